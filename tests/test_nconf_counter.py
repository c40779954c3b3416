"""The restart counter of io.hh:251-305 (su2b_update_nconf_counter / su2b_read_nconf_counter).
Host-only entry points of the library: they run without a GPU.

The expected bytes follow io::update_nconf_counter (io.hh:299-304): the header line
"heat i path_conf", then heat, i and the path separated by single spaces, no newline at the
end; the file name is conf_dir + "nconf_counter.txt" with no separator added."""
import pytest

import su2_b200 as sb


def test_counter_bytes_and_round_trip(tmp_path):
    d = str(tmp_path) + "/"
    sb.update_nconf_counter(d, True, 1200, d + "run.conf.1200")
    raw = (tmp_path / "nconf_counter.txt").read_bytes()
    assert raw == ("heat i path_conf\n1 1200 " + d + "run.conf.1200").encode()
    assert sb.read_nconf_counter(d) == (True, 1200, d + "run.conf.1200")
    sb.update_nconf_counter(d, False, 7, "c.7")  # overwritten, not appended
    assert (tmp_path / "nconf_counter.txt").read_bytes() == b"heat i path_conf\n0 7 c.7"
    assert sb.read_nconf_counter(d) == (False, 7, "c.7")


def test_conf_dir_is_a_prefix(tmp_path):
    # the reference concatenates conf_dir and the file name as they are
    sb.update_nconf_counter(str(tmp_path / "pre_"), True, 3, "x")
    assert (tmp_path / "pre_nconf_counter.txt").exists()
    assert sb.read_nconf_counter(str(tmp_path / "pre_")) == (True, 3, "x")


def test_reads_a_counter_written_by_hand(tmp_path):
    # the reader takes the second line and splits it at spaces; a trailing newline is fine
    (tmp_path / "nconf_counter.txt").write_text("heat i path_conf\n0 40 /data/conf.40\n")
    assert sb.read_nconf_counter(str(tmp_path) + "/") == (False, 40, "/data/conf.40")


@pytest.mark.parametrize("body", ["heat i path_conf\n", "heat i path_conf\n2 4 c",
                                  "heat i path_conf\n1 x c", "heat i path_conf\n1 4", ""])
def test_malformed_counter_is_an_error(tmp_path, body):
    (tmp_path / "nconf_counter.txt").write_text(body)
    with pytest.raises(sb.Su2bError):
        sb.read_nconf_counter(str(tmp_path) + "/")


def test_missing_counter_is_an_error(tmp_path):
    # the reference aborts (io.hh:270-274); the library returns an error status
    with pytest.raises(sb.Su2bError):
        sb.read_nconf_counter(str(tmp_path) + "/")
