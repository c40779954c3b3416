"""Gauge configuration files in the reference's binary format (gaugeconfig.hh:225-252),
written from and read into the device (su2b_save_gauge / su2b_load_gauge), against files
the reference itself writes and reads."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(0, (4, 4, 4, 6), 4), (0, (6, 4, 1, 4), 3), (1, (4, 4, 4, 4), 4), (1, (8, 1, 1, 6), 2)]
IDS = ["su2-d4", "su2-d3", "u1-d4", "u1-d2"]


def make(gpu, group, dims, nd, precision="fp64"):
    Lx, Ly, Lz, Lt = dims
    return gpu.gaugeconfig(Lx, Ly, Lz, Lt, nd, 2.0, group="su2" if group == 0 else "u1",
                           precision=precision)


@pytest.mark.parametrize("group,dims,nd", CASES, ids=IDS)
def test_save_is_the_reference_file(gpu, orc, ref, tmp_path, group, dims, nd):
    U = orc.hotstart(group, dims, nd, 5, 1.0, 654321)
    ref.save_gauge(group, dims, nd, U, tmp_path / "ref.conf")
    with make(gpu, group, dims, nd) as c:
        c.upload(U)
        c.save(tmp_path / "dev.conf")
    assert (tmp_path / "dev.conf").read_bytes() == (tmp_path / "ref.conf").read_bytes()


@pytest.mark.parametrize("group,dims,nd", CASES, ids=IDS)
def test_load_reads_the_reference_file(gpu, orc, ref, tmp_path, group, dims, nd):
    U = orc.hotstart(group, dims, nd, 6, 1.0, 654321)
    ref.save_gauge(group, dims, nd, U, tmp_path / "ref.conf")
    with make(gpu, group, dims, nd) as c:
        c.load(tmp_path / "ref.conf")
        assert np.array_equal(c.download(), U)
        assert c.gauge_energy() == pytest.approx(orc.gauge_energy(group, dims, nd, U), rel=1e-13)
    # and the reference reads what the device wrote
    with make(gpu, group, dims, nd) as c:
        c.upload(U)
        c.save(tmp_path / "dev.conf")
    assert np.array_equal(ref.load_gauge(group, dims, nd, tmp_path / "dev.conf"), U)


def test_large_file_round_trip_and_mixed_precision(gpu, orc, tmp_path):
    """16^4: several double-buffered chunks each way; FP32 links are written widened."""
    group, dims, nd = 0, (16, 16, 16, 16), 4
    U = orc.hotstart(group, dims, nd, 7, 1.0, 654321)
    with make(gpu, group, dims, nd) as c:
        c.upload(U)
        c.save(tmp_path / "a.conf")
        c.upload(np.tile([1.0, 0.0, 0.0, 0.0], U.size // 4))
        c.load(tmp_path / "a.conf")
        assert np.array_equal(c.download(), U)
    with make(gpu, group, dims, nd, precision="mixed") as c:
        c.upload(U)
        c.save(tmp_path / "m.conf")
    rec = np.fromfile(tmp_path / "m.conf", dtype=np.dtype([("nc", "<u8"), ("v", "<f8", (4,))]))
    assert np.array_equal(rec["v"].reshape(-1), U.astype(np.float32).astype(np.float64))


def test_load_rejects_short_and_foreign_files(gpu, orc, ref, tmp_path):
    import su2_b200
    U = orc.hotstart(0, (4, 4, 4, 4), 4, 8, 1.0, 654321)
    ref.save_gauge(0, (4, 4, 4, 4), 4, U, tmp_path / "su2.conf")
    data = (tmp_path / "su2.conf").read_bytes()
    (tmp_path / "short.conf").write_bytes(data[: len(data) // 2])
    with make(gpu, 0, (4, 4, 4, 4), 4) as c:
        with pytest.raises(su2_b200.Su2bError):
            c.load(tmp_path / "short.conf")
        with pytest.raises(su2_b200.Su2bError):
            c.load(tmp_path / "missing.conf")
    Uu = orc.hotstart(1, (4, 4, 4, 4), 4, 8, 1.0, 654321)
    ref.save_gauge(1, (4, 4, 4, 4), 4, Uu, tmp_path / "u1.conf")
    with make(gpu, 0, (4, 4, 2, 2), 4) as c:  # as many bytes as the U(1) file
        with pytest.raises(su2_b200.Su2bError):
            c.load(tmp_path / "u1.conf")


def test_restart_from_the_counter(gpu, orc, tmp_path):
    # base_program.hpp:284-296 and :440-454: save, update the counter, restart elsewhere
    dims, nd = (4, 4, 4, 6), 4
    U = orc.hotstart(0, dims, nd, 9, 1.0, 654321)
    d = str(tmp_path) + "/"
    with make(gpu, 0, dims, nd) as c:
        c.upload(U)
        c.save(d + "run.conf.50")
    gpu.update_nconf_counter(d, True, 50, d + "run.conf.50")
    with make(gpu, 0, dims, nd) as c:
        assert c.restart(d) == (True, 50)
        assert np.array_equal(c.download(), U)
    with make(gpu, 0, dims, nd) as c:
        with pytest.raises(gpu.Su2bError):
            c.restart(str(tmp_path / "nowhere") + "/")
