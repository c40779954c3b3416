"""The drop-in boundary compiled on the reference's side.

oracle/shim_check (built by ``make -C oracle ref`` against the reference's headers, the shim
include/su2b_device.hpp and su2_b200/libsu2b.so) re-enacts the su2 HMC driver
(hmc.hpp:86-101 after base_program.hpp:276-317): a hot start with random_gauge_trafo, then
trajectories i = 0..5 with std::mt19937(seed + i), once through the reference's md_update and
once through device_lattice::md_update with the same engine.  It prints one JSON line; this
test runs it on the GPU and checks that both sides take the same accept decisions with the
same Delta H, plaquette and clover energy, end on the same links, and give the same gauge
derivative, for SU(2) d=4 8^4 and U(1) d=2 16x16.
"""
import json
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "shim_check")


def test_reference_driver_through_the_shim(gpu):
    if not os.path.exists(BIN):
        if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libsu2ref.so")):
            pytest.fail("oracle/_ref was built without shim_check")
        pytest.skip("the reference checkout was not available to build oracle/_ref")
    r = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [ln for ln in r.stdout.strip().split("\n") if ln.startswith("{")][-1]
    res = json.loads(line)
    for name in ("su2", "u1"):
        g = res[name]
        assert g["ntraj"] == 6 and g["accept_mismatch"] == 0, g
        assert g["dH_err"] <= 1e-7, g
        assert g["plaq_rel_err"] <= 1e-11, g
        assert g["E_rel_err"] <= 1e-10, g
        assert g["U_max_err"] <= 1e-9, g
        assert g["deriv_rel_err"] <= 1e-12, g
        assert g["philox_ok"], g
    # the chain is not trivially all-accept or all-reject
    assert 0 < res["su2"]["accepted"] <= 6
