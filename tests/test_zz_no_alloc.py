"""The allocation-free plaquette entry point, su2b_gauge_energy_noalloc.

It exists for callers that cannot allocate device memory (a host framework that owns all of
the GPU's memory through its own pool, or code running during CUDA graph capture).  Through
the C ABI it must give the same sums as the context-based entry point (gauge_energy, full and
spatial-only) within the 1e-12 relative tolerance of the other FP64 reductions, on two calls
in a row (its scratch array is shared and reused), and reject lattices larger than its fixed
scratch array.  The device buffers here belong to the test, as they would to such a caller.
This file is collected last so that a run stopping at the first failure has run everything
else first; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = [(0, (8, 8, 8, 8), 4), (0, (6, 4, 1, 4), 3), (1, (16, 1, 1, 10), 2), (1, (4, 4, 4, 4), 4)]


@pytest.mark.parametrize("group,dims,nd", CASES)
def test_noalloc_matches_context_entry_point(gpu, orc, group, dims, nd):
    import torch
    from su2_b200 import _abi
    lib = _abi.load()
    U = orc.hotstart(group, dims, nd, 2024, 1.0, 654321)
    Lx, Ly, Lz, Lt = dims
    with gpu.gaugeconfig(Lx, Ly, Lz, Lt, nd, 2.0, group="su2" if group == 0 else "u1") as c:
        c.upload(U)
        want = np.array([c.gauge_energy(False), c.gauge_energy(True)])
    U_dev = torch.from_numpy(U).to("cuda")
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    for _ in range(2):  # the shared scratch array keeps the previous call's contents
        rc = lib.su2b_gauge_energy_noalloc(group, Lx, Ly, Lz, Lt, nd, ctypes.c_void_p(U_dev.data_ptr()),
                                           ctypes.c_void_p(out.data_ptr()), None)
        assert rc == _abi.OK
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12)
        out.fill_(float("nan"))


def test_noalloc_rejects_lattices_beyond_its_scratch(gpu):
    import torch
    from su2_b200 import _abi
    lib = _abi.load()
    dummy = torch.zeros(4, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    # 48^4 = 5,308,416 sites > 4,194,304
    assert lib.su2b_gauge_energy_noalloc(0, 48, 48, 48, 48, 4, p, p, None) == _abi.ERR_INVALID
    assert lib.su2b_gauge_energy_noalloc(0, 8, 8, 8, 8, 4, None, p, None) == _abi.ERR_INVALID
    # extents whose product wraps a 64-bit integer (65536^4 = 2^64) or an int stride
    assert lib.su2b_gauge_energy_noalloc(0, 65536, 65536, 65536, 65536, 4, p, p,
                                         None) == _abi.ERR_INVALID
    assert lib.su2b_gauge_energy_noalloc(1, 2 ** 30, 1, 1, 4, 2, p, p, None) == _abi.ERR_INVALID
