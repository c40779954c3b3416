"""Error behaviour of the C ABI with a live context: every context entry point called with
zero and NULL arguments either refuses (SU2B_ERR_INVALID or SU2B_ERR_UNSUPPORTED, with a
message from su2b_last_error) or does the harmless thing zero asks for, never reports a
CUDA error, and leaves the context usable.  The reference ends such calls in
spacetime_lattice::fatal_error (geometry.hh:43-48); the shim maps a refusal to that."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# entry points whose zero/NULL call must be refused: a required buffer or path is NULL, or a
# count or step size is zero
MUST_REFUSE = {
    "su2b_ctx_stream", "su2b_upload_gauge", "su2b_download_gauge", "su2b_gauge_energy",
    "su2b_retr_sum_plaquettes", "su2b_gauge_action", "su2b_energy_density",
    "su2b_gauge_force", "su2b_update_gauge", "su2b_hmc_trajectory", "su2b_metropolis_sweep",
    "su2b_gradient_flow", "su2b_staggered_apply", "su2b_solve", "su2b_fermion_force",
    "su2b_fermion_action", "su2b_kernel_launches", "su2b_polyakov_loop", "su2b_save_gauge",
    "su2b_pion_correlator", "su2b_load_gauge", "su2b_restart", "su2b_wilson_loop",
    "su2b_force_vjp", "su2b_flow_adjoint", "su2b_tune_get"}
# not called: they end or reconfigure the context rather than act on it
SKIP = {"su2b_ctx_destroy", "su2b_set_beta"}


@pytest.mark.parametrize("group,precision,dims,nd", [
    ("su2", "fp64", (4, 4, 4, 4), 4), ("su2", "mixed", (4, 4, 4, 4), 4),
    ("u1", "fp64", (8, 1, 1, 8), 2)], ids=["su2-fp64", "su2-mixed", "u1-2d"])
def test_zero_arguments_refused_and_context_usable(gpu, orc, group, precision, dims, nd):
    from su2_b200 import _abi
    lib = _abi.load()
    Lx, Ly, Lz, Lt = dims
    U = orc.hotstart(0 if group == "su2" else 1, dims, nd, 4711, 1.0, 654321)
    with gpu.gaugeconfig(Lx, Ly, Lz, Lt, nd, 2.3, group=group, precision=precision) as c:
        c.upload(U)
        e0 = c.gauge_energy()
        checked = 0
        for name, (res, args) in _abi.SIGNATURES.items():
            if name in SKIP or not args or args[0] is not _abi._P or \
                    name.startswith(("su2b_batch", "su2b_slabs")):
                continue
            vals = [0 if a in (C.c_int, C.c_uint32, C.c_uint64, C.c_long)
                    else 0.0 if a is C.c_double else None for a in args[1:]]
            rc = getattr(lib, name)(c.ctx, *vals)
            if name == "su2b_last_error":
                continue
            assert rc in (_abi.OK, _abi.ERR_INVALID, _abi.ERR_UNSUPPORTED), (name, rc)
            if name in MUST_REFUSE:
                assert rc != _abi.OK, name
                assert lib.su2b_last_error(c.ctx), name
            checked += 1
        assert checked > 30
        # the context still works: the same field gives the same plaquette sum
        c.upload(U)
        assert c.gauge_energy() == e0
        assert np.isfinite(c.md_update("leapfrog", 2, 0.2, seed=1, traj=0).dH)


def _zero_calls(lib, prefix, handle, skip, must_refuse, silent=()):
    """Calls every entry point named prefix* whose first argument is a handle with zeros and
    NULLs; returns the number called."""
    from su2_b200 import _abi
    checked = 0
    for name, (res, args) in _abi.SIGNATURES.items():
        if not name.startswith(prefix) or name in skip or not args or args[0] is not _abi._P:
            continue
        vals = [0 if a in (C.c_int, C.c_uint32, C.c_uint64, C.c_long)
                else 0.0 if a is C.c_double else None for a in args[1:]]
        rc = getattr(lib, name)(handle, *vals)
        if name.endswith("last_error"):
            continue
        assert rc in (_abi.OK, _abi.ERR_INVALID, _abi.ERR_UNSUPPORTED), (name, rc)
        if name in must_refuse:
            assert rc != _abi.OK, name
            if name not in silent:
                assert getattr(lib, prefix + "last_error")(handle), name
        checked += 1
    return checked


def test_batch_zero_arguments(gpu, orc):
    from su2_b200 import _abi
    from su2_b200.batch import chain_batch
    chains = [dict(dims=(4, 4, 4, 4), ndims=4, beta=2.3, seed=1),
              dict(dims=(6, 4, 1, 4), ndims=3, beta=2.1, seed=2)]
    starts = [orc.hotstart(0, ch["dims"], ch["ndims"], 10 + i, 1.0, 654321)
              for i, ch in enumerate(chains)]
    with chain_batch(chains, precision="mixed") as b:
        for i, U in enumerate(starts):
            b.upload(i, U)
        ref = [r.dH for r in b.md_update("leapfrog", 2, 0.2, traj=0)]
        v0 = b.variant
        must = {"su2b_batch_stream", "su2b_batch_kernel_launches", "su2b_batch_upload",
                "su2b_batch_download", "su2b_batch_hmc", "su2b_batch_tune_get"}
        n = _zero_calls(_abi.load(), "su2b_batch_", b.h, {"su2b_batch_destroy"}, must)
        assert n >= 8
        b.variant = v0  # the zero calls retuned the launch shape
        for i, U in enumerate(starts):  # usable: the same start gives the same trajectory
            b.upload(i, U)
        assert [r.dH for r in b.md_update("leapfrog", 2, 0.2, traj=0)] == pytest.approx(
            ref, rel=1e-12)


def test_slabs_zero_arguments(gpu, orc):
    from su2_b200 import _abi
    from su2_b200.slabs import slab_lattice
    dims, nd = (4, 4, 4, 8), 4
    U = orc.hotstart(0, dims, nd, 4711, 1.0, 654321)
    with slab_lattice(dims, nd, 2.3, 2, precision="fp64") as s:
        s.upload(U)
        e0 = s.gauge_energy()
        must = {"su2b_slabs_connect", "su2b_slabs_upload", "su2b_slabs_download",
                "su2b_slabs_hmc_trajectory", "su2b_slabs_metropolis_sweep",
                "su2b_slabs_energy_density", "su2b_slabs_gradient_flow",
                "su2b_slabs_gauge_energy", "su2b_slabs_tune_get", "su2b_slabs_get_overlap",
                "su2b_slabs_kernel_launches", "su2b_slabs_stream"}
        # su2b_slabs_nccl_id takes an id buffer, not a handle
        n = _zero_calls(_abi.load(), "su2b_slabs_", s.h,
                        {"su2b_slabs_destroy", "su2b_slabs_nccl_id"}, must,
                        silent={"su2b_slabs_get_overlap"})
        assert n >= 15
        s.upload(U)
        assert s.gauge_energy() == pytest.approx(e0, rel=1e-14)
