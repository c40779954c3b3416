"""ctypes declarations of include/su2b.h and the loader of the in-tree libsu2b.so.

There is no fallback: if the compiled library is missing the import fails with the build
command to run.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsu2b.so")

OK, ERR_INVALID, ERR_CUDA, ERR_NOT_CONVERGED, ERR_UNSUPPORTED, ERR_NOMEM, ERR_TIMEOUT = range(7)
GROUP_SU2, GROUP_U1 = 0, 1
PREC_FP64, PREC_MIXED = 0, 1
LEAPFROG, LP_LEAPFROG, OMF4, LP_OMF4, EULER, RUTH, OMF2 = 0, 1, 2, 3, 4, 5, 6
OP_D, OP_DDAG, OP_DDDAG = 0, 1, 2
SOLVER_CG, SOLVER_BICGSTAB, SOLVER_CG_MIXED = 0, 1, 2
TOL_ABS, TOL_REL = 0, 1
CG_START_REFERENCE, CG_START_ZERO = 0, 1

_ERRNAMES = {ERR_INVALID: "invalid argument", ERR_CUDA: "CUDA error",
             ERR_NOT_CONVERGED: "not converged", ERR_UNSUPPORTED: "unsupported",
             ERR_NOMEM: "out of device memory", ERR_TIMEOUT: "device wait timed out"}

_D = C.POINTER(C.c_double)


class HmcParams(C.Structure):
    _fields_ = [("integrator", C.c_int), ("n_steps", C.c_int), ("tau", C.c_double),
                ("seed", C.c_uint64), ("traj", C.c_uint32), ("revtest", C.c_int),
                ("accept_reject", C.c_int), ("momenta_host", _D), ("uniform_host", C.c_double),
                ("fermion_mass", C.c_double), ("cg_tol", C.c_double), ("cg_max_iter", C.c_int),
                ("pf_source_host", _D), ("pf_complex", C.c_int), ("cg_start", C.c_int),
                ("pf_seed", C.c_long), ("round_exponent", C.c_int)]


class TrajResult(C.Structure):
    _fields_ = [("accepted", C.c_int), ("dH", C.c_double), ("ddH", C.c_double),
                ("H_old", C.c_double * 3), ("H_new", C.c_double * 3),
                ("plaquette", C.c_double), ("cg_iterations", C.c_long)]


class ChainDesc(C.Structure):
    _fields_ = [("Lx", C.c_int), ("Ly", C.c_int), ("Lz", C.c_int), ("Lt", C.c_int),
                ("ndims", C.c_int), ("beta", C.c_double), ("seed", C.c_uint64)]


class SolveParams(C.Structure):
    _fields_ = [("solver", C.c_int), ("op", C.c_int), ("mass", C.c_double), ("tol", C.c_double),
                ("tol_mode", C.c_int), ("max_iter", C.c_int), ("delta", C.c_double)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_long), ("restarts", C.c_long), ("residual", C.c_double),
                ("true_residual", C.c_double)]


_P = C.c_void_p
i32, f64, u32, u64, i64 = C.c_int, C.c_double, C.c_uint32, C.c_uint64, C.c_long

# every entry point of include/su2b.h: name -> (restype, argtypes)
SIGNATURES = {
    "su2b_ctx_create": (i32, [i32, i32, i32, i32, i32, i32, f64, f64, i32, i32, C.POINTER(_P)]),
    "su2b_ctx_destroy": (i32, [_P]),
    "su2b_last_error": (C.c_char_p, [_P]),
    "su2b_ctx_stream": (i32, [_P, C.POINTER(_P)]),
    "su2b_set_beta": (i32, [_P, f64]),
    "su2b_synchronize": (i32, [_P]),
    "su2b_upload_gauge": (i32, [_P, _D]),
    "su2b_download_gauge": (i32, [_P, _D]),
    "su2b_gauge_energy": (i32, [_P, i32, _D]),
    "su2b_retr_sum_plaquettes": (i32, [_P, i32, _D]),
    "su2b_gauge_action": (i32, [_P, _D]),
    "su2b_energy_density": (i32, [_P, i32, i32, _D, _D]),
    "su2b_gauge_force": (i32, [_P, f64, _D]),
    "su2b_restore_su": (i32, [_P]),
    "su2b_update_gauge": (i32, [_P, _D, f64]),
    "su2b_hmc_trajectory": (i32, [_P, C.POINTER(HmcParams), C.POINTER(TrajResult)]),
    "su2b_metropolis_sweep": (i32, [_P, f64, i32, u64, u32, _D]),
    "su2b_flow_step": (i32, [_P, f64]),
    "su2b_gradient_flow": (i32, [_P, f64, f64, f64, _D, i32, C.POINTER(C.c_int)]),
    "su2b_staggered_apply": (i32, [_P, i32, f64, _D, _D]),
    "su2b_solve": (i32, [_P, C.POINTER(SolveParams), _D, _D, _D, C.POINTER(SolveStats)]),
    "su2b_fermion_force": (i32, [_P, f64, _D, f64, i32, _D, i64, _D, C.POINTER(C.c_long)]),
    "su2b_fermion_action": (i32, [_P, f64, _D, f64, i32, _D, i64, _D]),
    "su2b_profile": (i32, [_P, i32]),
    "su2b_profile_read": (i32, [_P, i32, C.POINTER(C.c_long), C.POINTER(C.c_double)]),
    "su2b_kernel_launches": (i32, [_P, C.POINTER(C.c_long)]),
    "su2b_gauge_energy_noalloc": (i32, [i32, i32, i32, i32, i32, i32, _P, _P, _P]),
    "su2b_autotune": (i32, [_P, C.c_char_p, i32, _D]),
    "su2b_batch_create": (i32, [i32, C.POINTER(ChainDesc), i32, i32, C.POINTER(_P)]),
    "su2b_batch_destroy": (i32, [_P]),
    "su2b_batch_last_error": (C.c_char_p, [_P]),
    "su2b_batch_stream": (i32, [_P, C.POINTER(_P)]),
    "su2b_batch_kernel_launches": (i32, [_P, C.POINTER(C.c_long)]),
    "su2b_batch_upload": (i32, [_P, i32, _D]),
    "su2b_batch_download": (i32, [_P, i32, _D]),
    "su2b_batch_hmc": (i32, [_P, i32, i32, f64, u32, C.POINTER(TrajResult)]),
    "su2b_batch_autotune": (i32, [_P, _D]),
    "su2b_polyakov_loop": (i32, [_P, _D]),
    "su2b_save_gauge": (i32, [_P, C.c_char_p]),
    "su2b_pion_correlator": (i32, [_P, f64, f64, i32, i64, _D, C.POINTER(i64)]),
    "su2b_load_gauge": (i32, [_P, C.c_char_p]),
    "su2b_update_nconf_counter": (i32, [C.c_char_p, i32, C.c_long, C.c_char_p]),
    "su2b_read_nconf_counter": (i32, [C.c_char_p, C.POINTER(i32), C.POINTER(C.c_long),
                                      C.c_char_p, C.c_size_t]),
    "su2b_restart": (i32, [_P, C.c_char_p, C.POINTER(i32), C.POINTER(C.c_long)]),
    "su2b_wilson_loop": (i32, [_P, i32, i32, _D]),
    "su2b_ape_smear": (i32, [_P, f64, i32]),
    "su2b_batch_tune_get": (i32, [_P, C.POINTER(i32)]),
    "su2b_batch_tune_set": (i32, [_P, i32]),
    "su2b_action_backward": (i32, [_P, f64, _D, _D]),
    "su2b_force_vjp": (i32, [_P, _D, _D]),
    "su2b_flow_adjoint": (i32, [_P, f64, i32, i32, _D, _D]),
    "su2b_tune_get": (i32, [_P, i32, C.POINTER(C.c_int)]),
    "su2b_tune_set": (i32, [_P, i32, i32]),
    "su2b_slabs_create": (i32, [i32, i32, i32, i32, i32, f64, f64, i32, i32, i32, i32, i32,
                                C.POINTER(_P)]),
    "su2b_slabs_destroy": (i32, [_P]),
    "su2b_slabs_last_error": (C.c_char_p, [_P]),
    "su2b_slabs_info": (i32, [_P, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32),
                              C.POINTER(i32)]),
    "su2b_slabs_nccl_id": (i32, [_P]),
    "su2b_slabs_connect": (i32, [_P, _P, i32, i32]),
    "su2b_slabs_upload": (i32, [_P, _D]),
    "su2b_slabs_download": (i32, [_P, _D]),
    "su2b_slabs_hmc_trajectory": (i32, [_P, C.POINTER(HmcParams), C.POINTER(TrajResult)]),
    "su2b_slabs_gauge_energy": (i32, [_P, i32, _D]),
    "su2b_slabs_metropolis_sweep": (i32, [_P, f64, i32, u64, u32, _D]),
    "su2b_slabs_flow_step": (i32, [_P, f64]),
    "su2b_slabs_energy_density": (i32, [_P, i32, i32, _D, _D]),
    "su2b_slabs_gradient_flow": (i32, [_P, f64, f64, f64, _D, i32, C.POINTER(C.c_int)]),
    "su2b_slabs_autotune": (i32, [_P, _D]),
    "su2b_slabs_tune_get": (i32, [_P, C.POINTER(i32)]),
    "su2b_slabs_tune_set": (i32, [_P, i32]),
    "su2b_slabs_set_overlap": (i32, [_P, i32]),
    "su2b_slabs_get_overlap": (i32, [_P, C.POINTER(i32)]),
    "su2b_slabs_kernel_launches": (i32, [_P, C.POINTER(C.c_long)]),
    "su2b_slabs_stream": (i32, [_P, C.POINTER(_P)]),
}
FORCE_VARIANTS = 12
BATCH_VARIANTS = 4
# (threads per block, min blocks per SM) of the batched force kernel
BATCH_SHAPES = [(64, 8), (128, 4), (128, 6), (256, 3)]
# (threads per block, min resident blocks per SM) of the force kernel's launch shapes; the
# "split" shapes run two threads per site (d = 4; other d use (128, 8)), "xsplit" with the
# cross-plane products formed once per site and swapped in shared memory; the anisotropic
# action always runs (128, 6)
FORCE_SHAPES = [(256, 4), (128, 8), (128, 4), (128, 6), (256, 2), (256, 3), ("split", 128, 8),
                (64, 16), ("xsplit", 128, 8), ("link", 128, 6), ("split", 128, 5), ("pair", 128, 8)]

K_FORCE, K_UPDATE, K_PLAQUETTE, K_MOMENTA, K_RESTORE, K_METROPOLIS, K_CLOVER, K_STAGGERED, \
    K_OTHER = range(9)
K_NAMES = ["force", "update", "plaquette", "momenta", "restore", "metropolis", "clover",
           "staggered", "other"]

_lib = None


def load() -> C.CDLL:
    """Load libsu2b.so and declare its signatures; raises if the library was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m su2_b200.build`")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


class Su2bError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"su2b error {code} ({_ERRNAMES.get(code, '?')}): {msg}")
        self.code = code


def check(rc: int, ctx=None) -> None:
    if rc != OK:
        msg = ""
        if ctx is not None:
            m = load().su2b_last_error(ctx)
            msg = m.decode() if m else ""
        raise Su2bError(rc, msg)
