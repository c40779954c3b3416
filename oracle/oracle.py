"""ctypes front-end for the two CPU checkers (TEST INFRASTRUCTURE ONLY).

``Oracle("orc")`` loads ``oracle/libsu2oracle.so`` -- the C restatement of the reference
hot path (su2_oracle.c).  ``Oracle("ref")`` loads ``oracle/_ref/libsu2ref.so`` -- the
reference's own headers behind a C ABI (ref_harness.cc).  Both expose the same calls with
the same argument meaning, on numpy arrays in the reference host layout
(gaugeconfig.hh:211-222).  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
legs import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PATHS = {"orc": os.path.join(HERE, "libsu2oracle.so"),
         "ref": os.path.join(HERE, "_ref", "libsu2ref.so")}

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
i32, f64, i64, u32, u64 = C.c_int, C.c_double, C.c_long, C.c_uint32, C.c_uint64

# name -> (restype, argtypes); "G" marks the group+geometry prefix (group, Lx, Ly, Lz, Lt, nd)
_G = [i32] * 6
_L = [i32] * 5  # U(1)-only calls: Lx, Ly, Lz, Lt, nd
_SIGS = {
    "hotstart": (None, _G + [i32, f64, i32, _D]),
    "random_gauge_trafo": (None, _G + [i32, _D]),
    "retr_sum_plaquettes": (f64, _G + [_D, f64, i32, i32]),
    "gauge_energy": (f64, _G + [_D, i32]),
    "polyakov_loop": (f64, _G + [_D]),
    "wilson_loop": (f64, _G + [_D, i32, i32]),
    "ape_smear": (None, _G + [f64, i32, _D]),
    "pion_correlator": (None, [i32, i32, i32, i32, i32, _D, f64, f64, i64, _D]),
    "S_G_hmc": (f64, _G + [f64, _D, f64, i32]),
    "gauge_derivative": (None, _G + [f64, f64, _D, f64, _D]),
    "md_injected": (f64, _G + [f64, f64, i32, i32, f64, _D, _D, _D]),
    "md_injected_lp": (f64, _G + [f64, f64, i32, i32, f64, _D, _D, _D, i32]),
    "hmc_run": (None, _G + [f64, f64, i32, i32, f64, i64, i32, i32, _D, _I, _D, _D]),
    "energy_density": (None, _G + [_D, i32, i32, _D, _D]),
    "runge_kutta": (None, _G + [f64, f64, f64, _D]),
    "staggered_apply": (None, _L + [_D, f64, i32, _D, _D]),
    "cg_ddag": (i64, _L + [_D, f64, _D, _D, f64, _D]),
    "bicgstab_d": (i64, _L + [_D, f64, _D, _D, f64, _D]),
    "ddag_inv": (None, _L + [_D, f64, _D, f64, i64, _D]),
    "fermion_heatbath": (f64, _L + [_D, f64, i64, _D]),
    "fermion_accept": (f64, _L + [_D, f64, _D, f64, i64]),
    "fermion_derivative": (None, _L + [_D, f64, _D, f64, i64, _D]),
    "md_injected_fermion": (f64, _L + [f64, f64, f64, i64, i32, i32, f64, _D, _D, _D, _D]),
    "md_injected_fermion_lp": (f64, _L + [f64, f64, f64, i64, i32, i32, f64, _D, _D, _D, _D,
                                          i32]),
    "eta": (f64, [i32] * 5),
    "initnormal": (f64, _G + [i64, _D]),
    "gaussian_spinor": (None, [i32] * 4 + [f64, f64, i64, _D]),
}
_ORC_ONLY = {
    "sweep_checkerboard": None,
    "restore_su": (None, _G + [_D]),
    "update_gauge": (None, _G + [_D, _D, f64]),
    "integrate": (None, _G + [f64, f64, i32, i32, f64, _D, _D]),
    "gradient_flow": (i32, _G + [f64, f64, _D, f64, f64, f64, _D, i32]),
    "fermion_force_from_chi": (None, _L + [_D, f64, _D, _D]),
    "cg_dense": (i64, [i32, _D, _D, _D, f64, _D]),
    "bicgstab_dense": (i64, [i32, _D, _D, _D, f64, _D]),
    "philox4x32_10": (None, [C.POINTER(C.c_uint32)] * 3),
    "philox_momenta": (None, _G + [u64, u32, _D]),
    "philox_accept_uniform": (f64, [u64, u32]),
    "philox_pf_source": (None, [i32] * 4 + [u64, u32, i32, _D]),
    "metropolis_checkerboard": (None, _G + [f64, f64, f64, i32, u64, u32, _D, _D]),
    "exp_su2": (None, [_D, _D]),
    "last_solve_calls": (i64, []),
}
_REF_ONLY = {
    "sweep": (None, _G + [f64, f64, i32, f64, i32, i64, i64, _D, _D]),
    "gradient_flow": (None, _G + [f64, f64, _D, f64, f64, f64, C.c_char_p]),
    "omp_threads": (i32, []),
    "save_gauge": (None, _G + [_D, C.c_char_p]),
    "load_gauge": (i32, _G + [C.c_char_p, _D]),
}


def build(which: str = "oracle") -> None:
    """Compile a checker with oracle/Makefile (``oracle`` or ``ref``)."""
    subprocess.run(["make", "-s", "-C", HERE, which], check=True)


def reference_dir() -> str | None:
    """The reference checkout oracle/Makefile reads ($SU2_REFERENCE overrides its default),
    or None where it is absent (the GPU box, a fresh clone without the reference)."""
    try:
        r = subprocess.run(["make", "-s", "-C", HERE, "refdir"], capture_output=True,
                           text=True, check=True)
    except (OSError, subprocess.CalledProcessError):
        return None
    d = r.stdout.strip()
    return d or None


def available(kind: str) -> bool:
    return os.path.exists(PATHS[kind])


def dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


class Oracle:
    """One checker library; calls take numpy float64 arrays (modified in place where the
    reference function modifies its argument)."""

    def __init__(self, kind: str = "orc"):
        self.kind = kind
        self.lib = C.CDLL(PATHS[kind])
        prefix = "orc_" if kind == "orc" else "ref_"
        sigs = dict(_SIGS)
        sigs.update({k: v for k, v in (_ORC_ONLY if kind == "orc" else _REF_ONLY).items()
                     if v is not None})
        for name, (res, args) in sigs.items():
            f = getattr(self.lib, prefix + name)
            f.restype = res
            f.argtypes = args
            setattr(self, "_" + name, f)

    # ---------------- gauge fields ----------------
    @staticmethod
    def nlinks(dims, nd):
        Lx, Ly, Lz, Lt = dims
        return Lx * Ly * Lz * Lt * nd

    def hotstart(self, group, dims, nd, seed, delta=1.0, trafo_seed=-1):
        n = self.nlinks(dims, nd) * (4 if group == 0 else 1)
        out = np.zeros(n)
        self._hotstart(group, *dims, nd, seed, delta, trafo_seed, dp(out))
        return out

    def random_gauge_trafo(self, group, dims, nd, U, seed):
        U = np.ascontiguousarray(U, dtype=np.float64).copy()
        self._random_gauge_trafo(group, *dims, nd, seed, dp(U))
        return U

    def retr_sum_plaquettes(self, group, dims, nd, U, xi=1.0, aniso=False, spatial_only=False):
        return self._retr_sum_plaquettes(group, *dims, nd, dp(U), xi, int(aniso),
                                         int(spatial_only))

    def gauge_energy(self, group, dims, nd, U, spatial_only=False):
        return self._gauge_energy(group, *dims, nd, dp(U), int(spatial_only))

    def polyakov_loop(self, group, dims, nd, U):
        return self._polyakov_loop(group, *dims, nd, dp(U))

    def wilson_loop(self, group, dims, nd, U, r, t):
        return self._wilson_loop(group, *dims, nd, dp(U), r, t)

    def ape_smear(self, group, dims, nd, U, alpha, spatial=True):
        U = np.ascontiguousarray(U, dtype=np.float64).copy()
        self._ape_smear(group, *dims, nd, alpha, int(spatial), dp(U))
        return U

    def pion_correlator(self, dims, nd, U, m, tol, seed):
        C = np.zeros(dims[3])
        self._pion_correlator(*dims, nd, dp(U), m, tol, seed, dp(C))
        return C

    def save_gauge(self, group, dims, nd, U, path):
        """gaugeconfig::save of the reference (reference harness only)."""
        self._save_gauge(group, *dims, nd, dp(np.ascontiguousarray(U, dtype=np.float64)),
                         str(path).encode())

    def load_gauge(self, group, dims, nd, path):
        out = np.zeros(self.nlinks(dims, nd) * (4 if group == 0 else 1))
        rc = self._load_gauge(group, *dims, nd, str(path).encode(), dp(out))
        if rc != 0:
            raise OSError(f"reference could not load {path}")
        return out

    def S_G_hmc(self, group, dims, nd, beta, U, xi=1.0, aniso=False):
        return self._S_G_hmc(group, *dims, nd, beta, dp(U), xi, int(aniso))

    def gauge_derivative(self, group, dims, nd, beta, U, xi=1.0, fac=1.0):
        out = np.zeros(self.nlinks(dims, nd) * (3 if group == 0 else 1))
        self._gauge_derivative(group, *dims, nd, beta, xi, dp(U), fac, dp(out))
        return out

    def md_injected(self, group, dims, nd, beta, integ, nsteps, tau, U, P, xi=1.0,
                    exponent=None):
        """exponent: the rounding exponent of the low-precision integrators (ids 1 and 3);
        None uses 16, the reference's default when the integrator is built without one."""
        U = U.copy()
        P = P.copy()
        H = np.zeros(4)
        if exponent is None and integ in (1, 3):
            exponent = 16
        if exponent is None:
            dH = self._md_injected(group, *dims, nd, beta, xi, integ, nsteps, tau, dp(U),
                                   dp(P), dp(H))
        else:
            dH = self._md_injected_lp(group, *dims, nd, beta, xi, integ, nsteps, tau, dp(U),
                                      dp(P), dp(H), exponent)
        return dH, U, P, H

    def hmc_run(self, group, dims, nd, beta, integ, nsteps, tau, seed, i0, ntraj, U, xi=1.0):
        U = U.copy()
        acc = np.zeros(ntraj, dtype=np.int32)
        dH = np.zeros(ntraj)
        plaq = np.zeros(ntraj)
        self._hmc_run(group, *dims, nd, beta, xi, integ, nsteps, tau, seed, i0, ntraj, dp(U),
                      acc.ctypes.data_as(_I), dp(dH), dp(plaq))
        return U, acc, dH, plaq

    def energy_density(self, group, dims, nd, U, cloverdef=True, ss=False):
        E = C.c_double()
        Q = C.c_double()
        self._energy_density(group, *dims, nd, dp(U), int(cloverdef), int(ss), C.byref(E),
                             C.byref(Q))
        return E.value, Q.value

    def runge_kutta(self, group, dims, nd, beta, eps, U, xi=1.0):
        U = U.copy()
        self._runge_kutta(group, *dims, nd, beta, xi, eps, dp(U))
        return U

    def initnormal(self, group, dims, nd, seed):
        P = np.zeros(self.nlinks(dims, nd) * (3 if group == 0 else 1))
        u = self._initnormal(group, *dims, nd, seed, dp(P))
        return P, u

    # ---------------- staggered (U(1)) ----------------
    def staggered_apply(self, dims, nd, U, m, op, psi):
        out = np.zeros_like(psi)
        self._staggered_apply(*dims, nd, dp(U), m, op, dp(psi), dp(out))
        return out

    def cg_ddag(self, dims, nd, U, m, b, x0, tol):
        x = np.zeros_like(b)
        it = self._cg_ddag(*dims, nd, dp(U), m, dp(b), dp(x0), tol, dp(x))
        return x, it

    def bicgstab_d(self, dims, nd, U, m, b, x0, tol):
        x = np.zeros_like(b)
        it = self._bicgstab_d(*dims, nd, dp(U), m, dp(b), dp(x0), tol, dp(x))
        return x, it

    def ddag_inv(self, dims, nd, U, m, psi, tol, seed):
        x = np.zeros_like(psi)
        self._ddag_inv(*dims, nd, dp(U), m, dp(psi), tol, seed, dp(x))
        return x

    def fermion_heatbath(self, dims, nd, U, m, seed_pf):
        V = dims[0] * dims[1] * dims[2] * dims[3]
        phi = np.zeros(2 * V)
        h = self._fermion_heatbath(*dims, nd, dp(U), m, seed_pf, dp(phi))
        return phi, h

    def fermion_accept(self, dims, nd, U, m, phi, tol, seed):
        return self._fermion_accept(*dims, nd, dp(U), m, dp(phi), tol, seed)

    def fermion_derivative(self, dims, nd, U, m, phi, tol, seed):
        out = np.zeros(self.nlinks(dims, nd))
        self._fermion_derivative(*dims, nd, dp(U), m, dp(phi), tol, seed, dp(out))
        return out

    def md_injected_fermion(self, dims, nd, beta, m, tol, seed, integ, nsteps, tau, U, P, R,
                            exponent=None):
        """exponent: as md_injected (the low-precision integrators, ids 1 and 3)."""
        U = U.copy()
        P = P.copy()
        H = np.zeros(6)
        if exponent is None and integ in (1, 3):
            exponent = 16
        if exponent is None:
            dH = self._md_injected_fermion(*dims, nd, beta, m, tol, seed, integ, nsteps, tau,
                                           dp(U), dp(P), dp(R), dp(H))
        else:
            dH = self._md_injected_fermion_lp(*dims, nd, beta, m, tol, seed, integ, nsteps, tau,
                                              dp(U), dp(P), dp(R), dp(H), exponent)
        return dH, U, P, H

    def gaussian_spinor(self, dims, avr, sigma, seed):
        V = dims[0] * dims[1] * dims[2] * dims[3]
        out = np.zeros(2 * V)
        self._gaussian_spinor(*dims, avr, sigma, seed, dp(out))
        return out

    def eta(self, t, x, y, z, mu):
        return self._eta(t, x, y, z, mu)

    # ---------------- reference-only ----------------
    def sweep(self, group, dims, nd, beta, delta, N_hit, seed, i, U, xi=1.0, aniso=False):
        U = U.copy()
        rates = np.zeros(2)
        self._sweep(group, *dims, nd, beta, xi, int(aniso), delta, N_hit, seed, i, dp(U),
                    dp(rates))
        return U, rates

    def gradient_flow_rows(self, group, dims, nd, beta, U, tmax, eps, tstart=0.0, xi=1.0,
                           path=None):
        """Flow records {t, xi_R, P, P_ss, Ep, Ep_ss, Ec, Ec_ss, Q} as an (n, 9) array."""
        if self.kind == "orc":
            rows = np.zeros((4096, 9))
            n = self._gradient_flow(group, *dims, nd, beta, xi, dp(U), tmax, eps, tstart,
                                    dp(rows), rows.shape[0])
            return rows[:n].copy()
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            p = os.path.join(d, "flow.dat")
            self._gradient_flow(group, *dims, nd, beta, xi, dp(U), tmax, eps, tstart,
                                p.encode())
            lines = [ln.split() for ln in open(p).read().splitlines()[1:] if ln.strip()]
        return np.array([[float(v) for v in ln] for ln in lines]).reshape(-1, 9)

    # ---------------- restatement-only ----------------
    def update_gauge(self, group, dims, nd, U, P, dtau):
        U = U.copy()
        self._update_gauge(group, *dims, nd, dp(U), dp(P), dtau)
        return U

    def restore_su(self, group, dims, nd, U):
        U = U.copy()
        self._restore_su(group, *dims, nd, dp(U))
        return U

    def integrate(self, group, dims, nd, beta, integ, nsteps, tau, U, P, xi=1.0):
        U = U.copy()
        P = P.copy()
        self._integrate(group, *dims, nd, beta, xi, integ, nsteps, tau, dp(U), dp(P))
        return U, P

    def fermion_force_from_chi(self, dims, nd, U, m, chi):
        out = np.zeros(self.nlinks(dims, nd))
        self._fermion_force_from_chi(*dims, nd, dp(U), m, dp(chi), dp(out))
        return out

    def cg_dense(self, A, b, x0, tol):
        n = b.size // 2
        x = np.zeros_like(b)
        it = self._cg_dense(n, dp(A), dp(b), dp(x0), tol, dp(x))
        return x, it

    def bicgstab_dense(self, A, b, x0, tol):
        n = b.size // 2
        x = np.zeros_like(b)
        it = self._bicgstab_dense(n, dp(A), dp(b), dp(x0), tol, dp(x))
        return x, it

    def philox(self, ctr, key):
        c = (C.c_uint32 * 4)(*ctr)
        k = (C.c_uint32 * 2)(*key)
        o = (C.c_uint32 * 4)()
        self._philox4x32_10(c, k, o)
        return list(o)

    def philox_momenta(self, group, dims, nd, seed, traj):
        P = np.zeros(self.nlinks(dims, nd) * (3 if group == 0 else 1))
        self._philox_momenta(group, *dims, nd, seed, traj, dp(P))
        return P

    def philox_accept_uniform(self, seed, traj):
        return self._philox_accept_uniform(seed, traj)

    def philox_pf_source(self, dims, seed, traj, complex_source=False):
        V = dims[0] * dims[1] * dims[2] * dims[3]
        R = np.zeros(2 * V)
        self._philox_pf_source(*dims, seed, traj, int(complex_source), dp(R))
        return R

    def metropolis_checkerboard(self, group, dims, nd, beta, delta, N_hit, seed, sweep, U,
                                xi=1.0):
        U = U.copy()
        rates = np.zeros(2)
        self._metropolis_checkerboard(group, *dims, nd, beta, xi, delta, N_hit, seed, sweep,
                                      dp(U), dp(rates))
        return U, rates

    def exp_su2(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        o = np.zeros(4)
        self._exp_su2(dp(x), dp(o))
        return o
