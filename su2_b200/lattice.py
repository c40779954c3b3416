"""Host-side mirror of the su2 hot-path interface on top of the libsu2b C ABI.

The names follow the reference so that a caller of the reference finds the same operations:
``gaugeconfig`` (gaugeconfig.hh) holds the device-resident field, and its methods are the
free functions of the reference applied to it -- ``gauge_energy``, ``retr_sum_Wplaquettes``,
``get_S_G_hmc``, ``energy_density``, ``md_update``, ``sweep``, ``runge_kutta``,
``gradient_flow``, ``apply_D``/``apply_Ddag``/``DDdag`` and the Krylov solvers.  Arrays are
numpy float64 in the reference host layout (see include/su2b.h).  Errors raise Su2bError
with the library's message (the reference aborts via fatal_error instead).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import check

_D = C.POINTER(C.c_double)

INTEGRATORS = {"leapfrog": _abi.LEAPFROG, "lp_leapfrog": _abi.LP_LEAPFROG, "omf4": _abi.OMF4,
               "lp_omf4": _abi.LP_OMF4, "euler": _abi.EULER, "ruth": _abi.RUTH,
               "omf2": _abi.OMF2}


def _dp(a: np.ndarray):
    return a.ctypes.data_as(_D)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


@dataclass
class TrajectoryResult:
    accepted: bool
    dH: float
    ddH: float
    H_old: tuple
    H_new: tuple
    plaquette: float
    cg_iterations: int


@dataclass
class SolveResult:
    x: np.ndarray
    iterations: int
    restarts: int
    residual: float
    true_residual: float
    converged: bool


def update_nconf_counter(conf_dir, heat, i, path_conf):
    """io::update_nconf_counter (io.hh:294-305): conf_dir + "nconf_counter.txt" names the
    last saved configuration.  Host only."""
    check(_abi.load().su2b_update_nconf_counter(str(conf_dir).encode(), int(bool(heat)), int(i),
                                                 str(path_conf).encode()))


def read_nconf_counter(conf_dir):
    """io::read_nconf_counter (io.hh:267-285): (heat, i, path_conf).  Host only."""
    heat, i = C.c_int(), C.c_long()
    buf = C.create_string_buffer(4096)
    check(_abi.load().su2b_read_nconf_counter(str(conf_dir).encode(), C.byref(heat), C.byref(i),
                                               buf, len(buf)))
    return bool(heat.value), i.value, buf.value.decode()


class gaugeconfig:
    """Device-resident gauge field: gaugeconfig<G>(Lx, Ly, Lz, Lt, ndims, beta)
    (gaugeconfig.hh:49-63).  group: "su2" or "u1"; precision: "fp64" or "mixed"."""

    def __init__(self, Lx, Ly, Lz, Lt, ndims=4, beta=0.0, group="su2", xi=1.0,
                 precision="fp64", device=0):
        self.lib = _abi.load()
        self.group = _abi.GROUP_SU2 if group == "su2" else _abi.GROUP_U1
        self.dims = (Lx, Ly, Lz, Lt)
        self.ndims = ndims
        self.beta = beta
        self.xi = xi
        self.precision = precision
        self.volume = Lx * Ly * Lz * Lt
        self.n_links = self.volume * ndims
        ctx = C.c_void_p()
        prec = _abi.PREC_FP64 if precision == "fp64" else _abi.PREC_MIXED
        check(self.lib.su2b_ctx_create(self.group, Lx, Ly, Lz, Lt, ndims, beta, xi, prec, device,
                                       C.byref(ctx)))
        self.ctx = ctx

    # ---- lifetime ----
    def close(self):
        if getattr(self, "ctx", None):
            self.lib.su2b_ctx_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, rc):
        check(rc, self.ctx)

    @property
    def link_reals(self):
        return 4 if self.group == _abi.GROUP_SU2 else 1

    @property
    def adj_reals(self):
        return 3 if self.group == _abi.GROUP_SU2 else 1

    def stream(self) -> int:
        s = C.c_void_p()
        self._c(self.lib.su2b_ctx_stream(self.ctx, C.byref(s)))
        return s.value or 0

    def synchronize(self):
        """Waits for all work queued on the context's stream."""
        self._c(self.lib.su2b_synchronize(self.ctx))

    def profile(self, enable=True):
        """Per-kernel-class device timers (CUDA events on the context's stream)."""
        self._c(self.lib.su2b_profile(self.ctx, int(enable)))

    def profile_read(self) -> dict:
        out = {}
        for k, name in enumerate(_abi.K_NAMES):
            n, ms = C.c_long(), C.c_double()
            self._c(self.lib.su2b_profile_read(self.ctx, k, C.byref(n), C.byref(ms)))
            out[name] = (n.value, ms.value)
        return out

    def autotune(self, cache_path=None, retune=False):
        """Time the launch shapes of the force kernel on this field and keep the fastest;
        returns {variant: microseconds}."""
        t = np.zeros(_abi.FORCE_VARIANTS)
        cp = cache_path.encode() if cache_path else None
        self._c(self.lib.su2b_autotune(self.ctx, cp, int(retune), _dp(t)))
        return {v: float(t[v]) for v in range(_abi.FORCE_VARIANTS)}

    @property
    def force_variant(self) -> int:
        v = C.c_int()
        self._c(self.lib.su2b_tune_get(self.ctx, 0, C.byref(v)))
        return v.value

    @force_variant.setter
    def force_variant(self, v):
        self._c(self.lib.su2b_tune_set(self.ctx, 0, int(v)))

    @property
    def plain_trajectory(self) -> bool:
        """True: SU(2) trajectories run in the plain form (start-field copy, integrator steps
        launched one by one, no graph); False (default): the fused, graph-captured form."""
        v = C.c_int()
        self._c(self.lib.su2b_tune_get(self.ctx, 1, C.byref(v)))
        return v.value == 1

    @plain_trajectory.setter
    def plain_trajectory(self, on):
        self._c(self.lib.su2b_tune_set(self.ctx, 1, 1 if on else 0))

    def kernel_launches(self) -> int:
        n = C.c_long()
        self._c(self.lib.su2b_kernel_launches(self.ctx, C.byref(n)))
        return n.value

    def setBeta(self, beta):
        self.beta = beta
        self._c(self.lib.su2b_set_beta(self.ctx, beta))

    # ---- transfer ----
    def upload(self, U):
        U = _f64(U)
        assert U.size == self.n_links * self.link_reals
        self._c(self.lib.su2b_upload_gauge(self.ctx, _dp(U)))

    def download(self, out=None) -> np.ndarray:
        """The links in the reference's host layout.  out: a C-contiguous float64 buffer of
        the right size to write into (pinned memory makes the copy a direct DMA)."""
        n = self.n_links * self.link_reals
        if out is None:
            out = np.empty(n)
        elif out.dtype != np.float64 or out.size != n or not out.flags.c_contiguous:
            raise ValueError(f"out must be a contiguous float64 array of {n} elements")
        self._c(self.lib.su2b_download_gauge(self.ctx, _dp(out)))
        return out

    def save(self, path):
        """gaugeconfig::save (gaugeconfig.hh:225-230): the reference's binary format."""
        self._c(self.lib.su2b_save_gauge(self.ctx, str(path).encode()))

    def load(self, path):
        """gaugeconfig::load (gaugeconfig.hh:241-252); raises on a short or foreign file."""
        self._c(self.lib.su2b_load_gauge(self.ctx, str(path).encode()))

    def restart(self, conf_dir):
        """The restart of base_program.hpp:284-296: reads conf_dir + "nconf_counter.txt" and
        loads the configuration it names.  Returns (heat, i) as the counter holds them."""
        heat, i = C.c_int(), C.c_long()
        self._c(self.lib.su2b_restart(self.ctx, str(conf_dir).encode(), C.byref(heat),
                                      C.byref(i)))
        return bool(heat.value), i.value

    # ---- reductions ----
    def gauge_energy(self, spatial_only=False) -> float:
        out = C.c_double()
        self._c(self.lib.su2b_gauge_energy(self.ctx, int(spatial_only), C.byref(out)))
        return out.value

    def retr_sum_Wplaquettes(self, spatial_only=False) -> float:
        out = C.c_double()
        self._c(self.lib.su2b_retr_sum_plaquettes(self.ctx, int(spatial_only), C.byref(out)))
        return out.value

    def get_S_G_hmc(self) -> float:
        out = C.c_double()
        self._c(self.lib.su2b_gauge_action(self.ctx, C.byref(out)))
        return out.value

    def energy_density(self, cloverdef=True, ss=False):
        E, Q = C.c_double(), C.c_double()
        self._c(self.lib.su2b_energy_density(self.ctx, int(cloverdef), int(ss), C.byref(E),
                                             C.byref(Q)))
        return E.value, Q.value

    # ---- observables between trajectories ----
    def polyakov_loop_spatial_average(self) -> float:
        """polyakov_loop.hh:48-63 (normalised by the full volume, as the reference)."""
        out = C.c_double()
        self._c(self.lib.su2b_polyakov_loop(self.ctx, C.byref(out)))
        return out.value

    def wilsonloop(self, r, t) -> float:
        """Planar r x t Wilson loops averaged over the (mu, 0) planes (wilsonloop.hh:147-157)."""
        out = C.c_double()
        self._c(self.lib.su2b_wilson_loop(self.ctx, int(r), int(t), C.byref(out)))
        return out.value

    def APEsmearing(self, alpha, spatial=True):
        """APE smearing of the links in place (smearape.hh:97-131)."""
        self._c(self.lib.su2b_ape_smear(self.ctx, alpha, int(spatial)))

    # ---- force / updates ----
    def derivative(self, fac=1.0) -> np.ndarray:
        out = np.empty(self.n_links * self.adj_reals)
        self._c(self.lib.su2b_gauge_force(self.ctx, fac, _dp(out)))
        return out

    def restoreSU(self):
        self._c(self.lib.su2b_restore_su(self.ctx))

    def update_gauge(self, P, dtau):
        P = _f64(P)
        self._c(self.lib.su2b_update_gauge(self.ctx, _dp(P), dtau))

    # ---- derivatives (SU(2)) ----
    def action_backward(self, grad_out=1.0):
        """(S, grad_out * dS/dU): the Wilson action and its left derivative."""
        S = C.c_double()
        out = np.empty(self.n_links * 3)
        self._c(self.lib.su2b_action_backward(self.ctx, grad_out, C.byref(S), _dp(out)))
        return S.value, out

    def force_vjp(self, mu):
        mu = _f64(mu)
        out = np.empty(self.n_links * 3)
        self._c(self.lib.su2b_force_vjp(self.ctx, _dp(mu), _dp(out)))
        return out

    def flow_objective(self, eps, n_steps, grad=True, checkpoint_every=0):
        """t^2 E_p(t) after n_steps flow steps and (if grad) its derivative w.r.t. the links."""
        O = C.c_double()
        g = np.empty(self.n_links * 3) if grad else None
        self._c(self.lib.su2b_flow_adjoint(self.ctx, eps, n_steps, checkpoint_every, C.byref(O),
                                           _dp(g) if grad else None))
        return (O.value, g) if grad else O.value

    # ---- HMC ----
    def md_update(self, integrator="leapfrog", n_steps=10, tau=1.0, seed=0, traj=0,
                  momenta=None, uniform=None, revtest=False, accept_reject=True,
                  fermion_mass=0.0, cg_tol=1e-10, cg_max_iter=100000, pf_source=None,
                  pf_complex=False, cg_start="reference", pf_seed=97234719,
                  exponent=0) -> TrajectoryResult:
        """One HMC trajectory (md_update, md_update.hh:18-81).  momenta/uniform replay a host
        random stream; otherwise the device Philox streams keyed by (seed, traj) are used.
        exponent: rounding exponent of lp_leapfrog / lp_omf4 (the reference's default 0)."""
        p = _abi.HmcParams()
        p.integrator = INTEGRATORS[integrator] if isinstance(integrator, str) else integrator
        p.n_steps = n_steps
        p.tau = tau
        p.seed = seed
        p.traj = traj
        p.revtest = int(revtest)
        p.accept_reject = int(accept_reject)
        keep = []
        if momenta is not None:
            m = _f64(momenta)
            keep.append(m)
            p.momenta_host = _dp(m)
        p.uniform_host = -1.0 if uniform is None else float(uniform)
        p.fermion_mass = fermion_mass
        p.cg_tol = cg_tol
        p.cg_max_iter = cg_max_iter
        if pf_source is not None:
            r = _f64(pf_source)
            keep.append(r)
            p.pf_source_host = _dp(r)
        p.pf_complex = int(pf_complex)
        p.cg_start = _abi.CG_START_REFERENCE if cg_start == "reference" else _abi.CG_START_ZERO
        p.pf_seed = pf_seed
        p.round_exponent = exponent
        r = _abi.TrajResult()
        self._c(self.lib.su2b_hmc_trajectory(self.ctx, C.byref(p), C.byref(r)))
        return TrajectoryResult(bool(r.accepted), r.dH, r.ddH, tuple(r.H_old), tuple(r.H_new),
                                r.plaquette, r.cg_iterations)

    # ---- Metropolis ----
    def sweep(self, delta, N_hit, seed, sweep_index):
        """N_hit Metropolis updates of every link (flat_spacetime::sweep); returns the
        acceptance rates {overall, temporal} (flat-sweep.hh:154-157)."""
        rates = np.zeros(2)
        self._c(self.lib.su2b_metropolis_sweep(self.ctx, delta, N_hit, seed, sweep_index,
                                               _dp(rates)))
        return rates

    # ---- flow ----
    def runge_kutta(self, eps):
        self._c(self.lib.su2b_flow_step(self.ctx, eps))

    def gradient_flow(self, tmax, eps, tstart=0.0, max_rows=100000) -> np.ndarray:
        """Records {t, xi_R, P, P_ss, Ep, Ep_ss, Ec, Ec_ss, Q} (flat-gradient_flow.hh:70-197)."""
        rows = np.zeros((max_rows, 9))
        n = C.c_int()
        self._c(self.lib.su2b_gradient_flow(self.ctx, tmax, eps, tstart, _dp(rows), max_rows,
                                            C.byref(n)))
        return rows[:min(n.value, max_rows)].copy()

    # ---- staggered fermions (U(1)) ----
    def _apply(self, op, m, psi):
        psi = _f64(psi)
        out = np.empty_like(psi)
        self._c(self.lib.su2b_staggered_apply(self.ctx, op, m, _dp(psi), _dp(out)))
        return out

    def apply_D(self, m, psi):
        return self._apply(_abi.OP_D, m, psi)

    def apply_Ddag(self, m, psi):
        return self._apply(_abi.OP_DDAG, m, psi)

    def DDdag(self, m, psi):
        return self._apply(_abi.OP_DDDAG, m, psi)

    def solve(self, b, m, tol=1e-10, solver="CG", x0=None, tol_mode="abs", max_iter=100000,
              delta=0.1) -> SolveResult:
        """LinearCG on D Ddag ("CG"), LinearBiCGStab on D ("BiCGStab") or the mixed-precision
        CG ("CG_mixed")."""
        p = _abi.SolveParams()
        p.solver = {"CG": _abi.SOLVER_CG, "BiCGStab": _abi.SOLVER_BICGSTAB,
                    "CG_mixed": _abi.SOLVER_CG_MIXED}[solver]
        p.op = _abi.OP_D if solver == "BiCGStab" else _abi.OP_DDDAG
        p.mass = m
        p.tol = tol
        p.tol_mode = _abi.TOL_REL if tol_mode == "rel" else _abi.TOL_ABS
        p.max_iter = max_iter
        p.delta = delta
        b = _f64(b)
        x = np.empty_like(b)
        x0p = None
        if x0 is not None:
            x0 = _f64(x0)
            x0p = _dp(x0)
        st = _abi.SolveStats()
        rc = self.lib.su2b_solve(self.ctx, C.byref(p), _dp(b), x0p, _dp(x), C.byref(st))
        if rc not in (_abi.OK, _abi.ERR_NOT_CONVERGED):
            self._c(rc)
        return SolveResult(x, st.iterations, st.restarts, st.residual, st.true_residual,
                           rc == _abi.OK)

    def C_pion(self, m, tol=1e-10, seed=97234719, max_iter=100000):
        """staggered::C_pion (propagator.hpp:25-65): the pion correlator at rest, Lt values."""
        C_ = np.zeros(self.dims[3])
        it = C.c_long()
        self._c(self.lib.su2b_pion_correlator(self.ctx, m, tol, max_iter, seed, _dp(C_),
                                              C.byref(it)))
        return C_

    def fermion_derivative(self, m, phi, tol=1e-10, seed=97234719, x0=None, max_iter=100000):
        phi = _f64(phi)
        out = np.empty(self.n_links)
        it = C.c_long()
        x0p = _dp(_f64(x0)) if x0 is not None else None
        self._c(self.lib.su2b_fermion_force(self.ctx, m, _dp(phi), tol, max_iter, x0p, seed,
                                            _dp(out), C.byref(it)))
        return out, it.value

    def fermion_action(self, m, phi, tol=1e-10, seed=97234719, x0=None, max_iter=100000):
        phi = _f64(phi)
        out = C.c_double()
        x0p = _dp(_f64(x0)) if x0 is not None else None
        self._c(self.lib.su2b_fermion_action(self.ctx, m, _dp(phi), tol, max_iter, x0p, seed,
                                             C.byref(out)))
        return out.value
