"""Ensembles of independent SU(2) chains advanced together (su2b_batch_* of the C ABI)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .lattice import INTEGRATORS, TrajectoryResult, _dp, _f64


class chain_batch:
    """chains: list of dicts {dims: (Lx, Ly, Lz, Lt), ndims, beta, seed}."""

    def __init__(self, chains, precision="mixed", device=0):
        self.lib = _abi.load()
        self.chains = [dict(c) for c in chains]
        arr = (_abi.ChainDesc * len(chains))()
        for i, c in enumerate(chains):
            Lx, Ly, Lz, Lt = c["dims"]
            arr[i] = _abi.ChainDesc(Lx, Ly, Lz, Lt, c["ndims"], c["beta"], c["seed"])
        h = C.c_void_p()
        prec = _abi.PREC_FP64 if precision == "fp64" else _abi.PREC_MIXED
        rc = self.lib.su2b_batch_create(len(chains), arr, prec, device, C.byref(h))
        if rc != _abi.OK:
            raise _abi.Su2bError(rc, "batch creation failed")
        self.h = h

    def _c(self, rc):
        if rc != _abi.OK:
            m = self.lib.su2b_batch_last_error(self.h)
            raise _abi.Su2bError(rc, m.decode() if m else "")

    def close(self):
        if getattr(self, "h", None):
            self.lib.su2b_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def n_links(self, i):
        c = self.chains[i]
        Lx, Ly, Lz, Lt = c["dims"]
        return Lx * Ly * Lz * Lt * c["ndims"]

    def upload(self, i, U):
        U = _f64(U)
        self._c(self.lib.su2b_batch_upload(self.h, i, _dp(U)))

    def download(self, i):
        U = np.empty(self.n_links(i) * 4)
        self._c(self.lib.su2b_batch_download(self.h, i, _dp(U)))
        return U

    def stream(self):
        s = C.c_void_p()
        self._c(self.lib.su2b_batch_stream(self.h, C.byref(s)))
        return s.value or 0

    def kernel_launches(self):
        n = C.c_long()
        self._c(self.lib.su2b_batch_kernel_launches(self.h, C.byref(n)))
        return n.value

    def autotune(self):
        """Times the batched force step of every launch shape on the current fields (which it
        leaves unchanged), keeps the fastest; returns {variant: microseconds per launch}."""
        t = np.zeros(_abi.BATCH_VARIANTS)
        self._c(self.lib.su2b_batch_autotune(self.h, _dp(t)))
        return {v: float(t[v]) for v in range(_abi.BATCH_VARIANTS)}

    @property
    def variant(self) -> int:
        v = C.c_int()
        self._c(self.lib.su2b_batch_tune_get(self.h, C.byref(v)))
        return v.value

    @variant.setter
    def variant(self, v):
        self._c(self.lib.su2b_batch_tune_set(self.h, int(v)))

    def md_update(self, integrator="leapfrog", n_steps=10, tau=1.0, traj=0):
        res = (_abi.TrajResult * len(self.chains))()
        integ = INTEGRATORS[integrator] if isinstance(integrator, str) else integrator
        self._c(self.lib.su2b_batch_hmc(self.h, integ, n_steps, tau, traj, res))
        return [TrajectoryResult(bool(r.accepted), r.dH, r.ddH, tuple(r.H_old), tuple(r.H_new),
                                 r.plaquette, r.cg_iterations) for r in res]
