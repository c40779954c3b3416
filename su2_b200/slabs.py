"""One SU(2) lattice over time slabs (su2b_slabs_* of the C ABI).

The lattice is cut into ``nslabs`` slabs of ``Lt / nslabs`` time slices (an even number).  A
``slab_lattice`` holds the slabs ``first .. first + count - 1``:

- ``count == nslabs`` (the default): every slab on one device; the ghost slices between them
  are device copies and a trajectory is one CUDA graph;
- one slab per process (``count == 1``, one GPU per rank): the ranks exchange ghost slices and
  sums over NCCL once ``connect_process_group`` has joined them.

A trajectory equals the one of a single-lattice ``gaugeconfig`` with the same seed and
trajectory index (the momenta are the Philox streams of the whole lattice): the same links
and accept decisions, energies to rounding.  The reference splits the same site loops over
OpenMP threads along t (flat-gaugemonomial.hh:105-131, flat-sweep.hh:83,128).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .lattice import INTEGRATORS, TrajectoryResult, _dp, _f64

NCCL_ID_BYTES = 128


def slab_bounds(Lt: int, nslabs: int, slab: int) -> tuple[int, int]:
    """The time slices [t0, t1) of one slab; raises where su2b_slabs_create returns
    SU2B_ERR_INVALID (Lt below 2 or not a multiple of nslabs, or an odd slab thickness)."""
    if nslabs < 1 or not 0 <= slab < nslabs:
        raise ValueError(f"bad slab {slab} of {nslabs}")
    if Lt < 2 or Lt % nslabs or (Lt // nslabs) % 2:
        raise ValueError(f"Lt = {Lt} does not split into {nslabs} slabs of an even thickness")
    tl = Lt // nslabs
    return slab * tl, (slab + 1) * tl


def nccl_unique_id() -> bytes:
    """ncclGetUniqueId through the library (one process makes it, all join with it)."""
    lib = _abi.load()
    buf = C.create_string_buffer(NCCL_ID_BYTES)
    rc = lib.su2b_slabs_nccl_id(buf)
    if rc != _abi.OK:
        raise _abi.Su2bError(rc, "ncclGetUniqueId failed (is libnccl.so.2 loadable?)")
    return buf.raw


def broadcast_unique_id(dist, make_id=nccl_unique_id) -> bytes:
    """Rank 0 makes the id, every rank of the process group returns it (gloo or NCCL)."""
    obj = [make_id() if dist.get_rank() == 0 else None]
    dist.broadcast_object_list(obj, src=0)
    return obj[0]


class slab_lattice:
    """dims = (Lx, Ly, Lz, Lt); precision "mixed" (FP32 links, FP64 sums) or "fp64"."""

    def __init__(self, dims, ndims, beta, nslabs, xi=1.0, precision="mixed", first=0,
                 count=None, device=0):
        self.lib = _abi.load()
        Lx, Ly, Lz, Lt = dims
        self.dims = tuple(dims)
        self.ndims = ndims
        self.nslabs = nslabs
        self.first = first
        self.count = nslabs - first if count is None else count
        prec = _abi.PREC_FP64 if precision == "fp64" else _abi.PREC_MIXED
        h = C.c_void_p()
        rc = self.lib.su2b_slabs_create(Lx, Ly, Lz, Lt, ndims, beta, xi, prec, nslabs, first,
                                        self.count, device, C.byref(h))
        if rc != _abi.OK:
            raise _abi.Su2bError(rc, f"slab creation failed ({dims}, {nslabs} slabs)")
        self.h = h
        self.n_links = Lx * Ly * Lz * Lt * ndims

    def _c(self, rc):
        if rc != _abi.OK:
            m = self.lib.su2b_slabs_last_error(self.h)
            raise _abi.Su2bError(rc, m.decode() if m else "")

    def close(self):
        if getattr(self, "h", None):
            self.lib.su2b_slabs_destroy(self.h)
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

    def slices(self) -> tuple[int, int]:
        """The time slices [t0, t1) this handle holds."""
        tl = self.dims[3] // self.nslabs
        return self.first * tl, (self.first + self.count) * tl

    def connect(self, unique_id: bytes, nranks: int, rank: int):
        buf = C.create_string_buffer(bytes(unique_id), NCCL_ID_BYTES)
        self._c(self.lib.su2b_slabs_connect(self.h, buf, nranks, rank))

    def upload(self, U):
        """U: the whole lattice's field in the reference host layout."""
        U = _f64(U)
        assert U.size == self.n_links * 4
        self._c(self.lib.su2b_slabs_upload(self.h, _dp(U)))

    def download(self, out=None) -> np.ndarray:
        """Writes this handle's slices into out (the whole lattice's field; a new zero array
        if None) and returns it."""
        n = self.n_links * 4
        if out is None:
            out = np.zeros(n)
        elif out.dtype != np.float64 or out.size != n or not out.flags.c_contiguous:
            raise ValueError(f"out must be a contiguous float64 array of {n} elements")
        self._c(self.lib.su2b_slabs_download(self.h, _dp(out)))
        return out

    def md_update(self, integrator="omf2", n_steps=10, tau=1.0, seed=0, traj=0, uniform=None,
                  accept_reject=True, momenta=None) -> TrajectoryResult:
        """One trajectory (md_update, md_update.hh:18-81) over all slabs."""
        p = _abi.HmcParams()
        p.integrator = INTEGRATORS[integrator] if isinstance(integrator, str) else integrator
        p.n_steps = n_steps
        p.tau = tau
        p.seed = seed
        p.traj = traj
        p.accept_reject = int(accept_reject)
        keep = None
        if momenta is not None:
            keep = _f64(momenta)
            p.momenta_host = _dp(keep)
        p.uniform_host = -1.0 if uniform is None else float(uniform)
        r = _abi.TrajResult()
        self._c(self.lib.su2b_slabs_hmc_trajectory(self.h, C.byref(p), C.byref(r)))
        del keep
        return TrajectoryResult(bool(r.accepted), r.dH, r.ddH, tuple(r.H_old), tuple(r.H_new),
                                r.plaquette, r.cg_iterations)

    def sweep(self, delta, N_hit, seed, sweep_index):
        """N_hit Metropolis updates of every link (flat_spacetime::sweep) over the slabs;
        returns the acceptance rates {overall, temporal} of the whole lattice."""
        rates = np.zeros(2)
        self._c(self.lib.su2b_slabs_metropolis_sweep(self.h, delta, N_hit, seed, sweep_index,
                                                     _dp(rates)))
        return rates

    def runge_kutta(self, eps):
        """One RK3 flow step of the current field (runge_kutta, flat-gradient_flow.hh:17-50)."""
        self._c(self.lib.su2b_slabs_flow_step(self.h, eps))

    def energy_density(self, cloverdef=True, ss=False):
        """(E, Q) of the whole lattice (flat-energy_density.hh:57-164)."""
        E, Q = C.c_double(), C.c_double()
        self._c(self.lib.su2b_slabs_energy_density(self.h, int(cloverdef), int(ss), C.byref(E),
                                                   C.byref(Q)))
        return E.value, Q.value

    def gradient_flow(self, tmax, eps, tstart=0.0) -> np.ndarray:
        """Records {t, xi_R, P, P_ss, Ep, Ep_ss, Ec, Ec_ss, Q} of the whole lattice
        (flat-gradient_flow.hh:70-197); the current field stays unchanged."""
        max_rows = int((tmax - tstart) / (2 * eps)) + 4
        rows = np.zeros((max_rows, 9))
        n = C.c_int()
        self._c(self.lib.su2b_slabs_gradient_flow(self.h, tmax, eps, tstart, _dp(rows), max_rows,
                                                  C.byref(n)))
        return rows[:min(n.value, max_rows)].copy()

    def gauge_energy(self, spatial_only=False) -> float:
        out = C.c_double()
        self._c(self.lib.su2b_slabs_gauge_energy(self.h, int(spatial_only), C.byref(out)))
        return out.value

    def autotune(self) -> np.ndarray:
        t = np.full(_abi.FORCE_VARIANTS, -1.0)
        self._c(self.lib.su2b_slabs_autotune(self.h, _dp(t)))
        return t

    def tune_get(self) -> int:
        v = C.c_int()
        self._c(self.lib.su2b_slabs_tune_get(self.h, C.byref(v)))
        return v.value

    def tune_set(self, variant: int):
        """The force kernel's launch shape (an index of _abi.FORCE_SHAPES) on every slab."""
        self._c(self.lib.su2b_slabs_tune_set(self.h, int(variant)))

    @property
    def overlap(self) -> bool:
        """Boundary slices first, their exchange overlapping the interior (su2b_slabs_set_overlap)."""
        v = C.c_int()
        self._c(self.lib.su2b_slabs_get_overlap(self.h, C.byref(v)))
        return bool(v.value)

    @overlap.setter
    def overlap(self, on: bool):
        self._c(self.lib.su2b_slabs_set_overlap(self.h, int(bool(on))))

    def kernel_launches(self) -> int:
        n = C.c_long()
        self._c(self.lib.su2b_slabs_kernel_launches(self.h, C.byref(n)))
        return n.value

    def stream(self) -> int:
        s = C.c_void_p()
        self._c(self.lib.su2b_slabs_stream(self.h, C.byref(s)))
        return s.value or 0


def connect_process_group(lat: slab_lattice, dist, make_id=nccl_unique_id):
    """Joins the handles of all ranks (one slab each, rank = slab) into one NCCL
    communicator; the id (made by make_id on rank 0) travels over the torch.distributed
    process group.  Every rank must call it: it is a collective of the group."""
    bad = lat.count != 1 or lat.first != dist.get_rank() or lat.nslabs != dist.get_world_size()
    # every rank takes part in the broadcast before any raises, so none is left waiting
    uid = broadcast_unique_id(dist, make_id)
    if bad:
        raise ValueError("one slab per rank: nslabs = world size, first = rank")
    lat.connect(uid, dist.get_world_size(), dist.get_rank())
