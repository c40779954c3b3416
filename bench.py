#!/usr/bin/env python
"""Headline benchmark: SU(2) d=4 32^4 HMC at beta = 2.4, omf2 integrator, tau = 1, 16 steps.

One step = one HMC trajectory (Philox momenta, 33 force evaluations, 32 link updates,
FP64 accept/reject).  ``value`` is the trajectory rate of the mixed-precision path (FP32
links and forces, FP64 reductions / accept / reunitarisation) over all ranks; the FP64 path
runs the same trajectories from the same thermalised configuration for the comparison at
equal Delta H and plaquette.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

With N > 1 (torchrun, one process per GPU) every rank runs an independent chain (replicas,
no collective in the timed path); the slowest rank's device time sets the rate.
``--impl reference`` times the reference's own CPU implementation (md_update from the su2
headers, built in oracle/_ref) on the host cores for the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L = 32
BETA = 2.4
NSTEPS = 16
TAU = 1.0
METRIC = "SU(2) 32^4 HMC traj/s mixed vs FP64 at equal ΔH/plaq; kernel HBM GB/s vs peak"
WORKLOAD = "SU(2) d=4 32^4, beta=2.4, omf2 tau=1 n=16 HMC trajectory"
THERM_TRAJ = 20  # untimed HMC trajectories after the Metropolis thermalisation


class quiet_stdout:
    """Silences file descriptor 1 (the reference's integrator factory prints its name)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.null)
        os.close(self.saved)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback (6.65 TB/s)"


def haar_links(n_links, seed):
    """Haar-uniform SU(2) links (normalised Gaussian 4-vectors), reference host layout."""
    rng = np.random.default_rng(seed)
    q = rng.normal(size=(n_links, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return np.ascontiguousarray(q.reshape(-1))


class Clocks:
    """Samples the SM clock and the clock-event (throttle) reasons during the timed region.

    An NVML polling thread reads them every 2 ms, so that even a timed region of a few tens
    of milliseconds carries a clock record; the sampler only reads, it changes no setting.
    """

    # NVML clocks-event reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown"}

    def __init__(self, device):
        self.device = device
        self.h = None
        self.samples = []
        self.reasons = 0
        self.max_mhz = None
        self.stop_flag = threading.Event()
        self.t = None
        try:
            import pynvml as N
            import torch
            N.nvmlInit()
            self.N = N
            pr = torch.cuda.get_device_properties(device)
            try:
                bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
                self.h = N.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                self.h = N.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = float(N.nvmlDeviceGetMaxClockInfo(self.h, N.NVML_CLOCK_SM))
        except Exception:
            self.h = None

    def _poll(self):
        N = self.N
        get_r = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            N.nvmlDeviceGetCurrentClocksThrottleReasons
        while True:
            try:
                self.samples.append(float(N.nvmlDeviceGetClockInfo(self.h, N.NVML_CLOCK_SM)))
                self.reasons |= int(get_r(self.h))
            except Exception:
                pass
            self.running.set()
            if self.stop_flag.wait(0.002):
                break

    def start(self):
        """Starts polling and returns once the poller runs (first sample taken)."""
        if self.h is None:
            return
        self.samples, self.reasons = [], 0
        self.stop_flag.clear()
        self.running = threading.Event()
        self.t = threading.Thread(target=self._poll, daemon=True)
        self.t.start()
        self.running.wait(5.0)

    def stop(self):
        if self.t is None:
            return None
        self.stop_flag.set()
        self.t.join()
        self.t = None
        if not self.samples:
            return None
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(v for b, v in self.REASONS.items() if self.reasons & b),
                "samples": len(self.samples), "source": "NVML, 2 ms polling"}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    # a process group whenever torchrun launched the run, one rank included, so that the
    # collective code of an N-GPU run is the code a one-GPU torchrun executes
    if ws > 1 or "TORCHELASTIC_RUN_ID" in os.environ:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    return ws, rank, local, dist


def barrier(dist):
    if dist is not None:
        import torch
        dist.barrier()
        torch.cuda.synchronize()


def allmax(dist, x):
    from su2_b200 import replicas
    return replicas.max_over_ranks(x) if dist is not None else x


# --------------------------------------------------------------------------------------
def run_chain(c, K, seed, traj0, events):
    """K timed trajectories on context c; returns (device seconds, results)."""
    import torch
    s = torch.cuda.ExternalStream(c.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    res = []
    e0.record(s)
    for k in range(K):
        res.append(c.md_update("omf2", NSTEPS, TAU, seed=seed, traj=traj0 + k))
    e1.record(s)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3, res


def stats(res, V):
    dH = [r.dH for r in res]
    return {"acceptance": sum(r.accepted for r in res) / len(res),
            "dH_mean": float(np.mean(dH)), "dH_rms": float(np.sqrt(np.mean(np.square(dH)))),
            "exp_minus_dH": float(np.mean(np.exp(-np.array(dH)))),
            "plaquette": float(np.mean([r.plaquette for r in res])) / (V * 6 * 2)}


def blocked(x, nblocks=20):
    """Mean and its standard error from nblocks consecutive blocks of a chain's series."""
    x = np.asarray(x, dtype=np.float64)
    n = len(x) // nblocks * nblocks
    b = x[:n].reshape(nblocks, -1).mean(axis=1)
    return float(x.mean()), float(b.std(ddof=1) / np.sqrt(nblocks))


def ks_effective(a, b):
    """Two-sample Kolmogorov-Smirnov test of two Markov chains' samples.  The statistic D is
    the samples' own; its p-value takes each chain's effective size n / (2 tau), with
    2 tau = (20-block error / naive error)^2 of the chain's mean (at least 1), in the
    asymptotic Kolmogorov distribution.  Correlated samples (a rejected trajectory leaves the
    field, and the next Delta H is drawn on it) make the plain p-value far too small."""
    from scipy import stats as st
    D = float(st.ks_2samp(a, b).statistic)

    def neff(x):
        x = np.asarray(x, dtype=np.float64)
        naive = np.std(x, ddof=1) / np.sqrt(len(x))
        r = max(1.0, (blocked(x)[1] / naive) ** 2)
        return len(x) / r, r

    (na, ra), (nb, rb) = neff(a), neff(b)
    return D, float(st.kstwobign.sf(D * np.sqrt(na * nb / (na + nb)))), ra, rb


def chain_statistics(c, U_start, n, seed, V):
    """n untimed trajectories of one precision from U_start (a Markov chain with Philox
    momenta and accept uniforms keyed by seed): Delta H, acceptance, exp(-Delta H) and the
    plaquette after each trajectory, each with its 20-block standard error."""
    c.upload(U_start)
    res = [c.md_update("omf2", NSTEPS, TAU, seed=seed, traj=k) for k in range(n)]
    dH = np.array([r.dH for r in res])
    out = {"dH": blocked(dH), "acc": blocked([float(r.accepted) for r in res]),
           "exp_mdH": blocked(np.exp(-dH)),
           "plaq": blocked([r.plaquette / (V * 6 * 2) for r in res])}
    return out, dH


def equal_dH_plaq(mixed, fp64, U_start, n, pairs, seed, V):
    """The metric's comparison of the two precisions at equal Delta H and plaquette.

    Chains: each precision runs n trajectories from the same thermalised field with its own
    seed (independent samples); the observables are compared by their difference in combined
    standard errors (z) and the Delta H samples by a two-sample Kolmogorov-Smirnov test;
    <exp(-Delta H)> = 1 (Creutz) is checked in each arm.
    Pairs: from the same field with the same seed and trajectory index both precisions draw
    the same momenta (FP32 storage evaluates the FP64 stream's uniforms in FP32) and the same
    accept uniform, so their Delta H differ only by the FP32 arithmetic of the trajectory."""
    from scipy import stats as st
    sm, dm = chain_statistics(mixed, U_start, n, seed + 11, V)
    sd, dd = chain_statistics(fp64, U_start, n, seed + 12, V)
    # exp(-Delta H) is heavy-tailed at <Delta H> ~ 3: for Gaussian Delta H (variance v) its
    # standard deviation is sqrt(exp(v) - 1), far above what a finite sample shows, so its
    # error is the larger of the blocked one and sqrt(expm1(v) / n)
    for s_, d_ in ((sm, dm), (sd, dd)):
        m, e = s_["exp_mdH"]
        s_["exp_mdH"] = (m, max(e, float(np.sqrt(np.expm1(np.var(d_)) / len(d_)))))
    z = {k: (sm[k][0] - sd[k][0]) / float(np.hypot(sm[k][1], sd[k][1])) for k in sm}
    creutz = {a: (s_["exp_mdH"][0] - 1.0) / s_["exp_mdH"][1] for a, s_ in (("mixed", sm),
                                                                           ("fp64", sd))}
    # the Gaussian form of <exp(-Delta H)> = 1: <Delta H> = var(Delta H) / 2
    half_var = {a: round(float(np.mean(d_) - np.var(d_) / 2), 3) for a, d_ in (("mixed", dm),
                                                                              ("fp64", dd))}
    diff, same = [], 0
    for k in range(pairs):
        r = []
        for c in (mixed, fp64):
            c.upload(U_start)
            r.append(c.md_update("omf2", NSTEPS, TAU, seed=seed + 13, traj=k))
        diff.append(r[0].dH - r[1].dH)
        same += r[0].accepted == r[1].accepted
    diff = np.array(diff)
    ks = ks_effective(dm, dd)
    rnd = lambda v: [float(f"{v[0]:.6g}"), float(f"{v[1]:.2g}")]  # noqa: E731
    return {"trajectories_per_arm": n, "errors": "20-block (exp_mdH: lognormal bound)",
            "mixed": {k: rnd(v) for k, v in sm.items()},
            "fp64": {k: rnd(v) for k, v in sd.items()},
            "z_mixed_minus_fp64": {k: round(v, 2) for k, v in z.items()},
            "creutz_z": {k: round(v, 2) for k, v in creutz.items()},
            "dH_mean_minus_half_var": half_var,
            "ks_p_dH": float(f"{ks[1]:.3g}"),
            "ks_dH": {"D": round(ks[0], 4), "p_iid": float(f"{st.ks_2samp(dm, dd).pvalue:.3g}"),
                      "two_tau": {"mixed": round(ks[2], 2), "fp64": round(ks[3], 2)},
                      "p": "asymptotic, effective sizes n / (2 tau)"},
            "paired": {"pairs": pairs, "same_momenta": True,
                       "dH_diff_mean": float(f"{diff.mean():.3g}"),
                       "dH_diff_rms": float(f"{np.sqrt(np.mean(diff ** 2)):.3g}"),
                       "dH_diff_max": float(f"{np.abs(diff).max():.3g}"),
                       "same_decision": same / pairs}}


def force_in_graph(c, t_traj, n_traj, bytes_per_link, NL, seed):
    """Device time of one force launch inside the captured trajectory: the trajectory's
    device time (graph replay, CUDA events) minus the device time of its other kernels (each
    timed with CUDA events in a direct-launch run of the same trajectory), shared over its
    force launches.  Launch gaps stay in the figure, so it is an upper bound on the kernel."""
    c.profile(True)
    for k in range(n_traj):
        c.md_update("omf2", NSTEPS, TAU, seed=seed, traj=300000 + k)
    prof = c.profile_read()
    c.profile(False)
    n_force = prof["force"][0] / n_traj
    other_ms = sum(ms for name, (n, ms) in prof.items() if name != "force") / n_traj
    t_force = (t_traj * 1e3 - other_ms) / n_force / 1e3
    per = {name: {"launches": n // n_traj, "us": round(ms * 1e3 / n, 2)}
           for name, (n, ms) in prof.items() if n}
    return {"avg_launch_us": t_force * 1e6, "GB/s": bytes_per_link * NL / t_force / 1e9,
            "force_launches_per_traj": n_force, "other_kernels_ms_per_traj": other_ms,
            "direct_launch_us": prof["force"][1] * 1e3 / prof["force"][0]}, per


def ours(args):
    import torch

    import su2_b200
    ws, rank, local, dist = dist_setup()
    torch.cuda.set_device(local)
    K, W = args.steps, args.warmup
    V = L ** 4
    NL = V * 4
    from su2_b200 import replicas
    seed = replicas.replica_seed(20240, rank)

    # ---- thermalised start (untimed): Haar start, Metropolis sweeps, HMC warm-up ----
    U0 = haar_links(NL, seed)
    mixed = su2_b200.gaugeconfig(L, L, L, L, 4, BETA, precision="mixed", device=local)
    mixed.upload(U0)
    for sweep in range(args.therm_sweeps):
        mixed.sweep(0.15, 8, seed, sweep)
    for k in range(THERM_TRAJ + max(W, 3)):
        mixed.md_update("omf2", NSTEPS, TAU, seed=seed, traj=100000 + k)
    U_th = mixed.download()
    # one FP64 start for all arms: FP32 links widened to double are unitary to about 1e-7
    # only, so the thermalised field is reunitarised in FP64 first
    Uq = U_th.reshape(-1, 4)
    Uq /= np.sqrt(np.einsum("ij,ij->i", Uq, Uq))[:, None]
    mixed.upload(U_th)
    tune_m = mixed.autotune()  # launch shape of the force kernel, timed on this field
    mixed.upload(U_th)
    for k in range(W):
        mixed.md_update("omf2", NSTEPS, TAU, seed=seed + 5, traj=k)
    mixed.upload(U_th)

    # ---- headline: mixed precision, K trajectories ----
    clocks = Clocks(local)
    barrier(dist)
    n0 = mixed.kernel_launches()
    clocks.start()
    t_mixed, res_m = run_chain(mixed, K, seed, 0, None)
    clk = clocks.stop()
    launches = mixed.kernel_launches() - n0
    t_mixed = allmax(dist, t_mixed)
    value = ws * K / t_mixed

    # ---- FP64, fused and graph-captured, same start and seeds ----
    fp64 = su2_b200.gaugeconfig(L, L, L, L, 4, BETA, precision="fp64", device=local)
    fp64.upload(U_th)
    tune_d = fp64.autotune()
    fp64.upload(U_th)
    for k in range(W):
        fp64.md_update("omf2", NSTEPS, TAU, seed=seed + 7, traj=200000 + k)
    fp64.upload(U_th)
    barrier(dist)
    t_fp64, res_d = run_chain(fp64, K, seed, 0, None)
    t_fp64 = allmax(dist, t_fp64)

    # ---- the plain form: FP64, integrator steps launched one by one (no graph, no link
    #      update fused into the force launch, a copy of the start field), the default force
    #      launch shape (no autotuning) ----
    plain = su2_b200.gaugeconfig(L, L, L, L, 4, BETA, precision="fp64", device=local)
    plain.plain_trajectory = True
    plain.upload(U_th)
    for k in range(W):
        plain.md_update("omf2", NSTEPS, TAU, seed=seed + 9, traj=200000 + k)
    plain.upload(U_th)
    barrier(dist)
    t_plain, res_p = run_chain(plain, K, seed, 0, None)
    t_plain = allmax(dist, t_plain)
    plain_shape = su2_b200._abi.FORCE_SHAPES[plain.force_variant]
    plain.close()

    # ---- roofline of the dominant kernel (fused staples/force/momentum/link update) ----
    hbm, peak_src = peaks()
    nprof = max(2, K // 2)
    roof, kernels = {}, {}
    for name, c, bpl, t in (("mixed", mixed, 56, t_mixed / K), ("fp64", fp64, 112, t_fp64 / K)):
        c.upload(U_th)
        roof[name], kernels[name] = force_in_graph(c, t, nprof, bpl, NL, seed)
    # measured DRAM bytes of the launch shape the tuner chose, from an ncu capture
    traffic = None
    tp = os.path.join(ROOT, "profiles", "force_kernel_traffic.json")
    if os.path.exists(tp):
        shape = su2_b200._abi.FORCE_SHAPES[mixed.force_variant]
        key = shape[0] if isinstance(shape[0], str) else str(shape)
        traffic = json.load(open(tp)).get("mixed_bytes_per_launch", {}).get(key)

    # ---- mixed against FP64 at equal Delta H and plaquette (untimed statistics) ----
    eq = equal_dH_plaq(mixed, fp64, U_th, args.stat_traj, args.pairs, seed, V)

    # ---- e2e through the C ABI with host buffers (pinned), per trajectory:
    #      upload the host gaugeconfig, one trajectory, download the gaugeconfig ----
    Uh = torch.empty(NL * 4, dtype=torch.float64, pin_memory=True).numpy()
    Uh[:] = U_th
    mixed.upload(Uh)
    barrier(dist)
    t0 = time.perf_counter()
    for k in range(K):
        mixed.upload(Uh)
        mixed.md_update("omf2", NSTEPS, TAU, seed=seed, traj=400000 + k)
        mixed.download(out=Uh)
    t_e2e = allmax(dist, time.perf_counter() - t0)

    # ---- side measurements of the workload (Metropolis sweep, flow step) ----
    mixed.upload(U_th)
    s = torch.cuda.ExternalStream(mixed.stream())
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record(s)
    for sweep in range(5):
        mixed.sweep(0.15, 8, seed, 5000 + sweep)
    ev[1].record(s)
    fp64.upload(U_th)
    s2 = torch.cuda.ExternalStream(fp64.stream())
    ev[2].record(s2)
    for _ in range(10):
        fp64.runge_kutta(0.01)
    ev[3].record(s2)
    torch.cuda.synchronize()
    metro = 5 / (ev[0].elapsed_time(ev[1]) / 1e3)
    flow = 10 / (ev[2].elapsed_time(ev[3]) / 1e3)
    # the same two in the other precision: FP64 Metropolis, mixed-precision flow
    fp64.upload(U_th)
    mixed.upload(U_th)
    ev2 = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev2[0].record(s2)
    for sweep in range(5):
        fp64.sweep(0.15, 8, seed, 5000 + sweep)
    ev2[1].record(s2)
    ev2[2].record(s)
    for _ in range(10):
        mixed.runge_kutta(0.01)
    ev2[3].record(s)
    torch.cuda.synchronize()
    metro64 = 5 / (ev2[0].elapsed_time(ev2[1]) / 1e3)
    flow32 = 10 / (ev2[2].elapsed_time(ev2[3]) / 1e3)

    # ---- one lattice over time slabs on this GPU: what the decomposition adds (per-slab
    #      launches, a ghost-slice exchange after each force launch, the cross-slab sums),
    #      mixed precision with the tuned force shape, device time of K trajectories ----
    from su2_b200.slabs import slab_lattice
    slab_rate = {}
    for nsl, ov in ((2, False), (4, False), (2, True), (4, True)):
        with slab_lattice((L, L, L, L), 4, BETA, nsl, precision="mixed", device=local) as sl:
            sl.upload(U_th)
            sl.tune_set(mixed.force_variant)
            sl.overlap = ov
            for k in range(10):  # graph capture of the buffer assignments met
                sl.md_update("omf2", NSTEPS, TAU, seed=seed, traj=600000 + k)
            ss = torch.cuda.ExternalStream(sl.stream())
            ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ea.record(ss)
            for k in range(K):
                sl.md_update("omf2", NSTEPS, TAU, seed=seed, traj=600010 + k)
            eb.record(ss)
            eb.synchronize()
            slab_rate[f"{nsl}{' overlapped' if ov else ''}"] = K / (ea.elapsed_time(eb) / 1e3)

    # ---- the measurements taken between trajectories (FP64 context, thermalised field):
    #      wall time per call, each call returns its value to the host ----
    def per_call(fn, n=5):
        fn()
        fp64.synchronize()
        t0 = time.perf_counter()
        for _ in range(n):
            fn()
        fp64.synchronize()
        return 1e3 * (time.perf_counter() - t0) / n

    fp64.upload(U_th)
    obs = {"plaquette_ms": per_call(fp64.gauge_energy),
           "clover_E_Q_ms": per_call(fp64.energy_density),
           "polyakov_loop_ms": per_call(fp64.polyakov_loop_spatial_average),
           "wilson_loop_4x4_ms": per_call(lambda: fp64.wilsonloop(4, 4)),
           "ape_smear_spatial_ms": per_call(lambda: fp64.APEsmearing(0.5))}
    fp64.upload(U_th)
    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "conf.0")
        t0 = time.perf_counter()
        fp64.save(path)
        t_save = time.perf_counter() - t0
        nbytes = os.path.getsize(path)
        t0 = time.perf_counter()
        fp64.load(path)
        t_load = time.perf_counter() - t0
    obs["gaugeconfig_file_bytes"] = nbytes
    obs["save_GB_per_s"] = nbytes / t_save / 1e9
    obs["load_GB_per_s"] = nbytes / t_load / 1e9
    # the workload's flow measurement: Wilson flow to t = 4 with eps = 0.01 on the thermalised
    # field, records every second step (flat-gradient_flow.hh:70-197), t^2 E_clover at the end
    fp64.upload(U_th)
    fp64.synchronize()
    t0 = time.perf_counter()
    rows = fp64.gradient_flow(4.0, 0.01)
    t_flow = time.perf_counter() - t0
    obs["flow_to_t4"] = {"s": t_flow, "records": int(len(rows)), "t_last": float(rows[-1, 0]),
                         "t2_Ec_last": float(rows[-1, 0] ** 2 * rows[-1, 6]),
                         "t2_Ep_last": float(rows[-1, 0] ** 2 * rows[-1, 4])}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(U_th)

    if rank == 0:
        shapes = su2_b200._abi.FORCE_SHAPES
        # details first (one JSON line of their own); the headline line comes last
        print(json.dumps({
            "detail": "bench.py headline run: per-kernel timers, tuner and side measurements",
            "kernels_us": kernels, "roofline_fp64_kernel": roof["fp64"],
            "roofline_mixed_kernel": roof["mixed"],
            "autotune_force_us": {"mixed": {str(shapes[k]): v for k, v in tune_m.items()},
                                  "fp64": {str(shapes[k]): v for k, v in tune_d.items()}},
            "timed_chain_stats": {"mixed": stats(res_m, V), "fp64": stats(res_d, V),
                                  "plain_fp64": stats(res_p, V)},
            "metropolis_sweeps_per_s": {"mixed": metro, "fp64": metro64},
            "flow_rk3_steps_per_s": {"fp64": flow, "mixed": flow32},
            "time_slabs_one_gpu_mixed_traj_per_s": {"1 (the lattice)": K / t_mixed,
                                                   **slab_rate},
            "between_trajectories_fp64": obs,
            # the long forms of the headline line's entries
            "headline_notes": {
                "data": "synthetic: seeded Haar-random start, Metropolis-thermalised on device",
                "config": {"workload": WORKLOAD + " (mixed precision)", "lattice": [L] * 4,
                           "replicas": ws,
                           "l2": "working set (three link buffers, P) > 126 MB L2; no flush"},
                "fp64_form": "fused, graph, tuned",
                "plain_fp64_form": f"steps launched one by one, no graph, default shape "
                                   f"{plain_shape}",
                "roofline": {"kernel": "fused staple/force/momentum/link update FP32 "
                                       f"{shapes[mixed.force_variant]}",
                             "bytes_per_launch": 56 * NL,
                             "avg_launch_us": roof["mixed"]["avg_launch_us"],
                             "timing": "in-graph: trajectory device time minus its other "
                                       "kernels, per force launch",
                             "peak_source": peak_src,
                             "traffic": "ncu DRAM bytes per launch of the chosen shape"},
                "e2e": "host FP64 gaugeconfig up, trajectory, down; wall clock",
                "clocks": clk,
                "cpu_baseline": cpu,
                "equal_dH_plaq": eq}}), flush=True)
        r3 = lambda v: float(f"{v:.4g}")  # noqa: E731
        # the headline line stays under 1,400 characters, so that a 1,500-character log tail
        # holds it whole; the detail line above carries the long forms
        line = {
            "metric": METRIC, "value": r3(value), "unit": "traj/s", "n_gpus": ws, "steps": K,
            "warmup": W, "ms_per_step": r3(1e3 * t_mixed / K), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32 links + fp64 sums/accept",
            "data": "synthetic, seeded",
            "config": {"workload": "SU(2) 32^4 beta 2.4 omf2 tau 1 n 16, mixed",
                       "parallelism": f"replicas x{ws}", "l2": "working set > L2, no flush"},
            "fp64": r3(ws * K / t_fp64), "plain_fp64": r3(ws * K / t_plain),
            "speedup_mixed_vs_fp64": r3(t_fp64 / t_mixed),
            "speedup_mixed_vs_plain_fp64": r3(t_plain / t_mixed),
            "fp64_gpu_over_reference_cpu": r3(ws * K / t_fp64 / cpu["value"]) if cpu else None,
            "equal_dH_plaq": {"n": eq["trajectories_per_arm"], "mixed": eq["mixed"],
                              "fp64": eq["fp64"], "z": eq["z_mixed_minus_fp64"],
                              "ks_p": eq["ks_p_dH"], "creutz_z": eq["creutz_z"],
                              "paired_dH_rms": eq["paired"]["dH_diff_rms"]},
            "roofline": {"bound": "hbm", "achieved": r3(roof["mixed"]["GB/s"]), "peak": hbm,
                         "unit": "GB/s", "frac": r3(roof["mixed"]["GB/s"] / hbm),
                         "traffic": traffic, "peak_of": peak_src.split()[0],
                         "fp64_frac": r3(roof["fp64"]["GB/s"] / hbm)},
            "e2e": {"value": r3(ws * K / t_e2e), "unit": "traj/s",
                    "h2d_bytes_per_step": int(NL * 4 * 8), "d2h_bytes_per_step": int(NL * 4 * 8)},
            "gpu_launches": int(launches),
            "clocks": {k: clk[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")} if clk else None,
            "cpu_baseline": ({"value": r3(cpu["value"]), "unit": cpu["unit"],
                              "cores": cpu["cores"], "kind": cpu["kind"],
                              "sample": "1 trajectory"} if cpu else None),
        }
        print(json.dumps(line, separators=(",", ":")), flush=True)
    mixed.close()
    fp64.close()
    if dist is not None:
        dist.destroy_process_group()


def cpu_baseline(U_th):
    """The reference's md_update code (oracle/_ref) on the host cores: one omf2 trajectory of
    the same 32^4 workload with injected momenta (a bounded sample)."""
    from oracle import oracle as O
    if not O.available("ref"):
        return None
    r = O.Oracle("ref")
    threads = r._omp_threads()
    P = np.random.default_rng(5).normal(size=L ** 4 * 4 * 3)
    with quiet_stdout():
        t0 = time.perf_counter()
        r.md_injected(0, (L, L, L, L), 4, BETA, 6, NSTEPS, TAU, U_th.copy(), P)
        dt = time.perf_counter() - t0
    return {"value": 1.0 / dt, "unit": "traj/s", "cores": threads, "kind": "reference",
            "sample": "1 omf2 trajectory of the 32^4 workload, reference md_update code, "
                      "OpenMP"}


def slabs_run(args):
    """--slabs N: one 32^4 lattice cut into N time slabs (strong scaling).  Under torchrun
    each rank holds one slab (N = world size) and the ranks exchange ghost slices and sums
    over NCCL; as one process, all N slabs share its GPU.  Rank 0 thermalises the field and
    broadcasts it; value = trajectories of the lattice per second over the slowest rank's
    device time; e2e uploads each rank's slices (with ghosts) and downloads them per step."""
    import torch

    import su2_b200
    from su2_b200.slabs import connect_process_group, slab_lattice
    ws, rank, local, dist = dist_setup()
    torch.cuda.set_device(local)
    K, W, N = args.steps, args.warmup, args.slabs
    if dist is not None and N != ws:
        raise SystemExit(f"--slabs {N} under {ws} ranks: one slab per rank (N = world size)")
    NL = L ** 4 * 4
    seed = 20240
    therm = su2_b200.gaugeconfig(L, L, L, L, 4, BETA, precision="mixed", device=local)
    if rank == 0:
        therm.upload(haar_links(NL, seed))
        for sweep in range(args.therm_sweeps):
            therm.sweep(0.15, 8, seed, sweep)
        for k in range(THERM_TRAJ):
            therm.md_update("omf2", NSTEPS, TAU, seed=seed, traj=100000 + k)
        U_th = therm.download()
        Uq = U_th.reshape(-1, 4)
        Uq /= np.sqrt(np.einsum("ij,ij->i", Uq, Uq))[:, None]
        therm.upload(U_th)
        therm.autotune()
        variant = therm.force_variant
    else:
        U_th, variant = np.empty(NL * 4), 0
    therm.close()
    if dist is not None:
        t = torch.from_numpy(U_th).cuda()
        v = torch.tensor([variant], device="cuda")
        dist.broadcast(t, 0)
        dist.broadcast(v, 0)
        U_th, variant = t.cpu().numpy(), int(v.item())
    if dist is not None:
        lat = slab_lattice((L, L, L, L), 4, BETA, N, precision="mixed", first=rank, count=1,
                           device=local)
        connect_process_group(lat, dist)
    else:
        lat = slab_lattice((L, L, L, L), 4, BETA, N, precision="mixed", device=local)
    lat.upload(U_th)
    lat.tune_set(variant)
    for k in range(max(W, 3) + 6):
        lat.md_update("omf2", NSTEPS, TAU, seed=seed, traj=300000 + k)
    lat.upload(U_th)
    s = torch.cuda.ExternalStream(lat.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = Clocks(local)
    barrier(dist)
    n0 = lat.kernel_launches()
    clocks.start()
    e0.record(s)
    res = [lat.md_update("omf2", NSTEPS, TAU, seed=seed, traj=k) for k in range(K)]
    e1.record(s)
    e1.synchronize()
    clk = clocks.stop()
    launches = lat.kernel_launches() - n0
    t = allmax(dist, e0.elapsed_time(e1) / 1e3)
    # the workload's other steps over the same slabs: Metropolis sweeps and RK3 flow steps
    side = {}
    for name, fn, n in (("metropolis_sweeps_per_s", lambda k: lat.sweep(0.15, 8, seed, 7000 + k), 5),
                        ("flow_rk3_steps_per_s", lambda k: lat.runge_kutta(0.01), 10)):
        lat.upload(U_th)
        fn(0)
        barrier(dist)
        e0.record(s)
        for k in range(n):
            fn(k + 1)
        e1.record(s)
        e1.synchronize()
        side[name] = n / allmax(dist, e0.elapsed_time(e1) / 1e3)
    lat.upload(U_th)
    Uh = torch.empty(NL * 4, dtype=torch.float64, pin_memory=True).numpy()
    Uh[:] = U_th
    t0, t1 = lat.slices()
    row = L ** 3 * 4 * 4
    barrier(dist)
    w0 = time.perf_counter()
    for k in range(K):
        lat.upload(Uh)
        lat.md_update("omf2", NSTEPS, TAU, seed=seed, traj=400000 + k)
        lat.download(Uh)
    t_e2e = allmax(dist, time.perf_counter() - w0)
    if rank == 0:
        line = {
            "metric": METRIC, "value": K / t, "unit": "traj/s", "n_gpus": ws, "steps": K,
            "warmup": W, "ms_per_step": 1e3 * t / K, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "fp32 links/forces + fp64 reductions/accept",
            "data": "synthetic: seeded Haar-random start, Metropolis-thermalised on device",
            "config": {"workload": WORKLOAD + " (mixed precision), one lattice over time slabs",
                       "lattice": [L] * 4, "slabs": N, "slices_per_slab": L // N,
                       "parallelism": f"t-slabs x{N}" + (" on one GPU" if ws == 1 else ""),
                       "l2": "working set > 126 MB L2; no flush"},
            "acceptance": sum(r.accepted for r in res) / K,
            "side": side,
            "e2e": {"value": K / t_e2e, "unit": "traj/s",
                    "h2d_bytes_per_step": int(lat.count * (L // N + 2) * row * 8),
                    "d2h_bytes_per_step": int((t1 - t0) * row * 8),
                    "note": "per rank: its slices and ghost slices up, trajectory, its slices "
                            "down; wall clock"},
            "gpu_launches": int(launches),
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    lat.close()
    if dist is not None:
        dist.destroy_process_group()


def reference(args):
    """--impl reference: the reference's stock md_update (std::mt19937 momenta, accept/reject,
    hmc.hpp:86-101) on the host cores, one trajectory per step."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    if not O.available("ref"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libsu2ref.so was not "
                          "built (needs the reference checkout at build time)"}))
        return
    r = O.Oracle("ref")
    threads = r._omp_threads()
    U = haar_links(L ** 4 * 4, 20240)
    with quiet_stdout():
        for k in range(args.warmup):
            U, *_ = r.hmc_run(0, (L, L, L, L), 4, BETA, 6, NSTEPS, TAU, 13526463, k, 1, U)
        t0 = time.perf_counter()
        for k in range(args.steps):
            U, acc, dH, plaq = r.hmc_run(0, (L, L, L, L), 4, BETA, 6, NSTEPS, TAU, 13526463,
                                         args.warmup + k, 1, U)
        dt = time.perf_counter() - t0
    v = args.steps / dt
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "traj/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
        "data": "synthetic: seeded Haar-random start",
        "config": {"workload": WORKLOAD + " (reference CPU, FP64)", "lattice": [L] * 4},
        "cpu_baseline": {"value": v, "unit": "traj/s", "cores": threads, "kind": "reference",
                         "sample": f"{args.steps} full trajectories of the workload"},
        "e2e": {"value": v, "unit": "traj/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def profile_run(args):
    """--profile-run: a bare loop of one operation of the 32^4 workload, for ncu.

    A Haar-random 32^4 start (untimed work does not change what a kernel reads or writes),
    the force kernel's launch shape fixed by --force-variant instead of the tuner, then W
    warm-up and K steps of one precision.  --profile-op picks the step: an omf2 trajectory
    (hmc), a Metropolis sweep (delta 0.15, 8 hits), an RK3 Wilson-flow step (eps 0.01), or
    (all) each of these plus every other kernel of the path once: plaquette, clover, Polyakov
    and Wilson loops, APE smearing, gauge-file save/load, download, CG / BiCGStab (and the
    mixed CG, or in FP64 a pseudofermion trajectory) on the U(1) 256^2 staggered workload,
    and a leapfrog trajectory of eight chains of the batched ensemble.
    Prints one JSON line with the number of kernel launches made before the K steps (the ncu
    ``-s`` to skip to them) and per step.
    """
    import torch

    import su2_b200
    V = L ** 4
    c = su2_b200.gaugeconfig(L, L, L, L, 4, BETA, precision=args.precision)
    c.upload(haar_links(V * 4, 20240))
    c.force_variant = args.force_variant

    u1 = batch = None
    if args.profile_op == "all":
        # the staggered solvers run on the U(1) 256^2 workload (vectors of 65,536 sites)
        u1 = su2_b200.gaugeconfig(256, 1, 1, 256, 2, 4.0, group="u1", precision=args.precision)
        u1.upload(np.random.default_rng(4242).uniform(-np.pi, np.pi, size=256 * 256 * 2))
        b = np.random.default_rng(4243).normal(size=2 * 256 * 256)
        # the batched kernels on the first eight chains of the 64-chain ensemble
        from su2_b200.batch import chain_batch
        from su2_b200 import replicas
        chains = ensemble_chains()[:8]
        batch = chain_batch(chains, precision="mixed")
        for i, ch in enumerate(chains):
            batch.upload(i, haar_links(replicas.chain_sites(ch) * ch["ndims"], ch["seed"]))
    td = tempfile.mkdtemp()

    def step(k):
        if args.profile_op in ("hmc", "all"):
            c.md_update("omf2", NSTEPS, TAU, seed=20240, traj=k)
        if args.profile_op in ("metropolis", "all"):
            c.sweep(0.15, 8, 20240, k)
        if args.profile_op in ("flow", "all"):
            c.runge_kutta(0.01)
        if args.profile_op == "all":  # every other kernel of the path, once
            c.gauge_energy()
            c.energy_density()
            c.polyakov_loop_spatial_average()
            c.wilsonloop(2, 2)
            path = os.path.join(td, "conf")
            c.save(path)
            c.load(path)
            c.APEsmearing(0.5)
            c.download()
            u1.solve(b, 0.05, tol=1e-10, solver="CG", tol_mode="rel")
            u1.solve(b, 0.05, tol=1e-10, solver="BiCGStab", tol_mode="rel")
            if args.precision == "mixed":
                u1.solve(b, 0.05, tol=1e-10, solver="CG_mixed", tol_mode="rel")
            else:  # pseudofermion trajectory (det D D^+ monomial, FP64 U(1) only)
                u1.md_update("omf2", 2, 0.2, seed=7, traj=k, fermion_mass=0.05, cg_tol=1e-10)
            batch.md_update("leapfrog", 10, 1.0, traj=k)

    def launches():  # over every context of the loop
        n = c.kernel_launches()
        if u1 is not None:
            n += u1.kernel_launches() + batch.kernel_launches()
        return n

    for k in range(args.warmup):
        step(k)
    c.synchronize()
    if u1 is not None:
        u1.synchronize()
        torch.cuda.synchronize()
    n0 = launches()
    for k in range(args.steps):
        # an NVTX range per timed step, so that a profiler can select exactly these launches
        # (ncu --nvtx --nvtx-include "profile_step/")
        torch.cuda.nvtx.range_push("profile_step")
        step(args.warmup + k)
        torch.cuda.nvtx.range_pop()
    c.synchronize()
    n1 = launches()
    print(json.dumps({"profile_run": f"SU(2) d=4 {L}^4, beta={BETA}", "op": args.profile_op,
                      "precision": args.precision,
                      "force_variant": su2_b200._abi.FORCE_SHAPES[args.force_variant],
                      "setup_launches": n0, "launches_per_step": (n1 - n0) / max(1, args.steps),
                      "steps": args.steps, "warmup": args.warmup}), flush=True)
    c.close()
    if u1 is not None:
        u1.close()
        batch.close()
    torch.cuda.synchronize()


# --------------------------------------------------------------------------------------
# The other workloads of the su2 hot path (``--config N``).  Each prints one JSON line of
# its own; the default run (config 2) is the headline above.

def _line(metric, value, unit, args, ws, ms_per_step, config, **extra):
    d = {"metric": metric, "value": value, "unit": unit, "n_gpus": ws, "steps": args.steps,
         "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
         "scaling": "weak", "vs_baseline": None, "data": "synthetic (seeded)",
         "config": config}
    d.update(extra)
    print(json.dumps(d), flush=True)


def _events(stream):
    import torch
    s = torch.cuda.ExternalStream(stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    return s, a, b


def config1(args):
    """SU(2) d=4 8^4, beta 2.3, leapfrog tau 1 n 10, FP64, plaquette every trajectory: the
    reference's own CPU run and the plain method.  K trajectories (default 200) after W."""
    import torch

    import su2_b200
    ws, rank, local, dist = dist_setup()
    torch.cuda.set_device(local)
    from su2_b200 import replicas
    seed = replicas.replica_seed(13526463, rank)
    K, W = args.steps, args.warmup
    c = su2_b200.gaugeconfig(8, 8, 8, 8, 4, 2.3, precision="fp64", device=local)
    c.upload(haar_links(8 ** 4 * 4, seed))
    tune = c.autotune()  # the launch shape that suits 8^4 is not the one of 32^4
    c.upload(haar_links(8 ** 4 * 4, seed))
    for k in range(W):
        c.md_update("leapfrog", 10, 1.0, seed=seed, traj=k)
    s, e0, e1 = _events(c.stream())
    barrier(dist)
    n0 = c.kernel_launches()
    e0.record(s)
    res = [c.md_update("leapfrog", 10, 1.0, seed=seed, traj=W + k) for k in range(K)]
    e1.record(s)
    e1.synchronize()
    t = allmax(dist, e0.elapsed_time(e1) / 1e3)
    plaq = [r.plaquette / (8 ** 4 * 6 * 2) for r in res]
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        if O.available("ref"):
            r = O.Oracle("ref")
            U = haar_links(8 ** 4 * 4, seed)
            n = 200
            with quiet_stdout():
                t0 = time.perf_counter()
                r.hmc_run(0, (8, 8, 8, 8), 4, 2.3, 0, 10, 1.0, 13526463, 0, n, U)
                dt = time.perf_counter() - t0
            cpu = {"value": n / dt, "unit": "traj/s", "cores": r._omp_threads(),
                   "kind": "reference", "sample": f"{n} leapfrog trajectories of the 8^4 "
                                                  "workload, md_update + accept/reject"}
    if rank == 0:
        _line("SU(2) 8^4 leapfrog HMC traj/s (FP64)", ws * K / t, "traj/s", args, ws,
              1e3 * t / K, {"workload": "SU(2) d=4 8^4 beta=2.3 leapfrog tau=1 n=10, FP64, "
                                        "Haar start", "replicas": ws},
              dtype="fp64", acceptance=sum(r.accepted for r in res) / K,
              plaquette_mean=float(np.mean(plaq)), plaquette_last=plaq[-1],
              gpu_launches=c.kernel_launches() - n0, cpu_baseline=cpu,
              autotune_force_us={str(su2_b200._abi.FORCE_SHAPES[k]): v for k, v in tune.items()},
              force_shape=su2_b200._abi.FORCE_SHAPES[c.force_variant])
    c.close()


def config3(args):
    """U(1) d=2 256^2, beta 4.0, staggered m 0.05: CG on D D^+ to relative 1e-10 in FP64 and
    FP32-inner / FP64-reliable-update, BiCGStab on D with the same right-hand side, and the
    HMC trajectory with the det(D D^+) monomial (omf2 tau 1, n 10)."""
    import torch

    import su2_b200
    ws, rank, local, dist = dist_setup()
    torch.cuda.set_device(local)
    L, m, beta = 256, 0.05, 4.0
    V = L * L
    rng = np.random.default_rng(4242 + rank)
    U = rng.uniform(-np.pi, np.pi, size=V * 2)
    b = rng.normal(size=2 * V)
    out = {}
    solves = {}
    for name, prec, solver in (("cg_fp64", "fp64", "CG"), ("cg_mixed", "mixed", "CG_mixed"),
                               ("bicgstab_fp64", "fp64", "BiCGStab")):
        c = su2_b200.gaugeconfig(L, 1, 1, L, 2, beta, group="u1", precision=prec, device=local)
        c.upload(U)
        for _ in range(max(1, args.warmup)):
            c.solve(b, m, tol=1e-10, solver=solver, tol_mode="rel")
        s, e0, e1 = _events(c.stream())
        barrier(dist)
        e0.record(s)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            r = c.solve(b, m, tol=1e-10, solver=solver, tol_mode="rel")
        e1.record(s)
        e1.synchronize()
        wall = time.perf_counter() - t0
        t = allmax(dist, e0.elapsed_time(e1) / 1e3)
        solves[name] = {"ms_per_solve": 1e3 * t / args.steps, "iterations": r.iterations,
                        "restarts": r.restarts,
                        "true_residual_rel": r.true_residual / float(np.linalg.norm(b)),
                        "wall_ms_per_solve": 1e3 * wall / args.steps}
        if name == "cg_fp64":
            x64 = r.x
        elif name == "cg_mixed":
            solves[name]["x_rel_diff_vs_cg_fp64"] = float(np.linalg.norm(r.x - x64) /
                                                          np.linalg.norm(x64))
        if name == "cg_fp64":
            # pseudofermion HMC trajectory (det D D^+ monomial), FP64
            c.md_update("omf2", 10, 1.0, seed=7, traj=0, fermion_mass=m, cg_tol=1e-10)
            acc = []
            e0.record(s)
            nt = max(2, args.steps // 2)
            for k in range(nt):
                acc.append(c.md_update("omf2", 10, 1.0, seed=7, traj=1 + k, fermion_mass=m,
                                       cg_tol=1e-10))
            e1.record(s)
            e1.synchronize()
            out["hmc"] = {"traj_per_s": nt / (e0.elapsed_time(e1) / 1e3),
                          "acceptance": sum(a.accepted for a in acc) / nt,
                          "cg_iterations_per_traj": float(np.mean([a.cg_iterations
                                                                   for a in acc]))}
            # pion correlator (propagator.hpp:25-65): one CG solve and the time-slice sums
            c.upload(U)
            C_pi = c.C_pion(m, tol=1e-10)
            npi = max(2, args.steps // 2)
            t0 = time.perf_counter()
            for _ in range(npi):
                C_pi = c.C_pion(m, tol=1e-10)
            out["pion"] = {"ms_per_correlator": 1e3 * (time.perf_counter() - t0) / npi,
                           "C1": float(C_pi[1]), "timeslices": len(C_pi),
                           "note": "C(0) is skipped, as the reference does (contact term)"}
        c.close()
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        if O.available("ref"):
            r = O.Oracle("ref")
            tol_abs = 1e-10 * float(np.linalg.norm(b))  # CG.hpp stops on |r| < tol
            t0 = time.perf_counter()
            xr, it = r.cg_ddag((L, 1, 1, L), 2, U, m, b, np.zeros_like(b), tol_abs)
            dt = time.perf_counter() - t0
            cpu = {"value": 1.0 / dt, "unit": "solves/s", "cores": r._omp_threads(),
                   "kind": "reference", "sample": f"1 LinearCG solve on D D^+ to |r| < 1e-10 |b| "
                                                  f"({it} iterations incl. restarts)",
                   "x_rel_diff_vs_cg_fp64": float(np.linalg.norm(xr - x64) /
                                                  np.linalg.norm(xr))}
    if rank == 0:
        v = ws * 1e3 / solves["cg_fp64"]["ms_per_solve"]
        _line("U(1) 256^2 staggered CG on DD^+ to rel 1e-10: solves/s", v, "solves/s", args,
              ws, solves["cg_fp64"]["ms_per_solve"],
              {"workload": "U(1) d=2 256x256 beta=4.0 staggered m=0.05, hot start",
               "replicas": ws}, dtype="fp64 (and fp32-inner mixed CG)", solvers=solves,
              fermion_hmc=out.get("hmc"), pion_correlator=out.get("pion"), cpu_baseline=cpu)


def ensemble_chains(n=64, seed=20250):
    """Seeded ensemble: SU(2) d=4 with L in {8..24} and d=3 with L in {16..48} (even extents,
    as the even/odd layout and the checkerboard require), beta uniform in [2.0, 2.6]."""
    rng = np.random.default_rng(seed)
    chains = []
    for i in range(n):
        if i % 2 == 0:
            L = int(rng.integers(4, 13)) * 2
            chains.append(dict(dims=(L, L, L, L), ndims=4, beta=float(rng.uniform(2.0, 2.6)),
                               seed=7000 + i))
        else:
            L = int(rng.integers(8, 25)) * 2
            chains.append(dict(dims=(L, L, 1, L), ndims=3, beta=float(rng.uniform(2.0, 2.6)),
                               seed=7000 + i))
    return chains


def config4(args):
    """64 independent SU(2) chains of uneven sizes, leapfrog tau 1 n 10, FP32 links with FP64
    sums: one batched graph per trajectory (persistent kernels over all chains' tiles) against
    the same chains run one by one (one context and graph per chain).  Site-updates = sites x
    trajectories.  With N ranks the chains are partitioned by replicas.partition_chains."""
    import torch

    import su2_b200
    from su2_b200 import replicas
    from su2_b200.batch import chain_batch
    ws, rank, local, dist = dist_setup()
    torch.cuda.set_device(local)
    chains = ensemble_chains()
    mine = [chains[i] for i in replicas.partition_chains(chains, ws, rank)]
    sites = sum(replicas.chain_sites(c) for c in mine)
    starts = [haar_links(replicas.chain_sites(c) * c["ndims"], c["seed"]) for c in mine]
    K, W = args.steps, args.warmup
    with chain_batch(mine, precision="mixed", device=local) as b:
        for i, U in enumerate(starts):
            b.upload(i, U)
        tune = b.autotune()  # launch shape of the batched kernels, timed on this ensemble
        for k in range(W):
            b.md_update("leapfrog", 10, 1.0, traj=k)
        s, e0, e1 = _events(b.stream())
        barrier(dist)
        n0 = b.kernel_launches()
        e0.record(s)
        res = [b.md_update("leapfrog", 10, 1.0, traj=W + k) for k in range(K)]
        e1.record(s)
        e1.synchronize()
        t_b = allmax(dist, e0.elapsed_time(e1) / 1e3)
        launches = b.kernel_launches() - n0
    total_sites = replicas.sum_over_ranks(sites) if dist is not None else sites
    # one by one: every chain its own context and trajectory graph, run back to back, in the
    # same precision (mixed) and in the plain form (FP64)
    def one_by_one(precision):
        ctxs = []
        for c, U in zip(mine, starts):
            Lx, Ly, Lz, Lt = c["dims"]
            g = su2_b200.gaugeconfig(Lx, Ly, Lz, Lt, c["ndims"], c["beta"],
                                     precision=precision, device=local)
            g.upload(U)
            g.autotune(os.path.join(tempfile.gettempdir(), "su2b_tune_cache.txt"))
            for k in range(W):
                g.md_update("leapfrog", 10, 1.0, seed=c["seed"], traj=k)
            ctxs.append(g)
        torch.cuda.synchronize()
        barrier(dist)
        t0 = time.perf_counter()
        for k in range(K):
            for c, g in zip(mine, ctxs):
                g.md_update("leapfrog", 10, 1.0, seed=c["seed"], traj=W + k)
        torch.cuda.synchronize()
        t = allmax(dist, time.perf_counter() - t0)
        for g in ctxs:
            g.close()
        return t

    t_1 = one_by_one("mixed")
    t_64 = one_by_one("fp64")
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        if O.available("ref"):
            r = O.Oracle("ref")
            c = max(chains, key=replicas.chain_cost)
            Lx, Ly, Lz, Lt = c["dims"]
            U = haar_links(replicas.chain_sites(c) * c["ndims"], 1)
            with quiet_stdout():
                t0 = time.perf_counter()
                r.hmc_run(0, c["dims"], c["ndims"], c["beta"], 0, 10, 1.0, 1, 0, 1, U)
                dt = time.perf_counter() - t0
            cpu = {"value": replicas.chain_sites(c) / dt, "unit": "site-updates/s",
                   "cores": r._omp_threads(), "kind": "reference",
                   "sample": f"1 leapfrog trajectory of the largest chain {c['dims']} "
                             f"d={c['ndims']}"}
    if rank == 0:
        _line("64-chain SU(2) ensemble leapfrog HMC site-updates/s (batched)",
              total_sites * K / t_b, "site-updates/s", args, ws, 1e3 * t_b / K,
              {"workload": "64 SU(2) chains, d=4 L in 8..24 and d=3 L in 16..48 (even), beta "
                           "U[2.0,2.6], leapfrog tau=1 n=10, FP32 links + FP64 sums",
               "chains": len(chains), "sites_total": int(total_sites),
               "parallelism": f"chains partitioned over {ws} rank(s)"},
              dtype="fp32 links + fp64 sums", one_by_one_site_updates_per_s=total_sites * K / t_1,
              batch_autotune_force_us={str(su2_b200._abi.BATCH_SHAPES[v]): us
                                       for v, us in tune.items()},
              batched_over_one_by_one=t_1 / t_b,
              one_by_one_fp64_site_updates_per_s=total_sites * K / t_64,
              batched_mixed_over_one_by_one_fp64=t_64 / t_b,
              acceptance=float(np.mean([r.accepted for rr in res for r in rr])),
              gpu_launches=int(launches), cpu_baseline=cpu)


def config5(args):
    """SU(2) d=4 24^4 beta 2.4 from a GPU-thermalised field: the Wilson action's backward
    against central finite differences (eps 1e-6, FP64) on 1000 random links and against the
    gauge force, and the gradient of t^2 E(t = 2) (eps 0.01, 200 RK3 steps, checkpoints every
    14 steps) in FP64 and FP32 with the FP32 error against FP64."""
    import torch

    import su2_b200
    ws, rank, local, dist = dist_setup()
    torch.cuda.set_device(local)
    L = 24
    NL = L ** 4 * 4
    c = su2_b200.gaugeconfig(L, L, L, L, 4, 2.4, precision="fp64", device=local)
    c.upload(haar_links(NL, 99 + rank))
    for sweep in range(100):
        c.sweep(0.15, 8, 99, sweep)
    for k in range(10):
        c.md_update("omf2", 16, 1.0, seed=99, traj=k)
    U = c.download()
    S, dS = c.action_backward()
    F = c.derivative()
    force_rel = float(np.linalg.norm(dS - F) / np.linalg.norm(F))
    rng = np.random.default_rng(5)
    links = rng.choice(NL, size=1000, replace=False)
    comps = rng.integers(0, 3, size=1000)
    eps = 1e-6
    fd_err = []
    V_ = U.copy()
    t0 = time.perf_counter()
    for l, k in zip(links, comps):
        vals = []
        for sgn in (1.0, -1.0):
            x = np.zeros(3)
            x[k] = sgn * eps
            q = U[4 * l:4 * l + 4]
            # exp(x) (exp_gauge.cc:8-18) times the link, in the (a, b) form of su2.hh
            al = np.linalg.norm(x)
            e = np.array([np.cos(al), np.sin(al) * x[2] / al, np.sin(al) * x[1] / al,
                          np.sin(al) * x[0] / al])
            a = complex(e[0], e[1]) * complex(q[0], q[1]) - complex(e[2], e[3]) * \
                complex(q[2], -q[3])
            bb = complex(e[0], e[1]) * complex(q[2], q[3]) + complex(e[2], e[3]) * \
                complex(q[0], -q[1])
            V_[4 * l:4 * l + 4] = [a.real, a.imag, bb.real, bb.imag]
            c.upload(V_)
            vals.append(c.get_S_G_hmc())
            V_[4 * l:4 * l + 4] = q
        fd = (vals[0] - vals[1]) / (2 * eps)
        fd_err.append(abs(fd - dS[3 * l + k]) / max(1.0, abs(dS[3 * l + k])))
    t_fd = time.perf_counter() - t0
    c.upload(U)
    out = {}
    grads = {}
    for prec in ("fp64", "mixed"):
        g = c if prec == "fp64" else su2_b200.gaugeconfig(L, L, L, L, 4, 2.4, precision=prec,
                                                           device=local)
        g.upload(U)
        g.flow_objective(0.01, 200, grad=True, checkpoint_every=14)  # warm-up
        s, e0, e1 = _events(g.stream())
        barrier(dist)
        e0.record(s)
        for _ in range(args.steps):
            O, grad = g.flow_objective(0.01, 200, grad=True, checkpoint_every=14)
        e1.record(s)
        e1.synchronize()
        t = allmax(dist, e0.elapsed_time(e1) / 1e3) / args.steps
        out[prec] = {"ms_per_gradient": 1e3 * t, "objective": O}
        grads[prec] = grad
        if g is not c:
            g.close()
    out["mixed"]["grad_rel_err_vs_fp64"] = float(np.linalg.norm(grads["mixed"] - grads["fp64"]) /
                                                 np.linalg.norm(grads["fp64"]))
    out["mixed"]["objective_rel_err_vs_fp64"] = abs(out["mixed"]["objective"] -
                                                    out["fp64"]["objective"]) / \
        abs(out["fp64"]["objective"])
    c.close()
    if rank == 0:
        t = out["fp64"]["ms_per_gradient"] / 1e3
        _line("SU(2) 24^4 gradient of t^2 E(t=2) w.r.t. the initial links: gradients/s (FP64)",
              ws / t, "gradients/s", args, ws, 1e3 * t,
              {"workload": "SU(2) d=4 24^4 beta=2.4, GPU-thermalised (100 Metropolis sweeps + "
                           "10 omf2 trajectories); flow eps=0.01 to t=2, checkpoints every 14",
               "replicas": ws},
              dtype="fp64 (and fp32)", flow_gradient=out,
              action_backward={"S": S, "rel_diff_vs_gauge_force": force_rel,
                               "fd_links": 1000, "fd_eps": eps,
                               "fd_max_rel_err": float(np.max(fd_err)),
                               "fd_median_rel_err": float(np.median(fd_err)),
                               "fd_seconds": t_fd})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--therm-sweeps", type=int, default=300)
    ap.add_argument("--stat-traj", type=int, default=5000,
                    help="untimed trajectories per precision for the Delta H / plaquette "
                         "comparison")
    ap.add_argument("--pairs", type=int, default=32,
                    help="paired trajectories (same start, same momenta) per precision")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-run", action="store_true",
                    help="only the timed loop of one precision, for ncu (no bench line)")
    ap.add_argument("--profile-op", default="hmc", choices=["hmc", "metropolis", "flow", "all"],
                    help="with --profile-run: the step of the loop")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--force-variant", type=int, default=3)
    ap.add_argument("--config", type=int, default=2, choices=[1, 2, 3, 4, 5],
                    help="2: the headline 32^4 HMC; 1, 3, 4, 5: the other workloads")
    ap.add_argument("--slabs", type=int, default=0,
                    help="one 32^4 lattice over N time slabs: one per rank under torchrun "
                         "(NCCL), all on the GPU as one process (strong scaling)")
    args = ap.parse_args()
    if args.profile_run:
        profile_run(args)
    elif args.impl == "ours" and args.slabs:
        slabs_run(args)
    elif args.impl == "ours" and args.config != 2:
        {1: config1, 3: config3, 4: config4, 5: config5}[args.config](args)
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            dist.destroy_process_group()
    elif args.impl == "reference":
        reference(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
