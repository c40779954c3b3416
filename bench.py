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
            if self.stop_flag.wait(0.002):
                break

    def start(self):
        if self.h is None:
            return
        self.samples, self.reasons = [], 0
        self.stop_flag.clear()
        self.t = threading.Thread(target=self._poll, daemon=True)
        self.t.start()

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
    if ws > 1:
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
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allsum(dist, x):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


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


def ours(args):
    import torch

    import su2_b200
    ws, rank, local, dist = dist_setup()
    torch.cuda.set_device(local)
    K, W = args.steps, args.warmup
    V = L ** 4
    NL = V * 4
    seed = 20240 + 1000 * rank

    # ---- thermalised start (untimed): Haar start, Metropolis sweeps, HMC warm-up ----
    U0 = haar_links(NL, seed)
    mixed = su2_b200.gaugeconfig(L, L, L, L, 4, BETA, precision="mixed", device=local)
    mixed.upload(U0)
    for sweep in range(args.therm_sweeps):
        mixed.sweep(0.15, 8, seed, sweep)
    for k in range(THERM_TRAJ + max(W, 3)):
        mixed.md_update("omf2", NSTEPS, TAU, seed=seed, traj=100000 + k)
    U_th = mixed.download()
    tune_m = mixed.autotune()  # launch shape of the force kernel, timed on this field

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

    # ---- FP64 path, same start and seeds ----
    fp64 = su2_b200.gaugeconfig(L, L, L, L, 4, BETA, precision="fp64", device=local)
    fp64.upload(U_th)
    tune_d = fp64.autotune()
    fp64.upload(U_th)
    for k in range(min(W, 2)):
        fp64.md_update("omf2", NSTEPS, TAU, seed=seed + 7, traj=200000 + k)
    fp64.upload(U_th)
    barrier(dist)
    t_fp64, res_d = run_chain(fp64, K, seed, 0, None)
    t_fp64 = allmax(dist, t_fp64)

    # ---- roofline of the dominant kernel (fused staple/force/momentum), live timers ----
    roof = {}
    kernels = {}
    hbm, peak_src = peaks()
    # every force launch of the fused trajectory reads U and P, writes P and writes the next
    # link buffer (exp(dt P) U, or restoreSU(U) after the last step): 56 B/link in FP32
    # storage, 112 B/link in FP64
    for name, c, bpl in (("mixed", mixed, 56), ("fp64", fp64, 112)):
        c.upload(U_th)
        c.profile(True)
        for k in range(max(2, K // 2)):
            c.md_update("omf2", NSTEPS, TAU, seed=seed, traj=300000 + k)
        prof = c.profile_read()
        c.profile(False)
        n, ms = prof["force"]
        avg = ms / 1e3 / n
        roof[name] = {"avg_us": avg * 1e6, "GB/s": bpl * NL / avg / 1e9}
        per = {}
        nb = {"force": bpl, "plaquette": 32 if name == "fp64" else 16,
              "momenta": 24 if name == "fp64" else 12}
        for kname, (kn, kms) in prof.items():
            if kn:
                d = {"launches": kn, "avg_us": kms * 1e3 / kn}
                if kname in nb:
                    d["GB/s"] = nb[kname] * NL / (kms / 1e3 / kn) / 1e9
                per[kname] = d
        kernels[name] = per
    traffic = None
    tp = os.path.join(ROOT, "profiles", "force_kernel_traffic.json")
    if os.path.exists(tp):
        traffic = json.load(open(tp)).get("mixed_bytes_per_launch")

    # ---- e2e through the C ABI with host buffers (pinned), per trajectory:
    #      upload the host gaugeconfig, one trajectory, download the gaugeconfig ----
    Uh = torch.empty(NL * 4, dtype=torch.float64, pin_memory=True).numpy()
    Uh[:] = U_th
    mixed.upload(Uh)
    barrier(dist)
    t0 = time.perf_counter()
    for k in range(K):
        mixed.upload(Uh)
        r = mixed.md_update("omf2", NSTEPS, TAU, seed=seed, traj=400000 + k)
        Uh[:] = mixed.download()
    t_e2e = allmax(dist, time.perf_counter() - t0)

    # ---- side measurements of config 2 (Metropolis sweep, flow step) ----
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

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(U_th)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "traj/s", "n_gpus": ws, "steps": K,
            "warmup": W, "ms_per_step": 1e3 * t_mixed / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "fp32 links/forces + fp64 reductions/accept",
            "data": "synthetic: seeded Haar-random start, Metropolis-thermalised on device",
            "config": {"workload": WORKLOAD + " (mixed precision)", "lattice": [L] * 4,
                       "beta": BETA, "integrator": "omf2", "n_steps": NSTEPS, "tau": TAU,
                       "replicas": ws, "parallelism": f"replicas x{ws}",
                       "l2": "working set per step (U, U_old, P) > 126 MB L2; no flush"},
            "mixed": dict(traj_per_s=value, **stats(res_m, V)),
            "fp64": dict(traj_per_s=ws * K / t_fp64, **stats(res_d, V)),
            "speedup_mixed_vs_fp64": t_fp64 / t_mixed,
            "roofline": {"bound": "hbm",
                         "kernel": "k_force_su2<float,4>: staples, force, momentum step and the "
                                   "following link update, fused (FP32 storage)",
                         "achieved": roof["mixed"]["GB/s"], "peak": hbm, "unit": "GB/s",
                         "frac": roof["mixed"]["GB/s"] / hbm, "traffic": traffic,
                         "bytes_per_launch": 56 * NL, "avg_launch_us": roof["mixed"]["avg_us"],
                         "peak_source": peak_src,
                         "fp64_kernel": {"achieved": roof["fp64"]["GB/s"],
                                         "frac": roof["fp64"]["GB/s"] / hbm,
                                         "bytes_per_launch": 112 * NL,
                                         "avg_launch_us": roof["fp64"]["avg_us"]}},
            "kernels": kernels,
            "autotune_force_us": {"mixed": {str(su2_b200._abi.FORCE_SHAPES[k]): v
                                            for k, v in tune_m.items()},
                                  "fp64": {str(su2_b200._abi.FORCE_SHAPES[k]): v
                                           for k, v in tune_d.items()},
                                  "chosen": {"mixed": su2_b200._abi.FORCE_SHAPES[mixed.force_variant],
                                             "fp64": su2_b200._abi.FORCE_SHAPES[fp64.force_variant]}},
            "metropolis_sweeps_per_s": metro, "flow_rk3_steps_per_s_fp64": flow,
            "e2e": {"value": ws * K / t_e2e, "unit": "traj/s",
                    "h2d_bytes_per_step": int(NL * 4 * 8), "d2h_bytes_per_step": int(NL * 4 * 8),
                    "note": "upload of the host gaugeconfig (reference layout, FP64, pinned) "
                            "+ trajectory + download, wall clock"},
            "gpu_launches": int(launches),
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
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
            "sample": "1 omf2 trajectory (16 steps, 33 force evaluations) of the 32^4 workload "
                      "through the reference's integrator/monomial code, OpenMP"}


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
    """--profile-run: the bare timed loop of the headline workload, for ncu.

    A Haar-random 32^4 start (untimed work does not change what a kernel reads or writes),
    the force kernel's launch shape fixed by --force-variant instead of the tuner, W warm-up
    and K trajectories of one precision.  Prints one JSON line with the number of kernel
    launches made before the K trajectories (the ncu ``-s`` to skip to them) and per
    trajectory.
    """
    import torch

    import su2_b200
    V = L ** 4
    c = su2_b200.gaugeconfig(L, L, L, L, 4, BETA, precision=args.precision)
    c.upload(haar_links(V * 4, 20240))
    c.force_variant = args.force_variant
    for k in range(args.warmup):
        c.md_update("omf2", NSTEPS, TAU, seed=20240, traj=k)
    c.synchronize()
    n0 = c.kernel_launches()
    for k in range(args.steps):
        c.md_update("omf2", NSTEPS, TAU, seed=20240, traj=args.warmup + k)
    c.synchronize()
    n1 = c.kernel_launches()
    print(json.dumps({"profile_run": WORKLOAD, "precision": args.precision,
                      "force_variant": su2_b200._abi.FORCE_SHAPES[args.force_variant],
                      "setup_launches": n0, "launches_per_traj": (n1 - n0) / max(1, args.steps),
                      "steps": args.steps, "warmup": args.warmup}), flush=True)
    c.close()
    torch.cuda.synchronize()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--therm-sweeps", type=int, default=300)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-run", action="store_true",
                    help="only the timed loop of one precision, for ncu (no bench line)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--force-variant", type=int, default=3)
    args = ap.parse_args()
    if args.profile_run:
        profile_run(args)
    elif args.impl == "reference":
        reference(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
