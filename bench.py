"""Throughput of the HMC hot path: force+logdet evaluations/s on a 32x32
triangular lattice with Nt = 64 (beta = 20, J = (1,-.5,-.5), lambda = (.3,.15,.15),
mu0 = -3, omega0 = 0.05), on synthetic N(0,1) phonon fields.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one evaluation = construct_M_hat + LU log det/inverse + force
(the body of leap_frog, simulation/organic_hmc.c:177-180).  The headline
`value` is the mixed-precision adjoint path (FP64 M_hat, LU and log det,
FP32 force sweep); the FP64 reference-algorithm path and the FP64 adjoint are
measured beside it on the same GPU (`paths`).  N GPUs run independent
replicas (one process per GPU, no data-path collective).

`--impl reference` times the reference's own C/OpenMP implementation
(oracle/_ref, compiled unmodified) on this host's cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "electron-phonon-hmc_b200"))

METRIC = "force+logdet evals/s, 32x32 lattice Nt=64: mixed vs FP64 plain, same B200"
UNIT = "evals/s"
L, NT, BETA = 32, 64, 20.0
J, LAM, MU0, OMEGA0 = (1.0, -0.5, -0.5), (0.3, 0.15, 0.15), -3.0, 0.05
WORKLOAD = "32x32 triangular lattice (V=1024), Nt=64, beta=20, force+logdet eval"

# Algorithmic work of one evaluation (reference algorithm, Taylor-4 as two pairs):
# FLOP = V^2 Nt (84 (1 + log2 Nt) + 170) + 2 V^3 ; per slice application 84 V^2 flop.
V = L * L
FLOP_PER_EVAL = V * V * NT * (84 * (1 + 6) + 170) + 2 * V ** 3
# adjoint force sweep (one launch): per vector, site and slice 7 stencils (7 FMA each),
# 3 pair combinations, link contraction (3 links x 8 products) ~ 173 flop
ADJ_SWEEP_FLOP = 173 * V * V * NT
# sweep 1 (M_hat and the q stack): Nt slice applications of 84 flop per site and vector
SWEEP1_FLOP = 84 * V * V * NT
# LU + inverse (getrf + getri): 2 V^3
LU_FLOP = 2 * V ** 3


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([s.strip() for s in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 5 + i and s[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def cpu_baseline(max_seconds=25.0):
    """The reference's C/OpenMP path (oracle/_ref) on this host's cores; bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Model, Reference
    ref = Reference()
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    m = Model.physical(L, L, NT, BETA, J, LAM, MU0, OMEGA0)
    ctx = ref.context(m)
    times = []
    seed = 1
    t_start = time.perf_counter()
    while True:
        x = ref.random_x(seed, m.dim)
        ctx.eval(x)
        times.append(ctx.last_time())
        seed += 1
        if time.perf_counter() - t_start > max_seconds or len(times) >= 20:
            break
    ctx.close()
    per = sum(times) / len(times)
    return {"value": 1.0 / per, "unit": UNIT, "cores": cores, "kind": "reference",
            "sample": f"{len(times)} evals (seeds 1..{len(times)}) of the 32x32 Nt=64 workload, "
                      f"reference C sources + OpenBLAS, OMP/OpenBLAS threads={cores}",
            "s_per_eval": per}


def run_reference_arm(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Model, Reference
    ref = Reference()
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    m = Model.physical(L, L, NT, BETA, J, LAM, MU0, OMEGA0)
    ctx = ref.context(m)
    # bounded: at most 3 untimed warm-up evals and a sample capped at ~120 s of CPU time
    for w in range(min(args.warmup, 3)):
        ctx.eval(ref.random_x(1000 + w, m.dim))
    times = []
    budget = 120.0
    t0 = time.perf_counter()
    for k in range(args.steps):
        ctx.eval(ref.random_x(1 + k, m.dim))
        times.append(ctx.last_time())
        if time.perf_counter() - t0 > budget:
            break
    ctx.close()
    per = sum(times) / len(times)
    val = 1.0 / per
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": ws, "steps": len(times),
            "warmup": min(args.warmup, 3), "ms_per_step": per * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "global_batch": 1, "seq_len": NT, "parallelism": "host cores"},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"{len(times)} evals of the workload (capped at {budget:.0f} s)"},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(value, dist, device):
    """The largest of `value` over all ranks (the slowest replica sets the
    whole-job time); `value` itself when not distributed."""
    if dist is None:
        return float(value)
    import torch
    tt = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def whole_job_rate(n_ranks, steps, max_seconds):
    """Evaluations per second of all replicas together: every rank runs
    `steps` evaluations; the job takes as long as its slowest rank."""
    return n_ranks * steps / max_seconds


def load_ncu_summary():
    p = os.path.join(ROOT, "profiles", "ncu_summary.json")
    if os.path.exists(p):
        try:
            return json.load(open(p))
        except Exception:
            return {}
    return {}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--paths", default="mixed,adjoint,reference")
    ap.add_argument("--profile", action="store_true",
                    help="run only warm-up + timed evaluations of --paths (for ncu); print nothing")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    W = max(3, args.warmup)
    K = max(1, args.steps)

    import torch
    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    import ephmc
    lib = ephmc.load_library()
    t, kappa, mu, omega = ephmc.convert_params(BETA, NT, J, LAM, MU0, OMEGA0)
    ctx = ephmc.Context(L, L, NT, t, kappa, mu, omega, device=local)
    dim = ctx.dim
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234 + rank)
    xs = [torch.randn(dim, dtype=torch.float64, device=dev, generator=gen) for _ in range(K + W)]
    pd = torch.empty(dim, dtype=torch.float64, device=dev)
    # L2 flush buffer (larger than the 126 MB L2), written between timed steps
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    lib.ephmc_ctx_set_stream(ctx.h, stream.cuda_stream)

    paths = [p for p in args.paths.split(",") if p]
    results = {}
    phase = {}
    for path in paths:
        for w in range(W):
            ctx.eval(xs[K + w], pd, mode=path)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        launches0 = lib.ephmc_launch_count()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        ph = []
        sampler = ClockSampler(local) if path == "mixed" else None
        if sampler:
            sampler.__enter__()
        for k in range(K):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            ctx.eval(xs[k], pd, mode=path)
            ev[k][1].record(stream)
            ph.append(ctx.timings())
        torch.cuda.synchronize()
        if sampler:
            sampler.__exit__()
        launches = lib.ephmc_launch_count() - launches0
        ms = [a.elapsed_time(b) for a, b in ev]
        total_ms = max_over_ranks(sum(ms), dist, dev)
        results[path] = {"ms_per_step": total_ms / K, "value": whole_job_rate(ws, K, total_ms / 1e3),
                         "launches": launches,
                         "clocks": sampler.summary() if sampler else None}
        phase[path] = {"mhat_ms": statistics.median(p[0] for p in ph), "lu_ms": statistics.median(p[1] for p in ph),
                       "force_ms": statistics.median(p[2] for p in ph)}

    if args.profile:
        # profiling mode (under ncu): only the warm-up and timed evaluations above
        ctx.close()
        return 0

    head = "mixed" if "mixed" in results else paths[0]
    r = results[head]

    # e2e: the public C ABI with host buffers (pinned), H2D of x and D2H of the force inside
    xh = torch.empty(dim, dtype=torch.float64, pin_memory=True)
    ph_ = torch.empty(dim, dtype=torch.float64, pin_memory=True)
    xh.copy_(xs[0].cpu())
    xnp, pnp = xh.numpy(), ph_.numpy()
    lib.ephmc_ctx_set_stream(ctx.h, None)
    for _ in range(W):
        ctx.eval(xnp, pnp, mode=head)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(K):
        ctx.eval(xnp, pnp, mode=head)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, dev)
    e2e = {"value": whole_job_rate(ws, K, e2e_s), "unit": UNIT, "h2d_bytes_per_step": 8 * dim,
           "d2h_bytes_per_step": 8 * dim + 8}

    line = None
    if rank == 0:
        fp32 = C_float_peak(lib, False)
        fp64 = C_float_peak(lib, True)
        ncu = load_ncu_summary()
        # per kernel of the headline path: algorithmic flop per launch / in-run duration
        ph = phase[head]
        sweep_peak = fp32 if head == "mixed" else fp64

        def frac(flop, ms, peak):
            ach = flop / (ms * 1e-3) / 1e12 if ms > 0 else None
            return ach, (ach / peak if (ach and peak) else None)

        kernels = {}
        for name, flop, ms, pk, bound in (
                ("k_gj_dataflow (LU, inverse, log det)", LU_FLOP, ph["lu_ms"], fp64, "fp64"),
                ("k_adjoint_strip (force sweep)" if head == "mixed" else "k_adjoint (force sweep)",
                 ADJ_SWEEP_FLOP, ph["force_ms"], sweep_peak, "fp32" if head == "mixed" else "fp64"),
                ("k_slices_strip (M_hat + q stack)", SWEEP1_FLOP, ph["mhat_ms"], fp64, "fp64")):
            ach, fr = frac(flop, ms, pk)
            kernels[name] = {"ms": ms, "achieved_tflops": ach, "peak_tflops": pk, "frac": fr, "bound": bound,
                             "algorithmic_flop_per_launch": flop}
        # the dominant kernel (largest share of the step) is the LU
        ach, fr = frac(LU_FLOP, ph["lu_ms"], fp64)
        roofline = {"bound": "fp64", "kernel": "k_gj_dataflow (LU + inverse + log det, one cooperative launch)",
                    "achieved": ach, "peak": fp64, "unit": "TFLOP/s", "frac": fr,
                    "peak_source": "measured in this run (CUDA-core FP64 FMA probe, ephmc_measure_fma_peak)",
                    "traffic": ncu.get("k_gj_dataflow_dram_bytes_per_launch"),
                    "algorithmic_flop_per_launch": LU_FLOP,
                    "note": "latency-bound: 1024 sequential pivot steps and 127 panel hand-offs",
                    "kernels": kernels}
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            try:
                cpu = cpu_baseline()
            except Exception as e:  # reported, not fatal
                cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                       "sample": f"unavailable: {e}"}
        line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
                "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64+f32" if head == "mixed" else "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "path": head, "global_batch": ws, "seq_len": NT,
                           "parallelism": f"replicas x{ws}", "l2": "flushed between steps (256 MB write), per-step CUDA events",
                           "inputs": "x ~ N(0,1) i.i.d. per link and slice (torch.randn, seed 1234+rank)"},
                "paths": {p: {"evals_per_s": v["value"], "ms_per_step": v["ms_per_step"], **phase[p]}
                          for p, v in results.items()},
                "mixed_over_fp64_plain": (results["mixed"]["value"] / results["reference"]["value"])
                if ("mixed" in results and "reference" in results) else None,
                "trajectories_per_s_estimate": r["value"] / 22.0,
                "roofline": roofline, "fp64_fma_peak_tflops": fp64, "fp32_fma_peak_tflops": fp32,
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": results[head]["launches"],
                "clocks": results[head]["clocks"]}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def C_float_peak(lib, fp64):
    import ctypes as C
    v = C.c_float(0)
    st = lib.ephmc_measure_fma_peak(1 if fp64 else 0, C.byref(v))
    return float(v.value) if st == 0 else None


if __name__ == "__main__":
    sys.exit(main())
