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

`--workload batch` measures 64 independent chains of uneven lattice, Nt, beta
and coupling evaluated together (ephmc_batch_eval), against the same chains
one at a time.

`--workload stabilised` times the mixed force on the re-stabilised FP64 chain
(ephmc_ctx_set_stabilize) at 48x48, Nt = 128, beta = 40.

`--workload trans_loc` measures the static-disorder mode instead:
disorder samples/s of hist_trans_loc (simulation/organic_trans_loc.c:25-83) on
a 64x64 lattice (V = 4096) with 512 frequency bins, beta = 40, one step = one
batch of `--tl-batch` samples (ephmc_tl_run); with `--impl reference` the
reference's hist_trans_loc on the host, one sample per step.
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
TRAJ_BETA = 10.0  # the timed trajectory (beta = 20 diverges in the MD, in the reference as well)
DH_TRAJ = 20      # trajectories of the mixed-vs-FP64 dH comparison in the headline line

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
# the segmented mixed force (segments of 16 slices, m = Nt/16): the M_hat phase
# is sweep 1 plus the FP32 stacks of segments 1..m-1 from the identity
# (C - 1 slices each); the force phase is the FP64 y chain (Nt - C slices),
# m - 1 DGEMMs of 2 V^3 for the segments' start rows, and the FP32 sweep
SEG_C = 16
SEG_M = NT // SEG_C
MIXED_MHAT_FLOP = 84 * V * V * (NT + (SEG_M - 1) * (SEG_C - 1))
MIXED_FORCE_FLOP = 84 * V * V * (NT - SEG_C) + 2 * V ** 3 * (SEG_M - 1) + ADJ_SWEEP_FLOP


# static-disorder workload: input.txt units, converted as organic_main does with
# STATIC_DISORDER.  mu0 = 0: then run_trans_loc's default bin width spans the
# whole band; with mu0 < 0 the reference writes bins past the end of greens.
TL_L, TL_BINS, TL_BETA, TL_MU0 = 64, 512, 40.0, 0.0
TL_A, TL_B = (1.0, 0.0), (0.5, 0.8660254)
TL_METRIC = "disorder samples/s, TL mode 64x64 lattice (V=4096), 512 bins, beta=40"
TL_UNIT = "samples/s"
TL_WORKLOAD = "static disorder: 64x64 triangular lattice (V=4096), 512 frequency bins, beta=40, mu0=0"


# the checkpointing configuration at its own temperature, where the raw slice
# product loses log det to rounding: the re-stabilised chain (48x48, Nt = 128,
# beta = 40, checkpoints every 12 slices, stabilisation segments of 6)
STAB_L, STAB_NT, STAB_BETA, STAB_CKPT = 48, 128, 40.0, 12
STAB_METRIC = "stabilised force+logdet evals/s, 48x48 lattice Nt=128 beta=40 (re-stabilised FP64 chain)"


def run_stabilised_bench(args):
    """evals/s of the mixed force on the re-stabilised chain (ephmc_ctx_set_stabilize):
    W warm-up and K timed evaluations on device-resident N(0,1) fields, beside
    the unstabilised evaluation of the same context for comparison."""
    import torch

    import ephmc
    ws, rank, local = dist_env()
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    lib = ephmc.load_library()
    L_, nt = args.stab_l, STAB_NT
    t, kappa, mu, omega = ephmc.convert_params(STAB_BETA, nt, J, LAM, MU0, OMEGA0)
    ctx = ephmc.Context(L_, L_, nt, t, kappa, mu, omega, device=local)
    ctx.set_checkpoint(STAB_CKPT)
    gen = torch.Generator(device=dev)
    gen.manual_seed(99 + rank)
    x = torch.randn(ctx.dim, dtype=torch.float64, device=dev, generator=gen)
    pd = torch.empty_like(x)
    W, K = max(1, min(args.warmup, 3)), max(1, min(args.steps, 10))
    out = {}
    for stab in ((True,) if args.profile else (False, True)):
        ctx.set_stabilize(stab)
        for _ in range(W):
            ctx.eval(x, pd, mode="mixed")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(K):
            ctx.eval(x, pd, mode="mixed")
        torch.cuda.synchronize()
        out[stab] = (time.perf_counter() - t0) / K
    ctx.close()
    if args.profile or rank != 0:
        return 0
    print(json.dumps({"metric": STAB_METRIC, "value": 1.0 / out[True], "unit": UNIT, "n_gpus": 1, "steps": K,
                      "warmup": W, "ms_per_step": 1e3 * out[True], "higher_is_better": True, "scaling": "weak",
                      "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
                      "config": {"workload": f"{L_}x{L_} lattice, Nt={nt}, beta={STAB_BETA}, checkpoints every "
                                             f"{STAB_CKPT} slices, stabilisation segments of 6, mixed force",
                                 "inputs": "x ~ N(0,1) (torch.randn)"},
                      "unstabilised_ms_per_eval": 1e3 * out[False]}), flush=True)
    return 0


CKPT_METRIC = "force+logdet evals/s, 48x48 lattice Nt=128 beta=40, checkpoints every 12 slices (mixed force)"


def checkpointed_measure(local, rank, L_, W, K):
    """W warm-up and K timed checkpointed mixed evaluations at L_ x L_,
    Nt = 128, beta = 40, checkpoints every 12 slices, on device-resident
    N(0,1) fields: seconds per evaluation (wall clock around K evaluations,
    synchronized on both sides), median phases (M_hat, LU, force) from the
    context's CUDA events, context bytes."""
    import numpy as np
    import torch

    import ephmc
    dev = torch.device("cuda", local)
    nt = STAB_NT
    t, kappa, mu, omega = ephmc.convert_params(STAB_BETA, nt, J, LAM, MU0, OMEGA0)
    ctx = ephmc.Context(L_, L_, nt, t, kappa, mu, omega, device=local)
    ctx.set_checkpoint(STAB_CKPT)
    gen = torch.Generator(device=dev)
    gen.manual_seed(99 + rank)
    x = torch.randn(ctx.dim, dtype=torch.float64, device=dev, generator=gen)
    pd = torch.empty_like(x)
    for _ in range(W):
        ctx.eval(x, pd, mode="mixed")
    torch.cuda.synchronize()
    phases = []
    t0 = time.perf_counter()
    for _ in range(K):
        ctx.eval(x, pd, mode="mixed")
        phases.append(ctx.timings())
    torch.cuda.synchronize()
    per = (time.perf_counter() - t0) / K
    mem = ctx.memory()
    ctx.close()
    ph = np.median(np.array(phases), axis=0)
    return {"s_per_eval": per, "phases_ms": {"mhat": float(ph[0]), "lu": float(ph[1]), "force": float(ph[2])},
            "context_bytes": int(mem)}


def run_checkpointed_bench(args):
    """evals/s of the checkpointed mixed evaluation (the reference's raw slice
    product, no re-stabilisation) at 48x48, Nt = 128, beta = 40, checkpoints
    every 12 slices, with its phases (M_hat, LU, force) from the context's
    events: W warm-up and K timed evaluations on device-resident N(0,1)
    fields.  The raw product's log det is resolved only to about 1e-6 at this
    beta; the timing is that of the method as the reference runs it."""
    import torch

    import ephmc
    ws, rank, local = dist_env()
    torch.cuda.set_device(torch.device("cuda", local))
    ephmc.load_library()
    W, K = max(1, min(args.warmup, 3)), max(1, min(args.steps, 20))
    m = checkpointed_measure(local, rank, args.stab_l, W, K)
    if args.profile or rank != 0:
        return 0
    L_ = args.stab_l
    print(json.dumps({"metric": CKPT_METRIC, "value": 1.0 / m["s_per_eval"], "unit": UNIT, "n_gpus": 1, "steps": K,
                      "warmup": W, "ms_per_step": 1e3 * m["s_per_eval"], "higher_is_better": True,
                      "scaling": "weak", "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
                      "config": {"workload": f"{L_}x{L_} lattice, Nt={STAB_NT}, beta={STAB_BETA}, checkpoints every "
                                             f"{STAB_CKPT} slices, mixed force (segments of {STAB_CKPT})",
                                 "inputs": "x ~ N(0,1) (torch.randn)"},
                      "phases_ms": m["phases_ms"], "context_bytes": m["context_bytes"]}), flush=True)
    return 0


def tl_params():
    sys.path.insert(0, os.path.join(ROOT, "electron-phonon-hmc_b200"))
    import ephmc
    t, kappa, mu, _ = ephmc.convert_params(TL_BETA, TL_BINS, J, LAM, TL_MU0, OMEGA0, static_disorder=True)
    return t, kappa, mu, ephmc.contraction_matrix(TL_A, TL_B)


def tl_flop_per_sample(V):
    """Nominal FP64 work of one sample: tridiagonalisation 4/3 V^3, eigenvector
    back-transformation 2 V^3, the two triangular matrix-element products
    2 x V^3 (the tridiagonal divide and conquer is not counted)."""
    return (4.0 / 3.0 + 2.0 + 2.0) * V ** 3


# batched chains: 64 independent chains of uneven lattice, Nt, beta and coupling
BATCH_N, BATCH_SEED = 64, 2024
BATCH_METRIC = "chain force+logdet evals/s, 64 uneven chains (L 8-32, Nt 16-64, beta 5-40) in one batch"
BATCH_UNIT = "chain evals/s"


def batch_chains():
    """The 64 chains: L in {8,12,16,24,32} (square), Nt in {16,32,64},
    beta ~ U[5,40], lambda scaled by U[0.5,1.5]; seeded.  Returns
    (L, Nt, beta, lambda-scale) tuples."""
    rng = np.random.default_rng(BATCH_SEED)
    out = []
    for _ in range(BATCH_N):
        out.append((int(rng.choice([8, 12, 16, 24, 32])), int(rng.choice([16, 32, 64])), float(rng.uniform(5, 40)),
                    float(rng.uniform(0.5, 1.5))))
    return out


def batch_flop(chains):
    return sum((L * L) ** 2 * nt * (84 * (1 + np.log2(nt)) + 170) + 2 * (L * L) ** 3 for L, nt, _, _ in chains)


def run_batch_bench(args):
    """chain evals/s of the 64-chain mix: W warm-up and K timed batches of one
    mixed-precision evaluation per chain through ephmc_batch_eval (fields
    resident in HBM), the same chains one at a time through ephmc_eval for
    comparison, and the batch through the C ABI with host buffers (e2e)."""
    import torch
    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    import ephmc
    lib = ephmc.load_library()
    chains = batch_chains()
    W, K = max(3, args.warmup), max(1, min(args.steps, 50))
    res = batch_measure(lib, dev, local, chains, W, K, dist, tune=True)
    ctxs, batch_s, seq_s, launches, sampler, tune_gain, e2e = (res[k] for k in (
        "ctxs", "batch_s", "seq_s", "launches", "sampler", "tune_gain", "e2e"))
    n = len(ctxs)
    value = ws * K * n / batch_s
    if rank == 0:
        fp64 = C_float_peak(lib, True)
        flop = batch_flop(chains)
        ach = flop * K / batch_s / 1e12
        cpu = None
        if ws == 1 and not args.no_cpu_baseline:
            try:
                cpu = batch_cpu_baseline(chains)
            except Exception as e:
                cpu = {"value": None, "unit": BATCH_UNIT, "cores": os.cpu_count(), "kind": "reference",
                       "sample": f"unavailable: {e}"}
        line = {"metric": BATCH_METRIC, "value": value, "unit": BATCH_UNIT, "n_gpus": ws, "steps": K, "warmup": W,
                "ms_per_step": batch_s / K * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64+f32", "data": "synthetic",
                "config": {"workload": f"{n} chains, L in {{8,12,16,24,32}}, Nt in {{16,32,64}}, beta ~ U[5,40], "
                                       f"lambda x U[0.5,1.5] (seed {BATCH_SEED}); one mixed evaluation per chain "
                                       "per step", "global_batch": n * ws, "parallelism": f"replicas x{ws}",
                           "l2": "fields of all chains resident; no flush (a step touches the 64 contexts' "
                                 "buffers, several GB)"},
                "one_chain_at_a_time": {"value": ws * K * n / seq_s, "ms_per_step": seq_s / K * 1e3},
                "autotune": {"chains_tuned": len(tune_gain),
                             "sum_ms_per_eval_before": sum(b for b, _ in tune_gain),
                             "sum_ms_per_eval_after": sum(a for _, a in tune_gain)},
                "roofline": {"bound": "fp64", "kernel": "whole batch (sweeps + LU of all chains)", "achieved": ach,
                             "peak": fp64, "unit": "TFLOP/s", "frac": ach / fp64 if fp64 else None,
                             "peak_source": "measured in this run (CUDA-core FP64 FMA probe)",
                             "algorithmic_flop_per_step": flop, "traffic": None},
                "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": sampler.summary()}
        print(json.dumps(line), flush=True)
    for c in ctxs:
        c.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def batch_measure(lib, dev, local, chains, W, K, dist, tune=True):
    """The 64-chain batch: contexts and N(0,1) fields on the device, optional
    per-chain autotuning, W warm-up and K timed batches (ephmc_batch_eval),
    the same chains one at a time, and the batch through the C ABI with host
    buffers.  Returns the timings and the contexts (the caller closes them)."""
    import torch

    import ephmc
    ws, rank, _ = dist_env()
    ctxs, xs, pds = [], [], []
    gen = torch.Generator(device=dev)
    gen.manual_seed(77 + rank)
    for L, nt, beta, s in chains:
        t, kappa, mu, omega = ephmc.convert_params(beta, nt, J, tuple(s * v for v in LAM), MU0, OMEGA0)
        c = ephmc.Context(L, L, nt, t, kappa, mu, omega, device=local)
        ctxs.append(c)
        xs.append(torch.randn(c.dim, dtype=torch.float64, device=dev, generator=gen))
        pds.append(torch.empty(c.dim, dtype=torch.float64, device=dev))

    def run_batch(x, p):
        try:
            ephmc.batch_eval(ctxs, x, p, mode="mixed")
        except ephmc.EphmcError as e:  # chains outside the Taylor regime may give a non-finite log det
            if e.status != 5:
                raise

    def run_seq():
        for c, x, p in zip(ctxs, xs, pds):
            try:
                c.eval(x, p, mode="mixed")
            except ephmc.EphmcError as e:
                if e.status != 5:
                    raise

    # launch shapes per chain, by measurement (ephmc_ctx_autotune), before any timing
    tune_gain = []
    for c, x in zip(ctxs, xs):
        if not tune:
            break
        try:
            b, a, _ = c.autotune(x, "mixed")
            tune_gain.append((b, a))
        except ephmc.EphmcError as e:
            if e.status != 5:
                raise
    for _ in range(W):
        run_batch(xs, pds)
    run_seq()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    launches0 = lib.ephmc_launch_count()
    with clock_sampler(local) as sampler:
        t0 = time.perf_counter()
        for _ in range(K):
            run_batch(xs, pds)
        torch.cuda.synchronize()
        batch_s = time.perf_counter() - t0
    launches = lib.ephmc_launch_count() - launches0
    t0 = time.perf_counter()
    for _ in range(K):
        run_seq()
    torch.cuda.synchronize()
    seq_s = time.perf_counter() - t0
    batch_s = max_over_ranks(batch_s, dist, dev)
    seq_s = max_over_ranks(seq_s, dist, dev)
    n = len(ctxs)
    # e2e: host fields and forces (pinned) through the C ABI
    xh = [torch.empty(c.dim, dtype=torch.float64, pin_memory=True) for c in ctxs]
    ph = [torch.empty(c.dim, dtype=torch.float64, pin_memory=True) for c in ctxs]
    for a, b in zip(xh, xs):
        a.copy_(b.cpu())
    xnp, pnp = [a.numpy() for a in xh], [a.numpy() for a in ph]
    run_batch(xnp, pnp)
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(K):
        run_batch(xnp, pnp)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, dev)
    nbytes = sum(8 * c.dim for c in ctxs)
    e2e = {"value": ws * K * n / e2e_s, "unit": BATCH_UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes}
    return {"ctxs": ctxs, "batch_s": batch_s, "seq_s": seq_s, "launches": launches, "sampler": sampler,
            "tune_gain": tune_gain, "e2e": e2e}


def batch_cpu_baseline(chains, budget=60.0):
    """The reference (oracle/_ref) on the host: one evaluation of each chain in
    turn until all are done or `budget` seconds have passed."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Model, Reference
    ref = Reference()
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    done, spent = 0, 0.0
    for i, (L, nt, beta, s) in enumerate(chains):
        m = Model.physical(L, L, nt, beta, J, tuple(s * v for v in LAM), MU0, OMEGA0)
        ctx = ref.context(m)
        ctx.eval(ref.random_x(1 + i, m.dim))
        spent += ctx.last_time()
        ctx.close()
        done += 1
        if spent > budget:
            break
    return {"value": done / spent, "unit": BATCH_UNIT, "cores": cores, "kind": "reference",
            "sample": f"one evaluation of each of the first {done} of the {len(chains)} chains, reference C "
                      f"sources + OpenBLAS, OMP/OpenBLAS threads={cores}"}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class NvmlClockSampler:
    """SM clocks and throttle reasons during the timed region, polled in-process
    through NVML every 20 ms (a one-sample nvidia-smi record of a sub-second
    region says little)."""

    def __init__(self, index):
        import pynvml
        self.nv = pynvml
        self.BITS = {"hw_slowdown": pynvml.nvmlClocksThrottleReasonHwSlowdown,
                     "sw_thermal_slowdown": pynvml.nvmlClocksThrottleReasonSwThermalSlowdown,
                     "hw_thermal_slowdown": pynvml.nvmlClocksThrottleReasonHwThermalSlowdown,
                     "sw_power_cap": pynvml.nvmlClocksThrottleReasonSwPowerCap}
        pynvml.nvmlInit()
        self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
        self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                self.samples.append((mhz, reasons))
            except Exception:
                pass
            self._stop.wait(0.02)

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
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["NVML returned no sample"], "samples": 0}
        reasons = sorted({n for _, r in self.samples for n, bit in self.BITS.items() if r & bit})
        return {"sm_mhz": statistics.median(m for m, _ in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples), "source": "NVML, every 20 ms"}


def clock_sampler(index):
    try:
        return NvmlClockSampler(index)
    except Exception:
        return ClockSampler(index)


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


def run_reference_trans_loc(args):
    """The reference's hist_trans_loc (oracle/_ref) on the host, one disorder
    sample of the TL workload per step; at most one untimed warm-up sample and
    a sample capped at about 5 minutes."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Reference
    ref = Reference()
    cores = os.cpu_count() or 1
    ref.set_threads(cores)
    t, kappa, mu, cm = tl_params()
    width = (-2 * mu + 8 * np.abs(kappa).sum()) / TL_BINS
    times = []
    budget = 300.0
    t0 = time.perf_counter()
    for k in range(max(1, args.steps)):
        a = time.perf_counter()
        ref.trans_loc_samples(100 + k, TL_L, TL_L, TL_BINS, t, kappa, mu, cm, width, 1)
        times.append(time.perf_counter() - a)
        if time.perf_counter() - t0 > budget:
            break
    per = sum(times) / len(times)
    val = 1.0 / per
    line = {"impl": "reference", "metric": TL_METRIC, "value": val, "unit": TL_UNIT, "n_gpus": ws,
            "steps": len(times), "warmup": 0, "ms_per_step": per * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": TL_WORKLOAD, "global_batch": 1, "parallelism": "host cores"},
            "cpu_baseline": {"value": val, "unit": TL_UNIT, "cores": cores, "kind": "reference",
                             "sample": f"{len(times)} disorder samples of the workload (LAPACKE dsyev on "
                                       f"{cores} OpenBLAS threads, pair loop single-threaded as written)"},
            "e2e": {"value": val, "unit": TL_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_trans_loc_bench(args):
    """Disorder samples/s of the GPU path: W warm-up and K timed batches of
    --tl-batch samples through ephmc_tl_run, bond fields resident in HBM; then
    the same through the C ABI with host buffers (e2e)."""
    import torch
    ws, rank, local = dist_env()
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    import ephmc
    lib = ephmc.load_library()
    t, kappa, mu, cm = tl_params()
    B = max(1, args.tl_batch)
    W = max(3, args.warmup)
    K = max(1, args.steps)
    if args.profile:  # under ncu: one warm-up and one timed sample, nothing printed
        B, W, K = 1, 1, 1
    Lt = args.tl_l
    V = Lt * Lt
    tl = ephmc.TransLoc(Lt, Lt, TL_BINS, t, kappa, mu, cm, lanes=args.tl_lanes, device=local)
    width = tl.default_width()
    stream = torch.cuda.current_stream(dev)
    tl.set_stream(stream.cuda_stream)
    gen = torch.Generator(device=dev)
    gen.manual_seed(4321 + rank)
    xs = torch.randn((K + W) * B, 3 * V, dtype=torch.float64, device=dev, generator=gen)
    hist = torch.zeros(TL_BINS, dtype=torch.float64, device=dev)
    z = torch.zeros(B, dtype=torch.float64, device=dev)
    for w in range(W):
        tl.run(xs[(K + w) * B:(K + w + 1) * B], width, hist, z)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = lib.ephmc_launch_count()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    stages = []
    with ClockSampler(local) as sampler:
        for k in range(K):
            ev[k][0].record(stream)
            tl.run(xs[k * B:(k + 1) * B], width, hist, z)
            ev[k][1].record(stream)
            stages.append(tl.last_timings())
        torch.cuda.synchronize()
    launches = lib.ephmc_launch_count() - launches0
    total_ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev), dist, dev)
    value = ws * K * B / (total_ms / 1e3)
    if args.profile:
        tl.close()
        return 0
    # e2e: host bond fields (pinned) in, host histogram and partition sums out
    xh = torch.empty(B, 3 * V, dtype=torch.float64, pin_memory=True)
    xh.copy_(xs[:B].cpu())
    hh = np.zeros(TL_BINS)
    zh = np.zeros(B)
    tl.set_stream(0)
    tl.run(xh.numpy(), width, hh, zh)
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for k in range(K):
        tl.run(xh.numpy(), width, hh, zh)
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist, dev)
    e2e = {"value": ws * K * B / e2e_s, "unit": TL_UNIT, "h2d_bytes_per_step": 8 * B * 3 * V,
           "d2h_bytes_per_step": 8 * (TL_BINS + B)}
    if rank == 0:
        a = torch.randn(4096, 4096, dtype=torch.float64, device=dev)
        for _ in range(2):
            torch.mm(a, a)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(5):
            torch.mm(a, a)
        e1.record()
        torch.cuda.synchronize()
        dgemm_tflops = 5 * 2 * 4096 ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12
        st = [statistics.median(s[i] for s in stages) for i in range(5)]
        flop = tl_flop_per_sample(V)
        ach = flop * ws * K * B / (total_ms / 1e3) / 1e12 / ws
        prod_flop = 2.0 * V ** 3
        # the two triangular products and the binning pass, from lane 0's stage events
        kernels = {
            "cusolverDnDsyevd (library)": {"ms": st[1]},
            "cublasDsyrkx x2 (library)": {"ms": st[3], "achieved_tflops": prod_flop / (st[3] * 1e-3) / 1e12,
                                          "peak_tflops": dgemm_tflops},
            "k_tl_current": {"ms": st[2], "bytes": 8 * 3 * V * V,
                             "achieved_gbs": 8 * 3 * V * V / (st[2] * 1e-3) / 1e9},
            "k_tl_boltzmann + k_tl_bin": {"ms": st[4], "bytes": 8 * V * (V + 1),
                                          "achieved_gbs": 8 * V * (V + 1) / (st[4] * 1e-3) / 1e9},
            "k_tl_hamilton + memset": {"ms": st[0]}}
        line = {"metric": TL_METRIC, "value": value, "unit": TL_UNIT, "n_gpus": ws, "steps": K, "warmup": W,
                "ms_per_step": total_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64", "data": "synthetic",
                "config": {"workload": TL_WORKLOAD if Lt == TL_L else f"static disorder: {Lt}x{Lt} lattice (V={V}), "
                                                                      f"512 bins, beta=40, mu0=0",
                           "global_batch": B * ws, "samples_per_step_per_gpu": B,
                           "lanes": args.tl_lanes, "parallelism": f"replicas x{ws}",
                           "l2": f"inputs larger than L2 (each sample's matrices: {7 * 8 * V * V / 1e6:.0f} MB)",
                           "inputs": "bond fields x ~ N(0,1) (torch.randn, seed 4321+rank)"},
                "roofline": {"bound": "fp64 tensor", "kernel": "whole sample (eigensolver-dominated)",
                             "achieved": ach, "peak": dgemm_tflops, "unit": "TFLOP/s",
                             "frac": ach / dgemm_tflops if dgemm_tflops else None,
                             "peak_source": "cuBLAS DGEMM 4096^3 measured in this run",
                             "algorithmic_flop_per_sample": flop, "traffic": None,
                             "stage_ms_lane0": dict(zip(["hamiltonian", "eigensolver", "current", "products",
                                                         "binning"], st)),
                             "kernels": kernels},
                "cpu_baseline": None, "e2e": e2e, "gpu_launches": launches, "clocks": sampler.summary()}
        print(json.dumps(line), flush=True)
    tl.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
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
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the 64-chain batch field of the headline line")
    ap.add_argument("--no-checkpointed", action="store_true",
                    help="skip the 48x48 checkpointed-evaluation field of the headline line")
    ap.add_argument("--paths", default="mixed,adjoint,reference")
    ap.add_argument("--profile", action="store_true",
                    help="run only warm-up + timed evaluations of --paths (for ncu); print nothing")
    ap.add_argument("--workload", default="hmc", choices=["hmc", "trans_loc", "batch", "stabilised", "checkpointed"])
    ap.add_argument("--stab-l", type=int, default=STAB_L, help="stabilised: lattice extent")
    ap.add_argument("--tl-batch", type=int, default=16, help="trans_loc: disorder samples per step")
    ap.add_argument("--tl-lanes", type=int, default=2, help="trans_loc: samples diagonalised concurrently")
    ap.add_argument("--tl-l", type=int, default=TL_L, help="trans_loc: lattice extent (profiling on smaller cases)")
    args = ap.parse_args()
    if args.workload == "stabilised":
        return 0 if args.impl == "reference" else run_stabilised_bench(args)
    if args.workload == "checkpointed":
        return 0 if args.impl == "reference" else run_checkpointed_bench(args)
    if args.workload == "trans_loc":
        return run_reference_trans_loc(args) if args.impl == "reference" else run_trans_loc_bench(args)
    if args.workload == "batch":
        if args.impl == "reference":
            ws, rank, _ = dist_env()
            if rank != 0:
                return 0
            cpu = batch_cpu_baseline(batch_chains(), budget=240.0)
            print(json.dumps({"impl": "reference", "metric": BATCH_METRIC, "value": cpu["value"], "unit": BATCH_UNIT,
                              "n_gpus": ws, "steps": 1, "warmup": 0, "ms_per_step": BATCH_N / cpu["value"] * 1e3,
                              "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                              "data": "synthetic", "config": {"workload": "the 64-chain mix", "parallelism": "host cores"},
                              "cpu_baseline": cpu, "e2e": {"value": cpu["value"], "unit": BATCH_UNIT,
                                                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
            return 0
        return run_batch_bench(args)
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
        sampler = clock_sampler(local) if path == "mixed" else None
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

    # One whole HMC trajectory (trajectory, simulation/organic_hmc.c:192-294,
    # without the measurement rows): momenta drawn N(0,1) on the device and
    # Fourier-accelerated (sample_fourier_momenta), their energy and the
    # action, Nmd = 20 leapfrog steps with Fourier acceleration over pi/2
    # (ephmc_leapfrog), the accept-step evaluation with its FP64 log det, the
    # new action and the Metropolis decision on the host; wall clock per
    # trajectory.  beta = 10: at beta = 20 the molecular dynamics diverges
    # within two steps, in the reference's own HMC as here (acceptance 0,
    # e^-dH NaN on 8x8, Nt = 64).
    tt, tk, tmu, tom = ephmc.convert_params(TRAJ_BETA, NT, J, LAM, MU0, OMEGA0)
    tctx = ephmc.Context(L, L, NT, tt, tk, tmu, tom, device=local)
    lib.ephmc_ctx_set_stream(tctx.h, stream.cuda_stream)
    urng = np.random.default_rng(4321 + rank)

    def hmc_trajectory(c, x, ld_x, mode):
        p0 = torch.randn(dim, dtype=torch.float64, device=dev, generator=gen)
        c.fa_scale_momenta(p0)
        h0 = c.hamilton(x, ld_x, c.fa_energy(p0))
        x1 = x.clone()
        c.leapfrog(x1, p0, 20, float(np.pi / 2), mode)
        ld1, _ = c.eval(x1, pd, mode=mode)
        dh = c.hamilton(x1, ld1, c.fa_energy(p0)) - h0
        accept = urng.random() < np.exp(-dh)
        return (x1, ld1, dh, accept) if accept else (x, ld_x, dh, accept)

    xt = torch.randn(dim, dtype=torch.float64, device=dev, generator=gen)
    tctx.fa_scale_free_bosons(xt)
    traj_ms, traj_fail, traj_acc = [], None, []
    try:
        ldt, _ = tctx.eval(xt, pd, mode=head)
        for k in range(12):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            xt, ldt, _, acc = hmc_trajectory(tctx, xt, ldt, head)
            torch.cuda.synchronize()
            if k >= 2:
                traj_ms.append(1e3 * (time.perf_counter() - t0))
                traj_acc.append(acc)
    except ephmc.EphmcError as e:
        traj_fail = str(e)
    tctx.close()
    traj = max_over_ranks(statistics.median(traj_ms), dist, dev) if traj_ms else None

    # The mixed force's Hamiltonian error: trajectories from the same field and
    # momenta with the FP64 adjoint force and with the mixed force, at beta = 10
    # and mu0 = 0 (with the band empty at mu0 = -3 the fermion force hardly
    # enters dH; at mu0 = 0 |dH| ~ 1e-2); the chain follows the FP64 run.
    dh_stats = None
    if head == "mixed":
        ht, hk, hmu, hom = ephmc.convert_params(TRAJ_BETA, NT, J, LAM, 0.0, OMEGA0)
        hctx = ephmc.Context(L, L, NT, ht, hk, hmu, hom, device=local)
        lib.ephmc_ctx_set_stream(hctx.h, stream.cuda_stream)
        xh0 = torch.randn(dim, dtype=torch.float64, device=dev, generator=gen)
        hctx.fa_scale_free_bosons(xh0)
        try:
            ld_h, _ = hctx.eval(xh0, pd, mode="adjoint")
            d64, dmx, a64, amx = [], [], [], []
            for _ in range(DH_TRAJ):
                p0 = torch.randn(dim, dtype=torch.float64, device=dev, generator=gen)
                hctx.fa_scale_momenta(p0)
                h0 = hctx.hamilton(xh0, ld_h, hctx.fa_energy(p0))
                u = urng.random()
                ends = {}
                for mode, dl, al in (("adjoint", d64, a64), ("mixed", dmx, amx)):
                    x1, p1 = xh0.clone(), p0.clone()
                    hctx.leapfrog(x1, p1, 20, float(np.pi / 2), mode)
                    ld1, _ = hctx.eval(x1, pd, mode="adjoint")
                    dl.append(hctx.hamilton(x1, ld1, hctx.fa_energy(p1)) - h0)
                    al.append(bool(u < np.exp(-dl[-1])))
                    ends[mode] = (x1, ld1)
                if a64[-1]:
                    xh0, ld_h = ends["adjoint"]
            diff = np.array(dmx) - np.array(d64)
            dh_stats = {"trajectories": DH_TRAJ, "beta": TRAJ_BETA, "mu0": 0.0,
                        "mean_abs_dH_fp64": float(np.mean(np.abs(d64))), "mean_dH_fp64": float(np.mean(d64)),
                        "mean_dH_mixed": float(np.mean(dmx)), "bias": float(np.mean(diff)),
                        "median_difference": float(np.median(diff)), "max_abs_difference": float(np.max(np.abs(diff))),
                        "acceptance_fp64": float(np.mean(a64)), "acceptance_mixed": float(np.mean(amx)),
                        "same_decisions": int(np.sum(np.array(a64) == np.array(amx)))}
        except ephmc.EphmcError as e:
            dh_stats = {"failed": str(e)}
        hctx.close()

    # the 64-chain batch (ephmc_batch_eval), untuned, a few steps
    batch = None
    if not args.no_batch:
        bres = batch_measure(lib, dev, local, batch_chains(), 2, 5, dist, tune=False)
        nb = len(bres["ctxs"])
        batch = {"metric": BATCH_METRIC, "value": ws * 5 * nb / bres["batch_s"], "unit": BATCH_UNIT,
                 "ms_per_step": bres["batch_s"] / 5 * 1e3,
                 "one_chain_at_a_time": ws * 5 * nb / bres["seq_s"], "e2e": bres["e2e"],
                 "gpu_launches": bres["launches"], "steps": 5, "warmup": 2,
                 "workload": f"{nb} chains, L in {{8,12,16,24,32}}, Nt in {{16,32,64}}, beta ~ U[5,40], lambda x "
                             f"U[0.5,1.5] (seed {BATCH_SEED}), one mixed evaluation per chain per step, not autotuned"}
        for c in bres["ctxs"]:
            c.close()
    ckpt = None
    if not args.no_checkpointed:
        cm = checkpointed_measure(local, rank, STAB_L, 2, 5)
        ckpt = {"metric": CKPT_METRIC, "value": 1.0 / cm["s_per_eval"], "unit": UNIT,
                "ms_per_step": 1e3 * cm["s_per_eval"], "phases_ms": cm["phases_ms"],
                "context_bytes": cm["context_bytes"], "steps": 5, "warmup": 2,
                "workload": f"{STAB_L}x{STAB_L} lattice, Nt={STAB_NT}, beta={STAB_BETA}, checkpoints every "
                            f"{STAB_CKPT} slices, mixed force; N(0,1) fields; wall clock around the 5 evaluations"}

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
        if head == "mixed":
            phases = (("k_gj_dataflow (LU, inverse, log det)", LU_FLOP, ph["lu_ms"], fp64, "fp64"),
                      ("force phase: FP64 y chain (k_slices_strip), segment DGEMMs, k_adjoint_strip FP32 sweep",
                       MIXED_FORCE_FLOP, ph["force_ms"], fp32, "fp32 sweep + fp64 chain/GEMMs"),
                      ("M_hat phase: k_slices_strip FP64 sweep 1 + segment stacks from the identity",
                       MIXED_MHAT_FLOP, ph["mhat_ms"], fp64, "fp64"))
        else:
            phases = (("k_gj_dataflow (LU, inverse, log det)", LU_FLOP, ph["lu_ms"], fp64, "fp64"),
                      ("k_adjoint (force sweep)", ADJ_SWEEP_FLOP, ph["force_ms"], sweep_peak, "fp64"),
                      ("k_slices_strip (M_hat + q stack)", SWEEP1_FLOP, ph["mhat_ms"], fp64, "fp64"))
        for name, flop, ms, pk, bound in phases:
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
                "trajectory": {"ms": traj, "trajectories_per_s": (ws * 1e3 / traj) if traj else None,
                               "beta": TRAJ_BETA, "failed": traj_fail,
                               "acceptance": float(np.mean(traj_acc)) if traj_acc else None,
                               "what": "wall clock of one whole HMC trajectory at 32x32, Nt=64, beta=10: momentum "
                                       "draw and Fourier acceleration, action, 20 leapfrog steps with Fourier "
                                       "acceleration over pi/2 (ephmc_leapfrog), the accept-step evaluation, new "
                                       "action, Metropolis decision (median of 10 after 2). At beta=20 the MD "
                                       "diverges, in the reference too"},
                "mixed_dH": dh_stats, "batch": batch, "checkpointed": ckpt,
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
