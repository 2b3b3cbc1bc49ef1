"""Throughput of the MLFMA forward solve path: forward solves/s at true relative
residual 1e-5 on the 1024x1024-pixel workload (102.4 wavelengths, 8 tree
levels, 20 random lossy ellipses, 256 plane-wave transmitters), complex64 with
FP64 reductions.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step solves all 256 transmitters as one batched, masked BiCGSTAB launch
sequence on the tensor engine.  Beside it, on bounded samples: the plain
single-RHS solver (one transmitter per launch sequence, complex FP32 SIMT: the
metric's denominator) and the same single-RHS solver on the tensor engine; the
learned warm start, trained inside the run on solver-generated fields; the
reference's own CPU path (oracle/_ref, all host threads); and the field error
of a sampled transmitter against the reference's FP64 solver converged to
1e-10.  With N > 1 (torchrun) every rank solves its own 256 transmitters; there
is no collective on the data path.  One JSON line is printed by rank 0.

--impl reference times the reference's own CPU implementation on the same
workload; its inputs come from the oracle's restatement of the seeded
generators (bit-identical) and the reference's own tree ordering, so that arm
loads no library of this package.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "inverse-solver-gpu_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

LEVEL = 8             # 1024 x 1024 pixels (reference `level`, mom.cpp:6,137)
NTX = 256
NELL = 20
EPS = (1.1, 2.0)
TAND = 0.1
TOL = 1e-5
SEED = 2000
METRIC = "forward solves/s at rel. residual 1e-5: batched+learned vs plain FP32, 1 B200"


def workload_config(world: int) -> dict:
    """The workload, identical for both arms (how each arm runs it is reported beside)."""
    return {"workload": "1024x1024 px (102.4 lambda, lambda/10), 8 levels (7 MLFMA levels), 8x8 leaves; "
                        "20 random ellipses eps_r U[1.1,2.0](1+i tan d), tan d U[0,0.1]; 256 plane-wave Tx; "
                        "BiCGSTAB to true rel. residual 1e-5",
            "grid": 1024, "levels": LEVEL, "transmitters": NTX, "tol": TOL, "seed": SEED,
            "parallelism": f"tx-sharded x{world}" if world > 1 else "single GPU",
            "l2_policy": "inputs larger than L2 (26 GB working set per step)"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self) -> dict:
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows]
        reasons = set()
        for r in rows:
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": sorted(reasons),
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


def make_inputs(s, rank: int):
    chi = s.phantom(seed=SEED + rank, count=NELL, axis=(1.0, 3.0), eps=EPS, tand_max=TAND)
    g = (s.opts.k0 ** 2) * s.raster_to_tree(chi)          # tree order, as mom.cpp:288-289
    b = s.plane_waves(NTX, order=0)                        # tree order (setup_born.cpp:62-65)
    return g, b


def reference_inputs(ref, rank: int, txs):
    """The same inputs for the reference arm, without this package's library:
    the oracle's bit-identical restatement of the seeded generators, mapped to
    tree order with the reference's own unkmap (setup_mlfma.cpp:177-185)."""
    from _oracle import seeded_ellipses, seeded_plane_waves
    side = 8 * 2 ** (LEVEL - 1)
    um = ref.table("unkmap", 0, side * side, "i")
    chi = seeded_ellipses(side, SEED + rank, NELL, (1.0, 3.0), EPS, TAND)
    tree = np.empty_like(chi)
    tree[um] = chi
    g = (2 * math.pi) ** 2 * tree
    b = {tx: seeded_plane_waves(side, NTX, tx, 1, um)[0] for tx in txs}
    return g, b


def peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"], "src": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "src": "fallback"}


def algorithmic_bytes_per_matvec(s) -> float:
    """8 (3U + 4S), S = sum over levels >= 2 of clusters x samples."""
    S = sum((4 ** i) * s.numsamp(i) for i in range(2, s.level))
    return 8.0 * (3 * s.numunk + 4 * S)


def near_field_flops_per_rhs(s) -> tuple[float, float]:
    """(tensor FLOPs executed, useful complex FLOPs) of the near-field + L2P
    kernel for one RHS.  Executed: per 16 x 8-leaf tile, 9 neighbour slots x 4
    K-chunks x 2 K-steps x 3 split products (hi hi, hi lo, lo hi) of
    128 x 128 x 16 MMAs, plus the L2P chunks (2 ns reals padded to 32) the same
    way.  Useful: (9 x 64 + ns) complex MACs x 8 flops per pixel."""
    tiles = -(-s.side // 8 // 16) * -(-s.side // 8 // 8)
    ns = s.numsamp(s.level - 1)
    mma = 2 * 128 * 128 * 16
    stages = 36 + -(-2 * ns // 32)
    executed = tiles * stages * 6 * mma
    useful = s.numunk * (9 * 64 + ns) * 8
    return float(executed), float(useful)


# DRAM bytes (read + write) of one near-field launch over 16 RHS of the 1024^2
# workload: a constant captured once with ncu (dram__bytes_read.sum +
# dram__bytes_write.sum, one launch, --set full), not measured by this run;
# the traffic grows with the RHS processed, so a launch over R RHS is R / 16
# of it scaled.
NEAR_TRAFFIC_16RHS_CAPTURED = 326.4e6 + 102.9e6


def cpu_reference_sample(ref, g, b, budget_s: float, max_solves: int):
    """The reference's own CPU path (oracle/_ref) on the host cores; also
    returns the first solve's field (Tx 0), the FP64 run at the same tolerance."""
    threads = ref.L.ref_omp_threads()
    solved, t_total, x0 = 0, 0.0, None
    while solved < max_solves and t_total < budget_s:
        t0 = time.perf_counter()
        x, _ = ref.bicgs(g, b[solved % len(b)], False, TOL, 300)
        t_total += time.perf_counter() - t0
        x0 = x if x0 is None else x0
        solved += 1
    return {"value": solved / t_total, "unit": "solves/s", "cores": threads, "kind": "reference",
            "sample": f"{solved} forward solves (Tx 0..{solved - 1}) of the same 1024^2 workload, FP64, "
                      f"{threads} OpenMP threads, {t_total:.1f} s"}, x0


def field_parity(ref, g, b_tx, x_ours, x_fp64_same_tol, tx: int):
    """Relative L2 error of our field against the reference's FP64 solver
    converged to 1e-10 (and of the reference's own 1e-5 run against it);
    returns the record and that FP64 field."""
    from _oracle import rel
    t0 = time.perf_counter()
    x10, it10 = ref.bicgs(g, b_tx, False, 1e-10, 2000)
    out = {"tx": tx, "field_err_vs_fp64": rel(x_ours, x10),
           "fp64_reference": "reference CPU solver (bicgs.cpp + solve.cpp, FP64) converged to 1e-10",
           "fp64_iterations": it10, "fp64_seconds": time.perf_counter() - t0, "bar": 1e-4}
    if x_fp64_same_tol is not None:
        out["fp64_at_tol_field_err_vs_fp64"] = rel(x_fp64_same_tol, x10)
        out["field_err_vs_fp64_at_tol"] = rel(x_ours, x_fp64_same_tol)
    return out, x10


def max_over_ranks(v: float, dist, device) -> float:
    """The largest of every rank's v (the job's time is its slowest rank's)."""
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference_gpu(args):
    """--impl reference-gpu (a helper process of the one-GPU run): forward
    solves of the workload through the reference's own GPU path (FP64,
    oracle/_ref/libisgref_gpu.so), timed by the host clock around each
    synchronous call; Tx 0's field goes to --ref-gpu-out."""
    from _oracle import ReferenceGpu
    if args.ref_gpu_in:  # another workload's inputs: level, numrx, g and b in tree order
        d = np.load(args.ref_gpu_in)
        ref = ReferenceGpu(int(d["level"]), 2 * math.pi, int(d["numrx"]))
        g = d["g"]
        b = dict(enumerate(d["b"]))
        txs = [k % len(b) for k in range(args.warmup + args.steps)]
    else:
        ref = ReferenceGpu(LEVEL, 2 * math.pi, 32)
        txs = list(range(args.warmup + args.steps))
        g, b = reference_inputs(ref, 0, txs)
    times, its = [], []
    for k, tx in enumerate(txs):
        t0 = time.perf_counter()
        x, it = ref.bicgs(g, b[tx], False, TOL, 300)
        dt = time.perf_counter() - t0
        if tx == 0 and args.ref_gpu_out:
            np.save(args.ref_gpu_out, x)
        if k >= args.warmup:
            times.append(dt)
            its.append(it)
    print(json.dumps({"value": len(times) / sum(times), "unit": "solves/s", "solves": len(times),
                      "mean_iterations": float(np.mean(its)), "seconds_per_solve": sum(times) / len(times)}))


def reference_gpu_sample(x10, inputs: dict | None = None, steps: int = 2, warmup: int = 1) -> dict:
    """The reference's own GPU path on this GPU, in a child process (its error
    handler exits on a CUDA error); x10: the FP64 solution of Tx 0 for the
    error of the reference's field.  inputs: another workload's level, numrx,
    g and b (tree order) instead of the headline workload's."""
    from _oracle import ReferenceGpu, rel
    if not ReferenceGpu.available():
        return {"unavailable": "oracle/_ref/libisgref_gpu.so was not built"}
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "x0.npy")
        cmd = [sys.executable, os.path.abspath(__file__), "--impl", "reference-gpu", "--steps", str(steps),
               "--warmup", str(warmup), "--ref-gpu-out", out]
        if inputs is not None:
            np.savez(os.path.join(d, "in.npz"), **inputs)
            cmd += ["--ref-gpu-in", os.path.join(d, "in.npz")]
        try:
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
        except subprocess.TimeoutExpired:
            return {"unavailable": f"the reference's GPU path did not finish {steps + warmup} solves in 900 s"}
        lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
        if r.returncode != 0 or not lines:
            return {"unavailable": f"the reference's GPU path exited with {r.returncode}: {r.stderr[-300:]}"}
        res = json.loads(lines[-1])
        res["kind"] = ("the reference's own GPU path (gpu.cu, kernels.cu, matvec_gpu.cu, bicgs_gpu.cu; FP64, "
                       "one transmitter per solve), compiled for sm_100a")
        if x10 is not None and os.path.exists(out):
            res["tx0_field_err_vs_fp64"] = rel(np.load(out), x10)
        return res


def run_reference_arm(args, rank: int, world: int):
    """--impl reference: the reference's own CPU implementation, rank 0 only."""
    if rank != 0:
        return
    from _oracle import Reference
    if not Reference.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libisgref.so was not built"}))
        return
    ref = Reference(LEVEL, 2 * math.pi, 32)
    threads = ref.L.ref_omp_threads()
    txs = [k % NTX for k in range(args.warmup + args.steps)]
    g, b = reference_inputs(ref, 0, sorted(set(txs)))
    times = []
    for k, tx in enumerate(txs):
        t0 = time.perf_counter()
        ref.bicgs(g, b[tx], False, TOL, 300)
        dt = time.perf_counter() - t0
        if k >= args.warmup:
            times.append(dt)
    ms = 1000 * sum(times) / len(times)
    v = 1000.0 / ms
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": workload_config(world),
        "solver": {"impl": "reference CPU path (solve.cpp MLFMA + bicgs.cpp BiCGSTAB, FP64, OpenMP)",
                   "batch": 1, "step": "one forward solve (Tx k mod 256)"},
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": threads, "kind": "reference",
                         "sample": f"one forward solve per step (Tx k), {threads} threads"},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def single_rhs_rate(s, g, b, opts, stream, n: int) -> dict:
    """One transmitter per launch sequence (the first solve is a warm-up)."""
    import torch
    ms, its = [], []
    for j in range(n + 1):
        xj = torch.zeros_like(b[j])
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        inf = s.bicgs(xj, g, b[j], opts=opts, stream=stream)[0]
        a1.record(stream)
        torch.cuda.synchronize()
        if j:
            ms.append(a0.elapsed_time(a1))
            its.append(inf["iterations"])
    return {"value": 1000.0 / (sum(ms) / len(ms)), "unit": "solves/s", "solves": len(ms),
            "mean_iterations": float(np.mean(its)), "ms_per_solve": float(np.mean(ms))}


def learned_arm(s, isg, g, b, stream, pairs: int, steps: int, zero_iterations: float) -> dict:
    """Trains the neural-operator warm start on solver-generated fields of the
    workload's contrast distribution (other seeds, random transmitters), then
    times one 256-RHS solve started from it."""
    import torch
    t0 = time.perf_counter()
    rng = np.random.default_rng(SEED + 17)
    G, B = [], []
    for j in range(pairs):
        chi = s.phantom(seed=SEED + 100 + j, count=NELL, axis=(1.0, 3.0), eps=EPS, tand_max=TAND)
        G.append((s.opts.k0 ** 2) * s.raster_to_tree(chi))
        B.append(s.plane_waves(NTX, first=int(rng.integers(NTX)), count=1)[0])
    dev = b.device
    gt = torch.from_numpy(np.array(G).astype(np.complex64)).to(dev)
    bt = torch.from_numpy(np.array(B).astype(np.complex64)).to(dev)
    ut = torch.zeros_like(bt)
    opts = isg.default_solve_opts(tol=TOL, maxit=300, engine=isg.ENGINE_TENSOR, check_every=2)
    s.bicgs(ut, gt, bt, opts=opts, stream=stream)
    t_data = time.perf_counter() - t0
    s.fno_create(width=32, modes=12, layers=4, batch=4, seed=1)
    losses = []
    for k in range(steps):
        sel = torch.from_numpy(rng.choice(pairs, 4, replace=False)).to(dev)
        losses.append(s.fno_train_step(gt[sel], bt[sel], ut[sel], lr=3e-3 if k < 2 * steps // 3 else 1e-3,
                                       stream=stream))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0 - t_data
    lo = isg.default_solve_opts(tol=TOL, maxit=300, engine=isg.ENGINE_TENSOR, check_every=2,
                                guess=isg.GUESS_LEARNED)
    x = torch.zeros_like(b)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    infos = s.bicgs(x, g, b, opts=lo, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    its = float(np.mean([i["iterations"] for i in infos]))
    ok = all(i["status"] == 0 and 0 <= i["true_residual"] <= TOL for i in infos)
    return {"value": NTX * 1000.0 / ms, "unit": "solves/s", "mean_iterations": its,
            "zero_start_mean_iterations": zero_iterations, "all_converged": ok,
            "network": "FNO width 32, 4 spectral layers, 12x24 modes, BF16 tcgen05 products, FP32 accumulate",
            "training": {"pairs": pairs, "steps": steps, "batch": 4, "data_s": round(t_data, 2),
                         "train_s": round(t_train, 2), "loss_first": losses[0], "loss_last": losses[-1]},
            "pays": its < zero_iterations}


def status_counts(infos) -> dict:
    names = {0: "ok", 1: "not_converged", 2: "breakdown", 3: "nonfinite", 6: "timeout"}
    c = {}
    for i in infos:
        k = names.get(i["status"], str(i["status"]))
        c[k] = c.get(k, 0) + 1
    return c


def run_config1(isg, torch, dev, reps: int = 5) -> dict:
    """The reference's own small case: 128 x 128 pixels (12.8 lambda, 4 MLFMA
    levels, 8 x 8 leaves), three ellipses with eps_r U[1.1, 1.5] (seed 1000),
    32 line-source transmitters and 32 near-field receivers on a 20-lambda
    circle, every transmitter solved to true residual 1e-5.  GPU: the 32 solves
    as one batch on the tensor engine, device-resident, `reps` timed repeats
    after a warm-up (median).  CPU: the reference's compiled FP64 solver
    (oracle/_ref: bicgs.cpp over solve.cpp) on all 32 transmitters with every
    host thread, from the same complex64-rounded inputs.  Parity: every GPU
    field against the reference's FP64 solve converged to 1e-10, and every
    iteration count against the reference's at 1e-5."""
    from _oracle import Reference, rel
    level, ntx, nrx, radius = 5, 32, 32, 20.0
    s = isg.Solver(level, numrx=nrx, max_rhs=ntx, device=dev.index or 0)
    s.setup_gpu()
    s.set_nearfield_receivers(radius)
    chi = s.raster_to_tree(s.phantom(seed=1000, count=3, axis=(1.0, 3.0), eps=(1.1, 1.5)))
    g_np = ((s.opts.k0 ** 2) * chi).astype(np.complex64)
    b_np = s.line_sources(ntx, radius).astype(np.complex64)
    g, b = torch.from_numpy(g_np).to(dev), torch.from_numpy(b_np).to(dev)
    stream = torch.cuda.Stream(dev)
    opts = isg.default_solve_opts(tol=TOL, maxit=1000, engine=isg.ENGINE_TENSOR, check_every=2)
    x = torch.zeros_like(b)
    s.bicgs(x, g, b, opts=opts, stream=stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    times = []
    for _ in range(reps):
        e0.record(stream)
        infos = s.bicgs(x, g, b, opts=opts, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = statistics.median(times)
    rx = s.receive(g * x).cpu().numpy()
    X = x.cpu().numpy().astype(np.complex128)
    out = {"workload": "128x128 px (12.8 lambda), 4 MLFMA levels, 3 ellipses eps_r U[1.1,1.5], 32 line-source Tx "
                       "and 32 near-field Rx on r=20 lambda, BiCGSTAB to true rel. residual 1e-5",
           "gpu": {"value": ntx * 1000.0 / ms, "unit": "solves/s", "ms_per_batch": ms, "batch": ntx,
                   "engine": "tensor", "mean_iterations": float(np.mean([i["iterations"] for i in infos])),
                   "all_converged": all(i["status"] == 0 and 0 <= i["true_residual"] <= TOL for i in infos)}}
    if not Reference.available():
        out["cpu_baseline"] = {"unavailable": "oracle/_ref (the compiled reference) is not built"}
        return out
    ref = Reference(level, 2 * math.pi, nrx)
    threads = ref.L.ref_omp_threads()
    g64, b64 = g_np.astype(np.complex128), b_np.astype(np.complex128)
    t0 = time.perf_counter()
    ref_its = [ref.bicgs(g64, b64[j], False, TOL, 1000)[1] for j in range(ntx)]
    t_cpu = time.perf_counter() - t0
    out["cpu_baseline"] = {"value": ntx / t_cpu, "unit": "solves/s", "cores": threads, "kind": "reference",
                           "sample": f"all {ntx} forward solves, FP64, {threads} OpenMP threads, {t_cpu:.2f} s"}
    x10s = [ref.bicgs(g64, b64[j], False, 1e-10, 2000)[0] for j in range(ntx)]
    errs = [rel(X[j], x10s[j]) for j in range(ntx)]
    dits = [infos[j]["iterations"] - ref_its[j] for j in range(ntx)]
    out["parity"] = {"max_field_err_vs_fp64": max(errs), "mean_field_err_vs_fp64": float(np.mean(errs)),
                     "bar": 1e-4, "iterations_minus_reference": sorted(set(dits)),
                     "fp64_reference": "reference CPU solver (bicgs.cpp + solve.cpp, FP64) converged to 1e-10",
                     "receivers": f"{nrx} near-field samples per Tx computed (isg_receive)",
                     "rx_norm": float(np.linalg.norm(rx))}
    out["speedup_gpu_vs_cpu"] = out["gpu"]["value"] / out["cpu_baseline"]["value"]
    out["reference_gpu"] = reference_gpu_sample(x10s[0], {"level": level, "numrx": nrx, "g": g64, "b": b64},
                                                steps=ntx, warmup=2)
    if "value" in out["reference_gpu"]:
        out["speedup_gpu_vs_reference_gpu"] = out["gpu"]["value"] / out["reference_gpu"]["value"]
    return out


def run_config3(isg, torch, dev, seed: int = 3000) -> dict:
    """64 independent forward problems, grid sides drawn from {128, 256, 512,
    1024}, 16-128 plane-wave transmitters each, random ellipses eps_r in
    [1.1, 1.8], solved together by isg.multi.MultiSolver (one multi-RHS block
    per grid size, per-RHS contrasts and masks, the sizes' iteration blocks as
    branches of one CUDA graph per poll, isg_bicgs_group) to true residual
    1e-5."""
    from isg.multi import MultiSolver, level_of
    rng = np.random.default_rng(seed)
    ms = MultiSolver(max_rhs=256, device=dev.index or 0, engine=isg.ENGINE_TENSOR)
    ellipses = {5: 3, 6: 5, 7: 10, 8: 20}
    problems = []
    for p in range(64):
        lvl = int(rng.choice([5, 6, 7, 8]))
        s = ms.solver(lvl)
        chi = s.raster_to_tree(s.phantom(seed=seed + p, count=ellipses[lvl], axis=(1.0, 3.0), eps=(1.1, 1.8)))
        ntx = int(rng.integers(16, 129))
        b = s.plane_waves(ntx, order=isg.ORDER_TREE)
        problems.append((torch.from_numpy(((2 * np.pi) ** 2 * chi).astype(np.complex64)).to(dev),
                         torch.from_numpy(b.astype(np.complex64)).to(dev)))
    ms.solve(problems[:4], tol=TOL, maxit=1000)  # warm-up: graphs, kernels, launch attributes
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = ms.solve(problems, tol=TOL, maxit=1000)
    e1.record()
    torch.cuda.synchronize()
    ms_total = e0.elapsed_time(e1)
    infos = [i for _, inf in out for i in inf]
    by = {}
    for (g, b), (_, inf) in zip(problems, out):
        n = int(round(g.shape[-1] ** 0.5))
        d = by.setdefault(n, {"problems": 0, "solves": 0, "iterations": []})
        d["problems"] += 1
        d["solves"] += b.shape[0]
        d["iterations"] += [i["iterations"] for i in inf]
    for d in by.values():
        d["mean_iterations"] = float(np.mean(d.pop("iterations")))
    return {"workload": "64 problems, sides U{128,256,512,1024}, 16-128 plane-wave Tx, ellipses eps_r U[1.1,1.8]",
            "solves": len(infos), "seconds": ms_total / 1e3, "value": len(infos) * 1000.0 / ms_total,
            "unit": "solves/s", "all_converged": all(i["status"] == 0 and 0 <= i["true_residual"] <= TOL
                                                    for i in infos),
            "status_counts": status_counts(infos), "max_true_residual": max(i["true_residual"] for i in infos),
            "by_side": {str(k): v for k, v in sorted(by.items())}}


def run_config4(isg, torch, dev, fp64_fields: int = 2, nrhs: int = 64) -> dict:
    """4096 x 4096 pixels (409.6 wavelengths, 9 MLFMA levels), Gaussian
    random field contrast (correlation length 2 wavelengths).  Timed: one batch
    of `nrhs` plane-wave illuminations (128 illuminations are two such
    batches) at eps_r in [1.0, 1.1], tensor engine, true residual 1e-5.
    Probed: the configured eps_r in [1.0, 1.6] on 8 illuminations for 400
    iterations (the residual it reaches).  FP64: for `fp64_fields` fields, the
    FP64 solution of the same system obtained by iterative refinement whose
    residuals b - (x - G(g x)) come from the reference's own FP64 MLFMA
    operator (oracle/_ref, solve.cpp:25-248), refined until that FP64 residual
    is below 1e-10; the error of the 1e-5 field against it is reported."""
    from _oracle import Reference, rel
    level = 10
    s = isg.Solver(level, numrx=32, max_rhs=nrhs, device=dev.index or 0)
    s.setup_gpu()
    out = {"workload": "4096x4096 px (409.6 lambda), 9 MLFMA levels, GRF corr 2 lambda", "nrhs": nrhs}
    chi = s.phantom(seed=4010, kind=1, eps=(1.0, 1.1), corr_len=2.0)
    g_np = (s.opts.k0 ** 2) * s.raster_to_tree(chi)
    b_np = s.plane_waves(128, first=0, count=nrhs)
    g = torch.from_numpy(g_np.astype(np.complex64)).to(dev)
    b = torch.from_numpy(b_np.astype(np.complex64)).to(dev)
    opts = isg.default_solve_opts(tol=TOL, maxit=3000, engine=isg.ENGINE_TENSOR, check_every=4)
    stream = torch.cuda.Stream(dev)
    x = torch.zeros_like(b)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    infos = s.bicgs(x, g, b, opts=opts, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    out["eps_1.0_1.1"] = {"value": nrhs * 1000.0 / ms, "unit": "solves/s", "seconds": ms / 1e3,
                          "mean_iterations": float(np.mean([i["iterations"] for i in infos])),
                          "all_converged": all(i["status"] == 0 and 0 <= i["true_residual"] <= TOL for i in infos),
                          "status_counts": status_counts(infos),
                          "max_true_residual": max(i["true_residual"] for i in infos)}
    # the configured contrast, bounded
    chi6 = s.phantom(seed=4010, kind=1, eps=(1.0, 1.6), corr_len=2.0)
    g6 = torch.from_numpy(((s.opts.k0 ** 2) * s.raster_to_tree(chi6)).astype(np.complex64)).to(dev)
    x6 = torch.zeros_like(b[:8])
    i6 = s.bicgs(x6, g6, b[:8], opts=isg.default_solve_opts(tol=TOL, maxit=400, engine=isg.ENGINE_TENSOR,
                                                             check_every=4), stream=stream)
    out["eps_1.0_1.6_probe"] = {"iterations": 400, "residuals": [i["residual"] for i in i6]}
    # FP64 solutions by refinement with the reference's FP64 operator
    if fp64_fields and Reference.available():
        ref = Reference(level, 2 * math.pi, 32)
        x_h = x[:fp64_fields].cpu().numpy().astype(np.complex128)
        errs = []
        o1 = isg.default_solve_opts(tol=1e-6, maxit=3000, engine=isg.ENGINE_TENSOR, check_every=4)
        for j in range(fp64_fields):
            bj = b_np[j]
            xr = x_h[j].copy()
            hist = []
            for _ in range(6):
                r = bj - (xr - ref.mlfma(g_np * xr))
                hist.append(float(np.linalg.norm(r) / np.linalg.norm(bj)))
                if hist[-1] < 1e-10:
                    break
                rd = torch.from_numpy(r.astype(np.complex64)).to(dev)
                dd = torch.zeros_like(rd)
                s.bicgs(dd, g, rd, opts=o1, stream=stream)
                xr = xr + dd.cpu().numpy().astype(np.complex128)
            # the same field solved to 1e-6: what is left at 1e-5 is the stopping tolerance, not the arithmetic
            xt = torch.zeros_like(b[j])
            s.bicgs(xt, g, b[j], opts=isg.default_solve_opts(tol=1e-6, maxit=5000, engine=isg.ENGINE_TENSOR,
                                                            check_every=4), stream=stream)
            errs.append({"tx": j, "field_err_vs_fp64": rel(x_h[j], xr), "fp64_residual_history": hist,
                         "tol_1e-6_field_err_vs_fp64": rel(xt.cpu().numpy().astype(np.complex128), xr)})
        out["parity"] = errs
    return out


def run_config5(isg, torch, dev, triples: int = 4096, epochs: float = 2.0, iters: int = 10,
                regs=(0.0, 1e-3, 3e-3, 1e-2, 3e-2), fno_batch: int = 8, train_budget_s: float = 240.0) -> dict:
    """Full inversion with the learned warm start: 512 x 512 pixels (51.2
    lambda, 7 MLFMA levels), 128 line-source transmitters and 256 near-field
    receivers on a 40-wavelength circle, an 8-ellipse contrast (semi-axes 1-3
    lambda) with eps_r in [1.1, 1.5], measurements with 1 % complex Gaussian
    noise, `iters` Polak-Ribiere iterations with Tikhonov regularisation,
    every forward and adjoint solve to true residual 1e-5 on the tensor engine.
    The Tikhonov weight (the reference's `regular`, 0 in mom.cpp:32) is the
    largest of `regs` whose zero-start inversion ends at a misfit within 1.5x
    of the unregularised one; the whole sweep is reported.  Each inversion is
    run twice and the second run is timed.

    The network (width 32, 4 spectral layers, 12 x 24 modes, BF16 tcgen05
    products with FP32 accumulation) is trained first on `triples`
    solver-generated (contrast, incident field, total field) triples: contrasts
    of the same distribution (other seeds), 16 random transmitters each, for
    `epochs` passes or `train_budget_s` seconds, whichever ends first.  The
    same inversion then runs with every solve from zero (the reference's
    method), from the previous iteration's fields, from the network (forward
    and adjoint solves), and from both (network on the first iteration, then
    the previous fields); each is timed on the device.  The plain single-RHS
    FP32 solver (one transmitter at a time, SIMT engine, zero start) runs the
    same inversion for the comparison the metric names."""
    level, ntx, nrx, radius = 7, 128, 256, 40.0
    s = isg.Solver(level, numrx=nrx, max_rhs=ntx, device=dev.index or 0)
    s.setup_gpu()
    s.set_nearfield_receivers(radius)
    k2 = s.opts.k0 ** 2
    U = s.numunk
    stream = torch.cuda.Stream(dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn):
        ev[0].record(stream)
        out = fn()
        ev[1].record(stream)
        torch.cuda.synchronize()
        return out, ev[0].elapsed_time(ev[1]) / 1e3

    def ellipses(seed):
        return s.raster_to_tree(s.phantom(seed=seed, count=8, axis=(1.0, 3.0), eps=(1.1, 1.5)))

    inc = torch.from_numpy(s.line_sources(ntx, radius).astype(np.complex64)).to(dev)
    chi_true = torch.from_numpy(ellipses(5000)).to(dev)
    mes = s.measure(inc, chi_true, noise=0.01, seed=5001, tol=1e-6, engine=isg.ENGINE_TENSOR, stream=stream)
    out = {"workload": "512x512 px (51.2 lambda), 128 line-source Tx x 256 near-field Rx on r=40 lambda, "
                       f"8 ellipses eps_r U[1.1,1.5], 1% noise, {iters} PR iterations, Tikhonov",
           "tol": TOL}

    def inversion(solver, engine, reg, reps=2, **kw):
        chi0 = torch.zeros(U, dtype=torch.complex128, device=dev)
        for _ in range(reps):
            (chi, hist), sec = timed(lambda: solver.dbim(inc, mes, chi=chi0, chi_true=chi_true, iterations=iters,
                                                          regular=reg, stream=stream, tol=TOL, maxit=1000,
                                                          engine=engine, check_every=2, **kw))
        return {"seconds": round(sec, 3), "seconds_per_iteration": round(sec / iters, 4),
                "solves": int(hist[-1]["solves"]), "bicgs_iterations": int(hist[-1]["iterations"]),
                "misfit": [round(h["misfit"], 6) for h in hist], "object_error_last": hist[-1]["object_error"]}, chi

    sweep = {f"{r:g}": inversion(s, isg.ENGINE_TENSOR, r, reps=1)[0] for r in regs}
    m0 = sweep[f"{regs[0]:g}"]["misfit"][-1]
    reg = max(r for r in regs if sweep[f"{r:g}"]["misfit"][-1] <= 1.5 * m0)
    out["tikhonov"] = {"chosen": reg, "sweep": {k: {"misfit_last": v["misfit"][-1],
                                                    "object_error_last": v["object_error_last"]}
                                                for k, v in sweep.items()}}

    # training triples: contrast j (one of triples / 16), transmitter t, total field u
    rng = np.random.default_rng(5100)
    ncon = triples // 16
    t0 = time.perf_counter()
    gall = torch.from_numpy(np.stack([k2 * ellipses(6000 + j) for j in range(ncon)]).astype(np.complex64)).to(dev)
    cid = np.repeat(np.arange(ncon), 16)
    tid = np.concatenate([rng.choice(ntx, 16, replace=False) for _ in range(ncon)])
    cid_t, tid_t = torch.from_numpy(cid).to(dev), torch.from_numpy(tid).to(dev)
    uall = torch.zeros((ncon * 16, U), dtype=torch.complex64, device=dev)
    data_its = []
    opts_t = isg.default_solve_opts(tol=TOL, maxit=1000, engine=isg.ENGINE_TENSOR, check_every=2)
    for j in range(0, ncon * 16, ntx):
        sl = slice(j, min(j + ntx, ncon * 16))
        ub = torch.zeros_like(uall[sl])
        info = s.bicgs(ub, gall[cid_t[sl]], inc[tid_t[sl]], opts=opts_t, stream=stream)
        uall[sl] = ub
        data_its += [i["iterations"] for i in info]
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    s.fno_create(width=32, modes=12, layers=4, batch=fno_batch, seed=1)
    steps = int(epochs * ncon * 16 / fno_batch)
    losses = []
    t0 = time.perf_counter()
    for k in range(steps):
        sel = torch.from_numpy(rng.choice(ncon * 16, fno_batch, replace=False)).to(dev)
        losses.append(s.fno_train_step(gall[cid_t[sel]], inc[tid_t[sel]], uall[sel],
                                       lr=3e-3 if k < 2 * steps // 3 else 1e-3, stream=stream))
        if k % 128 == 0:
            print("c5 training step %d / %d, loss %.4g, %.1f s" % (k, steps, losses[-1], time.perf_counter() - t0),
                  file=sys.stderr, flush=True)
        if time.perf_counter() - t0 > train_budget_s:
            break
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    del uall
    out["training"] = {"triples": ncon * 16, "contrasts": ncon, "data_s": round(t_data, 2),
                       "data_mean_iterations": float(np.mean(data_its)), "steps": len(losses), "batch": fno_batch,
                       "train_s": round(t_train, 2), "loss_first": float(np.mean(losses[:20])),
                       "loss_last": float(np.mean(losses[-20:])),
                       "network": "FNO width 32, 4 spectral layers, 12x24 modes, BF16 tcgen05 products, FP32 accumulate"}

    # what the network gains on the forward solves at the true contrast (held out)
    g_true = (k2 * chi_true).to(torch.complex64)
    fwd = {}
    for name, guess in (("zero", isg.GUESS_ZERO), ("learned", isg.GUESS_LEARNED)):
        x = torch.zeros_like(inc)
        o = isg.default_solve_opts(tol=TOL, maxit=1000, engine=isg.ENGINE_TENSOR, check_every=2, guess=guess)
        info, sec = timed(lambda: s.bicgs(x, g_true, inc, opts=o, stream=stream))
        fwd[name] = {"mean_iterations": float(np.mean([i["iterations"] for i in info])), "seconds": round(sec, 4),
                     "all_converged": all(i["status"] == 0 and 0 <= i["true_residual"] <= TOL for i in info)}
    out["forward_at_true_contrast"] = fwd

    runs, chis = {}, {}
    for name, kw in (("zero_start", {}), ("previous_iterate", {"warm_start": True}),
                     ("learned", {"guess": isg.GUESS_LEARNED}),
                     ("learned_then_previous", {"guess": isg.GUESS_LEARNED, "warm_start": True})):
        runs[name], chis[name] = inversion(s, isg.ENGINE_TENSOR, reg, **kw)
    ref = chis["zero_start"].cpu().numpy()
    for name in runs:
        runs[name]["contrast_vs_zero_start"] = float(np.linalg.norm(chis[name].cpu().numpy() - ref) /
                                                     np.linalg.norm(ref))
    del s
    s1 = isg.Solver(level, numrx=nrx, max_rhs=1, device=dev.index or 0)
    s1.setup_gpu()
    s1.set_nearfield_receivers(radius)
    runs["plain_single_rhs_fp32"], _ = inversion(s1, isg.ENGINE_SIMT, reg, reps=1)
    base = runs["plain_single_rhs_fp32"]["seconds"]
    for name in runs:
        runs[name]["speedup_vs_plain_single_rhs"] = round(base / runs[name]["seconds"], 2)
    out["inversions"] = runs
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu"])
    ap.add_argument("--ref-gpu-out", default="", help=argparse.SUPPRESS)
    ap.add_argument("--ref-gpu-in", default="", help=argparse.SUPPRESS)
    ap.add_argument("--engine", default="auto", choices=["auto", "simt", "tensor"])
    ap.add_argument("--plain-sample", type=int, default=4, help="single-RHS solves timed for the plain solvers")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline and the FP64 field check")
    ap.add_argument("--learned-pairs", type=int, default=16, help="solver-generated training pairs (0: no learned arm)")
    ap.add_argument("--learned-steps", type=int, default=150)
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5"],
                    help="c2: the headline 1024^2 / 256-Tx line (default); c1, c3, c4, c5: the reference's small "
                         "case, the mixed-size, 4096^2 and learned-warm-start inversion measurements, one JSON "
                         "line of their own")
    ap.add_argument("--stages-only", type=int, default=0,
                    help="only time the matvec stages on this many RHS of the workload (profiling case)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    if args.impl == "reference-gpu":
        run_reference_gpu(args)
        return

    import torch
    import isg
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    if args.workload != "c2":
        dev = torch.device("cuda", local)
        res = {"c1": run_config1, "c3": run_config3, "c4": run_config4, "c5": run_config5}[args.workload](isg, torch,
                                                                                                          dev)
        print(json.dumps({"workload": args.workload, **res}))
        return
    if args.stages_only:
        s = isg.Solver(LEVEL, numrx=32, max_rhs=args.stages_only, device=local)
        for eng in ([isg.ENGINE_SIMT, isg.ENGINE_TENSOR] if args.engine == "auto" else
                    [isg.ENGINE_SIMT if args.engine == "simt" else isg.ENGINE_TENSOR]):
            try:
                print(json.dumps({"engine": eng, "nrhs": args.stages_only,
                                  "stage_ms": s.time_stages(args.stages_only, eng, reps=3)}))
            except isg.IsgError as e:
                print(json.dumps({"engine": eng, "error": str(e)}))
        return
    s = isg.Solver(LEVEL, numrx=32, max_rhs=NTX, device=local)
    s.setup_gpu()
    g_np, b_np = make_inputs(s, rank)
    dev = torch.device("cuda", local)
    g = torch.from_numpy(g_np.astype(np.complex64)).to(dev)
    b = torch.from_numpy(b_np.astype(np.complex64)).to(dev)
    x = torch.zeros_like(b)
    stream = torch.cuda.Stream(dev)
    engine = {"simt": isg.ENGINE_SIMT, "tensor": isg.ENGINE_TENSOR, "auto": isg.ENGINE_TENSOR}[args.engine]
    opts = isg.default_solve_opts(tol=TOL, maxit=300, engine=engine, check_every=2)
    tuned = s.autotune(NTX, engine, stream=stream)  # launch shapes for this batch (untimed set-up)
    torch.cuda.synchronize()

    # Learned warm start: trained here on solver-generated fields; the timed
    # steps use it only if it saved iterations over the zero start.
    zero_its = None
    infos = s.bicgs(x, g, b, opts=opts, stream=stream)
    zero_its = float(np.mean([i["iterations"] for i in infos]))
    learned = None
    if args.learned_pairs > 0 and engine == isg.ENGINE_TENSOR:
        learned = learned_arm(s, isg, g, b, stream, args.learned_pairs, args.learned_steps, zero_its)
        if learned["pays"] and learned["all_converged"]:
            opts = isg.default_solve_opts(tol=TOL, maxit=300, engine=engine, check_every=2,
                                          guess=isg.GUESS_LEARNED)
    torch.cuda.cudart().cudaProfilerStart()  # a profiler started with profiling off sees the solves only

    def step():
        return s.bicgs(x, g, b, opts=opts, stream=stream)

    for _ in range(args.warmup):
        infos = step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches0 = isg.kernel_launches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    iters = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            infos = step()
            iters.append([i["iterations"] for i in infos])
        ev1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = isg.kernel_launches() - launches0
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dist, dev)
    bad = [i for i in infos if i["status"] != 0 or not (0 <= i["true_residual"] <= TOL)]
    value = world * NTX * 1000.0 / ms
    x_tx0 = x[0].cpu().numpy().astype(np.complex128)

    # End to end through the public API from pinned host buffers: every step
    # copies its contrast and incident fields in and its total fields out, on a
    # copy stream and double-buffered, so step i + 1's inputs and step i's
    # results cross PCIe while the solves run; the timed region runs from the
    # first input copy to the last result copy.
    b_host = torch.from_numpy(b_np.astype(np.complex64)).pin_memory()
    g_host = torch.from_numpy(g_np.astype(np.complex64)).pin_memory()
    x_host = torch.empty_like(b_host).pin_memory()
    e2e_steps = max(1, min(args.steps, 5))
    copy = torch.cuda.Stream(dev)
    gd = [torch.empty_like(g) for _ in range(2)]
    bd = [torch.empty_like(b) for _ in range(2)]
    xd = [torch.empty_like(b) for _ in range(2)]
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()

    def copy_in(j):
        with torch.cuda.stream(copy):
            gd[j].copy_(g_host, non_blocking=True)
            bd[j].copy_(b_host, non_blocking=True)
            ev_in[j].record(copy)

    with torch.cuda.stream(stream):
        e0.record(stream)
        copy.wait_stream(stream)
        copy_in(0)
        for i in range(e2e_steps):
            j = i & 1
            stream.wait_event(ev_in[j])
            if i + 1 < e2e_steps:
                copy_in(1 - j)  # buffers 1 - j: step i - 1's solve has returned, its result copy is queued before
            s.bicgs(xd[j], gd[j], bd[j], opts=opts, stream=stream)
            ev_out[j].record(stream)
            copy.wait_event(ev_out[j])
            with torch.cuda.stream(copy):
                x_host.copy_(xd[j], non_blocking=True)
        stream.wait_stream(copy)
        e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps, dist, dev)

    # Plain single-RHS FP32 solvers: one transmitter per launch sequence.
    plain = single_rhs_rate(s, g, b, isg.default_solve_opts(tol=TOL, maxit=300, engine=isg.ENGINE_SIMT,
                                                            check_every=1), stream, args.plain_sample)
    plain_tc = single_rhs_rate(s, g, b, isg.default_solve_opts(tol=TOL, maxit=300, engine=isg.ENGINE_TENSOR,
                                                               check_every=1), stream, args.plain_sample)

    # Roofline: the dominant kernel (near field + L2P on the tensor cores) and,
    # beside it, the whole matvec against HBM; both on the step's own batch of
    # NTX RHS (the launch shape of the timed region), each stage timed alone
    # with CUDA events on the launching stream.
    RB = NTX
    st = s.time_stages(nrhs=RB, engine=engine, reps=3)
    pk = peaks()
    bytes_mv = algorithmic_bytes_per_matvec(s) * RB
    achieved = bytes_mv / (st["total"] * 1e-3) / 1e9
    exe, useful = near_field_flops_per_rhs(s)
    near_useful = RB * useful / (st["near"] * 1e-3) / 1e12
    tc = engine == isg.ENGINE_TENSOR

    out = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        # No number is published for this metric; its own baseline is the plain single-RHS FP32 solver.
        "vs_baseline": value / (world * plain["value"]),
        "vs_baseline_basis": "value / (n_gpus x plain single-RHS complex-FP32 SIMT solver on the same workload)",
        "dtype": "c64 (FP64 dots)", "data": "synthetic",
        "config": workload_config(world),
        "solver": {"engine": "simt" if engine == isg.ENGINE_SIMT else "tensor", "batch": NTX,
                   "initial_guess": "learned" if opts.guess == isg.GUESS_LEARNED else "zero",
                   "autotuned": tuned},
        "mean_iterations": float(np.mean(iters)), "all_converged": not bad,
        "max_true_residual": max(i["true_residual"] for i in infos),
        "roofline": ({"bound": "tensor",
                      "kernel": f"k_tc_near_pipe (near field + L2P, 3xFP16 split tcgen05), {RB} RHS per launch",
                      "achieved": near_useful, "peak": pk["bf16_tflops"], "unit": "TFLOP/s",
                      "frac": near_useful / pk["bf16_tflops"], "peak_src": pk["src"] + " (bf16 burst)",
                      "flops": "useful complex work: (9 x 64 + ns_leaf) complex MACs x 8 per pixel",
                      "traffic": NEAR_TRAFFIC_16RHS_CAPTURED * RB / 16,
                      "traffic_src": "one ncu capture of a 16-RHS launch, scaled by RHS",
                      "launch_ms": st["near"],
                      "executed_tflops": RB * exe / (st["near"] * 1e-3) / 1e12,
                      "executed_flops_per_rhs": exe} if tc else
                     {"bound": "hbm", "kernel": f"MLFMA matvec (SIMT engine), {RB} RHS", "achieved": achieved,
                      "peak": pk["hbm_gbs"], "unit": "GB/s", "frac": achieved / pk["hbm_gbs"], "peak_src": pk["src"],
                      "traffic": None}),
        "roofline_matvec": {"bound": "hbm", "kernel": f"MLFMA matvec (P2M, M2M, M2L+L2L, L2P+near), {RB} RHS",
                            "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                            "frac": achieved / pk["hbm_gbs"], "peak_src": pk["src"], "stage_ms": st,
                            "algorithmic_bytes_per_rhs": algorithmic_bytes_per_matvec(s)},
        "plain": plain,
        "plain_tensor": plain_tc,
        "batching_factor": value / (world * plain_tc["value"]),
        "learned": learned,
        "e2e": {"value": world * NTX * 1000.0 / e2e_ms, "unit": "solves/s", "steps": e2e_steps,
                "h2d_bytes_per_step": int(b_host.numel() * 8 + g_host.numel() * 8),
                "d2h_bytes_per_step": int(x_host.numel() * 8)},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu:  # the CPU baseline and the FP64 check: one GPU only
        from _oracle import Reference
        if Reference.available():
            ref = Reference(LEVEL, 2 * math.pi, 32)
            out["cpu_baseline"], x5 = cpu_reference_sample(ref, g_np, b_np, args.cpu_budget, 8)
            out["parity"], x10 = field_parity(ref, g_np, b_np[0], x_tx0, x5, 0)
            out["reference_gpu"] = reference_gpu_sample(x10)
            if "value" in out["reference_gpu"]:
                out["reference_gpu"]["e2e_vs_reference_gpu"] = out["e2e"]["value"] / out["reference_gpu"]["value"]
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
