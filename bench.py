"""Benchmark: 64^3 Poisson multifrontal factor + solve on B200 (libmfgpu).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload poisson3d-64|poisson3d-48|poisson2d-100] [--forms fp64,mixed]

One step = numeric multifrontal factorization of A = poisson3d(64) (SCALE_SUM
row scaling, AMD order) followed by solve(F, B; refine) for 256 N(0,1)
right-hand sides (seed 4), with the refinement count each form needs to bring
the normwise backward error of every right-hand side to <= 1e-14.  The
pattern analysis (ordering + symbolic, done once per sparsity pattern) is
timed separately and reported as `analyze_s`.

`value` is the step time (seconds, lower is better) of the fastest form whose
solutions reach the accuracy target; both forms are reported under `forms`.  Inputs (A's values, Rs, B) are resident in HBM when the timed
region starts; `e2e` repeats the step through the C ABI with pinned host
buffers, host<->device copies included.  `--impl reference` times the CPU
oracle (the reference's algorithm restated in C++ over OpenBLAS) on the same
workload, on the host cores.

With N > 1 (torchrun), every rank factors and solves its own copy of the
system (replicas: one sparse system does not shard), the step time is the max
over ranks, and value = that time / N (seconds per system, whole job).

`--workload batch-1024` is the batched configuration instead: 1,024
independent shifted grid Laplacians (half 2-D with side U[16,64], half 3-D
with side U[8,20], 4 right-hand sides each) factored and solved by one
batched handle per GPU; one step = factor + solve(refine) of every system to
backward error <= 1e-14 per system.  With N > 1 the systems are split across
ranks by predicted flops (no collective); value = the max over ranks of the
step time (strong scaling: the batch is fixed).

`--method gplu` measures splu's default method instead, the Gilbert-Peierls
factorization (one warp per system) with solve(refine=2), on poisson2d-100
or a batch-N workload, beside the oracle's restatement on the host cores;
a single-GPU default run also reports it for poisson2d-100 under `gplu`
(`--no-gplu` skips it).
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
sys.path[:0] = [ROOT, os.path.join(ROOT, "pureumfpack.jl_b200")]

TARGET_ETA = 1e-14
CPU_FRONT_LIMIT = 2e10    # front elements beyond which the CPU oracle baseline is not run
MAX_REFINE = 8
REF_TIMED_STEPS = 3       # timed oracle steps of the reference arm (each is a full CPU factorization)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="poisson3d-64")
    ap.add_argument("--nrhs", type=int, default=256)
    ap.add_argument("--forms", default="fp64,mixed")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--records", default=None,
                    help="write the profiled step's launch records of every form (kernel class, level, tasks, ms, "
                         "algorithmic flops and bytes, tunable index) as JSON to this path")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the untimed comparison of the GPU factors with the oracle's (and mixed with FP64)")
    ap.add_argument("--solve-mode", default="auto", choices=["auto", "step", "persistent"],
                    help="solve launches: library default by rhs count, per step, or one persistent launch per pass")
    ap.add_argument("--relax", action="store_true",
                    help="relaxed amalgamation (opt-in; the factors then store explicit zeros)")
    ap.add_argument("--no-merge", action="store_true",
                    help="one front per supernode (default: supernode chains share a front; same factors)")
    ap.add_argument("--dtype", default="float64", choices=["float64", "float32"],
                    help="float32: the workload as a Float32 matrix through the Float32 C ABI (a side line, "
                         "not the headline metric)")
    ap.add_argument("--method", default="multifrontal", choices=["multifrontal", "gplu"],
                    help="gplu: splu(A; method=:gplu) (Gilbert-Peierls, one warp per system) on --workload "
                         "poisson2d-100 (default for this method) or batch-N")
    ap.add_argument("--no-gplu", action="store_true",
                    help="skip the side measurement of splu's default Gilbert-Peierls method on poisson2d-100")
    ap.add_argument("--no-autotune", action="store_true",
                    help="mixed form: keep the built-in GEMM variant rule instead of the learned autotuner")
    return ap.parse_args()


def make_workload(name: str, nrhs: int):
    from pureumfpack import matrices as M

    kind, k = name.rsplit("-", 1)
    k = int(k)
    if kind == "poisson3d":
        A = M.poisson3d(k)
        seed = 4
    elif kind == "poisson3d_shift":
        A = M.poisson3d(k).add_diagonal(1e-3)
        seed = 1
    elif kind == "poisson2d":
        A = M.poisson2d(k)
        seed = 0
    elif kind == "convdiff":
        A = M.convdiff3d(k)
        seed = 2
    elif kind == "random":
        A = M.random_unsym(k, 5, 10.0, seed=3)
        seed = 3
    else:
        raise SystemExit(f"unknown workload {name}")
    B = M.rhs(A.n, seed=seed, nrhs=nrhs)
    if B.ndim == 1:
        B = B.reshape(-1, 1)
    return A, np.asfortranarray(B)


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.15)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def fp_peak_tflops(torch, dtype, device) -> float:
    """In-run cuBLAS GEMM throughput (TFLOP/s) as the roofline denominator for
    a precision MEASURED_PEAKS.json does not cover (FP64, FP32 SIMT)."""
    n = 8192 if dtype == torch.float64 else 8192
    a = torch.randn(n, n, dtype=dtype, device=device)
    b = torch.randn(n, n, dtype=dtype, device=device)
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    torch.backends.cuda.matmul.allow_tf32 = prev
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


# ---------------------------------------------------------------------------
def _oracle_eta(A, X, B):
    """Largest normwise backward error over the columns (host, FP64)."""
    S = A.to_scipy()
    r = B - S @ X
    anorm = np.max(np.asarray(abs(S).sum(axis=1)).ravel())
    return float(np.max(np.abs(r).max(axis=0) / (anorm * np.abs(X).max(axis=0) + np.abs(B).max(axis=0))))


def cpu_baseline(A, B, sample_rhs: int = 4, order: str = "amd", scale: int = 1, threads: int = 0,
                 refine: int | None = None, keep_factors: bool = False):
    """The oracle (C++ restatement of the reference over OpenBLAS): symbolic +
    numeric multifrontal_lu of the full matrix, then solve(F, b; refine) for
    `sample_rhs` right-hand sides, scaled to the full RHS count.  `refine`
    None: the fewest refinements that bring the sampled right-hand sides to
    backward error <= TARGET_ETA, the oracle's own need (the same rule the GPU
    forms follow); only the solve with that count is timed.  threads 0: all
    host cores for BLAS.  Returns (seconds per step, details, oracle factors
    or None)."""
    from oracle import oracle as O

    cores = threads or (os.cpu_count() or 1)
    O.blas_threads(cores)
    t0 = time.perf_counter()
    S = O.symbolic_mf(A, q=O.colamd_order(A) if order == "colamd" else None)
    t1 = time.perf_counter()
    Rs = O.row_scaling(A, scale)
    As = O.apply_row_scaling(A, Rs)
    Fo = O.numeric(S, As, check=False)
    t2 = time.perf_counter()
    F = O.PureLU(Fo, Rs, A)
    nrhs = B.shape[1]
    k = min(sample_rhs, nrhs)
    Bk = np.asfortranarray(B[:, :k])
    etas = []
    if refine is None:
        for refine in range(MAX_REFINE + 1):
            etas.append(_oracle_eta(A, O.solve(F, Bk, refine=refine), Bk))
            if etas[-1] <= TARGET_ETA:
                break
    t3 = time.perf_counter()
    X = O.solve(F, Bk, refine=refine)
    t4 = time.perf_counter()
    numeric = t2 - t1
    solve_full = (t4 - t3) * nrhs / k
    return numeric + solve_full, {
        "symbolic_s": t1 - t0, "numeric_s": numeric, "solve_s_per_rhs": (t4 - t3) / k, "cores": cores,
        "refine": refine, "bwd_err": _oracle_eta(A, X, Bk), "bwd_err_by_refine": etas or None,
        "sample": f"full {A.n}-unknown numeric factorization (OpenBLAS, {cores} threads) + solve(refine={refine}, "
                  f"the oracle's fewest refinements to backward error <= {TARGET_ETA:g}) of {k} of {nrhs} "
                  f"right-hand sides, scaled x{nrhs / k:g}; symbolic phase reported separately",
    }, (Fo if keep_factors else None)


def run_reference(args):
    """The reference's CPU path on the host cores: the oracle, all host
    threads, on this arm's workload.  Each timed step is one full numeric
    factorization plus the sampled solve (about 15-20 s at poisson3d-64), so
    at most REF_TIMED_STEPS of the requested steps are timed; one extra
    untimed run measures the same step with one BLAS thread."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    A, B = make_workload(args.workload, args.nrhs)
    order, scale = workload_setup(args.workload)
    _, det0, _ = cpu_baseline(A, B, order=order, scale=scale)        # warm-up; fixes the refine count
    refine = det0["refine"]
    times, det = [], None
    timed = max(1, min(args.steps, REF_TIMED_STEPS))
    for _ in range(timed):
        t, det, _ = cpu_baseline(A, B, order=order, scale=scale, refine=refine)
        times.append(t)
    v = float(np.mean(times))
    t1, det1, _ = cpu_baseline(A, B, order=order, scale=scale, refine=refine, threads=1)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, A),
        "cpu_baseline": {"value": v, "unit": "s", "cores": det["cores"], "kind": "port", "sample": det["sample"],
                         "symbolic_s": det["symbolic_s"], "numeric_s": det["numeric_s"], "refine": refine,
                         "bwd_err": det["bwd_err"], "timed_steps": timed,
                         "threads_1": {"value": t1, "unit": "s", "cores": 1, "numeric_s": det1["numeric_s"],
                                       "sample": det1["sample"]}},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


METRIC = "64^3 Poisson factor+solve s at bwd err <=1e-14: mixed vs FP64 on 1 B200; %roofline"


def workload_setup(name: str):
    """(ordering, scale kind) of a workload: the unsymmetric pair runs with
    COLAMD through multifrontal_lu(As; q) and SCALE_MAX, the rest with AMD
    (as splu(A; method=:multifrontal)) and SCALE_SUM."""
    kind = name.rsplit("-", 1)[0]
    return ("colamd", 2) if kind in ("convdiff", "random") else ("amd", 1)


def workload_config(args, A):
    order, scale = workload_setup(args.workload)
    return {"workload": f"{args.workload} n={A.n} nnz={A.nnz()} nrhs={args.nrhs} {order.upper()} "
                        f"{'SCALE_MAX' if scale == 2 else 'SCALE_SUM'}, numeric factor + "
                        f"solve(refine) to normwise backward error <= 1e-14",
            "nrhs": args.nrhs, "relaxed_amalgamation": bool(getattr(args, "relax", False)),
            "merged_fronts": not getattr(args, "no_merge", False),
            "l2": "working set (fronts) larger than L2; no explicit flush",
            "parallelism": f"replicas x{args.gpus}" if args.gpus > 1 else "1 GPU"}


# ---------------------------------------------------------------------------
TUNE_TRAIN = ("poisson3d-24", "poisson3d-32", "poisson3d-40", "poisson3d-48", "convdiff-20", "poisson2d-200")


def autotune_mixed(ctx, run, R, device):
    """Learned GEMM-variant schedule for the mixed form: the cost model is
    trained on the GPU on exhaustive tables of smaller matrices (TUNE_TRAIN,
    same right-hand-side count), picks each launch's variant here, and this
    workload's own exhaustive table judges the choice.  The timed steps run
    the model's schedule."""
    import torch
    from pureumfpack import GpuContext, PRECISION_MIXED, row_scaling, symbolic_mf
    from pureumfpack import autotune as AT

    t0 = time.perf_counter()
    tables = []
    for name in TUNE_TRAIN:
        A, B = make_workload(name, R)
        c = GpuContext(device=device, precision=PRECISION_MIXED)
        c.analyze(A, symbolic_mf(A))
        dv = torch.device("cuda", device)
        ax = torch.from_numpy(A.nzval).to(dv)
        rs = torch.from_numpy(row_scaling(A, 1)).to(dv)
        bb = torch.from_numpy(np.asfortranarray(B).ravel(order="F")).to(dv)
        xx = torch.empty(A.n * R, dtype=torch.float64, device=dv)
        torch.cuda.synchronize()

        def r(c=c, ax=ax, rs=rs, bb=bb, xx=xx, n=A.n):
            c.factor_device(ax.data_ptr(), rs.data_ptr(), True)
            c.solve_device(R, bb.data_ptr(), n, xx.data_ptr(), n, 0)

        r()
        tables.append(AT.exhaustive_table(c, r, R))
        del c
    tuner = AT.train(tables, hidden=32, iters=3000, lr=3e-3, seed=0, device=device)
    t_train = time.perf_counter() - t0
    run()
    feats = AT.tune_features(ctx, R)
    choice = tuner.choose(feats, AT.rule_choice(feats, R))
    table = AT.exhaustive_table(ctx, run, R)
    j = AT.judge(tuner, table)
    AT.set_choice(ctx, choice)
    return {"launches": j["launches"], "mispredicted": j["mispredicted"], "model_ms": round(j["model_ms"], 3),
            "exhaustive_ms": round(j["table_ms"], 3), "rule_ms": round(j["rule_ms"], 3),
            "train_loss": round(tuner.loss, 4), "train_matrices": list(TUNE_TRAIN), "train_s": round(t_train, 2),
            "tensor_core_launches": int(np.sum(choice == 1))}


def bx3_peak(peaks):
    """Useful FP32 TFLOP/s ceiling of the BF16x3 tensor-core GEMMs: six bf16
    products per useful product on the sustained bf16 rate."""
    if "bf16_tflops_sustained" in peaks:
        return peaks["bf16_tflops_sustained"] / 6.0, ("MEASURED_PEAKS.json bf16_tflops_sustained / 6 (of measured): "
                                                       "BF16x3 issues six BF16 tensor-core products per useful "
                                                       "FP32 product")
    return 1400.0 / 6.0, "fallback sustained bf16 1.4 PFLOP/s / 6 (BF16x3: six bf16 products per useful product)"


def roofline_of(P, primary, fp64_peak, peaks):
    """Roofline entry for the dominant kernel class of one profiled step."""
    kern = P["stats"]["kernels"]
    dom = max(kern, key=lambda k: kern[k]["ms"])
    kd = kern[dom]
    per_launch_ms = kd["ms"] / max(kd["launches"], 1)
    if dom.startswith("gemm"):
        if primary == "fp64":
            peak, peak_src = fp64_peak, "in-run cuBLAS DGEMM 8192^3 (FP64 peak is not in MEASURED_PEAKS.json)"
        else:
            peak, peak_src = bx3_peak(peaks)
        achieved = kd["flops"] / (kd["ms"] * 1e-3) / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak,
                "unit": "TFLOP/s", "frac": achieved / peak, "peak_source": peak_src}
    else:
        peak = peaks.get("hbm_gbs", 6650.0)
        achieved = kd["bytes"] / (kd["ms"] * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks else "fallback"}
    traffic, tnote = None, None
    ratio = NCU_TRAFFIC_RATIO.get((dom, primary))
    if ratio is not None:
        traffic = ratio[0] * kd["bytes"] / max(kd["launches"], 1)
        tnote = (f"DRAM bytes per launch: ncu dram__bytes_read+write over algorithmic bytes ({ratio[0]:.3f}, "
                 f"{ratio[1]}) x this class's algorithmic bytes per launch")
    roof.update({"kernel": dom, "launches": kd["launches"], "avg_launch_ms": per_launch_ms,
                 "traffic": traffic, "algorithmic_bytes_per_launch": kd["bytes"] / max(kd["launches"], 1),
                 "note": "achieved = algorithmic work of the kernel class / its CUDA-event time over one profiled step"
                         + (f"; traffic: {tnote}" if tnote else "")})
    return roof


SOLVE_CLASSES = ("fwd_small", "fwd_assemble", "fwd_thin", "gemm_solve", "bwd_small", "bwd_gather",
                 "solve_finish")


def class_rooflines(f, form, fp64_peak, peaks, nrhs):
    """Per-class roofline entries of one form's profiled step: the factor
    GEMMs against the tensor peak of their precision, assembly and the CSC
    scatter against HBM bandwidth, and one solve pass (forward + backward
    over the resident fronts) both in GB/s and in TFLOP/s.  A solve pass's
    algorithmic work: flops 2 (nnz(L) + nnz(U)) nrhs; bytes: the factor values
    read once plus the right-hand side, solution and factor-order copy
    (es (nnz(L) + nnz(U)) + 24 n nrhs)."""
    st = f["stats"]
    kern = st["kernels"]
    hbm = peaks.get("hbm_gbs", 6650.0)
    es = 8 if form == "fp64" else 4
    tpeak, tsrc = (fp64_peak, "in-run cuBLAS DGEMM") if form == "fp64" else bx3_peak(peaks)
    out = {}
    if "gemm_factor" in kern:
        k = kern["gemm_factor"]
        a = k["flops"] / (k["ms"] * 1e-3) / 1e12
        out["gemm_factor"] = {"bound": "tensor", "achieved": a, "peak": tpeak, "unit": "TFLOP/s", "frac": a / tpeak,
                              "ms": k["ms"], "launches": k["launches"], "peak_source": tsrc}
        ratio = NCU_TRAFFIC_RATIO.get(("gemm_factor", form))
        if ratio is not None:
            out["gemm_factor"]["traffic_per_launch"] = ratio[0] * k["bytes"] / max(k["launches"], 1)
            out["gemm_factor"]["traffic_source"] = f"ncu DRAM / algorithmic bytes {ratio[0]:.3f} ({ratio[1]})"
    for name in ("assemble_columns", "scatter_csc"):
        if name in kern and kern[name]["bytes"] > 0:
            k = kern[name]
            a = k["bytes"] / (k["ms"] * 1e-3) / 1e9
            out[name] = {"bound": "hbm", "achieved": a, "peak": hbm, "unit": "GB/s", "frac": a / hbm, "ms": k["ms"],
                         "launches": k["launches"], "algorithmic_bytes": k["bytes"]}
            ratio = NCU_TRAFFIC_RATIO.get((name, form))
            if ratio is not None:
                out[name]["traffic_per_launch"] = ratio[0] * k["bytes"] / max(k["launches"], 1)
                out[name]["traffic_source"] = f"ncu DRAM / algorithmic bytes {ratio[0]:.3f} ({ratio[1]})"
    passes = f["refine"] + 1
    ms = sum(kern[c]["ms"] for c in SOLVE_CLASSES if c in kern) / passes
    if ms > 0:
        nnz = float(st["nnz_l"] + st["nnz_u"])
        flops = 2.0 * nnz * nrhs
        by = es * nnz + 24.0 * st["n"] * nrhs
        gbs = by / (ms * 1e-3) / 1e9
        tfs = flops / (ms * 1e-3) / 1e12
        out["solve_pass"] = {"ms": ms, "passes": passes, "GB/s": gbs, "hbm_frac": gbs / hbm, "TFLOP/s": tfs,
                             "tensor_frac": tfs / tpeak, "algorithmic_bytes": by, "flops": flops,
                             "bound": "tensor" if flops / by > tpeak * 1e3 / hbm else "hbm"}
    return out


def _colwise(colptr, ref, got):
    """(max over columns of ||got - ref|| / ||ref||, max entry-wise relative
    error over entries with |ref| > 1e-6 max|column|) for CSC values."""
    ref = np.asarray(ref, dtype=np.float64)
    got = np.asarray(got, dtype=np.float64)
    cnt = np.diff(np.asarray(colptr, np.int64))
    if ref.size == 0:
        return 0.0, 0.0
    starts = np.asarray(colptr, np.int64)[:-1][cnt > 0] - 1
    aref = np.abs(ref)
    d = np.abs(got - ref)
    colmax = np.maximum.reduceat(aref, starts)
    c2 = np.add.reduceat(aref * aref, starts)
    e2 = np.add.reduceat(d * d, starts)
    nz = c2 > 0
    big = aref > np.repeat(1e-6 * colmax, cnt[cnt > 0])
    return (float(np.max(np.sqrt(e2[nz] / c2[nz]))) if nz.any() else 0.0,
            float(np.max(d[big] / aref[big])) if big.any() else 0.0)


def factor_parity(ref, got):
    """Structure and values of factors `got` against `ref` (dicts of 1-based
    CSC arrays Lcolptr, Lrowval, Lnzval, Ucolptr, Urowval, Unzval, p, q,
    pinv): fill, patterns and pivots bit-equal, values per column."""
    eq = lambda k: bool(np.array_equal(ref[k], got[k]))  # noqa: E731
    fill = int(ref["Lcolptr"][-1] - 1 + ref["Ucolptr"][-1] - 1)
    out = {"fill": fill, "fill_equal": fill == int(got["Lcolptr"][-1] - 1 + got["Ucolptr"][-1] - 1),
           "pattern_equal": all(eq(k) for k in ("Lcolptr", "Lrowval", "Ucolptr", "Urowval")),
           "pivots_equal": all(eq(k) for k in ("p", "q", "pinv"))}
    if out["pattern_equal"]:
        ln, le = _colwise(ref["Lcolptr"], ref["Lnzval"], got["Lnzval"])
        un, ue = _colwise(ref["Ucolptr"], ref["Unzval"], got["Unzval"])
        out.update({"max_colwise": max(ln, un), "max_entrywise": max(le, ue)})
    return out


def gpu_factors(ctx):
    L, U, p, q, pinv = ctx.factors()
    return {"Lcolptr": L.colptr, "Lrowval": L.rowval, "Lnzval": L.nzval, "Ucolptr": U.colptr, "Urowval": U.rowval,
            "Unzval": U.nzval, "p": p, "q": q, "pinv": pinv}


# DRAM traffic over algorithmic bytes per kernel class, from ncu captures of
# a few launches on smaller cases (dram__bytes_read.sum + dram__bytes_write.sum
# over the class's algorithmic bytes of the same launches); scaled to this
# run's launches by their algorithmic bytes.  The captures' commands and
# figures are summarised under profiles/.
NCU_TRAFFIC_RATIO = {
    ("gemm_factor", "fp64"): (0.743, "k_gemm_f64 factor updates, poisson3d-48"),
    ("gemm_factor", "mixed"): (0.673, "five k_gemm_bx3 factor-update launches of 112-1305 tiles, poisson3d-48"),
    ("assemble_columns", "mixed"): (0.732, "one k_assemble_columns launch (4821 front columns), poisson3d-48"),
}


def run_f32(args):
    """The workload as a Float32 matrix (the reference's generic Tv =
    Float32): splu's Float32 row scaling on the host, mfgpu_factor_f32 +
    mfgpu_solve_f32 with host buffers, copies included, timed with CUDA events
    on the library's stream; beside it the oracle's Float32 path (sgetrf /
    strsm / sgemm fronts, Float32 solve) on the host cores.  One GPU."""
    import torch

    from pureumfpack import GpuContext, colamd_order, row_scaling, symbolic_mf

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    A64, B64 = make_workload(args.workload, args.nrhs)
    A = A64.astype(np.float32)
    B = np.asfortranarray(B64.astype(np.float32))
    n, R = A.n, B.shape[1]
    order, scale = workload_setup(args.workload)
    q = colamd_order(A) if order == "colamd" else None
    S = symbolic_mf(A, q=q)
    Rs = row_scaling(A, scale)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    ctx = GpuContext(device=0)
    ctx.set_stream(stream.cuda_stream)
    ctx.analyze(A, S)
    Sd = A64.to_scipy()
    refine = 0

    def step(r):
        ctx.factor_f32(A.nzval, Rs, False)
        return ctx.solve(B, r)   # Float32 b and x after factor_f32

    # fewest refinements reaching the Float32 residual level of the reference
    # check (normwise relative residual <= 1e-6, i.e. a few Float32 ulps)
    for r in range(4):
        x = step(r)
        res = float(np.max(np.linalg.norm(Sd @ x.astype(np.float64) - B, axis=0) / np.linalg.norm(B, axis=0)))
        refine = r
        if res <= 1e-6:
            break
    for _ in range(args.warmup):
        step(refine)
    clk = ClockSampler(0)
    clk.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        step(refine)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    sec = ev0.elapsed_time(ev1) / 1e3 / args.steps
    cpu = None
    if not args.no_cpu_baseline:
        from oracle import oracle as O

        cores = os.cpu_count() or 1
        O.blas_threads(cores)
        k = min(4, R)
        t0 = time.perf_counter()
        Fo = O.splu_f32(A, scale=scale, check=False, q=q)
        t1 = time.perf_counter()
        O.solve_f32(Fo, np.asfortranarray(B[:, :k]), refine=refine)
        t2 = time.perf_counter()
        cpu = {"value": (t1 - t0) + (t2 - t1) * R / k, "unit": "s", "cores": cores, "kind": "port",
               "sample": f"oracle Float32 splu (symbolic + numeric, OpenBLAS sgetrf/strsm/sgemm, {cores} threads) "
                         f"+ Float32 solve(refine={refine}) of {k} of {R} right-hand sides, scaled x{R / k:g}"}
    line = {"metric": f"{args.workload} Float32 factor+solve s (host buffers, copies included)", "value": sec,
            "unit": "s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "dtype": "f32", "data": "synthetic", "refine": refine, "residual": res,
            "config": {"workload": f"{args.workload} as Float32, n={n}, nrhs={R}, {order.upper()}",
                       "l2": "working set (fronts) larger than L2; no explicit flush"},
            "e2e": {"value": sec, "unit": "s", "h2d_bytes_per_step": int(A.nnz() * 4 + Rs.size * 4 + B.nbytes),
                    "d2h_bytes_per_step": int(B.nbytes)},
            "cpu_baseline": cpu, "clocks": clocks, "stats": {k: ctx.stats().get(k) for k in ("nsuper", "fronts", "nnz_l")}}
    print(json.dumps(line), flush=True)
    return 0


def gplu_measure(wl: str, steps: int, warmup: int, cpu: bool = True) -> dict:
    """splu(A; method=:gplu, ordering=:amd, tol=0.1, scale=SCALE_SUM) then
    solve(F, b; refine=2) (src/interface.jl:93-120,170-177) on one system or
    a batch of independent systems (`batch-N`), with host buffers; beside it
    the oracle's restatement of the same Gilbert-Peierls factorization and
    solve on the host cores (one system per thread).  s = the device time of
    the library's kernels (factor, finish, solve; CUDA events on its stream,
    median over the timed steps), e2e_s = the API calls' wall time
    (ordering, scaling, copies included)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle as O
    from pureumfpack import SCALE_SUM, BatchGPLU
    from pureumfpack import matrices as M

    if wl.startswith("batch-"):
        sysl = M.batched_set(int(wl.split("-", 1)[1]), seed=0, nrhs=4)
        desc = "2-D side U[16,64] / 3-D side U[8,20], shift U[0,1], 4 rhs each"
    else:
        A, B = make_workload(wl, 1)
        sysl = [(A, np.asfortranarray(B.reshape(A.n, -1)))]
        desc = f"n={A.n} nnz={A.nnz()} 1 rhs"
    As, Bs = [a for a, _ in sysl], [b for _, b in sysl]
    refine = 2
    dev_ms, wall = [], []
    for it in range(warmup + steps):
        t0 = time.perf_counter()
        F = BatchGPLU(As, ordering="amd", tol=0.1, scale=SCALE_SUM)
        Xs = F.solve(Bs, refine=refine)
        t1 = time.perf_counter()
        if it >= warmup:
            tm = F.ctx.timings()
            dev_ms.append(tm["factor_ms"] + tm["finish_ms"] + tm["solve_ms"])
            wall.append(t1 - t0)
    tm = F.ctx.timings()
    eta = max(_oracle_eta(A, X, B) for A, X, B in zip(As, Xs, Bs))
    # parity: every system's factors and solution against the oracle (sampled for large batches)
    idx = list(range(0, len(As), max(1, len(As) // 64)))
    exact = True
    for i in idx:
        Fo = O.splu_gplu(As[i], ordering="amd", tol=0.1, scale=O.SCALE_SUM)
        L, U, p, q, pinv = F.factors(i)
        exact &= (np.array_equal(L.rowval, Fo.F.Lrowval) and np.array_equal(L.nzval, Fo.F.Lnzval)
                  and np.array_equal(U.rowval, Fo.F.Urowval) and np.array_equal(U.nzval, Fo.F.Unzval)
                  and np.array_equal(p, Fo.F.p) and np.array_equal(Xs[i], O.solve(Fo, Bs[i], refine=refine)))
    cpu_line = None
    if cpu:
        cores = os.cpu_count() or 1

        def one(i):
            Fo = O.splu_gplu(As[i], ordering="amd", tol=0.1, scale=O.SCALE_SUM)
            O.solve(Fo, Bs[i], refine=refine)

        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=cores) as ex:
            list(ex.map(one, range(len(As))))
        cpu_line = {"value": time.perf_counter() - t0, "unit": "s", "cores": min(cores, len(As)), "kind": "port",
                    "sample": f"the oracle's splu(method=:gplu, AMD) + solve(refine={refine}) of every system, "
                              f"one system per host thread"}
    return {"workload": f"{wl}: {len(As)} system(s), {desc}, AMD, SCALE_SUM, tol 0.1, refine {refine}",
            "s": float(np.median(dev_ms)) / 1e3, "e2e_s": float(np.median(wall)),
            "h2d_bytes": int(sum(A.nnz() * 16 + A.n * 16 + B.nbytes for A, B in sysl)),
            "d2h_bytes": int(sum(B.nbytes for B in Bs)),
            "kernels_ms": {"factor": tm["factor_ms"], "finish": tm["finish_ms"], "solve": tm["solve_ms"]},
            "factor_launches": tm["factor_launches"], "reruns": tm["reruns"], "bwd_err": eta,
            "parity": {"systems_checked": len(idx), "bitwise_equal": bool(exact)}, "cpu_baseline": cpu_line}


def run_gplu(args):
    """`--method gplu`: the Gilbert-Peierls path (gplu_measure) as its own
    JSON line; `--workload` poisson2d-100 (the default for this method) or
    batch-N.  One GPU."""
    import torch

    torch.cuda.set_device(0)
    wl = args.workload if args.workload != "poisson3d-64" else "poisson2d-100"
    g = gplu_measure(wl, args.steps, args.warmup, cpu=not args.no_cpu_baseline)
    line = {"metric": f"{wl} splu(method=:gplu) factor+solve s", "value": g["s"], "unit": "s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": False, "dtype": "f64",
            "data": "synthetic", "config": {"workload": g["workload"]},
            "e2e": {"value": g["e2e_s"], "unit": "s", "h2d_bytes_per_step": g["h2d_bytes"],
                    "d2h_bytes_per_step": g["d2h_bytes"]},
            "kernels_ms": g["kernels_ms"], "factor_launches": g["factor_launches"], "reruns": g["reruns"],
            "bwd_err": g["bwd_err"], "parity": g["parity"], "cpu_baseline": g["cpu_baseline"]}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.method == "gplu":
        return run_gplu(args)
    if args.dtype == "float32":
        return run_f32(args)
    if args.workload.startswith("batch-"):
        return run_batch(args)
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)

    from pureumfpack import GpuContext, colamd_order, row_scaling, symbolic_mf, PRECISION_FP64, PRECISION_MIXED

    A, B = make_workload(args.workload, args.nrhs)
    n, R = A.n, B.shape[1]
    t0 = time.perf_counter()
    order, scale = workload_setup(args.workload)
    S = symbolic_mf(A, q=colamd_order(A) if order == "colamd" else None, relax=args.relax)
    Rs = row_scaling(A, scale)
    t_sym = time.perf_counter() - t0

    # a dedicated stream shared with the library: CUDA events recorded on it
    # bracket exactly the library's kernels (and it can be graph-captured)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    d_ax = torch.from_numpy(A.nzval).to(dev)
    d_rs = torch.from_numpy(Rs).to(dev)
    d_b = torch.from_numpy(np.asfortranarray(B).ravel(order="F")).to(dev)
    d_x = torch.empty(n * R, dtype=torch.float64, device=dev)

    forms = {}
    all_records = {}
    kept, par_mixed = {}, None
    peaks = measured_peaks()
    for form in [f for f in args.forms.split(",") if f]:
        prec = PRECISION_MIXED if form == "mixed" else PRECISION_FP64
        ctx = GpuContext(device=local, precision=prec,
                         persistent_solve={"auto": None, "step": False, "persistent": True}[args.solve_mode],
                         merge_fronts=not args.no_merge)
        ctx.set_stream(stream.cuda_stream)
        t0 = time.perf_counter()
        ctx.analyze(A, S)
        t_an = time.perf_counter() - t0

        def step(refine):
            st = ctx.factor_device(d_ax.data_ptr(), d_rs.data_ptr(), True)
            if st != 0:
                raise RuntimeError(f"singular pivot at column {st}")
            ctx.solve_device(R, d_b.data_ptr(), n, d_x.data_ptr(), n, refine)

        tune = None
        if form == "mixed" and not args.no_autotune:
            tune = autotune_mixed(ctx, lambda: step(0), R, local)

        # refinement count that reaches the accuracy target on every rhs
        refine, eta, etas = 0, None, []
        for refine in range(0, MAX_REFINE + 1):
            step(refine)
            eta = ctx.backward_error_device(R, d_b.data_ptr(), n, d_x.data_ptr(), n)
            etas.append(eta)
            if eta <= TARGET_ETA:
                break
        for _ in range(args.warmup):
            step(refine)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        ctx.set_profiling(False)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step(refine)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        clk = clocks.stop()
        ms = e0.elapsed_time(e1) / args.steps
        launches = ctx.stats()["launches"]
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
            dist.barrier()
        eta = ctx.backward_error_device(R, d_b.data_ptr(), n, d_x.data_ptr(), n)
        # profiled pass (not timed): per-kernel-class device times
        ctx.set_profiling(True)
        step(refine)
        torch.cuda.synchronize()
        st = ctx.stats()
        if args.records:
            all_records[form] = ctx.launch_records()
        ctx.set_profiling(False)
        # end to end through the C ABI with pinned host buffers
        e2e = None
        if not args.no_e2e:
            h_ax = torch.from_numpy(A.nzval).pin_memory()
            h_rs = torch.from_numpy(Rs).pin_memory()
            h_b = torch.from_numpy(np.asfortranarray(B).ravel(order="F")).pin_memory()
            h_x = torch.empty(n * R, dtype=torch.float64).pin_memory()
            lib = ctx._lib
            import ctypes

            dp = ctypes.POINTER(ctypes.c_double)

            def e2e_step():
                # solve(splu(A), B; refine) through one C-ABI call: the
                # right-hand sides cross the bus while the factorization runs
                rc = lib.mfgpu_factor_solve(ctx._h, ctypes.cast(h_ax.data_ptr(), dp),
                                            ctypes.cast(h_rs.data_ptr(), dp), 1, R, ctypes.cast(h_b.data_ptr(), dp),
                                            n, ctypes.cast(h_x.data_ptr(), dp), n, refine)
                if rc != 0:
                    raise RuntimeError(f"mfgpu_factor_solve -> {rc}")

            e2e_step()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                e2e_step()
            torch.cuda.synchronize()
            e2e_s = (time.perf_counter() - t0) / args.steps
            if world > 1:
                t = torch.tensor([e2e_s], device=dev)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                e2e_s = float(t.item())
            e2e = {"value": e2e_s / world, "unit": "s", "h2d_bytes_per_step": 8 * (A.nnz() + n + n * R),
                   "d2h_bytes_per_step": 8 * n * R}
        forms[form] = {"ms_per_step": ms, "refine": refine, "eta": eta, "analyze_s": t_an + t_sym,
                       "stats": st, "clocks": clk, "launches_timed": launches, "e2e": e2e, "etas": etas,
                       "autotune": tune}
        # parity (untimed): the FP64 form's factors are kept for the oracle
        # comparison; the mixed form's structure and values are compared with
        # the FP64 form's at once
        if world == 1 and not args.no_parity:
            fac = gpu_factors(ctx)
            if form == "fp64":
                kept["fp64"] = fac
            elif "fp64" in kept:
                par_mixed = factor_parity(kept["fp64"], fac)
            del fac
        del ctx
        torch.cuda.empty_cache()

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0
    if args.records:
        with open(args.records, "w") as fh:
            json.dump(all_records, fh)

    # the headline form: the fastest one whose solution meets the accuracy target
    ok = [k for k, f in forms.items() if f["eta"] is not None and f["eta"] <= TARGET_ETA]
    primary = min(ok or list(forms), key=lambda k: forms[k]["ms_per_step"])
    P = forms[primary]
    fp64_peak = fp_peak_tflops(torch, torch.float64, dev)
    roof = roofline_of(P, primary, fp64_peak, peaks)
    classes = {k: class_rooflines(f, k, fp64_peak, peaks, R) for k, f in forms.items()}

    cpu, parity = None, {}
    if par_mixed is not None:
        parity["mixed_vs_fp64"] = par_mixed
    # the oracle factors one front per supernode of the reference's structure
    # (no merged fronts): sum of (np + nu)^2 over the original supernodes
    npv, nuv = np.diff(S.sstart).astype(np.float64), np.diff(S.upd_ptr).astype(np.float64)
    oracle_front_elems = float(np.sum((npv + nuv) ** 2))
    if not args.no_cpu_baseline and world == 1 and oracle_front_elems > CPU_FRONT_LIMIT:
        cpu = {"value": None, "skipped": f"the oracle's full numeric factorization would materialise "
                                         f"{oracle_front_elems:.3g} front elements, far beyond a "
                                         f"bounded CPU sample"}
    elif not args.no_cpu_baseline and world == 1:
        try:
            order, scale = workload_setup(args.workload)
            v, det, Fo = cpu_baseline(A, B, order=order, scale=scale, keep_factors="fp64" in kept)
            cpu = {"value": v, "unit": "s", "cores": det["cores"], "kind": "port", "sample": det["sample"],
                   "symbolic_s": det["symbolic_s"], "numeric_s": det["numeric_s"], "refine": det["refine"],
                   "bwd_err": det["bwd_err"]}
            if Fo is not None:
                ref = {k: getattr(Fo, k) for k in ("Lcolptr", "Lrowval", "Lnzval", "Ucolptr", "Urowval", "Unzval",
                                                    "p", "q", "pinv")}
                parity["fp64_vs_oracle"] = factor_parity(ref, kept.pop("fp64"))
                del ref, Fo
        except Exception as e:  # the baseline must not kill the GPU number
            cpu = {"value": None, "error": str(e)}
    kept.clear()

    value = P["ms_per_step"] / 1e3 / world
    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": P["ms_per_step"], "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if primary == "fp64" else "f32+f64", "data": "synthetic", "form": primary,
        "config": workload_config(args, A),
        "forms": {k: {"s_per_step": f["ms_per_step"] / 1e3, "refine": f["refine"], "bwd_err": f["eta"],
                      "bwd_err_by_refine": f.get("etas"),
                      "factor_ms": f["stats"]["factor_ms"], "solve_ms": f["stats"]["solve_ms"],
                      "analyze_s": f["analyze_s"], "e2e_s": f["e2e"]["value"] if f["e2e"] else None,
                      "kernels_ms": {kk: round(vv["ms"], 3) for kk, vv in f["stats"]["kernels"].items()},
                      **({"autotune": f["autotune"]} if f.get("autotune") else {})}
                  for k, f in forms.items()},
        "roofline": roof,
        "roofline_classes": classes,
        "parity": parity or None,
        "cpu_baseline": cpu,
        "e2e": P["e2e"],
        "gpu_launches": P["launches_timed"],
        "clocks": P["clocks"],
        "stats": {k: P["stats"].get(k) for k in ("n", "nsuper", "levels", "nnz_l", "nnz_u", "max_front", "flops",
                                                 "front_elems", "front_elems_full", "pool_elems", "lean",
                                                 "flops_inverse", "fronts", "merged", "flops_exec")},
    }
    if world == 1 and not args.no_gplu:
        # splu's default method (Gilbert-Peierls) on the 2-D Poisson matrix of
        # the reference's CPU-runnable configuration, beside the headline
        try:
            line["gplu"] = gplu_measure("poisson2d-100", 3, 3, cpu=not args.no_cpu_baseline)
        except Exception as e:  # a side measurement must not kill the headline
            line["gplu"] = {"error": str(e)}
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


BATCH_METRIC = "{} batched systems factor+solve s at bwd err <=1e-14 per system on B200"


def _batch_eta(As, offs, B, X):
    """Largest normwise backward error over the systems and right-hand sides."""
    worst = 0.0
    for A, o in zip(As, offs[:-1]):
        S = A.to_scipy()
        b, x = B[o:o + A.n], X[o:o + A.n]
        r = b - S @ x
        anorm = np.max(np.asarray(abs(S).sum(axis=1)).ravel())
        eta = np.abs(r).max(axis=0) / (anorm * np.abs(x).max(axis=0) + np.abs(b).max(axis=0))
        worst = max(worst, float(eta.max()))
    return worst


def run_batch(args):
    from pureumfpack import PRECISION_FP64, PRECISION_MIXED, analyze_batch, row_scaling
    from pureumfpack import matrices as M
    from pureumfpack.shard import partition_by_cost, system_cost

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    count = int(args.workload.split("-", 1)[1])
    sysl = M.batched_set(count, seed=0, nrhs=4)
    t0 = time.perf_counter()
    costs = [system_cost(A) for A, _ in sysl]
    t_cost = time.perf_counter() - t0
    mine = partition_by_cost(costs, world)[rank]
    As = [sysl[i][0] for i in mine]
    Bs = [sysl[i][1] for i in mine]
    offs = np.cumsum([0] + [A.n for A in As])
    N, R = int(offs[-1]), 4
    nz = np.concatenate([A.nzval for A in As])
    rs = np.concatenate([row_scaling(A, 1) for A in As])
    B = np.zeros((N, R), order="F")
    for b, o in zip(Bs, offs[:-1]):
        B[o:o + b.shape[0]] = b
    flops_total = float(sum(costs))
    config = {"workload": f"{args.workload}: {count} systems (2-D side U[16,64] / 3-D side U[8,20], shift U[0,1], "
                          f"seed 0), {R} right-hand sides each, AMD, SCALE_SUM, factor + solve(refine) to backward "
                          f"error <= 1e-14 on every system",
              "systems": count, "unknowns": int(sum(A.n for A, _ in sysl)), "nrhs": R,
              "l2": "whole-batch working set (fronts) larger than L2; no explicit flush",
              "parallelism": f"systems split by predicted flops over {world} GPUs" if world > 1 else "1 GPU"}

    if args.impl == "reference":
        if rank != 0:
            return 0
        v, det = batch_cpu_baseline(sysl, costs)
        line = {"impl": "reference", "metric": BATCH_METRIC.format(count), "value": v, "unit": "s", "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False,
                "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                "cpu_baseline": {"value": v, "unit": "s", "kind": "port", **det},
                "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    d_ax = torch.from_numpy(nz).to(dev)
    d_rs = torch.from_numpy(rs).to(dev)
    d_b = torch.from_numpy(B.ravel(order="F")).to(dev)
    d_x = torch.empty(N * R, dtype=torch.float64, device=dev)
    forms, peaks = {}, measured_peaks()
    for form in [f for f in args.forms.split(",") if f]:
        prec = PRECISION_MIXED if form == "mixed" else PRECISION_FP64
        t0 = time.perf_counter()
        ctx = analyze_batch(As, "amd", device=local, precision=prec)
        t_an = time.perf_counter() - t0
        ctx.set_stream(stream.cuda_stream)

        def step(refine):
            ctx.factor_device(d_ax.data_ptr(), d_rs.data_ptr(), False)
            ctx.solve_device(R, d_b.data_ptr(), N, d_x.data_ptr(), N, refine)

        refine, eta = 0, None
        for refine in range(0, MAX_REFINE + 1):
            step(refine)
            torch.cuda.synchronize()
            eta = _batch_eta(As, offs, B, d_x.cpu().numpy().reshape(N, R, order="F"))
            if eta <= TARGET_ETA:
                break
        for _ in range(args.warmup):
            step(refine)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        clocks = ClockSampler(local)
        clocks.start()
        ctx.set_profiling(False)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            step(refine)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        clk = clocks.stop()
        ms = e0.elapsed_time(e1) / args.steps
        launches = ctx.stats()["launches"]
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
            dist.barrier()
        ctx.set_profiling(True)
        step(refine)
        torch.cuda.synchronize()
        st = ctx.stats()
        ctx.set_profiling(False)
        e2e = None
        if not args.no_e2e:
            import ctypes

            from pureumfpack import _lib as L

            lib = ctx._lib
            vals = [np.ascontiguousarray(A.nzval) for A in As]
            bs = [np.asfortranarray(b) for b in Bs]
            xs = [np.empty_like(b) for b in bs]
            pv, pb, px = L.ptr_array(vals), L.ptr_array(bs), L.ptr_array(xs)
            status = np.zeros(len(As), np.int64)

            def e2e_step():
                rc = lib.mfgpu_batch_factor(ctx._h, pv, 1, 0, L.ptr(status))
                if rc != 0:
                    raise RuntimeError(f"mfgpu_batch_factor -> {rc}")
                rc = lib.mfgpu_batch_solve(ctx._h, R, pb, px, refine)
                if rc != 0:
                    raise RuntimeError(f"mfgpu_batch_solve -> {rc}")

            e2e_step()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                e2e_step()
            torch.cuda.synchronize()
            e2e_s = (time.perf_counter() - t0) / args.steps
            if world > 1:
                t = torch.tensor([e2e_s], device=dev)
                dist.all_reduce(t, op=dist.ReduceOp.MAX)
                e2e_s = float(t.item())
            e2e = {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 8 * (len(nz) + N * R),
                   "d2h_bytes_per_step": 8 * N * R}
        forms[form] = {"ms_per_step": ms, "refine": refine, "eta": eta, "analyze_s": t_an, "stats": st,
                       "clocks": clk, "launches_timed": launches, "e2e": e2e}
        del ctx
        torch.cuda.empty_cache()
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return 0
    ok = [k for k, f in forms.items() if f["eta"] is not None and f["eta"] <= TARGET_ETA]
    primary = min(ok or list(forms), key=lambda k: forms[k]["ms_per_step"])
    P = forms[primary]
    fp64_peak = fp_peak_tflops(torch, torch.float64, dev)
    roof = roofline_of(P, primary, fp64_peak, peaks)
    classes = {k: class_rooflines(f, k, fp64_peak, peaks, R) for k, f in forms.items()}
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        try:
            v, det = batch_cpu_baseline(sysl, costs)
            cpu = {"value": v, "unit": "s", "kind": "port", **det}
        except Exception as e:
            cpu = {"value": None, "error": str(e)}
    line = {
        "metric": BATCH_METRIC.format(count), "value": P["ms_per_step"] / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": P["ms_per_step"], "higher_is_better": False, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64" if primary == "fp64" else "f32+f64", "data": "synthetic",
        "form": primary, "config": config,
        "forms": {k: {"s_per_step": f["ms_per_step"] / 1e3, "refine": f["refine"], "bwd_err": f["eta"],
                      "factor_ms": f["stats"]["factor_ms"], "solve_ms": f["stats"]["solve_ms"],
                      "analyze_s": f["analyze_s"], "e2e_s": f["e2e"]["value"] if f["e2e"] else None,
                      "kernels_ms": {kk: round(vv["ms"], 3) for kk, vv in f["stats"]["kernels"].items()}}
                  for k, f in forms.items()},
        "roofline": roof, "roofline_classes": classes, "cpu_baseline": cpu, "e2e": P["e2e"],
        "gpu_launches": P["launches_timed"],
        "clocks": P["clocks"], "predicted_gflop": flops_total / 1e9, "cost_model_s": t_cost,
        "stats": {k: P["stats"].get(k) for k in ("n", "nsuper", "levels", "nnz_l", "nnz_u", "max_front", "flops",
                                                 "front_elems", "front_elems_full", "pool_elems", "lean",
                                                 "flops_inverse", "fronts", "merged", "flops_exec")},
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def batch_cpu_baseline(sysl, costs, refine: int | None = None, stride: int = 16):
    """The oracle on every `stride`-th system of the batch (numeric factor +
    solve(refine) of its 4 right-hand sides, all host threads for BLAS),
    scaled to the whole batch by predicted flops.  `refine` None: the fewest
    refinements that bring every sampled system to backward error <=
    TARGET_ETA (untimed search), then the timed pass with that count."""
    from oracle import oracle as O

    cores = os.cpu_count() or 1
    O.blas_threads(cores)
    idx = list(range(0, len(sysl), stride))
    facs = []
    for i in idx:
        A, B = sysl[i]
        Rs = O.row_scaling(A, O.SCALE_SUM)
        facs.append(O.PureLU(O.numeric(O.symbolic_mf(A), O.apply_row_scaling(A, Rs), check=False), Rs, A))
    if refine is None:
        for refine in range(MAX_REFINE + 1):
            worst = max(_oracle_eta(sysl[i][0], O.solve(F, sysl[i][1], refine=refine), sysl[i][1])
                        for i, F in zip(idx, facs))
            if worst <= TARGET_ETA:
                break
    del facs
    t = 0.0
    for i in idx:
        A, B = sysl[i]
        S = O.symbolic_mf(A)
        t0 = time.perf_counter()
        Rs = O.row_scaling(A, O.SCALE_SUM)
        Fo = O.numeric(S, O.apply_row_scaling(A, Rs), check=False)
        O.solve(O.PureLU(Fo, Rs, A), B, refine=refine)
        t += time.perf_counter() - t0
    scale = float(sum(costs)) / float(sum(costs[i] for i in idx))
    return t * scale, {"cores": cores, "refine": refine,
                       "sample": f"{len(idx)} of {len(sysl)} systems (every {stride}th): numeric factor + "
                                 f"solve(refine={refine}, the oracle's fewest refinements to backward error <= "
                                 f"{TARGET_ETA:g}) of 4 rhs, symbolic excluded; scaled x{scale:.2f} by predicted "
                                 f"flops"}


if __name__ == "__main__":
    sys.exit(main())
