#!/usr/bin/env python
"""Swift SpMM benchmark (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

A step is one product C = A B over the workload (default: the 1,048,576 x 1,048,576 R-MAT
matrix, a,b,c,d = .57,.19,.19,.05, 16,777,216 edge draws with duplicates merged, values
U[-1,1] FP32, B 1,048,576 x 128 FP32 U[-1,1]).  `value` is whole-job GFLOP/s (2 nnz N per
step, summed over ranks) with A, B and C resident in HBM; `e2e` is the same metric through the
library's public call with B copied in from pinned host memory and C copied back every step.
Several GPUs run independent replicas (the product has no exchange step).

--impl reference times the reference's own CPU product (Swift_cpu, compiled from the
reference sources under oracle/_ref; the oracle's restatement if that build is absent) on
the host cores: each step is one whole product of the same workload (or, where warm-up and
steps would not fit --ref-seconds, the next equal share of one, in the reference's order).

--mtx FILE [--n N] [--dtype f32|f64] runs the same product on a MatrixMarket file (the
reference's input format) instead of a synthetic matrix.

--impl reference-gpu (context, one GPU) runs the reference's own GPU SpMM wrappers, compiled
from its sources for sm_100a under oracle/_ref, on the same workload and times the library's
product beside them in the same process.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "swift-high-performance-sparse-dense-matrix-multiplication-on-gpus_b200")
sys.path[:0] = [PKG_DIR, os.path.join(ROOT, "oracle")]

import numpy as np  # noqa: E402

WORKLOADS = {
    # the scale workloads (R-MAT scale 20, avg degree 16)
    "rmat20_n128_f32": dict(kind="rmat", scale=20, edges=16 << 20, N=128, dtype="f32"),
    "rmat20_n32_f32": dict(kind="rmat", scale=20, edges=16 << 20, N=32, dtype="f32"),
    "rmat20_n128_f64": dict(kind="rmat", scale=20, edges=16 << 20, N=128, dtype="f64"),
    "rmat20_n32_f64": dict(kind="rmat", scale=20, edges=16 << 20, N=32, dtype="f64"),
    # half-size case for full ncu captures (B and C still exceed L2)
    "rmat19_n128_f32": dict(kind="rmat", scale=19, edges=8 << 20, N=128, dtype="f32"),
    # precision workload: R-MAT scale 19 avg degree 32 merged with a 64-wide band, 16-bit B/C
    "rmat19band_n128_bf16": dict(kind="rmatband", scale=19, edges=16 << 20, N=128, dtype="bf16"),
    "rmat19band_n128_f16": dict(kind="rmatband", scale=19, edges=16 << 20, N=128, dtype="f16"),
    "rmat19band_n128_f32": dict(kind="rmatband", scale=19, edges=16 << 20, N=128, dtype="f32"),
    # half-size banded case for full ncu captures of the band engine (B and C exceed L2)
    "rmat18band_n128_f32": dict(kind="rmatband", scale=18, edges=8 << 20, N=128, dtype="f32"),
    "rmat18band_n128_bf16": dict(kind="rmatband", scale=18, edges=8 << 20, N=128, dtype="bf16"),
    # precision ratios (FP32 vs BF16 vs FP16 B/C on one FP32-valued matrix)
    "precision_rmat19band_n128": dict(kind="precision", rk="rmatband", scale=19, edges=16 << 20, N=128),
    # differentiation: GNN layer on a symmetric-normalised R-MAT graph, fused vs plain
    "fwdbwd_rmat18sym_n64": dict(kind="fwdbwd", scale=18, edges=(32 << 18) // 2, N=64, dtype="f32"),
    # the batching workload: 512 independent products in one persistent launch
    "batch512_f32": dict(kind="batch", count=512, N=None, dtype="f32"),
    # standalone SDDMM (out[e] = U[row e] . V[col e]) at the dense widths of the reference's SDDMM
    # comparison scripts (32 and 128), on the scale matrix
    "sddmm_rmat20_n32_f32": dict(kind="sddmm", scale=20, edges=16 << 20, N=32, dtype="f32"),
    "sddmm_rmat20_n128_f32": dict(kind="sddmm", scale=20, edges=16 << 20, N=128, dtype="f32"),
    "sddmm_rmat19_n128_f32": dict(kind="sddmm", scale=19, edges=8 << 20, N=128, dtype="f32"),
    "sddmm_rmat19_n32_f32": dict(kind="sddmm", scale=19, edges=8 << 20, N=32, dtype="f32"),
    # the 4096 x 4096 parity workload (rows ~Poisson(16))
    "poisson4096_n32_f32": dict(kind="poisson", M=4096, K=4096, lam=16.0, N=32, dtype="f32"),
}
DEFAULT_WORKLOAD = "rmat20_n128_f32"
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def describe(name, wl, nnz):
    if wl["kind"] == "mtx":
        return (f"MatrixMarket file {os.path.basename(wl['path'])} read as the reference's reader reads it "
                f"({nnz} nnz), the file's values; B {wl['N']} columns U[-1,1] row-major; C = A*B {wl['dtype']}")
    if wl["kind"] in ("rmat", "sddmm"):
        M = 1 << wl["scale"]
        if wl["kind"] == "sddmm":
            return (f"SDDMM on R-MAT scale {wl['scale']} ({M}x{M}, {wl['edges']} edge draws, duplicates merged -> "
                    f"{nnz} nnz): out[e] = U[row e] . V[col e], U and V {M}x{wl['N']} U[-1,1] {wl['dtype']}")
        return (f"R-MAT scale {wl['scale']} ({M}x{M}, {wl['edges']} edge draws, a,b,c,d=.57,.19,.19,.05, "
                f"duplicates merged -> {nnz} nnz), values U[-1,1]; B {M}x{wl['N']} U[-1,1] row-major; "
                f"C = A*B {wl['dtype']}")
    if wl["kind"] == "rmatband":
        M = 1 << wl["scale"]
        return (f"R-MAT scale {wl['scale']} ({wl['edges']} draws) merged with |i-j|<32 band -> {nnz} nnz, "
                f"values U[-1,1] FP32; B {M}x{wl['N']} and C in {wl['dtype']}, FP32 accumulation")
    return (f"{wl['M']}x{wl['K']} rows ~Poisson({wl['lam']}), columns uniform without replacement -> "
            f"{nnz} nnz; B {wl['K']}x{wl['N']} U[-1,1]")


def data_desc(wl):
    if wl["kind"] == "mtx":
        return f"MatrixMarket file {os.path.basename(wl['path'])} (its pattern and values); B synthetic U[-1,1]"
    return "synthetic (seeded generator; the reference's SuiteSparse inputs are not available offline)"


def make_inputs(wl, device, seed=0):
    """Pattern and values (host numpy CSR) plus B on `device` (torch)."""
    import torch

    from swift_b200 import gen
    mtx_val = None
    if wl["kind"] == "mtx":
        from swift_b200.mtx import read_mtx
        mm = read_mtx(wl["path"], np.float64 if wl["dtype"] == "f64" else np.float32)
        M, K, rp, ci, mtx_val = mm.rows, mm.cols, mm.rowptr, mm.colidx, mm.val
    elif wl["kind"] in ("rmat", "sddmm"):
        rp, ci = gen.rmat(wl["scale"], wl["edges"], seed=seed, device=device)
        M = K = 1 << wl["scale"]
    elif wl["kind"] == "rmatband":
        rp, ci = gen.rmat_plus_band(wl["scale"], wl["edges"], 32, seed=seed, device=device)
        M = K = 1 << wl["scale"]
    else:
        M, K = wl["M"], wl["K"]
        rp, ci = gen.poisson_uniform(M, K, wl["lam"], seed=seed)
    nnz = int(rp[-1])
    g = torch.Generator(device=device)
    g.manual_seed(seed + 1)
    vdt = torch.float64 if wl["dtype"] == "f64" else torch.float32
    val = (torch.rand(nnz, generator=g, device=device, dtype=vdt) * 2 - 1)
    if mtx_val is not None:
        val = torch.from_numpy(mtx_val).to(device=device, dtype=vdt)
    g.manual_seed(seed + 2)
    if wl["dtype"] == "f64":
        B = torch.rand((K, wl["N"]), generator=g, device=device, dtype=torch.float64) * 2 - 1
    else:
        bdt = {"f32": torch.float32, "bf16": torch.bfloat16, "f16": torch.float16}[wl["dtype"]]
        B = (torch.rand((K, wl["N"]), generator=g, device=device, dtype=torch.float32) * 2 - 1).to(bdt)
    return M, K, rp, ci, val, B


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, gpu):
        self.gpu = gpu
        self.lines = []
        self.proc = None
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.gpu)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()
        time.sleep(0.15)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def stop(self, t0, t1):
        if self.proc is None:
            return None
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        inside = [ln for ts, ln in self.lines if t0 - 0.06 <= ts <= t1 + 0.06] or [ln for _, ln in self.lines]
        mhz, mx, reasons = [], None, set()
        for ln in inside:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                mhz.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(self.NAMES, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not mhz:
            return None
        return {"sm_mhz": statistics.median(mhz), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(mhz)}


def hbm_peak():
    try:
        with open(MEASURED_PEAKS) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def profile_summary(workload):
    """The committed ncu summary of this workload's top kernel: `key: value` lines of
    profiles/<kernel>_<workload>.txt (kernel, dram_bytes_per_launch, ...), or {}."""
    import glob
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", f"*_{workload}.txt"))):
        d = {}
        with open(path) as f:
            for line in f:
                if ":" in line and not line.startswith(" "):
                    k, v = line.split(":", 1)
                    d[k.strip()] = v.strip()
        if "dram_bytes_per_launch" in d and "kernel" in d and d.get("workload", "").split(" ")[0] == workload:
            d["file"] = os.path.relpath(path, ROOT)
            return d
    return {}


class _StdoutToStderr:
    """Routes C-level stdout to stderr (the reference's host code prints progress and
    diagnostic lines; stdout carries only the JSON line).

    One line is known to be spurious and is labelled as such on its way through: the
    reference's csr2csc prints "CSR 2 CSC error" whenever the last CSR value differs from
    the last CSC value (src/coo2csc.h:57-63), which is the normal case for any matrix whose
    last row and last column end in different nonzeros.  Every other line passes unchanged,
    so a real failure message still reads as one."""
    KNOWN = {"CSR 2 CSC error": "the reference's last-value comparison (src/coo2csc.h:57-63), "
                                "not a failure: its CSC is correct and is checked bit for bit"}

    def __enter__(self):
        import tempfile
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.tmp = tempfile.TemporaryFile(mode="w+b")
        os.dup2(self.tmp.fileno(), 1)

    def __exit__(self, *exc):
        import ctypes
        try:
            ctypes.CDLL(None).fflush(None)  # C stdio buffers of the reference code
        except Exception:
            pass
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        self.tmp.seek(0)
        for raw in self.tmp.read().decode(errors="replace").splitlines():
            note = self.KNOWN.get(raw.strip())
            sys.stderr.write(f"{raw}   [{note}]\n" if note else raw + "\n")
        sys.stderr.flush()
        self.tmp.close()


def cpu_swift(M, K, rp, ci, val_np, B_np, N, impl="ref"):
    """The reference's host pipeline (csr2csc, col_sort, formattransation, block_catgory,
    balance) and a Swift_cpu sampler over its format."""
    with _StdoutToStderr():
        return _cpu_swift(M, K, rp, ci, val_np, B_np, N, impl)


def _cpu_swift(M, K, rp, ci, val_np, B_np, N, impl):
    import oracle
    use = "ref" if (impl == "ref" and oracle.ref_available()) else "oracle"
    t0 = time.perf_counter()
    r, p, cnt, v = oracle.csr2csc(M, K, rp, ci, val_np, impl=use)
    t1 = time.perf_counter()
    pm = oracle.perm_stable(cnt)
    sr, sv, sn, sB = oracle.col_sort(K, N, cnt, pm, p, r, v, B=B_np, impl=use)
    t2 = time.perf_counter()
    del r, v
    sl = oracle.build(sr, sv, sn, M, K, impl=use, row_sort=False)
    t3 = time.perf_counter()
    cs = oracle.CpuSwift(sl, M, K, N, sB, impl=use)
    # the host preprocessing the reference runs before its SpMM, one thread (ms)
    cs.preprocessing_ms = {"csr_to_csc": (t1 - t0) * 1e3, "col_sort": (t2 - t1) * 1e3,
                           "formattransation+block_catgory+balance": (t3 - t2) * 1e3}
    return cs, use


def cpu_product(cs):
    """One whole Swift_cpu product (every regular tile and the reside part) into a zeroed C,
    as the reference's driver calls it on a freshly allocated result (src/main.cu:302).
    Returns (seconds, nonzeros)."""
    cs.C.fill(0)
    return cs.run(0, cs.tilenum, with_reside=True)


def run_cpu_products(cs, seconds):
    """Whole products repeated within `seconds` of CPU time (at least one; an untimed one
    first when three fit).  Returns (GFLOP/s, seconds timed, nonzeros, products timed)."""
    s0, n = cpu_product(cs)
    tot_s, prods = 0.0, 0
    if 3 * s0 > seconds:  # too slow for a warm-up: the first product is the sample
        tot_s, prods = s0, 1
    while prods == 0 or tot_s + tot_s / prods <= seconds:
        s, n = cpu_product(cs)
        tot_s += s
        prods += 1
    gf = 2.0 * n * prods * cs.N / tot_s / 1e9 if tot_s > 0 else 0.0
    return gf, tot_s, n * prods, prods


def oracle_call(name, *a):
    """One call of an oracle restatement (test-side C code, used here only as the CPU baseline)."""
    import oracle
    return getattr(oracle, name)(*a)


def cpu_port_line(fn, flops, seconds, what):
    """CPU baseline from an oracle restatement where the reference has no implementation: fn
    repeated within `seconds` (at least once), flops per call."""
    try:
        n, tot = 0, 0.0
        while n == 0 or tot + tot / n <= seconds:
            a = time.perf_counter()
            fn()
            tot += time.perf_counter() - a
            n += 1
        return {"value": flops * n / tot / 1e9, "unit": "GFLOP/s", "cores": 1, "kind": "port",
                "sample": f"{what}: {n} whole call(s) in {tot:.1f} s, one thread"}
    except Exception as ex:  # the baseline is reported, never required
        return {"value": None, "unit": "GFLOP/s", "cores": 1, "kind": "port", "sample": f"failed: {ex}"}


def cpu_baseline_line(cs, kind, seconds, what):
    gf, secs, snnz, prods = run_cpu_products(cs, seconds)
    return {"value": gf, "unit": "GFLOP/s", "cores": 1,
            "kind": "reference" if kind == "ref" else "port",
            "host_preprocessing_ms": getattr(cs, "preprocessing_ms", None),
            "sample": f"{what}: {prods} whole Swift_cpu product(s) of this workload ({snnz // max(prods, 1)} nonzeros "
                      f"x N={cs.N} each) in {secs:.1f} s; single-threaded by construction, as the reference is "
                      f"(host has {os.cpu_count()} threads)"}


# ------------------------------------------------------------------------------------ ours
def max_over_ranks(value, dist, device="cuda"):
    """The largest of every rank's value (a device time: the job takes as long as its slowest
    replica).  dist is torch.distributed or None (one process)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(work_per_rank, world, seconds):
    """Aggregate throughput of `world` replicas that each did `work_per_rank` in `seconds`."""
    return world * work_per_rank / seconds if seconds > 0 else 0.0


def _timed(fn, steps, warmup):
    """Device ms per call of fn (CUDA events on the current stream, after warm-up)."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _gpu_index(local):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    return vis.split(",")[local] if vis else local


def _timed_clocked(fn, steps, warmup, local=0):
    """As _timed, with nvidia-smi clocks and throttle reasons sampled over the timed region:
    returns (device ms per call, clocks record)."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    sampler = ClockSampler(_gpu_index(local))
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.time()
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop(w0, time.time())
    return e0.elapsed_time(e1) / steps, clocks


def merge_clocks(recs):
    """One clocks record over several timed regions: median of their medians, every reason."""
    recs = [r for r in recs if r]
    if not recs:
        return None
    return {"sm_mhz": statistics.median(r["sm_mhz"] for r in recs), "sm_max_mhz": recs[0]["sm_max_mhz"],
            "reasons": sorted(set().union(*[set(r["reasons"]) for r in recs])),
            "samples": sum(r["samples"] for r in recs), "regions": len(recs)}


def roofline_line(alg_bytes, ms, workload, default_kernel):
    """The roofline record of the line's dominant kernel: algorithmic bytes / device time
    against the measured copy bandwidth, and the DRAM traffic of the committed ncu summary."""
    peak, peak_kind = hbm_peak()
    achieved = alg_bytes / (ms / 1e3) / 1e9
    prof = profile_summary(workload)
    traffic = float(prof["dram_bytes_per_launch"].split()[0]) if prof else None
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "traffic_source": prof.get("file"), "kernel": prof.get("kernel", default_kernel),
            "peak_source": f"{peak_kind} ({'MEASURED_PEAKS.json hbm_gbs' if peak_kind == 'measured' else 'pool fallback'})",
            "algorithmic_bytes_per_launch": alg_bytes}


def _single_gpu_line(args, out):
    rank = int(os.environ.get("RANK", "0"))
    if rank == 0:
        print(json.dumps(out), flush=True)


def run_precision(args):
    """The precision workload: one FP32-valued plan, products with FP32, BF16 and FP16 B and C
    (FP32 accumulation); value = BF16 GFLOP/s; ratios against FP32 and errors against the
    deterministic FP64 product beside it."""
    import torch

    from swift_b200 import Plan
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    wl = WORKLOADS[args.workload]
    M, K, rp, ci, val, B32 = make_inputs(dict(wl, kind="rmatband", dtype="f32"), "cuda")
    N = wl["N"]
    nnz = int(rp[-1])
    plan = Plan.from_csr(torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), val, (M, K))
    ref = plan.spmm_f64_reference(B32.double())
    refmax = ref.abs().max().item()
    res = {}
    peak = hbm_peak()[0]
    for name, dt in (("f32", torch.float32), ("bf16", torch.bfloat16), ("f16", torch.float16)):
        B = B32.to(dt)
        C = torch.empty((M, N), dtype=dt, device="cuda")
        eng, _ = plan.autotune(B, C)
        rw = plan.rowwise_params(N, dt) if eng in ("rowwise", "band") else None
        ms, clk = _timed_clocked(lambda: plan.spmm(B, C), args.steps, args.warmup, local)
        plan.spmm(B, C)
        err = (C.double() - ref).abs().max().item() / refmax
        # error of the 16-bit result against the same product on 16-bit-rounded inputs in FP64
        err_in = None
        if dt != torch.float32:
            ref_q = plan.spmm_f64_reference(B.double())
            err_in = (C.double() - ref_q).abs().max().item() / ref_q.abs().max().item()
            del ref_q
        bytes_ = nnz * 8 + (K + M) * N * B.element_size()
        res[name] = {"ms": ms, "gflops": 2.0 * nnz * N / (ms / 1e3) / 1e9, "engine": eng,
                     "row_engine_params": rw, "err_vs_fp64": err, "err_vs_fp64_on_rounded_B": err_in,
                     "algorithmic_bytes": bytes_, "hbm_frac": bytes_ / (ms / 1e3) / 1e9 / peak, "clocks": clk}
    # 16-bit B and C with per-row power-of-two scales (swift_spmm_scaled): B rows stored as
    # B / b_scale with each row's maximum in [2^14, 2^15); error of c_scale * C against FP64
    m = B32.abs().amax(dim=1)
    bscale = torch.where(m > 0, torch.exp2(torch.floor(torch.log2(torch.where(m > 0, m, torch.ones_like(m)))) - 14),
                         torch.ones_like(m)).float().contiguous()
    for name, dt in (("bf16_scaled", torch.bfloat16), ("f16_scaled", torch.float16)):
        B = (B32 / bscale[:, None]).to(dt)
        C = torch.empty((M, N), dtype=dt, device="cuda")
        cs = torch.empty(M, dtype=torch.float32, device="cuda")
        ms, clk = _timed_clocked(lambda: plan.spmm_scaled(B, b_scale=bscale, C_out=C, c_scale=cs), args.steps,
                                 args.warmup, local)
        plan.spmm_scaled(B, b_scale=bscale, C_out=C, c_scale=cs)
        err = (C.double() * cs.double()[:, None] - ref).abs().max().item() / refmax
        bytes_ = nnz * 8 + (K + M) * (N * B.element_size() + 4)
        res[name] = {"ms": ms, "gflops": 2.0 * nnz * N / (ms / 1e3) / 1e9, "engine": "rowwise",
                     "err_vs_fp64": err, "algorithmic_bytes": bytes_,
                     "hbm_frac": bytes_ / (ms / 1e3) / 1e9 / peak, "clocks": clk}
    # the plain FP32 path: the row walk over all of A, whatever the autotuner picked above
    B = B32
    C = torch.empty((M, N), dtype=torch.float32, device="cuda")
    ms_rw, clk_rw = _timed_clocked(lambda: plan.spmm(B, C, engine="rowwise"), args.steps, args.warmup, local)
    plain_f32 = {"ms": ms_rw, "gflops": 2.0 * nnz * N / (ms_rw / 1e3) / 1e9, "engine": "rowwise", "clocks": clk_rw}
    del ref
    f32b, bfb = res["f32"]["algorithmic_bytes"], res["bf16"]["algorithmic_bytes"]
    # the band engine's own format: dense 8-row tiles (values only) + the rest as CSR
    hist, bw = plan.band_profile()
    band = None
    if bw >= 0:
        tw = (8 + 2 * bw + 3) // 4 * 4
        rows = np.repeat(np.arange(M, dtype=np.int64), np.diff(rp.astype(np.int64)))
        c0 = (rows & ~7) - bw
        cols = ci.astype(np.int64)
        rest_nnz = int(np.count_nonzero((cols < c0) | (cols >= c0 + tw)))
        del rows, c0, cols
        tile_bytes = ((M + 63) // 64) * 64 * tw * 4
        # 16-bit B runs the tiles on the tensor cores: 16-row windows of 8 + tw columns rounded up
        # to 16, each value as hi + lo parts of B's type (4 bytes), plus one FP32 row factor per row
        twm = (8 + tw + 15) // 16 * 16
        mma_bytes = ((M + 63) // 64) * 64 * (twm * 4 + 4)
        band = {"half_width": bw, "tile_width": tw, "tile_bytes": tile_bytes, "mma_window_width": twm,
                "mma_fragment_bytes": mma_bytes, "rest_nnz": rest_nnz, "in_tiles_nnz": nnz - rest_nnz}
        for name in ("f32", "bf16", "f16"):
            esz = 4 if name == "f32" else 2
            b = (tile_bytes if name == "f32" else mma_bytes) + rest_nnz * 8 + (K + M) * N * esz
            band[f"format_bytes_{name}"] = b
            if res[name]["engine"] == "band":
                res[name]["algorithmic_bytes_band_format"] = b
                res[name]["hbm_frac_band_format"] = b / (res[name]["ms"] / 1e3) / 1e9 / peak
        band["byte_ceiling_16bit_vs_f32"] = band["format_bytes_f32"] / band["format_bytes_bf16"]
    cpu = None
    if not args.no_cpu_baseline:
        try:  # the reference has no 16-bit path: its FP32 Swift_cpu on the same matrix and B
            cs_, kind = cpu_swift(M, K, rp, ci, val.cpu().numpy(), B32.cpu().numpy(), N, impl="ref")
            cpu = cpu_baseline_line(cs_, kind, args.cpu_seconds,
                                    "the reference's FP32 Swift_cpu (it has no BF16/FP16 path)")
            del cs_
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "GFLOP/s", "cores": 1, "kind": "reference", "sample": f"failed: {ex}"}
    out = {
        "metric": "spmm_gflops", "value": res["bf16"]["gflops"], "unit": "GFLOP/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["bf16"]["ms"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16 B/C, fp32 accumulate", "data": "synthetic",
        "config": {"workload": args.workload, "rows": M, "nnz_realised": nnz, "N": N,
                   "l2": "inputs larger than L2 (B and C exceed 126 MB in every precision); no flush between steps",
                   "description": describe(args.workload, dict(wl, kind="rmatband", dtype="bf16/f16/f32"), nnz)},
        "ratio_bf16_vs_f32": res["f32"]["ms"] / res["bf16"]["ms"],
        "ratio_f16_vs_f32": res["f32"]["ms"] / res["f16"]["ms"],
        "plain_f32_path": plain_f32,
        "ratio_bf16_vs_plain_f32_path": plain_f32["ms"] / res["bf16"]["ms"],
        "ratio_f16_vs_plain_f32_path": plain_f32["ms"] / res["f16"]["ms"],
        "ratios_note": ("ratio_*_vs_f32: against the autotuned FP32 product (the band engine on this matrix); "
                        "ratio_*_vs_plain_f32_path: against the FP32 row walk over all of A"),
        "byte_model_ceiling_16bit_vs_f32": f32b / bfb,
        "band_format": band,
        "roofline": roofline_line(res["bf16"].get("algorithmic_bytes_band_format", bfb), res["bf16"]["ms"],
                                  args.workload, "band_mma_kernel + merge_flag_kernel" if res["bf16"]["engine"] == "band"
                                  else "merge_flag_kernel"),
        "products": res,
        "gpu_launches": args.steps,
        "clocks": merge_clocks([r["clocks"] for r in res.values()] + [clk_rw]),
        "clocks_headline": res["bf16"]["clocks"],
        "cpu_baseline": cpu,
    }
    _single_gpu_line(args, out)


def run_sddmm(args):
    """Standalone SDDMM: out[e] = U[row e] . V[col e] for every nonzero e (the backward kernel
    for dA on its own).  value = 2 nnz N / time; bytes = nnz (index 4 + output s) + U once +
    V once; the vendor's CSR SDDMM (torch.sparse.sampled_addmm) is timed beside it."""
    import torch

    from swift_b200 import Plan
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    wl = WORKLOADS[args.workload]
    M, K, rp, ci, val, _ = make_inputs(wl, "cuda")
    N = wl["N"]
    nnz = int(rp[-1])
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    U = torch.rand((M, N), generator=g, device="cuda") * 2 - 1
    V = torch.rand((K, N), generator=g, device="cuda") * 2 - 1
    plan = Plan.from_csr(torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), val, (M, K))
    out = torch.empty(nnz, device="cuda")
    Un, Vn = (None, None) if args.no_cpu_baseline else (U.double().cpu().numpy(), V.double().cpu().numpy())
    ms, clocks = _timed_clocked(lambda: plan.sddmm(U, V, out), args.steps, args.warmup, local)
    flops = 2.0 * nnz * N
    alg_bytes = nnz * (4 + 4) + M * N * 4 + K * N * 4
    library = None
    try:
        A_t = torch.sparse_csr_tensor(torch.from_numpy(rp).cuda().long(), torch.from_numpy(ci).cuda().long(),
                                      torch.zeros(nnz, device="cuda"), size=(M, K))
        Vt = V.t()
        lib_ms = _timed(lambda: torch.sparse.sampled_addmm(A_t, U, Vt, beta=0.0, alpha=1.0), 5, 2)
        ref = torch.sparse.sampled_addmm(A_t, U, Vt, beta=0.0, alpha=1.0).values()
        diff = float((ref - out).abs().max() / ref.abs().max())
        library = {"what": "torch.sparse.sampled_addmm on a CSR tensor (cuSPARSE SDDMM)", "ms_per_step": lib_ms,
                   "gflops": flops / (lib_ms / 1e3) / 1e9, "max_rel_diff": diff}
        del A_t
    except Exception as ex:  # context row only
        library = {"what": "torch.sparse.sampled_addmm on a CSR tensor", "error": str(ex)[:200]}
    res = {
        "metric": "sddmm_gflops", "value": flops / (ms / 1e3) / 1e9, "unit": "GFLOP/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": data_desc(wl),
        "config": {"workload": args.workload, "description": describe(args.workload, wl, nnz), "rows": M,
                   "cols": K, "nnz": nnz, "N": N,
                   "l2": "inputs larger than L2 (U and V exceed 126 MB); no flush between steps"},
        "roofline": roofline_line(alg_bytes, ms, args.workload, "merge_bwd_kernel"),
        "gpu_launches": args.steps,
        "clocks": clocks,
        "cpu_baseline": None if args.no_cpu_baseline else cpu_port_line(
            lambda: oracle_call("sddmm_f64", M, K, rp, ci, Un, Vn), flops, args.cpu_seconds,
            "the oracle's FP64 SDDMM restatement (the reference has no SDDMM)"),
        "library_context": library,
    }
    _single_gpu_line(args, res)
    plan.close()


def run_fwdbwd(args):
    """The differentiation workload: Y = A X, dX = A^T dY, dA = SDDMM(dY, X) on a symmetric-
    normalised R-MAT graph; fused (one pass over A for Y and dA, then A^T) against the same
    three products run separately; value = fused GFLOP/s (3 x 2 nnz N per step)."""
    import torch

    from swift_b200 import Plan, gen
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    wl = WORKLOADS[args.workload]
    rp, ci = gen.rmat(wl["scale"], wl["edges"], seed=0, device="cuda", symmetric=True, self_loops=False)
    M = 1 << wl["scale"]
    N = wl["N"]
    nnz = int(rp[-1])
    vals = gen.sym_normalized_values(rp, ci, M, np.float32)
    plan = Plan.from_csr(torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), torch.from_numpy(vals).cuda(),
                         (M, M), build_transpose=True)
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    X = torch.randn((M, N), generator=g, device="cuda")
    dY = torch.randn((M, N), generator=g, device="cuda")
    Y = torch.empty_like(X)
    dX = torch.empty_like(X)
    dA = torch.empty(nnz, device="cuda")
    plan.autotune(X, Y)

    def plain():
        plan.spmm(X, Y)
        plan.spmm_t(dY, dX)
        plan.sddmm(dY, X, dA)

    def fused():
        plan.fused_forward_backward(X, dY, Y, dX, dA)

    clk = {}
    t_plain, clk["plain"] = _timed_clocked(plain, args.steps, args.warmup, local)
    symmetric = plan.is_symmetric()
    plan.set_symmetry(False)  # general path: Y and dA in one pass, dX over A^T
    t_fused_general, clk["fused_general"] = _timed_clocked(fused, args.steps, args.warmup, local)
    plan.set_symmetry(True)
    t_fused, clk["fused"] = _timed_clocked(fused, args.steps, args.warmup, local)
    t_fwd, clk["spmm"] = _timed_clocked(lambda: plan.spmm(X, Y), args.steps, args.warmup, local)
    t_bwd, clk["spmm_t"] = _timed_clocked(lambda: plan.spmm_t(dY, dX), args.steps, args.warmup, local)
    t_sddmm, clk["sddmm"] = _timed_clocked(lambda: plan.sddmm(dY, X, dA), args.steps, args.warmup, local)
    flops = 3 * 2.0 * nnz * N
    # fused pass over symmetric A: A once (value + index), X and dY read once, Y, dX and dA written once
    alg_bytes = nnz * (8 + 4) + 4 * M * N * 4
    cpu = None
    if not args.no_cpu_baseline:
        Xn, dYn = X.double().cpu().numpy(), dY.double().cpu().numpy()
        v64 = vals.astype(np.float64)

        def port():
            oracle_call("csr_spmm_f64", M, M, rp, ci, v64, Xn)
            oracle_call("csr_spmm_t_f64", M, M, rp, ci, v64, dYn)
            oracle_call("sddmm_f64", M, M, rp, ci, dYn, Xn)
        cpu = cpu_port_line(port, flops, args.cpu_seconds, "the oracle's FP64 restatements of Y = A X, "
                            "dX = A^T dY and dA = SDDMM(dY, X) (the reference has no backward pass)")
    out = {
        "metric": "spmm_gflops", "value": flops / (t_fused / 1e3) / 1e9, "unit": "GFLOP/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_fused, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": args.workload, "nodes": M, "nnz": nnz, "N": N,
                   "graph": f"R-MAT scale {wl['scale']} symmetrised, no self loops, values 1/sqrt(d_i d_j)"},
        "ratio_fused_vs_plain": t_plain / t_fused,
        "ratio_fused_general_vs_plain": t_plain / t_fused_general,
        "symmetric": symmetric,
        "ms": {"plain_fwd_bwd": t_plain, "fused_fwd_bwd": t_fused, "fused_fwd_bwd_general": t_fused_general,
               "spmm": t_fwd, "spmm_transposed": t_bwd, "sddmm": t_sddmm},
        "paths": {"plain": "swift_spmm + swift_spmm_transposed + swift_sddmm, each its own pass",
                  "fused": "one pass over A for Y, dX (A symmetric: dX = A dY) and dA",
                  "fused_general": "one pass over A for Y and dA, one over A^T for dX"},
        "roofline": roofline_line(alg_bytes, t_fused, args.workload, "merge_bwd_kernel"),
        "gpu_launches": args.steps,
        "clocks": merge_clocks(list(clk.values())),
        "clocks_by_region": clk,
        "cpu_baseline": cpu,
    }
    _single_gpu_line(args, out)


def run_batch(args):
    """The batching workload: 512 independent products in one persistent launch, replayed as
    a CUDA graph; value = the batch's total GFLOP/s."""
    import torch

    from swift_b200 import Batch, Plan, gen
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    wl = WORKLOADS[args.workload]
    mats = gen.batch_matrices(wl["count"], seed=0, device="cuda")
    g = torch.Generator(device="cuda")
    g.manual_seed(1)
    plans = []
    flops = alg_bytes = 0
    nnz_tot = rows_tot = 0
    # every member's B (and C) is a view into one flat buffer, so that a step's inputs and
    # results cross PCIe as one copy each way
    offs = [int(x) for x in np.cumsum([0] + [m["M"] * m["N"] for m in mats])]
    Bflat = torch.rand(int(offs[-1]), generator=g, device="cuda") * 2 - 1
    Cflat = torch.empty(int(offs[-1]), device="cuda")
    Bs = [Bflat[offs[i]:offs[i + 1]].view(m["M"], m["N"]) for i, m in enumerate(mats)]
    Cs = [Cflat[offs[i]:offs[i + 1]].view(m["M"], m["N"]) for i, m in enumerate(mats)]
    for i, m in enumerate(mats):
        M, N = m["M"], m["N"]
        nnz = int(m["rowptr"][-1])
        val = torch.rand(nnz, generator=g, device="cuda") * 2 - 1
        plans.append(Plan.from_csr(torch.from_numpy(m["rowptr"]).cuda(), torch.from_numpy(m["colidx"]).cuda(),
                                   val, (M, M)))
        flops += 2.0 * nnz * N
        alg_bytes += nnz * 8 + 2 * M * N * 4
        nnz_tot += nnz
        rows_tot += M
    batch = Batch(plans)
    batch.set_operands(Bs, Cs)
    torch.cuda.synchronize()
    tw0 = time.perf_counter()
    best_U, tune_ms = batch.autotune()
    torch.cuda.synchronize()
    tune_wall_ms = (time.perf_counter() - tw0) * 1e3
    for _ in range(args.warmup):
        batch.run_graph()
    stream = torch.cuda.current_stream()
    gpu_idx = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[local] if os.environ.get("CUDA_VISIBLE_DEVICES") else local
    sampler = ClockSampler(gpu_idx)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.time()
    e0.record(stream)
    for _ in range(args.steps):
        batch.run_graph()
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop(w0, time.time())
    ms = e0.elapsed_time(e1)
    ms = max_over_ranks(ms, dist)
    ms_step = ms / args.steps
    value = whole_job_rate(flops * args.steps, world, ms / 1e3) / 1e9
    # end to end: every member's B in from pinned host memory, every C out.  Copies in, the
    # batch and copies out run on three streams over two operand sets (a second batch object
    # over the same plans), so one step's C leaves while the next step's B arrives.
    Bflat2, Cflat2 = torch.empty_like(Bflat), torch.empty_like(Cflat)
    batch2 = Batch(plans)
    batch2.set_operands([Bflat2[offs[i]:offs[i + 1]].view(m["M"], m["N"]) for i, m in enumerate(mats)],
                        [Cflat2[offs[i]:offs[i + 1]].view(m["M"], m["N"]) for i, m in enumerate(mats)])
    batch2.autotune()
    sets = [(batch, Bflat, Cflat), (batch2, Bflat2, Cflat2)]
    Bh = Bflat.cpu().pin_memory()
    Ch = [torch.empty(Cflat.shape, dtype=Cflat.dtype).pin_memory() for _ in range(2)]
    h2d = Bh.numel() * 4
    d2h = Ch[0].numel() * 4
    n_e2e = max(2, min(args.e2e_steps, 4))
    s_in, s_c, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_c = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]

    def e2e_batch_steps(n):
        for i in range(n):
            j = i % 2
            bj, Bd, Cd = sets[j]
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(ev_c[j])  # operand set j free once its batch ran
                Bd.copy_(Bh, non_blocking=True)
                ev_in[j].record(s_in)
            s_c.wait_event(ev_in[j])
            if i >= 2:
                s_c.wait_event(ev_out[j])  # its C copied out
            bj.run_graph(stream=s_c)
            ev_c[j].record(s_c)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_c[j])
                Ch[j].copy_(Cd, non_blocking=True)
                ev_out[j].record(s_out)

    torch.cuda.synchronize()
    e2e_batch_steps(2)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(s_in)
    s_c.wait_event(t0)
    s_out.wait_event(t0)
    e2e_batch_steps(n_e2e)
    s_out.wait_stream(s_in)
    s_out.wait_stream(s_c)
    t1.record(s_out)
    torch.cuda.synchronize()
    e2e_ms = t0.elapsed_time(t1)
    e2e_ms = max_over_ranks(e2e_ms, dist)
    batch2.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            gf, secs, done, kind = cpu_batch_products(mats, args.cpu_seconds)
            cpu = {"value": gf, "unit": "GFLOP/s", "cores": 1, "kind": "reference" if kind == "ref" else "port",
                   "sample": f"the reference's Swift_cpu over whole products of the first {done} of {len(mats)} "
                             f"members in {secs:.1f} s (single-threaded by construction, as the reference is)"}
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "GFLOP/s", "cores": 1, "kind": "reference", "sample": f"failed: {ex}"}
    Ns = [m["N"] for m in mats]
    out = {
        "metric": "spmm_gflops", "value": value, "unit": "GFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded generator; 512 square matrices, M log-uniform in [1024, 65536], "
                "average degree U[4, 64], half uniform-random and half R-MAT; N from {32, 64, 128})",
        "config": {"workload": args.workload, "matrices": len(mats), "rows": rows_tot, "nnz": nnz_tot,
                   "N_counts": {str(n): Ns.count(n) for n in (32, 64, 128)}, "task_size": best_U,
                   "task_sizes_by_class": dict(zip(("N<=32", "N<=64", "N>64"), batch.task_sizes())),
                   "n_split_by_class": dict(zip(("N<=32", "N<=64", "N>64"), batch.n_split())),
                   "autotune_wall_ms": tune_wall_ms, "autotune_best_candidate_ms": tune_ms,
                   "launch": "one persistent kernel per step, replayed as a CUDA graph",
                   "l2": "B and C of the batch (about 5 GB) exceed L2; no flush between steps",
                   "parallelism": f"replicas x{world} (no exchange step)"},
        "roofline": roofline_line(alg_bytes, ms_step, args.workload, "merge_batch_kernel"),
        "e2e": {"value": world * flops * n_e2e / (e2e_ms / 1e3) / 1e9, "unit": "GFLOP/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": n_e2e,
                "ms_per_step": e2e_ms / n_e2e,
                "pipeline": "one H2D / the batch / one D2H per step on three streams, two operand sets"},
        "gpu_launches": args.steps,
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    print(json.dumps(out), flush=True)
    batch.close()


def run_block_histogram(args):
    """Block-density histograms of the workload's matrix, measured on the GPU: for each block
    shape, occupied blocks and their nonzeros per fill bin (bin k: fill in (2^-(k+1), 2^-k],
    the last bin sparser), in A's own column order and in the plan's sorted column order."""
    import torch

    from swift_b200 import Plan
    wl = dict(WORKLOADS[args.workload])
    if wl["kind"] == "precision":
        wl = dict(wl, kind=wl["rk"], dtype="f32")
    if wl["kind"] not in ("rmat", "rmatband", "poisson", "mtx"):
        raise SystemExit(f"--block-histogram: workload kind {wl['kind']} has no single matrix")
    M, K, rp, ci, val, _ = make_inputs(wl, "cuda")
    plan = Plan.from_csr(torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), val, (M, K))
    nbins = 8
    out = {"workload": args.workload, "rows": M, "cols": K, "nnz": int(rp[-1]),
           "bins": [f"({2.0 ** -(k + 1):g}, {2.0 ** -k:g}]" for k in range(nbins - 1)] + [f"<= {2.0 ** -(nbins - 1):g}"],
           "histograms": []}
    for shape in args.block_histogram.split(","):
        bh, bw = (int(x) for x in shape.lower().split("x"))
        for sorted_cols in (False, True):
            blocks, nnz = plan.block_histogram(bh, bw, sorted_columns=sorted_cols, nbins=nbins)
            out["histograms"].append({"block": f"{bh}x{bw}", "columns": "sorted" if sorted_cols else "original",
                                      "blocks": blocks.tolist(), "nnz": nnz.tolist(),
                                      "nnz_share": (nnz / max(1, nnz.sum())).round(4).tolist()})
    hist, bw_ = plan.band_profile()
    out["band_half_width"] = bw_
    out["nnz_within_distance"] = {str(d): int(hist[: d + 1].sum()) for d in (0, 3, 7, 15, 31, 63, 128)}
    print(json.dumps(out), flush=True)
    plan.close()


def run_ours(args):
    import torch

    from swift_b200 import Plan
    kind = WORKLOADS[args.workload]["kind"]
    if kind == "batch":
        return run_batch(args)
    if kind == "precision":
        return run_precision(args)
    if kind == "fwdbwd":
        return run_fwdbwd(args)
    if kind == "sddmm":
        return run_sddmm(args)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    wl = WORKLOADS[args.workload]
    N = wl["N"]
    M, K, rp, ci, val, B = make_inputs(wl, "cuda")
    nnz = int(rp[-1])
    d_rp = torch.from_numpy(rp).cuda()
    d_ci = torch.from_numpy(ci).cuda()
    plan = Plan.from_csr(d_rp, d_ci, val, (M, K))
    C = torch.empty((M, N), dtype=B.dtype, device="cuda")
    if args.rowwise_params:  # with --engine band they set the band engine's rest walk
        U, unr, vb, kern = (int(x) for x in args.rowwise_params.split(","))
        plan.set_rowwise_params(U, unr, vb, kern)
        engine, tune_ms, tune_wall_ms = ("band" if args.engine == "band" else "rowwise"), None, 0.0
    elif args.engine != "auto":  # a pinned engine (profiling): no autotuning
        engine, tune_ms, tune_wall_ms = args.engine, None, 0.0
    else:
        torch.cuda.synchronize()
        tw0 = time.perf_counter()
        engine, tune_ms = plan.autotune(B, C)
        torch.cuda.synchronize()
        tune_wall_ms = (time.perf_counter() - tw0) * 1e3
    rw_params = plan.rowwise_params(N, B.dtype) if engine == "rowwise" else None
    st = plan.stats()
    stream = torch.cuda.current_stream()
    run_engine = args.engine if (not args.rowwise_params or args.engine == "band") else "auto"
    for _ in range(args.warmup):
        plan.spmm(B, C, engine=run_engine)
    gpu_idx = os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",")[local] if os.environ.get("CUDA_VISIBLE_DEVICES") else local
    sampler = ClockSampler(gpu_idx)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    w0 = time.time()
    e0.record(stream)
    for _ in range(args.steps):
        plan.spmm(B, C, engine=run_engine)
    e1.record(stream)
    torch.cuda.synchronize()
    w1 = time.time()
    clocks = sampler.stop(w0, w1)
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    ms = max_over_ranks(ms, dist)
    ms_step = ms / args.steps
    flops = 2.0 * nnz * N
    value = whole_job_rate(flops * args.steps, world, ms / 1e3) / 1e9
    esz = B.element_size()
    vsz = 8 if val.dtype == torch.float64 else 4
    alg_bytes = nnz * (vsz + 4) + K * N * esz + M * N * esz
    peak, peak_kind = hbm_peak()
    achieved = alg_bytes / (ms_step / 1e3) / 1e9
    prof = profile_summary(args.workload)
    kernel = prof.get("kernel", "merge engine" if engine == "rowwise" else "tiled_rowmajor_kernel")
    traffic = float(prof["dram_bytes_per_launch"].split()[0]) if prof else None

    # the Swift tiled engine on the same inputs (reported beside the chosen engine)
    tiled = None
    if B.dtype in (torch.float32, torch.float64):
        for _ in range(2):
            plan.spmm(B, C, engine="tiled")
        n_t = 5
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(n_t):
            plan.spmm(B, C, engine="tiled")
        e1.record(stream)
        torch.cuda.synchronize()
        t_ms = e0.elapsed_time(e1) / n_t
        tiled = {"gflops": flops / (t_ms / 1e3) / 1e9, "ms_per_step": t_ms,
                 "hbm_frac_of_measured": alg_bytes / (t_ms / 1e3) / 1e9 / peak}
        plan.spmm(B, C, engine=run_engine)

    # the gather ceiling of row-ordered products on this matrix: a kernel that only gathers the
    # B rows of A's column stream (swift_gather_bound), and the same with L1-resident rows
    gather = None
    if B.dtype == torch.float32 and N in (32, 64, 128) and K >= 256:
        g_ms, g_l1, _ = plan.gather_bound(B, reps=10)
        gbytes = nnz * N * 4
        gather = {"what": "B rows gathered along A's column stream only (no values, no C)",
                  "gather_bytes_per_launch": gbytes, "ms_column_stream": g_ms, "ms_l1_resident": g_l1,
                  "tb_s_column_stream": gbytes / (g_ms / 1e3) / 1e12, "tb_s_l1_resident": gbytes / (g_l1 / 1e3) / 1e12,
                  "product_time_over_gather_time": ms_step / g_ms}
        plan.spmm(B, C, engine=run_engine)

    # context only: the vendor library's CSR SpMM (torch.sparse -> cuSPARSE) on the same inputs
    library = None
    try:
        A_t = torch.sparse_csr_tensor(torch.from_numpy(rp).cuda().long(), torch.from_numpy(ci).cuda().long(),
                                      val, size=(M, K))
        Bl = B if B.dtype == val.dtype else B.to(val.dtype)
        lib_ms = _timed(lambda: torch.sparse.mm(A_t, Bl), 5, 2)
        library = {"what": "torch.sparse.mm on a CSR tensor (cuSPARSE SpMM)", "ms_per_step": lib_ms,
                   "gflops": flops / (lib_ms / 1e3) / 1e9}
        del A_t
    except Exception as ex:  # context row only
        library = {"what": "torch.sparse.mm on a CSR tensor", "error": str(ex)[:200]}

    # end to end through the public call: every step copies its B in from pinned host memory
    # and its C out to pinned host memory.  Copies in, products and copies out run on three
    # streams over two device buffer sets, so step i's C leaves while step i+1's B arrives
    # (PCIe is full duplex); the products stay ordered on one stream (one plan).
    Bh = [B.cpu().pin_memory() for _ in range(2)]
    Ch = [torch.empty((M, N), dtype=C.dtype).pin_memory() for _ in range(2)]
    Bd = [B, torch.empty_like(B)]
    Cd = [C, torch.empty_like(C)]
    s_in, s_c, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_c = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]

    def e2e_steps(n):
        for i in range(n):
            j = i % 2
            with torch.cuda.stream(s_in):
                if i >= 2:
                    s_in.wait_event(ev_c[j])  # Bd[j] free once its product ran
                Bd[j].copy_(Bh[j], non_blocking=True)
                ev_in[j].record(s_in)
            s_c.wait_event(ev_in[j])
            if i >= 2:
                s_c.wait_event(ev_out[j])  # Cd[j] free once it was copied out
            plan.spmm(Bd[j], Cd[j], engine=run_engine, stream=s_c)
            ev_c[j].record(s_c)
            with torch.cuda.stream(s_out):
                s_out.wait_event(ev_c[j])
                Ch[j].copy_(Cd[j], non_blocking=True)
                ev_out[j].record(s_out)

    torch.cuda.synchronize()
    e2e_steps(2)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(s_in)
    s_c.wait_event(t0)
    s_out.wait_event(t0)
    e2e_steps(args.e2e_steps)
    s_out.wait_stream(s_in)
    s_out.wait_stream(s_c)
    t1.record(s_out)
    torch.cuda.synchronize()
    e2e_ms = t0.elapsed_time(t1)
    e2e_ms = max_over_ranks(e2e_ms, dist)
    e2e_value = world * flops * args.e2e_steps / (e2e_ms / 1e3) / 1e9
    # the copy bound of that loop: one step's B in and C out on the same two streams, no product
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    c0.record(s_in)
    s_out.wait_event(c0)
    for i in range(2):
        with torch.cuda.stream(s_in):
            Bd[i % 2].copy_(Bh[i % 2], non_blocking=True)
        with torch.cuda.stream(s_out):
            Ch[i % 2].copy_(Cd[i % 2], non_blocking=True)
    s_out.wait_stream(s_in)
    c1.record(s_out)
    torch.cuda.synchronize()
    copy_ms = c0.elapsed_time(c1) / 2

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cs, kind = cpu_swift(M, K, rp, ci, val.cpu().numpy(),
                                 B.float().cpu().numpy() if B.dtype in (torch.bfloat16, torch.float16) else B.cpu().numpy(),
                                 N, impl="ref")
            cpu = cpu_baseline_line(cs, kind, args.cpu_seconds, "the reference's Swift_cpu (oracle/_ref)")
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "GFLOP/s", "cores": 1, "kind": "reference", "sample": f"failed: {ex}"}

    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    dtype = wl["dtype"]
    out = {
        "metric": "spmm_gflops", "value": value, "unit": "GFLOP/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
        "data": data_desc(wl),
        "config": {"workload": args.workload, "description": describe(args.workload, wl, nnz),
                   "rows": M, "cols": K, "nnz": nnz, "N": N, "engine": engine,
                   "row_engine_params": rw_params,
                   "parallelism": f"replicas x{world} (no exchange step)",
                   "l2": "inputs larger than L2 (B and C exceed 126 MB); no flush between steps",
                   "plan_build_ms": st["build_ms"], "autotune_wall_ms": tune_wall_ms,
                   "autotune_best_candidate_ms": tune_ms,
                   "format": {k: st[k] for k in ("nsteps", "tilenum", "reside_col", "reside_nnz", "numblk",
                                                  "fmt_count", "long_rows", "long_pieces", "max_row_nnz")}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": f"{peak_kind} ({'MEASURED_PEAKS.json hbm_gbs' if peak_kind == 'measured' else 'pool fallback'})",
                     "kernel": kernel, "algorithmic_bytes_per_launch": alg_bytes,
                     "traffic_source": prof.get("file"),
                     "frac_of_8TBs_nominal": achieved / 8000.0},
        "e2e": {"value": e2e_value, "unit": "GFLOP/s",
                "h2d_bytes_per_step": int(Bh[0].numel() * Bh[0].element_size()),
                "d2h_bytes_per_step": int(Ch[0].numel() * Ch[0].element_size()), "steps": args.e2e_steps,
                "ms_per_step": e2e_ms / args.e2e_steps,
                "pipeline": "H2D / product / D2H on three streams, two buffer sets",
                "copy_bound_ms_per_step": copy_ms,
                "frac_of_copy_bound": copy_ms / (e2e_ms / args.e2e_steps)},
        "gpu_launches": args.steps * (1 if engine == "rowwise" else 2),
        "clocks": clocks,
        "cpu_baseline": cpu,
        "tiled_engine": tiled,
        "gather_bound": gather,
        "library_context": library,
    }
    print(json.dumps(out), flush=True)
    plan.close()


# ------------------------------------------------------------------------------------ reference
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    wl = WORKLOADS[args.workload]
    N = wl["N"]
    try:
        import torch
        dev = "cuda" if torch.cuda.is_available() else "cpu"
    except Exception:
        dev = "cpu"
    if wl["kind"] == "batch":
        return run_reference_batch(args, wl, dev)
    if wl["kind"] in ("sddmm", "fwdbwd"):
        print(json.dumps({"impl": "reference", "unavailable": f"the reference has no CPU path for the "
                          f"{wl['kind']} workload (SpMM only)"}), flush=True)
        return
    note = None
    if wl["kind"] == "precision":
        # the reference has no 16-bit operands: its FP32 Swift_cpu on the same matrix and B
        wl = dict(wl, kind=wl["rk"], dtype="f32")
        note = "the reference has no BF16/FP16 path; this is its FP32 Swift_cpu on the same matrix and B"
    M, K, rp, ci, val, B = make_inputs(wl, dev)
    import torch
    Bn = B.float().cpu().numpy() if B.dtype in (torch.bfloat16, torch.float16) else B.cpu().numpy()
    vn = val.cpu().numpy()
    nnz = int(rp[-1])
    cs, kind = cpu_swift(M, K, rp, ci, vn, Bn, N, impl="ref")
    del Bn
    T = cs.tilenum
    # a step is one whole product when warm-up + steps fit the time budget; otherwise each
    # step is the next of S equal shares of the tiles (the reside part with the last share),
    # so that S consecutive steps make one whole product in the reference's own order
    t_prod, _ = cpu_product(cs)
    S = 1
    while S < max(T, 1) and (args.steps + args.warmup) * t_prod / S > float(args.ref_seconds):
        S *= 2
    j = 0

    def step():
        nonlocal j
        if j == 0:
            cs.C.fill(0)
        t0, t1 = j * T // S, (j + 1) * T // S
        r = cs.run(t0, t1, with_reside=(j == S - 1))
        j = (j + 1) % S
        return r

    for _ in range(args.warmup):
        step()
    tot_s, tot_nnz = 0.0, 0
    for _ in range(args.steps):
        sec, n = step()
        tot_s += sec
        tot_nnz += n
    value = 2.0 * tot_nnz * N / tot_s / 1e9 if tot_s > 0 else 0.0
    if S == 1:
        sample = (f"each step: one whole Swift_cpu product of this workload ({nnz} nonzeros x N={N}) into a zeroed C; "
                  f"{args.steps} products in {tot_s:.2f} s")
    else:
        sample = (f"each step: the next 1/{S} of the tiles of one whole Swift_cpu product in the reference's order "
                  f"({S} steps make a product of {nnz} nonzeros x N={N}; a whole product takes {t_prod:.2f} s); "
                  f"{tot_nnz} nonzeros in {tot_s:.2f} s over {args.steps} steps")
    if note:
        sample += f"; {note}"
    out = {
        "metric": "spmm_gflops", "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tot_s * 1e3 / max(1, args.steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": wl["dtype"], "impl": "reference",
        "data": data_desc(wl),
        "config": {"workload": args.workload, "description": describe(args.workload, wl, nnz), "rows": M,
                   "cols": K, "nnz": nnz, "N": N, "parallelism": "host CPU, rank 0 only"},
        "cpu_baseline": {"value": value, "unit": "GFLOP/s", "cores": 1,
                         "kind": "reference" if kind == "ref" else "port", "sample": sample,
                         "host_preprocessing_ms": cs.preprocessing_ms},
        "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def cpu_batch_products(mats, seconds):
    """The reference's Swift_cpu over the batch members in order (whole products, each into a
    zeroed C), until `seconds` of CPU time; returns (GFLOP/s, seconds, members done, kind)."""
    rng = np.random.default_rng(1)
    tot_s = tot_f = 0.0
    done = 0
    kind = "ref"
    for m in mats:
        M, N = m["M"], m["N"]
        nnz = int(m["rowptr"][-1])
        val = rng.uniform(-1, 1, nnz).astype(np.float32)
        B = rng.uniform(-1, 1, (M, N)).astype(np.float32)
        cs, kind = cpu_swift(M, M, m["rowptr"], m["colidx"], val, B, N, impl="ref")
        sec, n = cpu_product(cs)
        tot_s += sec
        tot_f += 2.0 * n * N
        done += 1
        if tot_s >= seconds:
            break
    return (tot_f / tot_s / 1e9 if tot_s > 0 else 0.0), tot_s, done, kind


def run_reference_batch(args, wl, dev):
    """The reference's Swift_cpu over the batch members in order (whole products), until the
    time budget is spent; value = flops of the products run / their time."""
    from swift_b200 import gen
    world = int(os.environ.get("WORLD_SIZE", "1"))
    mats = gen.batch_matrices(wl["count"], seed=0, device=dev)
    value, tot_s, done, kind = cpu_batch_products(mats, args.ref_seconds)
    sample = f"Swift_cpu over whole products of the first {done} of {len(mats)} matrices in {tot_s:.2f} s"
    out = {
        "metric": "spmm_gflops", "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": done,
        "warmup": 0, "ms_per_step": tot_s * 1e3 / max(1, done), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "impl": "reference", "data": "synthetic (seeded generator)",
        "config": {"workload": args.workload, "matrices": len(mats), "parallelism": "host CPU, rank 0 only"},
        "cpu_baseline": {"value": value, "unit": "GFLOP/s", "cores": 1,
                         "kind": "reference" if kind == "ref" else "port", "sample": sample},
        "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def run_reference_gpu(args):
    """Context: the reference's own GPU SpMM wrappers (Swift_GPU, Swift_gpu1, Swift_gpu2,
    Swift_GPU_3, Swift_GPU_4; oracle/_ref/libswiftrefgpu_*.so, compiled from its sources for
    sm_100a) on this workload, fed the format the reference's own host preprocessing builds.
    Each wrapper times its kernels with its own CUDA events; `value` is the best variant, as
    the reference's result_check keeps the best of its variants (src/auxiliary.h:28-50).  The
    library's autotuned product on the same inputs is timed in the same process beside it."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch

    import oracle
    from swift_b200 import Plan
    wl = WORKLOADS[args.workload]
    if wl["kind"] not in ("rmat", "rmatband", "poisson", "mtx") or wl["dtype"] not in ("f32", "f64"):
        print(json.dumps({"impl": "reference_gpu", "unavailable": "the reference's GPU wrappers take FP32 or "
                          "FP64 B and C of one matrix; this workload is not one"}), flush=True)
        return
    if not oracle.ref_gpu_available():
        print(json.dumps({"impl": "reference_gpu", "unavailable": "oracle/_ref/libswiftrefgpu_*.so not built "
                          "(needs the reference checkout at build time)"}), flush=True)
        return
    torch.cuda.set_device(0)
    N = wl["N"]
    M, K, rp, ci, val, B = make_inputs(wl, "cuda")
    nnz = int(rp[-1])
    flops = 2.0 * nnz * N
    vn, Bn = val.cpu().numpy(), B.cpu().numpy()
    # the library on the same inputs: autotuned product, CUDA events over `steps` launches
    plan = Plan.from_csr(torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(), val, (M, K))
    C = torch.empty((M, N), dtype=B.dtype, device="cuda")
    engine, _ = plan.autotune(B, C)
    lib_ms, lib_clocks = _timed_clocked(lambda: plan.spmm(B, C), max(5, min(args.steps, 200)), args.warmup)
    plan.spmm(B, C)
    golden = C.cpu().numpy()
    plan.close()
    del C
    torch.cuda.empty_cache()
    t0 = time.time()
    with _StdoutToStderr():
        r, p, cnt, v = oracle.csr2csc(M, K, rp, ci, vn, impl="ref")
        sr, sv, sn, sB = oracle.col_sort(K, N, cnt, oracle.perm_stable(cnt), p, r, v, B=Bn, impl="ref")
        del r, v
        sl = oracle.build(sr, sv, sn, M, K, impl="ref", row_sort=True, N=N)
    prep_s = time.time() - t0
    fmt = dict(sl.arrays, tilenum=sl.tilenum, regular_nnz=sl.regular_nnz, reside_col=sl.reside_col,
               reside_nnz=sl.reside_nnz, segsum=sl.segsum, numblk=sl.numblk)
    fmt4 = dict(fmt, sortrowidx=sl.arrays["rowsorted_rowidx"])
    reps = max(1, min(args.steps, 5))
    variants = {}
    sampler = ClockSampler(_gpu_index(0))
    sampler.start()
    w0 = time.time()
    for var, name in oracle.REF_GPU_VARIANTS.items():
        f = fmt4 if var == 4 else fmt
        if not oracle.ref_gpu_accepts(var, f, N, sB.dtype):
            variants[name] = {"status": "not run: outside the inputs whose launches stay in bounds "
                                        "(oracle/ref_gpu.cu)"}
            continue
        times, st, Cr = [], 0, None
        with _StdoutToStderr():
            for i in range(1 + reps):  # the first call warms up
                st, ms, Cr = oracle.ref_gpu_spmm(var, f, M, K, N, nnz, sB, golden)
                if st != oracle.REF_GPU_OK:
                    break
                if i:
                    times.append(ms)
        if st != oracle.REF_GPU_OK:
            variants[name] = {"status": {1: "reference check failed", 2: "refused",
                                         3: "CUDA error"}.get(st, str(st))}
            continue
        ms = statistics.median(times)
        diff = float(np.abs(np.asarray(Cr, np.float64) - golden).max() / max(np.abs(golden).max(), 1e-300))
        variants[name] = {"status": "ok (reference check passed)", "ms": ms, "gflops": flops / (ms / 1e3) / 1e9,
                          "max_rel_diff_vs_library": diff}
    ref_clocks = sampler.stop(w0, time.time())
    ok = [x for x in variants.values() if "ms" in x]
    best = min(ok, key=lambda x: x["ms"]) if ok else None
    out = {
        "metric": "spmm_gflops", "value": best["gflops"] if best else None, "unit": "GFLOP/s",
        "impl": "reference_gpu", "n_gpus": 1, "steps": reps, "warmup": 1,
        "ms_per_step": best["ms"] if best else None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": wl["dtype"],
        "data": data_desc(wl),
        "config": {"workload": args.workload, "description": describe(args.workload, wl, nnz), "rows": M,
                   "cols": K, "nnz": nnz, "N": N, "reference_host_preprocessing_s": prep_s},
        "timing": "each wrapper's own CUDA events around its kernels; uploads, downloads and its host-side "
                  "check outside; median of the calls after the first",
        "variants": variants,
        "library": {"engine": engine, "ms": lib_ms, "gflops": flops / (lib_ms / 1e3) / 1e9,
                    "speedup_vs_best_reference_kernel": (best["ms"] / lib_ms) if best else None,
                    "clocks": lib_clocks},
        "clocks": ref_clocks,
    }
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference", "reference-gpu"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default=DEFAULT_WORKLOAD)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--ref-seconds", type=float, default=150.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--engine", choices=["auto", "rowwise", "tiled", "tiled_grouped", "band"], default="auto",
                    help="single-product workloads: run this engine instead of the autotuned choice (profiling)")
    ap.add_argument("--rowwise-params", help="task_size,loads_in_flight,vector_bytes,kernel: run the row "
                                             "engine with these instead of autotuning (e.g. for a profile)")
    ap.add_argument("--block-histogram", metavar="BHxBW[,BHxBW...]",
                    help="instead of timing: print the block-density histograms of the workload's matrix "
                         "(swift_plan_block_histogram, A's and the sorted column order) as one JSON line")
    ap.add_argument("--mtx", help="MatrixMarket coordinate file: run the product on this matrix instead "
                                  "of a synthetic workload")
    ap.add_argument("--n", type=int, default=128, help="dense columns with --mtx")
    ap.add_argument("--dtype", choices=["f32", "f64"], default="f32", help="value type with --mtx")
    args = ap.parse_args()
    if args.mtx:
        name = f"mtx:{os.path.splitext(os.path.basename(args.mtx))[0]}_n{args.n}_{args.dtype}"
        WORKLOADS[name] = dict(kind="mtx", path=args.mtx, N=args.n, dtype=args.dtype)
        args.workload = name
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.block_histogram:
        run_block_histogram(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.impl == "reference-gpu":
        run_reference_gpu(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
