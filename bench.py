"""Benchmark: matrix-free LMM REML + scan at N=50,000 samples, M=100,000 SNPs.

One step = the whole `gwas --model lmm --fastlmm --fastlmm-matrix-free --no-loco` null
model and scan on one B200 with the packed genotypes resident in HBM: randomized
subspace iteration (4 kinship applies with 266 right-hand sides, QR, eigendecomposition),
low-rank REML (81-point grid + golden section), and the score/Wald scan of all 100,000
SNPs, results copied to the host.  The workload is synthetic (seeded generator, two
Balding-Nichols populations, 2% missing calls, 3 covariates).  Inputs (1.25 GB packed)
exceed the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
    python bench.py --impl reference      # the reference's CPU algorithm on host cores

Multi-GPU runs (torchrun) are independent replicas (the path has no exchange step): each
rank runs its own job; value = seconds per job for the whole machine.
"""
from __future__ import annotations

import os

# The CPU restatement alternates OpenMP table decodes with multithreaded BLAS GEMMs; spinning
# idle OpenMP threads would steal the cores the GEMMs run on (set before any OpenMP runtime
# starts).
os.environ.setdefault("OMP_WAIT_POLICY", "PASSIVE")

import argparse
import json
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "REML+scan s (N=50k,M=100k)"
RANK, OVERSAMPLE = 256, 10


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--n", type=int, default=50000)
    ap.add_argument("--m", type=int, default=100000)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-out", default="")
    ap.add_argument("--apply-only", action="store_true",
                    help="time kinship applies alone (the profiling case), not the REML+scan job")
    ap.add_argument("--k", default="68",
                    help="right-hand sides for --apply-only (a comma-separated list: one line each)")
    ap.add_argument("--serve-requests", type=int, default=32,
                    help="requests in the serving stream measured after the job (0 skips)")
    ap.add_argument("--serve-config5", action="store_true",
                    help="serve on the serving configuration's resident matrix (--serve-n x "
                         "--serve-m) instead of the job's")
    ap.add_argument("--serve-n", type=int, default=200000)
    ap.add_argument("--serve-m", type=int, default=500000)
    ap.add_argument("--serve-fp64-sample", type=int, default=4,
                    help="requests the plain FP64 form serves one at a time beside the stream")
    ap.add_argument("--serve-only", action="store_true",
                    help="only the serving measurement")
    ap.add_argument("--no-fp64-compare", action="store_true",
                    help="skip the one-step timing of the plain FP64 GPU form")
    ap.add_argument("--dense-n", type=int, default=10000,
                    help="samples of the dense exact-route measurement (0 = skip)")
    ap.add_argument("--dense-m", type=int, default=50000, help="SNPs of the dense measurement")
    ap.add_argument("--dense-only", action="store_true",
                    help="only the dense exact-route measurement (the case its ncu captures use)")
    ap.add_argument("--config1", type=int, default=1,
                    help="run the small single-trait configuration leg (0 skips)")
    ap.add_argument("--config3", action="store_true",
                    help="run the multi-trait configuration leg (N=100k, M=500k, 8 traits)")
    ap.add_argument("--config3-iters", type=int, default=3)
    ap.add_argument("--config4", action="store_true",
                    help="run the repeatability configuration leg (N=100k, ~300k records, M=300k)")
    ap.add_argument("--config4-iters", type=int, default=6)
    ap.add_argument("--ref-budget", type=float, default=240.0,
                    help="seconds of whole CPU jobs the reference arm runs (at least one)")
    ap.add_argument("--aireml-iters", type=int, default=50,
                    help="AI-REML (PCG + Hutchinson) iterations of the timed full run (0 skips)")
    ap.add_argument("--precond-rank", type=int, default=64,
                    help="rank of the AI-REML's low-rank deflation preconditioner (0: scalar)")
    return ap.parse_args()


def max_over_ranks(x: float, world: int, device=None) -> float:
    """The largest value over the ranks of the process group (a multi-GPU time is the slowest
    rank's); the value itself with one rank."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def gpu_uuid(local: int):
    """The CUDA device's UUID in nvidia-smi's form (GPU-xxxxxxxx-...), or None."""
    try:
        import torch

        u = str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        return None
    return u if u.startswith("GPU-") else "GPU-" + u


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region.

    The GPU is selected by its UUID (nvidia-smi numbers GPUs in PCI order and ignores
    CUDA_VISIBLE_DEVICES, so on a shared machine an index can name another user's GPU), and
    every sample's UUID is checked against it; samples of any other GPU are dropped.
    A timed region can be shorter than nvidia-smi's start-up and its 200 ms cadence, so entry
    waits (up to 10 s) for the sampler's first line and exit waits (up to 1 s) for one sample
    taken after the region began; the summary uses the samples from the region's start on."""

    FIELDS = ("uuid,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local: int):
        self.uuid = gpu_uuid(local)
        self.idx = local
        self.proc = None
        self.lines: list[str] = []
        self.first = 0

    def __enter__(self):
        ident = self.uuid if self.uuid else str(self.idx)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={ident}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
            return self
        t0 = time.perf_counter()
        while not self.lines and self.proc.poll() is None and time.perf_counter() - t0 < 10.0:
            time.sleep(0.01)
        self.first = len(self.lines)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            t0 = time.perf_counter()
            while (len(self.lines) <= self.first and self.proc.poll() is None
                   and time.perf_counter() - t0 < 1.0):
                time.sleep(0.01)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons, other, idx = [], 0.0, set(), 0, None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines[self.first:]:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            if self.uuid and f[0] != self.uuid:
                other += 1
                continue
            try:
                sm.append(float(f[2]))
                smax = max(smax, float(f[3]))
                idx = int(f[1])
            except ValueError:
                continue
            for name, v in zip(names, f[6:10]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"],
                    "gpu_uuid": self.uuid}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "gpu_uuid": self.uuid, "nvidia_smi_index": idx,
                "selected_by": "uuid" if self.uuid else "index", "other_gpu_samples": other}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def fp64_peak_tflops(torch):
    """cuBLAS DGEMM 8192^3 throughput on this GPU (the FP64 denominator)."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(3):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def int8_peak_tops(torch):
    """cuBLASLt int8 GEMM 8192^3 throughput on this GPU (the int8 tensor-pipe denominator)."""
    a = torch.randint(-64, 64, (8192, 8192), dtype=torch.int8, device="cuda")
    b = torch.randint(-64, 64, (8192, 8192), dtype=torch.int8, device="cuda").t()
    for _ in range(2):
        torch._int_mm(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch._int_mm(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def profile_traffic():
    """DRAM bytes per packed byte of the tensor-core passes from the committed ncu summary
    (profiles/kinship_tc_pair_passes_n20000_m30000_k266.md), or None."""
    import re

    path = os.path.join(ROOT, "profiles", "kinship_tc_pair_passes_n20000_m30000_k266.md")
    try:
        text = open(path).read()
    except OSError:
        return None
    out = {}
    for name in ("rows", "samples"):
        m = re.search(rf"traffic_per_packed_byte_{name}:\s*([0-9.]+)", text)
        if m:
            out[name] = float(m.group(1))
    return out or None


def run_apply_only(args):
    """Kinship applies alone: the small case the ncu captures use."""
    import torch

    import cosmicscanner_b200 as cs
    from cosmicscanner_b200 import synth

    torch.cuda.set_device(0)
    d = synth.cohort(args.n, args.m, 20261203, n_pops=2, fst=0.01, missing=0.02, n_causal=100)
    g = cs.Genotypes.from_bed_bytes(d["bed"], args.n, args.m)
    op = cs.KinshipOperator(g, None, None)
    stream = torch.cuda.current_stream().cuda_stream
    for kk in [int(v) for v in str(args.k).split(",")]:
        X = torch.randn(kk, args.n, dtype=torch.float64, device="cuda")  # column-major n x k
        Y = torch.empty_like(X)
        for _ in range(args.warmup):
            op.apply_device(X.data_ptr(), args.n, kk, Y.data_ptr(), args.n, args.precision, stream)
        torch.cuda.synchronize()
        cs.profile_enable(True)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(args.steps):
            op.apply_device(X.data_ptr(), args.n, kk, Y.data_ptr(), args.n, args.precision, stream)
        e.record()
        torch.cuda.synchronize()
        prof = cs.profile_summary()
        cs.profile_enable(False)
        ms = s.elapsed_time(e) / args.steps
        flops = 4.0 * args.n * args.m * kk
        print(json.dumps({"metric": "kinship apply ms", "value": ms, "unit": "ms", "n": args.n,
                          "m": args.m, "k": kk, "precision": args.precision,
                          "tflops": flops / (ms * 1e-3) / 1e12,
                          "kernels": [(k["name"], k["launches"], k["ms"] / k["launches"])
                                      for k in prof["kernels"]]}), flush=True)
    return 0


def run_serve(cs, g, variants, d, args, window=None, max_batch_columns=4096, fp64_sample=0,
              label=""):
    """A Poisson stream of association requests against the resident genotypes: subsets of
    log-uniform size 5,000..N, 1..16 traits with h2 ~ U(0.1, 0.7), an intercept and 2..5 N(0,1)
    covariates, full low-rank REML on all SNPs and a scan of a random contiguous window
    (`window` SNPs, default M/2).  Arrivals at 80 % of the server's measured capacity.  With
    `fp64_sample` > 0, the plain FP64 form serves that many of the same requests one at a time
    (a bounded sample of the stream: its per-request latency gives its throughput).  Returns
    the server's latency / throughput statistics."""
    n, m = d["n"], d["m"]
    rng = np.random.default_rng(20261208)
    base = (d["y"] - d["y"].mean()) / d["y"].std()
    window = max(1, m // 2) if window is None else min(window, m)

    def request():
        n_sub = int(np.exp(rng.uniform(np.log(min(5000, n // 2)), np.log(n))))
        S = np.sort(rng.choice(n, n_sub, replace=False)).astype(np.int32)
        t = int(rng.integers(1, 17))
        h2 = rng.uniform(0.1, 0.7, size=t)
        Y = np.column_stack([np.sqrt(h2[j]) * base[S] + np.sqrt(1 - h2[j]) *
                             rng.standard_normal(n_sub) for j in range(t)])
        p = int(rng.integers(2, 6))
        X = np.column_stack([np.ones(n_sub)] + [rng.standard_normal(n_sub) for _ in range(p)])
        b = int(rng.integers(0, m - window + 1))
        return S, Y, X.astype(np.float32).astype(np.float64), b, b + window

    reqs = [request() for _ in range(args.serve_requests)]
    srv = cs.Server(g, variants, precision=args.precision, max_active=8,
                    max_batch_columns=max_batch_columns)
    # one untimed request (the server's threads, handles and buffers come up); the service time
    # of one request alone; the capacity: eight requests submitted at once, completed per
    # second.  Arrivals come at 80 % of that capacity.
    srv.wait(srv.submit(*reqs[0]))
    solo_id = srv.submit(*reqs[0])
    single = srv.wait(solo_id)["latency_s"]
    n_traits0 = reqs[0][1].shape[1]
    solo = [srv.result(solo_id, t) for t in range(n_traits0)]
    srv.release(solo_id)
    c0 = time.perf_counter()
    cal = [srv.submit(*q) for q in reqs[:8]]
    for rid in cal:
        srv.wait(rid)
    capacity = len(cal) / (time.perf_counter() - c0)
    for rid in cal:
        srv.release(rid)
    st0 = srv.stats()
    rate = 0.8 * capacity
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs)))
    t0 = time.perf_counter()
    ids, t_sub = [], []
    for (S, Y, X, b, e), at in zip(reqs, arrivals):
        delay = at - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        t_sub.append(time.perf_counter())
        ids.append(srv.submit(S, Y, X, b, e))
    lat, failed = [], []
    mix_vs_alone = None
    for i, rid in enumerate(ids):
        try:
            lat.append(srv.wait(rid)["latency_s"])
            if i == 0:
                # the stream's first request was also served alone: same result in the mix
                dp, dv = 0.0, 0.0
                for t in range(n_traits0):
                    a, b = srv.result(rid, t), solo[t]
                    tested = np.asarray(b["tested"], bool)
                    if not np.array_equal(np.asarray(a["tested"], bool), tested):
                        dp = float("inf")
                    else:
                        dp = max(dp, float(np.max(np.abs(a["log10p"][tested] - b["log10p"][tested]),
                                                  initial=0.0)))
                    dv = max(dv, abs(a["sigma2_g"] - b["sigma2_g"]) / max(abs(b["sigma2_g"]), 1e-300))
                mix_vs_alone = {"traits": n_traits0, "sigma2_g_rel": dv, "log10p_max_abs": dp}
        except cs.CosmicError as e:  # counted and reported, the stream goes on
            failed.append(str(e))
            lat.append(float("nan"))
        srv.release(rid)
    lat = np.array(lat)
    ok = ~np.isnan(lat)
    st = srv.stats()
    srv.close()
    done = np.array(t_sub)[ok] + lat[ok]
    wall = float(np.max(done) - t_sub[0]) if ok.any() else float("nan")
    applies = st["applies"] - st0["applies"]
    sizes = np.array([len(q[0]) for q in reqs])
    lok = lat[ok] if ok.any() else np.array([float("nan")])
    out = {
        "requests": len(reqs), "completed": int(ok.sum()), "req_per_s": int(ok.sum()) / wall,
        "p50_ms": float(np.percentile(lok, 50)) * 1e3, "p99_ms": float(np.percentile(lok, 99)) * 1e3,
        "mean_ms": float(lok.mean()) * 1e3,
        "single_request_ms": single * 1e3, "capacity_rps": capacity, "arrival_rate_per_s": rate,
        "stacked_applies": applies,
        "mean_columns_per_stacked_apply": (st["apply_columns"] - st0["apply_columns"]) / max(1, applies),
        "max_requests_per_apply": st["max_requests_per_apply"],
        "own_view_requests": st["own_view_requests"], "memory_budget_gb": st["memory_budget_gb"],
        "max_concurrent": st["max_concurrent"], "failed": st["failed"],
        "failure_messages": sorted(set(failed))[:3],
        "first_request_mix_vs_alone": mix_vs_alone,
        "cohort_size_median": float(np.median(sizes)), "cohort_size_mean": float(sizes.mean()),
        "config": f"{label}resident N={n} M={m}; {len(reqs)} requests; subsets log-U[5000,{n}], "
                  f"traits U{{1..16}}, intercept + U{{2..5}} N(0,1) covariates, window {window} "
                  f"SNPs, Poisson arrivals at 80% of the capacity (8 requests at once), "
                  f"{args.precision}; cohorts below N/2 on their own repacked subset operator",
    }
    if fp64_sample > 0:
        one = cs.Server(g, variants, precision="fp64", max_active=1,
                        max_batch_columns=max_batch_columns)
        lat64 = []
        for q in reqs[:fp64_sample]:
            rid = one.submit(*q)
            lat64.append(one.wait(rid)["latency_s"])
            one.release(rid)
        one.close()
        lat64 = np.array(lat64)
        mixed_same = lat[:fp64_sample]
        out["fp64_one_at_a_time"] = {
            "requests": fp64_sample, "mean_ms": float(lat64.mean()) * 1e3,
            "req_per_s": 1.0 / float(lat64.mean()),
            "p50_ms": float(np.percentile(lat64, 50)) * 1e3,
            "sample": f"the first {fp64_sample} requests of the stream, one at a time (the "
                      f"whole stream would take ~{lat64.mean() * len(reqs) / 60:.0f} min)",
            "throughput_ratio_mixed_batched_over_fp64": out["req_per_s"] * float(lat64.mean()),
            "mixed_latency_same_requests_ms": float(np.nanmean(mixed_same)) * 1e3}
    return out


def run_serve_config5(cs, args):
    """The serving configuration at its stated shape: a resident N=200,000 x M=500,000 packed
    matrix (~25 GB; MAF U(0.01, 0.5), three Balding-Nichols populations at Fst 0.02, 1% missing)
    and a stream of --serve-requests requests with 50,000-SNP scan windows."""
    import torch

    from cosmicscanner_b200 import synth

    t0 = time.perf_counter()
    d = synth.cohort(args.serve_n, args.serve_m, 20261203 + 5, maf_lo=0.01, n_pops=3, fst=0.02,
                     missing=0.01, n_causal=1000, h2=0.5)
    gen_s = time.perf_counter() - t0
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    variants = cs.grm_variant_selection(g.stats(), 0.01)
    del d["bed"]
    torch.cuda.synchronize()
    out = run_serve(cs, g, variants, d, args, window=50000, max_batch_columns=1024,
                    fp64_sample=args.serve_fp64_sample, label="serving configuration: ")
    out["generation_s"] = gen_s
    g.close()
    return out


def run_aireml(cs, op, d, args, iters=50, probes=64, precond_rank=64, compare_iters=6):
    """The PCG + Hutchinson AI-REML route (STCG_VCE with the single-record design, the
    configuration's 64 Rademacher probes, 1 + p right-hand sides, absolute CG tolerance 1e-10):
      * `full`: the reference's default run -- up to 50 iterations (probes are redrawn each
        iteration, so it seldom stops early), SLQ log-likelihood (30 probes x 15 steps) -- in the
        mixed form with the low-rank deflation preconditioner, timed end to end;
      * `compare`: `compare_iters` iterations (4 EM + AI steps, no SLQ) in the mixed form and the
        FP64 form with the same probes and preconditioner, and in the mixed form with the
        reference's scalar preconditioner: seconds per iteration, CG iterations per solve,
        kinship applies and their mean width, and the mixed form's VC error against FP64."""
    import torch

    def one(prec, it, slq, rank):
        vce = cs.StcgVce()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = vce.solve(op, d["y"], d["X"], kinship_divisor=float(d["m"]), max_iter=it,
                      mc_samples=probes, slq_probes=slq, precision=prec, precond_rank=rank)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        vce.close()
        solves = (1 + d["X"].shape[1] + probes + 3) * max(1, r["iterations"])
        return {"seconds": dt, "s_per_iteration": dt / max(1, r["iterations"]),
                "iterations": r["iterations"], "converged": bool(r["converged"]),
                "sigma2_g": r["sigma2_g"], "sigma2_e": r["sigma2_e"], "logl": r["logl"],
                "pcg_iterations": r["pcg_iterations"],
                "cg_iterations_per_solve": r["pcg_iterations"] / solves,
                "kinship_applies": r["operator_applies"],
                "rhs_per_apply": r["operator_columns"] / max(1, r["operator_applies"]),
                "ms_per_apply": 1e3 * dt / max(1, r["operator_applies"]),
                "precond_rank": rank, "precision": prec}

    out = {"full": one(args.precision, iters, 30, precond_rank)}
    cmp = {"mixed": one(args.precision, compare_iters, 0, precond_rank),
           "fp64": one("fp64", compare_iters, 0, precond_rank),
           "mixed_scalar_precond": one(args.precision, compare_iters, 0, 0)}
    for key in ("sigma2_g", "sigma2_e"):
        cmp[f"{key}_rel_mixed_vs_fp64"] = abs(cmp["mixed"][key] - cmp["fp64"][key]) / abs(cmp["fp64"][key])
    cmp["speedup_mixed_over_fp64"] = cmp["fp64"]["s_per_iteration"] / cmp["mixed"]["s_per_iteration"]
    cmp["speedup_deflation_over_scalar"] = (cmp["mixed_scalar_precond"]["s_per_iteration"] /
                                            cmp["mixed"]["s_per_iteration"])
    out["compare"] = cmp
    out["config"] = (f"N={d['n']} M={d['m']}, {probes} probes + y + {d['X'].shape[1]} covariates, "
                     f"pcg_tol 1e-10 absolute; full: up to {iters} iterations with SLQ (30 x 15), "
                     f"low-rank deflation rank {precond_rank}; compare: {compare_iters} iterations")
    return out


def run_config1(cs, args):
    """The small single-trait configuration (N=2,000, M=10,000, 1% missing, X = [1, N(0,1)],
    100 causal SNPs, h2 0.5): the low-rank REML + scan job in the mixed and FP64 GPU forms and
    the oracle's CPU restatement on the host cores, and the PCG + Hutchinson AI-REML with the
    configuration's 30 probes (reference defaults: up to 50 iterations, SLQ log-likelihood).
    Seconds per job (the second of two runs for the GPU forms)."""
    import torch

    import oracle
    from cosmicscanner_b200 import synth

    d = synth.config1()
    n, m = d["n"], d["m"]
    X = d["X"].astype(np.float32).astype(np.float64)
    g = cs.Genotypes.from_bed_bytes(d["bed"], n, m)
    variants = cs.grm_variant_selection(g.stats(), 0.01)
    op = cs.KinshipOperator(g, None, variants)
    keep = np.arange(n, dtype=np.int32)
    out = {"n": n, "m": m}
    res = {}
    for prec in ("mixed", "fp64"):
        eng = cs.LmmEngine()
        for _ in range(2):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            diag = eng.prepareLowRankMatrixFree(d["y"], X, op, rank=RANK, oversample=OVERSAMPLE,
                                                precision=prec)
            r = eng.scan(g, keep, min_maf=0.01, precision=prec)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
        res[prec] = (diag, r)
        out[f"lowrank_{prec}_s"] = dt
        eng.close()
    out["lowrank_accuracy_mixed_vs_fp64"] = accuracy(res["mixed"][0], res["mixed"][1],
                                                     res["fp64"][0], res["fp64"][1])
    B = oracle.Bed(d["bed"][3:].reshape(m, -1), n)
    t0 = time.perf_counter()
    cj = oracle.lowrank_job_blas(B, d["y"], X, variants=variants, rank=RANK, oversample=OVERSAMPLE,
                                 n_threads=host_threads())
    out["lowrank_cpu_restatement_s"] = time.perf_counter() - t0
    out["cpu_cores"] = host_threads()
    out["sigma2_g"] = {"mixed": res["mixed"][0]["sigma2_g"], "fp64": res["fp64"][0]["sigma2_g"],
                       "cpu": cj["sigma2_g"]}
    op_all = cs.KinshipOperator(g, None, None)
    for prec in ("mixed", "fp64"):
        vce = cs.StcgVce()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rv = vce.solve(op_all, d["y"], X, kinship_divisor=float(m), max_iter=50, mc_samples=30,
                       slq_probes=30, precision=prec)
        torch.cuda.synchronize()
        out[f"aireml_{prec}"] = {"seconds": time.perf_counter() - t0,
                                 "iterations": rv["iterations"], "sigma2_g": rv["sigma2_g"],
                                 "sigma2_e": rv["sigma2_e"], "logl": rv["logl"],
                                 "pcg_iterations": rv["pcg_iterations"]}
        vce.close()
    op_all.close()
    op.close()
    g.close()
    return out


def run_config3(cs, args):
    """The multi-trait configuration: N=100,000, M=500,000 (MAF U(0.01, 0.5)), 8 traits with
    LKJ(2) genetic correlation, h2 U(0.2, 0.6), residual correlation 0.3; the multi-trait
    matrix-free REML (EM on Vg (x) K + Ve (x) I with 32 probes: every kinship apply carries
    8 x (1 + 32) = 264 right-hand sides) in the mixed form, --config3-iters EM iterations.
    The reference's route (MvEigenVce) needs the dense N x N eigendecomposition (80 GB at
    N = 100,000) and is not run."""
    import torch

    from cosmicscanner_b200 import synth

    t0 = time.perf_counter()
    d = synth.config3()
    gen_s = time.perf_counter() - t0
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    op = cs.KinshipOperator(g, None, None)
    del d["bed"]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    Vg, Ve, r = cs.mv_stcg_solve(op, d["Y"], d["X"], kinship_divisor=float(d["m"]),
                                 max_iter=args.config3_iters, tol=0.0, mc_samples=32,
                                 precision=args.precision)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    op.close()
    g.close()
    h2_est = np.diag(Vg) / (np.diag(Vg) + np.diag(Ve))
    return {"n": d["n"], "m": d["m"], "traits": int(d["Y"].shape[1]), "seconds": dt,
            "s_per_iteration": dt / max(1, r["iterations"]), "iterations": r["iterations"],
            "kinship_applies": r["operator_applies"],
            "rhs_per_apply": r["operator_columns"] / max(1, r["operator_applies"]),
            "ms_per_apply": 1e3 * dt / max(1, r["operator_applies"]),
            "cg_iterations": r["pcg_iterations"], "h2_true": d["h2"].tolist(),
            "h2_after_iterations": h2_est.tolist(), "generation_s": gen_s,
            "precision": args.precision}


def run_config4(cs, args):
    """The repeatability configuration: N=100,000 individuals with 1..5 records each (~300k
    records), M=300,000 SNPs, y = X b + Zr (g + pe) + e with h2 0.3 and repeatability 0.5, fixed
    effects intercept, N(0,1) and a 4-level factor; the three-component matrix-free AI-REML
    (V = sg2 Zr K Zr' + spe2 Zr Zr' + se2 I) in the mixed form with 32 probes, --config4-iters
    iterations with the SLQ log-likelihood.  The record-level scan (scanSTCG) needs the dense
    q x q subject GRM as the reference builds it (80 GB at q = 100,000) and is not run here."""
    import torch

    from cosmicscanner_b200 import synth

    t0 = time.perf_counter()
    d = synth.config4()
    gen_s = time.perf_counter() - t0
    g = cs.Genotypes.from_bed_bytes(d["bed"], d["n"], d["m"])
    op = cs.KinshipOperator(g, None, None)
    del d["bed"]
    vce = cs.StcgVce()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r = vce.solve(op, d["y"], d["X"], rec_to_row=d["rec_to_row"], with_pe=True,
                  kinship_divisor=float(d["m"]), max_iter=args.config4_iters, mc_samples=32,
                  slq_probes=30, precision=args.precision)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    vce.close()
    op.close()
    g.close()
    return {"n": d["n"], "records": int(len(d["y"])), "m": d["m"], "seconds": dt,
            "s_per_iteration": dt / max(1, r["iterations"]), "iterations": r["iterations"],
            "sigma2_g": r["sigma2_g"], "sigma2_pe": r["sigma2_pe"], "sigma2_e": r["sigma2_e"],
            "logl": r["logl"], "pcg_iterations": r["pcg_iterations"],
            "kinship_applies": r["operator_applies"],
            "rhs_per_apply": r["operator_columns"] / max(1, r["operator_applies"]),
            "generation_s": gen_s, "precision": args.precision,
            "scan": "not run: scanSTCG needs the dense q x q subject GRM (80 GB at q = 100,000)"}


def run_dense(cs, args):
    """The dense exact route (`gwas --model lmm` without --fastlmm): GRM (VanRaden) over every
    sample, EigenVce with the covariate projection, Brent null model and the exact scan of
    every SNP, on its own synthetic cohort of --dense-n x --dense-m; seconds per stage (the
    second of two runs), and a CPU estimate of the same stages from numpy-BLAS samples: one
    2048-SNP GRM block, LAPACK eigh at n = 2000 scaled by n^3, one 512-SNP scan block."""
    import torch

    from cosmicscanner_b200 import synth

    n, m = args.dense_n, args.dense_m
    d = synth.cohort(n, m, 5, missing=0.02, n_causal=200, h2=0.4)
    g = cs.Genotypes.from_bed_bytes(d["bed"], n, m)
    y, X = d["y"], d["X"].astype(np.float32).astype(np.float64)
    keep = np.arange(n, dtype=np.int32)
    stages = None
    for _ in range(2):
        t = [time.perf_counter()]
        b = cs.GrmBuilder().compute(g)
        torch.cuda.synchronize()
        t.append(time.perf_counter())
        v = cs.EigenVce().prepare(y, X, b)
        t.append(time.perf_counter())
        r = v.runNullModel()
        t.append(time.perf_counter())
        eng = cs.LmmEngine()
        eng.prepareFromVce(v)
        out = eng.scan(g, keep, precision=args.precision)
        t.append(time.perf_counter())
        stages = {"grm_s": t[1] - t[0], "eigh_s": t[2] - t[1], "null_s": t[3] - t[2],
                  "scan_s": t[4] - t[3], "total_s": t[4] - t[0]}
        tested = int(out["tested"].sum())
        eng.close()
        v.close()
        b.close()
    g.close()
    # CPU estimate (the reference's Eigen GEMMs / SelfAdjointEigenSolver as numpy-BLAS)
    rng = np.random.default_rng(1)
    Z = rng.standard_normal((n, 2048))
    c0 = time.perf_counter()
    _ = Z @ Z.T
    grm_cpu = (time.perf_counter() - c0) * (m / 2048)
    del Z
    A = rng.standard_normal((2000, 2000))
    c0 = time.perf_counter()
    np.linalg.eigh(A + A.T)
    eig_cpu = (time.perf_counter() - c0) * (n / 2000) ** 3
    W = rng.standard_normal((n, 2048))
    G = rng.standard_normal((n, 512))
    c0 = time.perf_counter()
    _ = W.T @ G
    scan_cpu = (time.perf_counter() - c0) * (n / 2048) * (m / 512)
    return {"n": n, "m": m, "precision": args.precision, **stages, "tested": tested,
            "sigma2_g": r["sigma2_g"], "sigma2_e": r["sigma2_e"],
            "cpu_estimate_s": {"grm": grm_cpu, "eigh": eig_cpu, "scan": scan_cpu,
                               "total": grm_cpu + eig_cpu + scan_cpu,
                               "cores": os.cpu_count() or 1,
                               "sample": "numpy-BLAS: one 2048-SNP Z Z^T block x M/2048, "
                                         "eigh at n=2000 x (N/2000)^3, one 512-SNP W^T G "
                                         "block x (N/2048)(M/512)"}}


def job_config(n: int, m: int) -> dict:
    """The workload both arms print (identical dicts)."""
    return {"workload": f"lmm matrix-free low-rank REML+scan, N={n} M={m} rank={RANK} "
                        f"sketch={RANK + OVERSAMPLE} p=3 (synthetic, 2 pops Fst=0.01, 2% missing)",
            "n": n, "m": m, "rank": RANK, "sketch": RANK + OVERSAMPLE, "covariates": 3,
            "l2": "inputs (packed genotypes) larger than L2; no flush"}


def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_job(d, threads):
    """One whole job on the host cores: the oracle's restatement of the reference's CPU path
    (prepareLowRankMatrixFree + scanLowRank, numpy BLAS/LAPACK for Eigen, OpenMP decodes) on the
    same inputs and GRM variant selection as the GPU job.  The per-SNP statistics (the upload's
    counterpart) are computed before the clock starts.  Returns (seconds, result)."""
    import oracle

    n, m = d["n"], d["m"]
    B = oracle.Bed(d["bed"][3:].reshape(m, -1), n)
    freq = B.mean / 2.0
    maf = np.minimum(freq, 1.0 - freq)
    variants = np.nonzero((B.inv_std != 0.0) & ~(maf < 0.01) & ~(np.abs(maf) < 1e-8))[0]
    X = d["X"].astype(np.float32).astype(np.float64)
    t0 = time.perf_counter()
    r = oracle.lowrank_job_blas(B, d["y"], X, variants=variants, rank=RANK,
                                oversample=OVERSAMPLE, n_threads=threads)
    return time.perf_counter() - t0, r


CPU_SAMPLE = ("one whole job, not a sample: Omega, 4 kinship applies with 266 right-hand sides "
              "(512-SNP FP64 decode blocks, two BLAS GEMMs each), 3 QRs, B = Q^T K Q, eigh, "
              "REML grid + golden search, and the Woodbury scan of every SNP (one BLAS GEMM "
              "G^T [U|X|Py] per 512-SNP block) -- the oracle's restatement of the reference's "
              "CPU path with numpy's threaded OpenBLAS for Eigen")


def run_reference(args):
    """The reference's CPU algorithm (the oracle's restatement; the reference itself cannot be
    built here) timed as whole jobs on every host core.  A job takes a minute or more, so the
    arm runs whole jobs until --ref-budget seconds have passed (at least one, at most --steps)
    and reports how many it ran; it never scales a partial job."""
    world, rank, local = dist_setup()
    if rank != 0:
        return 0
    from cosmicscanner_b200 import synth

    d = synth.config2(n=args.n, m=args.m)
    threads = host_threads()
    # warm-up: the BLAS threads and decode tables on a small slice, not a whole job
    import oracle

    small = synth.cohort(2000, 2000, 3, missing=0.02, n_causal=20)
    oracle.lowrank_job_blas(oracle.Bed(small["bed"][3:].reshape(2000, -1), 2000), small["y"],
                            small["X"], rank=64, n_threads=threads)
    vals, last = [], None
    t_start = time.perf_counter()
    while len(vals) < max(1, args.steps):
        el, last = cpu_job(d, threads)
        vals.append(el)
        if time.perf_counter() - t_start + el > args.ref_budget:
            break
    value = float(np.mean(vals))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "s",
        "n_gpus": args.gpus, "steps": len(vals), "requested_steps": args.steps, "warmup": 0,
        "warmup_note": "one small job (N=2000, M=2000) warms the BLAS threads; no full-size warm-up",
        "ms_per_step": value * 1e3, "seconds_each": vals, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": job_config(args.n, args.m),
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "port",
                         "sample": CPU_SAMPLE, "stages_s": last["seconds"]},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "sigma2_g": last["sigma2_g"], "sigma2_e": last["sigma2_e"], "rank": last["rank"],
        "tested": int(last["tested"].sum()),
    }
    print(json.dumps(line))
    return 0


def accuracy(mixed_diag, mixed_res, fp_diag, fp_res):
    """The mixed step's error against the FP64 GPU step on the same inputs: relative error of
    the variance components, max |delta BETA| / max |BETA| and the same for SE over the SNPs
    both test, max |delta -log10 P|, and the number of SNPs whose tested flag differs."""
    t = fp_res["tested"] & mixed_res["tested"]
    out = {}
    for key in ("sigma2_g", "sigma2_e"):
        out[f"{key}_rel"] = abs(mixed_diag[key] - fp_diag[key]) / abs(fp_diag[key])
    for key in ("beta", "se"):
        out[f"{key}_max_rel"] = float(np.abs(mixed_res[key][t] - fp_res[key][t]).max() /
                                      np.abs(fp_res[key][t]).max())
    out["beta_max_abs_over_se"] = float((np.abs(mixed_res["beta"][t] - fp_res["beta"][t]) /
                                         fp_res["se"][t]).max())
    out["log10p_max_abs"] = float(np.abs(mixed_res["log10p"][t] - fp_res["log10p"][t]).max())
    out["tested_mismatch"] = int((fp_res["tested"] != mixed_res["tested"]).sum())
    out["freq_equal"] = bool(np.array_equal(mixed_res["freq"][t], fp_res["freq"][t]))
    out["bounds"] = {"vc_rel": 1e-5, "beta_se_rel": 1e-5, "log10p_abs": 1e-3}
    out["within_bounds"] = bool(max(out["sigma2_g_rel"], out["sigma2_e_rel"]) <= 1e-5 and
                                max(out["beta_max_rel"], out["se_max_rel"]) <= 1e-5 and
                                out["log10p_max_abs"] <= 1e-3 and out["tested_mismatch"] == 0)
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.apply_only:
        return run_apply_only(args)
    if args.serve_only:
        import torch

        import cosmicscanner_b200 as cs

        torch.cuda.set_device(0)
        print(json.dumps({"serve": run_serve_config5(cs, args) if args.serve_config5 else None}))
        return 0
    if args.dense_only:
        import torch

        import cosmicscanner_b200 as cs

        torch.cuda.set_device(0)
        print(json.dumps({"dense": run_dense(cs, args)}))
        return 0
    import torch

    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    import cosmicscanner_b200 as cs
    from cosmicscanner_b200 import synth

    d = synth.config2(n=args.n, m=args.m)
    n, m = d["n"], d["m"]
    y = d["y"]
    X = d["X"].astype(np.float32).astype(np.float64)
    keep = np.arange(n, dtype=np.int32)
    bed = d["bed"]
    # pinned host copy of the inputs for the end-to-end leg
    cudart = torch.cuda.cudart()
    pinned = cudart.cudaHostRegister(bed.ctypes.data, bed.nbytes, 0) == 0

    g = cs.Genotypes.from_bed_bytes(bed, n, m)
    variants = cs.grm_variant_selection(g.stats(), 0.01)
    op = cs.KinshipOperator(g, None, variants)
    eng = cs.LmmEngine()

    diag = {}

    def step():
        diag.update(eng.prepareLowRankMatrixFree(y, X, op, rank=RANK, oversample=OVERSAMPLE,
                                                 precision=args.precision))
        return eng.scan(g, keep, min_maf=0.01, precision=args.precision)

    for _ in range(args.warmup):
        res = step()
    barrier = (lambda: torch.distributed.barrier()) if world > 1 else (lambda: None)
    barrier()
    torch.cuda.synchronize()
    launches0 = cs.launch_count()
    cs.profile_enable(True)
    with ClockSampler(local) as clocks:
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(args.steps):
            res = step()
        stop.record()
        torch.cuda.synchronize()
    barrier()
    prof = cs.profile_summary()
    cs.profile_enable(False)
    launches = cs.launch_count() - launches0
    ms = max_over_ranks(start.elapsed_time(stop), world, device="cuda")
    sec_per_step = ms / 1e3 / args.steps
    value = sec_per_step / world

    # ---- end to end through the public API from pinned host buffers
    # one untimed end-to-end job first (the device memory pool grows to the job's size once)
    cs.run_lmm_matrix_free(bed, n, m, y, X, rank=RANK, oversample=OVERSAMPLE,
                           precision=args.precision)
    torch.cuda.synchronize()
    e2e_ms = []
    cs.profile_enable(True)
    for _ in range(max(1, args.e2e_steps)):
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        cs.run_lmm_matrix_free(bed, n, m, y, X, rank=RANK, oversample=OVERSAMPLE,
                               precision=args.precision)
        t1.record()
        torch.cuda.synchronize()
        e2e_ms.append(t0.elapsed_time(t1))
    e2e_prof = cs.profile_summary()
    cs.profile_enable(False)
    # median over the jobs: a host-side hiccup in one job (the OS, the interpreter) does not move it
    e2e_s = max_over_ranks(float(np.median(e2e_ms)) / 1e3, world, device="cuda")

    # ---- the plain FP64 GPU form of the same job, one step (the north-star comparison), with
    # its top kernel profiled and the mixed step's error against it
    fp64 = None
    if not args.no_fp64_compare and args.precision != "fp64":
        torch.cuda.synchronize()
        cs.profile_enable(True)
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record()
        fp_diag = eng.prepareLowRankMatrixFree(y, X, op, rank=RANK, oversample=OVERSAMPLE,
                                               precision="fp64")
        fp_res = eng.scan(g, keep, min_maf=0.01, precision="fp64")
        a1.record()
        torch.cuda.synchronize()
        fp_prof = cs.profile_summary()
        cs.profile_enable(False)
        fp64_s = a0.elapsed_time(a1) / 1e3
        ftop = max(fp_prof["kernels"], key=lambda k: k["ms"])
        f_ms = ftop["ms"] / ftop["launches"]
        f_ach = ftop["flops"] / ftop["launches"] / (f_ms * 1e-3) / 1e12
        dgemm = fp64_peak_tflops(torch)
        fp64 = {"value": fp64_s, "unit": "s", "speedup_mixed_over_fp64": fp64_s / sec_per_step,
                "roofline": {"bound": "fp64", "kernel": ftop["name"], "achieved": f_ach,
                             "peak": dgemm, "unit": "TFLOP/s", "frac": f_ach / dgemm,
                             "peak_kind": "cuBLAS DGEMM 8192^3 measured in this run",
                             "ms_per_launch": f_ms, "launches": ftop["launches"],
                             "share_of_step": ftop["ms"] / (fp64_s * 1e3)},
                "note": "the same REML+scan step with FP64 kinship applies and scan projection",
                "accuracy_of_mixed": accuracy(diag, res, fp_diag, fp_res)}
    serve = None
    if args.serve_requests > 0 and world == 1:
        serve = (run_serve_config5(cs, args) if args.serve_config5 else
                 run_serve(cs, g, variants, d, args, fp64_sample=args.serve_fp64_sample))
    dense = run_dense(cs, args) if args.dense_n > 0 and world == 1 else None
    config1 = run_config1(cs, args) if args.config1 and world == 1 else None
    config3 = run_config3(cs, args) if args.config3 and world == 1 else None
    config4 = run_config4(cs, args) if args.config4 and world == 1 else None
    aireml = None
    if args.aireml_iters > 0 and world == 1:
        op_all = cs.KinshipOperator(g, None, None)
        aireml = run_aireml(cs, op_all, d, args, iters=args.aireml_iters,
                            precond_rank=args.precond_rank)
        op_all.close()

    if rank == 0:
        peaks, peak_kind = measured_peaks()
        kernels = [k for k in prof["kernels"]]
        top = max(kernels, key=lambda k: k["ms"])
        per_launch_ms = top["ms"] / top["launches"]
        flops_per_launch = top["flops"] / top["launches"]
        if "fp64" in top["name"]:
            peak = fp64_peak_tflops(torch)
            roof = {"bound": "fp64", "peak_kind": "cuBLAS DGEMM 8192^3 measured in this run"}
        else:
            peak = peaks["bf16_tflops"]
            roof = {"bound": "tensor", "peak_kind": f"bf16_tflops ({peak_kind})"}
        achieved = flops_per_launch / (per_launch_ms * 1e-3) / 1e12
        bytes_per_launch = top["bytes"] / top["launches"]
        traffic = None
        tr = profile_traffic()
        if tr and "_tc" in top["name"]:
            key = "rows" if "rows" in top["name"] else "samples"
            if key in tr:
                traffic = tr[key] * bytes_per_launch
        roof.update({"kernel": top["name"], "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak, "traffic": traffic,
                     "traffic_note": "ncu DRAM bytes per packed byte at N=20000 M=30000 k=266, "
                                     "scaled by this launch's packed bytes",
                     "algorithmic_bytes_per_launch": bytes_per_launch,
                     "ms_per_launch": per_launch_ms,
                     "share_of_step": top["ms"] / ms})
        if "_tc" in top["name"]:
            # the int8 datapath: MMA columns per useful multiply-add on columns padded to the
            # plan's column tiles (width cap w, a last tile rounded up to 16): 5 (3 right-hand-
            # side pieces against the imputed-code tile, 2 against the missing-indicator tile),
            # or 6 in a samples pass over the sample-major copy with the fixed dosage table (W and
            # mu o W, 3 pieces each)
            k_rhs = RANK + OVERSAMPLE
            plan = next((e for e in (prof.get("autotune") or [])
                         if e["pass"] == ("rows" if "rows" in top["name"] else "samples")
                         and abs(e["k"] - k_rhs) < 16), None)
            w = plan["max_width"] if plan else 80
            sets = 6 if ("samples" in top["name"] and plan
                         and plan.get("tmem_a") in (32, 64, "pair64")) else 5
            tiles = -(-k_rhs // w)
            padded = w * (tiles - 1) + -(-(k_rhs - w * (tiles - 1)) // 16) * 16
            ops = achieved * sets * padded / k_rhs
            ipeak = int8_peak_tops(torch)
            roof["int8_datapath"] = {"mma_tops": ops, "peak_tops": ipeak, "operand_sets": sets,
                                     "column_tile": w,
                                     "peak_kind": "cuBLASLt int8 GEMM 8192^3 measured in this run",
                                     "frac": ops / ipeak}
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            threads = host_threads()
            el, cr = cpu_job(d, threads)
            cpu = {"value": el, "unit": "s", "cores": threads, "kind": "port", "sample": CPU_SAMPLE,
                   "stages_s": cr["seconds"], "sigma2_g": cr["sigma2_g"],
                   "sigma2_e": cr["sigma2_e"], "rank": cr["rank"],
                   "sigma2_g_rel_to_gpu": abs(cr["sigma2_g"] - diag["sigma2_g"]) / abs(cr["sigma2_g"])}
        h2d = bed.nbytes + y.nbytes + X.nbytes + keep.nbytes
        d2h = m * (5 * 8 + 4)
        line = {
            "metric": METRIC, "value": value, "unit": "s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec_per_step * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else
                     "i8xi8->i32 (tcgen05.mma kind::i8, right-hand sides as 3 int8 pieces) + f64 "
                     "epilogue, QR, eigh, REML and scan statistics",
            "data": "synthetic",
            "config": job_config(n, m),
            "precision": args.precision, "parallelism": f"replicas x{world}",
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_s / world, "unit": "s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "pinned_host": bool(pinned),
                    "statistic": f"median of {len(e2e_ms)} jobs", "ms_each": e2e_ms, "host_stages": e2e_prof.get("host", [])},
            "fp64_gpu": fp64,
            "accuracy": None if fp64 is None else fp64["accuracy_of_mixed"],
            "serve": serve,
            "aireml": aireml,
            "config1": config1,
            "config3": config3,
            "config4": config4,
            "dense": dense,
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
            "kernels": kernels,
            "autotune": prof.get("autotune", []),
            "host_stages": prof.get("host", []),
            "sigma2_g": eng.getSigma2g(), "sigma2_e": eng.getSigma2e(),
            "tested": int(res["tested"].sum()),
        }
        print(json.dumps(line))
        if args.profile_out:
            with open(args.profile_out, "w") as f:
                json.dump(line, f, indent=1)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
