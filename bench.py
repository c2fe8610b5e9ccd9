#!/usr/bin/env python
"""Headline benchmark: 3-way K2 exhaustive search, 4096 SNPs x 262,144 samples.

Metric (the reference's, src/tensor-episdet.cu:198): unique triplets x samples
per second / 1e12 ("tera (triplets x samples)/s").  One step = one complete
exhaustive 3-way K2 search over the synthetic dataset (131,072 cases +
131,072 controls, planted triplet {137, 2048, 3901}).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value : K timed searches with the planes already resident in HBM, CUDA events
        on the stream the library launches on, max over ranks.
e2e   : the same search through the public C-ABI with pinned host buffers,
        host->device copies and the result read-back inside the timed region.
With N > 1 (torchrun) the first-SNP range is split into N slabs of equal
work; each rank searches its slab and the per-rank candidate lists are
all-gathered and merged (the only exchange), so the N-GPU job computes the
same answer as one GPU (strong scaling).
--impl reference times the CPU restatement of the reference (the oracle, the
reference has no CPU path and cannot be built here) on bounded samples of the
same workload, with all host threads.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "tensor-episdet_b200")
ORACLE = os.path.join(ROOT, "oracle")
sys.path.insert(0, PKG)

M, NC, NN = 4096, 131072, 131072
PLANTED = (137, 2048, 3901)
SEED = 0xE917
PUBLISHED = 25.0  # the reference's published "> 25 x 10^12" on a GeForce RTX 2070 SUPER (README.md:54-61)
METRIC = "3-way K2 tera (triplets×samples)/s at 4096 SNP×262144; batched vs plain"
UNIT = "1e12 triplets*samples/s"
WORKLOAD = ("exhaustive 3-way K2 search, 4096 SNPs x 262144 samples (131072 cases + 131072 controls), "
            "HWE genotypes MAF~U[0.05,0.5], planted triplet {137,2048,3901}")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the 64-cohort batched vs plain comparison")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class Clocks:
    """nvidia-smi sampler (200 ms) covering the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=10)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------ CPU side
def cpu_sample(cases, controls, target_s=10.0):
    """Times the CPU oracle (scalar popcount, all host threads) on a bounded
    sample of the workload: first SNP X = 0, second SNP Y in [1, 1+ky), every
    Z > Y.  ky is calibrated so one sample takes about target_s seconds."""
    sys.path.insert(0, ORACLE)
    import pyoracle

    cores = os.cpu_count() or 1

    def run(ky):
        t = time.perf_counter()
        r = pyoracle.search(cases, controls, NC, NN, order=3, score="k2", top_k=16, threads=cores, first_begin=0,
                            first_end=1, second_begin=1, second_end=1 + ky)
        return r["sets"], time.perf_counter() - t

    k0 = min(M - 3, cores)  # one (X, Y) work item per thread
    sets, dt = run(k0)
    ky = max(1, min(M - 3, int(k0 * target_s / max(dt, 1e-3))))
    return ky, cores, run


def cpu_baseline(cases, controls, gpu_slab):
    """The oracle on all host threads over the first-SNP slab X = 0 (every
    triplet {0, Y, Z}: 8.4 M of the 11.4 G, the heaviest first SNP), timed,
    and its top-1024 list compared with the GPU's search of the same slab
    (sets, FP32 key bits, FP64 re-scores, best set)."""
    import numpy as np

    sys.path.insert(0, ORACLE)
    import pyoracle

    cores = os.cpu_count() or 1
    t = time.perf_counter()
    o = pyoracle.search(cases, controls, NC, NN, order=3, score="k2", top_k=1024, threads=cores, first_begin=0,
                        first_end=1)
    dt = time.perf_counter() - t
    r = gpu_slab
    n = len(o["top"])
    match = (tuple(r.snps) == tuple(o["best"]) and r.score == o["best_fp64"] and len(r.top_snps) == n
             and [tuple(x) for x in r.top_snps[:n]] == [tuple(x) for x in o["top"]]
             and np.array_equal(r.top_fp32[:n].view(np.uint32), o["top_fp32"].view(np.uint32))
             and np.array_equal(r.top_fp64[:n], o["top_fp64"]))
    return {"value": o["sets"] * (NC + NN) / dt / 1e12, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"first-SNP slab X=0 ({o['sets']} triplets, all Y<Z) in {dt:.1f} s (oracle/oracle.c, "
                      f"scalar 64-bit popcount, {cores} threads)"}, {
        "oracle_slab_match": bool(match),
        "slab": "first SNP X=0 of the 4096 x 262144 workload, top 1024 (sets, FP32 key bits, FP64 scores, best)",
        "best": list(o["best"]), "sets": o["sets"]}


def generate():
    import episdet

    return episdet.generate(SEED, M, NC, NN, maf=(0.05, 0.5), planted=[PLANTED], base_risk=0.5, effect=0.25)


def generate_oracle():
    """The same planes made by the oracle library alone (bit-identical to
    generate(); tests/test_bench_cpu.py checks it), so the reference arm's
    process never loads the product library."""
    sys.path.insert(0, ORACLE)
    import pyoracle

    return pyoracle.generate(SEED, M, NC, NN, maf=(0.05, 0.5), planted=[PLANTED], base_risk=0.5, effect=0.25)


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    cases, controls = generate_oracle()
    ky, cores, run = cpu_sample(cases, controls, target_s=8.0)
    for _ in range(args.warmup):
        run(ky)
    tot_sets, tot_t = 0, 0.0
    for _ in range(args.steps):
        s, dt = run(ky)
        tot_sets += s
        tot_t += dt
    v = tot_sets * (NC + NN) / tot_t / 1e12
    sample = (f"X=0, Y in [1,{1 + ky}), all Z>Y per step ({tot_sets // max(args.steps, 1)} triplets), "
              f"oracle/oracle.c scalar popcount on {cores} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / max(args.steps, 1), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": v / PUBLISHED, "dtype": "u64 popcount", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": sample},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference needs CUTLASS 1.3 (absent) and has no CPU path; its algorithm is timed as the "
                "project's CPU restatement (oracle/), on a bounded sample of the workload (the whole search "
                "would take hours on the host cores); planes made by the oracle's own generator, so this "
                "process loads no library of the product",
        "libraries_loaded": sorted({os.path.relpath(l.split()[-1], ROOT) for l in open("/proc/self/maps")
                                    if l.rstrip().endswith(".so") and l.split()[-1].startswith(ROOT)})}))


# ------------------------------------------------------------------ GPU side
COHORT_SEED = 0xE915 + 4


def cohorts64():
    """64 seeded cohorts: SNPs log-uniform in [256, 2048], samples log-uniform in
    [4096, 131072], case fraction uniform in [0.3, 0.7]; even ones 2-way, odd
    ones 3-way, K2."""
    import numpy as np
    import episdet

    rng = np.random.default_rng(COHORT_SEED)
    out = []
    for i in range(64):
        m = int(round(math.exp(rng.uniform(math.log(256), math.log(2048)))))
        n = int(round(math.exp(rng.uniform(math.log(4096), math.log(131072)))))
        nc = int(round(n * rng.uniform(0.3, 0.7)))
        c, k = episdet.generate(COHORT_SEED * 1000 + i, m, nc, n - nc, maf=(0.05, 0.5))
        out.append((c, k, nc, n - nc, m, 2 if i % 2 == 0 else 3))
    return out


def batched_vs_plain(reps=2):
    """The 64 cohorts searched one after another through episdet.search (plain)
    and in one episdet.search_batched call with per-shape autotuning of the
    triplet instance (the tuning probes run in the warm-up pass), device-resident
    planes, wall clock around each full pass (synchronised), best of `reps`
    after a warm-up pass; every batched result must equal its plain result."""
    import numpy as np
    import torch
    import episdet

    co = cohorts64()
    dev = [(torch.from_numpy(c.view(np.int32)).cuda(), torch.from_numpy(k.view(np.int32)).cuda(), nc, nn, m)
           for c, k, nc, nn, m, _ in co]
    opts = [{"order": o, "score": "k2", "top_k": 1024} for *_, o in co]
    work = sum(math.comb(m, o) * (nc + nn) for _, _, nc, nn, m, o in co)

    def plain():
        return [episdet.search(c, k, nc, nn, num_snps=m, **o) for (c, k, nc, nn, m), o in zip(dev, opts)]

    opts_b = [dict(o, flags=episdet.FLAG_AUTOTUNE) for o in opts]

    def batched():
        return episdet.search_batched(dev, opts_b)

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0, r

    plain(), batched()
    tp, tb, same = [], [], True
    for _ in range(reps):
        t, rp = timed(plain)
        tp.append(t)
        t, rb = timed(batched)
        tb.append(t)
        same = same and all(a.snps == b.snps and a.score == b.score and np.array_equal(a.top_snps, b.top_snps)
                            and np.array_equal(a.top_fp64, b.top_fp64) for a, b in zip(rp, rb))
    return {"workload": "64 cohorts, SNPs log-U[256,2048], samples log-U[4096,131072], case fraction U[0.3,0.7], "
                        "half 2-way half 3-way K2", "plain_s": min(tp), "batched_s": min(tb),
            "ratio": min(tp) / min(tb), "identical": same,
            "plain_rate": work / min(tp) / 1e12, "batched_rate": work / min(tb) / 1e12, "unit": UNIT,
            "batched_autotune": True,
            "tuned_staged": sorted({(nc_ if nc_ < nn_ else nn_).bit_length() - 1: episdet.tuned_stage(3, "k2", nc_, nn_)
                                    for _, _, nc_, nn_, _, o_ in co if o_ == 3}.items()),
            "timing": f"wall clock per pass, device-resident planes, best of {reps} after a warm-up pass"}


def ours(args):
    import numpy as np
    import torch
    import episdet
    import sharded

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    cases, controls = generate()
    fb, fe = sharded.work_slabs(M, 3, world)[rank]
    stream = torch.cuda.Stream()
    dc = torch.from_numpy(cases.view(np.int32)).cuda()
    dn = torch.from_numpy(controls.view(np.int32)).cuda()
    hc = torch.from_numpy(cases.view(np.int32)).pin_memory()
    hn = torch.from_numpy(controls.view(np.int32)).pin_memory()
    K = 1024

    def step(c, n, timing=False):
        r = episdet.search(c, n, NC, NN, num_snps=M, order=3, score="k2", top_k=K, device=local,
                           first_begin=fb, first_end=fe, stream=stream.cuda_stream,
                           flags=episdet.FLAG_TIMING if timing else 0)
        return r

    def gather(r):
        if world == 1:
            return [(r.top_snps, r.top_fp32, r.top_fp64)]
        return sharded.gather_candidates(r.top_snps, r.top_fp32, r.top_fp64, K, 3,
                                         device=torch.device("cuda", local))

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist

            dist.barrier()

    def timed(c, n, steps, timing):
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        res = []
        e0.record(stream)
        for _ in range(steps):
            r = step(c, n, timing)
            res.append((r, gather(r)))
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        barrier()
        if world > 1:
            import torch.distributed as dist

            t = torch.tensor([ms], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, res

    for _ in range(args.warmup):
        gather(step(dc, dn))
    clocks = Clocks(local)
    clocks.start()
    ms, res = timed(dc, dn, args.steps, True)
    clk = clocks.stop()
    ms_e2e, res_e2e = timed(hc, hn, args.steps, False)

    total_sets = math.comb(M, 3)
    ms_step = ms / args.steps
    value = total_sets * (NC + NN) / (ms_step * 1e-3) / 1e12
    value_e2e = total_sets * (NC + NN) / (ms_e2e / args.steps * 1e-3) / 1e12
    r0 = res[-1][0]
    rows, best = sharded.merge_candidates(res[-1][1], "k2", K)
    if rank != 0:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    # Roofline of the dominant kernel (the triplet tensor launches), this rank:
    # the e2m1 MACs it issues (2 ops each) per second of its launches, against
    # the best rate measured for that instruction at the shape it issues
    # (tcgen05.mma.cta_group::2.kind::mxf4, N = 112: four count segments of
    # 112 accumulator columns plus the scale-factor columns fill the 512 TMEM
    # columns; profiles/tcgen05_mma_peak.md), and beside it the N = 256 rate
    # (the instruction's best at any shape) and the measured bf16 x 4 figure.
    peaks = {}
    pp = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pp):
        peaks = json.load(open(pp))
    bf16 = peaks.get("bf16_tflops_sustained") or 1400.0
    inst = {}
    pk = os.path.join(ROOT, "profiles", "tcgen05_mma_peak.md")
    if os.path.exists(pk):
        for line in open(pk):
            for key in ("mxf4_pair_n112_peak_tflops", "mxf4_pair_n256_peak_tflops"):
                if line.startswith(key + ":"):
                    inst[key] = float(line.split(":")[1].split()[0])
    kern_ms = sum(r.count_kernel_ms for r, _ in res) / args.steps
    launches = sum(r.count_kernel_launches for r, _ in res) / args.steps
    slab_sets = r0.sets_evaluated
    alg_ops = 2.0 * 8.0 * slab_sets * (NC + NN)        # 2 ops per bit-MAC, 8 AND cells per triplet
    exe_ops = 2.0 * r0.executed_macs
    algorithmic = alg_ops / (kern_ms * 1e-3) / 1e12
    executed = exe_ops / (kern_ms * 1e-3) / 1e12
    peak = inst.get("mxf4_pair_n112_peak_tflops")
    p256 = inst.get("mxf4_pair_n256_peak_tflops")
    roof = {"bound": "tensor", "achieved": executed, "peak": peak, "unit": "TFLOP/s",
            "frac": (executed / peak) if peak else None, "traffic": None,
            "kernel": "episdet::tc::tc_kernel (triplets)",
            "peak_source": "measured on this pool: kind::mxf4 CTA-pair MMA, M=256 N=112, 64 MMAs per commit "
                           "(profiles/tcgen05_mma_peak.md)",
            "frac_of_n256_instruction_peak": (executed / p256) if p256 else None,
            "n256_instruction_peak_tflops": p256,
            "frac_of_4x_bf16_sustained": executed / (4.0 * bf16),
            "algorithmic_tflops": algorithmic,
            "kernel_ms_per_step": kern_ms, "launches_per_step": launches,
            "avg_launch_us": 1e3 * kern_ms / max(launches, 1),
            "note": "achieved = e2m1 MACs the kernel issues x 2 / its launch time; the engine regroups samples by "
                    "the first SNP's genotype (exact), so it issues 4.2x fewer MACs than the algorithmic 8 AND "
                    "cells x N per triplet counted in algorithmic_tflops"}
    prof = os.path.join(ROOT, "profiles", "tc_kernel_triplets.md")
    if os.path.exists(prof):
        for line in open(prof):
            if line.startswith("traffic_bytes_per_launch_scaled:"):
                roof["traffic"] = float(line.split(":")[1].split()[0])
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": value / PUBLISHED, "dtype": "e2m1", "data": "synthetic (seeded HWE generator, planted triplet)",
        "config": {"workload": WORKLOAD, "snps": M, "samples": NC + NN, "order": 3, "score": "K2", "top_k": K,
                   "engine": "tcgen05 kind::mxf4 CTA pairs (counts exact in FP32)",
                   "parallelism": f"first-SNP slabs over {world} GPU(s)",
                   "l2": "inputs larger than L2 (256 MiB packed planes; 4 x 1.1 GB regrouped e2m1 operand rows "
                         "per launch)"},
        "e2e": {"value": value_e2e, "unit": UNIT, "h2d_bytes_per_step": int(res_e2e[-1][0].h2d_bytes),
                "d2h_bytes_per_step": int(res_e2e[-1][0].d2h_bytes)},
        "gpu_launches": int(sum(r.kernel_launches for r, _ in res)),
        "roofline": roof,
        "clocks": clk,
        "best": {"snps": list(best[1]), "k2_fp64": best[2], "planted_recovered": tuple(best[1]) == PLANTED},
    }
    if world == 1 and not args.no_batched:
        out["batched_vs_plain"] = batched_vs_plain()
    # FP32 epilogue scores against their FP64 re-scores over the top-1024 list.
    err = np.abs(r0.top_fp32.astype(np.float64) - r0.top_fp64)
    out["fp32_vs_fp64"] = {"max_abs": float(err.max()), "max_rel": float((err / np.abs(r0.top_fp64)).max()),
                           "over": "the 1024 candidates of the full search (K2 values ~1.8e5)"}
    if world == 1 and not args.no_cpu_baseline:
        slab = episdet.search(dc, dn, NC, NN, num_snps=M, order=3, score="k2", top_k=K, device=local,
                              first_begin=0, first_end=1, stream=stream.cuda_stream)
        out["cpu_baseline"], out["oracle_slab"] = cpu_baseline(cases, controls, slab)
        out["oracle_slab_match"] = out["oracle_slab"]["oracle_slab_match"]
    print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
