"""Benchmark of the PCAone B200 hot path: window-based RSVD (--svd 2) of a PLINK .bed.

Workload (default): 20,000 samples x 500,000 SNPs, 5 Balding-Nichols populations
(Fst ~ U(0.01, 0.1) per population, ancestral allele frequency ~ U(0.01, 0.5)), HWE
genotypes, 0.5% of entries missing completely at random; k = 20 (l = 40), 64 windows, the
reference's default flags otherwise (maxp 20, tol 1e-4, seed 101, in-core SNP shuffle).
Data are synthetic, generated by the package's seeded simulator.

One step = one full top-k PCA (all power-iteration epochs) over the packed genotypes.
  value : bed GB/s = packed .bed bytes x epochs / step time, genotypes resident in HBM,
          device time from CUDA events on the library's stream (summed over ranks for N > 1).
  e2e   : the same metric through the C ABI from host buffers: every step uploads the
          packed matrix from pinned memory, permutes/transposes it on the device, runs the
          RSVD and reads U, S, V back.
The packed matrix (2.5 GB) is larger than L2 (126 MB), so no L2 flush is needed between steps.

--impl reference times the reference PCAone (built from its own sources into oracle/_ref)
on the host cores, on a bounded sample of the same workload (all samples, a slice of SNPs).
"""
from __future__ import annotations

import argparse
import re
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    "c2": dict(workload="winSVD k=20, 64 windows, 20000 samples x 500000 SNPs, 5 BN pops",
               n=20000, m=500000, pops=5, fst=(0.01, 0.1), pmin=0.01, pmax=0.5, miss=0.005,
               seed=2, k=20, svd=2, bands=64, maxp=20, tol=1e-4, cpu_sample_snps=8000),
    # profiling-size case of c2 (packed matrix 250 MB > L2), same shapes per window row/column
    "c2s": dict(workload="winSVD k=20, 64 windows, 20000 samples x 50000 SNPs, 5 BN pops",
                n=20000, m=50000, pops=5, fst=(0.01, 0.1), pmin=0.01, pmax=0.5, miss=0.005,
                seed=2, k=20, svd=2, bands=64, maxp=20, tol=1e-4, cpu_sample_snps=8000),
    "c1": dict(workload="Halko k=10 p=7, 2000 samples x 50000 SNPs, 3 BN pops",
               n=2000, m=50000, pops=3, fst=(0.05, 0.05), pmin=0.05, pmax=0.5, miss=0.01,
               seed=1, k=10, svd=1, bands=64, maxp=7, tol=0.0, cpu_sample_snps=50000),
}

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


_T0 = time.time()


def log(*a):
    print(f"[{time.time() - _T0:8.1f}s]", *a, file=sys.stderr, flush=True)


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), \
        int(os.environ.get("LOCAL_RANK", 0))


def make_data(cfg, out_prefix):
    """Generate the synthetic .bed/.bim/.fam with the package simulator (cached per box)."""
    sim = os.path.join(ROOT, "pcaone_b200", "bin", "pcaone-sim")
    bpr = (cfg["n"] + 3) // 4
    want = 3 + cfg["m"] * bpr
    if os.path.exists(out_prefix + ".bed") and os.path.getsize(out_prefix + ".bed") == want:
        return
    t = time.time()
    subprocess.check_call([sim, "--out", out_prefix, "--n", str(cfg["n"]), "--m", str(cfg["m"]),
                           "--pops", str(cfg["pops"]), "--fst-lo", str(cfg["fst"][0]),
                           "--fst-hi", str(cfg["fst"][1]), "--pmin", str(cfg["pmin"]),
                           "--pmax", str(cfg["pmax"]), "--miss", str(cfg["miss"]),
                           "--seed", str(cfg["seed"])])
    log(f"generated {out_prefix}.bed in {time.time() - t:.1f}s")


def write_sample(prefix, sample_prefix, nsnps):
    """First `nsnps` SNP records of a .bed as a standalone PLINK fileset."""
    import pcaone_b200 as pb

    packed, N, M = pb.read_bed(prefix)
    nsnps = min(nsnps, M)
    with open(sample_prefix + ".bed", "wb") as f:
        f.write(bytes([0x6C, 0x1B, 0x01]))
        f.write(np.ascontiguousarray(packed[:nsnps]).tobytes())
    with open(prefix + ".bim") as fi, open(sample_prefix + ".bim", "w") as fo:
        for i, line in enumerate(fi):
            if i >= nsnps:
                break
            fo.write(line)
    shutil.copy(prefix + ".fam", sample_prefix + ".fam")
    return N, nsnps


def run_reference_sample(cfg, prefix, workdir):
    """Time the reference PCAone binary on a bounded sample; returns a cpu_baseline dict."""
    ref = os.path.join(ROOT, "oracle", "_ref", "PCAone")
    if not os.path.exists(ref):
        return None, "reference binary oracle/_ref/PCAone not built"
    sp = os.path.join(workdir, "cpu_sample")
    N, ms = write_sample(prefix, sp, cfg["cpu_sample_snps"])
    cores = os.cpu_count() or 1
    args = [ref, "-b", sp, "-d", str(cfg["svd"]), "-k", str(cfg["k"]), "-n", str(cores),
            "-o", os.path.join(workdir, "cpu_out"), "-v", "1"]
    if cfg["svd"] == 2:
        args += ["-w", str(cfg["bands"])]
    else:
        args += ["-p", str(cfg["maxp"]), "--tol-rsvd", str(cfg["tol"])]
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    t = time.perf_counter()
    out = subprocess.run(args, capture_output=True, text=True, env=env)
    wall = time.perf_counter() - t
    if out.returncode != 0:
        return None, "reference run failed: " + out.stderr[-300:]
    epochs = None
    for line in out.stdout.splitlines():
        if "stops at epoch" in line:
            epochs = int(line.split("=")[-1])
    if epochs is None:
        epochs = cfg["maxp"] + 1
    bpr = (N + 3) // 4
    gbs = ms * bpr * epochs / wall / 1e9
    return {"value": round(gbs, 6), "unit": "bed GB/s", "cores": cores, "kind": "reference",
            "sample": f"{N} samples x {ms} SNPs (first SNPs of the workload), same flags, "
                      f"{epochs} epochs, {wall:.2f} s wall",
            "seconds": round(wall, 3), "epochs": epochs}, None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)], stdout=open(self.path, "w"),
                stderr=subprocess.DEVNULL)
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "samples": len(sm), "reasons": sorted(reasons)}


def peaks():
    try:
        with open(MEASURED_PEAKS) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return FALLBACK_PEAKS, "fallback"


def pinned_copy(packed):
    """The packed matrix in page-locked host memory (torch as the allocator)."""
    try:
        import torch

        t = torch.empty(packed.size, dtype=torch.uint8, pin_memory=True)
        a = t.numpy().reshape(packed.shape)
        a[:] = packed
        return a, t
    except Exception as e:  # no CUDA torch: fall back to pageable memory, say so
        log(f"pinned allocation unavailable ({e}); e2e uses pageable memory")
        return np.ascontiguousarray(packed), None


def run_ours(args, cfg):
    import pcaone_b200 as pb

    rank, world, local = dist_env()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    def barrier():
        if dist:
            dist.barrier()

    workdir = os.environ.get("PCAONE_BENCH_DIR", os.path.join(tempfile.gettempdir(), "pcaone_bench"))
    os.makedirs(workdir, exist_ok=True)
    prefix = os.path.join(workdir, args.config)
    if rank == 0:
        make_data(cfg, prefix)
    barrier()
    log("data ready")
    packed, N, M = pb.read_bed(prefix)
    bpr = (N + 3) // 4
    bed_bytes = M * bpr
    perm = pb.shuffle_perm(M) if cfg["svd"] == 2 else None
    log("bed read into host memory")
    rs_kw = dict(k=cfg["k"], oversamples=10, maxp=cfg["maxp"], svd=cfg["svd"], bands=cfg["bands"],
                 tol=cfg["tol"], seed=101)

    ctx = pb.GpuContext(local)
    ctx.load_bed(packed, N)
    if perm is not None:
        ctx.permute(perm)
    prec = args.precision
    log("loaded and permuted on the device")
    # warm-up (also builds the transposed copy and missing-entry lists once)
    for _ in range(args.warmup):
        r = ctx.rsvd(precision=prec, **rs_kw)
        log(f"warm-up step: {r.gpu_ms:.1f} ms, {r.epochs} epochs, {r.kernel_launches} launches")
    barrier()
    with ClockSampler(local) as clk:
        barrier()
        res = []
        for _ in range(args.steps):
            res.append(ctx.rsvd(precision=prec, **rs_kw))
        barrier()
    clocks = clk.summary()
    log(f"timed steps: {[round(r.gpu_ms, 2) for r in res]} ms")
    step_ms = [r.gpu_ms for r in res]
    epochs = res[-1].epochs
    ms_per_step = sum(step_ms) / len(step_ms)
    # max over ranks of the per-step time
    if dist:
        import torch

        t = torch.tensor([ms_per_step], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_per_step = float(t.item())
    gbs_rank = bed_bytes * epochs / (ms_per_step / 1e3) / 1e9
    value = gbs_rank * world

    # one profiled run: per-launch times of the decode-GEMM kernels (roofline)
    prof = ctx.rsvd(precision=prec, profile=True, **rs_kw)
    log(f"profiled step: gemm {prof.gemm_ms:.1f} of {prof.gpu_ms:.1f} ms over {prof.gemm_launches} launches; "
        f"epilogue {prof.epilogue_ms:.1f}, updates {prof.update_ms:.1f}, epoch tail {prof.tail_ms:.1f}")
    l = cfg["k"] + max(10, cfg["k"])
    alg_flops = 4.0 * M * N * l * prof.epochs  # two products per epoch, 2*M*N*l each
    gemm_avg_ms = prof.gemm_ms / max(prof.gemm_launches, 1)
    achieved_tflops = alg_flops / (prof.gemm_ms / 1e3) / 1e12
    pk, pk_kind = peaks()
    peak = pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))
    traffic = None  # DRAM bytes per launch from the committed ncu summary of this kernel
    tpath = os.path.join(ROOT, "profiles", "k_decode_gemm_tc_c2.md")
    if prec == "mixed" and args.config == "c2" and os.path.exists(tpath):
        with open(tpath) as f:
            mt = re.search(r"^traffic_bytes_per_launch:\s*([0-9]+)", f.read(), re.M)
        traffic = int(mt.group(1)) if mt else None
    roofline = {"bound": "tensor", "achieved": round(achieved_tflops, 2), "peak": peak,
                "unit": "TFLOP/s", "frac": round(achieved_tflops / peak, 4), "traffic": traffic,
                "peak_source": f"{pk_kind} bf16_tflops_sustained",
                "kernel": "k_decode_gemm_tc" if prec == "mixed" else "k_decode_gemm (SIMT)",
                "launches": prof.gemm_launches, "avg_launch_ms": round(gemm_avg_ms, 5),
                "algorithmic_flops_per_launch": alg_flops / max(prof.gemm_launches, 1),
                "issued_flops_factor": 2.0 if prec == "mixed" else 1.0,
                "gemm_share_of_step": round(prof.gemm_ms / prof.gpu_ms, 4),
                "step_breakdown_ms": {"gemm": round(prof.gemm_ms, 2), "epilogues": round(prof.epilogue_ms, 2),
                                      "omega_updates": round(prof.update_ms, 2),
                                      "epoch_tail": round(prof.tail_ms, 2), "total": round(prof.gpu_ms, 2)}}

    # comparison runs: the plain FP32 GPU path and the FP64 algorithm-matched path
    acc = {}
    fp32_ms = None
    if not args.skip_compare:
        r32 = ctx.rsvd(precision="fp32", **rs_kw)
        fp32_ms = r32.gpu_ms
        log(f"fp32 path: {r32.gpu_ms:.1f} ms")
        r64 = ctx.rsvd(precision="fp64", **rs_kw)
        log(f"fp64 path: {r64.gpu_ms:.1f} ms")
        e64 = r64.S ** 2
        for name, r in (("mixed" if prec == "mixed" else prec, res[-1]), ("fp32", r32)):
            e = r.S ** 2
            q1, _ = np.linalg.qr(r.U)
            q2, _ = np.linalg.qr(r64.U)
            ang = float(np.arccos(np.clip(np.linalg.svd(q1.T @ q2, compute_uv=False), -1, 1)).max())
            acc[name] = {"eig_rel_err_vs_fp64": float(np.max(np.abs(e / e64 - 1))),
                         "max_principal_angle_vs_fp64": ang, "epochs": r.epochs}
        acc["fp64_epochs"] = r64.epochs

    # e2e: host buffers -> device -> PCA -> host, through the C ABI
    pinned, keep = pinned_copy(packed)
    e2e_t = []
    for i in range(max(1, min(args.steps, 3)) + 1):
        t0 = time.perf_counter()
        ctx.load_bed(pinned, N)
        if perm is not None:
            ctx.permute(perm)
        r = ctx.rsvd(precision=prec, **rs_kw)
        t1 = time.perf_counter()
        if i > 0:  # first is warm-up (allocations)
            e2e_t.append(t1 - t0)
    e2e_s = sum(e2e_t) / len(e2e_t)
    log(f"e2e steps: {[round(x, 3) for x in e2e_t]} s")
    if dist:
        import torch

        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": round(bed_bytes * r.epochs / e2e_s / 1e9 * world, 4), "unit": "bed GB/s",
           "h2d_bytes_per_step": int(bed_bytes + (perm.nbytes if perm is not None else 0)),
           "d2h_bytes_per_step": int((N + M + 1) * cfg["k"] * 8),
           "seconds_per_pca": round(e2e_s, 4)}

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        cpu, why = run_reference_sample(cfg, prefix, workdir)
        log(f"cpu baseline: {cpu}")
        if cpu is None:
            cpu = {"value": None, "unavailable": why}
    ctx.close()
    if dist:
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": "top-k PCA bed GB/s (packed .bed bytes x epochs / s), mixed BF16 vs FP32 GPU path",
        "value": round(value, 4), "unit": "bed GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3),
        "pca_seconds": round(ms_per_step / 1e3, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16" if prec == "mixed" else prec,
        "data": "synthetic (seeded Balding-Nichols simulator)",
        "config": {"workload": cfg["workload"], "samples": N, "snps": M, "k": cfg["k"],
                   "oversamples": max(10, cfg["k"]), "windows": cfg["bands"] if cfg["svd"] == 2 else 1,
                   "svd": cfg["svd"], "epochs": epochs, "precision": prec,
                   "parallelism": f"replicas x{world}",
                   "l2": "inputs (2.5 GB packed) larger than L2; no flush needed"},
        "fp32_path_ms": round(fp32_ms, 3) if fp32_ms else None,
        "speedup_vs_fp32_path": round(fp32_ms / ms_per_step, 3) if fp32_ms else None,
        "accuracy": acc, "roofline": roofline, "e2e": e2e, "cpu_baseline": cpu,
        "gpu_launches": int(res[-1].kernel_launches), "clocks": clocks,
    }
    print(json.dumps(line), flush=True)


def run_reference_arm(args, cfg):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    workdir = os.environ.get("PCAONE_BENCH_DIR", os.path.join(tempfile.gettempdir(), "pcaone_bench"))
    os.makedirs(workdir, exist_ok=True)
    prefix = os.path.join(workdir, args.config)
    make_data(cfg, prefix)
    vals = []
    info = None
    for i in range(args.warmup + args.steps):
        cpu, why = run_reference_sample(cfg, prefix, workdir)
        if cpu is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return
        if i >= args.warmup:
            vals.append(cpu["value"])
            info = cpu
        if args.warmup + args.steps > 2 and i == 0 and cpu["seconds"] > 60:
            break  # keep the arm within a few minutes
    v = sum(vals) / len(vals) if vals else info["value"]
    print(json.dumps({
        "impl": "reference", "metric": "top-k PCA bed GB/s (packed .bed bytes x epochs / s), "
        "mixed BF16 vs FP32 GPU path", "value": round(v, 6), "unit": "bed GB/s", "n_gpus": world,
        "steps": len(vals), "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "dtype": "f64", "data": "synthetic (seeded Balding-Nichols simulator)",
        "config": {"workload": cfg["workload"], "sample": info["sample"]},
        "cpu_baseline": {"value": round(v, 6), "unit": "bed GB/s", "cores": info["cores"],
                         "kind": "reference", "sample": info["sample"]},
        "e2e": {"value": round(v, 6), "unit": "bed GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}), flush=True)


def run_profile_kernel(args, cfg):
    """Smallest command for ncu: one standardised product Z^T Omega through the C ABI on the
    configured matrix (the mixed path launches the tcgen05 decode-GEMM once), then exit. No
    child processes, no torch."""
    import pcaone_b200 as pb

    workdir = os.environ.get("PCAONE_BENCH_DIR", os.path.join(tempfile.gettempdir(), "pcaone_bench"))
    os.makedirs(workdir, exist_ok=True)
    prefix = os.path.join(workdir, args.config)
    make_data(cfg, prefix)
    packed, N, M = pb.read_bed(prefix)
    l = cfg["k"] + max(10, cfg["k"])
    B = pb.omega(101, N, l)
    with pb.GpuContext(0) as ctx:
        ctx.load_bed(packed, N)
        for _ in range(args.steps):
            out = ctx.product_t(B, precision=args.precision)
    print(json.dumps({"profile_kernel": args.precision, "samples": N, "snps": M, "l": l,
                      "checksum": float(np.abs(out).sum())}))


def run_profile_step(args, cfg):
    """Small command for ncu: --steps RSVD runs of the configured workload through the C ABI
    (load, shuffle, then the full power iteration), then exit. No child processes, no torch."""
    import pcaone_b200 as pb

    workdir = os.environ.get("PCAONE_BENCH_DIR", os.path.join(tempfile.gettempdir(), "pcaone_bench"))
    os.makedirs(workdir, exist_ok=True)
    prefix = os.path.join(workdir, args.config)
    make_data(cfg, prefix)
    packed, N, M = pb.read_bed(prefix)
    rs_kw = dict(k=cfg["k"], oversamples=10, maxp=cfg["maxp"], svd=cfg["svd"], bands=cfg["bands"],
                 tol=cfg["tol"], seed=101)
    with pb.GpuContext(0) as ctx:
        ctx.load_bed(packed, N)
        if cfg["svd"] == 2:
            ctx.permute(pb.shuffle_perm(M))
        for _ in range(args.steps):
            r = ctx.rsvd(precision=args.precision, **rs_kw)
    print(json.dumps({"profile_step": args.precision, "samples": N, "snps": M, "epochs": r.epochs,
                      "launches": r.kernel_launches, "gpu_ms": r.gpu_ms}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIGS))
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp32", "fp64"])
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-compare", action="store_true")
    ap.add_argument("--profile-kernel", action="store_true",
                    help="run --steps products Z^T Omega only (a small command for ncu)")
    ap.add_argument("--profile-step", action="store_true",
                    help="run --steps RSVDs of the config only (a small command for ncu)")
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    if args.profile_kernel:
        run_profile_kernel(args, cfg)
    elif args.profile_step:
        run_profile_step(args, cfg)
    elif args.impl == "reference":
        run_reference_arm(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
