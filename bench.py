"""Benchmark of the PCAone B200 hot path.

Default workload (config c2, the headline): window-based RSVD (--svd 2) of a PLINK .bed of
20,000 samples x 500,000 SNPs, 5 Balding-Nichols populations (Fst ~ U(0.01, 0.1) per
population, ancestral allele frequency ~ U(0.01, 0.5)), HWE genotypes, 0.5% of entries
missing completely at random; k = 20 (l = 40), 64 windows, the reference's default flags
otherwise (maxp 20, tol 1e-4, seed 101, in-core SNP shuffle). Data are synthetic, generated by
the package's seeded simulator (pcaone_b200/bin/pcaone-sim).

Other configurations (--config): c1 (Halko k=10 p=7, 2000 x 50000), c3 (EMU k=10 up to 50 EM
iterations, 10000 x 200000 admixed, Beta(2,18) per-sample missingness), c4 (PCAngsd k=6 on
genotype likelihoods, 5000 x 200000 sites, depth ~ Poisson(4), error 0.01).

One step = one full run of the configuration through the C ABI with the inputs resident in
device memory: all power-iteration epochs of one top-k PCA (c1, c2), or the whole EM loop
(c3, c4).
  value : c1-c3: bed GB/s = packed .bed bytes x epochs / step time; c4: GL GB/s = FP32
          likelihood-pair bytes x likelihood passes / step time. c1, c2: device time from CUDA
          events on the library's stream; c3, c4: host time around the EM loop, whose every
          library call synchronises (the loop's convergence test runs on the host).
  e2e   : the same metric from host buffers: every step uploads the inputs from pinned memory
          (and permutes them on the device), runs the step and reads U, S, V back.
The inputs are larger than L2 (126 MB), so no L2 flush is needed between steps.

--impl reference times the reference PCAone (built from its own sources into oracle/_ref) on
the host cores on bounded samples of the same workload (all samples, slices of SNPs); with
several slice sizes it fits the wall time per pass and reports the rate at the full size.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# CPU slices hold at least 64 x 64 SNPs: with fewer SNPs per window than windows the reference
# winSVD fails (std::bad_alloc), so no 64-window slice is smaller than 4096 SNPs.
BN5 = ["--pops", "5", "--fst-lo", "0.01", "--fst-hi", "0.1", "--pmin", "0.01", "--pmax", "0.5"]
CONFIGS = {
    "c2": dict(kind="rsvd", workload="winSVD k=20, 64 windows, 20000 samples x 500000 SNPs, 5 BN pops",
               n=20000, m=500000, sim=BN5 + ["--miss", "0.005", "--seed", "2"],
               k=20, svd=2, bands=64, maxp=20, tol=1e-4, cpu_fit_snps=(4096, 8192, 16384)),
    # profiling-size case of c2 (packed matrix 250 MB > L2), same shapes per window row/column
    "c2s": dict(kind="rsvd", workload="winSVD k=20, 64 windows, 20000 samples x 50000 SNPs, 5 BN pops",
                n=20000, m=50000, sim=BN5 + ["--miss", "0.005", "--seed", "2"],
                k=20, svd=2, bands=64, maxp=20, tol=1e-4, cpu_fit_snps=(4096, 8192, 16384)),
    "c1": dict(kind="rsvd", workload="Halko k=10 p=7, 2000 samples x 50000 SNPs, 3 BN pops",
               n=2000, m=50000, sim=["--pops", "3", "--fst-lo", "0.05", "--fst-hi", "0.05", "--pmin", "0.05",
                                     "--pmax", "0.5", "--miss", "0.01", "--seed", "1"],
               k=10, svd=1, bands=64, maxp=7, tol=0.0, cpu_fit_snps=(50000,)),
    "c3": dict(kind="emu", workload="EMU k=10, up to 50 EM iterations (tol-em 5e-7), 10000 samples x 200000 "
                                    "SNPs, 4 admixed pops (Dirichlet 0.5), per-sample missing rate ~ Beta(2,18)",
               n=10000, m=200000, sim=["--pops", "4", "--fst-lo", "0.02", "--fst-hi", "0.1", "--pmin", "0.01",
                                       "--pmax", "0.5", "--admix", "0.5", "--miss-beta", "2,18", "--seed", "3"],
               k=10, svd=2, bands=64, maxp=20, tol=1e-4, maxiter=50, tolem=5e-7, cpu_fit_snps=(4096, 8192)),
    "c4": dict(kind="pcangsd", workload="PCAngsd k=6 on genotype likelihoods, 5000 samples x 200000 sites, "
                                        "3 pops, depth ~ Poisson(4), error 0.01, unshuffled (-S)",
               n=5000, m=200000, sim=["--pops", "3", "--fst-lo", "0.05", "--fst-hi", "0.1", "--pmin", "0.05",
                                      "--pmax", "0.5", "--beagle", "4,0.01", "--seed", "4"],
               k=6, svd=2, bands=64, maxp=20, tol=1e-4, maxiter=100, tolem=1e-5, cpu_fit_snps=(4096, 8192)),
    "c5": dict(kind="ld", workload="LD r2 of every pair in 1 Mb windows (flow A: genotypes projected off the top 10 "
                                    "PCs), 10000 samples x 300000 SNPs, about 100-1900 SNPs per window, Markov "
                                    "haplotype LD (switch 0.01)",
               n=10000, m=300000, sim=["--pops", "3", "--fst-lo", "0.05", "--fst-hi", "0.1", "--pmin", "0.05",
                                       "--pmax", "0.5", "--miss", "0.01", "--bp-spacing", "1000",
                                       "--ld-switch", "0.01", "--seed", "5"],
               k=10, ld_bp=1000000, svd=1, maxp=7, tol=0.0, bands=64, cpu_fit_snps=(3000, 6000)),
}

METRIC = ("top-k PCA bed GB/s (packed .bed bytes x epochs / s), int8/BF16 tensor-core vs FP32 GPU "
          "path at matched eigval error")
METRIC_GL = "PCAngsd GL GB/s (FP32 likelihood-pair bytes x likelihood passes / s)"
METRIC_LD = "LD r2 pairs per second (every SNP pair of the --ld-bp windows, genotypes projected off the top k PCs)"
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "PCAone")
SIM = os.path.join(ROOT, "pcaone_b200", "bin", "pcaone-sim")
DTYPE = {"mixed": "int8 (3-piece fixed-point sketch, int32 accumulation)",
         "bf16": "bf16 (split hi+lo sketch, fp32 accumulation)",
         "int8": "int8 (exact integer genotype Gram, int32 accumulation; FP64 projection and normalisation)"}

_T0 = time.time()


def log(*a):
    print(f"[{time.time() - _T0:8.1f}s]", *a, file=sys.stderr, flush=True)


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), \
        int(os.environ.get("LOCAL_RANK", 0))


def workdir():
    d = os.environ.get("PCAONE_BENCH_DIR", os.path.join(tempfile.gettempdir(), "pcaone_bench"))
    os.makedirs(d, exist_ok=True)
    return d


def make_data(cfg, prefix, m=None, text_gl=False):
    """Generate the synthetic inputs with the package simulator (cached per box). PLINK
    configs write prefix.bed/.bim/.fam; c4 writes prefix.gl.f32 (binary likelihood pairs), or
    prefix.beagle.gz when text_gl (the reference's input, for its CPU samples)."""
    m = m or cfg["m"]
    n = cfg["n"]
    args = [SIM, "--out", prefix, "--n", str(n), "--m", str(m)] + cfg["sim"]
    if cfg["kind"] == "pcangsd":
        if text_gl:
            path, want = prefix + ".beagle.gz", None
        else:
            path, want = prefix + ".gl.f32", m * 2 * n * 4
            args.append("--gl-bin")
    else:
        path, want = prefix + ".bed", 3 + m * ((n + 3) // 4)
    if os.path.exists(path) and (want is None or os.path.getsize(path) == want):
        return
    t = time.time()
    subprocess.check_call(args)
    log(f"generated {path} in {time.time() - t:.1f}s")


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


def reference_run(cfg, prefix, wd, nsnps):
    """One run of the reference binary on the first nsnps SNPs (sites) of the workload, all
    cores. Returns dict(seconds, epochs, sweeps, snps, samples, cores); raises RuntimeError."""
    if not os.path.exists(REF_BIN):
        raise RuntimeError("reference binary oracle/_ref/PCAone not built")
    cores = os.cpu_count() or 1
    sp = os.path.join(wd, f"ref_sample_{cfg['kind']}_{cfg['n']}_{nsnps}")
    kind = cfg["kind"]
    if kind == "pcangsd":
        make_data(cfg, sp, m=nsnps, text_gl=True)
        N = cfg["n"]
        args = [REF_BIN, "-G", sp + ".beagle.gz", "-k", str(cfg["k"]), "-S", "-w", str(cfg["bands"]),
                "--maxiter", str(cfg["maxiter"]), "--tol-em", str(cfg["tolem"])]
    elif kind == "ld":
        N, nsnps = write_sample(prefix, sp, nsnps)
        # the projection factors come from the reference's own PCA of the slice (not timed)
        subprocess.run([REF_BIN, "-b", sp, "-k", str(cfg["k"]), "-d", "1", "-p", "3", "-n", str(cores), "-o",
                        sp + "_pcs", "-v", "0"], check=True, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL,
                       env=dict(os.environ, OMP_NUM_THREADS=str(cores)))
        args = [REF_BIN, "-b", sp, "--read-U", sp + "_pcs.eigvecs", "--ld-bp", str(cfg["ld_bp"]), "-R"]
    else:
        N, nsnps = write_sample(prefix, sp, nsnps)
        args = [REF_BIN, "-b", sp, "-k", str(cfg["k"])]
        if kind == "emu":
            args += ["--emu", "-w", str(cfg["bands"]), "--maxiter", str(cfg["maxiter"]), "--tol-em", str(cfg["tolem"])]
        elif cfg["svd"] == 2:
            args += ["-d", "2", "-w", str(cfg["bands"])]
        else:
            args += ["-d", "1", "-p", str(cfg["maxp"]), "--tol-rsvd", str(cfg["tol"])]
    args += ["-n", str(cores), "-o", os.path.join(wd, "cpu_out"), "-v", "1"]
    env = dict(os.environ, OMP_NUM_THREADS=str(cores))
    t = time.perf_counter()
    # PCAngsd: timed from the start (text parse, allele-frequency EM, EM-PCA) to the "estimate
    # GRM" line; the N x N Jacobi SVD after it is not part of the timed work, so the process is
    # stopped there
    proc = subprocess.Popen(args, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True, env=env)
    epochs, sweeps, lines = 0, 0, []
    for line in proc.stdout:
        lines.append(line)
        if "stops at epoch" in line:
            epochs += int(line.split("=")[-1])
        if "individual allele frequencies estimated" in line:
            sweeps += 1
        if kind == "pcangsd" and "estimate GRM" in line:
            break
    wall = time.perf_counter() - t
    if kind == "pcangsd":
        proc.kill()
    rc = proc.wait()
    if kind != "pcangsd" and rc != 0:
        raise RuntimeError("reference run failed: " + "".join(lines[-5:])[-300:])
    if kind == "rsvd" and epochs == 0:
        epochs = cfg["maxp"] + 1
    pairs = 0
    if kind == "ld":
        import pcaone_b200 as pb

        pos, ends = pb.read_bim_positions(sp + ".bim")
        pairs = int((pb.ld_windows(pos, ends, cfg["ld_bp"])[1] - 1).sum())
    # likelihood passes of PCAngsd: the initial posterior and one per EM iteration
    return {"seconds": wall, "epochs": epochs, "sweeps": sweeps + 1, "snps": nsnps, "samples": N, "cores": cores,
            "pairs": pairs}


def unit_bytes(cfg, nsnps):
    """Bytes of one pass over the input: packed .bed records, or FP32 likelihood pairs."""
    if cfg["kind"] == "pcangsd":
        return nsnps * 2 * cfg["n"] * 4
    return nsnps * ((cfg["n"] + 3) // 4)


def passes_of(cfg, r):
    return r["sweeps"] if cfg["kind"] == "pcangsd" else r["epochs"]


def fitted_rate_ld(cfg, runs, full_pairs):
    """LD pairs per second of the reference from its runs on SNP slices: wall time fitted as
    a + b * pairs over the slices and evaluated at the full workload's pairs (one slice: its
    own rate)."""
    x = np.array([r["pairs"] for r in runs], dtype=float)
    y = np.array([r["seconds"] for r in runs])
    desc = "; ".join(f"{r['samples']} x {r['snps']}: {r['pairs']} pairs in {r['seconds']:.2f} s" for r in runs)
    if len(set(x)) > 1:
        b, a = np.polyfit(x, y, 1)
        value = full_pairs / (a + b * full_pairs)
        sample = (f"wall time (text .ld.gz output included) fitted as a + b * pairs over [{desc}] "
                  f"(a = {a:.4g} s, b = {b:.4g} s/pair) and evaluated at {full_pairs} pairs")
    else:
        value = float(np.mean(x / y))
        sample = desc + " (a slice of the workload)"
    return value, sample


def full_ld_pairs(cfg, prefix):
    import pcaone_b200 as pb

    pos, ends = pb.read_bim_positions(prefix + ".bim")
    ws, we = pb.ld_windows(pos, ends, cfg["ld_bp"])
    return ws, we, int((we - 1).sum())


def fitted_rate(cfg, runs):
    """Rate of the metric from reference runs: with several slice sizes, wall time per pass is
    fitted as a + b * SNPs (least squares) and evaluated at the full size; one size is used
    as measured."""
    passes = [passes_of(cfg, r) for r in runs]
    x = np.array([r["snps"] for r in runs], dtype=float)
    yp = np.array([r["seconds"] for r in runs]) / np.array(passes)
    desc = "; ".join(f"{r['samples']} x {r['snps']}: {r['seconds']:.2f} s, {p} passes" for r, p in zip(runs, passes))
    if len(set(x)) > 1:
        b, a = np.polyfit(x, yp, 1)
        value = unit_bytes(cfg, cfg["m"]) / (a + b * cfg["m"]) / 1e9
        sample = (f"wall time per pass fitted as a + b * SNPs over [{desc}] (a = {a:.4g} s, b = {b:.4g} s/SNP) "
                  f"and evaluated at {cfg['m']} SNPs")
    else:
        value = float(np.mean([unit_bytes(cfg, r["snps"]) * p / r["seconds"] for r, p in zip(runs, passes)])) / 1e9
        sample = desc + ("" if int(x[0]) == cfg["m"] else f" (a slice of the {cfg['m']}-SNP workload)")
    return value, sample


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


def pinned_copy(arr):
    """A copy of arr in page-locked host memory (torch as the allocator)."""
    try:
        import torch

        t = torch.empty(arr.nbytes, dtype=torch.uint8, pin_memory=True)
        a = t.numpy().view(arr.dtype).reshape(arr.shape)
        a[:] = arr
        return a, t
    except Exception as e:  # no CUDA torch: fall back to pageable memory, say so
        log(f"pinned allocation unavailable ({e}); e2e uses pageable memory")
        return np.ascontiguousarray(arr), None


def capture_traffic(profile, alg_bytes_per_launch):
    """DRAM traffic per launch scaled from a committed ncu summary of a smaller case of the same
    kernel (its `traffic_bytes_per_launch` over its `algorithmic_bytes_per_launch`, both read
    from the capture): the kernel's traffic grows with the packed bytes it streams."""
    path = os.path.join(ROOT, "profiles", profile)
    try:
        vals = {}
        for line in open(path):
            for key in ("traffic_bytes_per_launch", "algorithmic_bytes_per_launch"):
                if line.startswith(key + ":"):
                    vals[key] = float(line.split(":")[1])
        ratio = vals["traffic_bytes_per_launch"] / vals["algorithmic_bytes_per_launch"]
    except (OSError, KeyError, ValueError):
        return None, None
    return int(alg_bytes_per_launch * ratio), f"profiles/{profile}: ncu capture of a smaller case, " \
        f"traffic / algorithmic bytes = {ratio:.3f}, scaled to this launch size"


def tensor_roofline(prec, l, alg_flops, prof):
    """Roofline of the dominant decode-GEMM from one profiled run (CUDA events around every
    decode-GEMM launch on the library's stream)."""
    achieved = alg_flops / (prof.gemm_ms / 1e3) / 1e12
    pk, pk_kind = peaks()
    peak = pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))
    # issued tensor work per algorithmic flop: int8 issues three pieces on NP = 3 * round_up(l, 8)
    # rounded to 16 accumulator columns at twice the BF16 rate; split BF16 issues NP = 2l -> 16
    np8 = (3 * ((l + 7) // 8 * 8) + 15) // 16 * 16
    npbf = (2 * l + 15) // 16 * 16
    issued = {"mixed": np8 / l, "bf16": npbf / l}.get(prec, 1.0)
    rate = {"mixed": 2.0, "bf16": 1.0}.get(prec, 1.0)
    return {"bound": "tensor", "achieved": round(achieved, 2), "peak": peak, "unit": "TFLOP/s",
            "frac": round(achieved / peak, 4), "traffic": None,
            "peak_source": f"{pk_kind} bf16_tflops_sustained",
            "kernel": {"mixed": "k_decode_gemm_i8", "bf16": "k_decode_gemm_tc"}.get(prec, "k_decode_gemm (SIMT)"),
            "launches": prof.gemm_launches, "avg_launch_ms": round(prof.gemm_ms / max(prof.gemm_launches, 1), 5),
            "algorithmic_flops_per_launch": alg_flops / max(prof.gemm_launches, 1),
            "issued_ops_factor": round(issued, 4), "ceiling_frac_of_bf16_peak": round(rate / issued, 4),
            "gemm_share_of_step": round(prof.gemm_ms / prof.gpu_ms, 4),
            "step_breakdown_ms": {"gemm": round(prof.gemm_ms, 2), "epilogues": round(prof.epilogue_ms, 2),
                                  "omega_updates": round(prof.update_ms, 2), "epoch_tail": round(prof.tail_ms, 2),
                                  "waiting_for_host": round(prof.host_ms, 2), "total": round(prof.gpu_ms, 2)}}


def subspace_err(Ua, Sa, Ub, Sb, k=None):
    """Largest eigenvalue relative error and largest principal angle of the first k PCs."""
    k = k or len(Sa)
    e = np.abs(Sa[:k] ** 2 / Sb[:k] ** 2 - 1)
    q1, _ = np.linalg.qr(Ua[:, :k])
    q2, _ = np.linalg.qr(Ub[:, :k])
    ang = float(np.arccos(np.clip(np.linalg.svd(q1.T @ q2, compute_uv=False), -1, 1)).max())
    return float(e.max()), ang


class Run:
    """Process-group plumbing shared by the configurations (replicas, max over ranks)."""

    def __init__(self):
        self.rank, self.world, self.local = dist_env()
        self.dist = None
        self.device = "cpu"
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            # NCCL between the GPUs; gloo on hosts without one (the CPU tests of this plumbing)
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                self.device = "cuda"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.dist = dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max_over_ranks(self, x):
        if not self.dist:
            return x
        import torch

        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()


def prepare(cfg, config, run):
    wd = workdir()
    prefix = os.path.join(wd, config)
    if run.rank == 0:
        make_data(cfg, prefix)
    run.barrier()
    log("data ready")
    return wd, prefix


def run_rsvd_cfg(args, cfg, run):
    import pcaone_b200 as pb

    wd, prefix = prepare(cfg, args.config, run)
    packed, N, M = pb.read_bed(prefix)
    bed_bytes = M * ((N + 3) // 4)
    perm = pb.shuffle_perm(M) if cfg["svd"] == 2 else None
    rs_kw = dict(k=cfg["k"], oversamples=10, maxp=cfg["maxp"], svd=cfg["svd"], bands=cfg["bands"],
                 tol=cfg["tol"], seed=101)
    ctx = pb.GpuContext(run.local)
    ctx.load_bed(packed, N)
    if perm is not None:
        ctx.permute(perm)
    prec = args.precision
    log("loaded and permuted on the device")
    for _ in range(args.warmup):  # also builds the transposed copy and missing-entry lists once
        r = ctx.rsvd(precision=prec, **rs_kw)
        log(f"warm-up step: {r.gpu_ms:.1f} ms, {r.epochs} epochs, {r.kernel_launches} launches")
    run.barrier()
    with ClockSampler(run.local) as clk:
        run.barrier()
        res = [ctx.rsvd(precision=prec, **rs_kw) for _ in range(args.steps)]
        run.barrier()
    clocks = clk.summary()
    log(f"timed steps: {[round(r.gpu_ms, 2) for r in res]} ms")
    epochs = res[-1].epochs
    ms_per_step = run.max_over_ranks(sum(r.gpu_ms for r in res) / len(res))
    value = bed_bytes * epochs / (ms_per_step / 1e3) / 1e9 * run.world

    prof = ctx.rsvd(precision=prec, profile=True, **rs_kw)
    log(f"profiled step: gemm {prof.gemm_ms:.1f} of {prof.gpu_ms:.1f} ms over {prof.gemm_launches} launches; "
        f"epilogue {prof.epilogue_ms:.1f}, updates {prof.update_ms:.1f}, epoch tail {prof.tail_ms:.1f}")
    l = cfg["k"] + max(10, cfg["k"])
    roofline = tensor_roofline(prec, l, 4.0 * M * N * l * prof.epochs, prof)
    if prec == "mixed":  # each product streams the packed matrix once: 2 per epoch
        alg_b = 2.0 * bed_bytes * prof.epochs / max(prof.gemm_launches, 1)
        roofline["algorithmic_bytes_per_launch"] = int(alg_b)
        roofline["traffic"], roofline["traffic_source"] = capture_traffic("k_decode_gemm_i8_c2s.md", alg_b)

    acc, extra = {}, {}
    if not args.skip_compare:
        comp = {}
        for p2 in ("fp32", "bf16", "fp64"):
            if p2 != prec:
                comp[p2] = ctx.rsvd(precision=p2, **rs_kw)
                log(f"{p2} path: {comp[p2].gpu_ms:.1f} ms")
        r64 = comp.get("fp64", res[-1])
        runs = [(prec, res[-1])] + [(k2, v) for k2, v in comp.items() if k2 != "fp64"]
        for name, r in runs:
            e, a = subspace_err(r.U, r.S, r64.U, r64.S)
            acc[name] = {"eig_rel_err_vs_fp64": e, "max_principal_angle_vs_fp64": a, "epochs": r.epochs}
        # dense FP64 oracle for the population PCs (well separated from the noise): an FP64
        # Halko sketch of width 40 iterated for 40 epochs on the whole matrix
        pops = int(cfg["sim"][cfg["sim"].index("--pops") + 1])
        g = max(1, pops - 1)
        dense = ctx.rsvd(precision="fp64", k=max(cfg["k"], g), oversamples=40 - max(cfg["k"], g), maxp=39,
                         svd=1, tol=0.0, seed=7, want_v=False)
        log(f"dense FP64 reference for PCs 1-{g}: {dense.gpu_ms:.1f} ms")
        for name, r in runs + [("fp64", r64)]:
            e, a = subspace_err(r.U, r.S, dense.U, dense.S, g)
            acc.setdefault(name, {}).update({f"eig_rel_err_pcs1_{g}_vs_dense_fp64": e,
                                             f"max_angle_pcs1_{g}_vs_dense_fp64": a})
        for p2 in ("fp32", "bf16"):
            if p2 in comp:
                extra[f"{p2}_path_ms"] = round(comp[p2].gpu_ms, 3)
        if "fp32" in comp:
            extra["speedup_vs_fp32_path"] = round(comp["fp32"].gpu_ms / ms_per_step, 3)
            # the FP32 SIMT path's own rate: algorithmic flops of its products over its whole step
            extra["fp32_path_tflops_algorithmic"] = round(
                4.0 * M * N * l * comp["fp32"].epochs / (comp["fp32"].gpu_ms / 1e3) / 1e12, 2)

    # e2e: pinned host buffers -> device -> PCA -> host, through the C ABI
    pinned, keep = pinned_copy(packed)
    e2e_t = []
    for i in range(max(1, min(args.steps, 3)) + 1):
        t0 = time.perf_counter()
        ctx.load_bed(pinned, N)
        if perm is not None:
            ctx.permute(perm)
        r = ctx.rsvd(precision=prec, **rs_kw)
        t1 = time.perf_counter()
        if i > 0:  # the first is a warm-up (allocations)
            e2e_t.append(t1 - t0)
    log(f"e2e steps: {[round(x, 3) for x in e2e_t]} s")
    e2e_s = run.max_over_ranks(sum(e2e_t) / len(e2e_t))
    e2e = {"value": round(bed_bytes * r.epochs / e2e_s / 1e9 * run.world, 4), "unit": "bed GB/s",
           "h2d_bytes_per_step": int(bed_bytes + (perm.nbytes if perm is not None else 0)),
           "d2h_bytes_per_step": int((N + M + 1) * cfg["k"] * 8), "seconds_per_pca": round(e2e_s, 4)}
    launches = int(res[-1].kernel_launches)
    if cfg["svd"] == 2 and not args.skip_compare:
        extra["streamed"] = streamed_rsvd(ctx, packed, N, perm, prec, rs_kw, bed_bytes, res[-1])
    ctx.close()
    cpu = cpu_baseline(args, cfg, prefix, wd, run)
    run.close()
    if run.rank != 0:
        return
    emit(args, cfg, run, value, "bed GB/s", ms_per_step, prec, clocks, roofline, e2e, cpu, launches,
         {"samples": N, "snps": M, "k": cfg["k"], "oversamples": max(10, cfg["k"]),
          "windows": cfg["bands"] if cfg["svd"] == 2 else 1, "svd": cfg["svd"], "epochs": epochs},
         dict(extra, pca_seconds=round(ms_per_step / 1e3, 5), accuracy=acc))


def streamed_rsvd(ctx, packed, N, perm, prec, rs_kw, bed_bytes, resident):
    """The same PCA with the genotypes in pinned host memory (pcaone_gpu_load_bed_host, the
    out-of-core mode): every epoch copies the windows into two 1 GiB device slots over PCIe
    while the other slot's products run. Device time per PCA, the H2D bytes it moved and their
    rate, and the eigenvalue difference to the resident run."""
    ctx.load_bed_host(packed, N)
    if perm is not None:
        ctx.permute(perm)
    for _ in range(2):
        ctx.rsvd(precision=prec, **rs_kw)
    rs = [ctx.rsvd(precision=prec, **rs_kw) for _ in range(3)]
    ms = sum(r.gpu_ms for r in rs) / len(rs)
    h2d = int(rs[-1].h2d_bytes)
    out = {"ms_per_pca": round(ms, 2), "epochs": rs[-1].epochs, "h2d_bytes_per_pca": h2d,
           "h2d_gbs": round(h2d / (ms / 1e3) / 1e9, 2),
           "value_bed_gbs": round(bed_bytes * rs[-1].epochs / (ms / 1e3) / 1e9, 3),
           "eig_rel_err_vs_resident": float(np.max(np.abs(rs[-1].S ** 2 / resident.S ** 2 - 1))),
           "slots": "2 x 1 GiB (records, sample-major copy, int8 tiles of the windows they hold)"}
    log(f"streamed: {out}")
    return out


def run_emu_cfg(args, cfg, run):
    import pcaone_b200 as pb

    wd, prefix = prepare(cfg, args.config, run)
    packed, N, M = pb.read_bed(prefix)
    bed_bytes = M * ((N + 3) // 4)
    perm = pb.shuffle_perm(M)
    kw = dict(k=cfg["k"], svd=2, bands=cfg["bands"], maxp=cfg["maxp"], tol=cfg["tol"], maxiter=cfg["maxiter"],
              tolem=cfg["tolem"])
    prec = args.precision
    ctx = pb.GpuContext(run.local)
    ctx.load_bed(packed, N)
    ctx.permute(perm)
    for _ in range(args.warmup):
        t0 = time.perf_counter()
        out = pb.emu_loop(ctx, precision=prec, **kw)
        log(f"warm-up EMU: {time.perf_counter() - t0:.2f} s, {out[4]} iterations, {out[5]} epochs")
    run.barrier()
    times, outs = [], []
    with ClockSampler(run.local) as clk:
        run.barrier()
        for _ in range(args.steps):
            t0 = time.perf_counter()
            outs.append(pb.emu_loop(ctx, precision=prec, **kw))
            times.append(time.perf_counter() - t0)
        run.barrier()
    clocks = clk.summary()
    log(f"timed EMU runs: {[round(t, 3) for t in times]} s")
    sec = run.max_over_ranks(sum(times) / len(times))
    eig, S, U, V, it, epochs = outs[-1]
    value = bed_bytes * epochs / sec / 1e9 * run.world
    # roofline of the decode-GEMM inside the EM loop: one profiled RSVD with the imputed values
    # of the final factors active
    ctx.fit_emu(U, S, V, True)
    l = cfg["k"] + max(10, cfg["k"])
    prof = ctx.rsvd(k=cfg["k"], maxp=cfg["maxp"], svd=2, bands=cfg["bands"], tol=cfg["tol"], precision=prec,
                    standardize=False, carry=True, profile=True)
    ctx.clear_imputed()
    roofline = tensor_roofline(prec, l, 4.0 * M * N * l * prof.epochs, prof)
    acc = {}
    if not args.skip_compare:
        o64 = pb.emu_loop(ctx, precision="fp64", **kw)
        e, a = subspace_err(U, S, o64[2], o64[1])
        # the populations' PCs (4 admixed populations: PCs 1-3) carry the structure; the rest
        # are noise PCs with near-equal eigenvalues
        npc = int(cfg["sim"][cfg["sim"].index("--pops") + 1]) - 1
        e3, a3 = subspace_err(U, S, o64[2], o64[1], k=npc)
        acc = {prec: {"eig_rel_err_vs_fp64": e, "max_principal_angle_vs_fp64": a, "iterations": it,
                      f"eig_rel_err_pcs1_{npc}_vs_fp64": e3, f"max_angle_pcs1_{npc}_vs_fp64": a3},
               "fp64_iterations": o64[4]}
    pinned, keep = pinned_copy(packed)
    e2e_t = []
    for i in range(2):
        t0 = time.perf_counter()
        ctx.load_bed(pinned, N)
        ctx.permute(perm)
        o = pb.emu_loop(ctx, precision=prec, **kw)
        if i > 0:
            e2e_t.append(time.perf_counter() - t0)
    e2e_s = run.max_over_ranks(e2e_t[0])
    e2e = {"value": round(bed_bytes * o[5] / e2e_s / 1e9 * run.world, 4), "unit": "bed GB/s",
           "h2d_bytes_per_step": int(bed_bytes + perm.nbytes), "d2h_bytes_per_step": int((N + M + 1) * cfg["k"] * 8),
           "seconds_per_emu": round(e2e_s, 3)}
    ctx.close()
    cpu = cpu_baseline(args, cfg, prefix, wd, run)
    run.close()
    if run.rank != 0:
        return
    emit(args, cfg, run, value, "bed GB/s", sec * 1e3, prec, clocks, roofline, e2e, cpu, None,
         {"samples": N, "snps": M, "k": cfg["k"], "windows": cfg["bands"], "em_iterations": it,
          "epochs_total": epochs},
         {"emu_seconds": round(sec, 4), "accuracy": acc,
          "timing": "host clock around the EM loop (every library call synchronises)"})


def run_pcangsd_cfg(args, cfg, run):
    import pcaone_b200 as pb

    wd, prefix = prepare(cfg, args.config, run)
    N, M = cfg["n"], cfg["m"]
    P = np.fromfile(prefix + ".gl.f32", dtype=np.float32).reshape(M, 2 * N)  # = 2N x M column-major
    gl_bytes = P.nbytes
    k, bands = cfg["k"], cfg["bands"]
    ident = np.arange(M, dtype=np.int32)
    ctx = pb.GpuContext(run.local)
    ctx.load_gl(P.T)
    log("likelihoods loaded")

    def step():
        F, it_maf = ctx.gl_freq(cfg["maxiter"], 1e-6)
        ctx.gl_update()
        out = pb._pcangsd_em(ctx, ident, F, k, 2, bands, cfg["maxp"], 10, cfg["tol"], cfg["maxiter"],
                             cfg["tolem"], 101, 1, True, False)
        return out, it_maf

    for _ in range(args.warmup):
        t0 = time.perf_counter()
        out, itm = step()
        log(f"warm-up PCAngsd: {time.perf_counter() - t0:.2f} s, {out[4]} EM iterations, {itm} MAF sweeps")
    run.barrier()
    times = []
    with ClockSampler(run.local) as clk:
        run.barrier()
        for _ in range(args.steps):
            t0 = time.perf_counter()
            out, itm = step()
            times.append(time.perf_counter() - t0)
        run.barrier()
    clocks = clk.summary()
    log(f"timed PCAngsd runs: {[round(t, 3) for t in times]} s")
    sec = run.max_over_ranks(sum(times) / len(times))
    # likelihood passes counted as for the reference: the initial posterior and one posterior
    # per EM iteration (the allele-frequency EM sweeps are timed but not counted)
    passes = 1 + out[4]
    value = gl_bytes * passes / sec / 1e9 * run.world
    # HBM roofline of the posterior kernel: P read (FP64 pairs, 16 N bytes a site) + E write
    # (4 Npad bytes), device time of the kernel (CUDA events on the library's stream)
    reps = 5
    dev_ms, host_ms = [], []
    for _ in range(reps):
        t0 = time.perf_counter()
        ctx.gl_update(out[2], out[1], out[3])
        host_ms.append((time.perf_counter() - t0) * 1e3)
        dev_ms.append(ctx.gl_timing())
    upd_s = sum(dev_ms) / reps / 1e3
    npad = (N + 255) // 256 * 256
    alg = M * (16 * N + 4 * npad)
    pk, pk_kind = peaks()
    roofline = {"bound": "hbm", "achieved": round(alg / upd_s / 1e9, 1), "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": round(alg / upd_s / 1e9 / pk["hbm_gbs"], 4), "traffic": None,
                "peak_source": f"{pk_kind} hbm_gbs",
                "kernel": "k_posterior_e (device time, CUDA events)",
                "algorithmic_bytes_per_launch": alg, "avg_launch_ms": round(upd_s * 1e3, 3),
                "avg_gl_update_call_ms": round(sum(host_ms) / reps, 3)}
    pinned, keep = pinned_copy(P)
    e2e_t = []
    for i in range(2):
        t0 = time.perf_counter()
        ctx.load_gl(pinned.T)
        o, _ = step()
        if i > 0:
            e2e_t.append(time.perf_counter() - t0)
    e2e_s = run.max_over_ranks(e2e_t[0])
    e2e = {"value": round(gl_bytes * passes / e2e_s / 1e9 * run.world, 4), "unit": "GL GB/s",
           "h2d_bytes_per_step": int(gl_bytes), "d2h_bytes_per_step": int((N + M + 1) * k * 8),
           "seconds_per_pcangsd": round(e2e_s, 3)}
    ctx.close()
    cpu = cpu_baseline(args, cfg, prefix, wd, run)
    run.close()
    if run.rank != 0:
        return
    emit(args, cfg, run, value, "GL GB/s", sec * 1e3, "fp32", clocks, roofline, e2e, cpu, None,
         {"samples": N, "sites": M, "k": k, "windows": bands, "em_iterations": out[4], "maf_sweeps": itm,
          "likelihood_passes": passes},
         {"pcangsd_seconds": round(sec, 4),
          "timing": "host clock around the EM loop (every library call synchronises)"}, metric=METRIC_GL)


def ld_dense_check(packed, N, U, ws, we, r2, nwin=3):
    """Largest |r2 - r2_dense| over a few windows (first, middle, last long one), r2_dense
    from a dense FP64 evaluation in numpy: centred genotypes (missing 0), projected off U,
    Pearson r of every pair of the window."""
    off = np.concatenate([[0], np.cumsum(np.maximum(we.astype(np.int64) - 1, 0))])
    long_ = np.nonzero(we > 1)[0]
    picks = sorted({int(long_[0]), int(long_[len(long_) // 2]), int(long_[-1])})[:nwin]
    worst = 0.0
    lut = np.array([2.0, 0.0, 1.0, 0.0])  # A1 count per code (missing -> 0)
    for w in picks:
        i0, n = int(ws[w]), int(we[w])
        codes = np.unpackbits(packed[i0:i0 + n][:, :, None], axis=2, bitorder="little")
        codes = (codes[:, :, 0::2] + 2 * codes[:, :, 1::2]).reshape(n, -1)[:, :N]
        x = lut[codes] / 2.0
        nm = codes != 1
        F = (x * nm).sum(1) / np.maximum(nm.sum(1), 1)
        G = np.where(nm, x - F[:, None], 0.0).T  # N x n
        G = G - U @ (U.T @ G)
        r = (G[:, 1:].T @ G[:, 0]) / np.sqrt((G[:, 1:] ** 2).sum(0) * (G[:, 0] ** 2).sum())
        worst = max(worst, float(np.abs(r2[off[w]:off[w + 1]] - r * r).max()))
    return {"max_abs_r2_err_vs_dense_fp64": worst, "windows_checked": picks}


def run_ld_cfg(args, cfg, run):
    """LD r2 of every window pair through the C ABI (pcaone_gpu_ld_r2): the band Gram of the
    windows on the tensor cores. value = pairs / device time of the LD work (CUDA events on the
    library's stream around the diagonal, tiling and band-Gram launches; the packed genotypes
    and the projection factors resident); e2e = pairs / wall time of load + LD call with host
    buffers (packed genotypes in, r2 of every pair out)."""
    import pcaone_b200 as pb

    wd, prefix = prepare(cfg, args.config, run)
    packed, N, M = pb.read_bed(prefix)
    ws, we, pairs = full_ld_pairs(cfg, prefix)
    log(f"{len(ws)} windows, {pairs} pairs, window SNPs {int(we.min())}..{int(we.max())}")
    ctx = pb.GpuContext(run.local)
    ctx.load_bed(packed, N)
    pcs = ctx.rsvd(k=cfg["k"], svd=1, maxp=cfg["maxp"], tol=cfg["tol"], precision="mixed")
    U = pcs.U
    for _ in range(args.warmup):
        t0 = time.perf_counter()
        ctx.ld_r2(ws, we, U)
        log(f"warm-up LD: {time.perf_counter() - t0:.2f} s wall, device {ctx.ld_timing()}")
    run.barrier()
    dev, gram = [], []
    with ClockSampler(run.local) as clk:
        run.barrier()
        for _ in range(args.steps):
            ctx.ld_r2(ws, we, U)
            d, g = ctx.ld_timing()
            dev.append(d)
            gram.append(g)
        run.barrier()
    clocks = clk.summary()
    log(f"timed LD device ms: {[round(x, 2) for x in dev]}, band Gram ms: {[round(x, 2) for x in gram]}")
    ms = run.max_over_ranks(float(np.mean(dev)))
    value = pairs / (ms / 1e3) * run.world
    # tensor roofline of the band Gram: 4 integer Grams (RR, RN, NR, NN), 2 ops per product
    alg = 8.0 * pairs * N
    g_ms = float(np.mean(gram))
    pk, pk_kind = peaks()
    peak = pk.get("bf16_tflops_sustained", pk.get("bf16_tflops"))
    # issued: per (128 x 128) tile of SNP pairs two M = 128, N = 256 int8 MMAs per sample
    T = 128
    reach = {}
    for s, w in zip(ws, we):
        if w >= 2:
            b = int(s) // T
            reach[b] = max(reach.get(b, -1), int(s) + int(w) - 1)
    ntile = sum(v // T - b + 1 for b, v in reach.items())
    issued = ntile * 2.0 * 2 * T * 256 * ((N + 127) // 128 * 128)
    achieved = alg / (g_ms / 1e3) / 1e12
    roofline = {"bound": "tensor", "achieved": round(achieved, 2), "peak": peak, "unit": "TFLOP/s",
                "frac": round(achieved / peak, 4), "traffic": None, "peak_source": f"{pk_kind} bf16_tflops_sustained",
                "kernel": "k_ld_gram_i8", "launches": 1, "avg_launch_ms": round(g_ms, 4),
                "algorithmic_ops_per_launch": alg, "issued_ops_factor": round(issued / alg, 4),
                "ceiling_frac_of_bf16_peak": round(2.0 / (issued / alg), 4), "band_tiles": ntile,
                "gram_share_of_device_ms": round(g_ms / ms, 4)}
    pinned, keep = pinned_copy(packed)
    e2e_t = []
    for i in range(2):
        t0 = time.perf_counter()
        ctx.load_bed(pinned, N)
        out = ctx.ld_r2(ws, we, U)
        if i > 0:
            e2e_t.append(time.perf_counter() - t0)
    e2e_s = run.max_over_ranks(e2e_t[0])
    e2e = {"value": round(pairs / e2e_s * run.world, 1), "unit": "pairs/s",
           "h2d_bytes_per_step": int(packed.nbytes + U.nbytes + ws.nbytes + we.nbytes),
           "d2h_bytes_per_step": int(out.nbytes), "seconds_per_call": round(e2e_s, 3),
           "includes": "genotype upload, projection factors W = Gc^T U (FP64 product) and Y, r2 of every pair "
                       "copied back"}
    acc = {}
    if not args.skip_compare:
        acc = ld_dense_check(packed, N, U, ws, we, out)
    ctx.close()
    cpu = cpu_baseline(args, cfg, prefix, wd, run)
    run.close()
    if run.rank != 0:
        return
    emit(args, cfg, run, value, "pairs/s", ms, "int8", clocks, roofline, e2e, cpu, None,
         {"samples": N, "snps": M, "k": cfg["k"], "ld_bp": cfg["ld_bp"], "windows": int(len(ws)), "pairs": pairs,
          "window_snps": [int(we.min()), int(we.max())]},
         {"accuracy": acc, "timing": "CUDA events on the library stream (pcaone_gpu_ld_timing)"}, metric=METRIC_LD)


def cpu_baseline(args, cfg, prefix, wd, run):
    if run.rank != 0 or run.world != 1 or args.skip_cpu:
        return None
    try:
        runs = [reference_run(cfg, prefix, wd, s) for s in cfg["cpu_fit_snps"]]
    except (RuntimeError, subprocess.CalledProcessError) as e:
        return {"value": None, "unavailable": str(e)}
    if cfg["kind"] == "ld":
        value, sample = fitted_rate_ld(cfg, runs, full_ld_pairs(cfg, prefix)[2])
        cpu = {"value": round(value, 1), "unit": "pairs/s", "cores": runs[0]["cores"], "kind": "reference",
               "sample": sample}
        log(f"cpu baseline: {cpu}")
        return cpu
    value, sample = fitted_rate(cfg, runs)
    cpu = {"value": round(value, 6), "unit": "GL GB/s" if cfg["kind"] == "pcangsd" else "bed GB/s",
           "cores": runs[0]["cores"], "kind": "reference", "sample": sample}
    log(f"cpu baseline: {cpu}")
    return cpu


def emit(args, cfg, run, value, unit, ms_per_step, prec, clocks, roofline, e2e, cpu, launches, conf, extra,
         metric=METRIC):
    line = {
        "metric": metric, "value": round(value, 4), "unit": unit, "n_gpus": run.world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_per_step, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": DTYPE.get(prec, prec),
        "data": "synthetic (seeded simulator: " + " ".join(cfg["sim"]) + ")",
        "config": dict({"workload": cfg["workload"]}, **conf, precision=prec,
                       parallelism=f"replicas x{run.world}",
                       l2="inputs larger than L2 (126 MB); no flush needed"),
    }
    line.update(extra)
    line.update({"roofline": roofline, "e2e": e2e, "cpu_baseline": cpu, "clocks": clocks})
    if launches is not None:
        line["gpu_launches"] = launches
    print(json.dumps(line), flush=True)


def run_reference_arm(args, cfg):
    """The reference PCAone on the host cores, rank 0 only: W + K runs on slices of the
    workload cycling through the configured sizes, the rate fitted over the K timed runs and
    evaluated at the full size (one size: its own rate)."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    wd = workdir()
    prefix = os.path.join(wd, args.config)
    make_data(cfg, prefix)
    sizes = list(cfg["cpu_fit_snps"])
    runs = []
    t_start = time.perf_counter()
    for i in range(args.warmup + args.steps):
        try:
            r = reference_run(cfg, prefix, wd, sizes[i % len(sizes)])
        except (RuntimeError, subprocess.CalledProcessError) as e:
            print(json.dumps({"impl": "reference", "unavailable": str(e)}))
            return
        if i >= args.warmup:
            runs.append(r)
        if time.perf_counter() - t_start > 240 and len(runs) >= len(sizes):
            break  # keep the arm within a few minutes
    if cfg["kind"] == "ld":
        v, sample = fitted_rate_ld(cfg, runs, full_ld_pairs(cfg, prefix)[2])
        unit, metric = "pairs/s", METRIC_LD
    else:
        v, sample = fitted_rate(cfg, runs)
        unit = "GL GB/s" if cfg["kind"] == "pcangsd" else "bed GB/s"
        metric = METRIC_GL if cfg["kind"] == "pcangsd" else METRIC
    print(json.dumps({
        "impl": "reference", "metric": metric, "value": round(v, 6),
        "unit": unit, "n_gpus": world, "steps": len(runs), "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "dtype": "f64", "data": "synthetic (seeded simulator: " + " ".join(cfg["sim"]) + ")",
        "config": {"workload": cfg["workload"], "sample": f"{len(runs)} timed runs; " + sample},
        "cpu_baseline": {"value": round(v, 6), "unit": unit, "cores": runs[0]["cores"], "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(v, 6), "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)


def run_profile_kernel(args, cfg):
    """Smallest command for ncu: one standardised product Z^T Omega through the C ABI on the
    configured matrix (the tensor-core paths launch their decode-GEMM once), then exit. No
    child processes, no torch."""
    import pcaone_b200 as pb

    prefix = os.path.join(workdir(), args.config)
    make_data(cfg, prefix)
    if cfg["kind"] == "pcangsd":  # posterior, dense products and GRM on the first 40000 sites
        N, m, k = cfg["n"], 40000, cfg["k"]
        P = np.fromfile(prefix + ".gl.f32", dtype=np.float32, count=m * 2 * N).reshape(m, 2 * N)
        kw = dict(k=k, oversamples=10, maxp=cfg["maxp"], svd=2, bands=cfg["bands"], tol=cfg["tol"], seed=101,
                  rand=1, precision=pb.PREC_FP32, standardize=False)
        with pb.GpuContext(0) as ctx:
            ctx.load_gl(P.T)
            ctx.gl_freq(cfg["maxiter"], 1e-6)
            ctx.gl_update()
            r = ctx.rsvd(carry=False, **kw)
            for _ in range(args.steps):
                ctx.gl_update(r.U, r.S, r.V)
            C, _, _ = ctx.gl_grm(r.U, r.S, r.V, vectors=False)
        print(json.dumps({"profile_kernel": "pcangsd", "samples": N, "sites": m, "epochs": r.epochs,
                          "checksum": float(np.trace(C))}))
        return
    packed, N, M = pb.read_bed(prefix)
    if cfg["kind"] == "ld":  # one band-Gram launch over the first 60000 SNPs (150 MB packed)
        m = min(M, 60000)
        pos, ends = pb.read_bim_positions(prefix + ".bim")
        ws, we = pb.ld_windows(pos[:m], [e for e in ends if e < m - 1] + [m - 1], cfg["ld_bp"])
        U = np.linalg.qr(np.random.default_rng(1).standard_normal((N, cfg["k"])))[0]
        with pb.GpuContext(0) as ctx:
            ctx.load_bed(np.ascontiguousarray(packed[:m]), N)
            for _ in range(args.steps):
                r2 = ctx.ld_r2(ws, we, U)
            t = ctx.ld_timing()
        print(json.dumps({"profile_kernel": "ld", "samples": N, "snps": m, "pairs": int(r2.size),
                          "device_ms": t[0], "gram_ms": t[1], "checksum": float(r2.sum())}))
        return
    if cfg["kind"] == "emu":  # the EMU imputation and the weighted epilogue gathers, 50000 SNPs
        m = min(M, 50000)
        kw = dict(k=cfg["k"], oversamples=10, maxp=cfg["maxp"], svd=2, bands=cfg["bands"], tol=cfg["tol"],
                  seed=101, precision=args.precision)
        with pb.GpuContext(0) as ctx:
            ctx.load_bed(np.ascontiguousarray(packed[:m]), N)
            ctx.permute(pb.shuffle_perm(m))
            ctx.clear_imputed()
            r = ctx.rsvd(standardize=False, **kw)
            for _ in range(args.steps):
                ctx.fit_emu(r.U, r.S, r.V, True)
                r = ctx.rsvd(standardize=False, carry=True, **kw)
        print(json.dumps({"profile_kernel": "emu", "samples": N, "snps": m, "epochs": r.epochs,
                          "checksum": float(np.abs(r.S).sum())}))
        return
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

    prefix = os.path.join(workdir(), args.config)
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
    ap.add_argument("--precision", default="mixed", choices=["mixed", "bf16", "fp32", "fp64"])
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
        run = Run()
        {"rsvd": run_rsvd_cfg, "emu": run_emu_cfg, "pcangsd": run_pcangsd_cfg,
         "ld": run_ld_cfg}[cfg["kind"]](args, cfg, run)


if __name__ == "__main__":
    main()
