"""Regenerates the golden fixtures in this folder.

Inputs are small seeded synthetic datasets written by the package's simulator
(``pcaone_b200/bin/pcaone-sim``); outputs are produced by the unmodified reference PCAone
v0.6.0 binary built from its own sources by ``oracle/ref.mk`` into ``oracle/_ref/PCAone``.
Run from the repository root in the container that has the reference sources:

    make -f oracle/ref.mk -j8            # REF defaults to $PCAONE_REF, else /root/reference
    python tests/golden/make_golden.py             # every case
    python tests/golden/make_golden.py g4_pruneA   # only the named cases (others kept)

Each case in ``CASES`` is (name, dataset, reference arguments, output suffixes kept).
``cases.json`` records the exact commands so the tests can reproduce them.

``LARGE`` datasets are full benchmark shapes (config 1: 2000 samples x 50000 SNPs). They are
too large to commit: the tests regenerate them with the same simulator flags and check the
.bed against the sha256 recorded here; only the reference's outputs are kept (.loadings: the
first LARGE_LOADING_ROWS SNPs, gzip-compressed).
"""
from __future__ import annotations

import gzip
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
SIM = os.path.join(ROOT, "pcaone_b200", "bin", "pcaone-sim")
REF = os.path.join(ROOT, "oracle", "_ref", "PCAone")

DATASETS = {
    # odd N (not a multiple of 4) exercises the padded last byte of every SNP record
    "g1": ["--n", "203", "--m", "1500", "--pops", "3", "--fst", "0.05", "--pmin", "0.05",
           "--pmax", "0.5", "--miss", "0.01", "--seed", "11"],
    # heavy per-sample missingness for EMU
    "g2": ["--n", "120", "--m", "1200", "--pops", "3", "--fst", "0.08", "--pmin", "0.05",
           "--pmax", "0.5", "--miss-beta", "2,18", "--admix", "0.5", "--seed", "12"],
    # genotype likelihoods for PCAngsd
    "g3": ["--n", "80", "--m", "900", "--pops", "3", "--fst", "0.1", "--pmin", "0.05",
           "--pmax", "0.5", "--beagle", "4,0.01", "--seed", "13"],
    # two chromosomes with positions for LD windows
    "g4": ["--n", "100", "--m", "600", "--pops", "3", "--fst", "0.05", "--pmin", "0.05",
           "--pmax", "0.5", "--miss", "0.01", "--chroms", "2", "--bp-spacing", "500",
           "--seed", "14"],
}

# full-shape datasets, regenerated by the tests (not committed); same flags as bench.py "c1"
LARGE = {
    "c1": ["--n", "2000", "--m", "50000", "--pops", "3", "--fst-lo", "0.05", "--fst-hi", "0.05",
           "--pmin", "0.05", "--pmax", "0.5", "--miss", "0.01", "--seed", "1"],
}

LARGE_LOADING_ROWS = 5000

# assoc-like files for clumping, drawn from the g4 .bim: (file, seed, fraction of SNPs kept,
# fraction with a small p-value); columns CHR, SNP, BP, P (tab-separated, with a header);
# every p-value is distinct
ASSOC = {"g4_a.assoc": (21, 0.8, 0.15), "g4_b.assoc": (22, 0.6, 0.3)}


def write_assoc(bim: str, path: str, seed: int, keep: float, small: float) -> None:
    import numpy as np

    rng = np.random.default_rng(seed)
    rows = [line.split() for line in open(bim)]
    lines = ["CHR\tSNP\tBP\tP"]
    used = set()
    for r in rows:
        if rng.random() >= keep:
            continue
        while True:
            p = float(10 ** -rng.uniform(3, 6)) if rng.random() < small else float(rng.uniform(0.001, 1))
            p = float(f"{p:.6g}")
            if p not in used:
                used.add(p)
                break
        lines.append(f"{r[0]}\t{r[1]}\t{r[3]}\t{p:.6g}")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")

EIG = [".eigvals", ".sigvals", ".eigvecs"]
CASES = [
    ("g1_halko", "g1", ["-b", "{d}", "-d", "1", "-k", "4", "--oversamples", "10", "-p", "7",
                        "--tol-rsvd", "0", "-V"], EIG + [".loadings", ".mbim"]),
    ("g1_halko_p3", "g1", ["-b", "{d}", "-d", "1", "-k", "3", "-p", "3", "--seed", "7"],
     EIG),
    ("g1_win", "g1", ["-b", "{d}", "-d", "2", "-k", "4", "-w", "16", "-V"],
     EIG + [".loadings"]),
    ("g1_winS", "g1", ["-b", "{d}", "-d", "2", "-k", "4", "-w", "8", "-S", "-V"],
     EIG + [".loadings"]),
    ("g1_win_unif", "g1", ["-b", "{d}", "-d", "2", "-k", "3", "-w", "4", "--rand", "0",
                           "--seed", "3", "-p", "5"], EIG),
    ("g1_nostd", "g1", ["-b", "{d}", "-d", "1", "-k", "3", "-p", "5", "--tol-rsvd", "0",
                        "-C", "0"], EIG),
    ("g2_emu", "g2", ["-b", "{d}", "--emu", "-k", "3", "-w", "8", "--maxiter", "20",
                      "--tol-em", "1e-6", "-V"], EIG + [".loadings"]),
    ("g3_pcangsd", "g3", ["-G", "{d}.beagle.gz", "-k", "3", "-S", "-w", "8", "--maxiter", "30",
                          "-V"], EIG + [".loadings", ".cov"]),
    ("g3_pcangsd_shuf", "g3", ["-G", "{d}.beagle.gz", "-k", "3", "-w", "8", "--maxiter", "30"],
     EIG + [".cov"]),
    ("g4_pcs", "g4", ["-b", "{d}", "-d", "1", "-k", "3", "-p", "7", "--tol-rsvd", "0", "-V"],
     EIG + [".mbim"]),
    ("g4_ldA", "g4", ["-b", "{d}", "--read-U", "{g}/ref/g4_pcs.eigvecs", "-f",
                      "{g}/ref/g4_pcs.mbim", "--ld-bp", "5000", "-R"], [".ld.gz"]),
    ("g4_adj", "g4", ["-b", "{d}", "-d", "1", "-k", "3", "-p", "7", "--tol-rsvd", "0", "-D"],
     [".residuals", ".mbim"] + EIG),
    ("g4_ldB", "g4", ["-B", "{g}/ref/g4_adj.residuals", "-f", "{g}/ref/g4_adj.mbim",
                      "--ld-bp", "5000", "-R"], [".ld.gz"]),
    # LD pruning: flow A keeping the higher-MAF SNP (.mbim frequencies), flow A with a plain
    # .bim (the follower is dropped), flow B
    ("g4_pruneA", "g4", ["-b", "{d}", "--read-U", "{g}/ref/g4_pcs.eigvecs", "-f", "{g}/ref/g4_pcs.mbim",
                         "--ld-bp", "5000", "--ld-r2", "0.05"], [".ld.prune.in", ".ld.prune.out"]),
    ("g4_pruneA_bim", "g4", ["-b", "{d}", "--read-U", "{g}/ref/g4_pcs.eigvecs", "--ld-bp", "5000",
                             "--ld-r2", "0.05"], [".ld.prune.in", ".ld.prune.out"]),
    ("g4_pruneB", "g4", ["-B", "{g}/ref/g4_adj.residuals", "-f", "{g}/ref/g4_adj.mbim", "--ld-bp", "5000",
                         "--ld-r2", "0.05"], [".ld.prune.in", ".ld.prune.out"]),
    # LD clumping of two assoc-like files (flow A) and of one with other thresholds (flow B)
    ("g4_clumpA", "g4", ["-b", "{d}", "--read-U", "{g}/ref/g4_pcs.eigvecs", "-f", "{g}/ref/g4_pcs.mbim",
                         "--clump", "{g}/g4_a.assoc,{g}/g4_b.assoc", "--clump-p1", "0.01",
                         "--clump-p2", "0.2", "--clump-r2", "0.05", "--clump-bp", "5000"],
     [".p0.clump", ".p1.clump"]),
    ("g4_clumpB", "g4", ["-B", "{g}/ref/g4_adj.residuals", "-f", "{g}/ref/g4_adj.mbim",
                         "--clump", "{g}/g4_a.assoc", "--clump-p1", "0.05", "--clump-p2", "0.5",
                         "--clump-r2", "0.03", "--clump-bp", "3000"], [".p0.clump"]),
    # PCAngsd on PLINK input: pseudo-likelihoods from the genotypes (shuffled and -S)
    ("g1_pcangsd_bed", "g1", ["-b", "{d}", "--pcangsd", "-k", "3", "-w", "8", "--maxiter", "30",
                              "-V"], EIG + [".loadings"]),
    ("g1_pcangsd_bedS", "g1", ["-b", "{d}", "--pcangsd", "-k", "3", "-w", "8", "-S",
                               "--maxiter", "30", "-V"], EIG + [".loadings"]),
    # out-of-core winSVD (-m): permute_plink order and the block plan (24 blocks, band factor 3;
    # 8 blocks, band factor 1); -v 3 keeps the permuted .bim for the order's pin
    ("g1_win_m", "g1", ["-b", "{d}", "-d", "2", "-k", "4", "-w", "8", "-m", "0.0001", "-V", "-v", "3"],
     EIG + [".loadings", ".perm.bim"]),
    ("g1_win_m8", "g1", ["-b", "{d}", "-d", "2", "-k", "4", "-w", "8", "-m", "0.0003", "-V"],
     EIG + [".loadings"]),
    # IRAM (--svd 0): Spectra's restarted Lanczos on Z Z^T, converged to --itol 1e-6
    ("g1_iram", "g1", ["-b", "{d}", "-d", "0", "-k", "4", "-V"], EIG + [".loadings"]),
    # config 1 at its full shape: Halko k=10, oversampling 10, 8 epochs
    ("c1_halko", "c1", ["-b", "{d}", "-d", "1", "-k", "10", "--oversamples", "10", "-p", "7",
                        "--tol-rsvd", "0", "-V"], EIG + [".loadings"]),
    ("c1_iram", "c1", ["-b", "{d}", "-d", "0", "-k", "10"], EIG),
]


def sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for blk in iter(lambda: f.read(1 << 20), b""):
            h.update(blk)
    return h.hexdigest()


def main() -> int:
    if not os.path.exists(REF):
        print("reference binary missing: run make -f oracle/ref.mk first", file=sys.stderr)
        return 1
    if not os.path.exists(SIM):
        print("simulator missing: run the package build first", file=sys.stderr)
        return 1
    refdir = os.path.join(HERE, "ref")
    os.makedirs(refdir, exist_ok=True)
    for name, args in DATASETS.items():
        subprocess.check_call([SIM, "--out", os.path.join(HERE, name)] + args)
    for fname, (seed, keep, small) in ASSOC.items():
        write_assoc(os.path.join(HERE, "g4.bim"), os.path.join(HERE, fname), seed, keep, small)
    large_dir = tempfile.mkdtemp()
    large_sha = {}
    for name, args in LARGE.items():
        subprocess.check_call([SIM, "--out", os.path.join(large_dir, name)] + args)
        large_sha[name] = sha256(os.path.join(large_dir, name + ".bed"))
    only = set(sys.argv[1:])
    old = {}
    if only and os.path.exists(os.path.join(HERE, "cases.json")):
        with open(os.path.join(HERE, "cases.json")) as f:
            old = {c["name"]: c for c in json.load(f)["cases"]}
    record = {"datasets": DATASETS, "large_datasets": LARGE, "large_bed_sha256": large_sha,
              "cases": []}
    env = dict(os.environ, OMP_NUM_THREADS="4")
    for name, ds, args, keep in CASES:
        if only and name not in only and name in old:
            record["cases"].append(old[name])
            continue
        with tempfile.TemporaryDirectory() as tmp:
            dpath = os.path.join(large_dir if ds in LARGE else HERE, ds)
            argv = [a.format(d=dpath, g=HERE) for a in args]
            out = os.path.join(tmp, name)
            verb = [] if "-v" in argv else ["-v", "0"]
            subprocess.run([REF] + argv + ["-o", out] + verb, check=True, env=env,
                           stdout=subprocess.DEVNULL)
            for suf in keep:
                if ds in LARGE and suf == ".loadings":
                    text = []
                    with open(out + suf) as fi:
                        for i, line in enumerate(fi):
                            if i >= LARGE_LOADING_ROWS:
                                break
                            text.append(line)
                    # mtime 0: the compressed bytes do not depend on when they were made
                    with gzip.GzipFile(os.path.join(refdir, name + suf + ".gz"), "wb", mtime=0) as fo:
                        fo.write("".join(text).encode())
                else:
                    shutil.copy(out + suf, os.path.join(refdir, name + suf))
        record["cases"].append({"name": name, "dataset": ds, "args": args, "outputs": keep})
    shutil.rmtree(large_dir)
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(record, f, indent=1)
    return 0


if __name__ == "__main__":
    sys.exit(main())
