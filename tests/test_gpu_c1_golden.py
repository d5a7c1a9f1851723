"""Config 1 at its full shape against the reference binary: Halko k = 10, oversampling 10,
8 epochs (-p 7 --tol-rsvd 0) on 2000 samples x 50000 SNPs (3 Balding-Nichols populations, 1%
missing). The input is regenerated by the package's seeded simulator and checked against the
.bed sha256 recorded when the reference outputs were made (tests/golden/make_golden.py)."""
import gzip
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

import pcaone_b200 as pb
from oracle import pcaone_oracle as O
from tests.helpers import GOLDEN, assert_cols_close, assert_eig_close, ref_eigvals, ref_table

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def c1_prefix(tmp_path_factory):
    with open(os.path.join(GOLDEN, "cases.json")) as f:
        rec = json.load(f)
    prefix = str(tmp_path_factory.mktemp("c1") / "c1")
    sim = os.path.join(ROOT, "pcaone_b200", "bin", "pcaone-sim")
    subprocess.check_call([sim, "--out", prefix] + rec["large_datasets"]["c1"], stdout=subprocess.DEVNULL)
    h = hashlib.sha256()
    with open(prefix + ".bed", "rb") as f:
        for blk in iter(lambda: f.read(1 << 20), b""):
            h.update(blk)
    assert h.hexdigest() == rec["large_bed_sha256"]["c1"], "simulator output differs from the golden input"
    return prefix


def ref_loadings():
    with gzip.open(os.path.join(GOLDEN, "ref", "c1_halko.loadings.gz"), "rt") as f:
        return np.array([[float(t) for t in line.split()] for line in f])


@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed", "bf16"])
def test_c1_halko_matches_reference(gpu, c1_prefix, prec):
    packed, N, M = pb.read_bed(c1_prefix)
    gpu.load_bed(packed, N)
    r = gpu.rsvd(k=10, oversamples=10, maxp=7, svd=1, tol=0.0, precision=prec)
    assert r.epochs == 8
    assert_eig_close(r.S ** 2 / M * 2, ref_eigvals("c1_halko"), 1e-5)
    U_ref, V_ref = ref_table("c1_halko", ".eigvecs"), ref_loadings()
    if prec == "fp64":  # algorithm-matched: every PC, to the reference's printed digits
        assert_cols_close(r.U, U_ref, 2e-6)
        assert_cols_close(r.V[:V_ref.shape[0]], V_ref, 2e-6)
    else:  # the two population PCs (the rest are noise with near-equal eigenvalues)
        assert_cols_close(r.U[:, :2], U_ref[:, :2], 5e-4)
        assert_cols_close(r.V[:V_ref.shape[0], :2], V_ref[:, :2], 5e-4)


def test_c1_cli_matches_reference(c1_prefix, tmp_path):
    out = str(tmp_path / "c1")
    cli = os.path.join(ROOT, "pcaone_b200", "bin", "PCAone")
    subprocess.run([cli, "-b", c1_prefix, "-d", "1", "-k", "10", "--oversamples", "10", "-p", "7",
                    "--tol-rsvd", "0", "-V", "-o", out], check=True, stdout=subprocess.DEVNULL)
    assert_eig_close(O.read_table(out + ".eigvals")[:, 0], ref_eigvals("c1_halko"), 1e-5)
    assert_cols_close(O.read_table(out + ".eigvecs")[:, :2], ref_table("c1_halko", ".eigvecs")[:, :2], 5e-4)


def test_c1_iram_cli_matches_reference(c1_prefix, tmp_path):
    """Config 1 with --svd 0 (IRAM, k = 10): every eigenvalue to 1e-5 of the reference's."""
    out = str(tmp_path / "c1_iram")
    cli = os.path.join(ROOT, "pcaone_b200", "bin", "PCAone")
    subprocess.run([cli, "-b", c1_prefix, "-d", "0", "-k", "10", "-o", out], check=True, stdout=subprocess.DEVNULL)
    assert_eig_close(O.read_table(out + ".eigvals")[:, 0], ref_eigvals("c1_iram"), 1e-5)
    assert_cols_close(O.read_table(out + ".eigvecs")[:, :2], ref_table("c1_iram", ".eigvecs")[:, :2], 5e-4)
