"""GPU tests of the standardised decode-GEMM products through the C ABI, each precision
against the FP64 numpy restatement of Z (oracle): Z^T B and Z B."""
import numpy as np
import pytest

import pcaone_b200 as pb
from oracle import pcaone_oracle as O
from tests.test_gpu_rsvd import random_bed

pytestmark = pytest.mark.gpu

# max |err| / max |ref| per output column. mixed: int8 tensor cores with the sketch as three
# 8-bit fixed-point pieces per column (21 bits below the column maximum); bf16: split BF16
# hi+lo pairs (16 significant bits), FP32 accumulation.
TOL = {"fp64": 1e-12, "fp32": 2e-6, "mixed": 5e-6, "bf16": 5e-5}


def rel_col_err(got, ref):
    return float((np.abs(got - ref).max(axis=0) / np.abs(ref).max(axis=0)).max())


@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed", "bf16"])
@pytest.mark.parametrize("N,M,l", [(1003, 2500, 40), (517, 777, 20), (2048, 1300, 7), (300, 4100, 64)])
def test_products_match_dense(gpu, prec, N, M, l):
    bed = random_bed(N, M, seed=N * 7 + l, miss=0.02)
    Z, F = O.standardized_from_bed(bed)
    gpu.load_bed(bed.packed, N)
    rng = np.random.default_rng(l)
    B1 = rng.standard_normal((N, l))
    got1 = gpu.product_t(B1, precision=prec)
    assert rel_col_err(got1, Z.T @ B1) <= TOL[prec]
    B2 = rng.standard_normal((M, l))
    got2 = gpu.product(B2, precision=prec)
    assert rel_col_err(got2, Z @ B2) <= TOL[prec]


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
@pytest.mark.parametrize("N,M,l", [(1003, 2500, 40), (2048, 1300, 7), (300, 4100, 64)])
def test_int8_pipeline_variants_match_dense(gpu, monkeypatch, variant, N, M, l):
    """Every pipeline variant of the int8 decode-GEMM (the autotuner's choices), pinned one at
    a time: codes through shared memory or from global memory, one- or two-chunk units (wide
    sketches, l = 64, have the one-chunk forms 0 and 2 only)."""
    monkeypatch.setenv("PCAONE_I8_VARIANT", str(variant))
    bed = random_bed(N, M, seed=N * 3 + l + variant, miss=0.02)
    Z, F = O.standardized_from_bed(bed)
    gpu.load_bed(bed.packed, N)
    rng = np.random.default_rng(l + variant)
    B1 = rng.standard_normal((N, l))
    assert rel_col_err(gpu.product_t(B1, precision="mixed"), Z.T @ B1) <= TOL["mixed"]
    B2 = rng.standard_normal((M, l))
    assert rel_col_err(gpu.product(B2, precision="mixed"), Z @ B2) <= TOL["mixed"]


@pytest.mark.parametrize("prec", ["fp64", "mixed", "bf16"])
def test_products_unstandardised_haploid(gpu, prec):
    bed = random_bed(640, 900, seed=3, miss=0.05)
    codes = O.decode_codes(bed)
    F = O.allele_freq(codes)
    Zc = O.centered_matrix(codes, F)
    gpu.load_bed(bed.packed, bed.N)
    B = np.random.default_rng(0).standard_normal((bed.N, 12))
    assert rel_col_err(gpu.product_t(B, precision=prec, standardize=False), Zc.T @ B) <= TOL[prec]
    Zh = O.standardize(Zc, F, ploidy=1)
    assert rel_col_err(gpu.product_t(B, precision=prec, ploidy=1), Zh.T @ B) <= TOL[prec]


@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed", "bf16"])
def test_gram_product_matches_dense(gpu, prec):
    """The IRAM operator Z (Z^T X) in one device call against the oracle's Z."""
    bed = random_bed(777, 3001, seed=21, miss=0.02)
    Z, F = O.standardized_from_bed(bed)
    gpu.load_bed(bed.packed, bed.N)
    X = np.random.default_rng(3).standard_normal((bed.N, 5))
    got = gpu.gram_product(X, precision=prec)
    assert rel_col_err(got, Z @ (Z.T @ X)) <= 2 * TOL[prec]
