"""Windowed LD r2 (flow A: genotypes projected off U) through the C ABI against the
reference's .ld.gz output and the oracle."""
import os

import numpy as np
import pytest

import pcaone_b200 as pb
from oracle import pcaone_oracle as O
from tests.helpers import GOLDEN
from tests.test_gpu_rsvd import random_bed

pytestmark = pytest.mark.gpu


def test_ld_flow_a_matches_reference(gpu):
    bed = O.read_bed(os.path.join(GOLDEN, "g4"))
    U = O.read_usv(os.path.join(GOLDEN, "ref", "g4_pcs.eigvecs"))
    snp = O.read_snp_pos(os.path.join(GOLDEN, "ref", "g4_pcs.mbim"))
    O.divide_pos_by_window(snp, 5000)
    gpu.load_bed(bed.packed, bed.N)
    r2 = gpu.ld_r2(snp.ws, snp.we, U)
    head, ref = O.read_ld_gz(os.path.join(GOLDEN, "ref", "g4_ldA.ld.gz"))
    rr = np.array([float(x[6]) for x in ref])
    assert len(r2) == len(rr)
    assert np.abs(r2 - rr).max() <= 1e-5  # parity bar for LD r2 (absolute)


@pytest.mark.parametrize("N,M,with_u", [(1001, 700, True), (333, 500, False), (2048, 300, True)])
def test_ld_matches_oracle(gpu, N, M, with_u):
    bed = random_bed(N, M, seed=N + M, miss=0.03)
    rng = np.random.default_rng(1)
    U = np.linalg.qr(rng.standard_normal((N, 5)))[0] if with_u else None
    gpu.load_bed(bed.packed, N)
    snp = O.SnpLD(["1"], np.cumsum(rng.integers(1, 300, M)), [M - 1], [""] * M)
    O.divide_pos_by_window(snp, 4000)
    r2 = gpu.ld_r2(snp.ws, snp.we, U)
    G = O.centered_matrix(O.decode_codes(bed), O.allele_freq(O.decode_codes(bed)))
    if with_u:
        G = G - U @ (U.T @ G)
    i, k, r = O.ld_pairs(G, snp)
    assert np.abs(r2 - r * r).max() <= 1e-6


@pytest.mark.parametrize("N,M,k,bp,chroms", [
    (1001, 700, 5, 4000, 1),     # tensor-core band Gram, windows across several 128-SNP tiles
    (130, 2000, 0, 60000, 2),    # unprojected, long windows (up to ~1000 SNPs), two chromosomes
    (2049, 515, 16, 9000, 1),    # widest projection of the tensor-core path
    (777, 600, 20, 5000, 1),     # projection wider than 16: the bit-plane kernel
])
def test_ld_band_gram_matches_oracle_f64(gpu, N, M, k, bp, chroms):
    """FP64 r2 of every window pair (the pruning/clumping values) against the oracle's
    dense FP64 correlations, on shapes that are not multiples of the 128-SNP and 128-sample
    tiles."""
    bed = random_bed(N, M, seed=3 * N + M, miss=0.05)
    rng = np.random.default_rng(N)
    U = np.linalg.qr(rng.standard_normal((N, k)))[0] if k else None
    gpu.load_bed(bed.packed, N)
    pos = np.concatenate([np.cumsum(rng.integers(1, 120, M // chroms + (c < M % chroms))) for c in range(chroms)])
    ends, acc = [], 0
    for c in range(chroms):
        acc += M // chroms + (c < M % chroms)
        ends.append(acc - 1)
    snp = O.SnpLD([str(c + 1) for c in range(chroms)], pos, ends, [""] * M)
    O.divide_pos_by_window(snp, bp)
    r2 = gpu.ld_r2(snp.ws, snp.we, U, f64=True)
    G = O.centered_matrix(O.decode_codes(bed), O.allele_freq(O.decode_codes(bed)))
    if k:
        G = G - U @ (U.T @ G)
    i, kk, r = O.ld_pairs(G, snp)
    assert len(r2) == len(r) and int(np.max(snp.we)) > 60  # windows cross 128-SNP tile edges
    np.testing.assert_allclose(r2, r * r, rtol=1e-9, atol=1e-12)


def test_ld_flow_b_matches_reference(gpu):
    """Flow B: r2 on the reference's own .residuals matrix (loaded and re-centred on the
    device) against the reference's .ld.gz of -B g4_adj.residuals -f g4_adj.mbim."""
    path = os.path.join(GOLDEN, "ref", "g4_adj.residuals")
    with open(path, "rb") as f:
        M, N = (int(x) for x in np.frombuffer(f.read(8), dtype=np.uint32))
        X = np.frombuffer(f.read(4 * M * N), dtype=np.float32).reshape(M, N)
    snp = O.read_snp_pos(os.path.join(GOLDEN, "ref", "g4_adj.mbim"))
    O.divide_pos_by_window(snp, 5000)
    gpu.load_dense(X)
    r2 = gpu.ld_r2(snp.ws, snp.we)
    head, ref = O.read_ld_gz(os.path.join(GOLDEN, "ref", "g4_ldB.ld.gz"))
    rr = np.array([float(x[6]) for x in ref])
    assert len(r2) == len(rr)
    assert np.abs(r2 - rr).max() <= 1e-5
    i, k, r = O.ld_pairs(O.read_residuals(path), snp)
    assert np.abs(r2 - r * r).max() <= 1e-6


@pytest.mark.parametrize("N,M", [(517, 900), (64, 2000)])
def test_ld_dense_matches_oracle(gpu, N, M):
    """Dense r2 on an arbitrary float matrix with long windows (tiles across block edges)."""
    rng = np.random.default_rng(N)
    X = rng.standard_normal((M, N)).astype(np.float32) + 3.0
    snp = O.SnpLD(["1"], np.cumsum(rng.integers(1, 50, M)), [M - 1], [""] * M)
    O.divide_pos_by_window(snp, 3000)
    gpu.load_dense(X)
    r2 = gpu.ld_r2(snp.ws, snp.we)
    G = X.T.astype(np.float64)
    G = G - G.mean(axis=0, keepdims=True)
    i, k, r = O.ld_pairs(G, snp)
    assert np.abs(r2 - r * r).max() <= 1e-6


def test_residuals_match_reference(gpu):
    """The -D writer's rows (Data::write_residuals) from the reference's own factors of the
    g4_adj run against the reference's .residuals file."""
    bed = O.read_bed(os.path.join(GOLDEN, "g4"))
    gpu.load_bed(bed.packed, bed.N)
    with open(os.path.join(GOLDEN, "ref", "g4_adj.residuals"), "rb") as f:
        M, N = (int(x) for x in np.frombuffer(f.read(8), dtype=np.uint32))
        ref = np.frombuffer(f.read(4 * M * N), dtype=np.float32).reshape(M, N)
    # the centred genotypes (ld-stats 1) are independent of the factors: exact up to float rounding
    G = O.centered_matrix(O.decode_codes(bed), O.allele_freq(O.decode_codes(bed)))
    G = G - G.mean(axis=0, keepdims=True)
    got = gpu.residuals()
    np.testing.assert_allclose(got, G.T.astype(np.float32), atol=2e-7)
    # with factors: U S V^T from an FP64 GPU Halko run of the same flags (-d 1 -k 3 -p 7, unstandardised)
    r = gpu.rsvd(k=3, maxp=7, svd=1, tol=0.0, precision="fp64", standardize=False)
    res = gpu.residuals(r.U, r.S, r.V)
    assert np.abs(res - ref).max() <= 1e-5
