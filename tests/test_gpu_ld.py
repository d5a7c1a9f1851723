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
