"""GPU parity tests of the RSVD path through the C ABI: counts and F bit-exact against the
oracle, FP64/FP32 Halko and winSVD against the reference's golden outputs and the oracle."""
import os

import numpy as np
import pytest

import pcaone_b200 as pb
from oracle import pcaone_oracle as O
from tests.helpers import (GOLDEN, assert_cols_close, assert_eig_close, max_angle, ref_eigvals,
                           ref_table)

pytestmark = pytest.mark.gpu


def load(gpu, name):
    packed, N, M = pb.read_bed(os.path.join(GOLDEN, name))
    gpu.load_bed(packed, N)
    return O.read_bed(os.path.join(GOLDEN, name))


def random_bed(N, M, seed, miss=0.02):
    rng = np.random.default_rng(seed)
    p = rng.uniform(0.05, 0.5, M)
    d = (rng.random((M, N)) < p[:, None]).astype(np.uint8) + (rng.random((M, N)) < p[:, None])
    codes = np.where(d == 2, 0, np.where(d == 1, 2, 3)).astype(np.uint8)
    codes[rng.random((M, N)) < miss] = 1
    bpr = (N + 3) // 4
    pad = np.zeros((M, bpr * 4), dtype=np.uint8)
    pad[:, :N] = codes
    pad = pad.reshape(M, bpr, 4)
    packed = (pad[:, :, 0] | (pad[:, :, 1] << 2) | (pad[:, :, 2] << 4) | (pad[:, :, 3] << 6)).astype(np.uint8)
    return O.Bed(N, M, packed)


@pytest.mark.parametrize("N,M", [(203, 1500), (1001, 777), (1002, 300), (1003, 64), (4096, 2000)])
def test_counts_and_freq_bit_exact(gpu, N, M):
    bed = random_bed(N, M, seed=N + M)
    gpu.load_bed(bed.packed, N)
    a, c = gpu.counts()
    n00, n10, nonmiss = O.allele_counts(O.decode_codes(bed))
    np.testing.assert_array_equal(a, 2 * n00 + n10)
    np.testing.assert_array_equal(c, nonmiss)
    np.testing.assert_array_equal(gpu.allele_freq(), O.allele_freq(O.decode_codes(bed)))


def test_permute_then_counts(gpu):
    bed = random_bed(555, 1234, seed=9)
    gpu.load_bed(bed.packed, bed.N)
    a0, c0 = gpu.counts()
    perm = pb.shuffle_perm(bed.M)
    gpu.permute(perm)
    a1, c1 = gpu.counts()
    np.testing.assert_array_equal(a1, a0[perm])
    np.testing.assert_array_equal(c1, c0[perm])


def test_bad_permutation_rejected(gpu):
    bed = random_bed(100, 50, seed=1)
    gpu.load_bed(bed.packed, bed.N)
    with pytest.raises(pb.PcaoneError):
        gpu.permute(np.zeros(50, dtype=np.int32))


GOLDEN_CASES = [
    ("g1_halko", dict(svd=1, k=4, oversamples=10, maxp=7, tol=0.0), False),
    ("g1_halko_p3", dict(svd=1, k=3, maxp=3, seed=7), False),
    ("g1_win", dict(svd=2, k=4, bands=16), True),
    ("g1_winS", dict(svd=2, k=4, bands=8), False),
    ("g1_win_unif", dict(svd=2, k=3, bands=4, rand=0, seed=3, maxp=5), True),
    ("g1_nostd", dict(svd=1, k=3, maxp=5, tol=0.0, standardize=False), False),
]


def run_gpu(gpu, bed, shuffle, **kw):
    gpu.load_bed(bed.packed, bed.N)
    perm = pb.shuffle_perm(bed.M) if shuffle else None
    if shuffle:
        gpu.permute(perm)
    r = gpu.rsvd(**kw)
    V = r.V
    if shuffle:
        V = np.empty_like(r.V)
        V[perm] = r.V
    return r, V


@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed", "bf16"])
@pytest.mark.parametrize("name,kw,shuffle", GOLDEN_CASES)
def test_rsvd_matches_reference_golden(gpu, prec, name, kw, shuffle):
    bed = O.read_bed(os.path.join(GOLDEN, "g1"))
    r, V = run_gpu(gpu, bed, shuffle, precision=prec, **kw)
    eig = r.S ** 2 / bed.M * 2
    # reference prints 6 significant digits; FP32 path also within the 1e-5 parity bar
    assert_eig_close(eig, ref_eigvals(name), 1e-5)
    assert_cols_close(r.U, ref_table(name, ".eigvecs"), 2e-6 if prec == "fp64" else 5e-4)
    lpath = os.path.join(GOLDEN, "ref", name + ".loadings")
    if os.path.exists(lpath):
        assert_cols_close(V, O.read_table(lpath), 2e-6 if prec == "fp64" else 5e-4)
    if prec in ("mixed", "bf16"):
        assert r.gemm_launches > 0


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name,mem", [("g1_win_m", 0.0001), ("g1_win_m8", 0.0003)])
def test_rsvd_out_of_core_plan_matches_reference_golden(gpu, prec, name, mem):
    """-m: permute_plink order and winSVD windows of the -m block plan (src/Data.cpp:27-71,
    src/Halko.cpp:228-269); three blocks per band for g1_win_m, one for g1_win_m8."""
    bed = O.read_bed(os.path.join(GOLDEN, "g1"))
    bs, nblocks, bf = pb.block_plan(bed.N, bed.M, 4, 10, mem, 8)
    perm = pb.plink_perm(bed.M, bed.N, 8)
    gpu.load_bed(bed.packed, bed.N)
    gpu.permute(perm)
    r = gpu.rsvd(svd=2, k=4, bands=8, precision=prec, block_snps=bs, band_factor=bf)
    V = np.empty_like(r.V)
    V[perm] = r.V
    assert_eig_close(r.S ** 2 / bed.M * 2, ref_eigvals(name), 1e-5)
    tol = 2e-6 if prec == "fp64" else 5e-4
    assert_cols_close(r.U, ref_table(name, ".eigvecs"), tol)
    assert_cols_close(V, O.read_table(os.path.join(GOLDEN, "ref", name + ".loadings")), tol)
    eig_o, S_o, U_o, V_o, F_o, ep_o = O.run_pca(bed, k=4, bands=8, memory=mem)
    assert r.epochs == ep_o


@pytest.mark.parametrize("svd,bands", [(1, 0), (2, 16), (2, 64)])
def test_rsvd_matches_oracle_larger(gpu, svd, bands):
    bed = random_bed(1502, 9001, seed=5, miss=0.01)
    kw = dict(k=6, maxp=6, tol=0.0) if svd == 1 else dict(k=6, maxp=8, bands=bands)
    eig_o, S_o, U_o, V_o, F_o, ep_o = O.run_pca(bed, svd=svd, **kw)
    for prec, rtol, ang in [("fp64", 1e-9, 1e-7), ("fp32", 1e-5, 1e-3), ("mixed", 1e-5, 1e-3),
                            ("bf16", 1e-5, 1e-3)]:
        r, V = run_gpu(gpu, bed, svd == 2, precision=prec, svd=svd, **kw)
        assert r.epochs == ep_o
        assert_eig_close(r.S ** 2 / bed.M * 2, eig_o, rtol)
        assert max_angle(r.U, U_o) <= ang
        assert max_angle(V, V_o) <= ang


@pytest.mark.parametrize("prec", ["fp64", "mixed", "bf16"])
def test_emu_matches_reference_golden(gpu, prec):
    """EMU (--emu -k 3 -w 8 --maxiter 20 --tol-em 1e-6) against the reference's outputs."""
    packed, N, M = pb.read_bed(os.path.join(GOLDEN, "g2"))
    eig, S, U, V, iters = pb.run_emu(gpu, packed, N, k=3, bands=8, maxiter=20, tolem=1e-6,
                                     precision=prec)
    assert_eig_close(eig, ref_eigvals("g2_emu"), 1e-5)
    tol = 2e-6 if prec == "fp64" else 5e-4
    assert_cols_close(U, ref_table("g2_emu", ".eigvecs"), tol)
    assert_cols_close(V, ref_table("g2_emu", ".loadings"), tol)


def test_emu_matches_oracle_other_modes(gpu):
    """Halko (-d 1) and unshuffled EMU, where the reference itself crashes: oracle only."""
    bed = O.read_bed(os.path.join(GOLDEN, "g2"))
    for svd, shuffle in [(1, False), (2, False)]:
        eig_o, S_o, U_o, V_o, F_o, it_o, _ = O.run_emu(bed, k=3, svd=svd, bands=8, maxiter=10,
                                                       tolem=1e-6, shuffle=shuffle)
        eig, S, U, V, it = pb.run_emu(gpu, bed.packed, bed.N, k=3, svd=svd, bands=8, maxiter=10,
                                      tolem=1e-6, shuffle=shuffle, precision="fp64")
        assert it == it_o
        assert_eig_close(eig, eig_o, 1e-9)
        assert max_angle(U, U_o) < 1e-7


@pytest.mark.parametrize("name,shuffle", [("g1_pcangsd_bed", True), ("g1_pcangsd_bedS", False)])
def test_pcangsd_on_plink_matches_reference_golden(gpu, name, shuffle):
    """PCAngsd on PLINK input (-b g1 --pcangsd -k 3 -w 8 --maxiter 30, with and without -S):
    pseudo-likelihoods and the first RSVD on the centred genotypes, built on the device."""
    packed, N, M = pb.read_bed(os.path.join(GOLDEN, "g1"))
    eig, S, U, V, iters, F = pb.run_pcangsd_bed(gpu, packed, N, k=3, bands=8, maxiter=30, shuffle=shuffle)
    np.testing.assert_array_equal(F, O.allele_freq(O.decode_codes(O.read_bed(os.path.join(GOLDEN, "g1")))))
    assert_eig_close(eig, ref_eigvals(name), 1e-5)
    assert_cols_close(U, ref_table(name, ".eigvecs"), 5e-4)
    assert_cols_close(V, ref_table(name, ".loadings"), 5e-4)


@pytest.mark.parametrize("name,shuffle", [("g3_pcangsd", False), ("g3_pcangsd_shuf", True)])
def test_pcangsd_matches_reference_golden(gpu, name, shuffle):
    """PCAngsd (-G g3.beagle.gz -k 3 -w 8 --maxiter 30, with and without -S)."""
    P, N, M = O.parse_beagle(os.path.join(GOLDEN, "g3.beagle.gz"))
    eig, S, U, V, iters, F = pb.run_pcangsd(gpu, P, k=3, bands=8, maxiter=30, shuffle=shuffle)
    np.testing.assert_allclose(F, O.em_maf(P, 30, 1e-6), rtol=1e-6)
    assert_eig_close(eig, ref_eigvals(name), 1e-5)
    assert_cols_close(U, ref_table(name, ".eigvecs"), 5e-4)
    if not shuffle:
        assert_cols_close(V, ref_table(name, ".loadings"), 5e-4)


@pytest.fixture(scope="module")
def bench_shape_oracle():
    """The benchmark's schedule (k = 20, l = 40, 64 windows, shuffled, the reference's default
    maxp/tol) on a 4000 x 32000 matrix with 0.5% missing, run once by the FP64 oracle."""
    bed = random_bed(4000, 32000, seed=11, miss=0.005)
    return bed, O.run_pca(bed, svd=2, k=20, maxp=20, bands=64)


@pytest.mark.parametrize("prec", ["mixed", "bf16"])
def test_winsvd_bench_shape_matches_oracle(gpu, bench_shape_oracle, prec):
    """Eigenvalues to 1e-5 relative and a largest principal angle of 1e-3 rad (the mixed-precision
    bar) against the FP64 oracle; the leading four PCs to 1e-4 rad."""
    bed, (eig_o, S_o, U_o, V_o, F_o, ep_o) = bench_shape_oracle
    r, V = run_gpu(gpu, bed, True, precision=prec, svd=2, k=20, maxp=20, bands=64)
    assert r.epochs == ep_o
    assert_eig_close(r.S ** 2 / bed.M * 2, eig_o, 1e-5)
    assert max_angle(r.U, U_o) <= 1e-3
    assert max_angle(V, V_o) <= 1e-3
    assert max_angle(r.U[:, :4], U_o[:, :4]) <= 1e-4
