"""Streamed genotypes (pcaone_gpu_load_bed_host): the packed records stay in host memory and
the RSVD copies runs of windows into two device slots, the device side of the reference's
out-of-core mode (-m; src/FilePlink.cpp:133-294 over the block plan of src/Data.cpp:16-72).

With a slot large enough for every window the products see the same runs as the resident
path, so the results must be identical; with one window per slot they are checked against the
reference's -m goldens, the oracle and the resident path at each precision's tolerance."""
import os

import numpy as np
import pytest

import pcaone_b200 as pb
from oracle import pcaone_oracle as O
from tests.helpers import GOLDEN, assert_cols_close, assert_eig_close, max_angle, ref_eigvals, ref_table
from tests.test_gpu_rsvd import random_bed

pytestmark = pytest.mark.gpu

ONE_WINDOW = 1  # slot budget in bytes: one window (Halko: one 256-SNP block) per slot


def test_streamed_counts_match_resident(gpu):
    bed = random_bed(1003, 2500, seed=21, miss=0.03)
    gpu.load_bed(bed.packed, bed.N)
    a, c = gpu.counts()
    F = gpu.allele_freq()
    gpu.load_bed_host(bed.packed, bed.N, ONE_WINDOW)
    a2, c2 = gpu.counts()
    np.testing.assert_array_equal(a, a2)
    np.testing.assert_array_equal(c, c2)
    np.testing.assert_array_equal(F, gpu.allele_freq())
    perm = pb.shuffle_perm(bed.M)
    gpu.permute(perm)  # host records permuted, then counted again
    a3, c3 = gpu.counts()
    np.testing.assert_array_equal(a3, a[perm])
    np.testing.assert_array_equal(c3, c[perm])


@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed"])
def test_streamed_one_slot_identical_to_resident(gpu, prec):
    bed = random_bed(1502, 9001, seed=5, miss=0.01)
    perm = pb.shuffle_perm(bed.M)
    kw = dict(k=6, maxp=8, bands=16, svd=2, precision=prec)
    gpu.load_bed(bed.packed, bed.N)
    gpu.permute(perm)
    r = gpu.rsvd(**kw)
    gpu.load_bed_host(bed.packed, bed.N, 1 << 34)
    gpu.permute(perm)
    s = gpu.rsvd(**kw)
    assert s.epochs == r.epochs
    np.testing.assert_array_equal(s.S, r.S)
    np.testing.assert_array_equal(s.U, r.U)
    np.testing.assert_array_equal(s.V, r.V)


@pytest.mark.parametrize("prec", ["fp64", "fp32", "mixed"])
@pytest.mark.parametrize("name,mem", [("g1_win_m", 0.0001), ("g1_win_m8", 0.0003)])
def test_streamed_out_of_core_plan_matches_reference_golden(gpu, prec, name, mem):
    """-m with one window of the block plan per device slot: the reference's -m outputs."""
    bed = O.read_bed(os.path.join(GOLDEN, "g1"))
    bs, nblocks, bf = pb.block_plan(bed.N, bed.M, 4, 10, mem, 8)
    perm = pb.plink_perm(bed.M, bed.N, 8)
    gpu.load_bed_host(bed.packed, bed.N, ONE_WINDOW)
    gpu.permute(perm)
    r = gpu.rsvd(svd=2, k=4, bands=8, precision=prec, block_snps=bs, band_factor=bf)
    V = np.empty_like(r.V)
    V[perm] = r.V
    assert_eig_close(r.S ** 2 / bed.M * 2, ref_eigvals(name), 1e-5)
    tol = 2e-6 if prec == "fp64" else 5e-4
    assert_cols_close(r.U, ref_table(name, ".eigvecs"), tol)
    assert_cols_close(V, O.read_table(os.path.join(GOLDEN, "ref", name + ".loadings")), tol)


@pytest.mark.parametrize("svd,bands", [(1, 0), (2, 16)])
def test_streamed_small_slots_match_oracle(gpu, svd, bands):
    bed = random_bed(1502, 9001, seed=5, miss=0.01)
    kw = dict(k=6, maxp=6, tol=0.0) if svd == 1 else dict(k=6, maxp=8, bands=bands)
    eig_o, S_o, U_o, V_o, F_o, ep_o = O.run_pca(bed, svd=svd, **kw)
    perm = pb.shuffle_perm(bed.M) if svd == 2 else None
    for prec, rtol, ang in [("fp64", 1e-9, 1e-7), ("fp32", 1e-5, 1e-3), ("mixed", 1e-5, 1e-3)]:
        gpu.load_bed_host(bed.packed, bed.N, ONE_WINDOW)
        if perm is not None:
            gpu.permute(perm)
        r = gpu.rsvd(precision=prec, svd=svd, **kw)
        V = r.V
        if perm is not None:
            V = np.empty_like(r.V)
            V[perm] = r.V
        assert r.epochs == ep_o
        assert_eig_close(r.S ** 2 / bed.M * 2, eig_o, rtol)
        assert max_angle(r.U, U_o) <= ang
        assert max_angle(V, V_o) <= ang


def test_streamed_emu_matches_resident(gpu):
    """EMU on streamed genotypes (imputed values on the resident missing-entry lists)."""
    packed, N, M = pb.read_bed(os.path.join(GOLDEN, "g2"))
    eig, S, U, V, it = pb.run_emu(gpu, packed, N, k=3, bands=8, maxiter=20, tolem=1e-6, precision="fp64")
    perm = pb.shuffle_perm(M)
    gpu.load_bed_host(packed, N, ONE_WINDOW)
    gpu.permute(perm)
    eig2, S2, U2, V2, it2, _ = pb.emu_loop(gpu, k=3, svd=2, bands=8, maxiter=20, tolem=1e-6, precision="fp64")
    Vo = np.empty_like(V2)
    Vo[perm] = V2
    assert it2 == it
    assert_eig_close(eig2, eig, 1e-9)
    assert_cols_close(U2, U, 1e-7)
    assert_cols_close(Vo, V, 1e-7)
    assert_eig_close(eig2, ref_eigvals("g2_emu"), 1e-5)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", 2e-6), ("mixed", 5e-6)])
def test_streamed_gram_and_product_match_resident(gpu, prec, tol):
    """The IRAM operator Z (Z^T X) and the product Z^T B over streamed blocks (one window per
    slot) against the resident whole-matrix products, at the product tolerances."""
    bed = random_bed(777, 3001, seed=21, miss=0.02)
    rng = np.random.default_rng(3)
    X = rng.standard_normal((bed.N, 5))
    B = rng.standard_normal((bed.N, 6))
    gpu.load_bed(bed.packed, bed.N)
    y_res, g_res = gpu.gram_product(X, precision=prec), gpu.product_t(B, precision=prec)
    gpu.load_bed_host(bed.packed, bed.N, ONE_WINDOW)
    y_str, g_str = gpu.gram_product(X, precision=prec), gpu.product_t(B, precision=prec)
    rel = lambda a, b: float((np.abs(a - b).max(axis=0) / np.abs(b).max(axis=0)).max())
    assert rel(y_str, y_res) <= 2 * tol
    assert rel(g_str, g_res) <= 2 * tol


def test_streamed_rejects_resident_only_calls(gpu):
    bed = random_bed(300, 1200, seed=2)
    gpu.load_bed_host(bed.packed, bed.N)
    with pytest.raises(pb.PcaoneError) as e:
        gpu.product(np.zeros((bed.M, 4)), precision="fp32")
    assert e.value.status == 6 and "streamed" in str(e.value)
    with pytest.raises(pb.PcaoneError) as e:
        gpu.rsvd(k=4, svd=2, bands=8, precision="bf16")
    assert e.value.status == 1
    r = gpu.rsvd(k=4, svd=2, bands=8, precision="mixed")  # the context stays usable
    assert np.all(np.isfinite(r.S))
