"""CPU tests: the oracle is pinned against the reference's own outputs (golden fixtures
made by the reference binary, tests/golden/make_golden.py) and the reference's own RNG."""
import os
import subprocess

import numpy as np
import pytest

from oracle import pcaone_oracle as O
from tests.helpers import GOLDEN, assert_cols_close, assert_eig_close, ref_eigvals, ref_table

REF_OMEGA = os.path.join(os.path.dirname(O._HERE), "oracle", "_ref", "omega_ref")


def g(name):
    return O.read_bed(os.path.join(GOLDEN, name))


def test_allele_freq_matches_reference_mbim():
    bed = g("g1")
    F = O.allele_freq(O.decode_codes(bed))
    mbim = [float(line.split("\t")[6]) for line in open(os.path.join(GOLDEN, "ref", "g1_halko.mbim"))]
    # the .mbim prints F with 6 significant digits
    np.testing.assert_allclose(F, mbim, rtol=5e-6, atol=1e-12)


@pytest.mark.parametrize("name,svd,kw", [
    ("g1_halko", 1, dict(k=4, oversamples=10, maxp=7, tol=0.0)),
    ("g1_halko_p3", 1, dict(k=3, maxp=3, seed=7)),
    ("g1_win", 2, dict(k=4, bands=16)),
    ("g1_winS", 2, dict(k=4, bands=8, shuffle=False)),
    ("g1_win_unif", 2, dict(k=3, bands=4, rand=0, seed=3, maxp=5)),
    ("g1_nostd", 1, dict(k=3, maxp=5, tol=0.0, standardize_geno=False)),
    ("g1_win_m", 2, dict(k=4, bands=8, memory=0.0001)),
    ("g1_win_m8", 2, dict(k=4, bands=8, memory=0.0003)),
])
def test_oracle_rsvd_matches_reference(name, svd, kw):
    bed = g("g1")
    eig, S, U, V, F, ep = O.run_pca(bed, svd=svd, **kw)
    assert_eig_close(eig, ref_eigvals(name), 1e-5)
    assert_cols_close(U, ref_table(name, ".eigvecs"), 2e-6)
    if os.path.exists(os.path.join(GOLDEN, "ref", name + ".loadings")):
        assert_cols_close(V, ref_table(name, ".loadings"), 2e-6)


@pytest.mark.skipif(not os.path.exists(REF_OMEGA), reason="reference build not present")
@pytest.mark.parametrize("rand", [0, 1])
def test_oracle_rng_matches_reference_build(rand):
    N, l, pn = 777, 13, 3001
    raw = subprocess.run([REF_OMEGA, "101", str(rand), str(N), str(l), str(pn)],
                         capture_output=True, check=True).stdout
    ref = np.frombuffer(raw[:N * l * 8], dtype=np.float64).reshape(l, N).T
    perm = np.frombuffer(raw[N * l * 8:], dtype=np.int32)
    assert np.array_equal(O.omega(101, N, l, rand), ref)
    assert np.array_equal(O.shuffle_perm(pn), perm)


def test_oracle_householder_sign_recovery():
    # CholeskyQR2 + modified-LU signs reproduce the Householder thin Q (LAPACK convention)
    rng = np.random.default_rng(3)
    for _ in range(200):
        n, l = int(rng.integers(40, 300)), int(rng.integers(2, 24))
        H = rng.standard_normal((n, l)) @ rng.standard_normal((l, l))
        W = H.T @ H
        R = np.linalg.cholesky(W).T
        Q = np.linalg.solve(R.T, H.T).T
        R2 = np.linalg.cholesky(Q.T @ Q).T
        Q = np.linalg.solve(R2.T, Q.T).T
        A = Q[:l, :l].copy()
        D = np.zeros(l)
        for i in range(l):
            D[i] = -1.0 if A[i, i] >= 0 else 1.0
            A[i, i] -= D[i]
            A[i + 1:, i] /= A[i, i]
            A[i + 1:, i + 1:] -= np.outer(A[i + 1:, i], A[i, i + 1:])
        np.testing.assert_allclose(Q * D, O.householder_q(H), atol=1e-8)


def test_oracle_emu_matches_reference():
    bed = g("g2")
    eig, S, U, V, F, it, diffs = O.run_emu(bed, k=3, bands=8, maxiter=20, tolem=1e-6)
    assert_eig_close(eig, ref_eigvals("g2_emu"), 1e-5)
    assert_cols_close(U, ref_table("g2_emu", ".eigvecs"), 2e-6)
    assert_cols_close(V, ref_table("g2_emu", ".loadings"), 2e-6)


def _ld_check(G, mbim, ref_gz):
    snp = O.read_snp_pos(os.path.join(GOLDEN, "ref", mbim))
    O.divide_pos_by_window(snp, 5000)
    i, k, r = O.ld_pairs(G, snp)
    head, ref = O.read_ld_gz(os.path.join(GOLDEN, "ref", ref_gz))
    assert head == "CHR_A\tBP_A\tSNP_A\tCHR_B\tBP_B\tSNP_B\tR2\n"
    assert O.ld_lines(snp, i, k, r) == ["\t".join(x) for x in ref]


def test_oracle_ld_flow_a_matches_reference():
    U = O.read_usv(os.path.join(GOLDEN, "ref", "g4_pcs.eigvecs"))
    _ld_check(O.ld_flow_a(g("g4"), U), "g4_pcs.mbim", "g4_ldA.ld.gz")


def test_oracle_ld_flow_b_matches_reference():
    G = O.read_residuals(os.path.join(GOLDEN, "ref", "g4_adj.residuals"))
    _ld_check(G, "g4_adj.mbim", "g4_ldB.ld.gz")


def _ld_G(flow):
    if flow == "A":
        U = O.read_usv(os.path.join(GOLDEN, "ref", "g4_pcs.eigvecs"))
        return O.ld_flow_a(g("g4"), U)
    if flow == "A0":  # clumping on PLINK input: the centred genotypes, not projected off U
        return O.ld_flow_a(g("g4"), None)
    return O.read_residuals(os.path.join(GOLDEN, "ref", "g4_adj.residuals"))


def _r2_of(G):
    nrm = (G * G).sum(axis=0)
    return lambda a, b: float((G[:, a] @ G[:, b]) ** 2 / (nrm[a] * nrm[b]))


@pytest.mark.parametrize("name,flow,bim", [("g4_pruneA", "A", "ref/g4_pcs.mbim"), ("g4_pruneA_bim", "A", "g4.bim"),
                                           ("g4_pruneB", "B", "ref/g4_adj.mbim")])
def test_oracle_ld_prune_matches_reference(name, flow, bim):
    G = _ld_G(flow)
    filebim = os.path.join(GOLDEN, bim)
    snp = O.read_snp_pos(filebim)
    O.divide_pos_by_window(snp, 5000)
    i, k, r = O.ld_pairs(G, snp)
    r2 = {(int(a), int(b)): float(x * x) for a, b, x in zip(i, k, r)}
    keep = O.ld_prune(snp, r2, 0.05, O.read_bim_af(filebim))
    lines = open(filebim).read().splitlines()
    assert [x for x, kk in zip(lines, keep) if kk] == open(os.path.join(GOLDEN, "ref", name + ".ld.prune.in")).read().splitlines()
    assert [x for x, kk in zip(lines, keep) if not kk] == \
        open(os.path.join(GOLDEN, "ref", name + ".ld.prune.out")).read().splitlines()
    assert 0 < keep.sum() < len(keep)


@pytest.mark.parametrize("name,flow,mbim,files,p1,p2,r2,bp", [
    ("g4_clumpA", "A0", "ref/g4_pcs.mbim", ["g4_a.assoc", "g4_b.assoc"], 0.01, 0.2, 0.05, 5000),
    ("g4_clumpB", "B", "ref/g4_adj.mbim", ["g4_a.assoc"], 0.05, 0.5, 0.03, 3000),
])
def test_oracle_ld_clump_matches_reference(name, flow, mbim, files, p1, p2, r2, bp):
    G = _ld_G(flow)
    snp = O.read_snp_pos(os.path.join(GOLDEN, mbim))
    r2_of = _r2_of(G)
    clumped = 0
    for t, fname in enumerate(files):
        head, idx, snp_t, lines = O.read_assoc(os.path.join(GOLDEN, fname))
        pv = O.assoc_pvals(lines, idx, p2)
        ipc, bpc = O.target_snp_idx(snp_t, snp)
        out = O.ld_clump(head, bp, r2, p1, r2_of, ipc, bpc, pv)
        ref = open(os.path.join(GOLDEN, "ref", f"{name}.p{t}.clump")).read().splitlines()
        assert out == ref
        clumped += sum(not x.endswith("NONE") for x in out[1:])
    assert clumped > 0


@pytest.mark.parametrize("name,shuffle", [("g3_pcangsd", False), ("g3_pcangsd_shuf", True)])
def test_oracle_pcangsd_matches_reference(name, shuffle):
    eig, S, U, V, F, it, C, Dc = O.run_pcangsd(os.path.join(GOLDEN, "g3.beagle.gz"), k=3,
                                               shuffle=shuffle, bands=8, maxiter=30)
    assert_eig_close(eig, ref_eigvals(name), 1e-5)
    assert_cols_close(U, ref_table(name, ".eigvecs"), 2e-6)
    if not shuffle:
        assert_cols_close(V, ref_table(name, ".loadings"), 2e-6)
    # the GRM pairs each site's likelihoods with the loading row the EM updates use (with the
    # shuffle: the permuted index), which the shuffled run's .cov pins
    Cr = O.read_eigen_matrix(os.path.join(GOLDEN, "ref", name + ".cov"))
    np.testing.assert_allclose(C, Cr, atol=1e-5)


def test_eigen_aligned_format_reproduces_reference_cov():
    """The text rule the CLI writes .cov and .eigvecs2 rows with (Eigen's default aligned
    stream output) reproduces the reference's own .cov byte for byte."""
    from tests.helpers import eigen_aligned
    path = os.path.join(GOLDEN, "ref", "g3_pcangsd.cov")
    with open(path) as f:
        text = f.read()
    assert eigen_aligned(O.read_eigen_matrix(path)) + "\n" == text


def test_oracle_matches_reference_at_config1_shape(tmp_path):
    """Config 1 at its full shape (2000 x 50000, Halko k=10, oversampling 10, -p 7 --tol-rsvd 0):
    the oracle against the reference binary's outputs, on the input the seeded simulator
    regenerates (sha256 recorded with the outputs)."""
    import gzip
    import hashlib
    import json

    root = os.path.dirname(O._HERE)
    sim = os.path.join(root, "pcaone_b200", "bin", "pcaone-sim")
    if not os.path.exists(sim):
        pytest.skip("simulator not built")
    with open(os.path.join(GOLDEN, "cases.json")) as f:
        rec = json.load(f)
    prefix = str(tmp_path / "c1")
    subprocess.check_call([sim, "--out", prefix] + rec["large_datasets"]["c1"], stdout=subprocess.DEVNULL)
    with open(prefix + ".bed", "rb") as f:
        assert hashlib.sha256(f.read()).hexdigest() == rec["large_bed_sha256"]["c1"]
    bed = O.read_bed(prefix)
    eig, S, U, V, F, ep = O.run_pca(bed, svd=1, k=10, oversamples=10, maxp=7, tol=0.0)
    assert ep == 8
    assert_eig_close(eig, ref_eigvals("c1_halko"), 1e-5)
    assert_cols_close(U, ref_table("c1_halko", ".eigvecs"), 2e-6)
    with gzip.open(os.path.join(GOLDEN, "ref", "c1_halko.loadings.gz"), "rt") as f:
        Vref = np.array([[float(t) for t in line.split()] for line in f])
    assert_cols_close(V[:Vref.shape[0]], Vref, 2e-6)


@pytest.mark.parametrize("name,shuffle", [("g1_pcangsd_bed", True), ("g1_pcangsd_bedS", False)])
def test_oracle_pcangsd_on_plink_matches_reference(name, shuffle):
    """-b with --pcangsd: pseudo-likelihoods from the genotypes (src/FilePlink.cpp:89-105)."""
    eig, S, U, V, F, it, C, Dc = O.run_pcangsd_bed(g("g1"), k=3, bands=8, maxiter=30, shuffle=shuffle)
    assert_eig_close(eig, ref_eigvals(name), 1e-5)
    assert_cols_close(U, ref_table(name, ".eigvecs"), 2e-6)
    assert_cols_close(V, ref_table(name, ".loadings"), 2e-6)


def test_oracle_dense_eig_matches_reference_iram():
    """--svd 0 (IRAM, converged to --itol 1e-6) gives the exact leading eigenpairs: the oracle's
    dense FP64 SVD of Z matches the reference's -d 0 outputs."""
    eig, S, U, V = O.dense_eig(g("g1"), 4)
    assert_eig_close(eig, ref_eigvals("g1_iram"), 1e-5)
    assert_cols_close(U, ref_table("g1_iram", ".eigvecs"), 2e-5)
    assert_cols_close(V, ref_table("g1_iram", ".loadings"), 2e-5)


def test_oracle_plink_perm_matches_reference_perm_bim():
    # -m writes the permuted .bim (src/FilePlink.cpp:298-405); row i of it is SNP perm[i]
    bed = g("g1")
    ids = [line.split()[1] for line in open(os.path.join(GOLDEN, "g1.bim"))]
    ref = [line.split()[1] for line in open(os.path.join(GOLDEN, "ref", "g1_win_m.perm.bim"))]
    perm = O.plink_perm(bed.M, bed.N, 8)
    assert [ids[j] for j in perm] == ref


def test_oracle_block_plan_windows():
    # the plans behind the two -m fixtures (203 samples, 1500 SNPs, -w 8): three blocks of 63
    # SNPs per band, and one block of 188 SNPs per band
    bed = g("g1")
    assert O.block_plan(bed.N, bed.M, 4, 10, 0.0001, 8) == (63, 3)
    assert O.block_plan(bed.N, bed.M, 4, 10, 0.0003, 8) == (188, 1)


def test_reference_iram_out_of_core_equals_in_core(tmp_path):
    """The reference's -d 0 with -m (its block-by-block Arnoldi operator) prints the same
    outputs as its in-core IRAM golden, which the streamed IRAM CLI test compares against."""
    ref = os.path.join(os.path.dirname(O._HERE), "oracle", "_ref", "PCAone")
    if not os.path.exists(ref):
        pytest.skip("reference binary not built")
    out = str(tmp_path / "iram_m")
    r = subprocess.run([ref, "-b", os.path.join(GOLDEN, "g1"), "-d", "0", "-k", "4", "-V", "-m", "0.0001",
                        "-o", out], capture_output=True, text=True, timeout=300, cwd=tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "out-of-core" in open(out + ".log").read()
    for ext in (".eigvals", ".eigvecs", ".loadings"):
        assert_cols_close(O.read_table(out + ext), ref_table("g1_iram", ext), 1e-6)
