"""The PCAone drop-in CLI (pcaone_b200/bin/PCAone) against the reference's own output files
for the same flags (golden fixtures), plus its input-error behaviour."""
import gzip
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import pcaone_oracle as O
from tests.helpers import (GOLDEN, assert_cols_close, assert_eig_close, case, eigen_aligned, ref_out,
                           ref_table, top_vectors_match)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "pcaone_b200", "bin", "PCAone")


def run_cli(args, tmp_path, check=True):
    out = subprocess.run([CLI] + args + ["-v", "0"], capture_output=True, text=True, cwd=tmp_path)
    if check:
        assert out.returncode == 0, out.stdout + out.stderr
    return out


def golden_args(name, tmp_path):
    c = case(name)
    args = [a.format(d=os.path.join(GOLDEN, c["dataset"]), g=GOLDEN) for a in c["args"]]
    return args + ["-o", str(tmp_path / name)]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["mixed", "fp64"])
@pytest.mark.parametrize("name", ["g1_halko", "g1_win", "g1_winS", "g1_nostd", "g1_win_unif", "g1_win_m",
                                  "g1_win_m8"])
def test_cli_matches_reference_outputs(tmp_path, prec, name):
    run_cli(golden_args(name, tmp_path) + ["--precision", prec], tmp_path)
    out = str(tmp_path / name)
    assert_eig_close(O.read_table(out + ".eigvals")[:, 0], ref_table(name, ".eigvals")[:, 0], 1e-5)
    with open(out + ".sigvals") as f, open(ref_out(name, ".sigvals")) as g:
        assert f.readline() == g.readline()  # "#N,M"
    tol = 2e-6 if prec == "fp64" else 5e-4
    assert_cols_close(O.read_table(out + ".eigvecs"), ref_table(name, ".eigvecs"), tol)
    if os.path.exists(ref_out(name, ".loadings")):
        assert_cols_close(O.read_table(out + ".loadings"), ref_table(name, ".loadings"), tol)
    if os.path.exists(ref_out(name, ".mbim")):
        # allele frequencies are bit-exact, so the text is identical
        assert open(out + ".mbim").read() == open(ref_out(name, ".mbim")).read()
    lines = open(out + ".eigvecs2").read().splitlines()
    assert lines[0].startswith("#FID\tIID\tPC1")
    assert len(lines) == 1 + O.count_lines(os.path.join(GOLDEN, "g1.fam"))


@pytest.mark.gpu
def test_cli_out_of_core_writes_permuted_fileset(tmp_path):
    """-m leaves the permute_plink fileset (src/FilePlink.cpp:339-403) beside the outputs."""
    run_cli(golden_args("g1_win_m", tmp_path), tmp_path)
    out = str(tmp_path / "g1_win_m")
    assert open(out + ".perm.bim").read() == open(ref_out("g1_win_m", ".perm.bim")).read()
    bed = O.read_bed(os.path.join(GOLDEN, "g1"))
    perm = O.plink_perm(bed.M, bed.N, 8)
    raw = open(out + ".perm.bed", "rb").read()
    assert raw[:3] == bytes([0x6C, 0x1B, 0x01])
    bpr = (bed.N + 3) // 4
    assert np.array_equal(np.frombuffer(raw[3:], np.uint8).reshape(bed.M, bpr), bed.packed.reshape(bed.M, bpr)[perm])
    assert open(out + ".perm.fam").read() == open(os.path.join(GOLDEN, "g1.fam")).read()
    # one block only: the reference refuses -m (src/Data.cpp:51)
    r = run_cli(["-b", os.path.join(GOLDEN, "g1"), "-k", "4", "-m", "8", "-o", str(tmp_path / "one")], tmp_path,
                check=False)
    assert r.returncode != 0 and "only one block" in r.stdout + r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["g1_pcangsd_bed", "g1_pcangsd_bedS"])
def test_cli_pcangsd_on_plink_matches_reference_outputs(tmp_path, name):
    """-b with --pcangsd: pseudo-likelihoods from the genotypes (src/FilePlink.cpp:89-105)."""
    run_cli(golden_args(name, tmp_path), tmp_path)
    out = str(tmp_path / name)
    assert_eig_close(O.read_table(out + ".eigvals")[:, 0], ref_table(name, ".eigvals")[:, 0], 1e-5)
    assert_cols_close(O.read_table(out + ".eigvecs"), ref_table(name, ".eigvecs"), 5e-4)
    assert_cols_close(O.read_table(out + ".loadings"), ref_table(name, ".loadings"), 5e-4)


@pytest.mark.gpu
def test_cli_iram_matches_reference_outputs(tmp_path):
    """--svd 0: restarted Lanczos on the device gram product against the reference's IRAM."""
    run_cli(golden_args("g1_iram", tmp_path), tmp_path)
    out = str(tmp_path / "g1_iram")
    assert_eig_close(O.read_table(out + ".eigvals")[:, 0], ref_table("g1_iram", ".eigvals")[:, 0], 1e-5)
    assert_cols_close(O.read_table(out + ".eigvecs"), ref_table("g1_iram", ".eigvecs"), 5e-4)
    assert_cols_close(O.read_table(out + ".loadings"), ref_table("g1_iram", ".loadings"), 5e-4)


@pytest.mark.gpu
def test_cli_iram_out_of_core_matches_reference_outputs(tmp_path):
    """--svd 0 with -m: the same Lanczos on the Gram product of streamed genotypes (blocks
    staged into device slots) gives the reference's IRAM outputs."""
    run_cli(golden_args("g1_iram", tmp_path) + ["-m", "0.0001"], tmp_path)
    out = str(tmp_path / "g1_iram")
    assert "running IRAM SVD with out-of-core mode." in open(out + ".log").read()
    assert_eig_close(O.read_table(out + ".eigvals")[:, 0], ref_table("g1_iram", ".eigvals")[:, 0], 1e-5)
    assert_cols_close(O.read_table(out + ".eigvecs"), ref_table("g1_iram", ".eigvecs"), 5e-4)
    assert_cols_close(O.read_table(out + ".loadings"), ref_table("g1_iram", ".loadings"), 5e-4)


@pytest.mark.gpu
def test_cli_emu_matches_reference_outputs(tmp_path):
    run_cli(golden_args("g2_emu", tmp_path), tmp_path)
    out = str(tmp_path / "g2_emu")
    assert_eig_close(O.read_table(out + ".eigvals")[:, 0], ref_table("g2_emu", ".eigvals")[:, 0], 1e-5)
    assert_cols_close(O.read_table(out + ".eigvecs"), ref_table("g2_emu", ".eigvecs"), 5e-4)
    assert_cols_close(O.read_table(out + ".loadings"), ref_table("g2_emu", ".loadings"), 5e-4)


@pytest.mark.gpu
def test_cli_maf_filter(tmp_path):
    d = os.path.join(GOLDEN, "g1")
    run_cli(["-b", d, "-d", "1", "-k", "3", "-p", "4", "--maf", "0.2", "-V", "--precision", "fp64",
             "-o", str(tmp_path / "maf")], tmp_path)
    bed = O.read_bed(d)
    F = O.allele_freq(O.decode_codes(bed))
    maf = np.minimum(F, 1 - F)
    keep = np.where(maf > 0.2)[0]
    assert O.count_lines(str(tmp_path / "maf.mbim")) == len(keep)
    sub = O.Bed(bed.N, len(keep), bed.packed[keep])
    eig, *_ = O.run_pca(sub, k=3, svd=1, maxp=4)
    assert_eig_close(O.read_table(str(tmp_path / "maf.eigvals"))[:, 0], eig, 1e-5)  # 6 printed digits


def test_cli_rejects_unknown_option(tmp_path):
    out = run_cli(["-b", os.path.join(GOLDEN, "g1"), "--no-such-flag"], tmp_path, check=False)
    assert out.returncode == 1 and "unknown option" in out.stderr


def test_cli_rejects_out_of_scope_mode(tmp_path):
    out = run_cli(["-b", os.path.join(GOLDEN, "g1"), "--project", "1"], tmp_path, check=False)
    assert out.returncode == 1


def test_cli_rejects_bad_magic_and_truncation(tmp_path):
    for suf in (".bim", ".fam"):
        shutil.copy(os.path.join(GOLDEN, "g1" + suf), tmp_path / ("bad" + suf))
    raw = open(os.path.join(GOLDEN, "g1.bed"), "rb").read()
    (tmp_path / "bad.bed").write_bytes(b"\x6c\x1b\x00" + raw[3:])
    out = run_cli(["-b", str(tmp_path / "bad")], tmp_path, check=False)
    assert out.returncode == 1 and "magic" in out.stderr
    (tmp_path / "bad.bed").write_bytes(raw[: len(raw) // 2])
    out = run_cli(["-b", str(tmp_path / "bad")], tmp_path, check=False)
    assert out.returncode == 1 and "shorter" in out.stderr


def test_cli_rejects_odd_windows(tmp_path):
    out = run_cli(["-b", os.path.join(GOLDEN, "g1"), "-w", "5"], tmp_path, check=False)
    assert out.returncode == 1


@pytest.mark.gpu
def test_cli_ld_flow_a_matches_reference(tmp_path):
    run_cli(golden_args("g4_ldA", tmp_path), tmp_path)
    head, got = O.read_ld_gz(str(tmp_path / "g4_ldA.ld.gz"))
    rhead, ref = O.read_ld_gz(ref_out("g4_ldA", ".ld.gz"))
    assert head == rhead and len(got) == len(ref)
    assert [x[:6] for x in got] == [x[:6] for x in ref]
    diff = np.abs(np.array([float(x[6]) for x in got]) - np.array([float(x[6]) for x in ref]))
    assert diff.max() <= 1.01e-6  # 6 printed decimals; the r2 values agree to 1e-5 or better


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["g4_pruneA", "g4_pruneA_bim", "g4_pruneB"])
def test_cli_ld_prune_matches_reference(tmp_path, name):
    """--ld-r2: the kept and removed SNP lists are identical to the reference's (r2 from the
    device in FP64, the greedy pass of src/LD.cpp:141-242 on the host)."""
    run_cli(golden_args(name, tmp_path), tmp_path)
    for suf in (".ld.prune.in", ".ld.prune.out"):
        assert open(str(tmp_path / name) + suf).read() == open(ref_out(name, suf)).read()


@pytest.mark.gpu
@pytest.mark.parametrize("name,files", [("g4_clumpA", 2), ("g4_clumpB", 1)])
def test_cli_ld_clump_matches_reference(tmp_path, name, files):
    """--clump: one .pN.clump per assoc-like file, identical to the reference's."""
    run_cli(golden_args(name, tmp_path), tmp_path)
    for t in range(files):
        suf = f".p{t}.clump"
        assert open(str(tmp_path / name) + suf).read() == open(ref_out(name, suf)).read()


@pytest.mark.gpu
def test_ld_r2_f64_matches_oracle(tmp_path):
    """pcaone_gpu_ld_r2_f64 on flow A (projected) and on the unprojected genotypes."""
    import pcaone_b200 as pb
    bed = O.read_bed(os.path.join(GOLDEN, "g4"))
    snp = O.read_snp_pos(os.path.join(GOLDEN, "g4.bim"))
    O.divide_pos_by_window(snp, 5000)
    U = O.read_usv(os.path.join(GOLDEN, "ref", "g4_pcs.eigvecs"))
    with pb.GpuContext(0) as ctx:
        ctx.load_bed(bed.packed, bed.N)
        for Uuse in (U, None):
            got = ctx.ld_r2(snp.ws, snp.we, Uuse, f64=True)
            i, k, r = O.ld_pairs(O.ld_flow_a(bed, Uuse), snp)
            np.testing.assert_allclose(got, r * r, rtol=1e-9, atol=1e-12)


@pytest.mark.gpu
def test_cli_ld_flow_b_matches_reference(tmp_path):
    """Flow B end to end: -D writes the .residuals matrix and .mbim (compared with the
    reference's), then -B reads it back for the windowed r2 (.ld.gz)."""
    run_cli(golden_args("g4_adj", tmp_path), tmp_path)
    out = str(tmp_path / "g4_adj")
    assert open(out + ".mbim").read() == open(ref_out("g4_adj", ".mbim")).read()
    got = np.fromfile(out + ".residuals", dtype=np.uint8)
    ref = np.fromfile(ref_out("g4_adj", ".residuals"), dtype=np.uint8)
    assert got.size == ref.size and np.array_equal(got[:8], ref[:8])  # header: nsnps, nsamples
    diff = np.abs(got[8:].view(np.float32) - ref[8:].view(np.float32))
    assert diff.max() <= 1e-5
    c = case("g4_ldB")
    args = [a.format(d=os.path.join(GOLDEN, c["dataset"]), g=GOLDEN) for a in c["args"]]
    args[args.index("-B") + 1] = out + ".residuals"
    args[args.index("-f") + 1] = out + ".mbim"
    run_cli(args + ["-o", str(tmp_path / "g4_ldB")], tmp_path)
    head, got = O.read_ld_gz(str(tmp_path / "g4_ldB.ld.gz"))
    rhead, ref = O.read_ld_gz(ref_out("g4_ldB", ".ld.gz"))
    assert head == rhead and [x[:6] for x in got] == [x[:6] for x in ref]
    d = np.abs(np.array([float(x[6]) for x in got]) - np.array([float(x[6]) for x in ref]))
    assert d.max() <= 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["g3_pcangsd", "g3_pcangsd_shuf"])
def test_cli_pcangsd_matches_reference_outputs(tmp_path, name):
    run_cli(golden_args(name, tmp_path), tmp_path)
    out = str(tmp_path / name)
    assert_eig_close(O.read_table(out + ".eigvals")[:, 0], ref_table(name, ".eigvals")[:, 0], 1e-5)
    assert_cols_close(O.read_table(out + ".eigvecs"), ref_table(name, ".eigvecs"), 5e-4)
    # GRM stage: .cov in Eigen's aligned text, .eigvecs2 = sample names + singular vectors
    with open(out + ".cov") as f:
        text = f.read()
    C = O.read_eigen_matrix(out + ".cov")
    assert text == eigen_aligned(C) + "\n"
    N = C.shape[0]
    np.testing.assert_array_equal(C, C.T)
    # both runs: with the shuffle the GRM's site/loading pairing follows the EM updates' index
    np.testing.assert_allclose(C, O.read_eigen_matrix(ref_out(name, ".cov")), atol=1e-5)
    with open(out + ".eigvecs2") as f:
        lines = f.read().split("\n")
    assert lines[0] == "#FID\tIID" + "".join(f"\tPC{i + 1}" for i in range(N))
    with gzip.open(os.path.join(GOLDEN, "g3.beagle.gz"), "rt") as g:
        names = g.readline().split()[3::3]
    ev = np.empty((N, N))
    for i in range(N):
        a, b, row = lines[1 + i].split("\t")
        assert a == b == names[i]
        ev[i] = [float(t) for t in row.split()]
        assert row == eigen_aligned(ev[i])
    assert lines[1 + N] == ""
    top_vectors_match(ev, C, 3, 1e-4)
