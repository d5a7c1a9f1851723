"""ORACLE -- test infrastructure only.

A CPU restatement, in numpy (FP64), of the reference PCAone v0.6.0 hot path. It is the checker
for the CUDA path and is imported only by tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py``; the product never calls it.

Every function cites the reference file:line it restates (paths inside the PCAone project).
Its parity is pinned against the reference binary built by ``oracle/ref.mk`` (golden outputs
under ``tests/golden/``) and against the reference's own Omega/permutation draws
(``oracle/_ref/omega_ref``).
"""
from __future__ import annotations

import ctypes
import gzip
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))

# src/Common.hpp:57-58  BED2GENO = {1, -9 (missing), 0.5, 0} for codes 00, 01, 10, 11
BED2GENO = np.array([1.0, -9.0, 0.5, 0.0])
VAR_TOL = 1e-9  # src/Data.hpp:7


# --------------------------------------------------------------------------- RNG draws
def _rnglib():
    path = os.path.join(_HERE, "liboracle_rng.so")
    if not os.path.exists(path):
        import subprocess

        subprocess.check_call(["g++", "-O2", "-shared", "-fPIC", "-o", path,
                               os.path.join(_HERE, "rng.cpp")])
    lib = ctypes.CDLL(path)
    lib.oracle_omega.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_long,
                                 ctypes.c_void_p]
    lib.oracle_shuffle.argtypes = [ctypes.c_long, ctypes.c_void_p]
    return lib


def omega(seed: int, nrow: int, ncol: int, rand: int = 1) -> np.ndarray:
    """Omega as drawn by RsvdOpData::initOmg (src/Halko.cpp:14-22), column-major fill."""
    out = np.zeros(nrow * ncol)
    _rnglib().oracle_omega(seed, rand, nrow, ncol, out.ctypes.data)
    return out.reshape(ncol, nrow).T.copy()


def shuffle_perm(n: int) -> np.ndarray:
    """In-core SNP permutation of permute_matrix (src/RSVD.hpp:63-79)."""
    out = np.zeros(n, dtype=np.int32)
    _rnglib().oracle_shuffle(n, out.ctypes.data)
    return out


# --------------------------------------------------------------------------- PLINK input
@dataclass
class Bed:
    N: int
    M: int
    packed: np.ndarray  # (M, bpr) uint8, SNP-major as on disk

    @property
    def bpr(self) -> int:
        return (self.N + 3) >> 2


def count_lines(path: str) -> int:
    """count_lines (src/Utils.cpp:94-103)."""
    with open(path, "rb") as f:
        return sum(1 for _ in f)


def read_bed(prefix: str) -> Bed:
    """FileBed constructor (src/FilePlink.hpp:10-26): N from .fam, M from .bim, magic check."""
    N = count_lines(prefix + ".fam")
    M = count_lines(prefix + ".bim")
    raw = np.fromfile(prefix + ".bed", dtype=np.uint8)
    if raw.size < 3 or raw[0] != 0x6C or raw[1] != 0x1B or raw[2] != 0x01:
        raise ValueError("Incorrect magic number in plink bed file.")
    bpr = (N + 3) >> 2
    if raw.size < 3 + M * bpr:
        raise ValueError("truncated .bed")
    return Bed(N, M, raw[3:3 + M * bpr].reshape(M, bpr).copy())


def decode_codes(bed: Bed) -> np.ndarray:
    """2-bit codes as an (M, N) uint8 matrix (src/FilePlink.cpp:70-88, LSB-first)."""
    p = bed.packed
    codes = np.stack([(p >> (2 * k)) & 3 for k in range(4)], axis=2).reshape(bed.M, -1)
    return codes[:, :bed.N].copy()


def allele_counts(codes: np.ndarray):
    """Integer per-SNP counts (n_hom_A1, n_het, n_nonmissing) for FileBed::read_all
    (src/FilePlink.cpp:36-64)."""
    n00 = (codes == 0).sum(axis=1).astype(np.int64)
    n10 = (codes == 2).sum(axis=1).astype(np.int64)
    n01 = (codes == 1).sum(axis=1).astype(np.int64)
    nonmiss = codes.shape[1] - n01
    return n00, n10, nonmiss


def allele_freq(codes: np.ndarray) -> np.ndarray:
    """F_j = sum of BED2GENO over non-missing / count (src/FilePlink.cpp:36-57).
    The FP64 sum of {1, 0.5, 0} is exact, so F = ((2 n00 + n10) * 0.5) / c bit-for-bit."""
    n00, n10, c = allele_counts(codes)
    s = (2 * n00 + n10).astype(np.float64) * 0.5
    with np.errstate(invalid="ignore", divide="ignore"):
        F = np.where(c == 0, 0.0, s / np.maximum(c, 1))
    return F


def centered_matrix(codes: np.ndarray, F: np.ndarray) -> np.ndarray:
    """G (N x M) = BED2GENO[code] - F_j, missing -> 0 (src/FilePlink.cpp:70-115)."""
    G = BED2GENO[codes].T.copy()  # N x M
    miss = codes.T == 1
    G -= F[None, :]
    G[miss] = 0.0
    return G


def standardize(G: np.ndarray, F: np.ndarray, ploidy: int = 2) -> np.ndarray:
    """Data::standardize_E (src/Data.cpp:290-299): G_ij /= sqrt(ploidy F (1-F)) if > 1e-9."""
    sd = np.sqrt(float(ploidy) * F * (1 - F))
    out = G.copy()
    ok = sd > VAR_TOL
    out[:, ok] /= sd[ok][None, :]
    return out


def standardized_from_bed(bed: Bed, standardize_geno: bool = True) -> tuple[np.ndarray, np.ndarray]:
    codes = decode_codes(bed)
    F = allele_freq(codes)
    G = centered_matrix(codes, F)
    if standardize_geno:
        G = standardize(G, F)
    return G, F


# --------------------------------------------------------------------------- RSVD
def householder_q(H: np.ndarray) -> np.ndarray:
    """Thin Q of a Householder QR with R_ii = -sign(x_0)||x|| (Eigen::HouseholderQR and LAPACK
    dgeqrf share this sign convention)."""
    q, _ = np.linalg.qr(H, mode="reduced")
    return q


def flip_omg(Omg2: np.ndarray, Omg: np.ndarray) -> np.ndarray:
    """PCAone::flipOmg (src/RSVD.hpp:81-90). Returns the flipped Omg (also the new Omg2)."""
    out = Omg.copy()
    for i in range(out.shape[1]):
        if np.abs(Omg2[:, i] - out[:, i]).sum() > 2 * np.abs(Omg2[:, i] + out[:, i]).sum():
            out[:, i] *= -1
    return out


def mev(X: np.ndarray, Y: np.ndarray) -> float:
    """mev (src/Utils.cpp:192-198)."""
    return float(np.mean([np.linalg.norm(X.T @ Y[:, i]) for i in range(X.shape[1])]))


@dataclass
class RsvdResult:
    U: np.ndarray
    S: np.ndarray
    V: np.ndarray
    epochs: int
    diffs: list = field(default_factory=list)


def _usv_step(G, H, k):
    """One computeUSV epoch tail (src/Halko.cpp:54-69): QR(G) twice, B = R^-T H^T, SVD(B)."""
    Q1, R1 = np.linalg.qr(G, mode="reduced")
    Q2, R2 = np.linalg.qr(Q1, mode="reduced")
    R = R2 @ R1
    B = np.linalg.solve(R.T, H.T)
    ub, s, vbt = np.linalg.svd(B, full_matrices=False)
    return Q2, ub, s, vbt.T


class _HalkoState:
    def __init__(self, N, l, seed, rand):
        self.N, self.l, self.seed, self.rand = N, l, seed, rand
        self.init_omg()

    def init_omg(self):
        self.Omg = omega(self.seed, self.N, self.l, self.rand)
        self.Omg2 = self.Omg.copy()


def compute_usv(Z: np.ndarray, k: int, os_: int, p: int, tol: float, gandh, state,
                winsvd_bands: int | None = None) -> RsvdResult:
    """RsvdOpData::computeUSV (src/Halko.cpp:45-95). Z is N x M (samples x SNPs)."""
    N, M = Z.shape
    Upre = None
    diffs = []
    pi = 0
    Ucur = None
    while pi <= p:
        G, H = gandh(pi)
        Q2, ub, s, vb = _usv_step(G, H, k)
        Ucur = vb[:, :k]
        if pi > 0:
            diff = 1 - mev(Ucur, Upre)
            diffs.append(diff)
            if diff < tol or pi == p:
                if winsvd_bands is not None and 2 ** pi < winsvd_bands:
                    p = int(np.log2(winsvd_bands))
                else:
                    V = Q2 @ ub[:, :k]
                    return RsvdResult(Ucur, s[:k], V, pi + 1, diffs)
            else:
                Upre = Ucur
        else:
            Upre = Ucur
        pi += 1
    raise RuntimeError("unreachable")  # the loop always returns at pi == p


def halko(Z: np.ndarray, k: int, os_: int, p: int, tol: float, seed: int = 101,
          rand: int = 1) -> RsvdResult:
    """sSVD, NormalRsvdOpData::computeGandH in-core (src/Halko.cpp:97-125)."""
    N, M = Z.shape
    l = k + os_
    st = _HalkoState(N, l, seed, rand)
    last = {}

    def gandh(pi):
        if pi == 0:
            st.init_omg()
        else:
            st.Omg = flip_omg(st.Omg2, householder_q(last["H"]))
            st.Omg2 = st.Omg.copy()
        G = Z.T @ st.Omg
        H = Z @ G
        last["H"] = H
        return G, H

    return compute_usv(Z, k, os_, p, tol, gandh, st)


def plink_perm(nsnps: int, nsamples: int, nbands: int, gb: int = 2) -> np.ndarray:
    """permute_plink (src/FilePlink.cpp:298-405): the out-of-core SNP order. Each read buffer (a
    multiple of nbands SNPs, gb GB at most) deals its SNPs round-robin to nbands contiguous
    bands; perm[new] = old."""
    M, bpr = nsnps, (nsamples + 3) >> 2
    two = min(int(np.floor(1073741824 * gb / bpr)), M)
    bufsize = two // nbands
    two = bufsize * nbands
    nblocks = (M + two - 1) // two
    modr2 = M % two
    bufidx = bufsize
    modr, bandsize = M % nbands, (M + nbands - 1) // nbands
    bandidx = [b * bandsize if (modr == 0 or b < modr) else modr * bandsize + (bandsize - 1) * (b - modr)
               for b in range(nbands)]
    perm = np.full(M, -1, dtype=np.int64)
    for i in range(nblocks):
        if i == nblocks - 1 and modr2 != 0:
            two2 = M - (nblocks - 1) * two
            bufsize = (two2 + nbands - 1) // nbands
            modr2 = two2 % nbands
        for b in range(nbands):
            last = [bufsize - 1] if (i != nblocks - 1 or b < modr2 or modr2 == 0) else []
            for j in list(range(bufsize - 1)) + last:
                perm[i * bufidx + bandidx[b] + j] = i * two + j * nbands + b
    assert (perm >= 0).all()
    return perm.astype(np.int32)


def block_plan(nsamples: int, nsnps: int, k: int, os_: int, memory_gb: float, bands: int):
    """Data::prepare for the out-of-core winSVD (src/Data.cpp:27-71): (blocksize, band_factor)."""
    l = k + os_
    m = (3 * nsamples * l + 2 * nsnps * l + 5 * nsnps) / 134217728
    m = 0 if memory_gb > 1.1 * m else m
    bs = int(np.ceil(((m + memory_gb) * 134217728 - 3 * nsamples * l - 2 * nsnps * l - 5 * nsnps) / nsamples))
    nblocks = int(np.ceil(nsnps / bs))
    factor = 1
    if nblocks < bands:
        bs = int(np.ceil(nsnps / bands))
    else:
        factor = int(np.ceil(nblocks / bands))
        bs = int(np.ceil(nsnps / (bands * factor)))
    return bs, factor


def winsvd(Z: np.ndarray, k: int, os_: int, p: int, tol: float, bands: int, seed: int = 101,
           rand: int = 1, update_hook=None, state: dict | None = None, blocksize: int = 0,
           band_factor: int = 1) -> RsvdResult:
    """Window-based RSVD, FancyRsvdOpData::computeGandH in-core (src/Halko.cpp:153-226).
    Z must already be column-permuted when the reference permutes (src/Halko.cpp:181-184).

    `state` carries the window sums H1/H2 between successive calls: FancyRsvdOpData keeps
    them as members (src/Halko.hpp:68) and only zeroes them when 2^pi >= bands
    (src/Halko.cpp:159-163), so a second computeUSV on the same operator (the EM loops,
    src/Halko.cpp:301-336) starts from the previous call's leftover H2.

    blocksize > 0 gives the out-of-core schedule (src/Halko.cpp:228-269): the windows are the
    ceil(M / blocksize) blocks of the -m plan, bands start at band_factor blocks and the
    "adjacent" update falls on block 2^(pi-1) * band_factor."""
    N, M = Z.shape
    l = k + os_
    st = _HalkoState(N, l, seed, rand)
    if state is not None and "H1" in state:
        H1, H2 = state["H1"], state["H2"]
    else:
        H1 = np.zeros((N, l))
        H2 = np.zeros((N, l))
    if state is not None:
        state["H1"], state["H2"] = H1, H2
    sched = {"bandsize": 1}
    bf = band_factor if blocksize > 0 else 1
    blocksize = blocksize if blocksize > 0 else int(np.ceil(M / bands))
    nwin = int(np.ceil(M / blocksize))

    def gandh(pi):
        nonlocal H1, H2
        if pi == 0:
            st.init_omg()
        if 2 ** pi >= bands:
            H1[:] = 0
            H2[:] = 0
        if pi == 0:
            sched["bandsize"] = bf
        sched["bandsize"] = min(sched["bandsize"] * 2, nwin)
        bandsize = sched["bandsize"]
        G = np.zeros((M, l))
        H = None
        i = 1
        for b in range(nwin):
            s0 = b * blocksize
            s1 = M if (b + 1) * blocksize >= M else (b + 1) * blocksize
            if s0 < M:
                Gb = Z[:, s0:s1].T @ st.Omg
                G[s0:s1] = Gb
                if i <= bandsize // 2:
                    H1 += Z[:, s0:s1] @ Gb
                else:
                    H2 += Z[:, s0:s1] @ Gb
            adjacent = pi > 0 and (b + 1) == 2 ** (pi - 1) * bf and 2 ** pi < bands
            if (b + 1) < bandsize and not adjacent:
                i += 1
                continue
            if not (i == bandsize or i == bandsize // 2 or adjacent):
                i += 1
                continue
            H = H1 + H2
            st.Omg = flip_omg(st.Omg2, householder_q(H))
            st.Omg2 = st.Omg.copy()
            if update_hook is not None:
                update_hook(pi, b, st.Omg)
            if i == bandsize:
                H1[:] = 0
                i = 0
            else:
                H2[:] = 0
            i += 1
        return G, H

    return compute_usv(Z, k, os_, p, tol, gandh, st, winsvd_bands=bands)


def run_pca(bed: Bed, k: int = 10, svd: int = 2, maxp: int = 20, oversamples: int = 10,
            bands: int = 64, tol: float = 1e-4, seed: int = 101, rand: int = 1,
            shuffle: bool = True, standardize_geno: bool = True, memory: float = 0.0):
    """Plain (no EM) PLINK PCA, run_pca_with_halko (src/Halko.cpp:272-293, 338-342).
    Returns (eigvals, sigvals, U, V, F, epochs) with V in original SNP order."""
    os_ = max(oversamples, k)  # src/Cmd.cpp:190
    Z, F = standardized_from_bed(bed, standardize_geno)
    if svd == 1:
        res = halko(Z, k, os_, maxp, tol, seed, rand)
        V = res.V
    elif svd == 2 and memory > 0:  # out-of-core: permute_plink order and the block plan
        perm = plink_perm(bed.M, bed.N, bands) if shuffle else np.arange(bed.M, dtype=np.int32)
        bs, bf = block_plan(bed.N, bed.M, k, os_, memory, bands)
        res = winsvd(Z[:, perm], k, os_, maxp, tol, bands, seed, rand, blocksize=bs, band_factor=bf)
        V = np.empty_like(res.V)
        V[perm] = res.V
    elif svd == 2:
        perm = shuffle_perm(bed.M) if shuffle else np.arange(bed.M, dtype=np.int32)
        res = winsvd(Z[:, perm], k, os_, maxp, tol, bands, seed, rand)
        V = np.empty_like(res.V)
        V[perm] = res.V  # data->perm * V (src/Halko.cpp:340)
    else:
        raise ValueError("svd must be 1 or 2")
    eig = res.S ** 2 / bed.M * 2  # src/Halko.cpp:340, ploidy in src/Data.cpp:186
    return eig, res.S, res.U, V, F, res.epochs


def missing_mask(codes: np.ndarray) -> np.ndarray:
    """C: N x M boolean, True where the genotype is missing (src/FilePlink.cpp:79-85)."""
    return (codes == 1).T.copy()


def fit_emu(G: np.ndarray, miss: np.ndarray, U, S, V, Fclip) -> None:
    """Data::fit_with_pi EMU branch (src/Data.cpp:272-287), in place: missing entries of the
    centred G take clip(U S V^T, -F, 1 - F). G, miss are N x M in the current column order;
    Fclip[j] is the F the reference reads for column j."""
    pred = (U * S) @ V.T
    lo = -Fclip[None, :]
    hi = 1.0 - Fclip[None, :]
    G[miss] = np.clip(pred, lo, hi)[miss]


def run_emu(bed: Bed, k: int = 10, svd: int = 2, maxp: int = 20, oversamples: int = 10,
            bands: int = 64, tol: float = 1e-4, maxiter: int = 100, tolem: float = 1e-5,
            seed: int = 101, rand: int = 1, shuffle: bool = True, reference_index: bool = True):
    """EMU PCA, run_pca_with_halko impute branch with --emu (src/Halko.cpp:294-336, 338-342).

    Reference index semantics (reference_index=True): after the in-core shuffle G's columns
    are permuted but F stays in input order, so the clip bounds (src/Data.cpp:283) and the
    final standardize_E (src/Data.cpp:296) read F at the permuted position. The missing mask
    is read through the permutation (src/Data.cpp:277) and is correct.
    Returns (eigvals, S, U, V in input order, F, em_iterations, diffs)."""
    os_ = max(oversamples, k)
    codes = decode_codes(bed)
    F = allele_freq(codes)
    G = centered_matrix(codes, F)
    miss = missing_mask(codes)
    M = bed.M
    perm = shuffle_perm(M) if (svd == 2 and shuffle) else np.arange(M, dtype=np.int32)
    Gp = G[:, perm].copy()
    missp = miss[:, perm]
    Fclip = F if reference_index else F[perm]
    state = {}

    def rsvd(Z):
        if svd == 1:
            return halko(Z, k, os_, maxp, tol, seed, rand)
        return winsvd(Z, k, os_, maxp, tol, bands, seed, rand, state=state)

    res = rsvd(Gp)
    diffs = []
    it = 0
    for it in range(maxiter):
        Vpre = res.V
        fit_emu(Gp, missp, res.U, res.S, res.V, Fclip)
        res = rsvd(Gp)
        diff = 1.0 - mev(res.V, Vpre)
        diffs.append(diff)
        if diff < tolem:
            break
    # final standardised run (src/Halko.cpp:332-336)
    fit_emu(Gp, missp, res.U, res.S, res.V, Fclip)
    Gs = standardize(Gp, Fclip)
    res = rsvd(Gs)
    V = np.empty_like(res.V)
    V[perm] = res.V
    eig = res.S ** 2 / M * 2
    return eig, res.S, res.U, V, F, it + 1, diffs


def dense_eig(bed: Bed, k: int, standardize_geno: bool = True):
    """FP64 dense oracle: eigenvalues sigma^2/M*ploidy and U from the full SVD of Z."""
    Z, F = standardized_from_bed(bed, standardize_geno)
    u, s, vt = np.linalg.svd(Z, full_matrices=False)
    return s[:k] ** 2 / bed.M * 2, s[:k], u[:, :k], vt[:k].T


# --------------------------------------------------------------------------- comparisons
def principal_angles(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    qa, _ = np.linalg.qr(A)
    qb, _ = np.linalg.qr(B)
    s = np.linalg.svd(qa.T @ qb, compute_uv=False)
    return np.arccos(np.clip(s, -1.0, 1.0))


def max_col_err_up_to_sign(A: np.ndarray, B: np.ndarray) -> float:
    err = 0.0
    for i in range(A.shape[1]):
        e = min(np.abs(A[:, i] - B[:, i]).max(), np.abs(A[:, i] + B[:, i]).max())
        err = max(err, e)
    return err


# --------------------------------------------------------------------------- text IO
def fmt6(x: float) -> str:
    """One value as Eigen IOFormat(6, DontAlignCols, "\\t", "\\n") prints it (stream precision 6,
    default float format), i.e. C's %.6g."""
    return format(float(x), ".6g")


def read_table(path: str) -> np.ndarray:
    with open(path) as f:
        rows = [[float(t) for t in line.split("\t")] for line in f if line.strip()]
    return np.array(rows)


def read_ld_gz(path: str):
    with gzip.open(path, "rt") as f:
        head = f.readline()
        rows = [line.rstrip("\n").split("\t") for line in f]
    return head, rows


# --------------------------------------------------------------------------- LD r2
@dataclass
class SnpLD:
    chr: list
    pos: np.ndarray
    end_pos: list
    bims: list       # "chr\tpos\tid" per SNP (struct BIM, src/LD.hpp:18-28)
    ws: np.ndarray = None
    we: np.ndarray = None


def read_snp_pos(filebim: str) -> SnpLD:
    """get_snp_pos_bim (src/LD.cpp:51-74): chromosome runs, positions, and the BIM strings."""
    chrs, pos, end_pos, bims = [], [], [], []
    prev = None
    with open(filebim) as f:
        for i, line in enumerate(f):
            tok = [t for t in line.rstrip("\n").replace(" ", "\t").split("\t")]
            cur = tok[0]
            if prev is None:
                chrs.append(cur)
            elif prev != cur:
                end_pos.append(i - 1)
                chrs.append(cur)
            prev = cur
            pos.append(int(tok[3]))
            bims.append(tok[0] + "\t" + tok[3] + "\t" + tok[1])
    end_pos.append(len(pos) - 1)
    return SnpLD(chrs, np.array(pos, dtype=np.int64), end_pos, bims)


def divide_pos_by_window(snp: SnpLD, ld_bp: int) -> None:
    """divide_pos_by_window (src/LD.cpp:125-139): for each SNP i that is not at its
    chromosome's last position, the window holds the SNPs j >= i of that chromosome with
    pos_j - pos_i <= ld_bp (i included)."""
    ws, we = [], []
    c = 0
    n = len(snp.pos)
    for i in range(n):
        if snp.pos[i] == snp.pos[snp.end_pos[c]]:
            c += 1
            continue
        j = i
        while j <= snp.end_pos[c]:
            if snp.pos[j] - snp.pos[i] > ld_bp:
                break
            j += 1
        ws.append(i)
        we.append(j - i)
    snp.ws, snp.we = np.array(ws, dtype=np.int64), np.array(we, dtype=np.int64)


def ld_pairs(G: np.ndarray, snp: SnpLD):
    """ld_r2_big (src/LD.cpp:419-442): r = G_i.G_k * sds_i sds_k / (N-1), sds = 1/sd."""
    N = G.shape[0]
    sds = 1.0 / np.sqrt((G * G).sum(axis=0) / (N - 1))
    df = 1.0 / (N - 1)
    out_i, out_k, out_r = [], [], []
    for i, w in zip(snp.ws, snp.we):
        if w <= 1:
            continue
        ks = np.arange(i + 1, i + w)
        r = (G[:, ks].T @ G[:, i]) * (sds[i] * sds[ks] * df)
        out_i.append(np.full(len(ks), i))
        out_k.append(ks)
        out_r.append(r)
    if not out_i:
        return np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0)
    return np.concatenate(out_i), np.concatenate(out_k), np.concatenate(out_r)


def ld_flow_a(bed: Bed, U: np.ndarray | None):
    """run_ld_stuff with PLINK + --read-U (src/LD.cpp:444-468): centred G (not standardised,
    pca is off for LD, src/Cmd.cpp:166-169) projected off U: G = (I - U U^T) G. Clumping
    (src/LD.cpp:474-505) skips the projection and reads the centred G itself (U = None)."""
    codes = decode_codes(bed)
    F = allele_freq(codes)
    G = centered_matrix(codes, F)
    return G if U is None else G - U @ (U.T @ G)


def read_residuals(path: str) -> np.ndarray:
    """FileBin::read_all (src/FileBinary.cpp:21-30): int32 nsnps, nsamples, then float32
    columns; each column re-centred."""
    with open(path, "rb") as f:
        hdr = np.frombuffer(f.read(8), dtype=np.uint32)
        M, N = int(hdr[0]), int(hdr[1])
        G = np.frombuffer(f.read(4 * M * N), dtype=np.float32).reshape(M, N).T.astype(np.float64)
    return G - G.mean(axis=0, keepdims=True)


def ld_lines(snp: SnpLD, i, k, r) -> list:
    """Text lines of the .ld.gz output: bims[i] \\t bims[k] \\t std::to_string(r*r)."""
    return [f"{snp.bims[a]}\t{snp.bims[b]}\t{x * x:.6f}" for a, b, x in zip(i, k, r)]


def _maf(a: float) -> float:
    return 1 - a if a > 0.5 else a  # MAF (src/Common.hpp:25)


def read_bim_af(filebim: str) -> list:
    """The allele frequencies get_snp_pos_bim reads from a 7-column (.mbim) file, else []
    (src/LD.cpp:61)."""
    af = []
    with open(filebim) as f:
        for line in f:
            tok = [t for t in line.rstrip("\n").replace(" ", "\t").split("\t")]
            if len(tok) == 7:
                af.append(float(tok[6]))
    return af


def ld_prune(snp: SnpLD, r2: dict, r2_tol: float, af: list) -> np.ndarray:
    """ld_prune_big / ld_prune_small (src/LD.cpp:141-242): windows in order; a lead SNP i that
    is still kept compares every kept follower k of its window; r^2 > r2_tol drops k, or i
    when the .mbim frequencies give k the larger MAF. r2[(i, k)] holds the pair's r^2."""
    keep = np.ones(len(snp.pos), dtype=bool)
    pick_random = len(af) == 0
    for i, w in zip(snp.ws, snp.we):
        if not keep[i]:
            continue
        for j in range(1, int(w)):
            k = i + j
            if not keep[k]:
                continue
            if r2[(int(i), int(k))] > r2_tol:
                o = k
                if not pick_random:
                    o = i if _maf(af[k]) > _maf(af[i]) else k
                keep[o] = False
    return keep


def read_assoc(path: str, colnames: str = "CHR,BP,P"):
    """valid_assoc_file, get_snp_pos_bim(header) and map_index_snps (src/LD.cpp:245-300) for
    one assoc-like file: (header line, column indices, per-chromosome target positions,
    per-chromosome {bp: (p, line)} of the SNPs with p <= p2 built later). Returns the header,
    the column indices, the SnpLD of the targets and the raw lines."""
    with open(path) as f:
        lines = f.read().splitlines()
    head = lines[0]
    fields = head.split("\t")
    want = colnames.split(",")
    idx = [-1, -1, -1]
    for j, col in enumerate(fields):
        for t in range(3):
            if col == want[t]:
                idx[t] = j
    if min(idx) < 0:
        raise ValueError("the assoc-like file has no " + want[idx.index(-1)] + " column")
    chrs, pos, end_pos = [], [], []
    prev = None
    for i, line in enumerate(lines[1:]):
        tok = line.replace(" ", "\t").split("\t")
        cur = tok[idx[0]]
        if prev is None:
            chrs.append(cur)
        elif prev != cur:
            end_pos.append(i - 1)
            chrs.append(cur)
        prev = cur
        pos.append(int(tok[idx[1]]))
    end_pos.append(len(pos) - 1)
    return head, idx, SnpLD(chrs, np.array(pos, dtype=np.int64), end_pos, []), lines[1:]


def assoc_pvals(lines: list, idx: list, clump_p2: float) -> list:
    """map_index_snps (src/LD.cpp:272-297): per chromosome, {bp: (p, line)} of the lines with
    p <= clump_p2. The first line of a new chromosome is inserted before the switch, so it
    lands in the previous chromosome's map (the reference's order of operations); the first
    insert of a bp wins."""
    vm, m = [], {}
    prev = None
    for line in lines:
        tok = line.split("\t")
        cur = tok[idx[0]]
        bp = int(tok[idx[1]])
        p = float(tok[idx[2]])
        if p <= clump_p2 and bp not in m:
            m[bp] = (p, line)
        if prev is not None and prev != cur:
            vm.append(m)
            m = {}
        prev = cur
    vm.append(m)
    return vm


def target_snp_idx(snp_t: SnpLD, snp: SnpLD):
    """get_target_snp_idx (src/LD.cpp:79-123): per target chromosome, the indices in the LD
    matrix of the target SNPs whose position occurs on that chromosome, and their positions."""
    idx_per_chr, bp_per_chr = [], []
    for tc, ch in enumerate(snp_t.chr):
        c = snp.chr.index(ch)
        e = snp.end_pos[c]
        s = snp.end_pos[c - 1] if c > 0 else 0
        mpos = {int(snp.pos[i]): i for i in range(s, e + 1)}
        e = snp_t.end_pos[tc]
        s = snp_t.end_pos[tc - 1] if tc > 0 else 0
        idx, bp = [], []
        for i in range(s, e + 1):
            p = int(snp_t.pos[i])
            if p in mpos:
                bp.append(p)
                idx.append(mpos[p])
        idx_per_chr.append(idx)
        bp_per_chr.append(bp)
    return idx_per_chr, bp_per_chr


def ld_clump(head: str, clump_bp: int, clump_r2: float, clump_p1: float, r2_of, idx_per_chr,
             bp_per_chr, pvals_per_chr) -> list:
    """ld_clump_single_pheno (src/LD.cpp:299-367): index SNPs (p <= clump_p1) in increasing p;
    each takes the still unclumped targets within clump_bp on either side (backward first)
    with r^2 >= clump_r2; output lines = the index SNP's assoc line + tab + the clumped
    positions by increasing p, comma-separated, or NONE. r2_of(a, b) gives r^2 of matrix
    columns a < b."""
    out = [head + "\tSP2"]
    for c in range(len(bp_per_chr)):
        idx, bp = idx_per_chr[c], bp_per_chr[c]
        mbp = {}
        for j, b in enumerate(bp):
            mbp.setdefault(b, j)
        mpp = dict(pvals_per_chr[c])
        cand = sorted([(v[0], b) for b, v in mpp.items() if v[0] <= clump_p1])
        for _, p in cand:
            if p not in mpp or p not in mbp:
                continue
            j = mbp[p]
            clumped = []
            for direction in (-1, 1):
                k = j
                while True:
                    k += direction
                    if k < 0 or k >= len(bp):
                        break
                    if (direction < 0 and bp[k] < p - clump_bp) or (direction > 0 and bp[k] > p + clump_bp):
                        break
                    p2 = bp[k]
                    if p2 not in mpp:
                        continue
                    a, b = sorted((idx[j], idx[k]))
                    if r2_of(a, b) >= clump_r2:
                        clumped.append(p2)
                        del mpp[p2]
            line = pvals_per_chr[c][p][1] + "\t"
            if not clumped:
                line += "NONE"
            else:
                order = sorted(range(len(clumped)), key=lambda t: pvals_per_chr[c][clumped[t]][0])
                line += ",".join(str(clumped[t]) for t in order)
            out.append(line)
    return out


def read_usv(path: str) -> np.ndarray:
    """read_usv (src/Utils.cpp:255-286): the tab-separated table is read row by row into one
    vector, which is then viewed as a column-major (rows x cols) matrix
    (Eigen::Map<Mat2D>(V.data(), j, k)), so the returned U is the file's row-major values
    laid out column-major. LD flow A uses this U (src/LD.cpp:462)."""
    T = read_table(path)
    j, k = T.shape
    return T.ravel().reshape(k, j).T.copy()


# --------------------------------------------------------------------------- PCAngsd
def parse_beagle(path: str):
    """FileBeagle constructor + parse_beagle_file (src/FileBeagle.hpp:8-40,
    src/Utils.cpp:377-405): N = columns/3 - 1; P is 2N x M holding the first two of the three
    genotype likelihoods per sample (the third is implied as 1 - P0 - P1)."""
    with gzip.open(path, "rt") as f:
        head = f.readline().split()
        N = len(head) // 3 - 1
        rows = [line.split()[3:] for line in f if line.strip()]
    M = len(rows)
    gl = np.array(rows, dtype=np.float64).reshape(M, N, 3)
    P = np.empty((2 * N, M))
    P[0::2] = gl[:, :, 0].T
    P[1::2] = gl[:, :, 1].T
    return P, N, M


def _posterior(P, F, pt):
    """p0 = P0 (1-pt)^2, p1 = P1 2 pt (1-pt), p2 = (1 - P0 - P1) pt^2 (src/Data.cpp:264-266)."""
    P0, P1 = P[0::2], P[1::2]
    p0 = P0 * (1.0 - pt) * (1.0 - pt)
    p1 = P1 * 2 * pt * (1.0 - pt)
    p2 = (1 - P0 - P1) * pt * pt
    return p0, p1, p2


def em_maf(P: np.ndarray, maxiter: int = 100, tolmaf: float = 1e-6):
    """emMAF_with_GL (src/Utils.cpp:501-531), F0 = 0.25."""
    N = P.shape[0] // 2
    M = P.shape[1]
    F = np.full(M, 0.25)
    for it in range(maxiter):
        Ft = F.copy()
        p0, p1, p2 = _posterior(P, F[None, :], F[None, :])
        F = ((p1 + 2.0 * p2) / (p0 + p1 + p2)).sum(axis=0) * (1.0 / (2.0 * N))
        if np.sqrt(((F - Ft) ** 2).sum() / M) < tolmaf:
            break
    return F


def pcangsd_e(P: np.ndarray, F: np.ndarray, pred: np.ndarray | None):
    """Posterior expected genotype minus 2F: FileBeagle::read_all initial E (pt = F,
    src/FileBeagle.cpp:121-143) or Data::fit_with_pi PCAngsd branch (src/Data.cpp:249-270)
    with pt = clip((U S V^T + 2F)/2, 1e-4, 1 - 1e-4)."""
    if pred is None:
        pt = np.broadcast_to(F[None, :], (P.shape[0] // 2, P.shape[1]))
    else:
        pt = np.clip((pred + 2.0 * F[None, :]) / 2.0, 1e-4, 1 - 1e-4)
    p0, p1, p2 = _posterior(P, F[None, :], pt)
    return (p1 + 2.0 * p2) / (p0 + p1 + p2) - 2.0 * F[None, :]


def pcangsd_standardize(P, F, pred):
    """Data::pcangsd_standardize_E (src/Data.cpp:301-343): standardised E and the diagonal
    Dc_i = sum_j sum_g (g - 2F_j)^2 post_g / (2 F_j (1 - F_j))."""
    pt = np.clip((pred + 2.0 * F[None, :]) / 2.0, 1e-4, 1 - 1e-4)
    p0, p1, p2 = _posterior(P, F[None, :], pt)
    s = p0 + p1 + p2
    E = (p1 + 2 * p2) / s - 2.0 * F[None, :]
    norm = np.sqrt(2.0 * F * (1.0 - F))
    ok = norm > VAR_TOL
    E[:, ok] /= norm[ok][None, :]
    f2 = 2.0 * F[None, :]
    tmp = (0 - f2) ** 2 * (p0 / s) + (1 - f2) ** 2 * (p1 / s) + (2 - f2) ** 2 * (p2 / s)
    Dc = (tmp / (2.0 * F * (1.0 - F))[None, :]).sum(axis=1)
    return E, Dc


def run_pcangsd(beagle: str, k: int = 10, svd: int = 2, maxp: int = 20, oversamples: int = 10,
                bands: int = 64, tol: float = 1e-4, maxiter: int = 100, tolem: float = 1e-5,
                tolmaf: float = 1e-6, seed: int = 101, rand: int = 1, shuffle: bool = True,
                reference_index: bool = True):
    """PCAngsd, run_pca_with_halko impute branch for Beagle input (src/Halko.cpp:294-331).

    Reference index semantics after the in-core shuffle: every EM step rebuilds E for
    position j from P[:, j], F[j] and the loading row V[j] of the previous run, then permutes
    the columns again (src/Halko.cpp:164-184), so position j ends up with SNP perm[j]'s
    likelihoods and the prediction of loading row perm[j]. Returns
    (eigvals, S, U, V in input order, F, iterations, C (GRM), Dc)."""
    P, N, M = parse_beagle(beagle)
    F = em_maf(P, maxiter, tolmaf)
    return _pcangsd_loop(P, F, pcangsd_e(P, F, None), k, svd, maxp, oversamples, bands, tol,
                         maxiter, tolem, seed, rand, shuffle, reference_index)


def bed_pseudo_gl(bed: Bed):
    """FileBed::read_all with --pcangsd (src/FilePlink.cpp:36-115): F from the genotypes,
    pseudo-likelihood pairs RR -> (1, 0), AA -> (0, 0), RA -> (0, 1), missing ->
    (0.333333, 0.333333) (P is 2N x M), and the centred matrix E = BED2GENO - F with
    missing -> 0 (N x M, not standardised)."""
    codes = decode_codes(bed)
    F = allele_freq(codes)
    P = np.empty((2 * bed.N, bed.M))
    c = codes.T  # N x M
    P[0::2] = np.where(c == 3, 1.0, np.where(c == 1, 0.333333, 0.0))
    P[1::2] = np.where(c == 2, 1.0, np.where(c == 1, 0.333333, 0.0))
    return P, F, centered_matrix(codes, F)


def run_pcangsd_bed(bed: Bed, k: int = 10, svd: int = 2, maxp: int = 20, oversamples: int = 10,
                    bands: int = 64, tol: float = 1e-4, maxiter: int = 100, tolem: float = 1e-5,
                    seed: int = 101, rand: int = 1, shuffle: bool = True,
                    reference_index: bool = True):
    """PCAngsd on PLINK input (-b with --pcangsd, src/Cmd.cpp:205-207): the EM loop of
    run_pca_with_halko (src/Halko.cpp:294-316) on the pseudo-likelihoods of bed_pseudo_gl,
    starting from the centred genotypes. Same return value as run_pcangsd."""
    P, F, E0 = bed_pseudo_gl(bed)
    return _pcangsd_loop(P, F, E0, k, svd, maxp, oversamples, bands, tol, maxiter, tolem, seed,
                         rand, shuffle, reference_index)


def _pcangsd_loop(P, F, E, k, svd, maxp, oversamples, bands, tol, maxiter, tolem, seed, rand,
                  shuffle, reference_index):
    N, M = P.shape[0] // 2, P.shape[1]
    os_ = max(oversamples, k)
    perm = shuffle_perm(M) if (svd == 2 and shuffle) else np.arange(M, dtype=np.int32)
    state = {}

    def rsvd(Z):
        if svd == 1:
            return halko(Z, k, os_, maxp, tol, seed, rand)
        return winsvd(Z, k, os_, maxp, tol, bands, seed, rand, state=state)

    res = rsvd(E[:, perm])
    it = 0
    for it in range(maxiter):
        Vpre = res.V
        if reference_index:
            pred = (res.U * res.S) @ res.V.T          # position j <- loading row j
            Z = pcangsd_e(P, F, pred)[:, perm]
        else:
            Vo = np.empty_like(res.V)
            Vo[perm] = res.V                            # loadings in input order
            Z = pcangsd_e(P, F, (res.U * res.S) @ Vo.T)[:, perm]
        res = rsvd(Z)
        if 1.0 - mev(res.V, Vpre) < tolem:
            break
    if reference_index:
        pred = (res.U * res.S) @ res.V.T
    else:
        Vo = np.empty_like(res.V)
        Vo[perm] = res.V
        pred = (res.U * res.S) @ Vo.T
    Es, Dc = pcangsd_standardize(P, F, pred)
    C = Es @ Es.T / M
    C[np.diag_indices(N)] = Dc / M
    V = np.empty_like(res.V)
    V[perm] = res.V
    return res.S ** 2 / M * 2, res.S, res.U, V, F, it + 1, C, Dc


def read_eigen_matrix(path: str) -> np.ndarray:
    """A matrix printed by Eigen's default stream format (space separated, aligned)."""
    with open(path) as f:
        return np.array([[float(t) for t in line.split()] for line in f if line.strip()])
