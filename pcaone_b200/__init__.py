"""Python binding of the PCAone B200 C ABI (include/pcaone_gpu.h) over ctypes.

This is the ctypes stub a Python caller binds: it loads the in-tree ``lib/libpcaone_gpu.so``
and fails loudly when that library is missing. There is no CPU fallback: every compute call
runs on the GPU through the C ABI.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libpcaone_gpu.so")
BIN_DIR = os.path.join(_HERE, "bin")

PREC_FP32, PREC_MIXED, PREC_FP64, PREC_BF16 = 0, 1, 2, 3
PRECISIONS = {"fp32": PREC_FP32, "mixed": PREC_MIXED, "int8": PREC_MIXED, "bf16": PREC_BF16,
              "fp64": PREC_FP64}

STATUS = {0: "OK", 1: "EBADARG", 2: "EOOM", 3: "ECUDA", 4: "ETIMEOUT", 5: "ENUMERIC",
          6: "ESTATE", 7: "ENODEV"}

# C ABI symbols declared in include/pcaone_gpu.h
EXPORTS = ["pcaone_gpu_create", "pcaone_gpu_destroy", "pcaone_gpu_last_error",
           "pcaone_gpu_load_bed", "pcaone_gpu_counts", "pcaone_gpu_allele_freq",
           "pcaone_gpu_permute", "pcaone_shuffle_perm", "pcaone_omega", "pcaone_gpu_rsvd",
           "pcaone_gpu_product", "pcaone_gpu_fit_emu", "pcaone_gpu_clear_imputed",
           "pcaone_gpu_ld_r2", "pcaone_gpu_load_gl", "pcaone_gpu_gl_freq",
           "pcaone_gpu_gl_update", "pcaone_gpu_gl_grm", "pcaone_gpu_product_t_noalloc",
           "pcaone_gpu_bed_to_gl", "pcaone_gpu_load_gl_f32", "pcaone_gpu_gram_product",
           "pcaone_gpu_residuals", "pcaone_gpu_load_dense", "pcaone_plink_perm",
           "pcaone_gpu_ld_r2_f64", "pcaone_gpu_ld_timing", "pcaone_gpu_load_bed_host",
           "pcaone_gpu_gl_timing"]


class PcaoneError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class RsvdOpts(ctypes.Structure):
    _fields_ = [("k", ctypes.c_int32), ("oversamples", ctypes.c_int32),
                ("maxp", ctypes.c_int32), ("svd", ctypes.c_int32), ("bands", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("standardize", ctypes.c_int32),
                ("ploidy", ctypes.c_int32), ("seed", ctypes.c_int32), ("rand", ctypes.c_int32),
                ("tol", ctypes.c_double), ("verbose", ctypes.c_int32),
                ("profile", ctypes.c_int32), ("carry_window_state", ctypes.c_int32),
                ("block_snps", ctypes.c_int32), ("band_factor", ctypes.c_int32)]


class RsvdReport(ctypes.Structure):
    _fields_ = [("epochs", ctypes.c_int32), ("omega_updates", ctypes.c_int32),
                ("last_diff", ctypes.c_double), ("gpu_ms", ctypes.c_double),
                ("gemm_ms", ctypes.c_double), ("kernel_launches", ctypes.c_int64),
                ("gemm_launches", ctypes.c_int64), ("epilogue_ms", ctypes.c_double),
                ("update_ms", ctypes.c_double), ("tail_ms", ctypes.c_double),
                ("host_ms", ctypes.c_double), ("h2d_bytes", ctypes.c_uint64)]


_lib = None


def lib() -> ctypes.CDLL:
    """Load the in-tree C ABI library; raise if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C pcaone_b200`")
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, u32, u64 = ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint64
        L.pcaone_gpu_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
        L.pcaone_gpu_destroy.argtypes = [vp]
        L.pcaone_gpu_last_error.argtypes = [vp]
        L.pcaone_gpu_last_error.restype = ctypes.c_char_p
        L.pcaone_gpu_load_bed.argtypes = [vp, vp, u64, u32]
        L.pcaone_gpu_counts.argtypes = [vp, vp, vp]
        L.pcaone_gpu_allele_freq.argtypes = [vp, vp]
        L.pcaone_gpu_permute.argtypes = [vp, vp]
        L.pcaone_shuffle_perm.argtypes = [u64, vp]
        L.pcaone_omega.argtypes = [ctypes.c_int, ctypes.c_int, u64, u32, vp]
        L.pcaone_gpu_rsvd.argtypes = [vp, ctypes.POINTER(RsvdOpts), vp, vp, vp,
                                      ctypes.POINTER(RsvdReport)]
        L.pcaone_gpu_product.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         vp, u32, vp]
        L.pcaone_gpu_fit_emu.argtypes = [vp, vp, vp, vp, u32, ctypes.c_int]
        L.pcaone_gpu_clear_imputed.argtypes = [vp]
        L.pcaone_gpu_ld_r2.argtypes = [vp, vp, u32, vp, vp, u64, vp]
        L.pcaone_gpu_ld_r2_f64.argtypes = [vp, vp, u32, vp, vp, u64, vp]
        L.pcaone_gpu_ld_timing.argtypes = [vp, vp, vp]
        L.pcaone_gpu_load_gl.argtypes = [vp, vp, u64, u32]
        L.pcaone_gpu_load_bed_host.argtypes = [vp, vp, u64, u32, u64]
        L.pcaone_gpu_gl_timing.argtypes = [vp, vp]
        L.pcaone_gpu_gl_freq.argtypes = [vp, ctypes.c_int, ctypes.c_double, vp, vp]
        L.pcaone_gpu_bed_to_gl.argtypes = [vp]
        L.pcaone_gpu_load_gl_f32.argtypes = [vp, vp, u64, u32]
        L.pcaone_gpu_gram_product.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, u32, vp]
        L.pcaone_gpu_residuals.argtypes = [vp, vp, vp, vp, u32, u64, u64, vp]
        L.pcaone_gpu_load_dense.argtypes = [vp, vp, u64, u32]
        L.pcaone_plink_perm.argtypes = [u64, u32, u32, u32, vp]
        L.pcaone_gpu_gl_update.argtypes = [vp, vp, vp, vp, u32]
        L.pcaone_gpu_gl_grm.argtypes = [vp, vp, vp, vp, u32, vp, vp, vp]
        L.pcaone_gpu_product_t_noalloc.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, u32, vp]
        for name in EXPORTS:
            getattr(L, name).restype = ctypes.c_int if name != "pcaone_gpu_last_error" else ctypes.c_char_p
        _lib = L
    return _lib


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def shuffle_perm(n: int) -> np.ndarray:
    """The reference's in-core SNP shuffle (src/RSVD.hpp:63-79)."""
    out = np.zeros(n, dtype=np.int32)
    lib().pcaone_shuffle_perm(n, _ptr(out))
    return out


def plink_perm(nsnps: int, nsamples: int, nbands: int, buffer_gb: int = 2) -> np.ndarray:
    """The reference's out-of-core SNP order (permute_plink, src/FilePlink.cpp:298-405)."""
    out = np.zeros(nsnps, dtype=np.int32)
    st = lib().pcaone_plink_perm(nsnps, nsamples, buffer_gb, nbands, _ptr(out))
    if st != 0:
        raise PcaoneError(st, "pcaone_plink_perm failed")
    return out


def block_plan(nsamples: int, nsnps: int, k: int, oversamples: int, memory_gb: float, bands: int):
    """Data::prepare's out-of-core plan for the winSVD (src/Data.cpp:27-71): (blocksize,
    nblocks, band_factor) for -m memory_gb, l = k + max(oversamples, k)."""
    import math
    l = k + max(oversamples, k)
    m = (3 * nsamples * l + 2 * nsnps * l + 5 * nsnps) / 134217728
    m = 0 if memory_gb > 1.1 * m else m
    bs = math.ceil(((m + memory_gb) * 134217728 - 3 * nsamples * l - 2 * nsnps * l - 5 * nsnps) / nsamples)
    nblocks = math.ceil(nsnps / bs)
    factor = 1
    if nblocks < bands:
        bs = math.ceil(nsnps / bands)
    else:
        factor = math.ceil(nblocks / bands)
        bs = math.ceil(nsnps / (bands * factor))
    return bs, math.ceil(nsnps / bs), factor


def omega(seed: int, nrow: int, ncol: int, rand: int = 1) -> np.ndarray:
    """The reference's sketch Omega (src/Halko.cpp:14-22), nrow x ncol."""
    out = np.zeros(nrow * ncol)
    lib().pcaone_omega(seed, rand, nrow, ncol, _ptr(out))
    return out.reshape(ncol, nrow).T.copy()


@dataclass
class RsvdResult:
    U: np.ndarray
    S: np.ndarray
    V: np.ndarray
    epochs: int
    omega_updates: int
    last_diff: float
    gpu_ms: float
    gemm_ms: float
    kernel_launches: int
    gemm_launches: int
    epilogue_ms: float = 0.0
    update_ms: float = 0.0
    tail_ms: float = 0.0
    host_ms: float = 0.0
    h2d_bytes: int = 0


class GpuContext:
    """One GPU context (device memory, stream) holding one genotype matrix."""

    def __init__(self, device: int = 0):
        h = ctypes.c_void_p()
        st = lib().pcaone_gpu_create(device, ctypes.byref(h))
        if st != 0:
            raise PcaoneError(st, "pcaone_gpu_create failed")
        self._h = h
        self.N = self.M = 0

    def _check(self, st: int):
        if st != 0:
            msg = lib().pcaone_gpu_last_error(self._h).decode()
            raise PcaoneError(st, msg)

    def close(self):
        if self._h:
            lib().pcaone_gpu_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_bed(self, packed: np.ndarray, nsamples: int):
        """packed: (M, ceil(N/4)) uint8 SNP-major records."""
        packed = np.ascontiguousarray(packed, dtype=np.uint8)
        M = packed.shape[0]
        if packed.ndim != 2 or packed.shape[1] != (nsamples + 3) // 4:
            raise ValueError("packed must be (nsnps, ceil(nsamples/4)) bytes")
        self._check(lib().pcaone_gpu_load_bed(self._h, _ptr(packed), M, nsamples))
        self.N, self.M = nsamples, M

    def load_bed_host(self, packed: np.ndarray, nsamples: int, slot_bytes: int = 0):
        """The same records kept in (pinned) host memory and streamed to the device by runs of
        windows during rsvd (pcaone_gpu_load_bed_host); slot_bytes: device bytes per slot
        (0: 1 GiB)."""
        packed = np.ascontiguousarray(packed, dtype=np.uint8)
        M = packed.shape[0]
        if packed.ndim != 2 or packed.shape[1] != (nsamples + 3) // 4:
            raise ValueError("packed must be (nsnps, ceil(nsamples/4)) bytes")
        self._check(lib().pcaone_gpu_load_bed_host(self._h, _ptr(packed), M, nsamples, int(slot_bytes)))
        self.N, self.M = nsamples, M

    def counts(self):
        a = np.zeros(self.M, dtype=np.uint32)
        c = np.zeros(self.M, dtype=np.uint32)
        self._check(lib().pcaone_gpu_counts(self._h, _ptr(a), _ptr(c)))
        return a, c

    def allele_freq(self) -> np.ndarray:
        F = np.zeros(self.M)
        self._check(lib().pcaone_gpu_allele_freq(self._h, _ptr(F)))
        return F

    def permute(self, perm: np.ndarray):
        perm = np.ascontiguousarray(perm, dtype=np.int32)
        self._check(lib().pcaone_gpu_permute(self._h, _ptr(perm)))

    def rsvd(self, k: int = 10, oversamples: int = 10, maxp: int = 20, svd: int = 2,
             bands: int = 64, precision: int | str = PREC_FP32, standardize: bool = True,
             ploidy: int = 2, seed: int = 101, rand: int = 1, tol: float = 1e-4,
             verbose: bool = False, profile: bool = False, want_v: bool = True,
             carry: bool = False, block_snps: int = 0, band_factor: int = 0) -> RsvdResult:
        if isinstance(precision, str):
            precision = PRECISIONS[precision]
        os_ = max(oversamples, k)  # src/Cmd.cpp:190
        o = RsvdOpts(k, os_, maxp, svd, bands, precision, int(standardize), ploidy, seed,
                     rand, tol, int(verbose), int(profile), int(carry), block_snps, band_factor)
        # column-major outputs (filled completely by the library): U and V are returned as
        # Fortran-ordered (N x k, M x k) views, without a transposing copy
        U = np.empty((k, self.N))
        S = np.zeros(k)
        V = np.empty((k, self.M)) if want_v else None
        rep = RsvdReport()
        self._check(lib().pcaone_gpu_rsvd(self._h, ctypes.byref(o), _ptr(U), _ptr(S),
                                          _ptr(V), ctypes.byref(rep)))
        return RsvdResult(U.T, S, V.T if V is not None else None, rep.epochs,
                          rep.omega_updates, rep.last_diff, rep.gpu_ms, rep.gemm_ms,
                          rep.kernel_launches, rep.gemm_launches, rep.epilogue_ms,
                          rep.update_ms, rep.tail_ms, rep.host_ms, rep.h2d_bytes)


def _product(ctx: "GpuContext", B: np.ndarray, transpose: int, precision, standardize, ploidy):
    if isinstance(precision, str):
        precision = PRECISIONS[precision]
    B = np.asarray(B, dtype=np.float64)
    if B.ndim == 1:
        B = B[:, None]
    rows_in, rows_out = (ctx.N, ctx.M) if transpose == 0 else (ctx.M, ctx.N)
    if B.shape[0] != rows_in:
        raise ValueError(f"B must have {rows_in} rows")
    Bc = np.asfortranarray(B)
    out = np.zeros((rows_out, B.shape[1]), order="F")
    ctx._check(lib().pcaone_gpu_product(ctx._h, precision, transpose, int(standardize), ploidy,
                                        _ptr(Bc), B.shape[1], _ptr(out)))
    return np.ascontiguousarray(out)


GpuContext.product_t = lambda self, B, precision=PREC_FP64, standardize=True, ploidy=2: \
    _product(self, B, 0, precision, standardize, ploidy)
GpuContext.product_t.__doc__ = "Z^T B (nsnps x ncols) for B nsamples x ncols."
GpuContext.product = lambda self, B, precision=PREC_FP64, standardize=True, ploidy=2: \
    _product(self, B, 1, precision, standardize, ploidy)
GpuContext.product.__doc__ = "Z B (nsamples x ncols) for B nsnps x ncols."


def _gram_product(self, X, precision=PREC_FP64, standardize=True, ploidy=2):
    """Z (Z^T X) (nsamples x ncols) for X nsamples x ncols, on the device in one call."""
    if isinstance(precision, str):
        precision = PRECISIONS[precision]
    X = np.asarray(X, dtype=np.float64)
    if X.ndim == 1:
        X = X[:, None]
    if X.shape[0] != self.N:
        raise ValueError(f"X must have {self.N} rows")
    Xc = np.asfortranarray(X)
    Y = np.zeros(X.shape, order="F")
    self._check(lib().pcaone_gpu_gram_product(self._h, precision, int(standardize), ploidy, _ptr(Xc),
                                              X.shape[1], _ptr(Y)))
    return np.ascontiguousarray(Y)


GpuContext.gram_product = _gram_product


def _residuals(self, U=None, S=None, V=None, snp0=0, nsnp=None):
    """Residual rows (nsnp x nsamples float32) of pcaone_gpu_residuals; V holds the loadings of
    the nsnp SNPs from snp0 (current SNP order); no factors gives the centred genotypes."""
    nsnp = self.M - snp0 if nsnp is None else nsnp
    out = np.zeros((nsnp, self.N), dtype=np.float32)
    if U is None:
        self._check(lib().pcaone_gpu_residuals(self._h, None, None, None, 0, snp0, nsnp, _ptr(out)))
    else:
        Uf, Vf = np.asfortranarray(U, dtype=np.float64), np.asfortranarray(V, dtype=np.float64)
        Sf = np.ascontiguousarray(S, dtype=np.float64)
        self._check(lib().pcaone_gpu_residuals(self._h, _ptr(Uf), _ptr(Sf), _ptr(Vf), len(Sf), snp0, nsnp,
                                               _ptr(out)))
    return out


def _load_dense(self, X):
    """X: nsnps x nsamples float32 (the .residuals body), centred per row on the device."""
    X = np.ascontiguousarray(X, dtype=np.float32)
    self._check(lib().pcaone_gpu_load_dense(self._h, _ptr(X), X.shape[0], X.shape[1]))
    self.M, self.N = X.shape


GpuContext.residuals = _residuals
GpuContext.load_dense = _load_dense


def _fit_emu(self, U, S, V, reference_index=True):
    """Data::fit_with_pi EMU step on the device (see pcaone_gpu_fit_emu)."""
    k = len(S)
    Uf = np.asfortranarray(U, dtype=np.float64)
    Vf = np.asfortranarray(V, dtype=np.float64)
    Sf = np.ascontiguousarray(S, dtype=np.float64)
    self._check(lib().pcaone_gpu_fit_emu(self._h, _ptr(Uf), _ptr(Sf), _ptr(Vf), k,
                                         int(reference_index)))


def _clear_imputed(self):
    self._check(lib().pcaone_gpu_clear_imputed(self._h))


def _ld_r2(self, ws, we, U=None, f64=False):
    """r2 of every window pair (see pcaone_gpu_ld_r2, pcaone_gpu_ld_r2_f64 with f64); ws, we
    as divide_pos_by_window."""
    ws = np.ascontiguousarray(ws, dtype=np.int64)
    we = np.ascontiguousarray(we, dtype=np.int32)
    out = np.zeros(int(np.maximum(we - 1, 0).sum()), dtype=np.float64 if f64 else np.float32)
    Uf = None if U is None else np.asfortranarray(U, dtype=np.float64)
    k = 0 if U is None else U.shape[1]
    fn = lib().pcaone_gpu_ld_r2_f64 if f64 else lib().pcaone_gpu_ld_r2
    self._check(fn(self._h, _ptr(Uf), k, _ptr(ws), _ptr(we), len(ws), _ptr(out)))
    return out


GpuContext.ld_r2 = _ld_r2


def _ld_timing(self):
    """(device ms, band-Gram ms) of the last LD r2 call (see pcaone_gpu_ld_timing)."""
    a, b = ctypes.c_double(), ctypes.c_double()
    self._check(lib().pcaone_gpu_ld_timing(self._h, ctypes.byref(a), ctypes.byref(b)))
    return a.value, b.value


GpuContext.ld_timing = _ld_timing


def read_bim_positions(path: str):
    """Chromosome runs and positions of a .bim (get_snp_pos_bim, src/LD.cpp:51-77): returns
    (positions int64, last index of each chromosome run)."""
    pos, ends, prev = [], [], None
    with open(path) as f:
        for i, line in enumerate(f):
            tok = line.split()
            if prev is not None and tok[0] != prev:
                ends.append(i - 1)
            prev = tok[0]
            pos.append(int(tok[3]))
    ends.append(len(pos) - 1)
    return np.array(pos, dtype=np.int64), ends


def ld_windows(pos, ends, bp: int):
    """divide_pos_by_window (src/LD.cpp:125-139): (ws, we) of the windows of SNPs within bp
    of each lead SNP on its chromosome (none for a SNP at its chromosome's last position)."""
    pos = np.asarray(pos, dtype=np.int64)
    ws, we = [], []
    c = 0
    starts = [0] + [e + 1 for e in ends[:-1]]
    ordered = all(np.all(np.diff(pos[s:e + 1]) >= 0) for s, e in zip(starts, ends))
    for i in range(len(pos)):
        e = ends[c]
        if pos[i] == pos[e]:
            c += 1
            continue
        if ordered:  # the first SNP past bp, by bisection
            j = int(np.searchsorted(pos[i:e + 1], pos[i] + bp, side="right")) + i
        else:
            far = np.nonzero(pos[i:e + 1] - pos[i] > bp)[0]
            j = i + int(far[0]) if len(far) else e + 1
        ws.append(i)
        we.append(j - i)
    return np.array(ws, dtype=np.int64), np.array(we, dtype=np.int32)


def _load_gl(self, P: np.ndarray):
    """P: 2N x M likelihood pairs (first two of the three per sample and site). FP32 input is
    passed as is (pcaone_gpu_load_gl_f32), anything else as FP64."""
    N, M = P.shape[0] // 2, P.shape[1]
    if P.dtype == np.float32:
        Pf = np.asfortranarray(P)
        self._check(lib().pcaone_gpu_load_gl_f32(self._h, _ptr(Pf), M, N))
    else:
        Pf = np.asfortranarray(P, dtype=np.float64)
        self._check(lib().pcaone_gpu_load_gl(self._h, _ptr(Pf), M, N))
    self.N, self.M = N, M


def _gl_freq(self, maxiter=100, tolmaf=1e-6):
    F = np.zeros(self.M)
    it = ctypes.c_int(0)
    self._check(lib().pcaone_gpu_gl_freq(self._h, maxiter, tolmaf, _ptr(F), ctypes.byref(it)))
    return F, it.value


def _gl_update(self, U=None, S=None, V=None):
    if U is None:
        self._check(lib().pcaone_gpu_gl_update(self._h, None, None, None, 0))
        return
    Uf, Vf = np.asfortranarray(U, dtype=np.float64), np.asfortranarray(V, dtype=np.float64)
    Sf = np.ascontiguousarray(S, dtype=np.float64)
    self._check(lib().pcaone_gpu_gl_update(self._h, _ptr(Uf), _ptr(Sf), _ptr(Vf), len(S)))


def _gl_timing(self) -> float:
    """Device ms of the posterior kernel of the last gl_update (pcaone_gpu_gl_timing)."""
    t = ctypes.c_double()
    self._check(lib().pcaone_gpu_gl_timing(self._h, ctypes.byref(t)))
    return t.value


def _gl_grm(self, U, S, V, vectors=True):
    """PCAngsd GRM from the final factors (pcaone_gpu_gl_grm): returns (C, evecs, svals) with
    C nsamples x nsamples, evecs its singular vectors as columns (None unless vectors) and
    svals the singular values (None unless vectors)."""
    Uf, Vf = np.asfortranarray(U, dtype=np.float64), np.asfortranarray(V, dtype=np.float64)
    Sf = np.ascontiguousarray(S, dtype=np.float64)
    n = Uf.shape[0]
    C = np.empty((n, n), dtype=np.float64, order="F")
    ev = np.empty((n, n), dtype=np.float64, order="F") if vectors else None
    sv = np.empty(n, dtype=np.float64) if vectors else None
    self._check(lib().pcaone_gpu_gl_grm(self._h, _ptr(Uf), _ptr(Sf), _ptr(Vf), len(Sf), _ptr(C),
                                        _ptr(ev) if vectors else None, _ptr(sv) if vectors else None))
    return C, ev, sv


def _product_t_noalloc(self, d_B: int, ncols: int, d_out: int, standardize=True, ploidy=2):
    """Allocation-free Z^T B on caller-owned device buffers (raw device addresses of column-major
    FP64 nsamples x ncols B and nsnps x ncols out); see pcaone_gpu_product_t_noalloc."""
    self._check(lib().pcaone_gpu_product_t_noalloc(self._h, int(standardize), ploidy,
                                                   ctypes.c_void_p(d_B), ncols, ctypes.c_void_p(d_out)))


def _bed_to_gl(self):
    """Switch the loaded (optionally permuted) genotypes to the PCAngsd likelihood mode with
    pseudo-likelihoods (pcaone_gpu_bed_to_gl)."""
    self._check(lib().pcaone_gpu_bed_to_gl(self._h))


GpuContext.product_t_noalloc = _product_t_noalloc
GpuContext.bed_to_gl = _bed_to_gl
GpuContext.load_gl = _load_gl
GpuContext.gl_timing = _gl_timing
GpuContext.gl_freq = _gl_freq
GpuContext.gl_update = _gl_update
GpuContext.gl_grm = _gl_grm


def run_pcangsd(ctx: "GpuContext", P: np.ndarray, k: int = 10, svd: int = 2, bands: int = 64,
                maxp: int = 20, oversamples: int = 10, tol: float = 1e-4, maxiter: int = 100,
                tolem: float = 1e-5, tolmaf: float = 1e-6, seed: int = 101, rand: int = 1,
                shuffle: bool = True, reference_index: bool = True, grm: bool = False):
    """PCAngsd on the GPU: the impute branch of run_pca_with_halko for Beagle input
    (src/Halko.cpp:294-316). Returns (eigvals, S, U, V in input order, iterations, F); with
    grm, also (C, evecs, svals) of the GRM stage (src/Halko.cpp:317-331) from the final
    factors.

    The in-core shuffle is applied by feeding the RSVD the permuted posterior matrix: the
    likelihood columns are loaded in permuted order, and under the reference's index
    semantics each EM step predicts position j from loading row perm[j]."""
    M = P.shape[1]
    perm = shuffle_perm(M) if (svd == 2 and shuffle) else np.arange(M, dtype=np.int32)
    ctx.load_gl(P[:, perm])
    F_perm, _ = ctx.gl_freq(maxiter, tolmaf)
    ctx.gl_update()
    return _pcangsd_em(ctx, perm, F_perm, k, svd, bands, maxp, oversamples, tol, maxiter, tolem,
                       seed, rand, reference_index, grm)


def run_pcangsd_bed(ctx: "GpuContext", packed: np.ndarray, N: int, k: int = 10, svd: int = 2,
                    bands: int = 64, maxp: int = 20, oversamples: int = 10, tol: float = 1e-4,
                    maxiter: int = 100, tolem: float = 1e-5, seed: int = 101, rand: int = 1,
                    shuffle: bool = True, reference_index: bool = True):
    """PCAngsd on PLINK input (-b with --pcangsd): pseudo-likelihoods from the genotypes and F
    from the genotype counts (src/FilePlink.cpp:36-115), then the same EM loop as for Beagle
    input (src/Halko.cpp:294-316); the first RSVD runs on the centred, unstandardised
    genotypes. Returns (eigvals, S, U, V in input order, iterations, F)."""
    M = packed.shape[0]
    perm = shuffle_perm(M) if (svd == 2 and shuffle) else np.arange(M, dtype=np.int32)
    ctx.load_bed(packed, N)
    ctx.permute(perm)
    F_perm = ctx.allele_freq()
    ctx.bed_to_gl()
    return _pcangsd_em(ctx, perm, F_perm, k, svd, bands, maxp, oversamples, tol, maxiter, tolem,
                       seed, rand, reference_index, False)


def _pcangsd_em(ctx, perm, F_perm, k, svd, bands, maxp, oversamples, tol, maxiter, tolem, seed,
                rand, reference_index, grm):
    """The PCAngsd EM loop (src/Halko.cpp:294-316) on the likelihood matrix of ctx, whose SNP
    order is perm; returns the outputs of run_pcangsd."""
    M = len(perm)
    kw = dict(k=k, oversamples=oversamples, maxp=maxp, svd=svd, bands=bands, tol=tol,
              seed=seed, rand=rand, precision=PREC_FP32, standardize=False)
    r = ctx.rsvd(carry=False, **kw)
    it = 0
    for it in range(maxiter):
        Vpre = r.V
        Vuse = r.V[perm] if reference_index else r.V
        ctx.gl_update(r.U, r.S, Vuse)
        r = ctx.rsvd(carry=True, **kw)
        if 1.0 - mev(r.V, Vpre) < tolem:
            break
    V = np.empty_like(r.V)
    V[perm] = r.V
    F = np.empty_like(F_perm)
    F[perm] = F_perm
    out = (r.S ** 2 / M * 2, r.S, r.U, V, it + 1, F)
    if grm:
        out += ctx.gl_grm(r.U, r.S, r.V[perm] if reference_index else r.V)
    return out


GpuContext.fit_emu = _fit_emu
GpuContext.clear_imputed = _clear_imputed


def mev(X: np.ndarray, Y: np.ndarray) -> float:
    """1/k sum_i ||X^T Y_i|| (src/Utils.cpp:192-198)."""
    C = X.T @ Y
    return float(np.mean(np.linalg.norm(C, axis=0)))


def run_emu(ctx: "GpuContext", packed: np.ndarray, N: int, k: int = 10, svd: int = 2,
            bands: int = 64, maxp: int = 20, oversamples: int = 10, tol: float = 1e-4,
            maxiter: int = 100, tolem: float = 1e-5, seed: int = 101, rand: int = 1,
            shuffle: bool = True, precision=PREC_MIXED, reference_index: bool = True):
    """EMU PCA on the GPU: the impute branch of run_pca_with_halko with --emu
    (src/Halko.cpp:294-336). Returns (eigvals, S, U, V in input SNP order, iterations)."""
    ctx.load_bed(packed, N)
    M = packed.shape[0]
    perm = shuffle_perm(M) if (svd == 2 and shuffle) else None
    if perm is not None:
        ctx.permute(perm)
    eig, S, U, V, iters, _ = emu_loop(ctx, k, svd, bands, maxp, oversamples, tol, maxiter, tolem, seed,
                                      rand, precision, reference_index)
    if perm is not None:
        Vo = np.empty_like(V)
        Vo[perm] = V
        V = Vo
    return eig, S, U, V, iters


def emu_loop(ctx: "GpuContext", k: int = 10, svd: int = 2, bands: int = 64, maxp: int = 20,
             oversamples: int = 10, tol: float = 1e-4, maxiter: int = 100, tolem: float = 1e-5,
             seed: int = 101, rand: int = 1, precision=PREC_MIXED, reference_index: bool = True):
    """The EM iterations of EMU on the genotypes already loaded (and permuted) on ctx
    (src/Halko.cpp:294-336). Returns (eigvals, S, U, V in the context's SNP order, iterations,
    total epochs over all RSVD runs)."""
    kw = dict(k=k, oversamples=oversamples, maxp=maxp, svd=svd, bands=bands, tol=tol,
              seed=seed, rand=rand, precision=precision)
    ctx.clear_imputed()
    r = ctx.rsvd(standardize=False, carry=False, **kw)
    epochs = r.epochs
    it = 0
    for it in range(maxiter):
        Vpre = r.V
        ctx.fit_emu(r.U, r.S, r.V, reference_index)
        r = ctx.rsvd(standardize=False, carry=True, **kw)
        epochs += r.epochs
        if 1.0 - mev(r.V, Vpre) < tolem:
            break
    ctx.fit_emu(r.U, r.S, r.V, reference_index)
    r = ctx.rsvd(standardize=True, carry=True, **kw)
    epochs += r.epochs
    ctx.clear_imputed()
    return r.S ** 2 / ctx.M * 2, r.S, r.U, r.V, it + 1, epochs


def read_bed(prefix: str):
    """Read PLINK .bed/.bim/.fam: returns (packed (M, bpr) uint8, N, M)."""
    with open(prefix + ".fam", "rb") as f:
        N = sum(1 for _ in f)
    with open(prefix + ".bim", "rb") as f:
        M = sum(1 for _ in f)
    raw = np.fromfile(prefix + ".bed", dtype=np.uint8)
    if raw.size < 3 or raw[0] != 0x6C or raw[1] != 0x1B or raw[2] != 0x01:
        raise ValueError("Incorrect magic number in plink bed file.")
    bpr = (N + 3) // 4
    if raw.size < 3 + M * bpr:
        raise ValueError("truncated .bed file")
    return raw[3:3 + M * bpr].reshape(M, bpr), N, M
