"""CPU tests of the C ABI library: it loads, exports every declared symbol, and its host-side
RNG entry points reproduce the reference's draws (no GPU needed for these)."""
import ctypes
import os
import re

import numpy as np

import pcaone_b200 as pb
from oracle import pcaone_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "pcaone_gpu.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(pcaone_\w+)\s*\(", src, re.M)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(pb.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 10
    for s in syms:
        assert hasattr(lib, s), s
    assert set(pb.EXPORTS) <= set(syms)


def test_omega_and_shuffle_match_oracle():
    for seed, rand in [(101, 1), (7, 0), (3, 1)]:
        np.testing.assert_array_equal(pb.omega(seed, 500, 17, rand), O.omega(seed, 500, 17, rand))
    np.testing.assert_array_equal(pb.shuffle_perm(10007), O.shuffle_perm(10007))


def test_plink_perm_and_block_plan_match_oracle():
    # single read buffer (g1-like sizes) and many buffers (1e8 samples -> 40 SNPs per 1 GB
    # buffer with 4 bands), with and without a ragged last buffer and ragged bands
    for M, N, nb, gb in [(1000, 100, 8, 2), (1013, 100, 8, 2), (1000, 100_000_000, 4, 1),
                         (1013, 100_000_000, 4, 1), (997, 100_000_000, 8, 1), (64, 7, 64, 2)]:
        p = pb.plink_perm(M, N, nb, gb)
        np.testing.assert_array_equal(p, O.plink_perm(M, N, nb, gb))
        assert np.array_equal(np.sort(p), np.arange(M))
    for N, M, k, os_, mem, nb in [(100, 1000, 4, 10, 0.0001, 8), (100, 1000, 4, 10, 0.0003, 8),
                                  (2000, 50000, 10, 10, 0.05, 64)]:
        bs, nblocks, bf = pb.block_plan(N, M, k, os_, mem, nb)
        assert (bs, bf) == O.block_plan(N, M, k, max(os_, k), mem, nb)
        assert nblocks == -(-M // bs)


def test_create_without_device_fails_cleanly():
    import subprocess
    import sys
    code = ("import pcaone_b200 as pb\n"
            "try:\n    pb.GpuContext(999)\nexcept pb.PcaoneError as e:\n    print('ERR', e.status)\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT)
    assert "ERR 7" in out.stdout, out.stdout + out.stderr


def test_ld_windows_match_oracle():
    """The package's window helper (bisection on sorted positions, a scan otherwise) against
    the oracle's restatement of divide_pos_by_window: the golden .bim, a synthetic three-
    chromosome layout with repeated positions, and an unsorted chromosome."""
    import os

    import numpy as np

    import pcaone_b200 as pb
    from oracle import pcaone_oracle as O
    from tests.helpers import GOLDEN

    bim = os.path.join(GOLDEN, "g4.bim")
    pos, ends = pb.read_bim_positions(bim)
    for bp in (1, 500, 5000, 10 ** 9):
        ws, we = pb.ld_windows(pos, ends, bp)
        snp = O.read_snp_pos(bim)
        O.divide_pos_by_window(snp, bp)
        np.testing.assert_array_equal(ws, snp.ws)
        np.testing.assert_array_equal(we, snp.we)
    rng = np.random.default_rng(4)
    chrom = [np.sort(rng.integers(0, 20000, 300)), np.sort(rng.integers(0, 5000, 120)),
             rng.integers(0, 9000, 200)]  # the last one unsorted
    pos = np.concatenate(chrom)
    ends = list(np.cumsum([len(c) for c in chrom]) - 1)
    for bp in (0, 37, 1000):
        ws, we = pb.ld_windows(pos, ends, bp)
        snp = O.SnpLD(["1", "2", "3"], pos.astype(np.int64), ends, [])
        O.divide_pos_by_window(snp, bp)
        np.testing.assert_array_equal(ws, snp.ws)
        np.testing.assert_array_equal(we, snp.we)


def test_header_is_plain_c(tmp_path):
    """include/pcaone_gpu.h is a C header (the boundary a cgo / ctypes / C caller binds): it
    compiles as C99 with -pedantic, and as C++11."""
    import os
    import shutil
    import subprocess

    import pytest

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = tmp_path / "use.c"
    src.write_text('#include <string.h>\n#include "pcaone_gpu.h"\nint main(void) {\n'
                   '  pcaone_rsvd_opts o; pcaone_rsvd_report r;\n'
                   '  memset(&o, 0, sizeof o); memset(&r, 0, sizeof r);\n'
                   '  int (*fn)(pcaone_ctx*, const pcaone_rsvd_opts*, double*, double*, double*,\n'
                   '            pcaone_rsvd_report*) = pcaone_gpu_rsvd;\n'
                   '  (void)fn;\n  return o.k != 0 || r.epochs != 0;\n}\n')
    for cc, std, lang in (("gcc", "-std=c99", "c"), ("g++", "-std=c++11", "c++")):
        if shutil.which(cc) is None:
            pytest.skip(f"{cc} not available")
        r = subprocess.run([cc, std, "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only", "-x", lang,
                            "-I", os.path.join(root, "include"), str(src)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
