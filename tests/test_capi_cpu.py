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


def test_create_without_device_fails_cleanly():
    import subprocess
    import sys
    code = ("import pcaone_b200 as pb\n"
            "try:\n    pb.GpuContext(999)\nexcept pb.PcaoneError as e:\n    print('ERR', e.status)\n")
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT)
    assert "ERR 7" in out.stdout, out.stdout + out.stderr
