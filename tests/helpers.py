"""Shared comparison helpers for the parity tests."""
import json
import os

import numpy as np

from oracle import pcaone_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def case(name):
    with open(os.path.join(GOLDEN, "cases.json")) as f:
        rec = json.load(f)
    for c in rec["cases"]:
        if c["name"] == name:
            return c
    raise KeyError(name)


def ref_out(name, suffix):
    return os.path.join(GOLDEN, "ref", name + suffix)


def ref_table(name, suffix):
    return O.read_table(ref_out(name, suffix))


def ref_eigvals(name):
    return ref_table(name, ".eigvals")[:, 0]


def assert_eig_close(got, ref, rtol):
    got, ref = np.asarray(got), np.asarray(ref)
    rel = np.abs(got / ref - 1)
    assert rel.max() <= rtol, f"eigval rel err {rel.max():.3e} > {rtol:.1e}\n{got}\n{ref}"


def assert_cols_close(got, ref, atol):
    err = O.max_col_err_up_to_sign(got, ref)
    assert err <= atol, f"max column error up to sign {err:.3e} > {atol:.1e}"


def max_angle(A, B):
    return float(O.principal_angles(A, B).max())


def eigen_aligned(A) -> str:
    """Eigen's default `stream << matrix` text of A (stream precision 6): every coefficient
    printed as "%.6g", right-aligned to the widest one, " " between coefficients, "\\n" between
    rows, nothing after the last row."""
    A = np.atleast_2d(np.asarray(A, dtype=np.float64))
    cells = [["%.6g" % v for v in row] for row in A]
    w = max(len(c) for row in cells for c in row)
    return "\n".join(" ".join(c.rjust(w) for c in row) for row in cells)


def top_vectors_match(got, C, ncols, atol):
    """The first ncols columns of got against the eigenvectors of the symmetric C ordered by
    decreasing |eigenvalue|, up to sign; columns whose eigenvalue is not separated from its
    neighbours by 1e-6 relative are skipped."""
    w, Q = np.linalg.eigh(C)
    order = np.argsort(-np.abs(w), kind="stable")
    a = np.abs(w[order])
    checked = 0
    for c in range(ncols):
        gap = min(abs(a[c] - a[c - 1]) if c else np.inf, abs(a[c] - a[c + 1]) if c + 1 < len(a) else np.inf)
        if gap <= 1e-6 * a[0]:
            continue
        q = Q[:, order[c]]
        err = min(np.abs(got[:, c] - q).max(), np.abs(got[:, c] + q).max())
        assert err <= atol, f"vector {c}: error up to sign {err:.3e} > {atol:.1e}"
        checked += 1
    assert checked > 0
