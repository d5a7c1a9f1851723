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
