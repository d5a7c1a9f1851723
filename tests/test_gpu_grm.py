"""PCAngsd GRM stage (src/Halko.cpp:317-331 with Data::pcangsd_standardize_E,
src/Data.cpp:301-343) through the C ABI: pcaone_gpu_gl_grm against the oracle restatement on
the same inputs, and the whole GPU PCAngsd run against the reference's .cov."""
import os

import numpy as np
import pytest

import pcaone_b200 as pb
from tests.helpers import GOLDEN, ref_out, top_vectors_match
from oracle import pcaone_oracle as O

pytestmark = pytest.mark.gpu

BEAGLE = os.path.join(GOLDEN, "g3.beagle.gz")


def grm_oracle(P, F, U, S, V):
    """C = E E^T / M with diag Dc / M from the oracle's pcangsd_standardize (the device keeps
    the likelihoods in FP64, as the reference does)."""
    Es, Dc = O.pcangsd_standardize(P, F, (U * S) @ V.T)
    C = Es @ Es.T / P.shape[1]
    C[np.diag_indices(len(Dc))] = Dc / P.shape[1]
    return C


def test_gl_grm_matches_oracle_and_repeats(gpu):
    P, N, M = O.parse_beagle(BEAGLE)
    gpu.load_gl(P)
    F, _ = gpu.gl_freq(30, 1e-6)
    rng = np.random.default_rng(7)
    k = 3
    U = np.linalg.qr(rng.standard_normal((N, k)))[0]
    V = np.linalg.qr(rng.standard_normal((M, k)))[0]
    S = np.array([40.0, 25.0, 12.0])
    C, ev, sv = gpu.gl_grm(U, S, V)
    Co = grm_oracle(P, F, U, S, V)
    # FP64 on the same inputs: only the summation order of E E^T differs
    np.testing.assert_allclose(C, Co, rtol=1e-10, atol=1e-13)
    np.testing.assert_array_equal(C, C.T)
    w = np.linalg.eigvalsh(Co)
    np.testing.assert_allclose(sv, np.sort(np.abs(w))[::-1], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(ev.T @ ev, np.eye(N), atol=1e-10)
    top_vectors_match(ev, Co, 5, 1e-8)
    C2, ev2, sv2 = gpu.gl_grm(U, S, V)
    np.testing.assert_array_equal(C, C2)
    np.testing.assert_array_equal(sv, sv2)


def test_gl_grm_multi_tile_and_chunks_match_oracle(gpu, monkeypatch):
    """An odd sample count over several 128 x 128 tiles of the SYRK kernel (zero-filled past
    N) and the sites in chunks with a ragged last chunk (accumulated into the same lower
    triangle): synthetic normalised likelihoods, FP64 against the oracle."""
    rng = np.random.default_rng(11)
    N, M, k = 389, 1000, 4
    g = rng.dirichlet(np.ones(3) * 0.7, size=(M, N))  # per sample-site likelihood triple
    P = np.empty((2 * N, M))
    P[0::2, :] = g[:, :, 0].T
    P[1::2, :] = g[:, :, 1].T
    monkeypatch.setenv("PCAONE_GRM_CHUNK_SITES", "333")
    gpu.load_gl(P)
    F, _ = gpu.gl_freq(30, 1e-6)
    U = np.linalg.qr(rng.standard_normal((N, k)))[0]
    V = np.linalg.qr(rng.standard_normal((M, k)))[0]
    S = np.array([30.0, 20.0, 10.0, 5.0])
    C, _, sv = gpu.gl_grm(U, S, V)
    Co = grm_oracle(P, F, U, S, V)
    np.testing.assert_allclose(C, Co, rtol=1e-10, atol=1e-13)
    np.testing.assert_array_equal(C, C.T)
    np.testing.assert_allclose(sv, np.sort(np.abs(np.linalg.eigvalsh(Co)))[::-1], rtol=1e-9, atol=1e-12)


def test_gl_grm_rejects_missing_factors(gpu):
    P, N, M = O.parse_beagle(BEAGLE)
    gpu.load_gl(P)
    with pytest.raises(pb.PcaoneError):
        gpu.gl_grm(np.zeros((N, 0)), np.zeros(0), np.zeros((M, 0)))


def test_pcangsd_grm_matches_reference_cov(gpu):
    """-G g3.beagle.gz -k 3 -S -w 8 --maxiter 30: the GRM of the final factors against the
    reference's .cov (printed to 6 significant digits), its vectors up to sign."""
    P, N, M = O.parse_beagle(BEAGLE)
    out = pb.run_pcangsd(gpu, P, k=3, bands=8, maxiter=30, shuffle=False, grm=True)
    C, ev, sv = out[6], out[7], out[8]
    Cr = O.read_eigen_matrix(ref_out("g3_pcangsd", ".cov"))
    np.testing.assert_allclose(C, Cr, atol=1e-5)
    top_vectors_match(ev, Cr, 3, 2e-3)
