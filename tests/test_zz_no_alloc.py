"""The allocation-free product entry point (pcaone_gpu_product_t_noalloc).

Callers that cannot let a library call cudaMalloc (code inside another framework's device
memory pool, or a solver loop that must not allocate per call) pass their own device
buffers; the entry point keeps its scratch in one fixed device array inside the library.
Here torch plays the caller's allocator. On two calls in a row the result must match the
allocating pcaone_gpu_product (FP32, Z^T B) and the oracle's standardised Z^T B, free
device memory must not change across a call, and oversize problems must be rejected with a
clear error. The test uses its own context and data, so it passes alone in a fresh process
and after the other tests.
"""
import numpy as np
import pytest

import pcaone_b200 as pb
from oracle import pcaone_oracle as O

pytestmark = pytest.mark.gpu

TOL = 2e-6  # the FP32 product tolerance used by tests/test_gpu_product.py


def _random_bed(N, M, seed, miss):
    rng = np.random.default_rng(seed)
    p = rng.uniform(0.05, 0.5, M)
    d = (rng.random((M, N)) < p[:, None]).astype(np.uint8) + (rng.random((M, N)) < p[:, None])
    codes = np.where(d == 2, 0, np.where(d == 1, 2, 3)).astype(np.uint8)
    codes[rng.random((M, N)) < miss] = 1
    bpr = (N + 3) // 4
    pad = np.full((M, bpr * 4), 3, dtype=np.uint8)
    pad[:, :N] = codes
    pad = pad.reshape(M, bpr, 4)
    packed = (pad[:, :, 0] | (pad[:, :, 1] << 2) | (pad[:, :, 2] << 4) | (pad[:, :, 3] << 6))
    return O.Bed(N, M, packed.astype(np.uint8))


def _rel(got, ref):
    return float((np.abs(got - ref).max(axis=0) / np.abs(ref).max(axis=0)).max())


def test_product_noalloc_matches_allocating_product_and_oracle():
    torch = pytest.importorskip("torch")
    bed = _random_bed(1003, 2500, seed=42, miss=0.02)
    Z, _ = O.standardized_from_bed(bed)
    l = 40
    rng = np.random.default_rng(7)
    with pb.GpuContext(0) as ctx:
        ctx.load_bed(bed.packed, bed.N)
        for call in range(2):  # two calls in a row share (and overwrite) the scratch array
            B = rng.standard_normal((bed.N, l))
            ref = ctx.product_t(B, precision="fp32")  # existing entry point
            d_B = torch.tensor(B.T.copy(), dtype=torch.float64, device="cuda")  # column-major N x l
            d_out = torch.full((l, bed.M), float("nan"), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()  # d_B is written on torch's stream: complete it first
            free0 = torch.cuda.mem_get_info()[0]
            ctx.product_t_noalloc(d_B.data_ptr(), l, d_out.data_ptr())
            free1 = torch.cuda.mem_get_info()[0]
            got = d_out.cpu().numpy().T
            assert _rel(got, ref) <= TOL
            assert _rel(got, Z.T @ B) <= TOL
            if call == 1:  # after the first call has resolved the array's address
                assert free1 == free0, (free0, free1)


def test_product_noalloc_rejects_oversize_and_unprepared():
    torch = pytest.importorskip("torch")
    bed = _random_bed(8, 300000, seed=3, miss=0.0)
    l = 64  # 300000 SNPs x 64 columns x 4 bytes of partial sums exceeds the 64 MiB array
    with pb.GpuContext(0) as ctx:
        ctx.load_bed(bed.packed, bed.N)
        d_B = torch.zeros((l, bed.N), dtype=torch.float64, device="cuda")
        d_out = torch.zeros((l, bed.M), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        with pytest.raises(pb.PcaoneError) as e:  # missing-entry list not built yet
            ctx.product_t_noalloc(d_B.data_ptr(), l, d_out.data_ptr())
        assert e.value.status == 6
        ctx.product_t(np.zeros((bed.N, l)), precision="fp32")
        with pytest.raises(pb.PcaoneError) as e:
            ctx.product_t_noalloc(d_B.data_ptr(), l, d_out.data_ptr())
        assert e.value.status == 1 and "maximum" in str(e.value)
