"""bench.py helpers that need no GPU: the decode-GEMM's DRAM traffic scaled from the committed
ncu summary (its two byte counts must stay readable), and the roofline arithmetic."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_capture_traffic_reads_the_committed_summary():
    traffic, source = bench.capture_traffic("k_decode_gemm_i8_c2s.md", 250e6)
    assert traffic is not None and source.startswith("profiles/k_decode_gemm_i8_c2s.md")
    # the capture streams 250 MB of packed codes; DRAM bytes are those plus the partial sums
    assert 1.0 <= traffic / 250e6 <= 1.2


def test_capture_traffic_missing_profile_gives_none():
    assert bench.capture_traffic("no_such_profile.md", 1e6) == (None, None)


def test_tensor_roofline_ceiling_of_the_int8_pieces():
    class Prof:
        gemm_ms, gpu_ms, gemm_launches = 50.0, 180.0, 322
        epilogue_ms = update_ms = tail_ms = host_ms = 0.0

    r = bench.tensor_roofline("mixed", 40, 4.0 * 500000 * 20000 * 40 * 21, Prof)
    assert r["issued_ops_factor"] == 3.2 and r["ceiling_frac_of_bf16_peak"] == 0.625
    assert abs(r["achieved"] - 4.0 * 500000 * 20000 * 40 * 21 / 0.05 / 1e12) < 0.01
