"""The CLI's argument checks, which run before any device is opened: the same refusals (exit
code 1, the same message) as the reference's Param checks (src/Cmd.cpp:125-128, 195-212), and
clean refusals where the reference aborts. The reference binary built by oracle/ref.mk is
run beside it when it is present."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(ROOT, "pcaone_b200", "bin", "PCAone")
REF = os.path.join(ROOT, "oracle", "_ref", "PCAone")
G1 = os.path.join(ROOT, "tests", "golden", "g1")


def run(binary, args, tmp_path):
    r = subprocess.run([binary] + args + ["-o", str(tmp_path / "out")], capture_output=True, text=True,
                       timeout=60, cwd=tmp_path)
    return r.returncode, r.stdout + r.stderr


SAME = [
    (["--bogus"], "unknown option: --bogus"),
    (["-b", G1, "-k", "3", "-w", "3"], "the -w/--batches must be a power of 2 and the minimun is 4."),
    (["-b", G1, "-k", "3", "-m", "2", "--maf", "0.1"], "does not support --maf filters for out-of-core mode yet!"),
]


@pytest.mark.parametrize("args,msg", SAME)
def test_cli_refuses_like_the_reference(tmp_path, args, msg):
    if not os.path.exists(OURS):
        pytest.skip("CLI not built")
    rc, out = run(OURS, args, tmp_path)
    assert rc == 1 and msg in out, out
    if os.path.exists(REF):
        rc_r, out_r = run(REF, args, tmp_path)
        assert rc_r == 1 and msg in out_r, out_r


@pytest.mark.parametrize("args,msg", [
    (["-k", "3"], "no input"),                                    # the reference aborts (std::runtime_error)
    (["-b", G1, "-k", "3", "--emu", "--pcangsd"], "exclusive"),  # the reference aborts (std::bad_alloc)
    (["-b", G1, "-k", "3", "--precision", "int4"], "--precision must be"),
])
def test_cli_refuses_cleanly(tmp_path, args, msg):
    if not os.path.exists(OURS):
        pytest.skip("CLI not built")
    rc, out = run(OURS, args, tmp_path)
    assert rc == 1 and msg in out, out
