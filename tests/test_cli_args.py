"""Option parsing of bin/kssd3a needs no GPU: usage errors exit 64 (argp's
EX_USAGE) before any device work, as the reference's do."""
import os
import subprocess

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(ROOT, "kssd3a-public_b200", "bin", "kssd3a")


@pytest.mark.parametrize("argv", [
    ["ani", "-s", "0", "-q", "x"],
    ["ani", "--format", "bogus", "-q", "x"],
    ["ani", "-q", "x"],
    ["ani", "--unique-ctx", "-r", "a", "-q", "b"],
    ["ani", "-n", "95", "-r", "a", "-q", "b"],
])
def test_usage_errors_exit_64(argv):
    r = subprocess.run([OURS, *argv], capture_output=True)
    assert r.returncode == 64
    if oracle.ref_available():
        assert subprocess.run([oracle.REF_BIN, *argv], capture_output=True).returncode == 64
