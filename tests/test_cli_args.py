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


def _msg(stderr: bytes) -> str:
    """argp's first line without the program-name prefix."""
    line = stderr.decode(errors="replace").splitlines()[0] if stderr else ""
    return line.split(": ", 1)[-1]


@pytest.mark.parametrize("argv", [
    ["matrix", "--format", "edges", "x"],
    ["matrix", "--format", "bogus", "x"],
    ["matrix", "--format", "clusters", "--cut", "0.1", "-r", "a", "-q", "b"],
    ["matrix", "--keep-out", "k", "--format", "edges", "--cut", "0.1", "x"],
    ["matrix", "--dedup-strategy", "greedy", "--format", "clusters", "--cut", "0.1", "x"],
    ["matrix", "--dedup-strategy", "bogus", "x"],
    ["matrix", "--format", "dedup-plan", "--cut", "0.1", "--keep-matrix-format", "phylip", "x"],
    ["matrix", "--format", "dedup-plan", "--cut", "0.1", "--keep-matrix-out", "m", "--keep-matrix-idmap", "i", "x"],
    ["matrix", "--format", "dedup-plan", "--cut", "0.1", "--keep-out", "a", "--remove-out", "a", "x"],
    ["matrix", "--format", "dedup-plan", "--cut", "0.1", "--edge-out", "o", "-o", "o", "x"],
    ["matrix", "--format", "dedup-plan", "--cut", "0.1", "--keep-matrix-out", "m", "--keep-matrix-format", "phy",
     "--keep-matrix-idmap", "m", "x"],
    ["matrix", "--matrix-format", "fillip", "--format", "triangle", "x"],
    ["matrix", "--keep-matrix-format", "csv", "x"],
    ["matrix", "--progress", "maybe", "x"],
    ["matrix", "-m", "ctx-naive&aaf", "x"],
    ["matrix", "-m", "naive&|aaf", "--format", "edges", "--cut", "1", "x"],
    ["matrix", "--max-afcut", "1.5", "x"],
    ["matrix", "--index-min-votes", "0", "x"],
])
def test_matrix_usage_messages(argv):
    r = subprocess.run([OURS, *argv], capture_output=True)
    assert r.returncode == 64, r.stderr
    if oracle.ref_available():
        want = subprocess.run([oracle.REF_BIN, *argv], capture_output=True)
        assert want.returncode == 64
        assert _msg(r.stderr) == _msg(want.stderr)
