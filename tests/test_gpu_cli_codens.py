"""The 9- and 10-coden builds (kssd3a-public_b200/build/codens{9,10}/bin/kssd3a, from
`make -C kssd3a-public_b200 codens`) print the same bytes as the reference CLI
compiled with -DNUM_CODENS=9 / 10 (oracle/_ref/kssd3a_c9, kssd3a_c10) when those are
present, else as the committed golden outputs (tests/golden/cli_codens/)."""
import gzip
import os
import subprocess

import pytest

import oracle
from cli_cases import CODENS_BUILD_CASES, materialize, with_threads

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "cli_codens")


def _ours(codens):
    path = os.path.join(ROOT, "kssd3a-public_b200", "build", f"codens{codens}", "bin", "kssd3a")
    assert os.path.exists(path), f"{path} missing: run `make -C kssd3a-public_b200 codens`"
    return path


def _run(binary, argv):
    env = dict(os.environ, OMP_NUM_THREADS="4")
    for k in [k for k in env if k.startswith("KSSD3A_")]:
        env.pop(k, None)
    return subprocess.run([binary, *with_threads(argv)], capture_output=True, env=env, timeout=600)


@pytest.fixture(scope="module")
def workdir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("cli_codens"))


@pytest.mark.parametrize("codens", [9, 10])
@pytest.mark.parametrize("case", CODENS_BUILD_CASES, ids=[c[0] for c in CODENS_BUILD_CASES])
def test_codens_build_bytes_match_reference(codens, case, workdir):
    name, argv = case
    mine = _run(_ours(codens), materialize(workdir, argv, f"ours_c{codens}_" + name))
    assert mine.returncode == 0, mine.stderr.decode()[-2000:]
    ref_bin = f"{oracle.REF_BIN}_c{codens}"
    if os.path.exists(ref_bin):
        theirs = _run(ref_bin, materialize(workdir, argv, f"ref_c{codens}_" + name))
        assert theirs.returncode == 0, theirs.stderr.decode()[-2000:]
        want = theirs.stdout
    else:
        want = gzip.open(os.path.join(GOLDEN, f"c{codens}_{name}.out.gz")).read()
    if mine.stdout != want:
        a, b = mine.stdout.decode().splitlines(), want.decode().splitlines()
        for i, (x, y) in enumerate(zip(a, b)):
            if x != y:
                pytest.fail(f"first differing line {i}:\n ours: {x[:300]}\n want: {y[:300]}")
        pytest.fail(f"line counts differ: ours {len(a)} want {len(b)}")


def test_codens_builds_differ_from_default_models(workdir):
    """The 9/10-coden model coefficients are in effect: the default build's BestDist
    column differs from the 9-coden build's on the same inputs."""
    argv = ["ani", "-r", "{refs40c9i}", "-q", "{qry50c9}", "-n", "0.5"]
    default = _run(os.path.join(ROOT, "kssd3a-public_b200", "bin", "kssd3a"), materialize(workdir, argv, "d11"))
    c9 = _run(_ours(9), materialize(workdir, argv, "d9"))
    assert default.returncode == 0 and c9.returncode == 0
    assert default.stdout != c9.stdout
