"""bin/kssd3a (GPU counting + host epilogue) prints the same bytes as the reference
`kssd3a ani` on the same sketch directories: live against oracle/_ref/kssd3a when it
is present, else against the committed golden outputs (tests/golden/cli/*.out.gz)."""
import gzip
import os
import subprocess

import pytest

import oracle
from cli_cases import CASES, materialize, out_files, with_threads

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(ROOT, "kssd3a-public_b200", "bin", "kssd3a")
GOLDEN = os.path.join(ROOT, "tests", "golden", "cli")


def _run(binary, argv, env_extra):
    env = dict(os.environ, OMP_NUM_THREADS="4")
    for k in [k for k in env if k.startswith("KSSD3A_")]:
        env.pop(k, None)
    env.update({k: v for k, v in env_extra.items() if not k.startswith("_")})
    return subprocess.run([binary, *with_threads(argv)], capture_output=True, env=env, timeout=600)


@pytest.fixture(scope="module")
def workdir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("cli"))


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_cli_bytes_match_reference(case, workdir):
    name, argv, env = case
    mine = _run(OURS, materialize(workdir, argv, "ours_" + name), env)
    assert mine.returncode == 0, mine.stderr.decode()[-2000:]
    if oracle.ref_available():
        theirs = _run(oracle.REF_BIN, materialize(workdir, argv, "ref_" + name), env)
        assert theirs.returncode == 0, theirs.stderr.decode()[-2000:]
        want = theirs.stdout
    else:
        path = os.path.join(GOLDEN, name + ".out.gz")
        if not os.path.exists(path):
            pytest.skip("no reference binary and no golden output for this case")
        want = gzip.open(path).read()
    if env.get("_sorted"):
        # header first, rows in any order
        mine_lines, want_lines = mine.stdout.decode().splitlines(), want.decode().splitlines()
        assert mine_lines[:1] == want_lines[:1]
        assert sorted(mine_lines[1:]) == sorted(want_lines[1:])
    elif mine.stdout != want:
        a, b = mine.stdout.decode().splitlines(), want.decode().splitlines()
        for i, (x, y) in enumerate(zip(a, b)):
            if x != y:
                pytest.fail(f"first differing line {i}:\n ours: {x[:300]}\n want: {y[:300]}")
        pytest.fail(f"line counts differ: ours {len(a)} want {len(b)}")
    # extra output files (edge lists, keep/remove lists, kept matrices, id maps, glists)
    if oracle.ref_available():
        for f in out_files(argv):
            po = os.path.join(workdir, "ours_" + name, f)
            pr = os.path.join(workdir, "ref_" + name, f)
            assert os.path.exists(po) == os.path.exists(pr), f
            if os.path.exists(po):
                a, b = open(po, "rb").read(), open(pr, "rb").read()
                if env.get("_sorted_out") == f:
                    a, b = sorted(a.splitlines()), sorted(b.splitlines())
                assert a == b, f
    # automatic index creation leaves identical files behind
    if oracle.ref_available():
        for a in argv:
            if a.startswith("{"):
                d_o = os.path.join(workdir, "ours_" + name, a[1:-1])
                d_r = os.path.join(workdir, "ref_" + name, a[1:-1])
                for f in ("sortedcomb_ctxgid64obj32", "sortedcomb_ctxgid64obj32.unique_bits"):
                    po, pr = os.path.join(d_o, f), os.path.join(d_r, f)
                    assert os.path.exists(po) == os.path.exists(pr), (f, a)
                    if os.path.exists(po):
                        assert open(po, "rb").read() == open(pr, "rb").read(), (f, a)


def test_unique_ctx_report_matches_reference(workdir):
    if not oracle.ref_available():
        pytest.skip("reference binary not present")
    argv = ["ani", "-r", "{refs120i}", "--qraw", "{reads6}", "-n0", "-f0", "-t1"]
    outs = []
    for tag, binary in (("ours_report", OURS), ("ref_report", oracle.REF_BIN)):
        a = materialize(workdir, argv, tag)
        rep = os.path.join(workdir, tag, "report.tsv")
        r = _run(binary, [*a, "--unique-ctx-report", rep], {})
        assert r.returncode == 0, r.stderr.decode()[-1000:]
        outs.append((r.stdout, open(rep, "rb").read()))
    assert outs[0] == outs[1]
