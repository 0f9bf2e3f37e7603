"""bin/kssd3a against the reference CLI (oracle/_ref/kssd3a) on the benchmark
configurations' own shapes, byte for byte:

  - 64 genomes of 1 Mbp written as FASTA by a seeded sequence generator and sketched
    by the reference's own sketcher (`kssd3a sketch`, default -T -f8; `sketch -i` for
    the index): detail without an index (hash path), detail with the index (mem_eff),
    the direct self matrix, the ANI matrix and `kssd3a matrix`;
  - the 2,000-genome self ANI matrix of the headline configuration (indexed self
    full path, 36 MB of TSV) and its detail run.

Skipped where the reference build is absent (it is built from the reference sources
by oracle/Makefile)."""
import os
import subprocess

import numpy as np
import pytest

import kssdgpu
import oracle

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
OURS = os.path.join(ROOT, "kssd3a-public_b200", "bin", "kssd3a")
THREADS = str(min(16, os.cpu_count() or 4))


def _run(binary, argv):
    env = {k: v for k, v in os.environ.items() if not k.startswith("KSSD3A_")}
    env["OMP_NUM_THREADS"] = THREADS
    r = subprocess.run([binary, *argv], capture_output=True, env=env, timeout=900)
    assert r.returncode == 0, (binary, argv, r.stderr.decode()[-2000:])
    return r.stdout


def _same(argv):
    mine = _run(OURS, argv)
    want = _run(oracle.REF_BIN, argv)
    if mine != want:
        a, b = mine.decode().splitlines(), want.decode().splitlines()
        for i, (x, y) in enumerate(zip(a, b)):
            if x != y:
                pytest.fail(f"{argv}: first differing line {i}:\n ours: {x[:300]}\n want: {y[:300]}")
        pytest.fail(f"{argv}: line counts differ: ours {len(a)} want {len(b)}")
    return mine


@pytest.fixture(scope="module")
def config1(tmp_path_factory):
    if not oracle.ref_available():
        pytest.skip("reference build not present")
    import fasta_synth
    root = str(tmp_path_factory.mktemp("config1"))
    paths = fasta_synth.write_genomes(os.path.join(root, "fa"))
    plain = os.path.join(root, "refs")
    r = subprocess.run([oracle.REF_BIN, "sketch", "-p", THREADS, "-o", plain, *paths], capture_output=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr.decode()[-2000:]
    indexed = os.path.join(root, "refsi")
    r = subprocess.run([oracle.REF_BIN, "sketch", "-p", THREADS, "-o", indexed, *paths], capture_output=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr.decode()[-2000:]
    r = subprocess.run([oracle.REF_BIN, "sketch", "-i", indexed], capture_output=True, timeout=600)
    assert r.returncode == 0, r.stderr.decode()[-2000:]
    return plain, indexed


def test_config1_sketch_is_reference_made(config1):
    plain, _ = config1
    sk = kssdgpu.read_sketch_dir(plain)
    assert sk.n == 64
    per = np.diff(sk.offs.astype(np.int64))
    assert 3000 < per.mean() < 5000  # ~1 key per 256 bp of a 1 Mbp genome
    # clusters share contexts: well above one posting per context
    _, k = np.unique(sk.keys >> np.uint64(20), return_counts=True)
    assert len(sk.keys) / len(k) > 1.3


@pytest.mark.parametrize("argv", [
    ["ani", "-p", THREADS, "-r", "{plain}", "-q", "{plain}"],
    ["ani", "-p", THREADS, "-r", "{indexed}", "-q", "{indexed}"],
    ["ani", "-p", THREADS, "-r", "{indexed}", "-q", "{indexed}", "--anicut", "0.9", "-N", "5"],
    ["ani", "-p", THREADS, "-r", "{plain}", "-q", "{plain}", "--format", "matrix"],
    ["ani", "-p", THREADS, "-q", "{indexed}", "--format", "matrix", "--values", "ani"],
    ["matrix", "-p", THREADS, "-q", "{plain}"],
], ids=["detail_hash", "detail_mem_eff", "detail_top5", "matrix_direct", "self_ani_matrix", "matrix_cmd"])
def test_config1_cli_bytes(config1, argv):
    plain, indexed = config1
    argv = [plain if a == "{plain}" else indexed if a == "{indexed}" else a for a in argv]
    out = _same(argv)
    assert len(out.splitlines()) > 1


@pytest.fixture(scope="module")
def genomes2k(tmp_path_factory):
    if not oracle.ref_available():
        pytest.skip("reference build not present")
    sk = kssdgpu.synth(n_samples=2000, n_clusters=200, size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e6,
                       len_sigma=0.37, len_min=1e6, len_max=12e6, sub_lo=0.001, sub_hi=0.2, seed=20261203 + 2,
                       sample_seed=20261203 + 2, threads=os.cpu_count() or 8)
    d = str(tmp_path_factory.mktemp("g2k"))
    kssdgpu.write_sketch_dir(d, sk)
    rec = oracle.build_index(sk.keys, sk.offs)
    rec.tofile(os.path.join(d, "sortedcomb_ctxgid64obj32"))
    oracle.unique_bits(rec).tofile(os.path.join(d, "sortedcomb_ctxgid64obj32.unique_bits"))
    return d


def test_headline_2000_genome_ani_matrix_bytes(genomes2k):
    out = _same(["ani", "-p", THREADS, "-q", genomes2k, "--format", "matrix", "--values", "ani"])
    assert len(out.splitlines()) == 2001


@pytest.mark.parametrize("fmt", ["matrix", "triangle"])
def test_headline_2000_genome_matrix_to_file(genomes2k, tmp_path, fmt):
    """-o FILE (a regular file: rows go out as positioned writes from all host threads)
    gives the bytes the reference writes, also when the file already holds longer content."""
    want = _run(oracle.REF_BIN, ["ani", "-p", THREADS, "-q", genomes2k, "--format", fmt, "--values", "ani"])
    dst = tmp_path / "m.tsv"
    dst.write_bytes(b"x" * (len(want) + 12345))
    _run(OURS, ["ani", "-p", THREADS, "-q", genomes2k, "--format", fmt, "--values", "ani", "-o", str(dst)])
    assert dst.read_bytes() == want


def test_headline_2000_genome_detail_bytes(genomes2k):
    out = _same(["ani", "-p", THREADS, "-r", genomes2k, "-q", genomes2k])
    assert len(out.splitlines()) > 2000
