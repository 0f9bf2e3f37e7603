"""Device sketching (kssdgpu_sketch) against the reference sketcher's own output on the
golden FASTA/FASTQ inputs, and against the oracle's restatement on seeded sequence with
many layouts (coden pattern, manual context/object lengths, drfold, conflict mode,
short and empty records, empty samples, IUPAC noise, read sets)."""
import os

import numpy as np
import pytest

import kssdgpu
import oracle
from fixtures import read_fastx_records

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "sketch")
INPUTS = ["g0.fa", "g1.fasta", "g2.fna", "g3.fa.gz", "r0.fq"]


@pytest.mark.parametrize("mode", ["default", "conflict", "asone"])
def test_sketch_matches_reference_sketcher(mode):
    d = os.path.join(GOLDEN, mode)
    want_keys = np.fromfile(os.path.join(d, "comblco"), dtype=np.uint64)
    want_offs = np.fromfile(os.path.join(d, "comblco.index"), dtype=np.uint64)
    recs = [read_fastx_records(os.path.join(GOLDEN, "inputs", x)) for x in INPUTS]
    samples = [sum(recs, [])] if mode == "asone" else recs
    keys, offs = kssdgpu.sketch(samples, conflict=(mode == "conflict"))
    np.testing.assert_array_equal(offs, want_offs)
    np.testing.assert_array_equal(keys, want_keys)
    stat = np.fromfile(os.path.join(d, "lcofiles.stat"), dtype=np.uint32, count=1)
    assert kssdgpu.sketch_hash_id() == int(stat[0])


def _noisy(rng, n):
    s = np.frombuffer(b"ACGT", dtype=np.uint8)[rng.integers(0, 4, size=n)].copy()
    low = rng.random(n) < 0.1
    s[low] += 32  # lower case
    for p in rng.integers(0, n, size=max(1, n // 3000)):
        s[p] = ord("N")
    return s.tobytes()


def _samples(rng, kind):
    if kind == "genomes":
        anc = _noisy(rng, 50000)
        out = []
        for _ in range(5):
            b = bytearray(anc)
            for p in rng.integers(0, len(b), size=1500):
                b[p] = ord("ACGT"[rng.integers(0, 4)])
            cut = sorted(rng.integers(0, len(b), size=3).tolist())
            out.append([bytes(b[:cut[0]]), bytes(b[cut[0]:cut[1]]), b"", bytes(b[cut[1]:])])
        out.insert(2, [])                       # a sample without records
        out.append([b"ACGT" * 7, b"A" * 31])    # records shorter than k only
        return out
    if kind == "reads":
        g = _noisy(rng, 30000)
        reads = []
        for _ in range(3000):
            p = int(rng.integers(0, len(g) - 150))
            reads.append(g[p:p + 150])
        return [reads[:1000], reads[1000:], [g]]
    raise ValueError(kind)


LAYOUTS = [dict(klen=32, coden_len=11, drfold=8), dict(klen=32, coden_len=11, drfold=0),
           dict(klen=32, coden_len=11, drfold=4), dict(klen=20, coden_len=0, hclen=6, holen=1, drfold=2),
           dict(klen=31, coden_len=0, hclen=8, holen=0, drfold=3), dict(klen=16, coden_len=0, hclen=4, holen=2,
                                                                         drfold=1)]


@pytest.mark.parametrize("kind", ["genomes", "reads"])
@pytest.mark.parametrize("layout", range(len(LAYOUTS)))
@pytest.mark.parametrize("conflict", [False, True])
def test_sketch_matches_oracle(kind, layout, conflict):
    rng = np.random.default_rng(layout * 7 + (kind == "reads") * 3 + conflict)
    samples = _samples(rng, kind)
    lay = LAYOUTS[layout]
    keys, offs = kssdgpu.sketch(samples, conflict=conflict, **lay)
    assert len(offs) == len(samples) + 1
    for i, smp in enumerate(samples):
        want = oracle.sketch_records(smp, conflict=conflict, **lay)
        np.testing.assert_array_equal(keys[offs[i]:offs[i + 1]], want, err_msg=f"sample {i}")
    assert offs[-1] > 0


def test_sketch_edge_cases():
    # nothing to sketch
    keys, offs = kssdgpu.sketch([])
    assert len(keys) == 0 and list(offs) == [0]
    keys, offs = kssdgpu.sketch([[], [b""], [b"N" * 100]])
    assert len(keys) == 0 and list(offs) == [0, 0, 0, 0]
    # a sample spanning many thread tiles and records ending on tile edges
    rng = np.random.default_rng(5)
    g = _noisy(rng, 3 * 16384 + 77)
    recs = [g[:16384], g[16384:16384 + 64], g[16384 + 64:2 * 16384 - 1], g[2 * 16384 - 1:]]
    for lay in LAYOUTS[:2]:
        keys, offs = kssdgpu.sketch([recs, [g]], **lay)
        np.testing.assert_array_equal(keys[offs[0]:offs[1]], oracle.sketch_records(recs, **lay))
        np.testing.assert_array_equal(keys[offs[1]:offs[2]], oracle.sketch_records([g], **lay))
    # invalid arguments are refused, not run
    with pytest.raises(kssdgpu.KssdGpuError):
        kssdgpu.sketch([[b"ACGT" * 20]], klen=33, coden_len=0, hclen=4)
    with pytest.raises(kssdgpu.KssdGpuError):
        kssdgpu.sketch([[b"ACGT" * 20]], klen=20, coden_len=0, hclen=8, holen=3)
