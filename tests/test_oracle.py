"""The oracle (C restatement) pinned against the reference: its own counting
functions compiled from its sources (oracle/_ref/refharness.so), its CLI
(oracle/_ref/kssd3a), and committed golden vectors from that CLI (tests/golden)."""
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
from fixtures import mutate_from, random_samples, samples_to_sketch

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
needs_ref = pytest.mark.skipif(not oracle.ref_available(), reason="reference build (oracle/_ref) not present")


def _cases():
    # (seed, refs, queries, ctx_space, obj_space, conflict) — the shapes of the reference's
    # randomized oracle test (tests/test_unique_context.py:268-278) plus larger ones
    out = []
    for seed in range(20):
        out.append((seed, 4, 2, 35, 256, True))
    for seed in range(20, 26):
        out.append((seed, 40, 12, 300, 1 << 20, True))
    for seed in range(26, 30):
        out.append((seed, 64, 16, 2000, 1 << 20, False))
    return out


def _fixture(seed, nref, nq, ctx_space, obj_space, conflict):
    rng = np.random.default_rng(seed)
    refs = random_samples(rng, nref, 40, ctx_space, obj_space, conflict)
    qrys = random_samples(rng, nq, 40, ctx_space, obj_space, conflict)
    # queries derived from references so that objects also match or differ by few bases
    for i in range(min(nq, nref)):
        if rng.random() < 0.5 and refs[i]:
            qrys[i] = mutate_from(rng, refs[i], 0.05)
    rk, ro = samples_to_sketch(refs)
    qk, qo = samples_to_sketch(qrys)
    rec = oracle.build_index(rk, ro)
    return rk, ro, qk, qo, rec


@needs_ref
@pytest.mark.parametrize("case", _cases())
@pytest.mark.parametrize("ignoreconflict", [False, True])
def test_count_block_matches_reference(case, ignoreconflict):
    rk, ro, qk, qo, rec = _fixture(*case)
    nref = len(ro) - 1
    mine = oracle.count_block(rec, nref, qk, qo, ignoreconflict=ignoreconflict, unique=True)
    theirs = oracle.count_block(rec, nref, qk, qo, ignoreconflict=ignoreconflict, unique=True, ref=True)
    for a, b in zip(mine, theirs):
        np.testing.assert_array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("case", _cases()[::3])
@pytest.mark.parametrize("ignoreconflict", [False, True])
def test_count_lower_matches_reference(case, ignoreconflict):
    rk, ro, _, _, rec = _fixture(*case)
    nref = len(ro) - 1
    for off in range(0, nref, 7):
        nb = min(7, nref - off)
        qo = ro[off: off + nb + 1]
        qk = rk[int(qo[0]): int(qo[-1])]
        mine = oracle.count_lower(rec, nref, off, qk, qo, ignoreconflict=ignoreconflict)
        theirs = oracle.count_lower(rec, nref, off, qk, qo, ignoreconflict=ignoreconflict, ref=True)
        for a, b in zip(mine, theirs):
            np.testing.assert_array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("seed", range(10))
def test_pair_features_match_reference(seed):
    rng = np.random.default_rng(100 + seed)
    samples = random_samples(rng, 2, 60, 50, 1 << 20, True, empty_prob=0.05)
    k, o = samples_to_sketch(samples)
    a, b = k[o[0]:o[1]], k[o[1]:o[2]]
    for ign in (False, True):
        np.testing.assert_array_equal(oracle.pair_features(a, b, ignore_b_conflict=ign),
                                      oracle.pair_features(a, b, ignore_b_conflict=ign, ref=True))


@pytest.mark.parametrize("seed", range(5))
def test_self_lower_equals_pairwise_merge(seed):
    """count_lower over all blocks equals the per-pair merge (a10) for every lower pair."""
    rng = np.random.default_rng(200 + seed)
    samples = random_samples(rng, 12, 50, 80, 1 << 20, True)
    k, o = samples_to_sketch(samples)
    rec = oracle.build_index(k, o)
    for ign in (False, True):
        ctx, obj = oracle.self_lower_all(rec, k, o, ignoreconflict=ign)
        cell = 0
        for q in range(1, len(o) - 1):
            for r in range(q):
                f = oracle.pair_features(k[o[q]:o[q + 1]], k[o[r]:o[r + 1]], ignore_b_conflict=ign)
                assert (ctx[cell, 0], obj[cell, 0], obj[cell, 1], ctx[cell, 1]) == tuple(f)
                cell += 1


def test_dna_popcount():
    lib = oracle.oracle_lib()
    for x, want in [(0, 0), (1, 1), (2, 1), (3, 1), (4, 1), (0xF, 2), (0xFFFFF, 10), (0x55555555, 16)]:
        assert lib.orc_dna_popcount(x) == want


def test_index_build_matches_numpy_and_unique_bits():
    import kssdgpu
    rng = np.random.default_rng(7)
    samples = random_samples(rng, 30, 60, 500, 1 << 20, True)
    k, o = samples_to_sketch(samples)
    rec = oracle.build_index(k, o)
    sk = kssdgpu.Sketch(keys=k, offs=o, names=[f"s{i}" for i in range(len(o) - 1)], conflict=True)
    np.testing.assert_array_equal(rec.tobytes(), kssdgpu.build_records_np(sk).tobytes())
    np.testing.assert_array_equal(oracle.unique_bits(rec), kssdgpu.unique_bits_np(rec))


def _load_golden(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def _golden_cases():
    if not os.path.isdir(GOLDEN):
        return []
    return sorted(f for f in os.listdir(GOLDEN) if f.startswith("counts_") and f.endswith(".json"))


@pytest.mark.parametrize("name", _golden_cases())
def test_oracle_against_golden_cli_vectors(name):
    """Counts printed by the reference CLI (--unique-ctx-report) on committed fixtures."""
    g = _load_golden(name)
    refs = [[tuple(p) for p in s] for s in g["refs"]]
    qrys = [[tuple(p) for p in s] for s in g["queries"]]
    rk, ro = samples_to_sketch(refs)
    qk, qo = samples_to_sketch(qrys)
    rec = oracle.build_index(rk, ro)
    nref = len(ro) - 1
    ign = g["ignoreconflict"]
    ctx, obj, uctx, uobj = oracle.count_block(rec, nref, qk, qo, ignoreconflict=ign, unique=True)
    qcnt = oracle.sample_ctx_counts(qk, qo, 20, True, False)
    rcnt = oracle.ref_ctx_counts(rec, nref, ro, True, ign)
    utot = oracle.unique_ref_totals(rec, nref, ign)
    seen = set()
    for row in g["rows"]:
        q, r = row["q"], row["r"]
        seen.add((q, r))
        assert qcnt[q] == row["Qry_ctx"] and rcnt[r] == row["Ref_ctx"] and utot[r] == row["Unique_Ref_ctx"]
        assert (ctx[q, r, 0], obj[q, r, 0], obj[q, r, 1], ctx[q, r, 1]) == (
            row["XnY_ctx"], row["N_diff_obj"], row["N_diff_obj_section"], row["N_mut2_ctx"])
        assert (uctx[q, r, 0], uobj[q, r, 0], uobj[q, r, 1], uctx[q, r, 1]) == (
            row["Unique_XnY_ctx"], row["Unique_N_diff_obj"], row["Unique_N_diff_obj_section"],
            row["Unique_N_mut2_ctx"])
    # every cell with a shared context is in the report, and no other
    nz = {(int(q), int(r)) for q, r in zip(*np.nonzero(ctx[:, :, 0]))}
    assert nz == seen


@needs_ref
def test_reference_index_build_matches_oracle(tmp_path):
    """`kssd3a sketch -i` (the reference's index build) equals orc_build_index + unique bits."""
    import kssdgpu
    rng = np.random.default_rng(11)
    samples = random_samples(rng, 25, 80, 400, 1 << 20, True)
    k, o = samples_to_sketch(samples)
    sk = kssdgpu.Sketch(keys=k, offs=o, names=[f"s{i}" for i in range(len(o) - 1)], conflict=True)
    d = str(tmp_path / "sk")
    kssdgpu.write_sketch_dir(d, sk)
    subprocess.run([oracle.REF_BIN, "sketch", "-i", d], check=True, capture_output=True)
    ref_rec = kssdgpu.read_index_records(d)
    rec = oracle.build_index(k, o)
    assert ref_rec.tobytes() == rec.tobytes()
    ref_bits = np.fromfile(os.path.join(d, "sortedcomb_ctxgid64obj32.unique_bits"), dtype=np.uint8)
    np.testing.assert_array_equal(ref_bits, oracle.unique_bits(rec))


def test_workload_generator_builds_agree():
    """The generator built into oracle/libworkload.so (used by the timed reference arm)
    yields the same sketches as the product's host library."""
    import kssdgpu
    kw = dict(n_samples=60, n_clusters=6, size_dist=kssdgpu.SIZE_LOGNORMAL, len_median=4e5, len_min=1e5,
              len_max=1.2e6, sub_lo=0.001, sub_hi=0.2, seed=77, sample_seed=78)
    a = kssdgpu.synth(**kw)
    b = kssdgpu.synth(lib=kssdgpu.bind_synth(oracle.workload_lib()), **kw)
    np.testing.assert_array_equal(a.offs, b.offs)
    np.testing.assert_array_equal(a.keys, b.keys)


SKETCH_GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "sketch")
SKETCH_INPUTS = ["g0.fa", "g1.fasta", "g2.fna", "g3.fa.gz", "r0.fq"]


@pytest.mark.parametrize("mode", ["default", "conflict", "asone"])
def test_sketch_oracle_matches_reference_sketcher(mode):
    """The oracle's restatement of the reference's sketcher (canonical contexts, the
    splitmix64 hash filter at -f 8, the coden pattern, sort, dedup, conflict removal)
    gives the reference `kssd3a sketch` output byte for byte on the golden inputs:
    several records per file, lower case, N runs and IUPAC codes, CRLF line ends,
    records shorter than k, an empty record, gzip, FASTQ."""
    from fixtures import read_fastx_records
    d = os.path.join(SKETCH_GOLDEN, mode)
    keys = np.fromfile(os.path.join(d, "comblco"), dtype=np.uint64)
    offs = np.fromfile(os.path.join(d, "comblco.index"), dtype=np.uint64)
    recs = [read_fastx_records(os.path.join(SKETCH_GOLDEN, "inputs", x)) for x in SKETCH_INPUTS]
    samples = [sum(recs, [])] if mode == "asone" else recs
    assert len(offs) == len(samples) + 1
    for i, r in enumerate(samples):
        got = oracle.sketch_records(r, conflict=(mode == "conflict"))
        np.testing.assert_array_equal(got, keys[offs[i]:offs[i + 1]])
