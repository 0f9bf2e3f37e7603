"""Regenerates the golden vectors in this directory by running the reference CLI
(oracle/_ref/kssd3a, built from the reference sources by `make -C oracle ref`) on
small seeded fixtures.  Run from the repository root:

    python tests/golden/make_golden.py

counts_*.json : fixture samples + every row of `ani --unique-ctx-report` (the
                reference's full per-cell counters, src/command_ani.c:462-492)
cli/*.out.gz  : the reference CLI's stdout for every case of tests/cli_cases.py
                (seeded synthetic sketch directories, regenerated on demand)
cli_codens/c{9,10}_*.out.gz : the reference CLI compiled for 9 / 10 codens
                (`make -C oracle ref-codens`) on the CODENS_BUILD_CASES of
                tests/cli_cases.py (`python tests/golden/make_golden.py codens` alone)
"""
import csv
import io
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "kssd3a-public_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle  # noqa: E402
from fixtures import mutate_from, random_samples, samples_to_sketch  # noqa: E402
import kssdgpu  # noqa: E402

REF = oracle.REF_BIN


def write_dir(path, samples, prefix, with_index, conflict=True):
    k, o = samples_to_sketch(samples)
    sk = kssdgpu.Sketch(keys=k, offs=o, names=[f"{prefix}_{i}" for i in range(len(samples))], conflict=conflict)
    kssdgpu.write_sketch_dir(path, sk, with_index=with_index)


def counts_case(name, seed, nref, nq, ctx_space, obj_space, ignoreconflict):
    rng = np.random.default_rng(seed)
    refs = random_samples(rng, nref, 30, ctx_space, obj_space, True)
    qrys = random_samples(rng, nq, 30, ctx_space, obj_space, True)
    for i in range(min(nq, nref)):
        if refs[i] and rng.random() < 0.6:
            qrys[i] = mutate_from(rng, refs[i], 0.08)
    tmp = tempfile.mkdtemp(prefix="golden-")
    try:
        write_dir(os.path.join(tmp, "ref"), refs, "ref", True)
        write_dir(os.path.join(tmp, "qry"), qrys, "qry", False)
        rep = os.path.join(tmp, "rep.tsv")
        cmd = [REF, "ani", "-r", os.path.join(tmp, "ref"), "--qraw", os.path.join(tmp, "qry"), "-p2", "-n0", "-f0",
               "-t1", "--unique-ctx-report", rep]
        if ignoreconflict:
            cmd.append("--ignoreconflict")
        subprocess.run(cmd, check=True, capture_output=True)
        rows = []
        with open(rep) as f:
            for r in csv.DictReader(f, delimiter="\t"):
                row = {"q": int(r["Qry"].split("_")[1]), "r": int(r["Ref"].split("_")[1])}
                for k in ("Qry_ctx", "Ref_ctx", "XnY_ctx", "N_diff_obj", "N_diff_obj_section", "N_mut2_ctx",
                          "Unique_Ref_ctx", "Unique_XnY_ctx", "Unique_N_diff_obj", "Unique_N_diff_obj_section",
                          "Unique_N_mut2_ctx"):
                    row[k] = int(r[k])
                rows.append(row)
    finally:
        shutil.rmtree(tmp)
    out = {"command": " ".join(os.path.basename(c) if c.startswith(tmp) else c for c in cmd[1:]),
           "ignoreconflict": ignoreconflict,
           "refs": [[list(p) for p in sorted(set(s))] for s in refs],
           "queries": [[list(p) for p in sorted(set(s))] for s in qrys],
           "rows": rows}
    with open(os.path.join(HERE, f"counts_{name}.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print(name, len(rows), "rows")


def cli_cases():
    """stdout of the reference CLI for every tests/cli_cases.py case, gzip-compressed."""
    import gzip
    from cli_cases import CASES, materialize, with_threads
    out_dir = os.path.join(HERE, "cli")
    os.makedirs(out_dir, exist_ok=True)
    root = tempfile.mkdtemp(prefix="golden-cli-")
    try:
        for name, argv, env in CASES:
            a = materialize(root, argv, "ref_" + name)
            e = dict(os.environ, OMP_NUM_THREADS="4", **{k: v for k, v in env.items() if not k.startswith("_")})
            r = subprocess.run([REF, *with_threads(a)], capture_output=True, env=e, check=True)
            with gzip.GzipFile(os.path.join(out_dir, name + ".out.gz"), "wb", mtime=0) as f:
                f.write(r.stdout)
            print(name, len(r.stdout), "bytes")
    finally:
        shutil.rmtree(root)


def codens_cases():
    """stdout of the reference CLI compiled for 9 and 10 codens (oracle/_ref/kssd3a_c9,
    kssd3a_c10: `make -C oracle ref-codens`) for every CODENS_BUILD_CASES case."""
    import gzip
    from cli_cases import CODENS_BUILD_CASES, materialize, with_threads
    out_dir = os.path.join(HERE, "cli_codens")
    os.makedirs(out_dir, exist_ok=True)
    root = tempfile.mkdtemp(prefix="golden-codens-")
    try:
        for c in (9, 10):
            for name, argv in CODENS_BUILD_CASES:
                a = materialize(root, argv, f"ref_c{c}_" + name)
                e = dict(os.environ, OMP_NUM_THREADS="4")
                r = subprocess.run([f"{REF}_c{c}", *with_threads(a)], capture_output=True, env=e, check=True)
                with gzip.GzipFile(os.path.join(out_dir, f"c{c}_{name}.out.gz"), "wb", mtime=0) as f:
                    f.write(r.stdout)
                print(f"c{c}", name, len(r.stdout), "bytes")
    finally:
        shutil.rmtree(root)


def main():
    if sys.argv[1:] == ["codens"]:
        return codens_cases()
    if not os.path.exists(REF):
        sys.exit(f"{REF} missing: run `make -C oracle ref` first")
    counts_case("s0", 0, 4, 2, 35, 256, False)
    counts_case("s1", 1, 4, 2, 35, 256, True)
    counts_case("s2", 2, 12, 6, 60, 1 << 20, False)
    counts_case("s3", 3, 12, 6, 60, 1 << 20, True)
    counts_case("s4", 4, 30, 10, 400, 1 << 20, False)
    cli_cases()
    codens_cases()


if __name__ == "__main__":
    main()
