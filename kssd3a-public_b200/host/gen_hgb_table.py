"""Regenerates hgb_t11_model.c: the 160-tree gradient-boosted calibration model of
the reference (src/model_refaf_hgb.h, generated there by export_refaf_hgb.py for the
default NUM_CODENS = 11 pattern) as one array of node records.

The model is trained data: calibrated ANI must equal the reference's to the printed
digit, so every threshold and leaf value is carried over exactly (doubles written with
17 significant digits, which round-trip).  Run once where the reference sources exist:

    python kssd3a-public_b200/host/gen_hgb_table.py /path/to/reference/src/model_refaf_hgb.h
"""
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def array(text, name):
    m = re.search(r"static const [^=]*\b" + re.escape(name) + r"\[\d+\]\s*=\s*\{(.*?)\};", text, re.S)
    if not m:
        raise SystemExit(f"array {name} not found")
    return [t.strip() for t in m.group(1).replace("\n", " ").split(",") if t.strip()]


def main(path):
    text = open(path).read()
    text = text.split("#if NUM_CODENS == 11", 1)[1].split("#else", 1)[0]
    base = re.search(r"refaf_hgb_baseline\s*=\s*([-0-9.eE+]+)", text).group(1)
    offs = [int(x) for x in array(text, "refaf_hgb_tree_offsets")]
    feat = [int(x) for x in array(text, "refaf_hgb_feature_idx")]
    thr = [float(x) for x in array(text, "refaf_hgb_threshold")]
    val = [float(x) for x in array(text, "refaf_hgb_value")]
    left = [int(x) for x in array(text, "refaf_hgb_left")]
    right = [int(x) for x in array(text, "refaf_hgb_right")]
    leaf = [int(x) for x in array(text, "refaf_hgb_is_leaf")]
    miss = [int(x) for x in array(text, "refaf_hgb_missing_go_left")]
    n = len(feat)
    assert n == offs[-1] == len(thr) == len(val) == len(left) == len(right) == len(leaf) == len(miss)
    out = [
        "/* Generated by gen_hgb_table.py from the reference's src/model_refaf_hgb.h (NUM_CODENS = 11):",
        " * trained calibration trees, carried over exactly.  Do not edit. */",
        '#include "kssd_hgb.h"',
        "",
        f"const double kssd_hgb_baseline = {float(base)!r};",
        f"const unsigned kssd_hgb_tree_begin[KSSD_HGB_TREES + 1] = {{{', '.join(map(str, offs))}}};",
        "const kssd_hgb_node_t kssd_hgb_nodes[KSSD_HGB_NODES] = {",
    ]
    for i in range(n):
        # {threshold or leaf value, feature, flags (bit0 leaf, bit1 missing goes left), left, right}
        x = val[i] if leaf[i] else thr[i]
        out.append(f"    {{{x!r}, {feat[i]}, {leaf[i] | (miss[i] << 1)}, {left[i]}, {right[i]}}},")
    out.append("};")
    with open(os.path.join(HERE, "hgb_t11_model.c"), "w") as f:
        f.write("\n".join(out) + "\n")
    print(f"{n} nodes, {len(offs) - 1} trees")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: gen_hgb_table.py <reference src/model_refaf_hgb.h>")
    main(sys.argv[1])
