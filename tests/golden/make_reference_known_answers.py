"""Writes tests/golden/reference_known_answers.json.

The reference (Remade-With-Rust/rusty_h264) is Rust and cannot be built here,
so its golden vectors for the hot path are the literal values in its own unit
tests and tables.  This script collects them:

* QUANT_MF_OH[52][8] is extracted from crates/rusty_h264-common/src/transform.rs
  (the openh264 g_kiQuantMF table) by parsing the reference source, so no row is
  typed by hand;
* the small known-answer cases (MV prediction, median, flat-block transforms,
  edge-clamped MC) are restated below with the file:line of the test that holds
  each one.

Run it where the reference checkout is present:
    python tests/golden/make_reference_known_answers.py /path/to/rusty_h264
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def extract_quant_mf_oh(ref_root: str):
    src = open(os.path.join(ref_root, "crates/rusty_h264-common/src/transform.rs")).read()
    m = re.search(r"pub const QUANT_MF_OH: \[\[i16; 8\]; 52\] = \[(.*?)\n\];", src, re.S)
    rows = re.findall(r"\[([0-9,\s]+)\]", m.group(1))
    table = [[int(v) for v in r.split(",") if v.strip()] for r in rows]
    assert len(table) == 52 and all(len(r) == 8 for r in table)
    line = src[: m.start()].count("\n") + 1
    return table, f"crates/rusty_h264-common/src/transform.rs:{line}"


def extract_deblock_tables(ref_root: str):
    """ALPHA[52], BETA[52] and TC0[52][3] (spec Tables 8-16/8-17) as the
    reference's deblock.rs holds them."""
    path = "crates/rusty_h264-common/src/deblock.rs"
    src = open(os.path.join(ref_root, path)).read()
    out = {}
    for name in ("ALPHA", "BETA"):
        m = re.search(r"const " + name + r": \[i32; 52\] = \[(.*?)\];", src, re.S)
        vals = [int(v) for v in m.group(1).replace("\n", " ").split(",") if v.strip()]
        assert len(vals) == 52
        out[name.lower()] = {"source": f"{path}:{src[: m.start()].count(chr(10)) + 1}", "values": vals}
    m = re.search(r"const TC0: \[\[i32; 3\]; 52\] = \[(.*?)\n\];", src, re.S)
    rows = [[int(v) for v in r.split(",")] for r in re.findall(r"\[([0-9,\s]+)\]", m.group(1))]
    assert len(rows) == 52 and all(len(r) == 3 for r in rows)
    out["tc0"] = {"source": f"{path}:{src[: m.start()].count(chr(10)) + 1}", "rows": rows}
    return out


def main(ref_root: str):
    qmf, qmf_src = extract_quant_mf_oh(ref_root)
    out = {
        "quant_mf_oh": {"source": qmf_src, "rows": qmf},
        "deblock": extract_deblock_tables(ref_root),
        "median3": {
            "source": "crates/rusty_h264-common/src/inter.rs:1994-1999 (median_of_three)",
            "cases": [[1, 2, 3, 2], [3, 1, 2, 2], [-5, 0, 5, 0], [7, 7, 2, 7]],
        },
        # neighbours: [available, mvx, mvy, ref_idx]; cur_ref; expected
        "predict_mv": {
            "source": "crates/rusty_h264-common/src/inter.rs:2002-2034",
            "cases": [
                {"a": [1, 8, -4, 0], "b": [0, 0, 0, -1], "c": [0, 0, 0, -1], "cur_ref": 0, "want": [8, -4]},
                {"a": [1, 4, 0, 0], "b": [1, 8, 0, 0], "c": [1, 12, 0, 0], "cur_ref": 0, "want": [8, 0]},
                {"a": [1, 0, 0, -1], "b": [1, 5, 7, 0], "c": [1, 0, 0, -1], "cur_ref": 0, "want": [5, 7]},
                {"a": [1, 4, 4, 1], "b": [1, 5, 7, 0], "c": [1, 0, 0, -1], "cur_ref": 0, "want": [5, 7]},
                {"a": [1, 4, 4, 1], "b": [1, 5, 7, 0], "c": [1, 0, 0, -1], "cur_ref": 1, "want": [4, 4]},
            ],
        },
        "forward_core_flat": {
            "source": "crates/rusty_h264-common/src/transform.rs:1167-1176",
            "input": [4] * 16, "dc": 64,
        },
        "forward_core_8x8_flat": {
            "source": "crates/rusty_h264-common/src/transform.rs:1179-1188",
            "input": [4] * 64, "dc": 256,
        },
        "mc_luma": {
            "source": "crates/rusty_h264-common/src/inter.rs:2037-2063",
            "cases": [
                {"ref": [0, 1, 2, 3, 10, 11, 12, 13, 20, 21, 22, 23, 30, 31, 32, 33], "cw": 4, "ch": 4,
                 "x0": 1, "y0": 1, "bw": 2, "bh": 2, "mvx": 0, "mvy": 0, "want": [11, 12, 21, 22]},
                {"ref": [5, 6, 7, 8], "cw": 2, "ch": 2, "x0": 0, "y0": 0, "bw": 2, "bh": 2,
                 "mvx": -40, "mvy": -40, "want": [5, 5, 5, 5]},
            ],
            "flat": {"value": 100, "cw": 8, "ch": 8, "x0": 2, "y0": 2, "bw": 4, "bh": 4,
                     "phases": [[2, 0], [0, 2], [2, 2], [1, 1], [3, 3]]},
        },
        "quant_four_fixed": {
            "source": "crates/rusty_h264-accel/src/transform_quant.rs:199-222",
            "ff": [80, 85, 80, 85, 90, 95, 90, 95],
            "mf": [410, 420, 410, 420, 430, 440, 430, 440],
        },
    }
    path = os.path.join(HERE, "reference_known_answers.json")
    with open(path, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", path)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_reference_known_answers.py <path to the rusty_h264 checkout>")
    main(sys.argv[1])
