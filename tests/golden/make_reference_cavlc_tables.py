"""Writes tests/golden/reference_cavlc_tables.json.

The CAVLC VLC tables (the standard's Tables 9-4, 9-5, 9-7..9-10) as the
reference writes and reads them, parsed from its source
crates/rusty_h264-common/src/cavlc.rs (CBP_INTER :94, COEFF_TOKEN_LEN/BITS
:143/:175, CHROMA_DC_COEFF_TOKEN_LEN/BITS :208/:212, TOTAL_ZEROS_LEN/BITS
:218/:236, CHROMA_DC_TOTAL_ZEROS_LEN/BITS :256/:262, RUN_LEN/BITS :270/:280),
so no entry is typed by hand.  The tests compare the library's writer tables
with these and drive the oracle's decoder with them.

Run it where the reference checkout is present:
    python tests/golden/make_reference_cavlc_tables.py /path/to/rusty_h264
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ("CBP_INTER", "COEFF_TOKEN_LEN", "COEFF_TOKEN_BITS", "CHROMA_DC_COEFF_TOKEN_LEN", "CHROMA_DC_COEFF_TOKEN_BITS",
         "TOTAL_ZEROS_LEN", "TOTAL_ZEROS_BITS", "CHROMA_DC_TOTAL_ZEROS_LEN", "CHROMA_DC_TOTAL_ZEROS_BITS", "RUN_LEN",
         "RUN_BITS")


def parse(src: str, name: str):
    m = re.search(r"const\s+" + name + r"\s*:\s*\[[^=]*=\s*(\[.*?\]);", src, re.S)
    if not m:
        raise SystemExit(f"{name} not found")
    body = re.sub(r"//[^\n]*", "", m.group(1))
    return json.loads(re.sub(r",\s*\]", "]", body))


def main(root: str):
    src = open(os.path.join(root, "crates/rusty_h264-common/src/cavlc.rs")).read()
    out = {n: parse(src, n) for n in NAMES}
    path = os.path.join(HERE, "reference_cavlc_tables.json")
    with open(path, "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print("wrote", path)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_reference_cavlc_tables.py <path to the rusty_h264 checkout>")
    main(sys.argv[1])
