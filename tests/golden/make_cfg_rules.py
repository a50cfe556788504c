"""Extracts the rules of the reference's shipped tuning files into a fixture.

    python tests/golden/make_cfg_rules.py <reference root>

(or with the reference root in the environment variable HML_REFERENCE_DIR).
For each file under ``config/`` of the reference it records the rules in file
order -- duplicates included, since the reference's reader lets the last one
win -- as an int16 array: SGEMM ``K colStops type rowStops`` rows,
SGEMV ``N type blockStops rowStops`` rows.  The parsing restates the
reference's readers (src/hml_sgemm_kernel.cu:573-602,
src/hml_sgemv_kernel.cu:650-679): lines starting with '#' are skipped, every
other line gives four integers.  ``tests/test_cfg_roundtrip.py`` checks the
library's v1 reader and writer against this fixture.
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SGEMM_RULE = re.compile(r"^\s*(-?\d+)\s+(-?\d+)\s*:\s*(-?\d+)\s+(-?\d+)\s*$")
SGEMV_RULE = re.compile(r"^\s*(-?\d+)\s*:\s*(-?\d+)\s+(-?\d+)\s+(-?\d+)\s*$")


def parse(path, kind):
    rows = []
    pat = SGEMM_RULE if kind == "sgemm" else SGEMV_RULE
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                continue
            m = pat.match(line)
            if not m:
                raise SystemExit(f"{path}: unexpected line {line!r}")
            rows.append([int(g) for g in m.groups()])
    return np.array(rows, np.int16).reshape(-1, 4)


def main():
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HML_REFERENCE_DIR")
    if not root:
        raise SystemExit("usage: make_cfg_rules.py <reference root> (or set HML_REFERENCE_DIR)")
    cfg = os.path.join(root, "config")
    out = {}
    for name in sorted(os.listdir(cfg)):
        if not name.endswith(".cfg"):
            continue
        kind = "sgemm" if name.startswith("hml_sgemm") else "sgemv"
        out[name[:-4]] = parse(os.path.join(cfg, name), kind)
    np.savez_compressed(os.path.join(HERE, "cfg_rules.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
