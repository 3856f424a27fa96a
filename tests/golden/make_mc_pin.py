"""Writes mc_tables_pin.json: SHA-256 digests of the reference's marching-cubes
edge table and per-case vertex counts (Multiphase/Multiphase/tables.h:19-52,
318+), so the generated tables can be pinned where the reference tree is absent
(the digests identify the values without copying them). Run where the
reference is checked out:

    python tests/golden/make_mc_pin.py /path/to/reference/Multiphase/Multiphase/tables.h
"""
import hashlib
import json
import os
import re
import sys

import numpy as np


def parse(path):
    with open(path) as f:
        txt = f.read()

    def block(name):
        m = re.search(name + r"\s*\[[^\]]*\](?:\[[^\]]*\])?\s*=\s*\{(.*?)\};", txt, re.S)
        toks = re.findall(r"0x[0-9a-fA-F]+|\bX\b|-?\d+", m.group(1))
        return [255 if t == "X" else int(t, 0) for t in toks]

    return np.array(block("edgeTable"), np.int32), np.array(block("numVertsTable"), np.int32)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.int32).tobytes()).hexdigest()


if __name__ == "__main__":
    edge, nverts = parse(sys.argv[1])
    out = {"source": "Multiphase/Multiphase/tables.h (edgeTable, numVertsTable) as little-endian int32[256]",
           "edgeTable_sha256": digest(edge), "numVertsTable_sha256": digest(nverts)}
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "mc_tables_pin.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
