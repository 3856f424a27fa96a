"""Writes refhost_pin.json: the state digests after every stage of two
bubblesim frames (and the three surfaces' density fields and mesh counts) of
each configuration, computed with the reference's own kernels compiled for
the host (oracle/make_refhost.py).  tests/test_refhost_pin.py checks the
oracle against them where the reference tree is absent.  Run where the
reference is checked out:

    python tests/golden/make_refhost_pin.py
"""
import hashlib
import importlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "tests")]

CONFIGS = [1, 2, 3, 4, 5]
N = 16
FRAMES = 2
SEED = 2017_800


def inputs_digest(parts, rf, seeds):
    h = hashlib.sha256()
    for k in sorted(parts):
        if parts[k] is not None:
            h.update(k.encode())
            h.update(np.ascontiguousarray(parts[k]).tobytes())
    h.update(np.ascontiguousarray(rf, np.float32).tobytes())
    h.update(np.ascontiguousarray(seeds, np.int32).tobytes())
    return h.hexdigest()


def main():
    mp = importlib.import_module("2017multiphase_b200")
    from oracle import make_refhost
    make_refhost.build(quiet=True)
    from oracle import refhost
    from parity_util import staged_digests
    from test_refhost_stages import reference_mode
    out = {"source": "reference kernels (spray_k.cu) compiled for the host by oracle/make_refhost.py, "
                     "launched by oracle/refhost/stages.inc", "n": N, "frames": FRAMES, "configs": {}}
    for c in CONFIGS:
        p, parts, rf, seeds = reference_mode(mp, c, N, SEED + c)
        ref = refhost.RefHost(p, mp.FIELD_ID, mp.MPState)
        ref.upload_particles(**parts)
        ref.set_tables(rf, seeds)
        st = ref.state()
        st.n_real_solpoint = int((np.asarray(parts["flag"]) == mp.TYPESOLID).sum())
        ref.set_state(st)
        out["configs"][str(c)] = {"seed": SEED + c, "inputs_sha256": inputs_digest(parts, rf, seeds),
                                  "stages": staged_digests(ref, p, FRAMES)}
    # one line per stage
    lines = ["{", f' "source": {json.dumps(out["source"])},', f' "n": {N}, "frames": {FRAMES},', ' "configs": {']
    for ci, (c, d) in enumerate(out["configs"].items()):
        lines.append(f'  "{c}": {{"seed": {d["seed"]}, "inputs_sha256": "{d["inputs_sha256"]}", "stages": [')
        rows = [f"   {json.dumps(r)}" for r in d["stages"]]
        lines.append(",\n".join(rows))
        lines.append("  ]}" + ("," if ci + 1 < len(out["configs"]) else ""))
    lines += [" }", "}"]
    with open(os.path.join(HERE, "refhost_pin.json"), "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    main()
