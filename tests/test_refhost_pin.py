"""The oracle against digests of the reference's own kernels.

tests/golden/refhost_pin.json holds, for each configuration, the SHA-256 of the
whole state after every stage of two bubblesim frames and the three surfaces'
density fields and mesh counts, computed with the reference's kernels compiled
for the host (tests/golden/make_refhost_pin.py, oracle/make_refhost.py).  The
oracle, run stage by stage from the same inputs, must reproduce every digest:
the pin of tests/test_refhost_stages.py, carried without the reference tree.
The mesh counts, not the triangles, are pinned: the triangle lists follow the
generated case table."""
import hashlib
import json
import os

import numpy as np
import pytest

from parity_util import staged_digests
from test_refhost_stages import reference_mode

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "refhost_pin.json")) as _f:
    PIN = json.load(_f)


def _inputs_digest(parts, rf, seeds):
    h = hashlib.sha256()
    for k in sorted(parts):
        if parts[k] is not None:
            h.update(k.encode())
            h.update(np.ascontiguousarray(parts[k]).tobytes())
    h.update(np.ascontiguousarray(rf, np.float32).tobytes())
    h.update(np.ascontiguousarray(seeds, np.int32).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("config", sorted(PIN["configs"], key=int))
def test_oracle_reproduces_the_reference_kernels_digests(mp, oracle_mod, config):
    pin = PIN["configs"][config]
    c = int(config)
    p, parts, rf, seeds = reference_mode(mp, c, PIN["n"], pin["seed"])
    assert _inputs_digest(parts, rf, seeds) == pin["inputs_sha256"], \
        "the scene generator changed: regenerate tests/golden/refhost_pin.json"
    orc = oracle_mod.Oracle(p, mp.FIELD_ID, mp.MPState, mc_tables=mp.mc_tables())
    orc.upload_particles(**parts)
    orc.set_tables(rf, seeds)
    st = orc.state()
    st.n_real_solpoint = int((np.asarray(parts["flag"]) == mp.TYPESOLID).sum())
    orc.set_state(st)
    got = staged_digests(orc, p, PIN["frames"])
    assert len(got) == len(pin["stages"])
    for g, r in zip(got, pin["stages"]):
        assert g[:2] == r[:2]
        assert g == r, f"config {c}: state differs from the reference's kernels after frame {r[0]} stage {r[1]}"
