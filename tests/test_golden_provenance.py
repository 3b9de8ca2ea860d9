"""The committed golden vectors are what the reference itself produces.

tests/golden/make_golden.py runs the unmodified js/lbm.js, js/voxel.js and
js/shapes.js of a windtunnel checkout through tests/golden/jsmini.py. This
test reruns the whole generator in memory and requires the manifest (every
SHA-256 digest, body statistic and force value) and every stored array to
equal the committed golden.json / golden.npz exactly, so the fixtures the
oracle is pinned to can be reproduced from the reference at any time. The
checkout is found through WT_REFERENCE_ROOT, else at the path this machine
mounts it; where neither holds js/lbm.js (a GPU box) the test is skipped.
"""
import json
import os
import sys
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def _reference_root() -> Path | None:
    for cand in (os.environ.get("WT_REFERENCE_ROOT"), "/root/reference"):
        if cand and (Path(cand) / "js" / "lbm.js").is_file():
            return Path(cand)
    return None


def test_golden_vectors_regenerate_from_the_reference():
    ref = _reference_root()
    if ref is None:
        pytest.skip("no windtunnel checkout (set WT_REFERENCE_ROOT)")
    sys.path.insert(0, str(GOLDEN))
    try:
        import make_golden
    finally:
        sys.path.remove(str(GOLDEN))
    manifest, arrays = make_golden.generate(ref)
    committed = json.loads((GOLDEN / "golden.json").read_text())
    assert json.loads(json.dumps(manifest, default=float)) == committed
    stored = np.load(GOLDEN / "golden.npz")
    assert sorted(stored.files) == sorted(arrays)
    for k in stored.files:
        assert np.array_equal(stored[k], arrays[k]), k
