"""Loads the golden fixtures (tests/golden/*.npz) and rebuilds their inputs."""
from __future__ import annotations

import hashlib
import json
import pathlib

import numpy as np

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def names():
    """The seeded-system solve fixtures of tests/golden/make_golden.py (the real
    matrices of make_real.py and the Coupled cases of make_coupled.py have
    their own formats and tests, and the hierarchy-only fixtures their own
    loader)."""
    return sorted(p.stem for p in GOLDEN.glob("*.npz")
                  if not p.stem.startswith(("tmr_", "coupled_"))
                  and not p.stem.endswith("_hierarchy"))


def hierarchy_names():
    """Fixtures holding only the reference's AMG hierarchy (level sizes and
    array digests), for systems too large for a reference solve per fixture."""
    return sorted(p.stem for p in GOLDEN.glob("*_hierarchy.npz"))


def load(name):
    d = np.load(GOLDEN / f"{name}.npz")
    meta = json.loads(bytes(d["meta"]).decode())
    arrays = {k: d[k] for k in d.files if k != "meta"}
    return meta, arrays


def system(name):
    """The seeded input system of a fixture (checked against its stored digests)."""
    import sys
    sys.path.insert(0, str(GOLDEN))
    from make_golden import CASES, HIERARCHIES  # noqa: WPS433
    sys.path.pop(0)
    s = (CASES[name] if name in CASES else HIERARCHIES[name])[0]()
    meta, _ = load(name)
    assert digest(s.val) + digest(s.col) == meta["matrix_sha"], "generator drifted from fixture"
    if "rhs_sha" in meta:
        assert digest(s.b) == meta["rhs_sha"], "right-hand side drifted from fixture"
    return s


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
