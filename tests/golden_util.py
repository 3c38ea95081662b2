"""Helpers shared by the golden-vector tests (fixtures under tests/golden/)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def floating_equality(actual, gold, tol, zero_atol=1e-12):
    """Teuchos TEST_FLOATING_EQUALITY: |a-b| / max(|a|,|b|) <= tol.  Gold
    entries that are exactly zero are checked as |a| < zero_atol, as the
    reference's tests do for its zero residual entries."""
    actual = np.asarray(actual, dtype=np.float64)
    gold = np.asarray(gold, dtype=np.float64)
    assert actual.shape == gold.shape, (actual.shape, gold.shape)
    bad = []
    for i, (a, g) in enumerate(zip(actual.ravel(), gold.ravel())):
        if g == 0.0:
            if abs(a) >= zero_atol:
                bad.append((i, a, g))
        else:
            if abs(a - g) / max(abs(a), abs(g)) > tol:
                bad.append((i, a, g))
    assert not bad, f"{len(bad)} entries off (first: {bad[:3]})"


def derivative_case():
    d = load("derivative_tests_3d.json")
    cells = np.array(d["cells"], dtype=np.int32)
    coords = np.array(d["coords"], dtype=np.float64)
    u = 1e-4 * np.arange(1, 3 * coords.shape[0] + 1, dtype=np.float64)
    z = np.ones(coords.shape[0])
    return d, cells, coords, u, z


def star_graph(rowmap, cols, row0):
    """The sorted graph with row 0 in the reference's (Omega_h star) order."""
    cols = cols.copy()
    assert sorted(row0) == list(cols[rowmap[0]:rowmap[1]])
    cols[rowmap[0]:rowmap[1]] = row0
    return rowmap, cols
