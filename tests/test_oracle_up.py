"""CPU: the NumPy restatement of the stabilized u-p plasticity residual
(oracle/np_up.py) against the reference's gold values
(unit_tests/ElastoPlasticityTests.cpp:1967-2100, ElastoPlasticity_Residual3D_Elastic)."""
import json
import os

import numpy as np

from oracle import np_up

HERE = os.path.dirname(os.path.abspath(__file__))


def up_case():
    d = json.load(open(os.path.join(HERE, "golden", "up_residual_3d.json")))
    cells = np.array(d["cells"], np.int32)
    coords = np.array(d["coords"])
    ids = np.arange(coords.shape[0], dtype=np.float64)
    state = np.stack([1e-7 * ids, 2e-7 * ids, 3e-7 * ids, 4e-7 * ids], 1).ravel()
    ppg = np.array(d["projected_pressure_gradient"])
    return d, cells, coords, state, ppg


def test_up_residual_matches_reference_gold():
    d, cells, coords, state, ppg = up_case()
    m = d["material"]
    R = np_up.up_residual_cells(cells, coords, state, np.zeros((6, 14)), ppg.reshape(6, 4, 3), np.ones(8),
                                m["youngs_modulus"], m["poissons_ratio"], m["simp_exponent"], m["simp_min"],
                                m["pressure_scaling"])
    gold = np.array(d["gold"])
    assert d["numberings_matching"] == 1
    assert np.all(np.abs(R - gold) <= d["tolerance"] * np.abs(gold))
