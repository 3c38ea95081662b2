"""Generate the golden fixtures in tests/golden/ from the reference's own tests.

Run from the repository root with the path of a platoanalyze source tree,
as an argument or in the PA_REFERENCE environment variable:

    python tests/golden/make_golden.py <platoanalyze source tree>

The reference cannot be built here (it needs Trilinos, Omega_h and Kokkos), so
its unit tests are read as text and their gold arrays extracted:

* unit_tests/DerivativeTests.cpp, ElastostaticResidual3D and
  InternalElasticEnergy3D: 2x2x2 unit box, E=1e6, nu=0.3, SIMP p=1, min 0,
  z = 1, u_i = 1e-4 (i+1).
* unit_tests/PlasticityTests.cpp, J2PlasticityUtils_UpdatePlasticStep3D.
* unit_tests/ElastoPlasticityTests.cpp, ElastoPlasticity_Residual3D_Elastic
  (stabilized u-p residual on the single-hex box) and
  ElastoPlasticity_ElasticSolution3D (the u-p plasticity solve on the same
  box: one pseudo-time step, x = 0 face fixed, u_y = -1e-3 on x = 1).

The gold values depend on the vertex numbering of Omega_h's build_box, whose
source is not available.  It is identified here by search rather than
restated: the tet split is the one the reference's single-hex box test lists
(unit_tests/OmegaHUtilitiesTests.cpp:258-287, the six tets around the hex
diagonal, repeated in every hex), and the vertex permutation is the solution
of a 0/1 integer program (scipy.optimize.milp): a bijection from the 27 grid
points to vertex ids such that K(perm) u equals the 81 gold residual values.
The fixture records the permutation found, so tests never need the search.

The residual, Jacobian and energy gold are also invariant under the point
reflection x -> 1 - x, which the configuration gradient is not; the
orientation is taken from the sign of the first gold gradient_x entry.

The gold Jacobian and dR/dz arrays are raw block-CRS entry arrays whose
in-row column order is Omega_h's node-star order (not sorted).  Only row 0
is covered by the gold (45 and 24 entries); its column order is recovered by
matching each gold 3x3 / 1x3 block to exactly one neighbour block.
"""
import json
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import np_ref  # noqa: E402

REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("PA_REFERENCE", "")
OUT = os.path.dirname(os.path.abspath(__file__))


def grab(src, name, start):
    i = src.index(name, start)
    j = src.index("{", i)
    k = src.index("}", j)
    return [float(x) for x in re.findall(r"[-+]?[0-9]*\.?[0-9]+(?:[eE][-+]?[0-9]+)?", src[j + 1:k])]


def identify_numbering(R_gold):
    """Solve for the vertex permutation of the 2x2x2 box (see module doc)."""
    from scipy.optimize import Bounds, LinearConstraint, milp

    cells, coords = np_ref.box_mesh(2, 2, 2)  # grid numbering, same tet split
    prob = np_ref.Problem(cells, coords, E=1e6, nu=0.3, p=1.0, pmin=0.0)
    K = prob.stiffness_dense(np.ones(27))
    # u(vertex v) = 1e-4 (3v+1, 3v+2, 3v+3) = 3e-4 v (1,1,1) + rigid shift; K kills the shift.
    Kh = np.zeros((27, 3, 27))
    for g in range(27):
        for h in range(27):
            Kh[g, :, h] = K[3 * g:3 * g + 3, 3 * h:3 * h + 3].sum(1)
    R = np.asarray(R_gold).reshape(27, 3)
    nv = 27 * 27  # x[g*27 + v] = 1 iff grid point g carries vertex id v
    rows, lo, hi = [], [], []
    for g in range(27):
        r = np.zeros(nv); r[g * 27:(g + 1) * 27] = 1; rows.append(r); lo.append(1); hi.append(1)
    for v in range(27):
        r = np.zeros(nv); r[v::27] = 1; rows.append(r); lo.append(1); hi.append(1)
    for g in range(27):
        for d in range(3):
            r = np.zeros(nv)
            for h in range(27):
                r[h * 27:(h + 1) * 27] += 3e-4 * Kh[g, d, h] * np.arange(27)
            r[g * 27:(g + 1) * 27] -= R[:, d]
            rows.append(r / 100.0); lo.append(-1e-6); hi.append(1e-6)
    res = milp(c=np.zeros(nv), constraints=LinearConstraint(np.array(rows), lo, hi),
               integrality=np.ones(nv), bounds=Bounds(0, 1))
    assert res.status == 0, res.message
    perm = res.x.reshape(27, 27).round().astype(int).argmax(1)  # grid point -> vertex id
    v_coords = np.zeros((27, 3))
    v_coords[perm] = coords
    v_cells = perm[cells]
    return v_cells.astype(np.int32), v_coords


def choose_orientation(cells, coords, gold_dRdx00):
    """The residual, Jacobian and energy gold are invariant under the point
    reflection x -> 1 - x of the box (gradients flip sign, B^T C B does not),
    so the integer program cannot tell the two numberings apart; the
    configuration gradient can.  Keep the orientation whose dR_0x/dx_0x (the
    first gold gradient_x entry; node 0 is its own row-0 column) has the gold's
    sign, checked by a central difference."""
    u = 1e-4 * np.arange(1, 3 * coords.shape[0] + 1, dtype=np.float64)
    z = np.ones(coords.shape[0])
    h = 1e-6
    cp, cm = coords.copy(), coords.copy()
    cp[0, 0] += h
    cm[0, 0] -= h
    rp = np_ref.Problem(cells, cp, E=1e6, nu=0.3, p=1.0, pmin=0.0).value(u, z)
    rm = np_ref.Problem(cells, cm, E=1e6, nu=0.3, p=1.0, pmin=0.0).value(u, z)
    fd = (rp[0] - rm[0]) / (2 * h)
    if np.sign(fd) != np.sign(gold_dRdx00):
        coords = 1.0 - coords
    return cells, coords


def star_order_row0(blocks_gold, Kfull, cols_sorted, bi, bj):
    """Column order of row 0 that reproduces the gold block sequence."""
    order = []
    for b in blocks_gold:
        hits = [int(c) for c in cols_sorted
                if np.allclose(Kfull[0:bi, bj * c:bj * c + bj].ravel(), b, rtol=1e-12, atol=1e-9) and c not in order]
        assert len(hits) == 1, hits
        order.append(hits[0])
    return order


def derivative_tests():
    src = open(os.path.join(REF, "unit_tests/DerivativeTests.cpp")).read()
    s0 = src.index("DerivativeTests, ElastostaticResidual3D")
    s1 = src.index("DerivativeTests, InternalElasticEnergy3D")
    gold = {
        "residual": grab(src, "residual_gold", s0),
        "jacobian_entries": grab(src, "gold_jac_entries", s0),
        "gradient_z_entries": grab(src, "gold_grad_entries", s0),
        "gradient_x_entries": grab(src, "gold_grad_x_entries", s0),
        "energy_value": 46.125,
        "energy_grad_u": grab(src, "grad_u_gold", s1),
        "energy_grad_z": grab(src, "grad_z_gold", s1),
        "energy_grad_x": grab(src, "grad_x_gold", s1),
    }
    cells, coords = identify_numbering(gold["residual"])
    cells, coords = choose_orientation(cells, coords, gold["gradient_x_entries"][0])
    prob = np_ref.Problem(cells, coords, E=1e6, nu=0.3, p=1.0, pmin=0.0)
    z = np.ones(27)
    u = 1e-4 * np.arange(1, 82, dtype=np.float64)
    K = prob.stiffness_dense(z)
    G = prob.gradient_z_dense(u, z)
    rowmap, cols = np_ref.crs_graph(cells, 27)
    row0 = [int(c) for c in cols[rowmap[0]:rowmap[1]]]
    jac_order = star_order_row0(np.asarray(gold["jacobian_entries"]).reshape(-1, 9), K, row0, 3, 3)
    gz_order = star_order_row0(np.asarray(gold["gradient_z_entries"]).reshape(-1, 3), G, row0, 1, 3)
    assert gz_order[:len(jac_order)] == jac_order
    return {
        "source": "unit_tests/DerivativeTests.cpp:273-700 (ElastostaticResidual3D, InternalElasticEnergy3D)",
        "mesh": "Omega_h build_box 2x2x2 on the unit cube; numbering identified by tests/golden/make_golden.py",
        "material": {"youngs_modulus": 1.0e6, "poissons_ratio": 0.3, "simp_exponent": 1.0, "simp_min": 0.0},
        "state": "u_i = 1e-4 * (i + 1), z = 1",
        "tolerances": {"residual": 1e-13, "jacobian_entries": 1e-15, "gradient_z_entries": 2e-14,
                       "gradient_x_entries": 1e-13, "energy_value": 1e-13, "energy_grad_u": 1e-13,
                       "energy_grad_z": 1e-13},
        "cells": cells.tolist(),
        "coords": coords.tolist(),
        "row0_star_order": gz_order,
        "gold": gold,
    }


def j2_plastic_step():
    src = open(os.path.join(REF, "unit_tests/PlasticityTests.cpp")).read()
    s = src.index("J2PlasticityUtils_UpdatePlasticStep3D")
    e = src.index("TEUCHOS_UNIT_TEST", s + 10)
    body = src[s:e]
    i = body.index("tGold")
    j = body.index("{{", i)
    k = body.index("}};", j)
    rows = re.findall(r"\{([^{}]*)\}", body[j + 1:k + 1])
    gold = []
    for r in rows:
        vals = []
        for tok in re.findall(r"tHostPrevLocalState\(\d,\d\)|[-+]?[0-9]*\.?[0-9]+", r):
            m = re.match(r"tHostPrevLocalState\((\d),(\d)\)", tok)
            vals.append((int(m.group(1)) + 1.0) * (int(m.group(2)) + 1.0) if m else float(tok))
        gold.append(vals)
    return {
        "source": "unit_tests/PlasticityTests.cpp:283-333 (J2PlasticityUtils_UpdatePlasticStep3D)",
        "setup": "prev[i][j] = (i+1)(j+1); normal[i][j] = (i+1)(j+2)/5; local state starts as prev; H_kin = 3",
        "tolerance": 1e-4,
        "gold": gold,
    }


def up_residual_3d():
    """ElastoPlasticity_Residual3D_Elastic (unit_tests/ElastoPlasticityTests.cpp:1967-2100):
    stabilized u-p residual on the single-hex box (6 tets), E = 1e11, nu = 0.35,
    SIMP 3 / 1e-9, controls 1, zero local states, nodal state
    (1e-7, 2e-7, 3e-7, 4e-7) x vertex id, projected pressure gradient
    4e-7 (n+1)(d+1)(c+1) at node n of cell c.  The per-cell vertex coordinates
    are the reference's own (unit_tests/OmegaHUtilitiesTests.cpp:258-287, the
    six-tet split); the vertex ids of the eight corners are identified by
    exhaustive search over the 8! numberings against the gold residual."""
    import itertools
    from oracle import np_up
    src = open(os.path.join(REF, "unit_tests/ElastoPlasticityTests.cpp")).read()
    s = src.index("ElastoPlasticity_Residual3D_Elastic")
    i = src.index("tGold", s)
    j = src.index("{", i)
    k = src.index("};", j)
    rows = re.findall(r"\{([^{}]*)\}", src[j + 1:k + 1])
    gold = [[float(t) for t in re.findall(r"[-+]?[0-9]*\.?[0-9]+(?:[eE][-+]?[0-9]+)?", r)] for r in rows]
    gold = np.array(gold)
    assert gold.shape == (6, 16), gold.shape
    corners = [(a, b, c) for c in (0, 1) for b in (0, 1) for a in (0, 1)]
    tets = np_ref.HEX_TETS
    coords_c = np.array(corners, dtype=np.float64)
    cells_c = np.array([[corners.index(v) for v in t] for t in tets])
    ppg = np.array([[[4e-7 * (n + 1) * (d + 1) * (c + 1) for d in range(3)] for n in range(4)] for c in range(6)])
    local = np.zeros((6, 14))
    hits = []
    for perm in itertools.permutations(range(8)):
        perm = np.array(perm)  # corner -> vertex id
        ids = perm.astype(np.float64)
        state = np.zeros((8, 4))
        for d in range(4):
            state[:, d] = (d + 1) * 1e-7 * ids
        R = np_up.up_residual_cells(cells_c, coords_c, state.ravel(), local, ppg, np.ones(8), 1e11, 0.35)
        if np.all(np.abs(R - gold) <= 1e-4 * np.maximum(np.abs(gold), 1e-30) + 1e-12):
            hits.append(perm)
    assert len(hits) >= 1, "no numbering reproduces the gold"
    perm = hits[0]
    v_coords = np.zeros((8, 3))
    v_coords[perm] = coords_c
    v_cells = perm[cells_c]
    return {
        "source": "unit_tests/ElastoPlasticityTests.cpp:1967-2100 (ElastoPlasticity_Residual3D_Elastic)",
        "mesh": "Omega_h build_box 1x1x1, six tets; vertex ids identified by tests/golden/make_golden.py",
        "numberings_matching": len(hits),
        "material": {"youngs_modulus": 1e11, "poissons_ratio": 0.35, "simp_exponent": 3.0, "simp_min": 1e-9,
                     "pressure_scaling": 1.0},
        "state": "vertex v: (1e-7 v, 2e-7 v, 3e-7 v, 4e-7 v); controls 1; local states 0",
        "projected_pressure_gradient": ppg.reshape(6, 12).tolist(),
        "tolerance": 1e-4,
        "cells": v_cells.tolist(),
        "coords": v_coords.tolist(),
        "gold": gold.tolist(),
    }


def up_elastic_solution_3d(box):
    """ElastoPlasticity_ElasticSolution3D (unit_tests/ElastoPlasticityTests.cpp:2101-2233):
    PlasticityProblem::solution on the single-hex box of up_residual_3d (same
    Omega_h build_box mesh), controls 1, one pseudo-time step; the state
    (u_x, u_y, u_z, p per vertex) after the Newton solve, tolerance 1e-4."""
    src = open(os.path.join(REF, "unit_tests/ElastoPlasticityTests.cpp")).read()
    s = src.index("ElastoPlasticity_ElasticSolution3D")
    e = src.index("TEUCHOS_UNIT_TEST", s)
    body = src[s:e]

    def param(name):
        m = re.search(r"name='" + re.escape(name) + r"'\s+type='double'\s+value='([^']+)'", body)
        return float(m.group(1))

    i = body.index("tGold")
    j = body.index("{", i)
    k = body.index("};", j)
    rows = re.findall(r"\{([^{}]*)\}", body[j + 1:k + 1])
    gold = [float(t) for t in re.findall(r"[-+]?[0-9]*\.?[0-9]+(?:[eE][-+]?[0-9]+)?", rows[0])]
    assert len(gold) == 32, len(gold)
    assert "-0.001*t" in body and "Initial Num. Pseudo Time Steps' type='int' value='1'" in body
    return {
        "source": "unit_tests/ElastoPlasticityTests.cpp:2101-2233 (ElastoPlasticity_ElasticSolution3D)",
        "mesh": box["mesh"],
        "material": {"youngs_modulus": param("Youngs Modulus"), "poissons_ratio": param("Poissons Ratio"),
                     "simp_exponent": param("Exponent"), "simp_min": param("Minimum Value"), "pressure_scaling": 1.0},
        "j2": {"initial_yield_stress": param("Initial Yield Stress"),
               "hardening_modulus_isotropic": param("Hardening Modulus Isotropic"),
               "hardening_modulus_kinematic": param("Hardening Modulus Kinematic"),
               "elastic_penalty_exponent": param("Elastic Properties Penalty Exponent"),
               "elastic_min_ersatz": param("Elastic Properties Minimum Ersatz"),
               "plastic_penalty_exponent": param("Plastic Properties Penalty Exponent"),
               "plastic_min_ersatz": param("Plastic Properties Minimum Ersatz")},
        "steps": 1,
        "boundary": "x = 0 vertices: u_x = u_y = u_z = 0; x = 1 vertices: u_y = -0.001 t at t = 1",
        "tolerance": 1e-4,
        "cells": box["cells"],
        "coords": box["coords"],
        "gold": gold,
    }


def main():
    if not REF or not os.path.isdir(os.path.join(REF, "unit_tests")):
        sys.exit("usage: make_golden.py <platoanalyze source tree> (or set PA_REFERENCE)")
    with open(os.path.join(OUT, "derivative_tests_3d.json"), "w") as f:
        json.dump(derivative_tests(), f, indent=1)
    with open(os.path.join(OUT, "j2_plastic_step_3d.json"), "w") as f:
        json.dump(j2_plastic_step(), f, indent=1)
    box = up_residual_3d()
    with open(os.path.join(OUT, "up_residual_3d.json"), "w") as f:
        json.dump(box, f, indent=1)
    with open(os.path.join(OUT, "up_elastic_solution_3d.json"), "w") as f:
        json.dump(up_elastic_solution_3d(box), f, indent=1)
    print("wrote fixtures to", OUT)


if __name__ == "__main__":
    main()
