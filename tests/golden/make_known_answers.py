"""Writes reference_known_answers.json: the input vectors and expected values that the
reference's own tests and docs pin for this path, transcribed with their file:line.
Expected values are computed from the formulas those tests state (not from any code here).
Run: python tests/golden/make_known_answers.py
"""
import json
import math
import os

g = 9.81


def phys(U, n):
    h, hu, hv = U
    u, v = hu / h, hv / h
    un = u * n[0] + v * n[1]
    return [h * un, hu * un + 0.5 * g * h * h * n[0], hv * un + 0.5 * g * h * h * n[1]]


cases = {
    "flux_consistency": [
        # tests/unit/test_numerical_flux.cpp:17-40 (LF, n = x)
        {"kind": "lf", "U": [1.0, 0.5, 0.3], "n": [1.0, 0.0], "F": phys([1.0, 0.5, 0.3], [1, 0])},
        # :60-82 (HLLC, n = y)
        {"kind": "hllc", "U": [2.0, 1.0, -0.5], "n": [0.0, 1.0], "F": phys([2.0, 1.0, -0.5], [0, 1])},
        # :84-110 (Roe, 45 degree normal)
        {"kind": "roe", "U": [1.5, 0.75, 0.45], "n": [math.sqrt(0.5), math.sqrt(0.5)],
         "F": phys([1.5, 0.75, 0.45], [math.sqrt(0.5), math.sqrt(0.5)])},
    ],
    # :43-57 symmetry F*(L,R,n) = -F*(R,L,-n)
    "flux_symmetry": {"kind": "lf", "UL": [1.0, 0.5, 0.2], "UR": [1.2, 0.6, 0.1], "n": [1.0, 0.0]},
    # :150-172 conservation for LF, HLLC, Roe
    "flux_conservation": {"UL": [1.0, 0.5, 0.2], "UR": [1.5, 0.3, 0.4], "n": [0.6, 0.8]},
    # :131-148 dry-cell handling: finite result
    "flux_dry": {"UL": [1e-12, 0.0, 0.0], "UR": [1.0, 0.5, 0.0], "n": [1.0, 0.0]},
    # LGL nodes/weights tabulated in src/physics/vertical_velocity.cpp:190-200 (on [-1, 1])
    "lgl": {
        "3": {"x": [-1.0, -math.sqrt(1 / 5), math.sqrt(1 / 5), 1.0], "w": [1 / 6, 5 / 6, 5 / 6, 1 / 6]},
        "4": {"x": [-1.0, -math.sqrt(3 / 7), 0.0, math.sqrt(3 / 7), 1.0],
              "w": [1 / 10, 49 / 90, 32 / 45, 49 / 90, 1 / 10]},
        "2": {"x": [-1.0, 0.0, 1.0], "w": [1 / 3, 4 / 3, 1 / 3]},
    },
    # tests/integration/test_conservation.cpp:63-130: div(x, y, z) over [-1,1]^3 = 24
    "divergence_theorem": {"order": 3, "value": 24.0},
    # tests/unit/test_mode_splitting.cpp:11-37 element setup: N=2, h=100 m, f=1e-4
    "mode_split_element": {"order": 2, "h": 100.0, "f": 1e-4, "u_const": 1.5},
    # tests/integration/test_cg_cubic_bezier_bathymetry_smoother.cpp:935-966: 8x8 -> 625 DOFs
    "bezier_dofs": {"n": 8, "dofs": 625},
    # docs/cg_bezier_solver_verification.md:32-39 (16x16, lambda=1, C1 edges, direct KKT)
    "bezier_doc_16x16": {"objective": 25.235, "x_norm": 61.715, "data_residual": 0.1398,
                         "regularization": 0.0040, "dofs": 2401},
}

out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_known_answers.json")
with open(out, "w") as fh:
    json.dump(cases, fh, indent=1)
print(out)
