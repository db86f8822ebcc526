"""Writes tests/golden/tangent_logpfc_eps-0.9.json from the reference's common-tangent
test (tests/test_phase_diagram_common_tangent.py:43-77): the eps = -0.9 logPFC
triangle table (phi, fmin, q0*) and the coexistence densities it pins.

    python tests/golden/make_tangent_golden.py <reference checkout>
"""
import ast
import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit(f"usage: python {sys.argv[0]} <reference checkout>")
ref = sys.argv[1]
src = open(os.path.join(ref, "tests", "test_phase_diagram_common_tangent.py")).read()
tree = ast.parse(src)
vals = {}
for node in tree.body:
    if not (isinstance(node, ast.Assign) and len(node.targets) == 1):
        continue
    tgt = node.targets[0]
    if isinstance(tgt, ast.Tuple):   # BETA, G = 0.5, -2.0
        for n, v in zip(tgt.elts, ast.literal_eval(node.value)):
            vals[n.id] = v
    elif isinstance(tgt, ast.Name) and tgt.id in ("TRIANGLE_EPS_M0P9", "REF_PHI_L", "REF_PHI_S", "REF_MU",
                                                  "REF_OMEGA", "FSOLVE_P0201"):
        vals[tgt.id] = ast.literal_eval(node.value)
out = {
    "source": "tests/test_phase_diagram_common_tangent.py:33-77 (reference)",
    "beta": vals["BETA"], "g": vals["G"], "eps": -0.9,
    "triangle": [list(r) for r in vals["TRIANGLE_EPS_M0P9"]],
    "phi_l_notebook": vals["REF_PHI_L"], "phi_s_notebook": vals["REF_PHI_S"],
    "mu": vals["REF_MU"], "omega": vals["REF_OMEGA"],
    "fsolve": vals["FSOLVE_P0201"],
    # the reference module with the analytic liquid: notebook values + (2.064e-9, -2.612e-9)
    "phi_l_analytic": vals["REF_PHI_L"] + 2.064e-9, "phi_s_analytic": vals["REF_PHI_S"] - 2.612e-9,
}
dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tangent_logpfc_eps-0.9.json")
json.dump(out, open(dst, "w"), indent=1)
print(dst)
