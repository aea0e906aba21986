"""Extract the gold vectors of the reference's 3D elastostatic unit tests into a fixture.

Reads unit_tests/DerivativeTests.cpp of the Plato Analyze reference as text (nothing is
compiled or run) and writes tests/golden/derivative_tests_3d.json.  Run in a checkout that
has the reference tree:

    python tests/golden/make_golden.py /path/to/platoanalyze
"""
from __future__ import annotations

import json
import re
import sys
from pathlib import Path

NUM = re.compile(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?")

# (test name, variable, key in the fixture, scalar?)
WANTED = [
    ("DerivativeTests, 3D ", "gradient_gold", "cell_gradients", False),
    ("DerivativeTests, 3D ", "strain_gold", "cell_strain", False),
    ("DerivativeTests, 3D ", "stress_gold", "cell_stress", False),
    ("DerivativeTests, 3D ", "result_gold", "cell_residual", False),
    ("DerivativeTests, ElastostaticResidual3D ", "residual_gold", "residual", False),
    ("DerivativeTests, ElastostaticResidual3D ", "gold_jac_entries", "jacobian_entries", False),
    ("DerivativeTests, ElastostaticResidual3D ", "gold_grad_entries", "gradient_z_entries", False),
    ("DerivativeTests, InternalElasticEnergy3D ", "value_gold", "energy_value", True),
    ("DerivativeTests, InternalElasticEnergy3D ", "grad_u_gold", "energy_gradient_u", False),
    ("DerivativeTests, InternalElasticEnergy3D ", "grad_z_gold", "energy_gradient_z", False),
]


def extract(src: str, test: str, var: str, scalar: bool):
    start = src.index(f"TEUCHOS_UNIT_TEST( {test.strip()} )")
    i = src.index(var, start)
    line = src.index("\n", i) + 1
    if scalar:
        stmt = src[i:src.index(";", i)]
        return float(NUM.findall(stmt.split("=")[1])[0]), src[:i].count("\n") + 1
    j = src.index("{", i)
    k = src.index("};", j)
    return [float(x) for x in NUM.findall(src[j:k])], src[:line].count("\n")


def main(ref_root: str) -> None:
    path = Path(ref_root) / "unit_tests" / "DerivativeTests.cpp"
    src = path.read_text()
    out = {"source": "unit_tests/DerivativeTests.cpp", "mesh": "2x2x2 TET4 unit cube (48 tets, 27 nodes)",
           "inputs": {"youngs_modulus": 1.0e6, "poissons_ratio": 0.3, "penalty_exponent": 1.0,
                      "penalty_minimum": 0.0, "control": 1.0, "state": "u_i = 1e-4 * (i + 1)"},
           "lines": {}}
    for test, var, key, scalar in WANTED:
        vals, line = extract(src, test, var, scalar)
        out[key] = vals
        out["lines"][key] = f"unit_tests/DerivativeTests.cpp:{line}"
    dst = Path(__file__).resolve().parent / "derivative_tests_3d.json"
    dst.write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {dst}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference checkout root>")
    main(sys.argv[1])
