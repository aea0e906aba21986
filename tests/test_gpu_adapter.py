"""The C++ adapter (include/plato_b200.hpp) driven from C++ the way the reference's unit
tests drive VectorFunction / PhysicsScalarFunction / Problem, checked against the
reference golds and the CPU oracle."""
import subprocess
from pathlib import Path

import numpy as np
import pytest

from helpers import assert_floating_equality, load_golden, rel_l2
from oracle import Oracle
from platoanalyze_b200.problem import SolverOptions
from platoanalyze_b200.workloads import cantilever

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]
EXE = ROOT / "tests" / "cpp" / "_build" / "test_adapter"


@pytest.fixture(scope="module")
def output():
    from platoanalyze_b200 import build
    build.build_adapter_test()  # no-op when the binary is newer than its sources and the library
    r = subprocess.run([str(EXE)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    out = {}
    for line in r.stdout.splitlines():
        key, _, rest = line.partition(":")
        out[key.strip()] = rest.strip()
    return out


def vals(s):
    return np.array([float(x) for x in s.split()])


def test_adapter_matches_reference_golds(output):
    G = load_golden()
    assert_floating_equality(vals(output["residual"]), G["residual"], 1e-13, zero_abs=1e-11)
    assert_floating_equality(vals(output["jacobian"]), G["jacobian_entries"], 1e-13, zero_abs=1e-9)
    assert_floating_equality(vals(output["gradient_z"]), G["gradient_z_entries"], 2e-14)
    assert_floating_equality([float(output["energy"])], [G["energy_value"]], 1e-13)
    assert_floating_equality(vals(output["energy_gradient_u"]), G["energy_gradient_u"], 1e-13, zero_abs=1e-11)
    assert_floating_equality(vals(output["energy_gradient_z"]), G["energy_gradient_z"], 1e-13)


def test_adapter_problem_matches_oracle(output):
    spec = cantilever(6, 3, 3, SolverOptions(tolerance=1e-12))
    orc = Oracle.from_spec(spec)
    z = np.full(orc.N, 0.5)
    uo, _, _ = orc.solution_refined(z, tol=1e-13)
    u = vals(output["state"])
    assert rel_l2(u, uo) <= 1e-9
    f = float(output["compliance"])
    assert abs(f - orc.sf_value(u, z)) <= 1e-11 * abs(f)
    assert rel_l2(vals(output["dcdz"]), orc.criterion_gradient(z, u)) <= 1e-11
    assert "converged 1" in output["solve"]
    assert output["error_path"] == "status 1"


def test_adapter_helmholtz_matches_oracle(output):
    from platoanalyze_b200.mesh import X_PLUS, box_mesh

    m = box_mesh(6, 3, 3, 2.0, 1.0, 1.0)
    orc = Oracle(m.coords, m.connectivity)
    n = m.num_nodes
    i = np.arange(n)
    control = 0.25 + 0.5 * ((i * 7919) % 101) / 100.0
    w = 1.0 + 0.01 * (i % 13)
    cells, local = m.sideset(X_PLUS)
    S = (0.5, cells, local)
    fo, _ = orc.helmholtz_solution(0.2, control, tol=1e-14, surface=S)
    go, _ = orc.helmholtz_criterion_gradient(0.2, w, tol=1e-14, surface=S)
    assert rel_l2(vals(output["filtered"]), fo) <= 1e-10
    assert rel_l2(vals(output["filter_gradient"]), go) <= 1e-10
    assert rel_l2(vals(output["filter_jacobian"]), orc.helmholtz_gradient_u(0.2, surface=S)) <= 1e-13
