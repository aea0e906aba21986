"""The MPMD application on the GPU: operations run from the deck and the operations file give
the same values, gradients and states as the problem built directly through the C ABI, and
operation parameters rebuild the problem the way the reference's parse_inline does."""
from pathlib import Path

import numpy as np
import pytest
import torch

from helpers import rel_l2
from platoanalyze_b200 import capi
from platoanalyze_b200.app import AnalyzeApp
from platoanalyze_b200.mesh import X_MINUS, box_mesh, exterior_faces
from platoanalyze_b200.problem import EllipticProblem, HelmholtzFilter, SolverOptions, cantilever_spec
from platoanalyze_b200.workloads import splitmix_uniform

pytestmark = pytest.mark.gpu
DECKS = Path(__file__).resolve().parent / "decks"


@pytest.fixture(scope="module")
def app():
    a = AnalyzeApp("cantilever.xml", "operations.xml", base_dir=str(DECKS))
    yield a
    a.close()


@pytest.fixture(scope="module")
def direct():
    m = box_mesh(12, 6, 6, 2.0, 1.0, 1.0)
    spec = cantilever_spec(m, traction=(0.0, -1.0, 0.0), solver=SolverOptions(tolerance=1e-12))
    p = EllipticProblem(spec)
    yield p, m
    p.close()


def test_objective_value_and_gradient(app, direct):
    prob, m = direct
    z = splitmix_uniform(m.num_nodes, 41)
    app.import_field("Topology", z)
    app.compute("Compute Objective")
    f = app.export_value("Objective Value")
    g = app.export_field("Objective Gradient")
    zd = prob.to_dev(z)
    u, st = prob.solution(zd)
    assert st["converged"] == 1
    f0 = prob.criterion_value(zd, u)
    g0, _ = prob.criterion_gradient(zd, u)
    assert abs(f - f0) <= 1e-12 * abs(f0)
    assert rel_l2(g, g0.cpu().numpy()) <= 1e-12
    uh = u.cpu().numpy()
    for k, name in enumerate(("displacement X", "displacement Y", "displacement Z")):
        assert rel_l2(app.export_field(name), uh[k::3]) <= 1e-12
    assert np.array_equal(app.export_field("Topology"), z)


def test_volume_constraint(app, direct):
    prob, m = direct
    z = splitmix_uniform(m.num_nodes, 43)
    app.import_field("Topology", z)
    app.compute("Compute Constraint Value")
    app.compute("Compute Constraint Gradient")
    zd = prob.to_dev(z)
    v0 = prob.volume_value(zd, 1.0, 0.0)
    assert abs(app.export_value("Constraint Value") - (v0 - 0.4)) <= 1e-13 * abs(v0)
    assert rel_l2(app.export_field("Constraint Gradient"), prob.volume_gradient_z(zd, 1.0, 0.0).cpu().numpy()) <= 1e-14


def test_operation_parameter_rebuilds_the_problem(app):
    z = splitmix_uniform(app.num_nodes, 47)
    app.import_field("Topology", z)
    app.compute("Compute Scaled Load Solution")
    u1 = app.export_field("displacement Y")
    app.import_parameter("Compute Scaled Load Solution", "Tip Load Y", -2.5)
    app.compute("Compute Scaled Load Solution")
    u2 = app.export_field("displacement Y")
    assert rel_l2(u2, 2.5 * u1) <= 1e-10  # linear in the load
    app.import_parameter("Compute Scaled Load Solution", "Tip Load Y", -1.0)
    app.compute("Compute Scaled Load Solution")
    assert rel_l2(app.export_field("displacement Y"), u1) <= 1e-11
    assert np.array_equal(app.export_field("Topology"), z)  # the control survives the rebuild


def test_errors(app):
    with pytest.raises(capi.PlatoError) as e:
        app.compute("Compute Everything")
    assert e.value.status == capi.BAD_INPUT and "doesn't exist" in str(e.value)
    with pytest.raises(capi.PlatoError):
        app.import_field("Topology", np.ones(app.num_nodes + 1))
    with pytest.raises(capi.PlatoError) as e:
        app.import_parameter("Compute Objective", "Tip Load Y", 1.0)
    assert "wasn't defined for this operation" in str(e.value)
    with pytest.raises(capi.PlatoError):
        app.export_value("No Such Value")


def test_filter_operations():
    a = AnalyzeApp("filter.xml", "filter_operations.xml", base_dir=str(DECKS))
    m = box_mesh(12, 6, 6, 2.0, 1.0, 1.0)
    faces = exterior_faces(m.connectivity, m.nodeset(X_MINUS))
    filt = HelmholtzFilter(m.coords, m.connectivity, 0.15, surface_length_scale=0.5, surface_faces=faces)
    c = splitmix_uniform(m.num_nodes, 53)
    a.import_field("Topology", c)
    a.compute("Filter Control")
    f0, _ = filt.solution(filt.to_dev(c))
    assert rel_l2(a.export_field("Topology"), f0.cpu().numpy()) <= 1e-12
    assert rel_l2(a.export_field("filtered density"), f0.cpu().numpy()) <= 1e-12
    w = np.cos(np.arange(m.num_nodes) * 0.3)
    a.import_field("Topology", w)
    a.compute("Filter Gradient")
    g0, _ = filt.criterion_gradient(filt.to_dev(w))
    assert rel_l2(a.export_field("Topology"), g0.cpu().numpy()) <= 1e-12
    a.close()
    filt.close()
    torch.cuda.synchronize()


def test_exodus_input_mesh_matches_the_generated_box():
    """The same cantilever from an Exodus file and from the generator: same objective."""
    deck = (DECKS / "cantilever.xml").read_text()
    ops = (DECKS / "operations.xml").read_text()
    a = AnalyzeApp(deck.replace("box:12,6,6:2.0,1.0,1.0", "box:6,3,3:2.0,1.0,1.0"), ops)
    b = AnalyzeApp(deck.replace("box:12,6,6:2.0,1.0,1.0", "box_6x3x3.exo"), ops, base_dir=str(DECKS))
    z = splitmix_uniform(a.num_nodes, 59)
    for app_ in (a, b):
        app_.import_field("Topology", z)
        app_.compute("Compute Objective")
    assert abs(a.export_value("Objective Value") - b.export_value("Objective Value")) <= \
        1e-12 * abs(a.export_value("Objective Value"))
    assert rel_l2(b.export_field("Objective Gradient"), a.export_field("Objective Gradient")) <= 1e-12
    a.close()
    b.close()
