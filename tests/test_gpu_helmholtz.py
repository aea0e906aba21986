"""Helmholtz density filter through the C ABI against the CPU oracle: residual, Jacobian and
(dR/dcontrol)^T entries on the (bit-exact) node pattern, the filtered density, the chain rule,
and the reference's known answer (a uniform density is left unchanged)."""
import numpy as np
import pytest

from helpers import rel_l2
from oracle import Oracle
from platoanalyze_b200 import capi
from platoanalyze_b200.mesh import X_MINUS, box_mesh, exterior_faces
from platoanalyze_b200.problem import HelmholtzFilter
from platoanalyze_b200.workloads import splitmix_uniform

pytestmark = pytest.mark.gpu
TOL = 1e-11


def host(t):
    return t.detach().cpu().numpy()


def close(gpu, ref, tol=TOL):
    gpu, ref = np.asarray(gpu, np.float64), np.asarray(ref, np.float64)
    assert rel_l2(gpu, ref) <= tol, rel_l2(gpu, ref)
    assert np.abs(gpu - ref).max() <= tol * max(np.abs(ref).max(), 1e-300)


def jittered_mesh(nx, ny, nz, seed):
    m = box_mesh(nx, ny, nz, 1.3, 0.7, 0.9)
    rng = np.random.default_rng(seed)
    coords = m.coords.copy()
    h = np.array([1.3 / nx, 0.7 / ny, 0.9 / nz])
    interior = np.all((coords > 1e-12) & (coords < np.array([1.3, 0.7, 0.9]) - 1e-12), axis=1)
    coords[interior] += rng.uniform(-0.15, 0.15, (interior.sum(), 3)) * h
    perm = rng.permutation(m.num_nodes).astype(np.int32)
    new = np.empty_like(coords)
    new[perm] = coords
    return new, perm[m.connectivity].astype(np.int32)


@pytest.fixture(scope="module", params=["box", "jittered", "box-surface", "jittered-surface"])
def case(request):
    """(filter, oracle, L, num_nodes, surface): the surface cases carry the surface term on
    the exterior faces outside a symmetry plane at x = 0 (box) or on every exterior face
    (jittered, found by exterior_faces)."""
    if request.param.startswith("box"):
        m = box_mesh(10, 5, 5, 2.0, 1.0, 1.0)
        coords, conn, L = m.coords, m.connectivity, 0.1
        faces = exterior_faces(conn, m.nodeset(X_MINUS))
    else:
        coords, conn = jittered_mesh(7, 5, 4, 5)
        L = 0.13
        faces = exterior_faces(conn)
    surface = (0.6, faces[0], faces[1]) if request.param.endswith("surface") else None
    if surface:
        filt = HelmholtzFilter(coords, conn, L, surface_length_scale=0.6, surface_faces=faces, tolerance=1e-13)
    else:
        filt = HelmholtzFilter(coords, conn, L, tolerance=1e-13)
    orc = Oracle(coords, conn)
    return filt, orc, L, coords.shape[0], surface


def test_pattern_residual_and_matrices(case):
    filt, orc, L, n, S = case
    rm, cols = orc.graph()
    rmg, colsg = (host(t) for t in filt.pattern())
    assert np.array_equal(rmg, rm) and np.array_equal(colsg, cols)
    rng = np.random.default_rng(2)
    f, c = rng.standard_normal(n), splitmix_uniform(n, 3)
    close(host(filt.value(filt.to_dev(f), filt.to_dev(c))), orc.helmholtz_value(L, f, c, surface=S))
    close(host(filt.gradient_u()), orc.helmholtz_gradient_u(L, surface=S))
    close(host(filt.gradient_z()), orc.helmholtz_gradient_z())


def test_solution_and_chain_rule(case):
    filt, orc, L, n, S = case
    control = splitmix_uniform(n, 11)
    f, st = filt.solution(filt.to_dev(control))
    assert st["converged"] == 1 and st["relative_residual"] <= 1e-11
    fo, _ = orc.helmholtz_solution(L, control, tol=1e-14, surface=S)
    assert rel_l2(host(f), fo) <= 1e-10
    w = np.cos(np.arange(n) * 0.41)
    g, st = filt.criterion_gradient(filt.to_dev(w))
    assert st["converged"] == 1
    go, _ = orc.helmholtz_criterion_gradient(L, w, tol=1e-14, surface=S)
    assert rel_l2(host(g), go) <= 1e-10
    # adjoint identity: w . filtered(control) = dfdcontrol . control for a linear filter
    assert abs(w @ host(f) - host(g) @ control) <= 1e-10 * abs(w @ host(f))


def test_uniform_density_is_left_unchanged():
    m = box_mesh(12, 6, 6, 2.0, 1.0, 1.0)
    filt = HelmholtzFilter(m.coords, m.connectivity, 0.1, tolerance=1e-14)
    one = filt.to_dev(np.ones(m.num_nodes))
    assert np.abs(host(filt.value(one, one))).max() <= 1e-15
    f, st = filt.solution(one)
    assert np.abs(host(f) - 1.0).max() <= 1e-12


def test_filter_errors():
    m = box_mesh(2, 2, 2)
    with pytest.raises(capi.PlatoError) as e:
        HelmholtzFilter(m.coords, m.connectivity, -1.0)
    assert e.value.status == capi.BAD_INPUT
    cells, local = exterior_faces(m.connectivity)
    bad = local.copy()
    bad[0, 1] = 4
    with pytest.raises(capi.PlatoError) as e:
        HelmholtzFilter(m.coords, m.connectivity, 0.2, surface_length_scale=1.0, surface_faces=(cells, bad))
    assert e.value.status == capi.BAD_INPUT and "local node" in str(e.value)
    with pytest.raises(capi.PlatoError) as e:
        HelmholtzFilter(m.coords, m.connectivity, 0.2, surface_length_scale=-1.0, surface_faces=(cells, local))
    assert e.value.status == capi.BAD_INPUT
    filt = HelmholtzFilter(m.coords, m.connectivity, 0.2)
    assert filt.num_nodes == m.num_nodes
    # a mechanics handle refuses the filter's calls
    from platoanalyze_b200.problem import EllipticProblem, cantilever_spec

    prob = EllipticProblem(cantilever_spec(m))
    fake = HelmholtzFilter.__new__(HelmholtzFilter)
    fake.h, fake.torch = prob.h, filt.torch
    fake.num_nodes, fake.num_blocks = prob.num_nodes, prob.num_blocks
    try:
        with pytest.raises(capi.PlatoError) as e:
            fake.gradient_z()
        assert e.value.status == capi.BAD_INPUT and "Helmholtz" in str(e.value)
    finally:
        fake.h = None  # the handle belongs to prob
        prob.close()
