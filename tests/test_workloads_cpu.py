"""Synthetic workload generators (CPU): seeded densities, the batched-cantilever draw."""
import numpy as np

from platoanalyze_b200.workloads import BATCH_SIZES, batch_workload, grf_density, splitmix_uniform


def test_splitmix_uniform_is_seeded_and_in_range():
    a = splitmix_uniform(1000, 0x5EED0002)
    assert np.array_equal(a, splitmix_uniform(1000, 0x5EED0002))
    assert a.min() >= 0.01 and a.max() < 1.0
    assert abs(a.mean() - 0.505) < 0.03


def test_grf_density_covariance_and_range():
    z = grf_density(64, 32, 32, rng=np.random.default_rng(1))
    assert z.shape == (65 * 33 * 33,)
    assert z.min() >= 0.01 and z.max() <= 1.0
    f = np.log(z / (1 - z)).reshape(65, 33, 33)  # undo the logistic (nothing clips at this draw)
    h = 2.0 / 64
    for lag in (1, 3, 6):  # correlation exp(-r^2 / (2 * 0.1^2)) along x
        r = lag * h
        c = np.corrcoef(f[:-lag].ravel(), f[lag:].ravel())[0, 1]
        assert abs(c - np.exp(-r * r / 0.02)) < 0.05, (lag, c)


def test_batch_workload_draw():
    specs, zs, ns = batch_workload(count=8, sizes=(4, 6))
    assert len(specs) == len(zs) == len(ns) == 8
    assert set(ns) <= {4, 6}
    for s, z, n in zip(specs, zs, ns):
        assert s.coords.shape[0] == (n + 1) * (n // 2 + 1) ** 2 == z.size
        t = np.asarray(s.tractions[0][2])
        assert abs(np.linalg.norm(t) - 1.0) < 1e-12
    specs2, zs2, ns2 = batch_workload(count=8, sizes=(4, 6))
    assert ns == ns2 and all(np.array_equal(a, b) for a, b in zip(zs, zs2))
    assert BATCH_SIZES == (16, 24, 32, 48, 64)


def test_oracle_side_cantilever_equals_the_product_workload():
    """The reference arm builds its problem without the product library (oracle/workload.py);
    it must be the same problem, array for array."""
    import workload as ow

    from platoanalyze_b200.workloads import cantilever

    for size in ((3, 2, 2), (8, 4, 4), (5, 3, 7)):
        spec = cantilever(*size)
        orc = ow.cantilever_oracle(*size)
        assert np.array_equal(orc.coords, spec.coords)
        assert np.array_equal(orc.conn, spec.connectivity)
        assert np.array_equal(orc.bc_dofs, spec.bc_dofs)
        cells, local, vec = spec.tractions[0]
        assert np.array_equal(orc.fc, cells) and np.array_equal(orc.fl, local)
        assert tuple(vec) == (0.0, -1.0, 0.0)
    assert np.array_equal(ow.splitmix_uniform(4096, 0x5EED0002), splitmix_uniform(4096, 0x5EED0002))
