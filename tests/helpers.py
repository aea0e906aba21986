"""Shared fixtures of the test-suite: golden data, small problems, comparison helpers."""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_golden(name: str = "derivative_tests_3d.json") -> dict:
    return json.loads((GOLDEN / name).read_text())


def teuchos_rel_err(a, b) -> np.ndarray:
    """|a-b| / max(|a|,|b|) elementwise (Teuchos relErr); 0 where both are 0."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.maximum(np.abs(a), np.abs(b))
    num = np.abs(a - b)
    return np.where(den == 0.0, 0.0, num / np.where(den == 0.0, 1.0, den))


def assert_floating_equality(actual, gold, tol, zero_abs=None):
    """TEST_FLOATING_EQUALITY on every entry; gold zeros checked as |actual| < zero_abs."""
    actual = np.asarray(actual, dtype=np.float64).ravel()
    gold = np.asarray(gold, dtype=np.float64).ravel()
    assert actual.shape == gold.shape, (actual.shape, gold.shape)
    if zero_abs is not None:
        zmask = gold == 0.0
        assert np.all(np.abs(actual[zmask]) < zero_abs), np.abs(actual[zmask]).max()
        err = teuchos_rel_err(actual[~zmask], gold[~zmask])
    else:
        err = teuchos_rel_err(actual, gold)
    assert err.size == 0 or err.max() <= tol, f"max rel err {err.max():.3e} > {tol:.1e} at {np.argmax(err)}"


def rel_l2(a, b) -> float:
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def derivative_test_state(num_nodes: int) -> np.ndarray:
    """u_i = 1e-4 * (i + 1), accumulated the way DerivativeTests.cpp builds it."""
    u = np.empty(3 * num_nodes)
    disp = 0.0
    for i in range(u.size):
        disp += 0.0001
        u[i] = disp
    return u
