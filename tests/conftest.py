"""Shared fixtures and structure generators for the test suite.

Structures follow the seeded generator of the reference's
benchmarks/bench_force.py:152-158: n^3 cubic cells of a fractional basis,
Gaussian displacements from numpy.random.default_rng(seed).
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running")


DIAMOND = [[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0],
           [0.25, 0.25, 0.25], [0.25, 0.75, 0.75], [0.75, 0.25, 0.75],
           [0.75, 0.75, 0.25]]
FCC = [[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0]]

TERSOFF_SI = {"A": 1830.8, "B": 471.18, "lambda1": 2.4799, "lambda2": 1.7322,
              "lambda3": 0.0, "beta": 1.1e-6, "n": 0.78734, "c": 100390.0,
              "d": 16.217, "h": -0.59825, "R": 2.85, "D": 0.15}
SW_SI = {"epsilon": 2.1683, "sigma": 2.0951, "a": 1.80, "gamma": 1.20,
         "lambda": 21.0, "A": 7.049556277, "B": 0.6022245584, "p": 4.0,
         "q": 0.0, "costheta0": -1 / 3}
TERSOFF_XY = [
    {"i": "X", "j": "Y", "k": "Y", "A": 1830.8, "B": 471.18, "lambda1": 2.4799,
     "lambda2": 1.7322, "R": 2.85, "D": 0.15, "beta": 1.1e-6, "n": 0.78734,
     "c": 100390.0, "d": 16.217, "h": -0.59825, "lambda3": 1.7322},
    {"i": "Y", "j": "X", "k": "X", "A": 1500.0, "B": 400.0, "lambda1": 2.2,
     "lambda2": 1.5, "R": 2.85, "D": 0.15, "beta": 0.9e-6, "n": 0.7,
     "c": 90000.0, "d": 14.0, "h": -0.55, "lambda3": 1.5},
]
_TOMITA_KEYS = ("i", "j", "k", "sigma", "a", "lambda", "gamma", "A", "B", "p", "q")
_TOMITA_ROWS = [
    ("Ge", "Ge", "Ge", 2.181, 1.8110, 32.101, 1.1718, 10.093, 0.6862, 4.6973, 0.6588),
    ("Sn", "Sn", "Sn", 2.503, 1.7825, 28.747, 1.1610, 9.4315, 0.7012, 4.9827, 0.6252),
    ("Ge", "Ge", "Sn", 2.337, 1.7988, 29.858, 1.8136, 0.0, 0.0, 0.0, 0.0),
    ("Ge", "Sn", "Ge", 2.337, 1.7988, 29.858, 0.7232, 0.0, 0.0, 0.0, 0.0),
    ("Ge", "Sn", "Sn", 2.337, 1.7988, 24.460, 1.1484, 9.8864, 0.7021, 4.8537, 0.6482),
    ("Sn", "Ge", "Ge", 2.337, 1.7988, 24.460, 1.1484, 9.8864, 0.7021, 4.8537, 0.6482),
    ("Sn", "Ge", "Sn", 2.337, 1.7988, 26.074, 1.3564, 0.0, 0.0, 0.0, 0.0),
    ("Sn", "Sn", "Ge", 2.337, 1.7988, 26.074, 1.0924, 0.0, 0.0, 0.0, 0.0),
]
SW_GESN = [dict(zip(_TOMITA_KEYS, r), epsilon=1.0, costheta0=-0.333333)
           for r in _TOMITA_ROWS]


def nested_records(recs):
    out = {}
    for rec in recs:
        rec = dict(rec)
        out[(rec.pop("i"), rec.pop("j"), rec.pop("k"))] = rec
    return out


def cubic(basis, a, n, types, rattle=0.05, seed=0):
    rng = np.random.default_rng(seed)
    cells = np.array([[i, j, k] for i in range(n) for j in range(n) for k in range(n)])
    frac = (np.asarray(basis, float)[None] + cells[:, None]).reshape(-1, 3)
    pos = frac * a + rng.normal(0.0, rattle, frac.shape)
    return np.eye(3) * a * n, pos, list(types) * len(cells)


def strained(lat, pos, amp, seed):
    rng = np.random.default_rng(seed)
    e = rng.uniform(-amp, amp, (3, 3))
    e = 0.5 * (e + e.T)
    M = np.eye(3) + e
    return lat @ M, pos @ M


_golden_cache = {}


def golden(name):
    if name not in _golden_cache:
        with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
            _golden_cache[name] = {k: z[k] for k in z.files}
    return _golden_cache[name]


def has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cuda_device():
    if not has_cuda():
        pytest.skip("no CUDA device")
    import torch
    return torch.device("cuda:0")
