"""Kernels and data of the NLML Hessian checks: the reference's own cases
(src/gpr/tests.rs:1394-1493: an RBF, RBF × Constant, a nested composite,
distance and ARD leaves in one nested tree; noise variance 0.16) plus a
periodic product and a larger seeded ARD case.  Nodes are (kind, arg) pairs in
prefix order: Sum 1, Product 2, Rbf 10, RbfArd 11 (arg = d), Constant 12,
Periodic 13; params are log θ depth-first, then log σn².
"""

import math

import numpy as np

LN = math.log
NOISE = LN(0.16)


def col(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).T).reshape(-1)


def _rows(flat, d):
    return np.asarray(flat, dtype=np.float64).reshape(-1, d)


def reference_cases():
    """(name, nodes, params, x (n × d), y)"""
    x3 = _rows([0.0, 0.8, 1.7], 1)
    y3 = np.array([0.4, -0.2, 0.9])
    x4 = _rows([0.0, 0.8, 1.7, 2.1], 1)
    y4 = np.array([0.4, -0.2, 0.9, 0.1])
    xm = _rows([0.0, 0.8, 1.7, 2.1, 0.3, -0.4, 0.9, 1.2], 2)
    return [
        ("rbf", [[10, 0]], [LN(1.25), NOISE], x3, y3),
        ("rbf_x_constant", [[2, 2], [10, 0], [12, 0]], [LN(1.25), LN(1.4), NOISE], x3, y3),
        ("nested", [[1, 2], [2, 2], [10, 0], [1, 2], [2, 2], [10, 0], [12, 0], [12, 0], [10, 0]],
         [LN(1.25), LN(0.7), LN(1.3), LN(0.4), LN(2.0), NOISE], x4, y4),
        ("nested_mixed", [[2, 2], [1, 2], [10, 0], [11, 2], [1, 2], [2, 2], [12, 0], [10, 0], [12, 0]],
         [LN(1.1), LN(0.9), LN(1.4), LN(1.5), LN(2.0), LN(0.5), NOISE], xm, y4),
    ]


def periodic_case(n=7, seed=3):
    rs = np.random.RandomState(seed)
    x = rs.uniform(0, 3, size=(n, 1))
    y = np.sin(2 * x[:, 0]) + 0.1 * rs.standard_normal(n)
    nodes = [[1, 2], [2, 2], [13, 0], [12, 0], [10, 0]]  # Periodic × Constant + Rbf
    return ("periodic", nodes, [LN(0.8), LN(1.3), LN(0.9), LN(1.7), NOISE], x, y)


def ard_case(n, d=3, seed=5):
    rs = np.random.RandomState(seed)
    x = rs.uniform(0, 4, size=(n, d))
    y = np.sin(x[:, 0]) + 0.3 * np.cos(2 * x[:, 1]) + 0.1 * rs.standard_normal(n)
    # C × ARD + Rbf × C (a periodic leaf on a distance in d > 1 is not
    # positive definite in general, so it stays in the 1-d case)
    nodes = [[1, 2], [2, 2], [12, 0], [11, d], [2, 2], [10, 0], [12, 0]]
    ls = [(0.9, 1.4, 2.2)[f % 3] * (1.0 + 0.5 * (f // 3)) for f in range(d)]
    params = [LN(1.2)] + [LN(v) for v in ls] + [LN(2.5), LN(0.3), LN(0.05)]
    return ("ard%d" % n if d == 3 else "ard%d_d%d" % (n, d), nodes, params, x, y)
