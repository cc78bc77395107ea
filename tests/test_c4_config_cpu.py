"""The literal C4 configuration has no GP prior draw: gprx's periodic kernel
takes the Euclidean distance (src/kernel/periodic.rs:604-611), and in 3-d the
matrix K + 0.1 I of RbfKernel(1) + PeriodicKernel(1, p) with p in [0.5, 2] on
x in [0, 5]³ is indefinite, so the Cholesky of the oracle (and of the
reference) fails; with the periods of the batched benchmark ([10, 20]) the
same problems factor.  The problems follow the benchmark's seeded generator
(sizes log-uniform in [32, 1024]; of its first 40 problems the first 12 with
n ≤ 300).
"""

import math

import numpy as np

import bench
import oracle_lib as O

NODES = [[1, 2], [10, 0], [13, 0]]


def problems(first=40, count=4096, seed=3):
    """The batched benchmark's first problems, drawn as it draws them: the
    sizes of all problems, their periods, then per problem x and the normals
    of its prior draw."""
    rng = bench.SynthRng(seed)
    u = rng.unit(count)
    sizes = np.floor(np.exp(math.log(32) + u * (math.log(1024) - math.log(32)))).astype(int)
    rng.unit(count)  # the periods
    out = []
    for n in sizes[:first]:
        x = 5.0 * rng.unit(int(n) * 3)
        rng.normal(int(n))
        out.append((int(n), x))
    return out


def test_literal_c4_periods_do_not_factor_and_the_benchmark_periods_do():
    rs = np.random.RandomState(0)
    small = [(n, x) for n, x in problems() if n <= 300][:12]
    assert len(small) >= 6
    for n, x in small:
        y = rs.standard_normal(n)
        for per in (0.5, 1.0, 2.0):
            params = np.array([0.0, 0.0, math.log(per), math.log(0.1)])
            try:
                O.exact_eval(NODES, params, x, n, 3, y, grad=False)
                raise AssertionError("the literal C4 kernel factored at n=%d, p=%g" % (n, per))
            except O.OracleError:
                pass
        for per in (10.0, 20.0):
            params = np.array([0.0, 0.0, math.log(per), math.log(0.1)])
            O.exact_eval(NODES, params, x, n, 3, y, grad=False)
