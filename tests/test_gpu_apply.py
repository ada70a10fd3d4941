"""GPU parity of the matrix-free operator against the oracle's assembled
matrices: y = A x and y = HP_DSAT x through the C ABI, FP64 and FP32."""
import numpy as np
import pytest

from oracle.operators import Grid3, SplitNodeSystem

pytestmark = pytest.mark.gpu

# (n1, n2, n3, x1_extent, x2 range, x3 range, lam, mu, l_f)
CASES = [
    (11, 11, 11, 1.0, (-1, 1), (-1, 1), 2.0, 1.0, 0.4),            # reference test cubes
    (9, 13, 13, 1.0, (-1, 1), (-1, 1), 2.0, 1.0, 0.5),             # n1 != n23
    (9, 17, 21, 0.8, (-1.6, 1.6), (-2.0, 2.0), 1.5, 0.7, 0.0),     # unequal spacings per axis
    (12, 10, 9, 1.0, (-1, 1), (-1, 1), 2.0, 1.0, 1.0),             # even n1/n2, shortest axes
    (21, 33, 13, 2.0, (-1, 1), (-1, 1), 2.0, 1.0, 0.5),            # several x2 tiles
    (9, 17, 17, 800.0, (-800, 800), (-800, 800), 32.04e9, 32.04e9, 400.0),  # BP8 scale, h = 100 m
    (33, 17, 13, 800.0, (-400, 400), (-300, 300), 32.04e9, 32.04e9, 200.0),  # n1 = 33 (h = 25 m lines)
]


def oracle_system(c):
    n1, n2, n3, L1, x2, x3, lam, mu, _ = c
    gm = Grid3((-L1, x2[0], x3[0]), (0.0, x2[1], x3[1]), (n1, n2, n3))
    gp = Grid3((0.0, x2[0], x3[0]), (L1, x2[1], x3[1]), (n1, n2, n3))
    return SplitNodeSystem(gm, gp, lam, mu)


def gpu_fe(eqd, c):
    n1, n2, n3, L1, x2, x3, lam, mu, l_f = c
    return eqd.FaultElasticity(eqd.GridPair(n1, n2, n3, L1, x2, x3), lam, mu, l_f)


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}x{c[1]}x{c[2]}")
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 2e-5)])
def test_apply_matches_oracle(eqd, case, precision, tol):
    S = oracle_system(case)
    fe = gpu_fe(eqd, case)
    rng = np.random.default_rng(7)
    X = rng.standard_normal((S.Ntot, 3))
    for mode, M in (("A", S.A), ("HP_DSAT", S.HP_DSAT)):
        Y = eqd.apply_operator(fe, X, mode=mode, precision=precision)
        for j in range(X.shape[1]):
            ref = M @ X[:, j]
            sc = abs(M).dot(abs(X[:, j])).max()
            err = abs(Y[:, j] - ref).max() / sc
            assert err < tol, (mode, j, err)


def test_apply_output_in_range_of_P(eqd):
    """A x lands exactly in range(P): zero far-field rows, equal fault pairs."""
    case = CASES[0]
    S = oracle_system(case)
    fe = gpu_fe(eqd, case)
    x = np.random.default_rng(3).standard_normal(S.Ntot)
    for precision in ("fp64", "mixed"):
        y = eqd.apply_operator(fe, x, mode="A", precision=precision)
        assert np.abs(S.P @ y - y).max() == 0.0


def test_apply_columns_independent(eqd):
    """A column's result does not depend on the other columns of the batch."""
    case = CASES[4]
    S = oracle_system(case)
    fe = gpu_fe(eqd, case)
    X = np.random.default_rng(11).standard_normal((S.Ntot, 4))
    for precision in ("fp64", "mixed"):
        Y = eqd.apply_operator(fe, X, mode="A", precision=precision)
        y2 = eqd.apply_operator(fe, X[:, 2], mode="A", precision=precision)
        assert np.array_equal(Y[:, 2], y2)


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}x{c[1]}x{c[2]}")
@pytest.mark.parametrize("variant", list(range(11)))
def test_cg_path_kernel_every_variant(eqd, case, variant):
    """The kernel the CG iterations run (input already in range(P)), for each
    FP32 launch variant the autotuner may pick, and in FP64."""
    S = oracle_system(case)
    fe = gpu_fe(eqd, case)
    eqd.set_stencil_variant(fe, variant)
    X = S.P @ np.random.default_rng(5).standard_normal((S.Ntot, 2))
    for precision, tol in (("mixed", 2e-5), ("fp64", 1e-12)):
        Y = eqd.apply_operator(fe, X, mode="A_rangeP", precision=precision)
        for j in range(X.shape[1]):
            ref = S.A @ X[:, j]
            err = abs(Y[:, j] - ref).max() / abs(S.A).dot(abs(X[:, j])).max()
            assert err < tol, (precision, j, err)
