"""The ring-march FP32 stencil (launch variants 9 and 10 on the BP8 lines
n1 = 9, 21, 33) against the oracle: the operator, whole K builds, batch
independence, and its bounded-wait failure path."""
import ctypes as C

import numpy as np
import pytest

from oracle.cref import CRefStiffness
from oracle.fault import FaultElasticity as OracleFE, bp8_grids, lame_lambda
from oracle.operators import Grid3, SplitNodeSystem

pytestmark = pytest.mark.gpu

RING_VARIANTS = (9, 10)
MU = 32.04e9
K_TOL = 1e-8
# (n1, n2, n3, x1_extent, x2 range, x3 range, lam, mu, l_f): grids the ring
# variants run on (n1 in {9, 21, 33}, n2 >= 14)
CASES = [
    (9, 17, 21, 0.8, (-1.6, 1.6), (-2.0, 2.0), 1.5, 0.7, 0.0),       # unequal spacings, n3 != n2
    (9, 14, 9, 1.0, (-1, 1), (-1, 1), 2.0, 1.0, 1.0),                # two edge tiles only, shortest x3
    (21, 33, 13, 2.0, (-1, 1), (-1, 1), 2.0, 1.0, 0.5),              # middle tiles
    (21, 81, 21, 400.0, (-800, 800), (-200, 200), MU, MU, 200.0),    # h = 20 m lines, BP8 units
    (33, 17, 13, 800.0, (-400, 400), (-300, 300), MU, MU, 200.0),    # n1 = 33 (h = 25 m lines)
]


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def oracle_system(c):
    n1, n2, n3, L1, x2, x3, lam, mu, _ = c
    gm = Grid3((-L1, x2[0], x3[0]), (0.0, x2[1], x3[1]), (n1, n2, n3))
    gp = Grid3((0.0, x2[0], x3[0]), (L1, x2[1], x3[1]), (n1, n2, n3))
    return SplitNodeSystem(gm, gp, lam, mu)


def gpu_fe(eqd, c, **kw):
    n1, n2, n3, L1, x2, x3, lam, mu, l_f = c
    return eqd.FaultElasticity(eqd.GridPair(n1, n2, n3, L1, x2, x3), lam, mu, l_f, **kw)


def is_ring(eqd, fe, variant):
    """The variant's reported CTA size is the ring kernel's (a variant falls
    back to the generic plane march on grids the ring kernel does not cover)."""
    n1 = fe.grids.n1
    t2 = 7
    r32 = lambda x: (x + 31) // 32 * 32
    _, table = eqd.autotune(fe, 4)
    return table[variant][1] == 2 * r32(t2 * n1) + r32(2 * t2)


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}x{c[1]}x{c[2]}")
@pytest.mark.parametrize("variant", RING_VARIANTS)
def test_ring_operator_matches_oracle(eqd, case, variant):
    """y = A x for x in range(P) (the CG iterations' kernel), FP32 against
    the assembled FP64 A, relative to |A||x| (same bound as the other FP32
    variants)."""
    S = oracle_system(case)
    fe = gpu_fe(eqd, case)
    assert is_ring(eqd, fe, variant)
    eqd.set_stencil_variant(fe, variant)
    X = S.P @ np.random.default_rng(5).standard_normal((S.Ntot, 3))
    Y = eqd.apply_operator(fe, X, mode="A_rangeP", precision="mixed")
    for j in range(X.shape[1]):
        ref = S.A @ X[:, j]
        err = abs(Y[:, j] - ref).max() / abs(S.A).dot(abs(X[:, j])).max()
        assert err < 2e-5, (j, err)
    # exactly in range(P): far-field rows zero, fault pairs equal
    assert np.abs(S.P @ Y - Y).max() == 0.0


@pytest.mark.parametrize("variant", RING_VARIANTS)
def test_ring_columns_independent(eqd, variant):
    """A column's output does not depend on the other columns of the launch."""
    case = CASES[2]
    S = oracle_system(case)
    fe = gpu_fe(eqd, case)
    eqd.set_stencil_variant(fe, variant)
    X = S.P @ np.random.default_rng(11).standard_normal((S.Ntot, 5))
    Y = eqd.apply_operator(fe, X, mode="A_rangeP", precision="mixed")
    y3 = eqd.apply_operator(fe, X[:, 3], mode="A_rangeP", precision="mixed")
    assert np.array_equal(Y[:, 3], y3)


@pytest.fixture(scope="module")
def bp8_h100(eqd):
    """The reference's BP8 test model grid (17 x 17 x 9 per side, h = 100 m)
    with Omega_f = the whole fault plane: 578 columns, oracle at rtol 1e-13."""
    gm, gp = bp8_grids(100.0, 800.0, 800.0)
    ofe = OracleFE(gm, gp, lame_lambda(MU, 0.25), MU, 800.0)
    K_ref, _, ok = CRefStiffness(ofe).columns(np.arange(2 * ofe.nf), rtol=1e-13)
    assert ok.all()
    return K_ref


@pytest.mark.parametrize("variant", RING_VARIANTS)
def test_ring_K_matches_oracle(eqd, bp8_h100, variant):
    """The whole mixed-precision K (578 columns, BP8 units) with the ring
    kernel in the CG iterations, against the FP64 oracle: relative Frobenius
    and max-entry error <= 1e-8."""
    K_ref = bp8_h100
    fe = eqd.FaultElasticity(eqd.bp8_grids(100.0, 800.0, 800.0), lame_lambda(MU, 0.25), MU, 800.0,
                             precision="mixed", variant=variant + 1, itmax=5000)
    K = eqd.fault_stiffness(fe)
    assert rel(K, K_ref) < K_TOL
    assert abs(K - K_ref).max() / abs(K_ref).max() < K_TOL
    assert eqd.elastic_solver_report(fe)["unconverged"] == 0


@pytest.mark.parametrize("variant", RING_VARIANTS)
def test_ring_batched_equals_single(eqd, variant):
    """With the ring kernel, a K column built in a batch (two overlapping
    halves, slots refilled) is bit-identical to the same column alone."""
    fe = eqd.FaultElasticity(eqd.bp8_grids(100.0, 800.0, 800.0), lame_lambda(MU, 0.25), MU, 800.0,
                             precision="mixed", variant=variant + 1, itmax=5000)
    cols = np.arange(0, 2 * fe.nf, 3)
    Kb, itb, _ = eqd.stiffness_columns(fe, cols)
    for j in (0, 40, len(cols) - 1):
        K1, it1, _ = eqd.stiffness_columns(fe, [cols[j]])
        assert np.array_equal(K1[:, 0], Kb[:, j]) and it1[0] == itb[j]


def test_variant_option_is_per_call(eqd):
    """CGSolver(variant=k + 1) runs variant k for that call only; the grid's
    own selection is unchanged afterwards."""
    g = eqd.bp8_grids(100.0, 800.0, 800.0)
    lam = lame_lambda(MU, 0.25)
    fe = eqd.FaultElasticity(g, lam, MU, 800.0, precision="mixed")
    eqd.set_stencil_variant(fe, 1)
    cols = np.array([100, 144, 400])
    K_ring = eqd.stiffness_columns(fe, cols, solver=eqd.CGSolver(fe, variant=RING_VARIANTS[0] + 1))[0]
    K_pin = eqd.stiffness_columns(fe, cols)[0]
    fe2 = eqd.FaultElasticity(g, lam, MU, 800.0, precision="mixed")
    eqd.set_stencil_variant(fe2, RING_VARIANTS[0])
    assert np.array_equal(K_ring, eqd.stiffness_columns(fe2, cols)[0])
    fe3 = eqd.FaultElasticity(g, lam, MU, 800.0, precision="mixed")
    eqd.set_stencil_variant(fe3, 1)
    assert np.array_equal(K_pin, eqd.stiffness_columns(fe3, cols)[0])
    with pytest.raises(ValueError):
        eqd.stiffness_columns(fe, cols, solver=eqd.CGSolver(fe, variant=99))


def test_ring_wait_timeout_returns_error_and_recovers(eqd):
    """Failure path of the bounded waits: one launch whose copy of an x3
    plane is never issued. Its waits give up after a short poll limit, the
    kernel drains its other copies and returns, the call reports
    EQD_ERR_TIMEOUT, and the next call on the same grid gives the right
    result."""
    case = CASES[2]
    S = oracle_system(case)
    fe = gpu_fe(eqd, case)
    eqd.set_stencil_variant(fe, RING_VARIANTS[0])
    lib = eqd._abi.lib()
    X = S.P @ np.random.default_rng(2).standard_normal((S.Ntot, 2))
    good = eqd.apply_operator(fe, X, mode="A_rangeP", precision="mixed")
    eqd._abi.check(lib.eqd_test_inject_wait_timeout(fe.handle, C.c_int32(6), C.c_uint32(1 << 12)))
    with pytest.raises(eqd.EqdError) as e:
        eqd.apply_operator(fe, X, mode="A_rangeP", precision="mixed")
    assert e.value.code == eqd._abi.EQD_ERR_TIMEOUT
    again = eqd.apply_operator(fe, X, mode="A_rangeP", precision="mixed")
    assert np.array_equal(again, good)
    # the hook only applies to ring variants
    eqd.set_stencil_variant(fe, 1)
    rc = lib.eqd_test_inject_wait_timeout(fe.handle, C.c_int32(6), C.c_uint32(1 << 12))
    assert rc == eqd._abi.EQD_ERR_UNSUPPORTED
