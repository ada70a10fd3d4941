"""Jacobi preconditioning (`precond=:jacobi`, src/ElasticitySplitNode.jl:352-365)
on the GPU: diag(A) against the oracle's assembled A, preconditioned CG
against the oracle's Krylov-rule CG, and K with Jacobi against the exact K."""
import numpy as np
import pytest

from oracle.fault import FaultElasticity as OracleFE, cube_grids
from oracle.krylov_cg import krylov_cg, jacobi_preconditioner as oracle_jacobi
from oracle.operators import Grid3, SplitNodeSystem
from oracle.cref import CRefStiffness

pytestmark = pytest.mark.gpu

LAM, MU = 2.0, 1.0
CASES = [
    (11, 11, 11, 1.0, (-1, 1), (-1, 1), 2.0, 1.0, 0.4),
    (9, 17, 21, 0.8, (-1.6, 1.6), (-2.0, 2.0), 1.5, 0.7, 0.0),
    (12, 10, 9, 1.0, (-1, 1), (-1, 1), 2.0, 1.0, 1.0),
    (33, 17, 13, 800.0, (-400, 400), (-300, 300), 32.04e9, 32.04e9, 200.0),
]


def oracle_system(c):
    n1, n2, n3, L1, x2, x3, lam, mu, _ = c
    gm = Grid3((-L1, x2[0], x3[0]), (0.0, x2[1], x3[1]), (n1, n2, n3))
    gp = Grid3((0.0, x2[0], x3[0]), (L1, x2[1], x3[1]), (n1, n2, n3))
    return SplitNodeSystem(gm, gp, lam, mu)


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}x{c[1]}x{c[2]}")
def test_diag_matches_assembled_A(eqd, case):
    n1, n2, n3, L1, x2, x3, lam, mu, l_f = case
    S = oracle_system(case)
    fe = eqd.FaultElasticity(eqd.GridPair(n1, n2, n3, L1, x2, x3), lam, mu, l_f)
    d = eqd.operator_diagonal(fe)
    ref = S.A.diagonal()
    assert np.array_equal(d == 0, ref == 0)               # the same zero (far-field) rows
    assert np.abs(d - ref).max() <= 1e-12 * np.abs(ref).max()
    assert np.allclose(eqd.jacobi_preconditioner(fe), oracle_jacobi(S.A), rtol=1e-12, atol=0)


def test_jacobi_cg_matches_oracle(eqd):
    """Preconditioned FP64 CG: iteration count within one of the oracle's
    Krylov-rule PCG, same solution."""
    for n in (9, 13):
        gm, gp = cube_grids(n)
        S = SplitNodeSystem(gm, gp, LAM, MU)
        chi = S.build_chi(lambda x2, x3: (np.exp(-(x2 ** 2 + x3 ** 2) / 0.125), 0.0))
        b = S.HP_DSAT @ chi
        u_ref, it_ref, ok, _ = krylov_cg(S.A, b, 1e-10, Minv=oracle_jacobi(S.A))
        assert ok
        fe = eqd.FaultElasticity(eqd.cube_grids(n), LAM, MU, 0.0, precision="fp64", precond="jacobi")
        u = eqd.split_node_solve(fe.rs, b)
        rep = eqd.solver_report(fe.rs)
        assert rep["precond"] == "jacobi" and rep["unconverged"] == 0
        assert abs(rep["iterations"] - it_ref) <= 1, (rep, it_ref)
        U, U_ref = S.reconstruct_U(u, chi), S.reconstruct_U(u_ref, chi)
        assert np.linalg.norm(U - U_ref) / np.linalg.norm(U_ref) < 1e-8
        assert np.linalg.norm(b - S.A @ u) / np.linalg.norm(b) < 1e-8


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_jacobi_K_matches_exact(eqd, precision):
    gm, gp = cube_grids(11)
    ofe = OracleFE(gm, gp, LAM, MU, l_f=0.4)
    K_ref, _, ok = CRefStiffness(ofe).columns(np.arange(2 * ofe.nf), rtol=1e-13)
    fe = eqd.FaultElasticity(eqd.cube_grids(11), LAM, MU, 0.4, precision=precision, precond="jacobi")
    K = eqd.fault_stiffness(fe)
    assert np.linalg.norm(K - K_ref) / np.linalg.norm(K_ref) < 1e-8
    assert eqd.elastic_solver_report(fe)["unconverged"] == 0
