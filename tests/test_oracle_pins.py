"""The CPU oracle checked against the reference's own tests and published
numbers (the pin that makes it a trustworthy checker for the GPU path).

Mirrors test/elasticity_test.jl, test/elasticity_split_node_test.jl,
test/fault_response_test.jl and test/bp8_test.jl:27-37, plus the known
answers in tests/golden/reference_known_answers.json.
"""
import json
import os
from fractions import Fraction as Fr

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import sbp
from oracle.operators import Grid3, SplitNodeSystem, elastic_matrix, traction_blocks
from oracle.fault import FaultElasticity, bp8_grids, cube_grids, lame_lambda
from oracle.krylov_cg import CGSolver, krylov_cg, jacobi_preconditioner

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_known_answers.json")))
LAM, MU = 2.0, 1.0


# -- 1D SBP operators ---------------------------------------------------------
@pytest.mark.parametrize("n", [9, 12, 17])
def test_sbp_first_derivative_identity(n):
    w, D1 = sbp.h_weights_rational(n), sbp.d1_rational(n)
    for r in range(n):
        for c in range(n):
            q = w[r] * D1[r][c] + w[c] * D1[c][r]
            want = Fr(-1) if r == c == 0 else Fr(1) if r == c == n - 1 else Fr(0)
            assert q == want


@pytest.mark.parametrize("n", [9, 12, 17])
def test_sbp_second_derivative_compatible(n):
    """H D2 = -M + e_r d_r' - e_l d_l' with M symmetric positive semi-definite
    (src/Elasticity.jl:183-186)."""
    w, D2 = sbp.h_weights_rational(n), sbp.d2_rational(n)
    dl, dr = sbp.boundary_derivative_rational(n, False), sbp.boundary_derivative_rational(n, True)
    M = [[-(w[r] * D2[r][c] - ((1 if r == n - 1 else 0) * dr[c] - (1 if r == 0 else 0) * dl[c]))
          for c in range(n)] for r in range(n)]
    assert all(M[r][c] == M[c][r] for r in range(n) for c in range(n))
    ev = np.linalg.eigvalsh(np.array([[float(x) for x in row] for row in M]))
    assert ev.min() > -1e-12


def test_sbp_orders():
    """Interior order 4, boundary order 2 (test/convergence_test.jl:205-213)."""
    errs = {}
    for n in (101, 201, 401):
        ax = sbp.Axis(n, 1.0 / (n - 1))
        x = np.linspace(0, 1, n)
        f, f1, f2 = np.sin(2 * x + 0.3), 2 * np.cos(2 * x + 0.3), -4 * np.sin(2 * x + 0.3)
        e1 = ax.D1 @ f - f1
        e2 = ax.D2 @ f - f2
        errs[n] = (abs(e1[10:-10]).max(), abs(e1[:4]).max(), abs(e2[10:-10]).max(), abs(e2[:4]).max())
    for k, want in ((0, 3.8), (1, 1.8), (2, 3.8), (3, 1.8)):
        rate = np.log2(errs[101][k] / errs[201][k])
        assert rate > want, (k, rate)


# -- Elasticity ----------------------------------------------------------------
def test_sbp_property_E_T_compatible():
    """test/elasticity_test.jl:56-86."""
    n = 11
    g = Grid3((0, 0, 0), (1, 1, 1), (n, n, n))
    N = g.N
    E = elastic_matrix(g, LAM, MU)
    H = sp.block_diag([g.H()] * 3)
    i = np.arange(1, 3 * N + 1, dtype=float)
    u, v = np.sin(7.0 * i + 1.0), np.cos(3.0 * i + 2.0)
    volume = v @ (H @ (E @ u)) - u @ (H @ (E @ v))
    boundary = 0.0
    for a in range(3):
        for upper in (False, True):
            T = traction_blocks(g, LAM, MU, a, upper)
            e = g.e(a, upper)
            Hb = g.Hb(a)
            s = 1.0 if upper else -1.0
            Tmat = s * sp.bmat(T)
            eb = sp.block_diag([e] * 3)
            Hbb = sp.block_diag([Hb] * 3)
            boundary += (eb @ v) @ (Hbb @ (Tmat @ u)) - (eb @ u) @ (Hbb @ (Tmat @ v))
    scale = max(abs(volume), abs(boundary), 1.0)
    assert abs(volume - boundary) / scale < 1e-12


def test_polynomial_exactness():
    """u = [x, y^2, xz], lambda = mu = 1 -> [2, 6, 0] (test/elasticity_test.jl:88-97)."""
    g = Grid3((0, 0, 0), (1, 1, 1), (21, 21, 21))
    X = [g.coords(a) for a in range(3)]
    x, y, z = np.meshgrid(X[0], X[1], X[2], indexing="ij")
    flat = lambda f: f.flatten(order="F")
    u = np.concatenate([flat(x), flat(y ** 2), flat(x * z)])
    r = elastic_matrix(g, 1.0, 1.0) @ u
    N = g.N
    assert np.allclose(r[:N], 2.0) and np.allclose(r[N:2 * N], 6.0) and np.allclose(r[2 * N:], 0.0, atol=1e-8)


def test_traction_manufactured():
    """test/elasticity_test.jl:116-133 (5 %)."""
    n = 21
    g = Grid3((0, -1, -1), (1, 1, 1), (n, n, n))
    X = [g.coords(a) for a in range(3)]
    x, y, z = np.meshgrid(X[0], X[1], X[2], indexing="ij")
    pi = np.pi
    u1 = np.sin(pi * x) * np.cos(pi * y) * np.cos(pi * z)
    u2 = np.cos(pi * x) * np.sin(pi * y) * np.cos(pi * z)
    u3 = np.cos(pi * x) * np.cos(pi * y) * np.sin(pi * z)
    v = np.concatenate([a.flatten(order="F") for a in (u1, u2, u3)])
    T = traction_blocks(g, LAM, MU, 0, False)
    N = g.N
    tau = [sum(T[i][k] @ v[k * N:(k + 1) * N] for k in range(3)) for i in range(3)]
    yb, zb = np.meshgrid(X[1], X[2], indexing="ij")
    yb, zb = yb.flatten(order="F"), zb.flatten(order="F")
    # grad of ua at x = 0
    J11 = pi * np.cos(0) * np.cos(pi * yb) * np.cos(pi * zb)
    J22 = np.cos(0) * pi * np.cos(pi * yb) * np.cos(pi * zb)
    J33 = np.cos(0) * np.cos(pi * yb) * pi * np.cos(pi * zb)
    J21 = -pi * np.sin(0) * np.sin(pi * yb) * np.cos(pi * zb)
    J12 = -pi * np.sin(0) * np.sin(pi * yb) * np.cos(pi * zb)
    J31 = -pi * np.sin(0) * np.cos(pi * yb) * np.sin(pi * zb)
    J13 = J31
    true = [LAM * (J11 + J22 + J33) + 2 * MU * J11, MU * (J21 + J12), MU * (J31 + J13)]
    for i in range(3):
        scale = max(abs(true[i]).max(), 1.0)
        assert abs(tau[i] - true[i]).max() / scale < 0.05


# -- Split-node system -----------------------------------------------------------
def gauss_slip(x2, x3):
    return (np.exp(-(x2 ** 2 + x3 ** 2) / 0.125), 0.0)


@pytest.fixture(scope="module")
def sys11():
    gm, gp = cube_grids(11)
    return SplitNodeSystem(gm, gp, LAM, MU)


def test_nnz_pins(sys11):
    a = sys11.HP_DSAT.copy()
    a.data[:] = 1
    p = sys11.P.copy()
    p.data[:] = 1
    assert sys11.HP_DSAT.nnz == GOLD["nnz_HP_DSAT"]["n11"]
    assert (a @ p).nnz == GOLD["nnz_A_structural"]["n11"]


def test_nnz_pins_n15():
    gm, gp = cube_grids(15)
    S = SplitNodeSystem(gm, gp, LAM, MU)
    a = S.HP_DSAT.copy()
    a.data[:] = 1
    p = S.P.copy()
    p.data[:] = 1
    assert S.HP_DSAT.nnz == GOLD["nnz_HP_DSAT"]["n15"]
    assert (a @ p).nnz == GOLD["nnz_A_structural"]["n15"]


def test_cg_on_singular_system(sys11):
    """test/elasticity_split_node_test.jl:149-177."""
    S = sys11
    chi = S.build_chi(gauss_slip)
    b = S.HP_DSAT @ chi
    assert np.linalg.norm(b - S.P @ b) / np.linalg.norm(b) < 1e-14
    assert sp.linalg.norm(S.A - S.A.T) / sp.linalg.norm(S.A) < 1e-12
    cg = CGSolver(S.A)
    u = cg.solve(b)
    assert cg.report()["unconverged"] == 0
    assert np.linalg.norm(b - S.A @ u) / np.linalg.norm(b) < 1e-8
    assert np.linalg.norm(u - S.P @ u) / np.linalg.norm(u) < 1e-12


def test_jacobi_facts(sys11):
    """test/elasticity_split_node_test.jl:179-226."""
    S = sys11
    d = S.A.diagonal()
    zero = set(np.nonzero(d == 0)[0].tolist())
    ff = set(np.nonzero(np.diff(S.P.indptr) == 0)[0].tolist())
    assert zero and zero == ff
    assert (d[d != 0] > 0).all()
    M = sp.diags(jacobi_preconditioner(S.A))
    assert sp.linalg.norm(M @ S.P - S.P @ M) / sp.linalg.norm(M @ S.P) < 1e-14
    chi = S.build_chi(gauss_slip)
    b = S.HP_DSAT @ chi
    u0 = CGSolver(S.A).solve(b)
    sj = CGSolver(S.A, precond="jacobi")
    uj = sj.solve(b)
    U0, Uj = S.reconstruct_U(u0, chi), S.reconstruct_U(uj, chi)
    assert sj.report()["unconverged"] == 0 and sj.report()["precond"] == "jacobi"
    assert np.linalg.norm(Uj - U0) / np.linalg.norm(U0) < 1e-8
    with pytest.raises(ValueError):
        CGSolver(S.A, precond="nonsense")


def test_zero_diag_count():
    gm = Grid3((-1, -1, -1), (0, 1, 1), (9, 13, 13))
    gp = Grid3((0, -1, -1), (1, 1, 1), (9, 13, 13))
    S = SplitNodeSystem(gm, gp, LAM, MU)
    d = S.A.diagonal()
    assert S.Ntot == GOLD["zero_diag_A"]["ntot"]
    assert int((d == 0).sum()) == GOLD["zero_diag_A"]["count"]
    chi = S.build_chi(gauss_slip)
    b = S.HP_DSAT @ chi
    assert krylov_cg(S.A, b, 1e-10, Minv=jacobi_preconditioner(S.A))[1] == GOLD["jacobi_iterations_9x13x13"]["jacobi"]


def test_rank_P_A():
    gm, gp = cube_grids(9)
    S = SplitNodeSystem(gm, gp, LAM, MU)
    assert S.Ntot == GOLD["rank_P_A"]["ntot"]
    assert np.linalg.matrix_rank(S.P.toarray()) == GOLD["rank_P_A"]["rank"]
    assert np.linalg.matrix_rank(S.A.toarray()) == GOLD["rank_P_A"]["rank"]


@pytest.mark.parametrize("n", [9, 13])
def test_cg_iteration_counts(n):
    gm, gp = cube_grids(n)
    S = SplitNodeSystem(gm, gp, LAM, MU)
    b = S.HP_DSAT @ S.build_chi(gauss_slip)
    assert krylov_cg(S.A, b, 1e-10)[1] == GOLD["cg_iterations_gaussian_slip"][f"n{n}"]


def _gauss_patch(n):
    gm, gp = cube_grids(n)
    S = SplitNodeSystem(gm, gp, LAM, MU)
    chi = S.build_chi(lambda x2, x3: (np.exp(-(x2 ** 2 + x3 ** 2) / (2 * 0.25 ** 2)), 0.0))
    u = CGSolver(S.A).solve(S.HP_DSAT @ chi)
    U = S.reconstruct_U(u, chi)
    Nm = gm.N
    tm = [sp.hstack(S.Tm[j]) @ U[:3 * Nm] for j in range(3)]
    tp = [sp.hstack(S.Tp[j]) @ U[3 * Nm:] for j in range(3)]
    return S, U, tm, tp


def test_interface_conditions():
    """test/elasticity_split_node_test.jl:127-142."""
    S, U, tm, tp = _gauss_patch(13)
    gm, gp = S.gm, S.gp
    jump = lambda c: np.array([U[3 * gm.N + c * gp.N + ip] - U[c * gm.N + im] for im, ip in S.pairs])
    x2, x3 = gm.coords(1), gm.coords(2)
    n1, n2 = gm.n[0], gm.n[1]
    slip = np.array([np.exp(-(x2[(im // n1) % n2] ** 2 + x3[im // (n1 * n2)] ** 2) / 0.125) for im, _ in S.pairs])
    scale = abs(tm[1]).max()
    assert abs(jump(0)).max() < 1e-10
    assert abs(jump(1) - slip).max() < 1e-10
    assert abs(jump(2)).max() < 1e-10
    assert abs(tp[1] - tm[1]).max() / scale < 1e-10
    assert abs(tp[2] - tm[2]).max() / scale < 1e-10
    assert abs(abs(U).max() - 0.5) <= 1e-8 * 0.5


def test_normal_stress_vanishes_under_refinement():
    _, _, tm11, _ = _gauss_patch(11)
    _, _, tm15, _ = _gauss_patch(15)
    assert abs(tm11[0]).max() < 0.1 * abs(tm11[1]).max()
    assert abs(tm15[0]).max() < abs(tm11[0]).max()


# -- Fault response ------------------------------------------------------------------
@pytest.fixture(scope="module")
def fe13():
    gm, gp = cube_grids(13, L=1.2)
    return FaultElasticity(gm, gp, LAM, MU, l_f=0.6)


def test_boundary_selection_non_cube():
    g = Grid3((-1, -2, -3), (0, 2, 3), (9, 11, 13))
    sel = g.boundary_nodes(0, True)
    n1, n2 = 9, 11
    assert len(sel) == 11 * 13
    i2 = (sel // n1) % n2
    i3 = sel // (n1 * n2)
    assert (sel % n1 == n1 - 1).all()
    assert (i2 == np.tile(np.arange(11), 13)).all() and (i3 == np.repeat(np.arange(13), 11)).all()


def test_omega_endpoints(fe13):
    assert np.isclose(fe13.x2f[0], -0.6) and np.isclose(fe13.x2f[-1], 0.6)
    assert fe13.nf == len(fe13.x2f) * len(fe13.x3f) == 49
    gm, gp = cube_grids(13, L=1.2)
    with pytest.raises(ValueError):
        FaultElasticity(gm, gp, LAM, MU, l_f=0.55)


def test_stiffness_reproduces_direct_solve(fe13):
    nf = fe13.nf
    K = fe13.fault_stiffness()
    k = np.arange(1, nf + 1)
    s2, s3 = 0.01 * np.sin(3 * k), 0.02 * np.cos(2 * k)
    d2, d3 = fe13.shear_traction(s2, s3)
    st = K @ np.concatenate([s2, s3])
    assert np.allclose(st[:nf], d2, rtol=1e-8) and np.allclose(st[nf:], d3, rtol=1e-8)
    assert (np.diag(K) < 0).all()
    d2, _ = fe13.shear_traction(np.ones(nf), np.zeros(nf))
    assert d2.max() < 0
    z2, z3 = fe13.shear_traction(np.zeros(nf), np.zeros(nf))
    assert (z2 == 0).all() and (z3 == 0).all()


def test_toeplitz_approximates_exact():
    gm, gp = cube_grids(11)
    fe = FaultElasticity(gm, gp, LAM, MU, l_f=0.4)
    Ke = fe.fault_stiffness()
    Kt = fe.fault_stiffness_toeplitz()
    nf = fe.nf
    n2, n3 = len(fe.x2f), len(fe.x3f)
    c = ((n3 + 1) // 2 - 1) * n2 + (n2 + 1) // 2 - 1
    assert np.linalg.norm(Kt - Ke) / np.linalg.norm(Ke) < 0.05
    assert np.allclose(Kt[:nf, c], Ke[:nf, c], rtol=1e-6)
    assert np.allclose(Kt[nf:, nf + c], Ke[nf:, nf + c], rtol=1e-6)
    assert (np.diag(Kt)[:nf] < 0).all()
    assert np.isclose(Kt[c, c], Ke[c, c], rtol=1e-6)
    assert not np.isclose(Kt[0, 0], Ke[0, 0], rtol=1e-6)
    assert np.isclose(Kt[0, 0], Ke[0, 0], rtol=0.05)


# -- Production-size known answers (C restatement of the column loop) -------------------
def test_K_self_production():
    mu = 32.04e9
    gm, gp = bp8_grids(50.0, 800.0, 400.0)
    fe = FaultElasticity(gm, gp, lame_lambda(mu, 0.25), mu, 400.0)
    fe.rs.rtol = 1e-12
    ic = int(np.argmin(abs(fe.x2f)) + np.argmin(abs(fe.x3f)) * len(fe.x2f))
    col = fe.fault_stiffness([ic])[:, 0]
    assert f"{col[ic]:.5e}" == "-4.38404e+08"


def test_K_dz100_symmetry_and_diag():
    from oracle.cref import CRefStiffness
    mu = 32.04e9
    gm, gp = bp8_grids(100.0, 800.0, 800.0)
    fe = FaultElasticity(gm, gp, lame_lambda(mu, 0.25), mu, 400.0)
    K, it, ok = CRefStiffness(fe).columns(np.arange(2 * fe.nf))
    assert ok.all()
    assert K.shape == (2 * fe.nf, 2 * fe.nf)
    assert (np.diag(K) < 0).all()
    assert f"{np.diag(K).max():.2e}" == "-2.19e+08"
    asym = 100 * np.linalg.norm(K - K.T) / np.linalg.norm(K)
    assert f"{asym:.4f}" == "0.1827"
    assert np.linalg.norm(K - K.T) / np.linalg.norm(K) < 0.01
