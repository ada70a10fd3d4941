"""The time loop's right-hand side on the GPU (`eqd_rhs_*`, `eqd_friction_solve`)
against the oracle's restatement of src/RateStateFriction.jl and
src/BP8.jl:356-433, and the reference's own friction round-trip tests
(test/rate_state_friction_test.jl)."""
import math

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import friction as of

pytestmark = pytest.mark.gpu

A, B, DC, VS, FS = 0.016, 0.010, 0.5e-3, 1e-6, 0.6
SIG0 = 25.0e6
ETA = of.radiation_damping_coefficient(32.04e9, 3.464e3)
OP = of.FrictionParams(A, B, DC, VS, FS)


def test_friction_round_trips(eqd):
    fp = eqd.FrictionParams(A, B, DC, VS, FS)
    Vt = np.concatenate([10.0 ** np.linspace(-12, -2, 15), [1e-1, 1.0, 10.0, 100.0]])
    sig = np.full(Vt.size, SIG0)
    th = np.where(Vt >= 1e-1, DC / Vt, 1e4)
    T = np.array([ETA * v + of.fault_strength(v, t, SIG0, OP) for v, t in zip(Vt, th)])
    V = eqd.friction_solve(T, th, sig, ETA, fp)
    assert np.allclose(V, Vt, rtol=1e-8)
    V2 = eqd.friction_solve(T, th, sig, ETA, fp, V0=1e-8 * Vt)      # seeded far below the root
    assert np.allclose(V2, Vt, rtol=1e-8)
    T0 = np.array([of.fault_strength(v, 1e4, SIG0, OP) for v in Vt[:15]])
    assert np.allclose(eqd.friction_solve(T0, np.full(15, 1e4), sig[:15], 0.0, fp), Vt[:15], rtol=1e-8)
    # the same iterates as the oracle's scalar Newton
    ref = [of.solve_slip_rate(t, h, SIG0, ETA, OP) for t, h in zip(T, th)]
    assert np.allclose(V, ref, rtol=1e-13)


def test_friction_non_convergence_is_an_error(eqd):
    fp = eqd.FrictionParams(A, B, DC, VS, FS)
    th = DC / 1e-6
    T = ETA * 1e-6 + of.fault_strength(1e-6, th, SIG0, OP)
    with pytest.raises(eqd.EqdError) as e:
        eqd.friction_solve([T], [th], [SIG0], ETA, fp, V0=[1e-20], maxiter=1)
    assert e.value.code == eqd._abi.EQD_ERR_NOT_CONVERGED


def _model(nf_side=9, seed=0):
    rng = np.random.default_rng(seed)
    nf = nf_side * nf_side
    M = rng.standard_normal((2 * nf, 2 * nf))
    K = -(M @ M.T) / (2 * nf) * 2e8 - 4e8 * np.eye(2 * nf)    # stiffness-like: negative diagonal, Pa/m
    e = np.ones(nf_side)
    L1 = sp.diags([e[:-1], -2 * e, e[:-1]], [-1, 0, 1]).tolil()
    L1[0, 0] = L1[-1, -1] = -1.0                                 # zero-flux ends
    Ap = 0.05 / 100.0 ** 2 * (sp.kron(sp.eye(nf_side), L1) + sp.kron(L1, sp.eye(nf_side))).tocsr()
    x = np.linspace(-400, 400, nf_side)
    X2, X3 = np.meshgrid(x, x, indexing="ij")
    src = (np.exp(-(X2 ** 2 + X3 ** 2) / (2 * 50.0 ** 2)) / (2 * np.pi * 50.0 ** 2)).T.ravel()
    act = np.ones(nf, bool)
    act[[0, nf_side - 1, nf - nf_side, nf - 1]] = False
    return K, Ap, src, act


@pytest.mark.parametrize("injection", ["gaussian", "peaceman"])
def test_rhs_matches_oracle(eqd, injection):
    K, Ap, src, act = _model()
    nf = K.shape[0] // 2
    Vvec = np.array([1e-12, 1e-20])
    tau0 = 14.6e6 * Vvec / np.linalg.norm(Vvec)
    th0 = of.initial_state_from_strength(np.linalg.norm(Vvec), 14.6e6 - ETA * np.linalg.norm(Vvec), SIG0, OP)
    kw = dict(q0=0.003, beta=1e-8, phi=0.1, t_off=360000.0)
    if injection == "peaceman":
        kw.update(well_cell=nf // 2, WI=1e-11, S_e=1e-9, S_well=1e-7, Q0=0.003)
    om = of.RHSModel(K, Ap, src, act, OP, SIG0, 1e3, ETA, tau0, injection=injection, **kw)
    gpu = eqd.BP8Rhs(K, Ap, eqd.FrictionParams(A, B, DC, VS, FS), SIG0, 1e3, ETA, tau0, source=src, active=act,
                     injection=injection, **kw)
    rng = np.random.default_rng(3)
    n = 4 * nf + (1 if injection == "peaceman" else 0)
    for step, t in enumerate((0.0, 1000.0, 400000.0)):
        u = np.zeros(n)
        u[:2 * nf] = rng.standard_normal(2 * nf) * 1e-3 * (step + 1)
        u[2 * nf:3 * nf] = math.log(th0) + rng.standard_normal(nf) * 0.5
        u[3 * nf:4 * nf] = rng.uniform(0, 1e7, nf)
        u[3 * nf + 5] = 25.5e6                                    # one node past the floor
        if injection == "peaceman":
            u[4 * nf] = 2e7
        du_ref = om.rhs(u, t)
        du = gpu(u, t)
        scale = np.maximum(np.abs(du_ref), 1e-300)
        assert np.all(np.abs(du - du_ref) <= 1e-9 * scale + 1e-300), (step, np.max(np.abs(du - du_ref) / scale))
        tau, vp = gpu.fields()
        assert np.allclose(tau, om.tau, rtol=1e-12)
        assert np.allclose(vp, om.Vprev, rtol=1e-9)
    rep = gpu.report()
    assert rep["floor_hits"] == om.floor_hits and rep["floor_nodes"] == 1
    assert rep["sigma_lowest"] == SIG0 - 25.5e6
