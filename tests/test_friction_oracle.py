"""The oracle's rate-and-state friction, pinned to the reference's own tests
(test/rate_state_friction_test.jl:21-103, BP8-QD-GS parameters)."""
import math

import numpy as np
import pytest

from oracle.friction import (FrictionParams, NotConverged, aging_law_rhs, fault_strength,
                             initial_state_from_strength, radiation_damping_coefficient, solve_slip_rate,
                             solve_slip_velocity, RHSModel)

A, B, DC, VS, FS = 0.016, 0.010, 0.5e-3, 1e-6, 0.6
SIG0, TAU_INIT, V_INIT = 25.0e6, 14.6e6, 1e-12
P = FrictionParams(A, B, DC, VS, FS)
ETA = radiation_damping_coefficient(32.04e9, 3.464e3)


def test_aging_law_steady_state():
    for V in (1e-12, 1e-9, 1e-6, 1e-3):
        assert abs(aging_law_rhs(V, DC / V, P)) <= 1e-14


def test_strength_increasing():
    Fs = [fault_strength(V, 1e3, SIG0, P) for V in 10.0 ** np.linspace(-12, -2, 20)]
    assert all(np.diff(Fs) > 0)


@pytest.mark.parametrize("eta", [0.0, ETA])
def test_round_trip(eta):
    Vs = (1e-12, 1e-9, 1e-6, 1e-3, 1e-1) if eta == 0.0 else 10.0 ** np.linspace(-12, -2, 15)
    for Vt in Vs:
        T = eta * Vt + fault_strength(Vt, 1e4, SIG0, P)
        assert math.isclose(solve_slip_rate(T, 1e4, SIG0, eta, P), Vt, rel_tol=1e-8)


def test_velocity_direction_and_magnitude():
    tau0, dtau = np.array([3.0e6, -1.5e6]), np.array([0.5e6, 2.0e6])
    V = solve_slip_velocity(tau0, dtau, 1e4, SIG0, ETA, P)
    Tv = tau0 + dtau
    assert np.allclose(V / np.linalg.norm(V), Tv / np.linalg.norm(Tv), rtol=1e-10)
    assert math.isclose(np.linalg.norm(V), solve_slip_rate(np.linalg.norm(Tv), 1e4, SIG0, ETA, P), rel_tol=1e-10)


def test_initial_state():
    th = initial_state_from_strength(V_INIT, TAU_INIT, SIG0, P)
    assert th > 0 and math.isclose(fault_strength(V_INIT, th, SIG0, P), TAU_INIT, rel_tol=1e-10)


def test_seeded_far_below_root():
    for Vt in (1e-1, 1.0, 10.0, 100.0):
        for sig in (25.0e6, 10.0e6, 1.0e6):
            th = DC / Vt
            T = ETA * Vt + fault_strength(Vt, th, sig, P)
            assert math.isclose(solve_slip_rate(T, th, sig, ETA, P), Vt, rel_tol=1e-8)
            assert math.isclose(solve_slip_rate(T, th, sig, ETA, P, V0=1e-8 * Vt), Vt, rel_tol=1e-8)


def test_non_convergence_raises():
    th = DC / 1e-6
    T = ETA * 1e-6 + fault_strength(1e-6, th, SIG0, P)
    with pytest.raises(NotConverged):
        solve_slip_rate(T, th, SIG0, ETA, P, V0=1e-20, maxiter=1)


def test_zero_stress_zero_velocity():
    assert (solve_slip_velocity([0.0, 0.0], [0.0, 0.0], 1e4, SIG0, ETA, P) == 0).all()


def test_rhs_model_at_initial_state_is_steady():
    """At BP8's initial state (zero slip, zero pressure, theta from eq. 28-29)
    the slip rate is V_init along tau0 and the state rate is zero up to the
    damping term (src/BP8.jl:333-345)."""
    import scipy.sparse as sp
    nf = 4
    K = np.zeros((2 * nf, 2 * nf))
    Vvec = np.array([V_INIT, 1e-20])
    tau0 = TAU_INIT * Vvec / np.linalg.norm(Vvec)
    th0 = initial_state_from_strength(np.linalg.norm(Vvec), TAU_INIT - ETA * np.linalg.norm(Vvec), SIG0, P)
    m = RHSModel(K, sp.csr_matrix((nf, nf)), None, None, P, SIG0, 1e3, ETA, tau0)
    u = np.zeros(4 * nf)
    u[2 * nf:3 * nf] = math.log(th0)
    du = m.rhs(u, 0.0)
    assert np.allclose(du[:nf], V_INIT, rtol=1e-9)
    assert np.allclose(du[2 * nf:3 * nf], 1.0 / th0 - np.linalg.norm(Vvec) / DC, atol=1e-12 / th0)
