"""Rate-and-state friction and the coupled BP8 right-hand side (CPU oracle).

TEST INFRASTRUCTURE: the oracle. Only tests, the smoke check and the
benchmark's CPU-baseline leg use it.

Restates, in numpy, `src/RateStateFriction.jl` (friction coefficient :37-40,
fault strength :47, aging law :54, `solve_slip_rate` :77-100 -- Newton in
x = ln V with steps clamped to +-maxstep, stop when |dx| < tol, error after
maxiter -- `solve_slip_velocity` :109-117, `initial_state_from_strength`
:128-131) and the right-hand side `evaluate!`/`rhs!` of `src/BP8.jl:356-433`
with a caller-supplied pore-pressure operator Ap (the reference builds it
from Diffinitive's 2D SBP Laplacian with Neumann SATs; here it is an input).
"""
import math

import numpy as np


class FrictionParams:
    """`FrictionParams(a, b, Dc, V_star, f_star)` (src/RateStateFriction.jl:18-24)."""

    def __init__(self, a, b, Dc, V_star, f_star):
        self.a, self.b, self.Dc, self.V_star, self.f_star = float(a), float(b), float(Dc), float(V_star), float(f_star)


def radiation_damping_coefficient(mu, c_s):
    return mu / (2.0 * c_s)


def friction_coefficient(V, theta, p):
    return p.a * math.asinh(V / (2 * p.V_star) * math.exp((p.f_star + p.b * math.log(p.V_star * theta / p.Dc)) / p.a))


def fault_strength(V, theta, sigma, p):
    return sigma * friction_coefficient(V, theta, p)


def aging_law_rhs(V, theta, p):
    return 1.0 - V * theta / p.Dc


class NotConverged(RuntimeError):
    pass


def solve_slip_rate(T, theta, sigma, eta, p, V0=None, tol=1e-12, maxiter=50, maxstep=5.0):
    C = math.exp((p.f_star + p.b * math.log(p.V_star * theta / p.Dc)) / p.a)
    x = math.log(p.V_star if V0 is None else V0)
    for _ in range(maxiter):
        V = math.exp(x)
        u = V / (2 * p.V_star) * C
        g = eta * V + sigma * p.a * math.asinh(u) - T
        dg = eta * V + sigma * p.a * u / math.sqrt(1 + u * u)
        dx = min(max(-g / dg, -maxstep), maxstep)
        x += dx
        if abs(dx) < tol:
            return math.exp(x)
    raise NotConverged(f"solve_slip_rate failed to converge in {maxiter} iterations (T={T}, theta={theta})")


def solve_slip_velocity(tau0, dtau, theta, sigma, eta, p, **kw):
    Tv = np.asarray(tau0, dtype=float) + np.asarray(dtau, dtype=float)
    T = float(np.linalg.norm(Tv))
    if T == 0.0:
        return np.zeros(2)
    return solve_slip_rate(T, theta, sigma, eta, p, **kw) * Tv / T


def initial_state_from_strength(V, F_target, sigma, p):
    f = F_target / sigma
    return (p.Dc / p.V_star) * math.exp((p.a * math.log(2 * p.V_star * math.sinh(f / p.a) / V) - p.f_star) / p.b)


class RHSModel:
    """The pieces of `BP8Model` the right-hand side reads (src/BP8.jl:130-146),
    with the reference's cache (Vprev starts at 1e-12, :120-121)."""

    def __init__(self, K, Ap, source, active, fp, sigma0, sigma_min, eta, tau0, q0=0.0, beta=1.0, phi=1.0,
                 t_off=0.0, injection="gaussian", well_cell=0, WI=0.0, S_e=1.0, S_well=1.0, Q0=0.0):
        self.K, self.Ap = np.asarray(K), Ap
        self.nf = K.shape[0] // 2
        self.source = np.zeros(self.nf) if source is None else np.asarray(source, dtype=float)
        self.active = np.ones(self.nf, bool) if active is None else np.asarray(active, bool)
        self.fp, self.sigma0, self.sigma_min, self.eta = fp, sigma0, sigma_min, eta
        self.tau0 = np.asarray(tau0, dtype=float)
        self.q0, self.beta, self.phi, self.t_off = q0, beta, phi, t_off
        self.injection, self.well_cell, self.WI, self.S_e, self.S_well, self.Q0 = \
            injection, well_cell, WI, S_e, S_well, Q0
        self.Vprev = np.full(self.nf, 1e-12)
        self.tau = np.zeros(2 * self.nf)
        self.floor_hits = 0

    def rhs(self, u, t, tol=1e-12, maxiter=50, maxstep=5.0):
        nf = self.nf
        slip, ph, pres = u[:2 * nf], u[2 * nf:3 * nf], u[3 * nf:4 * nf]
        dtau = self.K @ slip
        du = np.zeros_like(u)
        for i in range(nf):
            V = np.zeros(2)
            if self.active[i]:
                sraw = self.sigma0 - pres[i]
                if sraw < self.sigma_min:
                    self.floor_hits += 1
                sigma = max(sraw, self.sigma_min)
                V = solve_slip_velocity(self.tau0, (dtau[i], dtau[nf + i]), math.exp(ph[i]), sigma, self.eta,
                                        self.fp, V0=self.Vprev[i], tol=tol, maxiter=maxiter, maxstep=maxstep)
                self.Vprev[i] = max(float(np.linalg.norm(V)), 1e-30)
            du[i], du[nf + i] = V
            du[2 * nf + i] = math.exp(-ph[i]) - float(np.linalg.norm(V)) / self.fp.Dc
            self.tau[i] = self.tau0[0] + dtau[i] - self.eta * V[0]
            self.tau[nf + i] = self.tau0[1] + dtau[nf + i] - self.eta * V[1]
        dp = self.Ap @ pres
        if self.injection == "gaussian":
            q = self.q0 if t < self.t_off else 0.0
            dp = dp + q / (self.beta * self.phi) * self.source
        else:
            transfer = self.WI * (u[4 * nf] - pres[self.well_cell])
            dp[self.well_cell] += transfer / self.S_e
            Qinj = self.Q0 if t < self.t_off else 0.0
            du[4 * nf] = (Qinj - transfer) / self.S_well
        du[3 * nf:4 * nf] = dp
        return du
