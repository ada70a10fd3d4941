"""The coupled BP8 time loop's right-hand side on the GPU.

`BP8Rhs` is `rhs!(du, u, m, t)` / `evaluate!(m, u, t)` (src/BP8.jl:356-433)
with K resident in HBM: the K s GEMV, the per-node force balance
(`solve_slip_velocity`, src/RateStateFriction.jl:77-117), the aging law and
the pore-pressure equation with a caller-supplied sparse operator Ap (the
reference's `pore_pressure_operator`, src/PorePressure.jl:36-43, built once
on the host). `friction_solve` is `solve_slip_rate` for a batch of nodes.

    rhs = BP8Rhs(K, Ap, params, source=src, active=act)
    du = rhs(u, t)            # u = [s2; s3; ln(theta); p] (+ p_well)
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import EqdArgumentError, check, lib, ptr, f64


class RhsParams(C.Structure):
    """`eqd_rhs_params` (include/eqd.h)."""
    _fields_ = [("a", C.c_double), ("b", C.c_double), ("Dc", C.c_double), ("V_star", C.c_double),
                ("f_star", C.c_double), ("sigma0", C.c_double), ("sigma_min", C.c_double), ("eta", C.c_double),
                ("tau0_2", C.c_double), ("tau0_3", C.c_double), ("q0", C.c_double), ("beta", C.c_double),
                ("phi", C.c_double), ("t_off", C.c_double), ("injection", C.c_int32), ("well_cell", C.c_int32),
                ("WI", C.c_double), ("S_e", C.c_double), ("S_well", C.c_double), ("Q0", C.c_double),
                ("newton_tol", C.c_double), ("newton_maxstep", C.c_double), ("newton_maxiter", C.c_int32),
                ("pad_", C.c_int32)]


@dataclass
class FrictionParams:
    """`FrictionParams(a, b, Dc, V_star, f_star)` (src/RateStateFriction.jl:18-24)."""
    a: float
    b: float
    Dc: float
    V_star: float
    f_star: float


def _params(fp, newton_tol=1e-12, newton_maxiter=50, newton_maxstep=5.0, **kw):
    p = RhsParams()
    p.a, p.b, p.Dc, p.V_star, p.f_star = fp.a, fp.b, fp.Dc, fp.V_star, fp.f_star
    p.newton_tol, p.newton_maxiter, p.newton_maxstep = newton_tol, newton_maxiter, newton_maxstep
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def friction_solve(T, theta, sigma, eta, fp, V0=None, tol=1e-12, maxiter=50, maxstep=5.0, device=0):
    """`solve_slip_rate` for arrays of nodes on the GPU; raises EqdError
    (EQD_ERR_NOT_CONVERGED) where the reference throws."""
    T, theta, sigma = f64(np.atleast_1d(T)), f64(np.atleast_1d(theta)), f64(np.atleast_1d(sigma))
    n = T.size
    if theta.size != n or sigma.size != n:
        raise EqdArgumentError(_abi.EQD_ERR_ARG, "T, theta and sigma must have the same length")
    V = np.empty(n)
    v0 = None if V0 is None else f64(np.broadcast_to(V0, (n,)))
    p = _params(fp, tol, maxiter, maxstep)
    check(lib().eqd_friction_solve(C.c_int32(device), C.c_int32(n), ptr(T), ptr(theta), ptr(sigma), C.c_double(eta),
                                   C.byref(p), None if v0 is None else ptr(v0), ptr(V)))
    return V


class BP8Rhs:
    """GPU right-hand side of the coupled model. `params` is a dict of
    `eqd_rhs_params` fields besides the friction ones: sigma0, sigma_min,
    eta, tau0 (2-vector), and for the Gaussian source q0, beta, phi, t_off,
    or for the Peaceman well injection="peaceman", well_cell, WI, S_e,
    S_well, Q0 (and t_off)."""

    def __init__(self, K, Ap, fp, sigma0, sigma_min, eta, tau0, source=None, active=None, injection="gaussian",
                 q0=0.0, beta=1.0, phi=1.0, t_off=0.0, well_cell=0, WI=0.0, S_e=1.0, S_well=1.0, Q0=0.0,
                 device=0, newton_tol=1e-12, newton_maxiter=50, newton_maxstep=5.0):
        import scipy.sparse as sp
        K = np.asfortranarray(K, dtype=np.float64)
        n = K.shape[0]
        if K.ndim != 2 or K.shape[1] != n or n % 2:
            raise EqdArgumentError(_abi.EQD_ERR_ARG, "K must be 2nf x 2nf")
        self.nf = n // 2
        A = sp.csr_matrix(Ap)
        if A.shape != (self.nf, self.nf):
            raise EqdArgumentError(_abi.EQD_ERR_ARG, "Ap must be nf x nf")
        A.sort_indices()
        self.peaceman = injection == "peaceman"
        if injection not in ("gaussian", "peaceman"):
            raise EqdArgumentError(_abi.EQD_ERR_ARG, f"injection must be :gaussian or :peaceman, got {injection}")
        p = _params(fp, newton_tol, newton_maxiter, newton_maxstep, sigma0=sigma0, sigma_min=sigma_min, eta=eta,
                    tau0_2=float(tau0[0]), tau0_3=float(tau0[1]), q0=q0, beta=beta, phi=phi, t_off=t_off,
                    injection=1 if self.peaceman else 0, well_cell=int(well_cell), WI=WI, S_e=S_e, S_well=S_well,
                    Q0=Q0)
        ap_ptr = np.ascontiguousarray(A.indptr, dtype=np.int32)
        ap_idx = np.ascontiguousarray(A.indices, dtype=np.int32)
        ap_val = f64(A.data)
        src = None if source is None else f64(source)
        act = None if active is None else np.ascontiguousarray(active, dtype=np.uint8)
        h = C.c_void_p()
        check(lib().eqd_rhs_create(C.c_int32(device), C.c_int32(self.nf), ptr(K), C.byref(p), ptr(ap_ptr), ptr(ap_idx),
                                   ptr(ap_val), None if src is None else ptr(src), None if act is None else ptr(act),
                                   C.byref(h)))
        self._h = h

    @property
    def state_length(self):
        return 4 * self.nf + (1 if self.peaceman else 0)

    def __call__(self, u, t):
        u = f64(u)
        if u.size != self.state_length:
            raise EqdArgumentError(_abi.EQD_ERR_ARG, f"state has {u.size} entries, expected {self.state_length}")
        du = np.empty_like(u)
        check(lib().eqd_rhs_eval(self._h, C.c_double(t), ptr(u), ptr(du)))
        return du

    def fields(self):
        """(tau: 2nf shear stress acting on the fault, Vprev: nf) of the last evaluation."""
        tau, vp = np.empty(2 * self.nf), np.empty(self.nf)
        check(lib().eqd_rhs_fields(self._h, ptr(tau), ptr(vp)))
        return tau, vp

    def report(self):
        s, hits, nodes = C.c_double(), C.c_int64(), C.c_int32()
        check(lib().eqd_rhs_report(self._h, C.byref(s), C.byref(hits), C.byref(nodes)))
        return dict(sigma_lowest=s.value, floor_hits=hits.value, floor_nodes=nodes.value)

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib().eqd_rhs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
