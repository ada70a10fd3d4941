"""eqd_b200 — B200 (sm_100a) fault-stiffness engine, host-side interface.

Mirrors the reference's API for the fault-stiffness path of
EarthquakeDiffinitive.jl (same names, argument meaning and error behaviour),
on top of the C ABI in include/eqd.h:

  reference (Julia)                                   here
  -------------------------------------------------   ---------------------------------
  FaultElasticity(g₋, g₊, λ, μ, set; l_f, kw...)     FaultElasticity(grids, lam, mu, l_f, **kw)
      src/FaultResponse.jl:96-146
  CGSolver(A; rtol, atol, itmax, precond)             CGSolver(rtol=, atol=, itmax=, precond=, precision=)
      src/ElasticitySplitNode.jl:365
  split_node_solve(s, rhs)          :378-396          split_node_solve(solver, rhs)
  duplicate / merge_stats! / solver_report :408-447   solver.duplicate() / merge_stats(a, b) / solver_report(s)
  shear_traction(fe, s2, s3)        FaultResponse:194 shear_traction(fe, s2, s3)
  fault_stiffness(fe; verbose, threaded)       :229   fault_stiffness(fe, verbose=False, threaded=None)
  fault_stiffness_toeplitz(fe; verbose)        :339   fault_stiffness_toeplitz(fe, verbose=False)
  elastic_solver_report / frictional_node_count / fault_grid_axes
  build_model(; Δz, L_fault, L_normal, stiffness) BP8.jl:184   build_model(dz=, L_fault=, L_normal=, stiffness=)
  mul!(Δτ, K, slip)                  BP8.jl:366        KMatrix(K).gemv(slip)

Misuse raises `EqdArgumentError` (a ValueError), where the reference calls
`error()`. A CG solve that does not converge is counted in the solver's
`unconverged` and warned about once, not raised — as in the reference.

There is no CPU path: every call runs the sm_100a kernels of libeqd.so and
fails loudly if the library or a GPU is missing.
"""
import ctypes as C
import os
import threading
import warnings

import numpy as np

from . import _abi
from ._abi import EqdError, EqdArgumentError, check, lib, ptr, f64

__all__ = [
    "GridPair", "bp8_grids", "cube_grids", "lame_lambda", "FaultElasticity", "CGSolver",
    "CGStats", "split_node_solve", "solver_report", "merge_stats", "duplicate",
    "elastic_solver_report", "frictional_node_count", "fault_grid_axes", "shear_traction",
    "fault_stiffness", "fault_stiffness_toeplitz", "stiffness_columns", "apply_operator", "assemble_operator",
    "KMatrix", "build_model", "EqdError", "EqdArgumentError", "library_path", "Server",
    "operator_diagonal", "jacobi_preconditioner", "cached_fault_stiffness", "BP8Rhs", "FrictionParams",
    "friction_solve",
]


def library_path():
    return _abi.LIB_PATH


# ---------------------------------------------------------------------------
# Grids
# ---------------------------------------------------------------------------
class GridPair:
    """The two blocks of the split-node system: minus x1 in [-x1_extent, 0],
    plus x1 in [0, x1_extent], both over [x2_lo, x2_hi] x [x3_lo, x3_hi] with
    n1 x n2 x n3 nodes (the reference's `g_minus`, `g_plus`)."""

    def __init__(self, n1, n2, n3, x1_extent, x2=(-1.0, 1.0), x3=(-1.0, 1.0)):
        self.n1, self.n2, self.n3 = int(n1), int(n2), int(n3)
        self.x1_extent = float(x1_extent)
        self.x2 = (float(x2[0]), float(x2[1]))
        self.x3 = (float(x3[0]), float(x3[1]))

    @property
    def ntot(self):
        return 6 * self.n1 * self.n2 * self.n3


def bp8_grids(dz, L_fault, L_normal):
    """`build_model`'s grids (src/BP8.jl:196-206)."""
    n1 = int(round(L_normal / dz)) + 1
    n23 = int(round(2 * L_fault / dz)) + 1
    return GridPair(n1, n23, n23, L_normal, (-L_fault, L_fault), (-L_fault, L_fault))


def cube_grids(n, L=1.0):
    """The test suites' `fr_grids(n; L)` (test/fault_response_test.jl:16-17)."""
    return GridPair(n, n, n, L, (-L, L), (-L, L))


def lame_lambda(mu, nu):
    """`lame_lambda` (src/BP8.jl:92)."""
    return 2 * mu * nu / (1 - 2 * nu)


# ---------------------------------------------------------------------------
# Solver options + stats
# ---------------------------------------------------------------------------
class CGStats:
    """`CGStats` (src/ElasticitySplitNode.jl:256-262)."""

    def __init__(self):
        self.solves = 0
        self.iterations = 0
        self.max_iterations = 0
        self.unconverged = 0
        self.seconds = 0.0
        self.device_seconds = 0.0

    def add(self, st):
        self.solves += st.solves
        self.iterations += st.iterations
        self.max_iterations = max(self.max_iterations, st.max_iterations)
        self.unconverged += st.unconverged
        self.seconds += st.seconds
        self.device_seconds += st.device_seconds


_PRECONDS = {"none": _abi.EQD_PRECOND_NONE, "jacobi": _abi.EQD_PRECOND_JACOBI}
_PRECISIONS = {"fp64": _abi.EQD_PREC_FP64, "mixed": _abi.EQD_PREC_MIXED}


class CGSolver:
    """`CGSolver(A; rtol=1e-10, atol=0.0, itmax=0, precond=:none)`.

    The operator is the matrix-free A of the grid the solver is attached to
    (a FaultElasticity attaches its own). `precision` selects the engine:
    "fp64" is plain FP64 CG with Krylov.jl's stopping rule (recursive
    residual); "mixed" is FP32 CG with FP64 reliable updates, stopping on the
    FP64 true residual. `chunk` caps the columns resident at once (0: as many
    as `hbm_budget_bytes` allows), `reliable_delta` is the mixed engine's
    residual-drop factor for an FP64 true-residual update; `variant` picks
    the FP32 stencil launch variant for this solver's calls (0: the grid's,
    chosen by `autotune` on first use or pinned by `set_stencil_variant`;
    k > 0: variant k - 1 of `autotune`'s list). `split` and `fuse` change
    only the schedule, never the result bits: `split=False` runs a large
    batch as one chain of kernels instead of two overlapping halves, and
    `fuse=True` forms the CG direction inside the stencil apply (slower on
    B200; for comparison)."""

    def __init__(self, fe=None, rtol=1e-10, atol=0.0, itmax=0, precond="none", precision="mixed",
                 chunk=0, reliable_delta=0.01, hbm_budget_bytes=0, variant=0, split=True, fuse=False):
        if precond not in _PRECONDS:
            raise EqdArgumentError(_abi.EQD_ERR_ARG, f"precond must be :none or :jacobi, got {precond}")
        if precision not in _PRECISIONS:
            raise EqdArgumentError(_abi.EQD_ERR_ARG, f"precision must be 'fp64' or 'mixed', got {precision}")
        self.fe = fe
        self.rtol, self.atol, self.itmax = float(rtol), float(atol), int(itmax)
        self.precond, self.precision = precond, precision
        self.chunk, self.reliable_delta = int(chunk), float(reliable_delta)
        self.hbm_budget_bytes, self.variant = int(hbm_budget_bytes), int(variant)
        self.split = bool(split)
        self.fuse = bool(fuse)
        self.stats = CGStats()
        self._warned = False

    def opts(self, **over):
        o = _abi.default_opts()
        o.rtol, o.atol, o.itmax = self.rtol, self.atol, self.itmax
        o.precond = _PRECONDS[self.precond]
        o.precision = _PRECISIONS[over.get("precision", self.precision)]
        o.chunk = self.chunk
        o.reliable_delta = self.reliable_delta
        o.hbm_budget_bytes = self.hbm_budget_bytes
        o.variant = self.variant
        if not self.split:
            o.flags |= _abi.EQD_FLAG_NO_SPLIT
        if self.fuse:
            o.flags |= _abi.EQD_FLAG_FUSE
        return o

    def record(self, st):
        self.stats.add(st)
        if st.unconverged and not self._warned:
            self._warned = True
            warnings.warn(
                f"CG did not converge on {st.unconverged} split-node solve(s). The returned "
                "displacement is not a solution, and fault_stiffness would fold it into K "
                f"silently. Raise itmax or loosen rtol. (rtol={self.rtol}, itmax={self.itmax})",
                RuntimeWarning, stacklevel=3)

    def duplicate(self):
        """`duplicate(solver)`: same operator and options, fresh counters."""
        return CGSolver(self.fe, self.rtol, self.atol, self.itmax, self.precond, self.precision,
                        self.chunk, self.reliable_delta, self.hbm_budget_bytes, self.variant, self.split,
                        self.fuse)

    def report(self):
        t = self.stats
        return dict(kind="cg", precond=self.precond, solves=t.solves, iterations=t.iterations,
                    mean_iterations=0.0 if t.solves == 0 else t.iterations / t.solves,
                    max_iterations=t.max_iterations, unconverged=t.unconverged)


def duplicate(solver):
    return solver.duplicate()


def merge_stats(into, frm):
    """`merge_stats!(into, from)`."""
    a, b = into.stats, frm.stats
    a.solves += b.solves
    a.iterations += b.iterations
    a.max_iterations = max(a.max_iterations, b.max_iterations)
    a.unconverged += b.unconverged
    return into


def solver_report(solver):
    return solver.report()


# ---------------------------------------------------------------------------
# FaultElasticity
# ---------------------------------------------------------------------------
class FaultElasticity:
    """`FaultElasticity(g_minus, g_plus, λ, μ, set; l_f, solver_kwargs...)`.

    Holds the device-resident operator metadata for the grid pair (a few KB;
    nothing is assembled). Omega_f = fault nodes with |x2|, |x3| <= l_f,
    ordered x2-fastest; a spacing that misses +-l_f raises, as the reference
    does."""

    def __init__(self, grids, lam, mu, l_f, device=0, **solver_kwargs):
        self.grids = grids
        self.lam, self.mu, self.l_f = float(lam), float(mu), float(l_f)
        d = _abi.GridDesc(grids.n1, grids.n2, grids.n3, grids.x1_extent,
                          grids.x2[0], grids.x2[1], grids.x3[0], grids.x3[1],
                          self.lam, self.mu, self.l_f, 4, int(device))
        h = C.c_void_p()
        check(lib().eqd_grid_create(C.byref(d), C.byref(h)))
        self._h = h
        ntot = C.c_int64()
        nf, n2f, n3f = C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().eqd_grid_info(h, C.byref(ntot), C.byref(nf), C.byref(n2f), C.byref(n3f)))
        self.Ntot, self.nf = ntot.value, nf.value
        self.n2f, self.n3f = n2f.value, n3f.value
        self.x2f = np.empty(self.n2f)
        self.x3f = np.empty(self.n3f)
        check(lib().eqd_grid_fault_axes(h, ptr(self.x2f), ptr(self.x3f)))
        self.rs = CGSolver(self, **solver_kwargs)
        self._lock = threading.Lock()

    @property
    def handle(self):
        if self._h is None:
            raise EqdError(_abi.EQD_ERR_ARG, "FaultElasticity was closed")
        return self._h

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib().eqd_grid_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_stencil_variant(fe, variant):
    """Pin the FP32 stencil launch variant of this grid (skips autotuning)."""
    check(lib().eqd_set_variant(fe.handle, C.c_int32(variant)))


def autotune(fe, ncols=256):
    """Time every FP32 stencil launch variant; returns (selected, [(tile_rows, threads, ms)]),
    the list indexed by variant (`set_stencil_variant`, CGSolver(variant=k + 1))."""
    sel, nv = C.c_int32(), C.c_int32()
    ms, tr, tt = (C.c_double * 16)(), (C.c_int32 * 16)(), (C.c_int32 * 16)()
    check(lib().eqd_autotune(fe.handle, C.c_int32(ncols), C.byref(sel), ms, tr, tt, C.byref(nv)))
    return sel.value, [(tr[i], tt[i], ms[i]) for i in range(nv.value)]


def tune_chunk(fe, widths=(32, 64, 128, 256, 512, 1024)):
    """Time mixed-precision CG iterations at each batch width; returns (best
    width, [(width, ms per column-iteration or None when out of range)]).
    Later calls on this grid with chunk=0 use the best width."""
    w = np.ascontiguousarray(widths, dtype=np.int32)
    ms = np.empty(len(w))
    best = C.c_int32()
    check(lib().eqd_tune_chunk(fe.handle, ptr(w), C.c_int32(len(w)), ptr(ms), C.byref(best)))
    return best.value, [(int(a), (float(b) if b >= 0 else None)) for a, b in zip(w, ms)]


def frictional_node_count(fe):
    return fe.nf


def fault_grid_axes(fe):
    return fe.x2f.copy(), fe.x3f.copy()


def elastic_solver_report(fe):
    return fe.rs.report()


def _solver_for(fe, solver):
    s = solver if solver is not None else fe.rs
    return s


def split_node_solve(solver, rhs):
    """`split_node_solve(s, rhs)`: solve A u = rhs (reference DOF layout)
    by FP64 CG with Krylov's stopping rule. `rhs` may hold several columns."""
    fe = solver.fe
    if fe is None:
        raise EqdArgumentError(_abi.EQD_ERR_ARG, "solver is not attached to a grid")
    b = f64(rhs)
    one = b.ndim == 1
    B = b.reshape(-1, 1) if one else b
    if B.shape[0] != fe.Ntot:
        raise EqdArgumentError(_abi.EQD_ERR_ARG, f"rhs has {B.shape[0]} rows, system has {fe.Ntot}")
    ncols = B.shape[1]
    Bc = np.ascontiguousarray(B.T)
    U = np.empty_like(Bc)
    st = _abi.Stats()
    check(lib().eqd_cg_solve(fe.handle, ptr(Bc), ptr(U), C.c_int32(ncols), C.byref(solver.opts()),
                             None, None, C.byref(st)))
    solver.record(st)
    return U[0].copy() if one else U.T.copy()


def operator_diagonal(fe):
    """diag(A) of the split-node operator A = -H P (D+SAT) P, reference DOF
    layout, computed on the GPU from the stencil tables (no assembly)."""
    d = np.empty(fe.Ntot)
    check(lib().eqd_diag(fe.handle, ptr(d)))
    return d


def jacobi_preconditioner(fe):
    """`jacobi_preconditioner(A)` (src/ElasticitySplitNode.jl:352-357):
    1 ./ diag(A), zero entries (the far-field rows) floored to 1; a negative
    diagonal entry raises."""
    d = operator_diagonal(fe)
    if np.any(d < 0):
        raise EqdArgumentError(_abi.EQD_ERR_ARG, "diag(A) has negative entries; A is not PSD and "
                                                 "a Jacobi preconditioner would not be SPD")
    out = np.ones_like(d)
    nz = d != 0
    out[nz] = 1.0 / d[nz]
    return out


def apply_operator(fe, x, mode="A", precision="fp64"):
    """y = A x (mode "A"), y = HP_DSAT x (mode "HP_DSAT"), or y = A x for x
    already in range(P) (mode "A_rangeP", the kernel CG iterates with), in the
    reference layout."""
    xx = f64(x)
    one = xx.ndim == 1
    X = np.ascontiguousarray((xx.reshape(-1, 1) if one else xx).T)
    Y = np.empty_like(X)
    m = {"A": 0, "HP_DSAT": 1, "A_rangeP": 2}[mode]
    check(lib().eqd_apply(fe.handle, ptr(X), ptr(Y), C.c_int32(X.shape[0]), C.c_int32(m),
                          C.c_int32(_PRECISIONS[precision])))
    return Y[0].copy() if one else Y.T.copy()


def assemble_operator(fe, which="A"):
    """The assembled sparse matrix of `split_node_system`
    (src/ElasticitySplitNode.jl:106-214): "A" = -H P (D+SAT) P or "HP_DSAT"
    = H P (D+SAT), as a scipy CSR matrix in the reference DOF order, built on
    the GPU by coloured probing of the matrix-free operator. Entries below
    1e-12 of their row's largest are left out (numerically zero)."""
    import scipy.sparse as sp
    w = {"A": 0, "HP_DSAT": 1}[which]
    nnz = C.c_int64()
    check(lib().eqd_assemble(fe.handle, C.c_int32(w), C.c_int64(0), None, None, None, C.byref(nnz)))
    n = fe.Ntot
    indptr = np.empty(n + 1, dtype=np.int64)
    indices = np.empty(max(nnz.value, 1), dtype=np.int32)
    values = np.empty(max(nnz.value, 1))
    check(lib().eqd_assemble(fe.handle, C.c_int32(w), C.c_int64(len(values)), ptr(indptr), ptr(indices),
                             ptr(values), C.byref(nnz)))
    k = nnz.value
    return sp.csr_matrix((values[:k], indices[:k], indptr), shape=(n, n))


def shear_traction(fe, s2, s3, solver=None):
    """`shear_traction(fe, s2, s3) -> (Δτ2, Δτ3)`; s2/s3 may be nf x nslip."""
    solver = _solver_for(fe, solver)
    a2, a3 = f64(s2), f64(s3)
    one = a2.ndim == 1
    S2 = np.ascontiguousarray((a2.reshape(-1, 1) if one else a2).T)
    S3 = np.ascontiguousarray((a3.reshape(-1, 1) if one else a3).T)
    if S2.shape != S3.shape or S2.shape[1] != fe.nf:
        raise EqdArgumentError(_abi.EQD_ERR_ARG, "s2 and s3 must both have nf rows")
    D2 = np.empty_like(S2)
    D3 = np.empty_like(S3)
    st = _abi.Stats()
    check(lib().eqd_shear_traction(fe.handle, ptr(S2), ptr(S3), C.c_int32(S2.shape[0]), ptr(D2), ptr(D3),
                                   C.byref(solver.opts()), C.byref(st)))
    solver.record(st)
    if one:
        return D2[0].copy(), D3[0].copy()
    return D2.T.copy(), D3.T.copy()


def stiffness_columns(fe, cols, solver=None):
    """Columns `cols` of K (2nf x len(cols)), with per-column iterations and
    status codes."""
    solver = _solver_for(fe, solver)
    cc = np.ascontiguousarray(cols, dtype=np.int32)
    out = np.empty((2 * fe.nf, len(cc)), order="F")
    iters = np.zeros(len(cc), dtype=np.int32)
    status = np.zeros(len(cc), dtype=np.int8)
    st = _abi.Stats()
    check(lib().eqd_stiffness_columns(fe.handle, ptr(cc), C.c_int32(len(cc)), C.byref(solver.opts()),
                                      ptr(out), ptr(iters), ptr(status), C.byref(st)))
    solver.record(st)
    return out, iters, status


def fault_stiffness(fe, verbose=False, threaded=None, solver=None):
    """`fault_stiffness(fe; verbose=false, threaded=...)` -> K (2nf x 2nf).

    All 2nf unit-slip columns run as batched multi-column CG on the GPU;
    `threaded` is accepted for API parity and has no effect (the batch is the
    parallelism)."""
    solver = _solver_for(fe, solver)
    n = 2 * fe.nf
    K = np.empty((n, n), order="F")
    st = _abi.Stats()
    check(lib().eqd_stiffness_exact(fe.handle, C.byref(solver.opts()), ptr(K), C.byref(st)))
    solver.record(st)
    if verbose:
        print(f"fault_stiffness: done seconds={st.seconds:.2f} columns={n} "
              f"mean_iterations={st.iterations / max(st.solves, 1):.1f}")
    return K


def fault_stiffness_toeplitz(fe, verbose=False, solver=None):
    """`fault_stiffness_toeplitz(fe)`: 5 sources x (s2, s3) = 10 solves."""
    solver = _solver_for(fe, solver)
    n = 2 * fe.nf
    K = np.empty((n, n), order="F")
    st = _abi.Stats()
    check(lib().eqd_stiffness_toeplitz(fe.handle, C.byref(solver.opts()), ptr(K), C.byref(st)))
    solver.record(st)
    if verbose:
        print(f"fault_stiffness_toeplitz: done seconds={st.seconds:.2f} solves={st.solves}")
    return K


# ---------------------------------------------------------------------------
# Resident K for the time loop
# ---------------------------------------------------------------------------
class KMatrix:
    """K resident in device memory; `gemv(slip)` is `mul!(Δτ, K, slip)`."""

    def __init__(self, K, device=0):
        K = np.asfortranarray(K, dtype=np.float64)
        if K.ndim != 2 or K.shape[0] != K.shape[1]:
            raise EqdArgumentError(_abi.EQD_ERR_ARG, "K must be square")
        self.n = K.shape[0]
        h = C.c_void_p()
        check(lib().eqd_kmat_create(C.c_int32(device), C.c_int32(self.n), ptr(K), C.byref(h)))
        self._h = h

    def gemv(self, s):
        """y = K s for one slip vector (n,) or several (n, nvec). A
        column-major (Fortran-ordered) (n, nvec) array goes to the device
        without a host transpose; the result of a matrix product is returned
        column-major."""
        s = np.asarray(s, dtype=np.float64)
        one = s.ndim == 1
        S = np.ascontiguousarray((s.reshape(-1, 1) if one else s).T)
        if S.shape[1] != self.n:
            raise EqdArgumentError(_abi.EQD_ERR_ARG, "slip length does not match K")
        Y = np.empty_like(S)
        check(lib().eqd_kmat_gemv(self._h, ptr(S), ptr(Y), C.c_int32(S.shape[0])))
        return Y[0] if one else Y.T

    def gemv_device(self, s, y, stream=None):
        """y = K s on device-resident vectors: `s` and `y` are contiguous
        float64 device tensors of shape (nvec, n) or (n,) (one slip vector per
        row), or `(pointer, nvec)` pairs. Launches on `stream` (a
        torch.cuda.Stream, a raw cudaStream_t, or None for the default stream)
        and returns without synchronizing."""
        def dev(a):
            if isinstance(a, tuple):
                return int(a[0]), int(a[1])
            if a.dtype.itemsize != 8 or not a.is_contiguous() or a.shape[-1] != self.n or a.dim() > 2:
                raise EqdArgumentError(_abi.EQD_ERR_ARG, "expected a contiguous float64 (nvec, n) device tensor")
            return a.data_ptr(), (1 if a.dim() == 1 else a.shape[0])
        sp, nv = dev(s)
        yp, nvy = dev(y)
        if nv != nvy:
            raise EqdArgumentError(_abi.EQD_ERR_ARG, "s and y hold different numbers of vectors")
        st = getattr(stream, "cuda_stream", stream) or 0
        check(lib().eqd_kmat_gemv_device(self._h, C.c_void_p(sp), C.c_void_p(yp), C.c_int32(nv), C.c_void_p(st)))

    def close(self):
        if getattr(self, "_h", None) is not None:
            lib().eqd_kmat_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def build_model(dz=50.0, L_fault=800.0, L_normal=400.0, l_f=400.0, mu=32.04e9, nu=0.25,
                stiffness="toeplitz", device=0, verbose=False, **solver_kwargs):
    """The elastic part of `build_model` (src/BP8.jl:184-258): grids, the
    FaultElasticity, and K by `stiffness` = "exact" | "toeplitz"."""
    if stiffness not in ("exact", "toeplitz"):
        raise EqdArgumentError(_abi.EQD_ERR_ARG, f"stiffness must be :exact or :toeplitz, got {stiffness}")
    if abs(l_f / dz - round(l_f / dz)) > 1e-9:
        raise EqdArgumentError(_abi.EQD_ERR_ARG, f"Δz={dz} must divide l_f={l_f} so the grid has nodes on ±l_f")
    if L_fault < l_f:
        raise EqdArgumentError(_abi.EQD_ERR_ARG, f"L_fault={L_fault} must be at least l_f={l_f}")
    g = bp8_grids(dz, L_fault, L_normal)
    if g.n1 < 9:
        raise EqdArgumentError(_abi.EQD_ERR_ARG,
                               f"L_normal/Δz gives only {g.n1} points across the fault-normal direction; "
                               "SBP order 4 needs at least 9. Increase L_normal or decrease Δz.")
    fe = FaultElasticity(g, lame_lambda(mu, nu), mu, l_f, device=device, **solver_kwargs)
    K = fault_stiffness(fe, verbose=verbose) if stiffness == "exact" else fault_stiffness_toeplitz(fe, verbose=verbose)
    info = dict(dz=dz, L_fault=L_fault, L_normal=L_normal, n1=g.n1, n23=g.n2, order=4,
                elastic_dofs=g.ntot, n2f=fe.n2f, n3f=fe.n3f)
    return dict(fe=fe, K=K, nf=fe.nf, x2=fe.x2f.copy(), x3=fe.x3f.copy(), grid_info=info)


from .serving import Server  # noqa: E402  (continuous-batching request server)
from .kcache import cached_fault_stiffness  # noqa: E402  (on-disk K cache with resume)
from .timeloop import BP8Rhs, FrictionParams, friction_solve  # noqa: E402  (time-loop RHS on the GPU)
