"""Conjugate gradients with Krylov.jl's `cg!` stopping rule (CPU oracle).

TEST INFRASTRUCTURE: the oracle. Only tests, the smoke check and the
benchmark's CPU-baseline leg use it.

The reference calls `Krylov.cg!` (Krylov.jl 0.10.9, pinned in
`Project.toml:24` and `context/demo/Manifest.toml:1123-1127`; not vendored) at
`src/ElasticitySplitNode.jl:379-380`, wrapped by `CGSolver`
(`src/ElasticitySplitNode.jl:324-370`) and `split_node_solve` (`:378-396`).
This restates the published algorithm for the unpreconditioned /
diagonally-preconditioned case with x0 = 0:

    r = b; z = M r; p = z; gamma = r.z; rNorm = sqrt(gamma)
    eps = atol + rtol * rNorm;  itmax = 0 -> 2n
    while !(rNorm <= eps || iter >= itmax):
        Ap = A p; pAp = p.Ap
        (pAp <= eps_mach * |p|^2 -> zero curvature, stop)
        alpha = gamma / pAp; x += alpha p; r -= alpha Ap; z = M r
        gamma' = r.z; rNorm = sqrt(gamma')
        beta = gamma'/gamma; p = z + beta p  (only if not yet solved)

The convergence test uses the recursively updated residual, as Krylov does.
"""
import numpy as np


class CGStats:
    """`CGStats` (`src/ElasticitySplitNode.jl:256-262`)."""

    def __init__(self):
        self.solves = 0
        self.iterations = 0
        self.max_iterations = 0
        self.unconverged = 0


def krylov_cg(A, b, rtol=1e-10, atol=0.0, itmax=0, Minv=None):
    """Returns (x, niter, solved, status)."""
    n = b.shape[0]
    x = np.zeros_like(b)
    r = b.copy()
    z = r if Minv is None else Minv * r
    p = z.copy()
    gamma = float(r @ z)
    rnorm = np.sqrt(gamma) if Minv is None else np.linalg.norm(r)
    if gamma == 0.0:
        return x, 0, True, "x = 0 is a zero-residual solution"
    eps = atol + rtol * rnorm
    itmax = 2 * n if itmax == 0 else itmax
    it = 0
    solved = rnorm <= eps
    tired = it >= itmax
    status = "unknown"
    while not (solved or tired):
        Ap = A @ p
        pAp = float(p @ Ap)
        if pAp <= np.finfo(float).eps * float(p @ p):
            status = "zero curvature"
            break
        alpha = gamma / pAp
        x += alpha * p
        r -= alpha * Ap
        z = r if Minv is None else Minv * r
        gamma_next = float(r @ z)
        rnorm = np.sqrt(gamma_next) if Minv is None else np.linalg.norm(r)
        it += 1
        solved = rnorm <= eps
        tired = it >= itmax
        if not solved:
            beta = gamma_next / gamma
            p = z + beta * p
        gamma = gamma_next
    if solved:
        status = "solution good enough given atol and rtol"
    elif tired:
        status = "maximum number of iterations exceeded"
    return x, it, solved, status


def jacobi_preconditioner(A):
    """`jacobi_preconditioner` (`src/ElasticitySplitNode.jl:352-357`)."""
    d = A.diagonal()
    if np.any(d < 0):
        raise ValueError("diag(A) has negative entries; A is not PSD and "
                         "a Jacobi preconditioner would not be SPD")
    out = np.ones_like(d)
    nz = d != 0
    out[nz] = 1.0 / d[nz]
    return out


class CGSolver:
    """`CGSolver(A; rtol=1e-10, atol=0.0, itmax=0, precond=:none)`."""

    def __init__(self, A, rtol=1e-10, atol=0.0, itmax=0, precond="none"):
        if precond not in ("none", "jacobi"):
            raise ValueError(f"precond must be :none or :jacobi, got {precond}")
        self.A = A
        self.precond = precond
        self.Minv = jacobi_preconditioner(A) if precond == "jacobi" else None
        self.rtol, self.atol, self.itmax = rtol, atol, itmax
        self.stats = CGStats()
        self.warned = False

    def solve(self, rhs):
        """`split_node_solve(s, rhs)`."""
        x, it, solved, status = krylov_cg(self.A, rhs, self.rtol, self.atol, self.itmax, self.Minv)
        t = self.stats
        t.solves += 1
        t.iterations += it
        t.max_iterations = max(t.max_iterations, it)
        if not solved:
            t.unconverged += 1
        return x

    def duplicate(self):
        d = CGSolver.__new__(CGSolver)
        d.A, d.precond, d.Minv = self.A, self.precond, self.Minv
        d.rtol, d.atol, d.itmax = self.rtol, self.atol, self.itmax
        d.stats = CGStats()
        d.warned = False
        return d

    def merge_stats(self, other):
        a, b = self.stats, other.stats
        a.solves += b.solves
        a.iterations += b.iterations
        a.max_iterations = max(a.max_iterations, b.max_iterations)
        a.unconverged += b.unconverged
        return self

    def report(self):
        t = self.stats
        return dict(kind="cg", precond=self.precond, solves=t.solves,
                    iterations=t.iterations,
                    mean_iterations=0.0 if t.solves == 0 else t.iterations / t.solves,
                    max_iterations=t.max_iterations, unconverged=t.unconverged)
