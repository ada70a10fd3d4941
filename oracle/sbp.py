"""Order-4 diagonal-norm SBP finite-difference operators (CPU oracle).

TEST INFRASTRUCTURE. This package is the CPU oracle of the fault-stiffness
path: only tests, the smoke check and the benchmark's CPU-baseline leg use it,
and only as the checker. The product path never imports it.

The reference takes every stencil coefficient from the third-party package
Diffinitive.jl (git rev 92d842cf1b9a137aa4952b59ad959abf588ba855, data file
`standard_diagonal.toml`, order 4), read at `src/BP8.jl:195` and in each test's
`stencil_set()` helper (e.g. `test/elasticity_test.jl:34-36`). That package is
not vendored, so this module restates the published operators it implements:
the Mattsson-Nordstrom (2004) order-4 diagonal-norm first-derivative operator
D1, the compatible narrow second-derivative operator D2 with its third-order
boundary derivative, and the norm H (`SYMMETRIC_SAT.md:133-134` names the
family).

The coefficients are pinned, not trusted:
  * `H D1 + D1^T H = diag(-1, 0, ..., 0, 1)` exactly (checked in rationals);
  * `H D2 - (e_r d_r^T - e_l d_l^T)` is symmetric (the narrow-operator SBP
    identity quoted at `src/Elasticity.jl:183-186`);
  * interior order 4 and boundary order 2 (`test/convergence_test.jl:205-213`);
  * the assembled operator reproduces the reference's published structure and
    values (nnz counts, `K_self`), see the oracle tests.

Conventions follow Diffinitive: an operator along an axis with `n` points and
spacing `h` is an `n x n` matrix; closures occupy the first and last four
rows; the right-end closure of D1 is the left one mirrored with a sign flip
(odd parity), of D2 mirrored without (even parity). `d_l`, `d_r` are the
boundary derivatives along the fixed +x axis, i.e. `normal_derivative` with
its outward sign removed (`src/Elasticity.jl:191-203`).
"""
from fractions import Fraction as Fr

import numpy as np
import scipy.sparse as sp

# Norm weights of the four closure points at each end (interior weight 1).
H_CLOSURE = [Fr(17, 48), Fr(59, 48), Fr(43, 48), Fr(49, 48)]

# First derivative: interior stencil at offsets -2..2, closure rows 1..4 over
# columns 1..6.
D1_INTERIOR = [Fr(1, 12), Fr(-2, 3), Fr(0), Fr(2, 3), Fr(-1, 12)]
D1_CLOSURE = [
    [Fr(-24, 17), Fr(59, 34), Fr(-4, 17), Fr(-3, 34), Fr(0), Fr(0)],
    [Fr(-1, 2), Fr(0), Fr(1, 2), Fr(0), Fr(0), Fr(0)],
    [Fr(4, 43), Fr(-59, 86), Fr(0), Fr(59, 86), Fr(-4, 43), Fr(0)],
    [Fr(3, 98), Fr(0), Fr(-59, 98), Fr(0), Fr(32, 49), Fr(-4, 49)],
]

# Narrow second derivative.
D2_INTERIOR = [Fr(-1, 12), Fr(4, 3), Fr(-5, 2), Fr(4, 3), Fr(-1, 12)]
D2_CLOSURE = [
    [Fr(2), Fr(-5), Fr(4), Fr(-1), Fr(0), Fr(0)],
    [Fr(1), Fr(-2), Fr(1), Fr(0), Fr(0), Fr(0)],
    [Fr(-4, 43), Fr(59, 43), Fr(-110, 43), Fr(59, 43), Fr(-4, 43), Fr(0)],
    [Fr(-1, 49), Fr(0), Fr(59, 49), Fr(-118, 49), Fr(64, 49), Fr(-4, 49)],
]

# Boundary derivative at the left end along +x (third order), columns 1..4.
D_BOUNDARY = [Fr(-11, 6), Fr(3), Fr(-3, 2), Fr(1, 3)]

N_MIN = 9  # 2*order + 1, `src/BP8.jl:198-204`


def _check_n(n):
    if n < N_MIN:
        raise ValueError(f"order-4 SBP needs at least {N_MIN} points per axis, got {n}")


def h_weights_rational(n):
    """Diagonal of H/h as Fractions."""
    _check_n(n)
    w = [Fr(1)] * n
    for i, c in enumerate(H_CLOSURE):
        w[i] = c
        w[n - 1 - i] = c
    return w


def d1_rational(n):
    """D1*h as a dense list-of-lists of Fractions."""
    _check_n(n)
    M = [[Fr(0)] * n for _ in range(n)]
    for r in range(4):
        for c in range(6):
            M[r][c] = D1_CLOSURE[r][c]
            M[n - 1 - r][n - 1 - c] = -D1_CLOSURE[r][c]
    for r in range(4, n - 4):
        for o in range(-2, 3):
            M[r][r + o] = D1_INTERIOR[o + 2]
    return M


def d2_rational(n):
    """D2*h^2 as a dense list-of-lists of Fractions."""
    _check_n(n)
    M = [[Fr(0)] * n for _ in range(n)]
    for r in range(4):
        for c in range(6):
            M[r][c] = D2_CLOSURE[r][c]
            M[n - 1 - r][n - 1 - c] = D2_CLOSURE[r][c]
    for r in range(4, n - 4):
        for o in range(-2, 3):
            M[r][r + o] = D2_INTERIOR[o + 2]
    return M


def boundary_derivative_rational(n, upper):
    """Row vector d*h: +x derivative at the left (upper=False) or right end."""
    _check_n(n)
    d = [Fr(0)] * n
    for i, c in enumerate(D_BOUNDARY):
        if upper:
            d[n - 1 - i] = -c
        else:
            d[i] = c
    return d


def _to_csr(M, scale):
    n = len(M)
    rows, cols, vals = [], [], []
    for r in range(n):
        for c in range(n):
            if M[r][c] != 0:
                rows.append(r)
                cols.append(c)
                vals.append(float(M[r][c]) * scale)
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


class Axis:
    """1D SBP operators on `n` equidistant points with spacing `h`."""

    def __init__(self, n, h):
        _check_n(n)
        self.n = n
        self.h = float(h)
        hinv = 1.0 / self.h
        self.w = np.array([float(x) for x in h_weights_rational(n)])
        self.H = sp.diags(self.h * self.w).tocsr()
        self.Hinv = sp.diags(1.0 / (self.h * self.w)).tocsr()
        self.D1 = _to_csr(d1_rational(n), hinv)
        self.D2 = _to_csr(d2_rational(n), hinv * hinv)
        self.d_lower = np.array([float(x) for x in boundary_derivative_rational(n, False)]) * hinv
        self.d_upper = np.array([float(x) for x in boundary_derivative_rational(n, True)]) * hinv
        self.I = sp.identity(n, format="csr")

    def e(self, upper):
        v = np.zeros(self.n)
        v[self.n - 1 if upper else 0] = 1.0
        return v

    def d(self, upper):
        return self.d_upper if upper else self.d_lower
