"""Slip -> shear-traction map and the dense fault stiffness K (CPU oracle).

TEST INFRASTRUCTURE: the oracle. Only tests, the smoke check and the
benchmark's CPU-baseline leg use it.

Restates `src/FaultResponse.jl`:
  * `FaultElasticity` constructor        -> `:96-146`  (Omega_f selection x2-fastest,
                                                          T2/T3 averaging, chi rows)
  * `build_chi!`                         -> `:176-185`
  * `shear_traction[!]`                  -> `:194-211`
  * `fault_stiffness`                    -> `:229-287`  (serial column loop; the
                                                          reference's threaded build is
                                                          bit-identical by construction)
  * `fault_stiffness_toeplitz`           -> `:339-393`
and the grid set-up of `build_model` (`src/BP8.jl:184-207`).
"""
import numpy as np

from .operators import Grid3, SplitNodeSystem
from .krylov_cg import CGSolver


def bp8_grids(dz, L_fault, L_normal):
    """The two blocks of `build_model` (`src/BP8.jl:196-206`)."""
    n1 = int(round(L_normal / dz)) + 1
    n23 = int(round(2 * L_fault / dz)) + 1
    gm = Grid3((-L_normal, -L_fault, -L_fault), (0.0, L_fault, L_fault), (n1, n23, n23))
    gp = Grid3((0.0, -L_fault, -L_fault), (L_normal, L_fault, L_fault), (n1, n23, n23))
    return gm, gp


def cube_grids(n, L=1.0):
    """The test suites' `fr_grids(n; L)` (`test/fault_response_test.jl:16-17`)."""
    gm = Grid3((-L, -L, -L), (0.0, L, L), (n, n, n))
    gp = Grid3((0.0, -L, -L), (L, L, L), (n, n, n))
    return gm, gp


def lame_lambda(mu, nu):
    """`lame_lambda` (`src/BP8.jl:92`)."""
    return 2 * mu * nu / (1 - 2 * nu)


class FaultElasticity:
    def __init__(self, gm, gp, lam, mu, l_f, system=None, **solver_kwargs):
        sysm = system if system is not None else SplitNodeSystem(gm, gp, lam, mu)
        self.sys = sysm
        Nm, Np = gm.N, gp.N
        self.Ntot = sysm.Ntot
        sel_minus = gm.boundary_nodes(0, True)
        sel_plus = gp.boundary_nodes(0, False)
        n2, n3 = gm.n[1], gm.n[2]
        x2_all = gm.coords(1)
        x3_all = gm.coords(2)
        tol = 1e-9 * max(l_f, 1.0)
        i2 = np.nonzero(np.abs(x2_all) <= l_f + tol)[0]
        i3 = np.nonzero(np.abs(x3_all) <= l_f + tol)[0]
        if len(i2) == 0:
            raise ValueError("no fault nodes inside Omega_f")
        for name, ax, idx in (("x2", x2_all, i2), ("x3", x3_all, i3)):
            if not (abs(ax[idx[0]] + l_f) <= tol and abs(ax[idx[-1]] - l_f) <= tol):
                raise ValueError(f"the elastic grid has no nodes exactly on {name} = ±l_f = ±{l_f}")
        self.i2f, self.i3f = i2, i3
        self.omega = np.array([a + n2 * b for b in i3 for a in i2], dtype=np.int64)
        self.x2f = x2_all[i2].copy()
        self.x3f = x3_all[i3].copy()
        self.l_f = l_f
        import scipy.sparse as sp
        Tm, Tp = sysm.Tm, sysm.Tp
        self.T2 = (0.5 * sp.hstack([sp.hstack(Tm[1]), sp.hstack(Tp[1])], format="csr")).tocsr()
        self.T3 = (0.5 * sp.hstack([sp.hstack(Tm[2]), sp.hstack(Tp[2])], format="csr")).tocsr()
        nf = len(self.omega)
        self.nf = nf
        self.chi_rows = np.empty((nf, 2), dtype=np.int64)
        self.chi_rows_plus = np.empty((nf, 2), dtype=np.int64)
        for k, b in enumerate(self.omega):
            for ci, comp in enumerate((1, 2)):
                self.chi_rows[k, ci] = comp * Nm + sel_minus[b]
                self.chi_rows_plus[k, ci] = 3 * Nm + comp * Np + sel_plus[b]
        self.P = sysm.P
        self.HP_DSAT = sysm.HP_DSAT
        self.rs = CGSolver(sysm.A, **solver_kwargs)

    def build_chi(self, chi, s2, s3):
        chi[:] = 0.0
        chi[self.chi_rows[:, 0]] = -s2 / 2
        chi[self.chi_rows_plus[:, 0]] = s2 / 2
        chi[self.chi_rows[:, 1]] = -s3 / 2
        chi[self.chi_rows_plus[:, 1]] = s3 / 2
        return chi

    def shear_traction(self, s2, s3, solver=None):
        solver = solver if solver is not None else self.rs
        chi = self.build_chi(np.zeros(self.Ntot), np.asarray(s2, float), np.asarray(s3, float))
        u = solver.solve(self.HP_DSAT @ chi)
        U = self.P @ u + chi
        t2 = self.T2 @ U
        t3 = self.T3 @ U
        return t2[self.omega].copy(), t3[self.omega].copy()

    def fault_stiffness(self, cols=None):
        """Dense K (2nf x 2nf), or only the columns `cols` (2nf x len(cols))."""
        nf = self.nf
        cols = range(2 * nf) if cols is None else cols
        cols = list(cols)
        K = np.empty((2 * nf, len(cols)))
        s2 = np.zeros(nf)
        s3 = np.zeros(nf)
        for j, col in enumerate(cols):
            s2[:] = 0.0
            s3[:] = 0.0
            if col < nf:
                s2[col] = 1.0
            else:
                s3[col - nf] = 1.0
            d2, d3 = self.shear_traction(s2, s3)
            K[:nf, j] = d2
            K[nf:, j] = d3
        return K

    def toeplitz_sources(self):
        n2, n3 = len(self.x2f), len(self.x3f)
        ac, bc = (n2 + 1) // 2, (n3 + 1) // 2
        idx = lambda a, b: (b - 1) * n2 + a   # 1-based, as in the reference
        return [idx(ac, bc), idx(1, 1), idx(n2, 1), idx(1, n3), idx(n2, n3)]

    def fault_stiffness_toeplitz(self, columns=None):
        """`columns`, if given, maps each 0-based unit-slip column index to its
        2nf-vector response (so callers can reuse solves); otherwise the 10
        solves are done here."""
        n2, n3 = len(self.x2f), len(self.x3f)
        nf = self.nf
        if nf != n2 * n3:
            raise ValueError("the Toeplitz expansion assumes the Omega_f nodes form a full grid")
        kernel = {}
        for src in self.toeplitz_sources():
            asrc, bsrc = (src - 1) % n2 + 1, (src - 1) // n2 + 1
            if columns is None:
                c2 = self.fault_stiffness([src - 1])[:, 0]
                c3 = self.fault_stiffness([nf + src - 1])[:, 0]
            else:
                c2 = columns[src - 1]
                c3 = columns[nf + src - 1]
            for i in range(1, nf + 1):
                ai, bi = (i - 1) % n2 + 1, (i - 1) // n2 + 1
                sep = (ai - asrc, bi - bsrc)
                if sep in kernel:
                    continue
                kernel[sep] = (c2[i - 1], c2[nf + i - 1], c3[i - 1], c3[nf + i - 1])
        K = np.zeros((2 * nf, 2 * nf))
        for j in range(1, nf + 1):
            aj, bj = (j - 1) % n2 + 1, (j - 1) // n2 + 1
            for i in range(1, nf + 1):
                ai, bi = (i - 1) % n2 + 1, (i - 1) // n2 + 1
                v = kernel.get((ai - aj, bi - bj))
                if v is None:
                    continue
                K[i - 1, j - 1] = v[0]
                K[nf + i - 1, j - 1] = v[1]
                K[i - 1, nf + j - 1] = v[2]
                K[nf + i - 1, nf + j - 1] = v[3]
        return K
