"""Assembled split-node SBP-SAT elastic system (CPU oracle, sparse FP64).

TEST INFRASTRUCTURE: the oracle. Only tests, the smoke check and the
benchmark's CPU-baseline leg use it.

Restates, in scipy, the reference's assembly:
  * `elastic_blocks` / `isotropic_lambda_mu`  -> `src/Elasticity.jl:44-89`
  * `traction_blocks`                          -> `src/Elasticity.jl:195-221`
  * `_prolongation`                            -> `src/ElasticitySplitNode.jl:63-68`
  * `fault_node_pairs`                         -> `src/ElasticitySplitNode.jl:85-93`
  * `split_node_system`                        -> `src/ElasticitySplitNode.jl:106-214`
  * `build_chi`, `reconstruct_U`               -> `src/ElasticitySplitNode.jl:223-243`
  * `dof_index_minus/plus`                     -> `src/ElasticitySplitNode.jl:41-42`

Grid functions are flattened exactly as in the reference: x1 fastest
(Julia column-major), component-major within a side, sides concatenated as
[u- (3Nm); u+ (3Np)]. All indices here are 0-based.
"""
import numpy as np
import scipy.sparse as sp

from .sbp import Axis


class Grid3:
    """Equidistant 3D grid on the box [lo, hi] with `n` points per axis
    (Diffinitive `equidistant_grid(lo, hi, n1, n2, n3)`)."""

    def __init__(self, lo, hi, n):
        self.lo = tuple(float(x) for x in lo)
        self.hi = tuple(float(x) for x in hi)
        self.n = tuple(int(x) for x in n)
        self.h = tuple((self.hi[a] - self.lo[a]) / (self.n[a] - 1) for a in range(3))
        self.axes = [Axis(self.n[a], self.h[a]) for a in range(3)]
        self.N = self.n[0] * self.n[1] * self.n[2]

    def coords(self, a):
        return np.linspace(self.lo[a], self.hi[a], self.n[a])

    def lin(self, i1, i2, i3):
        n1, n2, _ = self.n
        return i1 + n1 * (i2 + n2 * i3)

    # -- tensor-product lifting, x1 fastest --------------------------------
    def along(self, a, M):
        """Lift the 1D operator M (acting on axis a) to the full grid."""
        I = [sp.identity(self.n[b], format="csr") for b in range(3)]
        mats = [I[0], I[1], I[2]]
        mats[a] = sp.csr_matrix(M)
        return sp.kron(mats[2], sp.kron(mats[1], mats[0], format="csr"), format="csr")

    def D1(self, a):
        return self.along(a, self.axes[a].D1)

    def D2(self, a):
        return self.along(a, self.axes[a].D2)

    def H(self):
        ax = self.axes
        return sp.kron(ax[2].H, sp.kron(ax[1].H, ax[0].H, format="csr"), format="csr")

    def _boundary_lift(self, a, row):
        """Nb x N operator: the 1D row vector `row` on axis a, identity on the
        other two axes; boundary rows ordered column-major over the remaining
        axes (first remaining axis fastest)."""
        row = sp.csr_matrix(np.asarray(row).reshape(1, -1))
        I = [sp.identity(self.n[b], format="csr") for b in range(3)]
        mats = [I[0], I[1], I[2]]
        mats[a] = row
        return sp.kron(mats[2], sp.kron(mats[1], mats[0], format="csr"), format="csr")

    def e(self, a, upper):
        """`boundary_restriction(g, set, CartesianBoundary{a,Lower/Upper})`."""
        return self._boundary_lift(a, self.axes[a].e(upper))

    def dhat(self, a, upper):
        """Boundary derivative along the fixed +x_a axis (`s * normal_derivative`)."""
        return self._boundary_lift(a, self.axes[a].d(upper))

    def Hb(self, a):
        """`inner_product(boundary_grid(g, bid), set)`."""
        rest = [b for b in range(3) if b != a]
        return sp.kron(self.axes[rest[1]].H, self.axes[rest[0]].H, format="csr")

    def boundary_nodes(self, a, upper):
        """Linear indices of the boundary nodes of face (a, upper), in boundary
        grid order (`boundary_selection`, `src/FaultResponse.jl:57-68`)."""
        e = self.e(a, upper).tocoo()
        sel = np.empty(e.shape[0], dtype=np.int64)
        sel[e.row] = e.col
        return sel


def elastic_blocks(g, lam, mu):
    """M[j][k], the coefficient operator of u_k in equation j
    (`src/Elasticity.jl:80-89`)."""
    D1 = [g.D1(a) for a in range(3)]
    D2 = [g.D2(a) for a in range(3)]
    lap = (D2[0] + D2[1] + D2[2]) * mu
    M = [[None] * 3 for _ in range(3)]
    for j in range(3):
        for k in range(3):
            if j == k:
                M[j][k] = (lap + mu * D2[j] + lam * (D1[j] @ D1[j])).tocsr()
            else:
                M[j][k] = (mu * (D1[j] @ D1[k]) + lam * (D1[j] @ D1[k])).tocsr()
    return M


def elastic_matrix(g, lam, mu):
    M = elastic_blocks(g, lam, mu)
    return sp.bmat(M, format="csr")


def traction_blocks(g, lam, mu, a, upper):
    """T[i][k]: traction sigma_{i,a} on face (a, upper) along the fixed +x_a
    axis, from u_k (`src/Elasticity.jl:195-221`)."""
    e = g.e(a, upper)
    Dk = [g.D1(k) for k in range(3)]
    dh = g.dhat(a, upper)
    Nb = e.shape[0]
    T = [[sp.csr_matrix((Nb, g.N)) for _ in range(3)] for _ in range(3)]
    T[a][a] = (lam * (e @ Dk[a]) + 2 * mu * dh).tocsr()
    for k in range(3):
        if k != a:
            T[a][k] = (lam * (e @ Dk[k])).tocsr()
    for i in range(3):
        if i == a:
            continue
        T[i][a] = (mu * (e @ Dk[i])).tocsr()
        T[i][i] = (mu * dh).tocsr()
    return T


def prolongation(g, a, upper):
    """`-H^-1 e' H_gamma`, the SAT penalty prefactor (N x Nb)."""
    Hinv = sp.diags(1.0 / g.H().diagonal())
    return -(Hinv @ g.e(a, upper).T @ g.Hb(a)).tocsr()


def far_field_nodes(g, fault_upper):
    """Boundary nodes of every face except the fault face (dim 1, `fault_upper`)."""
    s = set()
    for a in range(3):
        for upper in (False, True):
            if a == 0 and upper == fault_upper:
                continue
            s.update(g.boundary_nodes(a, upper).tolist())
    return np.array(sorted(s), dtype=np.int64)


def check_pair(gm, gp):
    if gm.n[1:] != gp.n[1:] or not np.allclose(gm.lo[1:], gp.lo[1:]) or \
            not np.allclose(gm.hi[1:], gp.hi[1:]):
        raise ValueError("g_minus and g_plus must share the (x2, x3) discretization")


def fault_node_pairs(gm, gp):
    """[(Im, Ip)] linear-index pairs on the two fault faces sharing (x2, x3),
    ring excluded (`src/ElasticitySplitNode.jl:85-93`). Ordered like
    `boundary_indices` of the minus fault face, i.e. x2 fastest."""
    check_pair(gm, gp)
    ff = set(far_field_nodes(gm, fault_upper=True).tolist())
    fm = gm.boundary_nodes(0, True)
    fp = gp.boundary_nodes(0, False)
    return [(int(im), int(ip)) for im, ip in zip(fm, fp) if int(im) not in ff]


def dof_minus(gm, comp, I):
    return comp * gm.N + I


def dof_plus(gm, gp, comp, I):
    return 3 * gm.N + comp * gp.N + I


class SplitNodeSystem:
    """`split_node_system(g_minus, g_plus, λ, μ, set)` -> (A, HP_DSAT, P)."""

    def __init__(self, gm, gp, lam, mu):
        check_pair(gm, gp)
        self.gm, self.gp, self.lam, self.mu = gm, gp, float(lam), float(mu)
        Nm, Np = gm.N, gp.N
        self.Nm, self.Np = Nm, Np
        self.Ntot = Ntot = 3 * (Nm + Np)

        Dm = elastic_matrix(gm, lam, mu)
        Dp = elastic_matrix(gp, lam, mu)
        Dmat = sp.block_diag([Dm, Dp], format="csr")

        Tm = traction_blocks(gm, lam, mu, 0, True)
        Tp = traction_blocks(gp, lam, mu, 0, False)
        Pro_m = prolongation(gm, 0, True)
        Pro_p = prolongation(gp, 0, False)
        rows = []
        for j in range(3):
            Tm_j = sp.hstack(Tm[j], format="csr")
            Tp_j = sp.hstack(Tp[j], format="csr")
            blk_m = sp.hstack([0.5 * (Pro_m @ Tm_j), -0.5 * (Pro_m @ Tp_j)], format="csr")
            rows.append((j * Nm, blk_m))
            blk_p = sp.hstack([0.5 * (Pro_p @ Tm_j), -0.5 * (Pro_p @ Tp_j)], format="csr")
            rows.append((3 * Nm + j * Np, blk_p))
        SAT = sp.lil_matrix((Ntot, Ntot))
        SAT = sp.csr_matrix((Ntot, Ntot))
        parts = []
        for r0, blk in rows:
            c = blk.tocoo()
            parts.append((c.row + r0, c.col, c.data))
        I = np.concatenate([p[0] for p in parts])
        J = np.concatenate([p[1] for p in parts])
        V = np.concatenate([p[2] for p in parts])
        SAT = sp.csr_matrix((V, (I, J)), shape=(Ntot, Ntot))
        SAT.sum_duplicates()
        DSAT = (Dmat + SAT).tocsr()
        DSAT.eliminate_zeros()

        # P: identity; far-field rows zero; fault pairs averaged (all 3 comps).
        keep = np.ones(Ntot, dtype=bool)
        for comp in range(3):
            keep[dof_minus(gm, comp, far_field_nodes(gm, True))] = False
            keep[dof_plus(gm, gp, comp, far_field_nodes(gp, False))] = False
        pairs = fault_node_pairs(gm, gp)
        self.pairs = pairs
        pair_rows = np.zeros(Ntot, dtype=bool)
        pi, pj, pv = [], [], []
        for im, ip in pairs:
            for comp in range(3):
                rm = dof_minus(gm, comp, im)
                rp = dof_plus(gm, gp, comp, ip)
                for r in (rm, rp):
                    pair_rows[r] = True
                    pi += [r, r]
                    pj += [rm, rp]
                    pv += [0.5, 0.5]
        diag = np.nonzero(keep & ~pair_rows)[0]
        pi = np.concatenate([np.array(pi, dtype=np.int64), diag])
        pj = np.concatenate([np.array(pj, dtype=np.int64), diag])
        pv = np.concatenate([np.array(pv), np.ones(len(diag))])
        P = sp.csr_matrix((pv, (pi, pj)), shape=(Ntot, Ntot))
        self.P = P
        self.far_field_mask = ~keep

        Hm = gm.H().diagonal()
        Hp = gp.H().diagonal()
        Hdiag = np.concatenate([Hm, Hm, Hm, Hp, Hp, Hp])
        self.Hdiag = Hdiag
        H = sp.diags(Hdiag).tocsr()
        self.Dmat, self.SAT, self.DSAT = Dmat, SAT, DSAT
        self.HP_DSAT = (H @ P @ DSAT).tocsr()
        self.A = (-(self.HP_DSAT @ P)).tocsr()
        self.Tm, self.Tp = Tm, Tp

    # -- helpers used by the fault response and the tests -----------------
    def build_chi(self, slip_fn):
        """`build_chi(g_minus, g_plus, slip_fn)` (`src/ElasticitySplitNode.jl:223-235`)."""
        gm, gp = self.gm, self.gp
        chi = np.zeros(self.Ntot)
        x2 = gp.coords(1)
        x3 = gp.coords(2)
        n1p, n2p, _ = gp.n
        for im, ip in self.pairs:
            i2 = (ip // n1p) % n2p
            i3 = ip // (n1p * n2p)
            s2, s3 = slip_fn(x2[i2], x3[i3])
            chi[dof_plus(gm, gp, 1, ip)] = s2 / 2
            chi[dof_plus(gm, gp, 2, ip)] = s3 / 2
            chi[dof_minus(gm, 1, im)] = -s2 / 2
            chi[dof_minus(gm, 2, im)] = -s3 / 2
        return chi

    def reconstruct_U(self, u, chi):
        return self.P @ u + chi
