"""GPU K columns on the benchmark grids (BP8 units, mu = lambda = 32.04 GPa),
against the oracle:

  * the reference's published K_self = K[ic, ic] = -4.38404e8 Pa/m at
    dz = 50 m, L = (800, 400), l_f = 400 (PROGRESS.md:586; ic = the centre
    Omega_f node, scripts/bp8_domain_convergence.jl:73-77), through the GPU
    path in FP64 and in mixed precision;
  * h = 50 m with Omega_f = the whole fault plane (2,178 columns): 32 seeded
    columns including edge-ring and corner nodes, against the oracle's C
    restatement at rtol 1e-13;
  * h = 20 m (81 x 81 x 21 per side) and h = 25 m (129 x 129 x 33, L = 1600 /
    800) columns against oracle columns stored in tests/golden/
    config_columns.npz (made by tests/golden/make_config_columns.py).

Tolerance: relative Frobenius and max-entry error <= 1e-8 (the metric's bar).
"""
import os

import numpy as np
import pytest

from oracle.cref import CRefStiffness
from oracle.fault import FaultElasticity as OracleFE, bp8_grids, lame_lambda

pytestmark = pytest.mark.gpu

MU = 32.04e9
LAM = lame_lambda(MU, 0.25)
K_TOL = 1e-8
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "config_columns.npz")


def errs(K, K_ref):
    return (np.linalg.norm(K - K_ref) / np.linalg.norm(K_ref), abs(K - K_ref).max() / abs(K_ref).max())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_K_self_published_value(eqd, precision):
    fe = eqd.FaultElasticity(eqd.bp8_grids(50.0, 800.0, 400.0), LAM, MU, 400.0, precision=precision,
                             rtol=1e-12 if precision == "fp64" else 1e-10)
    x2, x3 = eqd.fault_grid_axes(fe)
    ic = int(np.argmin(abs(x2)) + np.argmin(abs(x3)) * len(x2))
    K, it, st = eqd.stiffness_columns(fe, [ic])
    assert st[0] == 1
    assert f"{K[ic, 0]:.5e}" == "-4.38404e+08"


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_h50_whole_plane_seeded_columns(eqd, precision):
    fe = eqd.FaultElasticity(eqd.bp8_grids(50.0, 800.0, 400.0), LAM, MU, 800.0, precision=precision, itmax=5000)
    nf, n2f = fe.nf, fe.n2f
    corners = [0, n2f - 1, nf - n2f, nf - 1]                 # fault-plane corners
    ring = [n2f // 2, (n2f // 2) * n2f, nf - n2f // 2 - 1]    # edge-ring nodes
    near = [n2f + 1, 2 * n2f - 2, nf - 2 * n2f + 1]          # next to the corners
    base = corners + ring + near
    fixed = base + [c + nf for c in base]                    # both shear components: 20 columns
    rest = np.setdiff1d(np.arange(2 * nf), fixed)
    rand = np.random.default_rng(50).choice(rest, size=32 - len(fixed), replace=False)
    cols = np.sort(np.concatenate([fixed, rand])).astype(np.int32)
    assert len(np.unique(cols)) == 32
    K, it, st = eqd.stiffness_columns(fe, cols)
    assert (st == 1).all(), st
    gm, gp = bp8_grids(50.0, 800.0, 400.0)
    K_ref, _, ok = CRefStiffness(OracleFE(gm, gp, LAM, MU, 800.0)).columns(cols, rtol=1e-13)
    assert ok.all()
    fro, mx = errs(K, K_ref)
    assert fro < K_TOL and mx < K_TOL, (fro, mx)
