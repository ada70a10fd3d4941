"""GPU assembly of A and HP_DSAT (`split_node_system`,
src/ElasticitySplitNode.jl:106-214) against the oracle's assembled matrices:
same numerically nonzero pattern, same values."""
import numpy as np
import pytest

from oracle.operators import Grid3, SplitNodeSystem

pytestmark = pytest.mark.gpu

# (n1, n2, n3, x1_extent, x2 range, x3 range, lam, mu, l_f); l_f only selects
# Omega_f (it does not enter the matrices) and must land on grid nodes
CASES = [
    (11, 11, 11, 1.0, (-1, 1), (-1, 1), 2.0, 1.0, 0.4),                  # the reference's test cubes
    (9, 17, 21, 0.8, (-1.6, 1.6), (-2.0, 2.0), 1.5, 0.7, 0.0),           # unequal spacings, periodic colours
    (12, 10, 9, 1.0, (-1, 1), (-1, 1), 2.0, 1.0, 1.0),                   # even / shortest axes
    (9, 17, 17, 800.0, (-800, 800), (-800, 800), 32.04e9, 32.04e9, 400.0),  # BP8 units, h = 100 m
]


def kept(M, rel):
    """CSR with the entries above rel x the row's largest, sorted columns."""
    M = M.tocsr().copy()
    M.sort_indices()
    rmax = abs(M).max(axis=1).toarray().ravel()
    thr = np.repeat(rel * rmax, np.diff(M.indptr))
    M.data[abs(M.data) <= thr] = 0.0
    M.eliminate_zeros()
    return M, rmax


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}x{c[1]}x{c[2]}")
@pytest.mark.parametrize("which", ["A", "HP_DSAT"])
def test_assembly_matches_oracle(eqd, case, which):
    n1, n2, n3, L1, x2, x3, lam, mu, l_f = case
    gm = Grid3((-L1, x2[0], x3[0]), (0.0, x2[1], x3[1]), (n1, n2, n3))
    gp = Grid3((0.0, x2[0], x3[0]), (L1, x2[1], x3[1]), (n1, n2, n3))
    S = SplitNodeSystem(gm, gp, lam, mu)
    ref = S.A if which == "A" else S.HP_DSAT
    fe = eqd.FaultElasticity(eqd.GridPair(n1, n2, n3, L1, x2, x3), lam, mu, l_f)
    M = eqd.assemble_operator(fe, which)
    assert M.shape == ref.shape
    R, rmax = kept(ref, 1e-10)
    G, _ = kept(M, 1e-10)
    # same pattern of clearly nonzero entries, values within 1e-11 of the row's largest
    assert np.array_equal(R.indptr, G.indptr)
    assert np.array_equal(R.indices, G.indices)
    scale = np.repeat(rmax, np.diff(R.indptr))
    assert (abs(G.data - R.data) <= 1e-11 * scale).all()
    # and nothing substantial among the entries either side dropped
    D = (M - ref).tocsr()
    assert abs(D).max() <= 1e-10 * rmax.max()
