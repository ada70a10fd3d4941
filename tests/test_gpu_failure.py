"""Non-convergence handling (`split_node_solve`, src/ElasticitySplitNode.jl:
386-393): a column that hits itmax is counted in `unconverged` and warned
about once, not raised; with EQD_FLAG_STRICT the call returns
EQD_ERR_NOT_CONVERGED. The bounded-wait failure path of the stencil is in
test_gpu_ring.py."""
import ctypes as C
import warnings

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LAM, MU = 2.0, 1.0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_itmax_counts_unconverged_and_warns_once(eqd, precision):
    fe = eqd.FaultElasticity(eqd.cube_grids(11), LAM, MU, 0.4, precision=precision, itmax=3)
    cols = np.arange(2 * fe.nf)
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        K, it, st = eqd.stiffness_columns(fe, cols)
        eqd.stiffness_columns(fe, cols[:5])
    assert (st == eqd._abi.COL_MAXITER).all(), st
    assert (it == 3).all(), it
    rep = eqd.elastic_solver_report(fe)
    assert rep["unconverged"] == len(cols) + 5
    assert rep["solves"] == len(cols) + 5
    ours = [x for x in w if issubclass(x.category, RuntimeWarning) and "did not converge" in str(x.message)]
    assert len(ours) == 1
    assert np.isfinite(K).all()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_strict_flag_returns_not_converged(eqd, precision):
    fe = eqd.FaultElasticity(eqd.cube_grids(11), LAM, MU, 0.4, precision=precision, itmax=3)
    lib = eqd._abi.lib()
    opts = fe.rs.opts()
    opts.flags |= eqd._abi.EQD_FLAG_STRICT
    cols = np.arange(6, dtype=np.int32)
    out = np.empty((2 * fe.nf, len(cols)), order="F")
    st = eqd._abi.Stats()
    rc = lib.eqd_stiffness_columns(fe.handle, eqd._abi.ptr(cols), C.c_int32(len(cols)), C.byref(opts),
                                   eqd._abi.ptr(out), None, None, C.byref(st))
    assert rc == eqd._abi.EQD_ERR_NOT_CONVERGED
    assert b"did not converge" in lib.eqd_last_error()
    assert st.unconverged == len(cols)
    # without the flag the same call succeeds and reports the count
    opts.flags &= ~eqd._abi.EQD_FLAG_STRICT
    st = eqd._abi.Stats()
    rc = lib.eqd_stiffness_columns(fe.handle, eqd._abi.ptr(cols), C.c_int32(len(cols)), C.byref(opts),
                                   eqd._abi.ptr(out), None, None, C.byref(st))
    assert rc == eqd._abi.EQD_OK and st.unconverged == len(cols)
