"""The request server (include/eqd.h `eqd_server_*`): continuous batching of
stiffness-column requests across grids. Each request's K columns must be the
same bits as the same columns built alone (`stiffness_columns`), whatever
else was in flight."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LAM, MU = 2.0, 1.0


def _grids(eqd, precision):
    a = eqd.FaultElasticity(eqd.cube_grids(11), LAM, MU, 0.4, precision=precision)          # nf 25
    b = eqd.FaultElasticity(eqd.cube_grids(13, L=1.2), LAM, MU, 0.6, precision=precision)   # nf 49
    for fe in (a, b):
        eqd.set_stencil_variant(fe, 1)
    return a, b


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_requests_in_the_mix_equal_alone(eqd, precision):
    ra, rb = _grids(eqd, precision)        # reference builds, alone
    sa, sb = _grids(eqd, precision)        # the server's grids
    rng = np.random.default_rng(5)
    with eqd.Server(hbm_budget_bytes=2 << 30, precision=precision) as srv:
        srv.add(sa, slots=8)                # fewer slots than columns: columns queue and refill
        srv.add(sb, slots=16)
        reqs = []
        for k in range(12):
            fe, ref = (sa, ra) if k % 3 else (sb, rb)
            n = int(rng.integers(1, 2 * fe.nf))
            cols = rng.choice(2 * fe.nf, size=n, replace=False)
            reqs.append((srv.submit(fe, cols), ref, cols))
        empty = srv.submit(sa, [])
        for req, ref, cols in reqs:
            K = req.result(timeout=300)
            K_alone, it_alone, _ = eqd.stiffness_columns(ref, cols)
            assert np.array_equal(K, K_alone)
            inf = req.info()
            assert inf["state"] == "done" and inf["unconverged"] == 0
            assert inf["iterations"] == int(it_alone.sum())
            assert inf["t_submit"] <= inf["t_start"] <= inf["t_done"]
        assert empty.result(timeout=10).shape == (2 * sa.nf, 0)
        # The same request again, now alone on the server: same bits.
        req, ref, cols = reqs[0]
        again = srv.submit(req.fe, cols).result(timeout=300)
        assert np.array_equal(again, req.result())


def test_server_owns_its_grids_and_validates(eqd):
    sa, _ = _grids(eqd, "mixed")
    srv = eqd.Server(hbm_budget_bytes=1 << 30)
    srv.add(sa, slots=4)
    with pytest.raises(ValueError):
        eqd.stiffness_columns(sa, [0])              # attached: the server's worker owns it
    with pytest.raises(ValueError):
        srv.submit(sa, [2 * sa.nf])                 # column out of range
    with pytest.raises(ValueError):
        srv.add(sa, slots=4)                        # attached twice
    K = srv.submit(sa, [3, 4]).result(timeout=120)
    srv.close()
    K2 = eqd.stiffness_columns(sa, [3, 4])[0]       # back with its owner
    assert np.array_equal(K, K2)


def test_budget_limits_slots(eqd):
    sa, _ = _grids(eqd, "mixed")
    with eqd.Server(hbm_budget_bytes=1 << 20) as srv:   # 1 MiB: room for a few slots of this grid, not 64
        with pytest.raises(eqd.EqdError):
            srv.add(sa, slots=64)


def test_server_with_jacobi(eqd):
    """Jacobi-preconditioned serving gives the same bits as a Jacobi batch."""
    ra = eqd.FaultElasticity(eqd.cube_grids(11), LAM, MU, 0.4, precond="jacobi")
    sa = eqd.FaultElasticity(eqd.cube_grids(11), LAM, MU, 0.4)
    for fe in (ra, sa):
        eqd.set_stencil_variant(fe, 1)
    cols = np.array([0, 7, 31, 49])
    with eqd.Server(hbm_budget_bytes=1 << 30, precond="jacobi") as srv:
        srv.add(sa, slots=3)
        K = srv.submit(sa, cols).result(timeout=120)
    K_ref, it_ref, _ = eqd.stiffness_columns(ra, cols)
    assert np.array_equal(K, K_ref)
