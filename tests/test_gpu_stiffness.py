"""GPU fault stiffness against the oracle, plus the reference's own K tests
(test/fault_response_test.jl, test/bp8_test.jl:27-37) run on the GPU path."""
import numpy as np
import pytest

from oracle.fault import FaultElasticity as OracleFE, cube_grids, bp8_grids, lame_lambda
from oracle.krylov_cg import krylov_cg
from oracle.operators import SplitNodeSystem
from oracle.cref import CRefStiffness

pytestmark = pytest.mark.gpu

LAM, MU = 2.0, 1.0
K_TOL = 1e-8   # relative Frobenius error of K against the tight FP64 oracle


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def small(eqd):
    """n = 11 cubes, l_f = 0.4: nf = 25, 50 columns (test/fault_response_test.jl:80-88)."""
    gm, gp = cube_grids(11)
    ofe = OracleFE(gm, gp, LAM, MU, l_f=0.4)
    K_ref, it, ok = CRefStiffness(ofe).columns(np.arange(2 * ofe.nf), rtol=1e-13)
    assert ok.all()
    return ofe, K_ref


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_K_matches_oracle(eqd, small, precision):
    ofe, K_ref = small
    fe = eqd.FaultElasticity(eqd.cube_grids(11), LAM, MU, 0.4, precision=precision)
    K = eqd.fault_stiffness(fe)
    assert K.shape == K_ref.shape
    assert rel(K, K_ref) < K_TOL
    assert abs(K - K_ref).max() / abs(K_ref).max() < K_TOL
    r = eqd.elastic_solver_report(fe)
    assert r["solves"] == 2 * fe.nf and r["unconverged"] == 0
    assert (np.diag(K) < 0).all()


def test_cg_solve_krylov_parity(eqd):
    """split_node_solve on the Gaussian slip patch: same iteration count as
    Krylov's rule on the assembled matrix (71 at n = 9, 108 at n = 13), same u."""
    for n, want in ((9, 71), (13, 108)):
        gm, gp = cube_grids(n)
        S = SplitNodeSystem(gm, gp, LAM, MU)
        chi = S.build_chi(lambda x2, x3: (np.exp(-(x2 ** 2 + x3 ** 2) / 0.125), 0.0))
        b = S.HP_DSAT @ chi
        u_ref, it_ref, _, _ = krylov_cg(S.A, b, 1e-10)
        assert it_ref == want
        fe = eqd.FaultElasticity(eqd.cube_grids(n), LAM, MU, 0.0, precision="fp64")
        u = eqd.split_node_solve(fe.rs, b)
        rep = eqd.solver_report(fe.rs)
        assert abs(rep["iterations"] - want) <= 1, rep
        assert rep["unconverged"] == 0
        U, U_ref = S.reconstruct_U(u, chi), S.reconstruct_U(u_ref, chi)
        assert rel(U, U_ref) < 1e-8
        assert np.linalg.norm(b - S.A @ u) / np.linalg.norm(b) < 1e-8


def test_reference_fault_response_suite(eqd):
    """test/fault_response_test.jl:43-88 on the GPU path (n = 13, L = 1.2, l_f = 0.6)."""
    fe = eqd.FaultElasticity(eqd.cube_grids(13, L=1.2), LAM, MU, 0.6)
    x2, x3 = eqd.fault_grid_axes(fe)
    assert np.isclose(x2[0], -0.6) and np.isclose(x2[-1], 0.6)
    assert fe.nf == len(x2) * len(x3)
    with pytest.raises(ValueError):
        eqd.FaultElasticity(eqd.cube_grids(13, L=1.2), LAM, MU, 0.55)
    K = eqd.fault_stiffness(fe)
    nf = fe.nf
    k = np.arange(1, nf + 1)
    s2, s3 = 0.01 * np.sin(3 * k), 0.02 * np.cos(2 * k)
    d2, d3 = eqd.shear_traction(fe, s2, s3)
    st = K @ np.concatenate([s2, s3])
    assert np.allclose(st[:nf], d2, rtol=1e-8) and np.allclose(st[nf:], d3, rtol=1e-8)
    assert (np.diag(K) < 0).all()
    d2, _ = eqd.shear_traction(fe, np.ones(nf), np.zeros(nf))
    assert d2.max() < 0
    z2, z3 = eqd.shear_traction(fe, np.zeros(nf), np.zeros(nf))
    assert (z2 == 0).all() and (z3 == 0).all()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_equals_single(eqd, precision):
    _batched_equals_single(eqd, precision, None)


@pytest.mark.parametrize("variant", list(range(11)))
def test_batched_equals_single_every_variant(eqd, variant):
    """Bit-identity holds for every stencil launch variant, including the
    two-columns-per-thread ones (a column's partner lane must not matter)."""
    _batched_equals_single(eqd, "mixed", variant)


def _batched_equals_single(eqd, precision, variant):
    """A column computed in a batch is bit-identical to the same column alone
    (the reference's `threaded K build matches serial`, :100-112)."""
    fe = eqd.FaultElasticity(eqd.cube_grids(11), LAM, MU, 0.4, precision=precision)
    if variant is not None:
        eqd.set_stencil_variant(fe, variant)
    cols = np.arange(2 * fe.nf)
    Kb, itb, stb = eqd.stiffness_columns(fe, cols)
    for c in (0, 7, fe.nf + 3):
        K1, it1, _ = eqd.stiffness_columns(fe, [c])
        assert np.array_equal(K1[:, 0], Kb[:, c])
        assert it1[0] == itb[c]
    Kp, itp, _ = eqd.stiffness_columns(fe, cols[::-1])
    assert np.array_equal(Kp[:, ::-1], Kb)


def test_tune_chunk(eqd, small):
    """The chunk-width tuner measures every width within range, skips the
    rest, and later builds (which then use its width) give the same K bits."""
    fe = eqd.FaultElasticity(eqd.cube_grids(11), LAM, MU, 0.4)
    eqd.set_stencil_variant(fe, 1)
    K0 = eqd.fault_stiffness(fe)
    best, table = eqd.tune_chunk(fe, (8, 16, 32, 1000))
    assert [w for w, _ in table] == [8, 16, 32, 1000]
    assert table[3][1] is None and all(ms > 0 for _, ms in table[:3])
    assert best in (8, 16, 32)
    assert np.array_equal(eqd.fault_stiffness(fe), K0)


def test_toeplitz(eqd, small):
    """test/fault_response_test.jl:128-171."""
    ofe, K_exact = small
    fe = eqd.FaultElasticity(eqd.cube_grids(11), LAM, MU, 0.4)
    Kt = eqd.fault_stiffness_toeplitz(fe)
    Kt_ref = ofe.fault_stiffness_toeplitz(
        columns={c: K_exact[:, c] for c in range(2 * ofe.nf)})
    assert rel(Kt, Kt_ref) < K_TOL
    nf = fe.nf
    n2, n3 = fe.n2f, fe.n3f
    c = ((n3 + 1) // 2 - 1) * n2 + (n2 + 1) // 2 - 1
    assert rel(Kt, K_exact) < 0.05
    assert np.allclose(Kt[:nf, c], K_exact[:nf, c], rtol=1e-6)
    assert np.allclose(Kt[nf:, nf + c], K_exact[nf:, nf + c], rtol=1e-6)
    assert (np.diag(Kt)[:nf] < 0).all()
    assert np.isclose(Kt[c, c], K_exact[c, c], rtol=1e-6)
    assert not np.isclose(Kt[0, 0], K_exact[0, 0], rtol=1e-6)
    assert np.isclose(Kt[0, 0], K_exact[0, 0], rtol=0.05)
    assert eqd.solver_report(fe.rs)["solves"] == 10


def test_bp8_dz100_model(eqd):
    """The reference's BP8 test model (test/bp8_test.jl:14, 27-37): dz = 100,
    L = (800, 800), l_f = 400 -> 17x17x9 per side; published max diag K
    -2.19e8 and asymmetry 0.1827 %."""
    m = eqd.build_model(dz=100.0, L_fault=800.0, L_normal=800.0, stiffness="exact")
    K, nf = m["K"], m["nf"]
    assert K.shape == (2 * nf, 2 * nf)
    assert (np.diag(K) < 0).all()
    assert np.linalg.norm(K - K.T) / np.linalg.norm(K) < 0.01
    assert f"{np.diag(K).max():.2e}" == "-2.19e+08"
    assert f"{100 * np.linalg.norm(K - K.T) / np.linalg.norm(K):.4f}" == "0.1827"
    mu = 32.04e9
    gm, gp = bp8_grids(100.0, 800.0, 800.0)
    ofe = OracleFE(gm, gp, lame_lambda(mu, 0.25), mu, 400.0)
    K_ref, _, ok = CRefStiffness(ofe).columns(np.arange(2 * nf), rtol=1e-13)
    assert rel(K, K_ref) < K_TOL


@pytest.mark.parametrize("n, nvec", [(578, 8), (1155, 64), (2178, 70), (1155, 12), (1155, 20), (4356, 24), (4356, 130),
                                     (6, 5), (7, 40), (130, 3)])
def test_batched_ks(eqd, n, nvec):
    """y = K S for many slip vectors (the blocked K S on the FP64 tensor
    cores: 16-, 32- and 64-vector tiles, odd n on 8-byte loads, more than 64
    vectors over several tiles) against numpy FP64, relative to |K||S|; the
    Fortran-ordered input gives the same bits as the C-ordered one."""
    rng = np.random.default_rng(n)
    K = rng.standard_normal((n, n))
    S = rng.standard_normal((n, nvec))
    M = eqd.KMatrix(K)
    Y = M.gemv(S)
    assert np.array_equal(M.gemv(np.asfortranarray(S)), Y)
    M.close()
    scale = abs(K).dot(abs(S)).max()
    assert Y.shape == (n, nvec)
    assert abs(Y - K @ S).max() <= 1e-13 * scale


@pytest.mark.parametrize("n, nvec", [(4356, 64), (1155, 33), (578, 5)])
def test_kmat_gemv_device(eqd, n, nvec):
    """y = K s on device-resident vectors (torch tensors, the library's
    stream-ordered entry) equals the host entry bit for bit, and numpy FP64
    to 1e-13 of |K||S|; a second call gives the same bits."""
    import torch
    rng = np.random.default_rng(n + nvec)
    K = rng.standard_normal((n, n))
    S = rng.standard_normal((n, nvec))
    M = eqd.KMatrix(K)
    Yh = M.gemv(S)
    s = torch.from_numpy(np.ascontiguousarray(S.T)).cuda()
    y = torch.empty_like(s)
    st = torch.cuda.current_stream()
    M.gemv_device(s, y, stream=st)
    st.synchronize()
    Yd = y.cpu().numpy().T
    y2 = torch.empty_like(s)
    M.gemv_device(s, y2, stream=st)
    st.synchronize()
    M.close()
    assert np.array_equal(Yd, Yh)
    assert torch.equal(y, y2)
    scale = abs(K).dot(abs(S)).max()
    assert abs(Yd - K @ S).max() <= 1e-13 * scale


@pytest.mark.parametrize("n, nvec", [(4356, 8), (2178, 16), (4356, 30), (578, 64)])
def test_ks_load_paths_same_bits(eqd, n, nvec):
    """The K S with 16-byte loads (slips 16-byte aligned) and with 8-byte
    loads (the same slips 8 bytes into a buffer) runs the same tiles, slices
    and k order: the same bits."""
    import torch
    rng = np.random.default_rng(n * nvec)
    K = rng.standard_normal((n, n))
    S = rng.standard_normal((nvec, n))
    M = eqd.KMatrix(K)
    buf = torch.zeros(nvec * n + 1, dtype=torch.float64, device="cuda")
    s_odd = buf[1:].view(nvec, n)
    s_odd.copy_(torch.from_numpy(S))
    s_al = torch.from_numpy(S).cuda()
    assert s_odd.data_ptr() % 16 == 8 and s_al.data_ptr() % 16 == 0
    y_al, y_odd = torch.empty_like(s_al), torch.empty_like(s_al)
    st = torch.cuda.current_stream()
    M.gemv_device(s_al, y_al, stream=st)
    M.gemv_device(s_odd, y_odd, stream=st)
    st.synchronize()
    M.close()
    assert torch.equal(y_al, y_odd)
    Y = y_al.cpu().numpy()
    assert abs(Y - S @ K.T).max() <= 1e-13 * abs(S).dot(abs(K).T).max()


def test_gemv(eqd):
    rng = np.random.default_rng(0)
    n = 578
    K = rng.standard_normal((n, n))
    M = eqd.KMatrix(K)
    s = rng.standard_normal(n)
    y = M.gemv(s)
    assert np.allclose(y, K @ s, rtol=1e-12, atol=1e-12 * abs(K).sum(1).max())
    for nv in (2, 3, 4, 9):  # the GEMV (1-2 vectors) and the tensor-core K S (3+)
        S = rng.standard_normal((n, nv))
        Y = M.gemv(S)
        assert np.allclose(Y, K @ S, rtol=1e-12, atol=1e-10)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_x3_segmented_equals_whole_columns(eqd, precision):
    """FP64-input stencil launches (the FP64 CG apply; the true residual of
    both precisions) of small batches split each column's march along x3
    (one column here runs as 4 segments of 8 planes, 38 columns as 2
    segments of 16); 338 columns run unsplit. The dot products are summed
    per block of 8 march steps whatever the split, so K columns and
    iteration counts are the same bits."""
    fe = eqd.FaultElasticity(eqd.cube_grids(25), LAM, MU, 0.5, precision=precision)   # 25^3 nodes, nf 169
    eqd.set_stencil_variant(fe, 1)
    cols = np.arange(2 * fe.nf)
    Kb, itb, stb = eqd.stiffness_columns(fe, cols)
    assert (stb == 1).all()
    part = cols[::9][:40]
    Km, itm, _ = eqd.stiffness_columns(fe, part)
    assert np.array_equal(Km, Kb[:, part]) and np.array_equal(itm, itb[part])
    for c in (0, fe.nf // 2, 2 * fe.nf - 1):
        K1, it1, _ = eqd.stiffness_columns(fe, [c])
        assert np.array_equal(K1[:, 0], Kb[:, c]) and it1[0] == itb[c]


@pytest.mark.parametrize("dz, L_fault, L_normal, l_f", [(100.0, 800.0, 800.0, 400.0), (40.0, 800.0, 800.0, 200.0),
                                                       (25.0, 200.0, 800.0, 100.0)])
def test_x3_segmented_bp8_grids(eqd, dz, L_fault, L_normal, l_f):
    """The x3 split on the BP8 grids' n1-specialised FP64 instances (n1 = 9:
    17 x 17 x 9, one x2 tile, 162 columns; n1 = 21: 41 x 41 x 21, five x2
    tiles, 242 columns; n1 = 33: 17 x 17 x 33, three edge-partitioned x2
    tiles, 162 columns): single columns (3 or 6 segments) give the same bits
    as the batch (2 segments, or none)."""
    mu = 32.04e9
    fe = eqd.FaultElasticity(eqd.bp8_grids(dz, L_fault, L_normal), eqd.lame_lambda(mu, 0.25), mu, l_f,
                             precision="fp64")
    cols = np.arange(2 * fe.nf)
    Kb, itb, stb = eqd.stiffness_columns(fe, cols)
    assert (stb == 1).all()
    for c in (0, fe.nf // 2 + 3, 2 * fe.nf - 1):
        K1, it1, _ = eqd.stiffness_columns(fe, [c])
        assert np.array_equal(K1[:, 0], Kb[:, c]) and it1[0] == itb[c]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("variant", [1, 3])
def test_fused_direction_update_equals_separate(eqd, precision, variant):
    """The CG direction p = r + beta p formed inside the stencil apply (from
    bulk copies of r and the previous p; opt-in) gives the same bits as the
    separate direction kernel: same K columns, same iteration counts.
    Variant 3 runs two columns per thread."""
    kw = dict(precision=precision)
    fe_f = eqd.FaultElasticity(eqd.cube_grids(13, L=1.2), LAM, MU, 0.6, fuse=True, **kw)
    fe_u = eqd.FaultElasticity(eqd.cube_grids(13, L=1.2), LAM, MU, 0.6, **kw)
    for fe in (fe_f, fe_u):
        eqd.set_stencil_variant(fe, variant)
    cols = np.arange(2 * fe_f.nf)
    Kf, itf, stf = eqd.stiffness_columns(fe_f, cols)
    Ku, itu, stu = eqd.stiffness_columns(fe_u, cols)
    assert (stf == 1).all()
    assert np.array_equal(Kf, Ku) and np.array_equal(itf, itu)
    K1, it1, _ = eqd.stiffness_columns(fe_f, [5])      # one column alone, fused
    assert np.array_equal(K1[:, 0], Ku[:, 5]) and it1[0] == itu[5]


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_slot_refill_equals_full_batch(eqd, precision):
    """With fewer slots than columns, columns enter as earlier ones finish
    (continuous batching); every K column is bit-identical to the one built
    with all columns resident at once, and iteration counts agree."""
    fe_all = eqd.FaultElasticity(eqd.cube_grids(11), LAM, MU, 0.4, precision=precision)
    fe_few = eqd.FaultElasticity(eqd.cube_grids(11), LAM, MU, 0.4, precision=precision, chunk=7)
    eqd.set_stencil_variant(fe_all, 1)
    eqd.set_stencil_variant(fe_few, 1)
    cols = np.arange(2 * fe_all.nf)
    Ka, ita, sta = eqd.stiffness_columns(fe_all, cols)
    Kf, itf, stf = eqd.stiffness_columns(fe_few, cols)
    assert np.array_equal(Ka, Kf)
    assert np.array_equal(ita, itf)
    assert (sta == stf).all()
    r = eqd.solver_report(fe_few.rs)
    assert r["solves"] == len(cols) and r["unconverged"] == 0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_split_halves_equal_single_chain(eqd, precision):
    """A batch of >= 64 columns runs as two halves on two streams whose
    stencil applies alternate; the K columns and iteration counts are the
    same bits as one chain of kernels."""
    kw = dict(precision=precision)
    fe_s = eqd.FaultElasticity(eqd.cube_grids(13, L=1.2), LAM, MU, 0.6, **kw)
    fe_1 = eqd.FaultElasticity(eqd.cube_grids(13, L=1.2), LAM, MU, 0.6, split=False, **kw)
    for fe in (fe_s, fe_1):
        eqd.set_stencil_variant(fe, 1)
    cols = np.arange(2 * fe_s.nf)
    assert len(cols) >= 64
    Ks, its, _ = eqd.stiffness_columns(fe_s, cols)
    K1, it1, _ = eqd.stiffness_columns(fe_1, cols)
    assert np.array_equal(Ks, K1) and np.array_equal(its, it1)


def test_mixed_corner_columns_bp8_scale(eqd):
    """BP8 units at h = 100 m with Omega_f = the whole fault plane: the
    columns next to the corners of the fault have right-hand sides whose
    dot-product terms exceed the FP32 range (|b_i q_i| ~ 5e38); the mixed
    solve must still converge to the FP64 K (dot products in FP64)."""
    mu = 32.04e9
    g = eqd.bp8_grids(100.0, 800.0, 800.0)
    fe = eqd.FaultElasticity(g, eqd.lame_lambda(mu, 0.25), mu, 800.0, precision="mixed", itmax=5000)
    fe64 = eqd.FaultElasticity(g, eqd.lame_lambda(mu, 0.25), mu, 800.0, precision="fp64", rtol=1e-12)
    nf = fe.nf
    corners = [18, 32, 256, 270]
    cols = np.array(corners + [c + nf for c in corners] + [144, nf + 144])
    K, it, st = eqd.stiffness_columns(fe, cols)
    K64 = eqd.stiffness_columns(fe64, cols)[0]
    assert (st == 1).all(), (st, it)
    assert rel(K, K64) < K_TOL


def test_cached_fault_stiffness(eqd, tmp_path):
    """The on-disk K cache built by the GPU in column blocks equals the
    one-call build bit for bit, and a second call loads it."""
    fe = eqd.FaultElasticity(eqd.cube_grids(11), LAM, MU, 0.4)
    eqd.set_stencil_variant(fe, 1)
    K = eqd.fault_stiffness(fe)
    Kc = eqd.cached_fault_stiffness(fe, str(tmp_path), block=16)
    assert np.array_equal(Kc, K)
    solves = eqd.solver_report(fe.rs)["solves"]
    Kc2 = eqd.cached_fault_stiffness(fe, str(tmp_path), block=16)
    assert np.array_equal(Kc2, K) and eqd.solver_report(fe.rs)["solves"] == solves
