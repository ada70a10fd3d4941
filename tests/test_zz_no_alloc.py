"""The allocation-free GEMV entry point, `eqd_kmat_gemv_static`.

It exists for callers that cannot allocate device memory (a time loop running
inside CUDA graph capture, or under a framework's own allocator): they pass K,
s and y as device buffers they own, and the library's only scratch is a static
array. This test calls it through the C ABI, twice in a row, and checks it
against the allocating entry point `eqd_kmat_gemv` on the same K and slips.
It lives in its own file, collected last, and passes alone in a fresh process
as well as after the other tests (the static array's set-up happens on the
first call either way).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12   # same bound as the allocating GEMV's test


def test_static_gemv_matches_allocating_gemv(eqd):
    import torch
    lib = eqd._abi.lib()
    rng = np.random.default_rng(42)
    n = 1156
    K = rng.standard_normal((n, n))
    ref = eqd.KMatrix(K)
    dK = torch.from_numpy(np.asfortranarray(K).T.copy()).to("cuda:0")   # column-major bytes
    for call, nvec in enumerate((1, 3)):
        S = rng.standard_normal((n, nvec))
        dS = torch.from_numpy(np.ascontiguousarray(S.T)).to("cuda:0")
        dY = torch.full((nvec, n), float("nan"), dtype=torch.float64, device="cuda:0")
        torch.cuda.synchronize()
        rc = lib.eqd_kmat_gemv_static(C.c_int32(0), C.c_int32(n), C.c_void_p(dK.data_ptr()),
                                      C.c_void_p(dS.data_ptr()), C.c_void_p(dY.data_ptr()),
                                      C.c_int32(nvec), C.c_void_p(0))
        eqd._abi.check(rc)
        torch.cuda.synchronize()
        Y = dY.cpu().numpy().T
        Yref = ref.gemv(S)
        scale = abs(K).dot(abs(S)).max()
        assert np.isfinite(Y).all(), call
        assert abs(Y - Yref.reshape(n, nvec)).max() <= TOL * scale, call
    ref.close()


def _static_gemv(eqd, n, K_ptr, S, stream_handle):
    """One call of the static entry point on device buffers; returns Y (n x nvec)."""
    import torch
    lib = eqd._abi.lib()
    nvec = S.shape[1]
    dS = torch.from_numpy(np.ascontiguousarray(S.T)).to("cuda:0")
    dY = torch.full((nvec, n), float("nan"), dtype=torch.float64, device="cuda:0")
    torch.cuda.synchronize()
    eqd._abi.check(lib.eqd_kmat_gemv_static(C.c_int32(0), C.c_int32(n), C.c_void_p(K_ptr),
                                            C.c_void_p(dS.data_ptr()), C.c_void_p(dY.data_ptr()),
                                            C.c_int32(nvec), C.c_void_p(stream_handle)))
    torch.cuda.synchronize()
    return dY.cpu().numpy().T


def test_static_gemv_scratch_clamp_stream_and_unaligned_k(eqd):
    """n * nvec close to the scratch limit (the column-slice count is clamped
    to fit the array), a caller's stream, and K given as an odd-sized matrix
    at an 8-byte offset (the GEMV then reads K with 8-byte loads)."""
    import torch
    rng = np.random.default_rng(7)
    stream = torch.cuda.Stream(device="cuda:0")
    for n, nvec, offset in ((2048, 200, 0), (1155, 3, 1)):
        K = rng.standard_normal((n, n))
        ref = eqd.KMatrix(K)
        flat = np.concatenate([np.zeros(offset), np.asfortranarray(K).T.ravel()])
        dK = torch.from_numpy(flat).to("cuda:0")
        S = rng.standard_normal((n, nvec))
        for _ in range(2):
            Y = _static_gemv(eqd, n, dK.data_ptr() + 8 * offset, S, stream.cuda_stream)
            Yref = ref.gemv(S).reshape(n, nvec)
            scale = abs(K).dot(abs(S)).max()
            assert np.isfinite(Y).all(), (n, nvec)
            assert abs(Y - Yref).max() <= TOL * scale, (n, nvec)
        ref.close()


def test_static_gemv_rejects_oversize(eqd):
    lib = eqd._abi.lib()
    rc = lib.eqd_kmat_gemv_static(C.c_int32(0), C.c_int32(600000), C.c_void_p(8), C.c_void_p(8), C.c_void_p(8),
                                  C.c_int32(1), C.c_void_p(0))
    assert rc == eqd._abi.EQD_ERR_ARG
    assert b"exceeds the static scratch" in lib.eqd_last_error()
