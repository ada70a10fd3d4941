"""Time y = K S on device-resident slip vectors (the FP64 tensor-core K S of
`eqd_kmat_gemv_device`, or the GEMV for 1-2 vectors).

    python profile_ks.py --n 13122 --nvec 64 [--reps 10]

K is a seeded N(0, 1) matrix of order n (13,122 = 2 nf at h = 20 m, 4,356
at h = 50 m), the slips N(0, 1). Prints milliseconds per call (CUDA events
on the launching stream, after warm-up), TFLOP/s (2 n^2 nvec per call) and
GB/s of K (8 n^2 bytes per call), and the error against a numpy product on
the first 64 rows. The launch count is small and fixed, so the script is
also the target for single-kernel profiler captures.
"""
import argparse
import sys

import numpy as np

from profile_apply import _package


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=13122)
    ap.add_argument("--nvec", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--reps", type=int, default=10)
    a = ap.parse_args(argv)
    import torch
    eqd = _package()
    rng = np.random.default_rng(a.n)
    K = rng.standard_normal((a.n, a.n))
    S = rng.standard_normal((a.nvec, a.n))       # one slip vector per row
    M = eqd.KMatrix(K)
    s = torch.from_numpy(S).cuda()
    y = torch.empty_like(s)
    st = torch.cuda.current_stream()
    for _ in range(a.warmup):
        M.gemv_device(s, y, stream=st)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(a.reps):
        M.gemv_device(s, y, stream=st)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(1, a.reps)
    Y = y.cpu().numpy()
    ref = S @ K[:64].T                           # rows 0..63 of K S, per vector
    err = abs(Y[:, :64] - ref).max() / abs(ref).max()
    M.close()
    print(f"n {a.n} nvec {a.nvec}: {ms:.4f} ms per call, {2.0 * a.n * a.n * a.nvec / ms / 1e9:.2f} TFLOP/s, "
          f"K at {8.0 * a.n * a.n / ms / 1e6:.0f} GB/s, max rel err (64 rows) {err:.2e}")
    return 0 if err < 1e-12 else 1


if __name__ == "__main__":
    sys.exit(main())
