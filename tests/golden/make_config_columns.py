"""Generate tests/golden/config_columns.npz: oracle K columns at the BP8
h = 20 m and h = 25 m grids, for the GPU parity tests on those grids.

    python tests/golden/make_config_columns.py [--threads N]

The columns come from the oracle's C restatement of the reference column loop
(assembled CSR A, FP64 Krylov-rule CG at rtol 1e-13), on seeded interior
Omega_f nodes. The grids are `build_model`'s (src/BP8.jl:196-206) with
mu = lambda = 32.04 GPa and Omega_f = the whole fault plane:
  h20: dz = 20 m, L_fault = 800 m, L_normal = 400 m (81 x 81 x 21 per side)
  h25: dz = 25 m, L_fault = 1600 m, L_normal = 800 m (129 x 129 x 33 per side)
"""
import argparse
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.cref import CRefStiffness, max_threads  # noqa: E402
from oracle.fault import FaultElasticity, bp8_grids, lame_lambda  # noqa: E402

MU = 32.04e9
GRIDS = {
    # name: dz, L_fault, L_normal, l_f, columns, seed
    "h20": (20.0, 800.0, 400.0, 800.0, 6, 20),
    "h25": (25.0, 1600.0, 800.0, 1600.0, 3, 25),
}


def interior_columns(n2f, n3f, ncols, seed):
    """Seeded K columns whose Omega_f node is off the fault plane's edge (edge
    nodes are far-field: their right-hand side is zero)."""
    nf = n2f * n3f
    rng = np.random.default_rng(seed)
    picked = []
    while len(picked) < ncols:
        c = int(rng.integers(0, 2 * nf))
        k = c % nf
        a, b = k % n2f, k // n2f
        if 0 < a < n2f - 1 and 0 < b < n3f - 1 and c not in picked:
            picked.append(c)
    return np.array(sorted(picked), dtype=np.int32)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=0)
    args = ap.parse_args()
    nt = args.threads or max_threads()
    out = {}
    for name, (dz, Lf, Ln, lf, ncols, seed) in GRIDS.items():
        t0 = time.time()
        gm, gp = bp8_grids(dz, Lf, Ln)
        fe = FaultElasticity(gm, gp, lame_lambda(MU, 0.25), MU, lf)
        cols = interior_columns(len(fe.x2f), len(fe.x3f), ncols, seed)
        K, it, ok = CRefStiffness(fe).columns(cols, rtol=1e-13, nthreads=nt)
        assert ok.all(), name
        out[f"{name}_cols"] = cols
        out[f"{name}_K"] = K
        out[f"{name}_iters"] = it
        print(f"{name}: {len(cols)} columns, iterations {list(it)}, {time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(os.path.join(HERE, "config_columns.npz"), **out)


if __name__ == "__main__":
    main()
