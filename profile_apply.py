"""Time the stencil apply (the CG iteration's kernel) on a BP8 grid.

    python profile_apply.py --dz 50 --columns 512 [--variant 2]

Grids follow `build_model` (src/BP8.jl:196-206): blocks of
(L_normal/dz+1) x (2 L_fault/dz+1)^2 nodes per side, mu = 32.04 GPa, nu = 0.25.
Prints milliseconds per launch and achieved GB/s over the algorithmic bytes
(one read of x and one write of y per column, in the apply's precision).
The launch count is small and fixed, so the script is also the target for
single-kernel profiler captures.
"""
import argparse
import ctypes as C
import importlib.util
import os
import sys

PKG_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "earthquakediffinitive.jl_b200")


def _package():
    if "eqd_b200" in sys.modules:
        return sys.modules["eqd_b200"]
    spec = importlib.util.spec_from_file_location(
        "eqd_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["eqd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--dz", type=float, default=50.0)
    ap.add_argument("--L-fault", type=float, default=800.0)
    ap.add_argument("--L-normal", type=float, default=400.0)
    ap.add_argument("--columns", type=int, default=512)
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--variant", type=int, default=-1, help="pin an FP32 launch variant (-1: autotune)")
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args(argv)
    eqd = _package()
    lib = eqd._abi.lib()
    mu = 32.04e9
    fe = eqd.FaultElasticity(eqd.bp8_grids(a.dz, a.L_fault, a.L_normal), eqd.lame_lambda(mu, 0.25), mu, a.L_fault)
    if a.variant >= 0:
        eqd.set_stencil_variant(fe, a.variant)
    else:
        print("autotune:", eqd.autotune(fe, min(a.columns, 512)))
    ms, by = C.c_double(), C.c_double()
    prec = eqd._abi.EQD_PREC_MIXED if a.precision == "mixed" else eqd._abi.EQD_PREC_FP64
    eqd._abi.check(lib.eqd_profile_apply(fe.handle, C.c_int32(a.columns), C.c_int32(prec), C.c_int32(a.warmup),
                                         C.c_int32(a.reps), C.byref(ms), C.byref(by)))
    print(f"dz {a.dz} columns {a.columns} precision {a.precision}: {ms.value:.4f} ms/launch, "
          f"{by.value / a.columns / 1e6:.3f} MB/column, {by.value / (ms.value * 1e-3) / 1e9:.1f} GB/s")


if __name__ == "__main__":
    main()
