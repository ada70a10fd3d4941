"""CPU oracle for the fault-stiffness path.

TEST INFRASTRUCTURE ONLY. Only `tests/`, `__graft_entry__.smoke()` and the
CPU-baseline leg of `bench.py` may import or run anything here, and only as
the checker. The product (`earthquakediffinitive.jl_b200`) never does.

`sbp`, `operators`, `krylov_cg`, `fault` restate the reference's FP64
algorithm (scipy sparse assembly + Krylov-rule CG); `cg_ref.c` restates the
same CG loop in C with OpenMP over columns for the timed CPU baseline.
"""
