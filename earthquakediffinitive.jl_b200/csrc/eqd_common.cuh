// Shared definitions for the sm_100a fault-stiffness kernels.
//
// Device vector layout (one column = one right-hand side):
//   v[col][side][comp][i3][plane]      plane = i2 * n1 + i1, padded to PS
// side 0 is the minus block (x1 in [-L, 0], fault at i1 = n1-1), side 1 the
// plus block (x1 in [0, L], fault at i1 = 0). Inside a side this is the
// reference's component-major, x1-fastest ordering (`dof_index_minus/plus`,
// src/ElasticitySplitNode.jl:41-42) with each (x1, x2) plane padded to a
// multiple of 16 bytes so it can be moved with one bulk-async copy. Pad
// entries are zero and stay zero.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define EQD_MAX_N1 40
#define EQD_NSLOT 6          // plane ring: p = s-3 .. s in use, two in flight
#define EQD_HALO 4           // i2 halo rows on each side of a tile (wide D1*D1)
#define EQD_PBLK 8           // x3 march steps per dot-product partial block

namespace eqd {

// Geometry and material of one grid pair (host-side bookkeeping).
struct GridConst {
    int n1, n2, n3;
    int PS;                    // padded plane length (elements), multiple of 4
    long long colstride;       // elements per column = 6 * n3 * PS
    double lam, mu;
    double hvol;               // h1*h2*h3
    double sat_c;              // 0.5 / (h1 * wq1[0]): interface SAT scale
    int i2f0, n2f, i3f0, n3f;  // Omega_f index box on the fault plane
    int nf;
};

// Per-launch column bookkeeping shared by all solver kernels.
struct ColumnSet {
    int ncols;
    const int *slip_node;      // unit-slip Omega_f node per column (or -1)
    const int *slip_comp;      // 0 -> s2, 1 -> s3
    const double *slip_dense;  // optional [ncols][2][nf] dense slip (may be null)
    const int8_t *status;      // per-column solve status (null: all active)
    const int8_t *flag;        // per-column "do this step" flag (null: all)
    const double *dinv;        // MODE_RHS: Jacobi weights (one column, device layout) for
                               // the second partial sum(dinv y^2); null: none
    const void *pold;          // MODE_AF: previous search direction (read), columns as the input
    void *pnew;                // MODE_AF: new search direction r + beta p (written)
    const double *beta;        // MODE_AF: per-column beta
};

enum ColStatus : int8_t {
    COL_ACTIVE = 0,
    COL_CONVERGED = 1,
    COL_MAXITER = 2,
    COL_BREAKDOWN = 3,
    COL_NONFINITE = 4,
    COL_IDLE = 5,
};

// Device error flags (bitmask in a global word).
enum DeviceError : unsigned {
    DERR_MBAR_TIMEOUT = 1u,
    DERR_BAD_LAUNCH = 2u,
};

// ---------------------------------------------------------------------------
// mbarrier + bulk async copy (cp.async.bulk, sm_90+), with bounded waits.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for phase `parity` of `bar` for at most ~2 s of wall time (and at
// most 2^24 polls); on expiry records the failure in *err and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, unsigned *err) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (int i = 0; i < (1 << 24); ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 63) == 63 && global_ns() - t0 > 2000000000ull) break;
    }
    atomicOr(err, DERR_MBAR_TIMEOUT);
    return false;
}

// Orders this thread's prior generic-proxy shared-memory writes before later
// async-proxy (bulk copy) accesses to the same locations.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Global -> shared bulk copy completing on `bar`. dst, src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// ---------------------------------------------------------------------------
// Deterministic block reduction of one double per thread (fixed tree order).
// `scratch` holds >= 32 doubles. Result valid in thread 0.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double block_sum(double v, double *scratch) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    if (warp == 0) {
        v = lane < nw ? scratch[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    return v;
}

}  // namespace eqd
