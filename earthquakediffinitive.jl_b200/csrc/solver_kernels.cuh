// Batched conjugate-gradient vector kernels, per-column scalar logic,
// traction extraction, Toeplitz expansion, dense GEMV and layout transforms.
//
// Every reduction is per column and in a fixed order (block tree, then the
// partials of that column in index order), so a column's result does not
// depend on which other columns share its batch.
#pragma once
#include "plane_march.cuh"

namespace eqd {

// Per-column CG state (device).
struct ColState {
    double *gamma;      // r.r of the current search direction
    double *beta;
    double *rr_ref;     // true ||r||^2 at the last reliable update (mixed)
    double *tol;        // atol + rtol ||b||
    double *bnorm;
    int *iters;
    int8_t *status;
    int8_t *flag;       // mixed: reliable update pending this iteration
};

struct SolveParams {
    double rtol, atol;
    long long itmax;    // 0 -> 2 * Ntot (the Krylov default)
    double delta;       // mixed: reliable update when ||r|| < delta * ||r_ref||
    int ntiles;         // apply partials per column
    int nchunks;        // update partials per column
    long long colstride;
    long long ntot;     // unpadded DOF count (for itmax default)
    int precond;        // 1: Jacobi (gamma = r.z, z = dinv r); 0: none (z = r)
};

// 16-byte group of vector elements: the CG vector kernels move whole groups
// (a column's storage is a multiple of 4 elements, its start 16-byte
// aligned), two groups of every vector per thread per pass. Beside the
// other half's stencil CTAs an SM has room for one 128-thread vector CTA
// (at most 64 registers a thread), so the bytes each thread keeps in flight
// set the memory parallelism the updates get there.
template <typename T>
struct alignas(16) Group {
    static constexpr int N = 16 / (int)sizeof(T);
    T v[N];
};

// ---------------------------------------------------------------------------
// x += alpha p ; r -= alpha q ; partial r.r   (alpha = gamma / p.q)
// X is the solution accumulator (FP64 for plain CG, FP32 correction d for the
// mixed inner solve).
// ---------------------------------------------------------------------------
// rr_part[col][chunk][2] = (r.r, r.z) partials; r.z = r.r without a
// preconditioner (`dinv` null), z = dinv r with one (Jacobi). A chunk is a
// contiguous range of 16-byte groups of the column.
// Grid-stride over (column, chunk) items: any grid size gives the same
// per-item partial sums, so a small grid (a few CTAs per SM, able to run
// beside the stencil apply) is as exact as one CTA per item.
template <typename T, typename TX>
__global__ void __launch_bounds__(256) cg_update_kernel(TX *__restrict__ x, T *__restrict__ r,
                                                        const T *__restrict__ p, const T *__restrict__ q,
                                                        const double *__restrict__ apply_part, ColState st,
                                                        SolveParams sp, double *__restrict__ rr_part,
                                                        const T *__restrict__ dinv, int ncols) {
    static_assert(sizeof(T) == sizeof(TX), "x and r share the group layout");
    using G = Group<T>;
    using GX = Group<TX>;
    constexpr int V = G::N;
    __shared__ double red[32];
    __shared__ double s_alpha;
    const int nitems = ncols * sp.nchunks;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int col = item / sp.nchunks;
        const int chunk = item % sp.nchunks;
        if (st.status[col] != COL_ACTIVE) continue;
        if (threadIdx.x == 0) {
            double pq = 0.0, pp = 0.0;
            for (int t = 0; t < sp.ntiles; ++t) {
                pq += apply_part[((long long)col * sp.ntiles + t) * 2 + 0];
                pp += apply_part[((long long)col * sp.ntiles + t) * 2 + 1];
            }
            double a = st.gamma[col] / pq;
            if (!(pq > 2.220446049250313e-16 * pp) || !isfinite(a)) a = 0.0;  // breakdown: scalar kernel flags it
            s_alpha = a;
        }
        __syncthreads();
        const double alpha = s_alpha;
        const long long ng = sp.colstride / V;
        const long long gbeg = ng * chunk / sp.nchunks, gend = ng * (chunk + 1) / sp.nchunks;
        const long long off = (long long)col * sp.colstride;
        GX *xg = reinterpret_cast<GX *>(x + off);
        G *rg = reinterpret_cast<G *>(r + off);
        const G *pg = reinterpret_cast<const G *>(p + off);
        const G *qg = reinterpret_cast<const G *>(q + off);
        const G *dg = reinterpret_cast<const G *>(dinv);
        double acc = 0.0, accz = 0.0;
        const T a_t = (T)alpha;
        const TX a_x = (TX)alpha;
        const long long bd = blockDim.x;
        auto one = [&](const G &pi, const G &qi, const G &ri0, const GX &xi0, long long gi) {
            G rn;
            GX xn;
#pragma unroll
            for (int k = 0; k < V; ++k) {
                xn.v[k] = (TX)(xi0.v[k] + a_x * (TX)pi.v[k]);
                rn.v[k] = ri0.v[k] - a_t * qi.v[k];
                acc += (double)rn.v[k] * (double)rn.v[k];
            }
            if (dinv) {
                const G z = dg[gi];
#pragma unroll
                for (int k = 0; k < V; ++k) accz += (double)z.v[k] * (double)rn.v[k] * (double)rn.v[k];
            }
            xg[gi] = xn;
            rg[gi] = rn;
        };
        long long gi = gbeg + threadIdx.x;
        for (; gi + bd < gend; gi += 2 * bd) {
            const G p0 = pg[gi], p1 = pg[gi + bd];
            const G q0 = qg[gi], q1 = qg[gi + bd];
            const G r0 = rg[gi], r1 = rg[gi + bd];
            const GX x0 = xg[gi], x1 = xg[gi + bd];
            one(p0, q0, r0, x0, gi);
            one(p1, q1, r1, x1, gi + bd);
        }
        if (gi < gend) one(pg[gi], qg[gi], rg[gi], xg[gi], gi);
        const double s = block_sum(acc, red);
        double sz = s;
        if (dinv) {
            __syncthreads();
            sz = block_sum(accz, red);
        }
        if (threadIdx.x == 0) {
            rr_part[((long long)col * sp.nchunks + chunk) * 2 + 0] = s;
            rr_part[((long long)col * sp.nchunks + chunk) * 2 + 1] = sz;
        }
        __syncthreads();
    }
}

// p = r + beta p for active columns (only the masked ones when `mask` is set:
// the first direction of columns that just entered the batch).
// With a preconditioner: p = dinv r + beta p.
template <typename T>
__global__ void __launch_bounds__(256) cg_pupdate_kernel(T *__restrict__ p, const T *__restrict__ r, ColState st,
                                                         SolveParams sp, const int8_t *__restrict__ mask,
                                                         const T *__restrict__ dinv, int ncols) {
    using G = Group<T>;
    constexpr int V = G::N;
    const int nitems = ncols * sp.nchunks;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int col = item / sp.nchunks;
        const int chunk = item % sp.nchunks;
        if (st.status[col] != COL_ACTIVE) continue;
        if (mask && !mask[col]) continue;
        const T b = (T)st.beta[col];
        const long long ng = sp.colstride / V;
        const long long gbeg = ng * chunk / sp.nchunks, gend = ng * (chunk + 1) / sp.nchunks;
        const long long off = (long long)col * sp.colstride;
        G *pg = reinterpret_cast<G *>(p + off);
        const G *rg = reinterpret_cast<const G *>(r + off);
        const G *dg = reinterpret_cast<const G *>(dinv);
        const long long bd = blockDim.x;
        auto one = [&](const G &ri, const G &pi, long long gi) {
            G pn;
            if (dinv) {
                const G z = dg[gi];
#pragma unroll
                for (int k = 0; k < V; ++k) pn.v[k] = z.v[k] * ri.v[k] + b * pi.v[k];
            } else {
#pragma unroll
                for (int k = 0; k < V; ++k) pn.v[k] = ri.v[k] + b * pi.v[k];
            }
            pg[gi] = pn;
        };
        long long gi = gbeg + threadIdx.x;
        for (; gi + 3 * bd < gend; gi += 4 * bd) {
            const G r0 = rg[gi], r1 = rg[gi + bd], r2 = rg[gi + 2 * bd], r3 = rg[gi + 3 * bd];
            const G p0 = pg[gi], p1 = pg[gi + bd], p2 = pg[gi + 2 * bd], p3 = pg[gi + 3 * bd];
            one(r0, p0, gi);
            one(r1, p1, gi + bd);
            one(r2, p2, gi + 2 * bd);
            one(r3, p3, gi + 3 * bd);
        }
        for (; gi < gend; gi += bd) one(rg[gi], pg[gi], gi);
    }
}

// ---------------------------------------------------------------------------
// Bulk-staged versions of the two iteration vector kernels. The vectors of a
// (column, chunk) item stream through shared memory in 4 KB tiles by bulk
// copies (two stages, completing on mbarriers), so the bytes in flight cost
// no registers: beside the other half's stencil CTAs an SM has about 8 K
// registers and 110 KB of shared memory left, and these kernels use 32
// registers a thread and 41 KB (update) or 25 KB (direction) a CTA. Same
// per-element arithmetic as the register versions above (which the batch
// setup and the FP64 iterations use); the partial sums of r.r are in a fixed
// order.
// ---------------------------------------------------------------------------
constexpr int kVecStages = 2;
constexpr int kVecTileBytes = 4096;
constexpr size_t kUpdateBulkSmem = 64 + (size_t)kVecStages * 5 * kVecTileBytes;
constexpr size_t kDirBulkSmem = 64 + (size_t)kVecStages * 3 * kVecTileBytes;
// Launched without a shared-memory opt-in: dynamic plus the update kernel's
// static 264 bytes must stay within the default 48 KB.
static_assert(kUpdateBulkSmem + 264 <= 48 * 1024 && kDirBulkSmem <= 48 * 1024, "bulk vector tiles exceed 48 KB");
static_assert(kVecTileBytes % 16 == 0, "bulk copies move multiples of 16 bytes");

// Tiles are counted over all items a CTA processes (`g`): tile g uses stage
// g % kVecStages and completes that stage's mbarrier phase (g / kVecStages) & 1.
__device__ __forceinline__ int vec_stage(unsigned g) { return (int)(g % kVecStages); }
__device__ __forceinline__ unsigned vec_parity(unsigned g) { return (g / kVecStages) & 1u; }

// After a bounded wait on tile g gave up (recorded in *err): wait (bounded)
// once more for tile g and for tile g + 1 if it was issued, so that no copy
// lands in shared memory after the CTA has left.
__device__ __forceinline__ void vec_bulk_drain(uint64_t *bar, unsigned g, bool next_issued, unsigned *err) {
    if (threadIdx.x == 0) {
        mbar_wait_bounded(&bar[vec_stage(g)], vec_parity(g), err);
        if (next_issued) mbar_wait_bounded(&bar[vec_stage(g + 1)], vec_parity(g + 1), err);
    }
    __syncthreads();
}

template <typename T, typename TX>
__global__ void __launch_bounds__(128, 16) cg_update_bulk_kernel(
    TX *__restrict__ x, T *__restrict__ r, const T *__restrict__ p, const T *__restrict__ q,
    const double *__restrict__ apply_part, ColState st, SolveParams sp, double *__restrict__ rr_part,
    const T *__restrict__ dinv, int ncols, unsigned *__restrict__ err) {
    static_assert(sizeof(T) == sizeof(TX), "x and r share the group layout");
    using G = Group<T>;
    using GX = Group<TX>;
    constexpr int V = G::N;
    constexpr int TE = kVecTileBytes / (int)sizeof(T);  // elements per vector tile
    constexpr int TG = TE / V;                          // groups per vector tile
    extern __shared__ __align__(128) unsigned char vsm[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(vsm);
    T *buf = reinterpret_cast<T *>(vsm + 64);  // [stage][p, q, r, x, dinv][TE]
    __shared__ double red[32];
    __shared__ double s_alpha;
    const unsigned nv = dinv ? 5u : 4u;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kVecStages; ++s) mbar_init(&bar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    unsigned g0 = 0;  // tiles this CTA started before the current item
    const int nitems = ncols * sp.nchunks;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int col = item / sp.nchunks;
        const int chunk = item % sp.nchunks;
        if (st.status[col] != COL_ACTIVE) continue;
        if (threadIdx.x == 0) {
            double pq = 0.0, pp = 0.0;
            for (int t = 0; t < sp.ntiles; ++t) {
                pq += apply_part[((long long)col * sp.ntiles + t) * 2 + 0];
                pp += apply_part[((long long)col * sp.ntiles + t) * 2 + 1];
            }
            double a = st.gamma[col] / pq;
            if (!(pq > 2.220446049250313e-16 * pp) || !isfinite(a)) a = 0.0;  // breakdown: scalar kernel flags it
            s_alpha = a;
        }
        __syncthreads();
        const double alpha = s_alpha;
        const long long ng = sp.colstride / V;
        const long long e0 = ng * chunk / sp.nchunks * V, e1 = ng * (chunk + 1) / sp.nchunks * V;
        const long long off = (long long)col * sp.colstride;
        const int ntile = (int)((e1 - e0 + TE - 1) / TE);
        auto issue = [&](int t) {
            const int s = vec_stage(g0 + t);
            const long long b0 = e0 + (long long)t * TE;
            const unsigned bytes = (unsigned)(min((long long)TE, e1 - b0) * (long long)sizeof(T));
            T *dst = buf + (size_t)s * 5 * TE;
            mbar_arrive_expect_tx(&bar[s], nv * bytes);
            bulk_g2s(dst + 0 * TE, p + off + b0, bytes, &bar[s]);
            bulk_g2s(dst + 1 * TE, q + off + b0, bytes, &bar[s]);
            bulk_g2s(dst + 2 * TE, r + off + b0, bytes, &bar[s]);
            bulk_g2s(dst + 3 * TE, x + off + b0, bytes, &bar[s]);
            if (dinv) bulk_g2s(dst + 4 * TE, dinv + b0, bytes, &bar[s]);
        };
        if (threadIdx.x == 0)
            for (int t = 0; t < min(kVecStages, ntile); ++t) issue(t);
        double acc = 0.0, accz = 0.0;
        const T a_t = (T)alpha;
        const TX a_x = (TX)alpha;
        for (int t = 0; t < ntile; ++t) {
            const int s = vec_stage(g0 + t);
            const bool landed = mbar_wait_bounded(&bar[s], vec_parity(g0 + t), err);
            if (!__syncthreads_and(landed)) {
                vec_bulk_drain(bar, g0 + t, t + 1 < ntile, err);
                return;
            }
            const long long b0 = e0 + (long long)t * TE;
            const int ngrp = (int)(min((long long)TE, e1 - b0) / V);
            const G *tile = reinterpret_cast<const G *>(buf + (size_t)s * 5 * TE);
            GX *xg = reinterpret_cast<GX *>(x + off + b0);
            G *rg = reinterpret_cast<G *>(r + off + b0);
            for (int gi = threadIdx.x; gi < ngrp; gi += blockDim.x) {
                const G pi = tile[gi], qi = tile[TG + gi], ri = tile[2 * TG + gi];
                const GX xi = reinterpret_cast<const GX *>(tile)[3 * TG + gi];
                G rn;
                GX xn;
#pragma unroll
                for (int k = 0; k < V; ++k) {
                    xn.v[k] = (TX)(xi.v[k] + a_x * (TX)pi.v[k]);
                    rn.v[k] = ri.v[k] - a_t * qi.v[k];
                    acc += (double)rn.v[k] * (double)rn.v[k];
                }
                if (dinv) {
                    const G z = tile[4 * TG + gi];
#pragma unroll
                    for (int k = 0; k < V; ++k) accz += (double)z.v[k] * (double)rn.v[k] * (double)rn.v[k];
                }
                xg[gi] = xn;
                rg[gi] = rn;
            }
            __syncthreads();  // stage s is read: refill it
            if (threadIdx.x == 0 && t + kVecStages < ntile) issue(t + kVecStages);
        }
        g0 += (unsigned)ntile;
        const double sum = block_sum(acc, red);
        double sz = sum;
        if (dinv) {
            __syncthreads();
            sz = block_sum(accz, red);
        }
        if (threadIdx.x == 0) {
            rr_part[((long long)col * sp.nchunks + chunk) * 2 + 0] = sum;
            rr_part[((long long)col * sp.nchunks + chunk) * 2 + 1] = sz;
        }
        __syncthreads();
    }
}

// p = r + beta p (with a preconditioner: p = dinv r + beta p), bulk-staged.
template <typename T>
__global__ void __launch_bounds__(128, 16) cg_pupdate_bulk_kernel(T *__restrict__ p, const T *__restrict__ r,
                                                                  ColState st, SolveParams sp,
                                                                  const T *__restrict__ dinv, int ncols,
                                                                  unsigned *__restrict__ err) {
    using G = Group<T>;
    constexpr int V = G::N;
    constexpr int TE = kVecTileBytes / (int)sizeof(T);
    constexpr int TG = TE / V;
    extern __shared__ __align__(128) unsigned char vsm[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(vsm);
    T *buf = reinterpret_cast<T *>(vsm + 64);  // [stage][r, p, dinv][TE]
    const unsigned nv = dinv ? 3u : 2u;
    if (threadIdx.x == 0) {
        for (int s = 0; s < kVecStages; ++s) mbar_init(&bar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();
    unsigned g0 = 0;  // tiles this CTA started before the current item
    const int nitems = ncols * sp.nchunks;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int col = item / sp.nchunks;
        const int chunk = item % sp.nchunks;
        if (st.status[col] != COL_ACTIVE) continue;
        const T b = (T)st.beta[col];
        const long long ng = sp.colstride / V;
        const long long e0 = ng * chunk / sp.nchunks * V, e1 = ng * (chunk + 1) / sp.nchunks * V;
        const long long off = (long long)col * sp.colstride;
        const int ntile = (int)((e1 - e0 + TE - 1) / TE);
        auto issue = [&](int t) {
            const int s = vec_stage(g0 + t);
            const long long b0 = e0 + (long long)t * TE;
            const unsigned bytes = (unsigned)(min((long long)TE, e1 - b0) * (long long)sizeof(T));
            T *dst = buf + (size_t)s * 3 * TE;
            mbar_arrive_expect_tx(&bar[s], nv * bytes);
            bulk_g2s(dst + 0 * TE, r + off + b0, bytes, &bar[s]);
            bulk_g2s(dst + 1 * TE, p + off + b0, bytes, &bar[s]);
            if (dinv) bulk_g2s(dst + 2 * TE, dinv + b0, bytes, &bar[s]);
        };
        if (threadIdx.x == 0)
            for (int t = 0; t < min(kVecStages, ntile); ++t) issue(t);
        for (int t = 0; t < ntile; ++t) {
            const int s = vec_stage(g0 + t);
            const bool landed = mbar_wait_bounded(&bar[s], vec_parity(g0 + t), err);
            if (!__syncthreads_and(landed)) {
                vec_bulk_drain(bar, g0 + t, t + 1 < ntile, err);
                return;
            }
            const long long b0 = e0 + (long long)t * TE;
            const int ngrp = (int)(min((long long)TE, e1 - b0) / V);
            const G *tile = reinterpret_cast<const G *>(buf + (size_t)s * 3 * TE);
            G *pg = reinterpret_cast<G *>(p + off + b0);
            for (int gi = threadIdx.x; gi < ngrp; gi += blockDim.x) {
                const G ri = tile[gi], pi = tile[TG + gi];
                G pn;
                if (dinv) {
                    const G z = tile[2 * TG + gi];
#pragma unroll
                    for (int k = 0; k < V; ++k) pn.v[k] = z.v[k] * ri.v[k] + b * pi.v[k];
                } else {
#pragma unroll
                    for (int k = 0; k < V; ++k) pn.v[k] = ri.v[k] + b * pi.v[k];
                }
                pg[gi] = pn;
            }
            __syncthreads();  // stage s is read: refill it
            if (threadIdx.x == 0 && t + kVecStages < ntile) issue(t + kVecStages);
        }
        g0 += (unsigned)ntile;
    }
}

// Mixed precision: fold the FP32 correction into the FP64 solution.
__global__ void __launch_bounds__(256) fold_correction_kernel(double *__restrict__ x, float *__restrict__ d, ColState st,
                                                              SolveParams sp, int ncols) {
    const int nitems = ncols * sp.nchunks;
    for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
        const int col = item / sp.nchunks;
        const int chunk = item % sp.nchunks;
        if (st.status[col] != COL_ACTIVE || !st.flag[col]) continue;
        const long long n = sp.colstride;
        const long long beg = n * chunk / sp.nchunks, end = n * (chunk + 1) / sp.nchunks;
        const long long off = (long long)col * n;
        for (long long i = beg + threadIdx.x; i < end; i += blockDim.x) {
            x[off + i] += (double)d[off + i];
            d[off + i] = 0.f;
        }
    }
}

__device__ __forceinline__ double sum_parts(const double *part, int col, int n, int stride, int k) {
    double s = 0.0;
    for (int t = 0; t < n; ++t) s += part[((long long)col * n + t) * stride + k];
    return s;
}

// After the update: count the iteration, test convergence (plain: Krylov's
// rule on the recursive residual), choose beta, or flag a reliable update.
__global__ void cg_scalar_kernel(ColState st, SolveParams sp, const double *__restrict__ apply_part,
                                 const double *__restrict__ rr_part, int ncols, int mixed) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncols || st.status[col] != COL_ACTIVE) return;
    const double pq = sum_parts(apply_part, col, sp.ntiles, 2, 0);
    const double pp = sum_parts(apply_part, col, sp.ntiles, 2, 1);
    const double rr = sum_parts(rr_part, col, sp.nchunks, 2, 0);
    const double rz = sum_parts(rr_part, col, sp.nchunks, 2, 1);
    const long long itmax = sp.itmax > 0 ? sp.itmax : 2 * sp.ntot;
    const int it = st.iters[col] + 1;
    st.iters[col] = it;
    if (!(pq > 2.220446049250313e-16 * pp)) {  // zero / negative curvature
        if (mixed) {
            st.flag[col] = 1;  // let the true residual decide
            return;
        }
        st.status[col] = COL_BREAKDOWN;
        return;
    }
    if (!isfinite(rr)) {
        st.status[col] = COL_NONFINITE;
        return;
    }
    if (!mixed) {
        if (sqrt(rr) <= st.tol[col]) {
            st.status[col] = COL_CONVERGED;
        } else if (it >= itmax) {
            st.status[col] = COL_MAXITER;
        } else {
            st.beta[col] = rz / st.gamma[col];
            st.gamma[col] = rz;
        }
        return;
    }
    const double tol = st.tol[col];
    if (rr <= tol * tol || rr <= sp.delta * sp.delta * st.rr_ref[col] || it >= itmax) {
        st.flag[col] = 1;
    } else {
        st.beta[col] = rz / st.gamma[col];
        st.gamma[col] = rz;
        st.flag[col] = 0;
    }
}

// After a true-residual evaluation (start of a solve, or a reliable update).
// `first`: this is r0 = b (sets ||b|| and the tolerance).
// `mask` (optional) restricts the kernel to the columns that just entered the
// batch (their r0 = b evaluation).
__global__ void cg_true_residual_kernel(ColState st, SolveParams sp, const double *__restrict__ res_part, int ncols,
                                        int mixed, const int8_t *__restrict__ mask = nullptr) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncols || st.status[col] != COL_ACTIVE) return;
    if (mask ? !mask[col] : (mixed && !st.flag[col])) return;
    const double rr = sum_parts(res_part, col, sp.ntiles, 2, 0);
    const double rz = sp.precond ? sum_parts(res_part, col, sp.ntiles, 2, 1) : rr;
    const int it = st.iters[col];
    if (it == 0) {
        const double bn = sqrt(rr);
        st.bnorm[col] = bn;
        st.tol[col] = sp.atol + sp.rtol * bn;
        st.beta[col] = 0.0;
        st.gamma[col] = rz;
        st.rr_ref[col] = rr;
        st.flag[col] = 0;
        if (rr == 0.0) st.status[col] = COL_CONVERGED;  // x = 0 solves it exactly
        else if (!isfinite(rr)) st.status[col] = COL_NONFINITE;
        else if (bn <= st.tol[col]) st.status[col] = COL_CONVERGED;
        return;
    }
    const long long itmax = sp.itmax > 0 ? sp.itmax : 2 * sp.ntot;
    st.flag[col] = 0;
    if (!isfinite(rr)) {
        st.status[col] = COL_NONFINITE;
    } else if (sqrt(rr) <= st.tol[col]) {
        st.status[col] = COL_CONVERGED;
    } else if (it >= itmax) {
        st.status[col] = COL_MAXITER;
    } else {
        st.beta[col] = rz / st.gamma[col];
        st.gamma[col] = rz;
        st.rr_ref[col] = rr;
    }
}

// Zero the vectors of the masked columns (padding included: the stencil's
// bulk copies read plane padding, which must stay zero).
template <typename T>
__global__ void __launch_bounds__(256) zero_columns_kernel(T *__restrict__ v, long long colstride, int nchunks,
                                                           const int8_t *__restrict__ mask) {
    const int col = blockIdx.x / nchunks;
    const int chunk = blockIdx.x % nchunks;
    if (!mask[col]) return;
    const long long beg = colstride * chunk / nchunks, end = colstride * (chunk + 1) / nchunks;
    T *vc = v + (long long)col * colstride;
    for (long long i = beg + threadIdx.x; i < end; i += blockDim.x) vc[i] = T(0);
}

// Per-column sum of squares of the masked columns, partials laid out as the
// stencil's [column][chunk][2] (slot 0) so cg_true_residual_kernel reads them.
template <typename T>
__global__ void __launch_bounds__(256) column_sumsq_kernel(const T *__restrict__ v, long long colstride, int nchunks,
                                                           const int8_t *__restrict__ mask, double *__restrict__ part,
                                                           const double *__restrict__ dinv = nullptr) {
    const int col = blockIdx.x / nchunks;
    const int chunk = blockIdx.x % nchunks;
    if (!mask[col]) return;
    __shared__ double red[32];
    const long long beg = colstride * chunk / nchunks, end = colstride * (chunk + 1) / nchunks;
    const T *vc = v + (long long)col * colstride;
    double acc = 0.0, accz = 0.0;
    for (long long i = beg + threadIdx.x; i < end; i += blockDim.x) {
        acc += (double)vc[i] * (double)vc[i];
        if (dinv) accz += dinv[i] * (double)vc[i] * (double)vc[i];
    }
    const double s = block_sum(acc, red);
    double sz = 0.0;
    if (dinv) {
        __syncthreads();
        sz = block_sum(accz, red);
    }
    if (threadIdx.x == 0) {
        part[((long long)col * nchunks + chunk) * 2 + 0] = s;
        part[((long long)col * nchunks + chunk) * 2 + 1] = sz;
    }
}

// ---------------------------------------------------------------------------
// Jacobi: diag(A) of A = -H P (D + SAT) P, one thread per DOF, device layout
// (`jacobi_preconditioner`, src/ElasticitySplitNode.jl:352-357, takes it from
// the assembled A). For comp j at a node off the fault face,
//   A_nn = -H_n (mu (D2_1 + D2_2 + D2_3) + mu D2_j + lam W_j)_nn ;
// at a fault pair (m minus, p plus; P averages both inputs and outputs)
//   A_mm = A_pp = -H_m/4 (D_mm + D_pp + 2c (t+ - t-)),
// t = d tau_j / d v_j at the own face node (tau on the fixed +x1 axis);
// far-field rows are zero. W = D1 D1 entries come from the D1 rows.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double d1_entry(const AxisT<double> &a, int n, int i, int k) {
    const int o = k - i;
    if (i < 4) return (o >= -3 && o <= 3) ? a.d1_cl[i][o + 3] : 0.0;
    if (i >= n - 4) return (o >= -3 && o <= 3) ? a.d1_cl[4 + (n - 1 - i)][o + 3] : 0.0;
    return (o >= -2 && o <= 2) ? a.d1_int[o + 2] : 0.0;
}

__device__ __forceinline__ double d2_diag(const AxisT<double> &a, int n, int i) {
    if (i < 4) return a.d2_cl[i][3];
    if (i >= n - 4) return a.d2_cl[4 + (n - 1 - i)][3];
    return a.d2_int[2];
}

__device__ __forceinline__ double w_diag(const AxisT<double> &a, int n, int i) {
    double s = 0.0;
    for (int k = max(i - 3, 0); k <= min(i + 3, n - 1); ++k) s += d1_entry(a, n, i, k) * d1_entry(a, n, k, i);
    return s;
}

__device__ __forceinline__ double hq(const AxisT<double> &a, int n, int i) {
    if (i < 4) return a.wq[i];
    if (i >= n - 4) return a.wq[n - 1 - i];
    return 1.0;
}

__global__ void jacobi_diag_kernel(const __grid_constant__ OpConst<double> C, int n1, int n2, int n3, int PS,
                                   double *__restrict__ diag, double *__restrict__ dinv64, float *__restrict__ dinv32,
                                   unsigned *__restrict__ negative) {
    const long long N = (long long)n1 * n2 * n3;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= 6 * N) return;
    const int sc = (int)(gid / N);
    const long long pt = gid % N;
    const int side = sc / 3, j = sc % 3;
    const int i3 = (int)(pt / ((long long)n1 * n2));
    const int i2 = (int)((pt / n1) % n2);
    const int i1 = (int)(pt % n1);
    const long long idx = ((long long)sc * n3 + i3) * PS + (long long)i2 * n1 + i1;
    const bool ff = (side == 0 && i1 == 0) || (side == 1 && i1 == n1 - 1) || i2 == 0 || i2 == n2 - 1 || i3 == 0 ||
                    i3 == n3 - 1;
    double d = 0.0;
    if (!ff) {
        const int nn[3] = {n1, n2, n3};
        auto Djj = [&](int a1) {
            const int ii[3] = {a1, i2, i3};
            double lap = 0.0;
            for (int a = 0; a < 3; ++a) lap += d2_diag(C.ax[a], nn[a], ii[a]);
            return C.mu * (lap + d2_diag(C.ax[j], nn[j], ii[j])) + C.lam * w_diag(C.ax[j], nn[j], ii[j]);
        };
        const double H = C.hvol * hq(C.ax[0], n1, i1) * hq(C.ax[1], n2, i2) * hq(C.ax[2], n3, i3);
        const bool face = (side == 0 && i1 == n1 - 1) || (side == 1 && i1 == 0);
        if (!face) {
            d = -H * Djj(i1);
        } else {
            const AxisT<double> &A1 = C.ax[0];
            const double dt = j == 0 ? C.lam * (d1_entry(A1, n1, 0, 0) - d1_entry(A1, n1, n1 - 1, n1 - 1)) +
                                           4.0 * C.mu * A1.dlo[0]
                                     : 2.0 * C.mu * A1.dlo[0];
            d = -0.25 * H * (Djj(n1 - 1) + Djj(0) + 2.0 * C.sat_c * dt);
        }
    }
    if (d < 0.0) atomicOr(negative, 1u);
    const double inv = d > 0.0 ? 1.0 / d : 1.0;
    if (diag) diag[idx] = d;
    if (dinv64) dinv64[idx] = inv;
    if (dinv32) dinv32[idx] = (float)inv;
}


// ---------------------------------------------------------------------------
// Traction extraction: K column entries from U = x + chi (FP64).
//   dtau_j(k) = 1/2 (tau_j^-(U^-) + tau_j^+(U^+)),  j = 2, 3,
//   tau_j = mu (D1_j U_1 + dhat U_j) at the fault node
// (`shear_traction!`, src/FaultResponse.jl:201-211, with T2/T3 of :130-132).
// One thread per (column, Omega_f node).
// ---------------------------------------------------------------------------
struct ExtractGeom {
    int n1, n2, n3, PS, nf, i2f0, n2f, i3f0, n3f;
    long long colstride;
    double mu;
};

// Full D1 row r of an axis of length n applied to f(0..n-1).
template <typename F>
__device__ __forceinline__ double d1_row(const AxisT<double> &a, int n, int r, F f) {
    double s = 0.0;
    for (int o = -2; o <= 2; ++o) {
        const int c = r + o;
        if (o != 0 && c >= 0 && c < n) s += a.d1_int[o + 2] * f(c);
    }
    if (r < 4) {
        for (int k = 0; k < 6; ++k) s += a.d1_corrL[r][k] * f(k);
    } else if (r >= n - 4) {
        const int rr = n - 1 - r;
        for (int k = 0; k < 6; ++k) s += a.d1_corrR[rr][k] * f(n - 1 - k);
    }
    return s;
}

// Entry j of the list extracts column slot slots[j] (j itself without a list)
// into K column dstcol[j] (j without a map), leading dimension kld.
__global__ void extract_traction_kernel(const __grid_constant__ OpConst<double> C, ExtractGeom g,
                                        const double *__restrict__ x, ColumnSet cs, double *__restrict__ K,
                                        long long kld, int nlist, const int *__restrict__ slots,
                                        const int *__restrict__ dstcol) {
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int j = (int)(gid / g.nf);
    const int k = (int)(gid % g.nf);
    if (j >= nlist) return;
    const int col = slots ? slots[j] : j;
    const long long kc = dstcol ? dstcol[j] : j;
    const int a = k % g.n2f, b = k / g.n2f;
    const int i2 = g.i2f0 + a, i3 = g.i3f0 + b;
    const int n1 = g.n1, n2 = g.n2, n3 = g.n3;
    const double *xc = x + (long long)col * g.colstride;
    auto chi = [&](int side, int comp, int ii2, int ii3) -> double {
        // chi of this column at the fault node (ii2, ii3), component comp (1, 2).
        if (comp == 0) return 0.0;
        if (ii2 < g.i2f0 || ii2 >= g.i2f0 + g.n2f || ii3 < g.i3f0 || ii3 >= g.i3f0 + g.n3f) return 0.0;
        const int kk = (ii2 - g.i2f0) + g.n2f * (ii3 - g.i3f0);
        double sl;
        if (cs.slip_dense)
            sl = cs.slip_dense[((long long)col * 2 + (comp - 1)) * g.nf + kk];
        else
            sl = (cs.slip_node[col] == kk && cs.slip_comp[col] == comp - 1) ? 1.0 : 0.0;
        return side == 0 ? -0.5 * sl : 0.5 * sl;
    };
    auto U = [&](int side, int comp, int ii1, int ii2, int ii3) -> double {
        double v = xc[((long long)(side * 3 + comp) * n3 + ii3) * g.PS + (long long)ii2 * n1 + ii1];
        const int fi1 = side == 0 ? n1 - 1 : 0;
        if (ii1 == fi1) v += chi(side, comp, ii2, ii3);
        return v;
    };
    double dt[2];
    for (int j = 0; j < 2; ++j) {  // j = 0 -> tau_2 (x2), j = 1 -> tau_3 (x3)
        double t = 0.0;
        for (int side = 0; side < 2; ++side) {
            const int fi1 = side == 0 ? n1 - 1 : 0;
            // tangential derivative of U_1 along x2 (j=0) or x3 (j=1)
            double tang;
            if (j == 0)
                tang = d1_row(C.ax[1], n2, i2, [&](int c) { return U(side, 0, fi1, c, i3); });
            else
                tang = d1_row(C.ax[2], n3, i3, [&](int c) { return U(side, 0, fi1, i2, c); });
            // boundary derivative of U_{j+1} along +x1
            double dh = 0.0;
            for (int q = 0; q < 4; ++q) {
                if (side == 1) dh += C.ax[0].dlo[q] * U(side, j + 1, q, i2, i3);
                else dh -= C.ax[0].dlo[q] * U(side, j + 1, n1 - 1 - q, i2, i3);
            }
            t += g.mu * (tang + dh);
        }
        dt[j] = 0.5 * t;
    }
    K[kc * kld + k] = dt[0];
    K[kc * kld + g.nf + k] = dt[1];
}

// ---------------------------------------------------------------------------
// Toeplitz expansion (`fault_stiffness_toeplitz`, src/FaultResponse.jl:339-393):
// K[i, j] from the response of the first source (priority order) that
// reaches the separation (a_i - a_j, b_i - b_j); unreachable -> 0.
// src_cols: [5 sources][2 (s2, s3)][2nf] responses, src_a/src_b 1-based.
// ---------------------------------------------------------------------------
__global__ void toeplitz_expand_kernel(const double *__restrict__ src_cols, const int *__restrict__ src_a,
                                       const int *__restrict__ src_b, int nsrc, int n2f, int n3f,
                                       double *__restrict__ K) {
    const int nf = n2f * n3f;
    const long long N = 2LL * nf;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (long long)nf * nf) return;
    const int i = (int)(gid % nf), j = (int)(gid / nf);
    const int ai = i % n2f + 1, bi = i / n2f + 1, aj = j % n2f + 1, bj = j / n2f + 1;
    const int da = ai - aj, db = bi - bj;
    double v0 = 0.0, v1 = 0.0, v2 = 0.0, v3 = 0.0;
    for (int s = 0; s < nsrc; ++s) {
        const int a = src_a[s] + da, b = src_b[s] + db;
        if (a >= 1 && a <= n2f && b >= 1 && b <= n3f) {
            const int node = (b - 1) * n2f + (a - 1);
            const double *c2 = src_cols + (long long)(s * 2 + 0) * N;
            const double *c3 = src_cols + (long long)(s * 2 + 1) * N;
            v0 = c2[node];
            v1 = c2[nf + node];
            v2 = c3[node];
            v3 = c3[nf + node];
            break;
        }
    }
    K[(long long)j * N + i] = v0;
    K[(long long)j * N + nf + i] = v1;
    K[(long long)(nf + j) * N + i] = v2;
    K[(long long)(nf + j) * N + nf + i] = v3;
}

// ---------------------------------------------------------------------------
// Dense FP64 GEMV y = K s (K column-major n x n), two passes: column slices
// write partial row sums, then a fixed-order reduction over slices. Vectors
// go four at a time, so one pass over K serves four right-hand sides (the
// time loop's Runge-Kutta stages or an ensemble): K is read ceil(nvec / 4)
// times instead of nvec times.
// VEC2: each thread reads its two rows of a column as one 16-byte load, which
// needs K 16-byte aligned and n even (then every column starts on a 16-byte
// boundary); gemv_vec2_ok() decides. Otherwise the two rows are read as two
// 8-byte loads. Both forms add the same products in the same order.
// ---------------------------------------------------------------------------
__host__ __device__ inline bool gemv_vec2_ok(const void *K, long long n) {
    return (n % 2 == 0) && ((reinterpret_cast<uintptr_t>(K) & 15u) == 0);
}

template <bool VEC2>
__device__ __forceinline__ double2 gemv_load2(const double *__restrict__ K, long long off) {
    if constexpr (VEC2) return *reinterpret_cast<const double2 *>(K + off);
    else return make_double2(K[off], K[off + 1]);
}

template <bool VEC2>
__global__ void __launch_bounds__(256) gemv_partial_kernel(const double *__restrict__ K, const double *__restrict__ s,
                                                           long long n, int nslice, int nvec,
                                                           double *__restrict__ part) {
    constexpr int VB = 4;
    const long long row2 = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 2;
    const int slice = blockIdx.y;
    const long long c0 = n * slice / nslice, c1 = n * (slice + 1) / nslice;
    for (int v0 = 0; v0 < nvec; v0 += VB) {
        const int nv = min(VB, nvec - v0);
        const double *sv[VB];
#pragma unroll
        for (int u = 0; u < VB; ++u) sv[u] = s + (long long)(v0 + (u < nv ? u : 0)) * n;
        double a0[VB], a1[VB];
#pragma unroll
        for (int u = 0; u < VB; ++u) a0[u] = a1[u] = 0.0;
        if (row2 + 1 < n) {
            long long c = c0;
            for (; c + 4 <= c1; c += 4) {  // four columns in flight per thread
                double2 kk[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) kk[j] = gemv_load2<VEC2>(K, (c + j) * n + row2);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
#pragma unroll
                    for (int u = 0; u < VB; ++u) {
                        if (u < nv) {
                            const double sc = sv[u][c + j];
                            a0[u] += kk[j].x * sc;
                            a1[u] += kk[j].y * sc;
                        }
                    }
                }
            }
            for (; c < c1; ++c) {
                const double2 kk = gemv_load2<VEC2>(K, c * n + row2);
#pragma unroll
                for (int u = 0; u < VB; ++u) {
                    if (u < nv) {
                        const double sc = sv[u][c];
                        a0[u] += kk.x * sc;
                        a1[u] += kk.y * sc;
                    }
                }
            }
#pragma unroll
            for (int u = 0; u < VB; ++u) {
                if (u < nv) {
                    part[((long long)(v0 + u) * nslice + slice) * n + row2] = a0[u];
                    part[((long long)(v0 + u) * nslice + slice) * n + row2 + 1] = a1[u];
                }
            }
        } else if (row2 < n) {
            for (long long c = c0; c < c1; ++c) {
                const double kk = K[c * n + row2];
#pragma unroll
                for (int u = 0; u < VB; ++u) a0[u] += kk * sv[u][c];
            }
#pragma unroll
            for (int u = 0; u < VB; ++u)
                if (u < nv) part[((long long)(v0 + u) * nslice + slice) * n + row2] = a0[u];
        }
    }
}

// ---------------------------------------------------------------------------
// Blocked FP64 K S for many slip vectors (Runge-Kutta stages, ensembles) on
// the FP64 tensor cores: K is read once per 64 vectors, and the products run
// as mma.sync m8n8k4 f64 (D = A B + C for an 8 x 4 by 4 x 8 tile per warp
// instruction, 512 flops), which issues 16 times fewer instructions than
// FP64 FMAs on the CUDA cores at the same peak.
//
// CTA tile: 128 rows of K x 16 NT vectors (NT = 1, 2, 4: 16, 32 or 64) over
// the k-range of one column slice, in steps of KB columns of K (16, or 32 for
// the narrow tiles, whose K stream needs more bytes in flight) staged in
// shared memory; each thread loads its share of the next step's tiles into
// registers while the current step is computed. The eight warps form a 4 x 2
// grid of 32-row x 8 NT-vector warp tiles (4 x NT mma tiles, 8 NT FP64
// accumulators per thread). Fragment layout of m8n8k4 f64 (lane = 4 g + t):
// A holds A[g][t], B holds B[t][g], C and D hold D[g][2t], D[g][2t + 1]. A
// 64-bit shared load is served per half-warp (g = 0..3 or 4..7, t = 0..3):
// row strides of 132 and KB + 4 doubles put the 16 doubles of each half on
// distinct banks (A: offsets 4t + g mod 16; B: 20 g + t or 36 g + t), so a
// fragment read takes two wavefronts. Tails (rows past n, columns past the
// slice, vectors past nvec) are zero-filled in registers, so every tile the
// tensor cores see is finite; that includes the columns of a step that lie
// past the slice's end. Slice bounds are multiples of 16 columns (the last
// ends at n). Partial sums go to part[(v * nslice + slice) * n + row], the
// GEMV's layout, and the same fixed-order reduction over slices finishes
// them; the tensor cores' own summation order is fixed, so results are the
// same bits on every run.
// VEC2: 16-byte loads (n even, K and S 16-byte aligned).
// ---------------------------------------------------------------------------
constexpr int kDmmaBM = 128, kDmmaBK = 16;
constexpr int kDmmaAStride = kDmmaBM + 4;  // doubles per k row of the staged K tile

__host__ __device__ inline long long dmma_slice_bound(long long n, int s, int nslice) {
    return s >= nslice ? n : (n * s / nslice) / kDmmaBK * kDmmaBK;
}

__device__ __forceinline__ void dmma_m8n8k4(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

template <bool VEC2, int NT, int KB>
__global__ void __launch_bounds__(256, 2) gemm_ks_dmma_kernel(const double *__restrict__ K,
                                                              const double *__restrict__ S, long long n,
                                                              int nslice, int nvec, double *__restrict__ part) {
    constexpr int BN = 16 * NT;                                  // vectors per CTA
    constexpr int BST = KB + 4;                                  // doubles per vector row of the S tile
    constexpr int BPAIRS = BN * KB / 2;                          // 16-byte pairs of an S tile
    constexpr int BQ2 = (BPAIRS + 255) / 256, BQ1 = BN * KB / 256;
    __shared__ __align__(16) double As[KB * kDmmaAStride];       // [k][row]
    __shared__ __align__(16) double Bs[BN * BST];                // [vector][k]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, t = lane & 3;
    const int wm = warp & 3, wn = warp >> 2;
    const long long row0 = (long long)blockIdx.x * kDmmaBM;
    const int slice = blockIdx.y;
    const int v0 = blockIdx.z * BN;
    const long long c0 = dmma_slice_bound(n, slice, nslice), c1 = dmma_slice_bound(n, slice + 1, nslice);

    // This thread's share of a step: KB / 2 entries of the K tile, up to 4 of the S tile.
    double ra[KB / 2], rb[4];
    auto load = [&](long long k0) {
        if constexpr (VEC2) {
            const int m = 2 * (tid & 63), kb = tid >> 6;
            const long long row = row0 + m;
#pragma unroll
            for (int q = 0; q < KB / 4; ++q) {
                const long long c = k0 + kb + 4 * q;
                double2 v = make_double2(0.0, 0.0);
                if (row < n && c < c1) v = *reinterpret_cast<const double2 *>(K + c * n + row);
                ra[2 * q] = v.x;
                ra[2 * q + 1] = v.y;
            }
#pragma unroll
            for (int q = 0; q < BQ2; ++q) {
                const int pidx = tid + 256 * q, j = pidx / (KB / 2);
                const long long cb = k0 + 2 * (pidx % (KB / 2));
                double2 v = make_double2(0.0, 0.0);
                if (pidx < BPAIRS && v0 + j < nvec && cb < c1)
                    v = *reinterpret_cast<const double2 *>(S + (long long)(v0 + j) * n + cb);
                rb[2 * q] = v.x;
                rb[2 * q + 1] = v.y;
            }
        } else {
            const int m = tid & 127, kb = tid >> 7;
            const long long row = row0 + m;
#pragma unroll
            for (int q = 0; q < KB / 2; ++q) {
                const long long c = k0 + kb + 2 * q;
                ra[q] = (row < n && c < c1) ? K[c * n + row] : 0.0;
            }
#pragma unroll
            for (int q = 0; q < BQ1; ++q) {
                const int e = tid + 256 * q, j = e / KB;
                const long long cb = k0 + (e % KB);
                rb[q] = (v0 + j < nvec && cb < c1) ? S[(long long)(v0 + j) * n + cb] : 0.0;
            }
        }
    };
    auto stage = [&]() {
        if constexpr (VEC2) {
            const int m = 2 * (tid & 63), kb = tid >> 6;
#pragma unroll
            for (int q = 0; q < KB / 4; ++q)
                *reinterpret_cast<double2 *>(&As[(kb + 4 * q) * kDmmaAStride + m]) = make_double2(ra[2 * q], ra[2 * q + 1]);
#pragma unroll
            for (int q = 0; q < BQ2; ++q) {
                const int pidx = tid + 256 * q;
                if (pidx < BPAIRS)
                    *reinterpret_cast<double2 *>(&Bs[(pidx / (KB / 2)) * BST + 2 * (pidx % (KB / 2))]) =
                        make_double2(rb[2 * q], rb[2 * q + 1]);
            }
        } else {
            const int m = tid & 127, kb = tid >> 7;
#pragma unroll
            for (int q = 0; q < KB / 2; ++q) As[(kb + 2 * q) * kDmmaAStride + m] = ra[q];
#pragma unroll
            for (int q = 0; q < BQ1; ++q) {
                const int e = tid + 256 * q;
                Bs[(e / KB) * BST + (e % KB)] = rb[q];
            }
        }
    };
    double acc[4][NT][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    if (c0 < c1) load(c0);
    for (long long k0 = c0; k0 < c1; k0 += KB) {
        stage();
        __syncthreads();
        if (k0 + KB < c1) load(k0 + KB);
#pragma unroll
        for (int kq = 0; kq < KB / 4; ++kq) {
            double a[4], b[NT];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[(kq * 4 + t) * kDmmaAStride + wm * 32 + i * 8 + g];
#pragma unroll
            for (int j = 0; j < NT; ++j) b[j] = Bs[(wn * 8 * NT + j * 8 + g) * BST + kq * 4 + t];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < NT; ++j) dmma_m8n8k4(acc[i][j], a[i], b[j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const long long row = row0 + wm * 32 + i * 8 + g;
        if (row >= n) continue;
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int v = v0 + wn * 8 * NT + j * 8 + 2 * t + e;
                if (v < nvec) part[((long long)v * nslice + slice) * n + row] = acc[i][j][e];
            }
    }
}

__global__ void gemv_reduce_kernel(const double *__restrict__ part, long long n, int nslice, int nvec,
                                   double *__restrict__ y) {
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= n * nvec) return;
    const int v = (int)(gid / n);
    const long long row = gid % n;
    double s = 0.0;
    for (int t = 0; t < nslice; ++t) s += part[((long long)v * nslice + t) * n + row];
    y[gid] = s;
}

// ---------------------------------------------------------------------------
// Sparse assembly of A or HP_DSAT by coloured probing (`split_node_system`,
// src/ElasticitySplitNode.jl:106-214, for callers that want the matrices).
// A DOF j of block sc (side * 3 + comp) at point (j1, j2, j3) has colour
//   ((sc * n1 + j1) * P2 + j2 mod P2) * P3 + j3 mod P3,
// with P = n on short axes and P = 2 R + 1 otherwise, R = the largest
// index distance between a row and a column of a nonzero along x2 and x3
// (measured: 5; R = 6 is used). Applying the operator to the indicator of
// one colour gives, in row i, the entry A[i, j] of the only column j of
// that colour within R of i along x2 and x3 (every colour-mate of j lies
// further away, where A[i, .] is zero).
// ---------------------------------------------------------------------------
struct ProbeGeom {
    int n1, n2, n3, PS;
    long long colstride, N;   // N = n1 n2 n3 points per block
    int P2, P3, R;
    long long ncolors;
};

__host__ __device__ inline long long probe_color(const ProbeGeom &g, int sc, int j1, int j2, int j3) {
    return (((long long)sc * g.n1 + j1) * g.P2 + j2 % g.P2) * g.P3 + j3 % g.P3;
}

// Indicators of colours [c0, c0 + nc), device layout, FP64.
__global__ void probe_fill_kernel(ProbeGeom g, long long c0, int nc, double *__restrict__ x) {
    const long long ntot = 6 * g.N;
    for (long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x; gid < ntot;
         gid += (long long)gridDim.x * blockDim.x) {
        const int sc = (int)(gid / g.N);
        const long long pt = gid % g.N;
        const int i3 = (int)(pt / ((long long)g.n1 * g.n2));
        const int i2 = (int)((pt / g.n1) % g.n2);
        const int i1 = (int)(pt % g.n1);
        const long long c = probe_color(g, sc, i1, i2, i3) - c0;
        if (c >= 0 && c < nc) x[c * g.colstride + ((long long)sc * g.n3 + i3) * g.PS + (long long)i2 * g.n1 + i1] = 1.0;
    }
}

// The column of colour c near row position (i2, i3): its reference index,
// or -1 when that colour has no column within R of the row along x2 / x3.
__device__ __forceinline__ long long probe_column(const ProbeGeom &g, long long c, int i2, int i3) {
    const int r3 = (int)(c % g.P3);
    const int r2 = (int)((c / g.P3) % g.P2);
    const int j1 = (int)((c / ((long long)g.P3 * g.P2)) % g.n1);
    const int sc = (int)(c / ((long long)g.P3 * g.P2 * g.n1));
    auto near_ = [&](int i, int r, int P, int n) -> int {
        if (P == n) return r;  // short axis: every index has its own colour
        const int lo = i - g.R;
        const int j = lo + (((r - lo) % P) + P) % P;
        return (j >= 0 && j < n) ? j : -1;
    };
    const int j2 = near_(i2, r2, g.P2, g.n2);
    const int j3 = near_(i3, r3, g.P3, g.n3);
    if (j2 < 0 || j3 < 0) return -1;
    return (long long)sc * g.N + ((long long)j3 * g.n2 + j2) * g.n1 + j1;
}

// Row i (reference order) takes, for each colour of the chunk, the entry the
// probe produced in that row, into a per-row buffer of kcap (column, value)
// pairs; rowmax tracks the largest magnitude of the row.
__global__ void probe_extract_kernel(ProbeGeom g, long long c0, int nc, const double *__restrict__ y, int kcap,
                                     int *__restrict__ rcnt, int *__restrict__ rcol, double *__restrict__ rval,
                                     double *__restrict__ rmax, unsigned *__restrict__ overflow) {
    const long long ntot = 6 * g.N;
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntot) return;
    const int sc = (int)(i / g.N);
    const long long pt = i % g.N;
    const int i3 = (int)(pt / ((long long)g.n1 * g.n2));
    const int i2 = (int)((pt / g.n1) % g.n2);
    const long long dev = ((long long)sc * g.n3 + i3) * g.PS + (pt % ((long long)g.n1 * g.n2));
    int cnt = rcnt[i];
    double mx = rmax[i];
    for (int k = 0; k < nc; ++k) {
        const long long j = probe_column(g, c0 + k, i2, i3);
        if (j < 0) continue;
        const double v = y[(long long)k * g.colstride + dev];
        if (v == 0.0) continue;
        if (cnt < kcap) {
            rcol[i * kcap + cnt] = (int)j;
            rval[i * kcap + cnt] = v;
        } else {
            atomicOr(overflow, 1u);
        }
        ++cnt;
        mx = fmax(mx, fabs(v));
    }
    rcnt[i] = cnt;
    rmax[i] = mx;
}

// Per row: sort the buffered entries by column and drop those below
// rel_drop times the row's largest (rounding residue of exactly cancelling
// terms); pass 0 writes the kept count, pass 1 the CSR entries at offset
// indptr[i].
__global__ void probe_compact_kernel(long long ntot, int kcap, int *__restrict__ rcnt, int *__restrict__ rcol,
                                     double *__restrict__ rval, const double *__restrict__ rmax, double rel_drop,
                                     int pass, const long long *__restrict__ indptr, int *__restrict__ indices,
                                     double *__restrict__ values, long long *__restrict__ kept) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntot) return;
    const int n = min(rcnt[i], kcap);
    int *cols = rcol + i * kcap;
    double *vals = rval + i * kcap;
    if (pass == 0) {
        for (int a = 1; a < n; ++a) {  // insertion sort by column
            const int cj = cols[a];
            const double vj = vals[a];
            int b = a - 1;
            while (b >= 0 && cols[b] > cj) {
                cols[b + 1] = cols[b];
                vals[b + 1] = vals[b];
                --b;
            }
            cols[b + 1] = cj;
            vals[b + 1] = vj;
        }
    }
    const double thr = rel_drop * rmax[i];
    long long o = pass == 1 ? indptr[i] : 0;
    long long m = 0;
    for (int a = 0; a < n; ++a) {
        if (fabs(vals[a]) <= thr) continue;
        if (pass == 1) {
            indices[o + m] = cols[a];
            values[o + m] = vals[a];
        }
        ++m;
    }
    if (pass == 0) kept[i] = m;
}

// Deterministic pseudo-random fill in [-1, 1) (measurement inputs).
template <typename T>
__global__ void fill_random_kernel(T *__restrict__ v, long long n, unsigned long long seed) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        unsigned long long z = (unsigned long long)i + seed * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        v[i] = (T)((double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0);
    }
}

// ---------------------------------------------------------------------------
// Layout transforms: reference DOF order (per column, Ntot contiguous) <->
// padded device layout. `T`/`U` allow precision conversion.
// ---------------------------------------------------------------------------
template <typename TS, typename TD>
__global__ void ref_to_dev_kernel(const TS *__restrict__ src, TD *__restrict__ dst, int n1, int n2, int n3, int PS,
                                  long long colstride, int ncols) {
    const long long N = (long long)n1 * n2 * n3;
    const long long ntot = 6 * N;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= ntot * ncols) return;
    const int col = (int)(gid / ntot);
    const long long r = gid % ntot;
    const long long sc = r / N, pt = r % N;
    const long long i3 = pt / ((long long)n1 * n2), pl = pt % ((long long)n1 * n2);
    dst[(long long)col * colstride + (sc * n3 + i3) * PS + pl] = (TD)src[gid];
}

template <typename TS, typename TD>
__global__ void dev_to_ref_kernel(const TS *__restrict__ src, TD *__restrict__ dst, int n1, int n2, int n3, int PS,
                                  long long colstride, int ncols) {
    const long long N = (long long)n1 * n2 * n3;
    const long long ntot = 6 * N;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= ntot * ncols) return;
    const int col = (int)(gid / ntot);
    const long long r = gid % ntot;
    const long long sc = r / N, pt = r % N;
    const long long i3 = pt / ((long long)n1 * n2), pl = pt % ((long long)n1 * n2);
    dst[gid] = (TD)src[(long long)col * colstride + (sc * n3 + i3) * PS + pl];
}

}  // namespace eqd
