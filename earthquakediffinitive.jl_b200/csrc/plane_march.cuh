// Matrix-free split-node SBP-SAT elastic operator, one sweep per column.
//
// Computes, for every column of a batch, one of
//   MODE_A   : y = -H P (D + SAT) v          (v already in range(P))
//   MODE_AP  : y = -H P (D + SAT) P x        (generic x; P applied in smem)
//   MODE_RHS : y = +H P (D + SAT) (x + chi)  (x in range(P); chi from the
//              column's slip) = b - A x, the true residual of the CG system
//   MODE_AF  : p' = r + beta p, y = -H P (D + SAT) p'  (the CG direction
//              update fused into the apply: r and p arrive by bulk copies,
//              p' is formed on the landed planes in shared memory and
//              written back; the input pointer is r)
// where, per side, D is the constant-coefficient Navier operator
//   (D v)_j = mu * sum_a D2_a v_j + mu * D2_j v_j + lam * D1_j D1_j v_j
//             + (lam + mu) * sum_{k != j} D1_j D1_k v_k
// (`elastic_blocks`, src/Elasticity.jl:80-89), SAT adds
// c * (tau_j^+ - tau_j^-) with c = 1 / (2 h1 w_0) on both fault faces
// (src/ElasticitySplitNode.jl:149-162 with `_prolongation`, :63-68), and P
// zeroes far-field rows and averages the two sides of each fault node
// (:171-203). The traction tau is `traction_blocks` (src/Elasticity.jl:195-221).
//
// Factorisation used here (exact in real arithmetic, reference composes the
// same D1 matrices):
//   w_1 = mu (2 D2_1 + D2_2 + D2_3) v_1 + D1_1 F_1
//   w_2 = mu (D2_1 + 2 D2_2 + D2_3) v_2 + lam W_2 v_2
//         + (lam + mu) (D1_1 H21 + D1_3 H23)
//   w_3 = mu (D2_1 + D2_2 + 2 D2_3) v_3 + D1_3 F_3
// with G_k = D1_k v_k, F_1 = lam G_1 + (lam+mu)(G_2+G_3),
// F_3 = lam G_3 + (lam+mu)(G_1+G_2), H21 = D1_2 v_1, H23 = D1_2 v_3 and
// W_2 = D1_2 D1_2 (the wide operator, as a 1D matrix).
//
// Work decomposition (one CTA per (column, x2 tile); FP64-input launches of
// small batches also split the x3 march into segments, one CTA each):
//   * one thread per point of the tile: both sides x all n1 points x the
//     tile's x2 rows, grouped into warp-uniform classes (x2-interior rows,
//     x2-closure rows, fault nodes with the two sides in adjacent lanes);
//   * x1 derivatives read the thread's own line from shared memory;
//   * x2 derivatives read neighbouring rows (tile + 4-row halo) from shared;
//   * x3 is marched plane by plane; x3 derivatives come from 7-deep register
//     windows (closure rows reach +-3 planes);
//   * planes arrive through a 6-slot ring filled by cp.async.bulk copies
//     completing on mbarriers, three planes ahead of use;
//   * one CTA barrier per plane (the x1 exchange of F1/H21, double-buffered
//     by step parity); the interface exchange between the two sides of a
//     fault node is a lane shuffle.
#pragma once
#include <type_traits>

#include "eqd_common.cuh"

namespace eqd {

enum { MODE_A = 0, MODE_AP = 1, MODE_RHS = 2, MODE_AF = 3 };

// Per-axis operator tables, built on the host from the exact 1D matrices of
// that axis length (so overlapping closures of short axes are exact).
//   *_cl[r][o]    : full rows of the 4 closure rows at each end, offsets -3..3
//                   (r = 0..3 lower end rows 0..3; r = 4..7 upper end rows
//                   n-1..n-4)
//   *_corrL[r][k] : row r minus the interior stencil, columns k (lower end)
//   *_corrR[r][k] : row n-1-r minus the interior stencil, columns n-1-k
// (rows of the wide operator W span up to 11 columns: both closures reach
// the middle row when n = 11)
template <typename T>
struct AxisT {
    T d1_int[5], d2_int[5], w_int[9];
    T d1_corrL[4][6], d1_corrR[4][6];
    T d2_corrL[4][6], d2_corrR[4][6];
    T w_corrL[6][11], w_corrR[6][11];
    T d1_cl[8][7], d2_cl[8][7];
    T dlo[4];
    T wq[4];
};

template <typename T>
struct OpConst {
    AxisT<T> ax[3];
    T lam, mu, lpm;        // lam + mu
    T sat_c;
    double hvol;
};

// Shared-memory geometry of a kernel compiled for a fixed n1 (N1 > 0): the
// chunk capacity and the exchange-array size are those of the largest tile
// the launch bound admits, so every offset is a compile-time constant.
__host__ __device__ constexpr int march_t2cap(int n1, int maxt) { return maxt / (2 * n1); }
__host__ __device__ constexpr int march_chcap(int n1, int maxt, int elem_bytes) {
    return (((march_t2cap(n1, maxt) + 2 * EQD_HALO) * n1 + 2 * (16 / elem_bytes)) + (16 / elem_bytes) - 1) /
           (16 / elem_bytes) * (16 / elem_bytes);
}

struct MarchGeom {
    int n1, n2, n3, PS;
    long long colstride;
    int ntiles;            // x2 tiles per column
    int t2max;             // rows per tile (upper bound)
    int nblk;              // x3 blocks of EQD_PBLK march steps: dot products are summed per
                           // (column, tile, block), so any x3 segmentation gives the same bits
    int nseg;              // x3 segments per (column, tile) in this launch
    int segblk;            // blocks per segment
    int edge;              // > 0: the first and last tiles have `edge` rows and the
                           // tiles between split the rest evenly; 0: all balanced
    int CH;                // ring chunk capacity (elements) per (side, comp)
    int i2f0, n2f, i3f0, n3f, nf;
};

// x3 derivatives from a 7-deep register window ordered by age: w[6] is the
// newest plane, the centre plane q sits in w[3]. Planes outside the domain
// hold zero and meet zero coefficients.
template <typename T>
__device__ __forceinline__ T x3_d1i(const AxisT<T> &a, const T (&w)[7]) {
    return a.d1_int[0] * w[1] + a.d1_int[1] * w[2] + a.d1_int[3] * w[4] + a.d1_int[4] * w[5];
}
template <typename T>
__device__ __forceinline__ T x3_d2i(const AxisT<T> &a, const T (&w)[7]) {
    return a.d2_int[0] * w[1] + a.d2_int[1] * w[2] + a.d2_int[2] * w[3] + a.d2_int[3] * w[4] + a.d2_int[4] * w[5];
}
// Closure row r (0..3 lower end, 4..7 upper end) of the x3 operators.
template <typename T>
__device__ __forceinline__ T x3_d1c(const AxisT<T> &a, const T (&w)[7], int r) {
    T s = T(0);
#pragma unroll
    for (int o = 0; o < 7; ++o) s += a.d1_cl[r][o] * w[o];
    return s;
}
template <typename T>
__device__ __forceinline__ T x3_d2c(const AxisT<T> &a, const T (&w)[7], int r) {
    T s = T(0);
#pragma unroll
    for (int o = 0; o < 7; ++o) s += a.d2_cl[r][o] * w[o];
    return s;
}

template <typename T>
__device__ __forceinline__ T x3_d1(const AxisT<T> &a, const T (&w)[7], int q, int n3) {
    if (q >= 4 && q <= n3 - 5)
        return a.d1_int[0] * w[1] + a.d1_int[1] * w[2] + a.d1_int[3] * w[4] + a.d1_int[4] * w[5];
    const int r = q < 4 ? q : 4 + (n3 - 1 - q);
    T s = T(0);
#pragma unroll
    for (int o = 0; o < 7; ++o) s += a.d1_cl[r][o] * w[o];
    return s;
}

template <typename T>
__device__ __forceinline__ T x3_d2(const AxisT<T> &a, const T (&w)[7], int q, int n3) {
    if (q >= 4 && q <= n3 - 5)
        return a.d2_int[0] * w[1] + a.d2_int[1] * w[2] + a.d2_int[2] * w[3] + a.d2_int[3] * w[4] +
               a.d2_int[4] * w[5];
    const int r = q < 4 ? q : 4 + (n3 - 1 - q);
    T s = T(0);
#pragma unroll
    for (int o = 0; o < 7; ++o) s += a.d2_cl[r][o] * w[o];
    return s;
}

// Quadrature weight H3/h3 of x3-plane q, zero on the far-field planes
// (q = 0, n3-1) and outside the domain.
template <typename T>
__device__ __forceinline__ T plane_weight(const AxisT<T> &a, int q, int n3) {
    if (q <= 0 || q >= n3 - 1) return T(0);
    if (q < 4) return a.wq[q];
    if (q >= n3 - 4) return a.wq[n3 - 1 - q];
    return T(1);
}

template <typename T>
__device__ __forceinline__ void push7(T (&w)[7], T v) {
#pragma unroll
    for (int k = 0; k < 6; ++k) w[k] = w[k + 1];
    w[6] = v;
}

// x2-direction operators at row r of a chunk pointer `c` (own element), row
// stride n1. The interior stencils are applied everywhere (rows beyond the
// domain read zero); threads on closure rows (`cl`) then add the closure
// corrections, one pass over the rows per input.
template <typename T>
__device__ __forceinline__ T x2_d1i(const AxisT<T> &a, const T *c, int n1) {
    return a.d1_int[0] * c[-2 * n1] + a.d1_int[1] * c[-n1] + a.d1_int[3] * c[n1] + a.d1_int[4] * c[2 * n1];
}

template <typename T>
__device__ __forceinline__ T x2_d2i(const AxisT<T> &a, const T *c, T self, int n1) {
    return a.d2_int[0] * c[-2 * n1] + a.d2_int[1] * c[-n1] + a.d2_int[2] * self + a.d2_int[3] * c[n1] +
           a.d2_int[4] * c[2 * n1];
}

template <typename T>
__device__ __forceinline__ T x2_wi(const AxisT<T> &a, const T *c, T self, int n1) {
    T s = a.w_int[4] * self;
#pragma unroll
    for (int o = 1; o <= 4; ++o) s += a.w_int[4 - o] * c[-o * n1] + a.w_int[4 + o] * c[o * n1];
    return s;
}

// Closure correction geometry of row r for an operator whose closure rows
// are the first / last `ncl` rows: whether row r is a closure row, its first
// boundary row (offset from the own element), the stride toward the
// interior, and the table row. For short axes where both closures reach a
// row, the lower-end table (built from the exact matrix) covers the whole row.
struct X2Corr {
    int off;
    int step;
    int row;
    bool left;
    bool on;
};

__device__ __forceinline__ X2Corr x2_geom(int r, int n1, int n2, int ncl) {
    X2Corr g;
    g.left = r < ncl;
    g.on = g.left || r >= n2 - ncl;
    g.row = g.left ? r : n2 - 1 - r;
    g.off = g.left ? -r * n1 : g.row * n1;
    g.step = g.left ? n1 : -n1;
    return g;
}

// D1 and D2 corrections on one input (closure rows 0..3 / n-4..n-1, 6 columns).
template <typename T>
__device__ __forceinline__ void x2_corr_dd(const AxisT<T> &a, const X2Corr &q, const T *c, T &d1, T &d2) {
    if (!q.on) return;
    const T *t1 = q.left ? a.d1_corrL[q.row] : a.d1_corrR[q.row];
    const T *t2 = q.left ? a.d2_corrL[q.row] : a.d2_corrR[q.row];
    const T *b = c + q.off;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const T x = b[k * q.step];
        d1 += t1[k] * x;
        d2 += t2[k] * x;
    }
}

// D1-only correction (for H23 at ingest).
template <typename T>
__device__ __forceinline__ void x2_corr_d1(const AxisT<T> &a, const X2Corr &q, const T *c, T &d1) {
    if (!q.on) return;
    const T *t1 = q.left ? a.d1_corrL[q.row] : a.d1_corrR[q.row];
    const T *b = c + q.off;
#pragma unroll
    for (int k = 0; k < 6; ++k) d1 += t1[k] * b[k * q.step];
}

// W correction (closure rows 0..5 / n-6..n-1, 11 columns).
template <typename T>
__device__ __forceinline__ void x2_corr_w(const AxisT<T> &a, const X2Corr &q, const T *c, T &w) {
    if (!q.on) return;
    const T *tw = q.left ? a.w_corrL[q.row] : a.w_corrR[q.row];
    const T *b = c + q.off;
#pragma unroll
    for (int k = 0; k < 11; ++k) w += tw[k] * b[k * q.step];
}

// N1 > 0 compiles the kernel for that fixed number of x1 points per side
// (every shared-memory offset becomes an immediate); N1 = 0 reads it from g.
// L = columns per thread: each thread carries the same point of L columns
// (own plane ring and exchange arrays per column), so every per-thread cost
// (addressing, branches, barriers, coefficient loads) is shared by L
// right-hand sides and the L independent arithmetic chains interleave.
template <typename T, typename TO, int MODE, int MAXT, int N1, int L>
__global__ void __launch_bounds__(MAXT, 1)
plane_march_kernel(const __grid_constant__ OpConst<T> C, const __grid_constant__ MarchGeom g,
                   const T *__restrict__ in, TO *__restrict__ out, ColumnSet cs,
                   double *__restrict__ partials, unsigned *__restrict__ err) {
    // FP64-input instances (the FP64 solve, and the true residual of both
    // precisions) sum their dot products per x3 step block and can split a
    // column's march along x3; FP32 instances (the mixed-precision CG apply)
    // sum per (column, tile) over the whole march.
    constexpr bool SEG = sizeof(T) == 8;
    // CTA -> (column group, x2 tile, x3 segment).
    const int nseg = SEG ? g.nseg : 1;
    const int per_grp = g.ntiles * nseg;
    const int grp = blockIdx.x / per_grp;
    const int tile = (blockIdx.x % per_grp) / nseg;
    const int seg = SEG ? blockIdx.x % nseg : 0;
    // Columns of this CTA; an inactive lane (past the end, not active, or not
    // flagged) mirrors an active one's input and stores nothing.
    int colv[L];
    bool act[L];
    int first = -1;
#pragma unroll
    for (int l = 0; l < L; ++l) {
        const int c = grp * L + l;
        bool a = c < cs.ncols;
        if (a && cs.status && cs.status[c] != COL_ACTIVE) a = false;
        if (a && cs.flag && !cs.flag[c]) a = false;
        colv[l] = c;
        act[l] = a;
        if (a && first < 0) first = c;
    }
    if (first < 0) return;
#pragma unroll
    for (int l = 0; l < L; ++l)
        if (!act[l]) colv[l] = first;

    const int n1 = N1 > 0 ? N1 : g.n1;
    const int n2 = g.n2, n3 = g.n3;
    // x3 segment (FP64-input instances). March step s ingests plane s, does
    // the in-plane work and finishes components 1, 2 of plane p = s - 3, and
    // finishes component 3 of plane z = s - 6. Steps are grouped in blocks of
    // EQD_PBLK: step s belongs to block min((s - 3) / EQD_PBLK, nblk - 1), and
    // the dot-product contributions of a block's steps are summed together. A
    // segment owns whole blocks [blk0, blk0 + nbs): steps [q0 + 3, q1 + 3)
    // (the last segment: to n3 + 6), so it stores components 1, 2 of planes
    // [q0, q1) and component 3 of planes [q0 - 3, q1 - 3). Before its first
    // owned step it marches from plane q0 - 9 or earlier to fill the windows
    // (z = q0 - 3 needs F3 of planes q0 - 6 .. q0, each from planes
    // p - 3 .. p + 3); the start is a multiple of the ring depth, so plane q
    // always uses ring slot q % EQD_NSLOT. FP32 instances march the whole
    // column: steps [0, n3 + 6).
    const int q0 = SEG ? seg * g.segblk * EQD_PBLK : 0;
    const int q1 = SEG ? min(q0 + g.segblk * EQD_PBLK, n3) : n3;
    const int blk0 = q0 / EQD_PBLK;
    const int nbs = (q1 - q0 + EQD_PBLK - 1) / EQD_PBLK;   // blocks of this segment
    const int o_beg = q0 + 3;                               // owned steps: [o_beg, s_end)
    const int s_end = q1 == n3 ? n3 + 6 : q1 + 3;
    const int s_beg = q0 > 9 ? (q0 - 9) / EQD_NSLOT * EQD_NSLOT : 0;
    const unsigned ph0 = (unsigned)(s_beg / EQD_NSLOT) & 1u;  // mbarrier phase parity of plane s_beg
    const int ing_end = min(n3, s_end);                     // planes ingested: [s_beg, ing_end)
    const int p_lo = max(q0 - 6, 0);                        // in-plane work: p in [p_lo, p_hi)
    const int p_hi = min(n3, s_end - 3);
    int a0, a1;
    if (g.edge > 0) {
        // Edge tiles hold every closure row (and read the 11 rows the wide
        // operator's closures reach); the middle tiles only need the halo.
        if (tile == 0) {
            a0 = 0;
            a1 = g.edge;
        } else if (tile == g.ntiles - 1) {
            a0 = n2 - g.edge;
            a1 = n2;
        } else {
            const int m = n2 - 2 * g.edge, nm = g.ntiles - 2, k = tile - 1;
            a0 = g.edge + (int)((long long)k * m / nm);
            a1 = g.edge + (int)((long long)(k + 1) * m / nm);
        }
    } else {
        a0 = (int)((long long)tile * n2 / g.ntiles);
        a1 = (int)((long long)(tile + 1) * n2 / g.ntiles);
    }
    constexpr int AE = 16 / (int)sizeof(T);  // elements per 16 bytes

    // Row range copied per plane (tile + halo, clipped), 16-byte aligned.
    const int r0 = max(a0 - EQD_HALO, 0), r1 = min(a1 + EQD_HALO, n2);
    const int lo_el = (a0 - EQD_HALO) * n1;
    const int base = lo_el >= 0 ? (lo_el / AE) * AE : -(((-lo_el) + AE - 1) / AE) * AE;
    const int e0 = ((r0 * n1) / AE) * AE;
    const int e1 = ((r1 * n1 + AE - 1) / AE) * AE;
    const unsigned bytes = (unsigned)((e1 - e0) * (int)sizeof(T));

    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem_raw);
    volatile int *s_dead = reinterpret_cast<volatile int *>(smem_raw + 56);  // [2], by step parity
    double *red = reinterpret_cast<double *>(smem_raw + 64);
    T *ring = reinterpret_cast<T *>(smem_raw + 64 + 32 * 8);  // [L][slot][side*3+comp][CH]
    constexpr int CHc = N1 > 0 ? march_chcap(N1, MAXT, (int)sizeof(T)) : 0;
    constexpr int NPc = N1 > 0 ? 2 * N1 * march_t2cap(N1, MAXT) : 0;
    const int CH = N1 > 0 ? CHc : g.CH;                     // chunk capacity per (side, comp)
    const int RS = EQD_NSLOT * 6 * CH;                        // ring size per column
    const int NP = N1 > 0 ? NPc : 2 * n1 * g.t2max;           // exchange entries per parity
    T *xF1 = ring + (size_t)L * RS;                           // [L][2 (step parity)][NP]
    T *xH21 = xF1 + (size_t)L * 2 * NP;                       // [L][2][NP]
    // Per-(block, warp) dot-product sums (FP64-input instances):
    // [L][segblk][warps][2].
    const int nwarps = (int)(blockDim.x >> 5);
    double *rblk = reinterpret_cast<double *>(
        (reinterpret_cast<uintptr_t>(xH21 + (size_t)L * 2 * NP) + 15) & ~(uintptr_t)15);
    // MODE_AF: ring of the r planes, [L][slot][side*3+comp][CH], beside the
    // ring of p planes (128-byte aligned, after the block sums).
    T *rring = reinterpret_cast<T *>(
        (reinterpret_cast<uintptr_t>(rblk) + (SEG ? (size_t)L * g.nblk * nwarps * 2 * sizeof(double) : 0) + 127) &
        ~(uintptr_t)127);

    // ---- thread -> point: warp-homogeneous classes --------------------------
    // class 0: x2-interior rows, not on the fault; class 1: x2-closure rows,
    // not on the fault; class 2: fault nodes, the two sides of a node in
    // adjacent lanes (partners exchange by shuffle).
    const int tid = threadIdx.x;
    const int T2 = a1 - a0;
    const int ilo = min(max(a0, 6), a1);
    const int ihi = max(min(a1, n2 - 6), ilo);
    const int nI = ihi - ilo;
    const int per = 2 * (n1 - 1);
    const int C0 = nI * per, C1 = (T2 - nI) * per, C2 = 2 * T2;  // threads per class
    // Each class starts on a warp boundary when the CTA has the threads for
    // it: a warp that mixed classes would pay for both classes' extra work
    // (x2 closure corrections and the fault-face SAT path), and the
    // per-plane barrier waits for the slowest warp.
    const int P0 = (C0 + 31) & ~31, P1 = (C1 + 31) & ~31;
    const bool aligned = P0 + P1 + C2 <= (int)blockDim.x;
    const int B0 = aligned ? P0 : C0;           // first thread of class 1
    const int B1 = B0 + (aligned ? P1 : C1);    // first thread of class 2 (even)
    int side = 0, i2 = a0, i1 = 0, cls = 3;
    if (tid < C0) {
        const int rr = tid / per, q = tid % per;
        side = q / (n1 - 1);
        const int j = q % (n1 - 1);
        i1 = side == 0 ? j : j + 1;
        i2 = ilo + rr;
        cls = 0;
    } else if (tid >= B0 && tid < B0 + C1) {
        const int k = tid - B0;
        const int rr = k / per, q = k % per;
        side = q / (n1 - 1);
        const int j = q % (n1 - 1);
        i1 = side == 0 ? j : j + 1;
        const int nlow = ilo - a0;
        i2 = rr < nlow ? a0 + rr : ihi + (rr - nlow);
        cls = 1;
    } else if (tid >= B1 && tid < B1 + C2) {
        const int k = tid - B1;
        side = k & 1;
        i1 = side == 0 ? n1 - 1 : 0;
        i2 = a0 + (k >> 1);
        cls = 2;
    }
    const bool valid = cls < 3;
    const bool is_face = cls == 2;
    const bool x2cl = cls != 0 && (i2 < 6 || i2 >= n2 - 6);
    const X2Corr gdd = x2_geom(i2, n1, n2, 4);
    const X2Corr gw = x2_geom(i2, n1, n2, 6);
    const unsigned facemask = __ballot_sync(0xffffffffu, is_face);
    const int i2l = i2 - a0;
    const int t2cap = N1 > 0 ? march_t2cap(N1, MAXT) : g.t2max;
    const int pidx = (side * t2cap + i2l) * n1 + i1;

    // Zero the rings (rows outside the domain must read as zero), init barriers.
    {
        const int nring = L * RS;
        for (int i = tid; i < nring; i += blockDim.x) ring[i] = T(0);
        if constexpr (MODE == MODE_AF)
            for (int i = tid; i < nring; i += blockDim.x) rring[i] = T(0);
        if constexpr (SEG) {
            const int nrb = L * g.segblk * nwarps * 2;
            for (int i = tid; i < nrb; i += blockDim.x) rblk[i] = 0.0;
        }
        fence_proxy_async_smem();
        if (tid == 0) {
            for (int k = 0; k < EQD_NSLOT; ++k) mbar_init(&mbar[k], 1);
            s_dead[0] = 0;
            s_dead[1] = 0;
            fence_mbar_init();
        }
    }
    __syncthreads();

    // MODE_AF: the p planes go to `ring` (where p' is formed) and the r
    // planes to `rring`, both completing on the slot's mbarrier.
    auto issue_plane = [&](int q) {
        const int slot = q % EQD_NSLOT;
        mbar_arrive_expect_tx(&mbar[slot], (unsigned)L * (MODE == MODE_AF ? 12u : 6u) * bytes);
#pragma unroll
        for (int l = 0; l < L; ++l) {
            const T *incol = (MODE == MODE_AF ? reinterpret_cast<const T *>(cs.pold) : in) + (long long)colv[l] * g.colstride;
            for (int sc = 0; sc < 6; ++sc) {
                T *dst = ring + (size_t)l * RS + ((size_t)slot * 6 + sc) * CH + (e0 - base);
                const T *src = incol + ((long long)sc * n3 + q) * g.PS + e0;
                bulk_g2s(dst, src, bytes, &mbar[slot]);
            }
            if constexpr (MODE == MODE_AF) {
                const T *rcol = in + (long long)colv[l] * g.colstride;
                for (int sc = 0; sc < 6; ++sc) {
                    T *dst = rring + (size_t)l * RS + ((size_t)slot * 6 + sc) * CH + (e0 - base);
                    const T *src = rcol + ((long long)sc * n3 + q) * g.PS + e0;
                    bulk_g2s(dst, src, bytes, &mbar[slot]);
                }
            }
        }
    };
    // MODE_AF: p' = r + beta p on landed plane q (every thread; the caller
    // orders it before the plane's readers with a CTA barrier). The same
    // expression as the unfused direction update, so the same bits.
    T beta_l[L];
#pragma unroll
    for (int l = 0; l < L; ++l) beta_l[l] = MODE == MODE_AF ? (T)cs.beta[colv[l]] : T(0);
    const int nel = (int)(bytes / sizeof(T));
    auto form_direction = [&](int q) {
        T *p0 = ring + (size_t)(q % EQD_NSLOT) * 6 * CH + (e0 - base);
        const long long roff = rring - ring;
        for (int j = tid; j < nel; j += blockDim.x) {
#pragma unroll
            for (int l = 0; l < L; ++l) {
                T *pp = p0 + (size_t)l * RS + j;
                const T *rp = pp + roff;
#pragma unroll
                for (int sc = 0; sc < 6; ++sc) pp[sc * CH] = rp[sc * CH] + beta_l[l] * pp[sc * CH];
            }
        }
        // The slot is refilled by bulk copies later: order these generic-proxy
        // writes before them.
        fence_proxy_async_smem();
    };
    int issued = min(s_beg + EQD_NSLOT, ing_end);  // planes [s_beg, issued) issued
    if (tid == 0) {
        for (int q = s_beg; q < issued; ++q) issue_plane(q);
    }
    bool lead_ok = true;
    if constexpr (MODE == MODE_AF) {
        // The first plane's direction; each step then forms the next plane's
        // before its barrier.
        if (s_beg < ing_end) {
            lead_ok = mbar_wait_bounded(&mbar[s_beg % EQD_NSLOT], ((unsigned)(s_beg / EQD_NSLOT) & 1u) ^ ph0, err);
            if (lead_ok) form_direction(s_beg);
        }
        lead_ok = __syncthreads_and(lead_ok);
    }

    // Per-thread x1 row operators (start column within the line + 6 taps).
    const AxisT<T> &A1 = C.ax[0];
    const AxisT<T> &A2 = C.ax[1];
    const AxisT<T> &A3 = C.ax[2];
    int s1;
    T c1[6], c2[6];
    if (i1 < 4) {
        s1 = 0;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int o = k - i1;
            c1[k] = (o >= -3 && o <= 3) ? A1.d1_cl[i1][o + 3] : T(0);
            c2[k] = (o >= -3 && o <= 3) ? A1.d2_cl[i1][o + 3] : T(0);
        }
    } else if (i1 >= n1 - 4) {
        s1 = n1 - 6;
        const int rr = n1 - 1 - i1;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int o = (s1 + k) - i1;
            c1[k] = (o >= -3 && o <= 3) ? A1.d1_cl[4 + rr][o + 3] : T(0);
            c2[k] = (o >= -3 && o <= 3) ? A1.d2_cl[4 + rr][o + 3] : T(0);
        }
    } else {
        s1 = i1 - 2;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            c1[k] = A1.d1_int[k];
            c2[k] = A1.d2_int[k];
        }
        c1[5] = T(0);
        c2[5] = T(0);
    }
    // Face threads: the +x1 boundary derivative of the fault node over the
    // same 6-wide x1 window (lower end of the plus block: window cols 0..3;
    // upper end of the minus block: cols 5..2, odd mirror).
    T cdh[6];
#pragma unroll
    for (int k = 0; k < 6; ++k)
        cdh[k] = !is_face ? T(0) : (side == 1 ? (k < 4 ? A1.dlo[k] : T(0)) : (k >= 2 ? -A1.dlo[5 - k] : T(0)));
    const bool ff_x12 = (side == 0 && i1 == 0) || (side == 1 && i1 == n1 - 1) || i2 == 0 || i2 == n2 - 1;
    const T wq1 = (i1 < 4) ? A1.wq[i1] : (i1 >= n1 - 4 ? A1.wq[n1 - 1 - i1] : T(1));
    const T wq2 = (i2 < 4) ? A2.wq[i2] : (i2 >= n2 - 4 ? A2.wq[n2 - 1 - i2] : T(1));
    // H weight of this (x1, x2) point with the sign of the mode; zero on the
    // x1/x2 far-field boundaries (P zeroes those rows).
    const T hpt = ff_x12 ? T(0) : (T)(C.hvol * (double)wq1 * (double)wq2 * (MODE == MODE_RHS ? 1.0 : -1.0));

    const int own = i2 * n1 + i1 - base + side * 3 * CH;      // comp-0 offset inside a plane slot
    const int lineoff = i2 * n1 + s1 - base + side * 3 * CH;  // comp-0 x1 window start
    const long long cstr = (long long)n3 * g.PS;                // component stride in the column
    const long long poff = (long long)(side * 3) * cstr + (long long)i2 * n1 + i1;

    T v1w[L][7], v2w[L][7], v3w[L][7], F3w[L][7], H23w[L][7], w3q[L][4];
#pragma unroll
    for (int l = 0; l < L; ++l) {
#pragma unroll
        for (int k = 0; k < 7; ++k) v1w[l][k] = v2w[l][k] = v3w[l][k] = F3w[l][k] = H23w[l][k] = T(0);
#pragma unroll
        for (int k = 0; k < 4; ++k) w3q[l][k] = T(0);
    }

    // Dot-product sums (FP64-input instances: of the current step block,
    // flushed per block).
    double acc0[L], acc1[L];
#pragma unroll
    for (int l = 0; l < L; ++l) acc0[l] = acc1[l] = 0.0;
    const T lam = C.lam, mu = C.mu, lpm = C.lpm, sat = C.sat_c;
    int dead_at = -1;
    const int lane = tid & 31, warp = tid >> 5;
    // Warp sums into this warp's slot of block b (all lanes take part).
    auto flush = [&](int b) {
#pragma unroll
        for (int l = 0; l < L; ++l) {
            double x = acc0[l], y = acc1[l];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                x += __shfl_down_sync(0xffffffffu, x, o);
                y += __shfl_down_sync(0xffffffffu, y, o);
            }
            if (lane == 0) {
                double *slot = rblk + (((size_t)l * g.segblk + b) * nwarps + warp) * 2;
                slot[0] += x;
                slot[1] += y;
            }
            acc0[l] = acc1[l] = 0.0;
        }
    };

    // One march step. Windows are ordered by age: index 6 holds plane s,
    // index 3 plane p = s - 3; the F3 window holds p at 6 and z = s - 6 at 3;
    // the w3 queue holds p at 3 and z at 0.
    auto step = [&](int s) -> bool {
        const int buf = s & 1;
        // ---- ingest plane s ----------------------------------------------------
        if (s < n3) {
            const int slot = s % EQD_NSLOT;
            if (!mbar_wait_bounded(&mbar[slot], ((unsigned)(s / EQD_NSLOT) & 1u) ^ ph0, err)) s_dead[buf] = 1;
            if (MODE == MODE_RHS || MODE == MODE_AP) {
                // Fix-up pass on the landed plane: chi (RHS) or P (generic input).
                const int nrows = r1 - r0;
#pragma unroll
                for (int l = 0; l < L; ++l) {
                    T *pl = ring + (size_t)l * RS + (size_t)slot * 6 * CH;
                    const int col = colv[l];
                    if (MODE == MODE_RHS) {
                        if (s >= g.i3f0 && s < g.i3f0 + g.n3f) {
                            for (int w = tid; w < nrows; w += blockDim.x) {
                                const int r = r0 + w;
                                if (r < g.i2f0 || r >= g.i2f0 + g.n2f) continue;
                                const int k = (r - g.i2f0) + g.n2f * (s - g.i3f0);
                                for (int j = 0; j < 2; ++j) {
                                    double sl;
                                    if (cs.slip_dense)
                                        sl = cs.slip_dense[((long long)col * 2 + j) * g.nf + k];
                                    else
                                        sl = (cs.slip_node[col] == k && cs.slip_comp[col] == j) ? 1.0 : 0.0;
                                    if (sl != 0.0) {
                                        pl[(0 * 3 + 1 + j) * CH + r * n1 + (n1 - 1) - base] -= (T)(0.5 * sl);
                                        pl[(1 * 3 + 1 + j) * CH + r * n1 + 0 - base] += (T)(0.5 * sl);
                                    }
                                }
                            }
                        }
                    } else {  // MODE_AP: v = P x
                        const bool plane_ff = (s == 0 || s == n3 - 1);
                        for (int w = tid; w < nrows * 3; w += blockDim.x) {
                            const int r = r0 + w / 3, j = w % 3;
                            T *m = pl + (0 * 3 + j) * CH + r * n1 - base;
                            T *pp = pl + (1 * 3 + j) * CH + r * n1 - base;
                            if (plane_ff || r == 0 || r == n2 - 1) {
                                for (int i = 0; i < n1; ++i) {
                                    m[i] = T(0);
                                    pp[i] = T(0);
                                }
                            } else {
                                m[0] = T(0);
                                pp[n1 - 1] = T(0);
                                const T avg = T(0.5) * (m[n1 - 1] + pp[0]);
                                m[n1 - 1] = avg;
                                pp[0] = avg;
                            }
                        }
                    }
                }
                fence_proxy_async_smem();
                __syncthreads();
            }
#pragma unroll
            for (int l = 0; l < L; ++l) {
                T a = T(0), b = T(0), c = T(0), h = T(0);
                if (valid) {
                    const T *pl = ring + (size_t)l * RS + (size_t)slot * 6 * CH;
                    const T *c3 = pl + 2 * CH + own;
                    a = pl[own];
                    b = pl[CH + own];
                    c = c3[0];
                    h = x2_d1i(A2, c3, n1);
                    if (x2cl) x2_corr_d1(A2, gdd, c3, h);
                    if constexpr (MODE == MODE_AF) {
                        // The new direction of this CTA's own points and planes.
                        if (act[l] && s >= q0 && s < q1) {
                            T *pn = reinterpret_cast<T *>(cs.pnew) + (long long)colv[l] * g.colstride + poff +
                                    (long long)s * g.PS;
                            pn[0] = a;
                            pn[cstr] = b;
                            pn[2 * cstr] = c;
                        }
                    }
                }
                push7(v1w[l], a);
                push7(v2w[l], b);
                push7(v3w[l], c);
                push7(H23w[l], h);
            }
        } else {
#pragma unroll
            for (int l = 0; l < L; ++l) {
                push7(v1w[l], T(0));
                push7(v2w[l], T(0));
                push7(v3w[l], T(0));
                push7(H23w[l], T(0));
            }
        }

        // ---- in-plane work at p = s - 3 ---------------------------------------
        const int p = s - 3;
        const bool pin = p >= p_lo && p < p_hi;
        const bool owned = s >= o_beg;          // (s < s_end always)
        const bool pout = owned && p < n3;      // components 1, 2 of plane p are stored here
        const bool x3i = p >= 4 && p <= n3 - 5;  // x3-interior plane (block-uniform)
        const int r3 = p < 4 ? p : 4 + (n3 - 1 - p);
        T w1[L], w2[L], w3p[L], F3[L];
#pragma unroll
        for (int l = 0; l < L; ++l) w1[l] = w2[l] = w3p[l] = F3[l] = T(0);
        if (valid && pin) {
#pragma unroll
            for (int l = 0; l < L; ++l) {
                const T *pl = ring + (size_t)l * RS + (size_t)(p % EQD_NSLOT) * 6 * CH;
                const T *l1 = pl + lineoff;
                const T *l2 = l1 + CH;
                const T *l3 = l2 + CH;
                const T *o1 = pl + own;
                const T *o2 = o1 + CH;
                const T *o3 = o2 + CH;
                const T v1 = v1w[l][3], v2 = v2w[l][3], v3 = v3w[l][3];
                T G1 = T(0), A11 = T(0), A21 = T(0), A31 = T(0);
                T xa[6], xb[6], xc[6];
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    xa[k] = l1[k];
                    xb[k] = l2[k];
                    xc[k] = l3[k];
                    G1 += c1[k] * xa[k];
                    A11 += c2[k] * xa[k];
                    A21 += c2[k] * xb[k];
                    A31 += c2[k] * xc[k];
                }
                T dh1 = T(0), dh2 = T(0), dh3 = T(0);
                if (is_face) {
#pragma unroll
                    for (int k = 0; k < 6; ++k) {
                        dh1 += cdh[k] * xa[k];
                        dh2 += cdh[k] * xb[k];
                        dh3 += cdh[k] * xc[k];
                    }
                }
                T G2 = x2_d1i(A2, o2, n1);
                T H21 = x2_d1i(A2, o1, n1);
                T A12 = x2_d2i(A2, o1, v1, n1);
                T A22 = x2_d2i(A2, o2, v2, n1);
                T A32 = x2_d2i(A2, o3, v3, n1);
                T W2 = x2_wi(A2, o2, v2, n1);
                if (x2cl) {
                    T dummy = T(0);
                    x2_corr_dd(A2, gdd, o1, H21, A12);
                    x2_corr_dd(A2, gdd, o2, G2, A22);
                    x2_corr_dd(A2, gdd, o3, dummy, A32);
                    x2_corr_w(A2, gw, o2, W2);
                }
                T G3, A13, A23, A33, D3H23;
                if (x3i) {
                    G3 = x3_d1i(A3, v3w[l]);
                    A13 = x3_d2i(A3, v1w[l]);
                    A23 = x3_d2i(A3, v2w[l]);
                    A33 = x3_d2i(A3, v3w[l]);
                    D3H23 = x3_d1i(A3, H23w[l]);
                } else {
                    G3 = x3_d1c(A3, v3w[l], r3);
                    A13 = x3_d2c(A3, v1w[l], r3);
                    A23 = x3_d2c(A3, v2w[l], r3);
                    A33 = x3_d2c(A3, v3w[l], r3);
                    D3H23 = x3_d1c(A3, H23w[l], r3);
                }
                const T F1 = lam * G1 + lpm * (G2 + G3);
                F3[l] = lam * G3 + lpm * (G1 + G2);
                w1[l] = mu * (T(2) * A11 + A12 + A13);
                w2[l] = mu * (A21 + T(2) * A22 + A23) + lam * W2 + lpm * D3H23;
                w3p[l] = mu * (A31 + A32 + T(2) * A33);
                if (is_face) {
                    // Traction on the fixed +x1 axis (`traction_blocks`), with the
                    // +x1 boundary derivatives dh (computed with the x1 window).
                    // SAT c (tau^+ - tau^-) on both faces; the partner (other
                    // side) is the adjacent lane.
                    const T D3v1 = x3i ? x3_d1i(A3, v1w[l]) : x3_d1c(A3, v1w[l], r3);
                    const T tau1 = lam * (G1 + G2 + G3) + T(2) * mu * dh1;
                    const T tau2 = mu * (H21 + dh2);
                    const T tau3 = mu * (D3v1 + dh3);
                    const T o1t = __shfl_xor_sync(facemask, tau1, 1);
                    const T o2t = __shfl_xor_sync(facemask, tau2, 1);
                    const T o3t = __shfl_xor_sync(facemask, tau3, 1);
                    const T sgn = side == 0 ? T(-1) : T(1);
                    w1[l] += sat * sgn * (tau1 - o1t);
                    w2[l] += sat * sgn * (tau2 - o2t);
                    w3p[l] += sat * sgn * (tau3 - o3t);
                }
                xF1[((size_t)l * 2 + buf) * NP + pidx] = F1;
                xH21[((size_t)l * 2 + buf) * NP + pidx] = H21;
            }
        }
#pragma unroll
        for (int l = 0; l < L; ++l) {
            push7(F3w[l], F3[l]);
#pragma unroll
            for (int k = 0; k < 3; ++k) w3q[l][k] = w3q[l][k + 1];
            w3q[l][3] = w3p[l];
        }
        if constexpr (MODE == MODE_AF) {
            // The next plane's direction, before the barrier that precedes its
            // ingest (its slot is not read during this step).
            if (s + 1 < ing_end) {
                if (mbar_wait_bounded(&mbar[(s + 1) % EQD_NSLOT], ((unsigned)((s + 1) / EQD_NSLOT) & 1u) ^ ph0, err))
                    form_direction(s + 1);
                else
                    s_dead[buf] = 1;
            }
        }
        __syncthreads();
        if (s_dead[buf]) {
            dead_at = s;
            return false;
        }
        // Slot of plane p is free: every thread has passed its last read.
        if (s - s_beg >= 3 && s + 3 < ing_end) {
            if (tid == 0) issue_plane(s + 3);
            issued = s + 4;
        }

        // ---- finish p: x1 derivatives of F1, H21; P, H; store -----------------
        if (valid && pout) {
            const T hw = hpt * plane_weight(A3, p, n3);
#pragma unroll
            for (int l = 0; l < L; ++l) {
                const T *xf = xF1 + ((size_t)l * 2 + buf) * NP + (pidx - i1 + s1);
                const T *xh = xH21 + ((size_t)l * 2 + buf) * NP + (pidx - i1 + s1);
                T E1 = T(0), E21 = T(0);
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    E1 += c1[k] * xf[k];
                    E21 += c1[k] * xh[k];
                }
                T u1 = w1[l] + E1;
                T u2 = w2[l] + lpm * E21;
                if (is_face) {
                    u1 = T(0.5) * (u1 + __shfl_xor_sync(facemask, u1, 1));
                    u2 = T(0.5) * (u2 + __shfl_xor_sync(facemask, u2, 1));
                }
                const T y1 = hw * u1, y2 = hw * u2;
                if (act[l]) {
                    TO *o = out + (long long)colv[l] * g.colstride + poff + (long long)p * g.PS;
                    o[0] = (TO)y1;
                    o[cstr] = (TO)y2;
                }
                const T va = v1w[l][3], vb = v2w[l][3];
                if (MODE == MODE_RHS) {
                    acc0[l] += (double)y1 * (double)y1 + (double)y2 * (double)y2;
                    if (cs.dinv) {
                        const double *dv = cs.dinv + poff + (long long)p * g.PS;
                        acc1[l] += dv[0] * (double)y1 * (double)y1 + dv[cstr] * (double)y2 * (double)y2;
                    }
                } else {
                    acc0[l] += (double)va * (double)y1 + (double)vb * (double)y2;
                    acc1[l] += (double)va * (double)va + (double)vb * (double)vb;
                }
            }
        }
        // ---- finish z = s - 6: comp 3 --------------------------------------------
        const int z = s - 6;
        const bool zout = owned && z >= 0 && z < n3;
        if (valid && zout) {
            const T hw = hpt * plane_weight(A3, z, n3);
            const bool x3iz = z >= 4 && z <= n3 - 5;
            const int r3z = z < 4 ? z : 4 + (n3 - 1 - z);
#pragma unroll
            for (int l = 0; l < L; ++l) {
                T w3 = w3q[l][0] + (x3iz ? x3_d1i(A3, F3w[l]) : x3_d1c(A3, F3w[l], r3z));
                if (is_face) w3 = T(0.5) * (w3 + __shfl_xor_sync(facemask, w3, 1));
                const T y3 = hw * w3;
                if (act[l]) out[(long long)colv[l] * g.colstride + poff + 2 * cstr + (long long)z * g.PS] = (TO)y3;
                const T vc = v3w[l][0];
                if (MODE == MODE_RHS) {
                    acc0[l] += (double)y3 * (double)y3;
                    if (cs.dinv) acc1[l] += cs.dinv[poff + 2 * cstr + (long long)z * g.PS] * (double)y3 * (double)y3;
                } else {
                    acc0[l] += (double)vc * (double)y3;
                    acc1[l] += (double)vc * (double)vc;
                }
            }
        }
        return true;
    };

    bool alive = lead_ok;
    if (!alive) dead_at = s_beg;
    if constexpr (SEG) {
        // Lead-in steps, then the owned step blocks, each closed by a flush
        // (every lane of every warp takes part).
        int s = s_beg;
        for (; s < o_beg && alive; ++s) alive = step(s);
        for (int b = blk0; b < blk0 + nbs && alive; ++b) {
            const int e = b == g.nblk - 1 ? s_end : min(b * EQD_PBLK + 3 + EQD_PBLK, s_end);
            for (; s < e && alive; ++s) alive = step(s);
            if (alive) flush(b - blk0);
        }
    } else {
        for (int s = 0; s < s_end && alive; ++s) alive = step(s);
    }

    if (!alive) {
        // A wait gave up (recorded in *err). Before the CTA's shared memory is
        // released, wait (bounded) for every plane copy issued and not yet
        // consumed: planes dead_at .. issued-1.
        if (tid == 0) {
            for (int q = max(dead_at, s_beg); q < issued; ++q)
                mbar_wait_bounded(&mbar[q % EQD_NSLOT], ((unsigned)(q / EQD_NSLOT) & 1u) ^ ph0, err);
        }
        __syncthreads();
        return;
    }

    if constexpr (SEG) {
        // Per (column, tile, step block): the warps' sums in warp order.
        __syncthreads();
        if (partials) {
#pragma unroll
            for (int l = 0; l < L; ++l) {
                if (!act[l]) continue;
                for (int i = tid; i < nbs * 2; i += blockDim.x) {
                    const int k = i & 1, b = i >> 1;
                    const double *src = rblk + ((size_t)l * g.segblk + b) * nwarps * 2 + k;
                    double sum = 0.0;
                    for (int w = 0; w < nwarps; ++w) sum += src[(size_t)w * 2];
                    partials[(((long long)colv[l] * g.ntiles + tile) * g.nblk + blk0 + b) * 2 + k] = sum;
                }
            }
        }
    } else {
        // Per (column, tile): block tree over the whole march.
#pragma unroll
        for (int l = 0; l < L; ++l) {
            const double s0 = block_sum(acc0[l], red);
            __syncthreads();
            const double s1v = block_sum(acc1[l], red);
            __syncthreads();
            if (tid == 0 && partials && act[l]) {
                double *pp = partials + ((long long)colv[l] * g.ntiles + tile) * 2;
                pp[0] = s0;
                pp[1] = s1v;
            }
        }
    }
}

}  // namespace eqd
