// The CG iterations' stencil apply, y = -H P (D + SAT) v for v in range(P),
// FP32, written for the instruction budget of one grid point.
//
// Same operator, factorisation and tables as plane_march_kernel (MODE_A; the
// reference's `elastic_blocks` src/Elasticity.jl:80-89, SAT and P of
// src/ElasticitySplitNode.jl:149-203, `traction_blocks` src/Elasticity.jl:
// 195-221). What differs is how the work reaches the SM:
//
//   * The x3 march is unrolled over the plane ring (8 slots, 8 march steps
//     per trip): every ring slot, register-window entry and exchange buffer
//     a step touches is a compile-time index, so a step issues no address
//     arithmetic, no register-window moves and no modulo; a shared-memory
//     operand is the thread's own offset plus an immediate.
//   * N1 (points across a side) and T2 (x2 rows per tile) are template
//     constants: the row stride of every x2 neighbour is an immediate.
//   * Thread -> point: lanes walk the tile's (x2, x1) plane of one side in
//     storage order, each side padded to whole warps, so the 32 addresses of
//     every warp-wide shared load are 32 consecutive words (no bank
//     conflicts). The fault-face point of each row is left to dedicated face
//     warps, where the two sides of a fault node sit in adjacent lanes (the
//     SAT coupling and the P averaging are lane shuffles).
//   * Component 2 finishes with component 3, three planes behind component 1:
//     H23 = D1_2 v3 is then formed from the same x2 neighbours of plane p as
//     the D2_2 v3 term, and a step reads only its own point of the newest plane.
//   * The interior x2 and x3 stencils are exact rationals (instruction
//     immediates) applied in unit spacing; 1/h and the Lame constants enter
//     through a handful of per-grid products, and one branch per phase picks
//     the interior or the closure form of all x3 derivatives. Idle lanes
//     compute on in-range data with their stores predicated off.
//   * Dot products p.q and p.p are accumulated in FP64 from FP64 products
//     (in BP8 units a single product can exceed the FP32 range), then reduced
//     per (column, tile) in a fixed order.
//
// Decomposition: one CTA per (column, x2 tile). Tiles: the first and last
// hold 7 rows (every x2 closure row, whose wide-operator rows reach 10 rows
// in) and the tiles between split the interior rows, at most T2 each. Planes
// arrive by cp.async.bulk into the 8-slot ring five planes ahead of use,
// completing on mbarriers; waits are bounded.
#pragma once
#include <type_traits>

#include "plane_march.cuh"

namespace eqd {

constexpr int kRing = 8;          // plane ring slots = march steps per unrolled trip
constexpr int kRingAhead = 5;     // planes in flight ahead of the newest ingested plane
constexpr int kRingEdge = 7;      // rows of the first and last x2 tiles

__host__ __device__ constexpr int ring_round32(int x) { return (x + 31) / 32 * 32; }
// Chunk (one side, component and plane: tile rows + 4-row halos) capacity in
// elements: 16-byte multiple with room for the 16-byte rounding of the copy.
__host__ __device__ constexpr int ring_chunk(int n1, int t2) { return ((t2 + 2 * EQD_HALO) * n1 + 8 + 3) / 4 * 4; }
// Regular lanes per side (whole warps), then the face warps.
__host__ __device__ constexpr int ring_side_lanes(int n1, int t2) { return ring_round32(t2 * n1); }
__host__ __device__ constexpr int ring_threads(int n1, int t2) {
    return 2 * ring_side_lanes(n1, t2) + ring_round32(2 * t2);
}
// Dynamic shared memory: 8 mbarriers (64 B), the step flags (64 B),
// reduction scratch (256 B), the ring, the F1 / H21 exchange (two step
// parities each).
constexpr int kRingHeader = 64 + 64 + 256;
__host__ __device__ constexpr size_t ring_smem(int n1, int t2) {
    return kRingHeader + (size_t)kRing * 6 * ring_chunk(n1, t2) * 4 + (size_t)2 * 2 * (2 * t2 * n1) * 4;
}

// Interior stencils of the order-4 operators as exact rationals (unit
// spacing): D1 = [1/12, -2/3, 0, 2/3, -1/12], D2 = [-1/12, 4/3, -5/2, 4/3,
// -1/12], W = D1 D1 = [1/144, -1/9, 4/9, 1/9, -65/72, ...] (symmetric). The
// ring march forms x2 and x3 derivatives in these raw units (the constants
// are instruction immediates) and applies 1/h and the material constants
// once, through the products below.
constexpr float kD1a = 1.f / 12.f, kD1b = 2.f / 3.f;
constexpr float kD2a = -1.f / 12.f, kD2b = 4.f / 3.f, kD2c = -5.f / 2.f;
constexpr float kWa = 1.f / 144.f, kWb = -1.f / 9.f, kWc = 4.f / 9.f, kWd = 1.f / 9.f, kWe = -65.f / 72.f;

// Per-grid scalars of the ring march: Lame constants times powers of the
// inverse spacings h2i = 1/h2, h3i = 1/h3, and the spacings (closure rows,
// which come from the tables in 1/h units, are converted to raw units).
struct RingScal {
    float lam, mu, mu2, lpm;                    // lambda, mu, 2 mu, lambda + mu
    float lpm_h2, lpm_h3, lam_h2, lam_h3;       // (lambda + mu) h2i, ..., lambda h3i
    float mu_h2, mu_h3;                         // mu h2i, mu h3i
    float mu_h2s, mu2_h2s, lam_h2s;             // mu h2i^2, 2 mu h2i^2, lambda h2i^2
    float mu_h3s, mu2_h3s;                      // mu h3i^2, 2 mu h3i^2
    float lpm_h2h3, h3i;                        // (lambda + mu) h2i h3i, h3i
    float h2, h2s, h3, h3s;                     // h2, h2^2, h3, h3^2
    float sat;                                  // SAT scale c = 1 / (2 h1 w0)
};

struct RingGeom {
    int n2, n3, PS;
    long long colstride;
    int ntiles;           // x2 tiles per column: [0, 7), middle tiles of <= T2 rows, [n2 - 7, n2)
    int nmid;             // middle tiles
    int drop_plane;       // test hook: the copy of this plane is never issued (-1: none)
    unsigned poll_limit;  // polls of a bounded wait before it gives up (0: the default bound)
    RingScal k;
};

__device__ __forceinline__ bool ring_wait(uint64_t *bar, unsigned parity, unsigned *err, unsigned limit) {
    if (limit == 0) return mbar_wait_bounded(bar, parity, err);
    for (unsigned i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    atomicOr(err, DERR_MBAR_TIMEOUT);
    return false;
}

template <int N>
using IC = std::integral_constant<int, N>;

// REGS caps the registers of a thread (with the CTA size, how many CTAs
// share an SM). DYN: the march is not unrolled; every step runs the code of
// slot 0 with ring slots, mbarrier and exchange buffer chosen at run time,
// and the register windows rotate by one entry after each step (a smaller
// code body at the price of the window moves).
template <int N1, int T2, int REGS, bool DYN = false>
__global__ void __maxnreg__(REGS)
ring_march_kernel(const __grid_constant__ OpConst<float> C, const __grid_constant__ RingGeom g,
                  const float *__restrict__ in, float *__restrict__ out, const int8_t *__restrict__ status,
                  double *__restrict__ partials, unsigned *__restrict__ err) {
    constexpr int CH = ring_chunk(N1, T2);
    constexpr int SL = ring_side_lanes(N1, T2);
    constexpr int NPT = 2 * T2 * N1;  // exchange entries per step parity
    constexpr int SLOT = 6 * CH;

    const int col = blockIdx.x / g.ntiles;
    const int tile = blockIdx.x % g.ntiles;
    if (status && status[col] != COL_ACTIVE) return;
    const int n2 = g.n2, n3 = g.n3;
    int a0, a1;
    if (tile == 0) {
        a0 = 0;
        a1 = kRingEdge;
    } else if (tile == g.ntiles - 1) {
        a0 = n2 - kRingEdge;
        a1 = n2;
    } else {
        const int m = n2 - 2 * kRingEdge, k = tile - 1;
        a0 = kRingEdge + (int)((long long)k * m / g.nmid);
        a1 = kRingEdge + (int)((long long)(k + 1) * m / g.nmid);
    }
    const int T2r = a1 - a0;

    // Copied rows [r0, r1) (tile + halo, clipped to the grid), as a 16-byte
    // aligned element range [e0, e1) of the plane. Chunk element 0 is plane
    // element `base` (row a0 - 4, rounded down to 16 bytes).
    const int r0 = max(a0 - EQD_HALO, 0), r1 = min(a1 + EQD_HALO, n2);
    const int lo_el = (a0 - EQD_HALO) * N1;
    const int base = lo_el >= 0 ? (lo_el / 4) * 4 : -(((-lo_el) + 3) / 4) * 4;
    const int e0 = ((r0 * N1) / 4) * 4;
    const int e1 = ((r1 * N1 + 3) / 4) * 4;
    const unsigned bytes = (unsigned)((e1 - e0) * 4);

    extern __shared__ __align__(128) unsigned char smem_raw[];
    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem_raw);
    volatile int *s_dead = reinterpret_cast<volatile int *>(smem_raw + 8 * kRing);  // [2], by step parity
    double *red = reinterpret_cast<double *>(smem_raw + 128);
    float *ring = reinterpret_cast<float *>(smem_raw + kRingHeader);  // [slot][side*3+comp][CH]
    float *xF1 = ring + kRing * SLOT;                                 // [2][NPT]
    float *xH21 = xF1 + 2 * NPT;                                      // [2][NPT]

    // ---- thread -> point ---------------------------------------------------
    const int tid = threadIdx.x;
    int side, row, i1;
    bool valid, is_face = false;
    if (tid < SL) {
        side = 0;
        row = tid / N1;
        i1 = tid % N1;
        valid = row < T2r && i1 != N1 - 1;
    } else if (tid < 2 * SL) {
        side = 1;
        row = (tid - SL) / N1;
        i1 = (tid - SL) % N1;
        valid = row < T2r && i1 != 0;
    } else {
        const int k = tid - 2 * SL;
        side = k & 1;
        row = k >> 1;
        i1 = side == 0 ? N1 - 1 : 0;
        is_face = true;
        valid = row < T2r;
    }
    if (!valid) row = 0;  // idle lanes: every derived index stays inside the grid and the buffers
    const int i2 = a0 + row;
    is_face = is_face && valid;  // idle face-warp lanes take the regular path (and store nothing)
    const unsigned facemask = __ballot_sync(0xffffffffu, is_face);
    const bool x2cl = i2 < 6 || i2 >= n2 - 6;

    // Zero the ring (rows outside the grid must read as zero), set up barriers.
    for (int i = tid; i < kRing * SLOT; i += blockDim.x) ring[i] = 0.f;
    fence_proxy_async_smem();
    if (tid == 0) {
        for (int k = 0; k < kRing; ++k) mbar_init(&mbar[k], 1);
        s_dead[0] = 0;
        s_dead[1] = 0;
        fence_mbar_init();
    }
    __syncthreads();

    const float *incol = in + (long long)col * g.colstride;
    auto issue_plane = [&](int q) {
        if (q == g.drop_plane) return;
        uint64_t *bar = &mbar[q & (kRing - 1)];
        mbar_arrive_expect_tx(bar, 6u * bytes);
        float *dst = ring + (q & (kRing - 1)) * SLOT + (e0 - base);
        const float *src = incol + (long long)q * g.PS + e0;
#pragma unroll
        for (int sc = 0; sc < 6; ++sc) bulk_g2s(dst + sc * CH, src + (long long)sc * n3 * g.PS, bytes, bar);
    };
    int issued = min(kRingAhead, n3);  // planes [0, issued) issued
    if (tid == 0)
        for (int q = 0; q < issued; ++q) issue_plane(q);

    // ---- per-thread operator rows --------------------------------------------
    const AxisT<float> &A1 = C.ax[0];
    const AxisT<float> &A2 = C.ax[1];
    const AxisT<float> &A3 = C.ax[2];
    int s1;
    float c1[6], c2[6];
    if (i1 < 4) {
        s1 = 0;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int o = k - i1;
            c1[k] = (o >= -3 && o <= 3) ? A1.d1_cl[i1][o + 3] : 0.f;
            c2[k] = (o >= -3 && o <= 3) ? A1.d2_cl[i1][o + 3] : 0.f;
        }
    } else if (i1 >= N1 - 4) {
        s1 = N1 - 6;
        const int rr = N1 - 1 - i1;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const int o = (s1 + k) - i1;
            c1[k] = (o >= -3 && o <= 3) ? A1.d1_cl[4 + rr][o + 3] : 0.f;
            c2[k] = (o >= -3 && o <= 3) ? A1.d2_cl[4 + rr][o + 3] : 0.f;
        }
    } else {
        s1 = i1 - 2;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            c1[k] = A1.d1_int[k];
            c2[k] = A1.d2_int[k];
        }
        c1[5] = 0.f;
        c2[5] = 0.f;
    }
    const bool ff_x12 = (side == 0 && i1 == 0) || (side == 1 && i1 == N1 - 1) || i2 == 0 || i2 == n2 - 1;
    const float wq1 = (i1 < 4) ? A1.wq[i1] : (i1 >= N1 - 4 ? A1.wq[N1 - 1 - i1] : 1.f);
    const float wq2 = (i2 < 4) ? A2.wq[i2] : (i2 >= n2 - 4 ? A2.wq[n2 - 1 - i2] : 1.f);
    const float hpt = (ff_x12 || !valid) ? 0.f : (float)(-C.hvol * (double)wq1 * (double)wq2);

    const int own = side * 3 * CH + i2 * N1 + i1 - base;   // component 1 of this point in a slot
    const int line = own - i1 + s1;                        // its x1 window
    const int pidx = (side * T2 + row) * N1 + i1;          // exchange entry
    const int pline = pidx - i1 + s1;
    const long long cstr = (long long)n3 * g.PS;
    float *ocol = out + (long long)col * g.colstride + (long long)side * 3 * cstr + i2 * N1 + i1;

    float v1w[kRing], v2w[kRing], v3w[kRing], F3w[kRing], H23w[kRing], w2q[4], w3q[4];
#pragma unroll
    for (int k = 0; k < kRing; ++k) v1w[k] = v2w[k] = v3w[k] = F3w[k] = H23w[k] = 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k) w2q[k] = w3q[k] = 0.f;
    double acc0 = 0.0, acc1 = 0.0;
    const RingScal K = g.k;
    const float sgn = side == 0 ? -1.f : 1.f;
    const int s_end = n3 + 6;
    int dead_at = -1;

    // Raw (unit-spacing) x3 first and second derivatives at the plane whose
    // window slot is Q: interior planes use the rational stencils, the
    // closure planes (table row r, in 1/h units) are converted to raw units.
    auto x3d1i = [&](const float (&w)[kRing], auto Qc) -> float {
        constexpr int Q = decltype(Qc)::value;
        return kD1a * (w[(Q - 2) & 7] - w[(Q + 2) & 7]) + kD1b * (w[(Q + 1) & 7] - w[(Q - 1) & 7]);
    };
    auto x3d2i = [&](const float (&w)[kRing], auto Qc) -> float {
        constexpr int Q = decltype(Qc)::value;
        return kD2a * (w[(Q - 2) & 7] + w[(Q + 2) & 7]) + kD2b * (w[(Q - 1) & 7] + w[(Q + 1) & 7]) + kD2c * w[Q & 7];
    };
    auto x3d1c = [&](const float (&w)[kRing], auto Qc, int r) -> float {
        constexpr int Q = decltype(Qc)::value;
        float s = 0.f;
#pragma unroll
        for (int o = 0; o < 7; ++o) s += A3.d1_cl[r][o] * w[(Q - 3 + o) & 7];
        return s * K.h3;
    };
    auto x3d2c = [&](const float (&w)[kRing], auto Qc, int r) -> float {
        constexpr int Q = decltype(Qc)::value;
        float s = 0.f;
#pragma unroll
        for (int o = 0; o < 7; ++o) s += A3.d2_cl[r][o] * w[(Q - 3 + o) & 7];
        return s * K.h3s;
    };
    // Quadrature weight of x3 plane q; zero on the far-field planes.
    auto plane_w = [&](int q) -> float {
        const int m = min(q, n3 - 1 - q);
        return m <= 0 ? 0.f : (m < 4 ? A3.wq[m] : 1.f);
    };

    // One march step s (slot U = s mod 8): ingest plane s; in-plane work and
    // component 1 of plane p = s - 3; components 2, 3 of plane z = s - 6.
    // Idle lanes compute on in-range data and store nothing (their H weight
    // is zero and their stores and sums are predicated off).
    auto step = [&](auto Uc, int s) -> bool {
        constexpr int U = decltype(Uc)::value;
        constexpr int UP = (U + kRing - 3) & 7;   // window slot of plane p
        constexpr int UZ = (U + kRing - 6) & 7;   // window slot of plane z
        const int RS = DYN ? (s & 7) : U;         // ring slot / mbarrier of plane s
        const int RP = DYN ? ((s + kRing - 3) & 7) : UP;  // ring slot of plane p
        const int BUF = DYN ? (s & 1) : (U & 1);
        constexpr int QP = (U + 1) & 3;           // queue entry of plane p  (p = s - 3)
        constexpr int QZ = (U + 2) & 3;           // queue entry of plane z  (z = s - 6)
        // ---- ingest plane s: the own point's three components ----------------
        float a = 0.f, b = 0.f, c = 0.f;
        if (s < n3) {
            if (!ring_wait(&mbar[RS], (unsigned)(s >> 3) & 1u, err, g.poll_limit)) s_dead[BUF] = 1;
            const float *pl = ring + RS * SLOT + own;
            a = pl[0];
            b = pl[CH];
            c = pl[2 * CH];
        }
        v1w[U] = a;
        v2w[U] = b;
        v3w[U] = c;

        // ---- in-plane work at p ----------------------------------------------
        const int p = s - 3;
        const bool pin = p >= 0 && p < n3;
        float w1 = 0.f, w2p = 0.f, w3p = 0.f, F3 = 0.f, h23r = 0.f;
        if (pin) {
            const float *pl = ring + RP * SLOT;
            const float *o1 = pl + own, *o2 = o1 + CH, *o3 = o2 + CH;
            const float *l1 = pl + line, *l2 = l1 + CH, *l3 = l2 + CH;
            const float v1 = v1w[UP], v2 = v2w[UP], v3 = v3w[UP];
            // x1 (per-thread rows, 1/h units)
            float G1 = 0.f, A11 = 0.f, A21 = 0.f, A31 = 0.f;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                const float xa = l1[k], xb = l2[k], xc = l3[k];
                G1 += c1[k] * xa;
                A11 += c2[k] * xa;
                A21 += c2[k] * xb;
                A31 += c2[k] * xc;
            }
            // x2 (raw units): sums and differences of the neighbour pairs
            const float a_m2 = o1[-2 * N1], a_m1 = o1[-N1], a_p1 = o1[N1], a_p2 = o1[2 * N1];
            const float b_m4 = o2[-4 * N1], b_m3 = o2[-3 * N1], b_m2 = o2[-2 * N1], b_m1 = o2[-N1];
            const float b_p1 = o2[N1], b_p2 = o2[2 * N1], b_p3 = o2[3 * N1], b_p4 = o2[4 * N1];
            const float c_m2 = o3[-2 * N1], c_m1 = o3[-N1], c_p1 = o3[N1], c_p2 = o3[2 * N1];
            float h21r = kD1a * (a_m2 - a_p2) + kD1b * (a_p1 - a_m1);
            float a12r = kD2a * (a_m2 + a_p2) + kD2b * (a_m1 + a_p1) + kD2c * v1;
            const float bs1 = b_m1 + b_p1, bs2 = b_m2 + b_p2;
            float g2r = kD1a * (b_m2 - b_p2) + kD1b * (b_p1 - b_m1);
            float a22r = kD2a * bs2 + kD2b * bs1 + kD2c * v2;
            float w2r = kWa * (b_m4 + b_p4) + kWb * (b_m3 + b_p3) + kWc * bs2 + kWd * bs1 + kWe * v2;
            h23r = kD1a * (c_m2 - c_p2) + kD1b * (c_p1 - c_m1);
            float a32r = kD2a * (c_m2 + c_p2) + kD2b * (c_m1 + c_p1) + kD2c * v3;
            if (x2cl) {
                // closure rows: table corrections (1/h units) converted to raw units
                const X2Corr gdd = x2_geom(i2, N1, n2, 4);
                const X2Corr gw = x2_geom(i2, N1, n2, 6);
                float e_h21 = 0.f, e_a12 = 0.f, e_g2 = 0.f, e_a22 = 0.f, e_h23 = 0.f, e_a32 = 0.f, e_w2 = 0.f;
                x2_corr_dd(A2, gdd, o1, e_h21, e_a12);
                x2_corr_dd(A2, gdd, o2, e_g2, e_a22);
                x2_corr_dd(A2, gdd, o3, e_h23, e_a32);
                x2_corr_w(A2, gw, o2, e_w2);
                h21r += e_h21 * K.h2;
                g2r += e_g2 * K.h2;
                h23r += e_h23 * K.h2;
                a12r += e_a12 * K.h2s;
                a22r += e_a22 * K.h2s;
                a32r += e_a32 * K.h2s;
                w2r += e_w2 * K.h2s;
            }
            // x3 (raw units), one branch for all five
            float g3r, a13r, a23r, a33r, d3v1r;
            if (p >= 4 && p <= n3 - 5) {
                g3r = x3d1i(v3w, IC<UP>{});
                a13r = x3d2i(v1w, IC<UP>{});
                a23r = x3d2i(v2w, IC<UP>{});
                a33r = x3d2i(v3w, IC<UP>{});
                d3v1r = x3d1i(v1w, IC<UP>{});
            } else {
                const int r3 = p < 4 ? p : 4 + (n3 - 1 - p);
                g3r = x3d1c(v3w, IC<UP>{}, r3);
                a13r = x3d2c(v1w, IC<UP>{}, r3);
                a23r = x3d2c(v2w, IC<UP>{}, r3);
                a33r = x3d2c(v3w, IC<UP>{}, r3);
                d3v1r = x3d1c(v1w, IC<UP>{}, r3);
            }
            const float F1 = K.lam * G1 + K.lpm_h2 * g2r + K.lpm_h3 * g3r;
            F3 = K.lam_h3 * g3r + K.lpm * G1 + K.lpm_h2 * g2r;
            w1 = K.mu2 * A11 + K.mu_h2s * a12r + K.mu_h3s * a13r;
            w2p = K.mu * A21 + K.mu2_h2s * a22r + K.mu_h3s * a23r + K.lam_h2s * w2r;
            w3p = K.mu * A31 + K.mu_h2s * a32r + K.mu2_h3s * a33r;
            if (is_face) {
                // Traction on the fixed +x1 axis and SAT c (tau+ - tau-) on both
                // faces; the other side of the node is the adjacent lane. The
                // +x1 boundary derivative runs over the same x1 window (plus
                // side: window columns 0..3; minus side: columns 5..2, odd mirror).
                float dh1 = 0.f, dh2 = 0.f, dh3 = 0.f;
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    const float cd = side == 1 ? (k < 4 ? A1.dlo[k] : 0.f) : (k >= 2 ? -A1.dlo[5 - k] : 0.f);
                    dh1 += cd * l1[k];
                    dh2 += cd * l2[k];
                    dh3 += cd * l3[k];
                }
                const float tau1 = K.lam * G1 + K.lam_h2 * g2r + K.lam_h3 * g3r + K.mu2 * dh1;
                const float tau2 = K.mu_h2 * h21r + K.mu * dh2;
                const float tau3 = K.mu_h3 * d3v1r + K.mu * dh3;
                const float o1t = __shfl_xor_sync(facemask, tau1, 1);
                const float o2t = __shfl_xor_sync(facemask, tau2, 1);
                const float o3t = __shfl_xor_sync(facemask, tau3, 1);
                const float cs = K.sat * sgn;
                w1 += cs * (tau1 - o1t);
                w2p += cs * (tau2 - o2t);
                w3p += cs * (tau3 - o3t);
            }
            if (valid) {
                xF1[BUF * NPT + pidx] = F1;
                xH21[BUF * NPT + pidx] = h21r;
            }
        }
        F3w[UP] = F3;
        H23w[UP] = h23r;
        __syncthreads();
        if (s_dead[BUF]) {
            dead_at = s;
            return false;
        }
        // The slot of plane p is free: every thread is past its reads.
        if (s + kRingAhead < n3) {
            if (tid == 0) issue_plane(s + kRingAhead);
            issued = s + kRingAhead + 1;
        }

        // ---- component 1 of p; components 2, 3 of p enter the queue ------------
        if (pin) {
            const float *xf = xF1 + BUF * NPT + pline;
            const float *xh = xH21 + BUF * NPT + pline;
            float E1 = 0.f, e21r = 0.f;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                E1 += c1[k] * xf[k];
                e21r += c1[k] * xh[k];
            }
            float u1 = w1 + E1;
            if (is_face) u1 = 0.5f * (u1 + __shfl_xor_sync(facemask, u1, 1));
            const float y1 = hpt * plane_w(p) * u1;
            if (valid) {
                ocol[(long long)p * g.PS] = y1;
                const double v1 = (double)v1w[UP];
                acc0 = fma(v1, (double)y1, acc0);
                acc1 = fma(v1, v1, acc1);
            }
            w2q[QP] = w2p + K.lpm_h2 * e21r;
            w3q[QP] = w3p;
        }
        // ---- components 2, 3 of z ----------------------------------------------
        const int z = s - 6;
        if (z >= 0 && z < n3) {
            float dh, df;
            if (z >= 4 && z <= n3 - 5) {
                dh = x3d1i(H23w, IC<UZ>{});
                df = x3d1i(F3w, IC<UZ>{});
            } else {
                const int r3z = z < 4 ? z : 4 + (n3 - 1 - z);
                dh = x3d1c(H23w, IC<UZ>{}, r3z);
                df = x3d1c(F3w, IC<UZ>{}, r3z);
            }
            float u2 = w2q[QZ] + K.lpm_h2h3 * dh;
            float u3 = w3q[QZ] + K.h3i * df;
            if (is_face) {
                u2 = 0.5f * (u2 + __shfl_xor_sync(facemask, u2, 1));
                u3 = 0.5f * (u3 + __shfl_xor_sync(facemask, u3, 1));
            }
            const float hw = hpt * plane_w(z);
            const float y2 = hw * u2, y3 = hw * u3;
            if (valid) {
                ocol[cstr + (long long)z * g.PS] = y2;
                ocol[2 * cstr + (long long)z * g.PS] = y3;
                const double v2 = (double)v2w[UZ], v3 = (double)v3w[UZ];
                acc0 = fma(v2, (double)y2, acc0);
                acc0 = fma(v3, (double)y3, acc0);
                acc1 = fma(v2, v2, acc1);
                acc1 = fma(v3, v3, acc1);
            }
        }
        return true;
    };

    bool alive = true;
    if constexpr (DYN) {
        // Slot 0 holds the newest plane; after a step every window moves one
        // entry toward older planes (slot k -> slot k - 1 mod 8).
        auto rot8 = [](float (&w)[kRing]) {
            const float t = w[0];
#pragma unroll
            for (int k = 0; k < kRing - 1; ++k) w[k] = w[k + 1];
            w[kRing - 1] = t;
        };
        auto rot4 = [](float (&w)[4]) {
            const float t = w[0];
#pragma unroll
            for (int k = 0; k < 3; ++k) w[k] = w[k + 1];
            w[3] = t;
        };
#pragma unroll 1
        for (int s = 0; s < s_end && alive; ++s) {
            alive = step(IC<0>{}, s);
            rot8(v1w);
            rot8(v2w);
            rot8(v3w);
            rot8(F3w);
            rot8(H23w);
            rot4(w2q);
            rot4(w3q);
        }
    }
    for (int s0 = 0; s0 < s_end && alive && !DYN; s0 += kRing) {
#define EQD_RING_STEP(U) \
    if (alive && s0 + U < s_end) alive = step(IC<U>{}, s0 + U);
        EQD_RING_STEP(0)
        EQD_RING_STEP(1)
        EQD_RING_STEP(2)
        EQD_RING_STEP(3)
        EQD_RING_STEP(4)
        EQD_RING_STEP(5)
        EQD_RING_STEP(6)
        EQD_RING_STEP(7)
#undef EQD_RING_STEP
    }

    if (!alive) {
        // A wait gave up (recorded in *err). Before the CTA's shared memory is
        // released, wait (with the default bound) for every plane copy issued
        // and not yet consumed: planes dead_at .. issued - 1 (a dropped plane
        // was never issued).
        if (tid == 0) {
            for (int q = dead_at; q < issued; ++q)
                if (q != g.drop_plane) ring_wait(&mbar[q & (kRing - 1)], (unsigned)(q >> 3) & 1u, err, 0u);
        }
        __syncthreads();
        return;
    }

    // Per (column, tile): block tree over the whole march.
    const double s0v = block_sum(acc0, red);
    __syncthreads();
    const double s1v = block_sum(acc1, red);
    if (tid == 0 && partials) {
        double *pp = partials + ((long long)col * g.ntiles + tile) * 2;
        pp[0] = s0v;
        pp[1] = s1v;
    }
}

}  // namespace eqd
