// libeqd host side: grid set-up, launch geometry, the batched CG driver and
// the C ABI declared in include/eqd.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <condition_variable>
#include <deque>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "../../include/eqd.h"
#include "ops_tables.h"
#include "solver_kernels.cuh"
#include "rhs_kernels.cuh"
#include "ring_march.cuh"

using namespace eqd;

// ---------------------------------------------------------------------------
// Errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

static int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

#define CUDA_OR_RETURN(call)                                                                       \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            return fail(e_ == cudaErrorMemoryAllocation ? EQD_ERR_OOM : EQD_ERR_CUDA,              \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                       \
        }                                                                                          \
    } while (0)

// ---------------------------------------------------------------------------
// Device buffers
// ---------------------------------------------------------------------------
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    cudaError_t ensure(size_t n) {
        if (n <= bytes) return cudaSuccess;
        release();
        cudaError_t e = cudaMalloc(&p, n);
        if (e == cudaSuccess) bytes = n;
        else p = nullptr;
        return e;
    }
    template <typename T> T *as() const { return static_cast<T *>(p); }
};

// Launch configuration of the plane-march apply for one precision.
struct MarchCfg {
    MarchGeom g;
    int threads = 0;
    size_t smem = 0;
    size_t smem_af = 0;  // MODE_AF (second plane ring); 0: does not fit, the direction update runs apart
    int ring_t2 = 0;     // > 0: the FP32 A-apply runs ring_march_kernel with this x2 tile capacity
    int ring_var = 0;    // which of the two ring-march instances of this n1 (0: A, 1: B)
    RingGeom rg{};
};

static constexpr int kMaxT32 = 640;   // generic FP32 instances
static constexpr int kMaxT32b = 512;  // FP32 A-apply variant without register spills
static constexpr int kMaxT32c = 384;  // FP32 A-apply, two columns per thread
static constexpr int kMaxT64 = 384;
static constexpr int kMaxT64b = 512;  // FP64 instances for wide x1 lines (n1 = 33 needs 7 x 66 threads)
static constexpr int kNumVariants = 11;  // 9 plane-march variants, then 2 ring-march variants
static constexpr int kFirstRingVariant = 9;

// Ring-march instances per n1: (x2 tile capacity, register cap per thread)
// of its two variants. A CTA's threads x registers must fit the SM's 65,536,
// with registers counted in units of 16 per thread (136 measured as too many
// for 480 threads); 128 registers spill a few bytes.
template <int N1> struct RingTraits;
// Variant A unrolls the march over the ring; variant B is the same tile
// without the unrolling (DYN: smaller code, window moves).
template <> struct RingTraits<9> { static constexpr int T2A = 7, MA = 128, T2B = 7, MB = 128; };
template <> struct RingTraits<21> { static constexpr int T2A = 7, MA = 128, T2B = 7, MB = 128; };
template <> struct RingTraits<33> { static constexpr int T2A = 7, MA = 96, T2B = 7, MB = 96; };
static_assert(ring_threads(9, RingTraits<9>::T2B) * RingTraits<9>::MB <= 65536, "ring CTA exceeds the register file");
static_assert(ring_threads(21, RingTraits<21>::T2B) * RingTraits<21>::MB <= 65536, "ring CTA exceeds the register file");
static_assert(ring_threads(33, RingTraits<33>::T2A) * RingTraits<33>::MA <= 65536, "ring CTA exceeds the register file");
static_assert(ring_threads(33, RingTraits<33>::T2B) * RingTraits<33>::MB <= 65536, "ring CTA exceeds the register file");

// The largest CTA the device will launch for a ring-march instance (its
// register use included).
template <int N1>
static int ring_max_threads(int which) {
    using R = RingTraits<N1>;
    cudaFuncAttributes fa{};
    cudaError_t e = which == 0 ? cudaFuncGetAttributes(&fa, ring_march_kernel<N1, R::T2A, R::MA>)
                               : cudaFuncGetAttributes(&fa, ring_march_kernel<N1, R::T2B, R::MB, true>);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return fa.maxThreadsPerBlock;
}

static int ring_launchable_threads(int n1, int which) {
    switch (n1) {
    case 9: return ring_max_threads<9>(which);
    case 21: return ring_max_threads<21>(which);
    case 33: return ring_max_threads<33>(which);
    default: return 0;
    }
}

static int ring_t2_for(int n1, int which) {
    switch (n1) {
    case 9: return which == 0 ? RingTraits<9>::T2A : RingTraits<9>::T2B;
    case 21: return which == 0 ? RingTraits<21>::T2A : RingTraits<21>::T2B;
    case 33: return which == 0 ? RingTraits<33>::T2A : RingTraits<33>::T2B;
    default: return 0;
    }
}

// Launch configuration of ring_march_kernel: 7-row tiles at both x2 ends,
// the rows between split into tiles of at most t2 rows.
static bool make_ring_cfg(const GridConst &gc, const double h[3], int which, MarchCfg &out, std::string &why) {
    const int t2 = ring_t2_for(gc.n1, which);
    if (t2 <= 0) {
        why = "ring march: n1 = " + std::to_string(gc.n1) + " has no specialised instance";
        return false;
    }
    if (gc.n2 < 2 * kRingEdge) {
        why = "ring march: n2 below 14";
        return false;
    }
    if (ring_threads(gc.n1, t2) > ring_launchable_threads(gc.n1, which)) {
        why = "ring march: the CTA does not fit the device's register file";
        return false;
    }
    const int m = gc.n2 - 2 * kRingEdge;
    const int nmid = m > 0 ? (m + t2 - 1) / t2 : 0;
    out = MarchCfg{};
    out.ring_t2 = t2;
    out.ring_var = which;
    out.rg.n2 = gc.n2;
    out.rg.n3 = gc.n3;
    out.rg.PS = gc.PS;
    out.rg.colstride = gc.colstride;
    out.rg.ntiles = nmid + 2;
    out.rg.nmid = std::max(nmid, 1);
    out.rg.drop_plane = -1;
    out.rg.poll_limit = 0;
    {
        const double lam = gc.lam, mu = gc.mu, lpm = gc.lam + gc.mu;
        const double h2 = h[1], h3 = h[2], h2i = 1.0 / h2, h3i = 1.0 / h3;
        RingScal &k = out.rg.k;
        k.lam = (float)lam;
        k.mu = (float)mu;
        k.mu2 = (float)(2 * mu);
        k.lpm = (float)lpm;
        k.lpm_h2 = (float)(lpm * h2i);
        k.lpm_h3 = (float)(lpm * h3i);
        k.lam_h2 = (float)(lam * h2i);
        k.lam_h3 = (float)(lam * h3i);
        k.mu_h2 = (float)(mu * h2i);
        k.mu_h3 = (float)(mu * h3i);
        k.mu_h2s = (float)(mu * h2i * h2i);
        k.mu2_h2s = (float)(2 * mu * h2i * h2i);
        k.lam_h2s = (float)(lam * h2i * h2i);
        k.mu_h3s = (float)(mu * h3i * h3i);
        k.mu2_h3s = (float)(2 * mu * h3i * h3i);
        k.lpm_h2h3 = (float)(lpm * h2i * h3i);
        k.h3i = (float)h3i;
        k.h2 = (float)h2;
        k.h2s = (float)(h2 * h2);
        k.h3 = (float)h3;
        k.h3s = (float)(h3 * h3);
        k.sat = (float)gc.sat_c;
    }
    out.g.n1 = gc.n1;
    out.g.n2 = gc.n2;
    out.g.n3 = gc.n3;
    out.g.PS = gc.PS;
    out.g.colstride = gc.colstride;
    out.g.ntiles = out.rg.ntiles;
    out.g.t2max = t2;
    out.g.nblk = 1;
    out.g.nseg = 1;
    out.g.segblk = 1;
    out.g.edge = kRingEdge;
    out.threads = ring_threads(gc.n1, t2);
    out.smem = ring_smem(gc.n1, t2);
    out.smem_af = 0;  // the direction update is not fused into this kernel
    return true;
}

static bool n1_specialized(int n1) { return n1 == 9 || n1 == 21 || n1 == 33; }

// `maxt` limits the threads of the tile; `kmaxt` is the launch bound of the
// kernel instance that will run it (it fixes the shared-memory geometry of
// the n1-specialized instances).
template <typename T>
static bool make_march_cfg(int n1, int n2, int n3, int PS, long long colstride, int maxt, int tile_rows,
                           const GridConst &gc, MarchCfg &out, std::string &why, int lanes = 1, int kmaxt = 0,
                           bool edge_mode = false) {
    if (kmaxt == 0) kmaxt = maxt;
    const int per_row = 2 * n1;
    int t2 = tile_rows > 0 ? std::min(tile_rows, maxt / per_row) : maxt / per_row;
    t2 = std::min(t2, n2);
    if (t2 * per_row > maxt) t2 = maxt / per_row;
    int ntiles = (n2 + t2 - 1) / t2;
    if (ntiles < 1) ntiles = 1;
    // Balanced tiles, every tile at least 7 rows: the wide operator's closure
    // rows reach 10 rows in from the boundary, and a tile reads 4 halo rows.
    while (ntiles > 1 && n2 / ntiles < 7) --ntiles;
    int t2max = (n2 + ntiles - 1) / ntiles;
    int edge = 0;
    // Edge partition: forced (a launch variant that keeps every x2 closure row
    // in 7-row edge tiles, so no CTA mixes closure and interior rows), or
    // needed when balanced tiles of >= 7 rows do not fit the thread limit.
    if ((edge_mode || t2max * per_row > maxt) && t2 >= 7 && n2 >= 14) {
        // Tiles of at most t2 rows: 7-row tiles at both ends carry the closure
        // rows, the tiles between (any height) split the interior.
        edge = 7;
        const int m = n2 - 2 * edge;
        const int nm = m > 0 ? (m + t2 - 1) / t2 : 0;
        ntiles = nm + 2;
        t2max = std::max(edge, nm > 0 ? (m + nm - 1) / nm : 0);
    }
    if (t2max * per_row > maxt || (edge == 0 && n2 / ntiles < std::min(7, n2))) {
        why = "grid too large in x1 for one CTA (n1=" + std::to_string(n1) + ")";
        return false;
    }
    constexpr int AE = 16 / (int)sizeof(T);
    int CH = (t2max + 2 * EQD_HALO) * n1 + 2 * AE;
    CH = (CH + AE - 1) / AE * AE;
    int NP = 2 * n1 * t2max;
    if (n1_specialized(n1)) {
        if (t2max > march_t2cap(n1, kmaxt)) {
            why = "tile exceeds the specialized kernel's capacity";
            return false;
        }
        CH = march_chcap(n1, kmaxt, (int)sizeof(T));
        NP = 2 * n1 * march_t2cap(n1, kmaxt);
    }
    out.g.n1 = n1;
    out.g.n2 = n2;
    out.g.n3 = n3;
    out.g.PS = PS;
    out.g.colstride = colstride;
    out.g.ntiles = ntiles;
    out.g.t2max = t2max;
    out.g.edge = edge;
    out.g.CH = CH;
    out.g.i2f0 = gc.i2f0;
    out.g.n2f = gc.n2f;
    out.g.i3f0 = gc.i3f0;
    out.g.n3f = gc.n3f;
    out.g.nf = gc.nf;
    // FP64-input instances sum dot products per x3 step block (and can split
    // a column along x3); FP32 ones per tile over the whole column.
    out.g.nblk = sizeof(T) == 8 ? (n3 + EQD_PBLK - 1) / EQD_PBLK : 1;
    out.g.nseg = 1;
    out.g.segblk = out.g.nblk;
    int threads = per_row * t2max;
    threads = (threads + 31) / 32 * 32;
    out.threads = threads;
    // barriers + flags, reduction scratch, and per column: plane ring, F1/H21
    // exchange [2][points] x 2; FP64: per-(step block, warp) dot-product sums
    out.smem = 64 + 32 * 8 + (size_t)lanes * ((size_t)EQD_NSLOT * 6 * CH + 4 * (size_t)NP) * sizeof(T);
    if (sizeof(T) == 8) out.smem += 16 + (size_t)lanes * out.g.nblk * (threads / 32) * 2 * sizeof(double);
    // MODE_AF adds the ring of r planes (aligned to 128 bytes after the rest).
    out.smem_af = out.smem + 144 + (size_t)lanes * EQD_NSLOT * 6 * CH * sizeof(T);
    return true;
}

// Dot-product partials per column of a launch configuration: one per
// (x2 tile, x3 step block) for FP64-input configurations, one per x2 tile
// for FP32 ones (nblk = 1).
static int nparts(const MarchCfg &m) { return m.g.ntiles * m.g.nblk; }

// x3 segmentation of an FP64-input launch: a batch too small to give every
// SM two CTAs is split along x3 into segments of whole step blocks (a
// segment marches 9 to 14 planes before its first block to fill its windows
// and 3 planes past its last). Partials are per step block, so the results
// do not depend on the split.
static MarchCfg segmented(const MarchCfg &m, long long groups, int num_sms) {
    MarchCfg r = m;
    const long long ctas = groups * m.g.ntiles;
    const long long target = 2LL * num_sms;
    if (ctas >= target || m.g.nblk <= 1) return r;
    const int want = (int)std::min<long long>((target + ctas - 1) / ctas, m.g.nblk);
    r.g.segblk = (m.g.nblk + want - 1) / want;
    r.g.nseg = (m.g.nblk + r.g.segblk - 1) / r.g.segblk;
    return r;
}

template <typename T>
static void fill_op(OpConst<T> &C, const GridConst &gc, const double h[3]) {
    for (int a = 0; a < 3; ++a) fill_axis<T>(C.ax[a], a == 0 ? gc.n1 : (a == 1 ? gc.n2 : gc.n3), h[a]);
    C.lam = (T)gc.lam;
    C.mu = (T)gc.mu;
    C.lpm = (T)(gc.lam + gc.mu);
    C.sat_c = (T)gc.sat_c;
    C.hvol = gc.hvol;
}

// Page-locked host array: device-to-host copies into it stay asynchronous.
template <typename E>
struct PinnedArr {
    E *p = nullptr;
    int n = 0;
    PinnedArr() = default;
    PinnedArr(const PinnedArr &) = delete;
    PinnedArr &operator=(const PinnedArr &) = delete;
    ~PinnedArr() {
        if (p) cudaFreeHost(p);
    }
    cudaError_t assign(int count, E v) {
        if (count > n) {
            if (p) cudaFreeHost(p);
            p = nullptr;
            n = 0;
            cudaError_t e = cudaHostAlloc((void **)&p, sizeof(E) * std::max(count, 1), cudaHostAllocDefault);
            if (e != cudaSuccess) return e;
            n = count;
        }
        for (int i = 0; i < count; ++i) p[i] = v;
        return cudaSuccess;
    }
    E *data() { return p; }
    E &operator[](int i) { return p[i]; }
    const E &operator[](int i) const { return p[i]; }
};

// Workspace of one batched solve (grown on demand, reused across calls).
struct Workspace {
    int cap = 0;            // columns
    int precision = -1;
    DevBuf x64, v0, v1, v2, v3;  // x64 + (r, p, q, d) in the working precision
    DevBuf v4;                   // fused direction update: the other p buffer (p alternates v1, v4)
    DevBuf apply_part, res_part, rr_part;
    DevBuf gamma, beta, rr_ref, tol, bnorm, iters, status, flag;
    DevBuf slip_node, slip_comp, slip_dense;
    DevBuf kout;
    DevBuf newmask, slot_list, dst_list;  // slot engine: entering columns, extraction lists
    DevBuf hbuf;                          // explicit-RHS staging (reference layout)
    PinnedArr<double> kstage;             // finished K columns on their way to a host K
    cudaGraphExec_t graph = nullptr;
    int graph_iters = 0;
    bool graph_split = false;  // the captured iterations run as two halves
    std::vector<uint64_t> graph_key;  // what the captured graph baked in (see SlotRun::setup)
    ~Workspace() {
        if (graph) cudaGraphExecDestroy(graph);
    }
};

struct eqd_grid {
    eqd_grid_desc desc;
    GridConst gc;
    double h[3];
    OpConst<float> c32;
    OpConst<double> c64;
    MarchCfg m32, m64;
    int m64_maxt = 384;   // launch bound of the FP64 instance the grid runs
    bool served = false;  // attached to an eqd_server (its worker owns the grid)
    int num_sms = 148;
    DevBuf dinv64, dinv32;   // Jacobi weights (one column, device layout)
    bool jacobi_ready = false;
    // FP32 A-apply launch variants (see make_variants) and the chosen one.
    MarchCfg v32[kNumVariants];
    int v32_maxt[kNumVariants] = {};
    int v32_lanes[kNumVariants] = {};
    int sel32 = 0;
    bool tuned = false;
    int chunk_tuned = 0;   // eqd_tune_chunk's choice of columns per batch (0: as many as the budget allows)
    double tune_ms[kNumVariants] = {};
    int nchunks = 1;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;          // second half of a split batch (graph capture only)
    cudaStream_t stream_hi = nullptr, stream2_hi = nullptr;  // high priority: vector kernels of the halves
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    cudaEvent_t evA = nullptr, evB = nullptr, evFork = nullptr, evJoin = nullptr, evArest = nullptr,
                evBrest = nullptr;
    DevBuf err;           // device error word
    Workspace ws;
    std::mutex mtx;
    std::vector<double> x2f, x3f;
    int tile_rows = 0;
    int test_drop_plane = -1;      // eqd_test_inject_wait_timeout: the next ring launch never copies this plane
    unsigned test_poll_limit = 0;
};

struct eqd_kmat {
    int device;
    int n;
    int ks_slots[3] = {296, 296, 296};  // resident CTAs of the blocked K S (16, 32, 64 vectors per CTA)
    DevBuf K, s, y, part;
    cudaStream_t stream = nullptr;
};

// ---------------------------------------------------------------------------
// Kernel launch helpers
// ---------------------------------------------------------------------------
// Kernel instances compiled for a fixed n1 (the BP8 grids' 9, 21, 33 points
// across a side); any other n1 runs the runtime-n1 instance.
#define EQD_FOR_N1(X) X(9) X(21) X(33)

template <typename T, typename TO, int MODE, int MAXT, int L = 1>
static void launch_n1(int n1, dim3 grid, const MarchCfg &m, cudaStream_t st, const OpConst<T> &C, const T *in,
                      TO *out, ColumnSet cs, double *partials, unsigned *err) {
    switch (n1) {
#define EQD_CASE(N)                                                                                       \
    case N:                                                                                               \
        plane_march_kernel<T, TO, MODE, MAXT, N, L><<<grid, m.threads, m.smem, st>>>(C, m.g, in, out, cs, \
                                                                                     partials, err);      \
        return;
        EQD_FOR_N1(EQD_CASE)
#undef EQD_CASE
    default:
        plane_march_kernel<T, TO, MODE, MAXT, 0, L><<<grid, m.threads, m.smem, st>>>(C, m.g, in, out, cs,
                                                                                     partials, err);
    }
}

template <int N1>
static void launch_ring_n1(int which, dim3 grid, const MarchCfg &m, const RingGeom &rg, cudaStream_t st,
                           const OpConst<float> &C, const float *in, float *out, const int8_t *status,
                           double *partials, unsigned *err) {
    using R = RingTraits<N1>;
    if (which == 0)
        ring_march_kernel<N1, R::T2A, R::MA><<<grid, m.threads, m.smem, st>>>(C, rg, in, out, status, partials, err);
    else
        ring_march_kernel<N1, R::T2B, R::MB, true><<<grid, m.threads, m.smem, st>>>(C, rg, in, out, status, partials,
                                                                                     err);
}

// The FP32 CG apply through ring_march_kernel (one CTA per column and x2
// tile). A pending test injection (eqd_test_inject_wait_timeout) applies to
// this launch only.
static cudaError_t launch_ring(eqd_grid *G, const MarchCfg &m, const float *in, float *out, const ColumnSet &cs,
                               double *partials, int ncols, cudaStream_t st) {
    RingGeom rg = m.rg;
    if (G->test_drop_plane >= 0) {
        rg.drop_plane = G->test_drop_plane;
        rg.poll_limit = G->test_poll_limit;
        G->test_drop_plane = -1;
    }
    const dim3 grid((unsigned)((long long)ncols * rg.ntiles));
    unsigned *err = G->err.as<unsigned>();
    switch (G->gc.n1) {
    case 9: launch_ring_n1<9>(m.ring_var, grid, m, rg, st, G->c32, in, out, cs.status, partials, err); break;
    case 21: launch_ring_n1<21>(m.ring_var, grid, m, rg, st, G->c32, in, out, cs.status, partials, err); break;
    case 33: launch_ring_n1<33>(m.ring_var, grid, m, rg, st, G->c32, in, out, cs.status, partials, err); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename T, typename TO, int MODE>
static cudaError_t launch_march(eqd_grid *G, const T *in, TO *out, ColumnSet cs, double *partials, int ncols,
                                int variant = -1, cudaStream_t stream = nullptr) {
    cs.ncols = ncols;
    cudaStream_t st = stream ? stream : G->stream;
    const int n1 = G->gc.n1;
    if constexpr (sizeof(T) == 4 && (MODE == MODE_A || MODE == MODE_AF)) {
        const int v = variant >= 0 ? variant : G->sel32;
        if (G->v32[v].ring_t2 > 0) {
            if (MODE == MODE_AF) return cudaErrorInvalidValue;  // not fused in this kernel (smem_af = 0)
            return launch_ring(G, G->v32[v], reinterpret_cast<const float *>(in), reinterpret_cast<float *>(out), cs,
                               partials, ncols, st);
        }
        const int lanes = G->v32_lanes[v];
        const long long groups = (ncols + lanes - 1) / lanes;
        MarchCfg m = segmented(G->v32[v], groups, G->num_sms);
        if (MODE == MODE_AF) m.smem = m.smem_af;
        dim3 grid((unsigned)(groups * m.g.ntiles * m.g.nseg));
        const float *fin = reinterpret_cast<const float *>(in);
        float *fout = reinterpret_cast<float *>(out);
        if (lanes == 2)
            launch_n1<float, float, MODE, kMaxT32c, 2>(n1, grid, m, st, G->c32, fin, fout, cs, partials,
                                                        G->err.as<unsigned>());
        else if (G->v32_maxt[v] == kMaxT32)
            launch_n1<float, float, MODE, kMaxT32>(n1, grid, m, st, G->c32, fin, fout, cs, partials,
                                                   G->err.as<unsigned>());
        else
            launch_n1<float, float, MODE, kMaxT32b>(n1, grid, m, st, G->c32, fin, fout, cs, partials,
                                                    G->err.as<unsigned>());
        return cudaGetLastError();
    }
    constexpr int MAXT = sizeof(T) == 4 ? kMaxT32 : kMaxT64;
    MarchCfg m = segmented(sizeof(T) == 4 ? G->m32 : G->m64, ncols, G->num_sms);
    if (MODE == MODE_AF) m.smem = m.smem_af;
    const OpConst<T> &C = *reinterpret_cast<const OpConst<T> *>(sizeof(T) == 4 ? (const void *)&G->c32
                                                                               : (const void *)&G->c64);
    dim3 grid((unsigned)(ncols * m.g.ntiles * m.g.nseg));
    const bool wide64 = sizeof(T) == 8 && G->m64_maxt == kMaxT64b;
    if (MODE == MODE_AP) {  // generic-input hook: runtime-n1 instance only
        if (wide64)
            plane_march_kernel<T, TO, MODE, kMaxT64b, 0, 1><<<grid, m.threads, m.smem, st>>>(
                C, m.g, in, out, cs, partials, G->err.as<unsigned>());
        else
            plane_march_kernel<T, TO, MODE, MAXT, 0, 1><<<grid, m.threads, m.smem, st>>>(
                C, m.g, in, out, cs, partials, G->err.as<unsigned>());
    } else if (wide64) {
        launch_n1<T, TO, MODE, kMaxT64b>(n1, grid, m, st, C, in, out, cs, partials, G->err.as<unsigned>());
    } else {
        launch_n1<T, TO, MODE, MAXT>(n1, grid, m, st, C, in, out, cs, partials, G->err.as<unsigned>());
    }
    return cudaGetLastError();
}

// Dynamic shared memory above 48 KB must be opted into per kernel.
static cudaError_t configure_kernels(int smem_max) {
#define EQD_KS(N)                                                                \
    (const void *)plane_march_kernel<float, float, MODE_A, kMaxT32, N, 1>,       \
        (const void *)plane_march_kernel<float, float, MODE_A, kMaxT32b, N, 1>,    \
        (const void *)plane_march_kernel<float, float, MODE_A, kMaxT32c, N, 2>,    \
        (const void *)plane_march_kernel<float, float, MODE_RHS, kMaxT32, N, 1>,   \
        (const void *)plane_march_kernel<double, double, MODE_A, kMaxT64, N, 1>,   \
        (const void *)plane_march_kernel<double, double, MODE_RHS, kMaxT64, N, 1>, \
        (const void *)plane_march_kernel<double, float, MODE_RHS, kMaxT64, N, 1>,   \
        (const void *)plane_march_kernel<double, double, MODE_A, kMaxT64b, N, 1>,  \
        (const void *)plane_march_kernel<double, double, MODE_RHS, kMaxT64b, N, 1>, \
        (const void *)plane_march_kernel<double, float, MODE_RHS, kMaxT64b, N, 1>,       \
        (const void *)plane_march_kernel<float, float, MODE_AF, kMaxT32, N, 1>,          \
        (const void *)plane_march_kernel<float, float, MODE_AF, kMaxT32b, N, 1>,         \
        (const void *)plane_march_kernel<float, float, MODE_AF, kMaxT32c, N, 2>,         \
        (const void *)plane_march_kernel<double, double, MODE_AF, kMaxT64, N, 1>,        \
        (const void *)plane_march_kernel<double, double, MODE_AF, kMaxT64b, N, 1>,
#define EQD_RING_KS(N)                                                                                     \
    (const void *)ring_march_kernel<N, RingTraits<N>::T2A, RingTraits<N>::MA>,                             \
        (const void *)ring_march_kernel<N, RingTraits<N>::T2B, RingTraits<N>::MB, true>,
    const void *ks[] = {
        EQD_FOR_N1(EQD_KS) EQD_KS(0)
        (const void *)plane_march_kernel<float, float, MODE_AP, kMaxT32, 0, 1>,
        (const void *)plane_march_kernel<double, double, MODE_AP, kMaxT64, 0, 1>,
        (const void *)plane_march_kernel<double, double, MODE_AP, kMaxT64b, 0, 1>,
        EQD_FOR_N1(EQD_RING_KS)
    };
#undef EQD_RING_KS
#undef EQD_KS
    for (const void *k : ks) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

static int check_device_error(eqd_grid *G) {
    unsigned h = 0;
    CUDA_OR_RETURN(cudaMemcpyAsync(&h, G->err.p, sizeof(unsigned), cudaMemcpyDeviceToHost, G->stream));
    CUDA_OR_RETURN(cudaStreamSynchronize(G->stream));
    if (h != 0) {
        cudaMemsetAsync(G->err.p, 0, sizeof(unsigned), G->stream);
        return fail(EQD_ERR_TIMEOUT, "a device-side bounded wait gave up (error word " + std::to_string(h) + ")");
    }
    return EQD_OK;
}

// ---------------------------------------------------------------------------
// Library info
// ---------------------------------------------------------------------------
extern "C" const char *eqd_last_error(void) { return g_last_error.c_str(); }
extern "C" const char *eqd_version(void) { return "eqd-b200 0.1 (sm_100a)"; }

extern "C" void eqd_default_opts(eqd_solve_opts *o) {
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->rtol = 1e-10;
    o->atol = 0.0;
    o->itmax = 0;
    o->precond = EQD_PRECOND_NONE;
    o->precision = EQD_PREC_MIXED;
    o->chunk = 0;
    o->reliable_delta = 0.01;
    o->hbm_budget_bytes = 0;
    o->variant = 0;
    o->flags = 0;
}

extern "C" int eqd_device_count(int32_t *count) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) n = 0;
    if (count) *count = n;
    return n > 0 ? EQD_OK : fail(EQD_ERR_NO_DEVICE, "no CUDA device visible");
}

// ---------------------------------------------------------------------------
// Grid
// ---------------------------------------------------------------------------
static bool on_node(double x, double l_f, double tol) { return std::fabs(x) <= l_f + tol; }

extern "C" int eqd_grid_create(const eqd_grid_desc *d, eqd_grid **out) {
    if (!d || !out) return fail(EQD_ERR_ARG, "null argument");
    *out = nullptr;
    if (d->order != 4) return fail(EQD_ERR_ARG, "only SBP order 4 (standard_diagonal.toml) is supported");
    if (d->n1 < 9 || d->n2 < 9 || d->n3 < 9)
        return fail(EQD_ERR_ARG, "SBP order 4 needs at least 9 points per axis (got " + std::to_string(d->n1) + "x" +
                                     std::to_string(d->n2) + "x" + std::to_string(d->n3) + ")");
    if (d->n1 > EQD_MAX_N1) return fail(EQD_ERR_ARG, "n1 above the supported maximum of " + std::to_string(EQD_MAX_N1));
    if (!(d->x1_extent > 0) || !(d->x2_hi > d->x2_lo) || !(d->x3_hi > d->x3_lo))
        return fail(EQD_ERR_ARG, "empty domain");
    if (!(d->mu > 0) || !std::isfinite(d->lambda)) return fail(EQD_ERR_ARG, "invalid Lame parameters");
    if (!(d->l_f >= 0)) return fail(EQD_ERR_ARG, "l_f must be non-negative");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(EQD_ERR_NO_DEVICE, "no CUDA device visible");
    if (d->device < 0 || d->device >= ndev) return fail(EQD_ERR_ARG, "device ordinal out of range");

    std::unique_ptr<eqd_grid> G(new eqd_grid());
    G->desc = *d;
    GridConst &gc = G->gc;
    gc.n1 = d->n1;
    gc.n2 = d->n2;
    gc.n3 = d->n3;
    G->h[0] = d->x1_extent / (d->n1 - 1);
    G->h[1] = (d->x2_hi - d->x2_lo) / (d->n2 - 1);
    G->h[2] = (d->x3_hi - d->x3_lo) / (d->n3 - 1);
    gc.PS = (d->n1 * d->n2 + 3) / 4 * 4;
    gc.colstride = 6LL * d->n3 * gc.PS;
    gc.lam = d->lambda;
    gc.mu = d->mu;
    gc.hvol = G->h[0] * G->h[1] * G->h[2];
    gc.sat_c = 0.5 / (G->h[0] * kHw[0].v());

    // Omega_f (src/FaultResponse.jl:112-126): |x| <= l_f + 1e-9 max(l_f, 1),
    // and the extreme selected nodes must sit on -l_f and +l_f.
    const double tol = 1e-9 * std::max(d->l_f, 1.0);
    auto select = [&](int n, double lo, double hi, const char *name, int &i0, int &cnt, std::vector<double> &ax) -> int {
        std::vector<double> x(n);
        for (int i = 0; i < n; ++i) x[i] = (i == n - 1) ? hi : lo + (hi - lo) * i / (n - 1);
        i0 = -1;
        cnt = 0;
        for (int i = 0; i < n; ++i)
            if (on_node(x[i], d->l_f, tol)) {
                if (i0 < 0) i0 = i;
                ++cnt;
            }
        if (cnt == 0) return fail(EQD_ERR_ARG, "no fault nodes inside Omega_f");
        if (!(std::fabs(x[i0] + d->l_f) <= tol && std::fabs(x[i0 + cnt - 1] - d->l_f) <= tol))
            return fail(EQD_ERR_ARG, std::string("the elastic grid has no nodes exactly on ") + name +
                                         " = +-l_f; pick a spacing that divides l_f");
        ax.assign(x.begin() + i0, x.begin() + i0 + cnt);
        return EQD_OK;
    };
    int rc = select(d->n2, d->x2_lo, d->x2_hi, "x2", gc.i2f0, gc.n2f, G->x2f);
    if (rc) return rc;
    rc = select(d->n3, d->x3_lo, d->x3_hi, "x3", gc.i3f0, gc.n3f, G->x3f);
    if (rc) return rc;
    gc.nf = gc.n2f * gc.n3f;

    CUDA_OR_RETURN(cudaSetDevice(d->device));  // launch limits below are queried for this device
    fill_op<float>(G->c32, gc, G->h);
    fill_op<double>(G->c64, gc, G->h);
    std::string why;
    if (!make_march_cfg<float>(gc.n1, gc.n2, gc.n3, gc.PS, gc.colstride, kMaxT32, 0, gc, G->m32, why))
        return fail(EQD_ERR_ARG, why);
    // FP64: the 384-thread instance where a tile fits, else the 512-thread one.
    G->m64_maxt = kMaxT64;
    if (!make_march_cfg<double>(gc.n1, gc.n2, gc.n3, gc.PS, gc.colstride, kMaxT64, 0, gc, G->m64, why)) {
        G->m64_maxt = kMaxT64b;
        if (!make_march_cfg<double>(gc.n1, gc.n2, gc.n3, gc.PS, gc.colstride, kMaxT64b, 0, gc, G->m64, why))
            return fail(EQD_ERR_ARG, why);
    }
    // FP32 A-apply variants: one large CTA per SM (640-thread bound, may
    // spill), one CTA of up to 512 threads (no spill), CTAs of up to 256
    // threads so that two share an SM, two columns per thread, and small
    // edge-partitioned tiles (closure rows and interior rows in different CTAs).
    {
        // thread limit, kernel launch bound, columns per thread, tile rows
        // (0: as many as fit), edge partition
        const int lim[kFirstRingVariant] = {kMaxT32, kMaxT32b, 256, kMaxT32c, 192, kMaxT32b, kMaxT32b, 192, 448};
        const int mt[kFirstRingVariant] = {kMaxT32, kMaxT32b, kMaxT32b, kMaxT32c, kMaxT32c, kMaxT32b, kMaxT32b,
                                           kMaxT32b, kMaxT32b};
        const int ln[kFirstRingVariant] = {1, 1, 1, 2, 2, 1, 1, 1, 1};
        const int rows[kFirstRingVariant] = {0, 0, 0, 0, 0, 7, 10, 0, 0};
        const bool edg[kFirstRingVariant] = {false, false, false, false, false, true, true, false, false};
        for (int v = 0; v < kNumVariants; ++v) {
            bool ok;
            if (v < kFirstRingVariant) {
                G->v32_maxt[v] = mt[v];
                G->v32_lanes[v] = ln[v];
                ok = make_march_cfg<float>(gc.n1, gc.n2, gc.n3, gc.PS, gc.colstride, lim[v], rows[v], gc, G->v32[v],
                                           why, ln[v], mt[v], edg[v]);
            } else {
                // Ring-march variants: the BP8 lines (n1 = 9, 21, 33) only.
                G->v32_maxt[v] = 0;
                G->v32_lanes[v] = 1;
                ok = make_ring_cfg(gc, G->h, v - kFirstRingVariant, G->v32[v], why);
            }
            if (!ok) {
                G->v32[v] = G->m32;  // fall back to the generic configuration
                G->v32_maxt[v] = kMaxT32;
                G->v32_lanes[v] = 1;
            }
        }
        G->sel32 = 1;
    }
    G->nchunks = (int)std::max<long long>(1, (gc.colstride + 16383) / 16384);

    CUDA_OR_RETURN(cudaSetDevice(d->device));
    {
        int optin = 0;
        CUDA_OR_RETURN(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, d->device));
        size_t need = std::max(G->m32.smem, G->m64.smem);
        for (int v = 0; v < kNumVariants; ++v) need = std::max(need, G->v32[v].smem);
        if ((size_t)optin < need)
            return fail(EQD_ERR_ARG, "stencil tile needs more shared memory than the device offers");
        // A configuration whose second ring does not fit runs the direction
        // update as its own kernel.
        for (MarchCfg *m : {&G->m32, &G->m64})
            if (m->smem_af > (size_t)optin) m->smem_af = 0;
        for (int v = 0; v < kNumVariants; ++v)
            if (G->v32[v].smem_af > (size_t)optin) G->v32[v].smem_af = 0;
        // The limit is a per-kernel attribute shared by every grid of the
        // process: set it to the device maximum, once per device.
        CUDA_OR_RETURN(configure_kernels(optin));
    }
    CUDA_OR_RETURN(cudaDeviceGetAttribute(&G->num_sms, cudaDevAttrMultiProcessorCount, d->device));
    CUDA_OR_RETURN(cudaStreamCreateWithFlags(&G->stream, cudaStreamNonBlocking));
    CUDA_OR_RETURN(cudaStreamCreateWithFlags(&G->stream2, cudaStreamNonBlocking));
    {
        int least = 0, greatest = 0;
        CUDA_OR_RETURN(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CUDA_OR_RETURN(cudaStreamCreateWithPriority(&G->stream_hi, cudaStreamNonBlocking, greatest));
        CUDA_OR_RETURN(cudaStreamCreateWithPriority(&G->stream2_hi, cudaStreamNonBlocking, greatest));
    }
    CUDA_OR_RETURN(cudaEventCreate(&G->ev0));
    CUDA_OR_RETURN(cudaEventCreate(&G->ev1));
    for (cudaEvent_t *e : {&G->evA, &G->evB, &G->evFork, &G->evJoin, &G->evArest, &G->evBrest})
        CUDA_OR_RETURN(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    CUDA_OR_RETURN(G->err.ensure(sizeof(unsigned)));
    CUDA_OR_RETURN(cudaMemset(G->err.p, 0, sizeof(unsigned)));
    *out = G.release();
    return EQD_OK;
}

extern "C" int eqd_grid_destroy(eqd_grid *G) {
    if (!G) return EQD_OK;
    {
        std::lock_guard<std::mutex> lk(G->mtx);
        if (G->served) return fail(EQD_ERR_ARG, "the grid is attached to a server; destroy the server first");
    }
    cudaSetDevice(G->desc.device);
    if (G->stream) cudaStreamSynchronize(G->stream);
    if (G->ev0) cudaEventDestroy(G->ev0);
    if (G->ev1) cudaEventDestroy(G->ev1);
    for (cudaEvent_t e : {G->evA, G->evB, G->evFork, G->evJoin, G->evArest, G->evBrest})
        if (e) cudaEventDestroy(e);
    for (cudaStream_t t : {G->stream2, G->stream_hi, G->stream2_hi})
        if (t) cudaStreamDestroy(t);
    if (G->stream) cudaStreamDestroy(G->stream);
    delete G;
    return EQD_OK;
}

extern "C" int eqd_grid_info(const eqd_grid *G, int64_t *ntot, int32_t *nf, int32_t *n2f, int32_t *n3f) {
    if (!G) return fail(EQD_ERR_ARG, "null grid");
    if (ntot) *ntot = 6LL * G->gc.n1 * G->gc.n2 * G->gc.n3;
    if (nf) *nf = G->gc.nf;
    if (n2f) *n2f = G->gc.n2f;
    if (n3f) *n3f = G->gc.n3f;
    return EQD_OK;
}

extern "C" int eqd_grid_fault_axes(const eqd_grid *G, double *x2f, double *x3f) {
    if (!G) return fail(EQD_ERR_ARG, "null grid");
    if (x2f) std::copy(G->x2f.begin(), G->x2f.end(), x2f);
    if (x3f) std::copy(G->x3f.begin(), G->x3f.end(), x3f);
    return EQD_OK;
}

// ---------------------------------------------------------------------------
// eqd_apply (operator hook)
// ---------------------------------------------------------------------------
template <typename T>
static int apply_impl(eqd_grid *G, const double *x, double *y, int ncols, int mode) {
    const GridConst &gc = G->gc;
    const long long ntot = 6LL * gc.n1 * gc.n2 * gc.n3;
    DevBuf hx, dx, dy;
    CUDA_OR_RETURN(hx.ensure(sizeof(double) * ntot * ncols));
    CUDA_OR_RETURN(dx.ensure(sizeof(T) * gc.colstride * ncols));
    CUDA_OR_RETURN(dy.ensure(sizeof(T) * gc.colstride * ncols));
    CUDA_OR_RETURN(cudaMemsetAsync(dx.p, 0, dx.bytes, G->stream));
    CUDA_OR_RETURN(cudaMemcpyAsync(hx.p, x, sizeof(double) * ntot * ncols, cudaMemcpyHostToDevice, G->stream));
    const long long nel = ntot * ncols;
    const int tb = 256;
    ref_to_dev_kernel<double, T><<<(unsigned)((nel + tb - 1) / tb), tb, 0, G->stream>>>(
        hx.as<double>(), dx.as<T>(), gc.n1, gc.n2, gc.n3, gc.PS, gc.colstride, ncols);
    CUDA_OR_RETURN(cudaGetLastError());
    ColumnSet cs{};
    std::vector<int> neg(ncols, -1), zero(ncols, 0);
    DevBuf sn, sc;
    CUDA_OR_RETURN(sn.ensure(sizeof(int) * ncols));
    CUDA_OR_RETURN(sc.ensure(sizeof(int) * ncols));
    CUDA_OR_RETURN(cudaMemcpyAsync(sn.p, neg.data(), sizeof(int) * ncols, cudaMemcpyHostToDevice, G->stream));
    CUDA_OR_RETURN(cudaMemcpyAsync(sc.p, zero.data(), sizeof(int) * ncols, cudaMemcpyHostToDevice, G->stream));
    cs.slip_node = sn.as<int>();
    cs.slip_comp = sc.as<int>();
    if (mode == 0) {
        CUDA_OR_RETURN((launch_march<T, T, MODE_AP>(G, dx.as<T>(), dy.as<T>(), cs, nullptr, ncols)));
    } else if (mode == 2) {
        DevBuf part;
        int nt = nparts(G->m64);
        for (int v = 0; v < kNumVariants; ++v) nt = std::max(nt, nparts(G->v32[v]));
        CUDA_OR_RETURN(part.ensure(sizeof(double) * 2 * ncols * nt));
        CUDA_OR_RETURN((launch_march<T, T, MODE_A>(G, dx.as<T>(), dy.as<T>(), cs, part.as<double>(), ncols)));
    } else {
        CUDA_OR_RETURN((launch_march<T, T, MODE_RHS>(G, dx.as<T>(), dy.as<T>(), cs, nullptr, ncols)));
    }
    dev_to_ref_kernel<T, double><<<(unsigned)((nel + tb - 1) / tb), tb, 0, G->stream>>>(
        dy.as<T>(), hx.as<double>(), gc.n1, gc.n2, gc.n3, gc.PS, gc.colstride, ncols);
    CUDA_OR_RETURN(cudaGetLastError());
    CUDA_OR_RETURN(cudaMemcpyAsync(y, hx.p, sizeof(double) * ntot * ncols, cudaMemcpyDeviceToHost, G->stream));
    CUDA_OR_RETURN(cudaStreamSynchronize(G->stream));
    return check_device_error(G);
}

extern "C" int eqd_apply(eqd_grid *G, const double *x, double *y, int32_t ncols, int32_t mode, int32_t precision) {
    if (!G || !x || !y) return fail(EQD_ERR_ARG, "null argument");
    if (ncols < 1) return fail(EQD_ERR_ARG, "ncols must be >= 1");
    if (mode < 0 || mode > 2) return fail(EQD_ERR_ARG, "mode must be 0 (A), 1 (HP_DSAT) or 2 (A, input in range(P))");
    std::lock_guard<std::mutex> lk(G->mtx);
    if (G->served) return fail(EQD_ERR_ARG, "the grid is attached to a server");
    CUDA_OR_RETURN(cudaSetDevice(G->desc.device));
    if (precision == EQD_PREC_FP64) return apply_impl<double>(G, x, y, ncols, mode);
    if (precision == EQD_PREC_MIXED) return apply_impl<float>(G, x, y, ncols, mode);
    return fail(EQD_ERR_ARG, "unknown precision");
}

// ---------------------------------------------------------------------------
// Autotuning of the FP32 A-apply launch variant (once per grid): each variant
// is timed on `ncols` device-resident columns; the fastest is kept. The
// choice is fixed for the grid's lifetime, so every column of every later
// call uses the same tile partition (and the same reduction order).
// ---------------------------------------------------------------------------

// ---------------------------------------------------------------------------
// Batched CG driver
// ---------------------------------------------------------------------------
struct BatchSpec {
    int ncols;
    const int *slip_node;        // host, per column (unit slip), or null
    const int *slip_comp;
    const double *slip_dense;    // host [ncols][2][nf] or null
    const double *rhs;           // host reference-layout RHS [ncols][ntot] (explicit-RHS solve) or null
    double *u_out;               // host reference-layout solution (explicit-RHS solve) or null
    double *kcols;               // host 2nf x ncols output (slip-driven) or null
    double *kdev;                // device 2nf x ncols output (slip-driven) or null
    int32_t *iters;
    int8_t *status;
};

static int resolve_chunk(eqd_grid *G, const eqd_solve_opts &o, int ncols, int prec, int &chunk) {
    const GridConst &gc = G->gc;
    // x64 + r, p, q (+ d) (+ the second direction buffer of the fused update).
    const int nvec = 3 + (prec == EQD_PREC_MIXED ? 1 : 0) + ((o.flags & EQD_FLAG_FUSE) ? 1 : 0);
    const size_t per_col = (size_t)gc.colstride * (8 + (size_t)nvec * (prec == EQD_PREC_MIXED ? 4 : 8)) +
                           (size_t)16 * gc.nf + 1024;
    size_t budget = o.hbm_budget_bytes;
    if (budget == 0) {
        size_t fr = 0, tot = 0;
        CUDA_OR_RETURN(cudaMemGetInfo(&fr, &tot));
        const size_t keep = (size_t)2 << 30;
        budget = fr > keep ? fr - keep : fr / 2;
    }
    long long cap = (long long)(budget / per_col);
    if (cap < 1) return fail(EQD_ERR_OOM, "HBM budget too small for one column");
    const long long want =
        o.chunk > 0 ? o.chunk : ((G->chunk_tuned > 0 && prec == EQD_PREC_MIXED) ? G->chunk_tuned : cap);
    chunk = (int)std::min<long long>(want, ncols);
    if ((long long)chunk > cap) chunk = (int)cap;
    return EQD_OK;
}

// Columns [c0, c0 + n) of the slot arrays, recorded on stream `s`: every
// pointer is offset to the span, so two spans are independent CG batches.
struct Span {
    int c0, n;
    cudaStream_t s;
    bool split;  // one of two halves whose kernels overlap
};

template <typename T>
struct IterPtrs {
    ColumnSet cs;
    ColState st;
    T *r, *p, *q;
    T *p2;  // fused direction update: the other direction buffer
    float *d;
    double *x64, *apply_part, *res_part, *rr_part;
};

template <typename T>
static IterPtrs<T> span_ptrs(eqd_grid *G, Workspace &W, const SolveParams &sp, const ColState &st0, const Span &sp_) {
    const GridConst &gc = G->gc;
    const long long c0 = sp_.c0;
    IterPtrs<T> P{};
    P.cs.ncols = sp_.n;
    P.cs.slip_node = W.slip_node.as<int>() + c0;
    P.cs.slip_comp = W.slip_comp.as<int>() + c0;
    P.cs.slip_dense = W.slip_dense.p ? W.slip_dense.as<double>() + c0 * 2 * gc.nf : nullptr;
    P.cs.status = W.status.as<int8_t>() + c0;
    P.st = ColState{st0.gamma + c0, st0.beta + c0, st0.rr_ref + c0, st0.tol + c0, st0.bnorm + c0,
                    st0.iters + c0, st0.status + c0, st0.flag + c0};
    P.r = W.v0.as<T>() + c0 * gc.colstride;
    P.p = W.v1.as<T>() + c0 * gc.colstride;
    P.q = W.v2.as<T>() + c0 * gc.colstride;
    P.p2 = W.v4.p ? W.v4.as<T>() + c0 * gc.colstride : nullptr;
    P.d = W.v3.p ? W.v3.as<float>() + c0 * gc.colstride : nullptr;
    P.x64 = W.x64.as<double>() + c0 * gc.colstride;
    P.apply_part = W.apply_part.as<double>() + c0 * sp.ntiles * 2;
    P.res_part = W.res_part.as<double>() + c0 * nparts(G->m64) * 2;
    P.rr_part = W.rr_part.as<double>() + c0 * G->nchunks * 2;
    return P;
}

// The direction of iteration k when the direction update is fused into the
// apply: iteration k reads the previous direction from one buffer and writes
// the new one to the other (v1 at even k, v4 at odd k; kIter is even, so a
// graph launch always starts with the current direction in v1).
template <typename T>
static T *dir_in(const IterPtrs<T> &P, int k) { return (k & 1) ? P.p2 : P.p; }
template <typename T>
static T *dir_out(const IterPtrs<T> &P, int k) { return (k & 1) ? P.p : P.p2; }

// The stencil apply of CG iteration k (q = A p, partial p.q); fused: with
// p = r + beta p formed on the way in.
template <typename T>
static void record_apply(eqd_grid *G, Workspace &W, int generic, int fused, int k, const SolveParams &sp,
                         const ColState &st0, const Span &sn) {
    IterPtrs<T> P = span_ptrs<T>(G, W, sp, st0, sn);
    if (generic) {
        launch_march<T, T, MODE_AP>(G, P.p, P.q, P.cs, P.apply_part, sn.n, -1, sn.s);
    } else if (fused) {
        ColumnSet cs = P.cs;
        cs.pold = dir_in(P, k);
        cs.pnew = dir_out(P, k);
        cs.beta = P.st.beta;
        launch_march<T, T, MODE_AF>(G, P.r, P.q, cs, P.apply_part, sn.n, -1, sn.s);
    } else {
        launch_march<T, T, MODE_A>(G, P.p, P.q, P.cs, P.apply_part, sn.n, -1, sn.s);
    }
}

// CTA size of the vector kernels inside the iterations: small enough to fit
// beside resident stencil CTAs on an SM (the update kernel's 128 threads x
// 62-70 registers take the 8 K registers that two 224-thread, 128-register
// stencil CTAs leave free), so the other half's updates can run while an
// apply is in flight.
static constexpr int kVecThreads = 128;
// With a split batch the vector kernels run on 4 CTAs per SM (grid-stride):
// they fit beside the other half's stencil CTAs and still stream at close to
// HBM speed (measured at h = 50 m: 1, 2, 4, 8 CTAs per SM and one CTA per item
// gave 6.0, 6.6, 6.5, 6.3 k columns/s; one chain with one CTA per item 6.2 k).
static constexpr int kVecCtasPerSm = 4;

// The rest of iteration k: x, r updates; scalars; reliable update (mixed);
// the next direction (unless the next apply forms it).
template <typename T>
static void record_rest(eqd_grid *G, Workspace &W, int mixed, int fused, int k, const SolveParams &sp,
                        const ColState &st0, const Span &sn) {
    IterPtrs<T> P = span_ptrs<T>(G, W, sp, st0, sn);
    const T *pk = fused ? dir_out(P, k) : P.p;  // this iteration's direction
    const int nch = G->nchunks;
    const double *dinv64 = sp.precond ? G->dinv64.as<double>() : nullptr;
    const float *dinv32 = sp.precond ? G->dinv32.as<float>() : nullptr;
    // Split: a few CTAs per SM (grid-stride over the items) so they fit
    // beside the other half's stencil CTAs; one chain: one CTA per item.
    const long long items = (long long)sn.n * nch;
    const unsigned nb = (unsigned)(sn.split ? std::min<long long>(items, (long long)G->num_sms * kVecCtasPerSm) : items);
    // Mixed precision: the bulk-staged vector kernels (measured at h = 50 m,
    // 2,178 columns: 7,213 vs 6,771 columns/s with the register versions).
    // FP64: the register versions (the bulk-staged ones measured 17 % slower
    // beside the FP64 stencil).
    unsigned *err = G->err.as<unsigned>();
    if (mixed) {
        cg_update_bulk_kernel<float, float><<<nb, kVecThreads, kUpdateBulkSmem, sn.s>>>(
            P.d, (float *)P.r, (const float *)pk, (const float *)P.q, P.apply_part, P.st, sp, P.rr_part, dinv32, sn.n,
            err);
    } else {
        cg_update_kernel<double, double><<<nb, kVecThreads, 0, sn.s>>>(P.x64, (double *)P.r, (const double *)pk,
                                                              (const double *)P.q, P.apply_part, P.st, sp,
                                                              P.rr_part, dinv64, sn.n);
    }
    const unsigned sb = (unsigned)((sn.n + 127) / 128);
    cg_scalar_kernel<<<sb, 128, 0, sn.s>>>(P.st, sp, P.apply_part, P.rr_part, sn.n, mixed);
    if (mixed) {
        // One CTA per item: in most iterations no column is flagged and every
        // CTA returns at once.
        fold_correction_kernel<<<(unsigned)items, kVecThreads, 0, sn.s>>>(P.x64, P.d, P.st, sp, sn.n);
        ColumnSet cf = P.cs;
        cf.flag = P.st.flag;
        cf.dinv = dinv64;
        launch_march<double, float, MODE_RHS>(G, P.x64, (float *)P.r, cf, P.res_part, sn.n, -1, sn.s);
        SolveParams sp2 = sp;
        sp2.ntiles = nparts(G->m64);
        cg_true_residual_kernel<<<sb, 128, 0, sn.s>>>(P.st, sp2, P.res_part, sn.n, 1);
    }
    if (!fused) {
        const T *dinvT = (const T *)(sizeof(T) == 4 ? (const void *)dinv32 : (const void *)dinv64);
        if (mixed)
            cg_pupdate_bulk_kernel<T><<<nb, kVecThreads, kDirBulkSmem, sn.s>>>(P.p, P.r, P.st, sp, dinvT, sn.n, err);
        else
            cg_pupdate_kernel<T><<<nb, kVecThreads, 0, sn.s>>>(P.p, P.r, P.st, sp, nullptr, dinvT, sn.n);
    }
}

// Capture kIter CG iterations over `cap` slots. Large batches are split in
// two halves on two streams whose stencil applies alternate: the
// arithmetic-bound apply of one half runs while the memory-bound vector
// updates of the other half stream through HBM.
template <typename T>
static void record_iterations(eqd_grid *G, Workspace &W, int cap, int mixed, int generic, int fused,
                              const SolveParams &sp, const ColState &st, int kIter, bool split) {
    if (!split) {
        const Span all{0, cap, G->stream, false};
        for (int k = 0; k < kIter; ++k) {
            record_apply<T>(G, W, generic, fused, k, sp, st, all);
            record_rest<T>(G, W, mixed, fused, k, sp, st, all);
        }
        return;
    }
    // Applies on normal-priority streams, the rest of each iteration on
    // high-priority streams (node priorities are kept at instantiation), so
    // that freed SM slots go to the short memory-bound kernels first.
    const int h0 = cap / 2;
    const Span A{0, h0, G->stream, true}, B{h0, cap - h0, G->stream2, true};
    const Span Ah{0, h0, G->stream_hi, true}, Bh{h0, cap - h0, G->stream2_hi, true};
    cudaEventRecord(G->evFork, A.s);
    for (cudaStream_t t : {B.s, Ah.s, Bh.s}) cudaStreamWaitEvent(t, G->evFork, 0);
    for (int k = 0; k < kIter; ++k) {
        if (k > 0) {
            cudaStreamWaitEvent(A.s, G->evB, 0);      // B's previous apply is done
            cudaStreamWaitEvent(A.s, G->evArest, 0);  // A's previous direction is ready
        }
        record_apply<T>(G, W, generic, fused, k, sp, st, A);
        cudaEventRecord(G->evA, A.s);
        cudaStreamWaitEvent(B.s, G->evA, 0);          // B's apply follows A's
        if (k > 0) cudaStreamWaitEvent(B.s, G->evBrest, 0);
        record_apply<T>(G, W, generic, fused, k, sp, st, B);
        cudaEventRecord(G->evB, B.s);
        cudaStreamWaitEvent(Ah.s, G->evA, 0);
        record_rest<T>(G, W, mixed, fused, k, sp, st, Ah);
        cudaEventRecord(G->evArest, Ah.s);
        cudaStreamWaitEvent(Bh.s, G->evB, 0);
        record_rest<T>(G, W, mixed, fused, k, sp, st, Bh);
        cudaEventRecord(G->evBrest, Bh.s);
    }
    cudaEventRecord(G->evJoin, B.s);
    cudaStreamWaitEvent(A.s, G->evJoin, 0);
    cudaStreamWaitEvent(A.s, G->evArest, 0);
    cudaStreamWaitEvent(A.s, G->evBrest, 0);
}

// Jacobi weights dinv = 1 / diag(A) (zeros floored to 1), computed once per
// grid; a negative diagonal entry is an error, as in the reference.
static int ensure_jacobi(eqd_grid *G) {
    if (G->jacobi_ready) return EQD_OK;
    const GridConst &gc = G->gc;
    CUDA_OR_RETURN(G->dinv64.ensure(sizeof(double) * gc.colstride));
    CUDA_OR_RETURN(G->dinv32.ensure(sizeof(float) * gc.colstride));
    CUDA_OR_RETURN(cudaMemsetAsync(G->dinv64.p, 0, sizeof(double) * gc.colstride, G->stream));
    CUDA_OR_RETURN(cudaMemsetAsync(G->dinv32.p, 0, sizeof(float) * gc.colstride, G->stream));
    DevBuf neg;
    CUDA_OR_RETURN(neg.ensure(sizeof(unsigned)));
    CUDA_OR_RETURN(cudaMemsetAsync(neg.p, 0, sizeof(unsigned), G->stream));
    const long long n = 6LL * gc.n1 * gc.n2 * gc.n3;
    jacobi_diag_kernel<<<(unsigned)((n + 255) / 256), 256, 0, G->stream>>>(
        G->c64, gc.n1, gc.n2, gc.n3, gc.PS, nullptr, G->dinv64.as<double>(), G->dinv32.as<float>(), neg.as<unsigned>());
    CUDA_OR_RETURN(cudaGetLastError());
    unsigned h = 0;
    CUDA_OR_RETURN(cudaMemcpyAsync(&h, neg.p, sizeof(unsigned), cudaMemcpyDeviceToHost, G->stream));
    CUDA_OR_RETURN(cudaStreamSynchronize(G->stream));
    if (h) return fail(EQD_ERR_ARG, "diag(A) has negative entries; A is not PSD and a Jacobi preconditioner "
                                    "would not be SPD");
    G->jacobi_ready = true;
    return EQD_OK;
}

// ---------------------------------------------------------------------------
// Slot engine: a fixed set of column slots, each holding one right-hand side's
// CG state. A column enters a free slot (its vectors are zeroed and r0 = b is
// evaluated for it alone), runs with every other occupied slot in the
// graph-captured iterations, and leaves when its status is final; its slot is
// then free for the next column. A column's arithmetic does not depend on the
// other slots (every reduction is per column, in a fixed order), so a column
// gives the same bits whenever and beside whatever it runs.
// ---------------------------------------------------------------------------
struct ColWork {
    int slip_node = -1;                  // unit slip at this Omega_f node (-1: none)
    int slip_comp = 0;                   // 0 -> s2, 1 -> s3
    const double *slip_dense = nullptr;  // host [2][nf] slip field, or null
    const double *rhs = nullptr;         // host reference-layout right-hand side (explicit-RHS solve), or null
    long long tag = 0;                   // the caller's id for the column
};

struct ColDone {
    long long tag;
    int slot;
    int iters;
    int8_t status;
};

static int tune_by_iterations(eqd_grid *G, const eqd_solve_opts &o, int ncols);

template <typename T>
struct SlotRun {
    eqd_grid *G = nullptr;
    Workspace *W = nullptr;
    int cap = 0, mixed = 0, generic = 0, dense = 0;
    int fused = 0;  // the direction update runs inside the stencil apply (MODE_AF)
    long long itmax = 0;
    SolveParams sp{};
    ColState st{};
    std::vector<int> hn, hc, hslot, hdst;
    std::vector<int8_t> hnew;
    PinnedArr<int> hit;     // per-slot iteration counts (read back every graph launch)
    PinnedArr<int8_t> hst;  // per-slot status
    std::vector<long long> tag;  // -1: free slot
    int held = 0;                // occupied slots (running or finished, not yet released)
    int64_t launches = 0;
    static constexpr int kIter = 10;

    int setup(eqd_grid *g, const eqd_solve_opts &o, int capacity, bool gen, bool dns) {
        G = g;
        W = &G->ws;
        cap = capacity;
        mixed = o.precision == EQD_PREC_MIXED;
        generic = gen;
        dense = dns;
        const GridConst &gc = G->gc;
        const long long ntot = 6LL * gc.n1 * gc.n2 * gc.n3;
        const size_t vec = (size_t)gc.colstride * cap;
        if (mixed && !G->tuned) {
            int rc = tune_by_iterations(G, o, std::min(cap, 1024));
            if (rc) return rc;
        }
        const int nt32 = nparts(G->v32[G->sel32]), nt64 = nparts(G->m64);
        Workspace &w = *W;
        CUDA_OR_RETURN(w.x64.ensure(sizeof(double) * vec));
        CUDA_OR_RETURN(w.v0.ensure(sizeof(T) * vec));
        CUDA_OR_RETURN(w.v1.ensure(sizeof(T) * vec));
        CUDA_OR_RETURN(w.v2.ensure(sizeof(T) * vec));
        if (mixed) CUDA_OR_RETURN(w.v3.ensure(sizeof(float) * vec));
        {
            const MarchCfg &mc = sizeof(T) == 4 ? G->v32[G->sel32] : G->m64;
            fused = !generic && o.precond != EQD_PRECOND_JACOBI && (o.flags & EQD_FLAG_FUSE) && mc.smem_af > 0;
        }
        if (fused) CUDA_OR_RETURN(w.v4.ensure(sizeof(T) * vec));
        else w.v4.release();
        int ntmax = std::max(nt64, nparts(G->m32));
        for (int v = 0; v < kNumVariants; ++v) ntmax = std::max(ntmax, nparts(G->v32[v]));
        CUDA_OR_RETURN(w.apply_part.ensure(sizeof(double) * 2 * cap * ntmax));
        CUDA_OR_RETURN(w.res_part.ensure(sizeof(double) * 2 * cap * std::max(nt64, G->nchunks)));
        CUDA_OR_RETURN(w.rr_part.ensure(sizeof(double) * 2 * cap * G->nchunks));
        for (DevBuf *b : {&w.gamma, &w.beta, &w.rr_ref, &w.tol, &w.bnorm}) CUDA_OR_RETURN(b->ensure(sizeof(double) * cap));
        CUDA_OR_RETURN(w.iters.ensure(sizeof(int) * cap));
        CUDA_OR_RETURN(w.status.ensure(cap));
        CUDA_OR_RETURN(w.flag.ensure(cap));
        CUDA_OR_RETURN(w.newmask.ensure(cap));
        CUDA_OR_RETURN(w.slot_list.ensure(sizeof(int) * cap));
        CUDA_OR_RETURN(w.dst_list.ensure(sizeof(int) * cap));
        CUDA_OR_RETURN(w.slip_node.ensure(sizeof(int) * cap));
        CUDA_OR_RETURN(w.slip_comp.ensure(sizeof(int) * cap));
        if (dense) CUDA_OR_RETURN(w.slip_dense.ensure(sizeof(double) * 2 * gc.nf * cap));
        else w.slip_dense.release();
        CUDA_OR_RETURN(w.kout.ensure(sizeof(double) * 2 * gc.nf * cap));
        if (generic) CUDA_OR_RETURN(w.hbuf.ensure(sizeof(double) * ntot * cap));

        st = ColState{w.gamma.as<double>(), w.beta.as<double>(), w.rr_ref.as<double>(), w.tol.as<double>(),
                      w.bnorm.as<double>(), w.iters.as<int>(), w.status.as<int8_t>(), w.flag.as<int8_t>()};
        sp = SolveParams{};
        sp.rtol = o.rtol;
        sp.atol = o.atol;
        sp.itmax = o.itmax;
        sp.delta = o.reliable_delta > 0 ? o.reliable_delta : 0.01;
        sp.ntiles = sizeof(T) == 4 ? nt32 : nt64;
        sp.nchunks = G->nchunks;
        sp.colstride = gc.colstride;
        sp.ntot = ntot;
        sp.precond = o.precond == EQD_PRECOND_JACOBI;
        if (sp.precond) {
            int rc = ensure_jacobi(G);
            if (rc) return rc;
        }
        itmax = o.itmax > 0 ? o.itmax : 2 * ntot;

        // Every slot starts free: status IDLE everywhere, vectors zeroed as
        // columns enter.
        hn.assign(cap, -1);
        hc.assign(cap, 0);
        CUDA_OR_RETURN(hit.assign(cap, 0));
        CUDA_OR_RETURN(hst.assign(cap, (int8_t)COL_IDLE));
        hnew.assign(cap, 0);
        tag.assign(cap, -1);
        hslot.resize(cap);
        hdst.resize(cap);
        held = 0;
        CUDA_OR_RETURN(cudaMemcpyAsync(w.status.p, hst.data(), cap, cudaMemcpyHostToDevice, G->stream));
        CUDA_OR_RETURN(cudaMemsetAsync(w.flag.p, 0, cap, G->stream));

        // Graph of kIter iterations over all slots, captured once per
        // (capacity, precision, mode, launch variant, preconditioner, split).
        const bool split = cap >= 64 && !(o.flags & EQD_FLAG_NO_SPLIT);
        // Everything the captured kernels bake in: sizes, options and every
        // workspace pointer (a buffer that grew or was released since the
        // capture must not be reached through the old graph).
        std::vector<uint64_t> kv = {(uint64_t)cap, (uint64_t)o.precision, (uint64_t)generic, (uint64_t)G->sel32,
                                    (uint64_t)o.precond, (uint64_t)split, (uint64_t)sp.itmax, (uint64_t)fused};
        for (double d : {sp.rtol, sp.atol, sp.delta}) {
            uint64_t b;
            std::memcpy(&b, &d, sizeof(b));
            kv.push_back(b);
        }
        for (const void *q : {w.x64.p, w.v0.p, w.v1.p, w.v2.p, w.v3.p, w.v4.p, w.apply_part.p, w.res_part.p, w.rr_part.p,
                              w.gamma.p, w.beta.p, w.rr_ref.p, w.tol.p, w.bnorm.p, w.iters.p, w.status.p, w.flag.p,
                              w.slip_node.p, w.slip_comp.p, w.slip_dense.p, G->dinv64.p, G->dinv32.p})
            kv.push_back((uint64_t)(uintptr_t)q);
        if (!w.graph || w.graph_key != kv) {
            if (w.graph) cudaGraphExecDestroy(w.graph);
            w.graph = nullptr;
            cudaGraph_t g;
            CUDA_OR_RETURN(cudaStreamBeginCapture(G->stream, cudaStreamCaptureModeThreadLocal));
            record_iterations<T>(G, w, cap, mixed, generic, fused, sp, st, kIter, split);
            cudaError_t ce = cudaStreamEndCapture(G->stream, &g);
            if (ce != cudaSuccess) return fail(EQD_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
            ce = cudaGraphInstantiate(&w.graph, g, cudaGraphInstantiateFlagUseNodePriority);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess) return fail(EQD_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce));
            w.graph_key = kv;
            w.graph_iters = kIter;
            w.graph_split = split;
        }
        return EQD_OK;
    }

    int free_slots() const { return cap - held; }

    ColumnSet colset() const {
        ColumnSet cs{};
        cs.ncols = cap;
        cs.slip_node = W->slip_node.as<int>();
        cs.slip_comp = W->slip_comp.as<int>();
        cs.slip_dense = dense ? W->slip_dense.as<double>() : nullptr;
        cs.status = W->status.as<int8_t>();
        return cs;
    }

    // Put up to n columns into free slots and evaluate their r0 = b; `taken`
    // is how many entered.
    int admit(const ColWork *work, int n, int &taken) {
        taken = 0;
        const GridConst &gc = G->gc;
        const long long ntot = 6LL * gc.n1 * gc.n2 * gc.n3;
        Workspace &w = *W;
        std::fill(hnew.begin(), hnew.end(), (int8_t)0);
        for (int s = 0; s < cap && taken < n; ++s) {
            if (tag[s] >= 0) continue;
            const ColWork &c = work[taken++];
            tag[s] = c.tag;
            hn[s] = c.slip_node;
            hc[s] = c.slip_comp;
            hst[s] = COL_ACTIVE;
            hit[s] = 0;
            hnew[s] = 1;
            ++held;
            if (dense) {
                if (c.slip_dense)
                    CUDA_OR_RETURN(cudaMemcpyAsync(w.slip_dense.as<double>() + (size_t)s * 2 * gc.nf, c.slip_dense,
                                                   sizeof(double) * 2 * gc.nf, cudaMemcpyHostToDevice, G->stream));
                else
                    CUDA_OR_RETURN(cudaMemsetAsync(w.slip_dense.as<double>() + (size_t)s * 2 * gc.nf, 0,
                                                   sizeof(double) * 2 * gc.nf, G->stream));
            }
        }
        if (taken == 0) return EQD_OK;
        CUDA_OR_RETURN(cudaMemcpyAsync(w.slip_node.p, hn.data(), sizeof(int) * cap, cudaMemcpyHostToDevice, G->stream));
        CUDA_OR_RETURN(cudaMemcpyAsync(w.slip_comp.p, hc.data(), sizeof(int) * cap, cudaMemcpyHostToDevice, G->stream));
        CUDA_OR_RETURN(cudaMemcpyAsync(w.status.p, hst.data(), cap, cudaMemcpyHostToDevice, G->stream));
        CUDA_OR_RETURN(cudaMemcpyAsync(w.iters.p, hit.data(), sizeof(int) * cap, cudaMemcpyHostToDevice, G->stream));
        CUDA_OR_RETURN(cudaMemcpyAsync(w.newmask.p, hnew.data(), cap, cudaMemcpyHostToDevice, G->stream));
        const int8_t *mask = w.newmask.as<int8_t>();
        const unsigned nb = (unsigned)(cap * G->nchunks);
        const long long cst = gc.colstride;
        zero_columns_kernel<double><<<nb, 256, 0, G->stream>>>(w.x64.as<double>(), cst, G->nchunks, mask);
        zero_columns_kernel<T><<<nb, 256, 0, G->stream>>>(w.v0.as<T>(), cst, G->nchunks, mask);
        zero_columns_kernel<T><<<nb, 256, 0, G->stream>>>(w.v1.as<T>(), cst, G->nchunks, mask);
        zero_columns_kernel<T><<<nb, 256, 0, G->stream>>>(w.v2.as<T>(), cst, G->nchunks, mask);
        if (mixed) zero_columns_kernel<float><<<nb, 256, 0, G->stream>>>(w.v3.as<float>(), cst, G->nchunks, mask);
        // Fused: the second direction buffer's plane padding must read as zero.
        if (fused) zero_columns_kernel<T><<<nb, 256, 0, G->stream>>>(w.v4.as<T>(), cst, G->nchunks, mask);
        launches += (mixed ? 5 : 4) + (fused ? 1 : 0);
        const unsigned sb = (unsigned)((cap + 127) / 128);
        if (!generic) {
            // r0 = b = H P (D+SAT) chi  (x = 0), in the working precision.
            ColumnSet cs = colset();
            cs.flag = mask;
            cs.dinv = sp.precond ? G->dinv64.as<double>() : nullptr;
            CUDA_OR_RETURN((launch_march<double, T, MODE_RHS>(G, w.x64.as<double>(), w.v0.as<T>(), cs,
                                                               w.res_part.as<double>(), cap)));
            SolveParams sp2 = sp;
            sp2.ntiles = nparts(G->m64);
            cg_true_residual_kernel<<<sb, 128, 0, G->stream>>>(st, sp2, w.res_part.as<double>(), cap, mixed, mask);
            launches += 2;
        } else {
            // r0 = b given explicitly (reference layout, FP64).
            int j = 0;
            for (int s = 0; s < cap && j < taken; ++s) {
                if (!hnew[s]) continue;
                const ColWork &c = work[j++];
                double *hb = w.hbuf.as<double>() + (size_t)s * ntot;
                CUDA_OR_RETURN(cudaMemcpyAsync(hb, c.rhs, sizeof(double) * ntot, cudaMemcpyHostToDevice, G->stream));
                const int tb = 256;
                ref_to_dev_kernel<double, T><<<(unsigned)((ntot + tb - 1) / tb), tb, 0, G->stream>>>(
                    hb, w.v0.as<T>() + (size_t)s * gc.colstride, gc.n1, gc.n2, gc.n3, gc.PS, gc.colstride, 1);
                ++launches;
            }
            column_sumsq_kernel<T><<<nb, 256, 0, G->stream>>>(w.v0.as<T>(), cst, G->nchunks, mask,
                                                               w.res_part.as<double>(),
                                                               sp.precond ? G->dinv64.as<double>() : nullptr);
            SolveParams sp2 = sp;
            sp2.ntiles = G->nchunks;
            cg_true_residual_kernel<<<sb, 128, 0, G->stream>>>(st, sp2, w.res_part.as<double>(), cap, 0, mask);
            launches += 2;
        }
        const T *dinvT = !sp.precond ? nullptr
                                     : (const T *)(sizeof(T) == 4 ? (const void *)G->dinv32.p : (const void *)G->dinv64.p);
        cg_pupdate_kernel<T><<<nb, 256, 0, G->stream>>>(w.v1.as<T>(), w.v0.as<T>(), st, sp, mask, dinvT, cap);
        ++launches;
        CUDA_OR_RETURN(cudaGetLastError());
        return EQD_OK;
    }

    // Run kIter iterations (when a column is running) and queue the status
    // read-back; collect() then lists the finished slots. Split in two so that
    // a caller driving several grids can have all of them running at once.
    int launch() {
        Workspace &w = *W;
        int running = 0;
        for (int s = 0; s < cap; ++s) running += tag[s] >= 0 && hst[s] == COL_ACTIVE;
        if (running > 0) {
            CUDA_OR_RETURN(cudaGraphLaunch(w.graph, G->stream));
            launches += (int64_t)kIter * ((mixed ? 7 : 4) - (fused ? 1 : 0)) * (w.graph_split ? 2 : 1);
        }
        CUDA_OR_RETURN(cudaMemcpyAsync(hst.data(), w.status.p, cap, cudaMemcpyDeviceToHost, G->stream));
        CUDA_OR_RETURN(cudaMemcpyAsync(hit.data(), w.iters.p, sizeof(int) * cap, cudaMemcpyDeviceToHost, G->stream));
        return EQD_OK;
    }

    int advance(std::vector<ColDone> &done) {
        int rc = launch();
        return rc ? rc : collect(done);
    }

    // Wait for the queued iterations; list the occupied slots whose status is
    // final.
    int collect(std::vector<ColDone> &done) {
        done.clear();
        Workspace &w = *W;
        CUDA_OR_RETURN(cudaStreamSynchronize(G->stream));
        int rc = check_device_error(G);
        if (rc) return rc;
        bool forced = false;
        for (int s = 0; s < cap; ++s) {
            if (tag[s] < 0) continue;
            if (hst[s] == COL_ACTIVE && hit[s] > itmax + 2 * kIter) {  // defensive: the kernels stop at itmax
                hst[s] = COL_MAXITER;
                forced = true;
            }
            if (hst[s] != COL_ACTIVE) done.push_back(ColDone{tag[s], s, hit[s], hst[s]});
        }
        if (forced)
            CUDA_OR_RETURN(cudaMemcpyAsync(w.status.p, hst.data(), cap, cudaMemcpyHostToDevice, G->stream));
        return EQD_OK;
    }

    // K columns of finished slots: into K (device) at column dst (the tag when
    // `to_tag`, else the position in `done`), leading dimension kld.
    int extract(const std::vector<ColDone> &done, double *K, long long kld, bool to_tag) {
        if (done.empty()) return EQD_OK;
        const GridConst &gc = G->gc;
        Workspace &w = *W;
        const int n = (int)done.size();
        for (int j = 0; j < n; ++j) {
            hslot[j] = done[j].slot;
            hdst[j] = to_tag ? (int)done[j].tag : j;
        }
        CUDA_OR_RETURN(cudaMemcpyAsync(w.slot_list.p, hslot.data(), sizeof(int) * n, cudaMemcpyHostToDevice, G->stream));
        CUDA_OR_RETURN(cudaMemcpyAsync(w.dst_list.p, hdst.data(), sizeof(int) * n, cudaMemcpyHostToDevice, G->stream));
        ExtractGeom eg{gc.n1, gc.n2, gc.n3, gc.PS, gc.nf, gc.i2f0, gc.n2f, gc.i3f0, gc.n3f, gc.colstride, gc.mu};
        const long long nthr = (long long)n * gc.nf;
        extract_traction_kernel<<<(unsigned)((nthr + 127) / 128), 128, 0, G->stream>>>(
            G->c64, eg, w.x64.as<double>(), colset(), K, kld, n, w.slot_list.as<int>(), w.dst_list.as<int>());
        ++launches;
        CUDA_OR_RETURN(cudaGetLastError());
        return EQD_OK;
    }

    // Explicit-RHS solve: the solution of a finished slot in reference layout.
    int solution(int slot, double *host_u) {
        const GridConst &gc = G->gc;
        const long long ntot = 6LL * gc.n1 * gc.n2 * gc.n3;
        Workspace &w = *W;
        double *hb = w.hbuf.as<double>() + (size_t)slot * ntot;
        const int tb = 256;
        dev_to_ref_kernel<double, double><<<(unsigned)((ntot + tb - 1) / tb), tb, 0, G->stream>>>(
            w.x64.as<double>() + (size_t)slot * gc.colstride, hb, gc.n1, gc.n2, gc.n3, gc.PS, gc.colstride, 1);
        ++launches;
        CUDA_OR_RETURN(cudaMemcpyAsync(host_u, hb, sizeof(double) * ntot, cudaMemcpyDeviceToHost, G->stream));
        return EQD_OK;
    }

    // Free the slots of finished columns.
    int release(const std::vector<ColDone> &done) {
        if (done.empty()) return EQD_OK;
        for (const ColDone &d : done) {
            tag[d.slot] = -1;
            hn[d.slot] = -1;
            hst[d.slot] = COL_IDLE;
            --held;
        }
        CUDA_OR_RETURN(cudaMemcpyAsync(W->status.p, hst.data(), cap, cudaMemcpyHostToDevice, G->stream));
        return EQD_OK;
    }
};

// Launch-variant tuner: time 20 CG iterations (two graph launches) of a
// batch of `ncols` unit-slip columns with each FP32 stencil variant and keep
// the fastest. The whole iteration is timed, not the stencil alone: a variant
// that packs more stencil CTAs per SM can leave less room for the other
// half's vector kernels (measured at h = 50 m: the fastest stencil alone was
// not the fastest iteration).
static int tune_by_iterations(eqd_grid *G, const eqd_solve_opts &o, int ncols) {
    const GridConst &gc = G->gc;
    ncols = std::max(1, std::min(ncols, 2 * gc.nf));
    std::vector<ColWork> work(ncols);
    for (int i = 0; i < ncols; ++i) {
        work[i].slip_node = (int)(((long long)i * 7919 + gc.nf / 2) % gc.nf);
        work[i].slip_comp = i & 1;
        work[i].tag = i;
    }
    eqd_solve_opts ot = o;
    ot.precision = EQD_PREC_MIXED;
    G->tuned = true;  // the slot engines below must not tune again
    double best = 1e30;
    int bestv = G->sel32;
    for (int v = 0; v < kNumVariants; ++v) {
        G->sel32 = v;
        SlotRun<float> R;
        int rc = R.setup(G, ot, ncols, false, false);
        if (rc) return rc;
        int taken = 0;
        rc = R.admit(work.data(), ncols, taken);
        if (!rc) rc = R.launch();  // first launch: warm-up
        if (rc) return rc;
        CUDA_OR_RETURN(cudaEventRecord(G->ev0, G->stream));
        rc = R.launch();
        if (!rc) rc = R.launch();
        if (rc) return rc;
        CUDA_OR_RETURN(cudaEventRecord(G->ev1, G->stream));
        CUDA_OR_RETURN(cudaEventSynchronize(G->ev1));
        float ms = 0.f;
        CUDA_OR_RETURN(cudaEventElapsedTime(&ms, G->ev0, G->ev1));
        G->tune_ms[v] = ms / (2.0 * SlotRun<float>::kIter);
        if (G->tune_ms[v] < best) {
            best = G->tune_ms[v];
            bestv = v;
        }
    }
    G->sel32 = bestv;
    return check_device_error(G);
}

// Batched solve through the slot engine: columns enter as slots free up; K
// columns go to the caller's device or host buffer as each column finishes.
template <typename T>
static int run_batch(eqd_grid *G, const eqd_solve_opts &o, const BatchSpec &B, eqd_stats *stats) {
    const GridConst &gc = G->gc;
    const int generic = B.rhs != nullptr;
    const long long ntot = 6LL * gc.n1 * gc.n2 * gc.n3;
    int chunk = 0;
    int rc = resolve_chunk(G, o, B.ncols, o.precision, chunk);
    if (rc) return rc;
    SlotRun<T> R;
    rc = R.setup(G, o, chunk, generic, B.slip_dense != nullptr);
    if (rc) return rc;

    std::vector<ColWork> work(B.ncols);
    for (int i = 0; i < B.ncols; ++i) {
        ColWork &c = work[i];
        c.tag = i;
        c.slip_node = B.slip_node ? B.slip_node[i] : -1;
        c.slip_comp = B.slip_comp ? B.slip_comp[i] : 0;
        c.slip_dense = B.slip_dense ? B.slip_dense + (size_t)i * 2 * gc.nf : nullptr;
        c.rhs = B.rhs ? B.rhs + (size_t)i * ntot : nullptr;
    }
    int64_t tot_it = 0, max_it = 0, unconv = 0;
    PinnedArr<double> &kstage = R.W->kstage;
    if (!generic && B.kcols && !B.kdev && kstage.n < 2 * gc.nf * chunk)
        CUDA_OR_RETURN(kstage.assign(2 * gc.nf * chunk, 0.0));
    // Host K output: finished columns are staged in pinned memory, and the
    // host copies them to the caller's K after the next graph launch, while
    // the GPU runs those iterations.
    const bool host_k = !generic && B.kcols && !B.kdev;
    cudaEvent_t kready = nullptr;  // the staged columns have landed
    if (host_k) CUDA_OR_RETURN(cudaEventCreateWithFlags(&kready, cudaEventDisableTiming));
    struct EventGuard {
        cudaEvent_t e;
        ~EventGuard() {
            if (e) cudaEventDestroy(e);
        }
    } kready_guard{kready};
    std::vector<ColDone> staged;
    auto copy_staged = [&]() -> int {
        if (staged.empty()) return EQD_OK;
        CUDA_OR_RETURN(cudaEventSynchronize(kready));
        for (size_t j = 0; j < staged.size(); ++j)
            std::memcpy(B.kcols + (size_t)staged[j].tag * 2 * gc.nf, kstage.data() + j * 2 * gc.nf,
                        sizeof(double) * 2 * gc.nf);
        staged.clear();
        return EQD_OK;
    };
    CUDA_OR_RETURN(cudaEventRecord(G->ev0, G->stream));
    int next = 0, finished = 0;
    std::vector<ColDone> done;
    while (finished < B.ncols) {
        // Explicit-RHS solves refill only an empty engine (their staging
        // buffer holds one wave of right-hand sides).
        if (next < B.ncols && R.free_slots() > 0 && (!generic || R.held == 0)) {
            int taken = 0;
            rc = R.admit(work.data() + next, B.ncols - next, taken);
            if (rc) return rc;
            next += taken;
        }
        rc = R.launch();
        if (!rc) rc = copy_staged();
        if (!rc) rc = R.collect(done);
        if (rc) return rc;
        if (done.empty()) continue;
        if (!generic) {
            if (B.kdev) {
                rc = R.extract(done, B.kdev, 2LL * gc.nf, true);
            } else {
                rc = R.extract(done, R.W->kout.template as<double>(), 2LL * gc.nf, false);
                if (!rc && B.kcols) {
                    CUDA_OR_RETURN(cudaMemcpyAsync(kstage.data(), R.W->kout.p, sizeof(double) * 2 * gc.nf * done.size(),
                                                   cudaMemcpyDeviceToHost, G->stream));
                    CUDA_OR_RETURN(cudaEventRecord(kready, G->stream));
                    staged = done;
                }
            }
            if (rc) return rc;
        } else if (B.u_out) {
            for (const ColDone &d : done) {
                rc = R.solution(d.slot, B.u_out + (size_t)d.tag * ntot);
                if (rc) return rc;
            }
            CUDA_OR_RETURN(cudaStreamSynchronize(G->stream));
        }
        for (size_t j = 0; j < done.size(); ++j) {
            const ColDone &d = done[j];
            tot_it += d.iters;
            max_it = std::max<int64_t>(max_it, d.iters);
            if (d.status != COL_CONVERGED) ++unconv;
            if (B.iters) B.iters[d.tag] = d.iters;
            if (B.status) B.status[d.tag] = d.status;
        }
        finished += (int)done.size();
        rc = R.release(done);
        if (rc) return rc;
    }
    rc = copy_staged();
    if (rc) return rc;
    CUDA_OR_RETURN(cudaEventRecord(G->ev1, G->stream));
    CUDA_OR_RETURN(cudaEventSynchronize(G->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, G->ev0, G->ev1);
    if (stats) {
        stats->solves += B.ncols;
        stats->iterations += tot_it;
        stats->max_iterations = std::max<int64_t>(stats->max_iterations, max_it);
        stats->unconverged += unconv;
        stats->kernel_launches += R.launches;
        stats->device_seconds += ms * 1e-3;
        stats->precision = o.precision;
        stats->precond = o.precond;
    }
    if ((o.flags & EQD_FLAG_STRICT) && unconv > 0)
        return fail(EQD_ERR_NOT_CONVERGED, std::to_string(unconv) + " column(s) did not converge");
    return EQD_OK;
}

static int run_batch_any(eqd_grid *G, const eqd_solve_opts *opts, const BatchSpec &B, eqd_stats *stats) {
    eqd_solve_opts o;
    if (opts) o = *opts;
    else eqd_default_opts(&o);
    if (!(o.rtol >= 0) || !(o.atol >= 0)) return fail(EQD_ERR_ARG, "rtol/atol must be non-negative");
    if (o.precond != EQD_PRECOND_NONE && o.precond != EQD_PRECOND_JACOBI)
        return fail(EQD_ERR_ARG, "precond must be :none or :jacobi");
    if (o.precision != EQD_PREC_FP64 && o.precision != EQD_PREC_MIXED) return fail(EQD_ERR_ARG, "unknown precision");
    if (B.rhs && o.precision != EQD_PREC_FP64) return fail(EQD_ERR_UNSUPPORTED, "explicit-RHS solves run in FP64");
    if (o.variant < 0 || o.variant > kNumVariants)
        return fail(EQD_ERR_ARG, "variant must be 0 (the grid's) or 1.." + std::to_string(kNumVariants));
    const auto t0 = std::chrono::steady_clock::now();
    std::lock_guard<std::mutex> lk(G->mtx);
    if (G->served) return fail(EQD_ERR_ARG, "the grid is attached to a server");
    CUDA_OR_RETURN(cudaSetDevice(G->desc.device));
    // A per-call variant replaces the grid's selection for this call only.
    const int sel_before = G->sel32;
    const bool tuned_before = G->tuned;
    if (o.variant > 0) {
        G->sel32 = o.variant - 1;
        G->tuned = true;
    }
    int rc = o.precision == EQD_PREC_MIXED ? run_batch<float>(G, o, B, stats) : run_batch<double>(G, o, B, stats);
    if (o.variant > 0) {
        G->sel32 = sel_before;
        G->tuned = tuned_before;
    }
    if (stats)
        stats->seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

extern "C" int eqd_stiffness_columns(eqd_grid *G, const int32_t *cols, int32_t ncols, const eqd_solve_opts *opts,
                                     double *out, int32_t *iters, int8_t *status, eqd_stats *stats) {
    if (!G || (!cols && ncols > 0) || (!out && ncols > 0)) return fail(EQD_ERR_ARG, "null argument");
    if (ncols < 0) return fail(EQD_ERR_ARG, "ncols must be >= 0");
    if (ncols == 0) return EQD_OK;
    const int nf = G->gc.nf;
    std::vector<int> node(ncols), comp(ncols);
    for (int i = 0; i < ncols; ++i) {
        if (cols[i] < 0 || cols[i] >= 2 * nf) return fail(EQD_ERR_ARG, "column index out of range");
        node[i] = cols[i] < nf ? cols[i] : cols[i] - nf;
        comp[i] = cols[i] < nf ? 0 : 1;
    }
    BatchSpec B{};
    B.ncols = ncols;
    B.slip_node = node.data();
    B.slip_comp = comp.data();
    B.kcols = out;
    B.iters = iters;
    B.status = status;
    return run_batch_any(G, opts, B, stats);
}

extern "C" int eqd_stiffness_columns_device(eqd_grid *G, const int32_t *cols, int32_t ncols,
                                            const eqd_solve_opts *opts, double *out_device, int32_t *iters,
                                            int8_t *status, eqd_stats *stats) {
    if (!G || (!cols && ncols > 0) || (!out_device && ncols > 0)) return fail(EQD_ERR_ARG, "null argument");
    if (ncols < 0) return fail(EQD_ERR_ARG, "ncols must be >= 0");
    if (ncols == 0) return EQD_OK;
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, out_device) != cudaSuccess || pa.type != cudaMemoryTypeDevice ||
        pa.device != G->desc.device) {
        cudaGetLastError();
        return fail(EQD_ERR_ARG, "out_device is not device memory of the grid's device");
    }
    const int nf = G->gc.nf;
    std::vector<int> node(ncols), comp(ncols);
    for (int i = 0; i < ncols; ++i) {
        if (cols[i] < 0 || cols[i] >= 2 * nf) return fail(EQD_ERR_ARG, "column index out of range");
        node[i] = cols[i] < nf ? cols[i] : cols[i] - nf;
        comp[i] = cols[i] < nf ? 0 : 1;
    }
    BatchSpec B{};
    B.ncols = ncols;
    B.slip_node = node.data();
    B.slip_comp = comp.data();
    B.kdev = out_device;
    B.iters = iters;
    B.status = status;
    return run_batch_any(G, opts, B, stats);
}

extern "C" int eqd_stiffness_exact(eqd_grid *G, const eqd_solve_opts *opts, double *K, eqd_stats *stats) {
    if (!G || !K) return fail(EQD_ERR_ARG, "null argument");
    const int n = 2 * G->gc.nf;
    std::vector<int32_t> cols(n);
    for (int i = 0; i < n; ++i) cols[i] = i;
    return eqd_stiffness_columns(G, cols.data(), n, opts, K, nullptr, nullptr, stats);
}

extern "C" int eqd_shear_traction(eqd_grid *G, const double *s2, const double *s3, int32_t nslip, double *dtau2,
                                  double *dtau3, const eqd_solve_opts *opts, eqd_stats *stats) {
    if (!G || !s2 || !s3 || !dtau2 || !dtau3) return fail(EQD_ERR_ARG, "null argument");
    if (nslip < 1) return fail(EQD_ERR_ARG, "nslip must be >= 1");
    const int nf = G->gc.nf;
    std::vector<double> dense((size_t)nslip * 2 * nf);
    for (int c = 0; c < nslip; ++c)
        for (int k = 0; k < nf; ++k) {
            dense[((size_t)c * 2 + 0) * nf + k] = s2[(size_t)c * nf + k];
            dense[((size_t)c * 2 + 1) * nf + k] = s3[(size_t)c * nf + k];
        }
    std::vector<int> node(nslip, -1), comp(nslip, 0);
    std::vector<double> out((size_t)2 * nf * nslip);
    BatchSpec B{};
    B.ncols = nslip;
    B.slip_node = node.data();
    B.slip_comp = comp.data();
    B.slip_dense = dense.data();
    B.kcols = out.data();
    int rc = run_batch_any(G, opts, B, stats);
    if (rc) return rc;
    for (int c = 0; c < nslip; ++c)
        for (int k = 0; k < nf; ++k) {
            dtau2[(size_t)c * nf + k] = out[(size_t)c * 2 * nf + k];
            dtau3[(size_t)c * nf + k] = out[(size_t)c * 2 * nf + nf + k];
        }
    return EQD_OK;
}

extern "C" int eqd_cg_solve(eqd_grid *G, const double *rhs, double *u, int32_t ncols, const eqd_solve_opts *opts,
                            int32_t *iters, int8_t *status, eqd_stats *stats) {
    if (!G || !rhs || !u) return fail(EQD_ERR_ARG, "null argument");
    if (ncols < 1) return fail(EQD_ERR_ARG, "ncols must be >= 1");
    eqd_solve_opts o;
    if (opts) o = *opts;
    else eqd_default_opts(&o);
    o.precision = EQD_PREC_FP64;
    BatchSpec B{};
    B.ncols = ncols;
    B.rhs = rhs;
    B.u_out = u;
    B.iters = iters;
    B.status = status;
    return run_batch_any(G, &o, B, stats);
}

extern "C" int eqd_stiffness_toeplitz(eqd_grid *G, const eqd_solve_opts *opts, double *K, eqd_stats *stats) {
    if (!G || !K) return fail(EQD_ERR_ARG, "null argument");
    const GridConst &gc = G->gc;
    const int n2 = gc.n2f, n3 = gc.n3f, nf = gc.nf;
    // Sources in priority order: centre, then the corners (1-based (a, b)).
    const int ac = (n2 + 1) / 2, bc = (n3 + 1) / 2;
    const int sa[5] = {ac, 1, n2, 1, n2}, sb[5] = {bc, 1, 1, n3, n3};
    std::vector<int32_t> cols(10);
    for (int s = 0; s < 5; ++s) {
        const int node = (sb[s] - 1) * n2 + (sa[s] - 1);
        cols[2 * s] = node;
        cols[2 * s + 1] = nf + node;
    }
    std::vector<double> resp((size_t)10 * 2 * nf);
    int rc = eqd_stiffness_columns(G, cols.data(), 10, opts, resp.data(), nullptr, nullptr, stats);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(G->mtx);
    if (G->served) return fail(EQD_ERR_ARG, "the grid is attached to a server");
    CUDA_OR_RETURN(cudaSetDevice(G->desc.device));
    const size_t N = 2 * (size_t)nf;
    DevBuf dK, dsrc, da, db;
    CUDA_OR_RETURN(dK.ensure(sizeof(double) * N * N));
    CUDA_OR_RETURN(dsrc.ensure(sizeof(double) * resp.size()));
    CUDA_OR_RETURN(da.ensure(sizeof(int) * 5));
    CUDA_OR_RETURN(db.ensure(sizeof(int) * 5));
    CUDA_OR_RETURN(cudaMemcpyAsync(dsrc.p, resp.data(), sizeof(double) * resp.size(), cudaMemcpyHostToDevice, G->stream));
    CUDA_OR_RETURN(cudaMemcpyAsync(da.p, sa, sizeof(sa), cudaMemcpyHostToDevice, G->stream));
    CUDA_OR_RETURN(cudaMemcpyAsync(db.p, sb, sizeof(sb), cudaMemcpyHostToDevice, G->stream));
    const long long ne = (long long)nf * nf;
    toeplitz_expand_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, G->stream>>>(dsrc.as<double>(), da.as<int>(),
                                                                              db.as<int>(), 5, n2, n3, dK.as<double>());
    CUDA_OR_RETURN(cudaGetLastError());
    CUDA_OR_RETURN(cudaMemcpyAsync(K, dK.p, sizeof(double) * N * N, cudaMemcpyDeviceToHost, G->stream));
    CUDA_OR_RETURN(cudaStreamSynchronize(G->stream));
    return EQD_OK;
}

template <typename T>
static int profile_apply_impl(eqd_grid *G, int ncols, int warmup, int reps, double *ms, double *bytes) {
    const GridConst &gc = G->gc;
    DevBuf x, y, part;
    const long long n = gc.colstride * (long long)ncols;
    CUDA_OR_RETURN(x.ensure(sizeof(T) * n));
    CUDA_OR_RETURN(y.ensure(sizeof(T) * n));
    if (sizeof(T) == 4 && !G->tuned) {
        eqd_solve_opts o;
        eqd_default_opts(&o);
        int rc = tune_by_iterations(G, o, std::min(ncols, 1024));
        if (rc) return rc;
    }
    int nt = nparts(G->m64);
    for (int v = 0; v < kNumVariants; ++v) nt = std::max(nt, nparts(G->v32[v]));
    CUDA_OR_RETURN(part.ensure(sizeof(double) * 2 * ncols * nt));
    fill_random_kernel<T><<<1184, 256, 0, G->stream>>>(x.as<T>(), n, 12345ull);
    CUDA_OR_RETURN(cudaGetLastError());
    ColumnSet cs{};
    for (int i = 0; i < warmup; ++i)
        CUDA_OR_RETURN((launch_march<T, T, MODE_A>(G, x.as<T>(), y.as<T>(), cs, part.as<double>(), ncols)));
    CUDA_OR_RETURN(cudaEventRecord(G->ev0, G->stream));
    for (int i = 0; i < reps; ++i)
        CUDA_OR_RETURN((launch_march<T, T, MODE_A>(G, x.as<T>(), y.as<T>(), cs, part.as<double>(), ncols)));
    CUDA_OR_RETURN(cudaEventRecord(G->ev1, G->stream));
    CUDA_OR_RETURN(cudaEventSynchronize(G->ev1));
    float t = 0.f;
    CUDA_OR_RETURN(cudaEventElapsedTime(&t, G->ev0, G->ev1));
    if (ms) *ms = (double)t / std::max(reps, 1);
    if (bytes) *bytes = 2.0 * 6.0 * gc.n1 * gc.n2 * gc.n3 * sizeof(T) * ncols;
    return check_device_error(G);
}

extern "C" int eqd_profile_apply(eqd_grid *G, int32_t ncols, int32_t precision, int32_t warmup, int32_t reps,
                                 double *ms_per_launch, double *bytes_per_launch) {
    if (!G || ncols < 1 || reps < 1 || warmup < 0) return fail(EQD_ERR_ARG, "invalid argument");
    std::lock_guard<std::mutex> lk(G->mtx);
    if (G->served) return fail(EQD_ERR_ARG, "the grid is attached to a server");
    CUDA_OR_RETURN(cudaSetDevice(G->desc.device));
    if (precision == EQD_PREC_MIXED) return profile_apply_impl<float>(G, ncols, warmup, reps, ms_per_launch, bytes_per_launch);
    if (precision == EQD_PREC_FP64) return profile_apply_impl<double>(G, ncols, warmup, reps, ms_per_launch, bytes_per_launch);
    return fail(EQD_ERR_ARG, "unknown precision");
}

extern "C" int eqd_autotune(eqd_grid *G, int32_t ncols, int32_t *selected, double *ms_per_variant,
                            int32_t *tile_rows, int32_t *threads, int32_t *nvariants) {
    if (!G || ncols < 0) return fail(EQD_ERR_ARG, "invalid argument");
    std::lock_guard<std::mutex> lk(G->mtx);
    if (G->served) return fail(EQD_ERR_ARG, "the grid is attached to a server");
    CUDA_OR_RETURN(cudaSetDevice(G->desc.device));
    if (ncols > 0) {
        eqd_solve_opts o;
        eqd_default_opts(&o);
        int rc = tune_by_iterations(G, o, ncols);
        if (rc) return rc;
    }
    if (selected) *selected = G->sel32;
    if (nvariants) *nvariants = kNumVariants;
    for (int v = 0; v < kNumVariants; ++v) {
        if (ms_per_variant) ms_per_variant[v] = G->tune_ms[v];
        if (tile_rows) tile_rows[v] = G->v32[v].g.t2max;
        if (threads) threads[v] = G->v32[v].threads;
    }
    return EQD_OK;
}

// Chunk-width tuner: the cost of one column-iteration of the mixed-precision
// CG at each batch width (unit-slip columns, two graph launches = 20
// iterations after one untimed launch), and the cheapest width, which later
// calls with opts.chunk = 0 use (capped by the HBM budget).
extern "C" int eqd_tune_chunk(eqd_grid *G, const int32_t *widths, int32_t nwidths, double *ms_per_column_iteration,
                              int32_t *best) {
    if (!G || !widths || nwidths < 1) return fail(EQD_ERR_ARG, "invalid argument");
    std::lock_guard<std::mutex> lk(G->mtx);
    if (G->served) return fail(EQD_ERR_ARG, "the grid is attached to a server");
    CUDA_OR_RETURN(cudaSetDevice(G->desc.device));
    const GridConst &gc = G->gc;
    eqd_solve_opts o;
    eqd_default_opts(&o);
    int cap = 0;
    int rc = resolve_chunk(G, o, 2 * gc.nf, EQD_PREC_MIXED, cap);
    if (rc) return rc;
    double bestms = 1e300;
    int bestw = 0;
    for (int k = 0; k < nwidths; ++k) {
        const int w = widths[k];
        if (w < 1 || w > 2 * gc.nf || w > cap) {
            if (ms_per_column_iteration) ms_per_column_iteration[k] = -1.0;  // not measured: out of range
            continue;
        }
        std::vector<ColWork> work(w);
        for (int i = 0; i < w; ++i) {
            work[i].slip_node = (int)(((long long)i * 7919 + gc.nf / 2) % gc.nf);
            work[i].slip_comp = i & 1;
            work[i].tag = i;
        }
        SlotRun<float> R;
        rc = R.setup(G, o, w, false, false);
        if (rc) return rc;
        int taken = 0;
        rc = R.admit(work.data(), w, taken);
        if (!rc) rc = R.launch();
        if (rc) return rc;
        CUDA_OR_RETURN(cudaEventRecord(G->ev0, G->stream));
        rc = R.launch();
        if (!rc) rc = R.launch();
        if (rc) return rc;
        CUDA_OR_RETURN(cudaEventRecord(G->ev1, G->stream));
        CUDA_OR_RETURN(cudaEventSynchronize(G->ev1));
        float ms = 0.f;
        CUDA_OR_RETURN(cudaEventElapsedTime(&ms, G->ev0, G->ev1));
        const double per = ms / (2.0 * SlotRun<float>::kIter * w);
        if (ms_per_column_iteration) ms_per_column_iteration[k] = per;
        if (per < bestms) {
            bestms = per;
            bestw = w;
        }
    }
    if (bestw == 0) return fail(EQD_ERR_ARG, "no width within 1 .. min(2 nf, the budget's columns)");
    G->chunk_tuned = bestw;
    if (best) *best = bestw;
    return check_device_error(G);
}

extern "C" int eqd_set_variant(eqd_grid *G, int32_t variant) {
    if (!G || variant < 0 || variant >= kNumVariants) return fail(EQD_ERR_ARG, "invalid variant");
    std::lock_guard<std::mutex> lk(G->mtx);
    if (G->served) return fail(EQD_ERR_ARG, "the grid is attached to a server");
    G->sel32 = variant;
    G->tuned = true;
    return EQD_OK;
}

extern "C" int eqd_test_inject_wait_timeout(eqd_grid *G, int32_t plane, uint32_t poll_limit) {
    if (!G || plane < 0 || plane >= G->gc.n3 || poll_limit == 0) return fail(EQD_ERR_ARG, "invalid argument");
    std::lock_guard<std::mutex> lk(G->mtx);
    if (G->served) return fail(EQD_ERR_ARG, "the grid is attached to a server");
    if (G->v32[G->sel32].ring_t2 <= 0)
        return fail(EQD_ERR_UNSUPPORTED, "the grid's FP32 apply variant is not a ring-march variant");
    G->test_drop_plane = plane;
    G->test_poll_limit = poll_limit;
    return EQD_OK;
}

// Sparse A (which = 0) or HP_DSAT (which = 1) in reference DOF order, CSR,
// by coloured probing with the FP64 operator kernels (probe_* kernels).
static constexpr int kProbeRowCap = 128;        // entries a row may hold before the drop (measured at most 96)
static constexpr double kProbeRelDrop = 1e-12;  // entries below this fraction of the row's largest are rounding

extern "C" int eqd_assemble(eqd_grid *G, int32_t which, int64_t capacity, int64_t *indptr, int32_t *indices,
                            double *values, int64_t *nnz) {
    if (!G || !nnz || (which != 0 && which != 1) || capacity < 0) return fail(EQD_ERR_ARG, "invalid argument");
    std::lock_guard<std::mutex> lk(G->mtx);
    if (G->served) return fail(EQD_ERR_ARG, "the grid is attached to a server");
    CUDA_OR_RETURN(cudaSetDevice(G->desc.device));
    const GridConst &gc = G->gc;
    ProbeGeom pg{};
    pg.n1 = gc.n1;
    pg.n2 = gc.n2;
    pg.n3 = gc.n3;
    pg.PS = gc.PS;
    pg.colstride = gc.colstride;
    pg.N = (long long)gc.n1 * gc.n2 * gc.n3;
    pg.R = 6;
    pg.P2 = gc.n2 <= 2 * pg.R + 1 ? gc.n2 : 2 * pg.R + 1;
    pg.P3 = gc.n3 <= 2 * pg.R + 1 ? gc.n3 : 2 * pg.R + 1;
    pg.ncolors = 6LL * gc.n1 * pg.P2 * pg.P3;
    const long long ntot = 6 * pg.N;
    if (ntot > INT32_MAX) return fail(EQD_ERR_UNSUPPORTED, "more DOFs than 32-bit column indices hold");
    // Probe chunk: at most 512 colours, within a quarter of free memory for x and y.
    size_t fr = 0, tot = 0;
    CUDA_OR_RETURN(cudaMemGetInfo(&fr, &tot));
    const size_t per = 2 * sizeof(double) * (size_t)gc.colstride;
    long long nc = std::min<long long>({512, pg.ncolors, (long long)(fr / 4 / per)});
    if (nc < 1) return fail(EQD_ERR_OOM, "no room for one probe");
    DevBuf x, y, sn, scomp, rcnt, rcol, rval, rmax, kept, dptr, dind, dval, ovf;
    CUDA_OR_RETURN(x.ensure(sizeof(double) * gc.colstride * nc));
    CUDA_OR_RETURN(y.ensure(sizeof(double) * gc.colstride * nc));
    CUDA_OR_RETURN(sn.ensure(sizeof(int) * nc));
    CUDA_OR_RETURN(scomp.ensure(sizeof(int) * nc));
    CUDA_OR_RETURN(rcnt.ensure(sizeof(int) * ntot));
    CUDA_OR_RETURN(rcol.ensure(sizeof(int) * ntot * kProbeRowCap));
    CUDA_OR_RETURN(rval.ensure(sizeof(double) * ntot * kProbeRowCap));
    CUDA_OR_RETURN(rmax.ensure(sizeof(double) * ntot));
    CUDA_OR_RETURN(kept.ensure(sizeof(long long) * ntot));
    CUDA_OR_RETURN(ovf.ensure(sizeof(unsigned)));
    cudaStream_t st = G->stream;
    CUDA_OR_RETURN(cudaMemsetAsync(rcnt.p, 0, sizeof(int) * ntot, st));
    CUDA_OR_RETURN(cudaMemsetAsync(rmax.p, 0, sizeof(double) * ntot, st));
    CUDA_OR_RETURN(cudaMemsetAsync(ovf.p, 0, sizeof(unsigned), st));
    {
        std::vector<int> neg(nc, -1);
        CUDA_OR_RETURN(cudaMemcpyAsync(sn.p, neg.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st));
        CUDA_OR_RETURN(cudaMemsetAsync(scomp.p, 0, sizeof(int) * nc, st));
        CUDA_OR_RETURN(cudaStreamSynchronize(st));
    }
    ColumnSet cs{};
    cs.slip_node = sn.as<int>();  // no slip: HP_DSAT x without the chi term
    cs.slip_comp = scomp.as<int>();
    const unsigned rb = (unsigned)((ntot + 255) / 256);
    for (long long c0 = 0; c0 < pg.ncolors; c0 += nc) {
        const int n = (int)std::min<long long>(nc, pg.ncolors - c0);
        CUDA_OR_RETURN(cudaMemsetAsync(x.p, 0, sizeof(double) * gc.colstride * n, st));
        probe_fill_kernel<<<1184, 256, 0, st>>>(pg, c0, n, x.as<double>());
        CUDA_OR_RETURN(cudaGetLastError());
        if (which == 0)
            CUDA_OR_RETURN((launch_march<double, double, MODE_AP>(G, x.as<double>(), y.as<double>(), cs, nullptr, n)));
        else
            CUDA_OR_RETURN((launch_march<double, double, MODE_RHS>(G, x.as<double>(), y.as<double>(), cs, nullptr, n)));
        probe_extract_kernel<<<rb, 256, 0, st>>>(pg, c0, n, y.as<double>(), kProbeRowCap, rcnt.as<int>(), rcol.as<int>(),
                                                 rval.as<double>(), rmax.as<double>(), ovf.as<unsigned>());
        CUDA_OR_RETURN(cudaGetLastError());
    }
    probe_compact_kernel<<<rb, 256, 0, st>>>(ntot, kProbeRowCap, rcnt.as<int>(), rcol.as<int>(), rval.as<double>(),
                                             rmax.as<double>(), kProbeRelDrop, 0, nullptr, nullptr, nullptr,
                                             kept.as<long long>());
    CUDA_OR_RETURN(cudaGetLastError());
    std::vector<long long> cnt(ntot);
    unsigned hovf = 0;
    CUDA_OR_RETURN(cudaMemcpyAsync(cnt.data(), kept.p, sizeof(long long) * ntot, cudaMemcpyDeviceToHost, st));
    CUDA_OR_RETURN(cudaMemcpyAsync(&hovf, ovf.p, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CUDA_OR_RETURN(cudaStreamSynchronize(st));
    int rc = check_device_error(G);
    if (rc) return rc;
    if (hovf) return fail(EQD_ERR_UNSUPPORTED, "a row holds more than " + std::to_string(kProbeRowCap) + " entries");
    std::vector<long long> off(ntot + 1, 0);
    for (long long i = 0; i < ntot; ++i) off[i + 1] = off[i] + cnt[i];
    *nnz = off[ntot];
    if (!indptr && !indices && !values) return EQD_OK;  // size query
    if (!indptr || !indices || !values) return fail(EQD_ERR_ARG, "indptr, indices and values go together");
    if (capacity < off[ntot])
        return fail(EQD_ERR_ARG, "capacity " + std::to_string(capacity) + " below nnz " + std::to_string(off[ntot]));
    CUDA_OR_RETURN(dptr.ensure(sizeof(long long) * (ntot + 1)));
    CUDA_OR_RETURN(dind.ensure(sizeof(int) * std::max<long long>(off[ntot], 1)));
    CUDA_OR_RETURN(dval.ensure(sizeof(double) * std::max<long long>(off[ntot], 1)));
    CUDA_OR_RETURN(cudaMemcpyAsync(dptr.p, off.data(), sizeof(long long) * (ntot + 1), cudaMemcpyHostToDevice, st));
    probe_compact_kernel<<<rb, 256, 0, st>>>(ntot, kProbeRowCap, rcnt.as<int>(), rcol.as<int>(), rval.as<double>(),
                                             rmax.as<double>(), kProbeRelDrop, 1, dptr.as<long long>(), dind.as<int>(),
                                             dval.as<double>(), nullptr);
    CUDA_OR_RETURN(cudaGetLastError());
    CUDA_OR_RETURN(cudaMemcpyAsync(indices, dind.p, sizeof(int) * off[ntot], cudaMemcpyDeviceToHost, st));
    CUDA_OR_RETURN(cudaMemcpyAsync(values, dval.p, sizeof(double) * off[ntot], cudaMemcpyDeviceToHost, st));
    CUDA_OR_RETURN(cudaStreamSynchronize(st));
    for (long long i = 0; i <= ntot; ++i) indptr[i] = off[i];
    return EQD_OK;
}

extern "C" int eqd_diag(eqd_grid *G, double *d) {
    if (!G || !d) return fail(EQD_ERR_ARG, "invalid argument");
    std::lock_guard<std::mutex> lk(G->mtx);
    if (G->served) return fail(EQD_ERR_ARG, "the grid is attached to a server");
    CUDA_OR_RETURN(cudaSetDevice(G->desc.device));
    const GridConst &gc = G->gc;
    const long long n = 6LL * gc.n1 * gc.n2 * gc.n3;
    DevBuf dev, ref, neg;
    CUDA_OR_RETURN(dev.ensure(sizeof(double) * gc.colstride));
    CUDA_OR_RETURN(ref.ensure(sizeof(double) * n));
    CUDA_OR_RETURN(neg.ensure(sizeof(unsigned)));
    CUDA_OR_RETURN(cudaMemsetAsync(neg.p, 0, sizeof(unsigned), G->stream));
    jacobi_diag_kernel<<<(unsigned)((n + 255) / 256), 256, 0, G->stream>>>(G->c64, gc.n1, gc.n2, gc.n3, gc.PS,
                                                                            dev.as<double>(), nullptr, nullptr,
                                                                            neg.as<unsigned>());
    dev_to_ref_kernel<double, double><<<(unsigned)((n + 255) / 256), 256, 0, G->stream>>>(
        dev.as<double>(), ref.as<double>(), gc.n1, gc.n2, gc.n3, gc.PS, gc.colstride, 1);
    CUDA_OR_RETURN(cudaGetLastError());
    CUDA_OR_RETURN(cudaMemcpyAsync(d, ref.p, sizeof(double) * n, cudaMemcpyDeviceToHost, G->stream));
    CUDA_OR_RETURN(cudaStreamSynchronize(G->stream));
    return EQD_OK;
}

// ---------------------------------------------------------------------------
// Resident K and the time-loop GEMV
// ---------------------------------------------------------------------------
extern "C" int eqd_kmat_create(int32_t device, int32_t n, const double *K, eqd_kmat **out) {
    if (!out || !K || n < 1) return fail(EQD_ERR_ARG, "invalid argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(EQD_ERR_NO_DEVICE, "no CUDA device visible");
    if (device < 0 || device >= ndev) return fail(EQD_ERR_ARG, "device ordinal out of range");
    CUDA_OR_RETURN(cudaSetDevice(device));
    std::unique_ptr<eqd_kmat> M(new eqd_kmat());
    M->device = device;
    M->n = n;
    CUDA_OR_RETURN(M->K.ensure(sizeof(double) * (size_t)n * n));
    CUDA_OR_RETURN(cudaStreamCreateWithFlags(&M->stream, cudaStreamNonBlocking));
    int sms = 0, per_sm[3] = {0, 0, 0};
    CUDA_OR_RETURN(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    CUDA_OR_RETURN(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[0], gemm_ks_dmma_kernel<true, 1, 32>, 256, 0));
    CUDA_OR_RETURN(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[1], gemm_ks_dmma_kernel<true, 2, 32>, 256, 0));
    CUDA_OR_RETURN(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[2], gemm_ks_dmma_kernel<true, 4, 16>, 256, 0));
    for (int k = 0; k < 3; ++k) M->ks_slots[k] = std::max(1, sms * per_sm[k]);
    CUDA_OR_RETURN(cudaMemcpyAsync(M->K.p, K, sizeof(double) * (size_t)n * n, cudaMemcpyHostToDevice, M->stream));
    CUDA_OR_RETURN(cudaStreamSynchronize(M->stream));
    *out = M.release();
    return EQD_OK;
}

// The GEMV's first pass: 16-byte loads of K where K and n allow them
// (gemv_vec2_ok), 8-byte loads otherwise.
static void launch_gemv_partial(dim3 grid, cudaStream_t st, const double *K, const double *s, long long n, int nslice,
                                int nvec, double *part) {
    if (gemv_vec2_ok(K, n))
        gemv_partial_kernel<true><<<grid, 256, 0, st>>>(K, s, n, nslice, nvec, part);
    else
        gemv_partial_kernel<false><<<grid, 256, 0, st>>>(K, s, n, nslice, nvec, part);
}

static int gemv_slices(int n) {
    // Enough CTAs to cover every SM several times over.
    const int rows_blocks = (n / 2 + 255) / 256;
    int s = std::max(1, (148 * 8) / std::max(1, rows_blocks));
    return std::min(s, std::max(1, n / 64));
}

// Vectors from which y = K s runs as the blocked K S on the FP64 tensor
// cores (K read once per 16-64 vectors) instead of the GEMV (K read once per
// 4). Measured at n = 13,122: GEMV 0.25 / 0.25 / 0.32 / 0.44 ms for 1-4
// vectors (1.1-1.8 ms for 5-8), the tensor-core path 0.27-0.32 ms for 2-8.
static constexpr int kGemmMinVectors = 3;

// Column slices of the blocked K S: the count (1..16, slices of at least 128
// columns) with the least time in whole waves of resident CTAs,
// ceil(tiles * ns / slots) / ns; the smallest count on ties.
static int ks_slices(long long n, int nvec, int bn, int slots) {
    const long long tiles = ((n + kDmmaBM - 1) / kDmmaBM) * ((nvec + bn - 1) / bn);
    const int max_ns = (int)std::max<long long>(1, std::min<long long>(16, n / 128));
    int best = 1;
    double best_t = 1e300;
    for (int ns = 1; ns <= max_ns; ++ns) {
        const double tm = (double)((tiles * ns + slots - 1) / slots) / ns;
        if (tm < best_t * (1.0 - 1e-9)) {
            best_t = tm;
            best = ns;
        }
    }
    return best;
}

// y = K s for nvec device-resident vectors (s, y: n x nvec, column-major) on
// stream st; returns after the launches. Scratch: M->part.
static int kmat_apply(eqd_kmat *M, const double *s, double *y, int nvec, cudaStream_t st) {
    const int n = M->n;
    const long long ne = (long long)n * nvec;
    const double *K = M->K.as<double>();
    if (nvec >= kGemmMinVectors) {
        // Vector tile: 16, 32 or 64 vectors per CTA, the narrowest that holds nvec.
        const int tk = nvec <= 16 ? 0 : nvec <= 32 ? 1 : 2, bn = 16 << tk;
        // The slice count depends only on n, nvec and the tile (the
        // occupancy of the 16-byte-load instance on either load path), so a
        // product is the same bits whatever the slips' alignment.
        const int ns = ks_slices(n, nvec, bn, M->ks_slots[tk]);
        CUDA_OR_RETURN(M->part.ensure(sizeof(double) * (size_t)ne * ns));
        const dim3 grid((unsigned)((n + kDmmaBM - 1) / kDmmaBM), (unsigned)ns, (unsigned)((nvec + bn - 1) / bn));
        const bool v2 = gemv_vec2_ok(K, n) && gemv_vec2_ok(s, n);
        double *pp = M->part.as<double>();
#define EQD_KS(V, NT) gemm_ks_dmma_kernel<V, NT, (NT < 4 ? 32 : 16)><<<grid, 256, 0, st>>>(K, s, n, ns, nvec, pp)
        if (tk == 0) { if (v2) EQD_KS(true, 1); else EQD_KS(false, 1); }
        else if (tk == 1) { if (v2) EQD_KS(true, 2); else EQD_KS(false, 2); }
        else { if (v2) EQD_KS(true, 4); else EQD_KS(false, 4); }
#undef EQD_KS
        gemv_reduce_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(M->part.as<double>(), n, ns, nvec, y);
    } else {
        const int nslice = gemv_slices(n);
        CUDA_OR_RETURN(M->part.ensure(sizeof(double) * (size_t)ne * nslice));
        dim3 grid((unsigned)(((n + 1) / 2 + 255) / 256), (unsigned)nslice);
        launch_gemv_partial(grid, st, K, s, n, nslice, nvec, M->part.as<double>());
        gemv_reduce_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(M->part.as<double>(), n, nslice, nvec, y);
    }
    CUDA_OR_RETURN(cudaGetLastError());
    return EQD_OK;
}

extern "C" int eqd_kmat_gemv(eqd_kmat *M, const double *s, double *y, int32_t nvec) {
    if (!M || !s || !y || nvec < 1) return fail(EQD_ERR_ARG, "invalid argument");
    CUDA_OR_RETURN(cudaSetDevice(M->device));
    const size_t bytes = sizeof(double) * (size_t)M->n * nvec;
    CUDA_OR_RETURN(M->s.ensure(bytes));
    CUDA_OR_RETURN(M->y.ensure(bytes));
    CUDA_OR_RETURN(cudaMemcpyAsync(M->s.p, s, bytes, cudaMemcpyHostToDevice, M->stream));
    const int rc = kmat_apply(M, M->s.as<double>(), M->y.as<double>(), nvec, M->stream);
    if (rc) return rc;
    CUDA_OR_RETURN(cudaMemcpyAsync(y, M->y.p, bytes, cudaMemcpyDeviceToHost, M->stream));
    CUDA_OR_RETURN(cudaStreamSynchronize(M->stream));
    return EQD_OK;
}

extern "C" int eqd_kmat_gemv_device(eqd_kmat *M, const double *s_device, double *y_device, int32_t nvec,
                                    void *stream) {
    if (!M || !s_device || !y_device || nvec < 1) return fail(EQD_ERR_ARG, "invalid argument");
    if ((reinterpret_cast<uintptr_t>(s_device) & 7u) || (reinterpret_cast<uintptr_t>(y_device) & 7u))
        return fail(EQD_ERR_ARG, "s and y must be 8-byte aligned");
    CUDA_OR_RETURN(cudaSetDevice(M->device));
    return kmat_apply(M, s_device, y_device, nvec, static_cast<cudaStream_t>(stream));
}

extern "C" int eqd_kmat_destroy(eqd_kmat *M) {
    if (!M) return EQD_OK;
    cudaSetDevice(M->device);
    if (M->stream) {
        cudaStreamSynchronize(M->stream);
        cudaStreamDestroy(M->stream);
    }
    delete M;
    return EQD_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free GEMV.
//
// For callers that must not allocate device memory at all: a time loop that
// runs inside a CUDA graph or under a framework's own device allocator (a
// Julia CuArray pool, a PyTorch caching allocator), where a hidden cudaMalloc
// would break capture or fragment the caller's pool, and latency-critical
// loops that may not block on the allocator. The caller passes K, s and y as
// device pointers it already owns; the only scratch (the per-slice partial
// row sums of the two-pass GEMV) lives in this file-scope array, 4 MiB per
// device, held by every GPU that loads the library until exit. The first call
// on a device looks the array's device address up (with that device current);
// make that first call before any stream capture. All calls on a device share
// the array: calls that overlap on the GPU race, so serialise them (one
// stream, or events). The array keeps the last call's contents; nothing in it
// needs to start at zero, because every partial sum read in a call was written
// in the same call.
// ---------------------------------------------------------------------------
#define EQD_GEMV_STATIC_SCRATCH_DOUBLES (1 << 19)

static __device__ __align__(256) double g_gemv_static_scratch[EQD_GEMV_STATIC_SCRATCH_DOUBLES];

static std::mutex g_gemv_static_mtx;
static double *g_gemv_static_ptr[128] = {nullptr};

extern "C" int eqd_kmat_gemv_static(int32_t device, int32_t n, const double *K_device, const double *s_device,
                                    double *y_device, int32_t nvec, void *stream) {
    if (n < 1 || nvec < 1 || !K_device || !s_device || !y_device) return fail(EQD_ERR_ARG, "invalid argument");
    if ((long long)n * nvec > EQD_GEMV_STATIC_SCRATCH_DOUBLES)
        return fail(EQD_ERR_ARG, "eqd_kmat_gemv_static: n * nvec = " + std::to_string((long long)n * nvec) +
                                     " exceeds the static scratch of " +
                                     std::to_string(EQD_GEMV_STATIC_SCRATCH_DOUBLES) + " doubles");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(EQD_ERR_NO_DEVICE, "no CUDA device visible");
    if (device < 0 || device >= ndev || device >= 128) return fail(EQD_ERR_ARG, "device ordinal out of range");
    int prev = 0;
    CUDA_OR_RETURN(cudaGetDevice(&prev));
    if (prev != device) CUDA_OR_RETURN(cudaSetDevice(device));
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_gemv_static_mtx);
        if (!g_gemv_static_ptr[device]) {
            void *ptr = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&ptr, g_gemv_static_scratch);
            if (e != cudaSuccess) {
                if (prev != device) cudaSetDevice(prev);
                return fail(EQD_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
            }
            g_gemv_static_ptr[device] = static_cast<double *>(ptr);
        }
        scratch = g_gemv_static_ptr[device];
    }
    int nslice = gemv_slices(n);
    nslice = std::max(1, std::min<int>(nslice, (int)(EQD_GEMV_STATIC_SCRATCH_DOUBLES / ((long long)n * nvec))));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    dim3 grid((unsigned)(((n + 1) / 2 + 255) / 256), (unsigned)nslice);
    launch_gemv_partial(grid, st, K_device, s_device, n, nslice, nvec, scratch);
    const long long ne = (long long)n * nvec;
    gemv_reduce_kernel<<<(unsigned)((ne + 255) / 256), 256, 0, st>>>(scratch, n, nslice, nvec, y_device);
    cudaError_t e = cudaGetLastError();
    if (prev != device) cudaSetDevice(prev);
    if (e != cudaSuccess) return fail(EQD_ERR_CUDA, std::string("eqd_kmat_gemv_static launch: ") + cudaGetErrorString(e));
    return EQD_OK;
}

// ---------------------------------------------------------------------------
// Server: continuous batching of stiffness-column requests across grids.
// Each attached grid has a slot engine and a worker thread of its own: it
// admits queued columns into free slots, runs the next graph of iterations
// on the grid's streams (grids overlap on the device), then collects
// finished columns and writes them to their requests' host buffers.
// ---------------------------------------------------------------------------
namespace {

struct SrvRequest {
    int64_t id = 0;
    double *k_out = nullptr;
    int ncols = 0, remaining = 0, unconverged = 0, max_it = 0;
    int64_t iterations = 0;
    int state = 0;  // 0 queued, 1 running, 2 done, 3 failed
    int err = EQD_OK;
    std::string msg;
    double t_submit = 0, t_start = -1, t_done = -1;
};

struct SrvGrid {
    eqd_grid *G = nullptr;
    int slots = 0;
    size_t bytes = 0;
    std::unique_ptr<SlotRun<float>> r32;
    std::unique_ptr<SlotRun<double>> r64;
    std::deque<ColWork> pending;  // guarded by the server mutex
    PinnedArr<double> kstage;     // finished K columns, compact
    std::vector<ColDone> done;
    std::thread worker;
    int held() const { return r32 ? r32->held : r64->held; }
    int free_slots() const { return r32 ? r32->free_slots() : r64->free_slots(); }
};

// Column tags carry the request id and the column's position in it.
constexpr int kTagBits = 24;

}  // namespace

struct eqd_server {
    eqd_solve_opts opts{};
    uint64_t budget = 0, used = 0;
    std::vector<std::unique_ptr<SrvGrid>> grids;
    std::map<int64_t, std::unique_ptr<SrvRequest>> reqs;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stop = false;
    int64_t next_id = 1;
    int fatal = EQD_OK;
    std::string fatal_msg;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    double now() const { return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count(); }
};

static void server_fail_all(eqd_server *S, int code, const std::string &msg) {
    std::lock_guard<std::mutex> lk(S->mu);
    S->fatal = code;
    S->fatal_msg = msg;
    for (auto &kv : S->reqs) {
        SrvRequest &r = *kv.second;
        if (r.state < 2) {
            r.state = 3;
            r.err = code;
            r.msg = msg;
            r.t_done = S->now();
        }
    }
    for (auto &g : S->grids) g->pending.clear();
    S->cv_done.notify_all();
}

// Admission order of a grid's queued columns: the request with the fewest
// columns still queued goes first (a small request is not held behind the
// columns of a large one that arrived earlier), unless the oldest queued
// request has waited longer than kServeAgeLimit seconds, which then goes
// first (no request starves). A request's columns stay in submission order.
// Queued columns of one request are contiguous in `pending` (submit appends
// them under the server lock).
constexpr double kServeAgeLimit = 2.0;

static void take_columns(eqd_server *S, SrvGrid &g, int nfree, std::vector<ColWork> &take) {
    struct Run {
        size_t beg, len;
        double t_submit;
    };
    while ((int)take.size() < nfree && !g.pending.empty()) {
        std::vector<Run> runs;
        for (size_t i = 0; i < g.pending.size();) {
            const int64_t id = g.pending[i].tag >> kTagBits;
            size_t j = i + 1;
            while (j < g.pending.size() && (g.pending[j].tag >> kTagBits) == id) ++j;
            auto it = S->reqs.find(id);
            runs.push_back(Run{i, j - i, it != S->reqs.end() ? it->second->t_submit : 0.0});
            i = j;
        }
        size_t pick = 0;  // runs[0] is the oldest
        if (S->now() - runs[0].t_submit <= kServeAgeLimit)
            for (size_t k = 1; k < runs.size(); ++k)
                if (runs[k].len < runs[pick].len) pick = k;
        const Run r = runs[pick];
        const size_t n = std::min(r.len, (size_t)(nfree - (int)take.size()));
        for (size_t k = 0; k < n; ++k) take.push_back(g.pending[r.beg + k]);
        g.pending.erase(g.pending.begin() + (long)r.beg, g.pending.begin() + (long)(r.beg + n));
    }
}

// One pass of a grid's worker: admit queued columns into free slots, run
// the next graph of iterations, deliver the columns that finished.
static int grid_pass(eqd_server *S, SrvGrid &g) {
    eqd_grid *G = g.G;
    std::vector<ColWork> take;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        take_columns(S, g, g.free_slots(), take);
        const double t = S->now();
        for (const ColWork &c : take) {
            auto it = S->reqs.find(c.tag >> kTagBits);
            if (it != S->reqs.end() && it->second->state == 0) {
                it->second->state = 1;
                it->second->t_start = t;
            }
        }
    }
    int rc = EQD_OK, taken = 0;
    if (!take.empty())
        rc = g.r32 ? g.r32->admit(take.data(), (int)take.size(), taken)
                   : g.r64->admit(take.data(), (int)take.size(), taken);
    if (rc) return rc;
    if (g.held() == 0) return EQD_OK;
    rc = g.r32 ? g.r32->advance(g.done) : g.r64->advance(g.done);
    if (rc) return rc;
    if (g.done.empty()) return EQD_OK;
    const int nf2 = 2 * G->gc.nf;
    rc = g.r32 ? g.r32->extract(g.done, G->ws.kout.as<double>(), nf2, false)
               : g.r64->extract(g.done, G->ws.kout.as<double>(), nf2, false);
    if (rc) return rc;
    CUDA_OR_RETURN(cudaMemcpyAsync(g.kstage.data(), G->ws.kout.p, sizeof(double) * nf2 * g.done.size(),
                                   cudaMemcpyDeviceToHost, G->stream));
    CUDA_OR_RETURN(cudaStreamSynchronize(G->stream));
    {
        std::lock_guard<std::mutex> lk(S->mu);
        const double t = S->now();
        bool any_done = false;
        for (size_t j = 0; j < g.done.size(); ++j) {
            const ColDone &d = g.done[j];
            auto it = S->reqs.find(d.tag >> kTagBits);
            if (it == S->reqs.end()) continue;
            SrvRequest &r = *it->second;
            const long long pos = d.tag & ((1LL << kTagBits) - 1);
            std::memcpy(r.k_out + (size_t)pos * nf2, g.kstage.data() + j * nf2, sizeof(double) * nf2);
            r.iterations += d.iters;
            r.max_it = std::max(r.max_it, d.iters);
            if (d.status != COL_CONVERGED) ++r.unconverged;
            if (--r.remaining == 0) {
                r.state = 2;
                r.t_done = t;
                any_done = true;
            }
        }
        if (any_done) S->cv_done.notify_all();
    }
    return g.r32 ? g.r32->release(g.done) : g.r64->release(g.done);
}

// One worker thread per grid: a grid advances at its own pace (its graphs
// run on its own streams), so a request on a small grid is not held behind
// the long iterations of a large one.
static void grid_loop(eqd_server *S, SrvGrid *g) {
    if (cudaSetDevice(g->G->desc.device) != cudaSuccess) {
        server_fail_all(S, EQD_ERR_CUDA, "cudaSetDevice failed in a server worker");
        return;
    }
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(S->mu);
            S->cv_work.wait(lk, [&] { return S->stop || S->fatal || !g->pending.empty() || g->held() > 0; });
            if (S->stop || S->fatal) return;
        }
        const int rc = grid_pass(S, *g);
        if (rc) {
            server_fail_all(S, rc, g_last_error);
            S->cv_work.notify_all();
            return;
        }
    }
}

extern "C" int eqd_server_create(const eqd_solve_opts *opts, uint64_t hbm_budget_bytes, eqd_server **out) {
    if (!out) return fail(EQD_ERR_ARG, "null argument");
    *out = nullptr;
    std::unique_ptr<eqd_server> S(new eqd_server());
    if (opts) S->opts = *opts;
    else eqd_default_opts(&S->opts);
    const eqd_solve_opts &o = S->opts;
    if (!(o.rtol >= 0) || !(o.atol >= 0)) return fail(EQD_ERR_ARG, "rtol/atol must be non-negative");
    if (o.precision != EQD_PREC_FP64 && o.precision != EQD_PREC_MIXED) return fail(EQD_ERR_ARG, "unknown precision");
    if (o.precond != EQD_PRECOND_NONE && o.precond != EQD_PRECOND_JACOBI)
        return fail(EQD_ERR_ARG, "precond must be :none or :jacobi");
    S->budget = hbm_budget_bytes;
    if (S->budget == 0) {
        size_t fr = 0, tot = 0;
        CUDA_OR_RETURN(cudaMemGetInfo(&fr, &tot));
        const size_t keep = (size_t)2 << 30;
        S->budget = fr > keep ? fr - keep : fr / 2;
    }
    *out = S.release();
    return EQD_OK;
}

// Stream priorities of a served grid: smaller grids get higher priority, so
// their short kernels take SM slots ahead of a large grid's long ones (a
// request on the h = 100 m grid is not starved by h = 25 m work). Within a
// grid the vector kernels stay one level above the stencil applies.
static int set_grid_priority(eqd_grid *G) {
    int least = 0, greatest = 0;
    CUDA_OR_RETURN(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    const double ntot = 6.0 * G->gc.n1 * G->gc.n2 * G->gc.n3;
    const int bucket = std::max(0, (int)std::floor(std::log10(std::max(ntot, 1.0))) - 4);  // 0: < 1e5 DOF
    const int step = least > greatest ? -1 : 1;                 // direction of "higher priority"
    const int span = std::abs(least - greatest);
    const int main_p = greatest - step * std::min(span, 1 + bucket);
    const int rest_p = greatest - step * std::min(span, bucket);
    CUDA_OR_RETURN(cudaStreamSynchronize(G->stream));
    for (cudaStream_t t : {G->stream, G->stream2, G->stream_hi, G->stream2_hi}) cudaStreamDestroy(t);
    CUDA_OR_RETURN(cudaStreamCreateWithPriority(&G->stream, cudaStreamNonBlocking, main_p));
    CUDA_OR_RETURN(cudaStreamCreateWithPriority(&G->stream2, cudaStreamNonBlocking, main_p));
    CUDA_OR_RETURN(cudaStreamCreateWithPriority(&G->stream_hi, cudaStreamNonBlocking, rest_p));
    CUDA_OR_RETURN(cudaStreamCreateWithPriority(&G->stream2_hi, cudaStreamNonBlocking, rest_p));
    G->ws.graph_key.clear();  // recapture on the new streams
    return EQD_OK;
}

extern "C" int eqd_server_add_grid(eqd_server *S, eqd_grid *G, int32_t slots) {
    if (!S || !G || slots < 0) return fail(EQD_ERR_ARG, "invalid argument");
    {
        std::lock_guard<std::mutex> lk(S->mu);
        for (auto &g : S->grids)
            if (g->G == G) return fail(EQD_ERR_ARG, "grid already attached");
    }
    std::lock_guard<std::mutex> glk(G->mtx);
    if (G->served) return fail(EQD_ERR_ARG, "the grid is attached to another server");
    CUDA_OR_RETURN(cudaSetDevice(G->desc.device));
    const GridConst &gc = G->gc;
    const int mixed = S->opts.precision == EQD_PREC_MIXED;
    const int nvec = 3 + (mixed ? 1 : 0) + ((S->opts.flags & EQD_FLAG_FUSE) ? 1 : 0);
    const size_t per_slot = (size_t)gc.colstride * (8 + (size_t)nvec * (mixed ? 4 : 8)) + (size_t)16 * gc.nf + 1024;
    std::unique_ptr<SrvGrid> g(new SrvGrid());
    {
        std::lock_guard<std::mutex> lk(S->mu);
        const uint64_t left = S->budget > S->used ? S->budget - S->used : 0;
        const long long fit = (long long)(left / per_slot);
        const int want = slots > 0 ? slots : (int)std::min<long long>(fit, 512);
        if (want < 1 || (long long)want > fit)
            return fail(EQD_ERR_OOM, "the server's HBM budget has room for " + std::to_string(fit) +
                                         " slot(s) of this grid");
        g->slots = want;
        g->bytes = (size_t)want * per_slot;
        S->used += g->bytes;
    }
    g->G = G;
    int rc = set_grid_priority(G);
    if (rc) {
        std::lock_guard<std::mutex> lk(S->mu);
        S->used -= g->bytes;
        return rc;
    }
    if (mixed) {
        g->r32.reset(new SlotRun<float>());
        rc = g->r32->setup(G, S->opts, g->slots, false, false);
    } else {
        g->r64.reset(new SlotRun<double>());
        rc = g->r64->setup(G, S->opts, g->slots, false, false);
    }
    if (!rc) {
        cudaError_t e = g->kstage.assign(2 * gc.nf * g->slots, 0.0);
        if (e != cudaSuccess) rc = fail(EQD_ERR_OOM, "pinned staging buffer");
    }
    if (!rc) {
        cudaError_t e = cudaStreamSynchronize(G->stream);
        if (e != cudaSuccess) rc = fail(EQD_ERR_CUDA, cudaGetErrorString(e));
    }
    if (rc) {
        std::lock_guard<std::mutex> lk(S->mu);
        S->used -= g->bytes;
        return rc;
    }
    G->served = true;
    std::lock_guard<std::mutex> lk(S->mu);
    SrvGrid *gp = g.get();
    S->grids.push_back(std::move(g));
    gp->worker = std::thread(grid_loop, S, gp);
    return EQD_OK;
}

extern "C" int eqd_server_submit(eqd_server *S, eqd_grid *G, const int32_t *cols, int32_t ncols, double *k_out,
                                 int64_t *request_id) {
    if (!S || !G || (!cols && ncols > 0) || ncols < 0 || (!k_out && ncols > 0) || !request_id)
        return fail(EQD_ERR_ARG, "invalid argument");
    if (ncols >= (1 << kTagBits)) return fail(EQD_ERR_ARG, "too many columns in one request");
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->fatal) return fail(S->fatal, "server stopped: " + S->fatal_msg);
    SrvGrid *g = nullptr;
    for (auto &x : S->grids)
        if (x->G == G) g = x.get();
    if (!g) return fail(EQD_ERR_ARG, "grid not attached to this server");
    const int nf = G->gc.nf;
    for (int i = 0; i < ncols; ++i)
        if (cols[i] < 0 || cols[i] >= 2 * nf) return fail(EQD_ERR_ARG, "column index out of range");
    std::unique_ptr<SrvRequest> r(new SrvRequest());
    r->id = S->next_id++;
    r->k_out = k_out;
    r->ncols = r->remaining = ncols;
    r->t_submit = S->now();
    if (ncols == 0) {
        r->state = 2;
        r->t_start = r->t_done = r->t_submit;
    }
    for (int i = 0; i < ncols; ++i) {
        ColWork c;
        c.slip_node = cols[i] % nf;
        c.slip_comp = cols[i] / nf;
        c.tag = (r->id << kTagBits) | i;
        g->pending.push_back(c);
    }
    *request_id = r->id;
    S->reqs[r->id] = std::move(r);
    S->cv_work.notify_all();
    return EQD_OK;
}

static SrvRequest *find_req(eqd_server *S, int64_t id) {
    auto it = S->reqs.find(id);
    return it == S->reqs.end() ? nullptr : it->second.get();
}

extern "C" int eqd_server_wait(eqd_server *S, int64_t id, double timeout_s) {
    if (!S) return fail(EQD_ERR_ARG, "null server");
    std::unique_lock<std::mutex> lk(S->mu);
    SrvRequest *r = find_req(S, id);
    if (!r) return fail(EQD_ERR_ARG, "unknown request id");
    const auto pred = [&] { return r->state >= 2; };
    if (timeout_s < 0) S->cv_done.wait(lk, pred);
    else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
        return fail(EQD_ERR_TIMEOUT, "request not done within the timeout");
    if (r->state == 3) return fail(r->err, r->msg);
    return EQD_OK;
}

extern "C" int eqd_server_poll(eqd_server *S, int64_t id, int32_t *done) {
    if (!S || !done) return fail(EQD_ERR_ARG, "invalid argument");
    std::lock_guard<std::mutex> lk(S->mu);
    SrvRequest *r = find_req(S, id);
    if (!r) return fail(EQD_ERR_ARG, "unknown request id");
    *done = r->state >= 2;
    if (r->state == 3) return fail(r->err, r->msg);
    return EQD_OK;
}

extern "C" int eqd_server_request_info(eqd_server *S, int64_t id, eqd_request_info *info) {
    if (!S || !info) return fail(EQD_ERR_ARG, "invalid argument");
    std::lock_guard<std::mutex> lk(S->mu);
    SrvRequest *r = find_req(S, id);
    if (!r) return fail(EQD_ERR_ARG, "unknown request id");
    info->state = r->state;
    info->ncols = r->ncols;
    info->unconverged = r->unconverged;
    info->max_iterations = r->max_it;
    info->iterations = r->iterations;
    info->t_submit = r->t_submit;
    info->t_start = r->t_start;
    info->t_done = r->t_done;
    return EQD_OK;
}

extern "C" int eqd_server_release(eqd_server *S, int64_t id) {
    if (!S) return fail(EQD_ERR_ARG, "null server");
    std::lock_guard<std::mutex> lk(S->mu);
    SrvRequest *r = find_req(S, id);
    if (!r) return fail(EQD_ERR_ARG, "unknown request id");
    if (r->state < 2) return fail(EQD_ERR_ARG, "request still in flight");
    S->reqs.erase(id);
    return EQD_OK;
}

extern "C" int eqd_server_destroy(eqd_server *S) {
    if (!S) return EQD_OK;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
    }
    S->cv_work.notify_all();
    for (auto &g : S->grids)
        if (g->worker.joinable()) g->worker.join();
    for (auto &g : S->grids) {
        cudaSetDevice(g->G->desc.device);
        cudaStreamSynchronize(g->G->stream);
        g->r32.reset();
        g->r64.reset();
        std::lock_guard<std::mutex> glk(g->G->mtx);
        g->G->served = false;
    }
    delete S;
    return EQD_OK;
}

// ---------------------------------------------------------------------------
// Time-loop right-hand side (eqd_rhs_*) and batched friction solves
// ---------------------------------------------------------------------------
struct eqd_rhs {
    int device = 0;
    int nf = 0;
    int nslice = 1;
    eqd_rhs_params p{};
    DevBuf K, part, u, du, ap_ptr, ap_idx, ap_val, source, active, vprev, tau, sigma_low, floor_nodes, floor_hits,
        status;
    cudaStream_t stream = nullptr;
};

static FrictionConst friction_const(const eqd_rhs_params &p) {
    return FrictionConst{p.a, p.b, p.Dc, p.V_star, p.f_star};
}

static bool newton_ok(const eqd_rhs_params &p) {
    return p.newton_tol > 0 && p.newton_maxiter > 0 && p.newton_maxstep > 0 && p.a > 0 && p.Dc > 0 && p.V_star > 0;
}

extern "C" int eqd_rhs_create(int32_t device, int32_t nf, const double *K, const eqd_rhs_params *params,
                              const int32_t *ap_ptr, const int32_t *ap_idx, const double *ap_val, const double *source,
                              const uint8_t *active, eqd_rhs **out) {
    if (!out || !K || !params || nf < 1 || !ap_ptr || (!ap_idx && ap_ptr[nf] > 0) || (!ap_val && ap_ptr[nf] > 0))
        return fail(EQD_ERR_ARG, "invalid argument");
    *out = nullptr;
    if (!newton_ok(*params)) return fail(EQD_ERR_ARG, "invalid friction or Newton parameters");
    if (params->injection == 1 && (params->well_cell < 0 || params->well_cell >= nf))
        return fail(EQD_ERR_ARG, "well_cell out of range");
    const int nnz = ap_ptr[nf];
    for (int i = 0; i < nf; ++i)
        if (ap_ptr[i + 1] < ap_ptr[i]) return fail(EQD_ERR_ARG, "Ap row pointers must be non-decreasing");
    for (int k = 0; k < nnz; ++k)
        if (ap_idx[k] < 0 || ap_idx[k] >= nf) return fail(EQD_ERR_ARG, "Ap column index out of range");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(EQD_ERR_NO_DEVICE, "no CUDA device visible");
    if (device < 0 || device >= ndev) return fail(EQD_ERR_ARG, "device ordinal out of range");
    CUDA_OR_RETURN(cudaSetDevice(device));
    std::unique_ptr<eqd_rhs> R(new eqd_rhs());
    R->device = device;
    R->nf = nf;
    R->p = *params;
    const long long n = 2LL * nf;
    R->nslice = gemv_slices((int)n);
    CUDA_OR_RETURN(cudaStreamCreateWithFlags(&R->stream, cudaStreamNonBlocking));
    CUDA_OR_RETURN(R->K.ensure(sizeof(double) * n * n));
    CUDA_OR_RETURN(R->part.ensure(sizeof(double) * n * R->nslice));
    CUDA_OR_RETURN(R->u.ensure(sizeof(double) * (4LL * nf + 1)));
    CUDA_OR_RETURN(R->du.ensure(sizeof(double) * (4LL * nf + 1)));
    CUDA_OR_RETURN(R->ap_ptr.ensure(sizeof(int) * (nf + 1)));
    CUDA_OR_RETURN(R->ap_idx.ensure(sizeof(int) * std::max(nnz, 1)));
    CUDA_OR_RETURN(R->ap_val.ensure(sizeof(double) * std::max(nnz, 1)));
    CUDA_OR_RETURN(R->source.ensure(sizeof(double) * nf));
    CUDA_OR_RETURN(R->active.ensure(nf));
    CUDA_OR_RETURN(R->vprev.ensure(sizeof(double) * nf));
    CUDA_OR_RETURN(R->tau.ensure(sizeof(double) * n));
    CUDA_OR_RETURN(R->sigma_low.ensure(sizeof(double) * nf));
    CUDA_OR_RETURN(R->floor_nodes.ensure(nf));
    CUDA_OR_RETURN(R->floor_hits.ensure(sizeof(unsigned long long)));
    CUDA_OR_RETURN(R->status.ensure(sizeof(unsigned)));
    cudaStream_t st = R->stream;
    CUDA_OR_RETURN(cudaMemcpyAsync(R->K.p, K, sizeof(double) * n * n, cudaMemcpyHostToDevice, st));
    CUDA_OR_RETURN(cudaMemcpyAsync(R->ap_ptr.p, ap_ptr, sizeof(int) * (nf + 1), cudaMemcpyHostToDevice, st));
    if (nnz > 0) {
        CUDA_OR_RETURN(cudaMemcpyAsync(R->ap_idx.p, ap_idx, sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
        CUDA_OR_RETURN(cudaMemcpyAsync(R->ap_val.p, ap_val, sizeof(double) * nnz, cudaMemcpyHostToDevice, st));
    }
    if (source) CUDA_OR_RETURN(cudaMemcpyAsync(R->source.p, source, sizeof(double) * nf, cudaMemcpyHostToDevice, st));
    else CUDA_OR_RETURN(cudaMemsetAsync(R->source.p, 0, sizeof(double) * nf, st));
    if (active) CUDA_OR_RETURN(cudaMemcpyAsync(R->active.p, active, nf, cudaMemcpyHostToDevice, st));
    else CUDA_OR_RETURN(cudaMemsetAsync(R->active.p, 1, nf, st));
    std::vector<double> init(nf, 1e-12), low(nf, INFINITY);
    CUDA_OR_RETURN(cudaMemcpyAsync(R->vprev.p, init.data(), sizeof(double) * nf, cudaMemcpyHostToDevice, st));
    CUDA_OR_RETURN(cudaMemcpyAsync(R->sigma_low.p, low.data(), sizeof(double) * nf, cudaMemcpyHostToDevice, st));
    CUDA_OR_RETURN(cudaMemsetAsync(R->floor_nodes.p, 0, nf, st));
    CUDA_OR_RETURN(cudaMemsetAsync(R->floor_hits.p, 0, sizeof(unsigned long long), st));
    CUDA_OR_RETURN(cudaMemsetAsync(R->tau.p, 0, sizeof(double) * n, st));
    CUDA_OR_RETURN(cudaStreamSynchronize(st));
    *out = R.release();
    return EQD_OK;
}

extern "C" int eqd_rhs_eval(eqd_rhs *R, double t, const double *u, double *du) {
    if (!R || !u || !du) return fail(EQD_ERR_ARG, "invalid argument");
    CUDA_OR_RETURN(cudaSetDevice(R->device));
    const int nf = R->nf;
    const long long nu = 4LL * nf + (R->p.injection == 1 ? 1 : 0);
    const long long n = 2LL * nf;
    cudaStream_t st = R->stream;
    CUDA_OR_RETURN(cudaMemcpyAsync(R->u.p, u, sizeof(double) * nu, cudaMemcpyHostToDevice, st));
    CUDA_OR_RETURN(cudaMemsetAsync(R->status.p, 0, sizeof(unsigned), st));
    dim3 g1((unsigned)(((n + 1) / 2 + 255) / 256), (unsigned)R->nslice);
    launch_gemv_partial(g1, st, R->K.as<double>(), R->u.as<double>(), n, R->nslice, 1, R->part.as<double>());
    RhsParams P{};
    P.fr = friction_const(R->p);
    P.sigma0 = R->p.sigma0;
    P.sigma_min = R->p.sigma_min;
    P.eta = R->p.eta;
    P.tau0_2 = R->p.tau0_2;
    P.tau0_3 = R->p.tau0_3;
    P.src_scale = t < R->p.t_off ? R->p.q0 / (R->p.beta * R->p.phi) : 0.0;
    P.tol = R->p.newton_tol;
    P.maxstep = R->p.newton_maxstep;
    P.maxiter = R->p.newton_maxiter;
    P.nf = nf;
    P.nslice = R->nslice;
    P.peaceman = R->p.injection == 1;
    P.well_cell = R->p.well_cell;
    P.WI = R->p.WI;
    P.S_e = R->p.S_e;
    P.S_well = R->p.S_well;
    P.Qinj = t < R->p.t_off ? R->p.Q0 : 0.0;
    rhs_node_kernel<<<(unsigned)((nf + 127) / 128), 128, 0, st>>>(
        P, R->part.as<double>(), R->u.as<double>(), R->du.as<double>(), R->ap_ptr.as<int>(), R->ap_idx.as<int>(),
        R->ap_val.as<double>(), R->source.as<double>(), R->active.as<unsigned char>(), R->vprev.as<double>(),
        R->tau.as<double>(), R->sigma_low.as<double>(), R->floor_nodes.as<unsigned char>(),
        R->floor_hits.as<unsigned long long>(), R->status.as<unsigned>());
    CUDA_OR_RETURN(cudaGetLastError());
    unsigned h = 0;
    CUDA_OR_RETURN(cudaMemcpyAsync(du, R->du.p, sizeof(double) * nu, cudaMemcpyDeviceToHost, st));
    CUDA_OR_RETURN(cudaMemcpyAsync(&h, R->status.p, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    CUDA_OR_RETURN(cudaStreamSynchronize(st));
    if (h & RHS_NEWTON_FAILED)
        return fail(EQD_ERR_NOT_CONVERGED, "solve_slip_rate did not converge at some fault node");
    return EQD_OK;
}

extern "C" int eqd_rhs_fields(eqd_rhs *R, double *tau, double *vprev) {
    if (!R) return fail(EQD_ERR_ARG, "invalid argument");
    CUDA_OR_RETURN(cudaSetDevice(R->device));
    if (tau)
        CUDA_OR_RETURN(cudaMemcpyAsync(tau, R->tau.p, sizeof(double) * 2 * R->nf, cudaMemcpyDeviceToHost, R->stream));
    if (vprev)
        CUDA_OR_RETURN(cudaMemcpyAsync(vprev, R->vprev.p, sizeof(double) * R->nf, cudaMemcpyDeviceToHost, R->stream));
    CUDA_OR_RETURN(cudaStreamSynchronize(R->stream));
    return EQD_OK;
}

extern "C" int eqd_rhs_report(eqd_rhs *R, double *sigma_lowest, int64_t *floor_hits, int32_t *floor_nodes) {
    if (!R) return fail(EQD_ERR_ARG, "invalid argument");
    CUDA_OR_RETURN(cudaSetDevice(R->device));
    std::vector<double> low(R->nf);
    std::vector<unsigned char> fn(R->nf);
    unsigned long long hits = 0;
    CUDA_OR_RETURN(cudaMemcpyAsync(low.data(), R->sigma_low.p, sizeof(double) * R->nf, cudaMemcpyDeviceToHost, R->stream));
    CUDA_OR_RETURN(cudaMemcpyAsync(fn.data(), R->floor_nodes.p, R->nf, cudaMemcpyDeviceToHost, R->stream));
    CUDA_OR_RETURN(cudaMemcpyAsync(&hits, R->floor_hits.p, sizeof(hits), cudaMemcpyDeviceToHost, R->stream));
    CUDA_OR_RETURN(cudaStreamSynchronize(R->stream));
    double m = INFINITY;
    int cnt = 0;
    for (int i = 0; i < R->nf; ++i) {
        m = std::min(m, low[i]);
        cnt += fn[i] != 0;
    }
    if (sigma_lowest) *sigma_lowest = m;
    if (floor_hits) *floor_hits = (int64_t)hits;
    if (floor_nodes) *floor_nodes = cnt;
    return EQD_OK;
}

extern "C" int eqd_rhs_destroy(eqd_rhs *R) {
    if (!R) return EQD_OK;
    cudaSetDevice(R->device);
    if (R->stream) {
        cudaStreamSynchronize(R->stream);
        cudaStreamDestroy(R->stream);
    }
    delete R;
    return EQD_OK;
}

extern "C" int eqd_friction_solve(int32_t device, int32_t n, const double *T, const double *theta, const double *sigma,
                                  double eta, const eqd_rhs_params *params, const double *V0, double *V) {
    if (n < 0 || (n > 0 && (!T || !theta || !sigma || !V)) || !params) return fail(EQD_ERR_ARG, "invalid argument");
    if (!newton_ok(*params)) return fail(EQD_ERR_ARG, "invalid friction or Newton parameters");
    if (n == 0) return EQD_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(EQD_ERR_NO_DEVICE, "no CUDA device visible");
    if (device < 0 || device >= ndev) return fail(EQD_ERR_ARG, "device ordinal out of range");
    CUDA_OR_RETURN(cudaSetDevice(device));
    DevBuf dT, dth, dsg, dv0, dV, dst;
    CUDA_OR_RETURN(dT.ensure(sizeof(double) * n));
    CUDA_OR_RETURN(dth.ensure(sizeof(double) * n));
    CUDA_OR_RETURN(dsg.ensure(sizeof(double) * n));
    CUDA_OR_RETURN(dV.ensure(sizeof(double) * n));
    CUDA_OR_RETURN(dst.ensure(sizeof(unsigned)));
    if (V0) CUDA_OR_RETURN(dv0.ensure(sizeof(double) * n));
    CUDA_OR_RETURN(cudaMemcpy(dT.p, T, sizeof(double) * n, cudaMemcpyHostToDevice));
    CUDA_OR_RETURN(cudaMemcpy(dth.p, theta, sizeof(double) * n, cudaMemcpyHostToDevice));
    CUDA_OR_RETURN(cudaMemcpy(dsg.p, sigma, sizeof(double) * n, cudaMemcpyHostToDevice));
    if (V0) CUDA_OR_RETURN(cudaMemcpy(dv0.p, V0, sizeof(double) * n, cudaMemcpyHostToDevice));
    CUDA_OR_RETURN(cudaMemset(dst.p, 0, sizeof(unsigned)));
    friction_solve_kernel<<<(unsigned)((n + 127) / 128), 128>>>(
        n, dT.as<double>(), dth.as<double>(), dsg.as<double>(), eta, friction_const(*params),
        V0 ? dv0.as<double>() : nullptr, params->newton_tol, params->newton_maxiter, params->newton_maxstep,
        dV.as<double>(), dst.as<unsigned>());
    CUDA_OR_RETURN(cudaGetLastError());
    unsigned h = 0;
    CUDA_OR_RETURN(cudaMemcpy(V, dV.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    CUDA_OR_RETURN(cudaMemcpy(&h, dst.p, sizeof(unsigned), cudaMemcpyDeviceToHost));
    if (h & RHS_NEWTON_FAILED)
        return fail(EQD_ERR_NOT_CONVERGED, "solve_slip_rate failed to converge");
    return EQD_OK;
}
