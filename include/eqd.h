/*
 * libeqd — B200 (sm_100a) fault-stiffness engine, C ABI.
 *
 * Drop-in for the dense fault-stiffness path of EarthquakeDiffinitive.jl:
 * one CG solve per unit-slip right-hand side on the split-node SBP-SAT
 * elastic operator A = -H P (D + SAT) P, assembled into K : [s2; s3] -> [dtau2; dtau3].
 * The Julia side binds these with `ccall`. All buffers in
 * the signatures are HOST memory owned by the caller; the library owns its
 * device memory. Matrices are column-major FP64, exactly the layout of the
 * reference's `Matrix{Float64}`.
 *
 * Conventions shared with the reference:
 *   - Omega_f nodes are ordered x2-fastest over an (n2f, n3f) grid
 *     (src/FaultResponse.jl:112-126).
 *   - K column c < nf is the response to unit s2 at node c, column nf + c to
 *     unit s3 at node c; rows 0..nf-1 are dtau2, nf..2nf-1 dtau3
 *     (src/FaultResponse.jl:249-255).
 *   - A "reference-layout" vector has Ntot = 6 n1 n2 n3 entries ordered
 *     [u1- u2- u3- u1+ u2+ u3+], each block x1-fastest
 *     (src/ElasticitySplitNode.jl:36-42).
 *
 * Every call returns an eqd_status; eqd_last_error() describes the last
 * failure on the calling thread.
 */
#ifndef EQD_H
#define EQD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    EQD_OK = 0,
    EQD_ERR_ARG = 1,          /* invalid argument (the reference's error() cases) */
    EQD_ERR_OOM = 2,          /* device allocation failed / over the HBM budget   */
    EQD_ERR_CUDA = 3,         /* CUDA runtime error                               */
    EQD_ERR_NOT_CONVERGED = 4,/* returned only when opts.flags has EQD_FLAG_STRICT */
    EQD_ERR_TIMEOUT = 5,      /* a device-side bounded wait gave up               */
    EQD_ERR_UNSUPPORTED = 6,
    EQD_ERR_NO_DEVICE = 7
} eqd_status;

/* Per-column solve outcome. */
typedef enum {
    EQD_COL_CONVERGED = 1,
    EQD_COL_MAXITER = 2,
    EQD_COL_BREAKDOWN = 3,    /* p.Ap <= eps |p|^2 (Krylov's zero curvature) */
    EQD_COL_NONFINITE = 4
} eqd_col_status;

typedef enum {
    EQD_PREC_FP64 = 0,        /* plain FP64 CG, Krylov.jl cg! rule (recursive residual) */
    EQD_PREC_MIXED = 1        /* FP32 CG with FP64 reliable updates; stops on the FP64 true residual */
} eqd_precision;

typedef enum { EQD_PRECOND_NONE = 0, EQD_PRECOND_JACOBI = 1 } eqd_precond;

#define EQD_FLAG_STRICT 1u    /* return EQD_ERR_NOT_CONVERGED if any column did not converge */
#define EQD_FLAG_NO_SPLIT 2u  /* run a large batch as one chain of kernels instead of two halves whose
                                 stencil applies alternate (for comparisons; results are identical) */
#define EQD_FLAG_FUSE 4u      /* form the CG direction p = r + beta p inside the stencil apply (from bulk
                                 copies of r and the previous p) instead of in its own kernel; results
                                 are identical. Off by default: the apply is instruction-issue bound,
                                 and the extra work there costs more than the separate memory-bound
                                 kernel, which overlaps the other half's apply. */

/*
 * Two equidistant blocks meeting at the fault plane x1 = 0:
 *   minus block x1 in [-x1_extent, 0], plus block x1 in [0, x1_extent],
 *   both x2 in [x2_lo, x2_hi], x3 in [x3_lo, x3_hi], n1 x n2 x n3 nodes each.
 * Replaces the grid pair built in `build_model` (src/BP8.jl:196-206) and the
 * `FaultElasticity(g_minus, g_plus, λ, μ, set; l_f)` constructor
 * (src/FaultResponse.jl:96-146): Omega_f = nodes with |x2|, |x3| <= l_f, which
 * must land exactly on grid nodes (same tolerance and error as the reference).
 */
typedef struct {
    int32_t n1, n2, n3;
    double x1_extent;
    double x2_lo, x2_hi, x3_lo, x3_hi;
    double lambda, mu;
    double l_f;
    int32_t order;            /* must be 4 (standard_diagonal.toml, order 4) */
    int32_t device;           /* CUDA device ordinal */
} eqd_grid_desc;

/* Mirrors `CGSolver(A; rtol=1e-10, atol=0.0, itmax=0, precond=:none)`
 * (src/ElasticitySplitNode.jl:365) plus the B200 engine's knobs. */
typedef struct {
    double rtol;              /* default 1e-10 */
    double atol;              /* default 0 */
    int64_t itmax;            /* 0 -> 2 Ntot, Krylov's default */
    int32_t precond;          /* eqd_precond */
    int32_t precision;        /* eqd_precision */
    int32_t chunk;            /* columns per device batch; 0 -> eqd_tune_chunk's choice if the grid was
                                 tuned, else as many as the HBM budget allows */
    double reliable_delta;    /* mixed: FP64 true-residual update when ||r|| drops by this factor (0 -> 0.01) */
    uint64_t hbm_budget_bytes;/* 0 -> free device memory minus 2 GiB */
    int32_t variant;          /* FP32 stencil launch variant for this call: 0 -> the grid's (chosen by
                                 eqd_autotune on first use, or pinned by eqd_set_variant); k > 0 ->
                                 variant k - 1 of eqd_autotune's list, for this call only */
    uint32_t flags;
} eqd_solve_opts;

/* Mirrors `CGStats` + `solver_report` (src/ElasticitySplitNode.jl:256-262, 442-447). */
typedef struct {
    int64_t solves;
    int64_t iterations;
    int64_t max_iterations;
    int64_t unconverged;
    int64_t reliable_updates; /* mixed precision only */
    double seconds;           /* wall time of the call */
    double device_seconds;    /* CUDA-event time of the solve loop */
    int32_t precond;
    int32_t precision;
    int64_t kernel_launches;  /* libeqd kernels launched by the call (graph nodes included) */
} eqd_stats;

typedef struct eqd_grid eqd_grid;
typedef struct eqd_kmat eqd_kmat;
typedef struct eqd_server eqd_server;

/* Library ------------------------------------------------------------------ */
const char *eqd_last_error(void);
const char *eqd_version(void);
void eqd_default_opts(eqd_solve_opts *opts);
int eqd_device_count(int32_t *count);

/* Grid (the FaultElasticity analogue) -------------------------------------- */
int eqd_grid_create(const eqd_grid_desc *desc, eqd_grid **out);
int eqd_grid_destroy(eqd_grid *grid);
/* ntot = 6 n1 n2 n3; nf = n2f * n3f (`frictional_node_count`, src/FaultResponse.jl:168). */
int eqd_grid_info(const eqd_grid *grid, int64_t *ntot, int32_t *nf, int32_t *n2f, int32_t *n3f);
/* Omega_f coordinates (`fault_grid_axes`, src/FaultResponse.jl:161). */
int eqd_grid_fault_axes(const eqd_grid *grid, double *x2f, double *x3f);

/* Operator hooks (test / adapter surface) ----------------------------------
 * x, y: ncols reference-layout vectors.
 * mode 0: y = A x          (A = -H P (D+SAT) P; `mul!(y, A, x)` on the
 *                            assembled matrix of src/ElasticitySplitNode.jl:211)
 * mode 1: y = HP_DSAT x    (= H P (D+SAT) x, the RHS operator of :210)
 * mode 2: y = A x for x already in range(P) (the kernel the CG iterations
 *         run; skips the input projection)
 * precision: EQD_PREC_FP64 or EQD_PREC_MIXED (FP32 arithmetic). */
int eqd_apply(eqd_grid *grid, const double *x, double *y, int32_t ncols, int32_t mode, int32_t precision);

/* `split_node_solve(solver, rhs)` (src/ElasticitySplitNode.jl:378-396) on the
 * matrix-free A: solves A u = rhs for ncols reference-layout right-hand
 * sides; iters/status per column (may be NULL). FP64 only. */
int eqd_cg_solve(eqd_grid *grid, const double *rhs, double *u, int32_t ncols, const eqd_solve_opts *opts,
                 int32_t *iters, int8_t *status, eqd_stats *stats);

/* `shear_traction(fe, s2, s3)` (src/FaultResponse.jl:194-211) for nslip slip
 * distributions: s2, s3, dtau2, dtau3 are nf x nslip, column-major. */
int eqd_shear_traction(eqd_grid *grid, const double *s2, const double *s3, int32_t nslip, double *dtau2,
                       double *dtau3, const eqd_solve_opts *opts, eqd_stats *stats);

/* `fault_stiffness(fe)` (src/FaultResponse.jl:229-287): the full 2nf x 2nf K
 * into the caller's buffer (>= 8 (2nf)^2 bytes). */
int eqd_stiffness_exact(eqd_grid *grid, const eqd_solve_opts *opts, double *K, eqd_stats *stats);

/* A subset of K's columns (0-based indices) into out (2nf x ncols);
 * iters / status per column may be NULL. Same column semantics as above. */
int eqd_stiffness_columns(eqd_grid *grid, const int32_t *cols, int32_t ncols, const eqd_solve_opts *opts,
                          double *out, int32_t *iters, int8_t *status, eqd_stats *stats);

/* Same as eqd_stiffness_columns, but `out_device` is a DEVICE pointer (on the
 * grid's device, 2nf x ncols FP64, column-major): K stays resident in HBM,
 * for device-side consumers (CuArray / torch). Returns when the columns are
 * written. */
int eqd_stiffness_columns_device(eqd_grid *grid, const int32_t *cols, int32_t ncols, const eqd_solve_opts *opts,
                                 double *out_device, int32_t *iters, int8_t *status, eqd_stats *stats);

/* `fault_stiffness_toeplitz(fe)` (src/FaultResponse.jl:339-393): 10 solves
 * (centre then the 4 corners, first source wins), expanded on the device. */
int eqd_stiffness_toeplitz(eqd_grid *grid, const eqd_solve_opts *opts, double *K, eqd_stats *stats);

/* Measurement hook: times `reps` launches of the stencil apply y = A x on
 * ncols device-resident random columns with CUDA events on the library's
 * stream (after `warmup` untimed launches). precision: EQD_PREC_MIXED (FP32)
 * or EQD_PREC_FP64. Writes the mean launch time (ms) and the algorithmic
 * bytes of one launch (2 * Ntot * sizeof(T) * ncols). */
int eqd_profile_apply(eqd_grid *grid, int32_t ncols, int32_t precision, int32_t warmup, int32_t reps,
                      double *ms_per_launch, double *bytes_per_launch);

/* Autotuner of the FP32 stencil launch configuration (x2 tile height, CTA
 * size, columns per thread, edge-partitioned tiles): times 20 mixed-precision
 * CG iterations of ncols unit-slip columns (<= 2nf) with every variant, keeps
 * the fastest for this grid (used by every later mixed-precision call) and
 * reports milliseconds per iteration. Arrays hold *nvariants (<= 16) entries.
 * ncols = 0 re-tunes nothing: it reports the current selection and the times
 * of the last tuning (zeros if the grid was never tuned). */
int eqd_autotune(eqd_grid *grid, int32_t ncols, int32_t *selected, double *ms_per_variant, int32_t *tile_rows,
                 int32_t *threads, int32_t *nvariants);

/* Chunk-width tuner (columns per batch): times 20 mixed-precision CG
 * iterations of `widths[k]` unit-slip columns for each width, writes the cost
 * of one column-iteration (ms; -1 for a width above 2nf or the HBM budget)
 * and the cheapest width, which later calls with opts.chunk = 0 use. */
int eqd_tune_chunk(eqd_grid *grid, const int32_t *widths, int32_t nwidths, double *ms_per_column_iteration,
                   int32_t *best);

/* Pins the FP32 stencil launch variant (0 .. *nvariants-1 of eqd_autotune)
 * for this grid instead of autotuning (reproducibility across processes). */
int eqd_set_variant(eqd_grid *grid, int32_t variant);

/* Failure-path test hook (no counterpart in the reference): the next FP32
 * stencil apply of this grid (its selected variant must be a ring-march
 * variant) never issues the copy of x3 plane `plane` and gives every bounded
 * wait `poll_limit` polls. The waits on that plane give up, the kernel drains
 * its other copies and returns, and the call that launched it returns
 * EQD_ERR_TIMEOUT; later calls run normally. One launch only. */
int eqd_test_inject_wait_timeout(eqd_grid *grid, int32_t plane, uint32_t poll_limit);

/* The assembled matrices of `split_node_system` (src/ElasticitySplitNode.jl:
 * 106-214) for callers that want them: which = 0 gives A = -H P (D+SAT) P,
 * which = 1 gives HP_DSAT = H P (D+SAT), CSR in reference DOF order (ntot
 * rows, 0-based, columns ascending), built on the GPU by coloured probing with
 * the FP64 operator kernels (no Julia-side assembly). Holds the numerically
 * nonzero entries: entries below 1e-12 of their row's largest (the rounding
 * of exactly cancelling terms, and the explicit zeros of the reference's
 * structural pattern) are left out. With indptr, indices and values all NULL
 * only *nnz is set; otherwise indptr holds ntot + 1 entries and indices and
 * values `capacity` >= *nnz entries (EQD_ERR_ARG with *nnz set when smaller). */
int eqd_assemble(eqd_grid *grid, int32_t which, int64_t capacity, int64_t *indptr, int32_t *indices,
                 double *values, int64_t *nnz);

/* Jacobi diagonal, `diag(A)` (src/ElasticitySplitNode.jl:352-357), reference layout. */
int eqd_diag(eqd_grid *grid, double *d);

/* Time-loop GEMV `mul!(Δτ, K, slip)` (src/BP8.jl:366) ----------------------
 * K stays resident on the device; y = K s for nvec vectors (n x nvec each,
 * column-major), any n >= 1. From 3 vectors on, K S runs blocked on the FP64
 * tensor cores (K read once per 64 vectors); fewer run as the GEMV. s and y
 * are host arrays; the call copies them and returns when y is written. */
int eqd_kmat_create(int32_t device, int32_t n, const double *K, eqd_kmat **out);
int eqd_kmat_gemv(eqd_kmat *kmat, const double *s, double *y, int32_t nvec);
/* The same y = K s with s and y DEVICE pointers (8-byte aligned, on the
 * kmat's device) for callers whose slip vectors are already resident, e.g.
 * Runge-Kutta stages of a time loop on the GPU (no counterpart in the
 * reference, which multiplies host arrays). Launches on `stream` (a
 * cudaStream_t, NULL = default stream) and returns without synchronizing.
 * Partial sums live in scratch owned by the kmat: calls on one kmat must be
 * serialised (one stream, or events), and the first call with a given n * nvec
 * may allocate it (make that call before any stream capture). */
int eqd_kmat_gemv_device(eqd_kmat *kmat, const double *s_device, double *y_device, int32_t nvec, void *stream);
int eqd_kmat_destroy(eqd_kmat *kmat);

/* Allocation-free y = K s (no counterpart in the reference: an addition for
 * callers that cannot allocate device memory, e.g. a time loop inside CUDA
 * graph capture or under a framework's own allocator). K (n x n, column-major),
 * s and y (n x nvec) are DEVICE pointers owned by the caller, on `device`;
 * any n >= 1 and any 8-byte-aligned K (16-byte loads are used only when K is
 * 16-byte aligned and n is even). Scratch is a static 4 MiB array per device:
 * n * nvec must not exceed 524,288 (EQD_ERR_ARG otherwise). The first call on
 * a device looks the array's address up and caches it for the life of the
 * process (make that call before any stream capture; the cached address does
 * not survive a reset of the device's primary context, e.g. cudaDeviceReset).
 * Launches on `stream` (a cudaStream_t, NULL = default stream) and returns
 * without synchronizing. All calls on a device share the scratch array:
 * serialise them (one stream, or events); calls that overlap on the GPU race. */
int eqd_kmat_gemv_static(int32_t device, int32_t n, const double *K_device, const double *s_device,
                         double *y_device, int32_t nvec, void *stream);

/* Time-loop right-hand side of the coupled BP8 model -----------------------
 * `rhs!(du, u, m, t)` / `evaluate!(m, u, t)` (src/BP8.jl:356-433) with K
 * resident on the GPU: Δτ = K·[s2; s3] (the GEMV), the slip velocity from
 * the radiation-damped rate-and-state force balance per fault node
 * (`solve_slip_velocity`, src/RateStateFriction.jl:77-117: Newton in ln V,
 * steps clamped to newton_maxstep, warm-started from the previous slip
 * rate), the aging law in φ = ln θ, and the pore-pressure equation
 * dp/dt = Ap·p + injection with the caller's sparse Ap (CSR, 0-based).
 * State u = [s2; s3; φ; p] (4nf), plus the well pressure for the Peaceman
 * well (4nf + 1); du has the same layout. */
typedef struct {
    double a, b, Dc, V_star, f_star;   /* FrictionParams (Dc = D_RS) */
    double sigma0, sigma_min;          /* effective normal stress and its floor (Pa) */
    double eta;                        /* radiation damping mu / (2 c_s) */
    double tau0_2, tau0_3;             /* background shear traction (Pa) */
    double q0, beta, phi, t_off;       /* Gaussian source: q0 / (beta phi) * source while t < t_off */
    int32_t injection;                 /* 0 Gaussian source, 1 Peaceman well */
    int32_t well_cell;                 /* 0-based node of the well */
    double WI, S_e, S_well, Q0;        /* Peaceman well */
    double newton_tol;                 /* 1e-12 */
    double newton_maxstep;             /* 5.0 */
    int32_t newton_maxiter;            /* 50 */
    int32_t pad_;
} eqd_rhs_params;

typedef struct eqd_rhs eqd_rhs;

/* K: 2nf x 2nf column-major (host); Ap: nf x nf CSR (ap_ptr[nf+1], ap_idx,
 * ap_val); source (nf, Gaussian injection) and active (nf, 0 = locked node)
 * may be NULL (zeros / all active). */
int eqd_rhs_create(int32_t device, int32_t nf, const double *K, const eqd_rhs_params *params, const int32_t *ap_ptr,
                   const int32_t *ap_idx, const double *ap_val, const double *source, const uint8_t *active,
                   eqd_rhs **out);
/* du = rhs(u, t) (host arrays). EQD_ERR_NOT_CONVERGED if a Newton solve did
 * not converge (the reference throws). */
int eqd_rhs_eval(eqd_rhs *rhs, double t, const double *u, double *du);
/* The cache fields of the last evaluation: shear stress acting on the fault
 * tau (2nf: τ2 then τ3) and the warm-start slip rate Vprev (nf); either may
 * be NULL. */
int eqd_rhs_fields(eqd_rhs *rhs, double *tau, double *vprev);
/* `effective_stress_report` inputs: lowest σ̄ = σ0 - p seen before the floor,
 * how many node evaluations hit the floor, and how many nodes ever did. */
int eqd_rhs_report(eqd_rhs *rhs, double *sigma_lowest, int64_t *floor_hits, int32_t *floor_nodes);
int eqd_rhs_destroy(eqd_rhs *rhs);

/* `solve_slip_rate` for n independent nodes (src/RateStateFriction.jl:77-100):
 * V[i] solves T = eta V + sigma a asinh(V/(2V*) C(theta)), seeded from V0[i]
 * (NULL: V*). Uses the friction and Newton fields of `params`. */
int eqd_friction_solve(int32_t device, int32_t n, const double *T, const double *theta, const double *sigma,
                       double eta, const eqd_rhs_params *params, const double *V0, double *V);

/* Serving: stiffness-column requests answered by continuous batching -------
 * The reference builds K in one blocking call (`fault_stiffness`,
 * src/FaultResponse.jl:229-287, its column loop `run_columns!` :244-263).
 * The server answers requests for subsets of K's columns on several grids as
 * they arrive: each attached grid keeps a pool of CG slots (operator tables,
 * Krylov vectors and per-column state resident in HBM); a request's columns
 * enter free slots as earlier columns finish, beside the columns of other
 * requests on the same grid; grids run concurrently on their own streams.
 * A column's result does not depend on what else is in flight. */
typedef struct {
    int32_t state;            /* 0 queued, 1 running, 2 done, 3 failed */
    int32_t ncols;
    int32_t unconverged;
    int32_t max_iterations;
    int64_t iterations;       /* sum over the request's columns */
    double t_submit;          /* seconds on the server clock */
    double t_start;           /* first column entered a slot */
    double t_done;            /* last column extracted */
} eqd_request_info;

/* `opts` fixes the solver for every grid (NULL: defaults); the slot pools of
 * all grids together stay within `hbm_budget_bytes` (0: free memory - 2 GiB). */
int eqd_server_create(const eqd_solve_opts *opts, uint64_t hbm_budget_bytes, eqd_server **out);
/* Attach a grid with `slots` CG slots (0: as many as the remaining budget
 * allows, at most 512). The grid then belongs to the server until
 * eqd_server_destroy: other calls on it fail with EQD_ERR_ARG. */
int eqd_server_add_grid(eqd_server *server, eqd_grid *grid, int32_t slots);
/* Queue K columns `cols` (0-based, < 2nf) of an attached grid; the result,
 * 2nf x ncols column-major FP64, goes to the caller-owned host buffer `k_out`,
 * which must stay valid until the request is done. */
int eqd_server_submit(eqd_server *server, eqd_grid *grid, const int32_t *cols, int32_t ncols, double *k_out,
                      int64_t *request_id);
/* Block until the request is done (EQD_OK), failed (its error), or
 * `timeout_s` passed (EQD_ERR_TIMEOUT; the request keeps running). */
int eqd_server_wait(eqd_server *server, int64_t request_id, double timeout_s);
int eqd_server_poll(eqd_server *server, int64_t request_id, int32_t *done);
int eqd_server_request_info(eqd_server *server, int64_t request_id, eqd_request_info *info);
/* Forget a finished request (its id becomes invalid). */
int eqd_server_release(eqd_server *server, int64_t request_id);
/* Stops the worker at the end of its current iteration; requests not yet done
 * are abandoned. Attached grids return to their owner. */
int eqd_server_destroy(eqd_server *server);

#ifdef __cplusplus
}
#endif

#endif /* EQD_H */
