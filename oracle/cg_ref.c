/*
 * CPU restatement of the reference's exact fault-stiffness column loop.
 *
 * TEST INFRASTRUCTURE: part of the oracle. Only tests and the CPU-baseline
 * leg of bench.py load this library, as the checker / the timed baseline.
 *
 * Restates, on the assembled CSR matrices the Python oracle builds:
 *   fault_stiffness / run_columns!   src/FaultResponse.jl:229-287
 *       (strided thread partition t:nt:ncols, one solver per thread, :265-281)
 *   shear_traction!                  src/FaultResponse.jl:201-211
 *   build_chi!                       src/FaultResponse.jl:176-185
 *   split_node_solve -> Krylov.cg!   src/ElasticitySplitNode.jl:378-396
 *       (Krylov.jl 0.10.9 rule: x0 = 0, stop when ||r_k|| <= atol + rtol*||b||
 *        on the recursive residual, itmax = 0 -> 2n)
 * in plain C with OpenMP threads over columns.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
    int64_t nrows;
    const int64_t *indptr;
    const int32_t *indices;
    const double *data;
} csr_t;

static void spmv(const csr_t *M, const double *x, double *y) {
    for (int64_t i = 0; i < M->nrows; ++i) {
        double s = 0.0;
        for (int64_t k = M->indptr[i]; k < M->indptr[i + 1]; ++k)
            s += M->data[k] * x[M->indices[k]];
        y[i] = s;
    }
}

static double dot(int64_t n, const double *a, const double *b) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* Krylov-rule CG from x0 = 0. Returns iterations; *solved set. */
static int64_t cg(const csr_t *A, const double *b, double *x, double *r, double *p,
                  double *Ap, double rtol, double atol, int64_t itmax, int *solved) {
    int64_t n = A->nrows;
    memset(x, 0, sizeof(double) * n);
    memcpy(r, b, sizeof(double) * n);
    memcpy(p, b, sizeof(double) * n);
    double gamma = dot(n, r, r);
    if (gamma == 0.0) { *solved = 1; return 0; }
    double rnorm = sqrt(gamma);
    double eps = atol + rtol * rnorm;
    if (itmax == 0) itmax = 2 * n;
    int64_t it = 0;
    int ok = rnorm <= eps;
    while (!(ok || it >= itmax)) {
        spmv(A, p, Ap);
        double pAp = dot(n, p, Ap);
        if (pAp <= DBL_EPSILON * dot(n, p, p)) break;
        double alpha = gamma / pAp;
        for (int64_t i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * Ap[i]; }
        double gnext = dot(n, r, r);
        rnorm = sqrt(gnext);
        ++it;
        ok = rnorm <= eps;
        if (!ok) {
            double beta = gnext / gamma;
            for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
        }
        gamma = gnext;
    }
    *solved = ok;
    return it;
}

/*
 * Computes the K columns `cols` (0-based; c < nf is unit s2 at Omega_f node c,
 * otherwise unit s3 at node c - nf) into out (2nf x ncols, column-major).
 * chi_rows / chi_rows_plus are nf x 2 row-major (component 2, 3).
 * nthreads <= 0 uses the OpenMP default.
 */
int eqdref_stiffness_columns(
    int64_t ntot,
    const int64_t *A_ip, const int32_t *A_ix, const double *A_v,
    const int64_t *B_ip, const int32_t *B_ix, const double *B_v,
    const int64_t *P_ip, const int32_t *P_ix, const double *P_v,
    int64_t nb,
    const int64_t *T2_ip, const int32_t *T2_ix, const double *T2_v,
    const int64_t *T3_ip, const int32_t *T3_ix, const double *T3_v,
    int32_t nf, const int64_t *chi_rows, const int64_t *chi_rows_plus, const int64_t *omega,
    int32_t ncols, const int32_t *cols, double rtol, double atol, int64_t itmax,
    int32_t nthreads, double *out, int64_t *iters, int8_t *solved) {
    csr_t A = {ntot, A_ip, A_ix, A_v}, B = {ntot, B_ip, B_ix, B_v}, P = {ntot, P_ip, P_ix, P_v};
    csr_t T2 = {nb, T2_ip, T2_ix, T2_v}, T3 = {nb, T3_ip, T3_ix, T3_v};
    int nt = 1;
#ifdef _OPENMP
    nt = nthreads > 0 ? nthreads : omp_get_max_threads();
    if (nt > ncols) nt = ncols > 0 ? ncols : 1;
#endif
    int err = 0;
#pragma omp parallel num_threads(nt) reduction(|:err)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        double *buf = (double *)malloc(sizeof(double) * (8 * ntot + 2 * nb));
        if (!buf) { err = 1; } else {
            double *chi = buf, *b = chi + ntot, *x = b + ntot, *r = x + ntot, *p = r + ntot,
                   *Ap = p + ntot, *U = Ap + ntot, *tmp = U + ntot, *t2 = tmp + ntot, *t3 = t2 + nb;
            for (int32_t j = t; j < ncols; j += nt) {   /* strided, as the reference */
                int32_t col = cols[j];
                memset(chi, 0, sizeof(double) * ntot);
                int comp = col < nf ? 0 : 1;
                int32_t k = col < nf ? col : col - nf;
                chi[chi_rows[2 * k + comp]] = -0.5;
                chi[chi_rows_plus[2 * k + comp]] = 0.5;
                spmv(&B, chi, b);
                int ok = 0;
                int64_t it = cg(&A, b, x, r, p, Ap, rtol, atol, itmax, &ok);
                spmv(&P, x, tmp);
                for (int64_t i = 0; i < ntot; ++i) U[i] = tmp[i] + chi[i];
                spmv(&T2, U, t2);
                spmv(&T3, U, t3);
                for (int32_t q = 0; q < nf; ++q) {
                    out[(int64_t)j * 2 * nf + q] = t2[omega[q]];
                    out[(int64_t)j * 2 * nf + nf + q] = t3[omega[q]];
                }
                iters[j] = it;
                solved[j] = (int8_t)ok;
            }
            free(buf);
        }
    }
    return err;
}

int eqdref_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
