// Time-loop right-hand side of the coupled BP8 model on the GPU: the slip
// velocity from the radiation-damped rate-and-state force balance, the aging
// law, and the pore-pressure equation, fused behind the K s GEMV.
//
//   Newton in x = ln V for  T = eta V + sigma a asinh(V/(2V*) C),
//   C = exp((f* + b ln(V* theta / Dc)) / a)       (src/RateStateFriction.jl:77-100)
//   V = V(|tau0 + dtau|) (tau0 + dtau) / |tau0 + dtau|          (:109-117)
//   du = [V2; V3; exp(-phi) - |V| / Dc; Ap p + injection]       (src/BP8.jl:356-433)
#pragma once
#include "solver_kernels.cuh"

namespace eqd {

struct FrictionConst {
    double a, b, Dc, V_star, f_star;
};

// Status bits reported by the RHS kernels.
enum : unsigned { RHS_NEWTON_FAILED = 1u };

// Newton in log space with clamped steps; returns false if it did not
// converge within maxiter (V holds the last iterate).
__device__ __forceinline__ bool slip_rate_newton(double T, double theta, double sigma, double eta,
                                                 const FrictionConst &p, double V0, double tol, int maxiter,
                                                 double maxstep, double &V) {
    const double C = exp((p.f_star + p.b * log(p.V_star * theta / p.Dc)) / p.a);
    double x = log(V0);
    for (int it = 0; it < maxiter; ++it) {
        const double v = exp(x);
        const double u = v / (2.0 * p.V_star) * C;
        const double g = eta * v + sigma * p.a * asinh(u) - T;
        const double dg = eta * v + sigma * p.a * u / sqrt(1.0 + u * u);
        const double dx = fmin(fmax(-g / dg, -maxstep), maxstep);
        x += dx;
        if (fabs(dx) < tol) {
            V = exp(x);
            return true;
        }
    }
    V = exp(x);
    return false;
}

// Batch of independent scalar solves (test hook and building block).
__global__ void friction_solve_kernel(int n, const double *__restrict__ T, const double *__restrict__ theta,
                                      const double *__restrict__ sigma, double eta, FrictionConst p,
                                      const double *__restrict__ V0, double tol, int maxiter, double maxstep,
                                      double *__restrict__ V, unsigned *__restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double v = 0.0;
    const bool ok = slip_rate_newton(T[i], theta[i], sigma[i], eta, p, V0 ? V0[i] : p.V_star, tol, maxiter,
                                     maxstep, v);
    V[i] = v;
    if (!ok) atomicOr(status, RHS_NEWTON_FAILED);
}

struct RhsParams {
    FrictionConst fr;
    double sigma0, sigma_min, eta, tau0_2, tau0_3;
    double src_scale;   // q0 / (beta phi) while t < t_off, else 0 (Gaussian source)
    double tol, maxstep;
    int maxiter;
    int nf, nslice;
    int peaceman;       // 1: Peaceman well at well_cell; 0: Gaussian source
    int well_cell;
    double WI, S_e, S_well, Qinj;
};

// One thread per fault node: finish the GEMV (fixed-order sum over column
// slices, as gemv_reduce_kernel), solve the force balance, aging law, and
// the node's row of the pore-pressure equation (CSR SpMV).
__global__ void rhs_node_kernel(RhsParams P, const double *__restrict__ part, const double *__restrict__ u,
                                double *__restrict__ du, const int *__restrict__ ap_ptr,
                                const int *__restrict__ ap_idx, const double *__restrict__ ap_val,
                                const double *__restrict__ source, const unsigned char *__restrict__ active,
                                double *__restrict__ Vprev, double *__restrict__ tau, double *__restrict__ sigma_low,
                                unsigned char *__restrict__ floor_nodes, unsigned long long *__restrict__ floor_hits,
                                unsigned *__restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nf = P.nf;
    if (i >= nf) return;
    const long long n = 2LL * nf;
    double d2 = 0.0, d3 = 0.0;
    for (int t = 0; t < P.nslice; ++t) {
        d2 += part[(long long)t * n + i];
        d3 += part[(long long)t * n + nf + i];
    }
    const double *phi = u + 2LL * nf;
    const double *pres = u + 3LL * nf;
    double V2 = 0.0, V3 = 0.0, Vm = 0.0;
    const double T2 = P.tau0_2 + d2, T3 = P.tau0_3 + d3;
    if (active[i]) {
        const double sraw = P.sigma0 - pres[i];
        if (sraw < sigma_low[i]) sigma_low[i] = sraw;
        if (sraw < P.sigma_min) {
            atomicAdd(floor_hits, 1ull);
            floor_nodes[i] = 1;
        }
        const double sigma = fmax(sraw, P.sigma_min);
        const double theta = exp(phi[i]);
        const double T = sqrt(T2 * T2 + T3 * T3);
        if (T != 0.0) {
            double v = 0.0;
            if (!slip_rate_newton(T, theta, sigma, P.eta, P.fr, Vprev[i], P.tol, P.maxiter, P.maxstep, v))
                atomicOr(status, RHS_NEWTON_FAILED);
            V2 = v * T2 / T;
            V3 = v * T3 / T;
            Vm = sqrt(V2 * V2 + V3 * V3);
        }
        Vprev[i] = fmax(Vm, 1e-30);
    }
    du[i] = V2;
    du[nf + i] = V3;
    du[2LL * nf + i] = exp(-phi[i]) - Vm / P.fr.Dc;
    tau[i] = T2 - P.eta * V2;
    tau[nf + i] = T3 - P.eta * V3;
    double dp = 0.0;
    for (int k = ap_ptr[i]; k < ap_ptr[i + 1]; ++k) dp += ap_val[k] * pres[ap_idx[k]];
    if (!P.peaceman) {
        dp += P.src_scale * source[i];
    } else if (i == P.well_cell) {
        const double transfer = P.WI * (u[4LL * nf] - pres[i]);
        dp += transfer / P.S_e;
        du[4LL * nf] = (P.Qinj - transfer) / P.S_well;
    }
    du[3LL * nf + i] = dp;
}

}  // namespace eqd
