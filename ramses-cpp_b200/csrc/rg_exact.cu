// rg_exact.cu -- batched exact Riemann solves, the stress workload and the
// training data of the learned Newton start (rg_mlp.cuh).
//
// The exact solver is RiemannSolver::solve_godunov_nr of RAMSES-CPP
// (src/solvers/hydro/RiemannSolver.cpp:194-307), in rg_physics.cuh.  Two modes:
// the reference's (10 iterations, |dp/(p+1e-10)| < 1e-6) and a converged one
// (tolerance 1e-14, larger iteration cap) in which the learned guess is judged:
// it must reach the same root with fewer Newton updates.
#include <cstdint>

#include "rg_face.cuh"
#include "rg_mlp.cuh"

namespace rg {

namespace {

// counter-based uniform doubles in [0, 1): splitmix64 of (seed, index, draw)
__device__ __forceinline__ double urand(unsigned long long seed, unsigned long long i, int k) {
    unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (i * 16ULL + (unsigned long long)k + 1ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// Stress workload of the exact solver: density ratio log-uniform up to 1e4,
// pressure ratio up to 1e6, 30 % strong double rarefactions (u_L < 0 < u_R with
// a jump from 0.2 to 1.5 times the vacuum-generating 2 (c_L + c_R)/(gamma-1)),
// the rest with velocities uniform in [-3, 3]; gamma 5/3 or 1.4.  Rotated
// primitive layout [ndim+2][n]: rho, u_n, u_t..., p.
template <int NDIM>
__global__ void k_stress_states(int n, unsigned long long seed, double* ql, double* qr, double* gam) {
    constexpr int NV = NDIM + 2, IP = NDIM + 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double g = urand(seed, i, 0) < 0.5 ? 5.0 / 3.0 : 1.4;
        double rl = pow(10.0, -2.0 + 4.0 * urand(seed, i, 1));
        double rr = rl * pow(10.0, -4.0 + 8.0 * urand(seed, i, 2)) ;
        double pl = pow(10.0, -3.0 + 6.0 * urand(seed, i, 3));
        double pr = pl * pow(10.0, -6.0 + 12.0 * urand(seed, i, 4));
        // keep both states inside log-uniform [1e-4,1e4] rho, [1e-6,1e6] p
        rr = fmin(fmax(rr, 1e-4), 1e4);
        pr = fmin(fmax(pr, 1e-6), 1e6);
        double ul, ur;
        if (urand(seed, i, 5) < 0.3) {
            double cl = sqrt(g * pl / rl), cr = sqrt(g * pr / rr);
            double du = (0.2 + 1.3 * urand(seed, i, 6)) * 2.0 * (cl + cr) / (g - 1.0);
            double f = 0.2 + 0.6 * urand(seed, i, 7);
            ul = -f * du;
            ur = (1.0 - f) * du;
        } else {
            ul = -3.0 + 6.0 * urand(seed, i, 6);
            ur = -3.0 + 6.0 * urand(seed, i, 7);
        }
        ql[i] = rl;
        qr[i] = rr;
        ql[(size_t)n + i] = ul;
        qr[(size_t)n + i] = ur;
        for (int d = 2; d <= NDIM; ++d) {
            ql[(size_t)d * n + i] = -1.0 + 2.0 * urand(seed, i, 6 + 2 * d);
            qr[(size_t)d * n + i] = -1.0 + 2.0 * urand(seed, i, 7 + 2 * d);
        }
        ql[(size_t)IP * n + i] = pl;
        qr[(size_t)IP * n + i] = pr;
        if (gam) gam[i] = g;
        (void)NV;
    }
}

// LEARNED: the network may be evaluated (out of line; it needs registers), so
// fewer resident blocks; the plain start keeps more warps in flight.
template <int NDIM, bool LEARNED>
__global__ void __launch_bounds__(256, LEARNED ? 2 : 4) k_exact_batch(int n, const double* __restrict__ ql, const double* __restrict__ qr,
                              const double* __restrict__ gam, double gamma0, double* flux, double* pstar, int* iters,
                              const float* __restrict__ mlp, int niter, double tol, DevStatus* st) {
    constexpr int NV = NDIM + 2;
    unsigned long long it_sum = 0, calls = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double a[NV], b[NV], f[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            a[v] = ql[(size_t)v * n + i];
            b[v] = qr[(size_t)v * n + i];
        }
        double gamma = gam ? gam[i] : gamma0;
        double smallp = 1e-10 * 1e-10 / gamma;
        double guess = LEARNED ? mlp_guess<NDIM>(mlp, a, b, gamma, smallp) : -1.0;
        double ps;
        int it = solve_exact_p<NDIM>(a, b, f, gamma, smallp, niter, tol, guess, &ps);
        if (flux) {
#pragma unroll
            for (int v = 0; v < NV; ++v) flux[(size_t)v * n + i] = f[v];
        }
        if (pstar) pstar[i] = ps;
        if (iters) iters[i] = it;
        it_sum += it;
        ++calls;
    }
    for (int o = 16; o > 0; o >>= 1) {
        it_sum += __shfl_xor_sync(0xffffffffu, it_sum, o);
        calls += __shfl_xor_sync(0xffffffffu, calls, o);
    }
    if ((threadIdx.x & 31) == 0 && calls) {
        atomicAdd(&st->exact_iters, it_sum);
        atomicAdd(&st->exact_calls, calls);
    }
}

// raw features [IN][n] and targets [n] = log(max(p*, 1e-30 pref) / base)
template <int NDIM>
__global__ void k_features(int n, const double* __restrict__ ql, const double* __restrict__ qr,
                           const double* __restrict__ gam, double gamma0, const double* __restrict__ pstar,
                           float* X, float* T) {
    constexpr int NV = NDIM + 2;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double a[NV], b[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            a[v] = ql[(size_t)v * n + i];
            b[v] = qr[(size_t)v * n + i];
        }
        double gamma = gam ? gam[i] : gamma0;
        float x[MLP_IN];
        double pref, base;
        mlp_features<NDIM>(a, b, gamma, 1e-10 * 1e-10 / gamma, x, &pref, &base);
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) X[(size_t)k * n + i] = x[k];
        if (T) T[i] = (float)log(smax(pstar[i], 1e-30 * pref) / base);
    }
}

inline int blocks_for(rg_ctx* c, long long n) {
    long long b = (n + 255) / 256, cap = (long long)c->sm_count * 16;
    return (int)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace

int launch_stress_states(rg_ctx* c, int n, unsigned long long seed, double* ql, double* qr, double* gam) {
    if (c->params.ndim == 1) k_stress_states<1><<<blocks_for(c, n), 256, 0, c->stream>>>(n, seed, ql, qr, gam);
    else k_stress_states<3><<<blocks_for(c, n), 256, 0, c->stream>>>(n, seed, ql, qr, gam);
    return check_cuda(c, cudaGetLastError(), "stress states");
}

int launch_exact_batch(rg_ctx* c, int n, const double* ql, const double* qr, const double* gam, double* flux,
                       double* pstar, int* iters, const float* mlp, int niter, double tol) {
    if (c->params.ndim == 1)
        if (mlp)
            k_exact_batch<1, true><<<blocks_for(c, n), 256, 0, c->stream>>>(n, ql, qr, gam, c->params.gamma, flux,
                                                                            pstar, iters, mlp, niter, tol, c->d_status);
        else
            k_exact_batch<1, false><<<blocks_for(c, n), 256, 0, c->stream>>>(n, ql, qr, gam, c->params.gamma, flux,
                                                                             pstar, iters, mlp, niter, tol, c->d_status);
    else
        if (mlp)
            k_exact_batch<3, true><<<blocks_for(c, n), 256, 0, c->stream>>>(n, ql, qr, gam, c->params.gamma, flux,
                                                                            pstar, iters, mlp, niter, tol, c->d_status);
        else
            k_exact_batch<3, false><<<blocks_for(c, n), 256, 0, c->stream>>>(n, ql, qr, gam, c->params.gamma, flux,
                                                                             pstar, iters, mlp, niter, tol, c->d_status);
    return check_cuda(c, cudaGetLastError(), "exact batch");
}

int launch_features(rg_ctx* c, int n, const double* ql, const double* qr, const double* gam, const double* pstar,
                    float* X, float* T) {
    if (c->params.ndim == 1)
        k_features<1><<<blocks_for(c, n), 256, 0, c->stream>>>(n, ql, qr, gam, c->params.gamma, pstar, X, T);
    else
        k_features<3><<<blocks_for(c, n), 256, 0, c->stream>>>(n, ql, qr, gam, c->params.gamma, pstar, X, T);
    return check_cuda(c, cudaGetLastError(), "features");
}

}  // namespace rg
