// rg_exact.cu -- batched exact Riemann solves, the stress workload and the
// training data of the learned Newton start (rg_mlp.cuh).
//
// The exact solver is RiemannSolver::solve_godunov_nr of RAMSES-CPP
// (src/solvers/hydro/RiemannSolver.cpp:194-307), in rg_physics.cuh.  Two modes:
// the reference's (10 iterations, |dp/(p+1e-10)| < 1e-6) and a converged one
// (tolerance 1e-14, larger iteration cap) in which the learned guess is evaluated:
// it must reach the same root with fewer Newton updates.
#include <algorithm>
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

// Exact solves of a batch; guess_in: per-interface Newton starts (-1: the
// two-shock start; k_mlp_guess_tc writes them), or null for the two-shock
// start everywhere.
template <int NDIM>
__global__ void __launch_bounds__(256, 4) k_exact_batch(int n, const double* __restrict__ ql, const double* __restrict__ qr,
                              const double* __restrict__ gam, double gamma0, double* flux, double* pstar, int* iters,
                              int niter, double tol, DevStatus* st, const double* __restrict__ guess_in) {
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
        double guess = guess_in ? guess_in[i] : -1.0;
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

// Learned starts for a batch, the network on the tensor cores.  A warp takes
// 32 interfaces (one per lane) and evaluates the network for all of them at
// once with mma.sync m16n8k16 (two 16-row tiles; BF16 operands, FP32
// accumulation) with the roundings of the training forward pass (rg_mlp.cu:
// features and H1 rounded to BF16 where they enter a product, W1 and W2
// rounded from the FP32 master copy, biases and the output layer in FP32),
// instead of 4,672 FP32 FMAs per lane; SiLU divides with the fast
// reciprocal (the result only starts Newton).  The gates are
// mlp_guess_eval's: weak waves keep the two-shock start and skip the
// network (a warp with no other lane skips it entirely), and a prediction
// that is not a finite positive number or lies within the gate band of the
// two-shock guess is dropped (-1: two-shock start).  The Newton solves run
// afterwards in k_exact_batch, which reads these starts at the occupancy of
// the plain solver.
constexpr int kTcWarps = 8;

struct TcInferSmem {
    __nv_bfloat16 w1[MLP_H][MLP_W1P];
    __nv_bfloat16 w2[MLP_H][MLP_W2P];  // [out][in]
    float b1[MLP_H], b2[MLP_H], w3[MLP_H];
    float xs[kTcWarps][32][MLP_IN + 1];  // standardised features, one row per lane
};

// SiLU as z * (1 + tanh(z / 2)) / 2 with the hardware tanh approximation:
// one special-function operation instead of an exponential and a reciprocal
__device__ __forceinline__ float silu_fast(float z) {
    float th;
    asm("tanh.approx.f32 %0, %1;" : "=f"(th) : "f"(0.5f * z));
    return z * fmaf(0.5f, th, 0.5f);
}

template <int NDIM>
__global__ void __launch_bounds__(kTcWarps * 32, 3)
    k_mlp_guess_tc(int n, const double* __restrict__ ql, const double* __restrict__ qr,
                   const double* __restrict__ gam, double gamma0, const float* __restrict__ w,
                   double* __restrict__ guess_out) {
    constexpr int NV = NDIM + 2, IP = NDIM + 1;
    __shared__ TcInferSmem S;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    for (int i = tid; i < MLP_H * 16; i += blockDim.x) {
        const int j = i / 16, k = i % 16;
        S.w1[j][k] = __float2bfloat16_rn(k < MLP_IN ? w[MLP_W1 + j * MLP_IN + k] : 0.f);
    }
    for (int i = tid; i < MLP_H * MLP_H; i += blockDim.x) S.w2[i / MLP_H][i % MLP_H] = __float2bfloat16_rn(w[MLP_W2 + i]);
    for (int i = tid; i < MLP_H; i += blockDim.x) {
        S.b1[i] = w[MLP_B1 + i];
        S.b2[i] = w[MLP_B2 + i];
        S.w3[i] = w[MLP_W3 + i];
    }
    __syncthreads();
    const float b3 = __ldg(w + MLP_B3), ym = __ldg(w + MLP_YM), ys = __ldg(w + MLP_YS);
    const double gate = (double)__ldg(w + MLP_GATE);
    const long long nwarp = (long long)gridDim.x * kTcWarps;
    for (long long base0 = ((long long)blockIdx.x * kTcWarps + warp) * 32; base0 < n; base0 += nwarp * 32) {
        const long long i = base0 + lane;
        const bool act = i < n;
        double a[NV], b[NV];
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            // lanes past the end carry a uniform unit state through the network
            a[v] = act ? ql[(size_t)v * n + i] : (v == 0 || v == IP ? 1.0 : 0.0);
            b[v] = act ? qr[(size_t)v * n + i] : (v == 0 || v == IP ? 1.0 : 0.0);
        }
        const double gamma = (act && gam) ? gam[i] : gamma0;
        const double smallp = 1e-10 * 1e-10 / gamma;
        bool want = act;
        {
            const double rl = smax(a[0], 1e-10), pl = smax(a[IP], rl * smallp);
            const double rr = smax(b[0], 1e-10), pr = smax(b[IP], rr * smallp);
            if (smax(pl, pr) < MLP_WEAK_P * smin(pl, pr)) {
                const double du = a[1] - b[1], cs = sqrt(gamma * pl / rl) + sqrt(gamma * pr / rr);
                if (fabs(du) < MLP_WEAK_U * cs) want = false;
            }
        }
        double guess = -1.0;
        if (__ballot_sync(0xffffffffu, want)) {
            float x[MLP_IN];
            double pref, basep, p2s;
            mlp_features<NDIM, true>(a, b, gamma, smallp, x, &pref, &basep, &p2s);
#pragma unroll
            for (int k = 0; k < MLP_IN; ++k)
                S.xs[warp][lane][k] = __fdividef(x[k] - __ldg(w + MLP_MU + k), __ldg(w + MLP_SD + k));
            __syncwarp();
            float yt[2][2];  // [row tile][row g / g + 8] of this thread's group
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const int r0 = mt * 16 + g, r1 = r0 + 8;
                const uint32_t xa0 = pack_bf16(S.xs[warp][r0][2 * t], S.xs[warp][r0][2 * t + 1]);
                const uint32_t xa1 = pack_bf16(S.xs[warp][r1][2 * t], S.xs[warp][r1][2 * t + 1]);
                uint32_t ha[4][4];
#pragma unroll
                for (int kt = 0; kt < 4; ++kt) {
                    float h[2][4];
#pragma unroll
                    for (int hh = 0; hh < 2; ++hh) {
                        const int nt = 2 * kt + hh, col = nt * 8 + 2 * t;
                        float c[4] = {0.f, 0.f, 0.f, 0.f};
                        const uint32_t b0 = *reinterpret_cast<const uint32_t*>(&S.w1[nt * 8 + g][2 * t]);
                        const uint32_t b1v = *reinterpret_cast<const uint32_t*>(&S.w1[nt * 8 + g][2 * t + 8]);
                        mma16816(c, xa0, xa1, 0u, 0u, b0, b1v);
                        h[hh][0] = silu_fast(c[0] + S.b1[col]);
                        h[hh][1] = silu_fast(c[1] + S.b1[col + 1]);
                        h[hh][2] = silu_fast(c[2] + S.b1[col]);
                        h[hh][3] = silu_fast(c[3] + S.b1[col + 1]);
                    }
                    ha[kt][0] = pack_bf16(h[0][0], h[0][1]);
                    ha[kt][1] = pack_bf16(h[0][2], h[0][3]);
                    ha[kt][2] = pack_bf16(h[1][0], h[1][1]);
                    ha[kt][3] = pack_bf16(h[1][2], h[1][3]);
                }
                float y0 = 0.f, y1 = 0.f;
#pragma unroll
                for (int nt = 0; nt < 8; ++nt) {
                    float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                    for (int kt = 0; kt < 4; ++kt) {
                        const uint32_t b0 = *reinterpret_cast<const uint32_t*>(&S.w2[nt * 8 + g][kt * 16 + 2 * t]);
                        const uint32_t b1v =
                            *reinterpret_cast<const uint32_t*>(&S.w2[nt * 8 + g][kt * 16 + 2 * t + 8]);
                        mma16816(c, ha[kt][0], ha[kt][1], ha[kt][2], ha[kt][3], b0, b1v);
                    }
                    const int col = nt * 8 + 2 * t;
                    y0 += S.w3[col] * silu_fast(c[0] + S.b2[col]) + S.w3[col + 1] * silu_fast(c[1] + S.b2[col + 1]);
                    y1 += S.w3[col] * silu_fast(c[2] + S.b2[col]) + S.w3[col + 1] * silu_fast(c[3] + S.b2[col + 1]);
                }
                yt[mt][0] = quad_sum(y0) + b3;
                yt[mt][1] = quad_sum(y1) + b3;
            }
            __syncwarp();  // the feature rows are rewritten by the next chunk
            // lane L's row: tile L >> 4, row (L & 15) of it, held by group L & 7
            const int src = (lane & 7) * 4;
            const float y00 = __shfl_sync(0xffffffffu, yt[0][0], src), y01 = __shfl_sync(0xffffffffu, yt[0][1], src);
            const float y10 = __shfl_sync(0xffffffffu, yt[1][0], src), y11 = __shfl_sync(0xffffffffu, yt[1][1], src);
            const bool hi = (lane >> 3) & 1;
            const float yl = (lane >> 4) ? (hi ? y11 : y10) : (hi ? y01 : y00);
            if (want) {
                // the prediction and the gate in FP32: log(guess / p2s) = y + log(base / p2s)
                const float yv = ym + ys * yl;
                const double gg = basep * (double)__expf(yv);
                const bool near = p2s > 0.0 && fabsf(yv + __logf((float)(basep / p2s))) < (float)gate;
                if (isfinite(gg) && gg > 0.0 && !near) guess = gg;
            }
        }
        if (act) guess_out[i] = guess;
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
    if (mlp) {
        // learned starts on the tensor cores into a scratch array, then the
        // plain solver's kernel (and occupancy) with those starts
        double* starts = nullptr;
        if (int rc = check_cuda(c, dev_alloc(c, &starts, sizeof(double) * (size_t)std::max(n, 1)), "learned starts"))
            return rc;
        const long long warps = ((long long)n + 31) / 32;
        const int gb = (int)std::max(1LL, std::min((warps + kTcWarps - 1) / kTcWarps, (long long)c->sm_count * 12));
        if (c->params.ndim == 1) {
            k_mlp_guess_tc<1><<<gb, kTcWarps * 32, 0, c->stream>>>(n, ql, qr, gam, c->params.gamma, mlp, starts);
            k_exact_batch<1><<<blocks_for(c, n), 256, 0, c->stream>>>(n, ql, qr, gam, c->params.gamma, flux, pstar,
                                                                     iters, niter, tol, c->d_status, starts);
        } else {
            k_mlp_guess_tc<3><<<gb, kTcWarps * 32, 0, c->stream>>>(n, ql, qr, gam, c->params.gamma, mlp, starts);
            k_exact_batch<3><<<blocks_for(c, n), 256, 0, c->stream>>>(n, ql, qr, gam, c->params.gamma, flux, pstar,
                                                                     iters, niter, tol, c->d_status, starts);
        }
        dev_free(c, starts);
        return check_cuda(c, cudaGetLastError(), "exact batch (learned start)");
    }
    if (c->params.ndim == 1)
        k_exact_batch<1><<<blocks_for(c, n), 256, 0, c->stream>>>(n, ql, qr, gam, c->params.gamma, flux, pstar, iters,
                                                                 niter, tol, c->d_status, nullptr);
    else
        k_exact_batch<3><<<blocks_for(c, n), 256, 0, c->stream>>>(n, ql, qr, gam, c->params.gamma, flux, pstar, iters,
                                                                 niter, tol, c->d_status, nullptr);
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
