// rg_mlp.cuh -- the learned initial guess of the exact Riemann solver.
//
// The reference's exact solver (RiemannSolver::solve_godunov_nr, RAMSES-CPP
// src/solvers/hydro/RiemannSolver.cpp:194-307) starts its two-shock Newton
// iteration from the linearised guess of :215.  Here a small MLP, trained on
// states the solver itself generates, predicts the converged star pressure;
// Newton then polishes it, so the converged flux is unchanged to tolerance
// while fewer iterations are needed.  The two-shock guess stays the fallback
// whenever the prediction is not a finite positive number, and also when the
// prediction lies within a relative band (MLP_GATE in log space) of the
// two-shock guess: there the linearised start is already as good as the
// network (it is exact for weak waves, where Newton stops after one update),
// and replacing it by a prediction carrying the network's few-percent error
// would add iterations.
//
// Network: 8 features -> 64 -> 64 -> 1, SiLU activations.
// Features of a rotated pair (ql, qr) with floors as in the solver, pref =
// max(pl, pr), c = sqrt(gamma p / rho):
//   x0 log(rl/rr)            x1 log(pl/pr)
//   x2 asinh((ul-ur)/(cl+cr)) x3 asinh(ul/cl)   x4 asinh(ur/cr)
//   x5 gamma                  x6 log(max(p_twoshock, 1e-30 pref)/pref)
//   x7 log(max(p_tworarefaction, 1e-30 pref)/pref)  (Toro's TRRS estimate)
// Base estimate: b = max(p_twoshock, p_tworarefaction, 1e-30 pref).
// Target: log(max(p*, 1e-30 pref) / b); the guess is b * exp(prediction).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#include "rg_physics.cuh"

namespace rg {

constexpr int MLP_IN = 8, MLP_H = 64;
// float offsets inside one contiguous parameter block
constexpr int MLP_W1 = 0;                          // [H][IN]
constexpr int MLP_B1 = MLP_W1 + MLP_H * MLP_IN;    // [H]
constexpr int MLP_W2 = MLP_B1 + MLP_H;             // [H][H]  (out, in)
constexpr int MLP_B2 = MLP_W2 + MLP_H * MLP_H;     // [H]
constexpr int MLP_W3 = MLP_B2 + MLP_H;             // [H]
constexpr int MLP_B3 = MLP_W3 + MLP_H;             // [1]
constexpr int MLP_NTRAIN = MLP_B3 + 1;             // 4801 trained parameters
constexpr int MLP_MU = MLP_NTRAIN;                 // [IN] feature means   (fixed at training start)
constexpr int MLP_SD = MLP_MU + MLP_IN;            // [IN] feature scales
constexpr int MLP_YM = MLP_SD + MLP_IN;            // target mean
constexpr int MLP_YS = MLP_YM + 1;                 // target scale
constexpr int MLP_GATE = MLP_YS + 1;               // keep the two-shock start when |log(guess/p2s)| < gate
constexpr int MLP_NPARAM = MLP_GATE + 1;           // 4820 floats in the parameter block
constexpr float MLP_GATE_DEFAULT = 0.2f;
constexpr float MLP_LOG_FLOOR = 1e-30f;

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
    float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// Features of a rotated pair; returns pref and the base estimate b.
template <int NDIM>
__device__ __forceinline__ void mlp_features(const double* ql, const double* qr, double gamma, double smallp,
                                             float* x, double* pref_out, double* base_out,
                                             double* p2s_out = nullptr) {
    constexpr int IP = Dims<NDIM>::IP;
    double rl = smax(ql[0], 1e-10), ul = ql[1], pl = smax(ql[IP], rl * smallp);
    double rr = smax(qr[0], 1e-10), ur = qr[1], pr = smax(qr[IP], rr * smallp);
    double cl = sqrt(gamma * pl / rl), cr = sqrt(gamma * pr / rr);
    double wl = sqrt(gamma * pl * rl), wr = sqrt(gamma * pr * rr);
    double p2s = smax((wr * pl + wl * pr + wl * wr * (ul - ur)) / (wl + wr + 1e-20), 0.0);
    double pref = smax(pl, pr);
    double z = (gamma - 1.0) / (2.0 * gamma);
    double num = cl + cr - 0.5 * (gamma - 1.0) * (ur - ul);
    double den = cl / pow(pl, z) + cr / pow(pr, z);
    double ptr = num > 0.0 ? pow(num / den, 1.0 / z) : 0.0;
    x[0] = (float)log(rl / rr);
    x[1] = (float)log(pl / pr);
    x[2] = (float)asinh((ul - ur) / (cl + cr));
    x[3] = (float)asinh(ul / cl);
    x[4] = (float)asinh(ur / cr);
    x[5] = (float)gamma;
    x[6] = (float)log(smax(p2s, 1e-30 * pref) / pref);
    x[7] = (float)log(smax(ptr, 1e-30 * pref) / pref);
    *pref_out = pref;
    *base_out = smax(smax(p2s, ptr), 1e-30 * pref);
    if (p2s_out) *p2s_out = p2s;
}

// FP32 forward pass on standardised features xs; w points to MLP_NPARAM
// floats (global memory, read through the read-only cache: every lane reads
// the same weight).  Returns the standardised prediction.
__device__ __forceinline__ float mlp_forward_std(const float* __restrict__ w, const float* x) {
    float h1[MLP_H];
#pragma unroll 8
    for (int j = 0; j < MLP_H; ++j) {
        float z = __ldg(w + MLP_B1 + j);
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) z = fmaf(__ldg(w + MLP_W1 + j * MLP_IN + k), x[k], z);
        h1[j] = silu(z);
    }
    float y = __ldg(w + MLP_B3);
#pragma unroll 2
    for (int j = 0; j < MLP_H; ++j) {
        float z = __ldg(w + MLP_B2 + j);
#pragma unroll
        for (int k = 0; k < MLP_H; ++k) z = fmaf(__ldg(w + MLP_W2 + j * MLP_H + k), h1[k], z);
        y = fmaf(__ldg(w + MLP_W3 + j), silu(z), y);
    }
    return y;
}

// Learned Newton start: pref * exp(prediction), or -1 (use the two-shock
// guess) when the network is absent or its output is not usable.
template <int NDIM>
__device__ __forceinline__ double mlp_guess(const float* __restrict__ w, const double* ql, const double* qr,
                                            double gamma, double smallp) {
    if (!w) return -1.0;
    float x[MLP_IN];
    double pref, base, p2s;
    mlp_features<NDIM>(ql, qr, gamma, smallp, x, &pref, &base, &p2s);
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) x[k] = (x[k] - __ldg(w + MLP_MU + k)) / __ldg(w + MLP_SD + k);
    float y = __ldg(w + MLP_YM) + __ldg(w + MLP_YS) * mlp_forward_std(w, x);
    double g = base * exp((double)y);
    if (!(isfinite(g) && g > 0.0)) return -1.0;
    if (p2s > 0.0 && fabs(log(g / p2s)) < (double)__ldg(w + MLP_GATE)) return -1.0;
    return g;
}

}  // namespace rg
