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
// two-shock guess, and without evaluating the network at all for weak waves
// (MLP_WEAK_*): there the linearised start is already as good as the
// network (it is exact for weak waves, where Newton stops after one update),
// and replacing it by a prediction carrying the network's few-percent error
// would add iterations.
//
// Network: 8 features -> 64 -> 64 -> 1, SiLU activations.
// Features of a rotated pair (ql, qr) with floors as in the solver, pref =
// max(pl, pr), c = sqrt(gamma p / rho), FP32:
//   x0 log(rl/rr)            x1 log(pl/pr)
//   x2 asinh((ul-ur)/(cl+cr)) x3 asinh(ul/cl)   x4 asinh(ur/cr)
//   x5 gamma                  x6 log(max(p_twoshock, 1e-30 pref)/pref)
//   x7 log(max(p_ts, 1e-30 pref)/pref), p_ts = Toro's two-shock estimate (the
//      linearised formula with the wave mass fluxes taken at the plain guess)
// Base estimate: b = max(p_ts, 1e-30 pref).
// Target: log(max(p*, 1e-30 pref) / b); the guess is b * exp(prediction).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

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
constexpr float MLP_GATE_DEFAULT = 0.05f;
// Weak-wave pre-gate: with pmax/pmin < MLP_WEAK_P and |ul-ur| < MLP_WEAK_U
// (cl+cr) the two-shock guess is within a few percent of p* (its error is
// second order in the wave strength) and the network is not evaluated.
constexpr double MLP_WEAK_P = 1.3, MLP_WEAK_U = 0.3;
constexpr float MLP_LOG_FLOOR = 1e-30f;

constexpr int MLP_W1P = 24;  // padded row stride (bf16) of W1 in shared memory [64][16 used]
constexpr int MLP_W2P = 72;  // padded row stride (bf16) of W2 / W2^T in shared memory [64][64]

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// d += A B on the tensor cores: one m16n8k16 tile, BF16 operands, FP32 accumulation
__device__ __forceinline__ void mma16816(float* d, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// sum over the 4 threads of an mma row group
__device__ __forceinline__ float quad_sum(float v) {
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    return v;
}

__device__ __forceinline__ float silu(float z) { return z / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu_grad(float z) {
    float s = 1.0f / (1.0f + __expf(-z));
    return s * (1.0f + z * (1.0f - s));
}

// Features of a rotated pair; returns pref and the base estimate b (and the
// two-shock guess).  Computed in FP32 on scale-free quantities -- pressures
// in units of pref, densities of rref = max(rl, rr), velocities of
// sqrt(pref/rref) -- so that every intermediate stays in FP32 range whatever
// the states' scale; the features are ratios and do not depend on the units.
// FAST: hardware approximations of log, asinh and the FP32 divides (the
// batched tensor-core guess, where the features only seed Newton); the
// training data and the in-solver guess use the accurate functions.
__device__ __forceinline__ float feat_div(float a, float b, bool fast) { return fast ? __fdividef(a, b) : a / b; }
__device__ __forceinline__ float feat_log(float a, bool fast) { return fast ? __logf(a) : logf(a); }
__device__ __forceinline__ float feat_asinh(float a, bool fast) {
    if (!fast) return asinhf(a);
    const float m = fabsf(a);
    return copysignf(__logf(m + sqrtf(fmaf(m, m, 1.0f))), a);
}

template <int NDIM, bool FAST = false>
__device__ __forceinline__ void mlp_features(const double* ql, const double* qr, double gamma, double smallp,
                                             float* x, double* pref_out, double* base_out,
                                             double* p2s_out = nullptr) {
    constexpr int IP = Dims<NDIM>::IP;
    double rl = smax(ql[0], 1e-10), pl = smax(ql[IP], rl * smallp);
    double rr = smax(qr[0], 1e-10), pr = smax(qr[IP], rr * smallp);
    double pref = smax(pl, pr), rref = smax(rl, rr);
    double ip = 1.0 / pref, ir = 1.0 / rref, iv = sqrt(rref * ip);
    const float g = (float)gamma;
    const float al = (float)(rl * ir), ar = (float)(rr * ir);
    const float bl = (float)(pl * ip), br = (float)(pr * ip);
    const float vl = (float)(ql[1] * iv), vr = (float)(qr[1] * iv);
    float cl = sqrtf(feat_div(g * bl, al, FAST)), cr = sqrtf(feat_div(g * br, ar, FAST));
    float wl = sqrtf(g * bl * al), wr = sqrtf(g * br * ar);
    float p2s = fmaxf(feat_div(wr * bl + wl * br + wl * wr * (vl - vr), wl + wr + 1e-30f, FAST), 0.f);
    // Toro's two-shock estimate: the linearised formula above with each wave's
    // mass flux W_k(p) = sqrt(gamma p_k rho_k (1 + (gamma+1)/(2 gamma) (p-p_k)/p_k))
    // -- the function the solver's Newton iteration works on -- taken at the
    // plain guess instead of at p_k
    const float g6 = (g + 1.f) / (2.f * g);
    const float wl0 = sqrtf(fmaxf(wl * wl * (1.f + feat_div(g6 * (p2s - bl), bl, FAST)), 0.f));
    const float wr0 = sqrtf(fmaxf(wr * wr * (1.f + feat_div(g6 * (p2s - br), br, FAST)), 0.f));
    const float pts = fmaxf(feat_div(wr0 * bl + wl0 * br + wl0 * wr0 * (vl - vr), wl0 + wr0 + 1e-30f, FAST), 0.f);
    x[0] = feat_log(feat_div(al, ar, FAST), FAST);
    x[1] = feat_log(feat_div(bl, br, FAST), FAST);
    x[2] = feat_asinh(feat_div(vl - vr, cl + cr, FAST), FAST);
    x[3] = feat_asinh(feat_div(vl, cl, FAST), FAST);
    x[4] = feat_asinh(feat_div(vr, cr, FAST), FAST);
    x[5] = g;
    x[6] = feat_log(fmaxf(p2s, MLP_LOG_FLOOR), FAST);
    x[7] = feat_log(fmaxf(pts, MLP_LOG_FLOOR), FAST);
    *pref_out = pref;
    *base_out = pref * (double)fmaxf(pts, MLP_LOG_FLOOR);
    if (p2s_out) *p2s_out = pref * (double)p2s;
}

// FP32 forward pass on standardised features xs; w points to MLP_NPARAM
// floats (global memory, 16-byte aligned, read through the read-only cache
// as float4: every lane reads the same weights, so each load is a broadcast
// feeding four FMAs).  Returns the standardised prediction.
__device__ __forceinline__ float mlp_forward_std(const float* __restrict__ w, const float* x) {
    const float4* __restrict__ w4 = reinterpret_cast<const float4*>(w);
    float h1[MLP_H];
#pragma unroll 8
    for (int j = 0; j < MLP_H; ++j) {
        float z = __ldg(w + MLP_B1 + j);
        float4 a = __ldg(w4 + (MLP_W1 + j * MLP_IN) / 4), b = __ldg(w4 + (MLP_W1 + j * MLP_IN) / 4 + 1);
        z = fmaf(a.x, x[0], z);
        z = fmaf(a.y, x[1], z);
        z = fmaf(a.z, x[2], z);
        z = fmaf(a.w, x[3], z);
        z = fmaf(b.x, x[4], z);
        z = fmaf(b.y, x[5], z);
        z = fmaf(b.z, x[6], z);
        z = fmaf(b.w, x[7], z);
        h1[j] = silu(z);
    }
    float y = __ldg(w + MLP_B3);
#pragma unroll 2
    for (int j = 0; j < MLP_H; ++j) {
        float z = __ldg(w + MLP_B2 + j);
#pragma unroll
        for (int k = 0; k < MLP_H; k += 4) {
            float4 a = __ldg(w4 + (MLP_W2 + j * MLP_H + k) / 4);
            z = fmaf(a.x, h1[k], z);
            z = fmaf(a.y, h1[k + 1], z);
            z = fmaf(a.z, h1[k + 2], z);
            z = fmaf(a.w, h1[k + 3], z);
        }
        y = fmaf(__ldg(w + MLP_W3 + j), silu(z), y);
    }
    return y;
}

// Features, network and gate: out of line, so the face kernels that inline
// the exact solver carry the network's 64-wide hidden layer only in the
// frame of this call, not in their own register allocation.
template <int NDIM>
__device__ __noinline__ double mlp_guess_eval(const float* __restrict__ w, const double* ql, const double* qr,
                                              double gamma, double smallp);

// Learned Newton start: pref * exp(prediction), or -1 (use the two-shock
// guess) when the network is absent or its output is not usable.
template <int NDIM>
__device__ __forceinline__ double mlp_guess(const float* __restrict__ w, const double* ql, const double* qr,
                                            double gamma, double smallp) {
    if (!w) return -1.0;
    return mlp_guess_eval<NDIM>(w, ql, qr, gamma, smallp);
}

template <int NDIM>
__device__ __noinline__ double mlp_guess_eval(const float* __restrict__ w, const double* ql, const double* qr,
                                              double gamma, double smallp) {
    {
        constexpr int IP = Dims<NDIM>::IP;
        double rl = smax(ql[0], 1e-10), pl = smax(ql[IP], rl * smallp);
        double rr = smax(qr[0], 1e-10), pr = smax(qr[IP], rr * smallp);
        if (smax(pl, pr) < MLP_WEAK_P * smin(pl, pr)) {
            double du = ql[1] - qr[1], cs = sqrt(gamma * pl / rl) + sqrt(gamma * pr / rr);
            if (fabs(du) < MLP_WEAK_U * cs) return -1.0;
        }
    }
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
