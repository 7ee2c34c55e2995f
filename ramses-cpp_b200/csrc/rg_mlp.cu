// rg_mlp.cu -- training of the learned Newton start (rg_mlp.cuh) on the GPU.
//
// Forward and backward of the 8 -> 64 -> 64 -> 1 SiLU network on tensor
// cores: BF16 operands, FP32 accumulation (mma.sync m16n8k16), FP32 master
// weights updated by Adam.  The layers are small (K <= 64), so each warp owns
// 16 samples and keeps the whole forward/backward in registers; the
// accumulator fragments of one layer are re-packed as the A operand of the
// next (same thread-to-row/column mapping), and the weight gradients are
// reduced over the block's 64 samples from shared memory in FP32.
//
// Rounding contract (mirrored exactly by the CPU gradient check): features,
// hidden activations H1 and the output-layer gradient dZ2 are rounded to BF16
// where they enter a tensor-core product; W1 and W2 are rounded to BF16 from
// the FP32 master copy; w3, biases, activations and all accumulations are FP32.
#include <cuda_bf16.h>

#include <cmath>
#include <cstdint>
#include <random>
#include <vector>

#include "rg_face.cuh"
#include "rg_mlp.cuh"

namespace rg {

namespace {

constexpr int TB = 128;       // threads per block: 4 warps
constexpr int SPB = 64;       // samples per block iteration (16 per warp)

struct TrainSmem {
    __nv_bfloat16 w1[MLP_H][MLP_W1P];
    __nv_bfloat16 w2[MLP_H][MLP_W2P];   // [out][in]
    __nv_bfloat16 w2t[MLP_H][MLP_W2P];  // [in][out]
    float b1[MLP_H], b2[MLP_H], w3[MLP_H];
    float h1b[SPB][MLP_H + 1];      // BF16-rounded H1 per sample
    float dz2[SPB][MLP_H + 1];
    float dz1[SPB][MLP_H + 1];
    float xb[SPB][MLP_IN + 1];
};

__device__ __forceinline__ float group_sum(float v) {  // over the 8 row groups of a warp
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 8);
    v += __shfl_xor_sync(0xffffffffu, v, 16);
    return v;
}

// Loss and gradients of the batch [n0, n0+nb) (standardised X [IN][N] and T
// [N]).  Block b writes the sums over its samples to its own row
// part[b][NTRAIN + 1] (gradients, then the squared error); k_grad_sum adds the
// rows in block order.  No atomics: the gradient, hence the trained network
// and every p* guess it makes, is the same bits on every run.
__global__ void __launch_bounds__(TB) k_mlp_grad(const float* __restrict__ X, const float* __restrict__ T, int N,
                                                 int n0, int nb, const float* __restrict__ w, float* part) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
    for (int i = tid; i < MLP_H * 16; i += TB) {
        int j = i / 16, k = i % 16;
        S.w1[j][k] = __float2bfloat16_rn(k < MLP_IN ? w[MLP_W1 + j * MLP_IN + k] : 0.f);
    }
    for (int i = tid; i < MLP_H * MLP_H; i += TB) {
        int o = i / MLP_H, in = i % MLP_H;
        __nv_bfloat16 v = __float2bfloat16_rn(w[MLP_W2 + i]);
        S.w2[o][in] = v;
        S.w2t[in][o] = v;
    }
    for (int i = tid; i < MLP_H; i += TB) {
        S.b1[i] = w[MLP_B1 + i];
        S.b2[i] = w[MLP_B2 + i];
        S.w3[i] = w[MLP_W3 + i];
    }
    const float b3 = w[MLP_B3];
    const float inv_nb = 1.0f / (float)nb;
    __syncthreads();

    // per-thread accumulators: columns col(nt, e) = nt*8 + 2t + e of this thread
    float acc_db1[8][2], acc_db2[8][2], acc_dw3[8][2];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int e = 0; e < 2; ++e) acc_db1[nt][e] = acc_db2[nt][e] = acc_dw3[nt][e] = 0.f;
    float acc_db3 = 0.f, acc_loss = 0.f;
    float acc_w2[32], acc_w1[4];
#pragma unroll
    for (int j = 0; j < 32; ++j) acc_w2[j] = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) acc_w1[j] = 0.f;

    const int ntile = (nb + SPB - 1) / SPB;
    for (int tile = blockIdx.x; tile < ntile; tile += gridDim.x) {
        const int sb = warp * 16;                 // first block-local sample of this warp
        const int base = n0 + tile * SPB + sb;    // first global sample of this warp
        const int lim = n0 + nb;
        const int r0 = base + g, r1 = base + g + 8;
        const bool v0 = r0 < lim, v1 = r1 < lim;
        // ---- layer 1: Z1 = X W1^T + b1 (K = 8 features padded to 16)
        float x00 = v0 ? X[(size_t)(2 * t) * N + r0] : 0.f, x01 = v0 ? X[(size_t)(2 * t + 1) * N + r0] : 0.f;
        float x10 = v1 ? X[(size_t)(2 * t) * N + r1] : 0.f, x11 = v1 ? X[(size_t)(2 * t + 1) * N + r1] : 0.f;
        S.xb[sb + g][2 * t] = bf16r(x00);
        S.xb[sb + g][2 * t + 1] = bf16r(x01);
        S.xb[sb + g + 8][2 * t] = bf16r(x10);
        S.xb[sb + g + 8][2 * t + 1] = bf16r(x11);
        const uint32_t xa0 = pack_bf16(x00, x01), xa1 = pack_bf16(x10, x11);
        float z1[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            uint32_t b0 = *reinterpret_cast<const uint32_t*>(&S.w1[nt * 8 + g][2 * t]);
            uint32_t b1v = *reinterpret_cast<const uint32_t*>(&S.w1[nt * 8 + g][2 * t + 8]);
            mma16816(c, xa0, xa1, 0u, 0u, b0, b1v);
            const int col = nt * 8 + 2 * t;
            z1[nt][0] = c[0] + S.b1[col];
            z1[nt][1] = c[1] + S.b1[col + 1];
            z1[nt][2] = c[2] + S.b1[col];
            z1[nt][3] = c[3] + S.b1[col + 1];
        }
        // H1 (BF16) as A fragments of layer 2, also staged for dW2
        uint32_t ha[4][4];
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            float h[2][4];
#pragma unroll
            for (int hh = 0; hh < 2; ++hh)
#pragma unroll
                for (int e = 0; e < 4; ++e) h[hh][e] = bf16r(silu(z1[2 * kt + hh][e]));
            ha[kt][0] = pack_bf16(h[0][0], h[0][1]);
            ha[kt][1] = pack_bf16(h[0][2], h[0][3]);
            ha[kt][2] = pack_bf16(h[1][0], h[1][1]);
            ha[kt][3] = pack_bf16(h[1][2], h[1][3]);
#pragma unroll
            for (int hh = 0; hh < 2; ++hh) {
                const int col = (2 * kt + hh) * 8 + 2 * t;
                S.h1b[sb + g][col] = h[hh][0];
                S.h1b[sb + g][col + 1] = h[hh][1];
                S.h1b[sb + g + 8][col] = h[hh][2];
                S.h1b[sb + g + 8][col + 1] = h[hh][3];
            }
        }
        // ---- layer 2: Z2 = H1 W2^T + b2; output y = w3 . silu(Z2) + b3
        float z2[8][4];
        float y0 = 0.f, y1 = 0.f;
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kt = 0; kt < 4; ++kt) {
                uint32_t b0 = *reinterpret_cast<const uint32_t*>(&S.w2[nt * 8 + g][kt * 16 + 2 * t]);
                uint32_t b1v = *reinterpret_cast<const uint32_t*>(&S.w2[nt * 8 + g][kt * 16 + 2 * t + 8]);
                mma16816(c, ha[kt][0], ha[kt][1], ha[kt][2], ha[kt][3], b0, b1v);
            }
            const int col = nt * 8 + 2 * t;
            z2[nt][0] = c[0] + S.b2[col];
            z2[nt][1] = c[1] + S.b2[col + 1];
            z2[nt][2] = c[2] + S.b2[col];
            z2[nt][3] = c[3] + S.b2[col + 1];
            y0 += S.w3[col] * silu(z2[nt][0]) + S.w3[col + 1] * silu(z2[nt][1]);
            y1 += S.w3[col] * silu(z2[nt][2]) + S.w3[col + 1] * silu(z2[nt][3]);
        }
        y0 = quad_sum(y0) + b3;
        y1 = quad_sum(y1) + b3;
        const float e0 = v0 ? y0 - T[r0] : 0.f, e1 = v1 ? y1 - T[r1] : 0.f;
        if (t == 0) acc_loss += e0 * e0 + e1 * e1;
        const float dy0 = 2.f * e0 * inv_nb, dy1 = 2.f * e1 * inv_nb;
        if (t == 0) acc_db3 += dy0 + dy1;
        // ---- backward through layer 2
        uint32_t da[4][4];
        float dz2v[8][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            const int col = nt * 8 + 2 * t;
            acc_dw3[nt][0] += dy0 * silu(z2[nt][0]) + dy1 * silu(z2[nt][2]);
            acc_dw3[nt][1] += dy0 * silu(z2[nt][1]) + dy1 * silu(z2[nt][3]);
            dz2v[nt][0] = dy0 * S.w3[col] * silu_grad(z2[nt][0]);
            dz2v[nt][1] = dy0 * S.w3[col + 1] * silu_grad(z2[nt][1]);
            dz2v[nt][2] = dy1 * S.w3[col] * silu_grad(z2[nt][2]);
            dz2v[nt][3] = dy1 * S.w3[col + 1] * silu_grad(z2[nt][3]);
            acc_db2[nt][0] += dz2v[nt][0] + dz2v[nt][2];
            acc_db2[nt][1] += dz2v[nt][1] + dz2v[nt][3];
            S.dz2[sb + g][col] = dz2v[nt][0];
            S.dz2[sb + g][col + 1] = dz2v[nt][1];
            S.dz2[sb + g + 8][col] = dz2v[nt][2];
            S.dz2[sb + g + 8][col + 1] = dz2v[nt][3];
        }
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            da[kt][0] = pack_bf16(dz2v[2 * kt][0], dz2v[2 * kt][1]);
            da[kt][1] = pack_bf16(dz2v[2 * kt][2], dz2v[2 * kt][3]);
            da[kt][2] = pack_bf16(dz2v[2 * kt + 1][0], dz2v[2 * kt + 1][1]);
            da[kt][3] = pack_bf16(dz2v[2 * kt + 1][2], dz2v[2 * kt + 1][3]);
        }
        // dH1 = dZ2 W2 (A = dZ2 in BF16, B = W2 read through its transpose), dZ1 = dH1 silu'(Z1)
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int kt = 0; kt < 4; ++kt) {
                uint32_t b0 = *reinterpret_cast<const uint32_t*>(&S.w2t[nt * 8 + g][kt * 16 + 2 * t]);
                uint32_t b1v = *reinterpret_cast<const uint32_t*>(&S.w2t[nt * 8 + g][kt * 16 + 2 * t + 8]);
                mma16816(c, da[kt][0], da[kt][1], da[kt][2], da[kt][3], b0, b1v);
            }
            const int col = nt * 8 + 2 * t;
            float d0 = c[0] * silu_grad(z1[nt][0]), d1 = c[1] * silu_grad(z1[nt][1]);
            float d2 = c[2] * silu_grad(z1[nt][2]), d3 = c[3] * silu_grad(z1[nt][3]);
            acc_db1[nt][0] += d0 + d2;
            acc_db1[nt][1] += d1 + d3;
            S.dz1[sb + g][col] = d0;
            S.dz1[sb + g][col + 1] = d1;
            S.dz1[sb + g + 8][col] = d2;
            S.dz1[sb + g + 8][col + 1] = d3;
        }
        __syncthreads();
        // ---- weight gradients over the block's 64 samples (FP32)
        {
            const int o = tid >> 1, half = tid & 1;
            for (int s = 0; s < SPB; ++s) {
                const float d2 = S.dz2[s][o], d1 = S.dz1[s][o];
#pragma unroll
                for (int j = 0; j < 32; ++j) acc_w2[j] += d2 * S.h1b[s][half * 32 + j];
#pragma unroll
                for (int k = 0; k < 4; ++k) acc_w1[k] += d1 * S.xb[s][half * 4 + k];
            }
        }
        __syncthreads();
    }
    // ---- flush to this block's row: W1 / W2 entries belong to one thread each;
    //      the per-warp sums of b1, b2, w3, b3 and the loss meet in shared
    //      memory (free after the loop's last barrier) and are added in warp order
    constexpr int NW = TB / 32;
    float* row = part + (size_t)blockIdx.x * (MLP_NTRAIN + 1);
    {
        const int o = tid >> 1, half = tid & 1;
#pragma unroll
        for (int j = 0; j < 32; ++j) row[MLP_W2 + o * MLP_H + half * 32 + j] = acc_w2[j];
#pragma unroll
        for (int k = 0; k < 4; ++k) row[MLP_W1 + o * MLP_IN + half * 4 + k] = acc_w1[k];
    }
    float* red = &S.dz2[0][0];  // [NW][3][H] column sums, then [NW][2] (loss, b3)
#pragma unroll
    for (int nt = 0; nt < 8; ++nt)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            float a = group_sum(acc_db1[nt][e]), b = group_sum(acc_db2[nt][e]), c = group_sum(acc_dw3[nt][e]);
            if (g == 0) {
                const int col = nt * 8 + 2 * t + e;
                red[(warp * 3 + 0) * MLP_H + col] = a;
                red[(warp * 3 + 1) * MLP_H + col] = b;
                red[(warp * 3 + 2) * MLP_H + col] = c;
            }
        }
    float l = acc_loss, d3 = acc_db3;
    for (int off = 16; off > 0; off >>= 1) {
        l += __shfl_xor_sync(0xffffffffu, l, off);
        d3 += __shfl_xor_sync(0xffffffffu, d3, off);
    }
    if (lane == 0) {
        red[NW * 3 * MLP_H + 2 * warp] = l;
        red[NW * 3 * MLP_H + 2 * warp + 1] = d3;
    }
    __syncthreads();
    for (int i = tid; i < 3 * MLP_H; i += TB) {
        const int q = i / MLP_H, col = i % MLP_H;
        float sum = 0.f;
#pragma unroll
        for (int wp = 0; wp < NW; ++wp) sum += red[(wp * 3 + q) * MLP_H + col];
        row[(q == 0 ? MLP_B1 : (q == 1 ? MLP_B2 : MLP_W3)) + col] = sum;
    }
    if (tid == 0) {
        float ls = 0.f, bs = 0.f;
#pragma unroll
        for (int wp = 0; wp < NW; ++wp) {
            ls += red[NW * 3 * MLP_H + 2 * wp];
            bs += red[NW * 3 * MLP_H + 2 * wp + 1];
        }
        row[MLP_B3] = bs;
        row[MLP_NTRAIN] = ls;
    }
}

// grad[p] += the blocks' rows summed in block order; column NTRAIN into *loss
__global__ void k_grad_sum(const float* __restrict__ part, int nblk, float* grad, float* loss) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= MLP_NTRAIN; p += gridDim.x * blockDim.x) {
        float sum = 0.f;
        for (int b = 0; b < nblk; ++b) sum += part[(size_t)b * (MLP_NTRAIN + 1) + p];
        if (p < MLP_NTRAIN) grad[p] += sum;
        else *loss += sum;
    }
}

__global__ void k_adam(float* w, float* m, float* v, float* grad, int n, float lr, float b1, float b2, float eps,
                       float bc1, float bc2) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        float gr = grad[p];
        float mm = b1 * m[p] + (1.f - b1) * gr;
        float vv = b2 * v[p] + (1.f - b2) * gr * gr;
        m[p] = mm;
        v[p] = vv;
        w[p] -= lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
        grad[p] = 0.f;
    }
}

__global__ void k_standardise(float* X, float* T, int n, const float* __restrict__ w) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) X[(size_t)k * n + i] = (X[(size_t)k * n + i] - w[MLP_MU + k]) / w[MLP_SD + k];
        if (T) T[i] = (T[i] - w[MLP_YM]) / w[MLP_YS];
    }
}

}  // namespace

int launch_exact_batch(rg_ctx* c, int n, const double* ql, const double* qr, const double* gam, double* flux,
                       double* pstar, int* iters, const float* mlp, int niter, double tol);
int launch_stress_states(rg_ctx* c, int n, unsigned long long seed, double* ql, double* qr, double* gam);
int launch_features(rg_ctx* c, int n, const double* ql, const double* qr, const double* gam, const double* pstar,
                    float* X, float* T);

// d_mlp: parameters [NPARAM], Adam moments m, v and the gradient [NTRAIN] each,
// the loss, one spare float, then the gradient kernel's per-block rows
// [sm_count][NTRAIN + 1]
constexpr size_t kPartOffset = MLP_NPARAM + 3 * MLP_NTRAIN + 2;

int mlp_ensure(rg_ctx* c) {
    if (c->d_mlp) return RG_OK;
    size_t bytes = sizeof(float) * (kPartOffset + (size_t)c->sm_count * (MLP_NTRAIN + 1));
    if (dev_alloc(c, &c->d_mlp, bytes) != cudaSuccess) {
        cudaGetLastError();
        c->d_mlp = nullptr;
        return set_error(c, RG_ERR_NOMEM, "MLP parameters");
    }
    cudaMemsetAsync(c->d_mlp, 0, bytes, c->stream);
    return check_cuda(c, cudaStreamSynchronize(c->stream), "MLP init");
}

static int grad_launch(rg_ctx* c, const float* X, const float* T, int N, int n0, int nb, float* grad, float* loss) {
    static bool attr_set[64] = {};  // per device: the shared-memory opt-in is a function attribute
    const int dev = c->device & 63;
    if (!attr_set[dev]) {
        if (int rc = check_cuda(c, cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                        (int)sizeof(TrainSmem)),
                                "MLP gradient kernel shared memory"))
            return rc;
        attr_set[dev] = true;
    }
    int tiles = (nb + SPB - 1) / SPB;
    int grid = tiles < c->sm_count ? tiles : c->sm_count;
    float* part = c->d_mlp + kPartOffset;
    k_mlp_grad<<<grid, TB, sizeof(TrainSmem), c->stream>>>(X, T, N, n0, nb, c->d_mlp, part);
    k_grad_sum<<<(MLP_NTRAIN + 256) / 256, 256, 0, c->stream>>>(part, grid, grad, loss);
    return check_cuda(c, cudaGetLastError(), "MLP gradient kernel");
}

// Host side of training: data from the solver itself (stress states, p* from
// the converged Newton iteration), standardisation, Adam with a cosine decay.
int mlp_train(rg_ctx* c, int nsamples, int epochs, int batch, float lr, unsigned long long seed, float* loss_out) {
    if (nsamples < 1024 || epochs < 1 || batch < 64) return set_error(c, RG_ERR_ARG, "bad training sizes");
    if (int rc = mlp_ensure(c)) return rc;
    const int nv = c->params.ndim + 2;
    double *ql = nullptr, *qr = nullptr, *gam = nullptr, *ps = nullptr;
    float *X = nullptr, *T = nullptr;
    size_t n = (size_t)nsamples;
    auto cleanup = [&]() {
        dev_free(c, ql); dev_free(c, qr); dev_free(c, gam); dev_free(c, ps); dev_free(c, X); dev_free(c, T);
    };
    if (dev_alloc(c, &ql, sizeof(double) * nv * n) != cudaSuccess || dev_alloc(c, &qr, sizeof(double) * nv * n) != cudaSuccess ||
        dev_alloc(c, &gam, sizeof(double) * n) != cudaSuccess || dev_alloc(c, &ps, sizeof(double) * n) != cudaSuccess ||
        dev_alloc(c, &X, sizeof(float) * MLP_IN * n) != cudaSuccess || dev_alloc(c, &T, sizeof(float) * n) != cudaSuccess) {
        cudaGetLastError();
        cleanup();
        return set_error(c, RG_ERR_NOMEM, "training data");
    }
    int rc = launch_stress_states(c, nsamples, seed, ql, qr, gam);
    if (!rc) rc = launch_exact_batch(c, nsamples, ql, qr, gam, nullptr, ps, nullptr, nullptr, 100, 1e-14);
    if (!rc) rc = launch_features(c, nsamples, ql, qr, gam, ps, X, T);
    if (rc) { cleanup(); return rc; }
    // standardisation from a strided sample of 65536 rows
    const int ns = 65536;
    std::vector<float> hx((size_t)MLP_IN * ns), ht(ns);
    size_t stride = n / ns > 0 ? n / ns : 1;
    for (int k = 0; k <= MLP_IN; ++k) {
        const float* src = (k < MLP_IN) ? X + (size_t)k * n : T;
        float* dst = (k < MLP_IN) ? hx.data() + (size_t)k * ns : ht.data();
        cudaMemcpy2DAsync(dst, sizeof(float), src, sizeof(float) * stride, sizeof(float), ns, cudaMemcpyDeviceToHost,
                          c->stream);
    }
    if ((rc = check_cuda(c, cudaStreamSynchronize(c->stream), "training sample"))) { cleanup(); return rc; }
    std::vector<float> hw(MLP_NPARAM, 0.f);
    std::mt19937_64 rng(seed ^ 0x5DEECE66DULL);
    auto uni = [&](float a) { return std::uniform_real_distribution<float>(-a, a)(rng); };
    for (int i = 0; i < MLP_H * MLP_IN; ++i) hw[MLP_W1 + i] = uni(std::sqrt(6.f / (MLP_IN + MLP_H)));
    for (int i = 0; i < MLP_H * MLP_H; ++i) hw[MLP_W2 + i] = uni(std::sqrt(6.f / (2 * MLP_H)));
    for (int i = 0; i < MLP_H; ++i) hw[MLP_W3 + i] = uni(std::sqrt(6.f / (MLP_H + 1)));
    for (int k = 0; k <= MLP_IN; ++k) {
        const float* a = (k < MLP_IN) ? hx.data() + (size_t)k * ns : ht.data();
        double s = 0, s2 = 0;
        for (int i = 0; i < ns; ++i) { s += a[i]; s2 += (double)a[i] * a[i]; }
        double mu = s / ns, sd = std::sqrt(std::max(s2 / ns - mu * mu, 1e-12));
        if (k < MLP_IN) { hw[MLP_MU + k] = (float)mu; hw[MLP_SD + k] = (float)sd; }
        else { hw[MLP_YM] = (float)mu; hw[MLP_YS] = (float)sd; }
    }
    hw[MLP_GATE] = MLP_GATE_DEFAULT;
    float* w = c->d_mlp;
    float* m = w + MLP_NPARAM;
    float* v = m + MLP_NTRAIN;
    float* grad = v + MLP_NTRAIN;
    float* dloss = grad + MLP_NTRAIN;
    cudaMemcpyAsync(w, hw.data(), sizeof(float) * MLP_NPARAM, cudaMemcpyHostToDevice, c->stream);
    cudaMemsetAsync(m, 0, sizeof(float) * (3 * MLP_NTRAIN + 2), c->stream);
    k_standardise<<<c->sm_count * 8, 256, 0, c->stream>>>(X, T, nsamples, w);
    const int steps_per_epoch = (int)(n / batch);
    const int total = steps_per_epoch * epochs;
    float b1 = 0.9f, b2 = 0.999f;
    double bc1 = 1, bc2 = 1;
    float last_loss = 0.f;
    for (int step = 0; step < total && !rc; ++step) {
        int n0 = (int)(((size_t)step % steps_per_epoch) * batch);
        bc1 *= b1;
        bc2 *= b2;
        float lr_t = (float)(0.05 * lr + 0.95 * lr * 0.5 * (1.0 + std::cos(M_PI * step / (double)total)));
        bool last_epoch = step >= total - steps_per_epoch;
        if (last_epoch && step == total - steps_per_epoch) cudaMemsetAsync(dloss, 0, sizeof(float), c->stream);
        rc = grad_launch(c, X, T, nsamples, n0, batch, grad, dloss);
        if (!rc) {
            k_adam<<<(MLP_NTRAIN + 255) / 256, 256, 0, c->stream>>>(w, m, v, grad, MLP_NTRAIN, lr_t, b1, b2, 1e-8f,
                                                                     (float)(1.0 - bc1), (float)(1.0 - bc2));
            rc = check_cuda(c, cudaGetLastError(), "adam");
        }
    }
    if (!rc) {
        float h = 0;
        cudaMemcpyAsync(&h, dloss, sizeof(float), cudaMemcpyDeviceToHost, c->stream);
        rc = check_cuda(c, cudaStreamSynchronize(c->stream), "training");
        last_loss = h / (float)((size_t)steps_per_epoch * batch);
    }
    cleanup();
    if (rc) return rc;
    c->mlp_valid = true;
    if (loss_out) *loss_out = last_loss;
    return RG_OK;
}

int mlp_grad(rg_ctx* c, int n, const float* x_host, const float* t_host, float* grad_host, float* loss_host) {
    if (int rc = mlp_ensure(c)) return rc;
    float *X = nullptr, *T = nullptr, *G = nullptr;
    if (dev_alloc(c, &X, sizeof(float) * MLP_IN * n) != cudaSuccess || dev_alloc(c, &T, sizeof(float) * n) != cudaSuccess ||
        dev_alloc(c, &G, sizeof(float) * (MLP_NTRAIN + 1)) != cudaSuccess) {
        cudaGetLastError();
        dev_free(c, X); dev_free(c, T); dev_free(c, G);
        return set_error(c, RG_ERR_NOMEM, "gradient check buffers");
    }
    cudaMemcpyAsync(X, x_host, sizeof(float) * MLP_IN * n, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(T, t_host, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream);
    cudaMemsetAsync(G, 0, sizeof(float) * (MLP_NTRAIN + 1), c->stream);
    int rc = grad_launch(c, X, T, n, 0, n, G, G + MLP_NTRAIN);
    if (!rc) {
        cudaMemcpyAsync(grad_host, G, sizeof(float) * MLP_NTRAIN, cudaMemcpyDeviceToHost, c->stream);
        cudaMemcpyAsync(loss_host, G + MLP_NTRAIN, sizeof(float), cudaMemcpyDeviceToHost, c->stream);
        rc = check_cuda(c, cudaStreamSynchronize(c->stream), "gradient check");
    }
    dev_free(c, X); dev_free(c, T); dev_free(c, G);
    return rc;
}

}  // namespace rg
