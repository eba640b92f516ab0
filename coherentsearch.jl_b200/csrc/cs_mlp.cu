// cs_mlp.cu -- the learned block proposal: per-block incoherent power-sum
// features and a small MLP (features -> 256 -> 256 -> 1, BF16 weights, FP32
// accumulation) with its training kernels.  No counterpart in the reference:
// it scores frequency blocks so that the coherent search, which reports
// every candidate, re-searches only the proposed ones.
//
// The network is tiny (147*256 + 256*256 + 256 weights): a training batch is
// a few MFLOP, so the layers are plain tiled SIMT products (FP32 accumulation
// of BF16 weights) rather than tensor-core tiles; their time is launch-bound.
#include "cohsearch.h"
#include "cs_internal.h"

#include <cuda_bf16.h>

#include <cmath>

namespace cs {

namespace {

// ---------------------------------------------------------------------------
// Features: for each decimation level (k, Hk) and each harmonic count
// H = 1..Hk, the incoherent power sum S(r) = sum_{i<=H} |X[rint(i*k*r)]|^2 at
// every trial r of the block (the coherent search's own grid), normalised as
// z = (S - H)/sqrt(H) (unit-mean exponential powers of a normalised spectrum:
// mean H, variance H); the feature is asinh of z's maximum over the block.
// Bins outside [1, namps) count as the mean power 1.  One CTA per block: each
// thread carries its trials' running sums over H, warps reduce the maxima.
// ---------------------------------------------------------------------------
constexpr int kFeatThreads = 256;
constexpr int kFeatTrials = 8;      // trials per thread and pass
constexpr int kFeatMax = 512;       // features per block

__global__ void __launch_bounds__(kFeatThreads) k_features(const float2* __restrict__ amps, int64_t namps,
                                                           double r_lo, double lodr, int64_t Nprof, int64_t total,
                                                           const DevLevel* __restrict__ levels, int nlev, int nfeat,
                                                           float* __restrict__ out) {
    __shared__ float red[kFeatThreads / 32][kFeatMax];
    const int64_t b = blockIdx.x;
    const int64_t t0 = b * Nprof;
    const int n = (int)min(Nprof, total - t0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int f = threadIdx.x; f < (kFeatThreads / 32) * nfeat; f += blockDim.x) red[f / nfeat][f % nfeat] = -INFINITY;
    __syncthreads();
    for (int j0 = 0; j0 < n; j0 += kFeatThreads * kFeatTrials) {
        double r[kFeatTrials];
        bool in[kFeatTrials];
#pragma unroll
        for (int q = 0; q < kFeatTrials; ++q) {
            const int j = j0 + q * kFeatThreads + threadIdx.x;
            in[q] = j < n;
            r[q] = r_lo + (double)(t0 + j) * lodr;
        }
        int f = 0;
        for (int l = 0; l < nlev; ++l) {
            const int k = levels[l].k, Hk = levels[l].Hk;
            float s[kFeatTrials];
#pragma unroll
            for (int q = 0; q < kFeatTrials; ++q) s[q] = 0.0f;
            for (int H = 1; H <= Hk; ++H, ++f) {
                float mx = -INFINITY;
                const float inv = rsqrtf((float)H);
#pragma unroll
                for (int q = 0; q < kFeatTrials; ++q) {
                    const int64_t bin = (int64_t)rint((double)(H * k) * r[q]);
                    float p = 1.0f;
                    if (bin >= 1 && bin < namps) {
                        const float2 x = __ldg(amps + bin);
                        p = x.x * x.x + x.y * x.y;
                    }
                    s[q] += p;
                    if (in[q]) mx = fmaxf(mx, (s[q] - (float)H) * inv);
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
                if (lane == 0) red[warp][f] = fmaxf(red[warp][f], mx);
            }
        }
    }
    __syncthreads();
    for (int f = threadIdx.x; f < nfeat; f += blockDim.x) {
        float mx = -INFINITY;
#pragma unroll
        for (int w = 0; w < kFeatThreads / 32; ++w) mx = fmaxf(mx, red[w][f]);
        out[b * nfeat + f] = asinhf(mx);
    }
}

// ---------------------------------------------------------------------------
// Dense products.  C[m][n] (row-major, ldc = N) = sum_k A(m,k) B(k,n) with
// A(m,k) = A[m*sam + k*sak], B(k,n) = B[k*sbk + n*sbn] (either operand FP32 or
// BF16), FP32 accumulation, then an epilogue: + bias[n], ReLU, or a ReLU mask
// (C *= (mask[m][n] > 0)).  64x64 tiles, K in steps of 16, 4x4 per thread.
// ---------------------------------------------------------------------------
constexpr int kBM = 64, kBN = 64, kBK = 16;

template <class T>
__device__ __forceinline__ float ld(const T* p, int64_t i);
template <>
__device__ __forceinline__ float ld<float>(const float* p, int64_t i) { return p[i]; }
template <>
__device__ __forceinline__ float ld<__nv_bfloat16>(const __nv_bfloat16* p, int64_t i) {
    return __bfloat162float(p[i]);
}

enum Epi { kEpiNone = 0, kEpiBias = 1, kEpiBiasRelu = 2, kEpiMask = 3 };

template <class TA, class TB>
__global__ void __launch_bounds__(256) k_gemm(const TA* __restrict__ A, int64_t sam, int64_t sak,
                                              const TB* __restrict__ B, int64_t sbk, int64_t sbn, float* __restrict__ C,
                                              int64_t M, int64_t N, int64_t K, int epi, const float* __restrict__ aux) {
    __shared__ float As[kBK][kBM + 4];
    __shared__ float Bs[kBK][kBN + 4];
    const int tid = threadIdx.x;
    const int64_t m0 = (int64_t)blockIdx.y * kBM, n0 = (int64_t)blockIdx.x * kBN;
    const int tm = (tid / 16) * 4, tn = (tid % 16) * 4;
    float acc[4][4] = {};
    for (int64_t k0 = 0; k0 < K; k0 += kBK) {
        for (int i = tid; i < kBK * kBM; i += 256) {
            const int kk = i / kBM, mm = i % kBM;
            const int64_t m = m0 + mm, k = k0 + kk;
            As[kk][mm] = (m < M && k < K) ? ld<TA>(A, m * sam + k * sak) : 0.0f;
        }
        for (int i = tid; i < kBK * kBN; i += 256) {
            const int kk = i / kBN, nn = i % kBN;
            const int64_t nc = n0 + nn, k = k0 + kk;
            Bs[kk][nn] = (nc < N && k < K) ? ld<TB>(B, k * sbk + nc * sbn) : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kBK; ++kk) {
            float a[4], bb[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][tm + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) bb[j] = Bs[kk][tn + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(a[i], bb[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int64_t m = m0 + tm + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int64_t nc = n0 + tn + j;
            if (nc >= N) continue;
            float v = acc[i][j];
            if (epi == kEpiBias || epi == kEpiBiasRelu) v += aux[nc];
            if (epi == kEpiBiasRelu) v = fmaxf(v, 0.0f);
            if (epi == kEpiMask && !(aux[m * N + nc] > 0.0f)) v = 0.0f;
            C[m * N + nc] = v;
        }
    }
}

template <class TA, class TB>
cudaError_t gemm(const TA* A, int64_t sam, int64_t sak, const TB* B, int64_t sbk, int64_t sbn, float* C, int64_t M,
                 int64_t N, int64_t K, int epi, const float* aux, cudaStream_t st) {
    if (M <= 0 || N <= 0) return cudaSuccess;
    dim3 grid((unsigned)((N + kBN - 1) / kBN), (unsigned)((M + kBM - 1) / kBM));
    k_gemm<TA, TB><<<grid, 256, 0, st>>>(A, sam, sak, B, sbk, sbn, C, M, N, K, epi, aux);
    return cudaGetLastError();
}

// z[s] = h2[s] . w3 + b3: one warp per row.
__global__ void k_out(const float* __restrict__ h2, const __nv_bfloat16* __restrict__ w3, const float* __restrict__ b3,
                      int64_t n, int dh, float* __restrict__ z) {
    const int64_t s = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= n) return;
    float acc = 0.0f;
    for (int j = lane; j < dh; j += 32) acc = fmaf(h2[s * dh + j], __bfloat162float(w3[j]), acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xFFFFFFFFu, acc, o);
    if (lane == 0) z[s] = acc + b3[0];
}

// Weighted binary cross-entropy with logits, mean over n: per row the loss
// w*(softplus(z) - y*z) with w = pos_weight for y = 1, 1 otherwise, and
// dz = w*(sigmoid(z) - y)/n.  The loss sum goes to *loss (atomic).
__global__ void k_bce(const float* __restrict__ z, const float* __restrict__ y, int64_t n, float pos_weight,
                      float* __restrict__ dz, float* __restrict__ loss) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.0f;
    if (s < n) {
        const float zz = z[s], yy = y[s];
        const float w = yy > 0.5f ? pos_weight : 1.0f;
        const float sp = zz > 0.0f ? zz + log1pf(expf(-zz)) : log1pf(expf(zz));   // softplus(z)
        l = w * (sp - yy * zz) / (float)n;
        const float sg = 1.0f / (1.0f + expf(-zz));
        dz[s] = w * (sg - yy) / (float)n;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xFFFFFFFFu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// dh2[s][j] = dz[s] * w3[j], masked by h2[s][j] > 0 (ReLU).
__global__ void k_dh2(const float* __restrict__ dz, const __nv_bfloat16* __restrict__ w3,
                      const float* __restrict__ h2, int64_t n, int dh, float* __restrict__ dh2) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * dh) return;
    const int64_t s = i / dh;
    const int j = (int)(i - s * dh);
    dh2[i] = h2[i] > 0.0f ? dz[s] * __bfloat162float(w3[j]) : 0.0f;
}

// out[j] = sum_s X[s*ld + j] (s < n), j < d: the bias gradients (and dW3 with
// X = h2 scaled by dz through k_colsum_w).
__global__ void k_colsum(const float* __restrict__ X, int64_t n, int d, int64_t ld, const float* __restrict__ w,
                         float* __restrict__ out) {
    __shared__ float red[8][33];
    const int j = blockIdx.x * 32 + (threadIdx.x & 31);
    const int r = threadIdx.x >> 5;   // 8 row lanes
    float acc = 0.0f;
    if (j < d)
        for (int64_t s = r; s < n; s += 8) acc += X[s * ld + j] * (w ? w[s] : 1.0f);
    red[r][threadIdx.x & 31] = acc;
    __syncthreads();
    if (r == 0 && j < d) {
        float t = 0.0f;
#pragma unroll
        for (int q = 0; q < 8; ++q) t += red[q][threadIdx.x & 31];
        out[j] = t;
    }
}

// Adam on an FP32 master tensor, then its BF16 copy (if any) refreshed.
__global__ void k_adam(float* __restrict__ p, __nv_bfloat16* __restrict__ pb, float* __restrict__ m1,
                       float* __restrict__ m2, const float* __restrict__ g, int64_t n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float a = b1 * m1[i] + (1.0f - b1) * gi;
    const float v = b2 * m2[i] + (1.0f - b2) * gi * gi;
    m1[i] = a;
    m2[i] = v;
    const float upd = lr * (a / c1) / (sqrtf(v / c2) + eps);
    p[i] -= upd;
    if (pb) pb[i] = __float2bfloat16_rn(p[i]);
}

__global__ void k_to_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ pb, int64_t n) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pb[i] = __float2bfloat16_rn(p[i]);
}

inline unsigned nblk(int64_t n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

cudaError_t launch_features(const float2* amps, int64_t namps, double r_lo, double lodr, int64_t Nprof, int64_t total,
                            const DevLevel* levels, int nlev, int nfeat, float* out, cudaStream_t st) {
    const int64_t nb = (total + Nprof - 1) / Nprof;
    if (nb <= 0) return cudaSuccess;
    if (nfeat > kFeatMax) return cudaErrorInvalidValue;
    k_features<<<(unsigned)nb, kFeatThreads, 0, st>>>(amps, namps, r_lo, lodr, Nprof, total, levels, nlev, nfeat, out);
    return cudaGetLastError();
}

cudaError_t launch_mlp_forward(const cs_mlp& net, const float* x, int64_t n, float* h1, float* h2, float* z,
                               cudaStream_t st) {
    const auto* w1 = reinterpret_cast<const __nv_bfloat16*>(net.w1);
    const auto* w2 = reinterpret_cast<const __nv_bfloat16*>(net.w2);
    const auto* w3 = reinterpret_cast<const __nv_bfloat16*>(net.w3);
    const int din = net.din, dh = net.dh;
    cudaError_t e = gemm<float, __nv_bfloat16>(x, din, 1, w1, 1, din, h1, n, dh, din, kEpiBiasRelu, net.b1, st);
    if (e == cudaSuccess) e = gemm<float, __nv_bfloat16>(h1, dh, 1, w2, 1, dh, h2, n, dh, dh, kEpiBiasRelu, net.b2, st);
    if (e == cudaSuccess && n > 0) {
        k_out<<<nblk(n * 32, 256), 256, 0, st>>>(h2, w3, net.b3, n, dh, z);
        e = cudaGetLastError();
    }
    return e;
}

cudaError_t launch_mlp_backward(const cs_mlp& net, const float* x, const float* h1, const float* h2, const float* z,
                                const float* y, int64_t n, float pos_weight, float* dz, float* dh1, float* dh2,
                                const cs_mlp_grads& g, float* loss, cudaStream_t st) {
    const auto* w2 = reinterpret_cast<const __nv_bfloat16*>(net.w2);
    const auto* w3 = reinterpret_cast<const __nv_bfloat16*>(net.w3);
    const int din = net.din, dh = net.dh;
    if (n <= 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(loss, 0, sizeof(float), st);
    if (e != cudaSuccess) return e;
    k_bce<<<nblk(n, 256), 256, 0, st>>>(z, y, n, pos_weight, dz, loss);
    // output layer: dW3[j] = sum_s dz[s] h2[s][j], db3 = sum_s dz[s]
    k_colsum<<<nblk(dh, 32), 256, 0, st>>>(h2, n, dh, dh, dz, g.w3);
    k_colsum<<<1, 256, 0, st>>>(dz, n, 1, 1, nullptr, g.b3);
    k_dh2<<<nblk(n * dh, 256), 256, 0, st>>>(dz, w3, h2, n, dh, dh2);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // layer 2: dW2 = dh2^T h1, db2 = colsum(dh2), dh1 = (dh2 W2) masked by h1 > 0
    e = gemm<float, float>(dh2, 1, dh, h1, dh, 1, g.w2, dh, dh, n, kEpiNone, nullptr, st);
    if (e != cudaSuccess) return e;
    k_colsum<<<nblk(dh, 32), 256, 0, st>>>(dh2, n, dh, dh, nullptr, g.b2);
    e = gemm<float, __nv_bfloat16>(dh2, dh, 1, w2, dh, 1, dh1, n, dh, dh, kEpiMask, h1, st);
    if (e != cudaSuccess) return e;
    // layer 1: dW1 = dh1^T x, db1 = colsum(dh1)
    e = gemm<float, float>(dh1, 1, dh, x, din, 1, g.w1, dh, din, n, kEpiNone, nullptr, st);
    if (e != cudaSuccess) return e;
    k_colsum<<<nblk(dh, 32), 256, 0, st>>>(dh1, n, dh, dh, nullptr, g.b1);
    return cudaGetLastError();
}

cudaError_t launch_adam(const cs_adam_param& p, float lr, float b1, float b2, float eps, int step, cudaStream_t st) {
    if (p.n <= 0) return cudaSuccess;
    const float c1 = 1.0f - std::pow(b1, (float)step), c2 = 1.0f - std::pow(b2, (float)step);
    k_adam<<<nblk(p.n, 256), 256, 0, st>>>(p.master, reinterpret_cast<__nv_bfloat16*>(p.bf16), p.m, p.v, p.grad, p.n,
                                           lr, b1, b2, eps, c1, c2);
    return cudaGetLastError();
}

cudaError_t launch_to_bf16(const float* p, uint16_t* pb, int64_t n, cudaStream_t st) {
    if (n <= 0) return cudaSuccess;
    k_to_bf16<<<nblk(n, 256), 256, 0, st>>>(p, reinterpret_cast<__nv_bfloat16*>(pb), n);
    return cudaGetLastError();
}

}  // namespace cs

// ---------------------------------------------------------------------------
// C ABI (declared in cohsearch.h)
// ---------------------------------------------------------------------------
extern "C" {

static cs_status mlp_status(cudaError_t e) { return e == cudaSuccess ? CS_OK : CS_ERR_CUDA; }

static bool mlp_ok(const cs_mlp* net) {
    return net && net->din > 0 && net->dh > 0 && net->w1 && net->b1 && net->w2 && net->b2 && net->w3 && net->b3;
}

cs_status cs_mlp_forward(const cs_mlp* net, const float* d_x, int64_t n, float* d_h1, float* d_h2, float* d_z,
                         void* stream) {
    if (!mlp_ok(net) || n < 0 || (n > 0 && (!d_x || !d_h1 || !d_h2 || !d_z))) return CS_ERR_INVALID_ARGUMENT;
    return mlp_status(cs::launch_mlp_forward(*net, d_x, n, d_h1, d_h2, d_z, static_cast<cudaStream_t>(stream)));
}

cs_status cs_mlp_backward(const cs_mlp* net, const float* d_x, const float* d_h1, const float* d_h2,
                          const float* d_z, const float* d_y, int64_t n, float pos_weight, float* d_dz, float* d_dh1,
                          float* d_dh2, const cs_mlp_grads* grads, float* d_loss, void* stream) {
    if (!mlp_ok(net) || !grads || n < 0 || !d_loss || !(pos_weight > 0.0f)) return CS_ERR_INVALID_ARGUMENT;
    if (n > 0 && (!d_x || !d_h1 || !d_h2 || !d_z || !d_y || !d_dz || !d_dh1 || !d_dh2)) return CS_ERR_INVALID_ARGUMENT;
    if (!grads->w1 || !grads->b1 || !grads->w2 || !grads->b2 || !grads->w3 || !grads->b3) return CS_ERR_INVALID_ARGUMENT;
    return mlp_status(cs::launch_mlp_backward(*net, d_x, d_h1, d_h2, d_z, d_y, n, pos_weight, d_dz, d_dh1, d_dh2,
                                              *grads, d_loss, static_cast<cudaStream_t>(stream)));
}

cs_status cs_adam_step(const cs_adam_param* params, int32_t nparams, float lr, float beta1, float beta2, float eps,
                       int32_t step, void* stream) {
    if (!params || nparams < 0 || step < 1) return CS_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < nparams; ++i) {
        const cs_adam_param& p = params[i];
        if (p.n < 0 || (p.n > 0 && (!p.master || !p.m || !p.v || !p.grad))) return CS_ERR_INVALID_ARGUMENT;
        const cudaError_t e = cs::launch_adam(p, lr, beta1, beta2, eps, step, static_cast<cudaStream_t>(stream));
        if (e != cudaSuccess) return CS_ERR_CUDA;
    }
    return CS_OK;
}

cs_status cs_mlp_to_bf16(const float* d_src, uint16_t* d_dst, int64_t n, void* stream) {
    if (n < 0 || (n > 0 && (!d_src || !d_dst))) return CS_ERR_INVALID_ARGUMENT;
    return mlp_status(cs::launch_to_bf16(d_src, d_dst, n, static_cast<cudaStream_t>(stream)));
}

}  // extern "C"
