// k_mlp.cu -- training and inference of the barotropic surrogate network.
//
// Network: x (175 features, padded to 176) -> Z1 = W1 x + b1 -> H1 = GELU(Z1)
// -> Z2 = W2 H1 + b2 -> H2 = GELU(Z2) -> out = W3 H2 + b3 (2 outputs); weights
// and activations feed the tensor cores as bf16 and every sum accumulates in
// fp32.  GELU is the tanh form 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))
// (Hendrycks & Gimpel, 2016).  Loss: mean squared error over the batch and
// both outputs.  Adam (Kingma & Ba, 2015) with bias correction updates fp32
// master weights, from which the bf16 operand copies are made.
//
// Tensor-core GEMMs (mlp_gemm.cuh), all "A[M x K] times B[N x K]^T" with K
// contiguous in both operands:
//   forward  Z1 = X W1^T           (A = X [B][176],   B = W1 [256][176])
//            Z2 = H1 W2^T  (+ W3)  (A = H1 [B][256],  B = W2 [256][256]), the
//                                   output layer folded into the epilogue
//   backward dH1 = dZ2 W2          (A = dZ2 [B][256], B = W2^T [256][256])
//            dW2 = dZ2^T H1        (A = dZ2^T [256][B], B = H1^T [256][B]), split-K
//            dW1 = dZ1^T X         (A = dZ1^T [256][B], B = X^T [176][B]),   split-K
// so the forward epilogues also write the transposed activations the weight
// gradients read.  The rank-2 output layer's backward, the bias gradients,
// the split-K reductions and Adam run on the CUDA cores.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "mlp.h"
#include "mlp_gemm.cuh"

namespace mom6b {

__device__ __forceinline__ float gelu_f(float z)
{
    const float c = 0.7978845608028654f;   // sqrt(2 / pi)
    const float t = tanhf(c * (z + 0.044715f * z * z * z));
    return 0.5f * z * (1.0f + t);
}

__device__ __forceinline__ float gelu_grad_f(float z)
{
    const float c = 0.7978845608028654f;
    const float z2 = z * z;
    const float t = tanhf(c * (z + 0.044715f * z2 * z));
    return 0.5f * (1.0f + t) + 0.5f * z * (1.0f - t * t) * c * (1.0f + 3.0f * 0.044715f * z2);
}

// ---- tensor-core layers -----------------------------------------------------
// Hidden layer: Z = acc + bias, H = GELU(Z) as bf16 (row-major and/or
// transposed); with out != nullptr also the output layer out = W3 H + b3 of
// the CTA's rows (N = 256 in one CTA).
template <int BN>
__global__ void __launch_bounds__(kGemmThreads, 2)
k_mlp_hidden(const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mB,
             int M, int N, int K, const float* __restrict__ bias, float* Z,
             __nv_bfloat16* H, __nv_bfloat16* HT, int ldt, const float* __restrict__ W3r,
             const float* __restrict__ b3, float* out, int* err)
{
    float o0 = 0.f, o1 = 0.f;
    gemm_tile<BN, kGemmStagesShort>(&mA, &mB, M, N, K, K, err, [&](int m, int n, const float* v) {
        // the thread's 16 consecutive columns: 64 B of Z and 32 B of H, stored
        // as 16-byte vectors (n is a multiple of 16)
        __align__(16) float z[16];
        __align__(16) __nv_bfloat16 hb[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            z[q] = v[q] + bias[n + q];
            hb[q] = __float2bfloat16_rn(gelu_f(z[q]));
        }
        if (Z) {
            float4* zd = (float4*)(Z + (size_t)m * N + n);
#pragma unroll
            for (int q = 0; q < 4; ++q) zd[q] = ((const float4*)z)[q];
        }
        if (H) {
            uint4* hd = (uint4*)(H + (size_t)m * N + n);
            hd[0] = ((const uint4*)hb)[0];
            hd[1] = ((const uint4*)hb)[1];
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            if (HT) HT[(size_t)(n + q) * ldt + m] = hb[q];
            if (out) {
                const float hr = __bfloat162float(hb[q]);
                o0 += hr * W3r[n + q];
                o1 += hr * W3r[N + n + q];
            }
        }
    });
    const int row = (int)blockIdx.x * kGemmBM + (int)threadIdx.x;
    if (out && row < M) {
        out[(size_t)row * 2] = o0 + b3[0];
        out[(size_t)row * 2 + 1] = o1 + b3[1];
    }
}

// Backward through a hidden layer: dZ = acc * GELU'(Z), stored transposed.
template <int BN>
__global__ void __launch_bounds__(kGemmThreads, 2)
k_mlp_dgelu(const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mB,
            int M, int N, int K, const float* __restrict__ Z, __nv_bfloat16* dZT, int ldt,
            int* err)
{
    gemm_tile<BN, kGemmStagesShort>(&mA, &mB, M, N, K, K, err, [&](int m, int n, const float* v) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            const float dz = v[q] * gelu_grad_f(Z[(size_t)m * N + n + q]);
            dZT[(size_t)(n + q) * ldt + m] = __float2bfloat16_rn(dz);
        }
    });
}

// Weight gradient, split-K partial sums part[z][m][n].
template <int BN>
__global__ void __launch_bounds__(kGemmThreads, 1)
k_mlp_wgrad(const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mB,
            int M, int N, int K, int kps, float* part, int* err)
{
    float* P = part + (size_t)blockIdx.z * M * N;
    gemm_tile<BN, kGemmStages>(&mA, &mB, M, N, K, kps, err, [&](int m, int n, const float* v) {
        float4* pd = (float4*)(P + (size_t)m * N + n);
#pragma unroll
        for (int q = 0; q < 4; ++q) pd[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    });
}

// ---- CUDA-core kernels ------------------------------------------------------
// Output layer backward for 32 rows per CTA (thread = hidden unit n):
// dOut = (out - y) / B, dZ2 = (W3^T dOut) * GELU'(Z2) (bf16, both layouts),
// and per-CTA partial sums of db2, dW3, db3 and the loss.
constexpr int kOutRows = 32;
constexpr int kOutPart = 3 * kMlpHidden + 3;

__global__ void __launch_bounds__(kMlpHidden)
k_mlp_out_bwd(int B, const float* __restrict__ out, const float* __restrict__ Y,
              const float* __restrict__ Z2, const __nv_bfloat16* __restrict__ H2,
              const float* __restrict__ W3r, __nv_bfloat16* dZ2, __nv_bfloat16* dZ2T,
              float* bpart)
{
    __shared__ float sdo[kOutRows][2];
    __shared__ __align__(16) __nv_bfloat16 tile[kMlpHidden][kOutRows + 8];
    __shared__ float sl[kOutRows];
    const int n = (int)threadIdx.x;
    const int r0 = (int)blockIdx.x * kOutRows;
    const float invB = 1.0f / (float)B;
    if (n < 2 * kOutRows) {
        const int r = n >> 1, o = n & 1, m = r0 + r;
        float d = 0.f;
        if (m < B) d = (out[(size_t)m * 2 + o] - Y[(size_t)m * 2 + o]);
        sdo[r][o] = d * invB;
        float sq = d * d;
        sq += __shfl_xor_sync(0xffffffffu, sq, 1);
        if (o == 0) sl[r] = sq;
    }
    __syncthreads();
    float adb2 = 0.f, aw0 = 0.f, aw1 = 0.f;
    const float w0 = W3r[n], w1 = W3r[kMlpHidden + n];
    for (int r = 0; r < kOutRows; ++r) {
        const int m = r0 + r;
        __nv_bfloat16 db = __float2bfloat16_rn(0.f);
        if (m < B) {
            const size_t o = (size_t)m * kMlpHidden + n;
            const float dh = sdo[r][0] * w0 + sdo[r][1] * w1;
            db = __float2bfloat16_rn(dh * gelu_grad_f(Z2[o]));
            dZ2[o] = db;
            const float h = __bfloat162float(H2[o]);
            adb2 += __bfloat162float(db);
            aw0 += sdo[r][0] * h;
            aw1 += sdo[r][1] * h;
        }
        tile[n][r] = db;
    }
    __syncthreads();
    // transposed rows: dZ2T[n][r0 .. r0+31]
    if (r0 + kOutRows <= B) {
        const uint4* src = (const uint4*)&tile[n][0];
        uint4* dst = (uint4*)(dZ2T + (size_t)n * B + r0);
#pragma unroll
        for (int q = 0; q < kOutRows / 8; ++q) dst[q] = src[q];
    } else {
        for (int r = 0; r < kOutRows && r0 + r < B; ++r) dZ2T[(size_t)n * B + r0 + r] = tile[n][r];
    }
    float* bp = bpart + (size_t)blockIdx.x * kOutPart;
    bp[n] = adb2;
    bp[kMlpHidden + n] = aw0;
    bp[2 * kMlpHidden + n] = aw1;
    if (n == 0) {
        float s0 = 0.f, s1 = 0.f, sq = 0.f;
        for (int r = 0; r < kOutRows; ++r) {
            s0 += sdo[r][0];
            s1 += sdo[r][1];
            sq += sl[r];
        }
        bp[3 * kMlpHidden] = s0;
        bp[3 * kMlpHidden + 1] = s1;
        bp[3 * kMlpHidden + 2] = sq;
    }
}

// Sum the output-layer partials of nb CTAs into the gradient (db2, dW3, db3)
// and the loss = sum (out - y)^2 / (2 B).
__global__ void k_mlp_out_reduce(int nb, int B, const float* __restrict__ bpart, float* G,
                                 float* loss)
{
    const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (t >= kOutPart) return;
    float s = 0.f;
    for (int b = 0; b < nb; ++b) s += bpart[(size_t)b * kOutPart + t];
    if (t < kMlpHidden) G[kOffB2 + t] = s;
    else if (t < 3 * kMlpHidden) G[kOffW3 + (t - kMlpHidden)] = s;
    else if (t < 3 * kMlpHidden + 2) G[kOffB3 + (t - 3 * kMlpHidden)] = s;
    else *loss = s / (2.0f * (float)B);
}

// Split-K reduction: G[off + m * N + n] = sum_z part[z][m][n].
__global__ void k_mlp_splitk_reduce(int S, int MN, const float* __restrict__ part, float* G,
                                    int off)
{
    const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (t >= MN) return;
    float s = 0.f;
    for (int z = 0; z < S; ++z) s += part[(size_t)z * MN + t];
    G[off + t] = s;
}

// db1[h] = sum_b dZ1T[h][b], one CTA per hidden unit.
__global__ void __launch_bounds__(256)
k_mlp_rowsum(int B, const __nv_bfloat16* __restrict__ dZT, float* G, int off)
{
    __shared__ float red[256];
    const __nv_bfloat16* row = dZT + (size_t)blockIdx.x * B;
    float s = 0.f;
    for (int b = (int)threadIdx.x; b < B; b += 256) s += __bfloat162float(row[b]);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) G[off + blockIdx.x] = red[0];
}

// Adam on the flat fp32 parameters; lr_t carries the bias corrections.
__global__ void k_mlp_adam(int n, float* P, const float* __restrict__ G, float* Mo, float* Vo,
                           float lr_t, float b1, float b2, float eps)
{
    const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (t >= n) return;
    const float g = G[t];
    const float m = b1 * Mo[t] + (1.0f - b1) * g;
    const float v = b2 * Vo[t] + (1.0f - b2) * g * g;
    Mo[t] = m;
    Vo[t] = v;
    P[t] -= lr_t * m / (sqrtf(v) + eps);
}

// bf16 operand copies of the fp32 weights: W1 [256][176], W2 [256][256] and
// its transpose, and W3 rounded to bf16 (kept as fp32).
__global__ void k_mlp_bf16(const float* __restrict__ P, __nv_bfloat16* W1b, __nv_bfloat16* W2b,
                           __nv_bfloat16* W2Tb, float* W3r)
{
    const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (t < kMlpHidden * kMlpInPad) W1b[t] = __float2bfloat16_rn(P[kOffW1 + t]);
    if (t < kMlpHidden * kMlpHidden) {
        const int r = t / kMlpHidden, c = t - r * kMlpHidden;
        const __nv_bfloat16 w = __float2bfloat16_rn(P[kOffW2 + t]);
        W2b[t] = w;
        W2Tb[(size_t)c * kMlpHidden + r] = w;
    }
    if (t < kMlpOut * kMlpHidden) W3r[t] = __bfloat162float(__float2bfloat16_rn(P[kOffW3 + t]));
}

// ---- host side ----------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// Tensor map of a row-major bf16 matrix [rows][cols] (cols contiguous) read in
// boxes of 64 columns x box_rows rows with the 128-byte swizzle.
static cudaError_t map_bf16(CUtensorMap* m, const void* base, uint64_t rows, uint64_t cols,
                            uint32_t box_rows)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn) return cudaErrorNotSupported;
    if (((uintptr_t)base & 15u) || (cols * 2) % 16 || box_rows > 256) return cudaErrorInvalidValue;
    cuuint64_t gdim[2] = {cols, rows};
    cuuint64_t gstride[1] = {cols * 2};
    cuuint32_t box[2] = {(cuuint32_t)kGemmBK, box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), gdim, gstride,
                    box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <class T>
static cudaError_t dev_alloc(T** p, size_t n)
{
    cudaError_t e = cudaMalloc((void**)p, n * sizeof(T) + 256);
    if (e == cudaSuccess) e = cudaMemset(*p, 0, n * sizeof(T) + 256);
    return e;
}

#define MLP_CK(x)                                  \
    do {                                           \
        cudaError_t e_ = (x);                      \
        if (e_ != cudaSuccess) return e_;          \
    } while (0)

Mlp::~Mlp()
{
    void* ptrs[] = {X, XT, Y, amp, gacc, out, loss, err, Xi, outi, ampi, d_norm, P, G, Mo, Vo, W1b,
                    W2b, W2Tb, W3r, Z1, Z2, H1, H1T, H2, dZ2, dZ2T, dZ1T, part, bpart, H1i};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}

// split count of the batch reduction of a weight gradient: K chunks that are
// whole 64-wide steps, about 64 of them
static int splitk_kps(int B)
{
    int kps = (B + 63) / 64;
    kps = ((kps + kGemmBK - 1) / kGemmBK) * kGemmBK;
    return kps < kGemmBK ? kGemmBK : kps;
}

cudaError_t Mlp::init(int batch, uint64_t seed, cudaStream_t s)
{
    if (batch < 128 || batch % 8) return cudaErrorInvalidValue;
    B_cap = batch;
    const size_t B = (size_t)batch;
    MLP_CK(dev_alloc(&P, kMlpParams));
    MLP_CK(dev_alloc(&G, kMlpParams));
    MLP_CK(dev_alloc(&Mo, kMlpParams));
    MLP_CK(dev_alloc(&Vo, kMlpParams));
    MLP_CK(dev_alloc(&W1b, (size_t)kMlpHidden * kMlpInPad));
    MLP_CK(dev_alloc(&W2b, (size_t)kMlpHidden * kMlpHidden));
    MLP_CK(dev_alloc(&W2Tb, (size_t)kMlpHidden * kMlpHidden));
    MLP_CK(dev_alloc(&W3r, (size_t)kMlpOut * kMlpHidden));
    MLP_CK(dev_alloc(&X, B * kMlpInPad));
    MLP_CK(dev_alloc(&XT, B * kMlpInPad));
    MLP_CK(dev_alloc(&Y, B * kMlpOut));
    MLP_CK(dev_alloc(&amp, B));
    MLP_CK(dev_alloc(&gacc, 4));
    MLP_CK(dev_alloc(&out, B * kMlpOut));
    MLP_CK(dev_alloc(&loss, 4));
    MLP_CK(dev_alloc(&err, 4));
    MLP_CK(dev_alloc(&d_norm, 16));
    MLP_CK(dev_alloc(&Z1, B * kMlpHidden));
    MLP_CK(dev_alloc(&Z2, B * kMlpHidden));
    MLP_CK(dev_alloc(&H1, B * kMlpHidden));
    MLP_CK(dev_alloc(&H1T, B * kMlpHidden));
    MLP_CK(dev_alloc(&H2, B * kMlpHidden));
    MLP_CK(dev_alloc(&dZ2, B * kMlpHidden));
    MLP_CK(dev_alloc(&dZ2T, B * kMlpHidden));
    MLP_CK(dev_alloc(&dZ1T, B * kMlpHidden));
    // kps >= B / 64, so a batch never has more than 64 splits
    MLP_CK(dev_alloc(&part, (size_t)64 * kMlpHidden * kMlpHidden));
    MLP_CK(dev_alloc(&bpart, (size_t)((batch + kOutRows - 1) / kOutRows) * kOutPart));
    // weights: uniform in +-1/sqrt(fan_in) from a splitmix64 stream; biases
    // zero; the padded input column of W1 stays zero
    std::vector<float> h(kMlpParams, 0.0f);
    uint64_t st = seed * 0x9E3779B97F4A7C15ULL + 0x1234567ULL;
    auto uni = [&]() {
        st += 0x9E3779B97F4A7C15ULL;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    };
    for (int r = 0; r < kMlpHidden; ++r)
        for (int c = 0; c < kMlpIn; ++c)
            h[kOffW1 + r * kMlpInPad + c] = (float)(uni() / std::sqrt((double)kMlpIn));
    for (int q = 0; q < kMlpHidden * kMlpHidden; ++q)
        h[kOffW2 + q] = (float)(uni() / std::sqrt((double)kMlpHidden));
    for (int q = 0; q < kMlpOut * kMlpHidden; ++q)
        h[kOffW3 + q] = (float)(uni() / std::sqrt((double)kMlpHidden));
    MLP_CK(cudaMemcpy(P, h.data(), kMlpParams * sizeof(float), cudaMemcpyHostToDevice));
    float nrm[16] = {0};
    for (int c = 0; c < kMlpChannels; ++c) nrm[c] = 1.0f / feat_std[c];
    nrm[7] = targ_std[0];
    nrm[8] = targ_std[1];
    MLP_CK(cudaMemcpy(d_norm, nrm, sizeof(nrm), cudaMemcpyHostToDevice));
    MLP_CK(bf16_copies(s));
    MLP_CK(cudaStreamSynchronize(s));
    return make_maps(batch);
}

cudaError_t Mlp::make_maps(int B)
{
    MLP_CK(map_bf16(&mX, X, B, kMlpInPad, kGemmBM));
    MLP_CK(map_bf16(&mH1, H1, B, kMlpHidden, kGemmBM));
    MLP_CK(map_bf16(&mdZ2, dZ2, B, kMlpHidden, kGemmBM));
    MLP_CK(map_bf16(&mdZ2T, dZ2T, kMlpHidden, B, kGemmBM));
    MLP_CK(map_bf16(&mdZ1T, dZ1T, kMlpHidden, B, kGemmBM));
    MLP_CK(map_bf16(&mW1, W1b, kMlpHidden, kMlpInPad, kMlpHidden));
    MLP_CK(map_bf16(&mW2, W2b, kMlpHidden, kMlpHidden, kMlpHidden));
    MLP_CK(map_bf16(&mW2T, W2Tb, kMlpHidden, kMlpHidden, kMlpHidden));
    MLP_CK(map_bf16(&mH1T_B, H1T, kMlpHidden, B, kMlpHidden));
    MLP_CK(map_bf16(&mXT_B, XT, kMlpInPad, B, kMlpInPad));
    maps_ok = true;
    map_B = B;
    return cudaSuccess;
}

cudaError_t Mlp::bf16_copies(cudaStream_t s)
{
    const int n = kMlpHidden * kMlpHidden;
    k_mlp_bf16<<<(n + 255) / 256, 256, 0, s>>>(P, W1b, W2b, W2Tb, W3r);
    ++launches;
    return cudaGetLastError();
}

cudaError_t Mlp::get_params(float* host) const
{
    return cudaMemcpy(host, P, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost);
}

cudaError_t Mlp::set_params(const float* host)
{
    MLP_CK(cudaMemcpy(P, host, kMlpParams * sizeof(float), cudaMemcpyHostToDevice));
    MLP_CK(bf16_copies(0));
    return cudaDeviceSynchronize();
}

template <class Kern>
static cudaError_t gemm_attr(Kern k, int bn, int stages)
{
    return cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                gemm_smem_bytes(bn, stages));
}

cudaError_t Mlp::forward(int B, bool keep, cudaStream_t s)
{
    static bool attr = false;
    if (!attr) {
        MLP_CK(gemm_attr(k_mlp_hidden<kMlpHidden>, kMlpHidden, kGemmStagesShort));
        MLP_CK(gemm_attr(k_mlp_dgelu<kMlpHidden>, kMlpHidden, kGemmStagesShort));
        MLP_CK(gemm_attr(k_mlp_wgrad<kMlpHidden>, kMlpHidden, kGemmStages));
        MLP_CK(gemm_attr(k_mlp_wgrad<kMlpInPad>, kMlpInPad, kGemmStages));
        attr = true;
    }
    const dim3 grid((B + kGemmBM - 1) / kGemmBM, 1, 1);
    const int sm = gemm_smem_bytes(kMlpHidden, kGemmStagesShort);
    k_mlp_hidden<kMlpHidden><<<grid, kGemmThreads, sm, s>>>(
        mX, mW1, B, kMlpHidden, kMlpInPad, P + kOffB1, keep ? Z1 : nullptr, H1,
        keep ? H1T : nullptr, B, nullptr, nullptr, nullptr, err);
    k_mlp_hidden<kMlpHidden><<<grid, kGemmThreads, sm, s>>>(
        mH1, mW2, B, kMlpHidden, kMlpHidden, P + kOffB2, keep ? Z2 : nullptr,
        keep ? H2 : nullptr, nullptr, B, W3r, P + kOffB3, out, err);
    launches += 2;
    return cudaGetLastError();
}

cudaError_t Mlp::backward(int B, cudaStream_t s)
{
    const int nb = (B + kOutRows - 1) / kOutRows;
    k_mlp_out_bwd<<<nb, kMlpHidden, 0, s>>>(B, out, Y, Z2, H2, W3r, dZ2, dZ2T, bpart);
    k_mlp_out_reduce<<<(kOutPart + 255) / 256, 256, 0, s>>>(nb, B, bpart, G, loss);
    // dH1 = dZ2 W2, dZ1 = dH1 * GELU'(Z1) (transposed)
    const dim3 grid((B + kGemmBM - 1) / kGemmBM, 1, 1);
    k_mlp_dgelu<kMlpHidden><<<grid, kGemmThreads, gemm_smem_bytes(kMlpHidden, kGemmStagesShort), s>>>(
        mdZ2, mW2T, B, kMlpHidden, kMlpHidden, Z1, dZ1T, B, err);
    // weight gradients, split over the batch
    const int kps = splitk_kps(B);
    const int S = (B + kps - 1) / kps;
    k_mlp_wgrad<kMlpHidden><<<dim3(kMlpHidden / kGemmBM, 1, S), kGemmThreads,
                              gemm_smem_bytes(kMlpHidden, kGemmStages), s>>>(mdZ2T, mH1T_B, kMlpHidden,
                                                                kMlpHidden, B, kps, part, err);
    k_mlp_splitk_reduce<<<(kMlpHidden * kMlpHidden + 255) / 256, 256, 0, s>>>(
        S, kMlpHidden * kMlpHidden, part, G, kOffW2);
    k_mlp_wgrad<kMlpInPad><<<dim3(kMlpHidden / kGemmBM, 1, S), kGemmThreads,
                             gemm_smem_bytes(kMlpInPad, kGemmStages), s>>>(mdZ1T, mXT_B, kMlpHidden,
                                                              kMlpInPad, B, kps, part, err);
    k_mlp_splitk_reduce<<<(kMlpHidden * kMlpInPad + 255) / 256, 256, 0, s>>>(
        S, kMlpHidden * kMlpInPad, part, G, kOffW1);
    k_mlp_rowsum<<<kMlpHidden, 256, 0, s>>>(B, dZ1T, G, kOffB1);
    launches += 8;
    return cudaGetLastError();
}

cudaError_t Mlp::gradients(int B, cudaStream_t s)
{
    if (B > B_cap || B < 128 || B % 8 || !maps_ok) return cudaErrorInvalidValue;
    if (B != map_B) MLP_CK(make_maps(B));   // the transposed buffers' row stride is B
    MLP_CK(forward(B, true, s));
    return backward(B, s);
}

cudaError_t Mlp::grads_to_host(float* host, cudaStream_t s) const
{
    MLP_CK(cudaStreamSynchronize(s));
    return cudaMemcpy(host, G, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost);
}

cudaError_t Mlp::train_step(int B, float lr, cudaStream_t s)
{
    MLP_CK(gradients(B, s));
    ++steps;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const double t = (double)steps;
    const float lr_t = (float)(lr * std::sqrt(1.0 - std::pow((double)b2, t)) /
                               (1.0 - std::pow((double)b1, t)));
    k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, s>>>(kMlpParams, P, G, Mo, Vo, lr_t, b1, b2,
                                                        eps);
    ++launches;
    return bf16_copies(s);
}

cudaError_t Mlp::prepare_inference(int n)
{
    if (n <= ni_cap && imaps_ok) return cudaSuccess;
    if (Xi) cudaFree(Xi);
    if (outi) cudaFree(outi);
    if (H1i) cudaFree(H1i);
    if (ampi) cudaFree(ampi);
    Xi = nullptr; outi = nullptr; H1i = nullptr; ampi = nullptr;
    const int cap = ((n + kGemmBM - 1) / kGemmBM) * kGemmBM;
    MLP_CK(dev_alloc(&Xi, (size_t)cap * kMlpInPad));
    MLP_CK(dev_alloc(&outi, (size_t)cap * kMlpOut));
    MLP_CK(dev_alloc(&ampi, (size_t)cap));
    MLP_CK(dev_alloc(&H1i, (size_t)cap * kMlpHidden));
    MLP_CK(map_bf16(&mXi, Xi, cap, kMlpInPad, kGemmBM));
    MLP_CK(map_bf16(&mH1i, H1i, cap, kMlpHidden, kGemmBM));
    ni_cap = cap;
    imaps_ok = true;
    return cudaSuccess;
}

cudaError_t Mlp::predict(int n, cudaStream_t s)
{
    if (n > ni_cap || !imaps_ok) return cudaErrorInvalidValue;
    const dim3 grid((n + kGemmBM - 1) / kGemmBM, 1, 1);
    const int sm = gemm_smem_bytes(kMlpHidden, kGemmStagesShort);
    k_mlp_hidden<kMlpHidden><<<grid, kGemmThreads, sm, s>>>(
        mXi, mW1, n, kMlpHidden, kMlpInPad, P + kOffB1, nullptr, H1i, nullptr, n, nullptr,
        nullptr, nullptr, err);
    k_mlp_hidden<kMlpHidden><<<grid, kGemmThreads, sm, s>>>(
        mH1i, mW2, n, kMlpHidden, kMlpHidden, P + kOffB2, nullptr, nullptr, nullptr, n, W3r,
        P + kOffB3, outi, err);
    launches += 2;
    return cudaGetLastError();
}

// ---- surrogate kernels ----------------------------------------------------------
__host__ __device__ inline uint64_t sur_mix(uint64_t z)
{
    z += 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Cell of sample s: uniform over the compute domain.
__device__ __forceinline__ void sur_sample(const Dims& D, uint64_t seed, int s, int& i, int& j)
{
    const int nx = D.ie - D.is + 1, ny = D.je - D.js + 1;
    const uint64_t h = sur_mix(seed * 0x100000001B3ULL + (uint64_t)s);
    const int idx = (int)((h >> 11) % (uint64_t)(nx * ny));
    i = D.is + idx % nx;
    j = D.js + idx / nx;
}

// Amplitude of the dynamic channels (eta, ubt, vbt, each divided by its
// channel std) over the 5 x 5 stencil of cell (i, j): their RMS.  The
// barotropic equations are linear in (eta, ubt, vbt), so the averaged
// transports are homogeneous of degree one in them; the network sees the
// stencil divided by this amplitude and its outputs are scaled back by it.
// gacc holds the sum of squares and the count of the same quantities over the
// whole compute domain (k_sur_amp_reduce); a tenth of their RMS floors the
// amplitude, so that a cell whose stencil is quiet while transports arrive
// from beyond it is not divided by (nearly) zero.
__device__ __forceinline__ float sur_amp(const SurGrid& g, const BtInputs& in,
                                         const float* norm, const double* gacc, int i, int j)
{
    double acc = 0.0;
    for (int r = 0; r < 25; ++r) {
        const int ii = i + r % 5 - 2, jj = j + r / 5 - 2;
        const size_t p = (size_t)(jj - 1) * g.D.n1 + (ii - 1);
        const double e = in.eta[p] * norm[0], u = in.ubt[p] * norm[1], v = in.vbt[p] * norm[2];
        acc += e * e + u * u + v * v;
    }
    const double glob = gacc[1] > 0.0 ? gacc[0] / gacc[1] : 0.0;
    return (float)(sqrt(acc / 75.0 + 0.01 * glob) + 1e-30);
}

__global__ void __launch_bounds__(256)
k_sur_amp_reduce(SurGrid g, BtInputs in, const float* __restrict__ norm, double* gacc)
{
    __shared__ double r0[256];
    const Dims& D = g.D;
    const int nx = D.ie - D.is + 1, ny = D.je - D.js + 1;
    double s0 = 0.0;
    for (int q = (int)(blockIdx.x * blockDim.x + threadIdx.x); q < nx * ny;
         q += (int)(gridDim.x * blockDim.x)) {
        const int i = D.is + q % nx, j = D.js + q / nx;
        const size_t p = (size_t)(j - 1) * D.n1 + (i - 1);
        const double e = in.eta[p] * norm[0], u = in.ubt[p] * norm[1], v = in.vbt[p] * norm[2];
        s0 += (e * e + u * u + v * v) / 3.0;
    }
    r0[threadIdx.x] = s0;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) r0[threadIdx.x] += r0[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicAdd(gacc, r0[0]);
        if (blockIdx.x == 0) atomicAdd(gacc + 1, (double)nx * ny);
    }
}

static cudaError_t sur_amp_reduce(const SurGrid& g, const BtInputs& in, const float* norm,
                                  double* gacc, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(gacc, 0, 2 * sizeof(double), s);
    if (e != cudaSuccess) return e;
    k_sur_amp_reduce<<<148, 256, 0, s>>>(g, in, norm, gacc);
    return cudaGetLastError();
}

// Feature f (channel f / 25, stencil offset f % 25 = (dj + 2) * 5 + (di + 2)) of
// cell (i, j); the dynamic channels are divided by the stencil amplitude amp.
__device__ __forceinline__ float sur_feature(const SurGrid& g, const BtInputs& in,
                                             const float* norm, float amp, int i, int j, int f)
{
    if (f >= kMlpIn) return 0.0f;
    const int c = f / 25, r = f - c * 25;
    const int ii = i + r % 5 - 2, jj = j + r / 5 - 2;
    const size_t p = (size_t)(jj - 1) * g.D.n1 + (ii - 1);
    double v;
    switch (c) {
    case 0: v = in.eta[p]; break;
    case 1: v = in.ubt[p]; break;
    case 2: v = in.vbt[p]; break;
    case 5: v = g.depth; break;
    case 6: v = g.cor[p]; break;
    default: v = 0.0; break;   // barotropic forcing: none in the barotropic solver
    }
    const double x = v * (double)norm[c];
    return (float)(c <= 2 ? x / (double)amp : x);
}

// amplitude of every sample (one thread per sample)
__global__ void k_sur_amp_train(SurGrid g, BtInputs in, const float* __restrict__ norm,
                                const double* __restrict__ gacc, int B, uint64_t seed, float* amp)
{
    const int s = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (s >= B) return;
    int i, j;
    sur_sample(g.D, seed, s, i, j);
    amp[s] = sur_amp(g, in, norm, gacc, i, j);
}

__global__ void k_sur_features_train(SurGrid g, BtInputs in, const float* __restrict__ norm,
                                     const float* __restrict__ amp, int B, uint64_t seed,
                                     __nv_bfloat16* X)
{
    const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);   // B * 176 < 2^31
    if (t >= B * kMlpInPad) return;
    const int s = t / kMlpInPad, f = t - s * kMlpInPad;
    int i, j;
    sur_sample(g.D, seed, s, i, j);
    X[t] = __float2bfloat16_rn(sur_feature(g, in, norm, amp[s], i, j, f));
}

__global__ void k_sur_features_train_t(SurGrid g, BtInputs in, const float* __restrict__ norm,
                                       const float* __restrict__ amp, int B, uint64_t seed,
                                       __nv_bfloat16* XT)
{
    const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (t >= B * kMlpInPad) return;
    const int f = t / B, s = t - f * B;
    int i, j;
    sur_sample(g.D, seed, s, i, j);
    XT[t] = __float2bfloat16_rn(sur_feature(g, in, norm, amp[s], i, j, f));
}

cudaError_t launch_sur_features_train(const SurGrid& g, const BtInputs& in, const float* norm,
                                      double* gacc, int B, uint64_t seed, __nv_bfloat16* X,
                                      __nv_bfloat16* XT, float* amp, cudaStream_t s)
{
    const long long n = (long long)B * kMlpInPad;
    if (n >= (1LL << 31)) return cudaErrorInvalidValue;
    const int nb = 256;
    const unsigned blocks = (unsigned)((n + nb - 1) / nb);
    cudaError_t e = sur_amp_reduce(g, in, norm, gacc, s);
    if (e != cudaSuccess) return e;
    k_sur_amp_train<<<(B + nb - 1) / nb, nb, 0, s>>>(g, in, norm, gacc, B, seed, amp);
    k_sur_features_train<<<blocks, nb, 0, s>>>(g, in, norm, amp, B, seed, X);
    k_sur_features_train_t<<<blocks, nb, 0, s>>>(g, in, norm, amp, B, seed, XT);
    return cudaGetLastError();
}

__global__ void k_sur_targets(SurGrid g, const double* __restrict__ uh_avg,
                              const double* __restrict__ vh_avg, const float* __restrict__ norm,
                              const float* __restrict__ amp, int B, uint64_t seed, float* Y)
{
    const int s = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (s >= B) return;
    int i, j;
    sur_sample(g.D, seed, s, i, j);
    const size_t p = (size_t)(j - 1) * g.D.n1 + (i - 1);
    const double a = (double)amp[s];
    Y[(size_t)s * 2] = (float)(uh_avg[p] / ((double)norm[7] * a));
    Y[(size_t)s * 2 + 1] = (float)(vh_avg[p] / ((double)norm[8] * a));
}

cudaError_t launch_sur_targets(const SurGrid& g, const double* uh_avg, const double* vh_avg,
                               const float* norm, const float* amp, int B, uint64_t seed,
                               float* Y, cudaStream_t s)
{
    k_sur_targets<<<(B + 255) / 256, 256, 0, s>>>(g, uh_avg, vh_avg, norm, amp, B, seed, Y);
    return cudaGetLastError();
}

__global__ void k_sur_amp_all(SurGrid g, BtInputs in, const float* __restrict__ norm,
                              const double* __restrict__ gacc, float* amp)
{
    const int nx = g.D.ie - g.D.is + 1, ny = g.D.je - g.D.js + 1;
    const int s = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (s >= nx * ny) return;
    amp[s] = sur_amp(g, in, norm, gacc, g.D.is + s % nx, g.D.js + s / nx);
}

__global__ void k_sur_features_all(SurGrid g, BtInputs in, const float* __restrict__ norm,
                                   const float* __restrict__ amp, __nv_bfloat16* X)
{
    const int nx = g.D.ie - g.D.is + 1, ny = g.D.je - g.D.js + 1;
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;   // < 2^32 (host checks)
    if (t >= (unsigned)nx * (unsigned)ny * (unsigned)kMlpInPad) return;
    const int s = (int)(t / (unsigned)kMlpInPad), f = (int)(t - (unsigned)s * kMlpInPad);
    const int i = g.D.is + s % nx, j = g.D.js + s / nx;
    X[t] = __float2bfloat16_rn(sur_feature(g, in, norm, amp[s], i, j, f));
}

cudaError_t launch_sur_features_all(const SurGrid& g, const BtInputs& in, const float* norm,
                                    double* gacc, __nv_bfloat16* X, float* amp, cudaStream_t s)
{
    const long long n = (long long)(g.D.ie - g.D.is + 1) * (g.D.je - g.D.js + 1) * kMlpInPad;
    if (n >= (1LL << 32)) return cudaErrorInvalidValue;
    cudaError_t e = sur_amp_reduce(g, in, norm, gacc, s);
    if (e != cudaSuccess) return e;
    const int nc = (g.D.ie - g.D.is + 1) * (g.D.je - g.D.js + 1);
    k_sur_amp_all<<<(nc + 255) / 256, 256, 0, s>>>(g, in, norm, gacc, amp);
    k_sur_features_all<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(g, in, norm, amp, X);
    return cudaGetLastError();
}

__global__ void k_sur_advance(SurGrid g, const float* __restrict__ outi,
                              const float* __restrict__ norm, const float* __restrict__ amp,
                              const double* eta_in, double* eta_out, double* u_av, double* v_av)
{
    const Dims& D = g.D;
    const int p = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (p >= D.n1 * D.n2) return;
    const int i = p % D.n1 + 1, j = p / D.n1 + 1;
    const int nx = D.ie - D.is + 1;
    const double su = (double)norm[7], sv = (double)norm[8];
    // predicted substep-averaged transports on their ranges, zero elsewhere
    auto U = [&](int a, int b) -> double {
        if (a < g.iu0 || a > g.iu1 || b < D.js || b > D.je || a < D.is) return 0.0;
        const size_t q = (size_t)((b - D.js) * nx + (a - D.is));
        return (double)outi[q * 2] * su * (double)amp[q];
    };
    auto V = [&](int a, int b) -> double {
        if (b < g.jv0 || b > g.jv1 || a < D.is || a > D.ie || b < D.js) return 0.0;
        const size_t q = (size_t)((b - D.js) * nx + (a - D.is));
        return (double)outi[q * 2 + 1] * sv * (double)amp[q];
    };
    double e = eta_in[p];
    if (i >= D.is && i <= D.ie && j >= D.js && j <= D.je)
        e = e - g.dt_total * g.IareaT[p] * ((U(i, j) - U(i - 1, j)) + (V(i, j) - V(i, j - 1)));
    eta_out[p] = e;
    const double uu = U(i, j), vv = V(i, j);
    u_av[p] = uu != 0.0 ? uu / g.Datu[p] : 0.0;
    v_av[p] = vv != 0.0 ? vv / g.Datv[p] : 0.0;
}

cudaError_t launch_sur_advance(const SurGrid& g, const float* outi, const float* norm,
                               const float* amp, const double* eta_in, double* eta_out,
                               double* u_av, double* v_av, cudaStream_t s)
{
    const int n = g.D.n1 * g.D.n2;
    k_sur_advance<<<(n + 255) / 256, 256, 0, s>>>(g, outi, norm, amp, eta_in, eta_out, u_av,
                                                  v_av);
    return cudaGetLastError();
}

__global__ void __launch_bounds__(256)
k_sur_diff(Dims D, const double* __restrict__ a, const double* __restrict__ b, double* acc)
{
    __shared__ double r0[256], r1[256];
    double s0 = 0.0, s1 = 0.0;
    const int nx = D.ie - D.is + 1, ny = D.je - D.js + 1;
    for (int q = (int)(blockIdx.x * blockDim.x + threadIdx.x); q < nx * ny;
         q += (int)(gridDim.x * blockDim.x)) {
        const int i = D.is + q % nx, j = D.js + q / nx;
        const size_t p = (size_t)(j - 1) * D.n1 + (i - 1);
        const double d = a[p] - b[p];
        s0 += d * d;
        s1 += b[p] * b[p];
    }
    r0[threadIdx.x] = s0;
    r1[threadIdx.x] = s1;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            r0[threadIdx.x] += r0[threadIdx.x + w];
            r1[threadIdx.x] += r1[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicAdd(acc, r0[0]);
        atomicAdd(acc + 1, r1[0]);
    }
}

__global__ void __launch_bounds__(256)
k_sur_transport_err(SurGrid g, const float* __restrict__ outi, const float* __restrict__ norm,
                    const float* __restrict__ amp, const double* __restrict__ uh,
                    const double* __restrict__ vh, double* acc)
{
    __shared__ double r0[256], r1[256];
    const Dims& D = g.D;
    const int nx = D.ie - D.is + 1, ny = D.je - D.js + 1;
    double s0 = 0.0, s1 = 0.0;
    for (int q = (int)(blockIdx.x * blockDim.x + threadIdx.x); q < nx * ny;
         q += (int)(gridDim.x * blockDim.x)) {
        const int i = D.is + q % nx, j = D.js + q / nx;
        const size_t p = (size_t)(j - 1) * D.n1 + (i - 1);
        const bool inu = i >= g.iu0 && i <= g.iu1, inv = j >= g.jv0 && j <= g.jv1;
        const double a = (double)amp[q];
        const double pu = inu ? (double)outi[(size_t)q * 2] * (double)norm[7] * a : 0.0;
        const double pv = inv ? (double)outi[(size_t)q * 2 + 1] * (double)norm[8] * a : 0.0;
        s0 += (pu - uh[p]) * (pu - uh[p]) + (pv - vh[p]) * (pv - vh[p]);
        s1 += uh[p] * uh[p] + vh[p] * vh[p];
    }
    r0[threadIdx.x] = s0;
    r1[threadIdx.x] = s1;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            r0[threadIdx.x] += r0[threadIdx.x + w];
            r1[threadIdx.x] += r1[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicAdd(acc, r0[0]);
        atomicAdd(acc + 1, r1[0]);
    }
}

cudaError_t launch_sur_transport_err(const SurGrid& g, const float* outi, const float* norm,
                                     const float* amp, const double* uh_avg,
                                     const double* vh_avg, double* acc, cudaStream_t s)
{
    k_sur_transport_err<<<148, 256, 0, s>>>(g, outi, norm, amp, uh_avg, vh_avg, acc);
    return cudaGetLastError();
}

cudaError_t launch_sur_diff(const Dims& D, const double* a, const double* b, double* acc,
                            cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(acc, 0, 2 * sizeof(double), s);
    if (e != cudaSuccess) return e;
    k_sur_diff<<<148, 256, 0, s>>>(D, a, b, acc);
    return cudaGetLastError();
}

} // namespace mom6b
