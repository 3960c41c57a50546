// The surrogate network of the adaptive energy sampler: a fully connected
// GELU network (hidden layers GELU, last layer linear) with BF16 operands and
// FP32 accumulation, trained with Adam on FP32 master weights.  No reference
// counterpart: NEGFtrans samples energies on a uniform grid only
// (main.f90:369-375).
//
// Layout: activations row-major (sample, feature); layer l maps width[l] ->
// width[l+1] with W_l row-major (out, in) and b_l (out).  Packed parameters:
// W_0, b_0, W_1, b_1, ...  Every GEMM is one kernel, C = A B, whose operands
// are read through strides (so the transposes of the backward pass need no
// copies), rounded to BF16 when staged in shared memory, and multiplied on the
// tensor cores with mma.sync m16n8k16 (FP32 accumulate).  The sizes involved
// (width 256, a few thousand samples) make each product a few hundred
// MFLOP: launch- and latency-bound, not tensor-bound.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "negf_mlp.h"

namespace {

constexpr int BM = 64, BN = 64, BK = 32, KP = BK + 8;  // tile and padded k pitch (bf16)
constexpr int GT = 128;                                  // 4 warps, 32x32 each

enum Epi { EPI_STORE = 0, EPI_BIAS = 1, EPI_BIAS_GELU = 2, EPI_GELU_GRAD = 3 };

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * expf(-0.5f * z * z) * 0.39894228040143268f;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat16 a = __float2bfloat16_rn(lo), b = __float2bfloat16_rn(hi);
    return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

struct Gemm {
    const float *A;  // A(m,k) = A[m*sam + k*sak]
    long sam, sak;
    const float *B;  // B(k,n) = B[k*sbk + n*sbn]
    long sbk, sbn;
    float *C;        // C(m,n) = C[m*ldc + n]
    int ldc;
    int M, N, K;
    int epi;
    const float *bias;  // [N]            (EPI_BIAS, EPI_BIAS_GELU)
    float *Z;           // pre-activation (EPI_BIAS_GELU), ld = ldc
    const float *gate;  // gelu'(gate) multiplies C (EPI_GELU_GRAD), ld = ldc
    int kchunk;         // split K: block z covers k in [z*kchunk, (z+1)*kchunk) (0 = all of K)
    long cz;            // split K: block z stores its partial C at C + z*cz (EPI_STORE only)
};

// C = A B with BF16 operands and FP32 accumulation.  Grid (ceil(N/BN), ceil(M/BM),
// K splits); with splits, each z-slice of the grid writes its partial product.
__global__ void __launch_bounds__(GT) k_gemm_bf16(Gemm g) {
    __shared__ __align__(16) __nv_bfloat16 sA[BM * KP];  // [m][k]
    __shared__ __align__(16) __nv_bfloat16 sB[BN * KP];  // [n][k]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
    const int gq = lane >> 2, tq = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[a][b][c] = 0.f;
    const int kbeg = g.kchunk ? blockIdx.z * g.kchunk : 0;
    const int kend = g.kchunk ? min(g.K, kbeg + g.kchunk) : g.K;
    float *C = g.C + (g.kchunk ? blockIdx.z * g.cz : 0);
    for (int k0 = kbeg; k0 < kend; k0 += BK) {
        // stage: pairs of k so that each shared word holds two BF16 values;
        // consecutive threads walk the operand's unit-stride index (coalesced)
        for (int e = tid; e < BM * BK / 2; e += GT) {
            const bool mfast = g.sam == 1;
            const int mm = mfast ? e % BM : e / (BK / 2);
            const int kk = 2 * (mfast ? e / BM : e % (BK / 2));
            const int m = m0 + mm, k = k0 + kk;
            float x0 = 0.f, x1 = 0.f;
            if (m < g.M) {
                if (k < kend) x0 = g.A[m * g.sam + k * g.sak];
                if (k + 1 < kend) x1 = g.A[m * g.sam + (k + 1) * g.sak];
            }
            *(uint32_t *)&sA[mm * KP + kk] = pack_bf16(x0, x1);
        }
        for (int e = tid; e < BN * BK / 2; e += GT) {
            const bool nfast = g.sbn == 1;
            const int nn = nfast ? e % BN : e / (BK / 2);
            const int kk = 2 * (nfast ? e / BN : e % (BK / 2));
            const int n = n0 + nn, k = k0 + kk;
            float x0 = 0.f, x1 = 0.f;
            if (n < g.N) {
                if (k < kend) x0 = g.B[k * g.sbk + n * g.sbn];
                if (k + 1 < kend) x1 = g.B[(k + 1) * g.sbk + n * g.sbn];
            }
            *(uint32_t *)&sB[nn * KP + kk] = pack_bf16(x0, x1);
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < BK; ks += 16) {
            uint32_t af[2][4], bfr[4][2];
#pragma unroll
            for (int a = 0; a < 2; ++a) {
                const __nv_bfloat16 *p = sA + (wm + 16 * a + gq) * KP + ks + 2 * tq;
                af[a][0] = *(const uint32_t *)p;
                af[a][1] = *(const uint32_t *)(p + 8 * KP);
                af[a][2] = *(const uint32_t *)(p + 8);
                af[a][3] = *(const uint32_t *)(p + 8 * KP + 8);
            }
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const __nv_bfloat16 *p = sB + (wn + 8 * b + gq) * KP + ks + 2 * tq;
                bfr[b][0] = *(const uint32_t *)p;
                bfr[b][1] = *(const uint32_t *)(p + 8);
            }
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b)
                    asm volatile(
                        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                        : "+f"(acc[a][b][0]), "+f"(acc[a][b][1]), "+f"(acc[a][b][2]), "+f"(acc[a][b][3])
                        : "r"(af[a][0]), "r"(af[a][1]), "r"(af[a][2]), "r"(af[a][3]), "r"(bfr[b][0]),
                          "r"(bfr[b][1]));
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int m = m0 + wm + 16 * a + gq + 8 * (c >> 1);
                const int n = n0 + wn + 8 * b + 2 * tq + (c & 1);
                if (m >= g.M || n >= g.N) continue;
                float v = acc[a][b][c];
                const long o = (long)m * g.ldc + n;
                if (g.epi == EPI_BIAS || g.epi == EPI_BIAS_GELU) v += g.bias[n];
                if (g.epi == EPI_BIAS_GELU) {
                    g.Z[o] = v;
                    v = gelu(v);
                }
                if (g.epi == EPI_GELU_GRAD) v *= gelu_grad(g.gate[o]);
                C[o] = v;
            }
}

// Weighted mean squared error: loss = sum w (y - t)^2 / sum w, dy = 2 w (y - t) / sum w.
// One block; the sums are formed in FP64.
__global__ void __launch_bounds__(1024) k_mse(const float *y, const float *t, const float *w, long n, float *dy,
                                             double *loss) {
    __shared__ double s0[32], s1[32];
    double a = 0.0, b = 0.0;
    for (long i = threadIdx.x; i < n; i += blockDim.x) {
        const double d = (double)y[i] - (double)t[i];
        a += (double)w[i] * d * d;
        b += (double)w[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    if ((threadIdx.x & 31) == 0) { s0[threadIdx.x >> 5] = a; s1[threadIdx.x >> 5] = b; }
    __syncthreads();
    if (threadIdx.x < 32) {
        const int nw = blockDim.x >> 5;
        a = threadIdx.x < nw ? s0[threadIdx.x] : 0.0;
        b = threadIdx.x < nw ? s1[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        if (threadIdx.x == 0) { s0[0] = a; s1[0] = b; }
    }
    __syncthreads();
    const double den = s1[0] > 0.0 ? s1[0] : 1.0;
    if (threadIdx.x == 0) *loss = s0[0] / den;
    const float sc = (float)(2.0 / den);
    for (long i = threadIdx.x; i < n; i += blockDim.x) dy[i] = sc * w[i] * (y[i] - t[i]);
}

// C[m*ldc + n] = sum over z < nz of ws[z*M*N + m*N + n]  (split-K partials, fixed order)
__global__ void k_splitk_sum(const float *ws, int nz, int M, int N, float *C, int ldc) {
    const long tot = (long)M * N;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < tot; e += (long)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int z = 0; z < nz; ++z) s += ws[z * tot + e];
        C[(e / N) * ldc + e % N] = s;
    }
}

// Adam on the packed parameters (FP32 master copy).
__global__ void k_adam(float *p, const float *g, float *m1, float *m2, long n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float a = b1 * m1[i] + (1.f - b1) * gi;
        const float b = b2 * m2[i] + (1.f - b2) * gi * gi;
        m1[i] = a;
        m2[i] = b;
        p[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
    }
}

// Gathers the rows idx[0..B) of the data set (x: nin per row, t and w: nout per row).
__global__ void k_gather(const float *x, const float *t, const float *w, const int *idx, int B, int nin, int nout,
                         float *xb, float *tb, float *wb) {
    const long tot = (long)B * (nin + 2 * nout);
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < tot; e += (long)gridDim.x * blockDim.x) {
        const int r = (int)(e / (nin + 2 * nout)), c = (int)(e % (nin + 2 * nout));
        const long src = idx[r];
        if (c < nin) xb[(long)r * nin + c] = x[src * nin + c];
        else if (c < nin + nout) tb[(long)r * nout + c - nin] = t[src * nout + c - nin];
        else wb[(long)r * nout + c - nin - nout] = w[src * nout + c - nin - nout];
    }
}

}  // namespace

struct negf_mlp {
    int device = 0, L = 0, max_batch = 0;
    std::vector<int> width;
    std::vector<long> woff, boff;  // offsets of W_l, b_l in the packed parameters
    long np = 0;
    float *p = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
    std::vector<float *> Z, Y;  // per layer: pre-activation and output [max_batch x width[l+1]]
    float *d0 = nullptr, *d1 = nullptr;  // gradient ping-pong [max_batch x max width]
    float *xb = nullptr, *tb = nullptr, *wb = nullptr, *dy = nullptr;
    float *ws = nullptr;    // split-K partial products
    float *ones = nullptr;  // [max_batch] of 1.0: bias gradients as products
    double *loss = nullptr;
    long step = 0;
    cudaStream_t st = nullptr;
};

namespace {

constexpr int MAX_SPLITS = 16;

// Launches C = A B; a product with few output tiles and a long K (the weight
// gradients, K = batch) is split along K into partial products that one more
// kernel sums in a fixed order.
int gemm(negf_mlp *mm, const Gemm &g0) {
    if (g0.M <= 0 || g0.N <= 0) return 0;
    Gemm g = g0;
    g.kchunk = 0;
    g.cz = 0;
    const int tiles = ((g.N + BN - 1) / BN) * ((g.M + BM - 1) / BM);
    int splits = 1;
    if (g.epi == EPI_STORE && tiles < 148 && g.K >= 8 * BK)
        splits = std::min({MAX_SPLITS, (2 * 148 + tiles - 1) / tiles, g.K / (4 * BK)});
    if (splits > 1) {
        const int kc = ((g.K + splits - 1) / splits + BK - 1) / BK * BK;
        splits = (g.K + kc - 1) / kc;
        g.kchunk = kc;
        g.C = mm->ws;
        g.ldc = g.N;
        g.cz = (long)g.M * g.N;
    }
    dim3 grid((g.N + BN - 1) / BN, (g.M + BM - 1) / BM, splits);
    k_gemm_bf16<<<grid, GT, 0, mm->st>>>(g);
    if (cudaGetLastError() != cudaSuccess) return NEGF_MLP_ERR_CUDA;
    if (splits > 1) {
        const int blocks = (int)std::min<long>(((long)g.M * g.N + 255) / 256, 148 * 4);
        k_splitk_sum<<<blocks, 256, 0, mm->st>>>(mm->ws, splits, g.M, g.N, g0.C, g0.ldc);
        if (cudaGetLastError() != cudaSuccess) return NEGF_MLP_ERR_CUDA;
    }
    return 0;
}

// Forward pass of B rows of m->xb; the outputs are m->Y[L-1].
int forward(negf_mlp *m, const float *x, int B) {
    const float *in = x;
    for (int l = 0; l < m->L; ++l) {
        const int K = m->width[l], N = m->width[l + 1];
        const bool last = l == m->L - 1;
        Gemm g{in, K, 1, m->p + m->woff[l], 1, K, m->Y[l], N, B, N, K,
               last ? EPI_BIAS : EPI_BIAS_GELU, m->p + m->boff[l], m->Z[l], nullptr};
        if (int rc = gemm(m, g)) return rc;
        in = m->Y[l];
    }
    return 0;
}

// Loss and gradient (into m->g) for B rows: x (B x width[0]), t, w (B x width[L]).
int backward(negf_mlp *m, const float *x, const float *t, const float *w, int B) {
    const int L = m->L, nout = m->width[L];
    k_mse<<<1, 1024, 0, m->st>>>(m->Y[L - 1], t, w, (long)B * nout, m->dy, m->loss);
    if (cudaGetLastError() != cudaSuccess) return NEGF_MLP_ERR_CUDA;
    const float *dz = m->dy;  // gradient w.r.t. the pre-activation of layer l
    for (int l = L - 1; l >= 0; --l) {
        const int K = m->width[l], N = m->width[l + 1];
        const float *in = l ? m->Y[l - 1] : x;
        // dW_l (N x K) = dz^T (N x B) * in (B x K)
        Gemm gw{dz, 1, N, in, K, 1, m->g + m->woff[l], K, N, K, B, EPI_STORE, nullptr, nullptr, nullptr};
        if (int rc = gemm(m, gw)) return rc;
        // db_l (N x 1) = dz^T (N x B) * ones (B x 1)
        Gemm gb{dz, 1, N, m->ones, 1, 0, m->g + m->boff[l], 1, N, 1, B, EPI_STORE, nullptr, nullptr, nullptr};
        if (int rc = gemm(m, gb)) return rc;
        if (l == 0) break;
        // dz_{l-1} (B x K) = (dz (B x N) * W_l (N x K)) * gelu'(Z_{l-1})
        float *dn = (dz == m->d0) ? m->d1 : m->d0;
        Gemm gd{dz, N, 1, m->p + m->woff[l], K, 1, dn, K, B, K, N, EPI_GELU_GRAD, nullptr, nullptr, m->Z[l - 1]};
        if (int rc = gemm(m, gd)) return rc;
        dz = dn;
    }
    return 0;
}

int adam(negf_mlp *m, float lr) {
    m->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)m->step), c2 = 1.f - powf(b2, (float)m->step);
    const int blocks = (int)std::min<long>((m->np + 255) / 256, 148 * 8);
    k_adam<<<blocks, 256, 0, m->st>>>(m->p, m->g, m->m1, m->m2, m->np, lr, b1, b2, 1e-8f, c1, c2);
    return cudaGetLastError() == cudaSuccess ? 0 : NEGF_MLP_ERR_CUDA;
}

int check_batch(const negf_mlp *m, int B) { return (B < 1 || B > m->max_batch) ? NEGF_MLP_ERR_ARG : 0; }

}  // namespace

extern "C" {

int negf_mlp_create(int32_t n_layers, const int32_t *widths, int32_t max_batch, int32_t device, negf_mlp **out) {
    if (!out || n_layers < 1 || !widths || max_batch < 1) return NEGF_MLP_ERR_ARG;
    *out = nullptr;
    for (int l = 0; l <= n_layers; ++l)
        if (widths[l] < 1 || widths[l] > 4096) return NEGF_MLP_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return NEGF_MLP_ERR_CUDA;
    negf_mlp *m = new negf_mlp();
    m->device = device;
    m->L = n_layers;
    m->max_batch = max_batch;
    m->width.assign(widths, widths + n_layers + 1);
    int wmax = 0;
    for (int l = 0; l < n_layers; ++l) {
        m->woff.push_back(m->np);
        m->np += (long)widths[l + 1] * widths[l];
        m->boff.push_back(m->np);
        m->np += widths[l + 1];
    }
    for (int l = 0; l <= n_layers; ++l) wmax = std::max(wmax, (int)widths[l]);
    bool ok = cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) == cudaSuccess;
    auto alloc = [&](float **p, size_t n) { if (ok) ok = cudaMalloc(p, sizeof(float) * n) == cudaSuccess; };
    alloc(&m->p, m->np);
    alloc(&m->g, m->np);
    alloc(&m->m1, m->np);
    alloc(&m->m2, m->np);
    m->Z.assign(n_layers, nullptr);
    m->Y.assign(n_layers, nullptr);
    for (int l = 0; l < n_layers; ++l) {
        alloc(&m->Z[l], (size_t)max_batch * widths[l + 1]);
        alloc(&m->Y[l], (size_t)max_batch * widths[l + 1]);
    }
    alloc(&m->d0, (size_t)max_batch * wmax);
    alloc(&m->d1, (size_t)max_batch * wmax);
    alloc(&m->xb, (size_t)max_batch * widths[0]);
    alloc(&m->tb, (size_t)max_batch * widths[n_layers]);
    alloc(&m->wb, (size_t)max_batch * widths[n_layers]);
    alloc(&m->dy, (size_t)max_batch * widths[n_layers]);
    size_t mn = 0;
    for (int l = 0; l < n_layers; ++l) mn = std::max(mn, (size_t)widths[l + 1] * widths[l]);
    alloc(&m->ws, MAX_SPLITS * mn);
    alloc(&m->ones, (size_t)max_batch);
    if (ok) {
        std::vector<float> one((size_t)max_batch, 1.0f);
        ok = cudaMemcpy(m->ones, one.data(), sizeof(float) * max_batch, cudaMemcpyHostToDevice) == cudaSuccess;
    }
    if (ok) ok = cudaMalloc(&m->loss, sizeof(double)) == cudaSuccess;
    if (ok) ok = cudaMemsetAsync(m->p, 0, sizeof(float) * m->np, m->st) == cudaSuccess &&
                 cudaMemsetAsync(m->m1, 0, sizeof(float) * m->np, m->st) == cudaSuccess &&
                 cudaMemsetAsync(m->m2, 0, sizeof(float) * m->np, m->st) == cudaSuccess &&
                 cudaStreamSynchronize(m->st) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        negf_mlp_destroy(m);
        return NEGF_MLP_ERR_NOMEM;
    }
    *out = m;
    return NEGF_MLP_OK;
}

int negf_mlp_destroy(negf_mlp *m) {
    if (!m) return NEGF_MLP_OK;
    cudaSetDevice(m->device);
    if (m->st) cudaStreamSynchronize(m->st);
    for (float *q : {m->p, m->g, m->m1, m->m2, m->d0, m->d1, m->xb, m->tb, m->wb, m->dy, m->ws, m->ones}) cudaFree(q);
    for (float *q : m->Z) cudaFree(q);
    for (float *q : m->Y) cudaFree(q);
    cudaFree(m->loss);
    if (m->st) cudaStreamDestroy(m->st);
    delete m;
    return NEGF_MLP_OK;
}

int64_t negf_mlp_param_count(const negf_mlp *m) { return m ? m->np : -1; }

int negf_mlp_set_params(negf_mlp *m, const float *params) {
    if (!m || !params) return NEGF_MLP_ERR_ARG;
    if (cudaSetDevice(m->device) != cudaSuccess) return NEGF_MLP_ERR_CUDA;
    m->step = 0;
    const size_t b = sizeof(float) * m->np;
    if (cudaMemcpyAsync(m->p, params, b, cudaMemcpyHostToDevice, m->st) != cudaSuccess ||
        cudaMemsetAsync(m->m1, 0, b, m->st) != cudaSuccess || cudaMemsetAsync(m->m2, 0, b, m->st) != cudaSuccess ||
        cudaStreamSynchronize(m->st) != cudaSuccess)
        return NEGF_MLP_ERR_CUDA;
    return NEGF_MLP_OK;
}

int negf_mlp_get_params(negf_mlp *m, float *params) {
    if (!m || !params) return NEGF_MLP_ERR_ARG;
    if (cudaSetDevice(m->device) != cudaSuccess) return NEGF_MLP_ERR_CUDA;
    if (cudaMemcpyAsync(params, m->p, sizeof(float) * m->np, cudaMemcpyDeviceToHost, m->st) != cudaSuccess ||
        cudaStreamSynchronize(m->st) != cudaSuccess)
        return NEGF_MLP_ERR_CUDA;
    return NEGF_MLP_OK;
}

int negf_mlp_forward(negf_mlp *m, const float *x, int32_t batch, float *y) {
    if (!m || !x || !y) return NEGF_MLP_ERR_ARG;
    if (cudaSetDevice(m->device) != cudaSuccess) return NEGF_MLP_ERR_CUDA;
    const int nin = m->width[0], nout = m->width[m->L];
    for (int32_t r0 = 0; r0 < batch; r0 += m->max_batch) {
        const int B = std::min(m->max_batch, batch - r0);
        if (cudaMemcpyAsync(m->xb, x + (size_t)r0 * nin, sizeof(float) * B * nin, cudaMemcpyHostToDevice,
                            m->st) != cudaSuccess)
            return NEGF_MLP_ERR_CUDA;
        if (int rc = forward(m, m->xb, B)) return rc;
        if (cudaMemcpyAsync(y + (size_t)r0 * nout, m->Y[m->L - 1], sizeof(float) * B * nout,
                            cudaMemcpyDeviceToHost, m->st) != cudaSuccess)
            return NEGF_MLP_ERR_CUDA;
    }
    return cudaStreamSynchronize(m->st) == cudaSuccess ? NEGF_MLP_OK : NEGF_MLP_ERR_CUDA;
}

int negf_mlp_grad(negf_mlp *m, const float *x, const float *t, const float *w, int32_t batch, double *loss,
                  float *grad) {
    if (!m || !x || !t || !w || !loss || !grad) return NEGF_MLP_ERR_ARG;
    if (int rc = check_batch(m, batch)) return rc;
    if (cudaSetDevice(m->device) != cudaSuccess) return NEGF_MLP_ERR_CUDA;
    const int nin = m->width[0], nout = m->width[m->L];
    if (cudaMemcpyAsync(m->xb, x, sizeof(float) * batch * nin, cudaMemcpyHostToDevice, m->st) != cudaSuccess ||
        cudaMemcpyAsync(m->tb, t, sizeof(float) * batch * nout, cudaMemcpyHostToDevice, m->st) != cudaSuccess ||
        cudaMemcpyAsync(m->wb, w, sizeof(float) * batch * nout, cudaMemcpyHostToDevice, m->st) != cudaSuccess)
        return NEGF_MLP_ERR_CUDA;
    if (int rc = forward(m, m->xb, batch)) return rc;
    if (int rc = backward(m, m->xb, m->tb, m->wb, batch)) return rc;
    if (cudaMemcpyAsync(grad, m->g, sizeof(float) * m->np, cudaMemcpyDeviceToHost, m->st) != cudaSuccess ||
        cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, m->st) != cudaSuccess ||
        cudaStreamSynchronize(m->st) != cudaSuccess)
        return NEGF_MLP_ERR_CUDA;
    return NEGF_MLP_OK;
}

int negf_mlp_train(negf_mlp *m, const float *x, const float *t, const float *w, int64_t n, int32_t batch,
                   int32_t steps, float lr, uint64_t seed, double *losses) {
    if (!m || !x || !t || !w || n < 1 || steps < 0) return NEGF_MLP_ERR_ARG;
    if (int rc = check_batch(m, batch)) return rc;
    if (cudaSetDevice(m->device) != cudaSuccess) return NEGF_MLP_ERR_CUDA;
    const int nin = m->width[0], nout = m->width[m->L];
    float *dx = nullptr, *dt = nullptr, *dw = nullptr;
    int *didx = nullptr;
    double *dl = nullptr;
    int rc = NEGF_MLP_OK;
    if (cudaMalloc(&dx, sizeof(float) * n * nin) != cudaSuccess ||
        cudaMalloc(&dt, sizeof(float) * n * nout) != cudaSuccess ||
        cudaMalloc(&dw, sizeof(float) * n * nout) != cudaSuccess ||
        cudaMalloc(&didx, sizeof(int) * (size_t)batch * std::max(steps, 1)) != cudaSuccess ||
        cudaMalloc(&dl, sizeof(double) * std::max(steps, 1)) != cudaSuccess)
        rc = NEGF_MLP_ERR_NOMEM;
    // minibatches: a fresh permutation of the data set per epoch (splitmix64 from seed)
    std::vector<int> idx((size_t)batch * std::max(steps, 1));
    if (!rc) {
        std::vector<int> perm(n);
        for (int64_t i = 0; i < n; ++i) perm[i] = (int)i;
        uint64_t s = seed;
        auto next = [&s]() {
            uint64_t z = (s += 0x9E3779B97F4A7C15ull);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            return z ^ (z >> 31);
        };
        int64_t pos = n;
        for (size_t i = 0; i < idx.size(); ++i) {
            if (pos == n) {
                for (int64_t j = n - 1; j > 0; --j) std::swap(perm[j], perm[next() % (uint64_t)(j + 1)]);
                pos = 0;
            }
            idx[i] = perm[pos++];
        }
        if (cudaMemcpyAsync(dx, x, sizeof(float) * n * nin, cudaMemcpyHostToDevice, m->st) != cudaSuccess ||
            cudaMemcpyAsync(dt, t, sizeof(float) * n * nout, cudaMemcpyHostToDevice, m->st) != cudaSuccess ||
            cudaMemcpyAsync(dw, w, sizeof(float) * n * nout, cudaMemcpyHostToDevice, m->st) != cudaSuccess ||
            cudaMemcpyAsync(didx, idx.data(), sizeof(int) * idx.size(), cudaMemcpyHostToDevice, m->st) !=
                cudaSuccess)
            rc = NEGF_MLP_ERR_CUDA;
    }
    for (int s = 0; s < steps && !rc; ++s) {
        const int blocks = std::min(148 * 4, (batch * (nin + 2 * nout) + 255) / 256);
        k_gather<<<blocks, 256, 0, m->st>>>(dx, dt, dw, didx + (size_t)s * batch, batch, nin, nout, m->xb, m->tb,
                                           m->wb);
        if (cudaGetLastError() != cudaSuccess) { rc = NEGF_MLP_ERR_CUDA; break; }
        if ((rc = forward(m, m->xb, batch))) break;
        if ((rc = backward(m, m->xb, m->tb, m->wb, batch))) break;
        if (cudaMemcpyAsync(dl + s, m->loss, sizeof(double), cudaMemcpyDeviceToDevice, m->st) != cudaSuccess) {
            rc = NEGF_MLP_ERR_CUDA;
            break;
        }
        if ((rc = adam(m, lr))) break;
    }
    if (!rc && losses && steps > 0 &&
        cudaMemcpyAsync(losses, dl, sizeof(double) * steps, cudaMemcpyDeviceToHost, m->st) != cudaSuccess)
        rc = NEGF_MLP_ERR_CUDA;
    if (cudaStreamSynchronize(m->st) != cudaSuccess && !rc) rc = NEGF_MLP_ERR_CUDA;
    cudaFree(dx);
    cudaFree(dt);
    cudaFree(dw);
    cudaFree(didx);
    cudaFree(dl);
    return rc;
}

}  // extern "C"
