// amrlbm_net.cu - the refine-flag forecaster of the learned regrid: a small
// convolutional network over one block with its ghost ring (4 channels on
// 18 x 18 cells for 16 x 16 blocks: C, |grad C| against the refine tolerance,
// Ux and Uy as cells moved over the forecast horizon), three 3x3 convolutions
// of 32 channels with ReLU, a global max pool and a dense output: the logit
// of "this block is flagged for refinement k steps from now". No counterpart
// in the reference, which flags blocks from the current field only
// (Err_Interface, Refine_Derefine.f90:327-351).
//
// Every contraction is one kernel: C = A B with BF16 operands and FP32
// accumulation on the tensor cores (mma.sync m16n8k16), A and B addressed
// through strides so that transposes cost nothing. A convolution is an
// im2col copy followed by that product; its backward pass is two more
// products (dW = colT dY, dcol = dY WT) and a col2im gather. Weights are
// kept in FP32 (Adam) and rounded to BF16 for every product.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "amrlbm.h"
#include "amrlbm_dev.cuh"
#include "amrlbm_launch.h"

namespace {

constexpr int CH = 32;        // channels of every hidden layer
constexpr int CIN = AMRLBM_NET_CHANNELS;
constexpr int TILE = AMRLBM_NET_TILE;  // 18
constexpr int PIX = TILE * TILE;       // 324
constexpr int K1 = CIN * 9, K1P = (K1 + 15) / 16 * 16;  // 36 -> 48
constexpr int K2 = CH * 9;                               // 288
// FP32 parameter vector: W1 [K1][CH], b1, W2 [K2][CH], b2, W3 [K2][CH], b3, wd [CH], bd
constexpr int O_W1 = 0, O_B1 = O_W1 + K1 * CH, O_W2 = O_B1 + CH, O_B2 = O_W2 + K2 * CH,
              O_W3 = O_B2 + CH, O_B3 = O_W3 + K2 * CH, O_WD = O_B3 + CH, O_BD = O_WD + CH,
              NPARAM = O_BD + 1;

// ---- the tensor-core product -----------------------------------------------
// C[M][N] (FP32, row stride ldc) = sum_k A(m, k) B(k, n), A(m, k) = A[m*sam + k*sak],
// B(k, n) = B[k*sbk + n*sbn], BF16. CTA: 4 warps, a 64 x 32 tile of C; each
// warp 16 rows x 4 n-tiles of 8. Operands go through shared memory with zero
// padding outside M, N, K.
constexpr int GM = 64, GN = 32, GK = 16;

__device__ __forceinline__ unsigned pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (unsigned)__bfloat16_as_ushort(lo) | ((unsigned)__bfloat16_as_ushort(hi) << 16);
}

__global__ void __launch_bounds__(128) k_gemm(int M, int N, int K, const __nv_bfloat16* A,
                                              long long sam, long long sak,
                                              const __nv_bfloat16* B, long long sbk,
                                              long long sbn, float* C, long long ldc) {
    __shared__ __nv_bfloat16 sA[GM][GK + 2];
    __shared__ __nv_bfloat16 sB[GK][GN + 2];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5, g = lane >> 2, q = lane & 3;
    const int m0 = blockIdx.x * GM, n0 = blockIdx.y * GN;
    float acc[4][4];
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[j][i] = 0.f;
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    for (int k0 = 0; k0 < K; k0 += GK) {
        for (int i = t; i < GM * GK; i += 128) {
            const int r = i / GK, c = i % GK, m = m0 + r, k = k0 + c;
            sA[r][c] = (m < M && k < K) ? A[(long long)m * sam + (long long)k * sak] : zero;
        }
        for (int i = t; i < GK * GN; i += 128) {
            const int r = i / GN, c = i % GN, k = k0 + r, n = n0 + c;
            sB[r][c] = (k < K && n < N) ? B[(long long)k * sbk + (long long)n * sbn] : zero;
        }
        __syncthreads();
        const int r = 16 * w;
        const unsigned a0 = pack_bf16(sA[r + g][2 * q], sA[r + g][2 * q + 1]);
        const unsigned a1 = pack_bf16(sA[r + g + 8][2 * q], sA[r + g + 8][2 * q + 1]);
        const unsigned a2 = pack_bf16(sA[r + g][2 * q + 8], sA[r + g][2 * q + 9]);
        const unsigned a3 = pack_bf16(sA[r + g + 8][2 * q + 8], sA[r + g + 8][2 * q + 9]);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const unsigned b0 = pack_bf16(sB[2 * q][8 * j + g], sB[2 * q + 1][8 * j + g]);
            const unsigned b1 = pack_bf16(sB[2 * q + 8][8 * j + g], sB[2 * q + 9][8 * j + g]);
            asm volatile(
                "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                : "+f"(acc[j][0]), "+f"(acc[j][1]), "+f"(acc[j][2]), "+f"(acc[j][3])
                : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int n = n0 + 8 * j + 2 * q;
        const int m = m0 + 16 * w + g;
        if (m < M) {
            if (n < N) C[(long long)m * ldc + n] = acc[j][0];
            if (n + 1 < N) C[(long long)m * ldc + n + 1] = acc[j][1];
        }
        if (m + 8 < M) {
            if (n < N) C[(long long)(m + 8) * ldc + n] = acc[j][2];
            if (n + 1 < N) C[(long long)(m + 8) * ldc + n + 1] = acc[j][3];
        }
    }
}

void gemm(cudaStream_t st, int M, int N, int K, const __nv_bfloat16* A, long long sam,
          long long sak, const __nv_bfloat16* B, long long sbk, long long sbn, float* C,
          long long ldc) {
    dim3 grid((M + GM - 1) / GM, (N + GN - 1) / GN);
    k_gemm<<<grid, 128, 0, st>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, ldc);
    count_launches(1);
}

// ---- elementwise parts -------------------------------------------------------
inline int blocks_for(long long n) { return (int)std::min<long long>((n + 255) / 256, 8192); }
#define GRID_STRIDE(i, n) for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

// input [n][CIN][TILE][TILE] (FP32) -> channels-last BF16 [n*PIX][CIN]
__global__ void k_input(int n, const float* x, __nv_bfloat16* a) {
    GRID_STRIDE(i, (long long)n * PIX * CIN) {
        const long long row = i / CIN;
        const int c = (int)(i % CIN), b = (int)(row / PIX), p = (int)(row % PIX);
        a[i] = __float2bfloat16(x[((long long)b * CIN + c) * PIX + p]);
    }
}
// im2col of a channels-last activation [n*PIX][cin]: col[row][k], k = o*cin + ci
// (tap-major: the 16 columns of one product step are whole taps of adjacent
// channels), o = (dy+1)*3 + (dx+1), zero outside the tile and for k >= cin*9
__global__ void k_im2col(int n, int cin, int kp, const __nv_bfloat16* a, __nv_bfloat16* col) {
    GRID_STRIDE(i, (long long)n * PIX * kp) {
        const long long row = i / kp;
        const int k = (int)(i % kp), b = (int)(row / PIX), p = (int)(row % PIX);
        __nv_bfloat16 v = __float2bfloat16(0.f);
        if (k < cin * 9) {
            const int o = k / cin, ci = k % cin, y = p / TILE + o / 3 - 1, x = p % TILE + o % 3 - 1;
            if (x >= 0 && x < TILE && y >= 0 && y < TILE)
                v = a[((long long)b * PIX + y * TILE + x) * cin + ci];
        }
        col[i] = v;
    }
}
// z [m][CH] + bias -> ReLU: activation in FP32 and BF16
__global__ void k_bias_relu(long long m, const float* z, const float* bias, float* af,
                            __nv_bfloat16* ab) {
    GRID_STRIDE(i, m * CH) {
        const float v = fmaxf(z[i] + bias[i % CH], 0.f);
        af[i] = v;
        ab[i] = __float2bfloat16(v);
    }
}
// global max pool of the last activation [n*PIX][CH] -> pooled [n][CH], argmax
__global__ void k_maxpool(int n, const float* a, float* pooled, int* arg) {
    GRID_STRIDE(i, (long long)n * CH) {
        const int b = (int)(i / CH), c = (int)(i % CH);
        float m = -1.f;
        int am = 0;
        for (int p = 0; p < PIX; ++p) {
            const float v = a[((long long)b * PIX + p) * CH + c];
            if (v > m) {
                m = v;
                am = p;
            }
        }
        pooled[i] = m;
        arg[i] = am;
    }
}
// dense output and the weighted binary cross-entropy on logits: logits[b],
// dlogit[b] = w (sigmoid(z) - y) / n, loss terms lterm[b]
__global__ void k_head(int n, const float* pooled, const float* w, const float* y, float posw,
                       float* logits, float* dlogit, float* lterm) {
    GRID_STRIDE(b, n) {
        float z = w[O_BD - O_WD];
        for (int c = 0; c < CH; ++c) z += w[c] * pooled[b * CH + c];
        logits[b] = z;
        if (y) {
            const float yy = y[b], wt = yy > 0.5f ? posw : 1.f;
            // log(1 + exp(-|z|)) + max(z, 0) - z y
            const float l = log1pf(expf(-fabsf(z))) + fmaxf(z, 0.f) - z * yy;
            lterm[b] = wt * l;
            dlogit[b] = wt * (1.f / (1.f + expf(-z)) - yy) / (float)n;
        }
    }
}
// dense backward: gradients of wd, bd (one CTA, fixed order) and dpooled
__global__ void k_head_back(int n, const float* pooled, const float* w, const float* dlogit,
                            float* dpooled, float* grad_wd) {
    const int t = threadIdx.x;
    if (t <= CH) {
        float s = 0.f;
        for (int b = 0; b < n; ++b) s += dlogit[b] * (t < CH ? pooled[b * CH + t] : 1.f);
        grad_wd[t] = s;  // [CH] weights then the bias
    }
    for (long long i = t; i < (long long)n * CH; i += blockDim.x) dpooled[i] = dlogit[i / CH] * w[i % CH];
}
// max-pool backward into dA [n*PIX][CH] (zero elsewhere)
__global__ void k_unpool(int n, const float* dpooled, const int* arg, float* dA) {
    GRID_STRIDE(i, (long long)n * PIX * CH) dA[i] = 0.f;
}
__global__ void k_unpool2(int n, const float* dpooled, const int* arg, float* dA) {
    GRID_STRIDE(i, (long long)n * CH) {
        const int b = (int)(i / CH), c = (int)(i % CH);
        dA[((long long)b * PIX + arg[i]) * CH + c] = dpooled[i];
    }
}
// ReLU backward: dz = dA where A > 0, as BF16 for the products
__global__ void k_relu_back(long long m, const float* dA, const float* A, float* dz,
                            __nv_bfloat16* dzb) {
    GRID_STRIDE(i, m * CH) {
        const float v = A[i] > 0.f ? dA[i] : 0.f;
        dz[i] = v;
        dzb[i] = __float2bfloat16(v);
    }
}
// bias gradient: column sums of dz [m][CH] (one CTA per channel, fixed order)
__global__ void k_colsum(long long m, const float* dz, float* out) {
    __shared__ float red[256];
    const int c = blockIdx.x;
    float s = 0.f;
    for (long long r = threadIdx.x; r < m; r += blockDim.x) s += dz[r * CH + c];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[c] = red[0];
}
// col2im: dA[row q][ci] = sum over the 3x3 offsets o of dcol[row q - o][o*cin + ci]
__global__ void k_col2im(int n, int cin, int kp, const float* dcol, float* dA) {
    GRID_STRIDE(i, (long long)n * PIX * cin) {
        const long long row = i / cin;
        const int ci = (int)(i % cin), b = (int)(row / PIX), p = (int)(row % PIX);
        const int y = p / TILE, x = p % TILE;
        float s = 0.f;
        for (int o = 0; o < 9; ++o) {
            const int py = y - (o / 3 - 1), px = x - (o % 3 - 1);
            if (px >= 0 && px < TILE && py >= 0 && py < TILE)
                s += dcol[((long long)b * PIX + py * TILE + px) * kp + o * cin + ci];
        }
        dA[i] = s;
    }
}
// Adam on the FP32 parameters
__global__ void k_adam(int np, float* p, const float* g, float* m1, float* m2, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
    GRID_STRIDE(i, np) {
        const float gi = g[i];
        m1[i] = b1 * m1[i] + (1.f - b1) * gi;
        m2[i] = b2 * m2[i] + (1.f - b2) * gi * gi;
        p[i] -= lr * (m1[i] / c1) / (sqrtf(m2[i] / c2) + eps);
    }
}
// BF16 weight matrices for the products: W1 padded to K1P rows
__global__ void k_pack(const float* p, __nv_bfloat16* w1, __nv_bfloat16* w2, __nv_bfloat16* w3) {
    GRID_STRIDE(i, (long long)K1P * CH) {
        const int k = (int)(i / CH);
        w1[i] = __float2bfloat16(k < K1 ? p[O_W1 + i] : 0.f);
    }
    GRID_STRIDE(i, (long long)K2 * CH) {
        w2[i] = __float2bfloat16(p[O_W2 + i]);
        w3[i] = __float2bfloat16(p[O_W3 + i]);
    }
}

// deterministic normal draws for the initial weights (splitmix64 + Box-Muller)
struct Rng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    double uniform() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
    double normal() { return std::sqrt(-2.0 * std::log(uniform())) * std::cos(6.283185307179586 * uniform()); }
};

}  // namespace

struct amrlbm_net {
    int max_n = 0;
    cudaStream_t st = nullptr;
    std::vector<void*> allocs;
    float *p = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;  // [NPARAM]
    __nv_bfloat16 *w1 = nullptr, *w2 = nullptr, *w3 = nullptr;
    // per batch row buffers
    float *x = nullptr, *y = nullptr;
    __nv_bfloat16 *a0 = nullptr, *col1 = nullptr, *col2 = nullptr, *col3 = nullptr;
    float *z = nullptr, *a1f = nullptr, *a2f = nullptr, *a3f = nullptr, *dA = nullptr, *dz = nullptr,
          *dcol = nullptr;
    __nv_bfloat16 *a1b = nullptr, *a2b = nullptr, *a3b = nullptr, *dzb = nullptr;
    float *pooled = nullptr, *dpooled = nullptr, *logits = nullptr, *dlogit = nullptr,
          *lterm = nullptr;
    int* arg = nullptr;
    int steps = 0;
    std::string err;
};

namespace {

template <class T>
T* nalloc(amrlbm_net* net, size_t n, cudaError_t* e) {
    void* q = nullptr;
    if (*e == cudaSuccess) *e = cudaMalloc(&q, n * sizeof(T));
    if (*e == cudaSuccess) {
        cudaMemset(q, 0, n * sizeof(T));
        net->allocs.push_back(q);
    }
    return (T*)q;
}

void repack(amrlbm_net* net) {
    k_pack<<<blocks_for((long long)K2 * CH), 256, 0, net->st>>>(net->p, net->w1, net->w2, net->w3);
    count_launches(1);
}

// forward of n samples already in net->x; the last activation in a3f
void forward(amrlbm_net* net, int n) {
    cudaStream_t st = net->st;
    const long long m = (long long)n * PIX;
    k_input<<<blocks_for(m * CIN), 256, 0, st>>>(n, net->x, net->a0);
    k_im2col<<<blocks_for(m * K1P), 256, 0, st>>>(n, CIN, K1P, net->a0, net->col1);
    gemm(st, (int)m, CH, K1P, net->col1, K1P, 1, net->w1, CH, 1, net->z, CH);
    k_bias_relu<<<blocks_for(m * CH), 256, 0, st>>>(m, net->z, net->p + O_B1, net->a1f, net->a1b);
    k_im2col<<<blocks_for(m * K2), 256, 0, st>>>(n, CH, K2, net->a1b, net->col2);
    gemm(st, (int)m, CH, K2, net->col2, K2, 1, net->w2, CH, 1, net->z, CH);
    k_bias_relu<<<blocks_for(m * CH), 256, 0, st>>>(m, net->z, net->p + O_B2, net->a2f, net->a2b);
    k_im2col<<<blocks_for(m * K2), 256, 0, st>>>(n, CH, K2, net->a2b, net->col3);
    gemm(st, (int)m, CH, K2, net->col3, K2, 1, net->w3, CH, 1, net->z, CH);
    k_bias_relu<<<blocks_for(m * CH), 256, 0, st>>>(m, net->z, net->p + O_B3, net->a3f, net->a3b);
    k_maxpool<<<blocks_for((long long)n * CH), 256, 0, st>>>(n, net->a3f, net->pooled, net->arg);
    count_launches(9);
}

// backward after forward with labels: gradients into net->g
void backward(amrlbm_net* net, int n) {
    cudaStream_t st = net->st;
    const long long m = (long long)n * PIX;
    k_head_back<<<1, 256, 0, st>>>(n, net->pooled, net->p + O_WD, net->dlogit, net->dpooled,
                                   net->g + O_WD);
    k_unpool<<<blocks_for(m * CH), 256, 0, st>>>(n, net->dpooled, net->arg, net->dA);
    k_unpool2<<<blocks_for((long long)n * CH), 256, 0, st>>>(n, net->dpooled, net->arg, net->dA);
    count_launches(3);
    // layer 3
    const float* A[3] = {net->a1f, net->a2f, net->a3f};
    const __nv_bfloat16* col[3] = {net->col1, net->col2, net->col3};
    const __nv_bfloat16* W[3] = {net->w1, net->w2, net->w3};
    const int kp[3] = {K1P, K2, K2}, kk[3] = {K1, K2, K2};
    const int ow[3] = {O_W1, O_W2, O_W3}, ob[3] = {O_B1, O_B2, O_B3};
    const int cin[3] = {CIN, CH, CH};
    for (int l = 2; l >= 0; --l) {
        k_relu_back<<<blocks_for(m * CH), 256, 0, st>>>(m, net->dA, A[l], net->dz, net->dzb);
        k_colsum<<<CH, 256, 0, st>>>(m, net->dz, net->g + ob[l]);
        count_launches(2);
        // dW = col^T dz: M = kk, N = CH, K = m (row strides of col are kp)
        gemm(st, kk[l], CH, (int)m, col[l], 1, kp[l], net->dzb, CH, 1, net->g + ow[l], CH);
        if (l == 0) break;
        // dcol = dz W^T: M = m, N = kp, K = CH
        gemm(st, (int)m, kp[l], CH, net->dzb, CH, 1, W[l], 1, CH, net->dcol, kp[l]);
        k_col2im<<<blocks_for(m * cin[l]), 256, 0, st>>>(n, cin[l], kp[l], net->dcol, net->dA);
        count_launches(1);
    }
}

int net_fail(amrlbm_net* net, int code, const std::string& m) {
    if (net) net->err = m;
    return code;
}
#define NCK(call)                                                                    \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) return net_fail(net, AMRLBM_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)

int load_batch(amrlbm_net* net, int n, const float* x, const float* y) {
    if (n < 1 || n > net->max_n || !x) return AMRLBM_ERR_ARG;
    NCK(cudaMemcpyAsync(net->x, x, sizeof(float) * (size_t)n * CIN * PIX, cudaMemcpyHostToDevice, net->st));
    if (y) NCK(cudaMemcpyAsync(net->y, y, sizeof(float) * (size_t)n, cudaMemcpyHostToDevice, net->st));
    return AMRLBM_OK;
}

}  // namespace

ForecastNet net_forecast_params(const amrlbm_net* net) {
    ForecastNet f;
    f.w1 = net->w1;
    f.w2 = net->w2;
    f.w3 = net->w3;
    f.b1 = net->p + O_B1;
    f.b2 = net->p + O_B2;
    f.b3 = net->p + O_B3;
    f.wd = net->p + O_WD;
    f.bd = net->p + O_BD;
    return f;
}

extern "C" {

int amrlbm_net_create(uint64_t seed, int32_t max_batch, amrlbm_net** out) {
    if (!out || max_batch < 1) return AMRLBM_ERR_ARG;
    *out = nullptr;
    int dev = 0, cc = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return AMRLBM_ERR_CUDA;
    cudaDeviceGetAttribute(&cc, cudaDevAttrComputeCapabilityMajor, dev);
    if (cc != 10) return AMRLBM_ERR_CUDA;
    amrlbm_net* net = new amrlbm_net();
    net->max_n = max_batch;
    cudaError_t e = cudaStreamCreateWithFlags(&net->st, cudaStreamNonBlocking);
    const size_t n = (size_t)max_batch, m = n * PIX;
    net->p = nalloc<float>(net, NPARAM, &e);
    net->g = nalloc<float>(net, NPARAM, &e);
    net->m1 = nalloc<float>(net, NPARAM, &e);
    net->m2 = nalloc<float>(net, NPARAM, &e);
    net->w1 = nalloc<__nv_bfloat16>(net, (size_t)K1P * CH, &e);
    net->w2 = nalloc<__nv_bfloat16>(net, (size_t)K2 * CH, &e);
    net->w3 = nalloc<__nv_bfloat16>(net, (size_t)K2 * CH, &e);
    net->x = nalloc<float>(net, n * CIN * PIX, &e);
    net->y = nalloc<float>(net, n, &e);
    net->a0 = nalloc<__nv_bfloat16>(net, m * CIN, &e);
    net->col1 = nalloc<__nv_bfloat16>(net, m * K1P, &e);
    net->col2 = nalloc<__nv_bfloat16>(net, m * K2, &e);
    net->col3 = nalloc<__nv_bfloat16>(net, m * K2, &e);
    net->z = nalloc<float>(net, m * CH, &e);
    net->a1f = nalloc<float>(net, m * CH, &e);
    net->a2f = nalloc<float>(net, m * CH, &e);
    net->a3f = nalloc<float>(net, m * CH, &e);
    net->a1b = nalloc<__nv_bfloat16>(net, m * CH, &e);
    net->a2b = nalloc<__nv_bfloat16>(net, m * CH, &e);
    net->a3b = nalloc<__nv_bfloat16>(net, m * CH, &e);
    net->dA = nalloc<float>(net, m * CH, &e);
    net->dz = nalloc<float>(net, m * CH, &e);
    net->dzb = nalloc<__nv_bfloat16>(net, m * CH, &e);
    net->dcol = nalloc<float>(net, m * K2, &e);
    net->pooled = nalloc<float>(net, n * CH, &e);
    net->dpooled = nalloc<float>(net, n * CH, &e);
    net->arg = nalloc<int>(net, n * CH, &e);
    net->logits = nalloc<float>(net, n, &e);
    net->dlogit = nalloc<float>(net, n, &e);
    net->lterm = nalloc<float>(net, n, &e);
    if (e != cudaSuccess) {
        amrlbm_net_destroy(net);
        return AMRLBM_ERR_CUDA;
    }
    // He-normal weights, zero biases
    std::vector<float> p(NPARAM, 0.f);
    Rng r{seed};
    auto fill = [&](int off, int count, int fan_in) {
        const double s = std::sqrt(2.0 / fan_in);
        for (int i = 0; i < count; ++i) p[off + i] = (float)(s * r.normal());
    };
    fill(O_W1, K1 * CH, K1);
    fill(O_W2, K2 * CH, K2);
    fill(O_W3, K2 * CH, K2);
    fill(O_WD, CH, CH);
    *out = net;
    return amrlbm_net_set(net, p.data());
}

int amrlbm_net_destroy(amrlbm_net* net) {
    if (!net) return AMRLBM_OK;
    if (net->st) cudaStreamSynchronize(net->st);
    for (void* q : net->allocs) cudaFree(q);
    if (net->st) cudaStreamDestroy(net->st);
    delete net;
    return AMRLBM_OK;
}

int32_t amrlbm_net_param_count(void) { return NPARAM; }

const char* amrlbm_net_last_error(const amrlbm_net* net) { return net ? net->err.c_str() : "no net"; }

int amrlbm_net_get(amrlbm_net* net, float* params) {
    if (!net || !params) return AMRLBM_ERR_ARG;
    NCK(cudaMemcpyAsync(params, net->p, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, net->st));
    NCK(cudaStreamSynchronize(net->st));
    return AMRLBM_OK;
}

int amrlbm_net_set(amrlbm_net* net, const float* params) {
    if (!net || !params) return AMRLBM_ERR_ARG;
    NCK(cudaMemcpyAsync(net->p, params, sizeof(float) * NPARAM, cudaMemcpyHostToDevice, net->st));
    NCK(cudaMemsetAsync(net->m1, 0, sizeof(float) * NPARAM, net->st));
    NCK(cudaMemsetAsync(net->m2, 0, sizeof(float) * NPARAM, net->st));
    net->steps = 0;
    repack(net);
    NCK(cudaStreamSynchronize(net->st));
    return AMRLBM_OK;
}

int amrlbm_net_forward(amrlbm_net* net, int32_t n, const float* x, float* logits) {
    if (!net || !logits) return AMRLBM_ERR_ARG;
    if (int r = load_batch(net, n, x, nullptr)) return r;
    forward(net, n);
    k_head<<<blocks_for(n), 256, 0, net->st>>>(n, net->pooled, net->p + O_WD, nullptr, 1.f,
                                               net->logits, net->dlogit, net->lterm);
    count_launches(1);
    NCK(cudaMemcpyAsync(logits, net->logits, sizeof(float) * n, cudaMemcpyDeviceToHost, net->st));
    NCK(cudaStreamSynchronize(net->st));
    return AMRLBM_OK;
}

// forward of samples already in device memory (the learned regrid's
// features), logits to the host; n may exceed the batch capacity
int amrlbm_net_forward_device(amrlbm_net* net, int32_t n, const float* x_dev, float* logits) {
    if (!net || !logits || n < 0 || (n > 0 && !x_dev)) return AMRLBM_ERR_ARG;
    const size_t per = (size_t)CIN * PIX;
    for (int i0 = 0; i0 < n; i0 += net->max_n) {
        const int b = std::min(net->max_n, n - i0);
        NCK(cudaMemcpyAsync(net->x, x_dev + per * i0, sizeof(float) * per * b,
                            cudaMemcpyDeviceToDevice, net->st));
        forward(net, b);
        k_head<<<blocks_for(b), 256, 0, net->st>>>(b, net->pooled, net->p + O_WD, nullptr, 1.f,
                                                   net->logits, net->dlogit, net->lterm);
        count_launches(1);
        NCK(cudaMemcpyAsync(logits + i0, net->logits, sizeof(float) * b, cudaMemcpyDeviceToHost, net->st));
    }
    NCK(cudaStreamSynchronize(net->st));
    return AMRLBM_OK;
}

int amrlbm_net_gradient(amrlbm_net* net, int32_t n, const float* x, const float* y,
                        float pos_weight, float* loss, float* grad) {
    if (!net || !y || !loss) return AMRLBM_ERR_ARG;
    if (int r = load_batch(net, n, x, y)) return r;
    forward(net, n);
    k_head<<<blocks_for(n), 256, 0, net->st>>>(n, net->pooled, net->p + O_WD, net->y, pos_weight,
                                               net->logits, net->dlogit, net->lterm);
    count_launches(1);
    backward(net, n);
    std::vector<float> lt(n);
    NCK(cudaMemcpyAsync(lt.data(), net->lterm, sizeof(float) * n, cudaMemcpyDeviceToHost, net->st));
    if (grad) NCK(cudaMemcpyAsync(grad, net->g, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, net->st));
    NCK(cudaStreamSynchronize(net->st));
    double s = 0.0;
    for (float v : lt) s += v;
    *loss = (float)(s / n);
    return AMRLBM_OK;
}

int amrlbm_net_train_step(amrlbm_net* net, int32_t n, const float* x, const float* y,
                          float pos_weight, float lr, float* loss) {
    if (int r = amrlbm_net_gradient(net, n, x, y, pos_weight, loss, nullptr)) return r;
    net->steps += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)net->steps), c2 = 1.f - std::pow(b2, (float)net->steps);
    k_adam<<<blocks_for(NPARAM), 256, 0, net->st>>>(NPARAM, net->p, net->g, net->m1, net->m2, lr, b1,
                                                    b2, 1e-8f, c1, c2);
    count_launches(1);
    repack(net);
    NCK(cudaStreamSynchronize(net->st));
    return AMRLBM_OK;
}

// the tensor-core product on its own, for its test: C = A B, A [M][K], B [K][N]
// (BF16 row-major on the host), C [M][N] FP32
int amrlbm_net_selftest_gemm(int32_t M, int32_t N, int32_t K, const uint16_t* A, const uint16_t* B,
                             float* C) {
    if (M < 1 || N < 1 || K < 1 || !A || !B || !C) return AMRLBM_ERR_ARG;
    __nv_bfloat16 *dA = nullptr, *dB = nullptr;
    float* dC = nullptr;
    cudaError_t e = cudaMalloc(&dA, sizeof(uint16_t) * (size_t)M * K);
    if (e == cudaSuccess) e = cudaMalloc(&dB, sizeof(uint16_t) * (size_t)K * N);
    if (e == cudaSuccess) e = cudaMalloc(&dC, sizeof(float) * (size_t)M * N);
    if (e == cudaSuccess) e = cudaMemcpy(dA, A, sizeof(uint16_t) * (size_t)M * K, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dB, B, sizeof(uint16_t) * (size_t)K * N, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        gemm(nullptr, M, N, K, dA, K, 1, dB, N, 1, dC, N);
        e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) e = cudaMemcpy(C, dC, sizeof(float) * (size_t)M * N, cudaMemcpyDeviceToHost);
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    return e == cudaSuccess ? AMRLBM_OK : AMRLBM_ERR_CUDA;
}

}  // extern "C"
