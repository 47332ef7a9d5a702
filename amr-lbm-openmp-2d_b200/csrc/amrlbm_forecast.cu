// amrlbm_forecast.cu - the learned regrid's forecast inside the time step:
// one fused kernel evaluates the refine-flag forecaster (amrlbm_net.cu) on
// every leaf that may still refine, between the error indicator of the
// regrid step (Err_Interface, Refine_Derefine.f90:327-351) and the refine
// flags (Refine_Derefine.f90:18-54), and raises the error of each leaf it
// forecasts to twice the refine tolerance. No counterpart in the reference,
// which flags blocks from the current field only.
//
// One CTA per leaf item, persistent over the leaf list. The item's samples
// (the four channels of amrlbm_block_features) are formed from the pool in
// shared memory, the three convolutions run as implicit products on the
// tensor cores (mma.sync m16n8k16, BF16 operands gathered straight from the
// channels-last activations, FP32 accumulation), bias and ReLU in the
// epilogue, the last layer reduced to its channel maxima in registers, and
// the dense output by one thread. The operands, their order along K and the
// rounding steps are those of the unfused network (k_input, k_im2col, k_gemm,
// k_bias_relu, k_maxpool, k_head), so the logits are bit for bit the same.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "amrlbm_dev.cuh"
#include "amrlbm_launch.h"

namespace {

constexpr int CH = 32, CIN = 4, TILE = 18, PIX = TILE * TILE;
constexpr int MTILES = (PIX + 15) / 16;  // 21 row tiles of 16 pixels
constexpr int K1P = 48, K2 = 9 * CH;     // layer 1 (36 padded to 48), layers 2 and 3
// shared row lengths (BF16) of the transposed weights W^T[n][k] and of the
// activations [pixel][channel]: chosen so that the 32 lanes of one fragment
// load hit 32 different banks
constexpr int KW1 = 72, KW2 = 328, AROW = 40;
constexpr int NT = 256, NWARP = NT / 32;

struct Smem {
    __nv_bfloat16 w1[CH][KW1];
    __nv_bfloat16 w2[CH][KW2];
    __nv_bfloat16 w3[CH][KW2];
    __nv_bfloat16 x0[PIX][CIN];  // the samples, channels last
    __nv_bfloat16 act[2][PIX][AROW];
    float b[3][CH], wd[CH], bd;
    float pmax[NWARP][CH];
    __align__(16) unsigned zero[4];  // the operand row outside the tile
};

__device__ __forceinline__ unsigned pack2(float lo, float hi) {
    return (unsigned)__bfloat16_as_ushort(__float2bfloat16(lo)) |
           ((unsigned)__bfloat16_as_ushort(__float2bfloat16(hi)) << 16);
}

// the im2col pair (k, k+1) of row `row` (k even, tap-major k = o*CI + ci):
// one 32-bit word of the activation (AW words per pixel), 0 outside
template <int CI, int AW>
__device__ __forceinline__ unsigned a_pair(const unsigned* act, int row, int k) {
    const int o = k / CI, ci = k % CI;
    if (o >= 9 || row >= PIX) return 0u;
    const int y = row / TILE + o / 3 - 1, x = row % TILE + o % 3 - 1;
    if (x < 0 || x >= TILE || y < 0 || y >= TILE) return 0u;
    return act[(y * TILE + x) * AW + (ci >> 1)];
}

// one row tile mt of a layer's product: acc[j][.] = columns 8j + 2q, +1 of
// rows 16mt + g (acc[j][0..1]) and 16mt + g + 8 (acc[j][2..3])
template <int CI, int AW, int K, int KW>
__device__ __forceinline__ void tile_product(const unsigned* act, const __nv_bfloat16 (*wt)[KW],
                                             int mt, int g, int q, float acc[4][4]) {
    const unsigned* w32 = reinterpret_cast<const unsigned*>(wt);
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[j][i] = 0.f;
    const int r0 = 16 * mt + g, r1 = r0 + 8;
#pragma unroll 2
    for (int k0 = 0; k0 < K; k0 += 16) {
        const unsigned a0 = a_pair<CI, AW>(act, r0, k0 + 2 * q);
        const unsigned a1 = a_pair<CI, AW>(act, r1, k0 + 2 * q);
        const unsigned a2 = a_pair<CI, AW>(act, r0, k0 + 2 * q + 8);
        const unsigned a3 = a_pair<CI, AW>(act, r1, k0 + 2 * q + 8);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int nrow = (8 * j + g) * (KW / 2);
            const unsigned b0 = w32[nrow + ((k0 + 2 * q) >> 1)];
            const unsigned b1 = w32[nrow + ((k0 + 2 * q + 8) >> 1)];
            asm volatile(
                "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                : "+f"(acc[j][0]), "+f"(acc[j][1]), "+f"(acc[j][2]), "+f"(acc[j][3])
                : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
        }
    }
}

// ReLU(acc + bias) of one row tile as BF16 into an activation
__device__ __forceinline__ void store_tile(const float acc[4][4], const float* bias, unsigned* o32,
                                           int mt, int g, int q) {
    const int r0 = 16 * mt + g, r1 = r0 + 8;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int n = 8 * j + 2 * q;
        if (r0 < PIX)
            o32[r0 * (AROW / 2) + (n >> 1)] =
                pack2(fmaxf(acc[j][0] + bias[n], 0.f), fmaxf(acc[j][1] + bias[n + 1], 0.f));
        if (r1 < PIX)
            o32[r1 * (AROW / 2) + (n >> 1)] =
                pack2(fmaxf(acc[j][2] + bias[n], 0.f), fmaxf(acc[j][3] + bias[n + 1], 0.f));
    }
}

// the first layer (4 input channels: one 16-column step spans four taps):
// operands gathered pair by pair
__device__ __forceinline__ void first_layer(const unsigned* x0, const __nv_bfloat16 (*wt)[KW1],
                                            const float* bias, __nv_bfloat16 (*out)[AROW], int warp,
                                            int g, int q) {
    unsigned* o32 = reinterpret_cast<unsigned*>(out);
    for (int mt = warp; mt < MTILES; mt += NWARP) {
        float acc[4][4];
        tile_product<CIN, CIN / 2, K1P, KW1>(x0, wt, mt, g, q, acc);
        store_tile(acc, bias, o32, mt, g, q);
    }
}

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void ldsm4(unsigned addr, unsigned& r0, unsigned& r1, unsigned& r2,
                                      unsigned& r3) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
                 : "r"(addr));
}

// a 32-channel layer: each 16-column step is one tap of 16 adjacent
// channels, so the operand fragments come by ldmatrix: A rows are the
// activation rows of the shifted pixels (a zero row outside the tile), B the
// transposed weights. The warp's row tiles mt = warp, warp + 8, warp + 16
// share each step's B fragments. Accumulation order along K as k_gemm's.
template <int KW>
__device__ __forceinline__ void conv32(const __nv_bfloat16 (*act)[AROW], const __nv_bfloat16 (*wt)[KW],
                                       unsigned zero_row, int warp, int lane, float acc[3][4][4]) {
    const int lr = lane & 15;
    int pix[3];
    unsigned vmask[3];  // bit o: tap o of this lane's row lies in the tile
#pragma unroll
    for (int u = 0; u < 3; ++u) {
        const int r = 16 * (warp + NWARP * u) + lr;
        pix[u] = r;
        vmask[u] = 0u;
        if (r < PIX) {
            const int y = r / TILE, x = r % TILE;
#pragma unroll
            for (int o = 0; o < 9; ++o) {
                const int yy = y + o / 3 - 1, xx = x + o % 3 - 1;
                if (yy >= 0 && yy < TILE && xx >= 0 && xx < TILE) vmask[u] |= 1u << o;
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int i = 0; i < 4; ++i) acc[u][j][i] = 0.f;
    }
    const unsigned abase = smem_addr(&act[0][0]) + (unsigned)((lane >> 4) * 8 * 2);
    const unsigned bbase = smem_addr(&wt[(lane & 7) + ((lane >> 4) << 3)][((lane >> 3) & 1) * 8]);
    const bool third = warp + 2 * NWARP < MTILES;
#pragma unroll
    for (int c = 0; c < K2 / 16; ++c) {
        const int o = c >> 1, c0 = (c & 1) * 16;
        const int shift = (o / 3 - 1) * TILE + (o % 3 - 1);
        unsigned b[8];
        ldsm4(bbase + (unsigned)(c * 32), b[0], b[1], b[2], b[3]);                    // n 0..15
        ldsm4(bbase + (unsigned)(16 * KW * 2 + c * 32), b[4], b[5], b[6], b[7]);      // n 16..31
#pragma unroll
        for (int u = 0; u < 3; ++u) {
            if (u == 2 && !third) break;
            const unsigned addr = ((vmask[u] >> o) & 1u)
                                      ? abase + (unsigned)(((pix[u] + shift) * AROW + c0) * 2)
                                      : zero_row;
            unsigned a0, a1, a2, a3;
            ldsm4(addr, a0, a1, a2, a3);
#pragma unroll
            for (int j = 0; j < 4; ++j)
                asm volatile(
                    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                    "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                    : "+f"(acc[u][j][0]), "+f"(acc[u][j][1]), "+f"(acc[u][j][2]), "+f"(acc[u][j][3])
                    : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b[2 * j]), "r"(b[2 * j + 1]));
        }
    }
}

template <bool MP>
__global__ void __launch_bounds__(NT, 2)
    k_forecast(const __grid_constant__ DevState s, ForecastNet net, int n_ids, const int* ids,
               float* logits, float horizon, double tol, float thr) {
    extern __shared__ __align__(16) unsigned char smraw[];
    Smem& S = *reinterpret_cast<Smem*>(smraw);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5, g = lane >> 2, q = lane & 3;
    {  // the weights, transposed, once per CTA
        const __nv_bfloat16* w1 = static_cast<const __nv_bfloat16*>(net.w1);
        const __nv_bfloat16* w2 = static_cast<const __nv_bfloat16*>(net.w2);
        const __nv_bfloat16* w3 = static_cast<const __nv_bfloat16*>(net.w3);
        for (int i = t; i < K1P * CH; i += NT) S.w1[i % CH][i / CH] = w1[i];
        for (int i = t; i < K2 * CH; i += NT) {
            S.w2[i % CH][i / CH] = w2[i];
            S.w3[i % CH][i / CH] = w3[i];
        }
        if (t < CH) {
            S.b[0][t] = net.b1[t];
            S.b[1][t] = net.b2[t];
            S.b[2][t] = net.b3[t];
            S.wd[t] = net.wd[t];
        }
        if (t == 0) S.bd = net.bd[0];
        if (t < 4) S.zero[t] = 0u;
    }
    const unsigned zero_row = smem_addr(S.zero);
    const bool explicit_ids = ids != nullptr;
    const int total = explicit_ids ? n_ids : s.cnt->nleaf;
    const int lmin = s.cnt->level_min, lmax = s.cnt->level_max;
    unsigned long long st_pred = 0, st_crit = 0, st_miss = 0, st_extra = 0;
    const int W = s.nx + 2;
    for (int i = blockIdx.x; i < total; i += gridDim.x) {
        const int n = explicit_ids ? ids[i] : s.leaf[i];
        if (!explicit_ids) {
            const int L = s.level[n];
            if (!(L < maxlv_of(s, n) && L >= lmin && L <= lmax)) continue;  // uniform in the CTA
        }
        __syncthreads();  // the previous item's reads of x0 and pmax are done
        // the samples (amrlbm_block_features): C, log(1 + e/tol), U horizon/dx
        const double dx = (double)s.dx[n];
        for (int c = t; c < PIX; c += NT) {
            const int x = c % W, y = c / W;
            double cc, cxp, cxm, cyp, cym, ux = 0.0, uy = 0.0;
            if (MP) {
                cc = s.mp.C[c_idx(s, n, x, y)];
                cxp = s.mp.C[c_idx(s, n, x + 1, y)];
                cxm = s.mp.C[c_idx(s, n, x - 1, y)];
                cyp = s.mp.C[c_idx(s, n, x, y + 1)];
                cym = s.mp.C[c_idx(s, n, x, y - 1)];
            } else {
                cc = s.C[c_idx(s, n, x, y)];
                cxp = s.C[c_idx(s, n, x + 1, y)];
                cxm = s.C[c_idx(s, n, x - 1, y)];
                cyp = s.C[c_idx(s, n, x, y + 1)];
                cym = s.C[c_idx(s, n, x, y - 1)];
            }
            const bool in = x >= 1 && x <= s.nx && y >= 1 && y <= s.ny;
            if (in) {
                ux = MP ? (double)s.mp.Ux[p_idx(s, n, x, y)] : s.Ux[p_idx(s, n, x, y)];
                uy = MP ? (double)s.mp.Uy[p_idx(s, n, x, y)] : s.Uy[p_idx(s, n, x, y)];
            }
            const double gx = cxp - cxm, gy = cyp - cym;
            const float f0 = (float)cc;
            const float f1 = (float)log1p(sqrt(gx * gx + gy * gy) / (2.0 * dx) / tol);
            const float f2 = in ? (float)(ux * horizon / dx) : 0.f;
            const float f3 = in ? (float)(uy * horizon / dx) : 0.f;
            unsigned* x32 = reinterpret_cast<unsigned*>(&S.x0[c][0]);
            x32[0] = pack2(f0, f1);
            x32[1] = pack2(f2, f3);
        }
        __syncthreads();
        first_layer(reinterpret_cast<const unsigned*>(S.x0), S.w1, S.b[0], S.act[0], warp, g, q);
        __syncthreads();
        {
            float acc[3][4][4];
            conv32<KW2>(S.act[0], S.w2, zero_row, warp, lane, acc);
#pragma unroll
            for (int u = 0; u < 3; ++u)
                if (warp + NWARP * u < MTILES)
                    store_tile(acc[u], S.b[1], reinterpret_cast<unsigned*>(S.act[1]), warp + NWARP * u,
                               g, q);
        }
        __syncthreads();
        // layer 3 reduced to the channel maxima (global max pool)
        float mx[4][2];
#pragma unroll
        for (int j = 0; j < 4; ++j) mx[j][0] = mx[j][1] = -1.f;
        {
            float acc[3][4][4];
            conv32<KW2>(S.act[1], S.w3, zero_row, warp, lane, acc);
#pragma unroll
            for (int u = 0; u < 3; ++u) {
                const int mt = warp + NWARP * u;
                if (mt >= MTILES) continue;
                const int r0 = 16 * mt + g, r1 = r0 + 8;
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int n2 = 8 * j + 2 * q;
                    if (r0 < PIX) {
                        mx[j][0] = fmaxf(mx[j][0], fmaxf(acc[u][j][0] + S.b[2][n2], 0.f));
                        mx[j][1] = fmaxf(mx[j][1], fmaxf(acc[u][j][1] + S.b[2][n2 + 1], 0.f));
                    }
                    if (r1 < PIX) {
                        mx[j][0] = fmaxf(mx[j][0], fmaxf(acc[u][j][2] + S.b[2][n2], 0.f));
                        mx[j][1] = fmaxf(mx[j][1], fmaxf(acc[u][j][3] + S.b[2][n2 + 1], 0.f));
                    }
                }
            }
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h)
#pragma unroll
                for (int o = 4; o < 32; o <<= 1)
                    mx[j][h] = fmaxf(mx[j][h], __shfl_xor_sync(0xffffffffu, mx[j][h], o));
        if (g == 0)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                S.pmax[warp][8 * j + 2 * q] = mx[j][0];
                S.pmax[warp][8 * j + 2 * q + 1] = mx[j][1];
            }
        __syncthreads();
        if (t == 0) {  // the dense output, in the order of k_head
            float z = S.bd;
            for (int c = 0; c < CH; ++c) {
                float p = S.pmax[0][c];
                for (int w = 1; w < NWARP; ++w) p = fmaxf(p, S.pmax[w][c]);
                z += S.wd[c] * p;
            }
            if (explicit_ids) {
                logits[i] = z;
            } else {
                const bool pr = z > thr, cr = s.err[n] > tol;
                st_pred += pr;
                st_crit += cr;
                st_miss += cr && !pr;
                st_extra += pr && !cr;
                if (pr && !cr) s.err[n] = 2.0 * tol;
            }
        }
    }
    if (!explicit_ids && t == 0 && (st_pred | st_crit)) {
        atomicAdd(&s.cnt->rstat[1], st_pred);
        atomicAdd(&s.cnt->rstat[2], st_crit);
        atomicAdd(&s.cnt->rstat[3], st_miss);
        atomicAdd(&s.cnt->rstat[4], st_extra);
    }
}

template <bool MP>
void forecast_launch(const DevState& s, const LaunchCfg& lc, cudaStream_t st, const ForecastNet& net,
                     int n_ids, const int* ids, float* logits, float horizon, double tol, float thr) {
    const size_t sm = sizeof(Smem);
    cudaFuncSetAttribute(k_forecast<MP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int grid = 2 * lc.num_sms;
    if (ids && n_ids < grid) grid = n_ids > 0 ? n_ids : 1;
    k_forecast<MP><<<grid, NT, sm, st>>>(s, net, n_ids, ids, logits, horizon, tol, thr);
}

}  // namespace

void launch_forecast(const DevState& s, const LaunchCfg& lc, cudaStream_t st, const ForecastNet& net,
                     int n_ids, const int* ids, float* logits, float horizon, double tol, float thr) {
    if (s.mp.fmt)
        forecast_launch<true>(s, lc, st, net, n_ids, ids, logits, horizon, tol, thr);
    else
        forecast_launch<false>(s, lc, st, net, n_ids, ids, logits, horizon, tol, thr);
    count_launches(1);
}
