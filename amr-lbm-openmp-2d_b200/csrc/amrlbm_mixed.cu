// amrlbm_mixed.cu - the mixed-precision time step: populations stored in 16
// bits (FP16 or BF16) as deviations, collision, ghost-cell interpolation and
// streaming in FP32 (compiled with FMA contraction: nothing here is compared
// bit for bit). The arithmetic is that of the FP64 kernels
// (LBM_Subroutines.f90:41-240, Fill_Ghost_Cells_*.f90, BC_Cell.f90) in FP32;
// the ghost cells come from the same fill plans and foreign-cell records.
//
// Storage (MpState, amrlbm_dev.cuh): per cell and field the rest population
// f_1 in FP32 and d_q = (f_q - r_q f_1) * scale in 16 bits, r_q = w_q/w_1
// (1/4 for the axis directions, 1/16 for the diagonals). At rest every
// population is w_q times the same moment, so d_q holds only the velocity,
// normal and forcing terms: a few per mille of f_q instead of f_q itself.
// A cell decodes from its own words, so a ghost cell interpolated from
// another block's cells needs nothing but those cells.
//
// One CTA of N*N threads per leaf item (one thread per cell), grid-stride
// over the items in work order. Items do not wait for one another where the
// plans' foreign cells make every ring depend on interiors only; where a
// coarse-to-fine stencil reads a coarser neighbour's ring cell that is itself
// coarse-to-fine or a wall cell, the launch takes the items in level order
// (see claim).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstddef>
#include <map>
#include <utility>

#include "amrlbm_fast.cuh"
#include "amrlbm_launch.h"
#include "amrlbm_plan.cuh"

void count_launches(int n);

namespace {

// floats of one block's C plane (both rings), as Geo<N>::cplane
__host__ __device__ constexpr int cplane_of(int N) { return (((N + 4) * (((N + 6 + 3) / 4) * 4) + 15) / 16) * 16; }

// ---- encoding ------------------------------------------------------------
template <int FMT>
__device__ __forceinline__ unsigned short enc(float v) {
    if (FMT == 1) return __half_as_ushort(__float2half_rn(v));
    return __bfloat16_as_ushort(__float2bfloat16_rn(v));
}
template <int FMT>
__device__ __forceinline__ float dec(unsigned short u) {
    if (FMT == 1) return __half2float(__ushort_as_half(u));
    return __bfloat162float(__ushort_as_bfloat16(u));
}
// Randomised rounding: a value rounds to one of its two neighbours in the
// narrower format, the one away from zero with probability equal to the
// dropped fraction, by adding random bits below the kept ones and
// truncating. Unbiased like round-to-nearest, but the errors of neighbouring
// cells holding nearly the same value are independent instead of equal, so
// they cancel in sums over the domain (the mass) instead of adding up step
// after step. The random bits hash the value with a salt (cell and
// population): the same state gives the same bits.
__device__ __forceinline__ unsigned rnd_bits(unsigned v, unsigned salt) {
    unsigned x = v ^ (salt * 0x9e3779b9u);
    x ^= x >> 16;
    x *= 0x7feb352du;  // multiplier of C. Wellons' lowbias32
    x ^= x >> 15;
    return x;
}
template <int FMT>
__device__ __forceinline__ unsigned short enc_sr(float v, unsigned salt) {
    const unsigned b = __float_as_uint(v), r = rnd_bits(b, salt);
    if (FMT == 2)  // BF16 keeps the upper 16 bits of the FP32 word
        return (unsigned short)((b + (r & 0xffffu)) >> 16);
    // FP16 keeps 10 of FP32's 23 mantissa bits in its normal range; below it
    // (|v| < 2^-14) its spacing is 2^-24
    if (fabsf(v) < 6.103515625e-05f)
        return __half_as_ushort(__float2half_rz(v + copysignf((float)(r >> 8) * 3.5527136788e-15f, v)));
    return __half_as_ushort(__float2half_rz(__uint_as_float(b + (r & 0x1fffu))));
}
// mass_encode: the eight deviations of a cell's h populations are rounded
// one after the other, each with the rounding error of the ones before it
// subtracted (error diffusion within the cell). Their sum, the cell's share
// of C and of the phase mass, then carries only the last rounding error
// instead of the sum of eight independent ones.

// FP64 -> FP32 the same way (29 dropped mantissa bits)
__device__ __forceinline__ float f32_sr(double d, unsigned salt) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(d);
    const unsigned r = rnd_bits((unsigned)(b >> 29), salt);
    return __double2float_rz(__longlong_as_double((long long)(b + (r & 0x1fffffffu))));
}

// r_q = w_q / w_1
__host__ __device__ __forceinline__ constexpr float rq(int q) { return q <= 5 ? 0.25f : 0.0625f; }
__device__ __forceinline__ float waf(int q) {
    return q == 1 ? 16.f / 36.f : (q <= 5 ? 4.f / 36.f : 1.f / 36.f);
}

// rest-plane index of A-pool offset off (= G.a(blk, 1, x, y))
template <int N>
__device__ __forceinline__ unsigned a_rest(const Geo<N>& G, unsigned off) {
    const unsigned blk = off / (9u * (unsigned)G.aplane);
    return off - 8u * (unsigned)G.aplane * blk;
}

// population q of field f (0 h, 1 g) of the cell at A offset off; CG: the
// cell may have been written by another CTA of the same launch (read through L2)
template <int N, int FMT, bool CG = false>
__device__ __forceinline__ float dec_a(const MpState& m, const Geo<N>& G, int f, unsigned off,
                                       int q) {
    const float* r = (f ? m.A1g : m.A1h) + a_rest(G, off);
    const float rest = CG ? __ldcg(r) : __ldg(r);
    if (q == 1) return rest;
    const unsigned short* dp = (f ? m.Adg : m.Adh) + off + (unsigned)(q - 1) * G.aplane;
    const unsigned short d = CG ? __ldcg(dp) : __ldg(dp);
    return dec<FMT>(d) * (f ? m.isg : m.ish) + rq(q) * rest;
}

// generic-proxy writes of earlier launches seen by the bulk copies that read them
__device__ __forceinline__ void fence_proxy_async_all() {
    asm volatile("fence.proxy.async;" ::: "memory");
}

// ---- level order ----------------------------------------------------------
// Fill q of a launch needs level order when a coarse-to-fine stencil reads a
// coarser neighbour's ring cell that is not a foreign cell (fillinfo[q]):
// then items are claimed in work order (coarser levels first) from queue q,
// each item publishes its block's flag once its ring and walls are in
// memory, and an item waits (bounded) for the flags of the coarser
// neighbours it reads. Without it, CTA b takes items b, b + grid, ...
// (the barrier first: the previous item's shared data has been read)
__device__ __forceinline__ int claim(const DevState& s, bool fast, int q, int k, int* sk) {
    __syncthreads();
    if (fast) return k < 0 ? (int)blockIdx.x : k + (int)gridDim.x;
    if (threadIdx.x == 0) *sk = (int)atomicAdd(&s.queue[4 * q], 1u);
    __syncthreads();
    return *sk;
}
// waits for the coarser neighbours whose rings item k's fill q reads;
// block-uniform, ends with a barrier
__device__ __forceinline__ void wait_for_coarser(const DevState& s, int q, int k) {
    const int* w = s.nbinfo + (size_t)k * NBI_STRIDE;
    const int mask = __ldg(w + (int)(offsetof(NbInfo, wait) / sizeof(int)) + q);
    const int t = threadIdx.x;
    if (t < 8 && ((mask >> (t + 1)) & 1))
        if (!spin_flag(fill_flags(s, q) + __ldg(w + t + 1), s.spin_limit))
            set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 300 + q);
    __syncthreads();
}
// all 9 populations of field f of the cell at A offset off
template <int N, int FMT>
__device__ __forceinline__ void dec_a9(const MpState& m, const Geo<N>& G, int f, unsigned off,
                                       float* v) {
    const float rest = __ldg((f ? m.A1g : m.A1h) + a_rest(G, off));
    const unsigned short* D = (f ? m.Adg : m.Adh) + off;
    const float is = f ? m.isg : m.ish;
    v[0] = rest;
#pragma unroll
    for (int q = 2; q <= 9; ++q) v[q - 1] = dec<FMT>(__ldg(D + (unsigned)(q - 1) * G.aplane)) * is + rq(q) * rest;
}
// writes the 9 populations v of field f of cell (x, y) of block n into A;
// rest (if given): v[0] before its rounding to FP32
template <int N, int FMT>
__device__ __forceinline__ void enc_a9(const MpState& m, const Geo<N>& G, int f, int n, int x,
                                       int y, float* v, const double* rest = nullptr) {
    const size_t off = G.a(n, 1, x, y);
    if (rest) v[0] = f32_sr(*rest, (unsigned)off * 2u + f + 0x51ed27u);
    (f ? m.A1g : m.A1h)[off - (size_t)8 * G.aplane * n] = v[0];
    unsigned short* D = (f ? m.Adg : m.Adh) + off;
    const float sc = f ? m.sg : m.sh;
    float e = 0.f;  // h: rounding error carried (mass_encode)
#pragma unroll
    for (int q = 2; q <= 9; ++q) {
        const float x = (v[q - 1] - rq(q) * v[0]) * sc - e;
        const unsigned short w = enc_sr<FMT>(x, (unsigned)(off + (size_t)(q - 1) * G.aplane) * 2u + f);
        D[(size_t)(q - 1) * G.aplane] = w;
        if (f == 0) e = dec<FMT>(w) - x;
    }
}

// Biquadratic_from_Fine / _Coarse (Interpolations.f90:2-138) of a plan entry
// in FP32 (same stencil as plan_combine)
__device__ __forceinline__ float combine_f(int meta, const float* g) {
    const int kind = plan_kind(meta);
    const int Jx = (meta >> 3) & 1, Jy = (meta >> 4) & 1;
    const float b = (kind == 2) ? 6.f : 30.f;
    const int ax = (kind == 2) ? 3 - 4 * Jx : 5 - 8 * Jx, ay = (kind == 2) ? 3 - 4 * Jy : 5 - 8 * Jy;
    const float Ax = (float)ax, Cx = (float)(2 - ax), Ay = (float)ay, Cy = (float)(2 - ay);
    float t[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) t[r] = Ay * g[3 * r] + b * g[3 * r + 1] + Cy * g[3 * r + 2];
    const float o = Ax * t[0] + b * t[1] + Cx * t[2];
    return (kind == 2) ? o * (1.f / 64.f) : o * (1.f / 1024.f);
}

// ---- C ghost rings ---------------------------------------------------------
// foreign cell j of a C fill (records fb) from the FP32 C pool
// (fb in memory or staged in shared memory)
__device__ __forceinline__ float foreign_cf(const int* fb, int fmax, int j, const float* C) {
    const int meta = fb[j];
    if (plan_kind(meta) == 1) return __ldg(C + (unsigned)fb[fmax + j]);
    float g[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) g[i] = __ldg(C + (unsigned)fb[(1 + i) * fmax + j]);
    return combine_f(meta, g);
}

// the C ring of width w of item k (block n) on the tile T (pool layout of
// one block) and in memory; foreign values in Fs. cg (level order): sources
// through L2, since a coarser neighbour's ring is written in this launch;
// without level order every source in memory is an interior cell that no
// item of the launch writes. Ends with a barrier.
template <int N>
__device__ void ring_c(const DevState& s, const Geo<N>& G, const int* pl, int R, int w,
                       const ItemRec& r, const float* Fs, float* T, bool cg) {
    const float* C = s.mp.C;
    for (int e = threadIdx.x; e < r.na + r.n2 + r.n3; e += blockDim.x) {
        const int meta = pl[e];
        const int kind = plan_kind(meta);
        if (kind == 0) continue;
        int x, y;
        if (w == 2)
            ring2_xy(meta >> 8, G.nx, G.ny, x, y);
        else
            ring1_xy(meta >> 8, G.nx, G.ny, x, y);
        if (kind < 0) {
            set_error(s, 4 /*AMRLBM_ERR_LEVEL_JUMP*/, r.n);
            continue;
        }
        float v;
        if (kind == 1) {
            v = __ldg(C + (unsigned)pl[R + e]);
        } else {
            float g[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) {
                const unsigned wd = (unsigned)pl[(1 + i) * R + e];
                g[i] = (kind == 3 && (wd & kIndirect)) ? Fs[wd & ~kIndirect]
                                                        : (cg ? __ldcg(C + wd) : __ldg(C + wd));
            }
            v = combine_f(meta, g);
        }
        T[G.c(0, x, y)] = v;
        s.mp.C[G.c(r.n, x, y)] = v;
    }
    __syncthreads();
}

// Symmetric_C(2)_3/4 (BC_Cell.f90:46-104) on the tile and in memory. Ends
// with a barrier.
template <int N>
__device__ void walls_c(const DevState& s, const Geo<N>& G, int n, int w, bool w3, bool w4,
                        float* T) {
    if (w3 || w4) {
        const int nx = G.nx, ny = G.ny;
        for (int idx = threadIdx.x; idx < (nx + 2 * w) * w * 2; idx += blockDim.x) {
            const int X = idx % (nx + 2 * w) + 1 - w, a = (idx / (nx + 2 * w)) % w + 1;
            const bool top = idx >= (nx + 2 * w) * w;
            if (top ? !w4 : !w3) continue;
            const int ys = top ? ny + 1 - a : a, yd = top ? ny + a : 1 - a;
            const float v = T[G.c(0, X, ys)];
            T[G.c(0, X, yd)] = v;
            s.mp.C[G.c(n, X, yd)] = v;
        }
    }
    __syncthreads();
}

// the block's C (both rings) into the tile; ends with a barrier
template <int N>
__device__ __forceinline__ void load_tile(const DevState& s, const Geo<N>& G, int n, float* T) {
    const float* src = s.mp.C + (size_t)n * G.cplane;
    for (int i = threadIdx.x; i < G.cplane; i += blockDim.x) T[i] = __ldg(src + i);
}

// ---- per-cell physics (LBM_Subroutines.f90) in FP32 -------------------------
template <int N>
struct CellC {
    const float* T;
    const Geo<N>& G;
    int x, y;
    __device__ __forceinline__ float operator()(int a, int b) const { return T[G.c(0, x + a, y + b)]; }
};

// Gradient_AMR (:293-312)
template <class CF>
__device__ __forceinline__ void grad_iso(CF Cs, float inv_dx, float& gx, float& gy) {
    gx = ((Cs(1, 0) - Cs(-1, 0)) * (1.f / 3.f) +
          (Cs(1, 1) + Cs(1, -1) - Cs(-1, 1) - Cs(-1, -1)) * (1.f / 12.f)) * inv_dx;
    gy = ((Cs(0, 1) - Cs(0, -1)) * (1.f / 3.f) +
          (Cs(1, 1) + Cs(-1, 1) - Cs(1, -1) - Cs(-1, -1)) * (1.f / 12.f)) * inv_dx;
}
// Laplacian_AMR + Chemical_Potential_AMR (:94-112, :316-333)
template <class CF>
__device__ __forceinline__ float chem_pot(CF Cs, const PhysF& ph, float inv_dx2) {
    const float D2C = (Cs(-1, -1) + Cs(1, -1) + Cs(-1, 1) + Cs(1, 1) +
                       4.f * (Cs(0, -1) + Cs(-1, 0) + Cs(1, 0) + Cs(0, 1)) - 20.f * Cs(0, 0)) *
                      (1.f / 6.f);
    const float c = Cs(0, 0);
    return ph.Beta4 * c * (c - 1.f) * (c - 0.5f) - ph.kappa * D2C * inv_dx2;
}
// Macroscopic_Values_g_AMR (:205-240): P, Ux, Uy from g[0..8] and the C stencil
template <class CF>
__device__ __forceinline__ void macro_g(CF Cs, const PhysF& ph, float inv_dx, const float* g,
                                        float& P, float& Ux, float& Uy) {
    float gx, gy;
    grad_iso(Cs, inv_dx, gx, gy);
    const float mu = chem_pot(Cs, ph, inv_dx * inv_dx);
    const float c0 = Cs(0, 0);
    const float Rho = ph.Rhol + c0 * ph.dRho;
    const float Fb = (ph.Rhoh - Rho) * ph.Gy;
    const float sx = g[1] - g[3] + g[5] - g[6] - g[7] + g[8];
    const float sy = g[2] - g[4] + g[5] + g[6] - g[7] - g[8];
    const float rr = __frcp_rn(Rho);
    Ux = (3.f * sx + 0.5f * (mu * gx)) * rr;
    Uy = (3.f * sy + 0.5f * (mu * gy + Fb)) * rr;
    float sp = 0.f;
#pragma unroll
    for (int k = 0; k < 9; ++k) sp += g[k];
    P = sp + ph.dRho6 * (Ux * gx + Uy * gy);
}

// Collision_h_g_AMR (:116-189) of one cell: h[0..8], g[0..8] post-streaming
// in, post-collision out. FUSED: P, U from Macroscopic_Values_g_AMR of g here.
template <bool FUSED, bool BGK, class CF>
__device__ __forceinline__ void collide(CF Cs, const PhysF& ph, float inv_dx, float* h, float* g,
                                        float& P, float& Ux, float& Uy, double& h1) {
    const float c0 = Cs(0, 0);
    const float mu = chem_pot(Cs, ph, inv_dx * inv_dx);
    auto Ec = [&](int k) { return (Cs(d_ex(k), d_ey(k)) - Cs(-d_ex(k), -d_ey(k))) * (0.5f * inv_dx); };
    auto Em = [&](int k) {
        return (-Cs(-d_ex(k), -d_ey(k)) - 3.f * c0 + 5.f * Cs(d_ex(k), d_ey(k)) -
                Cs(2 * d_ex(k), 2 * d_ey(k))) * (0.25f * inv_dx);
    };
    // Gradient_ED_AMR (:281-289)
    const float DcDx = (Ec(2) - Ec(4)) * (1.f / 3.f) + (Ec(6) - Ec(7) - Ec(8) + Ec(9)) * (1.f / 12.f);
    const float DcDy = (Ec(3) - Ec(5)) * (1.f / 3.f) + (Ec(6) + Ec(7) - Ec(8) - Ec(9)) * (1.f / 12.f);
    const float it = rsqrtf(DcDx * DcDx + DcDy * DcDy + 1.e-32f);  // normal_AMR (:25-37)
    const float ni = DcDx * it, nj = DcDy * it;
    const float Rho = ph.Rhol + c0 * ph.dRho;
    const float Fb = (ph.Rhoh - Rho) * ph.Gy;
    if (FUSED) macro_g(Cs, ph, inv_dx, g, P, Ux, Uy);
    const float tmp = 12.f * (1.f - c0) * ph.iW * ph.M0;
    const float U215 = 1.5f * (Ux * Ux + Uy * Uy);
    const float ud_c = Ux * DcDx + Uy * DcDy;
    const float DmX = (Em(2) - Em(4)) * (1.f / 3.f) + (Em(6) - Em(7) - Em(8) + Em(9)) * (1.f / 12.f);
    const float DmY = (Em(3) - Em(5)) * (1.f / 3.f) + (Em(6) + Em(7) - Em(8) - Em(9)) * (1.f / 12.f);
    const float ud_m = Ux * DmX + Uy * DmY;
    float tau;
    if (c0 < 0.f)
        tau = ph.taul5;
    else if (c0 > 1.f)
        tau = ph.tauh5;
    else
        tau = __frcp_rn(c0 * ph.itau_d + ph.itaul) + 0.5f;
    const float s9 = __frcp_rn(tau);
    // conservation of C: the rest equilibrium takes what the moving ones
    // leave of c0 (the FP32 weights sum to 1 + 8e-9, not 1), and each
    // population relaxes as h + wc (heq - h) (omwc + wc is not 1 in FP32
    // either); the rest population, which carries 4/9 of C and is stored in
    // FP32, is formed in FP64 (h1) for the caller's randomised rounding
    double heq1 = (double)c0;
    float f[9], hm[9];
#pragma unroll
    for (int k = 9; k >= 1; --k) {
        const float wk = waf(k);
        const float eU = (float)d_ex(k) * Ux + (float)d_ey(k) * Uy;
        const float eN = (float)d_ex(k) * ni + (float)d_ey(k) * nj;
        const float Gm = wk * (1.f + eU * (3.f + 4.5f * eU) - U215);
        if (k > 1) {
            const float heq = c0 * (Gm + tmp * wk * eN);
            heq1 -= (double)heq;
            h[k - 1] = h[k - 1] + ph.wc * (heq - h[k - 1]);
        } else {
            h1 = (double)h[0] + (double)ph.wc * (heq1 - (double)h[0]);
            h[0] = (float)h1;
        }
        const float Ak = (Gm - wk) * ph.dRho3 + Gm * mu;
        const float Bk = ((float)d_ey(k) - Uy) * Gm * Fb;
        const float hc = Ak * (Ec(k) - ud_c) + Bk;
        const float geq = P * wk + (Gm - wk) * Rho * (1.f / 3.f) - 0.5f * hc;
        f[k - 1] = BGK ? g[k - 1] * (1.f - s9) + geq * s9 : g[k - 1] - geq;
        hm[k - 1] = Ak * (Em(k) - ud_m) + Bk;
    }
    if (BGK) {
#pragma unroll
        for (int k = 0; k < 9; ++k) g[k] = f[k] + hm[k];
        return;
    }
    // MRT_Collision_AMR (:348-361)
    float m[10];
    m[1] = f[0] + f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8];
    m[2] = -4.f * f[0] - f[1] - f[2] - f[3] - f[4] + 2.f * (f[5] + f[6] + f[7] + f[8]);
    m[3] = 4.f * f[0] - 2.f * (f[1] + f[2] + f[3] + f[4]) + f[5] + f[6] + f[7] + f[8];
    m[4] = f[1] - f[3] + f[5] - f[6] - f[7] + f[8];
    m[5] = -2.f * (f[1] - f[3]) + f[5] - f[6] - f[7] + f[8];
    m[6] = f[2] - f[4] + f[5] + f[6] - f[7] - f[8];
    m[7] = -2.f * (f[2] - f[4]) + f[5] + f[6] - f[7] - f[8];
    m[8] = (f[1] - f[2] + f[3] - f[4]) * s9;
    m[9] = (f[5] - f[6] + f[7] - f[8]) * s9;
    const float b1 = 4.f * m[1] - m[2] - 2.f * m[3];
    const float b2 = 4.f * m[1] + 2.f * m[2] + m[3];
    float o[9];
    o[0] = 4.f * (m[1] - m[2] + m[3]);
    o[1] = b1 + 6.f * (m[4] - m[5]) + 9.f * m[8];
    o[2] = b1 + 6.f * (m[6] - m[7]) - 9.f * m[8];
    o[3] = b1 - 6.f * (m[4] - m[5]) + 9.f * m[8];
    o[4] = b1 - 6.f * (m[6] - m[7]) - 9.f * m[8];
    o[5] = b2 + 6.f * m[4] + 3.f * m[5] + 6.f * m[6] + 3.f * m[7] + 9.f * m[9];
    o[6] = b2 - 6.f * m[4] - 3.f * m[5] + 6.f * m[6] + 3.f * m[7] - 9.f * m[9];
    o[7] = b2 - 6.f * m[4] - 3.f * m[5] - 6.f * m[6] - 3.f * m[7] + 9.f * m[9];
    o[8] = b2 + 6.f * m[4] + 3.f * m[5] - 6.f * m[6] - 3.f * m[7] - 9.f * m[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) g[k] = (g[k] - o[k] * (1.f / 36.f)) + hm[k];
}

// post-streaming populations of cell (x, y) of block n (B pool)
template <int N, int FMT>
__device__ __forceinline__ void dec_b9(const MpState& m, const Geo<N>& G, int f, int n, int x,
                                       int y, float* v) {
    const size_t c = (size_t)(y - 1) * G.nx + (x - 1);
    const float rest = __ldg((f ? m.B1g : m.B1h) + (size_t)n * G.bplane + c);
    const unsigned short* D = (f ? m.Bdg : m.Bdh);
    const float is = f ? m.isg : m.ish;
    v[0] = rest;
#pragma unroll
    for (int q = 2; q <= 9; ++q) v[q - 1] = dec<FMT>(__ldg(D + G.bb(n, q, x, y))) * is + rq(q) * rest;
}
template <int N, int FMT>
__device__ __forceinline__ void enc_b9(const MpState& m, const Geo<N>& G, int f, int n, int x,
                                       int y, const float* v) {
    const size_t c = (size_t)(y - 1) * G.nx + (x - 1);
    (f ? m.B1g : m.B1h)[(size_t)n * G.bplane + c] = v[0];
    unsigned short* D = f ? m.Bdg : m.Bdh;
    const float sc = f ? m.sg : m.sh;
    float e = 0.f;  // h: rounding error carried (mass_encode)
#pragma unroll
    for (int q = 2; q <= 9; ++q) {
        const float xv = (v[q - 1] - rq(q) * v[0]) * sc - e;
        const unsigned short w = enc_sr<FMT>(xv, (unsigned)G.bb(n, q, x, y) * 2u + f + 0x9e3779b9u);
        D[G.bb(n, q, x, y)] = w;
        if (f == 0) e = dec<FMT>(w) - xv;
    }
}

// ---- K1: Fill_Ghost_Cells_C2 + Symmetric_C2 + collision ----------------------
// READ_PU: P, U of the current state are in memory (a tail ran before);
// else Macroscopic_Values_g_AMR runs inside the collision. wr: the last step of
// an amrlbm_step call (P, U written).
//
// Without level order each CTA takes items b, b + grid, ... with two shared
// stages: one bulk copy group (cp.async.bulk + mbarrier, this GPU's memory
// only) brings an item's C tile, its post-streaming h and g words and its C2
// plan and foreign records, and is issued for the next item once the current
// item's ring is on its tile, so it lands while the current item collides.

// one stage: C tile | h deviation planes | g deviation planes | h rest | g
// rest | plan words | foreign records (every part a multiple of 16 bytes)
template <int N>
struct K1Stage {
    static constexpr int R = 4 * (N + N) + 16;  // ring2_len
    static constexpr int FMAX = 2 * N + 28;     // foreign slots per leaf
    static constexpr int TILE = cplane_of(N) * 4, DEV = 9 * N * N * 2, REST = N * N * 4;
    static constexpr int PLAN = R * PLAN_INTS * 4, FRN = FMAX * FRN_INTS * 4;
    static constexpr int BYTES = TILE + 2 * DEV + 2 * REST + PLAN + FRN;
    static constexpr int O_DH = TILE, O_DG = O_DH + DEV, O_RH = O_DG + DEV, O_RG = O_RH + REST,
                         O_PL = O_RG + REST, O_FR = O_PL + PLAN;
};

// collision of cell (x, y) of block n from its decoded populations and the
// filled tile; writes A (and P, U where asked)
template <int N, int FMT, bool READ_PU, bool BGK>
__device__ __forceinline__ void collide_store(const DevState& s, const Geo<N>& G, int n, int x,
                                              int y, const float* T, float* h, float* g, int wr) {
    const MpState& m = s.mp;
    const float inv_dx = 1.f / (float)__ldg(s.dx + n);
    float P, Ux, Uy;
    if (READ_PU) {
        P = __ldg(m.P + G.p(n, x, y));
        Ux = __ldg(m.Ux + G.p(n, x, y));
        Uy = __ldg(m.Uy + G.p(n, x, y));
    }
    double h1;
    const PhysF& ph = s.n_inst ? m.phys[s.inst[n]] : m.ph;
    collide<!READ_PU, BGK>(CellC<N>{T, G, x, y}, ph, inv_dx, h, g, P, Ux, Uy, h1);
    enc_a9<N, FMT>(m, G, 0, n, x, y, h, &h1);
    enc_a9<N, FMT>(m, G, 1, n, x, y, g);
    if (wr && !READ_PU) {
        m.P[G.p(n, x, y)] = P;
        m.Ux[G.p(n, x, y)] = Ux;
        m.Uy[G.p(n, x, y)] = Uy;
    }
}

template <int N, int FMT, bool READ_PU, bool BGK>
__global__ void __launch_bounds__(N * N, (N == 16 ? 3 : 8)) k_mp_collide(const __grid_constant__ DevState s, int wr) {
    using SL = K1Stage<N>;
    extern __shared__ __align__(128) unsigned char sm[];
    const Geo<N> G(s);
    __shared__ __align__(16) int rec[2][REC_WORDS + 1];
    __shared__ int sk;
    const int t = threadIdx.x, total = s.lvl_off[AMR_MAXLV];
    const int R = SL::R;
    const MpState& m = s.mp;
    if (blockIdx.x == 0 && t == 0)
        atomicAdd(&s.cnt->updates, (unsigned long long)total * (unsigned long long)(N * N));
    const int x = t % N + 1, y = t / N + 1, c = t;
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(sm);  // [2]
    unsigned char* stages = sm + 128;
    float* Fs = reinterpret_cast<float*>(stages + 2 * SL::BYTES);  // [FMAX]
    const bool fast = s.fillinfo[Q_FILLC] == 0;
    if (!fast) {  // level order: items claimed in work order, no staging
        float* T = reinterpret_cast<float*>(stages);
        for (int k = claim(s, false, Q_FILLC, -1, &sk); k < total; k = claim(s, false, Q_FILLC, k, &sk)) {
            item_rec_stage(s, k, Q_FILLC, rec[0]);
            __syncthreads();
            const ItemRec r = item_rec_of(rec[0]);
            const int n = r.n;
            load_tile<N>(s, G, n, T);
            const int* fb = s.frn_c + (size_t)k * s.fmax * FRN_INTS;
            for (int j = t; j < r.nf; j += blockDim.x) Fs[j] = foreign_cf(fb, s.fmax, j, m.C);
            __syncthreads();
            wait_for_coarser(s, Q_FILLC, k);
            ring_c<N>(s, G, s.plan_c2 + (size_t)k * R * PLAN_INTS, R, 2, r, Fs, T, true);
            walls_c<N>(s, G, n, 2, r.w3, r.w4, T);
            publish_ring(s, Q_FILLC, n);
            float h[9], g[9];
            dec_b9<N, FMT>(m, G, 0, n, x, y, h);
            dec_b9<N, FMT>(m, G, 1, n, x, y, g);
            collide_store<N, FMT, READ_PU, BGK>(s, G, n, x, y, T, h, g, wr);
        }
        queue_done(s, Q_FILLC);
        return;
    }
    int k = blockIdx.x;
    if (k >= total) return;
    // thread 0 copies item kk (block nn) into stage st
    auto issue = [&](int st, int kk, int nn) {
        unsigned char* S = stages + st * SL::BYTES;
        fence_proxy_async_all();
        fence_proxy_async();
        mbar_expect_tx(&bar[st], SL::BYTES);
        bulk_g2s(S, m.C + (size_t)nn * G.cplane, SL::TILE, &bar[st]);
        bulk_g2s(S + SL::O_DH, m.Bdh + (size_t)nn * 9 * G.bplane, SL::DEV, &bar[st]);
        bulk_g2s(S + SL::O_DG, m.Bdg + (size_t)nn * 9 * G.bplane, SL::DEV, &bar[st]);
        bulk_g2s(S + SL::O_RH, m.B1h + (size_t)nn * G.bplane, SL::REST, &bar[st]);
        bulk_g2s(S + SL::O_RG, m.B1g + (size_t)nn * G.bplane, SL::REST, &bar[st]);
        bulk_g2s(S + SL::O_PL, s.plan_c2 + (size_t)kk * R * PLAN_INTS, SL::PLAN, &bar[st]);
        bulk_g2s(S + SL::O_FR, s.frn_c + (size_t)kk * s.fmax * FRN_INTS, SL::FRN, &bar[st]);
    };
    if (t == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
    }
    item_rec_stage(s, k, Q_FILLC, rec[0]);
    __syncthreads();
    if (t == 0) issue(0, k, rec[0][0]);
    unsigned phase = 0;
    int st = 0;
    while (k < total) {
        const int kn = k + gridDim.x;
        if (kn < total) item_rec_stage_async(s, kn, Q_FILLC, rec[st ^ 1]);
        if (__syncthreads_or(mbar_wait(&bar[st], (phase >> st) & 1u) ? 0 : 1)) {
            if (t == 0) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 110);
            mbar_wait(&bar[st], (phase >> st) & 1u);
            cp_async_wait_all();
            break;
        }
        phase ^= 1u << st;
        unsigned char* S = stages + st * SL::BYTES;
        float* T = reinterpret_cast<float*>(S);
        const ItemRec r = item_rec_of(rec[st]);
        const int n = r.n;
        const int* fb = reinterpret_cast<const int*>(S + SL::O_FR);
        for (int j = t; j < r.nf; j += blockDim.x) Fs[j] = foreign_cf(fb, s.fmax, j, m.C);
        __syncthreads();
        ring_c<N>(s, G, reinterpret_cast<const int*>(S + SL::O_PL), R, 2, r, Fs, T, false);
        walls_c<N>(s, G, n, 2, r.w3, r.w4, T);
        // the next item's copies, now that its record is in
        if (t < REC_WORDS) cp_async_wait_all();
        __syncthreads();
        if (t == 0 && kn < total) issue(st ^ 1, kn, rec[st ^ 1][0]);
        // decode this cell's post-streaming populations from the stage
        float h[9], g[9];
        {
            const unsigned short* DH = reinterpret_cast<const unsigned short*>(S + SL::O_DH);
            const unsigned short* DG = reinterpret_cast<const unsigned short*>(S + SL::O_DG);
            const float rh = reinterpret_cast<const float*>(S + SL::O_RH)[c];
            const float rg = reinterpret_cast<const float*>(S + SL::O_RG)[c];
            h[0] = rh;
            g[0] = rg;
#pragma unroll
            for (int q = 2; q <= 9; ++q) {
                h[q - 1] = dec<FMT>(DH[(q - 1) * N * N + c]) * m.ish + rq(q) * rh;
                g[q - 1] = dec<FMT>(DG[(q - 1) * N * N + c]) * m.isg + rq(q) * rg;
            }
        }
        collide_store<N, FMT, READ_PU, BGK>(s, G, n, x, y, T, h, g, wr);
        __syncthreads();  // the stage is read before it is refilled
        k = kn;
        st ^= 1;
    }
}

// ---- K2: Fill_Ghost_Cells_hg + Bounce_Back + streaming + macro h -----------
// As: both fields' 9 planes of the block (ring included), decoded, in the
// pool's plane layout. Without level order each CTA takes items b, b + grid,
// ... and copies the next item's words into the other of two shared stages
// while it works on the current one: the block's rest planes, plan words and
// foreign records by bulk copy (mbarrier), its 16-bit deviation planes by
// 8-byte cp.async (a block's 9 planes start on 8-byte boundaries only).
template <int N>
struct K2Stage {
    static constexpr int AP = (N + 2) * (N + 2), R = 2 * (N + N) + 4, FMAX = 2 * N + 28;
    static constexpr int DEV = 9 * AP * 2, REST = AP * 4, PLAN = R * PLAN_INTS * 4,
                         FRN = FMAX * FRN_INTS * 4;
    static constexpr int O_DG = DEV, O_RH = 2 * DEV, O_RG = O_RH + REST, O_PL = O_RG + REST,
                         O_FR = O_PL + PLAN, BYTES = O_FR + FRN;
    static_assert(O_RH % 16 == 0 && BYTES % 16 == 0 && DEV % 8 == 0, "stage alignment");
};

__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// the ring, the walls and the streaming of item k (block n) once As holds the
// block's planes: foreign cells (records fb), ring entries (plan words pl),
// Bounce_Back_3/4, the ring to memory where asked, then
// Perfect_Shift_AMR / Streaming_LaxWendroff_AMR (:41-90) into B and
// Macroscopic_Values_h_AMR (:193-201)
// (FAST: without level order, a compile-time flag so that each path gets its
// own code)
template <int N, int FMT, bool FAST>
__device__ void hg_item(const DevState& s, const Geo<N>& G, int k, const ItemRec& r, const int* fb,
                        const int* pl, float* As, float* Fs, bool wr) {
    constexpr bool fast = FAST;
    constexpr int AP = (N + 2) * (N + 2), FP = 9 * AP;
    const int t = threadIdx.x, n = r.n, RG = ring1_len(N, N), fmax = s.fmax;
    const MpState& m = s.mp;
    // foreign cells: one thread per (slot, field and population)
    for (int idx = t; idx < 18 * r.nf; idx += blockDim.x) {
        const int j = idx % r.nf, fq = idx / r.nf, f = fq / 9, q = fq % 9 + 1;
        const int meta = fb[j];
        float v;
        if (plan_kind(meta) == 1) {
            v = dec_a<N, FMT>(m, G, f, (unsigned)fb[fmax + j], q);
        } else {
            float gg[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) gg[i] = dec_a<N, FMT>(m, G, f, (unsigned)fb[(1 + i) * fmax + j], q);
            v = combine_f(meta, gg);
        }
        Fs[fq * fmax + j] = v;
    }
    __syncthreads();
    if (!fast) wait_for_coarser(s, Q_FILLHG, k);
    // the ring: copies per (cell, field), interpolated cells per (cell, population),
    // populations fastest, so that a cell's 9 threads share each source's rest load
    const int nC = 2 * r.na, nI = r.n2 + r.n3;
    for (int u = t; u < nC + 9 * nI; u += blockDim.x) {
        if (u < nC) {
            const int e = u % r.na, f = u / r.na;
            const int meta = pl[e];
            if (plan_kind(meta) < 0) {
                set_error(s, 4 /*AMRLBM_ERR_LEVEL_JUMP*/, n);
                continue;
            }
            int xx, yy;
            ring1_xy(meta >> 8, N, N, xx, yy);
            float v[9];
            dec_a9<N, FMT>(m, G, f, (unsigned)pl[RG + e], v);
#pragma unroll
            for (int q = 0; q < 9; ++q) As[f * FP + q * AP + yy * (N + 2) + xx] = v[q];
        } else {
            const int v2 = u - nC, e = r.na + v2 / 9, q = v2 % 9 + 1;
            const int meta = pl[e];
            const int kind = plan_kind(meta);
            int xx, yy;
            ring1_xy(meta >> 8, N, N, xx, yy);
            unsigned wd[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) wd[i] = (unsigned)pl[(1 + i) * RG + e];
#pragma unroll
            for (int f = 0; f < 2; ++f) {
                float gg[9];
#pragma unroll
                for (int i = 0; i < 9; ++i)
                    gg[i] = (kind == 3 && (wd[i] & kIndirect))
                                ? Fs[(f * 9 + q - 1) * fmax + (wd[i] & ~kIndirect)]
                                : (kind == 3 && !fast ? dec_a<N, FMT, true>(m, G, f, wd[i], q)
                                             : dec_a<N, FMT>(m, G, f, wd[i], q));
                As[f * FP + (q - 1) * AP + yy * (N + 2) + xx] = combine_f(meta, gg);
            }
        }
    }
    __syncthreads();
    // Bounce_Back_3/4 (BC_Cell.f90:2-42) on the staged planes
    if (r.w3 || r.w4) {
        for (int idx = t; idx < (N + 2) * 36; idx += blockDim.x) {
            const int X = idx % (N + 2), qf = (idx / (N + 2)) % 18;
            const bool top = idx >= (N + 2) * 18;
            if (top ? !r.w4 : !r.w3) continue;
            const int Y = top ? N + 1 : 0, Yi = top ? N : 1, sgn = top ? -1 : 1;
            const int i = qf % 9 + 1, f = qf / 9;
            int J = 1, Xn = X;
            if (i > 1) {
                Xn = min(max(0, X + sgn * d_ex(i) * d_ey(i)), N + 1);
                J = (i - 2) + 4 * ((i / 2) % 2);
            }
            As[f * FP + (i - 1) * AP + Y * (N + 2) + X] = As[f * FP + (J - 1) * AP + Yi * (N + 2) + Xn];
        }
    }
    __syncthreads();
    // the ring in memory where a later reader takes it from there: on the last
    // step of a call (the state is observed) or under level order
    if (wr || !fast) {
        for (int u = t; u < 2 * RG; u += blockDim.x) {
            const int f = u / RG;
            int xx, yy;
            ring1_xy(u % RG, N, N, xx, yy);
            float v[9];
#pragma unroll
            for (int q = 0; q < 9; ++q) v[q] = As[f * FP + q * AP + yy * (N + 2) + xx];
            enc_a9<N, FMT>(m, G, f, n, xx, yy, v);
        }
        if (!fast) {
            __syncthreads();
            publish_ring(s, Q_FILLHG, n);
        }
    }
    {
        const int x = t % N + 1, y = t / N + 1;
        const float cfl = 1.f / (float)__ldg(s.dx + n);
        const bool shift = cfl > 0.9f;
        const float cA = cfl * 0.5f * (1.f + cfl), cC = cfl * 0.5f * (1.f - cfl);
        double csum = 0.0;  // C = sum of h, in FP64, rounded to FP32 at random
#pragma unroll
        for (int f = 0; f < 2; ++f) {
            const float* Af = As + f * FP;
            float v[9];
#pragma unroll
            for (int i = 1; i <= 9; ++i) {
                auto at = [&](int q, int xx, int yy) { return Af[(q - 1) * AP + yy * (N + 2) + xx]; };
                if (i == 1)
                    v[0] = at(1, x, y);
                else if (shift)
                    v[i - 1] = at(i, x - d_ex(i), y - d_ey(i));
                else {  // cA f(x-e) + cB f(x) - cC f(x+e), cB = 1 - cA + cC, in
                        // increment form: exact on a uniform field in FP32
                    const float b = at(i, x, y);
                    v[i - 1] = b + (cA * (at(i, x - d_ex(i), y - d_ey(i)) - b) -
                                    cC * (at(i, x + d_ex(i), y + d_ey(i)) - b));
                }
                if (f == 0) csum += (double)v[i - 1];
            }
            enc_b9<N, FMT>(m, G, f, n, x, y, v);
        }
        m.C[G.c(n, x, y)] = f32_sr(csum, (unsigned)G.c(n, x, y) + 0x2545f491u);
    }
}

template <int N, int FMT>
__global__ void __launch_bounds__(N * N, (N == 16 ? 3 : 8))
    k_mp_fill_hg_stream(const __grid_constant__ DevState s, int wr) {
    using SL = K2Stage<N>;
    constexpr int AP = SL::AP, FP = 9 * AP;
    extern __shared__ __align__(128) unsigned char sm[];
    const Geo<N> G(s);
    __shared__ __align__(16) int rec[2][REC_WORDS + 1];
    __shared__ int sk, s_nn;
    const int t = threadIdx.x, total = s.lvl_off[AMR_MAXLV];
    const MpState& m = s.mp;
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(sm);  // [2]
    float* As = reinterpret_cast<float*>(sm + 128);                       // [2][9][AP]
    float* Fs = As + 2 * FP;                                              // [18][FMAX]
    unsigned char* stages = reinterpret_cast<unsigned char*>(Fs + 18 * SL::FMAX);
    const bool fast = s.fillinfo[Q_FILLHG] == 0;
    const int RG = SL::R;
    // the block's planes, ring included, from memory (level order) ...
    auto decode_mem = [&](int n) {
        for (int u = t; u < 2 * AP; u += blockDim.x) {
            const int f = u / AP, c = u % AP;
            float v[9];
            dec_a9<N, FMT>(m, G, f, (unsigned)G.a(n, 1, c % (N + 2), c / (N + 2)), v);
#pragma unroll
            for (int q = 0; q < 9; ++q) As[f * FP + q * AP + c] = v[q];
        }
    };
    if (!fast) {
        for (int k = claim(s, false, Q_FILLHG, -1, &sk); k < total; k = claim(s, false, Q_FILLHG, k, &sk)) {
            item_rec_stage(s, k, Q_FILLHG, rec[0]);
            __syncthreads();
            const ItemRec r = item_rec_of(rec[0]);
            decode_mem(r.n);
            hg_item<N, FMT, false>(s, G, k, r, s.frn_hg + (size_t)k * s.fmax * FRN_INTS,
                                   s.plan_hg + (size_t)k * RG * PLAN_INTS, As, Fs, wr != 0);
        }
        queue_done(s, Q_FILLHG);
        return;
    }
    int k = blockIdx.x;
    if (k >= total) return;
    // all threads: copies of item kk (block nn) into stage st
    auto issue = [&](int st, int kk, int nn) {
        unsigned char* S = stages + st * SL::BYTES;
        if (t == 0) {
            fence_proxy_async_all();
            fence_proxy_async();
            mbar_expect_tx(&bar[st], 2 * SL::REST + SL::PLAN + SL::FRN);
            bulk_g2s(S + SL::O_RH, m.A1h + (size_t)nn * AP, SL::REST, &bar[st]);
            bulk_g2s(S + SL::O_RG, m.A1g + (size_t)nn * AP, SL::REST, &bar[st]);
            bulk_g2s(S + SL::O_PL, s.plan_hg + (size_t)kk * RG * PLAN_INTS, SL::PLAN, &bar[st]);
            bulk_g2s(S + SL::O_FR, s.frn_hg + (size_t)kk * s.fmax * FRN_INTS, SL::FRN, &bar[st]);
        }
        const unsigned char* dh = reinterpret_cast<const unsigned char*>(m.Adh + (size_t)nn * 9 * AP);
        const unsigned char* dg = reinterpret_cast<const unsigned char*>(m.Adg + (size_t)nn * 9 * AP);
        for (int i = t; i < 2 * (SL::DEV / 8); i += blockDim.x) {
            const int f = i / (SL::DEV / 8), j = i % (SL::DEV / 8);
            cp_async8(S + f * SL::DEV + 8 * j, (f ? dg : dh) + 8 * j);
        }
        if (t < REC_WORDS) cp_async4(&rec[st][t], item_rec_word(s, kk, Q_FILLHG, t));
        cp_async_commit();
    };
    if (t == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        s_nn = __ldg(s.lvl_leaf + k);
    }
    __syncthreads();
    issue(0, k, s_nn);
    int n_after = 0;  // thread 0: block of the item after next
    if (t == 0 && k + (int)gridDim.x < total) n_after = __ldg(s.lvl_leaf + k + gridDim.x);
    __syncthreads();
    if (t == 0) s_nn = n_after;
    __syncthreads();
    unsigned phase = 0;
    int st = 0;
    while (k < total) {
        const int kn = k + gridDim.x;
        if (kn < total) issue(st ^ 1, kn, s_nn);
        else cp_async_commit();  // an empty group keeps the wait count uniform
        if (t == 0 && kn + (int)gridDim.x < total) n_after = __ldg(s.lvl_leaf + kn + gridDim.x);
        cp_async_wait_prev();
        if (__syncthreads_or(mbar_wait(&bar[st], (phase >> st) & 1u) ? 0 : 1)) {
            if (t == 0) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 111);
            mbar_wait(&bar[st], (phase >> st) & 1u);
            cp_async_wait_all();
            break;
        }
        phase ^= 1u << st;
        const unsigned char* S = stages + st * SL::BYTES;
        const ItemRec r = item_rec_of(rec[st]);
        // decode the staged planes into As
        {
            const unsigned short* DH = reinterpret_cast<const unsigned short*>(S);
            const unsigned short* DG = reinterpret_cast<const unsigned short*>(S + SL::O_DG);
            const float* RH = reinterpret_cast<const float*>(S + SL::O_RH);
            const float* RGs = reinterpret_cast<const float*>(S + SL::O_RG);
            for (int u = t; u < 2 * AP; u += blockDim.x) {
                const int f = u / AP, c = u % AP;
                const unsigned short* D = f ? DG : DH;
                const float rest = (f ? RGs : RH)[c], is = f ? m.isg : m.ish;
                As[f * FP + c] = rest;
#pragma unroll
                for (int q = 2; q <= 9; ++q) As[f * FP + (q - 1) * AP + c] = dec<FMT>(D[(q - 1) * AP + c]) * is + rq(q) * rest;
            }
        }
        hg_item<N, FMT, true>(s, G, k, r, reinterpret_cast<const int*>(S + SL::O_FR),
                              reinterpret_cast<const int*>(S + SL::O_PL), As, Fs, wr != 0);
        __syncthreads();  // As, Fs and the stage are read before they are refilled
        if (t == 0) s_nn = n_after;
        __syncthreads();
        k = kn;
        st ^= 1;
    }
    cp_async_wait_all();
}

// ---- K3: Fill_Ghost_Cells_C + Symmetric_C + Macroscopic_Values_g_AMR +
// Err_Interface (Refine_Derefine.f90:327-351, into the FP64 err of the block)
template <int N, int FMT>
__global__ void __launch_bounds__(N * N) k_mp_tail(const __grid_constant__ DevState s) {
    const Geo<N> G(s);
    __shared__ float T[cplane_of(N)];
    extern __shared__ float Fs[];
    __shared__ int rec[REC_WORDS + 1];
    __shared__ double red[32];
    const int t = threadIdx.x, total = s.lvl_off[AMR_MAXLV];
    const int R = ring1_len(N, N);
    const MpState& m = s.mp;
    const int x = t % N + 1, y = t / N + 1;
    const bool fast = s.fillinfo[Q_FILLC1] == 0;
    __shared__ int sk;
    for (int k = claim(s, fast, Q_FILLC1, -1, &sk); k < total; k = claim(s, fast, Q_FILLC1, k, &sk)) {
        item_rec_stage(s, k, Q_FILLC1, rec);
        __syncthreads();
        const ItemRec r = item_rec_of(rec);
        const int n = r.n;
        load_tile<N>(s, G, n, T);
        const int* fb = s.frn_c + (size_t)k * s.fmax * FRN_INTS;
        for (int j = t; j < r.nf; j += blockDim.x) Fs[j] = foreign_cf(fb, s.fmax, j, m.C);
        __syncthreads();
        if (!fast) wait_for_coarser(s, Q_FILLC1, k);
        // through L2 also without level order: measured faster here (the ring
        // of one width has little reuse of its sources)
        ring_c<N>(s, G, s.plan_c1 + (size_t)k * R * PLAN_INTS, R, 1, r, Fs, T, true);
        walls_c<N>(s, G, n, 1, r.w3, r.w4, T);
        if (!fast) publish_ring(s, Q_FILLC1, n);
        const float inv_dx = 1.f / (float)__ldg(s.dx + n);
        float g[9], P, Ux, Uy;
        dec_b9<N, FMT>(m, G, 1, n, x, y, g);
        const CellC<N> Cs{T, G, x, y};
        macro_g(Cs, s.n_inst ? m.phys[s.inst[n]] : m.ph, inv_dx, g, P, Ux, Uy);
        m.P[G.p(n, x, y)] = P;
        m.Ux[G.p(n, x, y)] = Ux;
        m.Uy[G.p(n, x, y)] = Uy;
        const double a = (double)Cs(1, 0) - (double)Cs(-1, 0), b = (double)Cs(0, 1) - (double)Cs(0, -1);
        double mx = a * a + b * b;
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if ((t & 31) == 0) red[t >> 5] = mx;
        __syncthreads();
        if (t == 0) {
            double mm = 0.0;
            for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) mm = fmax(mm, red[w]);
            s.err[n] = sqrt(mm) / (2.0 * s.dx[n]);
        }
    }
    if (!fast) queue_done(s, Q_FILLC1);
}

// ---- conversions between the FP64 pool and the mixed-precision state -------
// Blocks of list `mode`: 0 every leaf, 1 derefined parents, 2 their children,
// 3 refined parents, 4 their children. to_mp: FP64 -> 16-bit/FP32, else back.
// Converted per block: the post-streaming interior populations, the
// post-collision ring-1 populations, C with both rings, P, Ux, Uy.
__device__ __forceinline__ int conv_count(const DevState& s, int mode) {
    const Counters& c = *s.cnt;
    return mode == 0 ? c.nleaf : (mode <= 2 ? c.n_der : c.n_ref) * (mode == 2 || mode == 4 ? 4 : 1);
}
__device__ __forceinline__ int conv_block(const DevState& s, int mode, int i) {
    switch (mode) {
        case 0: return s.leaf[i];
        case 1: return s.der_list[i];
        case 2: return s.child[4 * s.der_list[i / 4]] + i % 4;
        case 3: return s.ref_list[i];
        default: return s.ref_c1[i / 4] + i % 4;
    }
}

template <int N, int FMT>
__global__ void __launch_bounds__(256) k_mp_convert(const __grid_constant__ DevState s, int mode,
                                                    int to_mp) {
    const Geo<N> G(s);
    const MpState& m = s.mp;
    const int cnt = conv_count(s, mode);
    const int RG = ring1_len(N, N);
    for (int i = blockIdx.x; i < cnt; i += gridDim.x) {
        const int n = conv_block(s, mode, i);
        for (int u = threadIdx.x; u < 2 * (N * N + RG); u += blockDim.x) {
            const int f = u / (N * N + RG), c = u % (N * N + RG);
            const bool interior = c < N * N;
            int x, y;
            if (interior) {
                x = c % N + 1;
                y = c / N + 1;
            } else {
                ring1_xy(c - N * N, N, N, x, y);
            }
            double v[9];
            const double* B = f ? s.Bg : s.Bh;
            double* Bw = f ? s.Bg : s.Bh;
            double* A = f ? s.Ag : s.Ah;
            const double sc = f ? m.sg : m.sh, is = f ? m.isg : m.ish;
            if (to_mp) {
#pragma unroll
                for (int q = 1; q <= 9; ++q) v[q - 1] = interior ? B[G.bb(n, q, x, y)] : A[G.a(n, q, x, y)];
                // the rest population and the deviations from the FP64 values,
                // each rounded once, at random (see enc_sr)
                const unsigned salt = (unsigned)(n * (N * N + RG) + c) * 2u + f + 0x1b873593u;
                const float o0 = f32_sr(v[0], salt);
                // h: the rounding errors carried from one deviation to the next
                // (mass_encode), in FP64 here
                double e = 0.0;
                unsigned short w[8];
#pragma unroll
                for (int q = 2; q <= 9; ++q) {
                    const double xv = (v[q - 1] - (double)rq(q) * (double)o0) * sc - e;
                    w[q - 2] = enc_sr<FMT>((float)xv, salt + 7u * q);
                    if (f == 0) e = (double)dec<FMT>(w[q - 2]) - xv;
                }
                if (interior) {
                    (f ? m.B1g : m.B1h)[(size_t)n * G.bplane + (size_t)(y - 1) * N + (x - 1)] = o0;
#pragma unroll
                    for (int q = 2; q <= 9; ++q) (f ? m.Bdg : m.Bdh)[G.bb(n, q, x, y)] = w[q - 2];
                } else {
                    const size_t off = G.a(n, 1, x, y);
                    (f ? m.A1g : m.A1h)[off - (size_t)8 * G.aplane * n] = o0;
#pragma unroll
                    for (int q = 2; q <= 9; ++q) (f ? m.Adg : m.Adh)[off + (size_t)(q - 1) * G.aplane] = w[q - 2];
                }
            } else {
                float w[9];
                if (interior) {
                    const size_t cc = (size_t)(y - 1) * N + (x - 1);
                    w[0] = (f ? m.B1g : m.B1h)[(size_t)n * G.bplane + cc];
#pragma unroll
                    for (int q = 2; q <= 9; ++q) w[q - 1] = dec<FMT>((f ? m.Bdg : m.Bdh)[G.bb(n, q, x, y)]);
                } else {
                    const size_t off = G.a(n, 1, x, y);
                    w[0] = (f ? m.A1g : m.A1h)[off - (size_t)8 * G.aplane * n];
#pragma unroll
                    for (int q = 2; q <= 9; ++q) w[q - 1] = dec<FMT>((f ? m.Adg : m.Adh)[off + (size_t)(q - 1) * G.aplane]);
                }
                v[0] = (double)w[0];
#pragma unroll
                for (int q = 2; q <= 9; ++q) v[q - 1] = (double)w[q - 1] * is + (double)rq(q) * v[0];
#pragma unroll
                for (int q = 1; q <= 9; ++q) {
                    if (interior)
                        Bw[G.bb(n, q, x, y)] = v[q - 1];
                    else
                        A[G.a(n, q, x, y)] = v[q - 1];
                }
            }
        }
        for (int u = threadIdx.x; u < G.cplane; u += blockDim.x) {
            const size_t o = (size_t)n * G.cplane + u;
            if (to_mp)
                m.C[o] = f32_sr(s.C[o], (unsigned)o + 0x2545f491u);
            else
                s.C[o] = (double)m.C[o];
        }
        for (int u = threadIdx.x; u < 3 * N * N; u += blockDim.x) {
            const int f = u / (N * N);
            const size_t o = (size_t)n * G.pplane + u % (N * N);
            double* D = f == 0 ? s.P : (f == 1 ? s.Ux : s.Uy);
            float* F = f == 0 ? m.P : (f == 1 ? m.Ux : m.Uy);
            if (to_mp)
                F[o] = (float)D[o];
            else
                D[o] = (double)F[o];
        }
    }
}

// persistent launch: as many CTAs as fit on the GPU at once (the items are
// distributed over them), the dynamic shared memory opted in where needed
// CTAs per SM of a kernel (queried once per kernel and shared-memory size,
// before any stream capture: amrlbm_set_precision prepares every variant)
template <class K>
int per_sm(K kern, int threads, size_t dyn) {
    static std::map<std::pair<const void*, size_t>, int> cache;
    const auto key = std::make_pair(reinterpret_cast<const void*>(kern), dyn);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    if (dyn > 48 * 1024) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn);
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, threads, dyn) != cudaSuccess || b < 1) b = 1;
    cache.emplace(key, b);
    return b;
}

// persistent launch: as many CTAs as fit on the GPU at once, the items
// distributed over them (prepare: only the occupancy query)
template <class K>
void grid_leaves_launch(K kern, const LaunchCfg& lc, int threads, size_t dyn, cudaStream_t st,
                        const DevState& s, int a, bool prepare = false) {
    int b = per_sm(kern, threads, dyn);
    if (prepare) return;
    if (lc.mp_ctas > 0 && lc.mp_ctas < b) b = lc.mp_ctas;
    kern<<<lc.num_sms * b, threads, dyn, st>>>(s, a);
    count_launches(1);
}

template <int N, int FMT>
void mp_collide(const DevState& s, const LaunchCfg& lc, cudaStream_t st, bool read_pu, int wr,
                bool prep = false) {
    const size_t dyn = 128 + 2 * (size_t)K1Stage<N>::BYTES + sizeof(float) * (size_t)s.fmax;
    if (s.g_model == 1 || prep) {
        if (read_pu || prep)
            grid_leaves_launch(k_mp_collide<N, FMT, true, true>, lc, N * N, dyn, st, s, wr, prep);
        if (!read_pu || prep)
            grid_leaves_launch(k_mp_collide<N, FMT, false, true>, lc, N * N, dyn, st, s, wr, prep);
    }
    if (s.g_model != 1 || prep) {
        if (read_pu || prep)
            grid_leaves_launch(k_mp_collide<N, FMT, true, false>, lc, N * N, dyn, st, s, wr, prep);
        if (!read_pu || prep)
            grid_leaves_launch(k_mp_collide<N, FMT, false, false>, lc, N * N, dyn, st, s, wr, prep);
    }
}
template <int N, int FMT>
void mp_fill_hg(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int wr, bool prep = false) {
    using SL = K2Stage<N>;
    const size_t dyn = 128 + sizeof(float) * (2 * 9 * (size_t)SL::AP + 18 * (size_t)SL::FMAX) +
                       2 * (size_t)SL::BYTES;
    grid_leaves_launch(k_mp_fill_hg_stream<N, FMT>, lc, N * N, dyn, st, s, wr, prep);
}
template <int N, int FMT>
void mp_tail(const DevState& s, const LaunchCfg& lc, cudaStream_t st) {
    k_mp_tail<N, FMT><<<lc.grid_leaves, N * N, sizeof(float) * (size_t)s.fmax, st>>>(s);
    count_launches(1);
}
template <int N, int FMT>
void mp_convert(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int mode, int to_mp) {
    k_mp_convert<N, FMT><<<lc.grid_leaves, 256, 0, st>>>(s, mode, to_mp);
    count_launches(1);
}

// dispatch over block size and storage format
template <template <int, int> class F, class... A>
void mp_dispatch(const DevState& s, A... a) {
    if (s.nx == 16 && s.mp.fmt == 1) F<16, 1>::run(s, a...);
    else if (s.nx == 16) F<16, 2>::run(s, a...);
    else if (s.mp.fmt == 1) F<8, 1>::run(s, a...);
    else F<8, 2>::run(s, a...);
}
template <int N, int FMT>
struct Collide {
    static void run(const DevState& s, const LaunchCfg& lc, cudaStream_t st, bool rp, int wr) {
        mp_collide<N, FMT>(s, lc, st, rp, wr);
    }
};
template <int N, int FMT>
struct FillHg {
    static void run(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int wr) {
        mp_fill_hg<N, FMT>(s, lc, st, wr);
    }
};
template <int N, int FMT>
struct Tail {
    static void run(const DevState& s, const LaunchCfg& lc, cudaStream_t st) { mp_tail<N, FMT>(s, lc, st); }
};
template <int N, int FMT>
struct Prepare {
    static void run(const DevState& s, const LaunchCfg& lc) {
        mp_collide<N, FMT>(s, lc, nullptr, false, 0, true);
        mp_fill_hg<N, FMT>(s, lc, nullptr, 0, true);
    }
};
template <int N, int FMT>
struct Convert {
    static void run(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int mode, int to_mp) {
        mp_convert<N, FMT>(s, lc, st, mode, to_mp);
    }
};

}  // namespace

void launch_mp_collide(const DevState& s, const LaunchCfg& lc, cudaStream_t st, bool read_pu,
                       int write_pu) {
    mp_dispatch<Collide>(s, lc, st, read_pu, write_pu);
}
void launch_mp_fill_hg_stream(const DevState& s, const LaunchCfg& lc, cudaStream_t st,
                              int write_ring) {
    mp_dispatch<FillHg>(s, lc, st, write_ring);
}
void launch_mp_tail(const DevState& s, const LaunchCfg& lc, cudaStream_t st) {
    mp_dispatch<Tail>(s, lc, st);
}
void launch_mp_prepare(const DevState& s, const LaunchCfg& lc) { mp_dispatch<Prepare>(s, lc); }
void launch_mp_convert(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int mode,
                       int to_mp) {
    mp_dispatch<Convert>(s, lc, st, mode, to_mp);
}
