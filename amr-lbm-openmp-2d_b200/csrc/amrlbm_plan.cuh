// amrlbm_plan.cuh - the ghost-cell fill plans and per-leaf records shared by
// the FP64 kernels (amrlbm_step.cu) and the mixed-precision kernels
// (amrlbm_mixed.cu): neighbour records, plan entries (kind, stencil side,
// source offsets), ring indexing, the biquadratic combination of a plan's
// sources, and the per-item record words. Device helpers with internal
// linkage: each translation unit gets its own copy.
#pragma once
#include <cstddef>

#include "amrlbm_fast.cuh"

namespace {

__device__ __forceinline__ int ghost_dir(int x, int y, int nx, int ny) {
    const bool xl = x < 1, xr = x > nx, yb = y < 1, yt = y > ny;
    if (xl) return yb ? 5 : (yt ? 6 : 1);
    if (xr) return yb ? 7 : (yt ? 8 : 2);
    return yb ? 3 : 4;
}

// per-direction neighbour data of the block being filled, loaded once into
// shared memory: resolved id, its level, leaf flag and first child (index 0:
// the block itself); per fill q: wait[q], the directions whose rings a
// level-ordered fill waits for, and nf[q], the number of foreign cells
struct NbInfo {
    int id[9], lev[9], leaf[9], c1[9];
    int bi, bj;
    int wait[NQUEUES];
    int nf[NQUEUES];
    // plan entries stored first: na of kinds 1 and -1, then n2 of kind 2, then
    // n3 of kind 3 (then those without a plan)
    int na[NQUEUES], n2[NQUEUES], n3[NQUEUES];
};
constexpr int NBI_INTS = (int)(sizeof(NbInfo) / sizeof(int));
static_assert(NBI_INTS <= NBI_STRIDE, "NbInfo record");

// ---------------------------------------------------------------------------
// Fill plan of ghost cell (x,y) of block n (level L) from its direction-d
// neighbour: what kind of value it takes and the offsets OFF(blk, x, y) of
// its sources. The cases, gathers and stencils follow Fill_Left_* ..
// Fill_Right_Top_* (Fill_Ghost_Cells_C.f90:44-416, Fill_Ghost_Cells_C2.f90:
// 44-416, Fill_Ghost_Cells_hg.f90:53-477) case by case; the weights are those
// of Biquadratic_from_Fine/_Coarse (Interpolations.f90:2-138).
// kind: 0 none / not filled, 1 copy of src[0], 2 Biquadratic_from_Fine,
// 3 Biquadratic_from_Coarse, -1 level jump. src[3*r+c] = G(i0+r, j0+c), the
// reference's gathered array around the stencil origin; w = (ax, cx, ay, cy).
struct GPlan {
    int kind, ax, cx, ay, cy;
    long long src[9];
};
template <class OF>
__device__ __forceinline__ void ghost_plan(const NbInfo& nbi, int nx, int ny, int L, int d, int x,
                                           int y, OF OFF, GPlan& P) {
    const int N = nbi.id[d];
    P.kind = 0;
    if (N <= 0) return;
    const int Ln = nbi.lev[d];
    const bool left = (d == 1 || d == 5 || d == 6), right = (d == 2 || d == 7 || d == 8);
    const bool bottom = (d == 3 || d == 5 || d == 7), top = (d == 4 || d == 6 || d == 8);
    const int a = left ? 1 - x : (right ? x - nx : 0);
    const int b = bottom ? 1 - y : (top ? y - ny : 0);
    int X, Y;  // output index of the reference's Cout(X,Y)
    if (d == 1 || d == 2) {
        X = a;
        Y = y;
    } else if (d == 3 || d == 4) {
        X = x;
        Y = b;
    } else {
        X = a;
        Y = b;
    }
    if (L == Ln) {
        if (nbi.leaf[d]) {
            P.kind = 1;
            P.src[0] = OFF(N, left ? nx + 1 - a : (right ? a : x), bottom ? ny + 1 - b : (top ? b : y));
            return;
        }
        P.kind = 2;
        const int Jy = (Y + 1) % 2, iy = 2 * Y - 1 - Jy, Jx = (X + 1) % 2, ix = 2 * X - 1 - Jx;
        P.ay = 3 - 4 * Jy;
        P.cy = 2 - P.ay;
        P.ax = 3 - 4 * Jx;
        P.cx = 2 - P.ax;
        const int c1 = nbi.c1[d];
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                const int i = ix + r, j = iy + c;  // G(i, j)
                long long o;
                if (d == 1 || d == 2) {
                    const int ch = (j <= ny) ? (d == 1 ? c1 + 1 : c1) : (d == 1 ? c1 + 3 : c1 + 2);
                    o = OFF(ch, (d == 1) ? nx - i + 1 : i, (j <= ny) ? j : j - ny);
                } else if (d == 3 || d == 4) {
                    const int ch = (i <= nx) ? (d == 3 ? c1 + 2 : c1) : (d == 3 ? c1 + 3 : c1 + 1);
                    o = OFF(ch, (i <= nx) ? i : i - nx, (d == 3) ? ny - j + 1 : j);
                } else {
                    const int ch = c1 + (d == 5 ? 3 : d == 6 ? 1 : d == 7 ? 2 : 0);
                    o = OFF(ch, left ? nx - i + 1 : i, bottom ? ny - j + 1 : j);
                }
                P.src[3 * r + c] = o;
            }
        return;
    }
    if (L == Ln + 1) {
        P.kind = 3;
        const int Iy = (Y + 1) / 2, Ix = (X + 1) / 2;
        P.ay = 5 - 8 * ((Y + 1) % 2);
        P.cy = 2 - P.ay;
        P.ax = 5 - 8 * ((X + 1) % 2);
        P.cx = 2 - P.ax;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                const int ii = Ix + r, jj = Iy + c;  // G(ii, jj)
                long long o;
                if (d == 1 || d == 2) {
                    const int Yo = (ny / 2) * (nbi.bj % 2);
                    o = OFF(N, (d == 1) ? nx + 2 - ii : ii - 1, jj - 1 + Yo);
                } else if (d == 3 || d == 4) {
                    const int Xo = (nx / 2) * (nbi.bi % 2);
                    o = OFF(N, ii - 1 + Xo, (d == 3) ? ny + 2 - jj : jj - 1);
                } else {
                    const int mi = nbi.bi % 2, mj = nbi.bj % 2;
                    const int I = left ? nx - (nx / 2) * mi - 1 : nx / 2 - (nx / 2) * mi;
                    const int J = bottom ? ny - (ny / 2) * mj - 1 : ny / 2 - (ny / 2) * mj;
                    o = OFF(N, left ? I + 3 - ii : I + ii - 1, bottom ? J + 3 - jj : J + jj - 1);
                }
                P.src[3 * r + c] = o;
            }
        return;
    }
    P.kind = -1;
}

// Packed plan of one ghost cell, stored plane by plane: plane 0 holds the
// meta word (bits 0-2 kind+1, bit 3 Jx, bit 4 Jy, bits 8- the cell's ring
// index; the stencil weights are
// ax = 3-4Jx (fine) or 5-8Jx (coarse), cx = 2-ax, the same along y), planes
// 1..9 the source offsets (in doubles, into the C pool or the first plane of
// the A pool). Plane i of entry t of a ring of R entries is base[i*R + t].
__device__ __forceinline__ void plan_store(int* base, int R, int t, const GPlan& P, int ring = 0) {
    int meta = ((P.kind + 1) & 7) | (ring << 8);
    if (P.kind == 2) meta |= ((P.ax == -1) ? 8 : 0) | ((P.ay == -1) ? 16 : 0);
    if (P.kind == 3) meta |= ((P.ax == -3) ? 8 : 0) | ((P.ay == -3) ? 16 : 0);
    base[t] = meta;
    const int ns = (P.kind == 1) ? 1 : ((P.kind >= 2) ? 9 : 0);
    for (int i = 0; i < 9; ++i) base[(1 + i) * R + t] = (i < ns) ? (int)(unsigned)P.src[i] : 0;
}
__device__ __forceinline__ int plan_kind(int meta) { return (meta & 7) - 1; }
// storage class of a plan entry: 0 copy or level jump, 1 fine-to-coarse,
// 2 coarse-to-fine, 3 no plan
__device__ __forceinline__ int plan_class(int kind) {
    return (kind == 1 || kind < 0) ? 0 : (kind == 2 ? 1 : (kind == 3 ? 2 : 3));
}

// Biquadratic_from_Fine / _Coarse (Interpolations.f90:2-138) at one output
// point from its 9 gathered sources g[3*r+c]: first along the reference's
// second index, then along the first, then /64 or /1024.
__device__ __forceinline__ double plan_combine(int meta, const double* g) {
    const int kind = plan_kind(meta);
    const int Jx = (meta >> 3) & 1, Jy = (meta >> 4) & 1;
    const double b = (kind == 2) ? 6.0 : 30.0;
    const int ax = (kind == 2) ? 3 - 4 * Jx : 5 - 8 * Jx, ay = (kind == 2) ? 3 - 4 * Jy : 5 - 8 * Jy;
    const double Ax = (double)ax, Cx = (double)(2 - ax), Ay = (double)ay, Cy = (double)(2 - ay);
    double t[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) t[r] = Ay * g[3 * r] + b * g[3 * r + 1] + Cy * g[3 * r + 2];
    const double o = Ax * t[0] + b * t[1] + Cx * t[2];
    return (kind == 2) ? o / 64.0 : o / 1024.0;
}

// ring 1 of a block: index r in [0, 2(nx+ny)+4) <-> (x,y)
__device__ __forceinline__ void ring1_xy(int r, int nx, int ny, int& x, int& y) {
    if (r < nx + 2) {
        x = r;
        y = 0;
    } else if (r < 2 * (nx + 2)) {
        x = r - (nx + 2);
        y = ny + 1;
    } else {
        const int t = r - 2 * (nx + 2);
        x = (t < ny) ? 0 : nx + 1;
        y = 1 + (t < ny ? t : t - ny);
    }
}
// rings 1-2 of C: index t in [0, 4(nx+ny)+16) <-> (x,y)
__device__ __forceinline__ void ring2_xy(int t, int nx, int ny, int& x, int& y) {
    const int W = nx + 4;
    if (t < 2 * W) {
        x = t % W - 1;
        y = t / W - 1;
    } else if (t < 4 * W) {
        const int u = t - 2 * W;
        x = u % W - 1;
        y = ny + 1 + u / W;
    } else {
        const int u = t - 4 * W, c = u / ny;
        x = (c < 2) ? c - 1 : nx - 1 + c;
        y = 1 + u % ny;
    }
}
__host__ __device__ __forceinline__ int ring2_len(int nx, int ny) { return 4 * (nx + ny) + 16; }
__host__ __device__ __forceinline__ int ring1_len(int nx, int ny) { return 2 * (nx + ny) + 4; }


// ---------------------------------------------------------------------------
// Source word of a packed plan: bit 31 clear: offset (doubles) of the source
// in the pool array; set: slot of a foreign cell of the item, a coarser
// neighbour's ghost cell that is a copy or a fine-to-coarse value of
// interiors, which the item evaluates itself before its coarse-to-fine
// cells. A foreign record (FRN_INTS ints, plane by plane over fmax slots)
// holds that ghost cell's plan (meta word, 9 sources) and its offset.
constexpr unsigned kIndirect = 0x80000000u;
constexpr int FRN_INTS = 11;

__device__ __forceinline__ int ring1_index(int x, int y, int nx, int ny) {
    if (y == 0) return x;
    if (y == ny + 1) return nx + 2 + x;
    return 2 * (nx + 2) + (x == 0 ? 0 : ny) + (y - 1);
}

// word offsets in a neighbour record
constexpr int REC_NF = (int)(offsetof(NbInfo, nf) / sizeof(int));
constexpr int REC_NA = (int)(offsetof(NbInfo, na) / sizeof(int));
constexpr int REC_N2 = (int)(offsetof(NbInfo, n2) / sizeof(int));
constexpr int REC_N3 = (int)(offsetof(NbInfo, n3) / sizeof(int));

// what an item of fill q needs from its record: block, foreign cells, plan
// entry classes, walls (id[3], id[4] < 0); staged in shared memory by
// threads 0..6 (REC_WORDS words), read from there by every thread
struct ItemRec {
    int n, nf, na, n2, n3;
    bool w3, w4;
};
constexpr int REC_WORDS = 7;
// word t of an item record: n, nf, na, n2, n3, id[3] (bottom), id[4] (top)
__device__ __forceinline__ const int* item_rec_word(const DevState& s, int c, int q, int t) {
    const int off = t == 0   ? 0
                    : t == 1 ? REC_NF + q
                    : t == 2 ? REC_NA + q
                    : t == 3 ? REC_N2 + q
                    : t == 4 ? REC_N3 + q
                             : t - 2;
    return s.nbinfo + (size_t)c * NBI_STRIDE + off;
}
__device__ __forceinline__ void item_rec_stage(const DevState& s, int c, int q, int* dst) {
    const int t = threadIdx.x;
    if (t < REC_WORDS) dst[t] = __ldg(item_rec_word(s, c, q, t));
}
// the same without waiting for the loads: threads 0..6 gather the words with
// cp.async and call cp_async_wait_all before the barrier that precedes the
// first read of dst (thread 0, which copies word 0, may read it after its
// own wait)
__device__ __forceinline__ void item_rec_stage_async(const DevState& s, int c, int q, int* dst) {
    const int t = threadIdx.x;
    if (t < REC_WORDS) cp_async4(dst + t, item_rec_word(s, c, q, t));
}
__device__ __forceinline__ ItemRec item_rec_of(const int* w) {
    ItemRec o;
    o.n = w[0];
    o.nf = w[1];
    o.na = w[2];
    o.n2 = w[3];
    o.n3 = w[4];
    o.w3 = w[5] < 0;
    o.w4 = w[6] < 0;
    return o;
}


// ---- level order: work queues and per-block ring flags ----------------------
__device__ __forceinline__ int ld_acquire_i(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_i(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ int* fill_flags(const DevState& s, int q) {
    return s.ring_done + (size_t)q * (s.max_blks + 1);
}

// End of a level-ordered launch of queue q, called by every CTA: the last CTA
// to finish clears the queue's counters and the flags of the leaves, for the
// next launch. (Launches without level order use neither.)
__device__ void queue_done(const DevState& s, int q) {
    __shared__ int last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&s.queue[4 * q + 2], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    int* f = fill_flags(s, q);
    const int total = s.lvl_off[AMR_MAXLV];
    for (int k = threadIdx.x; k < total; k += blockDim.x) f[s.lvl_leaf[k]] = 0;
    if (threadIdx.x == 0) {
        s.queue[4 * q] = 0;
        s.queue[4 * q + 1] = 0;
        s.queue[4 * q + 2] = 0;
    }
}

// bounded spin of one thread until *flag is set; false if it ran out
__device__ __forceinline__ bool spin_flag(const int* flag, int limit) {
    for (int it = 0; it < limit; ++it) {
        if (ld_acquire_i(flag) != 0) return true;
        __nanosleep(32);
    }
    return false;
}

// waits until every coarser neighbour of the item has its ring in memory;
// block-uniform, ends with a barrier
__device__ __forceinline__ void wait_coarse(const DevState& s, int q, const NbInfo& nbi) {
    const int t = threadIdx.x;
    if (t < 8 && ((nbi.wait[q] >> (t + 1)) & 1))
        if (!spin_flag(fill_flags(s, q) + nbi.id[t + 1], s.spin_limit)) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, q);
    __syncthreads();
}

// Raises block n's flag; call after the barrier that follows the ring's last
// writes. The release store is cumulative: it orders every write of the CTA
// that the barrier ordered before thread 0's store.
__device__ __forceinline__ void publish_ring(const DevState& s, int q, int n) {
    if (threadIdx.x == 0 && n != s.hold_flag) st_release_i(fill_flags(s, q) + n, 1);
}

}  // namespace
