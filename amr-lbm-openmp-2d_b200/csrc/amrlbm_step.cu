// amrlbm_step.cu - the per-step FP64 kernels (ghost fills fused with
// collision, streaming and macroscopic values). Compiled with -fmad=false:
// every operation the reference writes is rounded on its own and in its
// order; exact FMAs appear only inside the division of amrlbm_fast.cuh.
//
// Ghost fills without grid-wide level loops. The reference fills ghost cells
// level by level (Fill_Ghost_Cells_C.f90:8-38): a coarse-to-fine fill reads
// the coarse neighbour's ghost ring, written one level earlier. Here, after
// every topology change, each ghost cell of each leaf gets a fill plan (copy,
// fine-to-coarse or coarse-to-fine interpolation, with its source offsets).
// When every coarse-to-fine source is an interior cell or a coarser
// neighbour's ghost cell that is itself a copy or a fine-to-coarse value (the
// usual case), two flat launches fill all rings: copies and fine-to-coarse
// cells first, coarse-to-fine cells second; the consumer launch (collision,
// streaming or macroscopic values) applies the walls. Otherwise the consumer
// launch fills level by level first: CTAs claim leaves from a queue in which
// every leaf a finer neighbour reads precedes its readers, a leaf waits
// (bounded spin) for its coarser neighbours' flags, and no grid barrier is
// needed.
#include <cstdio>

#include "amrlbm_fast.cuh"
#include "amrlbm_launch.h"

void count_launches(int n);

namespace {

constexpr int kSpinLimit = 20000000;  // x ~64 ns: about a second

__device__ __forceinline__ int ld_acquire_i(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_i(int* p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// direction (1..8) of ghost cell (x,y)
__device__ __forceinline__ int ghost_dir(int x, int y, int nx, int ny) {
    const bool xl = x < 1, xr = x > nx, yb = y < 1, yt = y > ny;
    if (xl) return yb ? 5 : (yt ? 6 : 1);
    if (xr) return yb ? 7 : (yt ? 8 : 2);
    return yb ? 3 : 4;
}

// per-direction neighbour data of the block being filled, loaded once into
// shared memory: resolved id, its level, leaf flag and first child (index 0:
// the block itself); wait: the directions of coarser neighbours, whose rings
// a level-ordered fill waits for
struct NbInfo {
    int id[9], lev[9], leaf[9], c1[9];
    int bi, bj;
    int wait;
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
// meta word (bits 0-2 kind+1, bit 3 Jx, bit 4 Jy: the stencil weights are
// ax = 3-4Jx (fine) or 5-8Jx (coarse), cx = 2-ax, the same along y), planes
// 1..9 the source offsets (in doubles, into the C pool or the first plane of
// the A pool). Plane i of entry t of a ring of R entries is base[i*R + t].
__device__ __forceinline__ void plan_store(int* base, int R, int t, const GPlan& P) {
    int meta = (P.kind + 1) & 7;
    if (P.kind == 2) meta |= ((P.ax == -1) ? 8 : 0) | ((P.ay == -1) ? 16 : 0);
    if (P.kind == 3) meta |= ((P.ax == -3) ? 8 : 0) | ((P.ay == -3) ? 16 : 0);
    base[t] = meta;
    const int ns = (P.kind == 1) ? 1 : ((P.kind >= 2) ? 9 : 0);
    for (int i = 0; i < 9; ++i) base[(1 + i) * R + t] = (i < ns) ? (int)(unsigned)P.src[i] : 0;
}
__device__ __forceinline__ int plan_kind(int meta) { return (meta & 7) - 1; }

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
// Neighbour records and fill plans of every leaf, in work order (one CTA per
// leaf). The neighbour data is what Fill_Ghost_Cells_* reads through the
// block pointers (Fill_Ghost_Cells_C.f90:8-38): resolved neighbour ids, their
// levels, leaf flags and first children, plus the block's own id, level and
// ring_out flag.
//
// Coarse-to-fine cells read the coarser neighbour's ring, which the
// reference fills one level earlier. Where such a ring cell is itself a copy
// or a fine-to-coarse interpolation of interiors, the plan refers to that
// cell's own plan entry and the fill evaluates it in place, with the same
// operations the neighbour's fill uses, so the fill need not wait. Only where
// it is a coarse-to-fine or wall cell does the record's wait mask make the
// fill wait for the neighbour's flag.
__device__ void load_nbinfo(const DevState& s, int n, NbInfo& r) {
    for (int j = 0; j < 8; ++j) {
        const int b = s.nbr[8 * n + j];
        r.id[j + 1] = b;
        r.lev[j + 1] = (b > 0) ? s.level[b] : -1;
        r.leaf[j + 1] = (b > 0) ? (int)s.is_leaf[b] : 0;
        r.c1[j + 1] = (b > 0) ? s.child[4 * b] : 0;
    }
    r.id[0] = n;
    r.lev[0] = s.level[n];
    r.leaf[0] = (int)s.ring_out[n];
    r.c1[0] = 0;
    r.bi = s.bi[n];
    r.bj = s.bj[n];
    r.wait = 0;
}

template <int N>
__global__ void k_build_plans(DevState s) {
    const Geo<N> G(s);
    __shared__ NbInfo nbi;
    __shared__ NbInfo cnb[9];  // coarser neighbours' records
    const int nx = G.nx, ny = G.ny, R2 = ring2_len(nx, ny), R1 = ring1_len(nx, ny);
    const int total = s.lvl_off[AMR_MAXLV];
    const int t = threadIdx.x;
    for (int k = blockIdx.x; k < total; k += gridDim.x) {
        const int n = s.lvl_leaf[k];
        if (t == 0) load_nbinfo(s, n, nbi);
        __syncthreads();
        const int L = nbi.lev[0];
        if (t >= 1 && t <= 8 && nbi.id[t] > 0 && nbi.lev[t] == L - 1) {
            load_nbinfo(s, nbi.id[t], cnb[t]);
            atomicOr(&nbi.wait, 1 << t);
        }
        __syncthreads();
        // one plan type: queue q, plan array, unit lists of the flat fill
        // (copies (dest, source) from the front, fine-to-coarse cells (dest,
        // k*R + t) from the back, 2 ints each), ring length R, ring-2
        // indexing, offsets into the A pool (else C)
        auto build = [&](int q, int* plans, int* units, int R, bool two, bool afield) {
            auto off = [&](int blk, int xx, int yy) -> long long {
                return afield ? (long long)G.a(blk, 1, xx, yy) : (long long)G.c(blk, xx, yy);
            };
            const size_t cap2 = 2 * (size_t)(s.max_blks + 1) * R;
            for (int i = t; i < R; i += blockDim.x) {
                int x, y;
                if (two)
                    ring2_xy(i, nx, ny, x, y);
                else
                    ring1_xy(i, nx, ny, x, y);
                const int d = ghost_dir(x, y, nx, ny);
                bool deep = false;
                GPlan P;
                ghost_plan(nbi, nx, ny, L, d, x, y,
                           [&](int blk, int xx, int yy) -> long long {
                               // a coarser neighbour's ghost cell must be a copy or
                               // a fine-to-coarse value (its neighbour on that
                               // side exists and has its level) for the flat fill
                               const bool ring = xx < 1 || xx > nx || yy < 1 || yy > ny;
                               if (ring && blk == nbi.id[d] && nbi.lev[d] == L - 1) {
                                   const int dd = ghost_dir(xx, yy, nx, ny);
                                   if (!nbi.leaf[d] || cnb[d].id[dd] <= 0 || cnb[d].lev[dd] != L - 1)
                                       deep = true;
                               }
                               return off(blk, xx, yy);
                           },
                           P);
                plan_store(plans + (size_t)k * R * PLAN_INTS, R, i, P);
                if (deep || P.kind < 0) atomicOr(&s.fillinfo[q], 1);  // a level jump is reported there
                if (P.kind == 1) {
                    const size_t j = atomicAdd(&s.fillinfo[NQUEUES + q], 1);
                    units[2 * j] = (int)off(n, x, y);
                    units[2 * j + 1] = (int)(unsigned)P.src[0];
                } else if (P.kind == 2) {
                    const size_t j = atomicAdd(&s.fillinfo[2 * NQUEUES + q], 1);
                    units[cap2 - 2 - 2 * j] = (int)off(n, x, y);
                    units[cap2 - 1 - 2 * j] = k * R + i;
                }
            }
        };
        build(Q_FILLC, s.plan_c2, s.interp_c2, R2, true, false);
        build(Q_FILLC1, s.plan_c1, s.interp_c1, R1, false, false);
        build(Q_FILLHG, s.plan_hg, s.interp_hg, R1, false, true);
        __syncthreads();
        if (t < NBI_STRIDE)
            s.nbinfo[(size_t)k * NBI_STRIDE + t] = (t < NBI_INTS) ? reinterpret_cast<int*>(&nbi)[t] : 0;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Level-ordered launches: two phases in one launch.
//
// Fill phase: CTAs claim fill items (one leaf's ghost ring) in work order
// from queue[2q]. A fill item that reads a coarser neighbour's ring waits
// (bounded spin) for that neighbour's flag; every fill item raises its own
// block's flag when its ring, walls included, is in memory. Consumer phase:
// once the fill queue is empty, CTAs claim consumer items (the work that
// needs the block's own ring: collision, streaming, macroscopic values) from
// queue[2q+1]; a consumer item waits only for its own block's flag.
//
// A CTA claims its next item as soon as it starts the current one (the
// atomic's latency hides behind the work). Progress: the smallest unfinished
// fill item is held by a running CTA, as its current item or as the next one
// of a CTA whose current item is smaller (hence finished), and waits only on
// smaller items; consumer items are claimed after every fill item was. So
// every wait ends.

__device__ __forceinline__ int* fill_flags(const DevState& s, int q) {
    return s.ring_done + (size_t)q * (s.max_blks + 1);
}

// bounded spin of one thread until *flag is set; false if it ran out
__device__ __forceinline__ bool spin_flag(const int* flag) {
    for (int it = 0; it < kSpinLimit; ++it) {
        if (ld_acquire_i(flag) != 0) return true;
        __nanosleep(32);
    }
    return false;
}

// waits until every coarser neighbour of the item has its ring in memory;
// block-uniform, ends with a barrier
__device__ __forceinline__ void wait_coarse(const DevState& s, int q, const NbInfo& nbi) {
    const int t = threadIdx.x;
    if (t < 8 && ((nbi.wait >> (t + 1)) & 1))
        if (!spin_flag(fill_flags(s, q) + nbi.id[t + 1])) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, q);
    __syncthreads();
}

// Raises block n's flag; call after the barrier that follows the ring's last
// writes. The release store is cumulative: it orders every write of the CTA
// that the barrier ordered before thread 0's store.
__device__ __forceinline__ void publish_ring(const DevState& s, int q, int n) {
    if (threadIdx.x == 0) st_release_i(fill_flags(s, q) + n, 1);
}

// generic-proxy writes seen through an acquire, before bulk copies read them
__device__ __forceinline__ void fence_proxy_async_all() {
    asm volatile("fence.proxy.async;" ::: "memory");
}

// The fill phase of queue q: every claimed item runs fill(k, nbi) (its ring
// fill, with wait_coarse where the record's mask says so, block-uniform),
// then a barrier, walls(n, nbi), a barrier and the flag.
template <class FILL, class WALLS>
__device__ __forceinline__ void fill_phase(const DevState& s, int q, NbInfo* nbis, int* s_next,
                                           FILL fill, WALLS walls) {
    const int lmin = s.cnt->level_min, lmax = s.cnt->level_max;
    const int total = s.lvl_off[AMR_MAXLV];
    const int t = threadIdx.x;
    if (t == 0) *s_next = (int)atomicAdd(&s.queue[2 * q], 1u);
    __syncthreads();
    int k = *s_next;
    if (k < total && t < NBI_INTS)
        reinterpret_cast<int*>(&nbis[0])[t] = __ldg(s.nbinfo + (size_t)k * NBI_STRIDE + t);
    __syncthreads();
    int rb = 0;
    while (k < total) {
        const NbInfo& nbi = nbis[rb];
        unsigned kn = 0;
        if (t == 0) kn = atomicAdd(&s.queue[2 * q], 1u);  // the next item, claimed now
        const int n = nbi.id[0], L = nbi.lev[0];
        const bool do_fill = (L >= lmin && L <= lmax);
        if (do_fill) fill(k, n, nbi);
        if (t == 0) *s_next = (int)kn;
        __syncthreads();
        const int knext = *s_next;
        int pre = 0;
        if (knext < total && t < NBI_INTS) pre = __ldg(s.nbinfo + (size_t)knext * NBI_STRIDE + t);
        if (do_fill) {
            walls(n, nbi);
            __syncthreads();
        }
        publish_ring(s, q, n);
        if (t < NBI_INTS) reinterpret_cast<int*>(&nbis[rb ^ 1])[t] = pre;
        __syncthreads();
        k = knext;
        rb ^= 1;
    }
}

// The same walls for a block whose ring is in memory (written by an earlier
// launch) and, if T is given, in its shared C tile (index G.c(0,x,y)), which
// then is the source. No barrier inside: the rows read and written differ.
template <int N>
__device__ void wall_c_rows(const DevState& s, const Geo<N>& G, int n, int w, bool w3, bool w4,
                            double* T) {
    const int nx = G.nx, ny = G.ny;
    for (int idx = threadIdx.x; idx < (nx + 2 * w) * w * 2; idx += blockDim.x) {
        const int X = idx % (nx + 2 * w) + 1 - w, a = (idx / (nx + 2 * w)) % w + 1;
        const bool top = idx >= (nx + 2 * w) * w;
        if (top ? !w4 : !w3) continue;
        const int ys = top ? ny + 1 - a : a, yd = top ? ny + a : 1 - a;
        const double v = T ? T[G.c(0, X, ys)] : ldcg(s.C + G.c(n, X, ys));
        if (T) T[G.c(0, X, yd)] = v;
        s.C[G.c(n, X, yd)] = v;
    }
}

// which plan kinds a fill pass evaluates: 0 all, 1 all but coarse-to-fine
// (before a wait), 2 coarse-to-fine only (after it)
__device__ __forceinline__ bool pass_takes(int mode, int kind) {
    return mode == 0 || ((kind == 3) == (mode == 2));
}

// C ghost ring of width w of the item at work position k (block n) from its
// plans, into memory (level-ordered path). Kind 1 and 2 sources are
// interiors nothing writes during the launch; kind 3 sources include a
// coarser neighbour's ring written in it (read through L2 after the wait).
template <int N>
__device__ void fill_c_ring(const DevState& s, const Geo<N>& G, int k, int n, int w, int mode) {
    const int nx = G.nx, ny = G.ny;
    const int R = (w == 2) ? ring2_len(nx, ny) : ring1_len(nx, ny);
    const int* pl = ((w == 2) ? s.plan_c2 : s.plan_c1) + (size_t)k * R * PLAN_INTS;
    for (int t = threadIdx.x; t < R; t += blockDim.x) {
        const int meta = __ldg(pl + t);
        const int kind = plan_kind(meta);
        if (kind == 0 || !pass_takes(mode, kind)) continue;
        int x, y;
        if (w == 2)
            ring2_xy(t, nx, ny, x, y);
        else
            ring1_xy(t, nx, ny, x, y);
        if (kind < 0) {
            set_error(s, 4 /*AMRLBM_ERR_LEVEL_JUMP*/, n);
            continue;
        }
        double v;
        if (kind == 1) {
            v = __ldg(s.C + (unsigned)__ldg(pl + R + t));
        } else {
            double g[9];
            if (kind == 2) {
#pragma unroll
                for (int i = 0; i < 9; ++i) g[i] = __ldg(s.C + (unsigned)__ldg(pl + (1 + i) * R + t));
            } else {
#pragma unroll
                for (int i = 0; i < 9; ++i) g[i] = ldcg(s.C + (unsigned)__ldg(pl + (1 + i) * R + t));
            }
            v = plan_combine(meta, g);
        }
        s.C[G.c(n, x, y)] = v;
    }
}

// Symmetric_C_3/4 and Symmetric_C2_3/4 (BC_Cell.f90:46-104) on the walls of
// block n; after the ring fill and a barrier
template <int N>
__device__ void wall_c(const DevState& s, const Geo<N>& G, int n, const NbInfo& nbi, int w) {
    const int nx = G.nx, ny = G.ny;
    if (nbi.id[3] < 0) {
        for (int X = threadIdx.x + 1 - w; X <= nx + w; X += blockDim.x)
            for (int a = 1; a <= w; ++a)  // C(X,1-a) = C(X,a)
                s.C[G.c(n, X, 1 - a)] = ldcg(s.C + G.c(n, X, a));
    }
    if (nbi.id[4] < 0) {
        for (int X = threadIdx.x + 1 - w; X <= nx + w; X += blockDim.x)
            for (int a = 1; a <= w; ++a)  // C(X,ny+a) = C(X,ny+1-a)
                s.C[G.c(n, X, ny + a)] = ldcg(s.C + G.c(n, X, ny + 1 - a));
    }
}

// ---------------------------------------------------------------------------
// Collision_h_g_AMR (LBM_Subroutines.f90:116-189) of cell c of block n.
// T: shared C block (G.c(0,..)); the post-streaming populations B and (unless
// FUSED) P, Ux, Uy are read from memory, where nothing writes them during the
// launch. Writes the post-collision populations A to memory. FUSED: P, Ux,
// Uy come from Macroscopic_Values_g_AMR (:205-240) evaluated here on the
// same C ring.
template <bool SAFE, bool FUSED, int N>
__device__ __forceinline__ unsigned collide_cell(const DevState& s, const Geo<N>& G, int n, int c,
                                                 double inv_dx, const double* T) {
    const PhysD& ph = s.ph;
    const int nx = G.nx, BP = G.bplane, PP = G.pplane;
    const double inv_dx2 = inv_dx * inv_dx;
    const double* Hn = s.Bh + (size_t)n * 9 * BP + c;
    const double* Gn = s.Bg + (size_t)n * 9 * BP + c;
    Div<SAFE> dv;
    {
        const int x = c % nx + 1, y = c / nx + 1;
        auto Cs = [&](int a, int b) { return T[G.c(0, x + a, y + b)]; };
        const double c0 = Cs(0, 0);
        const double mu = chem_pot_f(dv, ph, inv_dx2, Cs);
        // ED_C_AMR (:244-258): (C(e)-C(-e))*0.5/dx
        auto Ec = [&](int k) {
            return ((Cs(d_ex(k), d_ey(k)) - Cs(-d_ex(k), -d_ey(k))) * 0.5) * inv_dx;
        };
        // ED_M_AMR (:262-277): (-C(-e)-3C(0)+5C(e)-C(2e))*0.25/dx
        auto Em = [&](int k) {
            return ((-Cs(-d_ex(k), -d_ey(k)) - 3.0 * c0 + 5.0 * Cs(d_ex(k), d_ey(k)) -
                     Cs(2 * d_ex(k), 2 * d_ey(k))) *
                    0.25) *
                   inv_dx;
        };
        double DcDx, DcDy, ni, nj;
        gradient_ed_f(dv, Ec, DcDx, DcDy);
        {  // normal_AMR (:25-37)
            const double t = sqrt(DcDx * DcDx + DcDy * DcDy + 1.e-32);
            const double rt = __drcp_rn(t);
            ni = dv(DcDx, t, rt);
            nj = dv(DcDy, t, rt);
        }
        const double Rho = ph.Rhol + c0 * ph.dRho;
        const double Fb = (ph.Rhoh - Rho) * ph.Gy;
        double P, Ux, Uy;
        if (FUSED) {
            double gx, gy;
            gradient_iso_f(dv, inv_dx, Cs, gx, gy);
            const double Fx = mu * gx;
            const double Fy = mu * gy + Fb;
            auto g = [&](int k) { return __ldg(Gn + (k - 1) * BP); };
            const double sx = ((((g(2) - g(4)) + g(6)) - g(7)) - g(8)) + g(9);
            const double sy = ((((g(3) - g(5)) + g(6)) + g(7)) - g(8)) - g(9);
            const double rr = __drcp_rn(Rho);
            Ux = dv(3.0 * sx + 0.5 * Fx, Rho, rr);
            Uy = dv(3.0 * sy + 0.5 * Fy, Rho, rr);
            double sp = 0.0;
#pragma unroll
            for (int k = 1; k <= 9; ++k) sp = sp + g(k);
            P = sp + ph.dRho6 * (Ux * gx + Uy * gy);
        } else {
            P = __ldg(s.P + (size_t)n * PP + c);
            Ux = __ldg(s.Ux + (size_t)n * PP + c);
            Uy = __ldg(s.Uy + (size_t)n * PP + c);
        }
        // Equilibrium_h_g_AMR (:2-21) scalars
        const double tmp = dv(12.0 * (1.0 - c0), ph.W, ph.yW) * ph.M0;
        const double U215 = 1.5 * (Ux * Ux + Uy * Uy);
        const double ud_c = Ux * DcDx + Uy * DcDy;
        double DmX, DmY;
        gradient_ed_f(dv, Em, DmX, DmY);
        const double ud_m = Ux * DmX + Uy * DmY;
        double tau;
        if (c0 < 0.0) {
            tau = ph.taul5;
        } else if (c0 > 1.0) {
            tau = ph.tauh5;
        } else {
            tau = c0 * ph.itau_d + ph.itaul;
            tau = __drcp_rn(tau) + 0.5;
        }
        const double s9 = __drcp_rn(tau);
        double f[10], hm[10];
#pragma unroll
        for (int k = 1; k <= 9; ++k) {
            const double wk = wa(k);
            const double eU = (double)d_ex(k) * Ux + (double)d_ey(k) * Uy;
            const double eN = (double)d_ex(k) * ni + (double)d_ey(k) * nj;
            const double Gm = wk * (1.0 + eU * (3.0 + 4.5 * eU) - U215);
            const double heq = c0 * (Gm + tmp * wk * eN);
            s.Ah[G.a(n, k, x, y)] = __ldg(Hn + (k - 1) * BP) * ph.omwc + heq * ph.wc;
            const double Ak = (Gm - wk) * ph.dRho3 + Gm * mu;
            const double Bk = ((double)d_ey(k) - Uy) * Gm * Fb;
            const double hc = Ak * (Ec(k) - ud_c) + Bk;
            const double geq = P * wk + dv.d3((Gm - wk) * Rho) - 0.5 * hc;
            f[k] = __ldg(Gn + (k - 1) * BP) - geq;
            hm[k] = Ak * (Em(k) - ud_m) + Bk;
        }
        // MRT_Collision_AMR (:348-361): Convert, relax 8 and 9, Reconvt, /36
        double m[10];
        m[1] = f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9];
        m[2] = -4.0 * f[1] - f[2] - f[3] - f[4] - f[5] + 2.0 * (f[6] + f[7] + f[8] + f[9]);
        m[3] = 4.0 * f[1] - 2.0 * (f[2] + f[3] + f[4] + f[5]) + f[6] + f[7] + f[8] + f[9];
        m[4] = f[2] - f[4] + f[6] - f[7] - f[8] + f[9];
        m[5] = -2.0 * (f[2] - f[4]) + f[6] - f[7] - f[8] + f[9];
        m[6] = f[3] - f[5] + f[6] + f[7] - f[8] - f[9];
        m[7] = -2.0 * (f[3] - f[5]) + f[6] + f[7] - f[8] - f[9];
        m[8] = (f[2] - f[3] + f[4] - f[5]) * s9;
        m[9] = (f[6] - f[7] + f[8] - f[9]) * s9;
        const double b1 = 4.0 * m[1] - m[2] - 2.0 * m[3];
        const double b2 = 4.0 * m[1] + 2.0 * m[2] + m[3];
        double o[10];
        o[1] = 4.0 * (m[1] - m[2] + m[3]);
        o[2] = b1 + 6.0 * (m[4] - m[5]) + 9.0 * m[8];
        o[3] = b1 + 6.0 * (m[6] - m[7]) - 9.0 * m[8];
        o[4] = b1 - 6.0 * (m[4] - m[5]) + 9.0 * m[8];
        o[5] = b1 - 6.0 * (m[6] - m[7]) - 9.0 * m[8];
        o[6] = b2 + 6.0 * m[4] + 3.0 * m[5] + 6.0 * m[6] + 3.0 * m[7] + 9.0 * m[9];
        o[7] = b2 - 6.0 * m[4] - 3.0 * m[5] + 6.0 * m[6] + 3.0 * m[7] - 9.0 * m[9];
        o[8] = b2 - 6.0 * m[4] - 3.0 * m[5] - 6.0 * m[6] - 3.0 * m[7] + 9.0 * m[9];
        o[9] = b2 + 6.0 * m[4] + 3.0 * m[5] - 6.0 * m[6] - 3.0 * m[7] - 9.0 * m[9];
#pragma unroll
        for (int k = 1; k <= 9; ++k)
            s.Ag[G.a(n, k, x, y)] = (__ldg(Gn + (k - 1) * BP) - dv.d36(o[k])) + hm[k];
    }
    return dv.bad;
}


// Macroscopic_Values_g_AMR (LBM_Subroutines.f90:205-240) of cell c of block n
// from T and the g populations in memory; dc = the Err_Interface term
// (Refine_Derefine.f90:327-351) of the cell
template <bool SAFE, int N>
__device__ __forceinline__ unsigned macro_g_cell_f(const DevState& s, const Geo<N>& G, int n, int c,
                                                   double inv_dx, const double* T, double& dc) {
    const PhysD& ph = s.ph;
    const int nx = G.nx, BP = G.bplane;
    const double inv_dx2 = inv_dx * inv_dx;
    Div<SAFE> dv;
    const int x = c % nx + 1, y = c / nx + 1;
    auto Cs = [&](int a, int b) { return T[G.c(0, x + a, y + b)]; };
    const double* Gn = s.Bg + (size_t)n * 9 * BP + c;
    auto g = [&](int k) { return __ldg(Gn + (k - 1) * BP); };
    double gx, gy;
    gradient_iso_f(dv, inv_dx, Cs, gx, gy);
    const double mu = chem_pot_f(dv, ph, inv_dx2, Cs);
    const double c0 = Cs(0, 0);
    const double Rho = ph.Rhol + c0 * ph.dRho;
    const double Fb = (ph.Rhoh - Rho) * ph.Gy;
    const double Fx = mu * gx;
    const double Fy = mu * gy + Fb;
    const double sx = ((((g(2) - g(4)) + g(6)) - g(7)) - g(8)) + g(9);
    const double sy = ((((g(3) - g(5)) + g(6)) + g(7)) - g(8)) - g(9);
    const double rr = __drcp_rn(Rho);
    const double Ux = dv(3.0 * sx + 0.5 * Fx, Rho, rr);
    const double Uy = dv(3.0 * sy + 0.5 * Fy, Rho, rr);
    double sp = 0.0;
#pragma unroll
    for (int k = 1; k <= 9; ++k) sp = sp + g(k);
    s.P[G.p(n, x, y)] = sp + ph.dRho6 * (Ux * gx + Uy * gy);
    s.Ux[G.p(n, x, y)] = Ux;
    s.Uy[G.p(n, x, y)] = Uy;
    const double a = Cs(1, 0) - Cs(-1, 0), b = Cs(0, 1) - Cs(0, -1);
    dc = a * a + b * b;
    return dv.bad;
}
// Collision of every cell of block n: the branch-free exact division path,
// and the IEEE path for a cell whose flag says a quotient left its range.
template <int N, bool FUSED>
__device__ __forceinline__ void collide_block(const DevState& s, const Geo<N>& G, int n,
                                              const double* T) {
    const double inv_dx = 1.0 / (double)__ldg(s.dx + n);  // dx is a power of two: exact
    for (int c = threadIdx.x; c < G.nx * G.ny; c += blockDim.x)
        if (collide_cell<false, FUSED>(s, G, n, c, inv_dx, T))
            collide_cell<true, FUSED>(s, G, n, c, inv_dx, T);
}

// Macroscopic_Values_g_AMR of every cell of block n; returns this thread's
// maximum of the Err_Interface terms
template <int N>
__device__ __forceinline__ double macro_g_block(const DevState& s, const Geo<N>& G, int n,
                                                const double* T) {
    const double inv_dx = 1.0 / (double)__ldg(s.dx + n);
    double mx = 0.0;
    for (int c = threadIdx.x; c < G.nx * G.ny; c += blockDim.x) {
        double dc;
        if (macro_g_cell_f<false>(s, G, n, c, inv_dx, T, dc))
            macro_g_cell_f<true>(s, G, n, c, inv_dx, T, dc);
        mx = fmax(mx, dc);
    }
    return mx;
}

// Err_Interface (Refine_Derefine.f90:327-351): err(n) = sqrt(max DC)/(2 dx)
// from each thread's running maximum. fmax drops a NaN term as the
// reference's MAX(err, DC) never selects one. Contains a barrier.
__device__ __forceinline__ void err_reduce(const DevState& s, int n, double mx, double* red) {
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) m = fmax(m, red[w]);
        s.err[n] = sqrt(m) / (2.0 * s.dx[n]);
    }
}

// ---------------------------------------------------------------------------
// Whether fill Q takes the flat path: no coarse-to-fine cell reads a coarser
// neighbour's ghost cell that is itself coarse-to-fine or a wall cell, and
// every leaf's level is in [LevelMin, LevelMax]. Else the consumer launch
// fills level by level.
__device__ __forceinline__ bool flat_fill(const DevState& s, int q) {
    return s.fillinfo[q] == 0 && s.cnt->level_min <= s.cnt->leaf_min &&
           s.cnt->level_max >= s.cnt->leaf_max;
}

// The copies and fine-to-coarse ghost cells of every leaf, one flat launch:
// one thread per copied cell (and field: its 9 populations together), one per
// fine-to-coarse cell (and field and population). Every source is an
// interior cell no launch of this fill writes. The coarse-to-fine cells (which
// read the copies and fine-to-coarse cells of coarser neighbours) and the
// walls are left to the consumer launch.
template <int N, int Q>
__global__ void __launch_bounds__(256) k_fill_flat(DevState s) {
    if (!flat_fill(s, Q)) return;
    const Geo<N> G(s);
    constexpr bool HG = (Q == Q_FILLHG);
    constexpr int F = HG ? 2 : 1;
    const int R = (Q == Q_FILLC) ? ring2_len(G.nx, G.ny) : ring1_len(G.nx, G.ny);
    const int* plans = (Q == Q_FILLC) ? s.plan_c2 : (Q == Q_FILLC1 ? s.plan_c1 : s.plan_hg);
    const int* units = (Q == Q_FILLC) ? s.interp_c2 : (Q == Q_FILLC1 ? s.interp_c1 : s.interp_hg);
    const size_t cap2 = 2 * (size_t)(s.max_blks + 1) * R;
    const int nc = s.fillinfo[NQUEUES + Q], ni = s.fillinfo[2 * NQUEUES + Q];
    const int nA = nc * F, nB = ni * (HG ? 18 : 1);
    for (int u = blockIdx.x * blockDim.x + threadIdx.x; u < nA + nB; u += gridDim.x * blockDim.x) {
        if (u < nA) {
            const int j = u % nc, f = u / nc;
            const unsigned dst = (unsigned)__ldg(units + 2 * j), src = (unsigned)__ldg(units + 2 * j + 1);
            double* A = HG ? (f ? s.Ag : s.Ah) : s.C;
            if (HG) {
                double v[9];
#pragma unroll
                for (int i = 0; i < 9; ++i) v[i] = __ldg(A + src + (size_t)i * G.aplane);
#pragma unroll
                for (int i = 0; i < 9; ++i) A[dst + (size_t)i * G.aplane] = v[i];
            } else {
                A[dst] = __ldg(A + src);
            }
            continue;
        }
        const int v = u - nA, j = HG ? v / 18 : v, fq = HG ? v % 18 : 0;
        const unsigned dst = (unsigned)__ldg(units + cap2 - 2 - 2 * (size_t)j);
        const int e = __ldg(units + cap2 - 1 - 2 * (size_t)j);
        const int* pl = plans + (size_t)(e / R) * R * PLAN_INTS + e % R;
        const int meta = __ldg(pl);
        double* A = HG ? (fq >= 9 ? s.Ag : s.Ah) : s.C;
        const size_t qo = (size_t)(fq % 9) * (HG ? G.aplane : 0);
        double g[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) g[i] = __ldg(A + (unsigned)__ldg(pl + (1 + i) * R) + qo);
        A[dst + qo] = plan_combine(meta, g);
    }
}

// The coarse-to-fine ghost cells of block n (work position c) on the flat
// path, into its staged copy and into memory. Sources: the coarser
// neighbour's interior and its copies / fine-to-coarse cells, written by
// k_fill_flat. T: shared C tile (index G.c(0,x,y)).
template <int N>
__device__ void c2f_cells_c(const DevState& s, const Geo<N>& G, int c, int n, int w, double* T) {
    const int nx = G.nx, ny = G.ny;
    const int R = (w == 2) ? ring2_len(nx, ny) : ring1_len(nx, ny);
    const int* pl = ((w == 2) ? s.plan_c2 : s.plan_c1) + (size_t)c * R * PLAN_INTS;
    for (int t = threadIdx.x; t < R; t += blockDim.x) {
        const int meta = __ldg(pl + t);
        if (plan_kind(meta) != 3) continue;
        int x, y;
        if (w == 2)
            ring2_xy(t, nx, ny, x, y);
        else
            ring1_xy(t, nx, ny, x, y);
        double g[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) g[i] = __ldg(s.C + (unsigned)__ldg(pl + (1 + i) * R + t));
        const double v = plan_combine(meta, g);
        if (T) T[G.c(0, x, y)] = v;
        s.C[G.c(n, x, y)] = v;
    }
}
// The same for the h and g planes staged in As ([field][q][pool plane
// layout]): one thread per (ghost cell, population), both fields.
template <int N>
__device__ void c2f_cells_hg(const DevState& s, const Geo<N>& G, int c, int n, double* As) {
    const int nx = G.nx, ny = G.ny, RG = ring1_len(nx, ny), FP = 9 * G.aplane;
    const int* pl = s.plan_hg + (size_t)c * RG * PLAN_INTS;
    for (int idx = threadIdx.x; idx < 9 * RG; idx += blockDim.x) {
        const int r = idx % RG, qq = idx / RG;
        const int meta = __ldg(pl + r);
        if (plan_kind(meta) != 3) continue;
        int x, y;
        ring1_xy(r, nx, ny, x, y);
        unsigned o[9];
#pragma unroll
        for (int i = 0; i < 9; ++i) o[i] = (unsigned)__ldg(pl + (1 + i) * RG + r) + qq * G.aplane;
#pragma unroll
        for (int f = 0; f < 2; ++f) {
            double* A = f ? s.Ag : s.Ah;
            double g[9];
#pragma unroll
            for (int i = 0; i < 9; ++i) g[i] = __ldg(A + o[i]);
            const double v = plan_combine(meta, g);
            As[f * FP + G.a(0, qq + 1, x, y)] = v;
            A[G.a(n, qq + 1, x, y)] = v;
        }
    }
}

__host__ __device__ constexpr int fill_c_min_blocks(int consumer) {
    return (consumer == CONS_COLLIDE_READ || consumer == CONS_COLLIDE_FUSED) ? 2 : 3;
}

// Level-ordered C ghost fill of width w (Fill_Ghost_Cells_C.f90:2-416,
// Fill_Ghost_Cells_C2.f90:2-416) and its consumer. Fill items: all leaves in
// work order; leaves of levels outside [LevelMin, LevelMax] are not filled
// (as the reference's DO L = LevelMin, LevelMax) but still get the consumer
// work. A consumer item bulk-copies its block's C tile, ring included, into
// one of two shared stages; the copy of the next item's tile starts while
// the current one is consumed (at once if that block's fill is done, else
// after the wait for it).
template <int N, int CONSUMER>
__global__ void __launch_bounds__(256, fill_c_min_blocks(CONSUMER))
    k_fill_c(DevState s, int w, int q) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const Geo<N> G(s);
    __shared__ NbInfo nbis[2];
    __shared__ double red[32];
    __shared__ int s_next;
    const int t = threadIdx.x;
    const int total = s.lvl_off[AMR_MAXLV];
    // fast: k_fill_flat has filled every ring; the walls are left to the
    // consumer items. Else the fill phase fills level by level, walls included.
    const bool fast = flat_fill(s, q);
    if (!fast)
        fill_phase(
            s, q, nbis, &s_next,
            [&](int k, int n, const NbInfo& nbi) {
                if (nbi.wait) {
                    fill_c_ring<N>(s, G, k, n, w, 1);
                    wait_coarse(s, q, nbi);
                    fill_c_ring<N>(s, G, k, n, w, 2);
                } else {
                    fill_c_ring<N>(s, G, k, n, w, 0);
                }
            },
            [&](int n, const NbInfo& nbi) { wall_c<N>(s, G, n, nbi, w); });
    // item c's level (record word lev[0]) and walls (id[3], id[4] < 0)
    auto rec_walls = [&](int c, int& L, bool& w3, bool& w4) {
        const int* rec = s.nbinfo + (size_t)c * NBI_STRIDE;
        L = __ldg(rec + 9);
        w3 = __ldg(rec + 3) < 0;
        w4 = __ldg(rec + 4) < 0;
    };
    if (CONSUMER == CONS_NONE) {  // flat path: coarse-to-fine cells and walls in memory
        if (fast)
            for (int c = blockIdx.x; c < total; c += gridDim.x) {
                int L;
                bool w3, w4;
                rec_walls(c, L, w3, w4);
                const int n = __ldg(s.lvl_leaf + c);
                c2f_cells_c<N>(s, G, c, n, w, nullptr);
                __syncthreads();
                if (w3 || w4) wall_c_rows<N>(s, G, n, w, w3, w4, nullptr);
                __syncthreads();
            }
        return;
    }

    constexpr bool collide = (CONSUMER == CONS_COLLIDE_READ || CONSUMER == CONS_COLLIDE_FUSED);
    if (collide && blockIdx.x == 0 && t == 0)
        atomicAdd(&s.cnt->updates, (unsigned long long)total * (unsigned long long)(G.nx * G.ny));
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smraw);  // [2]
    double* tiles = reinterpret_cast<double*>(smraw + 128);
    const unsigned tb = (unsigned)G.cplane * 8;
    const int* flags = fill_flags(s, q);
    // thread 0: copy item c's C tile into stage st once its fill is done;
    // without `block` only if it is done already (returns whether it started)
    auto start_tile = [&](int st, int c, bool block) {
        const int nn = __ldg(s.lvl_leaf + c);
        if (fast) {
            // the ring was written by the previous launch
        } else if (block) {
            if (!spin_flag(flags + nn)) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 200 + q);
        } else if (ld_acquire_i(flags + nn) == 0) {
            return false;
        }
        fence_proxy_async_all();
        mbar_expect_tx(&bar[st], tb);
        bulk_g2s(tiles + (size_t)st * G.cplane, s.C + (size_t)nn * G.cplane, tb, &bar[st]);
        return true;
    };
    bool pend = false;  // thread 0: the next item's copy is still to start
    if (t == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        const int c0 = (int)atomicAdd(&s.queue[2 * q + 1], 1u);
        s_next = c0;
        if (c0 < total) start_tile(0, c0, true);
    }
    __syncthreads();
    int c = s_next;
    unsigned phase = 0;  // bit st: parity of stage st's next completion
    int st = 0;
    while (c < total) {
        unsigned cn = 0;
        if (t == 0) cn = atomicAdd(&s.queue[2 * q + 1], 1u);
        const int n = __ldg(s.lvl_leaf + c);
        if (__syncthreads_or(mbar_wait(&bar[st], (phase >> st) & 1u) ? 0 : 1)) {
            if (t == 0) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 100 + q);
            mbar_wait(&bar[st], (phase >> st) & 1u);  // the copy must land before exit
            break;
        }
        phase ^= 1u << st;
        if (t == 0) {
            s_next = (int)cn;
            pend = ((int)cn < total) && !start_tile(st ^ 1, (int)cn, false);
        }
        double* T = tiles + (size_t)st * G.cplane;
        if (fast) {  // coarse-to-fine cells, then Symmetric_C(2)_3/4, on the tile and in memory
            int L;
            bool w3, w4;
            rec_walls(c, L, w3, w4);
            c2f_cells_c<N>(s, G, c, n, w, T);
            __syncthreads();
            if (w3 || w4) {
                wall_c_rows<N>(s, G, n, w, w3, w4, T);
                __syncthreads();
            }
        }
        if (CONSUMER == CONS_MACRO_G)
            err_reduce(s, n, macro_g_block<N>(s, G, n, T), red);
        else
            collide_block<N, CONSUMER == CONS_COLLIDE_FUSED>(s, G, n, T);
        __syncthreads();
        c = s_next;
        st ^= 1;
        if (t == 0 && pend) start_tile(st, c, true);
    }
}

// ---------------------------------------------------------------------------
// h/g ghost ring of the item at work position k (block n) from its plans,
// into memory (mode as fill_c_ring). A cell without a plan keeps its value in
// memory. Copies take one thread per (ring cell, field) with the 9
// populations' loads in flight together; interpolated cells one thread per
// (ring cell, field, population) with the 9 stencil loads in flight together.
template <int N>
__device__ void fill_hg_ring(const DevState& s, const Geo<N>& G, int k, int n, int mode) {
    const int nx = G.nx, ny = G.ny, RG = ring1_len(nx, ny);
    const int* pl = s.plan_hg + (size_t)k * RG * PLAN_INTS;
    if (mode != 2) {
        for (int idx = threadIdx.x; idx < 2 * RG; idx += blockDim.x) {
            const int r = idx % RG;
            const int kind = plan_kind(__ldg(pl + r));
            if (kind != 1 && kind != -1) continue;
            int x, y;
            ring1_xy(r, nx, ny, x, y);
            if (kind < 0) {
                set_error(s, 4 /*AMRLBM_ERR_LEVEL_JUMP*/, n);
                continue;
            }
            double* A = (idx >= RG) ? s.Ag : s.Ah;
            const double* src = A + (unsigned)__ldg(pl + RG + r);
            double v[9];
#pragma unroll
            for (int qq = 0; qq < 9; ++qq) v[qq] = __ldg(src + (size_t)qq * G.aplane);
#pragma unroll
            for (int qq = 0; qq < 9; ++qq) A[G.a(n, qq + 1, x, y)] = v[qq];
        }
    }
    for (int idx = threadIdx.x; idx < 18 * RG; idx += blockDim.x) {
        const int r = idx % RG, fq = idx / RG;
        const int meta = __ldg(pl + r);
        const int kind = plan_kind(meta);
        if (kind < 2 || !pass_takes(mode, kind)) continue;
        int x, y;
        ring1_xy(r, nx, ny, x, y);
        const int qq = fq % 9;
        double* A = (fq >= 9) ? s.Ag : s.Ah;
        const size_t qo = (size_t)qq * G.aplane;
        double g[9];
        if (kind == 2) {
#pragma unroll
            for (int i = 0; i < 9; ++i) g[i] = __ldg(A + (unsigned)__ldg(pl + (1 + i) * RG + r) + qo);
        } else {
#pragma unroll
            for (int i = 0; i < 9; ++i) g[i] = ldcg(A + (unsigned)__ldg(pl + (1 + i) * RG + r) + qo);
        }
        A[G.a(n, qq + 1, x, y)] = plan_combine(meta, g);
    }
}

// Bounce_Back_3/4 (BC_Cell.f90:2-42): f(i,X,wall row) = f(opposite(i), Xn,
// first row) on the walls of block n; after the ring fill and a barrier
template <int N>
__device__ void bounce_back(const DevState& s, const Geo<N>& G, int n, const NbInfo& nbi) {
    const int nx = G.nx, ny = G.ny;
    for (int wall = 3; wall <= 4; ++wall) {
        if (nbi.id[wall] >= 0) continue;
        const int Y = (wall == 3) ? 0 : ny + 1, Yi = (wall == 3) ? 1 : ny;
        const int sgn = (wall == 3) ? 1 : -1;
        for (int idx = threadIdx.x; idx < (nx + 2) * 18; idx += blockDim.x) {
            const int X = idx % (nx + 2), qf = idx / (nx + 2);
            const int i = qf % 9 + 1;
            int J = 1, Xn = X;
            if (i > 1) {
                Xn = min(max(0, X + sgn * d_ex(i) * d_ey(i)), nx + 1);
                J = (i - 2) + 4 * ((i / 2) % 2);
            }
            double* A = (qf >= 9) ? s.Ag : s.Ah;
            const double* src = A + G.a(n, J, Xn, Yi);
            A[G.a(n, i, X, Y)] = (Xn == 0 || Xn == nx + 1) ? ldcg(src) : __ldg(src);
        }
    }
}

// The same walls on a block's h and g planes staged in shared memory (As:
// [field][q][pool plane layout]), also written to memory. No barrier inside:
// wall rows are written, rows 1 and ny read.
template <int N>
__device__ void bounce_back_staged(const DevState& s, const Geo<N>& G, int n, bool w3, bool w4,
                                   double* As) {
    const int nx = G.nx, ny = G.ny, FP = 9 * G.aplane;
    for (int idx = threadIdx.x; idx < (nx + 2) * 36; idx += blockDim.x) {
        const int X = idx % (nx + 2), qf = (idx / (nx + 2)) % 18;
        const bool top = idx >= (nx + 2) * 18;
        if (top ? !w4 : !w3) continue;
        const int Y = top ? ny + 1 : 0, Yi = top ? ny : 1, sgn = top ? -1 : 1;
        const int i = qf % 9 + 1, f = qf / 9;
        int J = 1, Xn = X;
        if (i > 1) {
            Xn = min(max(0, X + sgn * d_ex(i) * d_ey(i)), nx + 1);
            J = (i - 2) + 4 * ((i / 2) % 2);
        }
        const double v = As[f * FP + G.a(0, J, Xn, Yi)];
        As[f * FP + G.a(0, i, X, Y)] = v;
        (f ? s.Ag : s.Ah)[G.a(n, i, X, Y)] = v;
    }
}

// Streaming (Perfect_Shift_AMR / Streaming_LaxWendroff_AMR,
// LBM_Subroutines.f90:41-90) of every cell of block n into B, and
// Macroscopic_Values_h_AMR (:193-201), from As: the block's h and g planes
// (ring included) in shared memory, each field 9 planes in the pool layout.
template <int N>
__device__ void stream_block(const DevState& s, const Geo<N>& G, int n, const double* As) {
    const int nx = G.nx, ny = G.ny;
    const int FP = 9 * G.aplane;
    const double cfl = 1.0 / (double)__ldg(s.dx + n);
    const bool shift = cfl > (double)0.9f;
    const double cA = cfl / 2.0 * (1.0 + cfl), cB = 1.0 - cfl * cfl, cC = cfl / 2.0 * (1.0 - cfl);
    for (int c = threadIdx.x; c < nx * ny; c += blockDim.x) {
        const int x = c % nx + 1, y = c / nx + 1;
        double csum = 0.0;
#pragma unroll
        for (int f = 0; f < 2; ++f) {
            const double* Af = As + f * FP;
            double* B = f ? s.Bg : s.Bh;
#pragma unroll
            for (int i = 1; i <= 9; ++i) {
                double v;
                if (i == 1) {
                    v = Af[G.a(0, 1, x, y)];
                } else if (shift) {
                    v = Af[G.a(0, i, x - d_ex(i), y - d_ey(i))];
                } else {
                    v = cA * Af[G.a(0, i, x - d_ex(i), y - d_ey(i))] + cB * Af[G.a(0, i, x, y)] -
                        cC * Af[G.a(0, i, x + d_ex(i), y + d_ey(i))];
                }
                B[G.bb(n, i, x, y)] = v;
                if (f == 0) csum = csum + v;
            }
        }
        s.C[G.c(n, x, y)] = csum;
    }
}

// Level-ordered Fill_Ghost_Cells_hg (Fill_Ghost_Cells_hg.f90:2-477) with
// Bounce_Back_3/4, then streaming and Macroscopic_Values_h_AMR of every leaf.
// The ghost ring goes to memory; a streaming item waits for its own block's
// fill, then bulk-copies the block's h and g planes into shared memory.
template <int N>
__global__ void __launch_bounds__(256, 3) k_fill_hg_stream(DevState s) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const Geo<N> G(s);
    __shared__ NbInfo nbis[2];
    __shared__ int s_next;
    const int q = Q_FILLHG;
    const int t = threadIdx.x;
    const int total = s.lvl_off[AMR_MAXLV];
    // fast: k_fill_flat has filled every ring; bounce-back is left to the
    // streaming items. Else the fill phase fills level by level, walls included.
    const bool fast = flat_fill(s, q);
    if (!fast)
        fill_phase(
            s, q, nbis, &s_next,
            [&](int k, int n, const NbInfo& nbi) {
                if (nbi.wait) {
                    fill_hg_ring<N>(s, G, k, n, 1);
                    wait_coarse(s, q, nbi);
                    fill_hg_ring<N>(s, G, k, n, 2);
                } else {
                    fill_hg_ring<N>(s, G, k, n, 0);
                }
            },
            [&](int n, const NbInfo& nbi) { bounce_back<N>(s, G, n, nbi); });
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smraw);
    double* As = reinterpret_cast<double*>(smraw + 128);  // [h|g][q][pool plane layout]
    const int FP = 9 * G.aplane;
    const unsigned fb = (unsigned)FP * 8;
    const int* flags = fill_flags(s, q);
    if (t == 0) {
        mbar_init(bar, 1);
        s_next = (int)atomicAdd(&s.queue[2 * q + 1], 1u);
    }
    __syncthreads();
    int c = s_next;
    unsigned phase = 0;
    while (c < total) {
        unsigned cn = 0;
        const int n = __ldg(s.lvl_leaf + c);
        if (t == 0) {
            cn = atomicAdd(&s.queue[2 * q + 1], 1u);
            if (!fast && !spin_flag(flags + n)) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 200 + q);
            fence_proxy_async_all();
            mbar_expect_tx(bar, 2 * fb);
            bulk_g2s(As, s.Ah + (size_t)n * FP, fb, bar);
            bulk_g2s(As + FP, s.Ag + (size_t)n * FP, fb, bar);
            s_next = (int)cn;
        }
        if (__syncthreads_or(mbar_wait(bar, phase) ? 0 : 1)) {
            if (t == 0) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 100 + q);
            mbar_wait(bar, phase);  // the copies must land before exit
            break;
        }
        phase ^= 1u;
        if (fast) {  // coarse-to-fine cells, then Bounce_Back_3/4, on the staged planes and in memory
            const int* rec = s.nbinfo + (size_t)c * NBI_STRIDE;
            const bool w3 = __ldg(rec + 3) < 0, w4 = __ldg(rec + 4) < 0;
            c2f_cells_hg<N>(s, G, c, n, As);
            __syncthreads();
            if (w3 || w4) {
                bounce_back_staged<N>(s, G, n, w3, w4, As);
                __syncthreads();
            }
        }
        stream_block<N>(s, G, n, As);
        c = s_next;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// grid-stride kernels over the leaf list (one CTA per block), C tile staged
// by plain loads

template <int N>
__device__ __forceinline__ void load_tile_c(const DevState& s, const Geo<N>& G, int n, double* T) {
    for (int i = threadIdx.x; i < G.cplane; i += blockDim.x) T[i] = s.C[(size_t)n * G.cplane + i];
    __syncthreads();
}

template <int N>
__global__ void __launch_bounds__(256, 2) k_collide(DevState s) {
    extern __shared__ __align__(16) double T[];
    const Geo<N> G(s);
    const int nleaf = s.cnt->nleaf;
    if (blockIdx.x == 0 && threadIdx.x == 0)
        atomicAdd(&s.cnt->updates, (unsigned long long)nleaf * (unsigned long long)(G.nx * G.ny));
    for (int m = blockIdx.x; m < nleaf; m += gridDim.x) {
        const int n = s.leaf[m];
        load_tile_c<N>(s, G, n, T);
        collide_block<N, false>(s, G, n, T);
        __syncthreads();
    }
}

template <int N>
__global__ void __launch_bounds__(256, 2) k_macro_g(DevState s) {
    extern __shared__ __align__(16) double T[];
    __shared__ double red[32];
    const Geo<N> G(s);
    const int nleaf = s.cnt->nleaf;
    for (int m = blockIdx.x; m < nleaf; m += gridDim.x) {
        const int n = s.leaf[m];
        load_tile_c<N>(s, G, n, T);
        err_reduce(s, n, macro_g_block<N>(s, G, n, T), red);
        __syncthreads();
    }
}

// Macroscopic_Values_h_AMR (LBM_Subroutines.f90:193-201)
template <int N>
__global__ void k_macro_h(DevState s) {
    const Geo<N> G(s);
    const int nleaf = s.cnt->nleaf, nn = G.nx * G.ny;
    for (int m = blockIdx.x; m < nleaf; m += gridDim.x) {
        const int n = s.leaf[m];
        for (int c = threadIdx.x; c < nn; c += blockDim.x) {
            const int x = c % G.nx + 1, y = c / G.nx + 1;
            double sum = 0.0;
#pragma unroll
            for (int q = 1; q <= 9; ++q) sum = sum + s.Bh[G.bb(n, q, x, y)];
            s.C[G.c(n, x, y)] = sum;
        }
    }
}

// Err_Interface (Refine_Derefine.f90:327-351) of every leaf
template <int N>
__global__ void k_err(DevState s) {
    __shared__ double red[32];
    const Geo<N> G(s);
    const int nleaf = s.cnt->nleaf, nx = G.nx, ny = G.ny;
    for (int m = blockIdx.x; m < nleaf; m += gridDim.x) {
        const int n = s.leaf[m];
        double mx = 0.0;
        for (int c = threadIdx.x; c < nx * ny; c += blockDim.x) {
            const int x = c % nx + 1, y = c / nx + 1;
            const double a = s.C[G.c(n, x + 1, y)] - s.C[G.c(n, x - 1, y)];
            const double b = s.C[G.c(n, x, y + 1)] - s.C[G.c(n, x, y - 1)];
            mx = fmax(mx, a * a + b * b);
        }
        err_reduce(s, n, mx, red);
        __syncthreads();
    }
}

// Div<false> (with its recompute on a flag) against IEEE division: a from a
// spread of binades, b a fixed
// divisor (b > 0) or random (b == 0); counts results whose bits differ.
__global__ void k_selftest_div(unsigned long long n, unsigned long long seed, double bfix,
                               unsigned long long* bad) {
    unsigned long long cnt = 0;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < n;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        unsigned long long z = seed + i * 0x9E3779B97F4A7C15ull;  // splitmix64
        auto next = [&]() {
            z += 0x9E3779B97F4A7C15ull;
            unsigned long long t = z;
            t = (t ^ (t >> 30)) * 0xBF58476D1CE4E5B9ull;
            t = (t ^ (t >> 27)) * 0x94D049BB133111EBull;
            return t ^ (t >> 31);
        };
        const unsigned long long ra = next(), rb = next();
        // mantissa random, exponent in [-1000, 1000] biased, random sign
        const unsigned long long ea = 23 + (ra >> 53) % 2000;
        const double a = __longlong_as_double((long long)((ra & 0x800FFFFFFFFFFFFFull) | (ea << 52)));
        double b = bfix;
        if (bfix == 0.0) {
            const unsigned long long eb = 523 + (rb >> 53) % 1000;
            b = __longlong_as_double((long long)((rb & 0x000FFFFFFFFFFFFFull) | (eb << 52)));
        }
        const double yb = __drcp_rn(b);
        Div<false> dv;
        double r1 = dv(a, b, yb);
        if (dv.bad) r1 = a / b;  // the recompute path of the kernels
        const double r2 = a / b;
        if (__double_as_longlong(r1) != __double_as_longlong(r2)) ++cnt;
    }
    if (cnt) atomicAdd(bad, cnt);
}

int block_threads(const DevState& s) {
    const int t = ((s.nx * s.ny + 31) / 32) * 32;  // whole warps (shuffle reductions)
    return t > 256 ? 256 : t;
}
int geo_n(const DevState& s) {
    if (s.nx == s.ny && (s.nx == 8 || s.nx == 16)) return s.nx;
    return 0;
}

template <class K>
void smem_optin(K kernel, size_t bytes) {
    if (bytes > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// CTAs of a level-ordered launch: as many as can be resident at once (more
// would only wait for a slot and find the queue empty)
template <class K>
int queue_grid(K kernel, int nt, size_t smem, const LaunchCfg& lc) {
    int occ = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, nt, smem) != cudaSuccess ||
        occ < 1)
        occ = 1;
    return lc.num_sms * occ;
}

// shared memory of a C-fill launch: mbarriers, two C tiles
size_t fill_c_smem(const DevState& s) { return 128 + 2 * sizeof(double) * (size_t)s.cplane; }

template <int N, int CONS>
void fill_c_launch(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int width, int q) {
    const size_t sm = fill_c_smem(s);
    const int nt = block_threads(s);
    smem_optin(k_fill_c<N, CONS>, sm);
    k_fill_c<N, CONS><<<queue_grid(k_fill_c<N, CONS>, nt, sm, lc), nt, sm, st>>>(s, width, q);
}

template <int N>
void fill_c_dispatch(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int width,
                     int consumer, int q) {
    switch (consumer) {
        case CONS_NONE: fill_c_launch<N, CONS_NONE>(s, lc, st, width, q); break;
        case CONS_COLLIDE_READ: fill_c_launch<N, CONS_COLLIDE_READ>(s, lc, st, width, q); break;
        case CONS_COLLIDE_FUSED: fill_c_launch<N, CONS_COLLIDE_FUSED>(s, lc, st, width, q); break;
        default: fill_c_launch<N, CONS_MACRO_G>(s, lc, st, width, q); break;
    }
}

#define DISPATCH(s, CALL)      \
    switch (geo_n(s)) {        \
        case 8: CALL(8); break;  \
        case 16: CALL(16); break; \
        default: CALL(0); break; \
    }

}  // namespace

// ---------------------------------------------------------------------------
void launch_fill_c(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int width,
                   int consumer) {
    const int q = (width == 2) ? Q_FILLC : Q_FILLC1;
    cudaMemsetAsync(s.queue + 2 * q, 0, 2 * sizeof(unsigned), st);
    cudaMemsetAsync(s.ring_done + (size_t)q * (s.max_blks + 1), 0,
                    sizeof(int) * (size_t)(s.max_blks + 1), st);
#define F_(N)                                                      \
    if (width == 2)                                                \
        k_fill_flat<N, Q_FILLC><<<lc.num_sms * 8, 256, 0, st>>>(s);  \
    else                                                           \
        k_fill_flat<N, Q_FILLC1><<<lc.num_sms * 8, 256, 0, st>>>(s)
    DISPATCH(s, F_);
#undef F_
    count_launches(1);
#define C_(N) fill_c_dispatch<N>(s, lc, st, width, consumer, q)
    DISPATCH(s, C_);
#undef C_
    count_launches(1);
}

void launch_fill_hg_stream(const DevState& s, const LaunchCfg& lc, cudaStream_t st) {
    cudaMemsetAsync(s.queue + 2 * Q_FILLHG, 0, 2 * sizeof(unsigned), st);
    cudaMemsetAsync(s.ring_done + (size_t)Q_FILLHG * (s.max_blks + 1), 0,
                    sizeof(int) * (size_t)(s.max_blks + 1), st);
#define F_(N) k_fill_flat<N, Q_FILLHG><<<lc.num_sms * 8, 256, 0, st>>>(s)
    DISPATCH(s, F_);
#undef F_
    count_launches(1);
    const int nt = block_threads(s);
    const size_t sm = 128 + 18 * sizeof(double) * (size_t)s.aplane;  // mbarrier, h and g planes
#define C_(N)                                                                            \
    smem_optin(k_fill_hg_stream<N>, sm);                                                 \
    k_fill_hg_stream<N><<<queue_grid(k_fill_hg_stream<N>, nt, sm, lc), nt, sm, st>>>(s)
    DISPATCH(s, C_);
#undef C_
    count_launches(1);
}

void launch_build_plans(const DevState& s, const LaunchCfg& lc, cudaStream_t st) {
    cudaMemsetAsync(s.fillinfo, 0, 3 * NQUEUES * sizeof(int), st);
#define C_(N) k_build_plans<N><<<lc.grid_leaves, 128, 0, st>>>(s)
    DISPATCH(s, C_);
#undef C_
    count_launches(1);
}

void launch_collide(const DevState& s, const LaunchCfg& lc, cudaStream_t st) {
    const size_t sm = sizeof(double) * (size_t)s.cplane;
#define C_(N)                      \
    smem_optin(k_collide<N>, sm); \
    k_collide<N><<<lc.grid_leaves, block_threads(s), sm, st>>>(s)
    DISPATCH(s, C_);
#undef C_
    count_launches(1);
}

void launch_macro_h(const DevState& s, const LaunchCfg& lc, cudaStream_t st) {
#define C_(N) k_macro_h<N><<<lc.grid_leaves, block_threads(s), 0, st>>>(s)
    DISPATCH(s, C_);
#undef C_
    count_launches(1);
}

void launch_macro_g(const DevState& s, const LaunchCfg& lc, cudaStream_t st) {
    const size_t sm = sizeof(double) * (size_t)s.cplane;
#define C_(N)                      \
    smem_optin(k_macro_g<N>, sm); \
    k_macro_g<N><<<lc.grid_leaves, block_threads(s), sm, st>>>(s)
    DISPATCH(s, C_);
#undef C_
    count_launches(1);
}

void launch_err(const DevState& s, const LaunchCfg& lc, cudaStream_t st) {
#define C_(N) k_err<N><<<lc.grid_leaves, block_threads(s), 0, st>>>(s)
    DISPATCH(s, C_);
#undef C_
    count_launches(1);
}

int selftest_division(unsigned long long n, unsigned long long seed, double divisor,
                      unsigned long long* mismatches) {
    unsigned long long* d = nullptr;
    if (cudaMalloc(&d, sizeof(unsigned long long)) != cudaSuccess) return 2;
    cudaMemset(d, 0, sizeof(unsigned long long));
    k_selftest_div<<<1184, 256>>>(n, seed, divisor, d);
    count_launches(1);
    const cudaError_t e = cudaMemcpy(mismatches, d, sizeof(unsigned long long),
                                     cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : 2;
}
