// amrlbm_step.cu - the per-step FP64 kernels (ghost fills fused with
// collision, streaming and macroscopic values). Compiled with -fmad=false:
// every operation the reference writes is rounded on its own and in its
// order; exact FMAs appear only inside the division of amrlbm_fast.cuh.
//
// Ghost fills without grid-wide level loops. The reference fills ghost cells
// level by level (Fill_Ghost_Cells_C.f90:8-38): a coarse-to-fine fill reads
// the coarse neighbour's ghost ring, written one level earlier. Here, after
// every topology change, each ghost cell of each leaf gets a fill plan (copy,
// fine-to-coarse or coarse-to-fine interpolation, with its source offsets);
// a coarser neighbour's ghost cell that a coarse-to-fine stencil reads and
// that is itself a copy or a fine-to-coarse value becomes a "foreign" cell of
// the reader, evaluated by the reader from interiors. Then every leaf's ring
// depends on interiors only (the usual case): each consumer item (collision,
// streaming or macroscopic values of one leaf) fills its own ring on its
// staged tile, applies the walls and consumes, with no ordering between
// leaves. Otherwise the consumer launch fills level by level first: CTAs
// claim leaves from a queue in which every leaf a finer neighbour reads
// precedes its readers, a leaf waits (bounded spin) for the flags of the
// coarser neighbours it reads, and no grid barrier is needed.
#include <cstddef>
#include <cstdio>

#include "amrlbm_fast.cuh"
#include "amrlbm_launch.h"
#include "amrlbm_plan.cuh"

void count_launches(int n);

namespace {


// direction (1..8) of ghost cell (x,y)
// ---------------------------------------------------------------------------
// Neighbour records and fill plans of every leaf, in work order (one CTA per
// leaf). The neighbour data is what Fill_Ghost_Cells_* reads through the
// block pointers (Fill_Ghost_Cells_C.f90:8-38): resolved neighbour ids, their
// levels, leaf flags and first children, plus the block's own id, level and
// ring_out flag.
//
// Coarse-to-fine cells read the coarser neighbour's ring, which the
// reference fills one level earlier. Where such a ring cell is a copy or a
// fine-to-coarse value, it becomes a foreign cell of the reading leaf: the
// leaf evaluates it from its plan, with the operations the neighbour's own
// fill uses, so the two leaves need not be ordered. Where it is itself
// coarse-to-fine or a wall cell, or a fill meets a level jump, the fill is
// marked as needing level order (fillinfo[q]), and the record's wait mask
// names the neighbours whose rings the leaf waits for then.
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
    for (int q = 0; q < NQUEUES; ++q) r.wait[q] = r.nf[q] = 0;
}

// One pass over the ghost cells of rings 1-2 serves all three fills: a cell's
// plan is the same in the C2, C1 and h/g fills (only the offsets differ, C
// pool or A pool), and a leaf's foreign cells are shared by the three.
template <int N>
__global__ void __launch_bounds__(128, 8) k_build_plans(DevState s) {
    const Geo<N> G(s);
    extern __shared__ int tab[];  // [9][ring1_len]: foreign cell -> slot
    __shared__ NbInfo nbi;
    __shared__ NbInfo cnb[9];     // coarser neighbours' records
    __shared__ int nfs;
    __shared__ int cls_n[2][4], cls_f[2][4];  // [C2 | ring-1 plans][class]: count, fill
    if (!s.cnt->topo_changed) return;  // the mesh did not change: the plans stand
    const int nx = G.nx, ny = G.ny, R2 = ring2_len(nx, ny), R1 = ring1_len(nx, ny);
    const int total = s.lvl_off[AMR_MAXLV];
    const int t = threadIdx.x, fmax = s.fmax;
    for (int k = blockIdx.x; k < total; k += gridDim.x) {
        const int n = s.lvl_leaf[k];
        if (t == 0) {
            load_nbinfo(s, n, nbi);
            nfs = 0;
        }
        if (t < 8) {
            cls_n[t / 4][t % 4] = 0;
            cls_f[t / 4][t % 4] = 0;
        }
        for (int i = t; i < 9 * R1; i += blockDim.x) tab[i] = -1;
        __syncthreads();
        const int L = nbi.lev[0];
        if (t >= 1 && t <= 8 && nbi.id[t] > 0 && nbi.lev[t] == L - 1) load_nbinfo(s, nbi.id[t], cnb[t]);
        __syncthreads();
        auto offc = [&](int blk, int xx, int yy) -> long long { return (long long)G.c(blk, xx, yy); };
        // ghost cell (xx,yy) of block blk, read from direction d: 1 a foreign
        // cell (the coarser neighbour's neighbour on that side has its level:
        // a copy or a fine-to-coarse value), -1 a coarser ring cell that is
        // not, 0 not a coarser neighbour's ghost cell
        auto foreign = [&](int d, int blk, int xx, int yy) {
            const bool ring = xx < 1 || xx > nx || yy < 1 || yy > ny;
            if (!ring || blk != nbi.id[d] || nbi.lev[d] != L - 1) return 0;
            const int dd = ghost_dir(xx, yy, nx, ny);
            return (nbi.leaf[d] && cnb[d].id[dd] > 0 && cnb[d].lev[dd] == L - 1) ? 1 : -1;
        };
        // 1: mark the foreign cells; anything else makes the fills wait
        for (int i = t; i < R2; i += blockDim.x) {
            int x, y;
            ring2_xy(i, nx, ny, x, y);
            const bool r1 = x >= 0 && x <= nx + 1 && y >= 0 && y <= ny + 1;
            const int d = ghost_dir(x, y, nx, ny);
            GPlan P;
            ghost_plan(nbi, nx, ny, L, d, x, y,
                       [&](int blk, int xx, int yy) -> long long {
                           const int f = foreign(d, blk, xx, yy);
                           if (f > 0) tab[d * R1 + ring1_index(xx, yy, nx, ny)] = -2;
                           if (f < 0) {
                               atomicOr(&nbi.wait[Q_FILLC], 1 << d);
                               if (r1) {
                                   atomicOr(&nbi.wait[Q_FILLC1], 1 << d);
                                   atomicOr(&nbi.wait[Q_FILLHG], 1 << d);
                               }
                           }
                           return 0;
                       },
                       P);
            // entries are stored by class: copies and level jumps,
            // fine-to-coarse cells, coarse-to-fine cells, cells without a plan
            const int cls = plan_class(P.kind);
            atomicAdd(&cls_n[0][cls], 1);
            if (r1) atomicAdd(&cls_n[1][cls], 1);
            if (P.kind < 0) {  // the level jump is reported by the level-ordered fills
                atomicOr(&s.fillinfo[Q_FILLC], 1);
                if (r1) {
                    atomicOr(&s.fillinfo[Q_FILLC1], 1);
                    atomicOr(&s.fillinfo[Q_FILLHG], 1);
                }
            }
        }
        __syncthreads();
        // 2: number the marked cells and write their records (C and A offsets)
        int* fc = s.frn_c + (size_t)k * fmax * FRN_INTS;
        int* fa = s.frn_hg + (size_t)k * fmax * FRN_INTS;
        for (int i = t; i < 9 * R1; i += blockDim.x) {
            if (tab[i] != -2) continue;
            const int j = atomicAdd(&nfs, 1);
            tab[i] = j;
            if (j >= fmax) {  // not reached: fmax bounds the cells a leaf reads
                set_error(s, 7 /*AMRLBM_ERR_STATE*/, n);
                continue;
            }
            const int d = i / R1;
            int xx, yy;
            ring1_xy(i % R1, nx, ny, xx, yy);
            long long aoff[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            int na = 0;
            GPlan sub;  // the coarser neighbour's plan of that ghost cell
            ghost_plan(cnb[d], nx, ny, L - 1, ghost_dir(xx, yy, nx, ny), xx, yy,
                       [&](int blk, int x2, int y2) -> long long {
                           aoff[na++ % 9] = (long long)G.a(blk, 1, x2, y2);
                           return offc(blk, x2, y2);
                       },
                       sub);
            plan_store(fc, fmax, j, sub);
            fc[10 * fmax + j] = (int)offc(nbi.id[d], xx, yy);
            for (int m = 0; m < 9; ++m) sub.src[m] = aoff[m];
            plan_store(fa, fmax, j, sub);
            fa[10 * fmax + j] = (int)G.a(nbi.id[d], 1, xx, yy);
        }
        __syncthreads();
        if (t < NQUEUES) {
            nbi.nf[t] = nfs;
            const int pt = (t == Q_FILLC) ? 0 : 1;
            nbi.na[t] = cls_n[pt][0];
            nbi.n2[t] = cls_n[pt][1];
            nbi.n3[t] = cls_n[pt][2];
            if (nbi.wait[t]) atomicOr(&s.fillinfo[t], 1);
        }
        // 3: the plans, foreign cells by slot
        for (int i = t; i < R2; i += blockDim.x) {
            int x, y;
            ring2_xy(i, nx, ny, x, y);
            const int d = ghost_dir(x, y, nx, ny);
            long long aoff[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            int na = 0;
            GPlan P;
            ghost_plan(nbi, nx, ny, L, d, x, y,
                       [&](int blk, int xx, int yy) -> long long {
                           long long w, wa;
                           if (foreign(d, blk, xx, yy) > 0) {
                               w = wa = (long long)(kIndirect |
                                                    (unsigned)tab[d * R1 + ring1_index(xx, yy, nx, ny)]);
                           } else {
                               w = offc(blk, xx, yy);
                               wa = (long long)G.a(blk, 1, xx, yy);
                           }
                           aoff[na++ % 9] = wa;
                           return w;
                       },
                       P);
            const int cls = plan_class(P.kind);
            auto slot = [&](int pt) {
                int base = 0;
                for (int m = 0; m < cls; ++m) base += cls_n[pt][m];
                return base + atomicAdd(&cls_f[pt][cls], 1);
            };
            plan_store(s.plan_c2 + (size_t)k * R2 * PLAN_INTS, R2, slot(0), P, i);
            if (x >= 0 && x <= nx + 1 && y >= 0 && y <= ny + 1) {
                const int i1 = ring1_index(x, y, nx, ny), e1 = slot(1);
                plan_store(s.plan_c1 + (size_t)k * R1 * PLAN_INTS, R1, e1, P, i1);
                for (int m = 0; m < 9; ++m) P.src[m] = aoff[m];
                plan_store(s.plan_hg + (size_t)k * R1 * PLAN_INTS, R1, e1, P, i1);
            }
        }
        __syncthreads();
        if (t < NBI_STRIDE)
            s.nbinfo[(size_t)k * NBI_STRIDE + t] = (t < NBI_INTS) ? reinterpret_cast<int*>(&nbi)[t] : 0;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Level-ordered launches, for fills that need level order: two phases in
// one launch. Fill phase: CTAs claim fill items (one leaf's ghost ring) in
// work order from queue[4q]. A fill item whose coarse-to-fine cells read a
// coarser neighbour's ring (other than its foreign cells) waits (bounded
// spin) for that neighbour's flag; every fill item raises its own block's
// flag when its ring, walls included, is in memory. Consumer phase: once the
// fill queue is empty, CTAs claim consumer items (the work that needs the
// block's own ring: collision, streaming, macroscopic values) from
// queue[4q+1]; a consumer item waits only for its own block's flag. Without
// level order there is no fill phase and consumer items fill their own rings.
//
// A CTA claims its next item as soon as it starts the current one (the
// atomic's latency hides behind the work). Progress: the smallest unfinished
// fill item is held by a running CTA, as its current item or as the next one
// of a CTA whose current item is smaller (hence finished), and waits only on
// smaller items; consumer items are claimed after every fill item was. So
// every wait ends.

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
    if (t == 0) *s_next = (int)atomicAdd(&s.queue[4 * q], 1u);
    __syncthreads();
    int k = *s_next;
    if (k < total && t < NBI_INTS)
        reinterpret_cast<int*>(&nbis[0])[t] = __ldg(s.nbinfo + (size_t)k * NBI_STRIDE + t);
    __syncthreads();
    int rb = 0;
    while (k < total) {
        const NbInfo& nbi = nbis[rb];
        unsigned kn = 0;
        if (t == 0) kn = atomicAdd(&s.queue[4 * q], 1u);  // the next item, claimed now
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
                            double* T, bool to_mem = true) {
    const int nx = G.nx, ny = G.ny;
    for (int idx = threadIdx.x; idx < (nx + 2 * w) * w * 2; idx += blockDim.x) {
        const int X = idx % (nx + 2 * w) + 1 - w, a = (idx / (nx + 2 * w)) % w + 1;
        const bool top = idx >= (nx + 2 * w) * w;
        if (top ? !w4 : !w3) continue;
        const int ys = top ? ny + 1 - a : a, yd = top ? ny + a : 1 - a;
        const double v = T ? T[G.c(0, X, ys)] : ldcg(s.C + G.c(n, X, ys));
        if (T) T[G.c(0, X, yd)] = v;
        if (to_mem) s.C[G.c(n, X, yd)] = v;
    }
}

// ---------------------------------------------------------------------------
// Ghost values from the plans. A fill item first evaluates its foreign cells
// into Fs (shared memory, Fs[plane * fmax + slot]), then its ghost cells.

// Whether fill q runs without level order: no leaf's fill waits for a
// coarser neighbour, no level jump, every leaf's level in [LevelMin,
// LevelMax]. Then every fill item depends on interiors only.
__device__ __forceinline__ bool fast_fill(const DevState& s, int q) {
    return s.fillinfo[q] == 0 && s.cnt->level_min <= s.cnt->leaf_min &&
           s.cnt->level_max >= s.cnt->leaf_max;
}

// Value of foreign cell j (records at fb) on the plane at qo of pool array A
// (C, or the first plane of Ah / Ag). live: the coarser neighbour is filled
// in this launch; if not, its ghost cell keeps the value in memory, as in the
// reference.
__device__ __forceinline__ double foreign_value(const int* fb, int fmax, int j, const double* A,
                                                size_t qo, bool live) {
    if (!live) return ldcg(A + (unsigned)fb[10 * fmax + j] + qo);
    const int meta = fb[j];
    if (plan_kind(meta) == 1) return __ldg(A + (unsigned)fb[fmax + j] + qo);
    double g[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) g[i] = __ldg(A + (unsigned)fb[(1 + i) * fmax + j] + qo);
    return plan_combine(meta, g);
}

// foreign cell records of item k of the C fills and of the h/g fill
__device__ __forceinline__ const int* frn_c_of(const DevState& s, int k) {
    return s.frn_c + (size_t)k * s.fmax * FRN_INTS;
}
__device__ __forceinline__ const int* frn_hg_of(const DevState& s, int k) {
    return s.frn_hg + (size_t)k * s.fmax * FRN_INTS;
}
// foreign cells of a C fill (records fb, in memory or shared memory) into
// Fs; ends with a barrier when there are any (nf is block-uniform)
template <int N>
__device__ void foreign_c(const DevState& s, const int* fb, int nf, bool live, double* Fs) {
    if (nf == 0) return;
    for (int j = threadIdx.x; j < nf; j += blockDim.x) Fs[j] = foreign_value(fb, s.fmax, j, s.C, 0, live);
    __syncthreads();
}
// the same for the h/g fill: one thread per (slot, field and population)
template <int N>
__device__ void foreign_hg(const DevState& s, const Geo<N>& G, const int* fb, int nf, bool live,
                           double* Fs) {
    if (nf == 0) return;
    for (int idx = threadIdx.x; idx < 18 * nf; idx += blockDim.x) {
        const int j = idx % nf, fq = idx / nf;
        Fs[fq * s.fmax + j] = foreign_value(fb, s.fmax, j, (fq >= 9) ? s.Ag : s.Ah,
                                            (size_t)(fq % 9) * G.aplane, live);
    }
    __syncthreads();
}

// a coarse-to-fine source: a foreign slot's value in Fs, or a cell in memory.
// cg (level order): the coarser neighbour's ring, written in this launch
// before a wait, so through L2. Without level order every source in memory
// is an interior cell that no item of the launch writes (the rings it could
// read are foreign cells), and the loads may go through L1.
__device__ __forceinline__ double c2f_source(unsigned w, const double* Fs, const double* A,
                                             size_t qo, bool cg) {
    return (w & kIndirect) ? Fs[w & ~kIndirect] : (cg ? ldcg(A + w + qo) : __ldg(A + w + qo));
}

// which plan kinds a fill pass evaluates: 0 all, 1 all but coarse-to-fine
// (before a wait), 2 coarse-to-fine only (after it)
__device__ __forceinline__ bool pass_takes(int mode, int kind) {
    return mode == 0 || ((kind == 3) == (mode == 2));
}

// One C ghost cell: plan entry e (plan words pl, in memory or shared memory;
// ring length R, width w) of
// block n, into memory (unless to_mem is false) and, if T is given, into the
// block's shared C tile (index G.c(0,x,y)). Kind 1 and 2 sources are
// interiors no launch of this fill writes; kind 3 sources are foreign slots
// (Fs) or cells in memory. Returns the kind.
template <int N>
__device__ __forceinline__ int c_entry(const DevState& s, const Geo<N>& G, const int* pl, int R,
                                       int e, int n, int w, const double* Fs, double* T,
                                       bool to_mem, bool cg) {
    const int meta = pl[e];
    const int kind = plan_kind(meta);
    if (kind == 0) return 0;
    int x, y;
    if (w == 2)
        ring2_xy(meta >> 8, G.nx, G.ny, x, y);
    else
        ring1_xy(meta >> 8, G.nx, G.ny, x, y);
    if (kind < 0) {
        set_error(s, 4 /*AMRLBM_ERR_LEVEL_JUMP*/, n);
        return kind;
    }
    double v;
    if (kind == 1) {
        v = __ldg(s.C + (unsigned)pl[R + e]);
    } else {
        double g[9];
        if (kind == 2) {
#pragma unroll
            for (int i = 0; i < 9; ++i) g[i] = __ldg(s.C + (unsigned)pl[(1 + i) * R + e]);
        } else {
#pragma unroll
            for (int i = 0; i < 9; ++i) g[i] = c2f_source((unsigned)pl[(1 + i) * R + e], Fs, s.C, 0, cg);
        }
        v = plan_combine(meta, g);
    }
    if (to_mem) s.C[G.c(n, x, y)] = v;
    if (T) T[G.c(0, x, y)] = v;
    return kind;
}

// C ghost ring of width w of item k (block n), level-ordered path, into
// memory: pass 0 all plan entries, 1 all but coarse-to-fine (before a
// wait), 2 coarse-to-fine only (after it). The foreign cells are in Fs.
template <int N>
__device__ void fill_ring_c(const DevState& s, const Geo<N>& G, int k, int n, int w, int mode,
                            const double* Fs) {
    const int R = (w == 2) ? ring2_len(G.nx, G.ny) : ring1_len(G.nx, G.ny);
    const int* pl = ((w == 2) ? s.plan_c2 : s.plan_c1) + (size_t)k * R * PLAN_INTS;
    for (int e = threadIdx.x; e < R; e += blockDim.x)
        if (pass_takes(mode, plan_kind(__ldg(pl + e))))
            c_entry<N>(s, G, pl, R, e, n, w, Fs, nullptr, true, true);
}

// One copied h/g ghost cell (plan entry e, field f): the 9 populations'
// loads in flight together.
template <int N>
__device__ __forceinline__ void hg_copy(const DevState& s, const Geo<N>& G, const int* pl, int RG,
                                        int e, int f, int n, double* As, bool to_mem) {
    const int meta = pl[e];
    int x, y;
    ring1_xy(meta >> 8, G.nx, G.ny, x, y);
    if (plan_kind(meta) < 0) {
        set_error(s, 4 /*AMRLBM_ERR_LEVEL_JUMP*/, n);
        return;
    }
    double* A = f ? s.Ag : s.Ah;
    const double* src = A + (unsigned)pl[RG + e];
    double v[9];
#pragma unroll
    for (int qq = 0; qq < 9; ++qq) v[qq] = __ldg(src + (size_t)qq * G.aplane);
#pragma unroll
    for (int qq = 0; qq < 9; ++qq) {
        if (to_mem) A[G.a(n, qq + 1, x, y)] = v[qq];
        if (As) As[f * 9 * G.aplane + G.a(0, qq + 1, x, y)] = v[qq];
    }
}
// One interpolated h/g ghost cell (plan entry e, population qq), both fields.
template <int N>
__device__ __forceinline__ void hg_interp(const DevState& s, const Geo<N>& G, const int* pl, int RG,
                                          int e, int qq, int n, const double* Fs, double* As,
                                          bool to_mem, bool cg) {
    const int meta = pl[e];
    const int kind = plan_kind(meta);
    int x, y;
    ring1_xy(meta >> 8, G.nx, G.ny, x, y);
    const size_t qo = (size_t)qq * G.aplane;
    unsigned wd[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) wd[i] = (unsigned)pl[(1 + i) * RG + e];
#pragma unroll
    for (int f = 0; f < 2; ++f) {
        double* A = f ? s.Ag : s.Ah;
        double g[9];
        if (kind == 2) {
#pragma unroll
            for (int i = 0; i < 9; ++i) g[i] = __ldg(A + wd[i] + qo);
        } else {
#pragma unroll
            for (int i = 0; i < 9; ++i) g[i] = c2f_source(wd[i], Fs + (f * 9 + qq) * s.fmax, A, qo, cg);
        }
        const double v = plan_combine(meta, g);
        if (to_mem) A[G.a(n, qq + 1, x, y)] = v;
        if (As) As[f * 9 * G.aplane + G.a(0, qq + 1, x, y)] = v;
    }
}

// h/g ghost ring of item k (block n), level-ordered path, into memory (pass
// as fill_ring_c). A cell without a plan keeps its value in memory.
template <int N>
__device__ void fill_ring_hg(const DevState& s, const Geo<N>& G, int k, int n, int mode,
                             const double* Fs) {
    const int RG = ring1_len(G.nx, G.ny);
    const int* pl = s.plan_hg + (size_t)k * RG * PLAN_INTS;
    if (mode != 2)
        for (int u = threadIdx.x; u < 2 * RG; u += blockDim.x) {
            const int kind = plan_kind(__ldg(pl + u % RG));
            if (kind == 1 || kind == -1) hg_copy<N>(s, G, pl, RG, u % RG, u / RG, n, nullptr, true);
        }
    for (int u = threadIdx.x; u < 9 * RG; u += blockDim.x) {
        const int kind = plan_kind(__ldg(pl + u % RG));
        if (kind >= 2 && pass_takes(mode, kind))
            hg_interp<N>(s, G, pl, RG, u % RG, u / RG, n, Fs, nullptr, true, true);
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
// T: shared C block (G.c(0,..)); Hb, Gb: the block's post-streaming h and g
// planes (plane stride nx*ny; staged in shared memory or in memory); unless
// FUSED, P, Ux, Uy are read from memory, where nothing writes them during the
// launch. Writes the post-collision populations A to memory. FUSED: P, Ux,
// Uy come from Macroscopic_Values_g_AMR (:205-240) evaluated here on the
// same C ring.
// BGK: the collision of g is BGK_Collision_AMR (LBM_Subroutines.f90:337-344,
// g*(1-s9) + geq*s9) instead of MRT_Collision_AMR, the alternative the
// reference leaves commented out at :180
template <bool SAFE, bool FUSED, bool SHH, bool SHG, int N, bool BGK = false, bool BATCH = false>
__device__ __forceinline__ unsigned collide_cell(const DevState& s, const Geo<N>& G, int n, int c,
                                                 double inv_dx, const double* T, const double* Hb,
                                                 const double* Gb) {
    const PhysD& ph = phys_of<BATCH>(s, n);
    const int nx = G.nx, BP = G.bplane, PP = G.pplane;
    const double inv_dx2 = inv_dx * inv_dx;
    const double* Hn = Hb + c;
    const double* Gn = Gb + c;
    auto ldh = [&](const double* p) { return SHH ? lds(p) : __ldg(p); };
    auto ldp = [&](const double* p) { return SHG ? lds(p) : __ldg(p); };
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
            auto g = [&](int k) { return ldp(Gn + (k - 1) * BP); };
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
            s.Ah[G.a(n, k, x, y)] = ldh(Hn + (k - 1) * BP) * ph.omwc + heq * ph.wc;
            const double Ak = (Gm - wk) * ph.dRho3 + Gm * mu;
            const double Bk = ((double)d_ey(k) - Uy) * Gm * Fb;
            const double hc = Ak * (Ec(k) - ud_c) + Bk;
            const double geq = P * wk + dv.d3((Gm - wk) * Rho) - 0.5 * hc;
            if (BGK)  // g(:)*(1.d0 - s9) + geq(:)*s9
                f[k] = ldp(Gn + (k - 1) * BP) * (1.0 - s9) + geq * s9;
            else
                f[k] = ldp(Gn + (k - 1) * BP) - geq;
            hm[k] = Ak * (Em(k) - ud_m) + Bk;
        }
        if (BGK) {
#pragma unroll
            for (int k = 1; k <= 9; ++k) s.Ag[G.a(n, k, x, y)] = f[k] + hm[k];
            return dv.bad;
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
            s.Ag[G.a(n, k, x, y)] = (ldp(Gn + (k - 1) * BP) - dv.d36(o[k])) + hm[k];
    }
    return dv.bad;
}


// Macroscopic_Values_g_AMR (LBM_Subroutines.f90:205-240) of cell c of block n
// from T and the block's g planes Gb (shared memory or memory); dc = the
// Err_Interface term (Refine_Derefine.f90:327-351) of the cell
template <bool SAFE, bool SH, int N, bool BATCH = false>
__device__ __forceinline__ unsigned macro_g_cell_f(const DevState& s, const Geo<N>& G, int n, int c,
                                                   double inv_dx, const double* T, const double* Gb,
                                                   double& dc) {
    const PhysD& ph = phys_of<BATCH>(s, n);
    const int nx = G.nx, BP = G.bplane;
    const double inv_dx2 = inv_dx * inv_dx;
    Div<SAFE> dv;
    const int x = c % nx + 1, y = c / nx + 1;
    auto Cs = [&](int a, int b) { return T[G.c(0, x + a, y + b)]; };
    const double* Gn = Gb + c;
    auto g = [&](int k) { return SH ? lds(Gn + (k - 1) * BP) : __ldg(Gn + (k - 1) * BP); };
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
// SHH, SHG: Hb, Gb point to shared memory (else to memory)
template <int N, bool FUSED, bool SHH, bool SHG, bool BGK = false, bool BATCH = false>
__device__ __forceinline__ void collide_block(const DevState& s, const Geo<N>& G, int n,
                                              const double* T, const double* Hb, const double* Gb) {
    const double inv_dx = 1.0 / (double)__ldg(s.dx + n);  // dx is a power of two: exact
    for (int c = threadIdx.x; c < G.nx * G.ny; c += blockDim.x)
        if (collide_cell<false, FUSED, SHH, SHG, N, BGK, BATCH>(s, G, n, c, inv_dx, T, Hb, Gb))
            collide_cell<true, FUSED, SHH, SHG, N, BGK, BATCH>(s, G, n, c, inv_dx, T, Hb, Gb);
}

// Macroscopic_Values_g_AMR of every cell of block n; returns this thread's
// maximum of the Err_Interface terms
template <int N, bool SH, bool BATCH = false>
__device__ __forceinline__ double macro_g_block(const DevState& s, const Geo<N>& G, int n,
                                                const double* T, const double* Gb) {
    const double inv_dx = 1.0 / (double)__ldg(s.dx + n);
    double mx = 0.0;
    for (int c = threadIdx.x; c < G.nx * G.ny; c += blockDim.x) {
        double dc;
        if (macro_g_cell_f<false, SH, N, BATCH>(s, G, n, c, inv_dx, T, Gb, dc))
            macro_g_cell_f<true, SH, N, BATCH>(s, G, n, c, inv_dx, T, Gb, dc);
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
                                   double* As, bool to_mem = true) {
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
        if (to_mem) (f ? s.Ag : s.Ah)[G.a(n, i, X, Y)] = v;
    }
}

// Streaming (Perfect_Shift_AMR / Streaming_LaxWendroff_AMR,
// LBM_Subroutines.f90:41-90) of every cell of block n into B, and
// Macroscopic_Values_h_AMR (:193-201), from As: the block's h and g planes
// (ring included) in shared memory, each field 9 planes in the pool layout.
// streaming coefficients of block n (dt/dx = 1/dx): Perfect_Shift_AMR where
// the Courant number exceeds 0.9, else Lax-Wendroff with cA, cB, cC
struct StreamCoef {
    double cA, cB, cC;
    bool shift;
    __device__ __forceinline__ StreamCoef(const DevState& s, int n) {
        const double cfl = 1.0 / (double)__ldg(s.dx + n);
        shift = cfl > (double)0.9f;
        cA = cfl / 2.0 * (1.0 + cfl);
        cB = 1.0 - cfl * cfl;
        cC = cfl / 2.0 * (1.0 - cfl);
    }
};
template <int N>
__device__ __forceinline__ void stream_cell(const DevState& s, const Geo<N>& G, int n, const double* As,
                                            const StreamCoef& k, int x, int y) {
    const int FP = 9 * G.aplane;
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
            } else if (k.shift) {
                v = Af[G.a(0, i, x - d_ex(i), y - d_ey(i))];
            } else {
                v = k.cA * Af[G.a(0, i, x - d_ex(i), y - d_ey(i))] + k.cB * Af[G.a(0, i, x, y)] -
                    k.cC * Af[G.a(0, i, x + d_ex(i), y + d_ey(i))];
            }
            B[G.bb(n, i, x, y)] = v;
            if (f == 0) csum = csum + v;
        }
    }
    s.C[G.c(n, x, y)] = csum;
}
template <int N>
__device__ void stream_block(const DevState& s, const Geo<N>& G, int n, const double* As) {
    const StreamCoef k(s, n);
    for (int c = threadIdx.x; c < G.nx * G.ny; c += blockDim.x)
        stream_cell<N>(s, G, n, As, k, c % G.nx + 1, c / G.nx + 1);
}
__host__ __device__ constexpr int fill_c_min_blocks(int consumer) {
    return (consumer == CONS_COLLIDE_READ || consumer == CONS_COLLIDE_FUSED) ? 2 : 3;
}

// Without level order: an item's C ring (block r.n; plan words pl, ring
// length R) on its tile T (if given) and in memory (if to_mem), its foreign
// cells in Fs already: one pass over
// the plan entries (stored by class: copies, fine-to-coarse, coarse-to-fine,
// so that a warp mostly takes one kind). Ends with a barrier.
template <int N>
__device__ void fast_ring_c(const DevState& s, const Geo<N>& G, const int* pl, int R, int w,
                            const ItemRec& r, const double* Fs, double* T, bool to_mem) {
    for (int e = threadIdx.x; e < r.na + r.n2 + r.n3; e += blockDim.x)
        c_entry<N>(s, G, pl, R, e, r.n, w, Fs, T, to_mem, false);
    __syncthreads();
}

// the same for the h/g ring on the staged planes As (if given): copies per
// field, interpolated cells per population (both fields)
template <int N>
__device__ void fast_ring_hg(const DevState& s, const Geo<N>& G, const int* pl, const ItemRec& r,
                             const double* Fs, double* As, bool to_mem) {
    const int RG = ring1_len(G.nx, G.ny);
    const int nC = 2 * r.na, nI = r.n2 + r.n3;
    for (int u = threadIdx.x; u < nC + 9 * nI; u += blockDim.x) {
        if (u < nC) {
            hg_copy<N>(s, G, pl, RG, u % r.na, u / r.na, r.n, As, to_mem);
        } else {
            const int v = u - nC;
            hg_interp<N>(s, G, pl, RG, r.na + v % nI, v / nI, r.n, Fs, As, to_mem, false);
        }
    }
    __syncthreads();
}

// C ghost fill of width w (Fill_Ghost_Cells_C.f90:2-416, Fill_Ghost_Cells_C2
// .f90:2-416) with Symmetric_C(2)_3/4 and its consumer, one item per leaf.
// Without level order (fast_fill) the items have no dependences: CTA b takes
// items b, b + gridDim.x, ..., bulk-copies the next item's C tile into the
// other of two shared stages while it consumes the current one, and fills
// each item's ring on its tile (and in memory if wr), applies the walls and
// consumes. With level order the fill phase fills every leaf first (leaves of
// levels outside [LevelMin, LevelMax] are not filled, as the reference's DO
// L = LevelMin, LevelMax, but still get the consumer work), and consumer
// items are claimed from a queue, their tile copy waiting for the block's flag.
// Shared memory: mbarriers (128 bytes), two stages (C tile and, for the
// consumer, the block's post-streaming h and / or g planes), the foreign
// values, and without level order each stage's plan words and foreign
// records (copied with the stage's tile).
__host__ __device__ constexpr bool stage_h(int consumer) {
    return consumer == CONS_COLLIDE_READ || consumer == CONS_COLLIDE_FUSED;
}
__host__ __device__ constexpr bool stage_g(int consumer) {
    return stage_h(consumer) || consumer == CONS_MACRO_G;
}
// doubles of one stage: C tile, h planes, g planes
__host__ __device__ inline size_t stage_doubles(int cplane, int bplane, int consumer) {
    return (size_t)cplane + (stage_h(consumer) ? 9 * (size_t)bplane : 0) +
           (stage_g(consumer) ? 9 * (size_t)bplane : 0);
}
// ints of one staged item's plan words (R entries) and foreign records; a
// multiple of 4 (16 bytes), as are both parts (R even, fmax a multiple of 4)
__host__ __device__ inline int plan_stage_ints(int R, int fmax) {
    return (PLAN_INTS * R + FRN_INTS * fmax + 3) & ~3;
}
// byte offset of a C fill's two staged plans: after the mbarriers, the two
// stages of SD doubles and the foreign values
__host__ __device__ inline size_t fill_c_plan_offset(size_t SD, int fmax) {
    return (128 + 8 * (2 * SD + (size_t)fmax) + 15) & ~(size_t)15;
}
template <int N, int CONSUMER, bool BGK, bool BATCH, bool FAST>
__device__ __forceinline__ void fill_c_body(const DevState& s, int w, int q, int wr) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const Geo<N> G(s);
    __shared__ NbInfo nbis[2];
    __shared__ double red[32];
    __shared__ int s_next;
    const int t = threadIdx.x;
    const int total = s.lvl_off[AMR_MAXLV];
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smraw);  // [2]
    double* tiles = reinterpret_cast<double*>(smraw + 128);
    const size_t SD = stage_doubles(G.cplane, G.bplane, CONSUMER);
    double* Fs = tiles + 2 * SD;
    const size_t HP = 9 * (size_t)G.bplane;  // doubles of 9 planes
    const bool fast = FAST;
    // without level order, stage st also holds its item's plan words and
    // foreign records (plans + st * PS)
    const int R = (w == 2) ? ring2_len(G.nx, G.ny) : ring1_len(G.nx, G.ny);
    const int PS = plan_stage_ints(R, s.fmax);
    int* plans = reinterpret_cast<int*>(smraw + fill_c_plan_offset(SD, s.fmax));
    const unsigned plb = (unsigned)(PLAN_INTS * R) * 4, frb = (unsigned)(FRN_INTS * s.fmax) * 4;
    constexpr bool collide = (CONSUMER == CONS_COLLIDE_READ || CONSUMER == CONS_COLLIDE_FUSED);
    if (collide && blockIdx.x == 0 && t == 0)
        atomicAdd(&s.cnt->updates, (unsigned long long)total * (unsigned long long)(G.nx * G.ny));
    // stage st: C tile at tiles + st*SD, then h planes (if staged), then g planes
    auto consume = [&](int n, const double* T) {
        const double* Hs = stage_h(CONSUMER) ? T + G.cplane : s.Bh + (size_t)n * HP;
        const double* Gs = stage_g(CONSUMER) ? T + G.cplane + (stage_h(CONSUMER) ? HP : 0)
                                             : s.Bg + (size_t)n * HP;
        if (CONSUMER == CONS_MACRO_G)
            err_reduce(s, n, macro_g_block<N, true, BATCH>(s, G, n, T, Gs), red);
        else if (CONSUMER != CONS_NONE)
            collide_block<N, CONSUMER == CONS_COLLIDE_FUSED, stage_h(CONSUMER), stage_g(CONSUMER), BGK,
                          BATCH>(s, G, n, T, Hs, Gs);
    };
    const unsigned tb = (unsigned)G.cplane * 8, hb = (unsigned)HP * 8;
    auto copy_tile = [&](int st, int nn, int c) {  // thread 0: item c, block nn
        double* T = tiles + st * SD;
        fence_proxy_async_all();
        mbar_expect_tx(&bar[st], tb + (stage_h(CONSUMER) ? hb : 0) + (stage_g(CONSUMER) ? hb : 0) +
                                     (fast ? plb + frb : 0));
        bulk_g2s(T, s.C + (size_t)nn * G.cplane, tb, &bar[st]);
        if (stage_h(CONSUMER)) bulk_g2s(T + G.cplane, s.Bh + (size_t)nn * HP, hb, &bar[st]);
        if (stage_g(CONSUMER))
            bulk_g2s(T + G.cplane + (stage_h(CONSUMER) ? HP : 0), s.Bg + (size_t)nn * HP, hb, &bar[st]);
        if (fast) {
            int* P = plans + st * PS;
            bulk_g2s(P, ((w == 2) ? s.plan_c2 : s.plan_c1) + (size_t)c * R * PLAN_INTS, plb, &bar[st]);
            bulk_g2s(P + PLAN_INTS * R, frn_c_of(s, c), frb, &bar[st]);
        }
    };

    const int lmin = s.cnt->level_min;
    if (!fast)
        fill_phase(
            s, q, nbis, &s_next,
            [&](int k, int n, const NbInfo& nbi) {
                foreign_c<N>(s, frn_c_of(s, k), nbi.nf[q], nbi.lev[0] - 1 >= lmin, Fs);
                if (nbi.wait[q]) {
                    fill_ring_c<N>(s, G, k, n, w, 1, Fs);
                    wait_coarse(s, q, nbi);
                    fill_ring_c<N>(s, G, k, n, w, 2, Fs);
                } else {
                    fill_ring_c<N>(s, G, k, n, w, 0, Fs);
                }
            },
            [&](int n, const NbInfo& nbi) { wall_c<N>(s, G, n, nbi, w); });
    // without level order: records of this and the next item (srec[st]: the
    // item of stage st)
    __shared__ int srec[2][REC_WORDS];
    if (CONSUMER == CONS_NONE) {  // Fill_Ghost_Cells_C(2) alone: without level order, the rings in memory
        if (fast)
            for (int c = blockIdx.x; c < total; c += gridDim.x) {
                item_rec_stage(s, c, q, srec[0]);
                __syncthreads();
                const ItemRec r = item_rec_of(srec[0]);
                foreign_c<N>(s, frn_c_of(s, c), r.nf, true, Fs);
                fast_ring_c<N>(s, G, ((w == 2) ? s.plan_c2 : s.plan_c1) + (size_t)c * R * PLAN_INTS,
                               R, w, r, Fs, nullptr, true);
                if (r.w3 || r.w4) wall_c_rows<N>(s, G, r.n, w, r.w3, r.w4, nullptr);
                __syncthreads();
            }
        else
            queue_done(s, q);
        return;
    }
    const int* flags = fill_flags(s, q);
    // thread 0: copy item c's C tile into stage st (with level order: once
    // its fill is done; without `block` only if it is done already; returns
    // whether the copy started)
    // (block nn; without level order the interior was written by the
    // previous launch)
    auto start_tile = [&](int st, int c, int nn, bool block) {
        if (fast) {
        } else if (block) {
            if (!spin_flag(flags + nn, s.spin_limit)) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 200 + q);
        } else if (ld_acquire_i(flags + nn) == 0) {
            return false;
        }
        copy_tile(st, nn, c);
        return true;
    };
    bool pend = false;  // thread 0: the next item's copy is still to start
    if (t == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        const int c0 = fast ? (int)blockIdx.x : (int)atomicAdd(&s.queue[4 * q + 1], 1u);
        s_next = c0;
        if (c0 < total) start_tile(0, c0, __ldg(s.lvl_leaf + c0), true);
    }
    if (fast && (int)blockIdx.x < total) item_rec_stage(s, blockIdx.x, q, srec[0]);
    __syncthreads();
    int c = s_next;
    unsigned phase = 0;  // bit st: parity of stage st's next completion
    int st = 0;
    while (c < total) {
        // the next item: the next of this CTA's share (without level order) or
        // the next in the queue, claimed now
        unsigned cn = c + gridDim.x;
        if (!fast && t == 0) cn = atomicAdd(&s.queue[4 * q + 1], 1u);
        int n;
        ItemRec r{};
        if (fast) {
            r = item_rec_of(srec[st]);
            n = r.n;
            if ((int)cn < total) item_rec_stage_async(s, cn, q, srec[st ^ 1]);  // for the next item
        } else {
            n = __ldg(s.lvl_leaf + c);
        }
        if (__syncthreads_or(mbar_wait(&bar[st], (phase >> st) & 1u) ? 0 : 1)) {
            if (t == 0) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 100 + q);
            mbar_wait(&bar[st], (phase >> st) & 1u);  // the copies must land before exit
            cp_async_wait_all();
            break;
        }
        phase ^= 1u << st;
        double* T = tiles + st * SD;
        if (fast) {  // the ring, then Symmetric_C(2)_3/4, on the tile (and in memory if wr)
            const int* P = plans + st * PS;
            foreign_c<N>(s, P + PLAN_INTS * R, r.nf, true, Fs);
            fast_ring_c<N>(s, G, P, R, w, r, Fs, T, wr != 0);
            if (r.w3 || r.w4) {
                wall_c_rows<N>(s, G, n, w, r.w3, r.w4, T, wr != 0);
                __syncthreads();
            }
        }
        if (t == 0) {
            s_next = (int)cn;
            int nn = 0;
            if ((int)cn < total) {
                if (fast) {
                    cp_async_wait_all();  // word 0 of the next record, copied by this thread
                    nn = srec[st ^ 1][0];
                } else {
                    nn = __ldg(s.lvl_leaf + cn);
                }
            }
            pend = ((int)cn < total) && !start_tile(st ^ 1, (int)cn, nn, false);
        }
        __syncwarp();  // warp 0 reconverges after thread 0's copies, before the consumer work
        consume(n, T);
        if (fast) cp_async_wait_all();  // the next item's record
        __syncthreads();
        c = s_next;
        st ^= 1;
        if (t == 0 && pend) start_tile(st, c, __ldg(s.lvl_leaf + c), true);
    }
    if (!fast) queue_done(s, q);
}
// The path without level order and the level-ordered one as two
// instantiations of the body, chosen once per launch, instead of one body
// with the two interleaved: the collision consumer's launch measured 6 %
// faster on the unordered path.
template <int N, int CONSUMER, bool BGK = false, bool BATCH = false>
__global__ void __launch_bounds__(256, fill_c_min_blocks(CONSUMER))
    k_fill_c(const __grid_constant__ DevState s, int w, int q, int wr) {
    if (fast_fill(s, q))
        fill_c_body<N, CONSUMER, BGK, BATCH, true>(s, w, q, wr);
    else
        fill_c_body<N, CONSUMER, BGK, BATCH, false>(s, w, q, wr);
}

// Fill_Ghost_Cells_hg (Fill_Ghost_Cells_hg.f90:2-477) with Bounce_Back_3/4,
// then streaming and Macroscopic_Values_h_AMR, one item per leaf. Each item
// bulk-copies its block's h and g planes into shared memory. Without level
// order (fast_fill) CTA b takes items b, b + gridDim.x, ..., fills each
// item's ring on the staged planes (and in memory if wr), applies the walls
// and streams; with level order the fill phase fills every leaf first and
// consumer items come from a queue, their copy waiting for the block's flag.
// Shared memory: mbarriers (128 bytes), h and g planes, the foreign values,
// and without level order one item's plan words and foreign records (copied
// once the previous item's ring is filled; a CTA's first item has its plan
// and planes copied at entry).

// byte offset of the h/g fill's staged plan: after the mbarriers, the
// h and g planes (FP doubles each) and the foreign values
__host__ __device__ inline size_t hg_plan_offset(size_t FP, int fmax) {
    return (128 + 8 * (2 * FP + 18 * (size_t)fmax) + 15) & ~(size_t)15;
}
template <int N, bool FAST>
__device__ __forceinline__ void fill_hg_stream_body(const DevState& s, int wr, int total, int first) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const Geo<N> G(s);
    __shared__ NbInfo nbis[2];
    __shared__ int s_next;
    const int q = Q_FILLHG;
    const int t = threadIdx.x;
    const int FP = 9 * G.aplane;
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smraw);
    double* As = reinterpret_cast<double*>(smraw + 128);  // [h|g][q][pool plane layout]
    double* Fs = As + 2 * (size_t)FP;
    const unsigned fb = (unsigned)FP * 8;
    auto copy_planes = [&](int nn) {  // thread 0
        fence_proxy_async_all();
        mbar_expect_tx(bar, 2 * fb);
        bulk_g2s(As, s.Ah + (size_t)nn * FP, fb, bar);
        bulk_g2s(As + FP, s.Ag + (size_t)nn * FP, fb, bar);
    };
    // without level order: plan words and foreign records of an item (Ps,
    // mbarrier bar[1]), copied once the previous item's ring is filled
    const int RG = ring1_len(G.nx, G.ny);
    int* Ps = reinterpret_cast<int*>(smraw + hg_plan_offset(FP, s.fmax));
    const unsigned plb = (unsigned)(PLAN_INTS * RG) * 4, frb = (unsigned)(FRN_INTS * s.fmax) * 4;
    auto copy_plan = [&](int c) {  // thread 0
        fence_proxy_async_all();
        mbar_expect_tx(&bar[1], plb + frb);
        bulk_g2s(Ps, s.plan_hg + (size_t)c * RG * PLAN_INTS, plb, &bar[1]);
        bulk_g2s(Ps + PLAN_INTS * RG, frn_hg_of(s, c), frb, &bar[1]);
    };
    const bool fast = FAST;
    if (t == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        // without level order the first item's plan and planes are copied at once
        if (fast && (int)blockIdx.x < total) {
            copy_plan(blockIdx.x);
            copy_planes(first);
        }
    }
    unsigned phase = 0;  // bit b: parity of bar[b]'s next completion

    if (fast) {
        __shared__ int srec[2][REC_WORDS];  // records of the current and the next item
        int c = blockIdx.x, rb = 0;
        if (c < total) item_rec_stage(s, c, q, srec[0]);
        __syncthreads();
        // bounded waits for the copies still in flight (bit b: bar[b]) before an exit
        auto drain = [&](unsigned bits) {
            for (int b = 0; b < 2; ++b)
                if ((bits >> b) & 1u) mbar_wait(&bar[b], (phase >> b) & 1u);
            cp_async_wait_all();
        };
        while (c < total) {
            const int cn = c + gridDim.x;
            const ItemRec r = item_rec_of(srec[rb]);
            if (t == 0 && c != (int)blockIdx.x) copy_planes(r.n);
            if (cn < total) item_rec_stage_async(s, cn, q, srec[rb ^ 1]);  // for the next iteration
            if (__syncthreads_or(mbar_wait(&bar[1], (phase >> 1) & 1u) ? 0 : 1)) {
                if (t == 0) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 100 + q);
                drain(3u);
                break;
            }
            phase ^= 2u;
            foreign_hg<N>(s, G, Ps + PLAN_INTS * RG, r.nf, true, Fs);  // while the planes land
            if (__syncthreads_or(mbar_wait(&bar[0], phase & 1u) ? 0 : 1)) {
                if (t == 0) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 100 + q);
                drain(1u);
                break;
            }
            phase ^= 1u;
            // the ring, then Bounce_Back_3/4, on the staged planes (and in memory if wr)
            fast_ring_hg<N>(s, G, Ps, r, Fs, As, wr != 0);
            if (t == 0 && cn < total) copy_plan(cn);  // the ring is filled: for the next iteration
            if (r.w3 || r.w4) {
                bounce_back_staged<N>(s, G, r.n, r.w3, r.w4, As, wr != 0);
                __syncthreads();
            }
            stream_block<N>(s, G, r.n, As);
            cp_async_wait_all();  // the next item's record
            __syncthreads();
            c = cn;
            rb ^= 1;
        }
        return;
    }

    __syncthreads();  // the mbarriers are initialised
    const int lmin = s.cnt->level_min;
    fill_phase(
        s, q, nbis, &s_next,
        [&](int k, int n, const NbInfo& nbi) {
            foreign_hg<N>(s, G, frn_hg_of(s, k), nbi.nf[q], nbi.lev[0] - 1 >= lmin, Fs);
            if (nbi.wait[q]) {
                fill_ring_hg<N>(s, G, k, n, 1, Fs);
                wait_coarse(s, q, nbi);
                fill_ring_hg<N>(s, G, k, n, 2, Fs);
            } else {
                fill_ring_hg<N>(s, G, k, n, 0, Fs);
            }
        },
        [&](int n, const NbInfo& nbi) { bounce_back<N>(s, G, n, nbi); });
    const int* flags = fill_flags(s, q);
    if (t == 0) s_next = (int)atomicAdd(&s.queue[4 * q + 1], 1u);
    __syncthreads();
    int c = s_next;
    while (c < total) {
        const int n = __ldg(s.lvl_leaf + c);
        if (t == 0) {
            const unsigned cn = atomicAdd(&s.queue[4 * q + 1], 1u);
            if (!spin_flag(flags + n, s.spin_limit)) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 200 + q);
            copy_planes(n);
            s_next = (int)cn;
        }
        if (__syncthreads_or(mbar_wait(bar, phase & 1u) ? 0 : 1)) {
            if (t == 0) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 100 + q);
            mbar_wait(bar, phase & 1u);
            break;
        }
        phase ^= 1u;
        stream_block<N>(s, G, n, As);
        c = s_next;
        __syncthreads();
    }
    queue_done(s, q);
}
// the unordered and the level-ordered path as two instantiations, as
// k_fill_c. The item count and the first item's block are loaded with the
// level-order flags, so that the first bulk copies wait for one round trip
// only (first: block of item blockIdx.x without level order)
template <int N>
__global__ void __launch_bounds__(256, 3) k_fill_hg_stream(DevState s, int wr) {
    const int total = s.lvl_off[AMR_MAXLV];
    const int first = (int)blockIdx.x <= s.max_blks ? __ldg(s.lvl_leaf + blockIdx.x) : 0;
    if (fast_fill(s, Q_FILLHG))
        fill_hg_stream_body<N, true>(s, wr, total, first);
    else
        fill_hg_stream_body<N, false>(s, wr, total, first);
}


// ---------------------------------------------------------------------------
// grid-stride kernels over the leaf list (one CTA per block), C tile staged
// by plain loads

template <int N>
__device__ __forceinline__ void load_tile_c(const DevState& s, const Geo<N>& G, int n, double* T) {
    for (int i = threadIdx.x; i < G.cplane; i += blockDim.x) T[i] = s.C[(size_t)n * G.cplane + i];
    __syncthreads();
}

template <int N, bool BGK = false, bool BATCH = false>
__global__ void __launch_bounds__(256, 2) k_collide(DevState s) {
    extern __shared__ __align__(16) double T[];
    const Geo<N> G(s);
    const int nleaf = s.cnt->nleaf;
    if (blockIdx.x == 0 && threadIdx.x == 0)
        atomicAdd(&s.cnt->updates, (unsigned long long)nleaf * (unsigned long long)(G.nx * G.ny));
    for (int m = blockIdx.x; m < nleaf; m += gridDim.x) {
        const int n = s.leaf[m];
        load_tile_c<N>(s, G, n, T);
        collide_block<N, false, false, false, BGK, BATCH>(s, G, n, T, s.Bh + (size_t)n * 9 * G.bplane,
                                                   s.Bg + (size_t)n * 9 * G.bplane);
        __syncthreads();
    }
}

template <int N, bool BATCH = false>
__global__ void __launch_bounds__(256, 2) k_macro_g(DevState s) {
    extern __shared__ __align__(16) double T[];
    __shared__ double red[32];
    const Geo<N> G(s);
    const int nleaf = s.cnt->nleaf;
    for (int m = blockIdx.x; m < nleaf; m += gridDim.x) {
        const int n = s.leaf[m];
        load_tile_c<N>(s, G, n, T);
        err_reduce(s, n, macro_g_block<N, false, BATCH>(s, G, n, T, s.Bg + (size_t)n * 9 * G.bplane), red);
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

// shared memory of a C-fill launch: mbarriers, two stages, foreign values
size_t fill_c_smem(const DevState& s, int consumer, int width) {
    const int R = (width == 2) ? ring2_len(s.nx, s.ny) : ring1_len(s.nx, s.ny);
    return fill_c_plan_offset(stage_doubles(s.cplane, s.bplane, consumer), s.fmax) +
           2 * sizeof(int) * (size_t)plan_stage_ints(R, s.fmax);
}

template <int N, int CONS, bool BGK = false, bool BATCH = false>
void fill_c_launch1(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int width, int q,
                    int wr) {
    const size_t sm = fill_c_smem(s, CONS, width);
    const int nt = block_threads(s);
    smem_optin(k_fill_c<N, CONS, BGK, BATCH>, sm);
    k_fill_c<N, CONS, BGK, BATCH><<<queue_grid(k_fill_c<N, CONS, BGK, BATCH>, nt, sm, lc), nt, sm,
                                    st>>>(s, width, q, wr);
}
// batched instances (per-instance physics) for the consumers that use it, on
// the 8x8 and 16x16 blocks that batches take
template <int N, int CONS, bool BGK = false>
void fill_c_launch(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int width, int q,
                   int wr) {
    if (N != 0 && CONS != CONS_NONE && s.n_inst)
        fill_c_launch1<N, CONS, BGK, (N != 0 && CONS != CONS_NONE)>(s, lc, st, width, q, wr);
    else
        fill_c_launch1<N, CONS, BGK, false>(s, lc, st, width, q, wr);
}

template <int N>
void fill_c_dispatch(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int width,
                     int consumer, int q, int wr) {
    switch (consumer) {
        case CONS_NONE: fill_c_launch<N, CONS_NONE>(s, lc, st, width, q, wr); break;
        case CONS_COLLIDE_READ:
            if (s.g_model == 1)
                fill_c_launch<N, CONS_COLLIDE_READ, true>(s, lc, st, width, q, wr);
            else
                fill_c_launch<N, CONS_COLLIDE_READ>(s, lc, st, width, q, wr);
            break;
        case CONS_COLLIDE_FUSED:
            if (s.g_model == 1)
                fill_c_launch<N, CONS_COLLIDE_FUSED, true>(s, lc, st, width, q, wr);
            else
                fill_c_launch<N, CONS_COLLIDE_FUSED>(s, lc, st, width, q, wr);
            break;
        default: fill_c_launch<N, CONS_MACRO_G>(s, lc, st, width, q, wr); break;
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
                   int consumer, int write_ring) {
    const int q = (width == 2) ? Q_FILLC : Q_FILLC1;
#define C_(N) fill_c_dispatch<N>(s, lc, st, width, consumer, q, write_ring)
    DISPATCH(s, C_);
#undef C_
    count_launches(1);
}

void launch_fill_hg_stream(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int write_ring) {
    const int nt = block_threads(s);
    // mbarriers, h and g planes, foreign values, the staged plan
    const size_t sm = hg_plan_offset(9 * (size_t)s.aplane, s.fmax) +
                      sizeof(int) * (size_t)plan_stage_ints(ring1_len(s.nx, s.ny), s.fmax);
#define C_(N)                                                                            \
    smem_optin(k_fill_hg_stream<N>, sm);                                                 \
    k_fill_hg_stream<N><<<queue_grid(k_fill_hg_stream<N>, nt, sm, lc), nt, sm, st>>>(s, write_ring)
    DISPATCH(s, C_);
#undef C_
    count_launches(1);
}

void launch_build_plans(const DevState& s, const LaunchCfg& lc, cudaStream_t st) {
#define C_(N) k_build_plans<N><<<lc.num_sms * 8, 128, 9 * sizeof(int) * ring1_len(s.nx, s.ny), st>>>(s)
    DISPATCH(s, C_);
#undef C_
    count_launches(1);
}

void launch_collide(const DevState& s, const LaunchCfg& lc, cudaStream_t st) {
    const size_t sm = sizeof(double) * (size_t)s.cplane;
#define C_(N)                      \
    smem_optin(k_collide<N>, sm); \
    smem_optin(k_collide<N, true>, sm); \
    smem_optin(k_collide<N, false, true>, sm); \
    smem_optin(k_collide<N, true, true>, sm); \
    if (s.g_model == 1 && s.n_inst) \
        k_collide<N, true, true><<<lc.grid_leaves, block_threads(s), sm, st>>>(s); \
    else if (s.g_model == 1) \
        k_collide<N, true><<<lc.grid_leaves, block_threads(s), sm, st>>>(s); \
    else if (s.n_inst) \
        k_collide<N, false, true><<<lc.grid_leaves, block_threads(s), sm, st>>>(s); \
    else \
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
    smem_optin(k_macro_g<N, true>, sm); \
    if (s.n_inst) \
        k_macro_g<N, true><<<lc.grid_leaves, block_threads(s), sm, st>>>(s); \
    else \
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

