// amrlbm_kernels.cu - FP64 sm_100a kernels of the block-structured AMR
// two-phase lattice Boltzmann path that run outside the time step: start-up
// fields, the regrid (flags, 2:1 balance, derefine with restriction, refine
// with neighbour pointers and prolongation, leaf lists) and diagnostics.
// Compiled with -fmad=false: every FP64 operation is rounded separately, in
// the reference's order. The per-step kernels are in amrlbm_step.cu.
//
#include <cstdio>

#include "amrlbm_launch.h"

namespace {

long long g_launches = 0;

__device__ __forceinline__ void load_tile(const DevState& s, int n, double* T) {
    const int nx = s.nx, ny = s.ny, W = nx + 4, H = ny + 4;
    for (int idx = threadIdx.x; idx < W * H; idx += blockDim.x)
        T[idx] = s.C[c_idx(s, n, idx % W - 1, idx / W - 1)];
    __syncthreads();
}

// ring 1 of a block: index r in [0, 2(nx+ny)+4) -> (x,y)
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

// Initialize_AMR_Rising_Bubble (AMR_Rising_2D_OMP.f90:186-226) given C
// hydro != 0: P also carries the light phase's hydrostatic head about the
// bubble centre y0, Gy*(Rhoh-Rhol)*(1-C)*(y-y0) (amrlbm_params.hydrostatic_start)
// p_given: P of every leaf was uploaded (several bubbles), not derived here
__global__ void __launch_bounds__(256) k_init_fields(DevState s, double R0, int hydro0, double Y00,
                                                     int p_given) {
    extern __shared__ double T[];
    const int nleaf = s.cnt->nleaf, nx = s.nx, ny = s.ny, TW = nx + 4;
    for (int m = blockIdx.x; m < nleaf; m += gridDim.x) {
        const int n = s.leaf[m];
        // the block's instance (batches) or the params' bubble
        const PhysD& ph = phys_any(s, n);
        const double* geo = s.n_inst ? s.inst_geo + 4 * s.inst[n] : nullptr;
        const double R = geo ? geo[0] : R0, Y0 = geo ? geo[2] : Y00;
        const int hydro = geo ? (geo[3] != 0.0) : hydro0;
        const double dRho3 = (ph.Rhoh - ph.Rhol) / 3.0;
        const int dx = s.dx[n];
        load_tile(s, n, T);
        for (int c = threadIdx.x; c < nx * ny; c += blockDim.x) {
            const int x = c % nx + 1, y = c / nx + 1;
            auto Cs = [&](int ddx, int ddy) { return T[(y + ddy + 1) * TW + (x + ddx + 1)]; };
            const double Cij = Cs(0, 0);
            const double Ux = 0, Uy = 0;
            double P = p_given ? s.P[p_idx(s, n, x, y)] : -ph.Sigma / R * Cij;
            if (hydro && !p_given) {
                const double Yc = (double)(s.bj[n] * dx * ny) + dx * (y - 0.5);
                P = P + ph.Gy * (ph.Rhoh - ph.Rhol) * (1.0 - Cij) * (Yc - Y0);
            }
            s.Ux[p_idx(s, n, x, y)] = Ux;
            s.Uy[p_idx(s, n, x, y)] = Uy;
            s.P[p_idx(s, n, x, y)] = P;
            const double mu = chem_pot(ph, dx, Cs);
            double E[10], Gamma[10], heq[10], DcDx, DcDy, ni, nj;
            ed_c(dx, Cs, E);
            gradient_ed(E, DcDx, DcDy);
            normal_vec(DcDx, DcDy, ni, nj);
            const double Rho = ph.Rhol + Cij * (ph.Rhoh - ph.Rhol);
            const double Fb = 0;
            equilibrium(ph, Cij, Ux, Uy, ni, nj, Gamma, heq);
            const double ud = Ux * DcDx + Uy * DcDy;
#pragma unroll
            for (int k = 1; k <= 9; ++k) {
                s.Bh[b_idx(s, n, k, x, y)] = heq[k];
                const double hlp = ((Gamma[k] - wa(k)) * dRho3 + Gamma[k] * mu) * (E[k] - ud) +
                                   ((double)d_ey(k) - Uy) * Gamma[k] * Fb;
                s.Bg[b_idx(s, n, k, x, y)] = P * wa(k) + (Gamma[k] - wa(k)) * Rho / 3.0 - 0.5 * hlp;
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// regrid (Refine_Derefine.f90): single-CTA topology passes + data kernels

// value of a neighbour pointer with the dangling check
__device__ __forceinline__ int resolve_chk(const DevState& s, int n, int k) {
    const int o = s.nb_owner[8 * n + k - 1];
    const int sl = s.nb_slot[8 * n + k - 1];
    if (sl == 0) return o;
    if (!s.child_alloc[o] || s.gen[o] != s.nb_gen[8 * n + k - 1]) set_error(s, 6, n);
    return s.child[4 * o + sl - 1];
}

// Block-wide exclusive scan of a 0/1 flag; returns the prefix, *total gets the sum.
__device__ int block_scan(int flag, int* total) {
    __shared__ int warp_sums[32];
    __shared__ int s_total;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned bal = __ballot_sync(0xffffffffu, flag);
    const int pre = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) warp_sums[wid] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        const int nw = (blockDim.x + 31) >> 5;
        for (int i = 0; i < nw; ++i) {
            const int t = warp_sums[i];
            warp_sums[i] = acc;
            acc += t;
        }
        s_total = acc;
    }
    __syncthreads();
    const int r = warp_sums[wid] + pre;
    *total = s_total;
    __syncthreads();
    return r;
}

// Stable compaction over ids 1..nb of pred(id) into out[base..] (out may be
// null: count only); returns count.
template <class Pred>
__device__ int compact(int nb, int* out, int base, Pred pred) {
    int count = 0;
    for (int start = 1; start <= nb; start += blockDim.x) {
        const int id = start + threadIdx.x;
        const int f = (id <= nb) ? (pred(id) ? 1 : 0) : 0;
        int tot;
        const int pos = block_scan(f, &tot);
        if (f && out) out[base + count + pos] = id;
        count += tot;
    }
    return count;
}

// Check_Level_Jump_Deref_2D (Refine_Derefine.f90:169-194)
__device__ __forceinline__ bool deref_ok(const DevState& s, int n, int dir, int c1, int c2) {
    const int b = resolve_chk(s, n, dir);
    if (b > 0 && !s.is_leaf[b]) {
        int c = s.child[4 * b + c1 - 1];
        for (int I = 1; I <= 2; ++I) {
            if (s.refin[c] || (!s.is_leaf[c] && !s.deref[c])) return false;
            c = s.child[4 * b + c2 - 1];
        }
    }
    return true;
}

// Flag_for_refinement + Enforce_1_Level_Jump (:18-93), Flag_for_derefinement
// + enforce_1_Level_jump_deref_2D (:97-165), and the list of blocks to
// derefine in ascending id order (Derefine, :198-211).
__global__ void __launch_bounds__(AMR_NTHREADS_TOPO) k_regrid_flags(DevState s, double refin_tol,
                                                                    double deref_tol) {
    const int nb = s.cnt->nblks;
    const int lmin = s.cnt->level_min, lmax = s.cnt->level_max;
    // levels that hold a block flagged for refinement / derefinement: the
    // closure passes of the other levels have nothing to do (each pass only
    // adds flags one level down, after the barrier that ends the pass before)
    __shared__ unsigned s_rmask, s_dmask, s_flagged;
    if (threadIdx.x == 0) s_rmask = s_dmask = s_flagged = 0u;
    __syncthreads();
    for (int n = 1 + threadIdx.x; n <= nb; n += blockDim.x) {
        uint8_t r = 0;
        if (s.is_leaf[n] && (!s.n_inst || s.inst_active[s.inst[n]])) {
            if (s.level[n] < s.min_levels) {
                r = 1;
            } else if (s.level[n] < maxlv_of(s, n) && s.err[n] > refin_tol) {
                r = 1;
                if (s.level[n] >= lmin && s.level[n] <= lmax) atomicAdd(&s_flagged, 1u);
            }
        }
        s.refin[n] = r;
        if (r) atomicOr(&s_rmask, 1u << s.level[n]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // statistics; with a forecaster it counts the flags itself
        s.cnt->rstat[0] += 1;
        if (!s.forecast) {
            s.cnt->rstat[2] += s_flagged;
            s.cnt->rstat[3] += s_flagged;
        }
    }
    // closure: a refining block's coarser (Level-1) leaf neighbours refine too;
    // processed from fine to coarse, every propagation goes one level down
    for (int L = s.max_levels; L >= 1; --L) {
        if (!((s_rmask >> L) & 1u)) continue;
        for (int n = 1 + threadIdx.x; n <= nb; n += blockDim.x) {
            if (s.level[n] != L || !s.refin[n]) continue;
            for (int I = 1; I <= 8; ++I) {
                const int b = resolve_chk(s, n, I);
                if (b > 0 && s.level[b] == L - 1 && s.is_leaf[b]) {
                    s.refin[b] = 1;
                    atomicOr(&s_rmask, 1u << (L - 1));
                }
            }
        }
        __syncthreads();
    }
    for (int n = 1 + threadIdx.x; n <= nb; n += blockDim.x) {
        uint8_t d = 0;
        if (s.has_leaf[n] && s.level[n] >= s.min_levels && (!s.n_inst || s.inst_active[s.inst[n]])) {
            const int c1 = s.child[4 * n];
            if (!(s.refin[c1] || s.refin[c1 + 1] || s.refin[c1 + 2] || s.refin[c1 + 3])) {
                d = 1;
                for (int c = c1; c <= c1 + 3; ++c)
                    if (s.err[c] > deref_tol) {
                        d = 0;
                        break;
                    }
            }
        }
        s.deref[n] = d;
        if (d) atomicOr(&s_dmask, 1u << s.level[n]);
    }
    __syncthreads();
    for (int L = lmax - 1; L >= lmin - 1; --L) {
        if (L < 0 || !((s_dmask >> L) & 1u)) continue;
        for (int n = 1 + threadIdx.x; n <= nb; n += blockDim.x) {
            if (s.level[n] != L || !s.deref[n]) continue;
            const bool ok = deref_ok(s, n, 1, 2, 4) && deref_ok(s, n, 2, 1, 3) &&
                            deref_ok(s, n, 3, 3, 4) && deref_ok(s, n, 4, 1, 2) &&
                            deref_ok(s, n, 5, 4, 4) && deref_ok(s, n, 6, 2, 2) &&
                            deref_ok(s, n, 7, 3, 3) && deref_ok(s, n, 8, 1, 1);
            if (!ok) s.deref[n] = 0;
        }
        __syncthreads();
    }
    const int nd = compact(nb, s.der_list, 0, [&](int id) { return s.deref[id] != 0; });
    // blocks the refinement of k_regrid_topo will take (levels lmin..lmax)
    const int nr = compact(nb, nullptr, 0, [&](int id) {
        return s.refin[id] != 0 && s.level[id] >= lmin && s.level[id] <= lmax;
    });
    if (threadIdx.x == 0) {
        s.cnt->n_der = nd;
        s.cnt->n_ref_flag = nr;
    }
}

// Restrict_Bilinear (Restrict.f90:14-65) for every block in der_list: the
// parent gets the 2x2 means of its children; ghost rings are zeroed.
__global__ void k_restrict(DevState s) {
    const int nd = s.cnt->n_der, nx = s.nx, ny = s.ny;
    for (int i = blockIdx.x; i < nd; i += gridDim.x) {
        const int par = s.der_list[i];
        const int c1 = s.child[4 * par];
        // zero C (all), P/U are written below, A rings
        for (int idx = threadIdx.x; idx < s.cplane; idx += blockDim.x)
            s.C[(size_t)par * s.cplane + idx] = 0.0;
        const int R = 2 * (nx + ny) + 4;
        for (int idx = threadIdx.x; idx < R * 18; idx += blockDim.x) {
            const int r = idx % R, qf = idx / R;
            int x, y;
            ring1_xy(r, nx, ny, x, y);
            double* A = (qf < 9) ? s.Ah : s.Ag;
            A[a_idx(s, par, qf % 9 + 1, x, y)] = 0.0;
        }
        __syncthreads();
        for (int c = threadIdx.x; c < nx * ny; c += blockDim.x) {
            const int x = c % nx + 1, y = c / nx + 1;
            // fine cell (X,Y) of the 2nx x 2ny assembly of the children
            auto F = [&](const double* base, int kind, int X, int Y, int q) {
                const int ch = c1 + (X > nx ? 1 : 0) + (Y > ny ? 2 : 0);
                const int xx = X > nx ? X - nx : X, yy = Y > ny ? Y - ny : Y;
                if (kind == 0) return base[b_idx(s, ch, q, xx, yy)];
                if (kind == 1) return base[c_idx(s, ch, xx, yy)];
                return base[p_idx(s, ch, xx, yy)];
            };
            auto bil = [&](const double* base, int kind, int q) {
                const double t0 = 0.5 * (F(base, kind, 2 * x - 1, 2 * y - 1, q) +
                                         F(base, kind, 2 * x - 1, 2 * y, q));
                const double t1 =
                    0.5 * (F(base, kind, 2 * x, 2 * y - 1, q) + F(base, kind, 2 * x, 2 * y, q));
                return 0.5 * (t0 + t1);
            };
            for (int q = 1; q <= 9; ++q) {
                s.Bh[b_idx(s, par, q, x, y)] = bil(s.Bh, 0, q);
                s.Bg[b_idx(s, par, q, x, y)] = bil(s.Bg, 0, q);
            }
            s.C[c_idx(s, par, x, y)] = bil(s.C, 1, 0);
            s.P[p_idx(s, par, x, y)] = bil(s.P, 2, 0);
            s.Ux[p_idx(s, par, x, y)] = bil(s.Ux, 2, 0);
            s.Uy[p_idx(s, par, x, y)] = bil(s.Uy, 2, 0);
        }
        __syncthreads();
    }
}

// Neighbor (Neighbors.f90:19-31)
__device__ void set_ptr(const DevState& s, int n, int k, int owner, int slot) {
    s.nb_owner[8 * n + k - 1] = owner;
    s.nb_slot[8 * n + k - 1] = slot;
    s.nb_gen[8 * n + k - 1] = slot ? s.gen[owner] : 0;
}
__device__ void copy_ptr(const DevState& s, int n, int k, int p) {
    s.nb_owner[8 * n + k - 1] = s.nb_owner[8 * p + k - 1];
    s.nb_slot[8 * n + k - 1] = s.nb_slot[8 * p + k - 1];
    s.nb_gen[8 * n + k - 1] = s.nb_gen[8 * p + k - 1];
}
__device__ void neighbor(const DevState& s, int p, int n, int n2, int c) {
    const int v = resolve_chk(s, p, n2);
    if (v < 0)
        copy_ptr(s, n, n2, p);
    else
        set_ptr(s, n, n2, v, c);
    const int n1 = n2 + 1 - 2 * ((n2 - 1) % 2);
    set_ptr(s, n, n1, p, c);
}
// through(k, slot): parent's pointer if negative, else child(slot) of it
__device__ void diag_through(const DevState& s, int p, int n, int k, int slot) {
    const int v = resolve_chk(s, p, k);
    if (v < 0)
        copy_ptr(s, n, k, p);
    else
        set_ptr(s, n, k, v, slot);
}
// fixed(kk, side, code, slot): the saved wall code if the side neighbour is external
__device__ void diag_fixed(const DevState& s, int p, int n, int kk, int side, int code, int slot) {
    const int v = resolve_chk(s, p, side);
    if (v < 0)
        set_ptr(s, n, kk, code, 0);
    else
        set_ptr(s, n, kk, v, slot);
}
// Find_Neighbors + Diagonal_Neighbor (Neighbors.f90:2-122)
__device__ void find_neighbors(const DevState& s, int par, int n, int I, int J) {
    const int c = 1 + I + 2 * J;
    neighbor(s, par, n, 1 + I, c + 1 - 2 * I);
    neighbor(s, par, n, 3 + J, c + 2 - 4 * J);
    if (c == 1) {
        diag_through(s, par, n, 5, 4);
        diag_fixed(s, par, n, 6, 1, -6, 4);
        diag_fixed(s, par, n, 7, 3, -7, 4);
        set_ptr(s, n, 8, par, 4);
    } else if (c == 2) {
        diag_fixed(s, par, n, 5, 3, -5, 3);
        set_ptr(s, n, 6, par, 3);
        diag_through(s, par, n, 7, 3);
        diag_fixed(s, par, n, 8, 2, -8, 3);
    } else if (c == 3) {
        diag_fixed(s, par, n, 5, 1, -5, 2);
        diag_through(s, par, n, 6, 2);
        set_ptr(s, n, 7, par, 2);
        diag_fixed(s, par, n, 8, 4, -8, 2);
    } else {
        set_ptr(s, n, 5, par, 1);
        diag_fixed(s, par, n, 6, 4, -6, 1);
        diag_fixed(s, par, n, 7, 2, -7, 1);
        diag_through(s, par, n, 8, 1);
    }
}

// Remove_Children (:215-258), Refine (:262-294) with Add_Child_Blocks
// (AMR_Rising_2D_OMP.f90:517-584), Array_of_Leaf_Blocks (:588-610) and the
// neighbour table of the new leaves.
__global__ void __launch_bounds__(AMR_NTHREADS_TOPO) k_regrid_topo(DevState s, int mode, int lmin_o,
                                                                   int lmax_o, int set_levels) {
    __shared__ int s_nr;
    Counters* cnt = s.cnt;
    const int nblks0 = cnt->nblks;
    const int lmin = lmin_o >= 0 ? lmin_o : cnt->level_min;
    const int lmax = lmax_o >= 0 ? lmax_o : cnt->level_max;
    if (mode == 0 && cnt->n_der == 0 && cnt->n_ref_flag == 0) {
        // nothing to refine or derefine: leaves, neighbours, work order and
        // fill plans stay as they are
        if (threadIdx.x == 0) {
            cnt->n_ref = 0;
            cnt->n_alloc_new = 0;
            cnt->topo_changed = 0;
            if (set_levels) {
                cnt->level_min = cnt->leaf_min;
                cnt->level_max = cnt->leaf_max;
            }
        }
        return;
    }
    if (mode != 2) {
        // ---- Derefine: Remove_Children for every listed parent (ascending ids)
        const int nd = (mode == 0) ? cnt->n_der : 0;
        const int head = cnt->fl_head, count = cnt->fl_count;
        for (int i = threadIdx.x; i < nd; i += blockDim.x) {
            const int par = s.der_list[i];
            const int c1 = s.child[4 * par];
            for (int c = c1; c <= c1 + 3; ++c) {
                s.level[c] = -1;
                s.is_leaf[c] = 0;
                s.alloc[c] = 0;
                s.child_alloc[c] = 0;
                s.gen[c] = s.gen[c] + 1;
            }
            for (int k = 0; k < 4; ++k) s.child[4 * par + k] = par;
            s.is_leaf[par] = 1;
            s.has_leaf[par] = 0;
            s.alloc[par] = 1;
            s.freelist[(head + count + i) % s.fl_cap] = c1;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nd; i += blockDim.x) {
            const int gp = s.parent[s.der_list[i]];
            if (gp > 0) {
                const int s1 = s.child[4 * gp], s4 = s.child[4 * gp + 3];
                bool all = true;
                for (int k = s1; k <= s4; ++k) all = all && s.is_leaf[k];
                if (all) s.has_leaf[gp] = 1;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            cnt->fl_count = count + nd;
            cnt->kk = cnt->kk + 4 * nd;
        }
        __syncthreads();
        // ---- Refine: blocks in (level ascending, id ascending) order
        int nr = 0;
        for (int L = lmin; L <= lmax; ++L)
            nr += compact(nblks0, s.ref_list, nr,
                          [&](int id) { return s.level[id] == L && s.refin[id] != 0; });
        const int F = cnt->fl_count, fh = cnt->fl_head;
        if (threadIdx.x == 0) {
            s_nr = nr;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < nr; k += blockDim.x) {
            const int c1 = (k < F) ? s.freelist[(fh + k) % s.fl_cap] : nblks0 + 1 + 4 * (k - F);
            if (c1 + 3 > s.max_blks) atomicMin(&s_nr, k);  // Add_Child_Blocks STOP
            s.ref_c1[k] = c1;
        }
        __syncthreads();
        if (s_nr < nr) {
            if (threadIdx.x == 0) set_error(s, 3 /*AMRLBM_ERR_POOL_FULL*/, s_nr);
            nr = s_nr;
        }
        const int used = nr < F ? nr : F;
        if (threadIdx.x == 0) {
            cnt->fl_head = (fh + used) % s.fl_cap;
            cnt->fl_count = F - used;
            cnt->kk = cnt->kk - 4 * used;
            cnt->nblks = nr > F ? nblks0 + 4 * (nr - F) : nblks0;
            cnt->n_ref = nr;
            cnt->n_alloc_new = nr > F ? nr - F : 0;
        }
        for (int L = lmin; L <= lmax; ++L) {
            for (int k = threadIdx.x; k < nr; k += blockDim.x) {
                const int par = s.ref_list[k];
                if (s.level[par] != L) continue;
                const int c1 = s.ref_c1[k];
                for (int i = 0; i < 4; ++i) s.child[4 * par + i] = c1 + i;
                s.is_leaf[par] = 0;
                s.has_leaf[par] = 1;
                const int gp = s.parent[par];
                if (gp > 0) s.has_leaf[gp] = 0;
                if (mode == 0) s.alloc[par] = 0;  // Prolong_Bilinear deallocates
                for (int J = 0; J <= 1; ++J)
                    for (int I = 0; I <= 1; ++I) {
                        const int N = c1 + I + 2 * J;
                        s.level[N] = L + 1;
                        s.dx[N] = s.dx[par] / 2;
                        if (s.n_inst) s.inst[N] = s.inst[par];
                        s.bi[N] = 2 * s.bi[par] + I;
                        s.bj[N] = 2 * s.bj[par] + J;
                        s.parent[N] = par;
                        for (int q = 0; q < 4; ++q) s.child[4 * N + q] = N;
                        s.child_alloc[N] = 1;
                        find_neighbors(s, par, N, I, J);
                        s.is_leaf[N] = 1;
                        s.has_leaf[N] = 0;
                        s.refin[N] = 0;
                        s.deref[N] = 0;
                        s.alloc[N] = 1;
                    }
            }
            __syncthreads();
        }
    }
    __syncthreads();
    // ---- Array_of_Leaf_Blocks, resolved neighbours, level range
    const int nb = cnt->nblks;
    const int nleaf = compact(nb, s.leaf, 0, [&](int id) { return s.is_leaf[id] != 0; });
    __shared__ int s_lo, s_hi;
    if (threadIdx.x == 0) {
        s_lo = 1 << 30;
        s_hi = -(1 << 30);
    }
    __syncthreads();
    for (int m = threadIdx.x; m < nleaf; m += blockDim.x) {
        const int n = s.leaf[m];
        for (int k = 1; k <= 8; ++k) s.nbr[8 * n + k - 1] = resolve_chk(s, n, k);
        s.ring_out[n] = 0;
        atomicMin(&s_lo, s.level[n]);
        atomicMax(&s_hi, s.level[n]);
    }
    __syncthreads();
    // leaves whose ghost rings (C and h/g) a finer neighbour's coarse-to-fine
    // fill reads: they publish their rings, their finer neighbours wait
    for (int m = threadIdx.x; m < nleaf; m += blockDim.x) {
        const int n = s.leaf[m];
        for (int k = 0; k < 8; ++k) {
            const int b = s.nbr[8 * n + k];
            if (b > 0 && s.level[b] == s.level[n] - 1) s.ring_out[b] = 1;
        }
    }
    __syncthreads();
    const int lo = s_lo, hi = s_hi;
    // work order of the level-ordered kernels: first the leaves others wait
    // on (by level), then the rest (by level); a waited-on leaf always comes
    // before its waiters
    int off = 0;
    for (int pass = 1; pass >= 0; --pass)
        for (int L = lo; L <= hi; ++L)
            off += compact(nleaf, s.lvl_leaf, off, [&](int m) {
                const int n = s.leaf[m - 1];
                return s.ring_out[n] == pass && s.level[n] == L;
            });
    // compact() stored positions 1..nleaf: turn them into block ids
    __syncthreads();
    for (int m = threadIdx.x; m < nleaf; m += blockDim.x) s.lvl_leaf[m] = s.leaf[s.lvl_leaf[m] - 1];
    if (threadIdx.x == 0) {
        cnt->topo_changed = 1;  // k_build_plans rebuilds the plans and fill flags
        for (int q = 0; q < NQUEUES; ++q) s.fillinfo[q] = 0;
        s.lvl_off[AMR_MAXLV] = nleaf;
        cnt->nleaf = nleaf;
        cnt->leaf_min = lo;
        cnt->leaf_max = hi;
        if (set_levels) {
            cnt->level_min = lo;
            cnt->level_max = hi;
        }
    }
}

// Prolong_Bilinear (Prolong.f90:12-39) + Fill_Children_Data (:105-130) for
// every refined block: children get bilinear h, g (with edge extrapolation)
// and C (ring 1 included), zero ghost rings, then Macroscopic_Values_g_AMR.
__global__ void __launch_bounds__(256) k_prolong(DevState s) {
    extern __shared__ double T[];
    const int nr = s.cnt->n_ref, nx = s.nx, ny = s.ny, TW = nx + 4;
    for (int i = blockIdx.x; i < nr; i += gridDim.x) {
        const int par = s.ref_list[i];
        const int c1 = s.ref_c1[i];
        for (int k = 0; k < 4; ++k) {
            const int ch = c1 + k;
            const int Ii = (k % 2) * nx, Jj = (k / 2) * ny;
            // h, g: Bilinear_Interpolate_Extrapolate (Prolong.f90:43-70)
            for (int c = threadIdx.x; c < nx * ny; c += blockDim.x) {
                const int x = c % nx + 1, y = c / nx + 1;
                const int xF = x + Ii, yF = y + Jj;
                const int Xx = max(1, min(nx - 1, xF / 2)), ax = 2 * xF - 4 * Xx + 1, bx = 4 - ax;
                const int Xy = max(1, min(ny - 1, yF / 2)), ay = 2 * yF - 4 * Xy + 1, by = 4 - ay;
                for (int f = 0; f < 2; ++f) {
                    const double* B = f ? s.Bg : s.Bh;
                    double* Bo = f ? s.Bg : s.Bh;
                    for (int q = 1; q <= 9; ++q) {
                        const double t0 = (double)bx * B[b_idx(s, par, q, Xx, Xy)] +
                                          (double)ax * B[b_idx(s, par, q, Xx + 1, Xy)];
                        const double t1 = (double)bx * B[b_idx(s, par, q, Xx, Xy + 1)] +
                                          (double)ax * B[b_idx(s, par, q, Xx + 1, Xy + 1)];
                        Bo[b_idx(s, ch, q, x, y)] = ((double)by * t0 + (double)ay * t1) / 16.0;
                    }
                }
            }
            // C: Bilinear_Interpolation (Prolong.f90:74-101) on 0..nx+1, zero ring 2
            const int W = nx + 4, H = ny + 4;
            for (int idx = threadIdx.x; idx < W * H; idx += blockDim.x) {
                const int x = idx % W - 1, y = idx / W - 1;
                double v = 0.0;
                if (x >= 0 && x <= nx + 1 && y >= 0 && y <= ny + 1) {
                    const int xF = x + Ii, yF = y + Jj;
                    const int Xx = xF / 2, ax = 2 * xF - 4 * Xx + 1, bx = 4 - ax;
                    const int Xy = yF / 2, ay = 2 * yF - 4 * Xy + 1, by = 4 - ay;
                    const double t0 = (double)bx * s.C[c_idx(s, par, Xx, Xy)] +
                                      (double)ax * s.C[c_idx(s, par, Xx + 1, Xy)];
                    const double t1 = (double)bx * s.C[c_idx(s, par, Xx, Xy + 1)] +
                                      (double)ax * s.C[c_idx(s, par, Xx + 1, Xy + 1)];
                    v = ((double)by * t0 + (double)ay * t1) / 16.0;
                }
                s.C[c_idx(s, ch, x, y)] = v;
                T[idx] = v;
            }
            const int R = 2 * (nx + ny) + 4;
            for (int idx = threadIdx.x; idx < R * 18; idx += blockDim.x) {
                const int r = idx % R, qf = idx / R;
                int x, y;
                ring1_xy(r, nx, ny, x, y);
                double* A = (qf < 9) ? s.Ah : s.Ag;
                A[a_idx(s, ch, qf % 9 + 1, x, y)] = 0.0;
            }
            __syncthreads();
            // Macroscopic_Values_g_AMR of the child
            const int dx = s.dx[ch];
            for (int c = threadIdx.x; c < nx * ny; c += blockDim.x) {
                const int x = c % nx + 1, y = c / nx + 1;
                auto Cs = [&](int ddx, int ddy) { return T[(y + ddy + 1) * TW + (x + ddx + 1)]; };
                double g[10];
                for (int q = 1; q <= 9; ++q) g[q] = s.Bg[b_idx(s, ch, q, x, y)];
                double P, Ux, Uy;
                macro_g_cell(phys_any(s, ch), dx, Cs, g, P, Ux, Uy);
                s.P[p_idx(s, ch, x, y)] = P;
                s.Ux[p_idx(s, ch, x, y)] = Ux;
                s.Uy[p_idx(s, ch, x, y)] = Uy;
            }
            __syncthreads();
        }
    }
}

// zeroed fields of the children created by Initial_Mesh (Add_Child_Blocks,
// AMR_Rising_2D_OMP.f90:572-577)
__global__ void k_zero_children(DevState s) {
    const int nr = s.cnt->n_ref;
    for (int i = blockIdx.x; i < nr; i += gridDim.x) {
        const int c1 = s.ref_c1[i];
        for (int k = 0; k < 4; ++k) {
            const int ch = c1 + k;
            for (size_t idx = threadIdx.x; idx < (size_t)9 * s.bplane; idx += blockDim.x) {
                s.Bh[(size_t)ch * 9 * s.bplane + idx] = 0.0;
                s.Bg[(size_t)ch * 9 * s.bplane + idx] = 0.0;
            }
            for (size_t idx = threadIdx.x; idx < (size_t)9 * s.aplane; idx += blockDim.x) {
                s.Ah[(size_t)ch * 9 * s.aplane + idx] = 0.0;
                s.Ag[(size_t)ch * 9 * s.aplane + idx] = 0.0;
            }
            for (int idx = threadIdx.x; idx < s.cplane; idx += blockDim.x)
                s.C[(size_t)ch * s.cplane + idx] = 0.0;
            for (int idx = threadIdx.x; idx < s.pplane; idx += blockDim.x) {
                s.P[(size_t)ch * s.pplane + idx] = 0.0;
                s.Ux[(size_t)ch * s.pplane + idx] = 0.0;
                s.Uy[(size_t)ch * s.pplane + idx] = 0.0;
            }
        }
    }
}

// Initial_Mesh: every leaf of `level` refines
__global__ void k_flag_level(DevState s, int level) {
    const int nb = s.cnt->nblks;
    for (int n = 1 + blockIdx.x * blockDim.x + threadIdx.x; n <= nb; n += gridDim.x * blockDim.x)
        s.refin[n] = (s.level[n] == level && s.is_leaf[n]) ? 1 : 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) s.cnt->n_der = 0;
}

// Determine_Min_Max_Levels (AMR_Rising_2D_OMP.f90:434-452)
__global__ void k_minmax(DevState s) {
    __shared__ int lo, hi;
    if (threadIdx.x == 0) {
        lo = 100;
        hi = -100;
    }
    __syncthreads();
    const int nleaf = s.cnt->nleaf;
    int l = 100, h = -100;
    for (int m = threadIdx.x; m < nleaf; m += blockDim.x) {
        const int L = s.level[s.leaf[m]];
        l = min(l, L);
        h = max(h, L);
    }
    atomicMin(&lo, l);
    atomicMax(&hi, h);
    __syncthreads();
    if (threadIdx.x == 0) {
        s.cnt->level_min = lo;
        s.cnt->level_max = hi;
    }
}

// Output (AMR_Rising_2D_OMP.f90:456-489) with a fixed summation order: per
// leaf block in (j,i) order, then over blocks in leaf-list order. out[8] =
// non-finite flag. part: 8 doubles per leaf (scratch, >= 8*nleaf).
// one CTA per leaf: the block's C and Uy staged in shared memory (coalesced),
// then thread 0 forms the block's sums in (j, i) order from there
__global__ void k_diag_blocks(DevState s, double* part) {
    extern __shared__ double sh[];  // [C | Uy] of one block, (j-1)*nx + (i-1)
    const int nleaf = s.cnt->nleaf, nx = s.nx, ny = s.ny, nc = nx * ny;
    for (int m = blockIdx.x; m < nleaf; m += gridDim.x) {
        const int n = s.leaf[m];
        for (int c = threadIdx.x; c < nc; c += blockDim.x) {
            const int i = c % nx + 1, j = c / nx + 1;
            sh[c] = s.C[c_idx(s, n, i, j)];
            sh[nc + c] = s.Uy[p_idx(s, n, i, j)];
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const int dx = s.dx[n];
            const double a = (double)(dx * dx);
            const PhysD& ph = phys_any(s, n);
            double mass = 0, rmin = 10, rmax = -10, umax = 0, vol = 0, ysum = 0, vsum = 0, phase = 0;
            bool finite = true;
            for (int j = 1; j <= ny; ++j)
                for (int i = 1; i <= nx; ++i) {
                    const double C = sh[(j - 1) * nx + (i - 1)];
                    const double Rho = ph.Rhol + C * (ph.Rhoh - ph.Rhol);
                    rmin = fmin(rmin, Rho);
                    rmax = fmax(rmax, Rho);
                    mass = mass + Rho * a;
                    const double uy = sh[nc + (j - 1) * nx + (i - 1)];
                    umax = fmax(umax, fabs(uy));
                    const double yc = (double)(s.bj[n] * dx * ny) + dx * (j - 0.5);
                    const double wgt = (C < 0.5) ? (1.0 - C) * a : 0.0;
                    vol = vol + wgt;
                    ysum = ysum + wgt * yc;
                    vsum = vsum + wgt * uy;
                    phase = phase + C * a;
                    if (!isfinite(C) || !isfinite(uy)) finite = false;
                }
            double* o = part + 9 * (size_t)m;
            o[0] = mass;
            o[1] = rmin;
            o[2] = rmax;
            o[3] = umax;
            o[4] = vol;
            o[5] = ysum;
            o[6] = vsum;
            o[7] = phase;
            o[8] = finite ? 0.0 : 1.0;
        }
        __syncthreads();
    }
}

// the per-block partials combined in leaf-list order: chunks of DIAG_CHUNK
// leaves staged in shared memory by all threads, thread k < 9 running
// quantity k's sum (or min / max) through them in order
#define DIAG_CHUNK 512
__global__ void k_diag_final(DevState s, const double* part, double* out) {
    __shared__ double sh[9 * DIAG_CHUNK];
    __shared__ double res[9];
    const int nleaf = s.cnt->nleaf, t = threadIdx.x;
    double acc = (t == 1) ? 10.0 : ((t == 2) ? -10.0 : 0.0);
    for (int base = 0; base < nleaf; base += DIAG_CHUNK) {
        const int cnt = min(DIAG_CHUNK, nleaf - base);
        for (int u = t; u < 9 * cnt; u += blockDim.x) sh[u] = part[9 * (size_t)base + u];
        __syncthreads();
        if (t < 9)
            for (int m = 0; m < cnt; ++m) {
                const double v = sh[9 * m + t];
                acc = (t == 1) ? fmin(acc, v) : ((t == 2 || t == 3) ? fmax(acc, v) : acc + v);
            }
        __syncthreads();
    }
    if (t < 9) res[t] = acc;
    __syncthreads();
    if (t == 0) {
        out[0] = res[0];
        out[1] = res[1];
        out[2] = res[2];
        out[3] = res[3];
        out[4] = res[4];
        out[5] = res[5] / res[4];
        out[6] = res[6] / res[4];
        out[7] = res[7];
        out[8] = res[8];
    }
}

// Samples of the refine-flag forecaster for blocks ids[0..n): per block 4
// channels on its (nx+2)^2 cells, ring 1 included ([i][channel][y][x]): C;
// log(1 + e/tol) with e the cell's Err_Interface term sqrt(dCx^2 + dCy^2)/(2dx)
// (Refine_Derefine.f90:327-351), so the refine criterion is e > tol; Ux and Uy
// times horizon/dx, the cells the flow moves over the horizon (0 on the ring).
// Needs C's ghost rings of the current state (between amrlbm_step calls).
__global__ void k_block_features(DevState s, int n, const int* ids, float horizon, double tol,
                                 float* out) {
    const int nx = s.nx, ny = s.ny, W = nx + 2, P = W * (ny + 2);
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const int b = ids[i];
        const double dx = (double)s.dx[b];
        float* o = out + (size_t)i * 4 * P;
        for (int c = threadIdx.x; c < P; c += blockDim.x) {
            const int x = c % W, y = c / W;
            const double gx = s.C[c_idx(s, b, x + 1, y)] - s.C[c_idx(s, b, x - 1, y)];
            const double gy = s.C[c_idx(s, b, x, y + 1)] - s.C[c_idx(s, b, x, y - 1)];
            o[c] = (float)s.C[c_idx(s, b, x, y)];
            o[P + c] = (float)log1p(sqrt(gx * gx + gy * gy) / (2.0 * dx) / tol);
            const bool in = x >= 1 && x <= nx && y >= 1 && y <= ny;
            o[2 * P + c] = in ? (float)(s.Ux[p_idx(s, b, x, y)] * horizon / dx) : 0.f;
            o[3 * P + c] = in ? (float)(s.Uy[p_idx(s, b, x, y)] * horizon / dx) : 0.f;
        }
    }
}

size_t tile_bytes(const DevState& s) { return (size_t)(s.nx + 4) * (s.ny + 4) * sizeof(double); }
int block_threads(const DevState& s) {
    const int t = ((s.nx * s.ny + 31) / 32) * 32;
    return t > 256 ? 256 : t;
}

}  // namespace

// ---------------------------------------------------------------------------
// launchers
long long launches_issued() { return g_launches; }
void count_launches(int n) { g_launches += n; }

void launch_reset_queues(const DevState& s, cudaStream_t st) {
    cudaMemsetAsync(s.queue, 0, sizeof(unsigned) * 4 * NQUEUES, st);
    cudaMemsetAsync(s.ring_done, 0, sizeof(int) * NQUEUES * (size_t)(s.max_blks + 1), st);
}







void launch_minmax(const DevState& s, cudaStream_t st) {
    k_minmax<<<1, 256, 0, st>>>(s);
    count_launches(1);
}

void launch_block_features(const DevState& s, cudaStream_t st, int n, const int* ids,
                           float horizon, double tol, float* out) {
    k_block_features<<<n < 4096 ? (n > 0 ? n : 1) : 4096, 128, 0, st>>>(s, n, ids, horizon, tol, out);
    count_launches(1);
}

void launch_init_fields(const DevState& s, const LaunchCfg& lc, cudaStream_t st, double radius,
                        int hydro, double y0, int p_given) {
    k_init_fields<<<lc.grid_leaves, block_threads(s), tile_bytes(s), st>>>(s, radius, hydro, y0, p_given);
    count_launches(1);
}

void launch_regrid_flags(const DevState& s, cudaStream_t st, double refin_tol, double deref_tol) {
    k_regrid_flags<<<1, AMR_NTHREADS_TOPO, 0, st>>>(s, refin_tol, deref_tol);
    count_launches(1);
}

void launch_restrict(const DevState& s, const LaunchCfg& lc, cudaStream_t st) {
    k_restrict<<<lc.grid_leaves, block_threads(s), 0, st>>>(s);
    count_launches(1);
}

void launch_regrid_topo(const DevState& s, cudaStream_t st, int mode, int lmin, int lmax,
                        int set_levels) {
    k_regrid_topo<<<1, AMR_NTHREADS_TOPO, 0, st>>>(s, mode, lmin, lmax, set_levels);
    count_launches(1);
}

void launch_prolong(const DevState& s, const LaunchCfg& lc, cudaStream_t st) {
    k_prolong<<<lc.grid_leaves, block_threads(s), tile_bytes(s), st>>>(s);
    count_launches(1);
}

void launch_zero_children(const DevState& s, const LaunchCfg& lc, cudaStream_t st) {
    k_zero_children<<<lc.grid_leaves, 256, 0, st>>>(s);
    count_launches(1);
}

void launch_flag_level(const DevState& s, cudaStream_t st, int level) {
    k_flag_level<<<64, 256, 0, st>>>(s, level);
    count_launches(1);
}

void launch_diag(const DevState& s, cudaStream_t st, double* out9) {
    // out9: device buffer of 9 + 9*max_blks doubles
    double* part = out9 + 9;
    k_diag_blocks<<<1184, 128, 2 * sizeof(double) * (size_t)s.nx * s.ny, st>>>(s, part);
    k_diag_final<<<1, 256, 0, st>>>(s, part, out9);
    count_launches(2);
}
