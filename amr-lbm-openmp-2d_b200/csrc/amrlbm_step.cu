// amrlbm_step.cu - the per-step FP64 kernels (ghost fills fused with
// collision, streaming and macroscopic values). Compiled with -fmad=false:
// every operation the reference writes is rounded on its own and in its
// order; exact FMAs appear only inside div_rn (amrlbm_fast.cuh).
//
// Level-ordered launches. The reference fills ghost cells level by level
// (Fill_Ghost_Cells_C.f90:8-38): a coarse-to-fine fill reads the coarse
// neighbour's ghost ring, written one level earlier. One launch serves all
// levels here: CTAs claim leaves from a queue sorted by level; a leaf whose
// fill reads a coarser neighbour's ring waits (bounded spin) until that
// neighbour has published it (a per-block flag). A waited-on leaf has a lower
// level, so it was claimed earlier by a CTA that is running, and the wait
// always ends. After its fill a CTA goes on with the
// work that needs only its own ring (collision, streaming, macroscopic
// values): one launch does "fill + consumer", no grid-wide barrier.
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

// Claims the next item of queue q; returns its index (block-uniform).
__device__ __forceinline__ int claim(const DevState& s, int q, int* slot) {
    __syncthreads();
    if (threadIdx.x == 0) *slot = (int)atomicAdd(&s.queue[2 * q], 1u);
    __syncthreads();
    return *slot;
}

// direction (1..8) of ghost cell (x,y)
__device__ __forceinline__ int ghost_dir(int x, int y, int nx, int ny) {
    const bool xl = x < 1, xr = x > nx, yb = y < 1, yt = y > ny;
    if (xl) return yb ? 5 : (yt ? 6 : 1);
    if (xr) return yb ? 7 : (yt ? 8 : 2);
    return yb ? 3 : 4;
}

// per-direction neighbour data of the block being filled, loaded once into
// shared memory: resolved id, its level, leaf flag and first child
struct NbInfo {
    int id[9], lev[9], leaf[9], c1[9];
    int bi, bj;
};

// Loads the block's neighbour data (threads 0..9), then waits until every
// coarser neighbour has published its ring for queue q (bounded spin).
__device__ __forceinline__ void load_nb_and_wait(const DevState& s, int q, int n, int L,
                                                 bool do_fill, NbInfo& nbi) {
    const int t = threadIdx.x;
    if (t < 8) {
        const int b = s.nbr[8 * n + t];
        nbi.id[t + 1] = b;
        if (b > 0) {
            nbi.lev[t + 1] = s.level[b];
            nbi.leaf[t + 1] = s.is_leaf[b];
            nbi.c1[t + 1] = s.child[4 * b];
        } else {
            nbi.lev[t + 1] = -1;
            nbi.leaf[t + 1] = 0;
            nbi.c1[t + 1] = 0;
        }
    } else if (t == 8) {
        nbi.bi = s.bi[n];
    } else if (t == 9) {
        nbi.bj = s.bj[n];
    }
    __syncthreads();
    if (do_fill && t < 8) {
        const int b = nbi.id[t + 1];
        if (b > 0 && nbi.lev[t + 1] == L - 1) {
            const int* flag = s.ring_done + (size_t)q * (s.max_blks + 1) + b;
            int it = 0;
            while (ld_acquire_i(flag) == 0) {
                if (++it > kSpinLimit) {
                    set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, q);
                    break;
                }
                __nanosleep(32);
            }
        }
    }
    __syncthreads();
}

// Marks block n's ring of queue q as written (after a barrier of the CTA).
__device__ __forceinline__ void publish_ring(const DevState& s, int q, int n) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        st_release_i(s.ring_done + (size_t)q * (s.max_blks + 1) + n, 1);
    }
}

// ---------------------------------------------------------------------------
// Value of ghost cell (x,y) of block n (level L) from its direction-d
// neighbour N, for one field F(blk, x, y) (C, or one population of h or g).
// Returns 1 if computed, -1 on a level jump. The gathers and stencils follow
// Fill_Left_* .. Fill_Right_Top_* (Fill_Ghost_Cells_C.f90:44-416,
// Fill_Ghost_Cells_C2.f90:44-416, Fill_Ghost_Cells_hg.f90:53-477) case by case.
template <class FF>
__device__ __forceinline__ int ghost_value(const NbInfo& nbi, int nx, int ny, int L, int d, int x,
                                           int y, FF F, double& v) {
    const int N = nbi.id[d];
    const int Ln = nbi.lev[d];
    const bool left = (d == 1 || d == 5 || d == 6), right = (d == 2 || d == 7 || d == 8);
    const bool bottom = (d == 3 || d == 5 || d == 7), top = (d == 4 || d == 6 || d == 8);
    const int a = left ? 1 - x : (right ? x - nx : 0);  // layer counted outward
    const int b = bottom ? 1 - y : (top ? y - ny : 0);
    if (L == Ln) {
        if (nbi.leaf[d]) {  // same-level leaf: copy
            const int sx = left ? nx + 1 - a : (right ? a : x);
            const int sy = bottom ? ny + 1 - b : (top ? b : y);
            v = F(N, sx, sy);
            return 1;
        }
        const int c1 = nbi.c1[d];  // same-level parent: Biquadratic_from_Fine
        if (d == 1 || d == 2) {
            v = biq_fine_pt(a, y, [&](int r, int J) {
                const int ch = (J <= ny) ? (d == 1 ? c1 + 1 : c1) : (d == 1 ? c1 + 3 : c1 + 2);
                return F(ch, (d == 1) ? nx - r + 1 : r, (J <= ny) ? J : J - ny);
            });
        } else if (d == 3 || d == 4) {
            v = biq_fine_pt(x, b, [&](int I, int r) {
                const int ch = (I <= nx) ? (d == 3 ? c1 + 2 : c1) : (d == 3 ? c1 + 3 : c1 + 1);
                return F(ch, (I <= nx) ? I : I - nx, (d == 3) ? ny - r + 1 : r);
            });
        } else {
            const int ch = c1 + (d == 5 ? 3 : d == 6 ? 1 : d == 7 ? 2 : 0);
            v = biq_fine_pt(a, b, [&](int k, int l) {
                return F(ch, left ? nx - k + 1 : k, bottom ? ny - l + 1 : l);
            });
        }
        return 1;
    }
    if (L == Ln + 1) {  // coarser neighbour: Biquadratic_from_Coarse
        if (d == 1 || d == 2) {
            const int Y = (ny / 2) * (nbi.bj % 2);
            v = biq_coarse_pt(a, y, [&](int ii, int jj) {
                return F(N, (d == 1) ? nx + 2 - ii : ii - 1, jj - 1 + Y);
            });
        } else if (d == 3 || d == 4) {
            const int X = (nx / 2) * (nbi.bi % 2);
            v = biq_coarse_pt(x, b, [&](int ii, int jj) {
                return F(N, ii - 1 + X, (d == 3) ? ny + 2 - jj : jj - 1);
            });
        } else {
            const int mi = nbi.bi % 2, mj = nbi.bj % 2;
            const int I = left ? nx - (nx / 2) * mi - 1 : nx / 2 - (nx / 2) * mi;
            const int J = bottom ? ny - (ny / 2) * mj - 1 : ny / 2 - (ny / 2) * mj;
            v = biq_coarse_pt(a, b, [&](int ii, int jj) {
                return F(N, left ? I + 3 - ii : I + ii - 1, bottom ? J + 3 - jj : J + jj - 1);
            });
        }
        return 1;
    }
    return -1;
}

// Fills the C ring of width w of block n into memory and into T, the
// shared copy of the block's C in its pool layout (index G.c(0,x,y)).
// Symmetric_C(2)_3/4 (BC_Cell.f90:46-104) at walls.
template <int N>
__device__ void fill_c_block(const DevState& s, const Geo<N>& G, int n, int L, const NbInfo& nbi,
                             int w, double* T) {
    const int nx = G.nx, ny = G.ny;
    const int W = nx + 2 * w, H = ny + 2 * w;
    auto F = [&](int blk, int xx, int yy) { return ldcg(&s.C[G.c(blk, xx, yy)]); };
    for (int idx = threadIdx.x; idx < W * H; idx += blockDim.x) {
        const int x = idx % W - w + 1, y = idx / W - w + 1;
        if (x >= 1 && x <= nx && y >= 1 && y <= ny) continue;
        const int d = ghost_dir(x, y, nx, ny);
        if (nbi.id[d] <= 0) continue;
        double v;
        if (ghost_value(nbi, nx, ny, L, d, x, y, F, v) < 0) {
            set_error(s, 4 /*AMRLBM_ERR_LEVEL_JUMP*/, n);
            continue;
        }
        s.C[G.c(n, x, y)] = v;
        T[G.c(0, x, y)] = v;
    }
    __syncthreads();
    if (nbi.id[3] < 0) {
        for (int X = threadIdx.x + 1 - w; X <= nx + w; X += blockDim.x)
            for (int a = 1; a <= w; ++a) {  // C(X,1-a) = C(X,a)
                const double v = T[G.c(0, X, a)];
                T[G.c(0, X, 1 - a)] = v;
                s.C[G.c(n, X, 1 - a)] = v;
            }
    }
    if (nbi.id[4] < 0) {
        for (int X = threadIdx.x + 1 - w; X <= nx + w; X += blockDim.x)
            for (int a = 1; a <= w; ++a) {  // C(X,ny+a) = C(X,ny+1-a)
                const double v = T[G.c(0, X, ny + 1 - a)];
                T[G.c(0, X, ny + a)] = v;
                s.C[G.c(n, X, ny + a)] = v;
            }
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Collision_h_g_AMR (LBM_Subroutines.f90:116-189) of every cell of block n.
// T: shared C block (G.c(0,..)); Hs, Gs: shared post-streaming populations
// [q][y][x]; Ps: shared P, Ux, Uy (used unless FUSED). Writes the
// post-collision populations A to memory. FUSED: P, Ux, Uy come from
// Macroscopic_Values_g_AMR (:205-240) evaluated here on the same C ring.
template <int N, bool FUSED>
__device__ __forceinline__ void collide_block(const DevState& s, const Geo<N>& G, int n,
                                              const double* T, const double* Hs,
                                              const double* Gs, const double* Ps) {
    const PhysD& ph = s.ph;
    const int nx = G.nx, ny = G.ny, BP = G.bplane, PP = G.pplane;
    const double inv_dx = 1.0 / (double)s.dx[n];  // dx is a power of two: exact
    const double inv_dx2 = inv_dx * inv_dx;
    for (int c = threadIdx.x; c < nx * ny; c += blockDim.x) {
        const int x = c % nx + 1, y = c / nx + 1;
        auto Cs = [&](int a, int b) { return T[G.c(0, x + a, y + b)]; };
        const double c0 = Cs(0, 0);
        const double mu = chem_pot_f(ph, inv_dx2, Cs);
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
        gradient_ed_f(Ec, DcDx, DcDy);
        {  // normal_AMR (:25-37)
            const double t = sqrt(DcDx * DcDx + DcDy * DcDy + 1.e-32);
            const double rt = __drcp_rn(t);
            ni = div_rn(DcDx, t, rt);
            nj = div_rn(DcDy, t, rt);
        }
        const double Rho = ph.Rhol + c0 * ph.dRho;
        const double Fb = (ph.Rhoh - Rho) * ph.Gy;
        double P, Ux, Uy;
        if (FUSED) {
            double gx, gy;
            gradient_iso_f(inv_dx, Cs, gx, gy);
            const double Fx = mu * gx;
            const double Fy = mu * gy + Fb;
            auto g = [&](int k) { return Gs[(k - 1) * BP + c]; };
            const double sx = ((((g(2) - g(4)) + g(6)) - g(7)) - g(8)) + g(9);
            const double sy = ((((g(3) - g(5)) + g(6)) + g(7)) - g(8)) - g(9);
            const double rr = __drcp_rn(Rho);
            Ux = div_rn(3.0 * sx + 0.5 * Fx, Rho, rr);
            Uy = div_rn(3.0 * sy + 0.5 * Fy, Rho, rr);
            double sp = 0.0;
#pragma unroll
            for (int k = 1; k <= 9; ++k) sp = sp + g(k);
            P = sp + ph.dRho6 * (Ux * gx + Uy * gy);
        } else {
            P = Ps[c];
            Ux = Ps[PP + c];
            Uy = Ps[2 * PP + c];
        }
        // Equilibrium_h_g_AMR (:2-21) scalars
        const double tmp = div_rn(12.0 * (1.0 - c0), ph.W, ph.yW) * ph.M0;
        const double U215 = 1.5 * (Ux * Ux + Uy * Uy);
        const double ud_c = Ux * DcDx + Uy * DcDy;
        double DmX, DmY;
        gradient_ed_f(Em, DmX, DmY);
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
            s.Ah[G.a(n, k, x, y)] = Hs[(k - 1) * BP + c] * ph.omwc + heq * ph.wc;
            const double Ak = (Gm - wk) * ph.dRho3 + Gm * mu;
            const double Bk = ((double)d_ey(k) - Uy) * Gm * Fb;
            const double hc = Ak * (Ec(k) - ud_c) + Bk;
            const double geq = P * wk + div3((Gm - wk) * Rho) - 0.5 * hc;
            f[k] = Gs[(k - 1) * BP + c] - geq;
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
            s.Ag[G.a(n, k, x, y)] = (Gs[(k - 1) * BP + c] - div36(o[k])) + hm[k];
    }
}

// Macroscopic_Values_g_AMR (LBM_Subroutines.f90:205-240) + Err_Interface
// (Refine_Derefine.f90:327-351) of block n from T and the shared g planes Gs
template <int N>
__device__ void macro_g_err_block(const DevState& s, const Geo<N>& G, int n, const double* T,
                                  const double* Gs, double* red) {
    const PhysD& ph = s.ph;
    const int nx = G.nx, ny = G.ny, BP = G.bplane;
    const int dx = s.dx[n];
    const double inv_dx = 1.0 / (double)dx, inv_dx2 = inv_dx * inv_dx;
    double mx = 0.0;
    for (int c = threadIdx.x; c < nx * ny; c += blockDim.x) {
        const int x = c % nx + 1, y = c / nx + 1;
        auto Cs = [&](int a, int b) { return T[G.c(0, x + a, y + b)]; };
        auto g = [&](int k) { return Gs[(k - 1) * BP + c]; };
        double gx, gy;
        gradient_iso_f(inv_dx, Cs, gx, gy);
        const double mu = chem_pot_f(ph, inv_dx2, Cs);
        const double c0 = Cs(0, 0);
        const double Rho = ph.Rhol + c0 * ph.dRho;
        const double Fb = (ph.Rhoh - Rho) * ph.Gy;
        const double Fx = mu * gx;
        const double Fy = mu * gy + Fb;
        const double sx = ((((g(2) - g(4)) + g(6)) - g(7)) - g(8)) + g(9);
        const double sy = ((((g(3) - g(5)) + g(6)) + g(7)) - g(8)) - g(9);
        const double rr = __drcp_rn(Rho);
        const double Ux = div_rn(3.0 * sx + 0.5 * Fx, Rho, rr);
        const double Uy = div_rn(3.0 * sy + 0.5 * Fy, Rho, rr);
        double sp = 0.0;
#pragma unroll
        for (int k = 1; k <= 9; ++k) sp = sp + g(k);
        s.P[G.p(n, x, y)] = sp + ph.dRho6 * (Ux * gx + Uy * gy);
        s.Ux[G.p(n, x, y)] = Ux;
        s.Uy[G.p(n, x, y)] = Uy;
        const double a = Cs(1, 0) - Cs(-1, 0), b = Cs(0, 1) - Cs(0, -1);
        mx = fmax(mx, a * a + b * b);
    }
    // block max; fmax drops NaN as MAX(err, DC) never selects a NaN DC
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) m = fmax(m, red[w]);
        s.err[n] = sqrt(m) / (2.0 * dx);
    }
}

// shared-memory stage of the C-fill kernels (doubles after a 128-byte header
// holding the mbarrier): C block, h planes, g planes, P/Ux/Uy, reduction
template <int N>
struct StageC {
    double *T, *Hs, *Gs, *Ps, *red;
    __device__ __forceinline__ StageC(unsigned char* raw, const Geo<N>& G) {
        T = reinterpret_cast<double*>(raw + 128);
        Hs = T + G.cplane;
        Gs = Hs + 9 * G.bplane;
        Ps = Gs + 9 * G.bplane;
        red = Ps + 3 * G.pplane;
    }
};
size_t stage_c_bytes(const DevState& s) {
    return 128 + sizeof(double) * ((size_t)s.cplane + 18 * (size_t)s.bplane + 3 * (size_t)s.pplane + 32);
}

// Level-ordered C ghost fill (+ consumer). Items: all leaves grouped by
// level; leaves of levels outside [LevelMin, LevelMax] are not filled (as the
// reference's DO L = LevelMin, LevelMax) but still get the consumer work.
// At claim time one thread starts bulk copies of the block's C and of the
// fields the consumer reads into shared memory; they land while the CTA
// loads the neighbour data and waits for coarser neighbours.
template <int N, int CONSUMER>
__global__ void __launch_bounds__(256, 2) k_fill_c(DevState s, int w, int q) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const Geo<N> G(s);
    const int nx = G.nx, ny = G.ny;
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smraw);
    const StageC<N> st(smraw, G);
    __shared__ int s_item;
    __shared__ NbInfo nbi;
    constexpr bool need_h = (CONSUMER == CONS_COLLIDE_READ || CONSUMER == CONS_COLLIDE_FUSED);
    constexpr bool need_g = need_h || CONSUMER == CONS_MACRO_G;
    constexpr bool need_p = (CONSUMER == CONS_COLLIDE_READ);
    const unsigned cb = G.cplane * 8, pb = G.bplane * 72, ppb = G.pplane * 8;
    const unsigned bytes = cb + (need_h ? pb : 0) + (need_g ? pb : 0) + (need_p ? 3 * ppb : 0);
    const int lmin = s.cnt->level_min, lmax = s.cnt->level_max;
    const int total = s.lvl_off[AMR_MAXLV];
    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();
    if (need_h)
        if (blockIdx.x == 0 && threadIdx.x == 0)
            atomicAdd(&s.cnt->updates, (unsigned long long)total * (unsigned long long)(nx * ny));
    unsigned phase = 0;
    for (;;) {
        const int k = claim(s, q, &s_item);
        if (k >= total) break;
        const int n = s.lvl_leaf[k];
        if (threadIdx.x == 0) {
            fence_proxy_async();
            mbar_expect_tx(bar, bytes);
            bulk_g2s(st.T, s.C + (size_t)n * G.cplane, cb, bar);
            if (need_h) bulk_g2s(st.Hs, s.Bh + (size_t)n * 9 * G.bplane, pb, bar);
            if (need_g) bulk_g2s(st.Gs, s.Bg + (size_t)n * 9 * G.bplane, pb, bar);
            if (need_p) {
                bulk_g2s(st.Ps, s.P + (size_t)n * G.pplane, ppb, bar);
                bulk_g2s(st.Ps + G.pplane, s.Ux + (size_t)n * G.pplane, ppb, bar);
                bulk_g2s(st.Ps + 2 * G.pplane, s.Uy + (size_t)n * G.pplane, ppb, bar);
            }
        }
        const int L = s.level[n];
        const bool do_fill = (L >= lmin && L <= lmax);
        load_nb_and_wait(s, q, n, L, do_fill, nbi);
        if (__syncthreads_or(mbar_wait(bar, phase) ? 0 : 1)) {
            if (threadIdx.x == 0) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 100 + q);
            mbar_wait(bar, phase);  // the copies in flight must land before exit
            break;
        }
        phase ^= 1u;
        if (do_fill) fill_c_block<N>(s, G, n, L, nbi, w, st.T);
        publish_ring(s, q, n);
        if (CONSUMER != CONS_NONE) {
            __syncthreads();
            if (CONSUMER == CONS_MACRO_G)
                macro_g_err_block<N>(s, G, n, st.T, st.Gs, st.red);
            else
                collide_block<N, CONSUMER == CONS_COLLIDE_FUSED>(s, G, n, st.T, st.Hs, st.Gs,
                                                                 st.Ps);
        }
    }
}

// ---------------------------------------------------------------------------
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

size_t stage_hg_bytes(const DevState& s) { return 128 + sizeof(double) * 18 * (size_t)s.aplane; }

// Level-ordered Fill_Ghost_Cells_hg (Fill_Ghost_Cells_hg.f90:2-477),
// Bounce_Back_3/4 (BC_Cell.f90:2-42), streaming (Perfect_Shift_AMR /
// Streaming_LaxWendroff_AMR, LBM_Subroutines.f90:41-90) from A into B, and
// Macroscopic_Values_h_AMR (:193-201). The block's post-collision h and g
// planes are bulk-copied into shared memory at claim time; the fill writes
// the ghost ring into that copy, so streaming reads shared memory only. The
// ring goes to memory only when a finer neighbour reads it (its
// coarse-to-fine fill) or when write_all is set (state a caller downloads).
template <int N>
__global__ void __launch_bounds__(256, 3) k_fill_hg_stream(DevState s, int write_all) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const Geo<N> G(s);
    const int nx = G.nx, ny = G.ny;
    const int RG = 2 * (nx + ny) + 4;
    const int FP = 9 * G.aplane;  // doubles of one field's planes
    unsigned long long* bar = reinterpret_cast<unsigned long long*>(smraw);
    double* As = reinterpret_cast<double*>(smraw + 128);  // [h|g][q][pool plane layout]
    __shared__ int s_item;
    __shared__ NbInfo nbi;
    const int q = Q_FILLHG;
    const unsigned fb = (unsigned)FP * 8;
    const int lmin = s.cnt->level_min, lmax = s.cnt->level_max;
    const int total = s.lvl_off[AMR_MAXLV];
    if (threadIdx.x == 0) mbar_init(bar, 1);
    __syncthreads();
    unsigned phase = 0;
    for (;;) {
        const int k = claim(s, q, &s_item);
        if (k >= total) break;
        const int n = s.lvl_leaf[k];
        if (threadIdx.x == 0) {
            fence_proxy_async();
            mbar_expect_tx(bar, 2 * fb);
            bulk_g2s(As, s.Ah + (size_t)n * FP, fb, bar);
            bulk_g2s(As + FP, s.Ag + (size_t)n * FP, fb, bar);
        }
        const int L = s.level[n];
        const bool do_fill = (L >= lmin && L <= lmax);
        const bool wr = write_all || s.ring_out[n];
        load_nb_and_wait(s, q, n, L, do_fill, nbi);
        if (__syncthreads_or(mbar_wait(bar, phase) ? 0 : 1)) {
            if (threadIdx.x == 0) set_error(s, 8 /*AMRLBM_ERR_TIMEOUT*/, 100 + q);
            mbar_wait(bar, phase);
            break;
        }
        phase ^= 1u;
        if (do_fill) {
            for (int idx = threadIdx.x; idx < RG * 18; idx += blockDim.x) {
                const int r = idx % RG, qf = idx / RG;
                const int qq = qf % 9 + 1, f = qf / 9;
                int x, y;
                ring1_xy(r, nx, ny, x, y);
                const int d = ghost_dir(x, y, nx, ny);
                if (nbi.id[d] <= 0) continue;  // wall rows come next; else unchanged
                const double* A = f ? s.Ag : s.Ah;
                auto F = [&](int blk, int xx, int yy) { return ldcg(&A[G.a(blk, qq, xx, yy)]); };
                double v;
                if (ghost_value(nbi, nx, ny, L, d, x, y, F, v) < 0) {
                    set_error(s, 4, n);
                    continue;
                }
                As[f * FP + G.a(0, qq, x, y)] = v;
                if (wr) const_cast<double*>(A)[G.a(n, qq, x, y)] = v;
            }
            __syncthreads();
            // Bounce_Back_3/4: f(i,X,wall) = f(opposite(i), Xn, first row)
            for (int wall = 3; wall <= 4; ++wall) {
                if (nbi.id[wall] >= 0) continue;
                const int Y = (wall == 3) ? 0 : ny + 1, Yi = (wall == 3) ? 1 : ny;
                const int sgn = (wall == 3) ? 1 : -1;
                for (int idx = threadIdx.x; idx < (nx + 2) * 18; idx += blockDim.x) {
                    const int X = idx % (nx + 2), qf = idx / (nx + 2);
                    const int i = qf % 9 + 1, f = qf / 9;
                    int J = 1, Xn = X;
                    if (i > 1) {
                        Xn = min(max(0, X + sgn * d_ex(i) * d_ey(i)), nx + 1);
                        J = (i - 2) + 4 * ((i / 2) % 2);
                    }
                    const double v = As[f * FP + G.a(0, J, Xn, Yi)];
                    As[f * FP + G.a(0, i, X, Y)] = v;
                    if (wr) (f ? s.Ag : s.Ah)[G.a(n, i, X, Y)] = v;
                }
            }
        }
        publish_ring(s, q, n);
        __syncthreads();
        const double cfl = 1.0 / (double)s.dx[n];
        const bool shift = cfl > (double)0.9f;
        const double cA = cfl / 2.0 * (1.0 + cfl), cB = 1.0 - cfl * cfl,
                     cC = cfl / 2.0 * (1.0 - cfl);
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
                        v = cA * Af[G.a(0, i, x - d_ex(i), y - d_ey(i))] +
                            cB * Af[G.a(0, i, x, y)] -
                            cC * Af[G.a(0, i, x + d_ex(i), y + d_ey(i))];
                    }
                    B[G.bb(n, i, x, y)] = v;
                    if (f == 0) csum = csum + v;
                }
            }
            s.C[G.c(n, x, y)] = csum;
        }
    }
}

// ---------------------------------------------------------------------------
// grid-stride kernels over the leaf list (one CTA per block)

// grid-stride kernels over the leaf list (one CTA per block), shared stage
// filled by plain loads
template <int N>
__device__ __forceinline__ void load_stage(const DevState& s, const Geo<N>& G, int n,
                                           const StageC<N>& st, bool h, bool g, bool p) {
    for (int i = threadIdx.x; i < G.cplane; i += blockDim.x) st.T[i] = s.C[(size_t)n * G.cplane + i];
    for (int i = threadIdx.x; i < 9 * G.bplane; i += blockDim.x) {
        if (h) st.Hs[i] = s.Bh[(size_t)n * 9 * G.bplane + i];
        if (g) st.Gs[i] = s.Bg[(size_t)n * 9 * G.bplane + i];
    }
    if (p)
        for (int i = threadIdx.x; i < G.pplane; i += blockDim.x) {
            st.Ps[i] = s.P[(size_t)n * G.pplane + i];
            st.Ps[G.pplane + i] = s.Ux[(size_t)n * G.pplane + i];
            st.Ps[2 * G.pplane + i] = s.Uy[(size_t)n * G.pplane + i];
        }
    __syncthreads();
}

template <int N>
__global__ void __launch_bounds__(256, 2) k_collide(DevState s) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const Geo<N> G(s);
    const StageC<N> st(smraw, G);
    const int nleaf = s.cnt->nleaf;
    if (blockIdx.x == 0 && threadIdx.x == 0)
        atomicAdd(&s.cnt->updates, (unsigned long long)nleaf * (unsigned long long)(G.nx * G.ny));
    for (int m = blockIdx.x; m < nleaf; m += gridDim.x) {
        const int n = s.leaf[m];
        load_stage<N>(s, G, n, st, true, true, true);
        collide_block<N, false>(s, G, n, st.T, st.Hs, st.Gs, st.Ps);
        __syncthreads();
    }
}

template <int N>
__global__ void __launch_bounds__(256, 2) k_macro_g(DevState s) {
    extern __shared__ __align__(128) unsigned char smraw[];
    const Geo<N> G(s);
    const StageC<N> st(smraw, G);
    const int nleaf = s.cnt->nleaf;
    for (int m = blockIdx.x; m < nleaf; m += gridDim.x) {
        const int n = s.leaf[m];
        load_stage<N>(s, G, n, st, false, true, false);
        macro_g_err_block<N>(s, G, n, st.T, st.Gs, st.red);
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
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
        __syncthreads();
        if (threadIdx.x == 0) {
            double r = 0.0;
            for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) r = fmax(r, red[w]);
            s.err[n] = sqrt(r) / (2.0 * s.dx[n]);
        }
        __syncthreads();
    }
}

// div_rn against IEEE division: a from a spread of binades, b a fixed
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
        const double r1 = div_rn(a, b, yb), r2 = a / b;
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

template <int N>
void fill_c_dispatch(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int width,
                     int consumer, int q) {
    const size_t sm = stage_c_bytes(s);
    smem_optin(k_fill_c<N, CONS_NONE>, sm);
    smem_optin(k_fill_c<N, CONS_COLLIDE_READ>, sm);
    smem_optin(k_fill_c<N, CONS_COLLIDE_FUSED>, sm);
    smem_optin(k_fill_c<N, CONS_MACRO_G>, sm);
    const int nt = block_threads(s);
    switch (consumer) {
        case CONS_NONE: k_fill_c<N, CONS_NONE><<<lc.grid_queue, nt, sm, st>>>(s, width, q); break;
        case CONS_COLLIDE_READ:
            k_fill_c<N, CONS_COLLIDE_READ><<<lc.grid_queue, nt, sm, st>>>(s, width, q);
            break;
        case CONS_COLLIDE_FUSED:
            k_fill_c<N, CONS_COLLIDE_FUSED><<<lc.grid_queue, nt, sm, st>>>(s, width, q);
            break;
        default: k_fill_c<N, CONS_MACRO_G><<<lc.grid_queue, nt, sm, st>>>(s, width, q); break;
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
#define C_(N) fill_c_dispatch<N>(s, lc, st, width, consumer, q)
    DISPATCH(s, C_);
#undef C_
    count_launches(1);
}

void launch_fill_hg_stream(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int write_all) {
    cudaMemsetAsync(s.queue + 2 * Q_FILLHG, 0, 2 * sizeof(unsigned), st);
    cudaMemsetAsync(s.ring_done + (size_t)Q_FILLHG * (s.max_blks + 1), 0,
                    sizeof(int) * (size_t)(s.max_blks + 1), st);
    const size_t sm = stage_hg_bytes(s);
#define C_(N)                                 \
    smem_optin(k_fill_hg_stream<N>, sm);      \
    k_fill_hg_stream<N><<<lc.grid_queue, block_threads(s), sm, st>>>(s, write_all)
    DISPATCH(s, C_);
#undef C_
    count_launches(1);
}

void launch_collide(const DevState& s, const LaunchCfg& lc, cudaStream_t st) {
#define C_(N)                                \
    smem_optin(k_collide<N>, stage_c_bytes(s)); \
    k_collide<N><<<lc.grid_leaves, block_threads(s), stage_c_bytes(s), st>>>(s)
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
#define C_(N)                                \
    smem_optin(k_macro_g<N>, stage_c_bytes(s)); \
    k_macro_g<N><<<lc.grid_leaves, block_threads(s), stage_c_bytes(s), st>>>(s)
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
