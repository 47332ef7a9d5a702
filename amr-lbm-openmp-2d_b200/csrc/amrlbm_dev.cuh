// amrlbm_dev.cuh - device-side state, layouts and FP64 lattice Boltzmann
// arithmetic of the B200 path. Every formula follows the reference's
// LBM_Subroutines.f90 operation by operation (same association order, x**2
// as x*x). The translation units that include this file are compiled with
// -fmad=false, so no multiply-add is contracted and every FP64 result equals
// the reference's IEEE double evaluation on a CPU without FMA.
#pragma once

#include <cstdint>

#define AMR_MAXLV 24          // levels 0..AMR_MAXLV-1
#define AMR_NTHREADS_TOPO 1024

// ---------------------------------------------------------------------------
// physical constants (D2Q9_Mod.f90:10-16)
struct PhysD {
    double W, Sigma, Beta, kappa, taul, tauh, Rhol, Rhoh, Gy, M0, wc;
    // constant sub-expressions of the reference's formulas, evaluated once on
    // the host with the same operations (so the values are identical)
    double Beta4;        // 4.d0*Beta                      (LBM_Subroutines.f90:108)
    double omwc;         // 1.d0-wc                        (:146)
    double dRho;         // Rhoh - Rhol                    (:150)
    double dRho3;        // (Rhoh - Rhol)/3.d0             (:129)
    double dRho6;        // (Rhoh-Rhol)/6.d0               (:216)
    double itau_d;       // 1.d0/tauh - 1.d0/taul          (:174)
    double itaul;        // 1.d0/taul                      (:174)
    double taul5, tauh5; // taul + 0.5d0, tauh + 0.5d0     (:170-172)
    double yW;           // RN(1/W)
};

// device counters of the block pool (Parameters.f90:6-10, 41-45)
struct Counters {
    unsigned long long updates;                  // leaf-cell updates done by collisions
    int nblks, nleaf, kk, level_min, level_max;  // Nblks, nLeaf, KK, LevelMin, LevelMax
    int fl_head, fl_count;                       // FIFO free list (ring buffer)
    int error, error_info;                       // sticky AMRLBM_ERR_* and detail
    int leaf_min, leaf_max;                      // level range of the current leaves
    int n_ref, n_der;                            // blocks refined / derefined by the last regrid
    int n_alloc_new;                             // refinements that appended new ids
    int n_ref_flag;    // blocks of the level range flagged for refinement by k_regrid_flags
    int topo_changed;  // whether the last k_regrid_topo changed the mesh (plans rebuilt)
    // regrid statistics (amrlbm_regrid_stats): regrids, leaves forecast,
    // leaves the criterion flagged, flagged ones not forecast, forecast ones
    // not flagged
    unsigned long long rstat[5];
};

// Work queues of the level-ordered kernels (queue[4q..4q+2]: next fill item,
// next consumer item, CTAs done; zero between launches).
enum { Q_FILLC = 0, Q_FILLHG = 1, Q_FILLC1 = 2, NQUEUES = 3 };
// per-leaf records of the level-ordered kernels, indexed by work-order
// position: neighbour record (NBI_STRIDE ints) and one fill plan per ghost
// cell (PLAN_INTS ints: kind/weights word + 9 source offsets)
enum { NBI_STRIDE = 64, PLAN_INTS = 10 };

// ---------------------------------------------------------------------------
// The block pool. Block ids are 1..max_blks (slot 0 unused).
//   Bh, Bg : populations after streaming = the reference's Blk%h/g interior,
//            [blk][q][y][x], x,y = 1..nx,ny
//   Ah, Ag : populations after collision with their ghost ring, the
//            reference's Blk%h/g(:,0:nx+1,0:ny+1) between collision and
//            streaming, [blk][q][y][x], x,y = 0..nx+1,ny+1 (rows of nx+2:
//            with nx, ny even, rows and planes are 16-byte multiples)
//   C      : order parameter with both ghost rings, [blk][y+1][col],
//            col = x+3 (x = -1..nx+2), y = -1..ny+2
//   P,Ux,Uy: [blk][y][x], x,y = 1..nx,ny
// Physical constants of the mixed-precision kernels (FP32 copies of PhysD's)
struct PhysF {
    float W, iW, Beta4, kappa, M0, wc, omwc, Rhol, Rhoh, dRho, dRho3, dRho6, Gy;
    float itau_d, itaul, taul5, tauh5;
};

// Mixed-precision state (amrlbm_set_precision): the same element layouts as
// the FP64 pools, so the fill plans' source offsets index them unchanged.
// A population f_q of a cell is stored as its rest population f_1 in FP32
// (A1 / B1, one plane per block) and, for q = 2..9, the deviation
// (f_q - (w_q/w_1) f_1) * scale in 16 bits (Ad / Bd, the 9-plane layout of
// Ah / Bh, plane 1 unused); w_q/w_1 is 1/4 or 1/16, and the scales are powers
// of two, so encoding adds only the 16-bit rounding. C (with both ghost
// rings), P, Ux, Uy are FP32.
struct MpState {
    int fmt;                  // 0 off, 1 FP16, 2 BF16
    float sh, sg, ish, isg;   // deviation scales of h and g, and their inverses
    float *C, *P, *Ux, *Uy;
    float *A1h, *A1g, *B1h, *B1g;
    unsigned short *Adh, *Adg, *Bdh, *Bdg;
    PhysF ph;
    const PhysF* phys;  // batched instances: per instance (else ph)
};

// default bound of a flag wait of the level-ordered fills: iterations of
// about 64 ns, about a second in all
constexpr int AMR_SPIN_LIMIT = 20000000;

struct DevState {
    int nx, ny, max_blks, fl_cap;
    int ap, aplane;  // A row pitch and plane stride (doubles)
    int bplane;      // B plane stride = nx*ny
    int cp, cplane;  // C row pitch and block stride
    int pplane;      // P/Ux/Uy block stride
    int min_levels, max_levels;
    int g_model;     // collision of g: 0 MRT (the reference's), 1 BGK
    double *Ah, *Ag, *Bh, *Bg, *C, *P, *Ux, *Uy, *err;
    int *level, *dx, *bi, *bj, *parent, *child;  // child[4*id + k-1]
    int *nb_owner, *nb_slot, *nb_gen;            // [8*id + k-1] neighbour pointers
    int *gen;                                    // generation of each child array
    int *nbr;                                    // resolved neighbours [8*id + k-1]
    uint8_t *is_leaf, *has_leaf, *refin, *deref, *alloc, *child_alloc;
    uint8_t* ring_out;  // leaf whose h/g ghost ring a finer neighbour reads
    int* ring_done;     // [NQUEUES][max_blks+1]: ring written in the running fill
    int *leaf;       // LeafBlks, ascending
    int *lvl_leaf;   // work order of the level-ordered kernels (see k_regrid_topo)
    int *lvl_off;    // lvl_off[AMR_MAXLV] = number of entries of lvl_leaf
    int *nbinfo;     // [k][NBI_STRIDE] neighbour record of lvl_leaf[k]
    int *plan_c2, *plan_c1, *plan_hg;  // [k][PLAN_INTS][ring] fill plans of lvl_leaf[k]
    int *frn_c, *frn_hg;               // [k][11][fmax] foreign cells (C / A offsets)
    int fmax;                          // foreign cells per leaf and fill, at most
    int* fillinfo;                     // [q]: fill q needs level order
    int *freelist;   // ring buffer of the first ids of freed quartets
    int *ref_list, *ref_c1, *der_list;
    Counters* cnt;
    int forecast;  // a forecaster runs before each regrid of the time step (it keeps the statistics)
    unsigned* queue;  // [4*NQUEUES]: per queue fill claims, consumer claims, CTAs done
    int spin_limit;   // iterations of a flag wait of the level-ordered fills
    int hold_flag;    // test hook: this block's ring flag is never raised (0: none)
    PhysD ph;
    MpState mp;
    // batched instances (amrlbm_create_batch): disconnected quadtrees in one
    // pool, each with its own physics, bubble and number of levels; n_inst 0:
    // one mesh, the params' (ph, max_levels)
    int n_inst;
    int* inst;             // instance of each block id
    const PhysD* phys;     // per instance
    const int* inst_maxlv; // maxLevels per instance
    const double* inst_geo;  // per instance: radius, xc, yc, hydrostatic start (0/1)
    const unsigned char* inst_active;  // per instance: regrids flag its blocks (start-up rounds)
};

// physics of block n's instance; BATCH: a compile-time choice, so the
// one-mesh kernels keep reading the launch's constant parameter
template <bool BATCH>
__device__ __forceinline__ const PhysD& phys_of(const DevState& s, int n) {
    if (BATCH) return s.phys[s.inst[n]];
    return s.ph;
}
__device__ __forceinline__ const PhysD& phys_any(const DevState& s, int n) {
    return s.n_inst ? s.phys[s.inst[n]] : s.ph;
}
__device__ __forceinline__ int maxlv_of(const DevState& s, int n) {
    return s.n_inst ? s.inst_maxlv[s.inst[n]] : s.max_levels;
}

// ---------------------------------------------------------------------------
// indexing
__device__ __forceinline__ size_t a_idx(const DevState& s, int b, int q, int x, int y) {
    return ((size_t)b * 9 + (q - 1)) * s.aplane + (size_t)y * s.ap + x;
}
__device__ __forceinline__ size_t b_idx(const DevState& s, int b, int q, int x, int y) {
    return ((size_t)b * 9 + (q - 1)) * s.bplane + (size_t)(y - 1) * s.nx + (x - 1);
}
__device__ __forceinline__ size_t c_idx(const DevState& s, int b, int x, int y) {
    return (size_t)b * s.cplane + (size_t)(y + 1) * s.cp + (x + 3);
}
__device__ __forceinline__ size_t p_idx(const DevState& s, int b, int x, int y) {
    return (size_t)b * s.pplane + (size_t)(y - 1) * s.nx + (x - 1);
}

// D2Q9 lattice (D2Q9_Mod.f90:6-8), 1-based:
// ex = [0,1,0,-1,0,1,-1,-1,1], ey = [0,0,1,0,-1,1,1,-1,-1]. Functions, not a
// __constant__ table, so that loops unrolled over k fold them into immediate
// offsets and constants.
__host__ __device__ __forceinline__ constexpr int cex(int k) {
    return (k == 2 || k == 6 || k == 9) ? 1 : ((k == 4 || k == 7 || k == 8) ? -1 : 0);
}
__host__ __device__ __forceinline__ constexpr int cey(int k) {
    return (k == 3 || k == 6 || k == 7) ? 1 : ((k == 5 || k == 8 || k == 9) ? -1 : 0);
}
#define d_ex(k) cex(k)
#define d_ey(k) cey(k)

__device__ __forceinline__ double wa(int i) {
    // [16,4,4,4,4,1,1,1,1]/36.d0, correctly rounded like the Fortran constant
    return i == 1 ? 16.0 / 36.0 : (i <= 5 ? 4.0 / 36.0 : 1.0 / 36.0);
}

// load bypassing L1: data written by other CTAs of the same kernel
__device__ __forceinline__ double ldcg(const double* p) { return __ldcg(p); }

// ---------------------------------------------------------------------------
// LBM_Subroutines.f90 arithmetic, per cell. Cs(dx, dy) returns C at the cell
// offset (dx, dy) from the current cell.

// Laplacian_AMR (:316-333) and Chemical_Potential_AMR (:94-112) at one cell
template <class CF>
__device__ __forceinline__ double chem_pot(const PhysD& ph, int dx, CF Cs) {
    const double D2C =
        (Cs(-1, -1) + Cs(1, -1) + Cs(-1, 1) + Cs(1, 1) +
         4.0 * (Cs(0, -1) + Cs(-1, 0) + Cs(1, 0) + Cs(0, 1)) - 20.0 * Cs(0, 0)) /
        6.0;
    const double c = Cs(0, 0);
    return 4.0 * ph.Beta * c * (c - 1.0) * (c - 0.5) - ph.kappa * D2C / (double)(dx * dx);
}

// Gradient_ED_AMR (:281-289)
__device__ __forceinline__ void gradient_ed(const double* E, double& Dx, double& Dy) {
    Dx = (E[2] - E[4]) / 3.0 + (E[6] - E[7] - E[8] + E[9]) / 12.0;
    Dy = (E[3] - E[5]) / 3.0 + (E[6] + E[7] - E[8] - E[9]) / 12.0;
}

// ED_C_AMR (:244-258)
template <class CF>
__device__ __forceinline__ void ed_c(int dx, CF Cs, double* E) {
#pragma unroll
    for (int k = 1; k <= 9; ++k) E[k] = Cs(d_ex(k), d_ey(k)) - Cs(-d_ex(k), -d_ey(k));
#pragma unroll
    for (int k = 1; k <= 9; ++k) E[k] = E[k] * 0.5 / (double)dx;
}

// ED_M_AMR (:262-277)
template <class CF>
__device__ __forceinline__ void ed_m(int dx, CF Cs, double* E) {
    const double c0 = Cs(0, 0);
#pragma unroll
    for (int k = 1; k <= 9; ++k)
        E[k] = (-Cs(-d_ex(k), -d_ey(k)) - 3.0 * c0 + 5.0 * Cs(d_ex(k), d_ey(k)) -
                Cs(2 * d_ex(k), 2 * d_ey(k)));
#pragma unroll
    for (int k = 1; k <= 9; ++k) E[k] = E[k] * 0.25 / (double)dx;
}

// normal_AMR (:25-37)
__device__ __forceinline__ void normal_vec(double DcDx, double DcDy, double& ni, double& nj) {
    const double tmp = sqrt(DcDx * DcDx + DcDy * DcDy + 1.e-32);
    ni = DcDx / tmp;
    nj = DcDy / tmp;
}

// Equilibrium_h_g_AMR (:2-21)
__device__ __forceinline__ void equilibrium(const PhysD& ph, double C, double U, double V,
                                            double ni, double nj, double* Gamma, double* heq) {
    const double tmp = (12.0 * (1.0 - C)) / ph.W * ph.M0;
    const double U2 = U * U + V * V;
#pragma unroll
    for (int i = 1; i <= 9; ++i) {
        const double eU = (double)d_ex(i) * U + (double)d_ey(i) * V;
        const double eN = (double)d_ex(i) * ni + (double)d_ey(i) * nj;
        Gamma[i] = wa(i) * (1.0 + eU * (3.0 + 4.5 * eU) - 1.5 * U2);
        heq[i] = C * (Gamma[i] + tmp * wa(i) * eN);
    }
}

// MRT_Collision_AMR (:348-361) with Convert/Reconvt_D2Q9_standard (:365-401)
__device__ __forceinline__ void mrt(double s9, const double* geq, double* g) {
    double f[10], m[10], o[10];
#pragma unroll
    for (int i = 1; i <= 9; ++i) f[i] = g[i] - geq[i];
    m[1] = f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9];
    m[2] = -4.0 * f[1] - f[2] - f[3] - f[4] - f[5] + 2.0 * (f[6] + f[7] + f[8] + f[9]);
    m[3] = 4.0 * f[1] - 2.0 * (f[2] + f[3] + f[4] + f[5]) + f[6] + f[7] + f[8] + f[9];
    m[4] = f[2] - f[4] + f[6] - f[7] - f[8] + f[9];
    m[5] = -2.0 * (f[2] - f[4]) + f[6] - f[7] - f[8] + f[9];
    m[6] = f[3] - f[5] + f[6] + f[7] - f[8] - f[9];
    m[7] = -2.0 * (f[3] - f[5]) + f[6] + f[7] - f[8] - f[9];
    m[8] = f[2] - f[3] + f[4] - f[5];
    m[9] = f[6] - f[7] + f[8] - f[9];
    // S = (1,...,1, s9, s9): tmp*S is exact for the unit rates
    m[8] = m[8] * s9;
    m[9] = m[9] * s9;
    o[1] = 4.0 * (m[1] - m[2] + m[3]);
    o[2] = 4.0 * m[1] - m[2] - 2.0 * m[3] + 6.0 * (m[4] - m[5]) + 9.0 * m[8];
    o[3] = 4.0 * m[1] - m[2] - 2.0 * m[3] + 6.0 * (m[6] - m[7]) - 9.0 * m[8];
    o[4] = 4.0 * m[1] - m[2] - 2.0 * m[3] - 6.0 * (m[4] - m[5]) + 9.0 * m[8];
    o[5] = 4.0 * m[1] - m[2] - 2.0 * m[3] - 6.0 * (m[6] - m[7]) - 9.0 * m[8];
    o[6] = 4.0 * m[1] + 2.0 * m[2] + m[3] + 6.0 * m[4] + 3.0 * m[5] + 6.0 * m[6] + 3.0 * m[7] +
           9.0 * m[9];
    o[7] = 4.0 * m[1] + 2.0 * m[2] + m[3] - 6.0 * m[4] - 3.0 * m[5] + 6.0 * m[6] + 3.0 * m[7] -
           9.0 * m[9];
    o[8] = 4.0 * m[1] + 2.0 * m[2] + m[3] - 6.0 * m[4] - 3.0 * m[5] - 6.0 * m[6] - 3.0 * m[7] +
           9.0 * m[9];
    o[9] = 4.0 * m[1] + 2.0 * m[2] + m[3] + 6.0 * m[4] + 3.0 * m[5] - 6.0 * m[6] - 3.0 * m[7] -
           9.0 * m[9];
#pragma unroll
    for (int i = 1; i <= 9; ++i) g[i] = g[i] - o[i] / 36.0;
}

// Gradient_AMR (:293-312) at one cell
template <class CF>
__device__ __forceinline__ void gradient_iso(int dx, CF Cs, double& DcDx, double& DcDy) {
    DcDx = ((Cs(1, 0) - Cs(-1, 0)) / 3.0 + (Cs(1, 1) + Cs(1, -1) - Cs(-1, 1) - Cs(-1, -1)) / 12.0) /
           (double)dx;
    DcDy = ((Cs(0, 1) - Cs(0, -1)) / 3.0 + (Cs(1, 1) + Cs(-1, 1) - Cs(1, -1) - Cs(-1, -1)) / 12.0) /
           (double)dx;
}

// Macroscopic_Values_g_AMR (:205-240) at one cell; g[1..9]
template <class CF>
__device__ __forceinline__ void macro_g_cell(const PhysD& ph, int dx, CF Cs, const double* g,
                                             double& P, double& Ux, double& Uy) {
    const double dRho6 = (ph.Rhoh - ph.Rhol) / 6.0;
    double DcDx, DcDy;
    gradient_iso(dx, Cs, DcDx, DcDy);
    const double mu = chem_pot(ph, dx, Cs);
    const double c = Cs(0, 0);
    const double Rho = ph.Rhol + c * (ph.Rhoh - ph.Rhol);
    const double Fb = (ph.Rhoh - Rho) * ph.Gy;
    const double Fx = mu * DcDx;
    const double Fy = mu * DcDy + Fb;
    // SUM(g(2:9)*ex(2:9)) from 0 in index order; the zero terms g*0 only
    // change the sign of an exact zero and are omitted
    const double sx = ((((g[2] - g[4]) + g[6]) - g[7]) - g[8]) + g[9];
    const double sy = ((((g[3] - g[5]) + g[6]) + g[7]) - g[8]) - g[9];
    Ux = (3.0 * sx + 0.5 * Fx) / Rho;
    Uy = (3.0 * sy + 0.5 * Fy) / Rho;
    double sp = 0.0;
#pragma unroll
    for (int k = 1; k <= 9; ++k) sp = sp + g[k];
    P = sp + dRho6 * (Ux * DcDx + Uy * DcDy);
}

// Collision_h_g_AMR (:116-189) at one cell: h[1..9], g[1..9] in/out
template <class CF>
__device__ __forceinline__ void collide_cell(const PhysD& ph, int dx, CF Cs, double P, double Ux,
                                             double Uy, double* h, double* g) {
    const double dRho3 = (ph.Rhoh - ph.Rhol) / 3.0;
    const double mu = chem_pot(ph, dx, Cs);
    const double Cij = Cs(0, 0);
    double E[10], Gamma[10], heq[10], hlp[10], geq[10];
    double DcDx, DcDy, ni, nj;
    ed_c(dx, Cs, E);
    gradient_ed(E, DcDx, DcDy);
    normal_vec(DcDx, DcDy, ni, nj);
    equilibrium(ph, Cij, Ux, Uy, ni, nj, Gamma, heq);
#pragma unroll
    for (int k = 1; k <= 9; ++k) h[k] = h[k] * (1.0 - ph.wc) + heq[k] * ph.wc;
    const double Rho = ph.Rhol + Cij * (ph.Rhoh - ph.Rhol);
    const double Fb = (ph.Rhoh - Rho) * ph.Gy;
    {
        const double ud = Ux * DcDx + Uy * DcDy;
#pragma unroll
        for (int k = 1; k <= 9; ++k)
            hlp[k] = ((Gamma[k] - wa(k)) * dRho3 + Gamma[k] * mu) * (E[k] - ud) +
                     ((double)d_ey(k) - Uy) * Gamma[k] * Fb;
    }
#pragma unroll
    for (int k = 1; k <= 9; ++k) geq[k] = P * wa(k) + (Gamma[k] - wa(k)) * Rho / 3.0 - 0.5 * hlp[k];
    ed_m(dx, Cs, E);
    gradient_ed(E, DcDx, DcDy);
    {
        const double ud = Ux * DcDx + Uy * DcDy;
#pragma unroll
        for (int k = 1; k <= 9; ++k)
            hlp[k] = ((Gamma[k] - wa(k)) * dRho3 + Gamma[k] * mu) * (E[k] - ud) +
                     ((double)d_ey(k) - Uy) * Gamma[k] * Fb;
    }
    double tau;
    if (Cij < 0.0) {
        tau = ph.taul + 0.5;
    } else if (Cij > 1.0) {
        tau = ph.tauh + 0.5;
    } else {
        tau = Cij * (1.0 / ph.tauh - 1.0 / ph.taul) + 1.0 / ph.taul;
        tau = 1.0 / tau + 0.5;
    }
    const double s9 = 1.0 / tau;
    mrt(s9, geq, g);
#pragma unroll
    for (int k = 1; k <= 9; ++k) g[k] = g[k] + hlp[k];
}

// ---------------------------------------------------------------------------
// Interpolations.f90 stencils evaluated at one output point. The reference
// reduces its gathered (dim1 = x, dim2 = y) array first along dim2, then
// along dim1; G(i, j) is 1-based.

// Biquadratic_from_Fine (:2-34): output (X, Y)
template <class GF>
__device__ __forceinline__ double biq_fine_pt(int X, int Y, GF G) {
    const int Jy = (Y + 1) % 2, iy = 2 * Y - 1 - Jy, ay = 3 - 4 * Jy, cy = 2 - ay;
    const int Jx = (X + 1) % 2, ix = 2 * X - 1 - Jx, ax = 3 - 4 * Jx, cx = 2 - ax;
    double t[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
        t[r] = (double)ay * G(ix + r, iy) + 6.0 * G(ix + r, iy + 1) + (double)cy * G(ix + r, iy + 2);
    const double o = (double)ax * t[0] + 6.0 * t[1] + (double)cx * t[2];
    return o / 64.0;
}

// Biquadratic_from_Coarse (:74-104): output (x, y)
template <class GF>
__device__ __forceinline__ double biq_coarse_pt(int x, int y, GF G) {
    const int Iy = (y + 1) / 2, ay = 5 - 8 * ((y + 1) % 2), cy = 2 - ay;
    const int Ix = (x + 1) / 2, ax = 5 - 8 * ((x + 1) % 2), cx = 2 - ax;
    double t[3];
#pragma unroll
    for (int r = 0; r < 3; ++r)
        t[r] = (double)ay * G(Ix + r, Iy) + 30.0 * G(Ix + r, Iy + 1) + (double)cy * G(Ix + r, Iy + 2);
    const double o = (double)ax * t[0] + 30.0 * t[1] + (double)cx * t[2];
    return o / 1024.0;
}

// ---------------------------------------------------------------------------
// neighbour pointers (Parameters.f90:23-31): value of Blk(n)%nghbr(k)%n
__device__ __forceinline__ int resolve_nb(const DevState& s, int n, int k) {
    const int o = s.nb_owner[8 * n + k - 1];
    const int sl = s.nb_slot[8 * n + k - 1];
    if (sl == 0) return o;
    return s.child[4 * o + sl - 1];
}

__device__ __forceinline__ void set_error(const DevState& s, int code, int info) {
    if (atomicCAS(&s.cnt->error, 0, code) == 0) s.cnt->error_info = info;
}
