/*
 * amrlbm_oracle.cpp - CPU oracle: a line-by-line C++17/OpenMP restatement of
 * the hot path of AMR-LBM-OpenMP-2D (Fortran 90 + OpenMP, GPL-3.0,
 * A. Fakhari). TEST INFRASTRUCTURE ONLY: tests/, the smoke check and the CPU
 * baseline leg of bench.py load it as the checker; the product never does.
 *
 * PARITY UNPINNED. The reference has no tests, golden vectors or fixtures and
 * cannot be compiled here (no Fortran compiler), so this restatement is
 * pinned only by known-answer tests derived from the reference's formulas and
 * by invariants (mass, symmetry, 2:1 balance, neighbour reciprocity).
 *
 * Faithfulness rules followed throughout:
 *   - Fortran evaluation order: left-to-right for +,-,*,/ of equal
 *     precedence, parentheses kept, x**2 (real or integer 2) evaluated as
 *     x*x, D**3 as (D*D)*D; built with -ffp-contract=off so no FMA contraction;
 *   - SUM(...) accumulates from 0 in index order;
 *   - 1-based block ids, the reference's array bounds and layouts;
 *   - a neighbour is a pointer to an integer (Parameters.f90:23-31): it is
 *     held as (owner, slot) and read at the time of use.
 * Deliberate generalisations (defaults reproduce the reference exactly):
 *   - nx, ny, L0/nx, minLevels, maxLevels, MaxBlks, physics, bubble geometry,
 *     tolerances and the regrid interval are run-time parameters;
 *   - the base grid is nbx x nby blocks, periodic in x, walls in y (the
 *     reference's 1 x 3 stack, AMR_Rising_2D_OMP.f90:54-57,119-138, is
 *     nbx=1, nby=3);
 *   - base blocks start with child(:) = self instead of -1
 *     (AMR_Rising_2D_OMP.f90:94). With minLevels >= 1, as in the reference,
 *     every base block is refined before the value can be read; with
 *     minLevels = 0 the -1 would make a refined block see a wall where its
 *     unrefined base neighbour is;
 *   - base blocks get field arrays when they stay leaves (minLevels = 0).
 */
#include "amrlbm_oracle.h"

#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <vector>

namespace {

/* D2Q9_Mod.f90:6-8, 1-based */
const int ex[10] = {0, 0, 1, 0, -1, 0, 1, -1, -1, 1};
const int ey[10] = {0, 0, 0, 1, 0, -1, 1, 1, -1, -1};
struct WaTable {
    double v[10];
    WaTable() {
        const int w[9] = {16, 4, 4, 4, 4, 1, 1, 1, 1};
        v[0] = 0.0;
        for (int i = 0; i < 9; ++i) v[i + 1] = w[i] / 36.0;
    }
};
const WaTable WA;
#define Wa(i) (WA.v[i])

struct Phys {
    double W, Sigma, Beta, kappa, taul, tauh, Rhol, Rhoh, Gy, M0, wc;
};

/* Pointer to an integer (Parameters.f90:23-25). slot 1..4: Blk(owner)%child(slot);
 * slot 0: a constant integer whose value is owner. gen: generation of owner's
 * child array when the pointer was made (catches use of a deallocated array). */
struct NbPtr {
    int owner = 0, slot = 0, gen = 0;
};

struct Block {
    int level = -1, dx = 0, I = 0, J = 0, parent = -1;
    int child[5] = {0, 0, 0, 0, 0};
    bool child_alloc = false;
    int gen = 0;
    NbPtr nb[9];
    bool isLeaf = false, hasLeaf = false, refin = false, deref = false;
    bool alloc = false;
    std::vector<double> h, g, C, P, Ux, Uy;
};

}  // namespace

struct orc_sim {
    amrlbm_params prm;
    Phys ph;
    int nx, ny, MaxBlks, nthreads;
    /* seconds per phase, as the timers of Main_Loop (AMR_Rising_2D_OMP.f90:
     * 366-375): Macroscopic_h, Macroscopic_g, collision, advection, Ghost_C,
     * Ghost_C2, Ghost_hg, refine */
    double phase_s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    std::vector<Block> blk; /* 1-based */
    int Nblks = 0, nLeaf = 0, KK = 0, LevelMin = 0, LevelMax = 0;
    std::vector<int> LeafBlks;
    std::deque<int> freelist; /* Root (front) ... emptyBlk (back) */
    long stepcount = 0;
    int err = 0;
    int level_jumps = 0;
    int g_model = 0; /* collision of g: 0 MRT (the reference's), 1 BGK */

    /* field accessors in the reference's layouts */
    int NX2() const { return nx + 2; }
    int NX4() const { return nx + 4; }
    size_t hsize() const { return (size_t)9 * (nx + 2) * (ny + 2); }
    size_t csize() const { return (size_t)(nx + 4) * (ny + 4); }
    size_t psize() const { return (size_t)nx * ny; }
    double& H(std::vector<double>& f, int q, int x, int y) const {
        return f[(q - 1) + 9 * (x + (nx + 2) * y)];
    }
    double H(const std::vector<double>& f, int q, int x, int y) const {
        return f[(q - 1) + 9 * (x + (nx + 2) * y)];
    }
    double& Cm(Block& b, int x, int y) const { return b.C[(x + 1) + (nx + 4) * (y + 1)]; }
    double Cm(const Block& b, int x, int y) const { return b.C[(x + 1) + (nx + 4) * (y + 1)]; }
    double& Pm(std::vector<double>& a, int x, int y) const { return a[(x - 1) + nx * (y - 1)]; }
    double Pm(const std::vector<double>& a, int x, int y) const {
        return a[(x - 1) + nx * (y - 1)];
    }

    void set_err(int e) {
        if (!err) err = e;
    }

    /* value of Blk(n)%nghbr(k)%n */
    int resolve(int n, int k) {
        const NbPtr& p = blk[n].nb[k];
        if (p.slot == 0) return p.owner;
        const Block& o = blk[p.owner];
        if (!o.child_alloc || o.gen != p.gen) {
            set_err(AMRLBM_ERR_DANGLING);
            return o.child_alloc ? o.child[p.slot] : -999999;
        }
        return o.child[p.slot];
    }
    int resolve_c(int n, int k) const { return const_cast<orc_sim*>(this)->resolve(n, k); }
    NbPtr child_ptr(int owner, int slot) const {
        NbPtr p;
        p.owner = owner;
        p.slot = slot;
        p.gen = blk[owner].gen;
        return p;
    }
    static NbPtr const_ptr(int v) {
        NbPtr p;
        p.owner = v;
        p.slot = 0;
        return p;
    }

    void alloc_fields(Block& b) {
        b.h.assign(hsize(), 0.0);
        b.g.assign(hsize(), 0.0);
        b.C.assign(csize(), 0.0);
        b.P.assign(psize(), 0.0);
        b.Ux.assign(psize(), 0.0);
        b.Uy.assign(psize(), 0.0);
        b.alloc = true;
    }
    void free_fields(Block& b) {
        std::vector<double>().swap(b.h);
        std::vector<double>().swap(b.g);
        std::vector<double>().swap(b.C);
        std::vector<double>().swap(b.P);
        std::vector<double>().swap(b.Ux);
        std::vector<double>().swap(b.Uy);
        b.alloc = false;
    }
};

namespace {

/* ======================================================================
 *  Set_Rising_Bubble_Parameters (AMR_Rising_2D_OMP.f90:235-263) and
 *  D2Q9_Mod (D2Q9_Mod.f90:10-11)
 * ====================================================================== */
Phys derive_phys(const amrlbm_params& p) {
    Phys ph;
    const double R = p.radius;
    const double D = 2.0 * R; /* AMR_Rising_2D_OMP.f90:155 */
    ph.Rhol = p.rho_l;
    ph.Rhoh = p.rho_h;
    ph.Gy = p.gy;
    ph.Sigma = ph.Gy * (ph.Rhoh - ph.Rhol) * (D * D) / p.bo;
    const double muh = std::sqrt(ph.Gy * ph.Rhoh * (ph.Rhoh - ph.Rhol) * ((D * D) * D)) / p.ar;
    const double mul = muh / p.visc_ratio;
    ph.tauh = 3.0 * (muh / ph.Rhoh);
    ph.taul = 3.0 * (mul / ph.Rhol);
    ph.W = p.w;
    ph.Beta = 12.0 * ph.Sigma / ph.W;
    ph.kappa = 1.5 * ph.Sigma * ph.W;
    ph.M0 = p.m0;
    ph.wc = 1.0 / (0.5 + ph.M0 * 3.0);
    return ph;
}

/* ======================================================================
 *  LBM_Subroutines.f90
 * ====================================================================== */

/* Equilibrium_h_g_AMR (LBM_Subroutines.f90:2-21) */
inline void equilibrium(const Phys& ph, double C, double U, double V, double ni, double nj,
                        double* Gamma, double* heq) {
    const double tmp = (12.0 * (1.0 - C)) / ph.W * ph.M0;
    const double U2 = U * U + V * V;
    for (int i = 1; i <= 9; ++i) {
        const double eU = (double)ex[i] * U + (double)ey[i] * V;
        const double eN = (double)ex[i] * ni + (double)ey[i] * nj;
        Gamma[i] = Wa(i) * (1.0 + eU * (3.0 + 4.5 * eU) - 1.5 * U2);
        heq[i] = C * (Gamma[i] + tmp * Wa(i) * eN);
    }
}

/* normal_AMR (LBM_Subroutines.f90:25-37); DcDx**2.d0 is folded to DcDx*DcDx */
inline void normal(double DcDx, double DcDy, double& ni, double& nj) {
    const double tmp = std::sqrt(DcDx * DcDx + DcDy * DcDy + 1.e-32);
    ni = DcDx / tmp;
    nj = DcDy / tmp;
}

/* Laplacian_AMR (LBM_Subroutines.f90:316-333) + Chemical_Potential_AMR (:94-112) */
void chemical_potential(const orc_sim& s, int dx, const Block& b, std::vector<double>& mu) {
    const int nx = s.nx, ny = s.ny;
    mu.resize((size_t)nx * ny);
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            auto C = [&](int x, int y) { return s.Cm(b, x, y); };
            const double D2C = (C(i - 1, j - 1) + C(i + 1, j - 1) + C(i - 1, j + 1) +
                                C(i + 1, j + 1) +
                                4 * (C(i, j - 1) + C(i - 1, j) + C(i + 1, j) + C(i, j + 1)) -
                                20 * C(i, j)) /
                               6;
            const double c = C(i, j);
            mu[(i - 1) + nx * (j - 1)] =
                4.0 * s.ph.Beta * c * (c - 1.0) * (c - 0.5) - s.ph.kappa * D2C / (double)(dx * dx);
        }
}

/* ED_C_AMR (LBM_Subroutines.f90:244-258) */
inline void ed_c(const orc_sim& s, int dx, const Block& b, int i, int j, double* E) {
    for (int k = 1; k <= 9; ++k)
        E[k] = s.Cm(b, i + ex[k], j + ey[k]) - s.Cm(b, i - ex[k], j - ey[k]);
    for (int k = 1; k <= 9; ++k) E[k] = E[k] * 0.5 / (double)dx;
}

/* ED_M_AMR (LBM_Subroutines.f90:262-277) */
inline void ed_m(const orc_sim& s, int dx, const Block& b, int i, int j, double* E) {
    for (int k = 1; k <= 9; ++k)
        E[k] = (-s.Cm(b, i - ex[k], j - ey[k]) - 3.0 * s.Cm(b, i, j) +
                5.0 * s.Cm(b, i + ex[k], j + ey[k]) - s.Cm(b, i + 2 * ex[k], j + 2 * ey[k]));
    for (int k = 1; k <= 9; ++k) E[k] = E[k] * 0.25 / (double)dx;
}

/* Gradient_ED_AMR (LBM_Subroutines.f90:281-289) */
inline void gradient_ed(const double* ED, double& Dx, double& Dy) {
    Dx = (ED[2] - ED[4]) / 3.0 + (ED[6] - ED[7] - ED[8] + ED[9]) / 12.0;
    Dy = (ED[3] - ED[5]) / 3.0 + (ED[6] + ED[7] - ED[8] - ED[9]) / 12.0;
}

/* Convert_D2Q9_standard (LBM_Subroutines.f90:365-380) */
inline void convert(const double* f, double* o) {
    o[1] = f[1] + f[2] + f[3] + f[4] + f[5] + f[6] + f[7] + f[8] + f[9];
    o[2] = -4.0 * f[1] - f[2] - f[3] - f[4] - f[5] + 2 * (f[6] + f[7] + f[8] + f[9]);
    o[3] = 4.0 * f[1] - 2.0 * (f[2] + f[3] + f[4] + f[5]) + f[6] + f[7] + f[8] + f[9];
    o[4] = f[2] - f[4] + f[6] - f[7] - f[8] + f[9];
    o[5] = -2.0 * (f[2] - f[4]) + f[6] - f[7] - f[8] + f[9];
    o[6] = f[3] - f[5] + f[6] + f[7] - f[8] - f[9];
    o[7] = -2.0 * (f[3] - f[5]) + f[6] + f[7] - f[8] - f[9];
    o[8] = f[2] - f[3] + f[4] - f[5];
    o[9] = f[6] - f[7] + f[8] - f[9];
}

/* Reconvt_D2Q9_standard (LBM_Subroutines.f90:384-401) */
inline void reconvt(const double* f, double* o) {
    o[1] = 4.0 * (f[1] - f[2] + f[3]);
    o[2] = 4.0 * f[1] - f[2] - 2.0 * f[3] + 6.0 * (f[4] - f[5]) + 9.0 * f[8];
    o[3] = 4.0 * f[1] - f[2] - 2.0 * f[3] + 6.0 * (f[6] - f[7]) - 9.0 * f[8];
    o[4] = 4.0 * f[1] - f[2] - 2.0 * f[3] - 6.0 * (f[4] - f[5]) + 9.0 * f[8];
    o[5] = 4.0 * f[1] - f[2] - 2.0 * f[3] - 6.0 * (f[6] - f[7]) - 9.0 * f[8];
    o[6] = 4.0 * f[1] + 2.0 * f[2] + f[3] + 6.0 * f[4] + 3.0 * f[5] + 6.0 * f[6] + 3.0 * f[7] +
           9.0 * f[9];
    o[7] = 4.0 * f[1] + 2.0 * f[2] + f[3] - 6.0 * f[4] - 3.0 * f[5] + 6.0 * f[6] + 3.0 * f[7] -
           9.0 * f[9];
    o[8] = 4.0 * f[1] + 2.0 * f[2] + f[3] - 6.0 * f[4] - 3.0 * f[5] - 6.0 * f[6] - 3.0 * f[7] +
           9.0 * f[9];
    o[9] = 4.0 * f[1] + 2.0 * f[2] + f[3] + 6.0 * f[4] + 3.0 * f[5] - 6.0 * f[6] - 3.0 * f[7] -
           9.0 * f[9];
    for (int i = 1; i <= 9; ++i) o[i] = o[i] / 36.0;
}

/* MRT_Collision_AMR (LBM_Subroutines.f90:348-361); g is 1-based g[1..9] */
inline void mrt(double s9, const double* geq, double* g) {
    double d[10], m[10], r[10];
    for (int i = 1; i <= 9; ++i) d[i] = g[i] - geq[i];
    convert(d, m);
    double S[10];
    for (int i = 1; i <= 7; ++i) S[i] = 1.0;
    S[8] = s9;
    S[9] = s9;
    for (int i = 1; i <= 9; ++i) m[i] = m[i] * S[i];
    reconvt(m, r);
    for (int i = 1; i <= 9; ++i) g[i] = g[i] - r[i];
}

/* BGK_Collision_AMR (LBM_Subroutines.f90:337-344), the alternative the
 * reference leaves commented out at :180: g = g*(1 - s9) + geq*s9 */
inline void bgk(double s9, const double* geq, double* g) {
    for (int i = 1; i <= 9; ++i) g[i] = g[i] * (1.0 - s9) + geq[i] * s9;
}

/* Collision_h_g_AMR (LBM_Subroutines.f90:116-189) */
void collision(const orc_sim& s, Block& b) {
    const Phys& ph = s.ph;
    const int nx = s.nx, ny = s.ny, dx = b.dx;
    const double dRho3 = (ph.Rhoh - ph.Rhol) / 3.0;
    std::vector<double> mu;
    chemical_potential(s, dx, b, mu);
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            double eDc[10], hlp[10], Gamma[10], heq[10], geq[10];
            double DcDx, DcDy, ni, nj;
            const double Cij = s.Cm(b, i, j);
            const double Ux = s.Pm(b.Ux, i, j), Uy = s.Pm(b.Uy, i, j), P = s.Pm(b.P, i, j);
            const double muij = mu[(i - 1) + nx * (j - 1)];
            ed_c(s, dx, b, i, j, eDc);
            gradient_ed(eDc, DcDx, DcDy);
            normal(DcDx, DcDy, ni, nj);
            equilibrium(ph, Cij, Ux, Uy, ni, nj, Gamma, heq);
            /* COLLISION (h) :146 */
            for (int k = 1; k <= 9; ++k)
                s.H(b.h, k, i, j) = s.H(b.h, k, i, j) * (1.0 - ph.wc) + heq[k] * ph.wc;
            /* COLLISION (g) :150-183 */
            const double Rho = ph.Rhol + Cij * (ph.Rhoh - ph.Rhol);
            const double Fb = (ph.Rhoh - Rho) * ph.Gy;
            for (int k = 1; k <= 9; ++k)
                hlp[k] = ((Gamma[k] - Wa(k)) * dRho3 + Gamma[k] * muij) *
                             (eDc[k] - (Ux * DcDx + Uy * DcDy)) +
                         ((double)ey[k] - Uy) * Gamma[k] * Fb;
            for (int k = 1; k <= 9; ++k)
                geq[k] = P * Wa(k) + (Gamma[k] - Wa(k)) * Rho / 3.0 - 0.5 * hlp[k];
            ed_m(s, dx, b, i, j, eDc);
            gradient_ed(eDc, DcDx, DcDy);
            for (int k = 1; k <= 9; ++k)
                hlp[k] = ((Gamma[k] - Wa(k)) * dRho3 + Gamma[k] * muij) *
                             (eDc[k] - (Ux * DcDx + Uy * DcDy)) +
                         ((double)ey[k] - Uy) * Gamma[k] * Fb;
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
            double gl[10];
            for (int k = 1; k <= 9; ++k) gl[k] = s.H(b.g, k, i, j);
            if (s.g_model == 1)
                bgk(s9, geq, gl);
            else
                mrt(s9, geq, gl);
            for (int k = 1; k <= 9; ++k) s.H(b.g, k, i, j) = gl[k] + hlp[k];
        }
}

/* Perfect_Shift_AMR (LBM_Subroutines.f90:41-62) and
 * Streaming_LaxWendroff_AMR (:66-90) */
void stream_field(const orc_sim& s, std::vector<double>& f, int dx) {
    const int nx = s.nx, ny = s.ny;
    const double cfl = 1.0 / (double)dx;
    std::vector<double> fnew((size_t)8 * nx * ny);
    auto FN = [&](int i, int X, int Y) -> double& {
        return fnew[(i - 2) + 8 * ((X - 1) + nx * (Y - 1))];
    };
    if (cfl > (double)0.9f) { /* 0.9 is a default-kind REAL literal (:416) */
        for (int Y = 1; Y <= ny; ++Y)
            for (int X = 1; X <= nx; ++X)
                for (int i = 2; i <= 9; ++i) FN(i, X, Y) = s.H(f, i, X - ex[i], Y - ey[i]);
    } else {
        for (int Y = 1; Y <= ny; ++Y)
            for (int X = 1; X <= nx; ++X)
                for (int i = 2; i <= 9; ++i)
                    FN(i, X, Y) = cfl / 2 * (1 + cfl) * s.H(f, i, X - ex[i], Y - ey[i]) +
                                  (1 - cfl * cfl) * s.H(f, i, X, Y) -
                                  cfl / 2 * (1 - cfl) * s.H(f, i, X + ex[i], Y + ey[i]);
    }
    for (int Y = 1; Y <= ny; ++Y)
        for (int X = 1; X <= nx; ++X)
            for (int i = 2; i <= 9; ++i) s.H(f, i, X, Y) = FN(i, X, Y);
}

/* Macroscopic_Values_h_AMR (LBM_Subroutines.f90:193-201) */
void macro_h(const orc_sim& s, Block& b) {
    for (int j = 1; j <= s.ny; ++j)
        for (int i = 1; i <= s.nx; ++i) {
            double sum = 0.0;
            for (int k = 1; k <= 9; ++k) sum = sum + s.H(b.h, k, i, j);
            s.Cm(b, i, j) = sum;
        }
}

/* Gradient_AMR (LBM_Subroutines.f90:293-312) */
inline void gradient(const orc_sim& s, int dx, const Block& b, int i, int j, double& DcDx,
                     double& DcDy) {
    auto C = [&](int x, int y) { return s.Cm(b, x, y); };
    DcDx = ((C(i + 1, j) - C(i - 1, j)) / 3.0 +
            (C(i + 1, j + 1) + C(i + 1, j - 1) - C(i - 1, j + 1) - C(i - 1, j - 1)) / 12.0) /
           (double)dx;
    DcDy = ((C(i, j + 1) - C(i, j - 1)) / 3.0 +
            (C(i + 1, j + 1) + C(i - 1, j + 1) - C(i + 1, j - 1) - C(i - 1, j - 1)) / 12.0) /
           (double)dx;
}

/* Macroscopic_Values_g_AMR (LBM_Subroutines.f90:205-240) */
void macro_g(const orc_sim& s, Block& b) {
    const Phys& ph = s.ph;
    const int nx = s.nx, ny = s.ny, dx = b.dx;
    const double dRho6 = (ph.Rhoh - ph.Rhol) / 6.0;
    std::vector<double> mu;
    chemical_potential(s, dx, b, mu);
    for (int j = 1; j <= ny; ++j)
        for (int i = 1; i <= nx; ++i) {
            double DcDx, DcDy;
            gradient(s, dx, b, i, j, DcDx, DcDy);
            const double Cij = s.Cm(b, i, j);
            const double Rho = ph.Rhol + Cij * (ph.Rhoh - ph.Rhol);
            const double Fb = (ph.Rhoh - Rho) * ph.Gy;
            const double muij = mu[(i - 1) + nx * (j - 1)];
            const double Fx = muij * DcDx;
            const double Fy = muij * DcDy + Fb;
            double sx = 0.0, sy = 0.0, sp = 0.0;
            for (int k = 2; k <= 9; ++k) sx = sx + s.H(b.g, k, i, j) * (double)ex[k];
            for (int k = 2; k <= 9; ++k) sy = sy + s.H(b.g, k, i, j) * (double)ey[k];
            const double Ux = (3.0 * sx + 0.5 * Fx) / Rho;
            const double Uy = (3.0 * sy + 0.5 * Fy) / Rho;
            for (int k = 1; k <= 9; ++k) sp = sp + s.H(b.g, k, i, j);
            s.Pm(b.Ux, i, j) = Ux;
            s.Pm(b.Uy, i, j) = Uy;
            s.Pm(b.P, i, j) = sp + dRho6 * (Ux * DcDx + Uy * DcDy);
        }
}

/* Err_Interface (Refine_Derefine.f90:327-351); (a)**2.d0 folded to a*a */
double err_interface(const orc_sim& s, const Block& b) {
    double err = 0.0;
    for (int J = 1; J <= s.ny; ++J)
        for (int I = 1; I <= s.nx; ++I) {
            const double a = s.Cm(b, I + 1, J) - s.Cm(b, I - 1, J);
            const double c = s.Cm(b, I, J + 1) - s.Cm(b, I, J - 1);
            const double DC = a * a + c * c;
            err = (DC > err) ? DC : err; /* MAX(err, DC) */
        }
    return std::sqrt(err) / (2.0 * b.dx);
}

/* ======================================================================
 *  Interpolations.f90 (arrays are 1-based, column-major; lead = 1 or 9)
 * ====================================================================== */

/* Biquadratic_from_Fine(_f) (Interpolations.f90:2-70) */
void biq_fine(int lead, int i2, int /*j2*/, int X2, int Y2, const double* Cin, double* Cout) {
    auto IN = [&](int q, int i, int j) { return Cin[q + lead * ((i - 1) + i2 * (j - 1))]; };
    std::vector<double> tmp((size_t)lead * i2 * Y2);
    auto T = [&](int q, int i, int j) -> double& { return tmp[q + lead * ((i - 1) + i2 * (j - 1))]; };
    auto OUT = [&](int q, int i, int j) -> double& {
        return Cout[q + lead * ((i - 1) + X2 * (j - 1))];
    };
    const int b = 6;
    for (int X = 1; X <= Y2; ++X) {
        const int J = (X + 1) % 2, i = 2 * X - 1 - J, a = 3 - 4 * J, c = 2 - a;
        for (int r = 1; r <= i2; ++r)
            for (int q = 0; q < lead; ++q)
                T(q, r, X) = a * IN(q, r, i) + b * IN(q, r, i + 1) + c * IN(q, r, i + 2);
    }
    for (int X = 1; X <= X2; ++X) {
        const int J = (X + 1) % 2, i = 2 * X - 1 - J, a = 3 - 4 * J, c = 2 - a;
        for (int r = 1; r <= Y2; ++r)
            for (int q = 0; q < lead; ++q)
                OUT(q, X, r) = a * T(q, i, r) + b * T(q, i + 1, r) + c * T(q, i + 2, r);
    }
    for (int k = 0; k < lead * X2 * Y2; ++k) Cout[k] = Cout[k] / 64.0;
}

/* Biquadratic_from_Coarse(_f) (Interpolations.f90:74-138) */
void biq_coarse(int lead, int I2, int J2, int x2, int y2, const double* Cin, double* Cout) {
    (void)J2;
    auto IN = [&](int q, int i, int j) { return Cin[q + lead * ((i - 1) + I2 * (j - 1))]; };
    std::vector<double> tmp((size_t)lead * I2 * y2);
    auto T = [&](int q, int i, int j) -> double& { return tmp[q + lead * ((i - 1) + I2 * (j - 1))]; };
    auto OUT = [&](int q, int i, int j) -> double& {
        return Cout[q + lead * ((i - 1) + x2 * (j - 1))];
    };
    const int b = 30;
    for (int x = 1; x <= y2; ++x) {
        const int I = (x + 1) / 2, a = 5 - 8 * ((x + 1) % 2), c = 2 - a;
        for (int r = 1; r <= I2; ++r)
            for (int q = 0; q < lead; ++q)
                T(q, r, x) = a * IN(q, r, I) + b * IN(q, r, I + 1) + c * IN(q, r, I + 2);
    }
    for (int x = 1; x <= x2; ++x) {
        const int I = (x + 1) / 2, a = 5 - 8 * ((x + 1) % 2), c = 2 - a;
        for (int r = 1; r <= y2; ++r)
            for (int q = 0; q < lead; ++q)
                OUT(q, x, r) = a * T(q, I, r) + b * T(q, I + 1, r) + c * T(q, I + 2, r);
    }
    for (int k = 0; k < lead * x2 * y2; ++k) Cout[k] = Cout[k] / 1024.0;
}

/* Bilinear_from_Fine(_f) (Interpolations.f90:142-194) */
void bil_fine(int lead, int i2, int j2, int X2, int Y2, const double* Cin, double* Cout) {
    (void)j2;
    auto IN = [&](int q, int i, int j) { return Cin[q + lead * ((i - 1) + i2 * (j - 1))]; };
    std::vector<double> tmp((size_t)lead * i2 * Y2);
    auto T = [&](int q, int i, int j) -> double& { return tmp[q + lead * ((i - 1) + i2 * (j - 1))]; };
    auto OUT = [&](int q, int i, int j) -> double& {
        return Cout[q + lead * ((i - 1) + X2 * (j - 1))];
    };
    for (int X = 1; X <= Y2; ++X) {
        const int i = 2 * X - 1;
        for (int r = 1; r <= i2; ++r)
            for (int q = 0; q < lead; ++q) T(q, r, X) = 0.5 * (IN(q, r, i) + IN(q, r, i + 1));
    }
    for (int X = 1; X <= X2; ++X) {
        const int i = 2 * X - 1;
        for (int r = 1; r <= Y2; ++r)
            for (int q = 0; q < lead; ++q) OUT(q, X, r) = 0.5 * (T(q, i, r) + T(q, i + 1, r));
    }
}

/* ======================================================================
 *  BC_Cell.f90
 * ====================================================================== */

/* Bounce_Back_3 (BC_Cell.f90:2-21) */
void bounce_back_3(const orc_sim& s, std::vector<double>& f) {
    const int nx = s.nx;
    const int Y = 0;
    for (int X = 0; X <= nx + 1; ++X) {
        s.H(f, 1, X, Y) = s.H(f, 1, X, Y + 1);
        for (int i = 2; i <= 9; ++i) {
            const int Xn = std::min(std::max(0, X + ex[i] * ey[i]), nx + 1);
            const int J = (i - 2) + 4 * ((i / 2) % 2);
            s.H(f, i, X, Y) = s.H(f, J, Xn, Y + 1);
        }
    }
}

/* Bounce_Back_4 (BC_Cell.f90:24-42) */
void bounce_back_4(const orc_sim& s, std::vector<double>& f) {
    const int nx = s.nx, ny = s.ny;
    const int Y = ny + 1;
    for (int X = 0; X <= nx + 1; ++X) {
        s.H(f, 1, X, Y) = s.H(f, 1, X, Y - 1);
        for (int i = 2; i <= 9; ++i) {
            const int Xn = std::min(std::max(0, X - ex[i] * ey[i]), nx + 1);
            const int J = (i - 2) + 4 * ((i / 2) % 2);
            s.H(f, i, X, Y) = s.H(f, J, Xn, Y - 1);
        }
    }
}

/* Symmetric_C_3/4 (BC_Cell.f90:46-72) and Symmetric_C2_3/4 (:76-104) */
void symmetric_3(const orc_sim& s, Block& b, int w) {
    if (w == 1) {
        for (int X = 0; X <= s.nx + 1; ++X) s.Cm(b, X, 0) = s.Cm(b, X, 1);
    } else {
        for (int X = -1; X <= s.nx + 2; ++X) {
            s.Cm(b, X, -1) = s.Cm(b, X, 2);
            s.Cm(b, X, 0) = s.Cm(b, X, 1);
        }
    }
}
void symmetric_4(const orc_sim& s, Block& b, int w) {
    const int ny = s.ny;
    if (w == 1) {
        for (int X = 0; X <= s.nx + 1; ++X) s.Cm(b, X, ny + 1) = s.Cm(b, X, ny);
    } else {
        for (int X = -1; X <= s.nx + 2; ++X) {
            s.Cm(b, X, ny + 1) = s.Cm(b, X, ny);
            s.Cm(b, X, ny + 2) = s.Cm(b, X, ny - 1);
        }
    }
}

/* ======================================================================
 *  Fill_Ghost_Cells_C.f90 (w = 1) and Fill_Ghost_Cells_C2.f90 (w = 2)
 * ====================================================================== */

void level_jump(orc_sim& s) {
#pragma omp atomic
    s.level_jumps++;
}

/* Fill_Left_C(2) (Fill_Ghost_Cells_C.f90:44-89, _C2.f90:44-89) */
void fill_left_c(orc_sim& s, int n, int L, int N1, int w) {
    const int nx = s.nx, ny = s.ny;
    Block& B = s.blk[n];
    const Block& Nb = s.blk[N1];
    const int L_nbr = Nb.level;
    std::vector<double> out((size_t)w * ny);
    if (L == L_nbr) {
        if (Nb.isLeaf) {
            for (int j = 1; j <= ny; ++j)
                for (int a = 1; a <= w; ++a) s.Cm(B, 1 - a, j) = s.Cm(Nb, nx + 1 - a, j);
            return;
        }
        const int nl = w + 2, child = Nb.child[1];
        std::vector<double> C((size_t)nl * 2 * ny);
        for (int J = 1; J <= ny; ++J)
            for (int I = nx - nl + 1; I <= nx; ++I) {
                C[(nx - I) + nl * (J - 1)] = s.Cm(s.blk[child + 1], I, J);
                C[(nx - I) + nl * (J + ny - 1)] = s.Cm(s.blk[child + 3], I, J);
            }
        biq_fine(1, nl, 2 * ny, w, ny, C.data(), out.data());
    } else if (L == L_nbr + 1) {
        const int Y = (ny / 2) * (B.J % 2);
        const int J2 = ny / 2 + 2;
        std::vector<double> C2((size_t)3 * J2);
        for (int j = 0; j <= ny / 2 + 1; ++j)
            for (int a = 0; a <= 2; ++a) C2[(2 - a) + 3 * j] = s.Cm(Nb, nx - 1 + a, j + Y);
        biq_coarse(1, 3, J2, w, ny, C2.data(), out.data());
    } else {
        level_jump(s);
        return;
    }
    for (int j = 1; j <= ny; ++j)
        for (int a = 1; a <= w; ++a) s.Cm(B, 1 - a, j) = out[(a - 1) + w * (j - 1)];
}

/* Fill_Right_C(2) (Fill_Ghost_Cells_C.f90:93-138) */
void fill_right_c(orc_sim& s, int n, int L, int N2, int w) {
    const int nx = s.nx, ny = s.ny;
    Block& B = s.blk[n];
    const Block& Nb = s.blk[N2];
    const int L_nbr = Nb.level;
    std::vector<double> out((size_t)w * ny);
    if (L == L_nbr) {
        if (Nb.isLeaf) {
            for (int j = 1; j <= ny; ++j)
                for (int a = 1; a <= w; ++a) s.Cm(B, nx + a, j) = s.Cm(Nb, a, j);
            return;
        }
        const int nl = w + 2, child = Nb.child[1];
        std::vector<double> C((size_t)nl * 2 * ny);
        for (int J = 1; J <= ny; ++J)
            for (int I = 1; I <= nl; ++I) {
                C[(I - 1) + nl * (J - 1)] = s.Cm(s.blk[child], I, J);
                C[(I - 1) + nl * (J + ny - 1)] = s.Cm(s.blk[child + 2], I, J);
            }
        biq_fine(1, nl, 2 * ny, w, ny, C.data(), out.data());
    } else if (L == L_nbr + 1) {
        const int Y = (ny / 2) * (B.J % 2);
        const int J2 = ny / 2 + 2;
        std::vector<double> C2((size_t)3 * J2);
        for (int j = 0; j <= ny / 2 + 1; ++j)
            for (int a = 0; a <= 2; ++a) C2[a + 3 * j] = s.Cm(Nb, a, j + Y);
        biq_coarse(1, 3, J2, w, ny, C2.data(), out.data());
    } else {
        level_jump(s);
        return;
    }
    for (int j = 1; j <= ny; ++j)
        for (int a = 1; a <= w; ++a) s.Cm(B, nx + a, j) = out[(a - 1) + w * (j - 1)];
}

/* Fill_Bottom_C(2) (Fill_Ghost_Cells_C.f90:142-187) */
void fill_bottom_c(orc_sim& s, int n, int L, int N3, int w) {
    const int nx = s.nx, ny = s.ny;
    Block& B = s.blk[n];
    const Block& Nb = s.blk[N3];
    const int L_nbr = Nb.level;
    std::vector<double> out((size_t)nx * w);
    if (L == L_nbr) {
        if (Nb.isLeaf) {
            for (int i = 1; i <= nx; ++i)
                for (int a = 1; a <= w; ++a) s.Cm(B, i, 1 - a) = s.Cm(Nb, i, ny + 1 - a);
            return;
        }
        const int nl = w + 2, child = Nb.child[1];
        std::vector<double> C((size_t)2 * nx * nl);
        for (int J = ny - nl + 1; J <= ny; ++J)
            for (int I = 1; I <= nx; ++I) {
                C[(I - 1) + 2 * nx * (ny - J)] = s.Cm(s.blk[child + 2], I, J);
                C[(I + nx - 1) + 2 * nx * (ny - J)] = s.Cm(s.blk[child + 3], I, J);
            }
        biq_fine(1, 2 * nx, nl, nx, w, C.data(), out.data());
    } else if (L == L_nbr + 1) {
        const int X = (nx / 2) * (B.I % 2);
        const int I2 = nx / 2 + 2;
        std::vector<double> C2((size_t)I2 * 3);
        for (int i = 0; i <= nx / 2 + 1; ++i)
            for (int a = 0; a <= 2; ++a) C2[i + I2 * (2 - a)] = s.Cm(Nb, i + X, ny - 1 + a);
        biq_coarse(1, I2, 3, nx, w, C2.data(), out.data());
    } else {
        level_jump(s);
        return;
    }
    for (int a = 1; a <= w; ++a)
        for (int i = 1; i <= nx; ++i) s.Cm(B, i, 1 - a) = out[(i - 1) + nx * (a - 1)];
}

/* Fill_Top_C(2) (Fill_Ghost_Cells_C.f90:191-236) */
void fill_top_c(orc_sim& s, int n, int L, int N4, int w) {
    const int nx = s.nx, ny = s.ny;
    Block& B = s.blk[n];
    const Block& Nb = s.blk[N4];
    const int L_nbr = Nb.level;
    std::vector<double> out((size_t)nx * w);
    if (L == L_nbr) {
        if (Nb.isLeaf) {
            for (int i = 1; i <= nx; ++i)
                for (int a = 1; a <= w; ++a) s.Cm(B, i, ny + a) = s.Cm(Nb, i, a);
            return;
        }
        const int nl = w + 2, child = Nb.child[1];
        std::vector<double> C((size_t)2 * nx * nl);
        for (int J = 1; J <= nl; ++J)
            for (int I = 1; I <= nx; ++I) {
                C[(I - 1) + 2 * nx * (J - 1)] = s.Cm(s.blk[child], I, J);
                C[(I + nx - 1) + 2 * nx * (J - 1)] = s.Cm(s.blk[child + 1], I, J);
            }
        biq_fine(1, 2 * nx, nl, nx, w, C.data(), out.data());
    } else if (L == L_nbr + 1) {
        const int X = (nx / 2) * (B.I % 2);
        const int I2 = nx / 2 + 2;
        std::vector<double> C2((size_t)I2 * 3);
        for (int i = 0; i <= nx / 2 + 1; ++i)
            for (int a = 0; a <= 2; ++a) C2[i + I2 * a] = s.Cm(Nb, i + X, a);
        biq_coarse(1, I2, 3, nx, w, C2.data(), out.data());
    } else {
        level_jump(s);
        return;
    }
    for (int a = 1; a <= w; ++a)
        for (int i = 1; i <= nx; ++i) s.Cm(B, i, ny + a) = out[(i - 1) + nx * (a - 1)];
}

/* The four corner fills (Fill_Ghost_Cells_C.f90:240-416, _C2.f90:240-416).
 * corner: 5 = left-bottom, 6 = left-top, 7 = right-bottom, 8 = right-top. */
void fill_corner_c(orc_sim& s, int n, int L, int Nn, int w, int corner) {
    const int nx = s.nx, ny = s.ny;
    Block& B = s.blk[n];
    const Block& Nb = s.blk[Nn];
    const int L_nbr = Nb.level;
    const bool left = (corner == 5 || corner == 6), bottom = (corner == 5 || corner == 7);
    /* ghost cell (a,b), a,b = 1..w, counted outward from the block */
    auto gx = [&](int a) { return left ? 1 - a : nx + a; };
    auto gy = [&](int b) { return bottom ? 1 - b : ny + b; };
    std::vector<double> out((size_t)w * w);
    if (L == L_nbr) {
        if (Nb.isLeaf) {
            /* e.g. Blk(n)%C(-1:0,-1:0) = Blk(N5)%C(nx-1:nx,ny-1:ny) */
            for (int b = 1; b <= w; ++b)
                for (int a = 1; a <= w; ++a) {
                    const int sx = left ? nx + 1 - a : a;
                    const int sy = bottom ? ny + 1 - b : b;
                    s.Cm(B, gx(a), gy(b)) = s.Cm(Nb, sx, sy);
                }
            return;
        }
        const int nl = w + 2;
        /* the neighbour's child touching the corner: 4 (LB), 2 (LT), 3 (RB), 1 (RT) */
        const int off = (corner == 5) ? 3 : (corner == 6) ? 1 : (corner == 7) ? 2 : 0;
        const Block& ch = s.blk[Nb.child[1] + off];
        std::vector<double> C((size_t)nl * nl);
        for (int J = 1; J <= nl; ++J)
            for (int I = 1; I <= nl; ++I) {
                /* C(k,l) with k,l counted from the corner: source cell index */
                const int sx = left ? nx - I + 1 : I;
                const int sy = bottom ? ny - J + 1 : J;
                C[(I - 1) + nl * (J - 1)] = s.Cm(ch, sx, sy);
            }
        biq_fine(1, nl, nl, w, w, C.data(), out.data());
    } else if (L == L_nbr + 1) {
        const int I = left ? nx - (nx / 2) * (B.I % 2) - 1 : nx / 2 - (nx / 2) * (B.I % 2);
        const int J = bottom ? ny - (ny / 2) * (B.J % 2) - 1 : ny / 2 - (ny / 2) * (B.J % 2);
        double C2[9];
        for (int b = 0; b <= 2; ++b)
            for (int a = 0; a <= 2; ++a) {
                const int ka = left ? 2 - a : a;
                const int kb = bottom ? 2 - b : b;
                C2[ka + 3 * kb] = s.Cm(Nb, I + a, J + b);
            }
        biq_coarse(1, 3, 3, w, w, C2, out.data());
    } else {
        level_jump(s);
        return;
    }
    for (int b = 1; b <= w; ++b)
        for (int a = 1; a <= w; ++a) s.Cm(B, gx(a), gy(b)) = out[(a - 1) + w * (b - 1)];
}

/* Fill_Ghost_Cells_C / _C2 (Fill_Ghost_Cells_C.f90:2-40) */
void fill_ghost_cells_c(orc_sim& s, int w) {
    for (int L = s.LevelMin; L <= s.LevelMax; ++L) {
#pragma omp parallel for schedule(static) num_threads(s.nthreads)
        for (int m = 0; m < s.nLeaf; ++m) {
            const int n = s.LeafBlks[m];
            if (L != s.blk[n].level) continue;
            int Nghbr[9];
            for (int I = 1; I <= 8; ++I) Nghbr[I] = s.resolve(n, I);
            if (Nghbr[1] > 0) fill_left_c(s, n, L, Nghbr[1], w);
            if (Nghbr[2] > 0) fill_right_c(s, n, L, Nghbr[2], w);
            if (Nghbr[3] > 0) fill_bottom_c(s, n, L, Nghbr[3], w);
            if (Nghbr[4] > 0) fill_top_c(s, n, L, Nghbr[4], w);
            for (int k = 5; k <= 8; ++k)
                if (Nghbr[k] > 0) fill_corner_c(s, n, L, Nghbr[k], w, k);
            if (Nghbr[3] < 0) symmetric_3(s, s.blk[n], w);
            if (Nghbr[4] < 0) symmetric_4(s, s.blk[n], w);
        }
    }
}

/* ======================================================================
 *  Fill_Ghost_Cells_hg.f90 (9 populations, h and g, ring 1)
 * ====================================================================== */

/* direction d: 1 left, 2 right, 3 bottom, 4 top, 5..8 corners */
void fill_hg_dir(orc_sim& s, int n, int L, int Nn, int d) {
    const int nx = s.nx, ny = s.ny;
    Block& B = s.blk[n];
    const Block& Nb = s.blk[Nn];
    const int L_nbr = Nb.level;
    const bool edge = d <= 4;
    const bool xdir = (d == 1 || d == 2); /* ghost column */
    /* output cells in the order of the reference's destination section */
    std::vector<std::pair<int, int>> dst;
    if (d == 1)
        for (int j = 1; j <= ny; ++j) dst.push_back({0, j});
    else if (d == 2)
        for (int j = 1; j <= ny; ++j) dst.push_back({nx + 1, j});
    else if (d == 3)
        for (int i = 1; i <= nx; ++i) dst.push_back({i, 0});
    else if (d == 4)
        for (int i = 1; i <= nx; ++i) dst.push_back({i, ny + 1});
    else if (d == 5)
        dst.push_back({0, 0});
    else if (d == 6)
        dst.push_back({0, ny + 1});
    else if (d == 7)
        dst.push_back({nx + 1, 0});
    else
        dst.push_back({nx + 1, ny + 1});
    const int nout = (int)dst.size();
    std::vector<double> oh((size_t)9 * nout), og((size_t)9 * nout);

    if (L == L_nbr) {
        if (Nb.isLeaf) {
            for (int m = 0; m < nout; ++m) {
                int sx = dst[m].first, sy = dst[m].second;
                if (d == 1 || d == 5 || d == 6) sx = nx;
                if (d == 2 || d == 7 || d == 8) sx = 1;
                if (d == 3 || d == 5 || d == 7) sy = ny;
                if (d == 4 || d == 6 || d == 8) sy = 1;
                for (int q = 1; q <= 9; ++q) {
                    s.H(B.h, q, dst[m].first, dst[m].second) = s.H(Nb.h, q, sx, sy);
                    s.H(B.g, q, dst[m].first, dst[m].second) = s.H(Nb.g, q, sx, sy);
                }
            }
            return;
        }
        const int child = Nb.child[1];
        if (edge) {
            /* gather 3 fine layers from 2 children, nearest layer first */
            const int i2 = xdir ? 3 : 2 * nx, j2 = xdir ? 2 * ny : 3;
            std::vector<double> th((size_t)9 * i2 * j2), tg((size_t)9 * i2 * j2);
            auto put = [&](int i, int j, const Block& c, int sx, int sy) {
                for (int q = 1; q <= 9; ++q) {
                    th[(q - 1) + 9 * ((i - 1) + i2 * (j - 1))] = s.H(c.h, q, sx, sy);
                    tg[(q - 1) + 9 * ((i - 1) + i2 * (j - 1))] = s.H(c.g, q, sx, sy);
                }
            };
            if (d == 1) {
                for (int J = 1; J <= ny; ++J)
                    for (int I = nx - 2; I <= nx; ++I) {
                        put(nx - I + 1, J, s.blk[child + 1], I, J);
                        put(nx - I + 1, J + ny, s.blk[child + 3], I, J);
                    }
            } else if (d == 2) {
                for (int J = 1; J <= ny; ++J)
                    for (int I = 1; I <= 3; ++I) {
                        put(I, J, s.blk[child], I, J);
                        put(I, J + ny, s.blk[child + 2], I, J);
                    }
            } else if (d == 3) {
                for (int J = ny - 2; J <= ny; ++J)
                    for (int I = 1; I <= nx; ++I) {
                        put(I, ny - J + 1, s.blk[child + 2], I, J);
                        put(I + nx, ny - J + 1, s.blk[child + 3], I, J);
                    }
            } else {
                for (int J = 1; J <= 3; ++J)
                    for (int I = 1; I <= nx; ++I) {
                        put(I, J, s.blk[child], I, J);
                        put(I + nx, J, s.blk[child + 1], I, J);
                    }
            }
            const int X2 = xdir ? 1 : nx, Y2 = xdir ? ny : 1;
            biq_fine(9, i2, j2, X2, Y2, th.data(), oh.data());
            biq_fine(9, i2, j2, X2, Y2, tg.data(), og.data());
        } else {
            const bool left = (d == 5 || d == 6), bottom = (d == 5 || d == 7);
            const int off = (d == 5) ? 3 : (d == 6) ? 1 : (d == 7) ? 2 : 0;
            const Block& ch = s.blk[child + off];
            double th[81], tg[81];
            for (int J = 1; J <= 3; ++J)
                for (int I = 1; I <= 3; ++I) {
                    const int sx = left ? nx - I + 1 : I;
                    const int sy = bottom ? ny - J + 1 : J;
                    for (int q = 1; q <= 9; ++q) {
                        th[(q - 1) + 9 * ((I - 1) + 3 * (J - 1))] = s.H(ch.h, q, sx, sy);
                        tg[(q - 1) + 9 * ((I - 1) + 3 * (J - 1))] = s.H(ch.g, q, sx, sy);
                    }
                }
            biq_fine(9, 3, 3, 1, 1, th, oh.data());
            biq_fine(9, 3, 3, 1, 1, tg, og.data());
        }
    } else if (L == L_nbr + 1) {
        if (edge) {
            int I2, J2;
            std::vector<double> H2, G2;
            auto put = [&](int a, int b, int sx, int sy) {
                for (int q = 1; q <= 9; ++q) {
                    H2[(q - 1) + 9 * (a + I2 * b)] = s.H(Nb.h, q, sx, sy);
                    G2[(q - 1) + 9 * (a + I2 * b)] = s.H(Nb.g, q, sx, sy);
                }
            };
            if (xdir) {
                I2 = 3;
                J2 = ny / 2 + 2;
                H2.resize((size_t)9 * I2 * J2);
                G2.resize((size_t)9 * I2 * J2);
                const int Y = (ny / 2) * (B.J % 2);
                for (int j = 0; j <= ny / 2 + 1; ++j)
                    for (int a = 0; a <= 2; ++a) {
                        if (d == 1)
                            put(2 - a, j, nx - 1 + a, j + Y);
                        else
                            put(a, j, a, j + Y);
                    }
                biq_coarse(9, I2, J2, 1, ny, H2.data(), oh.data());
                biq_coarse(9, I2, J2, 1, ny, G2.data(), og.data());
            } else {
                I2 = nx / 2 + 2;
                J2 = 3;
                H2.resize((size_t)9 * I2 * J2);
                G2.resize((size_t)9 * I2 * J2);
                const int X = (nx / 2) * (B.I % 2);
                for (int i = 0; i <= nx / 2 + 1; ++i)
                    for (int a = 0; a <= 2; ++a) {
                        if (d == 3)
                            put(i, 2 - a, i + X, ny - 1 + a);
                        else
                            put(i, a, i + X, a);
                    }
                biq_coarse(9, I2, J2, nx, 1, H2.data(), oh.data());
                biq_coarse(9, I2, J2, nx, 1, G2.data(), og.data());
            }
        } else {
            const bool left = (d == 5 || d == 6), bottom = (d == 5 || d == 7);
            const int I = left ? nx - (nx / 2) * (B.I % 2) - 1 : nx / 2 - (nx / 2) * (B.I % 2);
            const int J = bottom ? ny - (ny / 2) * (B.J % 2) - 1 : ny / 2 - (ny / 2) * (B.J % 2);
            double H2[81], G2[81];
            for (int b = 0; b <= 2; ++b)
                for (int a = 0; a <= 2; ++a) {
                    const int ka = left ? 2 - a : a, kb = bottom ? 2 - b : b;
                    for (int q = 1; q <= 9; ++q) {
                        H2[(q - 1) + 9 * (ka + 3 * kb)] = s.H(Nb.h, q, I + a, J + b);
                        G2[(q - 1) + 9 * (ka + 3 * kb)] = s.H(Nb.g, q, I + a, J + b);
                    }
                }
            biq_coarse(9, 3, 3, 1, 1, H2, oh.data());
            biq_coarse(9, 3, 3, 1, 1, G2, og.data());
        }
    } else {
        level_jump(s);
        return;
    }
    for (int m = 0; m < nout; ++m)
        for (int q = 1; q <= 9; ++q) {
            s.H(B.h, q, dst[m].first, dst[m].second) = oh[(q - 1) + 9 * m];
            s.H(B.g, q, dst[m].first, dst[m].second) = og[(q - 1) + 9 * m];
        }
}

/* Fill_Ghost_Cells_hg (Fill_Ghost_Cells_hg.f90:2-49) */
void fill_ghost_cells_hg(orc_sim& s) {
    for (int L = s.LevelMin; L <= s.LevelMax; ++L) {
#pragma omp parallel for schedule(static) num_threads(s.nthreads)
        for (int m = 0; m < s.nLeaf; ++m) {
            const int n = s.LeafBlks[m];
            if (L != s.blk[n].level) continue;
            int Nghbr[9];
            for (int I = 1; I <= 8; ++I) Nghbr[I] = s.resolve(n, I);
            for (int k = 1; k <= 8; ++k)
                if (Nghbr[k] > 0) fill_hg_dir(s, n, L, Nghbr[k], k);
            if (Nghbr[3] < 0) {
                bounce_back_3(s, s.blk[n].h);
                bounce_back_3(s, s.blk[n].g);
            }
            if (Nghbr[4] < 0) {
                bounce_back_4(s, s.blk[n].h);
                bounce_back_4(s, s.blk[n].g);
            }
        }
    }
}

/* ======================================================================
 *  Prolong.f90 and Restrict.f90
 * ====================================================================== */

/* Prolong_Bilinear (Prolong.f90:12-39) + Fill_Children_Data (:105-130) */
void prolong_bilinear(orc_sim& s, int n, int c) {
    const int nx = s.nx, ny = s.ny;
    Block& P = s.blk[n];
    /* Hnew_C, Gnew_C (9,nx,ny); C_C(0:nx+1,0:ny+1) */
    std::vector<double> HC((size_t)9 * nx * ny), GC((size_t)9 * nx * ny);
    std::vector<double> CC((size_t)(nx + 2) * (ny + 2));
    for (int y = 1; y <= ny; ++y)
        for (int x = 1; x <= nx; ++x)
            for (int q = 1; q <= 9; ++q) {
                HC[(q - 1) + 9 * ((x - 1) + nx * (y - 1))] = s.H(P.h, q, x, y);
                GC[(q - 1) + 9 * ((x - 1) + nx * (y - 1))] = s.H(P.g, q, x, y);
            }
    for (int y = 0; y <= ny + 1; ++y)
        for (int x = 0; x <= nx + 1; ++x) CC[x + (nx + 2) * y] = s.Cm(P, x, y);
    s.free_fields(P); /* newly added (02/26/2016), Prolong.f90:26 */

    /* Bilinear_Interpolate_Extrapolate (Prolong.f90:43-70) */
    auto interp_extrap = [&](const std::vector<double>& fin, std::vector<double>& fout) {
        std::vector<double> tmp((size_t)9 * 2 * nx * ny);
        fout.assign((size_t)9 * 2 * nx * 2 * ny, 0.0);
        for (int i = 1; i <= 2 * nx; ++i) {
            const int X = std::max(1, std::min(nx - 1, i / 2));
            const int a = 2 * i - 4 * X + 1, b = 4 - a;
            for (int y = 1; y <= ny; ++y)
                for (int q = 0; q < 9; ++q)
                    tmp[q + 9 * ((i - 1) + 2 * nx * (y - 1))] =
                        b * fin[q + 9 * ((X - 1) + nx * (y - 1))] + a * fin[q + 9 * (X + nx * (y - 1))];
        }
        for (int i = 1; i <= 2 * ny; ++i) {
            const int X = std::max(1, std::min(ny - 1, i / 2));
            const int a = 2 * i - 4 * X + 1, b = 4 - a;
            for (int x = 1; x <= 2 * nx; ++x)
                for (int q = 0; q < 9; ++q)
                    fout[q + 9 * ((x - 1) + 2 * nx * (i - 1))] =
                        b * tmp[q + 9 * ((x - 1) + 2 * nx * (X - 1))] +
                        a * tmp[q + 9 * ((x - 1) + 2 * nx * X)];
        }
        for (auto& v : fout) v = v / 16.0;
    };
    std::vector<double> hF, gF;
    interp_extrap(HC, hF);
    interp_extrap(GC, gF);

    /* Bilinear_Interpolation (Prolong.f90:74-101): C(0:2nx+1,0:2ny+1) */
    const int FX = 2 * nx + 2;
    std::vector<double> CF((size_t)FX * (2 * ny + 2)), tmp((size_t)FX * (ny + 2));
    for (int i = 0; i <= 2 * nx + 1; ++i) {
        const int X = i / 2, a = 2 * i - 4 * X + 1, b = 4 - a;
        for (int y = 0; y <= ny + 1; ++y)
            tmp[i + FX * y] = b * CC[X + (nx + 2) * y] + a * CC[(X + 1) + (nx + 2) * y];
    }
    for (int i = 0; i <= 2 * ny + 1; ++i) {
        const int X = i / 2, a = 2 * i - 4 * X + 1, b = 4 - a;
        for (int x = 0; x <= 2 * nx + 1; ++x)
            CF[x + FX * i] = b * tmp[x + FX * X] + a * tmp[x + FX * (X + 1)];
    }
    for (auto& v : CF) v = v / 16.0;

    /* Fill_Children_Data for c, c+1, c+2, c+3 */
    for (int k = 0; k < 4; ++k) {
        Block& Ch = s.blk[c + k];
        const int Ii = (k % 2) * nx, Jj = (k / 2) * ny;
        for (int J = 1; J <= ny; ++J)
            for (int I = 1; I <= nx; ++I)
                for (int q = 1; q <= 9; ++q) {
                    s.H(Ch.g, q, I, J) = gF[(q - 1) + 9 * ((I + Ii - 1) + 2 * nx * (J + Jj - 1))];
                    s.H(Ch.h, q, I, J) = hF[(q - 1) + 9 * ((I + Ii - 1) + 2 * nx * (J + Jj - 1))];
                }
        for (int J = 0; J <= ny + 1; ++J)
            for (int I = 0; I <= nx + 1; ++I) s.Cm(Ch, I, J) = CF[(I + Ii) + FX * (J + Jj)];
        macro_g(s, Ch);
    }
}

/* Restrict_Bilinear (Restrict.f90:14-65) */
void restrict_bilinear(orc_sim& s, int n) {
    const int nx = s.nx, ny = s.ny;
    Block& P = s.blk[n];
    s.alloc_fields(P); /* allocate and zero (Restrict.f90:155-164) */
    const int FX = 2 * nx;
    std::vector<double> h((size_t)9 * FX * 2 * ny), g(h.size());
    std::vector<double> C((size_t)FX * 2 * ny), Pp(C.size()), Ux(C.size()), Uy(C.size());
    int child = P.child[1];
    for (int j = 0; j <= 1; ++j)
        for (int i = 0; i <= 1; ++i) {
            const Block& ch = s.blk[child];
            for (int y = 1; y <= ny; ++y)
                for (int x = 1; x <= nx; ++x) {
                    const int X = x + nx * i, Y = y + ny * j;
                    for (int q = 1; q <= 9; ++q) {
                        h[(q - 1) + 9 * ((X - 1) + FX * (Y - 1))] = s.H(ch.h, q, x, y);
                        g[(q - 1) + 9 * ((X - 1) + FX * (Y - 1))] = s.H(ch.g, q, x, y);
                    }
                    C[(X - 1) + FX * (Y - 1)] = s.Cm(ch, x, y);
                    Pp[(X - 1) + FX * (Y - 1)] = s.Pm(ch.P, x, y);
                    Ux[(X - 1) + FX * (Y - 1)] = s.Pm(ch.Ux, x, y);
                    Uy[(X - 1) + FX * (Y - 1)] = s.Pm(ch.Uy, x, y);
                }
            child = child + 1;
        }
    std::vector<double> oh((size_t)9 * nx * ny), og(oh.size()), o((size_t)nx * ny);
    bil_fine(9, FX, 2 * ny, nx, ny, h.data(), oh.data());
    bil_fine(9, FX, 2 * ny, nx, ny, g.data(), og.data());
    for (int y = 1; y <= ny; ++y)
        for (int x = 1; x <= nx; ++x)
            for (int q = 1; q <= 9; ++q) {
                s.H(P.h, q, x, y) = oh[(q - 1) + 9 * ((x - 1) + nx * (y - 1))];
                s.H(P.g, q, x, y) = og[(q - 1) + 9 * ((x - 1) + nx * (y - 1))];
            }
    bil_fine(1, FX, 2 * ny, nx, ny, C.data(), o.data());
    for (int y = 1; y <= ny; ++y)
        for (int x = 1; x <= nx; ++x) s.Cm(P, x, y) = o[(x - 1) + nx * (y - 1)];
    bil_fine(1, FX, 2 * ny, nx, ny, Pp.data(), P.P.data());
    bil_fine(1, FX, 2 * ny, nx, ny, Ux.data(), P.Ux.data());
    bil_fine(1, FX, 2 * ny, nx, ny, Uy.data(), P.Uy.data());
}

/* ======================================================================
 *  Neighbors.f90
 * ====================================================================== */

/* Neighbor (Neighbors.f90:19-31) */
void neighbor(orc_sim& s, int p, int n, int n2, int c) {
    if (s.resolve(p, n2) < 0)
        s.blk[n].nb[n2] = s.blk[p].nb[n2]; /* same target as the parent's pointer */
    else
        s.blk[n].nb[n2] = s.child_ptr(s.resolve(p, n2), c);
    const int n1 = n2 + 1 - 2 * ((n2 - 1) % 2); /* opposite neighbour */
    s.blk[n].nb[n1] = s.child_ptr(p, c);
}

/* Diagonal_Neighbor (Neighbors.f90:41-122); SW/NW/SE/NE are the saved
 * targets -5/-6/-7/-8 */
void diagonal_neighbor(orc_sim& s, int p, int n, int c) {
    Block& B = s.blk[n];
    auto through = [&](int k, int slot) {
        return s.resolve(p, k) < 0 ? s.blk[p].nb[k] : s.child_ptr(s.resolve(p, k), slot);
    };
    auto fixed = [&](int k, int code, int slot) {
        return s.resolve(p, k) < 0 ? orc_sim::const_ptr(code) : s.child_ptr(s.resolve(p, k), slot);
    };
    if (c == 1) {
        B.nb[5] = through(5, 4);
        B.nb[6] = fixed(1, -6, 4);
        B.nb[7] = fixed(3, -7, 4);
        B.nb[8] = s.child_ptr(p, 4);
    } else if (c == 2) {
        B.nb[5] = fixed(3, -5, 3);
        B.nb[6] = s.child_ptr(p, 3);
        B.nb[7] = through(7, 3);
        B.nb[8] = fixed(2, -8, 3);
    } else if (c == 3) {
        B.nb[5] = fixed(1, -5, 2);
        B.nb[6] = through(6, 2);
        B.nb[7] = s.child_ptr(p, 2);
        B.nb[8] = fixed(4, -8, 2);
    } else if (c == 4) {
        B.nb[5] = s.child_ptr(p, 1);
        B.nb[6] = fixed(4, -6, 1);
        B.nb[7] = fixed(2, -7, 1);
        B.nb[8] = through(8, 1);
    }
}

/* Find_Neighbors (Neighbors.f90:2-15) */
void find_neighbors(orc_sim& s, int par, int n, int I, int J) {
    const int child = 1 + I + 2 * J;
    neighbor(s, par, n, 1 + I, child + 1 - 2 * I);
    neighbor(s, par, n, 3 + J, child + 2 - 4 * J);
    diagonal_neighbor(s, par, n, child);
}

/* ======================================================================
 *  Block pool (AMR_Rising_2D_OMP.f90:434-452, 517-610)
 * ====================================================================== */

/* Add_Child_Blocks (AMR_Rising_2D_OMP.f90:517-584) */
int add_child_blocks(orc_sim& s, int par, int FreeBlk) {
    int N = FreeBlk - 1;
    if (N + 4 > s.MaxBlks) {
        s.set_err(AMRLBM_ERR_POOL_FULL);
        return AMRLBM_ERR_POOL_FULL;
    }
    for (int i = 1; i <= 4; ++i) s.blk[par].child[i] = N + i;
    s.blk[par].isLeaf = false;
    s.blk[par].hasLeaf = true;
    const int grandpar = s.blk[par].parent;
    if (grandpar > 0) s.blk[grandpar].hasLeaf = false;
    for (int J = 0; J <= 1; ++J)
        for (int I = 0; I <= 1; ++I) {
            N = N + 1;
            Block& B = s.blk[N];
            B.level = s.blk[par].level + 1;
            B.dx = s.blk[par].dx / 2;
            B.I = 2 * s.blk[par].I + I;
            B.J = 2 * s.blk[par].J + J;
            B.parent = par;
            B.child_alloc = true;
            for (int k = 1; k <= 4; ++k) B.child[k] = N;
            find_neighbors(s, par, N, I, J);
            B.isLeaf = true;
            B.hasLeaf = false;
            B.refin = false;
            B.deref = false;
            s.alloc_fields(B);
        }
    s.Nblks = std::max(s.Nblks, N);
    return 0;
}

/* Array_of_Leaf_Blocks (AMR_Rising_2D_OMP.f90:588-610) */
void array_of_leaf_blocks(orc_sim& s) {
    s.LeafBlks.clear();
    for (int n = 1; n <= s.Nblks; ++n)
        if (s.blk[n].isLeaf) s.LeafBlks.push_back(n);
    s.nLeaf = (int)s.LeafBlks.size();
}

/* Determine_Min_Max_Levels (AMR_Rising_2D_OMP.f90:434-452) */
void determine_min_max_levels(orc_sim& s) {
    s.LevelMin = 100;
    s.LevelMax = -100;
    for (int m = 0; m < s.nLeaf; ++m) {
        const int L = s.blk[s.LeafBlks[m]].level;
        s.LevelMin = std::min(s.LevelMin, L);
        s.LevelMax = std::max(s.LevelMax, L);
    }
}

/* ======================================================================
 *  Refine_Derefine.f90
 * ====================================================================== */

void enforce_1_level_jump(orc_sim& s, int n);

/* Check_Level_Jump (Refine_Derefine.f90:74-93) */
void check_level_jump(orc_sim& s, int n, int I) {
    const int b = s.resolve(n, I);
    if (b > 0) {
        if (!s.blk[b].refin && s.blk[b].level == s.blk[n].level - 1) {
            if (s.blk[b].isLeaf) {
                s.blk[b].refin = true;
                enforce_1_level_jump(s, b);
            }
        }
    }
}

/* Enforce_1_Level_Jump (Refine_Derefine.f90:58-70) */
void enforce_1_level_jump(orc_sim& s, int n) {
    for (int I = 1; I <= 8; ++I) check_level_jump(s, n, I);
}

/* Flag_for_refinement (Refine_Derefine.f90:18-54) */
void flag_for_refinement(orc_sim& s, double refinTol) {
    const int minLevels = s.prm.min_levels, maxLevels = s.prm.max_levels;
#pragma omp parallel for schedule(static) num_threads(s.nthreads)
    for (int n = 1; n <= s.Nblks; ++n) {
        Block& B = s.blk[n];
        B.refin = false;
        if (B.isLeaf) {
            if (B.level < minLevels) {
                B.refin = true;
                continue;
            } else if (B.level < maxLevels) {
                const double err = err_interface(s, B);
                if (err > refinTol) {
                    B.refin = true;
                    continue;
                }
            }
        }
    }
    for (int n = 1; n <= s.Nblks; ++n)
        if (s.blk[n].refin) enforce_1_level_jump(s, n);
}

/* Check_Level_Jump_Deref_2D (Refine_Derefine.f90:169-194) */
void check_level_jump_deref(orc_sim& s, int n, int Nb, int c1, int c2) {
    if (!s.blk[n].deref) return;
    const int b = s.resolve(n, Nb);
    if (b > 0) {
        if (!s.blk[b].isLeaf) {
            int c = s.blk[b].child[c1];
            for (int I = 1; I <= 2; ++I) {
                const Block& C = s.blk[c];
                if (C.refin || (!C.isLeaf && !C.deref)) {
                    s.blk[n].deref = false;
                    return;
                }
                c = s.blk[b].child[c2];
            }
        }
    }
}

/* enforce_1_Level_jump_deref_2D (Refine_Derefine.f90:149-165) */
void enforce_deref(orc_sim& s, int n) {
    check_level_jump_deref(s, n, 1, 2, 4);
    check_level_jump_deref(s, n, 2, 1, 3);
    check_level_jump_deref(s, n, 3, 3, 4);
    check_level_jump_deref(s, n, 4, 1, 2);
    check_level_jump_deref(s, n, 5, 4, 4);
    check_level_jump_deref(s, n, 6, 2, 2);
    check_level_jump_deref(s, n, 7, 3, 3);
    check_level_jump_deref(s, n, 8, 1, 1);
}

/* Flag_for_derefinement (Refine_Derefine.f90:97-145) */
void flag_for_derefinement(orc_sim& s, double derefTol) {
    const int minLevels = s.prm.min_levels;
#pragma omp parallel for schedule(static) num_threads(s.nthreads)
    for (int n = 1; n <= s.Nblks; ++n) {
        Block& B = s.blk[n];
        B.deref = false;
        if (B.hasLeaf) {
            if (B.level < minLevels) continue;
            const int c1 = B.child[1], c4 = c1 + 3;
            bool any = false;
            for (int c = c1; c <= c4; ++c) any = any || s.blk[c].refin;
            if (any) continue;
            B.deref = true;
            for (int c = c1; c <= c4; ++c) {
                const double err = err_interface(s, s.blk[c]);
                if (err > derefTol) {
                    B.deref = false;
                    break;
                }
            }
        }
    }
    for (int L = s.LevelMax - 1; L >= s.LevelMin - 1; --L)
        for (int n = 1; n <= s.Nblks; ++n)
            if (s.blk[n].level == L && s.blk[n].deref) enforce_deref(s, n);
}

/* Remove_Children (Refine_Derefine.f90:215-258) */
void remove_children(orc_sim& s, int par) {
    const int c1 = s.blk[par].child[1], c4 = c1 + 3;
    for (int c = c1; c <= c4; ++c) {
        s.blk[c].level = -1;
        s.blk[c].isLeaf = false;
    }
    for (int k = 1; k <= 4; ++k) s.blk[par].child[k] = par;
    s.blk[par].isLeaf = true;
    s.blk[par].hasLeaf = false;
    const int grandpa = s.blk[par].parent;
    if (grandpa > 0) {
        const int s1 = s.blk[grandpa].child[1], s4 = s.blk[grandpa].child[4];
        bool all = true;
        for (int k = s1; k <= s4; ++k) all = all && s.blk[k].isLeaf;
        if (all) s.blk[grandpa].hasLeaf = true;
    }
    for (int c = c1; c <= c4; ++c) {
        s.free_fields(s.blk[c]);
        s.blk[c].child_alloc = false; /* DEALLOCATE( Blk(c)%child ) */
        s.blk[c].gen++;
    }
    s.freelist.push_back(c1);
    s.KK = s.KK + 4;
}

/* Derefine (Refine_Derefine.f90:198-211) */
void derefine(orc_sim& s) {
    for (int n = 1; n <= s.Nblks; ++n)
        if (s.blk[n].deref) {
            restrict_bilinear(s, n);
            remove_children(s, n);
        }
}

/* Refine (Refine_Derefine.f90:262-294) */
int refine(orc_sim& s) {
    for (int L = s.LevelMin; L <= s.LevelMax; ++L) {
        const int nb = s.Nblks; /* DO n = 1, Nblks: bound fixed at loop entry */
        for (int n = 1; n <= nb; ++n) {
            if (s.blk[n].level == L && s.blk[n].refin) {
                int c1;
                if (!s.freelist.empty()) {
                    c1 = s.freelist.front();
                    if (add_child_blocks(s, n, c1)) return s.err;
                    s.KK = s.KK - 4;
                    s.freelist.pop_front();
                } else {
                    c1 = s.Nblks + 1;
                    if (add_child_blocks(s, n, c1)) return s.err;
                }
                prolong_bilinear(s, n, c1);
            }
        }
    }
    return 0;
}

/* Refine_Derefine_Mesh (Refine_Derefine.f90:2-14) */
int refine_derefine_mesh(orc_sim& s, double refinTol, double derefTol) {
    flag_for_refinement(s, refinTol);
    flag_for_derefinement(s, derefTol);
    derefine(s);
    const int rc = refine(s);
    array_of_leaf_blocks(s);
    return rc;
}

/* ======================================================================
 *  Driver start-up (AMR_Rising_2D_OMP.f90:43-231, 493-513)
 * ====================================================================== */

/* Initialize_Base_Block + Fix_Initial_Neighbors_3Blocks
 * (AMR_Rising_2D_OMP.f90:79-138), generalised to nbx x nby */
void initialize_base_blocks(orc_sim& s) {
    const int nbx = s.prm.nbx, nby = s.prm.nby;
    auto id = [&](int bi, int bj) { return 1 + ((bi % nbx + nbx) % nbx) + nbx * bj; };
    for (int bj = 0; bj < nby; ++bj)
        for (int bi = 0; bi < nbx; ++bi) {
            const int N = id(bi, bj);
            Block& B = s.blk[N];
            B.level = 0;
            B.dx = s.prm.dx0;
            B.I = bi;
            B.J = bj;
            B.child_alloc = true;
            for (int k = 1; k <= 4; ++k) B.child[k] = N;
            B.parent = -1;
            const bool lo = bj > 0, hi = bj < nby - 1;
            B.nb[1] = orc_sim::const_ptr(id(bi - 1, bj));
            B.nb[2] = orc_sim::const_ptr(id(bi + 1, bj));
            B.nb[3] = orc_sim::const_ptr(lo ? id(bi, bj - 1) : -3);
            B.nb[4] = orc_sim::const_ptr(hi ? id(bi, bj + 1) : -4);
            B.nb[5] = orc_sim::const_ptr(lo ? id(bi - 1, bj - 1) : -5);
            B.nb[6] = orc_sim::const_ptr(hi ? id(bi - 1, bj + 1) : -6);
            B.nb[7] = orc_sim::const_ptr(lo ? id(bi + 1, bj - 1) : -7);
            B.nb[8] = orc_sim::const_ptr(hi ? id(bi + 1, bj + 1) : -8);
            B.isLeaf = true;
            B.hasLeaf = false;
            B.refin = false;
            B.deref = false;
            if (s.prm.min_levels == 0) s.alloc_fields(B);
        }
    s.Nblks = nbx * nby;
}

/* Initial_Mesh (AMR_Rising_2D_OMP.f90:493-513) */
int initial_mesh(orc_sim& s, int nLevels) {
    for (int L = 1; L <= nLevels; ++L) {
        const int nb = s.Nblks;
        for (int n = 1; n <= nb; ++n)
            if (s.blk[n].level == L - 1)
                if (add_child_blocks(s, n, s.Nblks + 1)) return s.err;
    }
    array_of_leaf_blocks(s);
    return 0;
}

/* Initialize_AMR_Rising_Bubble (AMR_Rising_2D_OMP.f90:142-231) */
void initialize_rising_bubble(orc_sim& s) {
    const Phys& ph = s.ph;
    const int nx = s.nx, ny = s.ny;
    const double R = s.prm.radius, X0 = s.prm.xc, Y0 = s.prm.yc;
    const double dRho3 = (ph.Rhoh - ph.Rhol) / 3.0;
#pragma omp parallel for schedule(static) num_threads(s.nthreads)
    for (int m = 0; m < s.nLeaf; ++m) {
        const int n = s.LeafBlks[m];
        Block& B = s.blk[n];
        const int dx = B.dx;
        for (int j = -1; j <= ny + 2; ++j)
            for (int i = -1; i <= nx + 2; ++i) {
                const double Xc = (double)(B.I * dx * nx) + dx * (i - 0.5);
                const double Yc = (double)(B.J * dx * ny) + dx * (j - 0.5);
                const double Ri = std::sqrt((Xc - X0) * (Xc - X0) + (Yc - Y0) * (Yc - Y0));
                s.Cm(B, i, j) = 0.5 + 0.5 * std::tanh(2.0 * (Ri - R) / ph.W);
            }
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                s.Pm(B.Ux, i, j) = 0;
                s.Pm(B.Uy, i, j) = 0;
                s.Pm(B.P, i, j) = -ph.Sigma / R * s.Cm(B, i, j);
                /* optional: the light phase's hydrostatic head about the
                   bubble centre (amrlbm_params.hydrostatic_start) */
                if (s.prm.hydrostatic_start) {
                    const double Yc = (double)(B.J * dx * ny) + dx * (j - 0.5);
                    s.Pm(B.P, i, j) = s.Pm(B.P, i, j) +
                                      ph.Gy * (ph.Rhoh - ph.Rhol) * (1.0 - s.Cm(B, i, j)) * (Yc - Y0);
                }
            }
        std::vector<double> mu;
        chemical_potential(s, dx, B, mu);
        for (int j = 1; j <= ny; ++j)
            for (int i = 1; i <= nx; ++i) {
                double eDc[10], hlp[10], Gamma[10], heq[10], DcDx, DcDy, ni, nj;
                ed_c(s, dx, B, i, j, eDc);
                gradient_ed(eDc, DcDx, DcDy);
                normal(DcDx, DcDy, ni, nj);
                const double Cij = s.Cm(B, i, j);
                const double Ux = s.Pm(B.Ux, i, j), Uy = s.Pm(B.Uy, i, j);
                const double Rho = ph.Rhol + Cij * (ph.Rhoh - ph.Rhol);
                const double Fb = 0;
                equilibrium(ph, Cij, Ux, Uy, ni, nj, Gamma, heq);
                for (int k = 1; k <= 9; ++k) s.H(B.h, k, i, j) = heq[k];
                const double muij = mu[(i - 1) + nx * (j - 1)];
                for (int k = 1; k <= 9; ++k)
                    hlp[k] = ((Gamma[k] - Wa(k)) * dRho3 + Gamma[k] * muij) *
                                 (eDc[k] - (Ux * DcDx + Uy * DcDy)) +
                             ((double)ey[k] - Uy) * Gamma[k] * Fb;
                const double P = s.Pm(B.P, i, j);
                for (int k = 1; k <= 9; ++k)
                    s.H(B.g, k, i, j) = P * Wa(k) + (Gamma[k] - Wa(k)) * Rho / 3.0 - 0.5 * hlp[k];
            }
    }
}

/* one iteration of the Main_Loop body (AMR_Rising_2D_OMP.f90:304-363) */
int main_loop_step(orc_sim& s) {
    double t = omp_get_wtime();
    auto lap = [&](int k) {  /* phase k's timer (Main_Loop, :316-362) */
        const double t2 = omp_get_wtime();
        s.phase_s[k] += t2 - t;
        t = t2;
    };
    determine_min_max_levels(s);
    fill_ghost_cells_c(s, 2);
    lap(5);
    /* Phase_Field_LBM_h_g_AMR (:381-430) */
#pragma omp parallel for schedule(static) num_threads(s.nthreads)
    for (int m = 0; m < s.nLeaf; ++m) collision(s, s.blk[s.LeafBlks[m]]);
    lap(2);
    fill_ghost_cells_hg(s);
    lap(6);
#pragma omp parallel for schedule(static) num_threads(s.nthreads)
    for (int m = 0; m < s.nLeaf; ++m) {
        Block& B = s.blk[s.LeafBlks[m]];
        stream_field(s, B.h, B.dx);
        stream_field(s, B.g, B.dx);
    }
    lap(3);
#pragma omp parallel for schedule(static) num_threads(s.nthreads)
    for (int m = 0; m < s.nLeaf; ++m) macro_h(s, s.blk[s.LeafBlks[m]]);
    lap(0);
    fill_ghost_cells_c(s, 1);
    lap(4);
#pragma omp parallel for schedule(static) num_threads(s.nthreads)
    for (int m = 0; m < s.nLeaf; ++m) macro_g(s, s.blk[s.LeafBlks[m]]);
    lap(1);
    s.stepcount++;
    if (s.stepcount % s.prm.regrid_every == 0) {
        const int r = refine_derefine_mesh(s, s.prm.refin_tol, s.prm.deref_tol);
        lap(7);
        return r;
    }
    return s.err;
}

}  // namespace

/* ======================================================================
 *  C interface
 * ====================================================================== */
extern "C" {

orc_sim* orc_create(const amrlbm_params* p, int nthreads) {
    if (!p || p->nx < 4 || p->ny < 4 || (p->nx % 2) || (p->ny % 2) || p->max_blks < 1)
        return nullptr;
    orc_sim* s = new orc_sim();
    s->prm = *p;
    if (s->prm.regrid_every < 1) s->prm.regrid_every = 1;
    s->ph = derive_phys(*p);
    s->nx = p->nx;
    s->ny = p->ny;
    s->MaxBlks = p->max_blks;
    s->nthreads = nthreads > 0 ? nthreads : omp_get_max_threads();
    s->blk.resize((size_t)s->MaxBlks + 1);
    return s;
}

void orc_destroy(orc_sim* s) { delete s; }
void orc_set_threads(orc_sim* s, int nthreads) {
    s->nthreads = nthreads > 0 ? nthreads : omp_get_max_threads();
}
int orc_last_error(const orc_sim* s) { return s->err; }
int orc_level_jump_count(const orc_sim* s) { return s->level_jumps; }

void orc_physics(const orc_sim* s, amrlbm_physics* o) {
    o->w = s->ph.W;
    o->sigma = s->ph.Sigma;
    o->beta = s->ph.Beta;
    o->kappa = s->ph.kappa;
    o->tau_l = s->ph.taul;
    o->tau_h = s->ph.tauh;
    o->rho_l = s->ph.Rhol;
    o->rho_h = s->ph.Rhoh;
    o->gy = s->ph.Gy;
    o->m0 = s->ph.M0;
}

void orc_set_physics(orc_sim* s, const amrlbm_physics* o) {
    s->ph.W = o->w;
    s->ph.Sigma = o->sigma;
    s->ph.Beta = o->beta;
    s->ph.kappa = o->kappa;
    s->ph.taul = o->tau_l;
    s->ph.tauh = o->tau_h;
    s->ph.Rhol = o->rho_l;
    s->ph.Rhoh = o->rho_h;
    s->ph.Gy = o->gy;
    s->ph.M0 = o->m0;
    s->ph.wc = 1.0 / (0.5 + s->ph.M0 * 3.0);
}

/* the collision model of g (LBM_Subroutines.f90:179-181): 0 MRT, 1 BGK */
int orc_set_g_collision(orc_sim* s, int model) {
    if (model != 0 && model != 1) return 1;
    s->g_model = model;
    return 0;
}

/* AMR_LBM_Rising_Bubble start-up (AMR_Rising_2D_OMP.f90:49-67) */
int orc_init_rising_bubble(orc_sim* s) {
    s->LevelMin = s->prm.min_levels;
    s->LevelMax = s->prm.min_levels;
    initialize_base_blocks(*s);
    if (initial_mesh(*s, s->LevelMin)) return s->err;
    initialize_rising_bubble(*s);
    while (s->LevelMax < s->prm.max_levels) {
        if (refine_derefine_mesh(*s, s->prm.refin_tol, s->prm.deref_tol)) return s->err;
        initialize_rising_bubble(*s);
        s->LevelMax = s->LevelMax + 1;
    }
    return s->err;
}

int orc_init_fields(orc_sim* s) {
    initialize_rising_bubble(*s);
    return s->err;
}

void orc_phase_times(const orc_sim* s, double out[8]) {
    for (int k = 0; k < 8; ++k) out[k] = s->phase_s[k];
}

int orc_step(orc_sim* s, int nsteps) {
    for (int t = 0; t < nsteps; ++t)
        if (main_loop_step(*s)) return s->err;
    return s->err;
}

void orc_min_max_levels(orc_sim* s) { determine_min_max_levels(*s); }
void orc_set_level_range(orc_sim* s, int lmin, int lmax) {
    s->LevelMin = lmin;
    s->LevelMax = lmax;
}
void orc_fill_c2(orc_sim* s) { fill_ghost_cells_c(*s, 2); }
void orc_fill_c(orc_sim* s) { fill_ghost_cells_c(*s, 1); }
void orc_fill_hg(orc_sim* s) { fill_ghost_cells_hg(*s); }
void orc_collide(orc_sim* s) {
#pragma omp parallel for schedule(static) num_threads(s->nthreads)
    for (int m = 0; m < s->nLeaf; ++m) collision(*s, s->blk[s->LeafBlks[m]]);
}
void orc_stream(orc_sim* s) {
#pragma omp parallel for schedule(static) num_threads(s->nthreads)
    for (int m = 0; m < s->nLeaf; ++m) {
        Block& B = s->blk[s->LeafBlks[m]];
        stream_field(*s, B.h, B.dx);
        stream_field(*s, B.g, B.dx);
    }
}
void orc_macro_h(orc_sim* s) {
#pragma omp parallel for schedule(static) num_threads(s->nthreads)
    for (int m = 0; m < s->nLeaf; ++m) macro_h(*s, s->blk[s->LeafBlks[m]]);
}
void orc_macro_g(orc_sim* s) {
#pragma omp parallel for schedule(static) num_threads(s->nthreads)
    for (int m = 0; m < s->nLeaf; ++m) macro_g(*s, s->blk[s->LeafBlks[m]]);
}
int orc_regrid(orc_sim* s, double refin_tol, double deref_tol) {
    return refine_derefine_mesh(*s, refin_tol, deref_tol);
}

void orc_counts(const orc_sim* s, int32_t out[5]) {
    out[0] = s->Nblks;
    out[1] = s->nLeaf;
    out[2] = s->KK;
    out[3] = s->LevelMin;
    out[4] = s->LevelMax;
}

int orc_get_topology(const orc_sim* s, int32_t* level, int32_t* dx, int32_t* bi, int32_t* bj,
                     int32_t* parent, int32_t* child, int32_t* nbr_owner, int32_t* nbr_slot,
                     uint8_t* flags, int32_t* n_free, int32_t* free_list) {
    for (int n = 1; n <= s->Nblks; ++n) {
        const Block& B = s->blk[n];
        const int i = n - 1;
        if (level) level[i] = B.level;
        if (dx) dx[i] = B.dx;
        if (bi) bi[i] = B.I;
        if (bj) bj[i] = B.J;
        if (parent) parent[i] = B.parent;
        for (int k = 1; k <= 4; ++k)
            if (child) child[4 * i + k - 1] = B.child_alloc ? B.child[k] : 0;
        for (int k = 1; k <= 8; ++k) {
            if (nbr_owner) nbr_owner[8 * i + k - 1] = B.nb[k].owner;
            if (nbr_slot) nbr_slot[8 * i + k - 1] = B.nb[k].slot;
        }
        if (flags)
            flags[i] = (B.isLeaf ? AMRLBM_F_LEAF : 0) | (B.hasLeaf ? AMRLBM_F_HASLEAF : 0) |
                       (B.refin ? AMRLBM_F_REFIN : 0) | (B.deref ? AMRLBM_F_DEREF : 0) |
                       (B.alloc ? AMRLBM_F_ALLOC : 0);
    }
    if (n_free) *n_free = (int32_t)s->freelist.size();
    if (free_list) {
        int k = 0;
        for (int c : s->freelist) free_list[k++] = c;
    }
    return 0;
}

int orc_set_topology(orc_sim* s, int32_t nblks, const int32_t* level, const int32_t* dx,
                     const int32_t* bi, const int32_t* bj, const int32_t* parent,
                     const int32_t* child, const int32_t* nbr_owner, const int32_t* nbr_slot,
                     const uint8_t* flags, int32_t n_free, const int32_t* free_list,
                     int32_t kk) {
    if (nblks < 1 || nblks > s->MaxBlks) return AMRLBM_ERR_ARG;
    for (int n = 1; n <= s->MaxBlks; ++n) {
        Block& B = s->blk[n];
        if (n > nblks) {
            B = Block();
            continue;
        }
        const int i = n - 1;
        B.level = level[i];
        B.dx = dx[i];
        B.I = bi[i];
        B.J = bj[i];
        B.parent = parent[i];
        B.child_alloc = B.level >= 0;
        B.gen = 0;
        for (int k = 1; k <= 4; ++k) B.child[k] = child[4 * i + k - 1];
        for (int k = 1; k <= 8; ++k) {
            B.nb[k].owner = nbr_owner[8 * i + k - 1];
            B.nb[k].slot = nbr_slot[8 * i + k - 1];
            B.nb[k].gen = 0;
        }
        B.isLeaf = flags[i] & AMRLBM_F_LEAF;
        B.hasLeaf = flags[i] & AMRLBM_F_HASLEAF;
        B.refin = flags[i] & AMRLBM_F_REFIN;
        B.deref = flags[i] & AMRLBM_F_DEREF;
        const bool want = flags[i] & AMRLBM_F_ALLOC;
        if (want && !B.alloc) s->alloc_fields(B);
        if (!want && B.alloc) s->free_fields(B);
    }
    s->Nblks = nblks;
    s->freelist.clear();
    for (int k = 0; k < n_free; ++k) s->freelist.push_back(free_list[k]);
    s->KK = kk;
    array_of_leaf_blocks(*s);
    return 0;
}

int orc_get_neighbours(const orc_sim* s, int32_t* nbr) {
    for (int n = 1; n <= s->Nblks; ++n)
        for (int k = 1; k <= 8; ++k)
            nbr[8 * (n - 1) + k - 1] = s->blk[n].isLeaf ? s->resolve_c(n, k) : 0;
    return 0;
}

int orc_get_leaves(const orc_sim* s, int32_t* leaves) {
    for (int m = 0; m < s->nLeaf; ++m) leaves[m] = s->LeafBlks[m];
    return s->nLeaf;
}

int orc_get_block(const orc_sim* s, int id, double* h, double* g, double* C, double* P,
                  double* Ux, double* Uy) {
    if (id < 1 || id > s->Nblks) return AMRLBM_ERR_ARG;
    const Block& B = s->blk[id];
    if (!B.alloc) return AMRLBM_ERR_STATE;
    if (h) std::memcpy(h, B.h.data(), B.h.size() * 8);
    if (g) std::memcpy(g, B.g.data(), B.g.size() * 8);
    if (C) std::memcpy(C, B.C.data(), B.C.size() * 8);
    if (P) std::memcpy(P, B.P.data(), B.P.size() * 8);
    if (Ux) std::memcpy(Ux, B.Ux.data(), B.Ux.size() * 8);
    if (Uy) std::memcpy(Uy, B.Uy.data(), B.Uy.size() * 8);
    return 0;
}

int orc_set_block(orc_sim* s, int id, const double* h, const double* g, const double* C,
                  const double* P, const double* Ux, const double* Uy) {
    if (id < 1 || id > s->Nblks) return AMRLBM_ERR_ARG;
    Block& B = s->blk[id];
    if (!B.alloc) s->alloc_fields(B);
    if (h) std::memcpy(B.h.data(), h, B.h.size() * 8);
    if (g) std::memcpy(B.g.data(), g, B.g.size() * 8);
    if (C) std::memcpy(B.C.data(), C, B.C.size() * 8);
    if (P) std::memcpy(B.P.data(), P, B.P.size() * 8);
    if (Ux) std::memcpy(B.Ux.data(), Ux, B.Ux.size() * 8);
    if (Uy) std::memcpy(B.Uy.data(), Uy, B.Uy.size() * 8);
    return 0;
}

int orc_block_error(const orc_sim* s, int id, double* err) {
    if (id < 1 || id > s->Nblks || !s->blk[id].alloc) return AMRLBM_ERR_ARG;
    *err = err_interface(*s, s->blk[id]);
    return 0;
}

/* Output (AMR_Rising_2D_OMP.f90:456-489) in a fixed order: every leaf's
 * partial sums in (j, i) order, then the partials in leaf-list order (the
 * reference's OpenMP reduction(+) has no fixed order); plus the bubble
 * (1-C) volume, centroid and rise velocity. */
int orc_diag(const orc_sim* s, double out[8]) {
    const Phys& ph = s->ph;
    double Mass = 0, Rho_min = 10, Rho_max = -10, U_max = 0;
    double vol = 0, ysum = 0, vsum = 0, phase = 0;
    bool finite = true;
    for (int m = 0; m < s->nLeaf; ++m) {
        const Block& B = s->blk[s->LeafBlks[m]];
        const int dx = B.dx;
        const double a = (double)(dx * dx);
        double bm = 0, bv = 0, by = 0, bu = 0, bp = 0;
        for (int j = 1; j <= s->ny; ++j)
            for (int i = 1; i <= s->nx; ++i) {
                const double C = s->Cm(B, i, j);
                const double Rho = ph.Rhol + C * (ph.Rhoh - ph.Rhol);
                Rho_min = std::fmin(Rho_min, Rho);
                Rho_max = std::fmax(Rho_max, Rho);
                bm = bm + Rho * a;
                const double uy = s->Pm(B.Uy, i, j);
                U_max = std::fmax(U_max, std::fabs(uy));
                const double yc = (double)(B.J * dx * s->ny) + dx * (j - 0.5);
                const double wgt = (C < 0.5) ? (1.0 - C) * a : 0.0;
                bv = bv + wgt;
                by = by + wgt * yc;
                bu = bu + wgt * uy;
                bp = bp + C * a;
                if (!std::isfinite(C) || !std::isfinite(uy)) finite = false;
            }
        Mass = Mass + bm;
        vol = vol + bv;
        ysum = ysum + by;
        vsum = vsum + bu;
        phase = phase + bp;
    }
    out[0] = Mass;
    out[1] = Rho_min;
    out[2] = Rho_max;
    out[3] = U_max;
    out[4] = vol;
    out[5] = ysum / vol;
    out[6] = vsum / vol;
    out[7] = phase;
    return finite ? 0 : AMRLBM_ERR_NAN;
}

/* ---- single routines ---------------------------------------------------- */
void orc_collision_block(const orc_sim* s, int dx, const double* C, const double* P,
                         const double* Ux, const double* Uy, double* h, double* g) {
    Block B;
    B.dx = dx;
    B.C.assign(C, C + s->csize());
    B.P.assign(P, P + s->psize());
    B.Ux.assign(Ux, Ux + s->psize());
    B.Uy.assign(Uy, Uy + s->psize());
    B.h.assign(h, h + s->hsize());
    B.g.assign(g, g + s->hsize());
    collision(*s, B);
    std::memcpy(h, B.h.data(), s->hsize() * 8);
    std::memcpy(g, B.g.data(), s->hsize() * 8);
}

void orc_macro_g_block(const orc_sim* s, int dx, const double* g, const double* C, double* P,
                       double* Ux, double* Uy) {
    Block B;
    B.dx = dx;
    B.g.assign(g, g + s->hsize());
    B.C.assign(C, C + s->csize());
    B.P.assign(s->psize(), 0.0);
    B.Ux.assign(s->psize(), 0.0);
    B.Uy.assign(s->psize(), 0.0);
    macro_g(*s, B);
    std::memcpy(P, B.P.data(), s->psize() * 8);
    std::memcpy(Ux, B.Ux.data(), s->psize() * 8);
    std::memcpy(Uy, B.Uy.data(), s->psize() * 8);
}

void orc_stream_block(const orc_sim* s, int dx, double* f) {
    std::vector<double> v(f, f + s->hsize());
    stream_field(*s, v, dx);
    std::memcpy(f, v.data(), s->hsize() * 8);
}

void orc_biquadratic_from_fine(int i2, int j2, int X2, int Y2, const double* cin,
                               double* cout) {
    biq_fine(1, i2, j2, X2, Y2, cin, cout);
}
void orc_biquadratic_from_coarse(int I2, int J2, int x2, int y2, const double* cin,
                                 double* cout) {
    biq_coarse(1, I2, J2, x2, y2, cin, cout);
}
void orc_bilinear_from_fine(int i2, int j2, int X2, int Y2, const double* cin, double* cout) {
    bil_fine(1, i2, j2, X2, Y2, cin, cout);
}
void orc_mrt(double s9, const double* geq, double* g) {
    double G[10], Q[10];
    for (int i = 0; i < 9; ++i) {
        G[i + 1] = g[i];
        Q[i + 1] = geq[i];
    }
    mrt(s9, Q, G);
    for (int i = 0; i < 9; ++i) g[i] = G[i + 1];
}
void orc_equilibrium(const orc_sim* s, double C, double U, double V, double ni, double nj,
                     double* gamma, double* heq) {
    double G[10], H[10];
    equilibrium(s->ph, C, U, V, ni, nj, G, H);
    for (int i = 0; i < 9; ++i) {
        gamma[i] = G[i + 1];
        heq[i] = H[i + 1];
    }
}

}  // extern "C"
