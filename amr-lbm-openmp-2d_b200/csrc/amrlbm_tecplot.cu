// amrlbm_tecplot.cu - TecPlot_CellCenter (TecPlot_ASCII.f90:2-86) without a
// graphics stack: the node and cell values of every leaf are evaluated on the
// device from the pool, copied to the host once, and written as the
// reference's ASCII file (FE quadrilateral zone, block data packing).
//
// File layout, as the reference writes it:
//   " Variables = X, Y, Ux, Uy, C, P"                     (list-directed)
//   "Zone N =" I6 ", E =" I6 ", ZONETYPE=FEquadrilateral, DATAPACKING=Block"
//   " VARLOCATION=([3,4,6]=CELLCENTERED), T = "<t>""      (list-directed)
//   X/L0, Y/L0 of the nodes (REAL(4) quotients)          9 per record, F10.3
//   Ux, Uy of the cells                                  8 per record, E14.6
//   C of the nodes (mean of the 4 adjacent cells - 1/2)  9 per record, E14.6
//   P*(D/2)/Sigma of the cells                           8 per record, E14.6
//   the 4 node numbers of every cell                     8 per record, I7
// Nodes are numbered per leaf (leaf-list order), (nx+1) x (ny+1) each, x
// fastest; cells likewise nx x ny. List-directed output is processor-
// dependent in Fortran; the two such lines are written with one leading
// blank and the time as %.17g.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "amrlbm_dev.cuh"
#include "amrlbm_launch.h"

namespace {

// one CTA per leaf m (leaf-list order): node values and coordinates, cell
// values. node_c[Nn], node_xy[2][Nn] (ints), cell[3][Ne]: Ux, Uy, scaled P.
__global__ void k_tecplot(DevState s, double* node_c, int* node_xy, double* cell, double D,
                          double sigma) {
    const int nleaf = s.cnt->nleaf, nx = s.nx, ny = s.ny;
    const size_t Nn = (size_t)nleaf * (nx + 1) * (ny + 1), Ne = (size_t)nleaf * nx * ny;
    for (int m = blockIdx.x; m < nleaf; m += gridDim.x) {
        const int n = s.leaf[m], dx = s.dx[n], bi = s.bi[n], bj = s.bj[n];
        for (int idx = threadIdx.x; idx < (nx + 1) * (ny + 1); idx += blockDim.x) {
            const int I = idx % (nx + 1) + 1, J = idx / (nx + 1) + 1;
            const size_t N = (size_t)m * (nx + 1) * (ny + 1) + idx;
            node_xy[N] = bi * dx * nx + dx * (I - 1);
            node_xy[Nn + N] = bj * dx * ny + dx * (J - 1);
            // 0.25d0*(C(i-1,j-1) + C(i,j-1) + C(i-1,j) + C(i,j)) - 0.5d0
            const double sum = ((s.C[c_idx(s, n, I - 1, J - 1)] + s.C[c_idx(s, n, I, J - 1)]) +
                                s.C[c_idx(s, n, I - 1, J)]) +
                               s.C[c_idx(s, n, I, J)];
            node_c[N] = 0.25 * sum - 0.5;
        }
        for (int idx = threadIdx.x; idx < nx * ny; idx += blockDim.x) {
            const int I = idx % nx + 1, J = idx / nx + 1;
            const size_t E = (size_t)m * nx * ny + idx;
            cell[E] = s.Ux[p_idx(s, n, I, J)];
            cell[Ne + E] = s.Uy[p_idx(s, n, I, J)];
            cell[2 * Ne + E] = ((s.P[p_idx(s, n, I, J)] * 0.5) * D) / sigma;  // P*0.5d0*D/Sigma
        }
    }
}

// Fortran edit descriptors on one record buffer
void put_stars(std::string& o, int w) { o.append((size_t)w, '*'); }

void put_i(std::string& o, long long v, int w) {  // Iw
    char b[32];
    const int k = std::snprintf(b, sizeof b, "%*lld", w, v);
    if (k > w) put_stars(o, w); else o.append(b, (size_t)k);
}

void put_f(std::string& o, double v, int w, int d) {  // Fw.d
    char b[64];
    const int k = std::snprintf(b, sizeof b, "%*.*f", w, d, v);
    if (k > w) put_stars(o, w); else o.append(b, (size_t)k);
}

// Ew.d with the default scale factor: [-]0.d1...dd E+ee (3 exponent digits
// without the E beyond 99), right-justified; NaN and Infinity as names
void put_e(std::string& o, double v, int w, int d) {
    char body[64];
    int k = 0;
    if (std::isnan(v) || std::isinf(v)) {
        const char* t = std::isnan(v) ? "NaN" : (v < 0 ? "-Infinity" : "Infinity");
        k = (int)std::strlen(t);
        std::memcpy(body, t, (size_t)k);
    } else {
        char digs[32];
        int e10 = 0;
        const double a = std::fabs(v);
        if (a == 0.0) {
            std::memset(digs, '0', (size_t)d);
        } else {
            char t[64];
            std::snprintf(t, sizeof t, "%.*e", d - 1, a);  // d.ddddde+XX, correctly rounded
            digs[0] = t[0];
            std::memcpy(digs + 1, t + 2, (size_t)(d - 1));
            e10 = std::atoi(std::strchr(t, 'e') + 1) + 1;
        }
        if (std::signbit(v)) body[k++] = '-';
        body[k++] = '0';
        body[k++] = '.';
        std::memcpy(body + k, digs, (size_t)d);
        k += d;
        const int ae = e10 < 0 ? -e10 : e10;
        k += (ae <= 99) ? std::snprintf(body + k, 16, "E%c%02d", e10 < 0 ? '-' : '+', ae)
                        : std::snprintf(body + k, 16, "%c%03d", e10 < 0 ? '-' : '+', ae);
    }
    if (k > w) {
        put_stars(o, w);
        return;
    }
    o.append((size_t)(w - k), ' ');
    o.append(body, (size_t)k);
}

// items of one array with `per` items a record (format reversion)
template <class PUT>
void put_records(std::string& o, size_t count, int per, PUT put) {
    for (size_t i = 0; i < count; ++i) {
        put(i);
        if ((i + 1) % per == 0 || i + 1 == count) o.push_back('\n');
    }
}

}  // namespace

void launch_tecplot(const DevState& s, cudaStream_t st, int num_sms, double* node_c, int* node_xy,
                    double* cell, double D, double sigma) {
    k_tecplot<<<num_sms * 8, 128, 0, st>>>(s, node_c, node_xy, cell, D, sigma);
    count_launches(1);
}

int tecplot_write(const char* path, int nx, int ny, int nleaf, int L0, double t_value,
                  const double* node_c, const int* node_xy, const double* cell) {
    const size_t Nn = (size_t)nleaf * (nx + 1) * (ny + 1), Ne = (size_t)nleaf * nx * ny;
    std::string o;
    o.reserve(Nn * 48 + Ne * 70 + 256);
    o += " Variables = X, Y, Ux, Uy, C, P\n";
    o += "Zone N =";
    put_i(o, (long long)Nn, 6);
    o += ", E =";
    put_i(o, (long long)Ne, 6);
    o += ", ZONETYPE=FEquadrilateral, DATAPACKING=Block\n";
    char tb[64];
    std::snprintf(tb, sizeof tb, "%.17g", t_value);
    o += " VARLOCATION=([3,4,6]=CELLCENTERED), T = \"";
    o += tb;
    o += "\"\n";
    const float fl0 = (float)L0;  // X(i) / FLOAT(L0): a REAL(4) quotient
    put_records(o, Nn, 9, [&](size_t i) { put_f(o, (double)((float)node_xy[i] / fl0), 10, 3); });
    put_records(o, Nn, 9, [&](size_t i) { put_f(o, (double)((float)node_xy[Nn + i] / fl0), 10, 3); });
    put_records(o, Ne, 8, [&](size_t i) { put_e(o, cell[i], 14, 6); });
    put_records(o, Ne, 8, [&](size_t i) { put_e(o, cell[Ne + i], 14, 6); });
    put_records(o, Nn, 9, [&](size_t i) { put_e(o, node_c[i], 14, 6); });
    put_records(o, Ne, 8, [&](size_t i) { put_e(o, cell[2 * Ne + i], 14, 6); });
    // connect(1:4, E) = N, N+1, N+1+nx+1, N+nx+1 (1-based node numbers)
    put_records(o, 4 * Ne, 8, [&](size_t k) {
        const size_t e = k / 4, c = e % ((size_t)nx * ny), m = e / ((size_t)nx * ny);
        const size_t I = c % nx, J = c / nx;
        const long long N = (long long)(m * (nx + 1) * (ny + 1) + J * (nx + 1) + I) + 1;
        const long long v[4] = {N, N + 1, N + 1 + nx + 1, N + nx + 1};
        put_i(o, v[k % 4], 7);
    });
    FILE* f = std::fopen(path, "wb");
    if (!f) return 1;
    const size_t wrote = std::fwrite(o.data(), 1, o.size(), f);
    const int closed = std::fclose(f);
    return (wrote == o.size() && closed == 0) ? 0 : 1;
}
