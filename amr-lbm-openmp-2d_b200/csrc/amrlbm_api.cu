// amrlbm_api.cu - the extern "C" boundary (include/amrlbm.h): context and
// device block pool, host<->device transfers in the reference's layouts, the
// driver's start-up, CUDA-graph stepping, diagnostics and timing.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "amrlbm.h"
#include "amrlbm_launch.h"

namespace {

size_t round_up(size_t v, size_t m) { return (v + m - 1) / m * m; }

struct GraphEntry {
    cudaGraphExec_t exec = nullptr;
    long long kernels = 0;  // kernels captured in the graph
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> prof;  // (kernel, events)
};

}  // namespace

struct amrlbm_ctx {
    amrlbm_params prm{};
    DevState s{};
    LaunchCfg lc{};
    cudaStream_t st = nullptr;
    std::string err;
    int64_t bytes = 0;
    long long stepcount = 0;
    bool tail_done = true;  // P,U and C ring 1 of the current state are materialised
    std::vector<void*> allocs;
    double* d_diag = nullptr;
    double* d_stage = nullptr;
    size_t stage_doubles = 0;
    int* d_ids = nullptr;
    size_t ids_cap = 0;
    void* d_flush = nullptr;
    size_t flush_bytes = 0;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    bool prof = false;
    double prof_ms[4] = {0, 0, 0, 0};
    long long prof_n[4] = {0, 0, 0, 0};
    long long prof_cells[4] = {0, 0, 0, 0};
    std::map<std::tuple<int, int, int, int, int>, GraphEntry> graphs;
    long long launches0 = 0;
    long long captured = 0, replayed = 0;  // graph kernels: captured once, run per replay
    GraphEntry* prof_pending = nullptr;    // replayed with profiling, events not read yet
    // mixed precision (amrlbm_set_precision): which state is current
    bool mp_stale = true;     // the FP64 pool is newer than the mixed-precision state
    bool fp64_stale = false;  // the mixed-precision state is newer than the FP64 pool
    std::vector<amrlbm_instance> insts;  // batched instances (amrlbm_create_batch)
    unsigned char* d_active = nullptr;   // s.inst_active
    std::vector<double> bubbles;         // several bubbles (x, y, R) (amrlbm_set_bubbles)
    // learned regrid (amrlbm_set_regrid_net)
    amrlbm_net* net = nullptr;
    float net_horizon = 16.f, net_logit = 0.f;
    ForecastNet fnet{};
    float* d_logits = nullptr;  // amrlbm_forecast_blocks: logits and block ids
    int* d_lids = nullptr;
    size_t logit_cap = 0;
    float* d_feat = nullptr;
    int* d_fids = nullptr;
    size_t feat_cap = 0;
};

namespace {

int fail(amrlbm_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

int cuda_fail(amrlbm_ctx* c, cudaError_t e, const char* where) {
    return fail(c, AMRLBM_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                              \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)

template <class T>
T* dalloc(amrlbm_ctx* ctx, size_t n, cudaError_t* e) {
    void* p = nullptr;
    *e = cudaMalloc(&p, n * sizeof(T));
    if (*e == cudaSuccess) {
        cudaMemset(p, 0, n * sizeof(T));
        ctx->allocs.push_back(p);
        ctx->bytes += (int64_t)(n * sizeof(T));
    }
    return (T*)p;
}

PhysD to_physd(const amrlbm_physics& p) {
    PhysD d;
    d.W = p.w;
    d.Sigma = p.sigma;
    d.Beta = p.beta;
    d.kappa = p.kappa;
    d.taul = p.tau_l;
    d.tauh = p.tau_h;
    d.Rhol = p.rho_l;
    d.Rhoh = p.rho_h;
    d.Gy = p.gy;
    d.M0 = p.m0;
    d.wc = 1.0 / (0.5 + d.M0 * 3.0);  // D2Q9_Mod.f90:11
    d.Beta4 = 4.0 * d.Beta;
    d.omwc = 1.0 - d.wc;
    d.dRho = d.Rhoh - d.Rhol;
    d.dRho3 = (d.Rhoh - d.Rhol) / 3.0;
    d.dRho6 = (d.Rhoh - d.Rhol) / 6.0;
    d.itau_d = 1.0 / d.tauh - 1.0 / d.taul;
    d.itaul = 1.0 / d.taul;
    d.taul5 = d.taul + 0.5;
    d.tauh5 = d.tauh + 0.5;
    d.yW = 1.0 / d.W;
    return d;
}

PhysF to_physf(const PhysD& d) {
    PhysF f;
    f.W = (float)d.W;
    f.iW = (float)(1.0 / d.W);
    f.Beta4 = (float)d.Beta4;
    f.kappa = (float)d.kappa;
    f.M0 = (float)d.M0;
    f.wc = (float)d.wc;
    f.omwc = (float)d.omwc;
    f.Rhol = (float)d.Rhol;
    f.Rhoh = (float)d.Rhoh;
    f.dRho = (float)d.dRho;
    f.dRho3 = (float)d.dRho3;
    f.dRho6 = (float)d.dRho6;
    f.Gy = (float)d.Gy;
    f.itau_d = (float)d.itau_d;
    f.itaul = (float)d.itaul;
    f.taul5 = (float)d.taul5;
    f.tauh5 = (float)d.tauh5;
    return f;
}

// ---- field transfer kernels (reference layouts <-> pool layouts) ----------

// Field offsets of a transfer of n blocks, field by field (h, g, C, P, Ux,
// Uy; -1: not transferred): field f of block i is at off[f] + i*size(f) of
// the staging buffer, in the reference's per-block layout.
struct XferLayout {
    long long off[6];
    size_t size[6], total;
};
XferLayout xfer_layout(int nx, int ny, int n, const void* const* fields) {
    XferLayout X;
    const size_t hs = (size_t)9 * (nx + 2) * (ny + 2), cs = (size_t)(nx + 4) * (ny + 4),
                 ps = (size_t)nx * ny;
    const size_t sz[6] = {hs, hs, cs, ps, ps, ps};
    X.total = 0;
    for (int f = 0; f < 6; ++f) {
        X.size[f] = sz[f];
        X.off[f] = fields[f] ? (long long)X.total : -1;
        if (fields[f]) X.total += (size_t)n * sz[f];
    }
    return X;
}

// dir 0: staging -> pool; 1: pool -> staging (layout of xfer_layout)
__global__ void k_transfer(DevState s, const int* ids, int n, double* stage, int dir,
                           XferLayout X) {
    const int nx = s.nx, ny = s.ny;
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const int b = ids[i];
        for (int f = 0; f < 2; ++f) {
            if (X.off[f] < 0) continue;
            double* A = f ? s.Ag : s.Ah;
            double* B = f ? s.Bg : s.Bh;
            double* r = stage + X.off[f] + (size_t)i * X.size[f];
            for (int e = threadIdx.x; e < (int)X.size[f]; e += blockDim.x) {
                const int q = e % 9 + 1, xy = e / 9, x = xy % (nx + 2), y = xy / (nx + 2);
                const bool in = x >= 1 && x <= nx && y >= 1 && y <= ny;
                double* p = in ? &B[b_idx(s, b, q, x, y)] : &A[a_idx(s, b, q, x, y)];
                if (dir == 0)
                    *p = r[e];
                else
                    r[e] = *p;
            }
        }
        if (X.off[2] >= 0) {
            double* r = stage + X.off[2] + (size_t)i * X.size[2];
            for (int e = threadIdx.x; e < (int)X.size[2]; e += blockDim.x) {
                double* p = &s.C[c_idx(s, b, e % (nx + 4) - 1, e / (nx + 4) - 1)];
                if (dir == 0)
                    *p = r[e];
                else
                    r[e] = *p;
            }
        }
        for (int f = 0; f < 3; ++f) {
            if (X.off[3 + f] < 0) continue;
            double* A = f == 0 ? s.P : (f == 1 ? s.Ux : s.Uy);
            double* r = stage + X.off[3 + f] + (size_t)i * X.size[3 + f];
            for (int e = threadIdx.x; e < (int)X.size[3 + f]; e += blockDim.x) {
                double* p = &A[(size_t)b * s.pplane + e];
                if (dir == 0)
                    *p = r[e];
                else
                    r[e] = *p;
            }
        }
    }
}

// device staging of at least `doubles` doubles and `nblocks` block ids;
// grows geometrically (the leaf count changes at every regrid)
int ensure_stage(amrlbm_ctx* ctx, size_t doubles, size_t nblocks) {
    if (doubles > ctx->stage_doubles) {
        const size_t need = doubles + doubles / 2 + 4096;
        if (ctx->d_stage) cudaFree(ctx->d_stage);
        ctx->d_stage = nullptr;
        ctx->stage_doubles = 0;
        CK(cudaMalloc(&ctx->d_stage, need * sizeof(double)));
        ctx->stage_doubles = need;
    }
    if (nblocks > ctx->ids_cap) {
        const size_t need = nblocks + nblocks / 2 + 16;
        if (ctx->d_ids) cudaFree(ctx->d_ids);
        ctx->d_ids = nullptr;
        ctx->ids_cap = 0;
        CK(cudaMalloc(&ctx->d_ids, need * sizeof(int)));
        ctx->ids_cap = need;
    }
    return 0;
}

int device_error(amrlbm_ctx* ctx) {
    int e[2] = {0, 0};
    CK(cudaMemcpy(e, &ctx->s.cnt->error, 2 * sizeof(int), cudaMemcpyDeviceToHost));
    if (e[0] == 0) return 0;
    const int zero[2] = {0, 0};
    CK(cudaMemcpy(&ctx->s.cnt->error, zero, 2 * sizeof(int), cudaMemcpyHostToDevice));
    static const char* names[] = {"ok", "argument", "cuda", "pool full (MaxBlks exceeded)",
                                  "level jump > 1 between neighbours", "non-finite value",
                                  "neighbour pointer into a freed block", "state",
                                  "bounded device wait ran out"};
    const char* nm = (e[0] >= 0 && e[0] <= 8) ? names[e[0]] : "unknown";
    return fail(ctx, e[0], std::string("device: ") + nm + " (info " + std::to_string(e[1]) + ")");
}

// reads the kernel events of the last profiled graph replay (stream idle)
void harvest_profile(amrlbm_ctx* ctx) {
    GraphEntry* ge = ctx->prof_pending;
    ctx->prof_pending = nullptr;
    if (!ge) return;
    for (auto& pe : ge->prof) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, pe.second.first, pe.second.second) == cudaSuccess) {
            ctx->prof_ms[pe.first] += ms;
            ctx->prof_n[pe.first] += 1;
        }
    }
}

int sync_check(amrlbm_ctx* ctx) {
    CK(cudaStreamSynchronize(ctx->st));
    CK(cudaGetLastError());
    harvest_profile(ctx);
    return device_error(ctx);
}

Counters read_counters(amrlbm_ctx* ctx) {
    Counters c;
    cudaMemcpy(&c, ctx->s.cnt, sizeof(Counters), cudaMemcpyDeviceToHost);
    return c;
}

// Refine_Derefine_Mesh as a fixed launch sequence (graph-capturable).
void enqueue_regrid(amrlbm_ctx* ctx, double rt, double dt, bool with_err, bool set_levels) {
    const DevState& s = ctx->s;
    if (with_err) launch_err(s, ctx->lc, ctx->st);
    launch_regrid_flags(s, ctx->st, rt, dt);
    launch_restrict(s, ctx->lc, ctx->st);
    launch_regrid_topo(s, ctx->st, 0, -1, -1, set_levels ? 1 : 0);
    launch_build_plans(s, ctx->lc, ctx->st);
    launch_prolong(s, ctx->lc, ctx->st);
}

// one Main_Loop iteration. consumer of K1 depends on whether the previous
// step materialised P,U; tail = Fill_Ghost_Cells_C + Macroscopic_Values_g_AMR.
struct ProfMark {
    amrlbm_ctx* ctx;
    GraphEntry* ge;
    int kernel;
    cudaEvent_t a = nullptr;
    ProfMark(amrlbm_ctx* c, GraphEntry* g, int k) : ctx(c), ge(g), kernel(k) {
        if (ge && ctx->prof) {
            cudaEvent_t b;
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecordWithFlags(a, ctx->st, cudaEventRecordExternal);
            ge->prof.push_back({kernel, {a, b}});
        }
    }
    ~ProfMark() {
        if (ge && ctx->prof) cudaEventRecordWithFlags(ge->prof.back().second.second, ctx->st,
                                                      cudaEventRecordExternal);
    }
};

// the learned regrid's forecast (a net attached): raises the error of the
// leaves it forecasts before the refine flags are taken
void enqueue_forecast(amrlbm_ctx* ctx) {
    if (ctx->net)
        launch_forecast(ctx->s, ctx->lc, ctx->st, ctx->fnet, 0, nullptr, nullptr, ctx->net_horizon,
                        ctx->prm.refin_tol, ctx->net_logit);
}

// Refine_Derefine_Mesh in a mixed-precision run: the flags from the err that
// the tail computed, and the FP64 restriction (Restrict.f90, FP64 sums) and
// prolongation kernels on FP64 copies of just the blocks they read, converted
// to FP64 before and back after.
void enqueue_regrid_mp(amrlbm_ctx* ctx, double rt, double dt) {
    const DevState& s = ctx->s;
    launch_regrid_flags(s, ctx->st, rt, dt);
    launch_mp_convert(s, ctx->lc, ctx->st, 2, 0);  // children of derefined parents
    launch_restrict(s, ctx->lc, ctx->st);
    launch_mp_convert(s, ctx->lc, ctx->st, 1, 1);  // the derefined parents
    launch_regrid_topo(s, ctx->st, 0, -1, -1, 1);
    launch_build_plans(s, ctx->lc, ctx->st);
    launch_mp_convert(s, ctx->lc, ctx->st, 3, 0);  // refined parents
    launch_prolong(s, ctx->lc, ctx->st);
    launch_mp_convert(s, ctx->lc, ctx->st, 4, 1);  // their new children
}

void enqueue_step_mp(amrlbm_ctx* ctx, GraphEntry* ge, bool prev_tail, bool tail, bool regrid,
                     bool last) {
    const DevState& s = ctx->s;
    {
        ProfMark m(ctx, ge, 0);
        launch_mp_collide(s, ctx->lc, ctx->st, prev_tail, last ? 1 : 0);
    }
    {
        ProfMark m(ctx, ge, 1);
        launch_mp_fill_hg_stream(s, ctx->lc, ctx->st, last ? 1 : 0);
    }
    if (tail) {
        ProfMark m(ctx, ge, 2);
        launch_mp_tail(s, ctx->lc, ctx->st);
    }
    if (regrid) {
        ProfMark m(ctx, ge, 3);
        enqueue_forecast(ctx);
        enqueue_regrid_mp(ctx, ctx->prm.refin_tol, ctx->prm.deref_tol);
    }
}

void enqueue_step(amrlbm_ctx* ctx, GraphEntry* ge, bool prev_tail, bool tail, bool regrid,
                  bool last) {
    const DevState& s = ctx->s;
    if (s.mp.fmt) {
        enqueue_step_mp(ctx, ge, prev_tail, tail, regrid, last);
        return;
    }
    {
        ProfMark m(ctx, ge, 0);
        launch_fill_c(s, ctx->lc, ctx->st, 2, prev_tail ? CONS_COLLIDE_READ : CONS_COLLIDE_FUSED,
                      last ? 1 : 0);
    }
    {
        ProfMark m(ctx, ge, 1);
        launch_fill_hg_stream(s, ctx->lc, ctx->st, last ? 1 : 0);
    }
    if (tail) {
        ProfMark m(ctx, ge, 2);
        launch_fill_c(s, ctx->lc, ctx->st, 1, CONS_MACRO_G);
    }
    if (regrid) {
        ProfMark m(ctx, ge, 3);
        enqueue_forecast(ctx);
        enqueue_regrid(ctx, ctx->prm.refin_tol, ctx->prm.deref_tol, false, true);
    }
}

int set_level_counters(amrlbm_ctx* ctx, int lmin, int lmax) {
    int v[2] = {lmin, lmax};
    CK(cudaMemcpyAsync(&ctx->s.cnt->level_min, v, 2 * sizeof(int), cudaMemcpyHostToDevice,
                       ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return 0;
}

// host copy of the topology arrays for blocks 1..nb (index id)
struct HostTopo {
    std::vector<int> level, dx, bi, bj;
};
int get_leaves_host(amrlbm_ctx* ctx, std::vector<int>& leaves, HostTopo& t) {
    Counters c = read_counters(ctx);
    leaves.resize(c.nleaf);
    if (c.nleaf)
        CK(cudaMemcpy(leaves.data(), ctx->s.leaf, c.nleaf * sizeof(int), cudaMemcpyDeviceToHost));
    const size_t nb = (size_t)c.nblks + 1;
    t.level.resize(nb);
    t.dx.resize(nb);
    t.bi.resize(nb);
    t.bj.resize(nb);
    CK(cudaMemcpy(t.level.data(), ctx->s.level, nb * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(t.dx.data(), ctx->s.dx, nb * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(t.bi.data(), ctx->s.bi, nb * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(t.bj.data(), ctx->s.bj, nb * sizeof(int), cudaMemcpyDeviceToHost));
    return 0;
}

int upload_blocks(amrlbm_ctx* ctx, int n, const int* ids, const double* h, const double* g,
                  const double* C, const double* P, const double* Ux, const double* Uy);

}  // namespace

// ===========================================================================
extern "C" {

void amrlbm_default_params(amrlbm_params* p) {
    const int L0 = 256, nx = 8;
    std::memset(p, 0, sizeof(*p));
    p->nx = nx;
    p->ny = nx;
    p->nbx = 1;
    p->nby = 3;
    p->dx0 = L0 / nx;
    p->min_levels = 1;
    p->max_levels = (int)std::lround(std::log((double)(L0 / nx)) / std::log(2.0));
    p->max_blks = 6 * (L0 / nx) * (L0 / nx);
    p->regrid_every = 1;
    p->rho_l = 0.001;
    p->rho_h = 1.0;
    p->visc_ratio = 100.0;
    p->bo = 40.0;
    p->ar = 40.0;
    p->gy = 0.000005;
    p->w = 5.0;
    p->m0 = 0.03;
    p->radius = L0 / 10.0;
    p->xc = L0 / 2;
    p->yc = L0 / 2;
    p->refin_tol = 0.002;
    p->deref_tol = 0.001;
}

// Set_Rising_Bubble_Parameters (AMR_Rising_2D_OMP.f90:235-263)
int amrlbm_derive_physics(const amrlbm_params* p, amrlbm_physics* o) {
    if (!p || !o) return AMRLBM_ERR_ARG;
    const double R = p->radius;
    const double D = 2.0 * R;
    o->rho_l = p->rho_l;
    o->rho_h = p->rho_h;
    o->gy = p->gy;
    o->sigma = o->gy * (o->rho_h - o->rho_l) * (D * D) / p->bo;
    const double muh = std::sqrt(o->gy * o->rho_h * (o->rho_h - o->rho_l) * ((D * D) * D)) / p->ar;
    const double mul = muh / p->visc_ratio;
    o->tau_h = 3.0 * (muh / o->rho_h);
    o->tau_l = 3.0 * (mul / o->rho_l);
    o->w = p->w;
    o->beta = 12.0 * o->sigma / o->w;
    o->kappa = 1.5 * o->sigma * o->w;
    o->m0 = p->m0;
    return AMRLBM_OK;
}

int amrlbm_create(const amrlbm_params* p, amrlbm_ctx** out) {
    if (!p || !out) return AMRLBM_ERR_ARG;
    *out = nullptr;
    if (p->nx < 4 || p->ny < 4 || (p->nx % 2) || (p->ny % 2) || p->nx * p->ny > 1024 ||
        p->nbx < 1 || p->nby < 1 || p->dx0 < 1 || p->min_levels < 0 ||
        p->max_levels < p->min_levels || p->max_levels >= AMR_MAXLV - 1 || p->max_blks < 1 ||
        p->max_blks < p->nbx * p->nby || p->hydrostatic_start < 0 || p->hydrostatic_start > 1)
        return AMRLBM_ERR_ARG;
    if ((p->dx0 >> p->max_levels) < 1) return AMRLBM_ERR_ARG;  // dx stays an integer >= 1
    if (p->dx0 & (p->dx0 - 1)) return AMRLBM_ERR_ARG;  // powers of two (L0/nx = 2**maxLevels)
    {  // fill plans hold 31-bit offsets into the A pool and 31-bit plan indices
        const size_t ap = (size_t)p->nx + 2;
        const size_t aplane = (p->ny + 2) * ap;
        const size_t r2 = 4 * ((size_t)p->nx + p->ny) + 16;
        if (((size_t)p->max_blks + 1) * 9 * aplane >= (1ull << 31) ||
            ((size_t)p->max_blks + 1) * r2 >= (1ull << 31))
            return AMRLBM_ERR_ARG;
    }
    int dev = 0, cc = 0, sms = 0;
    if (p->device >= 0 && cudaSetDevice(p->device) != cudaSuccess) return AMRLBM_ERR_CUDA;
    if (cudaGetDevice(&dev) != cudaSuccess) return AMRLBM_ERR_CUDA;
    cudaDeviceGetAttribute(&cc, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cc != 10) return AMRLBM_ERR_CUDA;  // built for sm_100a only
    amrlbm_ctx* ctx = new amrlbm_ctx();
    ctx->prm = *p;
    if (ctx->prm.regrid_every < 1) ctx->prm.regrid_every = 1;
    DevState& s = ctx->s;
    const int nx = p->nx, ny = p->ny;
    s.nx = nx;
    s.ny = ny;
    s.max_blks = p->max_blks;
    s.fl_cap = p->max_blks / 4 + 2;
    s.spin_limit = AMR_SPIN_LIMIT;
    s.hold_flag = 0;
    s.ap = nx + 2;                   // columns 0..nx+1 (nx even: rows and planes
    s.aplane = (ny + 2) * s.ap;      // of 16-byte multiples)
    s.bplane = nx * ny;
    s.cp = (int)round_up(nx + 6, 4);
    s.cplane = (int)round_up((size_t)(ny + 4) * s.cp, 16);
    s.pplane = nx * ny;
    s.min_levels = p->min_levels;
    s.g_model = AMRLBM_G_MRT;
    s.max_levels = p->max_levels;
    amrlbm_physics ph;
    amrlbm_derive_physics(p, &ph);
    s.ph = to_physd(ph);
    const size_t NB = (size_t)p->max_blks + 1;
    cudaError_t e = cudaSuccess;
#define AL(field, T, n)                                            \
    s.field = dalloc<T>(ctx, (n), &e);                             \
    if (e != cudaSuccess) {                                        \
        int r = cuda_fail(ctx, e, "cudaMalloc " #field);           \
        amrlbm_destroy(ctx);                                       \
        return r;                                                  \
    }
    AL(Ah, double, NB * 9 * s.aplane);
    AL(Ag, double, NB * 9 * s.aplane);
    AL(Bh, double, NB * 9 * s.bplane);
    AL(Bg, double, NB * 9 * s.bplane);
    AL(C, double, NB * s.cplane);
    AL(P, double, NB * s.pplane);
    AL(Ux, double, NB * s.pplane);
    AL(Uy, double, NB * s.pplane);
    AL(err, double, NB);
    AL(level, int, NB);
    AL(dx, int, NB);
    AL(bi, int, NB);
    AL(bj, int, NB);
    AL(parent, int, NB);
    AL(child, int, 4 * NB);
    AL(nb_owner, int, 8 * NB);
    AL(nb_slot, int, 8 * NB);
    AL(nb_gen, int, 8 * NB);
    AL(gen, int, NB);
    AL(nbr, int, 8 * NB);
    AL(is_leaf, uint8_t, NB);
    AL(has_leaf, uint8_t, NB);
    AL(refin, uint8_t, NB);
    AL(deref, uint8_t, NB);
    AL(alloc, uint8_t, NB);
    AL(child_alloc, uint8_t, NB);
    AL(ring_out, uint8_t, NB);
    AL(ring_done, int, NQUEUES * NB);
    AL(leaf, int, NB);
    AL(lvl_leaf, int, NB);
    AL(lvl_off, int, AMR_MAXLV + 1);
    AL(nbinfo, int, NB * NBI_STRIDE);
    AL(plan_c2, int, NB * PLAN_INTS * (size_t)(4 * (nx + ny) + 16));
    AL(plan_c1, int, NB * PLAN_INTS * (size_t)(2 * (nx + ny) + 4));
    AL(plan_hg, int, NB * PLAN_INTS * (size_t)(2 * (nx + ny) + 4));
    // a fine leaf reads at most half a side plus two cells of a coarser
    // neighbour's ring per side, and five cells per corner
    s.fmax = 2 * (nx > ny ? nx : ny) + 28;
    AL(frn_c, int, NB * 11 * (size_t)s.fmax);
    AL(frn_hg, int, NB * 11 * (size_t)s.fmax);
    AL(fillinfo, int, NQUEUES);
    AL(freelist, int, (size_t)s.fl_cap);
    AL(ref_list, int, NB);
    AL(ref_c1, int, NB);
    AL(der_list, int, NB);
    AL(cnt, Counters, 1);
    AL(queue, unsigned, 4 * NQUEUES);
    ctx->d_diag = dalloc<double>(ctx, 9 + 9 * NB, &e);
    if (e != cudaSuccess) {
        int r = cuda_fail(ctx, e, "cudaMalloc diag");
        amrlbm_destroy(ctx);
        return r;
    }
#undef AL
    ctx->lc.num_sms = sms;
    ctx->lc.grid_queue = sms * 4;
    ctx->lc.grid_leaves = sms * 4;
    if (cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&ctx->t0) != cudaSuccess || cudaEventCreate(&ctx->t1) != cudaSuccess) {
        amrlbm_destroy(ctx);
        return AMRLBM_ERR_CUDA;
    }
    launch_reset_queues(s, ctx->st);  // the level-ordered kernels start from zero counters
    cudaDeviceSynchronize();
    ctx->launches0 = launches_issued();
    *out = ctx;
    return AMRLBM_OK;
}

int amrlbm_destroy(amrlbm_ctx* ctx) {
    if (!ctx) return AMRLBM_OK;
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    for (auto& kv : ctx->graphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        for (auto& pe : kv.second.prof) {
            cudaEventDestroy(pe.second.first);
            cudaEventDestroy(pe.second.second);
        }
    }
    for (void* p : ctx->allocs) cudaFree(p);
    if (ctx->d_stage) cudaFree(ctx->d_stage);
    if (ctx->d_ids) cudaFree(ctx->d_ids);
    if (ctx->d_flush) cudaFree(ctx->d_flush);
    if (ctx->d_feat) cudaFree(ctx->d_feat);
    if (ctx->d_fids) cudaFree(ctx->d_fids);
    if (ctx->d_logits) cudaFree(ctx->d_logits);
    if (ctx->d_lids) cudaFree(ctx->d_lids);
    if (ctx->t0) cudaEventDestroy(ctx->t0);
    if (ctx->t1) cudaEventDestroy(ctx->t1);
    if (ctx->st) cudaStreamDestroy(ctx->st);
    delete ctx;
    return AMRLBM_OK;
}

// the captured intervals hold DevState by value and the kernel variants of
// the settings they were captured with
void drop_graphs(amrlbm_ctx* ctx) {
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    for (auto& kv : ctx->graphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        for (auto& pe : kv.second.prof) {
            cudaEventDestroy(pe.second.first);
            cudaEventDestroy(pe.second.second);
        }
    }
    ctx->graphs.clear();
    ctx->prof_pending = nullptr;
}

// The FP64 pool made current (converted back from the mixed-precision state
// after amrlbm_step ran in FP16/BF16) before a call that reads or writes it;
// `writes`: the call changes the FP64 state, which the next mixed-precision
// step then converts again.
void ensure_fp64(amrlbm_ctx* ctx, bool writes) {
    if (ctx->s.mp.fmt && ctx->fp64_stale) {
        launch_mp_convert(ctx->s, ctx->lc, ctx->st, 0, 0);
        ctx->fp64_stale = false;
    }
    if (writes) ctx->mp_stale = true;
}

int amrlbm_set_physics(amrlbm_ctx* ctx, const amrlbm_physics* phys) {
    if (!ctx || !phys) return AMRLBM_ERR_ARG;
    ctx->s.ph = to_physd(*phys);
    ctx->s.mp.ph = to_physf(ctx->s.ph);
    drop_graphs(ctx);
    return AMRLBM_OK;
}

int amrlbm_set_g_collision(amrlbm_ctx* ctx, int32_t model) {
    if (!ctx || (model != AMRLBM_G_MRT && model != AMRLBM_G_BGK)) return AMRLBM_ERR_ARG;
    ctx->s.g_model = model;
    drop_graphs(ctx);
    return AMRLBM_OK;
}

int amrlbm_set_precision(amrlbm_ctx* ctx, int32_t precision) {
    if (!ctx || precision < AMRLBM_FP64 || precision > AMRLBM_BF16) return AMRLBM_ERR_ARG;
    DevState& s = ctx->s;
    if (precision != AMRLBM_FP64 && (s.nx != s.ny || (s.nx != 8 && s.nx != 16)))
        return fail(ctx, AMRLBM_ERR_ARG, "mixed precision needs 8x8 or 16x16 blocks");
    if (precision == s.mp.fmt) return AMRLBM_OK;
    ensure_fp64(ctx, false);
    if (precision != AMRLBM_FP64 && !s.mp.C) {
        const size_t NB = (size_t)ctx->prm.max_blks + 1;
        cudaError_t e = cudaSuccess;
#define ALM(field, T, n)                                                   \
        s.mp.field = dalloc<T>(ctx, (n), &e);                              \
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaMalloc mp." #field);
        ALM(C, float, NB * s.cplane);
        ALM(P, float, NB * s.pplane);
        ALM(Ux, float, NB * s.pplane);
        ALM(Uy, float, NB * s.pplane);
        ALM(A1h, float, NB * s.aplane);
        ALM(A1g, float, NB * s.aplane);
        ALM(B1h, float, NB * s.bplane);
        ALM(B1g, float, NB * s.bplane);
        ALM(Adh, unsigned short, NB * 9 * s.aplane);
        ALM(Adg, unsigned short, NB * 9 * s.aplane);
        ALM(Bdh, unsigned short, NB * 9 * s.bplane);
        ALM(Bdg, unsigned short, NB * 9 * s.bplane);
#undef ALM
    }
    s.mp.fmt = precision;
    // FP16 keeps the deviations in its normal range with power-of-two scales
    // (exact); BF16 has FP32's exponent range and needs none
    s.mp.sh = precision == AMRLBM_FP16 ? 16.f : 1.f;
    s.mp.sg = precision == AMRLBM_FP16 ? 4096.f : 1.f;
    s.mp.ish = 1.f / s.mp.sh;
    s.mp.isg = 1.f / s.mp.sg;
    s.mp.ph = to_physf(s.ph);
    ctx->mp_stale = true;
    ctx->fp64_stale = false;
    drop_graphs(ctx);
    launch_mp_prepare(s, ctx->lc);
    return sync_check(ctx);
}

int amrlbm_set_launch(amrlbm_ctx* ctx, int32_t ctas_per_sm) {
    if (!ctx || ctas_per_sm < 0 || ctas_per_sm > 32) return AMRLBM_ERR_ARG;
    ctx->lc.mp_ctas = ctas_per_sm;
    drop_graphs(ctx);
    return AMRLBM_OK;
}

int amrlbm_get_fill_order(amrlbm_ctx* ctx, int32_t needs_order[3]) {
    if (!ctx || !needs_order) return AMRLBM_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->st));
    int f[NQUEUES];
    CK(cudaMemcpy(f, ctx->s.fillinfo, sizeof(f), cudaMemcpyDeviceToHost));
    needs_order[0] = f[Q_FILLC] != 0;
    needs_order[1] = f[Q_FILLC1] != 0;
    needs_order[2] = f[Q_FILLHG] != 0;
    return AMRLBM_OK;
}

int amrlbm_set_wait_test(amrlbm_ctx* ctx, int32_t spin_limit, int32_t hold_block) {
    if (!ctx || spin_limit < 0 || hold_block < 0 || hold_block > ctx->prm.max_blks)
        return AMRLBM_ERR_ARG;
    ctx->s.spin_limit = spin_limit > 0 ? spin_limit : AMR_SPIN_LIMIT;
    ctx->s.hold_flag = hold_block;
    drop_graphs(ctx);
    return AMRLBM_OK;
}

const char* amrlbm_last_error(const amrlbm_ctx* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int64_t amrlbm_device_bytes(const amrlbm_ctx* ctx) { return ctx ? ctx->bytes : 0; }

int amrlbm_get_counts(amrlbm_ctx* ctx, int32_t counts[5]) {
    if (!ctx || !counts) return AMRLBM_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->st));
    Counters c = read_counters(ctx);
    counts[0] = c.nblks;
    counts[1] = c.nleaf;
    counts[2] = c.kk;
    counts[3] = c.level_min;
    counts[4] = c.level_max;
    return AMRLBM_OK;
}

int amrlbm_set_level_range(amrlbm_ctx* ctx, int32_t lmin, int32_t lmax) {
    if (!ctx) return AMRLBM_ERR_ARG;
    return set_level_counters(ctx, lmin, lmax);
}

int amrlbm_set_topology(amrlbm_ctx* ctx, int32_t nblks, const int32_t* level, const int32_t* dx,
                        const int32_t* bi, const int32_t* bj, const int32_t* parent,
                        const int32_t* child, const int32_t* nbr_owner, const int32_t* nbr_slot,
                        const uint8_t* flags, int32_t n_free, const int32_t* free_list,
                        int32_t kk) {
    if (!ctx || nblks < 1 || nblks > ctx->prm.max_blks || n_free < 0 ||
        n_free > ctx->s.fl_cap - 1 || !level || !dx || !bi || !bj || !parent || !child ||
        !nbr_owner || !nbr_slot || !flags)
        return AMRLBM_ERR_ARG;
    ensure_fp64(ctx, true);
    DevState& s = ctx->s;
    const size_t NB = (size_t)ctx->prm.max_blks + 1;
    std::vector<int> lv(NB, -1), d(NB, 0), I(NB, 0), J(NB, 0), pa(NB, -1), ch(4 * NB, 0),
        no(8 * NB, 0), ns(8 * NB, 0), zero8(8 * NB, 0), zero(NB, 0);
    std::vector<uint8_t> fl[6];
    for (auto& v : fl) v.assign(NB, 0);
    for (int n = 1; n <= nblks; ++n) {
        const int i = n - 1;
        lv[n] = level[i];
        d[n] = dx[i];
        I[n] = bi[i];
        J[n] = bj[i];
        pa[n] = parent[i];
        for (int k = 0; k < 4; ++k) ch[4 * n + k] = child[4 * i + k];
        for (int k = 0; k < 8; ++k) {
            no[8 * n + k] = nbr_owner[8 * i + k];
            ns[8 * n + k] = nbr_slot[8 * i + k];
            if (ns[8 * n + k] < 0 || ns[8 * n + k] > 4) return AMRLBM_ERR_ARG;
            if (ns[8 * n + k] > 0 && (no[8 * n + k] < 1 || no[8 * n + k] > nblks))
                return AMRLBM_ERR_ARG;
        }
        fl[0][n] = (flags[i] & AMRLBM_F_LEAF) ? 1 : 0;
        fl[1][n] = (flags[i] & AMRLBM_F_HASLEAF) ? 1 : 0;
        fl[2][n] = (flags[i] & AMRLBM_F_REFIN) ? 1 : 0;
        fl[3][n] = (flags[i] & AMRLBM_F_DEREF) ? 1 : 0;
        fl[4][n] = (flags[i] & AMRLBM_F_ALLOC) ? 1 : 0;
        fl[5][n] = level[i] >= 0 ? 1 : 0;
        if (level[i] >= AMR_MAXLV - 1) return AMRLBM_ERR_ARG;
    }
    for (int k = 0; k < n_free; ++k)
        if (free_list[k] < 1 || free_list[k] + 3 > nblks) return AMRLBM_ERR_ARG;
    auto up = [&](void* dst, const void* src, size_t bytes) {
        return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->st);
    };
    CK(up(s.level, lv.data(), NB * 4));
    CK(up(s.dx, d.data(), NB * 4));
    CK(up(s.bi, I.data(), NB * 4));
    CK(up(s.bj, J.data(), NB * 4));
    CK(up(s.parent, pa.data(), NB * 4));
    CK(up(s.child, ch.data(), 4 * NB * 4));
    CK(up(s.nb_owner, no.data(), 8 * NB * 4));
    CK(up(s.nb_slot, ns.data(), 8 * NB * 4));
    CK(up(s.nb_gen, zero8.data(), 8 * NB * 4));
    CK(up(s.gen, zero.data(), NB * 4));
    CK(up(s.is_leaf, fl[0].data(), NB));
    CK(up(s.has_leaf, fl[1].data(), NB));
    CK(up(s.refin, fl[2].data(), NB));
    CK(up(s.deref, fl[3].data(), NB));
    CK(up(s.alloc, fl[4].data(), NB));
    CK(up(s.child_alloc, fl[5].data(), NB));
    if (n_free > 0) CK(up(s.freelist, free_list, (size_t)n_free * 4));
    Counters c = read_counters(ctx);
    c.nblks = nblks;
    c.kk = kk;
    c.fl_head = 0;
    c.fl_count = n_free;
    c.error = 0;
    CK(cudaMemcpyAsync(s.cnt, &c, sizeof(Counters), cudaMemcpyHostToDevice, ctx->st));
    launch_regrid_topo(s, ctx->st, 2, -1, -1, 0);
    launch_build_plans(s, ctx->lc, ctx->st);
    ctx->tail_done = true;
    return sync_check(ctx);
}

int amrlbm_get_topology(amrlbm_ctx* ctx, int32_t* level, int32_t* dx, int32_t* bi, int32_t* bj,
                        int32_t* parent, int32_t* child, int32_t* nbr_owner, int32_t* nbr_slot,
                        uint8_t* flags, int32_t* n_free, int32_t* free_list) {
    if (!ctx) return AMRLBM_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->st));
    DevState& s = ctx->s;
    Counters c = read_counters(ctx);
    const size_t nb = (size_t)c.nblks + 1;
    auto down = [&](std::vector<int>& v, const int* src, size_t n) {
        v.resize(n);
        return cudaMemcpy(v.data(), src, n * 4, cudaMemcpyDeviceToHost);
    };
    std::vector<int> lv, d, I, J, pa, ch, no, ns;
    CK(down(lv, s.level, nb));
    CK(down(d, s.dx, nb));
    CK(down(I, s.bi, nb));
    CK(down(J, s.bj, nb));
    CK(down(pa, s.parent, nb));
    CK(down(ch, s.child, 4 * nb));
    CK(down(no, s.nb_owner, 8 * nb));
    CK(down(ns, s.nb_slot, 8 * nb));
    std::vector<uint8_t> fl[6];
    const uint8_t* src[6] = {s.is_leaf, s.has_leaf, s.refin, s.deref, s.alloc, s.child_alloc};
    for (int k = 0; k < 6; ++k) {
        fl[k].resize(nb);
        CK(cudaMemcpy(fl[k].data(), src[k], nb, cudaMemcpyDeviceToHost));
    }
    for (int n = 1; n <= c.nblks; ++n) {
        const int i = n - 1;
        if (level) level[i] = lv[n];
        if (dx) dx[i] = d[n];
        if (bi) bi[i] = I[n];
        if (bj) bj[i] = J[n];
        if (parent) parent[i] = pa[n];
        if (child)
            for (int k = 0; k < 4; ++k) child[4 * i + k] = fl[5][n] ? ch[4 * n + k] : 0;
        for (int k = 0; k < 8; ++k) {
            if (nbr_owner) nbr_owner[8 * i + k] = no[8 * n + k];
            if (nbr_slot) nbr_slot[8 * i + k] = ns[8 * n + k];
        }
        if (flags)
            flags[i] = (fl[0][n] ? AMRLBM_F_LEAF : 0) | (fl[1][n] ? AMRLBM_F_HASLEAF : 0) |
                       (fl[2][n] ? AMRLBM_F_REFIN : 0) | (fl[3][n] ? AMRLBM_F_DEREF : 0) |
                       (fl[4][n] ? AMRLBM_F_ALLOC : 0);
    }
    if (n_free) *n_free = c.fl_count;
    if (free_list && c.fl_count > 0) {
        std::vector<int> ring(s.fl_cap);
        CK(cudaMemcpy(ring.data(), s.freelist, (size_t)s.fl_cap * 4, cudaMemcpyDeviceToHost));
        for (int k = 0; k < c.fl_count; ++k) free_list[k] = ring[(c.fl_head + k) % s.fl_cap];
    }
    return AMRLBM_OK;
}

int amrlbm_get_neighbours(amrlbm_ctx* ctx, int32_t* nbr) {
    if (!ctx || !nbr) return AMRLBM_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->st));
    Counters c = read_counters(ctx);
    const size_t nb = (size_t)c.nblks + 1;
    std::vector<int> v(8 * nb);
    std::vector<uint8_t> lf(nb);
    CK(cudaMemcpy(v.data(), ctx->s.nbr, 8 * nb * 4, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(lf.data(), ctx->s.is_leaf, nb, cudaMemcpyDeviceToHost));
    for (int n = 1; n <= c.nblks; ++n)
        for (int k = 0; k < 8; ++k) nbr[8 * (n - 1) + k] = lf[n] ? v[8 * n + k] : 0;
    return AMRLBM_OK;
}

int amrlbm_get_leaves(amrlbm_ctx* ctx, int32_t* leaves) {
    if (!ctx || !leaves) return AMRLBM_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->st));
    Counters c = read_counters(ctx);
    if (c.nleaf > 0)
        CK(cudaMemcpy(leaves, ctx->s.leaf, (size_t)c.nleaf * 4, cudaMemcpyDeviceToHost));
    return AMRLBM_OK;
}

int amrlbm_upload_fields(amrlbm_ctx* ctx, int32_t n, const int32_t* ids, const double* h,
                         const double* g, const double* C, const double* P, const double* Ux,
                         const double* Uy) {
    if (!ctx || n < 0 || (n > 0 && !ids)) return AMRLBM_ERR_ARG;
    if (n == 0) return AMRLBM_OK;
    ensure_fp64(ctx, true);
    int r = upload_blocks(ctx, n, ids, h, g, C, P, Ux, Uy);
    if (r) return r;
    ctx->tail_done = true;
    return sync_check(ctx);
}

int amrlbm_download_fields(amrlbm_ctx* ctx, int32_t n, const int32_t* ids, double* h, double* g,
                           double* C, double* P, double* Ux, double* Uy) {
    if (!ctx || n < 0 || (n > 0 && !ids)) return AMRLBM_ERR_ARG;
    if (n == 0) return AMRLBM_OK;
    ensure_fp64(ctx, false);
    for (int i = 0; i < n; ++i)
        if (ids[i] < 1 || ids[i] > ctx->prm.max_blks) return AMRLBM_ERR_ARG;
    double* dst[6] = {h, g, C, P, Ux, Uy};
    const void* fl[6] = {h, g, C, P, Ux, Uy};
    const XferLayout X = xfer_layout(ctx->prm.nx, ctx->prm.ny, n, fl);
    if (X.total == 0) return AMRLBM_OK;
    if (int r = ensure_stage(ctx, X.total, (size_t)n)) return r;
    CK(cudaMemcpyAsync(ctx->d_ids, ids, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->st));
    k_transfer<<<ctx->lc.grid_leaves, 256, 0, ctx->st>>>(ctx->s, ctx->d_ids, n, ctx->d_stage, 1, X);
    CK(cudaGetLastError());
    for (int f = 0; f < 6; ++f)  // straight into the caller's arrays
        if (dst[f])
            CK(cudaMemcpyAsync(dst[f], ctx->d_stage + X.off[f], (size_t)n * X.size[f] * 8,
                               cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return device_error(ctx);
}

int amrlbm_upload_block(amrlbm_ctx* ctx, int32_t id, const double* h, const double* g,
                        const double* C, const double* P, const double* Ux, const double* Uy) {
    return amrlbm_upload_fields(ctx, 1, &id, h, g, C, P, Ux, Uy);
}

int amrlbm_download_block(amrlbm_ctx* ctx, int32_t id, double* h, double* g, double* C,
                          double* P, double* Ux, double* Uy) {
    return amrlbm_download_fields(ctx, 1, &id, h, g, C, P, Ux, Uy);
}

int amrlbm_get_block_error(amrlbm_ctx* ctx, double* err) {
    if (!ctx || !err) return AMRLBM_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->st));
    Counters c = read_counters(ctx);
    std::vector<double> e((size_t)c.nblks + 1);
    std::vector<uint8_t> lf((size_t)c.nblks + 1);
    CK(cudaMemcpy(e.data(), ctx->s.err, e.size() * 8, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(lf.data(), ctx->s.is_leaf, lf.size(), cudaMemcpyDeviceToHost));
    for (int n = 1; n <= c.nblks; ++n) err[n - 1] = lf[n] ? e[n] : 0.0;
    return AMRLBM_OK;
}

// Initialize_AMR_Rising_Bubble (AMR_Rising_2D_OMP.f90:142-231): the analytic
// C (tanh profile, both ghost rings) is evaluated on the host like the
// driver does; P, U, h and g are derived from it on the device.
int amrlbm_init_fields(amrlbm_ctx* ctx) {
    if (!ctx) return AMRLBM_ERR_ARG;
    ensure_fp64(ctx, true);
    CK(cudaStreamSynchronize(ctx->st));
    std::vector<int> leaves;
    HostTopo t;
    if (int r = get_leaves_host(ctx, leaves, t)) return r;
    const int nx = ctx->prm.nx, ny = ctx->prm.ny;
    const size_t cs = (size_t)(nx + 4) * (ny + 4);
    std::vector<int> inst;  // batches: the instance of every block
    if (ctx->s.n_inst) {
        inst.resize(t.dx.size());
        CK(cudaMemcpy(inst.data(), ctx->s.inst, inst.size() * sizeof(int), cudaMemcpyDeviceToHost));
    }
    std::vector<double> C(leaves.size() * cs);
    const size_t ps = (size_t)nx * ny;
    const int nb = (int)ctx->bubbles.size() / 3;  // several bubbles: C and P from the nearest
    std::vector<double> P(nb ? leaves.size() * ps : 0);
    for (size_t m = 0; m < leaves.size(); ++m) {
        const int n = leaves[m];
        const int dx = t.dx[n];
        if (nb) {
            const double W = ctx->s.ph.W;
            const PhysD& ph = ctx->s.ph;
            for (int j = -1; j <= ny + 2; ++j)
                for (int i = -1; i <= nx + 2; ++i) {
                    const double Xc = (double)(t.bi[n] * dx * nx) + dx * (i - 0.5);
                    const double Yc = (double)(t.bj[n] * dx * ny) + dx * (j - 0.5);
                    double dmin = 1e300;
                    int kb = 0;
                    for (int k = 0; k < nb; ++k) {
                        const double* b = &ctx->bubbles[3 * k];
                        const double d = std::sqrt((Xc - b[0]) * (Xc - b[0]) + (Yc - b[1]) * (Yc - b[1])) - b[2];
                        if (d < dmin) {
                            dmin = d;
                            kb = k;
                        }
                    }
                    const double c = 0.5 + 0.5 * std::tanh(2.0 * dmin / W);
                    C[m * cs + (i + 1) + (nx + 4) * (j + 1)] = c;
                    if (i >= 1 && i <= nx && j >= 1 && j <= ny) {
                        const double* b = &ctx->bubbles[3 * kb];
                        double pv = -ph.Sigma / b[2] * c;
                        if (ctx->prm.hydrostatic_start)
                            pv = pv + ph.Gy * (ph.Rhoh - ph.Rhol) * (1.0 - c) * (Yc - b[1]);
                        P[m * ps + (i - 1) + nx * (j - 1)] = pv;
                    }
                }
            continue;
        }
        const amrlbm_instance* bi = ctx->s.n_inst ? &ctx->insts[inst[n]] : nullptr;
        const double R = bi ? bi->radius : ctx->prm.radius, X0 = bi ? bi->xc : ctx->prm.xc,
                     Y0 = bi ? bi->yc : ctx->prm.yc, W = bi ? bi->w : ctx->s.ph.W;
        double* c = C.data() + m * cs;
        for (int j = -1; j <= ny + 2; ++j)
            for (int i = -1; i <= nx + 2; ++i) {
                const double Xc = (double)(t.bi[n] * dx * nx) + dx * (i - 0.5);
                const double Yc = (double)(t.bj[n] * dx * ny) + dx * (j - 0.5);
                const double Ri = std::sqrt((Xc - X0) * (Xc - X0) + (Yc - Y0) * (Yc - Y0));
                c[(i + 1) + (nx + 4) * (j + 1)] = 0.5 + 0.5 * std::tanh(2.0 * (Ri - R) / W);
            }
    }
    if (!leaves.empty()) {
        if (int r = upload_blocks(ctx, (int)leaves.size(), leaves.data(), nullptr, nullptr,
                                  C.data(), nb ? P.data() : nullptr, nullptr, nullptr))
            return r;
    }
    launch_init_fields(ctx->s, ctx->lc, ctx->st, ctx->prm.radius, ctx->prm.hydrostatic_start,
                       ctx->prm.yc, nb ? 1 : 0);
    ctx->tail_done = true;
    return sync_check(ctx);
}

// AMR_LBM_Rising_Bubble (AMR_Rising_2D_OMP.f90:49-67) with the base grid
// generalised to nbx x nby blocks (periodic in x, walls in y).
int init_batch(amrlbm_ctx* ctx);

int init_single(amrlbm_ctx* ctx);

int amrlbm_init_rising_bubble(amrlbm_ctx* ctx) {
    if (!ctx) return AMRLBM_ERR_ARG;
    ensure_fp64(ctx, true);
    if (int r = ctx->s.n_inst ? init_batch(ctx) : init_single(ctx)) return r;
    // the regrid statistics count from here (not the start-up rounds)
    CK(cudaMemsetAsync(ctx->s.cnt->rstat, 0, sizeof(ctx->s.cnt->rstat), ctx->st));
    return sync_check(ctx);
}

int init_single(amrlbm_ctx* ctx) {
    const amrlbm_params& p = ctx->prm;
    const int nbx = p.nbx, nby = p.nby, nb = nbx * nby;
    // Initialize_Base_Block + Fix_Initial_Neighbors_3Blocks (:79-138)
    std::vector<int> level(nb, 0), dx(nb, p.dx0), bi(nb), bj(nb), parent(nb, -1), child(4 * nb),
        own(8 * nb), slot(8 * nb, 0);
    std::vector<uint8_t> flags(nb, AMRLBM_F_LEAF | (p.min_levels == 0 ? AMRLBM_F_ALLOC : 0));
    auto id = [&](int x, int y) { return 1 + ((x % nbx + nbx) % nbx) + nbx * y; };
    for (int y = 0; y < nby; ++y)
        for (int x = 0; x < nbx; ++x) {
            const int n = id(x, y), i = n - 1;
            bi[i] = x;
            bj[i] = y;
            for (int k = 0; k < 4; ++k) child[4 * i + k] = n;  // child(:) = self (see DESIGN)
            const bool lo = y > 0, hi = y < nby - 1;
            const int v[8] = {id(x - 1, y),
                              id(x + 1, y),
                              lo ? id(x, y - 1) : -3,
                              hi ? id(x, y + 1) : -4,
                              lo ? id(x - 1, y - 1) : -5,
                              hi ? id(x - 1, y + 1) : -6,
                              lo ? id(x + 1, y - 1) : -7,
                              hi ? id(x + 1, y + 1) : -8};
            for (int k = 0; k < 8; ++k) own[8 * i + k] = v[k];
        }
    if (int r = amrlbm_set_topology(ctx, nb, level.data(), dx.data(), bi.data(), bj.data(),
                                    parent.data(), child.data(), own.data(), slot.data(),
                                    flags.data(), 0, nullptr, 0))
        return r;
    // zero the base blocks' fields
    {
        std::vector<int> ids(nb);
        for (int n = 1; n <= nb; ++n) ids[n - 1] = n;
        const size_t hs = (size_t)9 * (p.nx + 2) * (p.ny + 2), cs = (size_t)(p.nx + 4) * (p.ny + 4),
                     ps = (size_t)p.nx * p.ny;
        std::vector<double> zh(nb * hs, 0.0), zc(nb * cs, 0.0), zp(nb * ps, 0.0);
        if (int r = upload_blocks(ctx, nb, ids.data(), zh.data(), zh.data(), zc.data(), zp.data(),
                                  zp.data(), zp.data()))
            return r;
    }
    // Initial_Mesh (:493-513)
    for (int L = 1; L <= p.min_levels; ++L) {
        launch_flag_level(ctx->s, ctx->st, L - 1);
        launch_regrid_topo(ctx->s, ctx->st, 1, L - 1, L - 1, 0);
        launch_build_plans(ctx->s, ctx->lc, ctx->st);
        launch_zero_children(ctx->s, ctx->lc, ctx->st);
    }
    if (int r = sync_check(ctx)) return r;
    int lmin = p.min_levels, lmax = p.min_levels;
    if (int r = set_level_counters(ctx, lmin, lmax)) return r;
    if (int r = amrlbm_init_fields(ctx)) return r;
    while (lmax < p.max_levels) {
        if (int r = amrlbm_regrid(ctx, p.refin_tol, p.deref_tol)) return r;
        if (int r = amrlbm_init_fields(ctx)) return r;
        lmax = lmax + 1;
        if (int r = set_level_counters(ctx, lmin, lmax)) return r;
    }
    ctx->stepcount = 0;
    ctx->tail_done = true;
    return AMRLBM_OK;
}

int amrlbm_min_max_levels(amrlbm_ctx* ctx, int32_t* lmin, int32_t* lmax) {
    if (!ctx) return AMRLBM_ERR_ARG;
    launch_minmax(ctx->s, ctx->st);
    if (int r = sync_check(ctx)) return r;
    Counters c = read_counters(ctx);
    if (lmin) *lmin = c.level_min;
    if (lmax) *lmax = c.level_max;
    return AMRLBM_OK;
}

int amrlbm_fill_ghost_c2(amrlbm_ctx* ctx) {
    if (!ctx) return AMRLBM_ERR_ARG;
    ensure_fp64(ctx, true);
    launch_fill_c(ctx->s, ctx->lc, ctx->st, 2, CONS_NONE);
    return sync_check(ctx);
}

int amrlbm_phase_field_step(amrlbm_ctx* ctx) {
    if (!ctx) return AMRLBM_ERR_ARG;
    ensure_fp64(ctx, true);
    launch_collide(ctx->s, ctx->lc, ctx->st);
    launch_fill_hg_stream(ctx->s, ctx->lc, ctx->st);
    ctx->tail_done = false;
    return sync_check(ctx);
}

int amrlbm_macro_h(amrlbm_ctx* ctx) {
    if (!ctx) return AMRLBM_ERR_ARG;
    ensure_fp64(ctx, true);
    launch_macro_h(ctx->s, ctx->lc, ctx->st);
    return sync_check(ctx);
}

int amrlbm_fill_ghost_c(amrlbm_ctx* ctx) {
    if (!ctx) return AMRLBM_ERR_ARG;
    ensure_fp64(ctx, true);
    launch_fill_c(ctx->s, ctx->lc, ctx->st, 1, CONS_NONE);
    return sync_check(ctx);
}

int amrlbm_macro_g(amrlbm_ctx* ctx) {
    if (!ctx) return AMRLBM_ERR_ARG;
    ensure_fp64(ctx, true);
    launch_macro_g(ctx->s, ctx->lc, ctx->st);
    ctx->tail_done = true;
    return sync_check(ctx);
}

int amrlbm_regrid(amrlbm_ctx* ctx, double refin_tol, double deref_tol) {
    if (!ctx) return AMRLBM_ERR_ARG;
    ensure_fp64(ctx, true);
    enqueue_regrid(ctx, refin_tol, deref_tol, true, false);
    ctx->tail_done = true;
    return sync_check(ctx);
}

int amrlbm_step(amrlbm_ctx* ctx, int32_t nsteps) {
    if (!ctx || nsteps < 0) return AMRLBM_ERR_ARG;
    if (nsteps == 0) return AMRLBM_OK;
    const int R = ctx->prm.regrid_every;
    if (ctx->s.mp.fmt) {
        if (ctx->mp_stale) launch_mp_convert(ctx->s, ctx->lc, ctx->st, 0, 1);
        ctx->mp_stale = false;
        ctx->fp64_stale = true;
    }
    launch_minmax(ctx->s, ctx->st);  // Determine_Min_Max_Levels
    int done = 0;
    while (done < nsteps) {
        const int phase = (int)(ctx->stepcount % R);
        int chunk = (R == 1) ? 16 : R - phase;  // up to the next regrid
        if (chunk > nsteps - done) chunk = nsteps - done;
        const bool final_chunk = (done + chunk == nsteps);
        const auto key = std::make_tuple(chunk, phase, ctx->tail_done ? 1 : 0, final_chunk ? 1 : 0,
                                         ctx->prof ? 1 : 0);
        if (ctx->prof_pending) {  // the previous replay's events must be read first
            CK(cudaStreamSynchronize(ctx->st));
            harvest_profile(ctx);
        }
        auto it = ctx->graphs.find(key);
        if (it == ctx->graphs.end()) {
            GraphEntry ge;
            const long long k0 = launches_issued();
            CK(cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeThreadLocal));
            bool prev_tail = ctx->tail_done;
            for (int t = 0; t < chunk; ++t) {
                const bool regrid = ((phase + t + 1) % R) == 0;
                const bool tail = regrid || (final_chunk && t == chunk - 1);
                enqueue_step(ctx, &ge, prev_tail, tail, regrid, final_chunk && t == chunk - 1);
                prev_tail = tail;
            }
            cudaGraph_t g;
            CK(cudaStreamEndCapture(ctx->st, &g));
            CK(cudaGraphInstantiate(&ge.exec, g, 0));
            cudaGraphDestroy(g);
            ge.kernels = launches_issued() - k0;
            ctx->captured += ge.kernels;
            it = ctx->graphs.emplace(key, ge).first;
        }
        CK(cudaGraphLaunch(it->second.exec, ctx->st));
        ctx->replayed += it->second.kernels;
        // regrid / tail state after the chunk
        bool last_tail = false;
        for (int t = 0; t < chunk; ++t) {
            const bool regrid = ((phase + t + 1) % R) == 0;
            last_tail = regrid || (final_chunk && t == chunk - 1);
        }
        if (ctx->prof) ctx->prof_pending = &it->second;
        ctx->stepcount += chunk;
        ctx->tail_done = last_tail;
        done += chunk;
    }
    CK(cudaGetLastError());
    return AMRLBM_OK;
}

int amrlbm_sync(amrlbm_ctx* ctx) {
    if (!ctx) return AMRLBM_ERR_ARG;
    return sync_check(ctx);
}

int amrlbm_diag(amrlbm_ctx* ctx, double out[8]) {
    if (!ctx || !out) return AMRLBM_ERR_ARG;
    ensure_fp64(ctx, false);
    launch_diag(ctx->s, ctx->st, ctx->d_diag);
    double o[9];
    CK(cudaMemcpyAsync(o, ctx->d_diag, 9 * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    if (int r = sync_check(ctx)) return r;
    for (int k = 0; k < 8; ++k) out[k] = o[k];
    if (o[8] != 0.0) return fail(ctx, AMRLBM_ERR_NAN, "non-finite C or Uy in a leaf");
    return AMRLBM_OK;
}

int amrlbm_write_tecplot(amrlbm_ctx* ctx, const char* path, int32_t t) {
    if (!ctx || !path) return AMRLBM_ERR_ARG;
    ensure_fp64(ctx, false);
    if (int r = sync_check(ctx)) return r;
    const Counters c = read_counters(ctx);
    const int nx = ctx->prm.nx, ny = ctx->prm.ny, nl = c.nleaf;
    const size_t Nn = (size_t)nl * (nx + 1) * (ny + 1), Ne = (size_t)nl * nx * ny;
    // staging: node C (Nn), cell Ux, Uy, P (3 Ne), node X, Y (2 Nn ints)
    if (int r = ensure_stage(ctx, Nn + 3 * Ne + Nn + 1, 0)) return r;
    double* node_c = ctx->d_stage;
    double* cell = node_c + Nn;
    int* node_xy = reinterpret_cast<int*>(cell + 3 * Ne);
    const double D = 2.0 * ctx->prm.radius;
    std::vector<double> hc(Nn), hcell(3 * Ne);
    std::vector<int> hxy(2 * Nn);
    if (nl > 0) {
        launch_tecplot(ctx->s, ctx->st, ctx->lc.num_sms, node_c, node_xy, cell, D, ctx->s.ph.Sigma);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(hc.data(), node_c, Nn * 8, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(hcell.data(), cell, 3 * Ne * 8, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(hxy.data(), node_xy, 2 * Nn * 4, cudaMemcpyDeviceToHost, ctx->st));
        if (int r = sync_check(ctx)) return r;
    }
    const double tv = (double)t * std::sqrt(ctx->s.ph.Gy / D);  // T*DSQRT(Gy/D)
    if (tecplot_write(path, nx, ny, nl, ctx->prm.dx0 * nx, tv, hc.data(), hxy.data(), hcell.data()))
        return fail(ctx, AMRLBM_ERR_IO, std::string("cannot write ") + path);
    return AMRLBM_OK;
}

int amrlbm_timer_start(amrlbm_ctx* ctx) {
    if (!ctx) return AMRLBM_ERR_ARG;
    CK(cudaEventRecord(ctx->t0, ctx->st));
    return AMRLBM_OK;
}

int amrlbm_timer_stop(amrlbm_ctx* ctx, float* ms) {
    if (!ctx || !ms) return AMRLBM_ERR_ARG;
    CK(cudaEventRecord(ctx->t1, ctx->st));
    CK(cudaEventSynchronize(ctx->t1));
    CK(cudaEventElapsedTime(ms, ctx->t0, ctx->t1));
    CK(cudaStreamSynchronize(ctx->st));
    harvest_profile(ctx);
    return device_error(ctx);
}

int amrlbm_profile_enable(amrlbm_ctx* ctx, int32_t enable) {
    if (!ctx) return AMRLBM_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->st));
    harvest_profile(ctx);
    ctx->prof = enable != 0;
    for (int k = 0; k < 4; ++k) {
        ctx->prof_ms[k] = 0;
        ctx->prof_n[k] = 0;
    }
    return AMRLBM_OK;
}

int amrlbm_profile_read(amrlbm_ctx* ctx, int32_t kernel, double* total_ms, int64_t* launches,
                        int64_t* cells) {
    if (!ctx || kernel < 0 || kernel > 3) return AMRLBM_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->st));
    harvest_profile(ctx);
    if (total_ms) *total_ms = ctx->prof_ms[kernel];
    if (launches) *launches = ctx->prof_n[kernel];
    if (cells) {
        Counters c = read_counters(ctx);
        *cells = (int64_t)c.updates;
    }
    return AMRLBM_OK;
}

int64_t amrlbm_launch_count(const amrlbm_ctx* ctx) {
    return ctx ? (int64_t)(launches_issued() - ctx->launches0 - ctx->captured + ctx->replayed) : 0;
}

int amrlbm_selftest_division(uint64_t n, uint64_t seed, double divisor, uint64_t* mismatches) {
    if (!mismatches) return AMRLBM_ERR_ARG;
    unsigned long long m = 0;
    const int r = selftest_division(n, seed, divisor, &m);
    *mismatches = m;
    return r;
}

int amrlbm_flush_l2(amrlbm_ctx* ctx) {
    if (!ctx) return AMRLBM_ERR_ARG;
    if (!ctx->d_flush) {
        int dev = 0, l2 = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev);
        ctx->flush_bytes = (size_t)(l2 > 0 ? l2 : (126 << 20)) * 2;
        CK(cudaMalloc(&ctx->d_flush, ctx->flush_bytes));
    }
    CK(cudaMemsetAsync(ctx->d_flush, ctx->flush_bytes & 0xff, ctx->flush_bytes, ctx->st));
    return AMRLBM_OK;
}

}  // extern "C"

namespace {
int upload_blocks(amrlbm_ctx* ctx, int n, const int* ids, const double* h, const double* g,
                  const double* C, const double* P, const double* Ux, const double* Uy) {
    for (int i = 0; i < n; ++i)
        if (ids[i] < 1 || ids[i] > ctx->prm.max_blks) return AMRLBM_ERR_ARG;
    const double* src[6] = {h, g, C, P, Ux, Uy};
    const void* fl[6] = {h, g, C, P, Ux, Uy};
    const XferLayout X = xfer_layout(ctx->prm.nx, ctx->prm.ny, n, fl);
    if (X.total == 0) return 0;
    if (int r = ensure_stage(ctx, X.total, (size_t)n)) return r;
    for (int f = 0; f < 6; ++f)  // straight from the caller's arrays
        if (src[f])
            CK(cudaMemcpyAsync(ctx->d_stage + X.off[f], src[f], (size_t)n * X.size[f] * 8,
                               cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->d_ids, ids, (size_t)n * 4, cudaMemcpyHostToDevice, ctx->st));
    k_transfer<<<ctx->lc.grid_leaves, 256, 0, ctx->st>>>(ctx->s, ctx->d_ids, n, ctx->d_stage, 0, X);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(ctx->st));  // the staging buffer is reused by the next call
    return 0;
}
}  // namespace

// ---------------------------------------------------------------------------
// Field download without allocation.
//
// amrlbm_download_fields stages through buffers it grows on demand: device
// memory for the block ids and the staged records (cudaMalloc) and
// page-locked host memory (cudaMallocHost). Some callers cannot have that:
// a host code that sizes all of its device memory once at start-up, as a
// Fortran driver sharing a GPU with other jobs under a fixed memory budget
// does, and an output hook that runs between time steps, where a call into
// the allocator may synchronise the device and would stall the stepping
// stream. The variant below stages through one fixed scratch area per
// device, a file-scope __device__ array, and copies each field straight into
// the caller's array.
//
// Limits: at most AMRLBM_NOALLOC_STAGE_DOUBLES doubles of requested field
// data and AMRLBM_NOALLOC_MAX_BLOCKS blocks per call; larger requests are
// rejected with AMRLBM_ERR_CAPACITY before anything runs. Nothing in the
// scratch has to start at zero: every element the call reads back was
// written earlier in the same call. The scratch is shared by every context
// on the device, so calls that overlap in time on one device (from two host
// threads, or on two contexts' streams) race on it; the caller serialises
// them.
namespace {

static __device__ __align__(256) double g_noalloc_stage[AMRLBM_NOALLOC_STAGE_DOUBLES];
static __device__ __align__(256) int g_noalloc_ids[AMRLBM_NOALLOC_MAX_BLOCKS];

constexpr int kNoallocDevices = 64;
struct NoallocScratch {
    std::atomic<double*> stage{nullptr};
    std::atomic<int*> ids{nullptr};
};
NoallocScratch g_noalloc_scratch[kNoallocDevices];

// Set-up, once per device, with that device current: the device addresses of
// the scratch arrays (cudaGetSymbolAddress allocates nothing). The first call
// on a device does this; a caller that records its work into a stream
// capture makes that first call before the capture starts.
cudaError_t noalloc_scratch(int dev, double** stage, int** ids) {
    if (dev < 0 || dev >= kNoallocDevices) return cudaErrorInvalidDevice;
    NoallocScratch& sc = g_noalloc_scratch[dev];
    double* st = sc.stage.load();
    int* id = sc.ids.load();
    if (!st || !id) {
        cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&st), g_noalloc_stage);
        if (e != cudaSuccess) return e;
        e = cudaGetSymbolAddress(reinterpret_cast<void**>(&id), g_noalloc_ids);
        if (e != cudaSuccess) return e;
        sc.stage.store(st);
        sc.ids.store(id);
    }
    *stage = st;
    *ids = id;
    return cudaSuccess;
}

// k_transfer's pool -> staging direction with the staging laid out field by
// field: field f of block i at stage[off[f] + i*size(f)], in the same
// per-block layout (off[f] < 0: field not requested)
__global__ void k_download_fieldwise(DevState s, const int* ids, int n, double* stage,
                                     long long off0, long long off1, long long off2, long long off3,
                                     long long off4, long long off5) {
    const int nx = s.nx, ny = s.ny;
    const int hs = 9 * (nx + 2) * (ny + 2), cs = (nx + 4) * (ny + 4), ps = nx * ny;
    const long long off[6] = {off0, off1, off2, off3, off4, off5};
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        const int b = ids[i];
        for (int f = 0; f < 2; ++f) {
            if (off[f] < 0) continue;
            const double* A = f ? s.Ag : s.Ah;
            const double* B = f ? s.Bg : s.Bh;
            double* r = stage + off[f] + (size_t)i * hs;
            for (int e = threadIdx.x; e < hs; e += blockDim.x) {
                const int q = e % 9 + 1, xy = e / 9, x = xy % (nx + 2), y = xy / (nx + 2);
                const bool in = x >= 1 && x <= nx && y >= 1 && y <= ny;
                r[e] = in ? B[b_idx(s, b, q, x, y)] : A[a_idx(s, b, q, x, y)];
            }
        }
        if (off[2] >= 0) {
            double* r = stage + off[2] + (size_t)i * cs;
            for (int e = threadIdx.x; e < cs; e += blockDim.x)
                r[e] = s.C[c_idx(s, b, e % (nx + 4) - 1, e / (nx + 4) - 1)];
        }
        for (int f = 0; f < 3; ++f) {
            if (off[3 + f] < 0) continue;
            const double* A = f == 0 ? s.P : (f == 1 ? s.Ux : s.Uy);
            double* r = stage + off[3 + f] + (size_t)i * ps;
            for (int e = threadIdx.x; e < ps; e += blockDim.x) r[e] = A[(size_t)b * s.pplane + e];
        }
    }
}

}  // namespace

extern "C" int amrlbm_download_fields_noalloc(amrlbm_ctx* ctx, int32_t n, const int32_t* ids,
                                              double* h, double* g, double* C, double* P,
                                              double* Ux, double* Uy) {
    if (!ctx || n < 0 || (n > 0 && !ids)) return AMRLBM_ERR_ARG;
    if (n == 0) return AMRLBM_OK;
    for (int i = 0; i < n; ++i)
        if (ids[i] < 1 || ids[i] > ctx->prm.max_blks) return AMRLBM_ERR_ARG;
    const int nx = ctx->prm.nx, ny = ctx->prm.ny;
    const size_t hs = (size_t)9 * (nx + 2) * (ny + 2), cs = (size_t)(nx + 4) * (ny + 4),
                 ps = (size_t)nx * ny;
    double* dst[6] = {h, g, C, P, Ux, Uy};
    const size_t sz[6] = {hs, hs, cs, ps, ps, ps};
    long long off[6];
    size_t used = 0;
    for (int f = 0; f < 6; ++f) {
        off[f] = dst[f] ? (long long)used : -1;
        if (dst[f]) used += (size_t)n * sz[f];
    }
    if (n > AMRLBM_NOALLOC_MAX_BLOCKS || used > (size_t)AMRLBM_NOALLOC_STAGE_DOUBLES)
        return AMRLBM_ERR_CAPACITY;
    if (used == 0) return AMRLBM_OK;
    ensure_fp64(ctx, false);  // kernels only: no allocation
    // the device that holds the context's pool, current for this call
    cudaPointerAttributes pa;
    if (cudaPointerGetAttributes(&pa, ctx->s.C) != cudaSuccess) return AMRLBM_ERR_CUDA;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return AMRLBM_ERR_CUDA;
    if (prev != pa.device && cudaSetDevice(pa.device) != cudaSuccess) return AMRLBM_ERR_CUDA;
    int rc = AMRLBM_OK;
    double* stage = nullptr;
    int* dids = nullptr;
    cudaError_t e = noalloc_scratch(pa.device, &stage, &dids);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dids, ids, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, ctx->st);
    if (e == cudaSuccess) {
        k_download_fieldwise<<<ctx->lc.grid_leaves, 256, 0, ctx->st>>>(
            ctx->s, dids, n, stage, off[0], off[1], off[2], off[3], off[4], off[5]);
        count_launches(1);
        e = cudaGetLastError();
    }
    for (int f = 0; f < 6 && e == cudaSuccess; ++f)
        if (dst[f])
            e = cudaMemcpyAsync(dst[f], stage + off[f], (size_t)n * sz[f] * sizeof(double),
                                cudaMemcpyDeviceToHost, ctx->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
    if (e != cudaSuccess) rc = AMRLBM_ERR_CUDA;
    if (rc == AMRLBM_OK) {  // a pending device-side error status, as the other calls report it
        int st[2] = {0, 0};
        if (cudaMemcpy(st, &ctx->s.cnt->error, sizeof(st), cudaMemcpyDeviceToHost) != cudaSuccess) {
            rc = AMRLBM_ERR_CUDA;
        } else if (st[0] != 0) {
            // reported once, then cleared as amrlbm_download_fields does, by a
            // copy from this stack array (no allocation)
            rc = st[0];
            const int zero[2] = {0, 0};
            if (cudaMemcpy(&ctx->s.cnt->error, zero, sizeof(zero), cudaMemcpyHostToDevice) !=
                cudaSuccess)
                rc = AMRLBM_ERR_CUDA;
        }
    }
    if (prev != pa.device) cudaSetDevice(prev);
    return rc;
}

// ===========================================================================
// Batched instances: many independent rising bubbles in one pool, advanced
// by the same launches. No counterpart in the reference, which runs one
// bubble per process.
namespace {

// the reference's parameter derivation (Set_Rising_Bubble_Parameters) for
// one instance on top of the batch's params
amrlbm_params instance_params(const amrlbm_params& base, const amrlbm_instance& in) {
    amrlbm_params q = base;
    q.nbx = in.nbx;
    q.nby = in.nby;
    q.dx0 = in.dx0;
    q.min_levels = 0;
    q.max_levels = in.max_levels;
    q.rho_l = in.rho_l;
    q.rho_h = in.rho_h;
    q.visc_ratio = in.visc_ratio;
    q.bo = in.bo;
    q.ar = in.ar;
    q.gy = in.gy;
    q.w = in.w;
    q.m0 = in.m0;
    q.radius = in.radius;
    q.xc = in.xc;
    q.yc = in.yc;
    q.hydrostatic_start = in.hydrostatic_start;
    return q;
}

int set_active(amrlbm_ctx* ctx, int round) {
    std::vector<unsigned char> a(ctx->insts.size());
    for (size_t i = 0; i < a.size(); ++i) a[i] = (round < 0 || round < ctx->insts[i].max_levels) ? 1 : 0;
    CK(cudaMemcpy(ctx->d_active, a.data(), a.size(), cudaMemcpyHostToDevice));
    return 0;
}

}  // namespace

// AMR_LBM_Rising_Bubble (AMR_Rising_2D_OMP.f90:49-67) for every instance of
// a batch: each instance's base blocks (periodic in x, walls in y) take
// consecutive ids, then the start-up rounds of Refine_Derefine_Mesh and the
// analytic bubble; an instance takes part in as many rounds as it has levels,
// so it goes through exactly the rounds of its own start-up.
int init_batch(amrlbm_ctx* ctx) {
    const auto& I = ctx->insts;
    int nb = 0, maxlv = 0;
    for (const auto& in : I) {
        nb += in.nbx * in.nby;
        maxlv = std::max(maxlv, in.max_levels);
    }
    if (nb > ctx->prm.max_blks) return fail(ctx, AMRLBM_ERR_POOL_FULL, "base blocks exceed max_blks");
    std::vector<int> level(nb, 0), dx(nb), bi(nb), bj(nb), parent(nb, -1), child(4 * nb),
        own(8 * nb), slot(8 * nb, 0), inst(ctx->prm.max_blks + 1, -1);
    std::vector<uint8_t> flags(nb, AMRLBM_F_LEAF | AMRLBM_F_ALLOC);
    int base = 0;
    for (size_t k = 0; k < I.size(); ++k) {
        const int nbx = I[k].nbx, nby = I[k].nby;
        auto id = [&](int x, int y) { return base + 1 + ((x % nbx + nbx) % nbx) + nbx * y; };
        for (int y = 0; y < nby; ++y)
            for (int x = 0; x < nbx; ++x) {
                const int n = id(x, y), i = n - 1;
                dx[i] = I[k].dx0;
                bi[i] = x;
                bj[i] = y;
                inst[n] = (int)k;
                for (int c = 0; c < 4; ++c) child[4 * i + c] = n;
                const bool lo = y > 0, hi = y < nby - 1;
                const int v[8] = {id(x - 1, y),  id(x + 1, y),
                                  lo ? id(x, y - 1) : -3,     hi ? id(x, y + 1) : -4,
                                  lo ? id(x - 1, y - 1) : -5, hi ? id(x - 1, y + 1) : -6,
                                  lo ? id(x + 1, y - 1) : -7, hi ? id(x + 1, y + 1) : -8};
                for (int c = 0; c < 8; ++c) own[8 * i + c] = v[c];
            }
        base += nbx * nby;
    }
    CK(cudaMemcpy(ctx->s.inst, inst.data(), inst.size() * sizeof(int), cudaMemcpyHostToDevice));
    if (int r = amrlbm_set_topology(ctx, nb, level.data(), dx.data(), bi.data(), bj.data(),
                                    parent.data(), child.data(), own.data(), slot.data(),
                                    flags.data(), 0, nullptr, 0))
        return r;
    {
        std::vector<int> ids(nb);
        for (int n = 1; n <= nb; ++n) ids[n - 1] = n;
        const size_t hs = (size_t)9 * (ctx->prm.nx + 2) * (ctx->prm.ny + 2),
                     cs = (size_t)(ctx->prm.nx + 4) * (ctx->prm.ny + 4),
                     ps = (size_t)ctx->prm.nx * ctx->prm.ny;
        std::vector<double> zh(nb * hs, 0.0), zc(nb * cs, 0.0), zp(nb * ps, 0.0);
        if (int r = upload_blocks(ctx, nb, ids.data(), zh.data(), zh.data(), zc.data(), zp.data(),
                                  zp.data(), zp.data()))
            return r;
    }
    int lmax = 0;
    if (int r = set_level_counters(ctx, 0, lmax)) return r;
    if (int r = amrlbm_init_fields(ctx)) return r;
    for (int round = 0; lmax < maxlv; ++round) {
        if (int r = set_active(ctx, round)) return r;
        if (int r = amrlbm_regrid(ctx, ctx->prm.refin_tol, ctx->prm.deref_tol)) return r;
        if (int r = amrlbm_init_fields(ctx)) return r;
        lmax = lmax + 1;
        if (int r = set_level_counters(ctx, 0, lmax)) return r;
    }
    if (int r = set_active(ctx, -1)) return r;
    ctx->stepcount = 0;
    ctx->tail_done = true;
    return AMRLBM_OK;
}

extern "C" {

int amrlbm_create_batch(const amrlbm_params* p, int32_t n_inst, const amrlbm_instance* inst,
                        amrlbm_ctx** out) {
    if (!p || !out || n_inst < 1 || !inst) return AMRLBM_ERR_ARG;
    *out = nullptr;
    if (p->nx != p->ny || (p->nx != 8 && p->nx != 16)) return AMRLBM_ERR_ARG;
    amrlbm_params q = *p;
    q.nbx = q.nby = 1;
    q.min_levels = 0;
    q.dx0 = 1;
    q.max_levels = 0;
    long long nb = 0;
    for (int i = 0; i < n_inst; ++i) {
        const amrlbm_instance& in = inst[i];
        if (in.nbx < 1 || in.nby < 1 || in.dx0 < 1 || (in.dx0 & (in.dx0 - 1)) || in.max_levels < 0 ||
            (in.dx0 >> in.max_levels) < 1 || in.hydrostatic_start < 0 || in.hydrostatic_start > 1)
            return AMRLBM_ERR_ARG;
        q.dx0 = std::max(q.dx0, in.dx0);
        q.max_levels = std::max(q.max_levels, in.max_levels);
        nb += (long long)in.nbx * in.nby;
    }
    if (nb > p->max_blks) return AMRLBM_ERR_ARG;
    // amrlbm_create checks dx0 >> max_levels >= 1 for the largest of each
    while ((q.dx0 >> q.max_levels) < 1) q.dx0 *= 2;
    if (int r = amrlbm_create(&q, out)) return r;
    amrlbm_ctx* ctx = *out;
    DevState& s = ctx->s;
    const size_t NB = (size_t)q.max_blks + 1;
    std::vector<PhysD> ph(n_inst);
    std::vector<PhysF> pf(n_inst);
    std::vector<int> mlv(n_inst);
    std::vector<double> geo(4 * (size_t)n_inst);
    for (int i = 0; i < n_inst; ++i) {
        const amrlbm_params ip = instance_params(q, inst[i]);
        amrlbm_physics phys;
        amrlbm_derive_physics(&ip, &phys);
        ph[i] = to_physd(phys);
        pf[i] = to_physf(ph[i]);
        mlv[i] = inst[i].max_levels;
        geo[4 * i] = inst[i].radius;
        geo[4 * i + 1] = inst[i].xc;
        geo[4 * i + 2] = inst[i].yc;
        geo[4 * i + 3] = inst[i].hydrostatic_start;
    }
    cudaError_t e = cudaSuccess;
    int* d_inst = dalloc<int>(ctx, NB, &e);
    PhysD* d_ph = e == cudaSuccess ? dalloc<PhysD>(ctx, n_inst, &e) : nullptr;
    PhysF* d_pf = e == cudaSuccess ? dalloc<PhysF>(ctx, n_inst, &e) : nullptr;
    int* d_mlv = e == cudaSuccess ? dalloc<int>(ctx, n_inst, &e) : nullptr;
    double* d_geo = e == cudaSuccess ? dalloc<double>(ctx, 4 * (size_t)n_inst, &e) : nullptr;
    unsigned char* d_act = e == cudaSuccess ? dalloc<unsigned char>(ctx, n_inst, &e) : nullptr;
    if (e == cudaSuccess) e = cudaMemcpy(d_ph, ph.data(), n_inst * sizeof(PhysD), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_pf, pf.data(), n_inst * sizeof(PhysF), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_mlv, mlv.data(), n_inst * sizeof(int), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_geo, geo.data(), geo.size() * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_act, 1, n_inst);
    if (e != cudaSuccess) {
        const int r = cuda_fail(ctx, e, "batch tables");
        amrlbm_destroy(ctx);
        *out = nullptr;
        return r;
    }
    s.n_inst = n_inst;
    s.inst = d_inst;
    s.phys = d_ph;
    s.mp.phys = d_pf;
    s.inst_maxlv = d_mlv;
    s.inst_geo = d_geo;
    s.inst_active = d_act;
    ctx->d_active = d_act;
    ctx->insts.assign(inst, inst + n_inst);
    return AMRLBM_OK;
}

int amrlbm_get_instances(amrlbm_ctx* ctx, int32_t* inst) {
    if (!ctx || !inst) return AMRLBM_ERR_ARG;
    CK(cudaStreamSynchronize(ctx->st));
    const Counters c = read_counters(ctx);
    if (!ctx->s.n_inst) {
        for (int n = 1; n <= c.nblks; ++n) inst[n - 1] = 0;
        return AMRLBM_OK;
    }
    CK(cudaMemcpy(inst, ctx->s.inst + 1, (size_t)c.nblks * sizeof(int), cudaMemcpyDeviceToHost));
    return AMRLBM_OK;
}

int amrlbm_diag_instances(amrlbm_ctx* ctx, double* out) {
    if (!ctx || !out) return AMRLBM_ERR_ARG;
    ensure_fp64(ctx, false);
    const int ni = ctx->s.n_inst ? ctx->s.n_inst : 1;
    launch_diag(ctx->s, ctx->st, ctx->d_diag);  // per-leaf partials after the first 9
    if (int r = sync_check(ctx)) return r;
    const Counters c = read_counters(ctx);
    std::vector<double> part(9 * (size_t)c.nleaf);
    std::vector<int> leaves(c.nleaf), inst(ctx->prm.max_blks + 1, 0);
    if (c.nleaf) {
        CK(cudaMemcpy(part.data(), ctx->d_diag + 9, part.size() * 8, cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(leaves.data(), ctx->s.leaf, c.nleaf * sizeof(int), cudaMemcpyDeviceToHost));
    }
    if (ctx->s.n_inst)
        CK(cudaMemcpy(inst.data(), ctx->s.inst, inst.size() * sizeof(int), cudaMemcpyDeviceToHost));
    // the fixed summation order of amrlbm_diag, per instance (leaf order)
    std::vector<double> acc(9 * (size_t)ni, 0.0);
    for (int i = 0; i < ni; ++i) {
        acc[9 * i + 1] = 10.0;
        acc[9 * i + 2] = -10.0;
    }
    for (int m = 0; m < c.nleaf; ++m) {
        double* a = &acc[9 * (size_t)inst[leaves[m]]];
        const double* v = &part[9 * (size_t)m];
        a[0] = a[0] + v[0];
        a[1] = std::fmin(a[1], v[1]);
        a[2] = std::fmax(a[2], v[2]);
        a[3] = std::fmax(a[3], v[3]);
        for (int k = 4; k < 9; ++k) a[k] = a[k] + v[k];
    }
    bool bad = false;
    for (int i = 0; i < ni; ++i) {
        const double* a = &acc[9 * (size_t)i];
        double* o = out + 8 * (size_t)i;
        o[0] = a[0];
        o[1] = a[1];
        o[2] = a[2];
        o[3] = a[3];
        o[4] = a[4];
        o[5] = a[5] / a[4];
        o[6] = a[6] / a[4];
        o[7] = a[7];
        if (a[8] != 0.0) bad = true;
    }
    if (bad) return fail(ctx, AMRLBM_ERR_NAN, "non-finite C or Uy in a leaf");
    return AMRLBM_OK;
}

}  // extern "C"

// ===========================================================================
// Several bubbles and the learned regrid. No counterpart in the reference
// (one bubble; Refine_Derefine_Mesh from the current field only).
extern "C" int amrlbm_net_forward_device(amrlbm_net* net, int32_t n, const float* x_dev,
                                         float* logits);

namespace {

// the forecaster's samples of blocks ids[0..n) into ctx->d_feat
int features_to_device(amrlbm_ctx* ctx, int n, const int* ids, float horizon) {
    const size_t per = (size_t)AMRLBM_NET_CHANNELS * (ctx->prm.nx + 2) * (ctx->prm.ny + 2);
    if ((size_t)n > ctx->feat_cap) {
        if (ctx->d_feat) cudaFree(ctx->d_feat);
        if (ctx->d_fids) cudaFree(ctx->d_fids);
        ctx->d_feat = nullptr;
        ctx->d_fids = nullptr;
        const size_t cap = (size_t)n + n / 2 + 64;
        CK(cudaMalloc(&ctx->d_feat, cap * per * sizeof(float)));
        CK(cudaMalloc(&ctx->d_fids, cap * sizeof(int)));
        ctx->feat_cap = cap;
    }
    if (n == 0) return AMRLBM_OK;
    CK(cudaMemcpyAsync(ctx->d_fids, ids, n * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    launch_block_features(ctx->s, ctx->st, n, ctx->d_fids, horizon, ctx->prm.refin_tol, ctx->d_feat);
    return AMRLBM_OK;
}

}  // namespace

extern "C" {

int amrlbm_set_bubbles(amrlbm_ctx* ctx, int32_t n, const double* xyr) {
    if (!ctx || n < 0 || (n > 0 && !xyr) || ctx->s.n_inst) return AMRLBM_ERR_ARG;
    for (int i = 0; i < n; ++i)
        if (!(xyr[3 * i + 2] > 0.0)) return AMRLBM_ERR_ARG;
    ctx->bubbles.assign(xyr, xyr + 3 * (size_t)n);
    return AMRLBM_OK;
}

int amrlbm_block_features(amrlbm_ctx* ctx, int32_t n, const int32_t* ids, float horizon, float* x) {
    if (!ctx || n < 0 || (n > 0 && (!ids || !x))) return AMRLBM_ERR_ARG;
    if (ctx->prm.nx + 2 != AMRLBM_NET_TILE || ctx->prm.ny + 2 != AMRLBM_NET_TILE)
        return fail(ctx, AMRLBM_ERR_ARG, "the forecaster takes 16x16 blocks");
    for (int i = 0; i < n; ++i)
        if (ids[i] < 1 || ids[i] > ctx->prm.max_blks) return AMRLBM_ERR_ARG;
    ensure_fp64(ctx, false);
    if (int r = features_to_device(ctx, n, ids, horizon)) return r;
    const size_t per = (size_t)AMRLBM_NET_CHANNELS * AMRLBM_NET_TILE * AMRLBM_NET_TILE;
    if (n) CK(cudaMemcpyAsync(x, ctx->d_feat, (size_t)n * per * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    return sync_check(ctx);
}

int amrlbm_set_regrid_net(amrlbm_ctx* ctx, amrlbm_net* net, float horizon, float threshold) {
    if (!ctx || (net && (!(horizon > 0.f) || !(threshold > 0.f) || !(threshold < 1.f))))
        return AMRLBM_ERR_ARG;
    if (net && (ctx->prm.nx != 16 || ctx->prm.ny != 16))
        return fail(ctx, AMRLBM_ERR_ARG, "the forecaster takes 16x16 blocks");
    ctx->net = net;
    ctx->net_horizon = horizon;
    ctx->net_logit = net ? std::log(threshold / (1.f - threshold)) : 0.f;
    if (net) ctx->fnet = net_forecast_params(net);
    ctx->s.forecast = net ? 1 : 0;
    drop_graphs(ctx);
    return AMRLBM_OK;
}

int amrlbm_regrid_stats(amrlbm_ctx* ctx, int64_t out[5]) {
    if (!ctx || !out) return AMRLBM_ERR_ARG;
    if (int r = sync_check(ctx)) return r;
    const Counters c = read_counters(ctx);
    for (int i = 0; i < 5; ++i) out[i] = (int64_t)c.rstat[i];
    return AMRLBM_OK;
}

int amrlbm_forecast_blocks(amrlbm_ctx* ctx, int32_t n, const int32_t* ids, float* logits) {
    if (!ctx || n < 0 || (n > 0 && (!ids || !logits))) return AMRLBM_ERR_ARG;
    if (!ctx->net) return fail(ctx, AMRLBM_ERR_STATE, "no forecaster attached");
    for (int i = 0; i < n; ++i)
        if (ids[i] < 1 || ids[i] > ctx->prm.max_blks) return AMRLBM_ERR_ARG;
    if (n == 0) return AMRLBM_OK;
    if ((size_t)n > ctx->logit_cap) {
        if (ctx->d_logits) cudaFree(ctx->d_logits);
        if (ctx->d_lids) cudaFree(ctx->d_lids);
        ctx->d_logits = nullptr;
        ctx->d_lids = nullptr;
        ctx->logit_cap = 0;
        CK(cudaMalloc(&ctx->d_logits, (size_t)n * sizeof(float)));
        CK(cudaMalloc(&ctx->d_lids, (size_t)n * sizeof(int)));
        ctx->logit_cap = (size_t)n;
    }
    if (ctx->s.mp.fmt && ctx->mp_stale) {  // the kernel reads the mixed-precision fields
        launch_mp_convert(ctx->s, ctx->lc, ctx->st, 0, 1);
        ctx->mp_stale = false;
        ctx->fp64_stale = true;
    }
    CK(cudaMemcpyAsync(ctx->d_lids, ids, n * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    launch_forecast(ctx->s, ctx->lc, ctx->st, ctx->fnet, n, ctx->d_lids, ctx->d_logits,
                    ctx->net_horizon, ctx->prm.refin_tol, ctx->net_logit);
    CK(cudaMemcpyAsync(logits, ctx->d_logits, n * sizeof(float), cudaMemcpyDeviceToHost, ctx->st));
    return sync_check(ctx);
}

}  // extern "C"
