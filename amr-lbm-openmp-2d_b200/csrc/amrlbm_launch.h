// amrlbm_launch.h - host-side launchers of the FP64 kernels (amrlbm_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "amrlbm_dev.cuh"

// consumer work fused after a C ghost fill in one level-ordered launch
enum FillCConsumer {
    CONS_NONE = 0,          // Fill_Ghost_Cells_C / _C2 alone
    CONS_COLLIDE_READ = 1,  // + Collision_h_g_AMR with P,Ux,Uy from memory
    CONS_COLLIDE_FUSED = 2, // + Macroscopic_Values_g_AMR in registers + collision
    CONS_MACRO_G = 3        // + Macroscopic_Values_g_AMR + Err_Interface
};

struct LaunchCfg {
    int num_sms;
    int grid_queue;     // CTAs of a level-ordered kernel
    int grid_leaves;    // CTAs of a grid-stride kernel over leaves
    int mp_ctas;        // CTAs per SM of the mixed-precision kernels (0: as many as fit)
};

// write_ring: without level order, the consumer items write the ghost rings
// they fill to memory only if set (their own launch reads them from shared
// memory; the state after a step holds them); fills with level order and
// CONS_NONE always write them
void launch_fill_c(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int width,
                   int consumer, int write_ring = 1);
void launch_fill_hg_stream(const DevState& s, const LaunchCfg& lc, cudaStream_t st,
                           int write_ring = 1);
void launch_collide(const DevState& s, const LaunchCfg& lc, cudaStream_t st);
void launch_macro_h(const DevState& s, const LaunchCfg& lc, cudaStream_t st);
void launch_macro_g(const DevState& s, const LaunchCfg& lc, cudaStream_t st);
void launch_err(const DevState& s, const LaunchCfg& lc, cudaStream_t st);
void launch_minmax(const DevState& s, cudaStream_t st);
void launch_init_fields(const DevState& s, const LaunchCfg& lc, cudaStream_t st, double radius,
                        int hydro, double y0, int p_given = 0);
void launch_block_features(const DevState& s, cudaStream_t st, int n, const int* ids,
                           float horizon, double tol, float* out);
void launch_regrid_flags(const DevState& s, cudaStream_t st, double refin_tol, double deref_tol);
void launch_restrict(const DevState& s, const LaunchCfg& lc, cudaStream_t st);
// mode 0: Refine_Derefine_Mesh; 1: Initial_Mesh level (no data movement);
// 2: rebuild lists only. lmin/lmax < 0: take LevelMin/LevelMax from the
// device counters. set_levels: LevelMin/LevelMax := level range of the new
// leaves (what the next Determine_Min_Max_Levels returns).
void launch_regrid_topo(const DevState& s, cudaStream_t st, int mode, int lmin, int lmax,
                        int set_levels);
// neighbour records and ghost-cell fill plans of the leaves in work order;
// after every change of the topology
void launch_build_plans(const DevState& s, const LaunchCfg& lc, cudaStream_t st);
void launch_prolong(const DevState& s, const LaunchCfg& lc, cudaStream_t st);
void launch_zero_children(const DevState& s, const LaunchCfg& lc, cudaStream_t st);
void launch_flag_level(const DevState& s, cudaStream_t st, int level);
void launch_diag(const DevState& s, cudaStream_t st, double* out8);
// TecPlot_CellCenter: node and cell values of every leaf (amrlbm_tecplot.cu)
void launch_tecplot(const DevState& s, cudaStream_t st, int num_sms, double* node_c, int* node_xy,
                    double* cell, double D, double sigma);
// writes the reference's ASCII file from those values; 0 on success
int tecplot_write(const char* path, int nx, int ny, int nleaf, int L0, double t_value,
                  const double* node_c, const int* node_xy, const double* cell);
void launch_reset_queues(const DevState& s, cudaStream_t st);
// number of kernels the launchers above issued (for the launch counter)
long long launches_issued();
void count_launches(int n);
// div_rn against IEEE division on n random operands (divisor 0: random)
int selftest_division(unsigned long long n, unsigned long long seed, double divisor,
                      unsigned long long* mismatches);

// mixed-precision time step (amrlbm_mixed.cu); s.mp.fmt != 0, nx = ny = 8 or 16.
// read_pu: P, U of the state are in memory (else the collision evaluates
// Macroscopic_Values_g_AMR); write_pu / write_ring: the last step of a call
void launch_mp_collide(const DevState& s, const LaunchCfg& lc, cudaStream_t st, bool read_pu,
                       int write_pu);
void launch_mp_fill_hg_stream(const DevState& s, const LaunchCfg& lc, cudaStream_t st,
                              int write_ring);
void launch_mp_tail(const DevState& s, const LaunchCfg& lc, cudaStream_t st);
// occupancy queries and shared-memory opt-ins of the kernels above (outside
// stream capture, once per block size and format)
void launch_mp_prepare(const DevState& s, const LaunchCfg& lc);
// mode: 0 every leaf, 1 derefined parents, 2 their children, 3 refined
// parents, 4 their children; to_mp: FP64 -> mixed, else back
void launch_mp_convert(const DevState& s, const LaunchCfg& lc, cudaStream_t st, int mode,
                       int to_mp);

// the refine-flag forecaster's device parameters (amrlbm_net.cu): BF16
// weight matrices W1 [48][32] (rows 36.. zero), W2, W3 [288][32], FP32
// biases, dense weights and bias
struct ForecastNet {
    const void *w1, *w2, *w3;
    const float *b1, *b2, *b3, *wd, *bd;
};
struct amrlbm_net;
ForecastNet net_forecast_params(const amrlbm_net* net);
// learned regrid (amrlbm_forecast.cu). ids == nullptr: every leaf of the
// level range that may still refine; a forecast (logit > thr) that the
// criterion (err > tol) does not flag raises err to 2 tol; statistics into
// the counters. Else logits[i] of blocks ids[0..n_ids) (device arrays).
void launch_forecast(const DevState& s, const LaunchCfg& lc, cudaStream_t st, const ForecastNet& net,
                     int n_ids, const int* ids, float* logits, float horizon, double tol, float thr);
