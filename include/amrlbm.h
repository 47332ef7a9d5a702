/*
 * amrlbm.h - C ABI of the B200 (sm_100a) block-structured AMR two-phase
 * lattice Boltzmann step (conservative phase field h + pressure/velocity g,
 * D2Q9, weighted MRT) of the rising-bubble solver AMR-LBM-OpenMP-2D.
 *
 * The library owns ONE device-resident block pool. A caller (the reference's
 * Fortran driver through ISO_C_BINDING, C, or Python through ctypes) keeps its
 * own host arrays and copies them in and out only through the upload/download
 * entry points below. Every entry point returns an int status: 0 = OK.
 *
 * Conventions shared with the reference (all cited paths are files of the
 * reference project):
 *   - block ids are 1-based Fortran indices into the pool Blk(1:MaxBlks)
 *     (Parameters.f90:39);
 *   - neighbour directions 1..8 = left, right, bottom, top, SW, NW, SE, NE
 *     (AMR_Rising_2D_OMP.f90:97-101); a negative neighbour is an external
 *     wall code;
 *   - child slot k = 1 + I + 2J for the child at (I,J) in {0,1}^2
 *     (AMR_Rising_2D_OMP.f90:542-551);
 *   - populations 1..9 = rest, E, N, W, S, NE, NW, SW, SE (D2Q9_Mod.f90:6-7);
 *   - field layouts are the reference's column-major arrays:
 *       h, g : (9, 0:nx+1, 0:ny+1)          (Parameters.f90:36)
 *       C    : (-1:nx+2, -1:ny+2)           (Parameters.f90:37)
 *       P, Ux, Uy : (nx, ny)                (Parameters.f90:37)
 *   - a neighbour is a POINTER to an integer, not a value
 *     (Parameters.f90:23-31, Neighbors.f90:19-31). It is exported as the pair
 *     (owner, slot): slot 1..4 means "child(slot) of block owner" and slot 0
 *     means "the constant owner" (wall codes and the base blocks' own
 *     neighbour integers). Its value is owner when slot == 0, else
 *     child(slot) of owner at the time it is read.
 *
 * One context per host thread; calls on one context are not re-entrant. All
 * device work of a context runs on that context's own CUDA stream.
 */
#ifndef AMRLBM_H
#define AMRLBM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (replace the reference's PRINT / STOP) ---------------- */
enum {
    AMRLBM_OK = 0,
    AMRLBM_ERR_ARG = 1,        /* bad argument or size                         */
    AMRLBM_ERR_CUDA = 2,       /* CUDA runtime error / no device / no sm_100   */
    AMRLBM_ERR_POOL_FULL = 3,  /* Add_Child_Blocks STOP, AMR_Rising_2D_OMP.f90:527-531 */
    AMRLBM_ERR_LEVEL_JUMP = 4, /* "Error in SUB_Fill_*", Fill_Ghost_Cells_C.f90:85-87 */
    AMRLBM_ERR_NAN = 5,        /* non-finite field value found by diagnostics  */
    AMRLBM_ERR_DANGLING = 6,   /* neighbour pointer into a freed block's child array */
    AMRLBM_ERR_STATE = 7,      /* call out of order (e.g. step before init)    */
    AMRLBM_ERR_TIMEOUT = 8,    /* a bounded device wait ran out                */
    AMRLBM_ERR_CAPACITY = 9,   /* request larger than a fixed scratch area      */
    AMRLBM_ERR_IO = 10         /* an output file could not be written           */
};

/* flag bits of amrlbm_get_topology / amrlbm_set_topology */
enum {
    AMRLBM_F_LEAF = 1,      /* Blk%IsLeaf  */
    AMRLBM_F_HASLEAF = 2,   /* Blk%hasLeaf */
    AMRLBM_F_REFIN = 4,     /* Blk%Refin   */
    AMRLBM_F_DEREF = 8,     /* Blk%Deref   */
    AMRLBM_F_ALLOC = 16     /* fields allocated (a leaf, or a derefined parent) */
};

/* Run-time parameters. The reference hard-codes these as PARAMETERs
 * (Parameters.f90:12-19, D2Q9_Mod.f90:10-11) or literals
 * (AMR_Rising_2D_OMP.f90:154-158,241-259,276-277); amrlbm_default_params()
 * returns the reference's values. */
typedef struct amrlbm_params {
    int32_t nx, ny;          /* cells per block side (even, >= 4)                    */
    int32_t nbx, nby;        /* base blocks in x (periodic) and y (walls)            */
    int32_t dx0;             /* base-level cell size in finest cells (L0/nx)         */
    int32_t min_levels;      /* minLevels                                            */
    int32_t max_levels;      /* maxLevels                                            */
    int32_t max_blks;        /* MaxBlks: pool capacity (blocks)                      */
    int32_t regrid_every;    /* regrid after every n-th step (reference: 1)          */
    int32_t device;          /* CUDA device of the pool; < 0: the current device     */
    double rho_l, rho_h;     /* Rhol, Rhoh                                            */
    double visc_ratio;       /* muh/mul (reference: 100)                              */
    double bo, ar;           /* Bond (=Eotvos) and Archimedes numbers                 */
    double gy;               /* gravity                                               */
    double w;                /* interface width W                                     */
    double m0;               /* mobility M0                                           */
    double radius, xc, yc;   /* bubble radius and centre (finest-cell units)          */
    double refin_tol;        /* refine if Err_Interface > refin_tol                   */
    double deref_tol;        /* derefine if all 4 children's error <= deref_tol       */
    /* Start-up pressure of Initialize_AMR_Rising_Bubble. 0 (the reference's,
     * AMR_Rising_2D_OMP.f90:193): the Laplace jump P = -Sigma/R*C.
     * 1: the same plus the hydrostatic head of the light phase about the
     * bubble centre, Gy*(Rhoh-Rhol)*(1-C)*(y-yc). The buoyancy force
     * Fb = (Rhoh-Rho)*Gy (LBM_Subroutines.f90:152) already removes the heavy
     * phase's head, so P stays uniform there, and inside the bubble the
     * head balances Fb from the first step instead of accelerating the light
     * phase from rest. */
    int32_t hydrostatic_start;
} amrlbm_params;

/* Derived physical constants (D2Q9_Mod.f90:13-16), as computed by
 * Set_Rising_Bubble_Parameters (AMR_Rising_2D_OMP.f90:235-263). */
typedef struct amrlbm_physics {
    double w, sigma, beta, kappa, tau_l, tau_h, rho_l, rho_h, gy, m0;
} amrlbm_physics;

typedef struct amrlbm_ctx amrlbm_ctx;

/* ---- set-up ------------------------------------------------------------- */
void amrlbm_default_params(amrlbm_params* p);
/* Set_Rising_Bubble_Parameters (AMR_Rising_2D_OMP.f90:235-263) for p. */
int amrlbm_derive_physics(const amrlbm_params* p, amrlbm_physics* out);
/* Allocates the device pool (max_blks blocks) on the current CUDA device. */
int amrlbm_create(const amrlbm_params* p, amrlbm_ctx** out);
int amrlbm_destroy(amrlbm_ctx* ctx);
/* Replaces the derived constants (the Fortran driver computes its own). */
int amrlbm_set_physics(amrlbm_ctx* ctx, const amrlbm_physics* phys);
/* Collision model of g in Collision_h_g_AMR (LBM_Subroutines.f90:179-181):
 * AMRLBM_G_MRT, MRT_Collision_AMR (:348-361), the reference's and the
 * default; or AMRLBM_G_BGK, BGK_Collision_AMR (:337-344), the alternative
 * the reference keeps commented out at :180. */
enum { AMRLBM_G_MRT = 0, AMRLBM_G_BGK = 1 };
int amrlbm_set_g_collision(amrlbm_ctx* ctx, int32_t model);
/* Storage precision of amrlbm_step; no counterpart in the reference, which
 * is FP64 throughout. AMRLBM_FP64 (the default) is the reference's
 * arithmetic, bit for bit. AMRLBM_FP16 / AMRLBM_BF16: the populations h and g
 * are stored in 16 bits as deviations (f_q - (w_q/w_1) f_1, the rest
 * population f_1 kept in FP32), C, P, Ux, Uy in FP32, and collision, ghost-cell
 * interpolation and streaming run in FP32; the regrid's restriction sums and
 * the diagnostics stay FP64 (Restrict.f90:14-65 on FP64 copies of the blocks
 * involved). Needs 8x8 or 16x16 blocks. The FP64 pool remains the state that
 * every other entry point reads and writes: after mixed-precision steps the
 * first such call converts the state back (rounded values), and the next
 * amrlbm_step converts it forward again. Results follow the FP64 trajectory
 * within the 16-bit rounding, not bit for bit. */
enum { AMRLBM_FP64 = 0, AMRLBM_FP16 = 1, AMRLBM_BF16 = 2 };
int amrlbm_set_precision(amrlbm_ctx* ctx, int32_t precision);
/* Launch shape of the mixed-precision kernels (one CTA of nx*ny threads per
 * leaf item, persistent over the items): at most ctas_per_sm CTAs on each SM,
 * 0 (the default) as many as fit. A tuning knob (amrlbm.autotune); results do
 * not depend on it. */
int amrlbm_set_launch(amrlbm_ctx* ctx, int32_t ctas_per_sm);
/* Whether the current mesh's ghost fills need level order (1) or not (0):
 * [0] Fill_Ghost_Cells_C2, [1] Fill_Ghost_Cells_C, [2] Fill_Ghost_Cells_hg.
 * A fill needs it where a coarse-to-fine stencil reads a coarser
 * neighbour's ghost cell that is itself coarse-to-fine or a wall cell (the
 * reference's DO L = LevelMin, LevelMax loops, Fill_Ghost_Cells_C.f90:8-38);
 * its kernels then take the leaves in level order with bounded waits. A
 * performance diagnostic; no counterpart in the reference. */
int amrlbm_get_fill_order(amrlbm_ctx* ctx, int32_t needs_order[3]);
/* Failure-detection test hook; no counterpart in the reference, whose
 * OpenMP barriers cannot time out. The level-ordered fills (a level range
 * narrower than the leaves) order their items by per-block flags, and every
 * wait on a flag is bounded: when it runs out the kernel records
 * AMRLBM_ERR_TIMEOUT, goes on and returns, and the next synchronising call
 * reports it. spin_limit > 0 replaces the bound (iterations of about 64 ns;
 * 0 restores the default of about a second); hold_block > 0 makes the fills
 * never raise that block's flag, so that every item waiting for it runs out
 * of its bound. (0, 0) restores normal operation. */
int amrlbm_set_wait_test(amrlbm_ctx* ctx, int32_t spin_limit, int32_t hold_block);
const char* amrlbm_last_error(const amrlbm_ctx* ctx);
/* Device memory held by the context, bytes. */
int64_t amrlbm_device_bytes(const amrlbm_ctx* ctx);

/* ---- state transfer (host <-> device) ----------------------------------- */
/* counts[0..4] = Nblks, nLeaf, KK, LevelMin, LevelMax (Parameters.f90:6-10) */
int amrlbm_get_counts(amrlbm_ctx* ctx, int32_t counts[5]);
/* Sets LevelMin/LevelMax as the driver does (AMR_Rising_2D_OMP.f90:51-52,66). */
int amrlbm_set_level_range(amrlbm_ctx* ctx, int32_t level_min, int32_t level_max);
/* Topology of blocks 1..nblks. Arrays are indexed by id-1; child has 4 entries
 * per block, nbr_owner / nbr_slot 8 per block (pointer model above). The
 * free list holds the first id of every freed quartet in FIFO order
 * (Parameters.f90:41-45, Refine_Derefine.f90:246-254). */
int amrlbm_set_topology(amrlbm_ctx* ctx, int32_t nblks, const int32_t* level,
                        const int32_t* dx, const int32_t* bi, const int32_t* bj,
                        const int32_t* parent, const int32_t* child,
                        const int32_t* nbr_owner, const int32_t* nbr_slot,
                        const uint8_t* flags, int32_t n_free, const int32_t* free_list,
                        int32_t kk);
int amrlbm_get_topology(amrlbm_ctx* ctx, int32_t* level, int32_t* dx, int32_t* bi,
                        int32_t* bj, int32_t* parent, int32_t* child,
                        int32_t* nbr_owner, int32_t* nbr_slot, uint8_t* flags,
                        int32_t* n_free, int32_t* free_list);
/* Resolved neighbour ids nbr[8*(id-1)+k-1] = Blk(id)%nghbr(k)%n of blocks
 * 1..Nblks (0 for blocks without fields). */
int amrlbm_get_neighbours(amrlbm_ctx* ctx, int32_t* nbr);
/* Leaf list LeafBlks(1:nLeaf) (AMR_Rising_2D_OMP.f90:588-610). */
int amrlbm_get_leaves(amrlbm_ctx* ctx, int32_t* leaves);
/* One block's fields in the reference layouts; any pointer may be NULL. */
int amrlbm_upload_block(amrlbm_ctx* ctx, int32_t id, const double* h, const double* g,
                        const double* C, const double* P, const double* Ux,
                        const double* Uy);
int amrlbm_download_block(amrlbm_ctx* ctx, int32_t id, double* h, double* g, double* C,
                          double* P, double* Ux, double* Uy);
/* Bulk transfer of n blocks ids[0..n-1]: each array holds n consecutive
 * blocks in the per-block layout above. Any field pointer may be NULL. */
int amrlbm_upload_fields(amrlbm_ctx* ctx, int32_t n, const int32_t* ids, const double* h,
                         const double* g, const double* C, const double* P,
                         const double* Ux, const double* Uy);
int amrlbm_download_fields(amrlbm_ctx* ctx, int32_t n, const int32_t* ids, double* h,
                           double* g, double* C, double* P, double* Ux, double* Uy);
/* Per-block interface error Err_Interface (Refine_Derefine.f90:327-351) of
 * blocks 1..Nblks as last computed by amrlbm_macro_g / amrlbm_regrid
 * (0 for blocks that are not leaves). */
int amrlbm_get_block_error(amrlbm_ctx* ctx, double* err);

/* ---- driver helpers ----------------------------------------------------- */
/* The reference driver's start-up, AMR_LBM_Rising_Bubble
 * (AMR_Rising_2D_OMP.f90:49-67): base blocks (generalised to nbx x nby,
 * periodic in x, walls in y), Initial_Mesh, the analytic bubble of
 * Initialize_AMR_Rising_Bubble and the start-up regrid loop. The tanh/sqrt
 * profile is evaluated on the host (as the driver does); everything else runs
 * on the device. */
int amrlbm_init_rising_bubble(amrlbm_ctx* ctx);
/* Initialize_AMR_Rising_Bubble (AMR_Rising_2D_OMP.f90:142-231) alone, for the
 * current leaves. */
int amrlbm_init_fields(amrlbm_ctx* ctx);

/* ---- phase entry points (the Main_Loop call sites) ---------------------- */
/* Determine_Min_Max_Levels (AMR_Rising_2D_OMP.f90:304,434-452). */
int amrlbm_min_max_levels(amrlbm_ctx* ctx, int32_t* level_min, int32_t* level_max);
/* Fill_Ghost_Cells_C2 (AMR_Rising_2D_OMP.f90:318). */
int amrlbm_fill_ghost_c2(amrlbm_ctx* ctx);
/* Phase_Field_LBM_h_g_AMR: collide all leaves, Fill_Ghost_Cells_hg, stream
 * (AMR_Rising_2D_OMP.f90:322,381-430). */
int amrlbm_phase_field_step(amrlbm_ctx* ctx);
/* Macroscopic_Values_h_AMR over leaves (AMR_Rising_2D_OMP.f90:328-335). */
int amrlbm_macro_h(amrlbm_ctx* ctx);
/* Fill_Ghost_Cells_C (AMR_Rising_2D_OMP.f90:341). */
int amrlbm_fill_ghost_c(amrlbm_ctx* ctx);
/* Macroscopic_Values_g_AMR over leaves (AMR_Rising_2D_OMP.f90:346-354);
 * also computes every leaf's Err_Interface for the next regrid. */
int amrlbm_macro_g(amrlbm_ctx* ctx);
/* Refine_Derefine_Mesh (AMR_Rising_2D_OMP.f90:360, Refine_Derefine.f90:2-14). */
int amrlbm_regrid(amrlbm_ctx* ctx, double refin_tol, double deref_tol);
/* nsteps iterations of the Main_Loop body (AMR_Rising_2D_OMP.f90:304-363)
 * without output, regridding after every regrid_every-th step (counted over
 * the context's lifetime). Steps that are not followed by a regrid run the
 * fused path (the next step's Fill_Ghost_Cells_C2 supplies the ring that
 * Fill_Ghost_Cells_C would write; Macroscopic_Values_g_AMR runs inside the
 * collision); on return the state equals the reference's at a step boundary.
 * Runs as CUDA graphs; does not synchronise the host. */
int amrlbm_step(amrlbm_ctx* ctx, int32_t nsteps);
/* Blocks the host until the context's stream is idle; returns a pending
 * device error status (pool full, level jump, ...), if any. */
int amrlbm_sync(amrlbm_ctx* ctx);

/* ---- diagnostics -------------------------------------------------------- */
/* Output (AMR_Rising_2D_OMP.f90:456-489) with a fixed summation order, plus
 * the bubble centroid and rise velocity. The bubble sums run over the cells
 * with C < 1/2 only, so that round-off of C around 1 in the heavy phase, summed
 * over the whole domain, does not move them:
 *   out[0] mass = sum rho*dx^2       out[1] rho_min   out[2] rho_max
 *   out[3] u_max = max |Uy|          out[4] bubble volume = sum_{C<1/2} (1-C)*dx^2
 *   out[5] yc = sum_{C<1/2} (1-C)*y*dx^2 / out[4]
 *   out[6] v_rise = sum_{C<1/2} (1-C)*Uy*dx^2 / out[4]
 *   out[7] phase volume sum C*dx^2
 * Returns AMRLBM_ERR_NAN if any leaf value is not finite. */
int amrlbm_diag(amrlbm_ctx* ctx, double out[8]);

/* TecPlot_CellCenter (TecPlot_ASCII.f90:2-86; call site
 * AMR_Rising_2D_OMP.f90:308): the leaves as one FE-quadrilateral zone in the
 * reference's ASCII layout, to `path` (the reference names its files
 * Rising_Bubble_2D_<nn>.dat from a call counter; the caller chooses here).
 * t: the time step T of the zone title T*sqrt(Gy/D), D = 2*radius. Node
 * values of C need the ghost ring 1 of C, as the reference's do: call it
 * between amrlbm_step calls (or after amrlbm_fill_ghost_c). Returns
 * AMRLBM_ERR_IO if the file cannot be written. */
int amrlbm_write_tecplot(amrlbm_ctx* ctx, const char* path, int32_t t);

/* ---- timing (CUDA events on the context's stream) ----------------------- */
int amrlbm_timer_start(amrlbm_ctx* ctx);
/* Milliseconds since amrlbm_timer_start; synchronises. */
int amrlbm_timer_stop(amrlbm_ctx* ctx, float* ms);
/* Per-kernel device time accounting of amrlbm_step: when enabled, every
 * launch of the collision kernel is bracketed by CUDA events on the
 * launching stream. kernel_ms returns the accumulated time and launches. */
int amrlbm_profile_enable(amrlbm_ctx* ctx, int32_t enable);
int amrlbm_profile_read(amrlbm_ctx* ctx, int32_t kernel, double* total_ms,
                        int64_t* launches, int64_t* cells);
/* Number of kernels this library launched since creation. */
int64_t amrlbm_launch_count(const amrlbm_ctx* ctx);
/* Self-test of the exact FP64 division used by the kernels (the FMA
 * correction of Markstein's theorem, given a correctly rounded reciprocal)
 * against IEEE division, on n random operands on the current device;
 * divisor 0 draws random divisors. mismatches = results whose bits differ. */
int amrlbm_selftest_division(uint64_t n, uint64_t seed, double divisor, uint64_t* mismatches);
/* Writes a buffer larger than the L2 cache on the context's stream. */
int amrlbm_flush_l2(amrlbm_ctx* ctx);

/* ---- batched instances ----------------------------------------------------
 * No counterpart in the reference, which runs one bubble per process. A batch
 * holds many independent rising-bubble problems in one pool; every entry
 * point above (amrlbm_step in FP64 or mixed precision, the transfers, the
 * regrid) advances all of them in the same launches. Each instance has its own
 * base grid (nbx x nby blocks of dx0 finest cells, periodic in x, walls in y),
 * number of levels, physics (derived as Set_Rising_Bubble_Parameters,
 * AMR_Rising_2D_OMP.f90:235-263, does for one) and bubble; block size, pool
 * size, tolerances and regrid interval are the batch's (amrlbm_params, whose
 * own physics and geometry fields are not used). Every instance's fields
 * equal, bit for bit, those of the same problem run alone; its block ids are
 * the pool's. amrlbm_init_rising_bubble starts every instance up
 * (AMR_Rising_2D_OMP.f90:49-67), each with as many start-up regrid rounds as
 * it has levels. 8x8 or 16x16 blocks. */
typedef struct amrlbm_instance {
    int32_t nbx, nby, dx0, max_levels;
    double rho_l, rho_h, visc_ratio, bo, ar, gy, w, m0;
    double radius, xc, yc;
    int32_t hydrostatic_start;
} amrlbm_instance;
int amrlbm_create_batch(const amrlbm_params* p, int32_t n_inst, const amrlbm_instance* inst,
                        amrlbm_ctx** out);
/* inst[id-1] = instance (0-based) of blocks 1..Nblks (0 for one mesh). */
int amrlbm_get_instances(amrlbm_ctx* ctx, int32_t* inst);
/* amrlbm_diag per instance: out[8*i .. 8*i+7] as amrlbm_diag's out[0..7],
 * each instance's sums in leaf-list order. */
int amrlbm_diag_instances(amrlbm_ctx* ctx, double* out);

/* ---- learned regrid: the refine-flag forecaster ---------------------------
 * No counterpart in the reference, which flags blocks from the current field
 * only (Err_Interface, Refine_Derefine.f90:327-351). A small convolutional
 * network over one 16x16 block with its ghost ring (AMRLBM_NET_CHANNELS
 * channels on AMRLBM_NET_TILE^2 cells, layout [n][channel][y][x]): three 3x3
 * convolutions of 32 channels with ReLU, a global max pool, a dense output;
 * the logit of "this block is flagged for refinement k steps from now". BF16
 * weights and activations on the tensor cores, FP32 accumulation, FP32 master
 * weights trained with Adam on a weighted binary cross-entropy. Parameter
 * vector (amrlbm_net_param_count floats): W1 [36][32], b1, W2 [288][32], b2,
 * W3 [288][32], b3, wd [32], bd, with W[((dy+1)*3 + (dx+1))*c_in + ci][co]. */
#define AMRLBM_NET_CHANNELS 4
#define AMRLBM_NET_TILE 18
typedef struct amrlbm_net amrlbm_net;
int amrlbm_net_create(uint64_t seed, int32_t max_batch, amrlbm_net** out);
int amrlbm_net_destroy(amrlbm_net* net);
int32_t amrlbm_net_param_count(void);
const char* amrlbm_net_last_error(const amrlbm_net* net);
int amrlbm_net_get(amrlbm_net* net, float* params);
/* also resets the optimiser state */
int amrlbm_net_set(amrlbm_net* net, const float* params);
/* logits of n samples x (host memory) */
int amrlbm_net_forward(amrlbm_net* net, int32_t n, const float* x, float* logits);
/* mean loss and its gradient (host, param_count floats; may be NULL) over n
 * samples with labels y in {0, 1}, positives weighted pos_weight */
int amrlbm_net_gradient(amrlbm_net* net, int32_t n, const float* x, const float* y,
                        float pos_weight, float* loss, float* grad);
/* one Adam step (learning rate lr) on the gradient of n samples */
int amrlbm_net_train_step(amrlbm_net* net, int32_t n, const float* x, const float* y,
                          float pos_weight, float lr, float* loss);
/* logits of n samples already in device memory (any n) */
int amrlbm_net_forward_device(amrlbm_net* net, int32_t n, const float* x_dev, float* logits);
/* the network's tensor-core product alone: C = A B, A [M][K] and B [K][N]
 * BF16 bit patterns, C FP32, row-major host arrays */
int amrlbm_net_selftest_gemm(int32_t M, int32_t N, int32_t K, const uint16_t* A,
                             const uint16_t* B, float* C);

/* The forecaster's samples of blocks ids[0..n) of the current state (16x16
 * blocks; between amrlbm_step calls, when C's ghost rings are filled), layout
 * [n][4][18][18] over the block's cells with ring 1: C; log(1 + e/refin_tol)
 * with e the cell's Err_Interface term sqrt(dCx^2 + dCy^2)/(2dx)
 * (Refine_Derefine.f90:327-351); Ux and Uy times horizon/dx (cells moved in
 * `horizon` steps; 0 on the ring). */
int amrlbm_block_features(amrlbm_ctx* ctx, int32_t n, const int32_t* ids, float horizon,
                          float* x);
/* Learned regrid: with net != NULL, every regrid of amrlbm_step refines the
 * leaves the forecaster flags (probability > threshold; its samples taken
 * with `horizon`) together with those the reference's criterion
 * (Err_Interface > refin_tol) flags; NULL restores the criterion alone. The
 * forecast runs on the device inside the step's graph, one fused kernel over
 * the leaves that may still refine, with the net's current weights (training
 * after this call is seen by later regrids). The net must outlive its use.
 * stats of the regrids of amrlbm_step and amrlbm_refine_derefine_mesh since
 * the start-up (amrlbm_init_rising_bubble resets them): [0] regrids, [1]
 * leaves forecast, [2] leaves the criterion flagged (leaves of the level
 * range that may still refine), [3] flagged leaves the forecast missed
 * (refined all the same; without a net every flagged leaf), [4] leaves
 * forecast but not flagged. */
int amrlbm_set_regrid_net(amrlbm_ctx* ctx, amrlbm_net* net, float horizon, float threshold);
int amrlbm_regrid_stats(amrlbm_ctx* ctx, int64_t out[5]);
/* logits[i] of the attached net (amrlbm_set_regrid_net) on block ids[i] of
 * the current state by the fused kernel of the learned regrid: equal, bit
 * for bit, to amrlbm_net_forward on amrlbm_block_features of the same
 * blocks. */
int amrlbm_forecast_blocks(amrlbm_ctx* ctx, int32_t n, const int32_t* ids, float* logits);
/* Several bubbles for amrlbm_init_rising_bubble / amrlbm_init_fields (n
 * triples x, y, R in finest cells; n = 0: the params' one bubble): C is the
 * tanh profile of the nearest bubble's surface, P as for one bubble with the
 * nearest bubble's radius and centre. No counterpart in the reference's
 * start-up (AMR_Rising_2D_OMP.f90:142-231), which places one bubble. */
int amrlbm_set_bubbles(amrlbm_ctx* ctx, int32_t n, const double* xyr);

/* ---- download without allocation ----------------------------------------
 * No counterpart in the reference, whose fields live in host memory.
 * amrlbm_download_fields with the same arguments and results, for callers
 * that must not allocate once set up (a host code with a fixed device-memory
 * budget, an output hook between time steps): it stages through a fixed
 * scratch area per device instead of buffers it allocates, and copies every
 * field straight into the caller's array. At most AMRLBM_NOALLOC_MAX_BLOCKS
 * blocks and AMRLBM_NOALLOC_STAGE_DOUBLES doubles of requested fields (n times
 * the sizes of the non-NULL fields) per call, else AMRLBM_ERR_CAPACITY and
 * nothing runs; split larger downloads into several calls. The scratch is
 * shared by all contexts on a device: calls that overlap in time on one
 * device race on it and must be serialised by the caller. The first call on
 * a device sets the scratch up (no allocation). A pending device error status
 * (pool full, level jump, ...) is returned once and cleared, as
 * amrlbm_download_fields does, but without a message through
 * amrlbm_last_error. */
#define AMRLBM_NOALLOC_STAGE_DOUBLES 524288 /* 4 MiB */
#define AMRLBM_NOALLOC_MAX_BLOCKS 16384
int amrlbm_download_fields_noalloc(amrlbm_ctx* ctx, int32_t n, const int32_t* ids, double* h,
                                   double* g, double* C, double* P, double* Ux, double* Uy);

#ifdef __cplusplus
}
#endif

#endif /* AMRLBM_H */
