/*
 * fdm.h — C-ABI of libfdm: the B200 (sm_100a) implementation of the
 * leaf-cell hot path of the cell-based quadtree AMR WCNS solver
 * (Jian-cd/FDM-cell-based-AMR-Cartesian).
 *
 * Every entry point replaces one OpenMP loop or subroutine of the reference
 * Fortran; the citation on each declaration names it (path:line within the
 * reference project).  A Fortran host binds these with ISO_C_BINDING
 * (`bind(C, name="fdm_time_advance_rk")`, `type(c_ptr), value :: h`); the
 * signatures use only plain pointers, sizes and C scalars.
 *
 * Ownership: the caller owns every host array (copied in/out on the call);
 * the library owns the device buffers, streams and CUDA graphs of a handle
 * for the handle's lifetime.  A handle is single-threaded: calls are
 * serialised on the handle's stream and outputs are synchronous on return.
 * The library never calls exit/abort and never throws across this ABI.
 */
#ifndef FDM_H
#define FDM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
#define FDM_OK            0
#define FDM_ERR_ARG       1   /* bad argument / size / inconsistent leaf set        */
#define FDM_ERR_CUDA      2   /* a CUDA runtime call failed (message in last_error) */
#define FDM_ERR_NAN       3   /* NaN residual: the reference stops here
                                 (src/solution.F90:209-215)                         */
#define FDM_ERR_TIMEOUT   4   /* a bounded device wait ran out                      */
#define FDM_ERR_NOMEM     5   /* device allocation failed                           */
#define FDM_ERR_STATE     6   /* call out of order (e.g. step before upload)        */
#define FDM_ERR_UNSUPPORTED 7 /* configuration outside what the kernels implement   */

/* -------------------------------------------------------- boundary kinds */
/* BCcyc = 6 is the only kind of the reference (src/module.F90:7).  The other
 * kinds are extensions for the four-quadrant Riemann and Mach-10 wall cases;
 * the reference has no counterpart for them. */
#define FDM_BC_PERIODIC      6
#define FDM_BC_TRANSMISSIVE  2
#define FDM_BC_WALL          3   /* reflecting wall (mirror, normal velocity negated) */
#define FDM_BC_INFLOW        4   /* fixed state bc_state[side]                        */
#define FDM_BC_DMR_BOTTOM    5   /* inflow for x <= dmr_x0, reflecting wall beyond    */
#define FDM_BC_DMR_TOP       7   /* exact moving oblique shock (post/pre states)      */
#define FDM_BC_EXCHANGE      8   /* y side of a strip: halo rows written by the caller
                                    (see "strips of one mesh" below)                  */

/* sides for bc_state[] */
#define FDM_SIDE_XM 0
#define FDM_SIDE_XP 1
#define FDM_SIDE_YM 2
#define FDM_SIDE_YP 3

/* ---------------------------------------------------------------- leaf keys
 * A quadtree node is named by a 64-bit key
 *     key = root << 34 | path << 4 | lvl
 * root : 0-based row-major index of the background cell, i.e. cell(root+1)
 *        of src/mesh.F90:15-37 (num(1) = root / m + 1, num(2) = root % m + 1)
 * lvl  : refinement level (0 = background cell), lvl <= FDM_LMAX
 * path : 2 bits per level, level 1 in the most significant pair of the 30-bit
 *        field; the pair is the child quadrant q = xbit | ybit << 1, so
 *        son1 (SW) = 0, son2 (SE) = 1, son4 (NW) = 2, son3 (NE) = 3
 *        (child placement of Refine_cell, src/mesh.F90:204-258).
 * Sorting leaf keys ascending yields exactly the reference leaf-list order of
 * IDNSgrid (roots row-major, children son1, son2, son4, son3 —
 * src/solution.F90:655-670). */
#define FDM_LMAX 15
#define FDM_KEY(root, lvl, path) \
    (((uint64_t)(root) << 34) | ((uint64_t)(path) << 4) | (uint64_t)(lvl))
#define FDM_KEY_ROOT(k) ((uint64_t)(k) >> 34)
#define FDM_KEY_LVL(k)  ((uint32_t)((k) & 15u))
#define FDM_KEY_PATH(k) (((uint64_t)(k) >> 4) & ((1ull << 30) - 1ull))

/* ------------------------------------------------------------- parameters
 * Mirrors the run parameters of module Global_Var (src/module.F90:16-68) as
 * set_parameter leaves them (src/MAIN.F90:29-71): the domain is already
 * padded by the three ghost layers, and every value is the one the Fortran
 * holds at run time (a REAL(4) literal such as gama = 1.4 is passed as its
 * promoted value 1.399999976158142). */
typedef struct fdm_params {
    double xmin, xmax, ymin, ymax;   /* padded domain (src/MAIN.F90:55-56)      */
    double h;                        /* background cell size                    */
    double x_factor;                 /* aspect factor dx = x_factor * dy        */
    int32_t m, n;                    /* background columns / rows incl. ghosts  */
    double gama, cv, ma;             /* cv = 1/(gama (gama-1) Ma^2)             */

    int32_t iflag_amr;               /* AMR on/off (src/solution.F90:221)       */
    int32_t lvl_amr;                 /* maximum AMR level                       */
    int32_t lvl_max;
    int32_t nstep_adapt, pstep_adapt;/* regrid when it>=Nstep and mod(it,P)==1  */
    double refine_goal_rot, refine_goal_div;
    double coarse_goal_rot, coarse_goal_div;

    int32_t kind_xpbc, kind_xmbc, kind_ypbc, kind_ymbc;

    int32_t iflag_localdt;           /* CFL time step (src/solution.F90:195)    */
    double cfl, tstep, t_end;

    /* boundary-extension data (no reference counterpart) */
    double bc_state[4][4];           /* (rho,u,v,p) per side for FDM_BC_INFLOW  */
    double dmr_x0;                   /* wall start for FDM_BC_DMR_BOTTOM        */
    double dmr_post[4], dmr_pre[4];  /* post/pre-shock states for the DMR BCs   */
    double dmr_shock_speed;          /* x-speed of the shock foot on y = ymax   */
    double dmr_angle_cot;            /* cot(angle) of the shock                 */
    int32_t flux_variant;            /* 0 = exact (reference op order, no FMA),
                                        1 = fast (FMA contraction)              */
    /* strip of the mesh held by this handle: root rows
     * [window_row0, window_row0 + window_rows) of the n padded rows above;
     * window_rows = 0 holds the whole mesh (see "strips of one mesh") */
    int32_t window_row0, window_rows;
    int32_t reserved[5];
} fdm_params;

typedef struct fdm_handle fdm_handle;

/* Counters the reference only prints (brinv "real matrix singularity!",
 * src/XuanGua.F90:616-619) or never notices. */
typedef struct fdm_counters {
    int64_t n_leaves;          /* all leaves incl. ghosts and corners         */
    int64_t n_interior;        /* nResgrid (src/solution.F90:599-613)         */
    int64_t n_ghost;           /* nBCgrid                                     */
    int64_t n_wls_requests;    /* hanging-node WLS-WENO evaluations per stage */
    int64_t n_restrict_requests;
    int64_t n_faces_x, n_faces_y;
    int64_t n_singular;        /* brinv singular pivots in the WLS geometry   */
    int64_t n_regrids;
    int64_t n_internal;        /* internal nodes of the tree                  */
    int64_t n_gm1_iterations;  /* fixpoint sweeps of gridmodify1 (all passes) */
    int64_t n_gm4_visits;      /* leaves gridmodify4 acted from               */
    int64_t n_gm4_nonleaf;     /* Refine_cell of a non-leaf by gridmodify4
                                  (src/mesh.F90:389-392)                      */
    int64_t n_gm4_triggers;    /* gridmodify4: leaves marked able to act at pass start */
    int64_t n_gm4_refines;     /* gridmodify4: Refine_cell calls */
    int64_t n_gm4_steps;       /* gridmodify4: replay iterations (batches and queued leaves) */
    int64_t gm4_replay_us;     /* gridmodify4: device time of the replay kernel, microseconds */
} fdm_counters;

/* ------------------------------------------------------------- lifecycle */
/* Create a handle on the current CUDA device.  Replaces nothing: the
 * reference keeps its state in module globals (src/module.F90:13-69). */
int fdm_create(const fdm_params *p, fdm_handle **out);
void fdm_destroy(fdm_handle *h);
int fdm_last_error(const fdm_handle *h, char *buf, size_t n);

/* Upload a complete leaf set (interior, ghost and corner leaves in any order)
 * with primitive values prim[4*i .. 4*i+3] = (rho, u, v, p).  Builds the
 * device leaf order, neighbour tables, stencil tables and hanging-node
 * requests.  Equivalent of the tree the reference holds after creat_mesh /
 * AMR + idneighbor + IDgrid (src/mesh.F90:9-47, src/neighbor.F90:399-449,
 * src/solution.F90:593-615). */
int fdm_upload_leaves(fdm_handle *h, int64_t n, const uint64_t *keys,
                      const double *prim);
int64_t fdm_num_leaves(const fdm_handle *h);
/* Download all leaves in key order; cap is the capacity of keys/prim.
 * keys or prim may be NULL (values only, or keys only). */
int fdm_download_leaves(fdm_handle *h, int64_t cap, int64_t *n_out,
                        uint64_t *keys, double *prim);
/* Overwrite the primitive values of the current leaf set (same keys as the
 * last upload/regrid, in key order).  No table rebuild. */
int fdm_set_values(fdm_handle *h, int64_t n, const double *prim);
/* Asynchronous forms (no reference counterpart): the copies run on copy
 * streams (one for uploads, one for read-backs) with double-buffered device
 * staging, ordered with the compute
 * stream by events, so an upload of the next input and a read-back of the
 * last result overlap the steps in between.  prim must be pinned host
 * memory and stay untouched until fdm_io_sync returns; the values are those
 * of the state at the point in the call sequence (uploads before the next
 * step, read-backs after the previous one). */
int fdm_set_values_async(fdm_handle *h, int64_t n, const double *prim);
int fdm_download_values_async(fdm_handle *h, int64_t cap, double *prim);
int fdm_io_sync(fdm_handle *h);

/* Scalars of the time loop: lambda_x, lambda_y, tstep, tt, it, l_max. */
int fdm_get_scalars(fdm_handle *h, double *lambda_x, double *lambda_y,
                    double *tstep, double *tt, int64_t *it, int32_t *l_max);
int fdm_set_scalars(fdm_handle *h, double lambda_x, double lambda_y,
                    double tstep, double tt, int64_t it);

/* ------------------------------------------------------------ time loop */
/* lambda / time-step control: monotone max of |u|+c, |v|+c over the interior
 * leaves, l_max, CFL step and t_end clamp (src/solution.F90:185-201). */
int fdm_step_control(fdm_handle *h, double *tstep, double *lambda_x,
                     double *lambda_y, int32_t *l_max);
/* One SSP-RK3 step with the current tstep: getRKn, 3 x (solution_cell loop,
 * updateRK, body_boundary_RK loop) — Time_advance_RK,
 * src/solution.F90:267-298. */
int fdm_time_advance_rk(fdm_handle *h, double tstep);
/* Fine-grained pieces of Time_advance_RK. */
int fdm_get_rkn(fdm_handle *h);                       /* src/solution.F90:372-384 */
int fdm_solution_cells(fdm_handle *h, int32_t krk);   /* src/solution.F90:279-284 */
int fdm_update_rk(fdm_handle *h, int32_t krk);        /* src/solution.F90:386-404 */
int fdm_body_boundary(fdm_handle *h, int32_t j);      /* src/solution.F90:288-293 */
/* Residual norms of the last stage, as Res_max / Res_rms after the
 * sqrt of src/solution.F90:209-210 (4 equations). */
int fdm_residual(fdm_handle *h, double res_max[4], double res_rms[4]);
/* One iteration of the solute loop (src/solution.F90:182-236) without file
 * output: step control, Time_advance_RK, tt update, NaN check, and AMR +
 * boundary refill when iflag_amr.  Returns FDM_ERR_NAN on a NaN residual. */
int fdm_solute_step(fdm_handle *h);
/* Run solute steps until tt >= t_end or nsteps were taken: the same
 * iterations as fdm_solute_step, replayed as a CUDA graph in chunks that end
 * at the next regrid, with the scalars read once per chunk.  On the device an
 * iteration after t_end or after a NaN residual changes nothing, so
 * *steps_done counts the iterations actually taken; returns FDM_ERR_NAN
 * after the iteration whose residual is NaN. */
int fdm_solute(fdm_handle *h, int64_t nsteps, int64_t *steps_done);

/* Run nsteps solute iterations on the device (step control, RK3 step,
 * tt/residual/NaN bookkeeping) through a captured CUDA graph, without host
 * synchronisation and without regrid: the timed window between two regrids
 * of the solute loop (src/solution.F90:182-219).  Returns when enqueued;
 * fdm_get_scalars synchronises. */
int fdm_advance(fdm_handle *h, int64_t nsteps);

/* AMR driver: indicators, refine/coarsen flags, smoothing / 2:1 balance,
 * neighbour and leaf-list rebuild (src/solution.F90:408-421). */
int fdm_amr(fdm_handle *h);

int fdm_get_counters(fdm_handle *h, fdm_counters *c);

/* Diagnostics of output_error (src/output_ADT.F90:18-75) on the device:
 * the density of every interior leaf against the isentropic vortex of
 * strength 5 at (5, 5), summed left to right in cell_NS (key) order as the
 * reference does.  norms[0..8] = L1_rho, L2_rho, Loo_rho over the interior
 * leaves, P1_rho, P2_rho, Poo_rho over the refined ones (0 when there are
 * none) and L1, L2, Loo over the level-0 ones; counts[0..2] = interior,
 * level-0 and refined leaf counts.  Only these numbers cross to the host.
 * The vortex density uses the device's exp and pow. */
int fdm_output_error(fdm_handle *h, double norms[9], int64_t counts[3]);
/* The leaf keys (key order) into pinned host memory, queued like
 * fdm_download_values_async on the read-back stream (a field dump of keys
 * and values overlaps the steps after it); complete at fdm_io_sync. */
int fdm_download_keys_async(fdm_handle *h, int64_t cap, uint64_t *keys);
/* Waits until every read-back queued so far (fdm_download_values_async,
 * fdm_download_keys_async) has landed in host memory.  It touches only the
 * read-back stream, so unlike every other call it may be made from another
 * host thread while the handle is in use (a writer thread of field dumps). */
int fdm_readback_wait(fdm_handle *h);

/* Paired runs, no reference counterpart: nsteps solute iterations of two
 * handles holding the same leaf set at the same iteration and time, in
 * lockstep.  `follow` takes `lead`'s lambda maxima before every step (so
 * the same time step) and, at every regrid, the refine/coarsen decisions of
 * `lead`'s indicators on `lead`'s state (so the same new leaf set); `lead`
 * advances exactly as fdm_solute advances it.  The two runs then differ only
 * by how their face fluxes are computed: with the learned gate on in
 * `follow` and off in `lead`, the difference of their states is the gate's
 * error alone, free of the regrid decisions that any perturbation flips.
 * Returns FDM_ERR_STATE if the handles do not start together, FDM_ERR_ARG
 * if a regrid finds different leaf sets. */
int fdm_solute_paired(fdm_handle *lead, fdm_handle *follow, int64_t nsteps,
                      int64_t *steps_done);

/* ----------------------------------------------- test / integration hooks */
/* The 8 stencil values per interior leaf (Tip, Tim, Tjp, Tjm, Tipp, Timm,
 * Tjpp, Tjmm of src/XuanGua.F90:401-590) for the current values, in interior
 * key order: out[(i*8 + s)*4 + v].  For parity tests. */
int fdm_debug_stencil(fdm_handle *h, int64_t cap, double *out);
/* Face-neighbour and diagonal-neighbour keys per leaf in key order
 * (idnei, src/neighbor.F90:412-449): out[i*8 + d], d = up, down, right,
 * left, upleft, upright, downleft, downright; ~0ull for a null pointer. */
int fdm_debug_neighbors(fdm_handle *h, int64_t cap, uint64_t *out);
/* Hanging-node stencils per interior leaf and entry (key order, entries as
 * in fdm_debug_stencil): kind 0 same-level leaf, 1 parent_value_weno WLS,
 * 2 parent_value_weno interpA fallback, 3 child_value_weno WLS, 4
 * child_value_weno copy fallback (src/XuanGua.F90:45-150); the node key the
 * value belongs to, the target point, (m1, m2) and up to 16 member keys of
 * the WLS stencil in the reference's list order. */
int fdm_debug_requests(fdm_handle *h, int64_t cap, int32_t *kind, uint64_t *node,
                       double *xy, int32_t *m12, uint64_t *mem);
/* The bounded waits of the batched kernel's grid barrier: two blocks wait
 * for a third that never arrives, give up at the default wait limit (2 s of
 * global-timer time) and return.  Returns FDM_ERR_TIMEOUT (the expected
 * outcome) with the device time of the waits in *seconds; the context stays
 * usable. */
int fdm_debug_barrier_timeout(double *seconds);
/* Host-side allocation-failure injection (no GPU fault): the next `after`
 * device buffer allocations of the library succeed and every later one
 * fails as if cudaMalloc had run out of memory, so the calls that need it
 * return FDM_ERR_NOMEM; after < 0 turns the injection off.  A handle whose
 * upload or regrid failed this way is left not loaded (FDM_ERR_STATE until
 * the next successful upload). */
int fdm_debug_fail_alloc(int64_t after);
/* AMR indicators rot/div of the interior leaves (src/solution.F90:424-466). */
int fdm_debug_rot_div(fdm_handle *h, int64_t cap, double *rot, double *div,
                      double *srot_sdiv_ne);
/* The device's left-to-right sums of two host arrays of n non-negative
 * addends (the kernel that forms Srot and Sdiv, src/solution.F90:430-457):
 * sums[0] = (...((0 + a[0]) + a[1]) + ...) + a[n-1], sums[1] the same over b.
 * For testing the summation on chosen inputs; runs on the current device. */
int fdm_debug_ordered_sum(const double *a, const double *b, int64_t n, double *sums);

/* Device-resident state for in-process callers (bench, Python mirror):
 * the CUDA stream of the handle and the device pointer of the (rho,u,v,p)
 * 32-byte slot records: interior leaves in key order, then ghost leaves,
 * corner leaves and hanging-node values; n receives the slot count. */
int fdm_device_state(fdm_handle *h, void **stream, double **prim_dev,
                     int64_t *n);

/* Measurement hooks.  fdm_time_kernels times the kernels of one stage on
 * the current state with CUDA events on the handle's stream, averaged over
 * reps launches: ms[0] face fluxes (x and y), ms[1] residual + RK update,
 * ms[2] hanging-node values, ms[3] ghost fill.  The stage-1/2 buffers are
 * scratch for this call.  fdm_fp64_peak measures the FP64 FMA throughput of
 * the current device (TFLOP/s, 2 flops per DFMA).  No reference
 * counterpart. */
int fdm_time_kernels(fdm_handle *h, int32_t reps, double *ms);
int fdm_fp64_peak(double *tflops);
/* Autotuner of the face-flux launch shape: times each of the
 * FDM_FACE_VARIANTS variants on the current leaf set (ms[v] = ms per x+y
 * launch pair; ms holds FDM_FACE_VARIANTS doubles), keeps the fastest for
 * this handle and reports it in *best.  fdm_set_variant forces one. */
#define FDM_FACE_VARIANTS 21
int fdm_autotune(fdm_handle *h, int32_t reps, int32_t *best, double *ms);
int fdm_set_variant(fdm_handle *h, int32_t face_variant);
/* Diagnostics: out[0], out[1] = x and y faces of the current state whose
 * branch-free division (face variants 7-10, 13, 14) meets an operand outside
 * its exact range and is computed again with the compiler's division. */
int fdm_debug_nr_fallbacks(fdm_handle *h, int64_t out[2]);

/* ------------------------------------------------------------ learned gate
 * No reference counterpart.  A BF16 MLP (8 -> 32 -> 32 -> 1, GELU, sigmoid,
 * FP32 accumulation on the tensor cores) decides per face whether the
 * linear WCNS weights suffice; such faces take a component-wise linear
 * reconstruction, all others the plain scheme.  Parameters are FP32, layout
 * W1[32][8], b1[32], W2[32][32], b2[32], w3[32], b3 (fdm_gate_param_count()
 * floats).  fdm_gate_set enables the gate on a handle (g >= threshold takes
 * the linear path) or disables it (enable = 0: the exact path).
 * fdm_gate_samples writes (features[8], target) of every stride-th face of
 * the current state to caller device buffers; target = exp(-dev/tau) with
 * dev the largest effect of a nonlinear-weight deviation on the face's 16
 * WCNS_Z3 reconstructions, |w1 - l1| |p1 - p2| over the magnitude of the
 * characteristic component on the stencil.  fdm_gate_train_step runs one
 * Adam step (forward and backward on the tensor cores) on a minibatch of B
 * samples idx0 + k*step (mod n) of caller device arrays, minimising
 * -(y log g + neg_weight (1-y) log(1-g)); loss receives the batch sum.
 * fdm_gate_eval: gate probabilities of feature rows. */
int fdm_gate_param_count(void);
int fdm_gate_set(fdm_handle *h, const float *params, float threshold, int32_t enable);
int fdm_gate_samples(fdm_handle *h, int64_t stride, int64_t phase, double tau,
                     float *feat_dev, float *target_dev, int64_t offset, int64_t cap,
                     int64_t *n_written);
int fdm_gate_train_step(const float *X, const float *Y, int64_t n, int64_t idx0,
                        int64_t step, int64_t B, float neg_weight, float *params,
                        float *grad, float *adam_m, float *adam_v, int64_t t,
                        float lr, float *loss, void *stream);
int fdm_gate_eval(const float *X, int64_t n, const float *params, float *prob,
                  void *stream);
/* The plain rule in place of the network, the baseline the network is
 * measured against: a face takes the linear path at stage 1 when the largest
 * of its normalised jumps (the gate's features before squashing) is at most
 * jump_threshold; jump_threshold < 0 restores the network.  Requires the
 * gate to be on (fdm_gate_set). */
int fdm_gate_set_jump_rule(fdm_handle *h, float jump_threshold);
/* faces that took the linear path in the last gated stage / all faces */
int fdm_gate_stats(fdm_handle *h, int64_t *gated, int64_t *total);

/* Diagnostics, no reference counterpart: device-timeline milliseconds of
 * the five regrid phases (indicators + ordered sums; flags + first node
 * sort; the lvlAMR gridmodify rounds; leaf/internal split; table rebuild),
 * ms[0..4] for the last regrid and ms[5..9] summed over all regrids. */
int fdm_amr_phase_ms(const fdm_handle *h, double ms[10]);

/* ------------------------------------------------------------ ensembles
 * No reference counterpart (the reference runs one mesh per process).  A
 * batch advances many loaded handles of one GPU together: one persistent,
 * cooperative kernel launch per RK3 stage covers every member, the blocks
 * taking (member, tile) work from a shared counter, with a grid barrier
 * (bounded waits) between the phases of a stage.  Each member keeps its own
 * tables, state, scalars and learned-gate setting, and ends in the state
 * that the same number of fdm_solute_step calls gives.  A member's regrid
 * rebuilds its tables; the batch notices and captures its step graph again.
 *
 * fdm_batch_advance: nsteps steps of every unfinished member without regrids
 * or host synchronisation (graph replays on the batch stream, ordered after
 * and before the members' own streams).  fdm_batch_solute: nsteps steps with
 * each member's regrids when due, stopping with FDM_ERR_NAN at a NaN.
 * fdm_batch_sync waits for the batch and reports a barrier that timed out.
 * A grid-barrier wait that runs past its limit (fdm_batch_set_wait_limit,
 * default 2 s) makes fdm_batch_solute / fdm_batch_sync return
 * FDM_ERR_TIMEOUT (the FDM_ERR_TIMEOUT of the error contract: a device wait
 * limit hit); the members' states of that step are then undefined and must
 * be restored (upload) by the caller, while the batch itself stays usable.
 * Members must stay alive and must not be used from another thread while
 * the batch exists. */
typedef struct fdm_batch fdm_batch;
int fdm_batch_create(fdm_handle *const *members, int32_t n, fdm_batch **out);
void fdm_batch_destroy(fdm_batch *b);
int fdm_batch_last_error(const fdm_batch *b, char *buf, size_t n);
int fdm_batch_advance(fdm_batch *b, int64_t nsteps);
int fdm_batch_solute(fdm_batch *b, int64_t nsteps, int64_t *steps_done);
int fdm_batch_sync(fdm_batch *b);
/* blocks_per_sm 1 or 2: resident blocks of the persistent kernel per SM;
 * 0: no persistent kernel, each member's own step graph on its own stream
 * (the batch stream is joined to the members' streams around every call,
 * so ordering and event timing on the batch stream are unchanged);
 * 3: no persistent kernel, one launch per phase of a stage covering the
 * tiles of every member (requests, faces, hard faces, cells, ghosts, each
 * with its own launch shape), ordered on the batch stream.  Results are the
 * same bits every way; which is faster depends on the members' sizes
 * (measure). */
int fdm_batch_set_blocks_per_sm(fdm_batch *b, int32_t blocks_per_sm);
/* Face phases of the persistent kernel: 0 the reference's operation order
 * (default), 1 the split order with the branch-free correctly rounded
 * division of face variants 7-10 (the same bits; one may be faster). */
int fdm_batch_set_face_flux(fdm_batch *b, int32_t branch_free);
/* Wait limit of one grid barrier of the persistent kernel in seconds
 * (0 < seconds <= 3600; default 2), measured on the GPU's global timer. */
int fdm_batch_set_wait_limit(fdm_batch *b, double seconds);
int fdm_batch_info(const fdm_batch *b, int32_t *grid, int32_t *blocks_per_sm,
                   int64_t *smem_bytes);
int fdm_batch_stream(const fdm_batch *b, void **stream);
/* diagnostics: microseconds of each phase of the last step, [3 stages][16] */
int fdm_batch_phase_us(fdm_batch *b, double us[48]);

/* ------------------------------------------------- no-allocation entry point
 * One SSP-RK3 step (the three stages of Time_advance_RK with periodic ghost
 * fill) on a uniform periodic grid of nx x ny cells, without allocating any
 * device memory.  No counterpart in the reference: it exists for callers
 * that cannot call cudaMalloc — a host whose GPU memory belongs to its own
 * allocator (an OpenACC or CUDA Fortran runtime that owns the device heap),
 * code that runs under a memory budget fixed at start-up, or a process that
 * forbids device allocation after initialisation.
 *
 * prim_in / prim_out: device arrays of (nx+6)*(ny+6) 32-byte records
 * (rho,u,v,p), 32-byte aligned, row-major over the background grid with its
 * three ghost layers (the order of cell(1..m*n)); prim_in holds filled
 * ghosts, prim_out receives the new interior, its periodic ghosts and the
 * input corners.  lambda_x/lambda_y are the global Lax-Friedrichs speeds of
 * the step.  Enqueued on `stream` (0 = legacy default stream); synchronise
 * before reading prim_out.
 *
 * Working memory (the two intermediate stage states and the face fluxes) is
 * a fixed 8.5 MiB static device array that every GPU loading libfdm holds
 * until the process exits.  Limits: 3 <= nx, ny <= FDM_STATIC_MAX_SIDE and
 * nx*ny <= FDM_STATIC_MAX_CELLS; larger sizes return FDM_ERR_ARG and enqueue
 * nothing.  Every call shares that array and every record a call reads was
 * written earlier by the same call, so nothing carries over from a previous
 * call; calls that overlap on the GPU (different streams, or different host
 * threads on one device) race on it and must be serialised by the caller.
 * Every call looks up the array's device address (cudaGetSymbolAddress)
 * with the caller's device current, so the address stays right after a
 * context is torn down and created again; the first call on each device
 * also loads the module there, so make that first call before any stream
 * capture.  prim_in and prim_out must not overlap (FDM_ERR_ARG).  A CUDA
 * error already pending when the call starts is returned as FDM_ERR_CUDA
 * before anything is enqueued (it belongs to earlier work). */
#define FDM_STATIC_MAX_SIDE  1024
#define FDM_STATIC_MAX_CELLS 65536
int fdm_time_advance_rk_uniform_static(const double *prim_in, double *prim_out,
                                       int32_t nx, int32_t ny, double h, double x_factor,
                                       double gama, double lambda_x, double lambda_y,
                                       double tstep, void *stream);

/* ------------------------------------------------------ checkpoint/restart
 * No reference counterpart (the reference writes only output files).  A
 * handle's state is its leaves (fdm_download_leaves), the scalars
 * (fdm_get_scalars) and the values of its internal nodes: every refined cell
 * keeps a value (its U when refined, the interpA mean when coarsened,
 * src/mesh.F90:199-260, 397-408) that a later gridmodify4 refinement of a
 * non-leaf copies into new sons (src/mesh.F90:389-392), while an upload
 * starts them as interpA means.  fdm_download_internal gives the internal
 * nodes (keys sorted, the ancestors of the leaves) and their (rho,u,v,p);
 * fdm_set_internal writes them back after an upload of the same leaf set
 * (FDM_ERR_ARG when the keys differ).  Upload + fdm_set_internal +
 * fdm_set_scalars restores a run that continues bit for bit. */
int fdm_download_internal(fdm_handle *h, int64_t cap, int64_t *n_out,
                          uint64_t *keys, double *vals);
int fdm_set_internal(fdm_handle *h, int64_t n, const uint64_t *keys,
                     const double *vals);

/* ----------------------------------------------------- strips of one mesh
 * No reference counterpart (the reference runs one OpenMP process).  One
 * mesh is split into horizontal strips of background rows, one handle per
 * strip (per GPU), exchanging halo rows after every stage.
 *
 * A strip handle is created with fdm_params.window_rows > 0: it holds the
 * root rows [window_row0, window_row0 + window_rows) of the padded root grid
 * that xmin..ymax, m and n describe.  Its leaf keys name roots relative to
 * the strip (root - window_row0 * m).  A y side of kind FDM_BC_EXCHANGE makes
 * the strip's three outer rows on that side a halo: their leaves are neither
 * advanced nor filled by fdm_body_boundary; the caller writes them after
 * every stage with the values of the strip that owns those rows.  Cell
 * centres and the neighbour classification use the global row, so a leaf
 * the strip owns is advanced by exactly the arithmetic the whole mesh gives
 * it.  Strips need non-periodic y sides where they are cut, at least three
 * owned rows each, and take no regrid (fdm_amr returns
 * FDM_ERR_UNSUPPORTED): the caller regrids the whole mesh.
 *
 * One step of a strip (every strip the same calls in the same order):
 *   fdm_step_control            local lambda, l_max
 *   (max of lambda_x, lambda_y, l_max over the strips)
 *   fdm_step_control_global     the step from the global maxima
 *   for krk = 1..3: fdm_solution_cells, fdm_update_rk, fdm_body_boundary(3),
 *                   fdm_pack_slots -> exchange -> fdm_unpack_slots
 *   fdm_set_scalars             tt + tstep, it + 1
 *
 * fdm_leaf_slots: the state slot of every leaf in key order (cap entries).
 * fdm_pack_slots / fdm_unpack_slots: gather the (rho,u,v,p) records of the
 * latest stage at the given slots into buf[4*i..4*i+3] / scatter them back;
 * slots and buf are DEVICE pointers (for NCCL or peer copies), the calls
 * return when the copy is complete.
 * fdm_step_control_global: sets lambda_x, lambda_y (monotone maxima) and
 * l_max and forms the time step of src/solution.F90:195-201 from them.
 * fdm_set_async(h, 1): fdm_solution_cells, fdm_update_rk, fdm_body_boundary
 * and the two halo copies return once enqueued on the handle's stream
 * (fdm_device_state), so the caller orders strips and transfers with CUDA
 * events instead of host waits; a slot error of a halo copy is then reported
 * by the next fdm_step_control_global.  fdm_set_async(h, 0) restores the
 * synchronous calls. */
int fdm_leaf_slots(fdm_handle *h, int64_t cap, int32_t *slot);
int fdm_pack_slots(fdm_handle *h, int64_t n, const int32_t *slots, double *buf);
int fdm_unpack_slots(fdm_handle *h, int64_t n, const int32_t *slots, const double *buf);
int fdm_step_control_global(fdm_handle *h, double lambda_x, double lambda_y,
                            int32_t l_max, double *tstep);
int fdm_set_async(fdm_handle *h, int32_t on);

#ifdef __cplusplus
}
#endif
#endif /* FDM_H */
