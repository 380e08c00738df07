/*
 * hfmm_b200 -- C ABI of the B200 Helmholtz KIFMM evaluate path.
 *
 * The reference (a JAX package) has no native boundary: its entry points are the
 * Python functions HFMM.setup / HFMM.evaluate (HFMM.py:55-91) and, one layer
 * down, kifmm.setup / kifmm.evaluate_setup (jaxfmm/kifmm/setup.py:19-261). This
 * header is the C-ABI those Python entry points bind through ctypes (see
 * hfmm_b200/_lib.py). Every function returns HFMM_OK (0) or a negative status;
 * hfmm_last_error() gives the message of the calling thread's last failure.
 * Pointers named *_dev are device pointers owned by the caller; the plan owns
 * every buffer it allocates. No C++ exception crosses this boundary.
 *
 * Life cycle of a plan (mirrors HFMM.setup, HFMM.py:55-80):
 *   hfmm_tree_build        tree + particle layout     (trees/cubic.py:316-695)
 *   hfmm_plan_info         depth, extent, sizes       (kifmm/setup.py:220-226 keys)
 *   hfmm_plan_set_level    per-level operator tables  (kifmm/operators.py:572-641)
 *   hfmm_plan_finalize     interaction lists + schedules (trees/lists.py:818-931)
 *   hfmm_evaluate          potential [+ field]        (HFMM.py:83-91, core.py:214-335)
 *   hfmm_plan_destroy
 */
#ifndef HFMM_B200_H
#define HFMM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HFMM_OK 0
#define HFMM_ERR_ARG -1       /* invalid argument (shape, range, null pointer)      */
#define HFMM_ERR_CUDA -2      /* a CUDA runtime call failed                          */
#define HFMM_ERR_STATE -3     /* call out of order (e.g. evaluate before finalize)    */
#define HFMM_ERR_CAPACITY -4  /* a size limit was exceeded                           */
#define HFMM_ERR_DEVICE -5    /* a kernel raised its device error flag               */

/* Kernel kinds of the kernel seam (hfmm_plan_set_kernel_kind; the reference's
 * Kernel specification, jaxfmm/kernels/spec.py:10-62). */
#define HFMM_KERNEL_HELMHOLTZ 0   /* cos(kr)/r and sin(kr)/r, HFMM.py:12-52            */
#define HFMM_KERNEL_YUKAWA 1      /* exp(-kappa r)/(4 pi r), kernels/yukawa/kernel.py:10-75;
                                     kappa = 0 is Laplace, kernels/laplace/kernel.py:104  */

#define HFMM_PREC_FP64 0      /* plain path: every phase in float64                  */
#define HFMM_PREC_MIXED 1     /* M2L as split 3xTF32 on tcgen05 (FP32 accumulation in
                                 short chains, folded into FP64), P2P in FP32 with an
                                 FP64 phase reduction; decodes, M2M, L2L, P2M, L2P FP64.
                                 M2L needs p >= 5 (ld = n_s rounded up to 32 >= 128);
                                 smaller p runs its FP64 GEMM.                         */

typedef struct hfmm_plan hfmm_plan;

/* Sizes of a built plan. Box indices follow the reference's packing
 * (finest level first, trees/cubic.py:371-372); boxes [0, n_boxes) are active. */
typedef struct hfmm_info {
    int64_t n_points;
    int32_t max_depth;        /* realised depth (build_fmm_tree_auto, cubic.py:530-600) */
    int32_t maxleaf;          /* largest leaf occupancy                                 */
    int64_t max_boxes;        /* the reference's box buffer size after doubling         */
    int64_t n_boxes;          /* active boxes                                           */
    int64_t n_leaves;
    int32_t adaptive;         /* leaves on more than one level (core.py:117)            */
    int32_t level_lo[16];     /* boxes of level l occupy [level_lo[l], level_hi[l])     */
    int32_t level_hi[16];
    double domain_extent;
    double pmin[3];
    int64_t n_v, n_u, n_w, n_x, n_near;   /* list lengths (0 until finalize)           */
    int32_t n_s;              /* surface points per box (0 until a kernel is set)       */
    int32_t p;
} hfmm_info;

/* Build the octree of n points (pos_dev: n x 3 float64, row-major, device).
 * n_max is the leaf size N_max; max_depth <= 0 selects the reference's automatic
 * depth (cubic.py:583-600). Replaces build_fmm_tree_auto + assign_particles
 * (trees/cubic.py:530-695) and core.setup_geometry's tree part (core.py:111-117). */
int hfmm_tree_build(const double* pos_dev, int64_t n, int32_t n_max, int32_t max_depth,
                    hfmm_plan** out);

/* Moving geometry (replaces the reference's fully-jit evaluator,
 * kifmm/fulljit.py:57-328, and its guarded driver, driver.py:556-640, for the
 * Helmholtz path): hfmm_tree_build with the domain cube [pmin, pmin + extent]^3
 * and the depth given instead of measured, so the level scales, and with them the
 * plan's operator tables, do not depend on where the points are. Then, per time
 * step, hfmm_plan_rebuild(plan, new_positions) rebuilds the tree, the U/V/W/X
 * lists and the schedules in place on the device and keeps the tables. Its
 * certificate: a point outside the domain returns HFMM_ERR_CAPACITY before
 * anything changes (the caller refits the domain and builds a new plan); a plan
 * in a batch returns HFMM_ERR_STATE. Same n as the plan; synchronises the device.
 * hfmm_plan_info then reports the realised counts. */
int hfmm_tree_build_in_domain(const double* pos_dev, int64_t n, int32_t n_max, int32_t max_depth,
                              const double* pmin, double extent, hfmm_plan** out);
int hfmm_plan_rebuild(hfmm_plan* plan, const double* pos_dev);

/* The sizes the reference's setup dict carries (max_depth, maxleaf, max_boxes,
 * domain_extent, pmin, list lengths: kifmm/setup.py:220-226, core.py:156-160). */
int hfmm_plan_info(const hfmm_plan* plan, hfmm_info* out);

/* Choose the kernel before hfmm_plan_set_kernel (default HFMM_KERNEL_HELMHOLTZ):
 * HFMM_KERNEL_YUKAWA takes kappa >= 0 as set_kernel's k, one family, and decode
 * tables of that kernel; every particle kernel, the device table generation, the
 * mixed near field and the direct-sum referee then evaluate exp(-kappa r)/(4 pi r)
 * (the reference's kifmm.setup(..., kernel=yukawa(kappa)) or kernel=LAPLACE,
 * kifmm/setup.py:19-226). */
int hfmm_plan_set_kernel_kind(hfmm_plan* plan, int32_t kind);

/* Kernel: wavenumber k, p points per cube edge, n_families = 2 (cos and sin
 * components, HFMM.py:65-80) or 1 (k == 0, HFMM.py:71-72). equiv_pts and
 * check_pts are the unit surfaces (n_s x 3, host, row-major) at radii 1.05 and
 * 2.95 (kifmm/surfaces.py:20-85); n_s = 6p^2 - 12p + 8. */
int hfmm_plan_set_kernel(hfmm_plan* plan, double k, int32_t p, int32_t n_families,
                         const double* equiv_pts, const double* check_pts);

/* Per-level tables of one kernel family (0 = cos, 1 = sin), host pointers, all
 * float64 row-major as the reference stacks them (operators.py:620-641):
 *   F_up_U, F_up_Vt, F_dn_U, F_dn_Vt : n_s x n_s;  F_up_d, F_dn_d : n_s
 *   M2M_K : 8 x n_s x n_s, M2M_K_lv[level]  (may be NULL when level == max_depth)
 *   L2L_K : 8 x n_s x n_s, L2L_K_lv[level-1] (may be NULL when level < 3)
 *   M2L_K : 343 x n_s x n_s, M2L_K_lv[level] (adjacent entries ignored)
 * Only levels 2..max_depth are consumed; the library copies and re-lays them out. */
int hfmm_plan_set_level(hfmm_plan* plan, int32_t family, int32_t level,
                        const double* F_up_U, const double* F_up_d, const double* F_up_Vt,
                        const double* F_dn_U, const double* F_dn_d, const double* F_dn_Vt,
                        const double* M2M_K, const double* L2L_K, const double* M2L_K);

/* Same as hfmm_plan_set_level, but only the damped-SVD decode factors come from
 * the host: the M2M, L2L and M2L kernel matrices (operators.py:363-403) are
 * evaluated on the device from the surfaces, k and the level scale. Entries agree
 * with the host NumPy tables to rounding (CUDA sincos vs the host libm). */
int hfmm_plan_set_level_decode(hfmm_plan* plan, int32_t family, int32_t level,
                               const double* F_up_U, const double* F_up_d, const double* F_up_Vt,
                               const double* F_dn_U, const double* F_dn_d, const double* F_dn_Vt);

/* Streaming M2L tables (no counterpart in the reference, whose M2L tables are
 * resident, kifmm/operators.py:612-613): instead of keeping the 316 M2L matrices
 * of every level (11 GB per family at p = 12, depth 5), the plan regenerates a
 * level's matrices on the device right before that level's M2L, into a
 * workspace of hfmm_plan_workspace_bytes bytes, bit-identical to the resident
 * tables. Choose the mode after hfmm_plan_set_kernel and before the level tables
 * (which must then come without M2L_K: hfmm_plan_set_level_decode). Without a
 * bound workspace, the first hfmm_evaluate allocates the plan's own (so make
 * that call outside stream capture). hfmm_plan_bind_workspace
 * points the plan at a caller-owned device buffer (256-byte aligned); plans that
 * share one must not run concurrently (a batch gives each stream its own). */
int hfmm_plan_set_streaming(hfmm_plan* plan, int32_t enable);
int hfmm_plan_workspace_bytes(const hfmm_plan* plan, int64_t* bytes);
int hfmm_plan_bind_workspace(hfmm_plan* plan, void* ws_dev, int64_t bytes);

/* Build the V, U, W, X lists and the evaluate schedules on the device
 * (trees/lists.py:818-931, core.py:119-140). */
int hfmm_plan_finalize(hfmm_plan* plan);

/* Evaluate for charges q_re (+ q_im, nullable for real charges) in the
 * original point order. phi_out: n complex128 (interleaved re, im).
 * field_out (nullable): n x 3 complex128, the field -grad(phi)
 * (kifmm/setup.py:242-246). With q_im == NULL this is HFMM.evaluate
 * (HFMM.py:83-91); with q_im the result follows by linearity,
 * phi = E_cos(q_re) - E_sin(q_im) + i (E_sin(q_re) + E_cos(q_im)).
 * precision: HFMM_PREC_FP64 or HFMM_PREC_MIXED. stream: a cudaStream_t or NULL.
 * Allocates nothing; asynchronous on the stream. */
int hfmm_evaluate(hfmm_plan* plan, const double* q_re_dev, const double* q_im_dev,
                  double* phi_out_dev, double* field_out_dev, int32_t precision,
                  void* stream);

/* Read and clear the plan's device error flag (synchronises the stream). No
 * counterpart: the reference's XLA programs have no device error path. */
int hfmm_plan_check(hfmm_plan* plan, void* stream);

/* Free the plan and everything it owns (the reference's state dict is freed by
 * Python's garbage collector, kifmm/setup.py:220-226). */
void hfmm_plan_destroy(hfmm_plan* plan);

/* Failure-path test hook of the mixed M2L kernel (process-wide; applies to the
 * launches that follow). wait_ns: the limit of each of its bounded mbarrier
 * waits (0 restores the default, 2 s). starve != 0 leaves the first operand
 * stage of every CTA without its gather arrivals, so a wait runs out: the kernel
 * then drains what it issued, frees its tensor memory, sets the timeout flag (4)
 * that hfmm_plan_check reports as HFMM_ERR_DEVICE, and returns. No counterpart
 * in the reference (XLA programs have no device error path). */
int hfmm_debug_m2l_wait(uint64_t wait_ns, int starve);

/* Source layout of the mixed M2L on complete tree levels (process-wide; applies to
 * the evaluates that follow): on != 0 (the default) lets a level whose every box is
 * present read its compressed densities, with complex charges, from a dense box
 * grid by strided TMA copies; on == 0 gathers them per target like every other
 * level. The two agree to the FP32 accumulation order. For tests and timing. No
 * counterpart in the reference. */
int hfmm_debug_m2l_grid(int on);

/* ---- inspection (tests compare these with the oracle bit for bit) ---- */
/* Tree arrays of the active boxes: m_id (uint64), p_id, lvls, counts (int32),
 * is_leaf (uint8), each of length n_boxes; sort_idx (int32, n). Host buffers. */
int hfmm_export_tree(const hfmm_plan* plan, uint64_t* m_id, int32_t* p_id, int32_t* lvls,
                     int32_t* counts, uint8_t* is_leaf, int32_t* sort_idx);
/* Particles-in-leaf table (n_boxes x maxleaf, -1 padded), cubic.py:683-693. Host buffer. */
int hfmm_export_pil(const hfmm_plan* plan, int32_t* pil);
/* List `which` (0 = V, 1 = U, 2 = W, 3 = X, 4 = near pairs) as (len x 2) int32, host. */
int hfmm_export_list(const hfmm_plan* plan, int32_t which, int32_t* pairs, int64_t cap);
/* Densities left by the last HFMM_PREC_FP64 evaluate, for per-phase checks: which = 0
 * the upward equivalent densities after P2M and M2M (phases.py:79-173), 1 the downward
 * local densities after M2L, P2L and L2L (phases.py:176-280, 1709-1770), both for the
 * boxes of levels 2..max_depth (other rows are 0). `columns` is that evaluate's charge
 * columns (1 real, 2 complex). Host buffer of n_families x n_boxes x columns x n_s
 * doubles, `cap` its capacity in doubles. Synchronises the device. The mixed path with a
 * compressed M2L keeps scaled SVD coordinates in these arrays instead. */
int hfmm_export_densities(const hfmm_plan* plan, int32_t which, int32_t columns, double* out,
                          int64_t cap);

/* ---- referee ---- */
/* Direct sum phi_t = sum_{s: r>0} q_s e^{ikr}/r (test.py:11-18) at n_t targets
 * (indices into the n points), with the field when field_out_dev != NULL.
 * Partial sums go to a scratch buffer the library allocates per call. */
int hfmm_direct(const double* pos_dev, const double* q_re_dev, const double* q_im_dev,
                int64_t n, const int32_t* targets_dev, int64_t n_t, double k,
                double* phi_out_dev, double* field_out_dev, void* stream);
/* hfmm_direct for a kernel kind: HFMM_KERNEL_YUKAWA sums q_s exp(-k r)/(4 pi r)
 * (field: q_s (1 + k r) exp(-k r)/(4 pi r^3) (x_t - x_s)) with complex charges by
 * linearity. Replaces the reference's own direct checks of its other kernels. */
int hfmm_direct_kernel(int32_t kind, const double* pos_dev, const double* q_re_dev,
                       const double* q_im_dev, int64_t n, const int32_t* targets_dev,
                       int64_t n_t, double k, double* phi_out_dev, double* field_out_dev,
                       void* stream);

/* hfmm_direct without allocation or synchronisation, for a check that overlaps
 * other work: the caller gives a device scratch of hfmm_direct_scratch_bytes(n,
 * n_t) bytes and a device int err_dev that out-of-range targets OR ERRF bits into
 * (the caller zeroes and reads it). Asynchronous on `stream`. No counterpart in
 * the reference. */
int64_t hfmm_direct_scratch_bytes(int64_t n, int64_t n_t);
int hfmm_direct_async(const double* pos_dev, const double* q_re_dev, const double* q_im_dev,
                      int64_t n, const int32_t* targets_dev, int64_t n_t, double k,
                      double* phi_out_dev, double* field_out_dev, double* scratch_dev,
                      int64_t scratch_bytes, int* err_dev, void* stream);

/* Same result as hfmm_direct without allocating anything, for callers that
 * cannot allocate device memory (a JAX/XLA process whose allocator owns the GPU
 * memory and runs foreign code inside that budget). No counterpart in the
 * reference. The partial
 * sums live in a fixed 8 MiB device array inside this library, so n_t is limited
 * to 131072 targets (HFMM_ERR_CAPACITY above that). The first call on a device
 * looks up that array's address (a one-time set-up on that device). All calls
 * share the array: calls that overlap on the GPU race. An out-of-range target
 * index gives HFMM_ERR_ARG; the error word is cleared at the start of every
 * call. Synchronises `stream`. */
int hfmm_direct_noalloc(const double* pos_dev, const double* q_re_dev, const double* q_im_dev,
                        int64_t n, const int32_t* targets_dev, int64_t n_t, double k,
                        double* phi_out_dev, double* field_out_dev, void* stream);

/* ---- phase timers ---- */
/* With profiling on, hfmm_evaluate records CUDA events around each phase on its
 * stream. hfmm_plan_phase_times synchronises and writes the milliseconds spent
 * per phase, summed over every evaluate since profiling was enabled or the
 * previous read (up to 8192 phase instances): 0 charge gather, 1 P2M, 2 M2M GEMM, 3 upward decode,
 * 4 M2L (with L2L fused on the FP64 path), 5 X-list P2L, 6 downward decode,
 * 7 P2P, 8 L2P, 9 W-list M2P, 10 combine, 11 TF32 splits of the mixed path,
 * 12 M2L table generation of a streaming plan, 13 the FP64 L2L GEMM of the mixed
 * path, 14 compress / expand GEMMs of a compressed M2L. (Replaces the reference's
 * wall-clock phase prints; it has no per-phase timers, util.py:692-724.) */
#define HFMM_N_PHASES 15
int hfmm_plan_set_profiling(hfmm_plan* plan, int32_t enable);
int hfmm_plan_phase_times(hfmm_plan* plan, double* ms_out);

/* Compressed M2L for the mixed path (no counterpart in the reference, which
 * applies each of a level's 316 M2L matrices densely, kifmm/phases.py:176-237):
 * with U (n_s x rank, row-major float64, device) spanning the level's dominant
 * M2L subspace and C (316 x rank x rank, row-major float64, device) with
 * C_d = U^T K_d U, the mixed evaluate computes M2L as U (sum_d C_d (U^T x_d)).
 * Give every level 2..max_depth of every family before hfmm_plan_finalize; the
 * FP64 evaluate keeps the dense tables (hfmm_b200/compress.py builds U and C). */
int hfmm_plan_set_m2l_compressed(hfmm_plan* plan, int32_t family, int32_t level, int32_t rank,
                                 const double* U_dev, const double* C_dev);

/* ---- batches (no counterpart in the reference: one problem per call there) ---- */
/* Many finalized plans (problems of uneven size and wavenumber) evaluated by one
 * CUDA-graph launch. hfmm_batch_create spreads the plans over n_streams streams
 * (longest work estimate first, onto the least loaded stream) and gives each
 * stream one M2L-table workspace shared by its streaming plans
 * (hfmm_plan_set_streaming). Set every problem's device charges and outputs
 * (same meaning as hfmm_evaluate), capture once, then launch as often as
 * wanted; changing a problem's pointers drops the graph until the next capture.
 * Read each plan's device error flag with hfmm_plan_check after a launch.
 * A plan belongs to at most one batch at a time; destroying the batch hands
 * streaming plans back to their own workspace (allocated at their next
 * hfmm_evaluate); destroying a plan first disables the batch's launches. */
typedef struct hfmm_batch hfmm_batch;
int hfmm_batch_create(hfmm_plan* const* plans, int32_t n_plans, int32_t n_streams,
                      hfmm_batch** out);
/* Stream index [0, n_streams) plan i runs on (>= 0), or a negative status. */
int hfmm_batch_stream_of(const hfmm_batch* batch, int32_t i);
int hfmm_batch_set_problem(hfmm_batch* batch, int32_t i, const double* q_re_dev,
                           const double* q_im_dev, double* phi_out_dev, double* field_out_dev,
                           int32_t precision);
/* Optional: check problem i in the graph against the FP64 direct sum (the referee
 * of test.py:11-18) at n_t target indices. pos_dev: the n x 3 positions (input
 * order) the plan was built from. After each launch sums_dev[0..3] hold
 * sum |phi - phi_ref|^2, sum |phi_ref|^2, sum |E - E_ref|^2, sum |E_ref|^2 over the
 * targets (the E terms are 0 without a field output). */
int hfmm_batch_set_check(hfmm_batch* batch, int32_t i, const double* pos_dev,
                         const int32_t* targets_dev, int32_t n_t, double* sums_dev);
int hfmm_batch_capture(hfmm_batch* batch);
int hfmm_batch_launch(hfmm_batch* batch, void* stream);
void hfmm_batch_destroy(hfmm_batch* batch);

/* Queued M2L of a batch (no counterpart in the reference): with on != 0 (the
 * default), a batch whose problems all run the low-rank mixed evaluate with the same
 * charge columns is captured as every plan's upward half, ONE persistent M2L kernel
 * draining a device queue of every plan's M2L work items (tile x row block of each
 * level and family, largest first; the CTAs take items with an atomic counter), and
 * every plan's downward half. on == 0 captures each plan's evaluate whole, on
 * streams. Takes effect at the next hfmm_batch_capture; hfmm_batch_queued reports
 * whether the captured graph uses the queue (1) or not (0), and
 * hfmm_batch_queue_note why not (an empty string when it does; valid until the
 * next capture or the batch's destruction). */
int hfmm_batch_set_queue(hfmm_batch* batch, int32_t on);
/* The low-rank mixed M2L of one plan's evaluate (no counterpart in the reference): with
 * on != 0 (the default) every level and family runs in ONE persistent launch over the
 * plan's own queue of (level, family, tile, row block) items, largest first, built at
 * finalize; on == 0 launches one kernel per level and family on the plan's side
 * streams. Results are the same bit for bit. */
int hfmm_plan_set_m2l_queue(hfmm_plan* plan, int32_t on);

/* Rotation-based M2L of the FP64 evaluate (the reference's rotation M2L is Laplace's,
 * kernels/laplace/transf.py:143-250; its Helmholtz path uses KIFMM tables,
 * kifmm/phases.py:176-237): per V pair, the source box's multipole coefficients of
 * order `order` are rotated into the frame whose z axis is the displacement, shifted
 * along z and rotated back, O(order^3). A displacement slot's ((dx+3)*49 + (dy+3)*7 +
 * (dz+3)) rotation R_y(-theta) R_z(-phi) has blocks T_n = D_n(theta) diag(e^{i m phi}):
 * D_host [n_theta][sum_{n<=order} (2n+1)^2] real holds D_n, row-major per block, for
 * each distinct polar angle; theta_host[343] each slot's angle index (-1 adjacent);
 * phase_host [343][2 order+1] complex (re, im interleaved) e^{i m phi}, m = -order..order;
 * dist_host[343] each slot's coaxial matrix index (-1 adjacent), n_dist of them. order 0
 * returns to the dense M2L tables. Then, per family and level,
 * hfmm_plan_set_rotation_level with Q [(order+1)^2][n_s] complex (multipole from
 * equivalent density), E [n_s][(order+1)^2] complex (check potential from local
 * coefficients, times pref, real part) and C [n_dist][2 order+1][order+1][order+1] real
 * (the coaxial shifts: C[d][m + order][n'][n] takes multipole (n, m) to local (n', m)).
 * The library keeps its own transposed copies. hfmm_b200/rotation.py builds all of
 * them. Only the FP64 evaluate uses it; after hfmm_plan_rebuild set it again. */
int hfmm_plan_set_m2l_rotation(hfmm_plan* plan, int32_t order, const double* D_host, int32_t n_theta,
                               const int32_t* theta_host, const double* phase_host,
                               const int32_t* dist_host, int32_t n_dist);
int hfmm_plan_set_rotation_level(hfmm_plan* plan, int32_t family, int32_t level, const double* Q_host,
                                 const double* E_host, const double* C_host, double pref);
int hfmm_batch_queued(const hfmm_batch* batch);
const char* hfmm_batch_queue_note(const hfmm_batch* batch);

/* ---- expansion-order network (no counterpart in the reference) ---- */
/* A 3 x 64 FP32 MLP (tanh hidden layers, linear output) over in_dim features
 * with out_dim outputs. Parameters are one flat device FP32 array of
 * hfmm_mlp_param_count(in_dim, out_dim) floats: W1[in][64] b1[64] W2[64][64] b2[64]
 * W3[64][64] b3[64] W4[64][out] b4[out]. X is (n, in_dim), targets/outputs
 * (n, out_dim), all row-major on the device. Loss = mean squared error over
 * samples and outputs. in_dim 1..64, out_dim 1..4. It picks the expansion order
 * that the reference takes from the caller (HFMM.py:55-80). */
int hfmm_mlp_param_count(int32_t in_dim, int32_t out_dim);
int hfmm_mlp_forward(const float* params_dev, const float* X_dev, int32_t n, int32_t in_dim,
                     int32_t out_dim, float* Y_dev, void* stream);
/* Full-batch gradient of the loss (written to grad_dev) and the loss itself. Synchronises. */
int hfmm_mlp_grad(const float* params_dev, const float* X_dev, const float* T_dev, int32_t n,
                  int32_t in_dim, int32_t out_dim, float* grad_dev, double* loss, void* stream);
/* `steps` full-batch Adam steps (b1 0.9, b2 0.999, eps 1e-8) continuing from
 * step number step0 with the moment arrays adam_m/adam_v (param_count floats
 * each, zero at step0 = 0); *loss is the loss after the last step. Synchronises. */
int hfmm_mlp_train(float* params_dev, float* adam_m_dev, float* adam_v_dev, int64_t step0,
                   const float* X_dev, const float* T_dev, int32_t n, int32_t in_dim,
                   int32_t out_dim, int32_t steps, float lr, double* loss, void* stream);

/* ---- diagnostics ---- */
const char* hfmm_last_error(void);
/* Kernels this library has launched since load (all plans, all threads). */
int64_t hfmm_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif /* HFMM_B200_H */
