/*
 * fmm_b200.h -- C ABI of the B200 evaluator for the FMM evaluation passes.
 *
 * Two layers, both plain C (pointers, sizes, status codes; no CUDA or torch types):
 *
 * 1. The FMM entry points (fmmgpu_fmm_*) mirror the user API of the reference,
 *    nd-fmm-exec's FmmBuilder / Fmm (fmm-exec/src/fmm.rs:1853 build, :3691 evaluate,
 *    :3719 evaluate_into): build once from source and target points in the caller's
 *    order, then evaluate charge vectors into potentials (and gradients) in the
 *    caller's order, with 1/(4 pi) applied (phi(x) = sum_j q_j / (4 pi |x - y_j|)).
 *    The build makes the plan on the host (octree, lists, f64 operator tables) and
 *    uploads it; an evaluation runs every pass on the GPU.
 *
 * 2. The operator entry points (fmmgpu_op_*) are the level calls of the reference's
 *    drop-in boundary, the FmmOperator trait (fmm-plan/src/operator.rs:434-492): one
 *    call per (level, kind) that queues device work and adds into its output in the
 *    trait's accumulation order (operator.rs:34-45).  A host that keeps its own plan
 *    (nd-fmm-exec's Engine::Device seam, fmm-exec/src/fmm.rs:2564-2568) drives an
 *    evaluation through these calls between fmmgpu_op_begin_evaluation and
 *    fmmgpu_op_read_output.
 *
 * Errors: every call returns an fmmgpu_status; a device error surfaces at the next
 * call that synchronises (evaluate, read_output), as the reference's device errors
 * surface at read_output (fmm-kernels/src/lib.rs:64-66).  fmmgpu_last_error() gives
 * the message of the last failure on the calling thread.
 */
#ifndef FMM_B200_H
#define FMM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    FMMGPU_OK = 0,
    FMMGPU_INVALID_ARGUMENT = 1,     /* settings or inputs rejected before any GPU work */
    FMMGPU_UNSUPPORTED = 2,          /* expansion order or precision not compiled in */
    FMMGPU_DEVICE_MEMORY = 3,        /* the device buffers do not fit */
    FMMGPU_DEVICE_ERROR = 4,         /* a CUDA call or kernel failed */
    FMMGPU_NO_DEVICE = 5             /* no CUDA device is visible */
} fmmgpu_status;

typedef enum {
    FMMGPU_PRECISION_F64 = 0,   /* the plain f64 evaluator (the drop-in) */
    FMMGPU_PRECISION_MIXED = 1  /* f32 points/expansions, f64 per-target accumulation */
} fmmgpu_precision;

/* FmmBuilder settings (fmm-exec/src/fmm.rs:1228-1270 names and defaults). */
typedef struct {
    int p;                    /* expansion order */
    int precision;            /* fmmgpu_precision */
    int gradients;            /* 0: potentials only, 1: potentials and gradients */
    int vectors;              /* m >= 1 charge vectors at the same points */
    int max_points_per_leaf;  /* refinement target (distinct level-16 keys per leaf) */
    int max_level;            /* deepest leaf level, 0-16 */
    int device;               /* CUDA device ordinal */
    int vectors_per_pass;     /* charge vectors per device pass: 0 (default) as many as fit in
                                 60% of the free device memory; rounded down to a divisor of
                                 `vectors`; the results do not depend on it */
    int autotune;             /* 1: time the launch shapes at build and keep the fastest
                                 (fmm-exec/src/fmm.rs:291-300, FmmBuilder::tuning_cache, with
                                 no cache file); 0 (default): the static shapes.  The results
                                 are the same bits either way */
    int64_t product_bytes;    /* M2L product buffer: 0 (default) every V pair's products at
                                 once when they fit beside the rest (else at most 20% of the
                                 free memory); > 0 at most this many bytes, the products
                                 then made and reduced level by level in chunks of target
                                 boxes.  The results do not depend on it */
    const char* table_cache;  /* directory of the operator-table cache (FmmBuilder::table_cache,
                                 fmm-exec/src/fmm.rs:1410-1425; the reference's TableCache
                                 files, fmm-tables/src/cache.rs): tables are loaded from it,
                                 or built and stored there; NULL (default): always built */
    const char* tuning_cache; /* directory of the autotuner's choices (FmmBuilder::tuning_cache,
                                 fmm.rs:1655-1669): with autotune on, a choice kept there for
                                 this device, precision and p is used instead of timing, and
                                 new timings are stored; NULL (default): no file */
} fmmgpu_settings;

typedef struct {
    int nlevels;
    int64_t nboxes, nleaves, nsources, ntargets;
    int64_t near_pairs;   /* source-target point pairs of P2P over all near rows */
    int64_t v_pairs;      /* M2L box pairs */
    int64_t w_pairs, x_pairs;
    int64_t device_bytes; /* device memory held by the evaluator */
    int64_t close_pairs;  /* near-singular P2P pairs the mixed form evaluates in f64 */
    int64_t launches;     /* kernels the last evaluation launched (0 before the first) */
    int64_t vectors_per_pass;  /* charge vectors per device pass (0 for a plan-only handle) */
    int64_t p2p_warps;    /* warps a block of the mixed P2P kernel (static 4, or the tuned one) */
    int64_t leaf_block;   /* threads a block of the L2P / M2P kernel (static 64, or the tuned one) */
    int64_t product_chunks; /* chunks of the M2L product path (0: every product at once) */
    int64_t p2p_stream_bytes; /* the mixed P2P's near-row source streams (0: mapped per flush) */
    int64_t tables_loaded;    /* tables the build took from the table cache: bit 0 M2L, 1 M2M, 2 L2L */
    int64_t tuning_loaded;    /* 1: the launch shapes came from the tuning cache */
    int64_t m2l_tile_columns; /* columns of a tensor-core M2L tile (the tuned one; 0: no tensor-core M2L) */
    int64_t vjp_forward_reused; /* VJPs that took the stored forward pass (fmmgpu_fmm_set_vjp_store) */
} fmmgpu_info;

typedef struct fmmgpu_fmm fmmgpu_fmm;

/* Settings with the reference's defaults: p = 6, f64, no gradients, one vector,
 * 64 points per leaf, max level 16, device 0 (and vectors per pass chosen by memory). */
void fmmgpu_default_settings(fmmgpu_settings* settings);

/* FmmBuilder::build (fmm.rs:1853): sources/targets are n x 3 doubles, caller order. */
int fmmgpu_fmm_build(const fmmgpu_settings* settings, size_t nsources, const double* sources,
                     size_t ntargets, const double* targets, fmmgpu_fmm** out);

/* The host half of a build only (plan, lists, tables), no device needed: the handle
 * answers info/boxes/list/tables and must be destroyed, but cannot evaluate. */
int fmmgpu_plan_build(const fmmgpu_settings* settings, size_t nsources, const double* sources,
                      size_t ntargets, const double* targets, fmmgpu_fmm** out);

/* A plan made outside the library (the reference's one-rank Plan, fmm-plan/src/plan.rs,
 * with the views its level calls receive, fmm-plan/src/operator.rs:170-317, and its list
 * CSRs, fmm-plan/src/lists.rs:172-282), flattened over all levels:
 *  - boxes level-major, key order within a level (box t of level l is global box
 *    level_start[l] + t: the reference's BoxIndex per level); keys are the reference's
 *    Morton keys (octree/src/morton.rs: 3 interleaved index bits a level, x highest,
 *    shifted left 15, the level in the low 15 bits);
 *  - leaves are the leaf boxes in box order (the reference's leaf index); leaf j holds the
 *    leaf-order points source_offsets[j] .. source_offsets[j + 1] (targets likewise), and
 *    source_order[a] / target_order[a] is the caller index of leaf-order point a;
 *  - the cubic domain: lower corner and side (fmm-exec/src/geometry.rs:120-147);
 *  - the lists as CSR (row offsets int64, entries int32), rows in the reference's
 *    accumulation order (operator.rs:34-45): near (per leaf: leaf indices, the leaf itself
 *    included, ascending), W (per leaf: box indices on the next level, ascending), X (per
 *    box: leaf indices, ascending), V (per box: source boxes of the same level with their
 *    offset indices 0..315, fmm-plan/src/lists.rs:100, by offset index; the batches of the
 *    reference's GroupedCsr are formed from them).
 * Every array is read during the call only. */
typedef struct {
    int nlevels;
    const int64_t* level_start;      /* nlevels + 1 */
    const uint64_t* keys;            /* level_start[nlevels] boxes */
    const uint8_t* is_leaf;          /* per box */
    double lower[3];
    double side;
    const int64_t* source_offsets;   /* nleaves + 1 */
    const int64_t* target_offsets;   /* nleaves + 1 */
    const int64_t* source_order;     /* nsources */
    const int64_t* target_order;     /* ntargets */
    const int64_t* near_rows;        /* nleaves + 1 */
    const int32_t* near;
    const int64_t* w_rows;           /* nleaves + 1 */
    const int32_t* w;
    const int64_t* x_rows;           /* nboxes + 1 */
    const int32_t* x;
    const int64_t* v_rows;           /* nboxes + 1 */
    const int32_t* v;
    const int32_t* v_offsets;        /* the offset index of each V entry */
} fmmgpu_plan_arrays;

/* The FmmOperator's device operator created on a caller's plan (the reference's
 * DeviceOperator::new, fmm-exec/src/device.rs:3032, which uploads the plan's views,
 * geometry and tables): the plan is checked (a complete octree of consistent keys, every
 * index in range, rows ordered, each point inside its leaf, near rows 2:1-balanced) and
 * uploaded with the f64 tables of settings->p and the points' leaf-scaled coordinates;
 * settings->max_points_per_leaf and max_level are not used.  The handle then answers every
 * call an fmmgpu_fmm_build handle does, the level calls on this plan.  A vector-Jacobian
 * product needs targets == sources here.  FMMGPU_INVALID_ARGUMENT names the first check
 * that failed. */
int fmmgpu_upload_plan(const fmmgpu_settings* settings, const fmmgpu_plan_arrays* plan, size_t nsources,
                       const double* sources, size_t ntargets, const double* targets, fmmgpu_fmm** out);
/* The same without a device (checks, host tables, a plan-only handle as fmmgpu_plan_build's). */
int fmmgpu_plan_from_arrays(const fmmgpu_settings* settings, const fmmgpu_plan_arrays* plan, size_t nsources,
                            const double* sources, size_t ntargets, const double* targets, fmmgpu_fmm** out);
/* The arrays of a handle's plan in that layout (pointers into the handle, valid while it
 * lives): what fmmgpu_upload_plan takes, so a plan round-trips. */
int fmmgpu_fmm_plan_arrays(const fmmgpu_fmm* fmm, fmmgpu_plan_arrays* plan);

/* Multi-cloud batch (no reference counterpart: the reference batches charge vectors
 * only, FmmBuilder::vectors, fmm.rs:200-227): `ncloud` independent clouds, cloud c with
 * nsources[c] sources and ntargets[c] targets (ntargets NULL: the targets are the
 * sources), their points consecutive in `sources` / `targets` (n x 3 doubles).  Each
 * cloud gets its own octree, exactly as fmmgpu_fmm_build would build it (in parallel
 * over the host's threads); the trees are merged level by level into one forest, so every
 * pass of an evaluation is one launch over all clouds and the M2L batches by offset span
 * the whole batch.  The handle is an ordinary fmmgpu_fmm: charges, potentials and
 * gradients are the clouds' arrays concatenated in cloud order, and each cloud's results
 * are the floats its own FMM gives. */
int fmmgpu_batch_build(const fmmgpu_settings* settings, size_t ncloud, const size_t* nsources,
                       const double* sources, const size_t* ntargets, const double* targets, fmmgpu_fmm** out);
/* The host half of a batch build only (no device), like fmmgpu_plan_build. */
int fmmgpu_batch_plan_build(const fmmgpu_settings* settings, size_t ncloud, const size_t* nsources,
                            const double* sources, const size_t* ntargets, const double* targets,
                            fmmgpu_fmm** out);

/* Fmm::evaluate_into (fmm.rs:3719) with HOST buffers: charges[i*m + v] (caller order,
 * m charges of a source adjacent); potential[v*nt + i]; gradient[(v*nt + i)*3 + k] (or
 * NULL without gradients).  Copies in, evaluates, copies out, synchronises. */
int fmmgpu_fmm_evaluate(fmmgpu_fmm* fmm, const double* charges, double* potential, double* gradient);

/* Fmm<f32>::evaluate_into (fmm.rs:3719 with T = f32, the value type of the reference's
 * f32 runs, fmm-bench/src/measure.rs:196) with HOST f32 buffers in the layouts of
 * fmmgpu_fmm_evaluate: the charges are widened to f64 on the device (exactly), the
 * evaluation is fmmgpu_fmm_evaluate's, and the potentials and gradients are rounded to
 * the nearest f32 on the device, so each element is the f64 call's result on the widened
 * charges, rounded; the copies move half the bytes.  Synchronises. */
int fmmgpu_fmm_evaluate_f32(fmmgpu_fmm* fmm, const float* charges, float* potential, float* gradient);

/* Vector-Jacobian product of the potentials (no reference counterpart; the reference has
 * no adjoint): for charges q and a cotangent w on the potentials (both HOST buffers, the
 * layouts of fmmgpu_fmm_evaluate: q[i*m + v], w[v*nt + i]) it returns
 *   dcharges[j*m + v] = sum_i w[v][i] G(t_i - s_j)             (the transpose FMM),
 *   dsources[3j + k]  = sum_v q[j][v] d/ds_jk sum_i w[v][i] G(t_i - s_j),
 *   dtargets[3i + k]  = sum_v w[v][i] d phi_v / dt_ik,
 * G = 1/(4 pi r), coincident pairs excluded as in the evaluation.  Two FMM passes, both
 * recomputed (no expansion is stored between them): the forward one with gradients and
 * the transpose one (charges w at the targets, evaluated with gradients at the sources),
 * which for an FMM built with targets == sources (the same pointer) is this FMM again;
 * otherwise the swapped FMM is built once at the first call and kept.  Needs gradients
 * on; not offered for multi-cloud batches.  Synchronises. */
int fmmgpu_fmm_vjp(fmmgpu_fmm* fmm, const double* charges, const double* cotangent, double* dcharges,
                   double* dsources, double* dtargets);

/* The same with DEVICE buffers on the evaluator's stream; does not synchronise. */
int fmmgpu_fmm_evaluate_device(fmmgpu_fmm* fmm, const double* charges, double* potential,
                               double* gradient);

/* The evaluator's CUDA stream (a cudaStream_t), for timing with events on it. */
void* fmmgpu_fmm_stream(fmmgpu_fmm* fmm);

/* Whole-sweep CUDA graph (on = 1): the next evaluation (fmmgpu_fmm_evaluate or
 * _evaluate_device) is captured into one CUDA graph, every pass of it, and later
 * evaluations with the same charge / potential / gradient buffers replay that graph
 * (one launch from the host); new buffers, or changed settings, re-capture.  The same
 * kernels run, so the results are the same floats.  Ignored while per-kind timing is on.
 * Off (0) by default.  Synchronises. */
int fmmgpu_fmm_set_graph(fmmgpu_fmm* fmm, int on);

/* Near field beside the far field (on = 1): an evaluation runs P2P on a second,
 * lower-priority stream, concurrently with the far-field passes, and one output pass adds
 * the two (the same addition as the serial order, so the same floats).  0, the default,
 * runs everything on one stream (on one B200 the two halves compete for the same FP32
 * pipes and the overlap measured no faster).  Per-kind timing always runs on one stream.
 * Synchronises. */
int fmmgpu_fmm_set_overlap(fmmgpu_fmm* fmm, int on);

/* Times the launch shapes that change no result on this handle's plan and device and
 * keeps the fastest (the reference's build-time tuner, fmm-exec/src/tune.rs:1-60, with
 * the P2P layout decision as the block of the mixed P2P kernel, 1, 2 or 4 warps, the
 * L2P / M2P block, 32, 64 or 128 threads, and the tensor-core M2L tile, its default or
 * its alternative column count: fmmgpu_fmm_set_m2l_tile, info.m2l_tile_columns).  `charges` as fmmgpu_fmm_evaluate's (host);
 * the handle's device outputs then hold their evaluation.  choice (may be NULL) receives
 * {p2p warps, leaf block}.  Every target sums the same terms in the same order whatever
 * the shape, so later evaluations give the same bits as before.  Drops a captured graph.
 * Synchronises. */
int fmmgpu_fmm_autotune(fmmgpu_fmm* fmm, const double* charges, int* choice);

/* Sets the launch shapes fmmgpu_fmm_autotune chooses (a choice kept from an earlier
 * tuning, as the reference's tuning cache keeps one, fmm-exec/src/fmm.rs:291-300):
 * p2p_warps 1, 2 or 4; leaf_block 32, 64 or 128.  The results are the same bits for
 * every pair.  Drops a captured graph.  Synchronises. */
int fmmgpu_fmm_set_launch_shapes(fmmgpu_fmm* fmm, int p2p_warps, int leaf_block);

/* The VJP's forward pass, stored or recomputed.  on = 1: every following evaluation with
 * gradients (host or device call, and a VJP's own forward pass) keeps a device copy of its
 * charges and target gradients (8 m (N_s + 3 N_t) bytes), and a VJP whose charges equal the
 * kept ones bit for bit (checked on the device) takes the kept gradients instead of running
 * the forward FMM (the same floats: the same evaluation).  on = 0 (the default, and what
 * memory asks for): every VJP recomputes its forward pass; the store is freed.  Refused with
 * FMMGPU_DEVICE_MEMORY when the store would take more than half the free device memory.
 * info.vjp_forward_reused counts the VJPs that used it.  Synchronises. */
int fmmgpu_fmm_set_vjp_store(fmmgpu_fmm* fmm, int on);

/* The tensor-core M2L tile of the following evaluations (mixed precision): 0 its default
 * columns (128 at p <= 6, 96 at p = 7, 8, 64 at p = 9, 10, 48 at p = 11, 12), 1 the
 * alternative (64 where the default has 96 or 128, else 32; more raw stages in flight).
 * Every product is the same float either way.  The autotuner picks one; a tuning cache
 * keeps it.  Drops a captured graph.  Synchronises. */
int fmmgpu_fmm_set_m2l_tile(fmmgpu_fmm* fmm, int tile);

/* Per-kind device timing of the following evaluations (the reference's KindTiming,
 * fmm-exec/src/fmm.rs:150-153): every launch is bracketed by CUDA events. */
int fmmgpu_fmm_set_kind_timing(fmmgpu_fmm* fmm, int on);
/* Which parts the following evaluations run, for tests: bit 0 the near field (P2P),
 * bit 1 the far field (everything that reaches L2P and M2P); 3, the default, is the FMM. */
int fmmgpu_fmm_set_kinds(fmmgpu_fmm* fmm, int kinds);
/* Which M2L the following evaluations use (mixed precision, p <= 8; f64 always runs 0):
 * 1 (default) the tensor-core products then the ordered local reduce, 2 the tensor-core
 * M2L fused with the local reduce (products added into the locals in row order, no
 * product array; at most 128 vectors a pass, 64 at p = 8), 0 SIMT products then the
 * reduce.  2 and 1 give the same bits.  Synchronises. */
int fmmgpu_fmm_set_m2l_path(fmmgpu_fmm* fmm, int path);
/* Where the mixed P2P takes its sources from, for tests: 1 (the default when the streams
 * were built: at most a quarter of the free device memory) every near row's sources
 * mapped into its target leaf's frame once, at build time, and copied per flush; 0 the
 * sources mapped per flush.  The same bits.  Synchronises. */
int fmmgpu_fmm_set_p2p_path(fmmgpu_fmm* fmm, int path);
/* Milliseconds of the last evaluation per kind: [0] charge load (in timed evaluations
 * with the mixed form's f64 sums of the near-singular pairs, which otherwise run beside
 * the far field), [1] P2M, [2] M2M, [3] L2L, [4] M2L, [5] P2L, [6] L2P + M2P, [7] P2P +
 * output pass.  Synchronises. */
int fmmgpu_fmm_kind_times(fmmgpu_fmm* fmm, double* ms);

/* Waits for the stream and returns the first device error, if any. */
int fmmgpu_fmm_synchronize(fmmgpu_fmm* fmm);

int fmmgpu_fmm_info(const fmmgpu_fmm* fmm, fmmgpu_info* info);

void fmmgpu_fmm_destroy(fmmgpu_fmm* fmm);

/* Plan export, for tests: level-major box keys (nboxes u64) and leaf flags (u8). */
int fmmgpu_fmm_boxes(const fmmgpu_fmm* fmm, uint64_t* keys, uint8_t* is_leaf);
/* The rows of one list (kind 0 near, 1 V, 2 W, 3 X) as box keys; row = leaf index for
 * near/W, box index for V/X.  Returns the count (writes at most cap keys), or -1. */
int64_t fmmgpu_fmm_list(const fmmgpu_fmm* fmm, int kind, int64_t row, uint64_t* keys, int64_t cap);
/* The f64 tables the plan uploaded: 316 M2L, 8 M2M, 8 L2L, column-major (p+1)^2 squares. */
int fmmgpu_fmm_tables(const fmmgpu_fmm* fmm, double* m2l, double* m2m, double* l2l);

/* ---- Operator level calls: the FmmOperator trait (fmm-plan/src/operator.rs:434-492) ----
 * The host drives an evaluation level by level on the plan the build made, in the
 * reference evaluator's schedule (fmm-plan/src/evaluator.rs:368-440):
 *   begin_evaluation(charges);
 *   for l = L..0:  p2m(l); if l > 0: m2m(l - 1)          upward
 *   for l = 1..L:  l2l(l); m2l(l); p2l(l)                downward
 *   for l = 0..L:  l2p(l); m2p(l); p2p(l)                leaves
 *   read_output(potential, gradient).
 * Every call queues work on the evaluator's stream and adds into its output (the
 * multipoles, the locals or the leaf-order target store) in the trait's accumulation
 * order (operator.rs:34-45); a call with nothing to do on its level is a no-op, as the
 * trait requires every call on every level (operator.rs:409-424).  Made in this order,
 * the calls give the same floats as fmmgpu_fmm_evaluate.  Level calls return
 * FMMGPU_INVALID_ARGUMENT for a level outside 0..nlevels-1 or before begin_evaluation;
 * device errors surface at read_output (fmm-kernels/src/lib.rs:64-66). */
typedef enum {
    FMMGPU_OP_P2M = 0,
    FMMGPU_OP_M2M = 1,  /* parents on `level` from their children on level + 1 */
    FMMGPU_OP_L2L = 2,  /* boxes on `level` from their parents on level - 1 */
    FMMGPU_OP_M2L = 3,
    FMMGPU_OP_P2L = 4,
    FMMGPU_OP_L2P = 5,
    FMMGPU_OP_M2P = 6,
    FMMGPU_OP_P2P = 7
} fmmgpu_op_kind;

/* DeviceOperator::begin_evaluation (fmm-exec/src/device.rs:4386): HOST charges in caller
 * order (charges[i*m + v]) to the device in leaf order; multipoles, locals and the
 * target store set to zero. */
int fmmgpu_op_begin_evaluation(fmmgpu_fmm* fmm, const double* charges);
int fmmgpu_op_p2m(fmmgpu_fmm* fmm, int level);
int fmmgpu_op_m2m(fmmgpu_fmm* fmm, int level);
int fmmgpu_op_l2l(fmmgpu_fmm* fmm, int level);
int fmmgpu_op_m2l(fmmgpu_fmm* fmm, int level);
int fmmgpu_op_p2l(fmmgpu_fmm* fmm, int level);
int fmmgpu_op_l2p(fmmgpu_fmm* fmm, int level);
int fmmgpu_op_m2p(fmmgpu_fmm* fmm, int level);
int fmmgpu_op_p2p(fmmgpu_fmm* fmm, int level);
/* FmmOperator::host_data (operator.rs:56-119): the exchange events of a distributed
 * evaluation; on one rank there is nothing to exchange and every event is accepted. */
int fmmgpu_op_host_data(fmmgpu_fmm* fmm, int event);
/* DeviceOperator::read_output (device.rs:4687) and the output pass (movement.rs:411,
 * fmm.rs:4750): phi = phi_hat / (4 pi r_t), g = g_hat / ((4 pi r_t) r_t) into HOST
 * buffers in caller order (layout of fmmgpu_fmm_evaluate); synchronises. */
int fmmgpu_op_read_output(fmmgpu_fmm* fmm, double* potential, double* gradient);

/* f64 direct sum on the GPU at the given targets: phi(x) = sum_j q_j / (4 pi |x - y_j|)
 * and its gradient (grad may be NULL), exactly coincident pairs skipped, Neumaier
 * compensation per target (fmm-ref/src/p2p.rs:147-186 with the FMM's 1/(4 pi)).
 * Host buffers in and out; allocates and frees its own device memory. */
int fmmgpu_direct_sum(size_t nsources, const double* sources, const double* charges, size_t ntargets,
                      const double* targets, double* potential, double* gradient, int device);

/* ---- Helmholtz, e^{ikr}/(4 pi r) (fmm-ref/src/helmholtz/p2p.rs; CONVENTIONS 3.15) ----
 * Complex values are (re, im) pairs of doubles; a complex gradient is (re x, im x, re y,
 * im y, re z, im z).  k = k_re + i k_im, finite.
 *
 * The f64 direct sum on the GPU (the reference's helmholtz::p2p::direct_sum: Neumaier per
 * real component, exactly coincident pairs skipped), with 1/(4 pi): charges[ns] complex,
 * potential[nt] and gradient[nt][3] complex (gradient may be NULL).  Host buffers. */
int fmmgpu_helmholtz_direct_sum(double k_re, double k_im, size_t nsources, const double* sources,
                                const double* charges, size_t ntargets, const double* targets, double* potential,
                                double* gradient, int device);

/* The Helmholtz near field of an FMM's plan: the P2P level calls of every level
 * (fmm-exec/src/helmholtz/operator.rs:2571-2615) on the near rows of the tree the build
 * made, in leaf-scaled coordinates with k_l = k r_l, in the handle's precision (f64, or
 * complex64 with the mixed form's f64 near-singular pairs).  charges[i*m + v] complex
 * (caller order), potential[v*nt + i] and gradient[(v*nt + i)*3 + k] complex (caller
 * order; the gradient when the FMM was built with gradients), with 1/(4 pi).  Host
 * buffers; synchronises.  fmmgpu_helmholtz_evaluate adds the far field. */
/* The dense M2L tables of one level for a real k > 0 (the reference's DenseM2l,
 * fmm-tables/src/helmholtz/dense.rs:1-30), built on the host in f64 by projection
 * (fmm-ref/src/helmholtz/direct.rs): boxes of half-width `half_width` (k in the same
 * units), degree p <= 30; writes 316 * 2 (p + 1)^4 doubles, per V-list offset d in index
 * order (target box at 2 half_width d from the source box) a real 2n x n matrix,
 * column-major, column j the local of the unit real multipole e_j (the real plane in rows
 * 0..n over the imaginary plane), n = (p + 1)^2.  No device needed. */
int fmmgpu_helmholtz_m2l_tables(int p, double k, double half_width, double* tables);
/* The M2M and L2L tables between a parent level of half-width `half_width` and its
 * children (the reference's per-level translation tables, fmm-ref/src/helmholtz/rcr.rs:129-156,
 * here by projection), 8 octants each in the layout above: child o centred at the parent
 * centre + half_width/2 (+-1, +-1, +-1), the sign of x from bit 2 of o, y bit 1, z bit 0;
 * m2m[o] takes the child's multipole to the parent's, l2l[o] the parent's local to the
 * child's.  Writes 8 * 2 (p + 1)^4 doubles to each.  No device needed. */
int fmmgpu_helmholtz_octant_tables(int p, double k, double half_width, double* m2m, double* l2l);

int fmmgpu_helmholtz_near(fmmgpu_fmm* fmm, double k_re, double k_im, const double* charges, double* potential,
                          double* gradient);

/* The whole Helmholtz FMM, e^{ikr}/(4 pi r), for a real wavenumber k = k_re > 0 (k_im must
 * be 0: the far field's tables are built for a real k), on the tree and lists the build
 * made: the reference's HelmholtzFmm evaluation (fmm-exec/src/helmholtz/fmm.rs; its
 * operator, fmm-exec/src/helmholtz/operator.rs:16-29, is host-only there).  Complex
 * expansions of degree p on every level in the real orthonormal harmonics and scaled
 * radial functions (fmm-ref/src/helmholtz/leaf.rs), the dense M2L tables of every level
 * (fmm-tables/src/helmholtz/dense.rs) and the M2M / L2L tables of every level built on the
 * host by projection (fmm-ref/src/helmholtz/direct.rs) when k is new (then kept for the
 * next calls with the same k), every pass on the GPU in the handle's precision (f64, or
 * f32 expansions and translations with complex64 near field and f64 near-singular pairs).
 * charges[i*m + v] complex (caller order), potential[v*nt + i] and gradient[(v*nt + i)*3 +
 * k] complex, with 1/(4 pi), HOST buffers; synchronises.  Not offered for multi-cloud
 * batches. */
int fmmgpu_helmholtz_evaluate(fmmgpu_fmm* fmm, double k_re, double k_im, const double* charges, double* potential,
                              double* gradient);
/* The same with complex64 HOST buffers (each complex number two floats, re then im; the
 * value type of a Helmholtz FMM of T = f32, fmm-exec/src/helmholtz/fmm.rs:2277): the
 * charges are widened to complex128 on the device, the evaluation is
 * fmmgpu_helmholtz_evaluate's, and the potentials and gradients are rounded to complex64
 * on the device, so the copies move half the bytes.  Synchronises. */
int fmmgpu_helmholtz_evaluate_f32(fmmgpu_fmm* fmm, double k_re, double k_im, const float* charges, float* potential,
                                  float* gradient);
/* The same with DEVICE buffers on the evaluator's stream; does not synchronise (the
 * tables of a new k are built, on the host, before the launches are queued). */
int fmmgpu_helmholtz_evaluate_device(fmmgpu_fmm* fmm, double k_re, double k_im, const double* charges,
                                     double* potential, double* gradient);
/* Host seconds the last new wavenumber's Helmholtz tables took to build. */
double fmmgpu_helmholtz_table_seconds(const fmmgpu_fmm* fmm);

/* The same direct sum on DEVICE buffers, allocating nothing.  No counterpart in the
 * reference (its direct_sum, fmm-ref/src/p2p.rs:147-186, is host code); the results are
 * bit-identical to fmmgpu_direct_sum's.
 *
 * For callers that cannot allocate: code that runs beside a built FMM whose plan and
 * stores fill the device (a cudaMalloc there fails or takes memory the evaluator needs),
 * and code on a stream that must not be stalled (cudaFree synchronises the whole device,
 * so the allocating entry point waits for every stream, the evaluator's included).
 *
 * Its scratch is one module-scope device array of FMMGPU_DIRECT_NOALLOC_SCRATCH_BYTES
 * (16 MiB) per device: ntargets x (128 if nsources > 65536, else 1) x 32 bytes must fit,
 * i.e. at most 4096 targets above 65536 sources and 524288 otherwise; larger calls
 * return FMMGPU_INVALID_ARGUMENT before any device work.  No part of the scratch has to
 * start at zero.  Queued on `stream` (a cudaStream_t; NULL = the default stream), not
 * synchronised; device errors surface at the caller's next synchronisation.
 *
 * Calls share that one scratch: two calls in flight at once on one device (different
 * streams, or threads without ordering) race on it and give wrong results.  Calls
 * queued one after another on one stream are safe.  The first call on each device does
 * one-time setup (the lookup of the scratch address, which may load the library's module
 * there): make that call before any stream capture begins.  The address is cached for the
 * life of the process, so do not reset a device (cudaDeviceReset) and then call again.
 * The calling thread's current device is restored before the call returns.  A CUDA
 * error left pending by earlier work on the thread is reported (FMMGPU_DEVICE_ERROR, not
 * cleared) and nothing is launched. */
#define FMMGPU_DIRECT_NOALLOC_SCRATCH_BYTES (16u << 20)
int fmmgpu_direct_sum_noalloc(size_t nsources, const double* sources, const double* charges, size_t ntargets,
                              const double* targets, double* potential, double* gradient, int device,
                              void* stream);

const char* fmmgpu_status_string(int status);
const char* fmmgpu_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* FMM_B200_H */
