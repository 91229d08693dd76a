/*
 * avbd_cuda.h -- C ABI of the B200 (sm_100a) AVBD step.
 *
 * The library replaces what runs under the reference's physics-backend seam:
 *   struct PhysicsBackend { virtual const char *name() const; virtual void step(Solver &); }
 *   (ts-jls/avbd-demo3d source/solver.h:410-417), installed as Solver::physicsBackend
 *   (solver.h:360) and called from Solver::step (solver.cpp:934-937).
 * One avbd_step() call performs what Solver::stepCpuReference does
 * (solver.cpp:1036-1041): broadphase, manifold creation and narrowphase, force
 * initialisation and warm start, body warm start, the primal/dual iterations and
 * the velocity update. Everything runs on the GPU; there is no CPU fallback.
 *
 * Conventions
 *  - Body index = position in the reference's Solver::bodies list (0 = list head =
 *    newest body). Forces carry a creation sequence number: a larger number is a
 *    newer force (the reference keeps per-body force lists newest first,
 *    force.cpp:25-36, and sums constraint rows in that order).
 *  - All functions return 0 on success or a negative AVBD_ERR_* code; the text of
 *    the last error is available from avbd_last_error(). Failures latch: after an
 *    error the context refuses to step until avbd_clear_error().
 *  - A context is single-threaded and bound to one device and one CUDA stream.
 *  - Floats are FP32 throughout, with the reference's operation order, so results
 *    are bit-identical to the reference CPU solver run in the same body order.
 */
#ifndef AVBD_CUDA_H
#define AVBD_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AVBD_OK 0
#define AVBD_ERR_ARGUMENT -1
#define AVBD_ERR_CUDA -2
#define AVBD_ERR_CAPACITY -3
#define AVBD_ERR_STATE -4
#define AVBD_ERR_LATCHED -5

#define AVBD_BROADPHASE_ALL_PAIRS 0
#define AVBD_BROADPHASE_GRID 1
#define AVBD_BROADPHASE_SAP 2
/* No counterpart in the reference: the uniform grid's pair set and creation order (mode
 * AVBD_BROADPHASE_GRID, solver.cpp:284-486) with the binned candidates found by a
 * sorted-Morton LBVH over each world's binned bodies instead of the grid's cell table. */
#define AVBD_BROADPHASE_LBVH 3

/* Body shapes (RigidShapeType, solver.h:47-53). */
#define AVBD_SHAPE_BOX 0
#define AVBD_SHAPE_SPHERE 1
#define AVBD_SHAPE_CAPSULE 2
#define AVBD_SHAPE_CYLINDER 3

/* How a step runs its solver iterations (avbd_set_iteration_mode). */
#define AVBD_ITERATIONS_PER_COLOUR 0 /* one launch per colour and iteration, then the dual sweep */
#define AVBD_ITERATIONS_PERSISTENT 1 /* all iterations in one cooperative launch (default) */

/* How a step is issued (avbd_set_step_mode). */
#define AVBD_STEP_DEVICE 0 /* counts stay on the device; no host wait inside a step (default) */
#define AVBD_STEP_HOST 1   /* the host reads the counts it needs at three points of each step */

#define AVBD_FORCE_MANIFOLD 0
#define AVBD_FORCE_JOINT 1
#define AVBD_FORCE_SPRING 2
#define AVBD_FORCE_IGNORE 3

typedef struct AvbdContext AvbdContext;

/* Solver parameters: Solver::dt, gravity, iterations, alpha, betaLin, betaAng, gamma,
 * broadphaseMode (solver.h:348-366). */
typedef struct AvbdParams
{
    float dt;
    float gravity;
    int32_t iterations;
    float alpha;
    float betaLin;
    float betaAng;
    float gamma;
    int32_t broadphase;
} AvbdParams;

/* Rigid state and properties (Rigid, solver.h:197-228), arrays of n entries in list order.
 * position3/velocity3/angular3/prev_velocity3/size3/moment3 hold 3 floats per body,
 * orientation4 holds x, y, z, w. */
typedef struct AvbdBodies
{
    int32_t count;
    const float *position3;
    const float *orientation4;
    const float *velocity3;
    const float *angular3;
    const float *prev_velocity3;
    const float *size3;
    const float *mass;
    const float *moment3;
    const float *friction;
    const float *radius;
    /* Shapes (RigidShape, solver.h:55-61; Rigid::makeSphere / makeCapsule / makeCylinder,
     * rigid.cpp:44-90), read when the world is loaded; NULL: every body is a box. shape:
     * AVBD_SHAPE_*; shape_radius: RigidShape::radius (a box's is length(size / 2));
     * half_length: capsule and cylinder half length (0 otherwise). size3 holds the shape's
     * bounding widths and radius the body's bounding radius, as on Rigid. */
    const int32_t *shape;
    const float *shape_radius;
    const float *half_length;
} AvbdBodies;

/* Body state written back after a step. Any pointer may be NULL to skip that field. */
typedef struct AvbdBodyState
{
    float *position3;
    float *orientation4;
    float *velocity3;
    float *angular3;
    float *prev_velocity3;
    float *initial_position3;
    float *initial_orientation4;
    float *inertial_position3;
    float *inertial_orientation4;
} AvbdBodyState;

/* Joints (Joint, solver.h:252-267). body_a may be -1 (anchored to world point rA).
 * state28 per joint: rA[3] rB[3] C0Lin[3] C0Ang[3] penaltyLin[3] penaltyAng[3]
 * lambdaLin[3] lambdaAng[3] stiffnessLin stiffnessAng fracture torqueArm. */
typedef struct AvbdJoints
{
    int32_t count;
    const int32_t *body_ab2;
    const int64_t *seq;
    const float *state28;
    const int32_t *broken;
} AvbdJoints;

/* Springs (Spring, solver.h:270-281). state8: rA[3] rB[3] rest stiffness. */
typedef struct AvbdSprings
{
    int32_t count;
    const int32_t *body_ab2;
    const int64_t *seq;
    const float *state8;
} AvbdSprings;

/* IgnoreCollision pairs (solver.h:284-291). */
typedef struct AvbdIgnores
{
    int32_t count;
    const int32_t *body_ab2;
    const int64_t *seq;
} AvbdIgnores;

/* Manifolds (Manifold, solver.h:294-334). Per manifold: bodies, sequence number, contact
 * count, basis (3 rows of 3), friction; per contact slot (8 per manifold): feature key,
 * contact15 = rA[3] rB[3] C0[3] penalty[3] lambda[3], stick flag. */
typedef struct AvbdManifolds
{
    int32_t count;
    const int32_t *body_ab2;
    const int64_t *seq;
    const int32_t *num_contacts;
    const float *basis9;
    const float *friction;
    const int32_t *keys8;
    const float *contact15x8;
    const int32_t *stick8;
} AvbdManifolds;

/* Writable views for readback (same layouts). */
typedef struct AvbdManifoldsOut
{
    int32_t *body_ab2;
    int64_t *seq;
    int32_t *num_contacts;
    float *basis9;
    float *friction;
    int32_t *keys8;
    float *contact15x8;
    int32_t *stick8;
} AvbdManifoldsOut;

typedef struct AvbdJointsOut
{
    int32_t *body_ab2;
    int64_t *seq;
    float *state28;
    int32_t *broken;
} AvbdJointsOut;

/* Per-step counters, in the spirit of SolverStats (solver.h:121-188). */
typedef struct AvbdStats
{
    int64_t body_count;
    int64_t pair_checks;
    int64_t sphere_hits;
    int64_t constrained_hits;
    int64_t manifolds_created;
    int64_t manifold_count;
    int64_t contact_count;
    int64_t joint_count;
    int64_t spring_count;
    int64_t solved_bodies;
    int64_t colours;
    int64_t colour_rounds;
    int64_t primal_rows;
    int64_t grid_rescaled; /* 1 if the grid hit the reference's 2^22-cell cap this step */
    int64_t device_steps;  /* steps issued without a host wait (since the world was loaded) */
    int64_t redone_steps;  /* of those, steps the host redid synchronously (see avbd_step) */
    float step_ms;
} AvbdStats;

/* Context lifetime. Replaces constructing a backend for Solver::physicsBackend
 * (makeCpuReferencePhysicsBackend, solver.cpp:676-680). stream may be NULL (the
 * context creates its own). The context also creates four non-blocking side streams on the
 * device, onto which a step forks independent parts of its work (the pair set, large bodies,
 * the LBVH tree, the initialisation of existing manifolds) and which it joins back with
 * events: every call's work is still ordered on `stream` as a whole. */
int avbd_create(AvbdContext **out, int32_t device_ordinal, void *cuda_stream);
void avbd_destroy(AvbdContext *ctx);
const char *avbd_last_error(const AvbdContext *ctx);
void avbd_clear_error(AvbdContext *ctx);
/* PhysicsBackend::name() (solver.h:413). */
const char *avbd_backend_name(void);

/* Solver parameters (Solver::dt .. broadphaseMode, solver.h:348-366). */
int avbd_set_params(AvbdContext *ctx, const AvbdParams *params);

/* Full world upload: replaces the device world (scene load, topology edits between
 * steps such as the drag joint of simulation_host.cpp:242-274). next_seq is the
 * sequence number the next created manifold receives (greater than every seq given). */
int avbd_load_world(AvbdContext *ctx, const AvbdBodies *bodies, const AvbdJoints *joints,
                    const AvbdSprings *springs, const AvbdIgnores *ignores, const AvbdManifolds *manifolds,
                    int64_t next_seq);

/* Batched worlds: num_worlds independent worlds in one context, stepped together by one
 * launch sequence per step (no counterpart in the reference, where each Solver is one
 * world). Bodies are given world by world: world w owns bodies [world_start[w],
 * world_start[w + 1]) in that world's list order; forces use these global indices and never
 * join two worlds; sequence numbers must increase with creation time within each world.
 * Every world keeps its own broadphase grid, so each evolves exactly as it would alone.
 * avbd_load_world is this call with one world. */
int avbd_load_batch(AvbdContext *ctx, int32_t num_worlds, const int32_t *world_start, const AvbdBodies *bodies,
                    const AvbdJoints *joints, const AvbdSprings *springs, const AvbdIgnores *ignores,
                    const AvbdManifolds *manifolds, int64_t next_seq);

/* Overwrite body state only (positions/orientations/velocities edited between steps,
 * e.g. scenes.h:45). Same layout and order as avbd_load_world's bodies. Arrays in
 * page-locked host memory that the device can address (cudaHostAlloc, cudaHostRegister, a
 * pinned torch tensor) are read in place by a kernel on the context stream, asynchronously:
 * keep them unchanged until the next call that waits for the device (a read,
 * avbd_synchronize); other arrays are copied before the call returns. avbd_read_bodies
 * likewise has its kernel write page-locked arrays in place before it returns. */
int avbd_write_bodies(AvbdContext *ctx, const AvbdBodies *bodies);

/* Solver::step() for nsteps steps (solver.cpp:934-937 via stepCpuReference 1036-1041).
 * Asynchronous on the context stream. In AVBD_STEP_DEVICE mode (the default, for the grid
 * broadphase with the single-launch iterations) a step keeps every count it needs on the
 * device and returns as soon as its launches are issued. A step that cannot run as issued
 * stops on the device before it changes anything, and so does every step issued after
 * it: new pairs that do not fit the manifold buffers, a grid that needs the reference's
 * cell-count cap (rescaled with the host's cbrtf), a joint broken in an earlier step (its
 * removal is compacted on the host). The next call that waits for the device (a read,
 * avbd_synchronize, avbd_get_stats, an edit) redoes those steps synchronously, so results
 * are always the same bits. In AVBD_STEP_HOST mode every step reads its counts on the host.
 * Errors of a step surface at the next call that waits for the device and latch:
 * AVBD_ERR_STATE when a bounded wait expires (a grid barrier, a row waiting for its
 * partner body's iteration count, the colouring's barrier) and when a body's position,
 * orientation or velocity is not finite at the start of a step (the step refuses it and
 * leaves the world as it was). */
int avbd_step(AvbdContext *ctx, int32_t nsteps);
/* Wait for the context stream (and redo or report any device-resident step, as above). */
int avbd_synchronize(AvbdContext *ctx);

/* Contacts injected for one step (ExternalManifoldContact, solver.h:336-344): per entry the
 * bodies (list indices a, b), up to 8 contacts and the contact basis (rows: normal pointing
 * from B to A, two tangents), in the layout avbd_read_manifolds writes: keys8 feature keys,
 * contact15x8 per contact rA(3) rB(3) C0(3, recomputed) penalty(3) lambda(3), stick8. */
typedef struct AvbdExternalContacts
{
    int32_t count;
    const int32_t *body_ab2;
    const int32_t *num_contacts;
    const float *basis9;
    const int32_t *keys8;
    const float *contact15x8;
    const int32_t *stick8;
    const int32_t *creates; /* per entry: nonzero = may make its pair's manifold (NULL: all) */
} AvbdExternalContacts;

/* One Solver::step with the broadphase replaced by the caller's pairs and, optionally, the
 * narrowphase replaced by the caller's contacts: Solver::stepCpuReferenceWithExternalBroadphase
 * (pairs[, contacts]) (solver.cpp:939-957, solver.h:403-404), whose pair handling is
 * broadphaseExternalPairs (solver.cpp:579-626) and whose contact lookup is
 * Manifold::initialize's (manifold.cpp:110-117). Bodies are list indices; the reference's
 * dense BodyIds map to them through the caller's body list.
 *  - pairs_ab2[2k], [2k+1]: pair k. Pairs naming no body, one body twice or bodies of two
 *    worlds are skipped. The others, in order: a bounding-sphere test, then a new manifold
 *    (bodies in the given order) unless a force already links the two bodies, counting an
 *    earlier pair of this call.
 *  - contacts (NULL: none): after the pairs, every valid entry with creates[e] != 0 in order
 *    makes its pair's manifold the same way, without the sphere test. The reference makes
 *    one only for entries whose dense ids increase (bodyA < bodyB): the caller sets creates
 *    from that. During this step every manifold whose bodies match an entry, as (a, b) or
 *    else as (b, a), takes that entry's basis and contacts instead of the narrowphase (the
 *    later of two entries with the same (a, b) wins); its penalty, multipliers and stick
 *    flags seed contacts that do not persist from the previous step.
 * Synchronous (returns when the step is done); counters land in avbd_get_stats. */
int avbd_step_external(AvbdContext *ctx, int32_t num_pairs, const int32_t *pairs_ab2,
                       const AvbdExternalContacts *contacts);

/* AVBD_STEP_DEVICE (default) or AVBD_STEP_HOST, for later steps; both give the same bits.
 * No counterpart in the reference (its CPU step has no device). */
int avbd_set_step_mode(AvbdContext *ctx, int32_t mode);
/* Manifold room kept beyond the live count for device-resident steps: spare = 0 restores
 * the default (twice the live count, and at least twice the body count more: bodies whose
 * bounding spheres overlap without touching get a manifold that lasts one step); a small spare
 * makes steps that create many pairs stop on the device and be redone on the host. */
int avbd_set_manifold_headroom(AvbdContext *ctx, int64_t spare);
/* Poll limits of the bounded waits: the colouring's grid barrier and the iteration
 * kernel's grid barriers and partner waits (0 = the defaults, 2^24 and 2^22 polls). A wait
 * that reaches its limit makes the step fail with AVBD_ERR_STATE, as described at
 * avbd_step; the context stays usable after avbd_clear_error and a reload. No counterpart
 * in the reference (its CPU solver never waits). */
int avbd_set_wait_limits(AvbdContext *ctx, uint32_t colouring_polls, uint32_t iteration_polls);

/* Solver::benchmarkBroadphaseOnly (solver.cpp:989-1034), the reference's collision-only
 * benchmark step (headless_server.cpp:664-690): every manifold is deleted and the selected
 * broadphase alone runs, leaving a contact-less manifold for every non-constrained hit pair.
 * Bodies do not move. Counters land in avbd_get_stats. */
int avbd_broadphase_only(AvbdContext *ctx);

/* Post-step readback (the contract of readbackAndApply, avbd_gpu_solver.cpp:1970-2022).
 * Waits for the pending steps; the packing is queued behind them first, so one wait serves
 * both. On an error return (a pending step failed) the output arrays may have been written
 * and hold no defined state. */
int avbd_read_bodies(AvbdContext *ctx, const AvbdBodyState *out);
int avbd_num_manifolds(AvbdContext *ctx, int32_t *count);
int avbd_read_manifolds(AvbdContext *ctx, const AvbdManifoldsOut *out);
int avbd_num_joints(AvbdContext *ctx, int32_t *count);
int avbd_read_joints(AvbdContext *ctx, const AvbdJointsOut *out);
int avbd_next_seq(AvbdContext *ctx, int64_t *next_seq);

/* Joint edits between steps, as SimulationHost makes them for a mouse drag
 * (beginDrag / updateDrag / releaseDrag, simulation_host.cpp:242-274; Joint constructor
 * joint.cpp:25-33, Force constructor / destructor force.cpp:14-39 / 42-). None of them
 * reloads the world.
 *
 * avbd_add_joints appends joints as the newest forces: their sequence numbers must be
 * strictly increasing and at or above avbd_next_seq (which then moves past the last);
 * body_a may be -1 (anchored to the world point rA) and both bodies lie in one world.
 * avbd_remove_joints deletes the joints with the given sequence numbers (every number
 * must name a joint; nothing changes otherwise).
 * avbd_write_joints overwrites state28 and broken of existing joints, matched by sequence
 * number; body_ab2 must equal the joint's bodies (it is a check, not an edit).
 * Each call drops the recorded forward of the differentiable step. */
/* Viewer-bridge snapshots of every body, written from the device state
 * (makeSnapshotBinary / makeSnapshotJson, viewer_bridge.cpp:748-842; the viewer's decoder
 * is decodeBinarySnapshot, viewer/src/main.js:986-1050).
 * Binary ("AVBS"): u32 magic 0x53425641, u32 version 1, u64 frame, u32 scene bytes, u32
 * body count, the scene name, then per body in ascending id order 64 bytes: u32 id, shape
 * (AVBD_SHAPE_*), material (materialIdForBody: 0 static, 1 box, 3 sphere, 4 cylinder,
 * 5 capsule), dynamic; f32 position[3], rotation[4] (x y z w), size[3] (full widths), shape
 * radius, half length. JSON: the same fields as text,
 * numbers with 5 decimals.
 * body_id: the SimWorld dense id of each body (list order), or NULL for the creation rank
 * (the dense id of a world built without deletions). *size receives the bytes needed
 * (the JSON text with its terminating zero); out = NULL only queries it. */
int avbd_snapshot_binary(AvbdContext *ctx, uint64_t frame, const char *scene_name, const int32_t *body_id,
                         uint8_t *out, int64_t capacity, int64_t *size);
int avbd_snapshot_json(AvbdContext *ctx, uint64_t frame, const char *scene_name, const int32_t *body_id, char *out,
                       int64_t capacity, int64_t *size);

/* Iteration mode: AVBD_ITERATIONS_PERSISTENT (default) runs every iteration of a step in
 * one cooperative launch with grid-wide barriers between colours and each contact's dual
 * update fused into the next iteration's primal row of the body that owns it;
 * AVBD_ITERATIONS_PER_COLOUR launches each colour and the dual sweep separately. Both give
 * the same bits. avbd_iteration_mode reports the mode the next step runs in (the
 * per-colour form where the device cannot hold the persistent launch, and while the
 * differentiable step records). */
int avbd_set_iteration_mode(AvbdContext *ctx, int32_t mode);
int avbd_iteration_mode(AvbdContext *ctx, int32_t *mode);

int avbd_add_joints(AvbdContext *ctx, const AvbdJoints *joints);
int avbd_remove_joints(AvbdContext *ctx, int32_t count, const int64_t *seq);
int avbd_write_joints(AvbdContext *ctx, const AvbdJoints *joints);

/* Parity dumps: colour per body of the last step (-1 = not solved) and colour count;
 * the primal sweep order (bodies grouped by colour). */
int avbd_read_colours(AvbdContext *ctx, int32_t *colour, int32_t *num_colours);
int avbd_read_solve_order(AvbdContext *ctx, int32_t *order, int32_t *count);
int avbd_get_stats(AvbdContext *ctx, AvbdStats *stats);

/* Device pointers of the resident body pose arrays (float4 xyz_ / xyzw per body) for
 * callers that keep data on the GPU. */
int avbd_device_pose(AvbdContext *ctx, void **position4, void **orientation4);

/* Per-phase GPU time, the counterpart of SolverStats' phase timers (broadphaseMs,
 * forceInitMs, bodyInitMs, primalSolveMs, dualUpdateMs, velocityUpdateMs; solver.h:121-188),
 * measured with CUDA events on the context stream. Profiling adds one stream sync per step. */
#define AVBD_PHASE_BROADPHASE 0
#define AVBD_PHASE_FORCE_INIT 1
#define AVBD_PHASE_ADJACENCY 2
#define AVBD_PHASE_BODY_INIT 3
#define AVBD_PHASE_COLOURING 4
#define AVBD_PHASE_PRIMAL 5
#define AVBD_PHASE_DUAL 6
#define AVBD_PHASE_VELOCITY 7
#define AVBD_PHASE_COUNT 8

typedef struct AvbdProfile
{
    int64_t steps;                         /* steps profiled since the last reset */
    double phase_ms[AVBD_PHASE_COUNT];     /* summed GPU time per phase */
    int64_t phase_spans[AVBD_PHASE_COUNT]; /* timed spans per phase (primal: one per launch) */
    int64_t launches;                      /* kernel launch calls issued (a library sort/scan call counts once) */
} AvbdProfile;

int avbd_set_profiling(AvbdContext *ctx, int32_t enable);

/* Colouring of the primal sweep (no counterpart in the reference, whose CPU sweep is
 * sequential in list order; the precedent is the WebGPU lane's greedy colouring in list
 * order, avbd_gpu_solver.cpp:1817-1866). GREEDY (default) gives exactly that greedy
 * colouring, computed in parallel as Jones-Plassmann with list-index priority; HASHED uses
 * hashed priorities, which needs fewer rounds but sweeps in an order further from the
 * reference's list order. */
#define AVBD_COLOUR_GREEDY 0
#define AVBD_COLOUR_HASHED 1
int avbd_set_colouring(AvbdContext *ctx, int32_t mode);

/* Constraint-graph colouring that allocates nothing. It has no counterpart in the
 * reference (the reference's CPU solver sweeps bodies one by one and never colours them).
 *
 * For callers that cannot call cudaMalloc: code that runs inside another framework's
 * memory pool or allocator, real-time loops that must not allocate after start-up, and
 * hosts that have already reserved the whole GPU. It computes the same colouring as the
 * primal sweep of avbd_step (Jones-Plassmann; mode AVBD_COLOUR_GREEDY or
 * AVBD_COLOUR_HASHED) for a graph the caller passes as a neighbour list, using only a
 * fixed scratch array compiled into the library: about 4 MiB that every GPU loading the
 * library keeps until the process exits.
 *
 * Inputs and outputs are device pointers except num_colours (host): n bodies (at most
 * AVBD_NOALLOC_MAX_BODIES), vertex[n] (non-zero = a body to colour), adj_start[n + 1] and
 * adj_other[adj_start[n]] (neighbours of body b are adj_other[adj_start[b] ..
 * adj_start[b + 1]); entries outside [0, n) are skipped), colour[n] receives the colour of
 * each vertex and -1 elsewhere. Runs on cuda_stream (NULL = default stream) and waits for
 * it before returning.
 *
 * The first call on a device sets that device up: it looks up the scratch array's device
 * address and the co-resident block count. Under CUDA 12's default lazy module loading
 * that first call is also when the driver loads this part of the library onto the device
 * and places the scratch array there, so it needs about 4 MiB free on the GPU and can
 * fail with AVBD_ERR_CUDA when the GPU is already full. Make the first call at start-up,
 * before the GPU is filled and before any stream capture begins (or set
 * CUDA_MODULE_LOADING=EAGER, which places the array when the library's context is
 * created); after it, calls allocate nothing. All calls share the one scratch array,
 * which keeps the last call's contents: calls that overlap on the GPU (other streams,
 * other threads) race and must be serialised by the caller.
 * Returns AVBD_OK, AVBD_ERR_ARGUMENT (bad arguments), AVBD_ERR_CAPACITY (n above the
 * maximum, or more than 256 colours), AVBD_ERR_STATE (colouring did not finish) or
 * AVBD_ERR_CUDA. */
#define AVBD_NOALLOC_MAX_BODIES (1 << 20)
int avbd_colour_graph_noalloc(int32_t n, const int32_t *vertex, const int32_t *adj_start, const int32_t *adj_other,
                              int32_t mode, int32_t *colour, int32_t *num_colours, void *cuda_stream);

/* Autotuner for the primal sweep (no counterpart in the reference, whose primal loop is a
 * serial CPU loop, solver.cpp:1177-1242). Variants differ in lanes per body and register
 * budget; every variant gives bit-identical results. avbd_autotune times each variant on
 * the current colouring (bodies' poses are restored after every trial) and selects the
 * fastest; variant_us receives one time per variant (may be NULL). */
int avbd_num_primal_variants(int32_t *count, int32_t *group, int32_t *min_blocks);
int avbd_set_primal_variant(AvbdContext *ctx, int32_t variant);
int avbd_autotune(AvbdContext *ctx, int32_t repeats, int32_t *best_variant, float *variant_us);
int avbd_read_profile(AvbdContext *ctx, AvbdProfile *out);
int avbd_reset_profile(AvbdContext *ctx);

/* Differentiable step: a forward / backward pair over several steps. The reference has no
 * differentiation; the map that is differentiated is its step (solver.cpp:1036-1298) with
 * the integer decisions of the run held fixed (contact set and contact geometry, colouring,
 * force clamps, friction-cone and penalty-ramp branches, warm-start clamps), which leaves
 * a smooth function of the initial body state, the masses and the friction coefficients.
 * The FP32 forward is the ordinary step; derivatives are evaluated and accumulated in
 * double precision.
 *
 * avbd_adjoint_forward runs nsteps steps exactly like avbd_step(ctx, nsteps) and keeps a
 * snapshot of the dynamic state every checkpoint_every steps. Worlds with joints or springs
 * are rejected (AVBD_ERR_ARGUMENT): the differentiable step covers contacts.
 *
 * Along the way it tapes every step's decisions and replays the frozen-branch map in double
 * precision, keeping a snapshot of that replay every checkpoint_every steps; the FP32 world
 * ends exactly where avbd_step(ctx, nsteps) would leave it.
 *
 * avbd_adjoint_backward takes the gradient of a loss with respect to the final state
 * (host arrays in list order: position n x 3, orientation n x 4 (x, y, z, w), velocity
 * n x 3, angular velocity n x 3; NULL = zero) and writes into the non-NULL host arrays of
 * AvbdAdjointGrad the gradient with respect to the state before the forward steps and the
 * parameters. Per checkpoint segment it replays the segment again, keeping the state at
 * every iteration, and sweeps it in reverse. It leaves the FP32 world untouched. The
 * forward must be the last thing that changed the world (a step, a body write or a load
 * in between is refused), and parameters and colouring mode must be the same.
 *
 * Friction parameters are per body pair: mu of every manifold between bodies a and b
 * (manifold.cpp:103, sqrt(mu_a mu_b) in the forward). Pairs are the (min, max) body pairs of
 * every manifold the forward met, in ascending order; avbd_adjoint_read_pairs lists them
 * and their nominal coefficients. body_friction chains the pair gradients through
 * mu = sqrt(mu_a mu_b) onto Rigid::friction. */
typedef struct AvbdAdjointGrad
{
    double *position;         /* n x 3 */
    double *orientation;      /* n x 4 */
    double *velocity;         /* n x 3 */
    double *angular_velocity; /* n x 3 */
    double *prev_velocity;    /* n x 3: Rigid::prevVelocityLin (the adaptive warm start reads it) */
    double *mass;             /* n: the moment scales with the mass (rigid.cpp:34-39) */
    double *pair_friction;    /* num_pairs */
    double *body_friction;    /* n */
} AvbdAdjointGrad;

int avbd_adjoint_forward(AvbdContext *ctx, int32_t nsteps, int32_t checkpoint_every);
int avbd_adjoint_num_pairs(AvbdContext *ctx, int32_t *count);
int avbd_adjoint_read_pairs(AvbdContext *ctx, int32_t *lohi2, float *friction);
int avbd_adjoint_backward(AvbdContext *ctx, const double *d_position3, const double *d_orientation4,
                          const double *d_velocity3, const double *d_angular_velocity3, const AvbdAdjointGrad *out);

/* Final state of the double-precision frozen-branch replay of the last forward (list
 * order; NULL outputs skipped): the state whose derivatives avbd_adjoint_backward takes.
 * It differs from the FP32 world only by rounding; evaluate a loss's gradient here for the
 * exact gradient of the differentiated map. */
int avbd_adjoint_replay_state(AvbdContext *ctx, double *position3, double *orientation4, double *velocity3,
                              double *angular_velocity3);

/* Parity dump of the forward's tape for one step: the manifold count, the branch outcomes
 * of every contact slot per iteration (iterations x num_manifolds x 8; bits 0-11 the dual
 * update, 12-13 the primal evaluation for body A, 14-15 for body B: 1 = normal force
 * clamped, 2 = friction cone; dual bits 4 tangential ramp, 8/16/32 penalty cap, 64/128/256
 * C < 0, 512/1024/2048 C > 0), the warm-start outcome per body (1 dynamic, 2 has forces,
 * 4 adaptive weight inside (0, 1), 8 weight clamped at 1) and the link of every contact to
 * the previous step's slot (manifold * 8 + contact, -1 = new). NULL outputs are skipped. */
int avbd_adjoint_tape_step(AvbdContext *ctx, int32_t step, int32_t *num_manifolds, uint16_t *flags,
                           uint8_t *body_flags, int32_t *link);

#ifdef __cplusplus
}
#endif

#endif
