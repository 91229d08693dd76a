/*
 * CPU oracle for the AVBD step (test infrastructure only).
 *
 * This is a plain-C restatement of the reference solver's per-step algorithm
 * (ts-jls/avbd-demo3d, source/solver.cpp, manifold.cpp, collide.cpp,
 * joint.cpp, spring.cpp, maths.h). It exists to check the CUDA path: only the
 * tests, the smoke check and the CPU-baseline leg of the benchmark load it.
 * It is pinned bit-for-bit against the reference compiled from its own
 * sources (oracle/Makefile, target `_ref`) and against the committed golden
 * fixtures in tests/golden/.
 *
 * Body indices in every query are LIST indices: index 0 is the head of the
 * reference's `Solver::bodies` list, i.e. the most recently created body
 * (Rigid constructor prepends, rigid.cpp:29-31). Scene descriptions passed to
 * oracle_create use CREATION indices (0 = first body created).
 */
#ifndef AVBD_ORACLE_H
#define AVBD_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleParams
{
    float dt;
    float gravity;
    int iterations;
    float alpha;
    float betaLin;
    float betaAng;
    float gamma;
    int broadphase; /* 0 = all pairs, 1 = uniform grid (reference default), 2 = sweep and prune */
    int orderMode;  /* 0 = primal sweep in list order; colour order with 1 = list-index (greedy)
                       priority, 2 = hashed priority */
} OracleParams;

enum
{
    ORACLE_FORCE_JOINT = 1,
    ORACLE_FORCE_SPRING = 2,
    ORACLE_FORCE_IGNORE = 3,
    ORACLE_FORCE_MANIFOLD = 4
};

typedef struct OracleWorld OracleWorld;

/* Scene in creation order. Body i is constructed like
 * `new Rigid(solver, size, density, friction, pos, vel)` (rigid.cpp:24-42) and
 * then given orientation quat4[i] (xyzw), as scenes.h:45 does. Forces follow in
 * the listed order: joints take fparam3 = {stiffnessLin, stiffnessAng, fracture},
 * springs {stiffness, rest, unused}; fa == -1 anchors a joint to the world. */
OracleWorld *oracle_create(const OracleParams *params, int nBodies, const float *size3, const float *density,
                           const float *friction, const float *pos3, const float *vel3, const float *quat4,
                           int nForces, const int *ftype, const int *fa, const int *fb, const float *frA3,
                           const float *frB3, const float *fparam3);
/* Body shapes (RigidShapeType, solver.h:47-53). */
enum
{
    ORACLE_SHAPE_BOX = 0,
    ORACLE_SHAPE_SPHERE = 1,
    ORACLE_SHAPE_CAPSULE = 2,
    ORACLE_SHAPE_CYLINDER = 3
};

/* As oracle_create, with a shape per body (creation order): boxes take size3; spheres,
 * capsules and cylinders are built like Rigid::makeSphere / makeCapsule / makeCylinder
 * (rigid.cpp:44-90) from dim2 = (radius, halfLength). shape NULL: all boxes. */
OracleWorld *oracle_create_shapes(const OracleParams *params, int nBodies, const int *shape, const float *dim2,
                                  const float *size3, const float *density, const float *friction,
                                  const float *pos3, const float *vel3, const float *quat4, int nForces,
                                  const int *ftype, const int *fa, const int *fb, const float *frA3,
                                  const float *frB3, const float *fparam3);
void oracle_destroy(OracleWorld *w);
void oracle_set_params(OracleWorld *w, const OracleParams *params);

/* Solver::benchmarkBroadphaseOnly (solver.cpp:989-1034): every manifold is deleted and the
 * broadphase alone runs, creating contact-less manifolds for the hit pairs. */
int oracle_broadphase_only(OracleWorld *w);

/* Joint edits between steps, as SimulationHost's drag makes them (simulation_host.cpp:242-274):
 * a new Joint (the newest force; a = -1 anchors it to the world point rA) returns its
 * sequence number; the anchor rA moves; the joint is deleted. Bodies in list order. */
int64_t oracle_add_joint(OracleWorld *w, int a, int b, const float *rA3, const float *rB3, float stiffLin,
                         float stiffAng, float fracture);
int oracle_set_joint_anchor(OracleWorld *w, int64_t seq, const float *rA3);
int oracle_remove_joint(OracleWorld *w, int64_t seq);

/* One full step = prepare + iterate + finish (solver.cpp:1036-1041). */
int oracle_step(OracleWorld *w, int nsteps);
int oracle_prepare(OracleWorld *w);
int oracle_iterate(OracleWorld *w);
int oracle_finish(OracleWorld *w);

int oracle_num_bodies(const OracleWorld *w);
void oracle_get_bodies(const OracleWorld *w, float *pos3, float *quat4, float *vel3, float *angvel3,
                       float *prevvel3);
void oracle_get_body_aux(const OracleWorld *w, float *initLin3, float *initAng4, float *inertLin3,
                         float *inertAng4);
void oracle_get_body_props(const OracleWorld *w, float *mass, float *moment3, float *radius, float *size3,
                           float *friction);
/* Overwrite body state between steps (list order). */
void oracle_set_bodies(OracleWorld *w, const float *pos3, const float *quat4, const float *vel3,
                       const float *angvel3, const float *prevvel3);

int oracle_num_manifolds(const OracleWorld *w);
/* Manifolds in creation order. contact15 holds per contact rA, rB, C0, penalty, lambda. */
void oracle_get_manifolds(const OracleWorld *w, int *ab2, int64_t *seq, int *ncontacts, float *basis9,
                          float *friction, int *keys8, float *contact15x8, int *stick8);

int oracle_num_joints(const OracleWorld *w);
/* Per joint: C0Lin, C0Ang, penaltyLin, penaltyAng, lambdaLin, lambdaAng (18 floats), broken flag. */
void oracle_get_joints(const OracleWorld *w, int *ab2, float *state18, int *broken);

/* Colouring of the last prepared step: colour per body (-1 = not solved), colour count. */
void oracle_get_colours(const OracleWorld *w, int *colour, int *nColours);
/* Bodies visited by the primal sweep of the last prepared step, in sweep order. */
int oracle_get_solve_order(const OracleWorld *w, int *order);

/* Counters of the last step: [0] pair checks, [1] sphere hits, [2] constrained hits,
 * [3] manifolds created, [4] manifolds alive, [5] contacts alive, [6] primal force visits,
 * [7] solved bodies per iteration, [8] colours. */
void oracle_get_counters(const OracleWorld *w, int64_t *out9);

/* Stand-alone box-box narrowphase (collide.cpp:898-955) for fixtures:
 * writes up to 8 contacts (key, rA, rB) and the basis, returns the count. */
int oracle_collide_boxes(const float *posA3, const float *quatA4, const float *sizeA3, const float *posB3,
                         const float *quatB4, const float *sizeB3, int *keys8, float *rA3x8, float *rB3x8,
                         float *basis9);

/* Colour priority used by the Jones-Plassmann colouring (shared contract with the CUDA path). */
uint32_t oracle_colour_priority(uint32_t bodyIndex);

void oracle_get_params(const OracleWorld *w, OracleParams *out);

/* ------------------------------------------------------------------------- */
/* Frozen-branch tape, for the checks of the differentiable step.            */
/* ------------------------------------------------------------------------- */

/* Branch outcomes recorded per contact evaluation (primal as body A, primal as body B,
 * dual), per carried-over contact and per body. The values equal the EvalFlags,
 * InitFlags and BodyFlags of avbd_demo3d_b200/csrc/avbd_diff.h. */
enum
{
    ORACLE_EF_NCLAMP = 1,   /* F.n >= 0 -> 0 (manifold.cpp:201) */
    ORACLE_EF_CONE = 2,     /* friction cone scaling (manifold.cpp:206-210) */
    ORACLE_EF_RAMP_T = 4,   /* dual: tangential ramp (manifold.cpp:271) */
    ORACLE_EF_CAP_X = 8,    /* dual: ramp reached PENALTY_MAX */
    ORACLE_EF_CAP_Y = 16,
    ORACLE_EF_CAP_Z = 32,
    ORACLE_EF_NEG_X = 64,   /* dual: C < 0 */
    ORACLE_EF_NEG_Y = 128,
    ORACLE_EF_NEG_Z = 256,
    ORACLE_EF_POS_X = 512,  /* dual: C > 0 */
    ORACLE_EF_POS_Y = 1024,
    ORACLE_EF_POS_Z = 2048,
    ORACLE_IF_LO_X = 1,     /* carried penalty * gamma < PENALTY_MIN (manifold.cpp:170) */
    ORACLE_IF_LO_Y = 2,
    ORACLE_IF_LO_Z = 4,
    ORACLE_IF_HI_X = 8,     /* carried penalty * gamma > PENALTY_MAX */
    ORACLE_IF_HI_Y = 16,
    ORACLE_IF_HI_Z = 32,
    ORACLE_BF_DYNAMIC = 1,  /* mass > 0 */
    ORACLE_BF_FORCES = 2,   /* non-empty force list */
    ORACLE_BF_ACCEL_IN = 4, /* adaptive warm-start weight inside (0, 1) (solver.cpp:1146-1150) */
    ORACLE_BF_ACCEL_ONE = 8 /* adaptive weight clamped at 1 */
};

/* One recorded step. Manifolds are the list after Manifold::initialize and removal, in
 * creation order; contact slot = manifold * 8 + contact. */
typedef struct OracleTapeStep
{
    int nMan, nSolve, nColours, iterations;
    float *bodyIn;            /* n x 16: pos3 quat4 vel3 angvel3 prevVel3 at step start */
    unsigned char *bodyFlags; /* n */
    int *ab;                  /* nMan x 2 */
    float *basis;             /* nMan x 9: rows normal, tangent 1, tangent 2 */
    float *friction;          /* nMan */
    int *ncontacts;           /* nMan */
    int *keys;                /* nMan x 8 */
    float *geo;               /* nMan x 8 x 6: rA, rB */
    float *init;              /* nMan x 8 x 9: C0, lambda, penalty after initialization */
    int *src;                 /* nMan x 8: slot in the previous step's list, -1 = new contact */
    unsigned char *initFlags; /* nMan x 8 */
    int *solveOrder;          /* nSolve, the primal sweep order */
    int *colourStart;         /* nColours + 1 */
    unsigned short *flags;    /* iterations x nMan x 8 x 3 */
} OracleTapeStep;

/* Start recording every following step (clears an earlier tape). Worlds with joints or
 * springs are not recorded: the differentiable step covers contacts. Returns 0, or -1. */
int oracle_tape_begin(OracleWorld *w);
void oracle_tape_end(OracleWorld *w);
int oracle_tape_steps(const OracleWorld *w);
const OracleTapeStep *oracle_tape_step(const OracleWorld *w, int s);

#ifdef __cplusplus
}
#endif

#endif
