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
void oracle_destroy(OracleWorld *w);
void oracle_set_params(OracleWorld *w, const OracleParams *params);

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

#ifdef __cplusplus
}
#endif

#endif
