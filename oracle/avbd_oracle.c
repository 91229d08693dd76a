/*
 * CPU oracle for the AVBD step -- TEST INFRASTRUCTURE, not part of the product.
 *
 * A plain-C restatement of the reference solver's step (ts-jls/avbd-demo3d):
 *   broadphase      source/solver.cpp:166-185 (all pairs), 284-486 (uniform grid), 488-577 (SAP)
 *   pair handling   source/solver.cpp:131-248, source/rigid.cpp:105-116
 *   narrowphase     source/collide.cpp:60-433, 898-955 (box-box only)
 *   manifold        source/manifold.cpp:100-280
 *   joint / spring  source/joint.cpp:14-182, source/spring.cpp:14-74
 *   warm start      source/solver.cpp:1134-1169
 *   primal / dual   source/solver.cpp:1172-1273
 *   finish          source/solver.cpp:1275-1298
 *   math            source/maths.h (operators, rotate, orthonormal, 6x6 LDL solve :481-547)
 *
 * Every floating-point expression keeps the reference's operation order, because
 * the step is chaotic: one ulp in a contact row changes the trajectory within a few
 * steps. Build with gcc -O2 and no FMA contraction (-ffp-contract=off), like the
 * reference (default x86-64, no -march). The oracle is pinned bit-for-bit against
 * the reference compiled from its own sources (oracle/Makefile `_ref`).
 *
 * Force order: the reference keeps per-body intrusive lists with the newest force
 * first (force.cpp:25-36). Here every force carries a creation sequence number and
 * per-body lists are rebuilt sorted by descending sequence, which is the same order.
 *
 * Colour order (orderMode 1 or 2): the primal sweep visits bodies grouped by a
 * Jones-Plassmann colouring of the dynamic-body constraint graph (mode 1: priority by
 * list index, equal to greedy colouring in list order; mode 2: hashed priority). Within
 * one colour no two bodies share a constraint, so this equals the reference run with its
 * body list relinked into colour order between prepareStep and iteratePrimalDualCpu.
 */
#include "avbd_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* Math (source/maths.h), same operation order                               */
/* ------------------------------------------------------------------------- */

typedef struct
{
    float x, y, z;
} V3;
typedef struct
{
    float x, y, z, w;
} Q4;
typedef struct
{
    V3 r[3];
} M3;

#define VE(v, i) (((float *)&(v))[i])
#define VEC(v, i) (((const float *)&(v))[i])

static inline V3 v3(float x, float y, float z)
{
    V3 v;
    v.x = x;
    v.y = y;
    v.z = z;
    return v;
}
static inline V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 vneg(V3 a) { return v3(-a.x, -a.y, -a.z); }
static inline V3 vmul(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 vdiv(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
static inline float vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline float vlensq(V3 a) { return vdot(a, a); }
static inline float vlen(V3 a) { return sqrtf(vlensq(a)); }
static inline V3 vcross(V3 a, V3 b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline V3 vabs(V3 a) { return v3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }

/* maths.h min/max/clamp keep their exact comparison semantics */
static inline float rmin(float a, float b) { return a < b ? a : b; }
static inline float rmax(float a, float b) { return a > b ? a : b; }
static inline float rclamp(float x, float a, float b) { return rmax(a, rmin(b, x)); }
static inline float rsign(float x) { return x < 0 ? -1.0f : x > 0 ? 1.0f : 0.0f; }
static inline V3 vminf(V3 a, float b) { return v3(rmin(a.x, b), rmin(a.y, b), rmin(a.z, b)); }
static inline V3 vclampf(V3 v, float a, float b) { return v3(rclamp(v.x, a, b), rclamp(v.y, a, b), rclamp(v.z, a, b)); }

static inline M3 m3rows(V3 a, V3 b, V3 c)
{
    M3 m;
    m.r[0] = a;
    m.r[1] = b;
    m.r[2] = c;
    return m;
}
static inline M3 mdiag(float a, float b, float c) { return m3rows(v3(a, 0, 0), v3(0, b, 0), v3(0, 0, c)); }
static inline V3 mcol(M3 m, int i) { return v3(VE(m.r[0], i), VE(m.r[1], i), VE(m.r[2], i)); }
static inline V3 mvmul(M3 a, V3 b) { return v3(vdot(a.r[0], b), vdot(a.r[1], b), vdot(a.r[2], b)); }
static inline M3 mmul(M3 a, M3 b)
{
    M3 c;
    for (int i = 0; i < 3; ++i)
        c.r[i] = v3(vdot(a.r[i], mcol(b, 0)), vdot(a.r[i], mcol(b, 1)), vdot(a.r[i], mcol(b, 2)));
    return c;
}
static inline M3 madd(M3 a, M3 b) { return m3rows(vadd(a.r[0], b.r[0]), vadd(a.r[1], b.r[1]), vadd(a.r[2], b.r[2])); }
static inline M3 mscale(M3 a, float s) { return m3rows(vmul(a.r[0], s), vmul(a.r[1], s), vmul(a.r[2], s)); }
static inline M3 mdivs(M3 a, float s) { return m3rows(vdiv(a.r[0], s), vdiv(a.r[1], s), vdiv(a.r[2], s)); }
static inline M3 mneg(M3 a) { return m3rows(vneg(a.r[0]), vneg(a.r[1]), vneg(a.r[2])); }
static inline M3 mtrans(M3 a)
{
    return m3rows(v3(a.r[0].x, a.r[1].x, a.r[2].x), v3(a.r[0].y, a.r[1].y, a.r[2].y),
                  v3(a.r[0].z, a.r[1].z, a.r[2].z));
}
static inline M3 mskew(V3 r) { return m3rows(v3(0, -r.z, r.y), v3(r.z, 0, -r.x), v3(-r.y, r.x, 0)); }
static inline M3 mouter(V3 a, V3 b) { return m3rows(vmul(b, a.x), vmul(b, a.y), vmul(b, a.z)); }
static inline M3 mdiagonalize(M3 m) { return mdiag(vlen(mcol(m, 0)), vlen(mcol(m, 1)), vlen(mcol(m, 2))); }

static inline Q4 q4(float x, float y, float z, float w)
{
    Q4 q;
    q.x = x;
    q.y = y;
    q.z = z;
    q.w = w;
    return q;
}
static inline V3 qvec(Q4 q) { return v3(q.x, q.y, q.z); }
static inline Q4 qmul(Q4 a, Q4 b)
{
    return q4(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
              a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}
static inline Q4 qadd(Q4 a, Q4 b) { return q4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
static inline Q4 qscale(Q4 a, float s) { return q4(a.x * s, a.y * s, a.z * s, a.w * s); }
static inline Q4 qdivs(Q4 a, float s) { return q4(a.x / s, a.y / s, a.z / s, a.w / s); }
static inline float qlensq(Q4 q) { return vlensq(qvec(q)) + q.w * q.w; }
static inline Q4 qnormalize(Q4 q) { return qdivs(q, sqrtf(qlensq(q))); }
static inline Q4 qconj(Q4 q) { return q4(-q.x, -q.y, -q.z, q.w); }
static inline Q4 qinverse(Q4 q) { return qdivs(qconj(q), qlensq(q)); }
/* quat - quat = 2 vec(a b^-1)   (maths.h:269-272) */
static inline V3 qdiff(Q4 a, Q4 b) { return vmul(qvec(qmul(a, qinverse(b))), 2.0f); }
/* quat + float3 = normalize(a + (b,0) a / 2)   (maths.h:274-277) */
static inline Q4 qstep(Q4 a, V3 b) { return qnormalize(qadd(a, qscale(qmul(q4(b.x, b.y, b.z, 0), a), 0.5f))); }
static inline V3 qrotate(Q4 q, V3 v)
{
    V3 u = qvec(q);
    V3 t = vmul(vcross(u, v), 2.0f);
    return vadd(vadd(v, vmul(t, q.w)), vcross(u, t));
}
static inline V3 xform(V3 p, Q4 q, V3 v) { return vadd(qrotate(q, v), p); }
static inline M3 orthonormal(V3 n)
{
    V3 t1 = fabsf(n.x) > fabsf(n.z) ? v3(-n.y, n.x, 0) : v3(0, -n.z, n.y);
    t1 = vdiv(t1, vlen(t1));
    V3 t2 = vcross(n, t1);
    return m3rows(n, t1, t2);
}

/* Unpivoted LDL^T of the 6x6 system [[aLin, aCross^T], [aCross, aAng]] read from lower
 * triangles (maths.h:481-547); same per-entry operation order, written as loops. */
static void ldl_solve6(M3 aLin, M3 aAng, M3 aCross, V3 bLin, V3 bAng, V3 *xLin, V3 *xAng)
{
    float A[6][6];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c <= r; ++c)
        {
            A[r][c] = VE(aLin.r[r], c);
            A[3 + r][3 + c] = VE(aAng.r[r], c);
        }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            A[3 + r][c] = VE(aCross.r[r], c);

    float L[6][6];
    float D[6];
    for (int j = 0; j < 6; ++j)
    {
        if (j == 0)
            D[0] = A[0][0];
        else
        {
            float s = L[j][0] * L[j][0] * D[0];
            for (int k = 1; k < j; ++k)
                s = s + L[j][k] * L[j][k] * D[k];
            D[j] = A[j][j] - s;
        }
        for (int i = j + 1; i < 6; ++i)
        {
            float v = A[i][j];
            for (int k = 0; k < j; ++k)
                v = v - L[j][k] * L[i][k] * D[k];
            L[i][j] = v / D[j];
        }
    }
    float b[6] = {bLin.x, bLin.y, bLin.z, bAng.x, bAng.y, bAng.z};
    float y[6], z[6], x[6];
    for (int i = 0; i < 6; ++i)
    {
        float v = b[i];
        for (int k = 0; k < i; ++k)
            v = v - L[i][k] * y[k];
        y[i] = v;
    }
    for (int i = 0; i < 6; ++i)
        z[i] = y[i] / D[i];
    for (int i = 5; i >= 0; --i)
    {
        float v = z[i];
        for (int k = i + 1; k < 6; ++k)
            v = v - L[k][i] * x[k];
        x[i] = v;
    }
    *xLin = v3(x[0], x[1], x[2]);
    *xAng = v3(x[3], x[4], x[5]);
}

/* ------------------------------------------------------------------------- */
/* World                                                                     */
/* ------------------------------------------------------------------------- */

#define PENALTY_MIN 1.0f
#define PENALTY_MAX 10000000000.0f
#define COLLISION_MARGIN 0.01f
#define STICK_THRESH 0.00001f

typedef struct
{
    V3 pos;
    Q4 q;
    V3 initLin;
    Q4 initAng;
    V3 inertLin;
    Q4 inertAng;
    V3 vel;
    V3 angvel;
    V3 prevVel;
    V3 size;
    float mass;
    V3 moment;
    float friction;
    float radius;
    int shape;            /* ORACLE_SHAPE_* (RigidShape::type) */
    float shapeRadius;    /* RigidShape::radius (a box's: length(size / 2)) */
    float halfLength;     /* RigidShape::halfLength (capsules, cylinders) */
} Body;

typedef struct
{
    int key;
    V3 rA, rB, C0, penalty, lambda;
    int stick;
} Contact;

typedef struct
{
    int a, b;
    int64_t seq;
    Contact c[8];
    M3 basis;
    int n;
    float friction;
    /* tape bookkeeping: index in the previous step's list (-1 = created this step), the
     * matched previous contact of each contact (-1 = new) and its penalty clamp flags */
    int oldIndex;
    int srcSlot[8];
    unsigned char iflags[8];
} Manifold;

typedef struct
{
    int a, b; /* a may be -1 (world anchor) */
    int64_t seq;
    V3 rA, rB, C0Lin, C0Ang, penLin, penAng, lamLin, lamAng;
    float stiffLin, stiffAng, fracture, torqueArm;
    int broken;
} Joint;

typedef struct
{
    int a, b;
    int64_t seq;
    V3 rA, rB;
    float rest, stiffness;
} Spring;

typedef struct
{
    int a, b;
    int64_t seq;
} Ignore;

/* adjacency entry: a force incident on a body */
typedef struct
{
    int body;
    int64_t seq;
    int type;  /* ORACLE_FORCE_* */
    int index; /* into the per-type array */
    int isA;
} Incidence;

struct OracleWorld
{
    OracleParams p;
    int n;
    Body *bodies;
    Manifold *man;
    int nMan, capMan;
    Joint *joints;
    int nJoints;
    Spring *springs;
    int nSprings;
    Ignore *ignores;
    int nIgnores;
    int64_t nextSeq;
    /* adjacency, rebuilt whenever the force set changes */
    Incidence *inc;
    int nInc, capInc;
    int *adjStart; /* n + 1 */
    /* colouring */
    int *colour;
    int nColours;
    int *solveOrder;
    int nSolve;
    int64_t counters[9];
    /* frozen-branch tape (oracle_tape_begin) */
    int recording;
    int curIter;
    OracleTapeStep *tape;
    int tapeSteps, tapeCap;
};

static int cmp_incidence(const void *pa, const void *pb)
{
    const Incidence *a = (const Incidence *)pa, *b = (const Incidence *)pb;
    if (a->body != b->body)
        return a->body < b->body ? -1 : 1;
    if (a->seq != b->seq)
        return a->seq > b->seq ? -1 : 1; /* newest first */
    return 0;
}

static void push_inc(OracleWorld *w, int body, int64_t seq, int type, int index, int isA)
{
    if (body < 0)
        return;
    if (w->nInc == w->capInc)
    {
        w->capInc = w->capInc ? w->capInc * 2 : 1024;
        w->inc = (Incidence *)realloc(w->inc, sizeof(Incidence) * (size_t)w->capInc);
    }
    Incidence e = {body, seq, type, index, isA};
    w->inc[w->nInc++] = e;
}

static void build_adjacency(OracleWorld *w)
{
    w->nInc = 0;
    for (int i = 0; i < w->nMan; ++i)
    {
        push_inc(w, w->man[i].a, w->man[i].seq, ORACLE_FORCE_MANIFOLD, i, 1);
        push_inc(w, w->man[i].b, w->man[i].seq, ORACLE_FORCE_MANIFOLD, i, 0);
    }
    for (int i = 0; i < w->nJoints; ++i)
    {
        push_inc(w, w->joints[i].a, w->joints[i].seq, ORACLE_FORCE_JOINT, i, 1);
        push_inc(w, w->joints[i].b, w->joints[i].seq, ORACLE_FORCE_JOINT, i, 0);
    }
    for (int i = 0; i < w->nSprings; ++i)
    {
        push_inc(w, w->springs[i].a, w->springs[i].seq, ORACLE_FORCE_SPRING, i, 1);
        push_inc(w, w->springs[i].b, w->springs[i].seq, ORACLE_FORCE_SPRING, i, 0);
    }
    for (int i = 0; i < w->nIgnores; ++i)
    {
        push_inc(w, w->ignores[i].a, w->ignores[i].seq, ORACLE_FORCE_IGNORE, i, 1);
        push_inc(w, w->ignores[i].b, w->ignores[i].seq, ORACLE_FORCE_IGNORE, i, 0);
    }
    qsort(w->inc, (size_t)w->nInc, sizeof(Incidence), cmp_incidence);
    for (int b = 0; b <= w->n; ++b)
        w->adjStart[b] = 0;
    for (int k = 0; k < w->nInc; ++k)
        w->adjStart[w->inc[k].body + 1]++;
    for (int b = 0; b < w->n; ++b)
        w->adjStart[b + 1] += w->adjStart[b];
}

static void force_bodies(const OracleWorld *w, const Incidence *e, int *a, int *b)
{
    switch (e->type)
    {
    case ORACLE_FORCE_MANIFOLD:
        *a = w->man[e->index].a;
        *b = w->man[e->index].b;
        break;
    case ORACLE_FORCE_JOINT:
        *a = w->joints[e->index].a;
        *b = w->joints[e->index].b;
        break;
    case ORACLE_FORCE_SPRING:
        *a = w->springs[e->index].a;
        *b = w->springs[e->index].b;
        break;
    default:
        *a = w->ignores[e->index].a;
        *b = w->ignores[e->index].b;
        break;
    }
}

static int degree(const OracleWorld *w, int b) { return w->adjStart[b + 1] - w->adjStart[b]; }

/* Rigid::constrainedTo via the shorter list (solver.cpp:197-205, rigid.cpp:105-116) */
static int constrained(const OracleWorld *w, int a, int b)
{
    int self = degree(w, a) <= degree(w, b) ? a : b;
    int other = self == a ? b : a;
    for (int k = w->adjStart[self]; k < w->adjStart[self + 1]; ++k)
    {
        int fa, fb;
        force_bodies(w, &w->inc[k], &fa, &fb);
        if ((fa == self && fb == other) || (fa == other && fb == self))
            return 1;
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Broadphase                                                                */
/* ------------------------------------------------------------------------- */

typedef struct
{
    int a, b;
} Pair;

typedef struct
{
    Pair *v;
    int n, cap;
} PairList;

static void pair_push(PairList *l, int a, int b)
{
    if (l->n == l->cap)
    {
        l->cap = l->cap ? l->cap * 2 : 1024;
        l->v = (Pair *)realloc(l->v, sizeof(Pair) * (size_t)l->cap);
    }
    l->v[l->n].a = a;
    l->v[l->n].b = b;
    l->n++;
}

/* A bounding-sphere hit (solver.cpp:131-164, classifyHit :197-213): pairs that already
 * share a force are dropped, the rest become new manifolds in hit order. */
static void sphere_hit(OracleWorld *w, PairList *out, int a, int b)
{
    w->counters[1]++;
    if (constrained(w, a, b))
        w->counters[2]++;
    else
        pair_push(out, a, b);
}

static void generate_pair(OracleWorld *w, PairList *out, int a, int b)
{
    w->counters[0]++;
    V3 dp = vsub(w->bodies[a].pos, w->bodies[b].pos);
    float r = w->bodies[a].radius + w->bodies[b].radius;
    if (vdot(dp, dp) <= r * r)
        sphere_hit(w, out, a, b);
}

static void broadphase_all_pairs(OracleWorld *w, PairList *out)
{
    for (int a = 0; a < w->n; ++a)
        for (int b = a + 1; b < w->n; ++b)
            generate_pair(w, out, a, b);
}

typedef struct
{
    uint32_t key;
    int body;
    V3 center;
    float radius;
    float slack;
} GridEntry;

typedef struct
{
    int body;
    V3 lo, hi;
    float slack;
} LargeBody;

static int cmp_float(const void *a, const void *b)
{
    float x = *(const float *)a, y = *(const float *)b;
    return x < y ? -1 : x > y ? 1 : 0;
}

static int cmp_grid(const void *pa, const void *pb)
{
    const GridEntry *a = (const GridEntry *)pa, *b = (const GridEntry *)pb;
    if (a->key != b->key)
        return a->key < b->key ? -1 : 1;
    return a->body < b->body ? -1 : a->body > b->body ? 1 : 0;
}

/* Uniform grid (solver.cpp:284-486). Hits come out in the reference's creation order:
 * sorted entry i, then own cell, then the 13 forward cells, then the large bodies;
 * large-large pairs last. */
static void broadphase_grid(OracleWorld *w, PairList *out)
{
    int n = w->n;
    if (n < 2)
        return;
    float *radii = (float *)malloc(sizeof(float) * (size_t)n);
    for (int i = 0; i < n; ++i)
        radii[i] = w->bodies[i].radius;
    size_t pct = (size_t)n * 95 / 100;
    if (pct > (size_t)n - 1)
        pct = (size_t)n - 1;
    qsort(radii, (size_t)n, sizeof(float), cmp_float);
    float binnedRadius = rmax(radii[pct], 1e-3f);
    free(radii);
    float cellSize = binnedRadius * 2.0f;

    GridEntry *entries = (GridEntry *)malloc(sizeof(GridEntry) * (size_t)n);
    LargeBody *large = (LargeBody *)malloc(sizeof(LargeBody) * (size_t)n);
    int nEntries = 0, nLarge = 0;
    V3 bmin = v3(FLT_MAX, FLT_MAX, FLT_MAX), bmax = v3(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    for (int i = 0; i < n; ++i)
    {
        const Body *body = &w->bodies[i];
        float slack = vlen(body->vel) * w->p.dt;
        if (body->radius > binnedRadius)
        {
            /* solver.cpp:314-326: boxes by their rotated extents, round shapes by radius */
            V3 h = v3(body->radius, body->radius, body->radius);
            if (body->shape == ORACLE_SHAPE_BOX)
            {
                V3 e = vmul(body->size, 0.5f);
                V3 cx = qrotate(body->q, v3(1, 0, 0));
                V3 cy = qrotate(body->q, v3(0, 1, 0));
                V3 cz = qrotate(body->q, v3(0, 0, 1));
                h = v3(fabsf(cx.x) * e.x + fabsf(cy.x) * e.y + fabsf(cz.x) * e.z,
                       fabsf(cx.y) * e.x + fabsf(cy.y) * e.y + fabsf(cz.y) * e.z,
                       fabsf(cx.z) * e.x + fabsf(cy.z) * e.y + fabsf(cz.z) * e.z);
            }
            large[nLarge].body = i;
            large[nLarge].lo = vsub(body->pos, h);
            large[nLarge].hi = vadd(body->pos, h);
            large[nLarge].slack = slack;
            nLarge++;
            continue;
        }
        V3 c = body->pos;
        bmin = v3(rmin(bmin.x, c.x), rmin(bmin.y, c.y), rmin(bmin.z, c.z));
        bmax = v3(rmax(bmax.x, c.x), rmax(bmax.y, c.y), rmax(bmax.z, c.z));
        entries[nEntries].key = 0;
        entries[nEntries].body = i;
        entries[nEntries].center = c;
        entries[nEntries].radius = body->radius;
        entries[nEntries].slack = slack;
        nEntries++;
    }

    int nx = 1, ny = 1, nz = 1;
    uint32_t *cellStart = NULL;
    if (nEntries > 0)
    {
        const uint64_t maxCells = 1ull << 22;
        V3 extent = vsub(bmax, bmin);
        nx = (int)(extent.x / cellSize) + 1;
        ny = (int)(extent.y / cellSize) + 1;
        nz = (int)(extent.z / cellSize) + 1;
        uint64_t numCells = (uint64_t)nx * (uint64_t)ny * (uint64_t)nz;
        while (numCells > maxCells)
        {
            cellSize *= rmax(cbrtf((float)numCells / (float)maxCells), 1.1f);
            nx = (int)(extent.x / cellSize) + 1;
            ny = (int)(extent.y / cellSize) + 1;
            nz = (int)(extent.z / cellSize) + 1;
            numCells = (uint64_t)nx * (uint64_t)ny * (uint64_t)nz;
        }
        for (int k = 0; k < nEntries; ++k)
        {
            GridEntry *e = &entries[k];
            int ix = (int)rclamp((e->center.x - bmin.x) / cellSize, 0.0f, (float)(nx - 1));
            int iy = (int)rclamp((e->center.y - bmin.y) / cellSize, 0.0f, (float)(ny - 1));
            int iz = (int)rclamp((e->center.z - bmin.z) / cellSize, 0.0f, (float)(nz - 1));
            e->key = (uint32_t)(ix + nx * (iy + ny * iz));
        }
        qsort(entries, (size_t)nEntries, sizeof(GridEntry), cmp_grid);
        cellStart = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)numCells);
        memset(cellStart, 0xFF, sizeof(uint32_t) * (size_t)numCells);
        for (int k = 0; k < nEntries; ++k)
            if (k == 0 || entries[k].key != entries[k - 1].key)
                cellStart[entries[k].key] = (uint32_t)k;
    }

    static const int fwd[13][3] = {{1, 0, 0},   {-1, 1, 0}, {0, 1, 0},  {1, 1, 0},  {-1, -1, 1},
                                   {0, -1, 1},  {1, -1, 1}, {-1, 0, 1}, {0, 0, 1},  {1, 0, 1},
                                   {-1, 1, 1},  {0, 1, 1},  {1, 1, 1}};
    for (int i = 0; i < nEntries; ++i)
    {
        const GridEntry *a = &entries[i];
#define TEST_ENTRY(bb)                                                                                         \
    do                                                                                                         \
    {                                                                                                          \
        w->counters[0]++;                                                                                      \
        V3 dp = vsub(a->center, (bb)->center);                                                                 \
        float r = a->radius + (bb)->radius;                                                                    \
        if (!(vdot(dp, dp) > r * r))                                                                           \
            sphere_hit(w, out, a->body, (bb)->body);                                                           \
    } while (0)
        for (int j = i + 1; j < nEntries && entries[j].key == a->key; ++j)
            TEST_ENTRY(&entries[j]);
        int ix = (int)(a->key % (uint32_t)nx);
        uint32_t t = a->key / (uint32_t)nx;
        int iy = (int)(t % (uint32_t)ny);
        int iz = (int)(t / (uint32_t)ny);
        for (int d = 0; d < 13; ++d)
        {
            int cx = ix + fwd[d][0], cy = iy + fwd[d][1], cz = iz + fwd[d][2];
            if (cx < 0 || cx >= nx || cy < 0 || cy >= ny || cz < 0 || cz >= nz)
                continue;
            uint32_t nkey = (uint32_t)(cx + nx * (cy + ny * cz));
            uint32_t s = cellStart[nkey];
            if (s == UINT32_MAX)
                continue;
            for (int j = (int)s; j < nEntries && entries[j].key == nkey; ++j)
                TEST_ENTRY(&entries[j]);
        }
#undef TEST_ENTRY
        for (int l = 0; l < nLarge; ++l)
        {
            const LargeBody *L = &large[l];
            w->counters[0]++;
            V3 qp = v3(rclamp(a->center.x, L->lo.x, L->hi.x), rclamp(a->center.y, L->lo.y, L->hi.y),
                       rclamp(a->center.z, L->lo.z, L->hi.z));
            V3 dp = vsub(a->center, qp);
            float reach = a->radius + a->slack + L->slack + 4.0f * COLLISION_MARGIN;
            if (vdot(dp, dp) > reach * reach)
                continue;
            sphere_hit(w, out, a->body, L->body);
        }
    }
    for (int i = 0; i < nLarge; ++i)
        for (int j = i + 1; j < nLarge; ++j)
            generate_pair(w, out, large[i].body, large[j].body);
    free(cellStart);
    free(entries);
    free(large);
}

typedef struct
{
    float lo, hi;
    int body;
    V3 center;
    float radius;
} SapInterval;

static int cmp_sap(const void *pa, const void *pb)
{
    const SapInterval *a = (const SapInterval *)pa, *b = (const SapInterval *)pb;
    if (a->lo != b->lo)
        return a->lo < b->lo ? -1 : 1;
    return a->body < b->body ? -1 : a->body > b->body ? 1 : 0;
}

/* Sweep and prune along the axis of largest centre variance (solver.cpp:488-577). */
static void broadphase_sap(OracleWorld *w, PairList *out)
{
    int n = w->n;
    if (n < 2)
        return;
    V3 mean = v3(0, 0, 0);
    for (int i = 0; i < n; ++i)
        mean = vadd(mean, w->bodies[i].pos);
    mean = vdiv(mean, (float)n);
    V3 var = v3(0, 0, 0);
    for (int i = 0; i < n; ++i)
    {
        V3 d = vsub(w->bodies[i].pos, mean);
        var = vadd(var, v3(d.x * d.x, d.y * d.y, d.z * d.z));
    }
    int axis = 0;
    if (var.y > VE(var, axis))
        axis = 1;
    if (var.z > VE(var, axis))
        axis = 2;
    SapInterval *iv = (SapInterval *)malloc(sizeof(SapInterval) * (size_t)n);
    for (int i = 0; i < n; ++i)
    {
        float c = VE(w->bodies[i].pos, axis);
        iv[i].lo = c - w->bodies[i].radius;
        iv[i].hi = c + w->bodies[i].radius;
        iv[i].body = i;
        iv[i].center = w->bodies[i].pos;
        iv[i].radius = w->bodies[i].radius;
    }
    qsort(iv, (size_t)n, sizeof(SapInterval), cmp_sap);
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j)
        {
            if (iv[j].lo > iv[i].hi)
                break;
            w->counters[0]++;
            V3 dp = vsub(iv[i].center, iv[j].center);
            float r = iv[i].radius + iv[j].radius;
            if (vdot(dp, dp) > r * r)
                continue;
            sphere_hit(w, out, iv[i].body, iv[j].body);
        }
    free(iv);
}

/* ------------------------------------------------------------------------- */
/* Box-box narrowphase (collide.cpp)                                         */
/* ------------------------------------------------------------------------- */

typedef struct
{
    V3 center;
    Q4 q;
    V3 half;
    V3 axis[3];
} Obb;

typedef struct
{
    int type; /* 0 face A, 1 face B, 2 edge */
    int ia, ib;
    float sep;
    V3 n;
    int valid;
} SatBest;

static Obb make_obb(V3 pos, Q4 q, V3 size)
{
    Obb o;
    o.center = pos;
    o.q = q;
    o.half = vmul(size, 0.5f);
    o.axis[0] = qrotate(q, v3(1.0f, 0.0f, 0.0f));
    o.axis[1] = qrotate(q, v3(0.0f, 1.0f, 0.0f));
    o.axis[2] = qrotate(q, v3(0.0f, 0.0f, 1.0f));
    return o;
}

static inline float absdot(V3 a, V3 b) { return fabsf(vdot(a, b)); }

static V3 support_point(const Obb *o, V3 dir)
{
    float sx = vdot(dir, o->axis[0]) >= 0.0f ? 1.0f : -1.0f;
    float sy = vdot(dir, o->axis[1]) >= 0.0f ? 1.0f : -1.0f;
    float sz = vdot(dir, o->axis[2]) >= 0.0f ? 1.0f : -1.0f;
    return vadd(vadd(vadd(o->center, vmul(o->axis[0], o->half.x * sx)), vmul(o->axis[1], o->half.y * sy)),
                vmul(o->axis[2], o->half.z * sz));
}

static void face_axes(const Obb *o, int ax, V3 *u, V3 *v, float *eu, float *ev)
{
    if (ax == 0)
    {
        *u = o->axis[1];
        *v = o->axis[2];
        *eu = o->half.y;
        *ev = o->half.z;
    }
    else if (ax == 1)
    {
        *u = o->axis[0];
        *v = o->axis[2];
        *eu = o->half.x;
        *ev = o->half.z;
    }
    else
    {
        *u = o->axis[0];
        *v = o->axis[1];
        *eu = o->half.x;
        *ev = o->half.y;
    }
}

static int clip_plane(const V3 *in, int cnt, V3 pn, float off, V3 *outv)
{
    if (cnt <= 0)
        return 0;
    int k = 0;
    V3 a = in[cnt - 1];
    float da = vdot(pn, a) - off;
    for (int i = 0; i < cnt; ++i)
    {
        V3 b = in[i];
        float db = vdot(pn, b) - off;
        int ain = da <= 1.0e-5f;
        int bin = db <= 1.0e-5f;
        if (ain != bin)
        {
            float t = 0.0f;
            float denom = da - db;
            if (fabsf(denom) > 1.0e-6f)
                t = rclamp(da / denom, 0.0f, 1.0f);
            if (k < 16)
                outv[k++] = vadd(a, vmul(vsub(b, a), t));
        }
        if (bin && k < 16)
            outv[k++] = b;
        a = b;
        da = db;
    }
    return k;
}

typedef struct
{
    int key;
    V3 rA, rB;
} NewContact;

static int add_contact(V3 pA, Q4 qA, V3 pB, Q4 qB, NewContact *cs, int *count, V3 *mids, V3 xA, V3 xB, int key)
{
    V3 mid = vmul(vadd(xA, xB), 0.5f);
    for (int i = 0; i < *count; ++i)
    {
        V3 d = vsub(mid, mids[i]);
        if (vlensq(d) < 1.0e-6f)
            return 0;
    }
    if (*count >= 8)
        return 0;
    NewContact *c = &cs[*count];
    c->key = key;
    c->rA = qrotate(qconj(qA), vsub(xA, pA));
    c->rB = qrotate(qconj(qB), vsub(xB, pB));
    mids[*count] = mid;
    (*count)++;
    return 1;
}

static int test_axis(const Obb *A, const Obb *B, V3 delta, V3 axis, int type, int ia, int ib, SatBest *best)
{
    float lenSq = vlensq(axis);
    if (lenSq < 1.0e-6f)
        return 1;
    float invLen = 1.0f / sqrtf(lenSq);
    V3 n = vmul(axis, invLen);
    if (vdot(n, delta) < 0.0f)
        n = vneg(n);
    float distance = fabsf(vdot(delta, n));
    float rA = A->half.x * absdot(n, A->axis[0]) + A->half.y * absdot(n, A->axis[1]) + A->half.z * absdot(n, A->axis[2]);
    float rB = B->half.x * absdot(n, B->axis[0]) + B->half.y * absdot(n, B->axis[1]) + B->half.z * absdot(n, B->axis[2]);
    float sep = distance - (rA + rB);
    if (sep > 0.0f)
        return 0;
    if (!best->valid || sep > best->sep)
    {
        best->valid = 1;
        best->type = type;
        best->ia = ia;
        best->ib = ib;
        best->sep = sep;
        best->n = n;
    }
    return 1;
}

static void support_edge(const Obb *o, int ax, V3 dir, V3 *ea, V3 *eb)
{
    int a1 = (ax + 1) % 3, a2 = (ax + 2) % 3;
    float s1 = vdot(dir, o->axis[a1]) >= 0.0f ? 1.0f : -1.0f;
    float s2 = vdot(dir, o->axis[a2]) >= 0.0f ? 1.0f : -1.0f;
    V3 ec = vadd(vadd(o->center, vmul(o->axis[a1], VEC(o->half, a1) * s1)), vmul(o->axis[a2], VEC(o->half, a2) * s2));
    *ea = vsub(ec, vmul(o->axis[ax], VEC(o->half, ax)));
    *eb = vadd(ec, vmul(o->axis[ax], VEC(o->half, ax)));
}

static void closest_segments(V3 p0, V3 p1, V3 q0, V3 q1, V3 *c0, V3 *c1)
{
    V3 d1 = vsub(p1, p0), d2 = vsub(q1, q0), r = vsub(p0, q0);
    float a = vdot(d1, d1), e = vdot(d2, d2), f = vdot(d2, r);
    float s = 0.0f, t = 0.0f;
    if (a <= 1.0e-6f && e <= 1.0e-6f)
    {
        *c0 = p0;
        *c1 = q0;
        return;
    }
    if (a <= 1.0e-6f)
        t = rclamp(f / e, 0.0f, 1.0f);
    else
    {
        float c = vdot(d1, r);
        if (e <= 1.0e-6f)
            s = rclamp(-c / a, 0.0f, 1.0f);
        else
        {
            float b = vdot(d1, d2);
            float denom = a * e - b * b;
            if (fabsf(denom) > 1.0e-6f)
                s = rclamp((b * f - c * e) / denom, 0.0f, 1.0f);
            t = (b * s + f) / e;
            if (t < 0.0f)
            {
                t = 0.0f;
                s = rclamp(-c / a, 0.0f, 1.0f);
            }
            else if (t > 1.0f)
            {
                t = 1.0f;
                s = rclamp((b - c) / a, 0.0f, 1.0f);
            }
        }
    }
    *c0 = vadd(p0, vmul(d1, s));
    *c1 = vadd(q0, vmul(d2, t));
}

static int face_manifold(const Obb *A, const Obb *B, int refIsA, int refAxis, V3 nAB, NewContact *cs)
{
    const Obb *R = refIsA ? A : B;
    const Obb *I = refIsA ? B : A;
    V3 outward = refIsA ? nAB : vneg(nAB);
    float sgn = vdot(outward, R->axis[refAxis]) >= 0.0f ? 1.0f : -1.0f;
    V3 rn = vmul(R->axis[refAxis], sgn);
    V3 rc = vadd(R->center, vmul(rn, VEC(R->half, refAxis)));
    V3 ru, rv;
    float reu, rev;
    face_axes(R, refAxis, &ru, &rv, &reu, &rev);

    int incAxis = 0;
    float best = -FLT_MAX;
    for (int i = 0; i < 3; ++i)
    {
        float d = absdot(I->axis[i], rn);
        if (d > best)
        {
            best = d;
            incAxis = i;
        }
    }
    V3 c0[16], c1[16];
    {
        float s = vdot(I->axis[incAxis], rn) > 0.0f ? -1.0f : 1.0f;
        V3 fn = vmul(I->axis[incAxis], s);
        V3 fc = vadd(I->center, vmul(fn, VEC(I->half, incAxis)));
        V3 u, v;
        float eu, ev;
        face_axes(I, incAxis, &u, &v, &eu, &ev);
        c0[0] = vadd(vadd(fc, vmul(u, eu)), vmul(v, ev));
        c0[1] = vadd(vsub(fc, vmul(u, eu)), vmul(v, ev));
        c0[2] = vsub(vsub(fc, vmul(u, eu)), vmul(v, ev));
        c0[3] = vsub(vadd(fc, vmul(u, eu)), vmul(v, ev));
    }
    int cnt = 4;
    V3 n0 = ru;
    cnt = clip_plane(c0, cnt, n0, vdot(n0, rc) + reu, c1);
    if (!cnt)
        return 0;
    V3 n1 = vneg(ru);
    cnt = clip_plane(c1, cnt, n1, vdot(n1, rc) + reu, c0);
    if (!cnt)
        return 0;
    V3 n2 = rv;
    cnt = clip_plane(c0, cnt, n2, vdot(n2, rc) + rev, c1);
    if (!cnt)
        return 0;
    V3 n3 = vneg(rv);
    cnt = clip_plane(c1, cnt, n3, vdot(n3, rc) + rev, c0);
    if (!cnt)
        return 0;

    int count = 0;
    V3 mids[8];
    int prefix = (refIsA ? 0 : 1) << 24;
    prefix |= (refAxis & 0xFF) << 16;
    prefix |= (incAxis & 0xFF) << 8;
    for (int i = 0; i < cnt && count < 8; ++i)
    {
        V3 p = c0[i];
        float dist = vdot(vsub(p, rc), rn);
        if (dist > 1.0e-5f)
            continue;
        V3 pr = vsub(p, vmul(rn, dist));
        V3 xA = refIsA ? pr : p;
        V3 xB = refIsA ? p : pr;
        add_contact(A->center, A->q, B->center, B->q, cs, &count, mids, xA, xB, prefix | (i & 0xFF));
    }
    if (!count)
        add_contact(A->center, A->q, B->center, B->q, cs, &count, mids, support_point(A, nAB),
                    support_point(B, vneg(nAB)), prefix);
    return count;
}

static int edge_contact(const Obb *A, const Obb *B, int axA, int axB, V3 nAB, NewContact *cs)
{
    V3 a0, a1, b0, b1, xA, xB;
    support_edge(A, axA, nAB, &a0, &a1);
    support_edge(B, axB, vneg(nAB), &b0, &b1);
    closest_segments(a0, a1, b0, b1, &xA, &xB);
    int count = 0;
    V3 mids[8];
    int key = (2 << 24) | ((axA & 0xFF) << 8) | (axB & 0xFF);
    add_contact(A->center, A->q, B->center, B->q, cs, &count, mids, xA, xB, key);
    if (!count)
        add_contact(A->center, A->q, B->center, B->q, cs, &count, mids, support_point(A, nAB),
                    support_point(B, vneg(nAB)), key);
    return count;
}

static int collide_boxes(V3 pA, Q4 qA, V3 sA, V3 pB, Q4 qB, V3 sB, NewContact *cs, M3 *basis)
{
    Obb A = make_obb(pA, qA, sA), B = make_obb(pB, qB, sB);
    V3 delta = vsub(B.center, A.center);
    SatBest face, edge;
    memset(&face, 0, sizeof(face));
    memset(&edge, 0, sizeof(edge));
    face.sep = -FLT_MAX;
    edge.sep = -FLT_MAX;
    for (int i = 0; i < 3; ++i)
        if (!test_axis(&A, &B, delta, A.axis[i], 0, i, -1, &face))
            return 0;
    for (int i = 0; i < 3; ++i)
        if (!test_axis(&A, &B, delta, B.axis[i], 1, -1, i, &face))
            return 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            if (!test_axis(&A, &B, delta, vcross(A.axis[i], B.axis[j]), 2, i, j, &edge))
                return 0;
    if (!face.valid)
        return 0;
    SatBest best = face;
    if (edge.valid && 0.95f * edge.sep > face.sep + 0.01f)
        best = edge;
    *basis = orthonormal(vneg(best.n));
    if (best.type == 2)
        return edge_contact(&A, &B, best.ia, best.ib, best.n, cs);
    if (best.type == 0)
        return face_manifold(&A, &B, 1, best.ia, best.n, cs);
    return face_manifold(&A, &B, 0, best.ib, best.n, cs);
}

/* ------------------------------------------------------------------------- */
/* Force initialisation                                                      */
/* ------------------------------------------------------------------------- */

/* ------------------------------------------------------------------------- */
/* Round shapes: spheres, capsules, cylinders (collide.cpp:435-1176)         */
/* ------------------------------------------------------------------------- */

#define SAT_EPS 1.0e-6f /* SAT_AXIS_EPSILON (collide.cpp:20) */

static int is_round(const Body *b) { return b->shape == ORACLE_SHAPE_SPHERE || b->shape == ORACLE_SHAPE_CAPSULE; }
static int is_cyl(const Body *b) { return b->shape == ORACLE_SHAPE_CYLINDER; }
static V3 vnormalize(V3 v) { return vdiv(v, vlen(v)); }

/* closestPointOnOBB, pointInsideOBB, localToOBBWorld (collide.cpp:435-456) */
static V3 obb_closest(const Obb *o, V3 p)
{
    V3 d = vsub(p, o->center);
    return vadd(vadd(vadd(o->center, vmul(o->axis[0], rclamp(vdot(d, o->axis[0]), -o->half.x, o->half.x))),
                     vmul(o->axis[1], rclamp(vdot(d, o->axis[1]), -o->half.y, o->half.y))),
                vmul(o->axis[2], rclamp(vdot(d, o->axis[2]), -o->half.z, o->half.z)));
}

static V3 obb_local(const Obb *o, V3 p)
{
    V3 d = vsub(p, o->center);
    return v3(vdot(d, o->axis[0]), vdot(d, o->axis[1]), vdot(d, o->axis[2]));
}

static V3 obb_world(const Obb *o, V3 l)
{
    return vadd(vadd(vadd(o->center, vmul(o->axis[0], l.x)), vmul(o->axis[1], l.y)), vmul(o->axis[2], l.z));
}

/* capsuleSegment / cylinderSegment (collide.cpp:468-488): a sphere is a point segment */
static void round_segment(const Body *b, V3 *a, V3 *c)
{
    if (b->shape == ORACLE_SHAPE_CAPSULE || b->shape == ORACLE_SHAPE_CYLINDER)
    {
        V3 axis = qrotate(b->q, v3(0.0f, 0.0f, 1.0f));
        *a = vsub(b->pos, vmul(axis, b->halfLength));
        *c = vadd(b->pos, vmul(axis, b->halfLength));
    }
    else
        *a = *c = b->pos;
}

/* closestPointOnSegment (collide.cpp:490-498) */
static V3 segment_closest(V3 a, V3 b, V3 p)
{
    V3 ab = vsub(b, a);
    float denom = vlensq(ab);
    if (denom < SAT_EPS)
        return a;
    float t = rclamp(vdot(vsub(p, a), ab) / denom, 0.0f, 1.0f);
    return vadd(a, vmul(ab, t));
}

/* addRoundContact (collide.cpp:500-517) */
static int round_contact(const Body *A, const Body *B, V3 cA, float rA, V3 cB, float rB, int key, NewContact *cs,
                         M3 *basis)
{
    V3 delta = vsub(cB, cA);
    float rs = rA + rB;
    float d2 = vlensq(delta);
    if (d2 > rs * rs)
        return 0;
    V3 n = d2 > SAT_EPS ? vdiv(delta, sqrtf(d2)) : v3(1.0f, 0.0f, 0.0f);
    V3 xA = vadd(cA, vmul(n, rA));
    V3 xB = vsub(cB, vmul(n, rB));
    *basis = orthonormal(vneg(n));
    int count = 0;
    V3 mids[8];
    add_contact(A->pos, A->q, B->pos, B->q, cs, &count, mids, xA, xB, key);
    return count;
}

/* thinStaticBoxTopFrame (collide.cpp:957-976): a static slab's thin axis and upward sign */
static int slab_frame(const Obb *o, const Body *box, int *thin, float *sign)
{
    if (box->mass > 0.0f)
        return 0;
    int t = 0;
    if (o->half.y < VEC(o->half, t))
        t = 1;
    if (o->half.z < VEC(o->half, t))
        t = 2;
    int a = (t + 1) % 3, b = (t + 2) % 3;
    if (VEC(o->half, t) * 4.0f > rmin(VEC(o->half, a), VEC(o->half, b)))
        return 0;
    *thin = t;
    *sign = vdot(o->axis[t], v3(0.0f, 0.0f, 1.0f)) >= 0.0f ? 1.0f : -1.0f;
    return 1;
}

/* sweptSphereBoxContact (collide.cpp:519-587) */
static int swept_sphere_box(const Obb *o, const Body *sph, const Body *box, float dt, V3 *nBoxToSphere, V3 *xBox)
{
    V3 rv = vsub(sph->vel, box->vel);
    if (dt <= 0.0f || vlensq(rv) < SAT_EPS)
        return 0;
    V3 cur = sph->pos;
    V3 prev = vsub(cur, vmul(rv, dt));
    V3 l0 = obb_local(o, prev), l1 = obb_local(o, cur);
    V3 delta = vsub(l1, l0);
    V3 eh = vadd(o->half, v3(sph->shapeRadius, sph->shapeRadius, sph->shapeRadius));
    float tEnter = 0.0f, tExit = 1.0f, hitSign = 1.0f;
    int hitAxis = -1;
    for (int ax = 0; ax < 3; ++ax)
    {
        float d = VEC(delta, ax), s0 = VEC(l0, ax), e = VEC(eh, ax);
        if (fabsf(d) < SAT_EPS)
        {
            if (s0 < -e || s0 > e)
                return 0;
            continue;
        }
        float inv = 1.0f / d;
        float t0 = (-e - s0) * inv, t1 = (e - s0) * inv, sg = -1.0f;
        if (t0 > t1)
        {
            float tmp = t0;
            t0 = t1;
            t1 = tmp;
            sg = 1.0f;
        }
        if (t0 > tEnter)
        {
            tEnter = t0;
            hitAxis = ax;
            hitSign = sg;
        }
        tExit = rmin(tExit, t1);
        if (tEnter > tExit)
            return 0;
    }
    if (hitAxis < 0 || tEnter < 0.0f || tEnter > 1.0f)
        return 0;
    V3 sl = vadd(l0, vmul(delta, tEnter));
    VE(sl, hitAxis) = VEC(o->half, hitAxis) * hitSign;
    for (int ax = 0; ax < 3; ++ax)
        if (ax != hitAxis)
            VE(sl, ax) = rclamp(VEC(sl, ax), -VEC(o->half, ax), VEC(o->half, ax));
    *nBoxToSphere = vmul(o->axis[hitAxis], hitSign);
    *xBox = obb_world(o, sl);
    return 1;
}

/* The slab-top point of a round body's centre (collide.cpp:651-684, 689-708), or 0. */
static int slab_point(const Obb *o, int thin, float sign, float radius, V3 center, V3 *xBox)
{
    V3 l = obb_local(o, center);
    float sd = VEC(l, thin) * sign - VEC(o->half, thin);
    if (sd > radius)
        return 0;
    for (int ax = 0; ax < 3; ++ax)
    {
        if (ax == thin)
            continue;
        if (VEC(l, ax) < -VEC(o->half, ax) - radius || VEC(l, ax) > VEC(o->half, ax) + radius)
            return 0;
    }
    VE(l, thin) = VEC(o->half, thin) * sign;
    for (int ax = 0; ax < 3; ++ax)
        if (ax != thin)
            VE(l, ax) = rclamp(VEC(l, ax), -VEC(o->half, ax), VEC(o->half, ax));
    *xBox = obb_world(o, l);
    return 1;
}

/* collideThinStaticBoxTopRound (collide.cpp:717-754): -1 when the box is no static slab */
static int slab_top_round(const Obb *o, const Body *rb, const Body *box, int roundIsA, NewContact *cs, M3 *basis)
{
    int thin;
    float sign;
    if (!slab_frame(o, box, &thin, &sign))
        return -1;
    V3 n = vmul(o->axis[thin], sign);
    V3 nAB = roundIsA ? vneg(n) : n;
    *basis = orthonormal(vneg(nAB));
    int count = 0;
    V3 mids[8], ends[2];
    int keys[2], nEnds;
    if (rb->shape == ORACLE_SHAPE_CAPSULE)
    {
        round_segment(rb, &ends[0], &ends[1]);
        keys[0] = 0x04000000;
        keys[1] = 0x04000001;
        nEnds = 2;
    }
    else
    {
        ends[0] = rb->pos;
        keys[0] = 0x02000000;
        nEnds = 1;
    }
    for (int e = 0; e < nEnds; ++e)
    {
        V3 xBox;
        if (!slab_point(o, thin, sign, rb->shapeRadius, ends[e], &xBox))
            continue;
        V3 xRound = vsub(ends[e], vmul(n, rb->shapeRadius));
        if (roundIsA)
            add_contact(rb->pos, rb->q, box->pos, box->q, cs, &count, mids, xRound, xBox, keys[e]);
        else
            add_contact(box->pos, box->q, rb->pos, rb->q, cs, &count, mids, xBox, xRound, keys[e]);
    }
    return count > 0 ? count : -1;
}

/* collideRoundRound (collide.cpp:756-765) */
static int collide_round_round(const Body *A, const Body *B, NewContact *cs, M3 *basis)
{
    V3 a0, a1, b0, b1, cA, cB;
    round_segment(A, &a0, &a1);
    round_segment(B, &b0, &b1);
    closest_segments(a0, a1, b0, b1, &cA, &cB);
    return round_contact(A, B, cA, A->shapeRadius, cB, B->shapeRadius, 0x03000000, cs, basis);
}

/* collideRoundBox (collide.cpp:767-896) */
static int collide_round_box(const Body *rb, const Body *box, int roundIsA, float dt, NewContact *cs, M3 *basis)
{
    Obb o = make_obb(box->pos, box->q, box->size);
    int top = slab_top_round(&o, rb, box, roundIsA, cs, basis);
    if (top >= 0)
        return top;
    V3 rc = rb->pos;
    if (rb->shape == ORACLE_SHAPE_CAPSULE)
    {
        V3 sa, sb;
        round_segment(rb, &sa, &sb);
        V3 ca = obb_closest(&o, sa), cb = obb_closest(&o, sb);
        rc = vlensq(vsub(sa, ca)) <= vlensq(vsub(sb, cb)) ? sa : sb;
    }
    float rr = rb->shapeRadius;
    V3 closest = obb_closest(&o, rc);
    V3 boxToRound = vsub(rc, closest);
    float d2 = vlensq(boxToRound);
    int onTop = 0;
    {
        /* thinStaticBoxTopContactRound (collide.cpp:632-685) */
        int thin;
        float sign;
        if (slab_frame(&o, box, &thin, &sign))
        {
            V3 n = vmul(o.axis[thin], sign);
            V3 sa, sb;
            round_segment(rb, &sa, &sb);
            float da = vdot(sa, n), db = vdot(sb, n);
            V3 topCenter;
            if (rb->shape == ORACLE_SHAPE_CAPSULE && fabsf(da - db) < 1.0e-4f)
                topCenter = segment_closest(sa, sb, rb->pos);
            else
                topCenter = da <= db ? sa : sb;
            V3 xBox;
            if (slab_point(&o, thin, sign, rr, topCenter, &xBox))
            {
                rc = topCenter;
                boxToRound = n;
                closest = xBox;
                d2 = 1.0f;
                onTop = 1;
            }
        }
    }
    V3 local = obb_local(&o, rc);
    int inside = fabsf(local.x) <= o.half.x && fabsf(local.y) <= o.half.y && fabsf(local.z) <= o.half.z;
    if (onTop)
    {
    }
    else if (inside)
    {
        V3 sn, sp;
        if (rb->shape == ORACLE_SHAPE_SPHERE && swept_sphere_box(&o, rb, box, dt, &sn, &sp))
        {
            boxToRound = sn;
            closest = sp;
            d2 = 1.0f;
        }
        else
        {
            int axis = 0;
            float sign = local.x >= 0.0f ? 1.0f : -1.0f;
            float best = o.half.x - fabsf(local.x);
            V3 rv = vsub(rb->vel, box->vel);
            if (box->mass <= 0.0f)
            {
                axis = 0;
                if (o.half.y < VEC(o.half, axis))
                    axis = 1;
                if (o.half.z < VEC(o.half, axis))
                    axis = 2;
                sign = vdot(o.axis[axis], v3(0.0f, 0.0f, 1.0f)) >= 0.0f ? 1.0f : -1.0f;
            }
            else if (vlensq(rv) > SAT_EPS)
            {
                V3 against = vneg(rv);
                float bestDot = -FLT_MAX;
                for (int ca = 0; ca < 3; ++ca)
                    for (int si = 0; si < 2; ++si)
                    {
                        float cs_ = si == 0 ? -1.0f : 1.0f;
                        float d = vdot(vmul(o.axis[ca], cs_), against);
                        if (d > bestDot)
                        {
                            bestDot = d;
                            axis = ca;
                            sign = cs_;
                        }
                    }
            }
            else
            {
                float dy = o.half.y - fabsf(local.y);
                if (dy < best)
                {
                    axis = 1;
                    sign = local.y >= 0.0f ? 1.0f : -1.0f;
                    best = dy;
                }
                float dz = o.half.z - fabsf(local.z);
                if (dz < best)
                {
                    axis = 2;
                    sign = local.z >= 0.0f ? 1.0f : -1.0f;
                }
            }
            V3 sl = local;
            VE(sl, axis) = VEC(o.half, axis) * sign;
            closest = obb_world(&o, sl);
            boxToRound = vmul(o.axis[axis], sign);
            d2 = 1.0f;
        }
    }
    else if (d2 > rr * rr)
    {
        V3 sn, sp;
        if (rb->shape != ORACLE_SHAPE_SPHERE || !swept_sphere_box(&o, rb, box, dt, &sn, &sp))
            return 0;
        boxToRound = sn;
        closest = sp;
        d2 = 1.0f;
    }
    V3 nBR = d2 > SAT_EPS ? vdiv(boxToRound, sqrtf(d2)) : v3(0.0f, 0.0f, 1.0f);
    V3 nAB = roundIsA ? vneg(nBR) : nBR;
    V3 xRound = vsub(rc, vmul(nBR, rr));
    *basis = orthonormal(vneg(nAB));
    int count = 0;
    V3 mids[8];
    int key = rb->shape == ORACLE_SHAPE_CAPSULE ? 0x04000000 : 0x02000000;
    if (roundIsA)
        add_contact(rb->pos, rb->q, box->pos, box->q, cs, &count, mids, xRound, closest, key);
    else
        add_contact(box->pos, box->q, rb->pos, rb->q, cs, &count, mids, closest, xRound, key);
    return count;
}

/* addThinStaticBoxTopCylinderContact (collide.cpp:978-1007) */
static void slab_cylinder_point(const Obb *o, const Body *cyl, const Body *box, int cylIsA, int thin, float sign, V3 xc,
                                int key, NewContact *cs, int *count, V3 *mids)
{
    V3 l = v3(vdot(vsub(xc, o->center), o->axis[0]), vdot(vsub(xc, o->center), o->axis[1]),
              vdot(vsub(xc, o->center), o->axis[2]));
    float sd = VEC(l, thin) * sign - VEC(o->half, thin);
    if (sd > COLLISION_MARGIN)
        return;
    for (int ax = 0; ax < 3; ++ax)
    {
        if (ax == thin)
            continue;
        if (VEC(l, ax) < -VEC(o->half, ax) - cyl->shapeRadius || VEC(l, ax) > VEC(o->half, ax) + cyl->shapeRadius)
            return;
    }
    VE(l, thin) = (VEC(o->half, thin) + COLLISION_MARGIN) * sign;
    for (int ax = 0; ax < 3; ++ax)
        if (ax != thin)
            VE(l, ax) = rclamp(VEC(l, ax), -VEC(o->half, ax), VEC(o->half, ax));
    V3 xBox = obb_world(o, l);
    if (cylIsA)
        add_contact(cyl->pos, cyl->q, box->pos, box->q, cs, count, mids, xc, xBox, key);
    else
        add_contact(box->pos, box->q, cyl->pos, cyl->q, cs, count, mids, xBox, xc, key);
}

static void across(V3 a, V3 *u, V3 *v)
{
    *u = fabsf(a.x) > fabsf(a.z) ? vnormalize(v3(-a.y, a.x, 0.0f)) : vnormalize(v3(0.0f, -a.z, a.y));
    *v = vnormalize(vcross(a, *u));
}

/* collideThinStaticBoxTopCylinder (collide.cpp:1009-1053) */
static int slab_top_cylinder(const Obb *o, const Body *cyl, const Body *box, int cylIsA, NewContact *cs, M3 *basis)
{
    int thin;
    float sign;
    if (!slab_frame(o, box, &thin, &sign))
        return -1;
    V3 n = vmul(o->axis[thin], sign);
    V3 nAB = cylIsA ? vneg(n) : n;
    *basis = orthonormal(vneg(nAB));
    V3 axis = qrotate(cyl->q, v3(0.0f, 0.0f, 1.0f));
    float ad = vdot(axis, n);
    int count = 0;
    V3 mids[8];
    if (fabsf(ad) > 0.65f)
    {
        float as = ad >= 0.0f ? 1.0f : -1.0f;
        V3 cap = vsub(cyl->pos, vmul(axis, cyl->halfLength * as));
        V3 u, v;
        across(axis, &u, &v);
        V3 offs[4] = {vmul(u, cyl->shapeRadius), vmul(vneg(u), cyl->shapeRadius), vmul(v, cyl->shapeRadius),
                      vmul(vneg(v), cyl->shapeRadius)};
        for (int i = 0; i < 4; ++i)
            slab_cylinder_point(o, cyl, box, cylIsA, thin, sign, vadd(cap, offs[i]), 0x05000000 | i, cs, &count, mids);
    }
    else
    {
        V3 radial = vsub(n, vmul(axis, ad));
        if (vlensq(radial) < SAT_EPS)
            radial = n;
        radial = vnormalize(radial);
        V3 a = vsub(cyl->pos, vmul(axis, cyl->halfLength));
        V3 b = vadd(cyl->pos, vmul(axis, cyl->halfLength));
        slab_cylinder_point(o, cyl, box, cylIsA, thin, sign, vsub(a, vmul(radial, cyl->shapeRadius)), 0x05000100, cs,
                            &count, mids);
        slab_cylinder_point(o, cyl, box, cylIsA, thin, sign, vsub(b, vmul(radial, cyl->shapeRadius)), 0x05000101, cs,
                            &count, mids);
    }
    return count > 0 ? count : -1;
}

/* addCylinderCapContacts (collide.cpp:1080-1091) */
static int cylinder_caps(const Body *A, const Body *B, V3 nAB, V3 capA, V3 capB, float radius, NewContact *cs, M3 *basis)
{
    *basis = orthonormal(vneg(nAB));
    int count = 0;
    V3 mids[8], u, v;
    across(nAB, &u, &v);
    V3 offs[4] = {vmul(u, radius), vmul(vneg(u), radius), vmul(v, radius), vmul(vneg(v), radius)};
    for (int i = 0; i < 4; ++i)
        add_contact(A->pos, A->q, B->pos, B->q, cs, &count, mids, vadd(capA, offs[i]), vadd(capB, offs[i]),
                    0x06000000 | i);
    return count;
}

/* collideCylinders (collide.cpp:1093-1150) */
static int collide_cylinders(const Body *A, const Body *B, NewContact *cs, M3 *basis)
{
    V3 axA = qrotate(A->q, v3(0.0f, 0.0f, 1.0f));
    V3 axB = qrotate(B->q, v3(0.0f, 0.0f, 1.0f));
    float par = vdot(axA, axB);
    V3 delta = vsub(B->pos, A->pos);
    if (fabsf(par) > 0.95f)
    {
        float axial = vdot(delta, axA);
        V3 radial = vsub(delta, vmul(axA, axial));
        float rl2 = vlensq(radial);
        float rs = A->shapeRadius + B->shapeRadius;
        if (rl2 > rs * rs)
            return 0;
        float overlap = A->halfLength + B->halfLength - fabsf(axial);
        if (overlap < -COLLISION_MARGIN)
            return 0;
        if (fabsf(axial) > (A->halfLength + B->halfLength) * 0.5f)
        {
            float side = axial >= 0.0f ? 1.0f : -1.0f;
            V3 nAB = vmul(axA, side);
            V3 capA = vadd(A->pos, vmul(nAB, A->halfLength));
            V3 capB = vsub(B->pos, vmul(nAB, B->halfLength));
            return cylinder_caps(A, B, nAB, capA, capB, rmin(A->shapeRadius, B->shapeRadius) * 0.85f, cs, basis);
        }
        V3 nAB = rl2 > SAT_EPS ? vdiv(radial, sqrtf(rl2)) : orthonormal(axA).r[1];
        *basis = orthonormal(vneg(nAB));
        int count = 0;
        V3 mids[8];
        float vals[2] = {rmax(-A->halfLength, axial - B->halfLength), rmin(A->halfLength, axial + B->halfLength)};
        for (int i = 0; i < 2; ++i)
        {
            float tA = vals[i], tB = tA - axial;
            V3 xA = vadd(vadd(A->pos, vmul(axA, tA)), vmul(nAB, A->shapeRadius));
            V3 xB = vsub(vadd(B->pos, vmul(axA, tB)), vmul(nAB, B->shapeRadius));
            add_contact(A->pos, A->q, B->pos, B->q, cs, &count, mids, xA, xB, 0x06000100 | i);
        }
        return count;
    }
    V3 a0, a1, b0, b1, cA, cB;
    round_segment(A, &a0, &a1);
    round_segment(B, &b0, &b1);
    closest_segments(a0, a1, b0, b1, &cA, &cB);
    return round_contact(A, B, cA, A->shapeRadius, cB, B->shapeRadius, 0x06000200, cs, basis);
}

/* collideCylinderRound (collide.cpp:1065-1078) */
static int collide_cylinder_round(const Body *cyl, const Body *rb, int cylIsA, NewContact *cs, M3 *basis)
{
    V3 c0, c1, r0, r1, cc, cr;
    round_segment(cyl, &c0, &c1);
    round_segment(rb, &r0, &r1);
    closest_segments(c0, c1, r0, r1, &cc, &cr);
    if (cylIsA)
        return round_contact(cyl, rb, cc, cyl->shapeRadius, cr, rb->shapeRadius, 0x07000000, cs, basis);
    return round_contact(rb, cyl, cr, rb->shapeRadius, cc, cyl->shapeRadius, 0x07000000, cs, basis);
}

/* Manifold::collide (collide.cpp:1154-1176) */
static int collide_shapes(const Body *A, const Body *B, float dt, NewContact *cs, M3 *basis)
{
    if (is_cyl(A) && is_cyl(B))
        return collide_cylinders(A, B, cs, basis);
    if (is_cyl(A) && is_round(B))
        return collide_cylinder_round(A, B, 1, cs, basis);
    if (is_round(A) && is_cyl(B))
        return collide_cylinder_round(B, A, 0, cs, basis);
    if (is_cyl(A) && B->shape == ORACLE_SHAPE_BOX)
    {
        Obb o = make_obb(B->pos, B->q, B->size);
        int top = slab_top_cylinder(&o, A, B, 1, cs, basis);
        return top >= 0 ? top : collide_boxes(A->pos, A->q, A->size, B->pos, B->q, B->size, cs, basis);
    }
    if (A->shape == ORACLE_SHAPE_BOX && is_cyl(B))
    {
        Obb o = make_obb(A->pos, A->q, A->size);
        int top = slab_top_cylinder(&o, B, A, 0, cs, basis);
        return top >= 0 ? top : collide_boxes(A->pos, A->q, A->size, B->pos, B->q, B->size, cs, basis);
    }
    if (is_round(A) && is_round(B))
        return collide_round_round(A, B, cs, basis);
    if (is_round(A) && B->shape == ORACLE_SHAPE_BOX)
        return collide_round_box(A, B, 1, dt, cs, basis);
    if (A->shape == ORACLE_SHAPE_BOX && is_round(B))
        return collide_round_box(B, A, 0, dt, cs, basis);
    return collide_boxes(A->pos, A->q, A->size, B->pos, B->q, B->size, cs, basis);
}

/* contactOffsetWorld (manifold.cpp:28-91) */
static V3 contact_offset(const Body *b, V3 lo, M3 basis, int isA, int key)
{
    if (b->shape == ORACLE_SHAPE_SPHERE)
        return vmul(basis.r[0], isA ? -b->shapeRadius : b->shapeRadius);
    if (b->shape == ORACLE_SHAPE_CAPSULE)
    {
        V3 axis = qrotate(b->q, v3(0.0f, 0.0f, 1.0f));
        V3 n = basis.r[0];
        V3 nl = qrotate(qconj(b->q), n);
        float cz = isA ? lo.z + nl.z * b->shapeRadius : lo.z - nl.z * b->shapeRadius;
        cz = rclamp(cz, -b->halfLength, b->halfLength);
        return vadd(vmul(axis, cz), vmul(n, isA ? -b->shapeRadius : b->shapeRadius));
    }
    if (b->shape == ORACLE_SHAPE_CYLINDER)
    {
        V3 sw = vmul(basis.r[0], isA ? -1.0f : 1.0f);
        V3 sl = qrotate(qconj(b->q), sw);
        float stored = sqrtf(lo.x * lo.x + lo.y * lo.y);
        int cap = (key & 0xFFFFFF00) == 0x05000000 || (key & 0xFFFFFF00) == 0x06000000;
        if (cap)
        {
            V3 l = v3(0.0f, 0.0f, 0.0f);
            if (stored > 1.0e-6f)
            {
                l.x = lo.x / stored * b->shapeRadius;
                l.y = lo.y / stored * b->shapeRadius;
            }
            float capSign = fabsf(lo.z) > 1.0e-6f ? (lo.z >= 0.0f ? 1.0f : -1.0f) : (sl.z >= 0.0f ? 1.0f : -1.0f);
            l.z = b->halfLength * capSign;
            return qrotate(b->q, l);
        }
        float radialLen = sqrtf(sl.x * sl.x + sl.y * sl.y);
        float z = fabsf(sl.z) > 0.15f ? (sl.z >= 0.0f ? b->halfLength : -b->halfLength)
                                      : rclamp(lo.z, -b->halfLength, b->halfLength);
        V3 l = v3(0.0f, 0.0f, z);
        if (radialLen > 1.0e-6f)
        {
            l.x = sl.x / radialLen * b->shapeRadius;
            l.y = sl.y / radialLen * b->shapeRadius;
        }
        else if (stored > 1.0e-6f)
        {
            l.x = lo.x / stored * b->shapeRadius;
            l.y = lo.y / stored * b->shapeRadius;
        }
        return qrotate(b->q, l);
    }
    return qrotate(b->q, lo);
}

/* Manifold::initialize (manifold.cpp:100-174), boxes only */
static int manifold_init(OracleWorld *w, Manifold *m)
{
    const Body *A = &w->bodies[m->a], *B = &w->bodies[m->b];
    m->friction = sqrtf(A->friction * B->friction);
    if (A->shape == ORACLE_SHAPE_SPHERE || B->shape == ORACLE_SHAPE_SPHERE)
        m->friction = 0.0f;
    /* manifold.cpp:120-147: round manifolds (cylinders included) refresh their contact
     * locations and restart the tangential rows every step */
    int round = A->shape != ORACLE_SHAPE_BOX || B->shape != ORACLE_SHAPE_BOX;
    NewContact nc[8];
    memset(nc, 0, sizeof(nc));
    M3 basis = m->basis;
    int nn = collide_shapes(A, B, w->p.dt, nc, &basis);
    m->basis = basis;
    Contact merged[8];
    memset(merged, 0, sizeof(merged));
    for (int i = 0; i < nn; ++i)
    {
        merged[i].key = nc[i].key;
        merged[i].rA = nc[i].rA;
        merged[i].rB = nc[i].rB;
        m->srcSlot[i] = -1;
        for (int j = 0; j < m->n; ++j)
            if (nc[i].key == m->c[j].key)
            {
                merged[i] = m->c[j];
                m->srcSlot[i] = j;
                if (round || !m->c[j].stick)
                {
                    merged[i].rA = nc[i].rA;
                    merged[i].rB = nc[i].rB;
                }
                if (round)
                {
                    merged[i].lambda.y = 0.0f;
                    merged[i].lambda.z = 0.0f;
                    merged[i].penalty.y = PENALTY_MIN;
                    merged[i].penalty.z = PENALTY_MIN;
                    merged[i].stick = 0;
                }
                break;
            }
    }
    m->n = nn;
    for (int i = 0; i < nn; ++i)
        m->c[i] = merged[i];
    for (int i = 0; i < nn; ++i)
    {
        Contact *c = &m->c[i];
        V3 xA = vadd(A->pos, contact_offset(A, c->rA, m->basis, 1, c->key));
        V3 xB = vadd(B->pos, contact_offset(B, c->rB, m->basis, 0, c->key));
        c->C0 = vadd(mvmul(m->basis, vsub(xA, xB)), v3(COLLISION_MARGIN, 0, 0));
        c->lambda = vmul(vmul(c->lambda, w->p.alpha), w->p.gamma);
        V3 pg = vmul(c->penalty, w->p.gamma);
        unsigned char f = 0;
        for (int k = 0; k < 3; ++k)
        {
            if (VE(pg, k) > PENALTY_MAX)
                f |= (unsigned char)(ORACLE_IF_HI_X << k);
            else if (VE(pg, k) < PENALTY_MIN)
                f |= (unsigned char)(ORACLE_IF_LO_X << k);
        }
        m->iflags[i] = f;
        c->penalty = vclampf(pg, PENALTY_MIN, PENALTY_MAX);
    }
    return nn > 0;
}

/* Joint::initialize (joint.cpp:35-54) */
static int joint_init(OracleWorld *w, Joint *j)
{
    const Body *B = &w->bodies[j->b];
    V3 pa = j->a >= 0 ? xform(w->bodies[j->a].pos, w->bodies[j->a].q, j->rA) : j->rA;
    j->C0Lin = vsub(pa, xform(B->pos, B->q, j->rB));
    Q4 qa = j->a >= 0 ? w->bodies[j->a].q : q4(0, 0, 0, 1);
    j->C0Ang = vmul(qdiff(qa, B->q), j->torqueArm);
    j->lamLin = vmul(vmul(j->lamLin, w->p.alpha), w->p.gamma);
    j->lamAng = vmul(vmul(j->lamAng, w->p.alpha), w->p.gamma);
    j->penLin = vclampf(vmul(j->penLin, w->p.gamma), PENALTY_MIN, PENALTY_MAX);
    j->penAng = vclampf(vmul(j->penAng, w->p.gamma), PENALTY_MIN, PENALTY_MAX);
    j->penLin = vminf(j->penLin, j->stiffLin);
    j->penAng = vminf(j->penAng, j->stiffAng);
    return !j->broken;
}

/* ------------------------------------------------------------------------- */
/* Colouring                                                                 */
/* ------------------------------------------------------------------------- */

uint32_t oracle_colour_priority(uint32_t b)
{
    uint32_t h = b * 0x9E3779B1u + 0x7F4A7C15u;
    h ^= h >> 16;
    h *= 0x85EBCA6Bu;
    h ^= h >> 13;
    h *= 0xC2B2AE35u;
    h ^= h >> 16;
    return h;
}

static int prio_greater(uint32_t pv, int v, uint32_t pu, int u) { return pv > pu || (pv == pu && v > u); }

/* orderMode 1: lower list index first, which makes the result the sequential greedy
 * colouring in list order; orderMode 2: hashed priorities (fewer rounds). */
static uint32_t priority_of(const OracleWorld *w, int v)
{
    return w->p.orderMode == 2 ? oracle_colour_priority((uint32_t)v) : 0xFFFFFFFFu - (uint32_t)v;
}

static int is_vertex(const OracleWorld *w, int b) { return b >= 0 && w->bodies[b].mass > 0 && degree(w, b) > 0; }

static int other_end(const OracleWorld *w, const Incidence *e, int self)
{
    if (e->type == ORACLE_FORCE_IGNORE)
        return -1;
    int a, b;
    force_bodies(w, e, &a, &b);
    return a == self ? b : a;
}

/* Jones-Plassmann: in round r every uncoloured vertex whose (priority, index) beats all
 * uncoloured neighbours takes the smallest colour unused by neighbours coloured before r. */
static void colour_graph(OracleWorld *w)
{
    int n = w->n;
    int *round = (int *)malloc(sizeof(int) * (size_t)n);
    int remaining = 0;
    for (int b = 0; b < n; ++b)
    {
        w->colour[b] = -1;
        round[b] = is_vertex(w, b) ? -1 : -2;
        if (round[b] == -1)
            remaining++;
    }
    int *pick = (int *)malloc(sizeof(int) * (size_t)n);
    int nColours = 0;
    for (int r = 0; remaining > 0; ++r)
    {
        for (int v = 0; v < n; ++v)
        {
            pick[v] = -1;
            if (round[v] != -1)
                continue;
            uint32_t pv = priority_of(w, v);
            int isMax = 1;
            uint64_t used[4] = {0, 0, 0, 0};
            for (int k = w->adjStart[v]; k < w->adjStart[v + 1]; ++k)
            {
                int u = other_end(w, &w->inc[k], v);
                if (!is_vertex(w, u))
                    continue;
                if (round[u] == -1)
                {
                    if (!prio_greater(pv, v, priority_of(w, u), u))
                    {
                        isMax = 0;
                        break;
                    }
                }
                else if (w->colour[u] < 256)
                    used[w->colour[u] >> 6] |= 1ull << (w->colour[u] & 63);
            }
            if (!isMax)
                continue;
            int c = 0;
            while (c < 256 && (used[c >> 6] >> (c & 63)) & 1ull)
                c++;
            pick[v] = c;
        }
        for (int v = 0; v < n; ++v)
            if (pick[v] >= 0)
            {
                w->colour[v] = pick[v];
                round[v] = r;
                remaining--;
                if (pick[v] + 1 > nColours)
                    nColours = pick[v] + 1;
            }
    }
    w->nColours = nColours;
    w->nSolve = 0;
    for (int c = 0; c < nColours; ++c)
        for (int b = 0; b < n; ++b)
            if (w->colour[b] == c)
                w->solveOrder[w->nSolve++] = b;
    free(round);
    free(pick);
}

/* ------------------------------------------------------------------------- */
/* Step                                                                      */
/* ------------------------------------------------------------------------- */

static void tape_begin_step(OracleWorld *w);
static void tape_record_prepared(OracleWorld *w);

/* Broadphase (solver.cpp:1074-1083) and the new manifolds in hit order
 * (applyBroadphaseChunks, solver.cpp:220-248). */
static void run_broadphase(OracleWorld *w)
{
    PairList hits = {0, 0, 0};
    if (w->p.broadphase == 1)
        broadphase_grid(w, &hits);
    else if (w->p.broadphase == 2)
        broadphase_sap(w, &hits);
    else
        broadphase_all_pairs(w, &hits);
    if (w->nMan + hits.n > w->capMan)
    {
        while (w->nMan + hits.n > w->capMan)
            w->capMan = w->capMan ? w->capMan * 2 : 1024;
        w->man = (Manifold *)realloc(w->man, sizeof(Manifold) * (size_t)w->capMan);
    }
    for (int k = 0; k < hits.n; ++k)
    {
        Manifold *m = &w->man[w->nMan++];
        memset(m, 0, sizeof(*m));
        m->a = hits.v[k].a;
        m->b = hits.v[k].b;
        m->seq = w->nextSeq++;
        m->oldIndex = -1;
    }
    w->counters[3] = hits.n;
    free(hits.v);
}

/* Solver::benchmarkBroadphaseOnly (solver.cpp:989-1034): delete every manifold, run the
 * broadphase alone; the new manifolds keep no contacts until a step initialises them. */
int oracle_broadphase_only(OracleWorld *w)
{
    for (int k = 0; k < 9; ++k)
        w->counters[k] = 0;
    w->nMan = 0;
    build_adjacency(w);
    run_broadphase(w);
    build_adjacency(w);
    w->counters[4] = w->nMan;
    return 0;
}

int oracle_prepare(OracleWorld *w)
{
    for (int k = 0; k < 9; ++k)
        w->counters[k] = 0;
    if (w->recording)
        tape_begin_step(w);
    for (int i = 0; i < w->nMan; ++i)
        w->man[i].oldIndex = i;
    run_broadphase(w);

    /* force initialisation and removal of inactive forces (solver.cpp:1085-1132) */
    int keep = 0;
    for (int i = 0; i < w->nMan; ++i)
        if (manifold_init(w, &w->man[i]))
            w->man[keep++] = w->man[i];
    w->nMan = keep;
    keep = 0;
    for (int i = 0; i < w->nJoints; ++i)
        if (joint_init(w, &w->joints[i]))
            w->joints[keep++] = w->joints[i];
    w->nJoints = keep;
    build_adjacency(w);
    w->counters[4] = w->nMan;
    for (int i = 0; i < w->nMan; ++i)
        w->counters[5] += w->man[i].n;

    /* body warm start (solver.cpp:1134-1169) */
    float dt = w->p.dt, g = w->p.gravity;
    for (int b = 0; b < w->n; ++b)
    {
        Body *body = &w->bodies[b];
        body->inertLin = vadd(body->pos, vmul(body->vel, dt));
        if (body->mass > 0)
            body->inertLin = vadd(body->inertLin, vmul(v3(0, 0, g), dt * dt));
        body->inertAng = qstep(body->q, vmul(body->angvel, dt));
        V3 accel = vdiv(vsub(body->vel, body->prevVel), dt);
        float accelExt = accel.z * rsign(g);
        float accelRaw = accelExt / fabsf(g);
        float accelWeight = rclamp(accelRaw, 0.0f, 1.0f);
        if (!isfinite(accelWeight))
            accelWeight = 0.0f;
        if (w->recording)
        {
            unsigned char f = 0;
            if (body->mass > 0)
                f |= ORACLE_BF_DYNAMIC;
            if (degree(w, b) > 0)
                f |= ORACLE_BF_FORCES;
            if (isfinite(accelWeight) && accelRaw > 0.0f && accelRaw < 1.0f)
                f |= ORACLE_BF_ACCEL_IN;
            else if (accelWeight == 1.0f)
                f |= ORACLE_BF_ACCEL_ONE;
            w->tape[w->tapeSteps - 1].bodyFlags[b] = f;
        }
        body->initLin = body->pos;
        body->initAng = body->q;
        if (body->mass > 0)
        {
            body->pos = vadd(vadd(body->pos, vmul(body->vel, dt)), vmul(v3(0, 0, g), accelWeight * dt * dt));
            body->q = qstep(body->q, vmul(body->angvel, dt));
        }
        if (body->mass > 0 && degree(w, b) == 0)
        {
            body->pos = body->inertLin;
            body->q = body->inertAng;
        }
    }
    if (w->p.orderMode == 1 || w->p.orderMode == 2)
        colour_graph(w);
    else
    {
        w->nColours = 0;
        w->nSolve = 0;
        for (int b = 0; b < w->n; ++b)
        {
            w->colour[b] = -1;
            if (w->bodies[b].mass > 0 && degree(w, b) > 0)
                w->solveOrder[w->nSolve++] = b;
        }
    }
    w->counters[7] = w->nSolve;
    w->counters[8] = w->nColours;
    if (w->recording)
        tape_record_prepared(w);
    return 0;
}

typedef struct
{
    M3 lhsLin, lhsAng, lhsCross;
    V3 rhsLin, rhsAng;
} System;

/* Manifold::updatePrimal (manifold.cpp:176-229) */
static void manifold_primal(const OracleWorld *w, const Manifold *m, int bodyIsA, float alpha, System *s)
{
    const Body *A = &w->bodies[m->a], *B = &w->bodies[m->b];
    V3 dqALin = vsub(A->pos, A->initLin);
    V3 dqAAng = qdiff(A->q, A->initAng);
    V3 dqBLin = vsub(B->pos, B->initLin);
    V3 dqBAng = qdiff(B->q, B->initAng);
    for (int i = 0; i < m->n; ++i)
    {
        const Contact *c = &m->c[i];
        V3 rAW = contact_offset(A, c->rA, m->basis, 1, c->key);
        V3 rBW = contact_offset(B, c->rB, m->basis, 0, c->key);
        M3 jALin = m->basis;
        M3 jBLin = mneg(m->basis);
        M3 jAAng = m3rows(vcross(rAW, jALin.r[0]), vcross(rAW, jALin.r[1]), vcross(rAW, jALin.r[2]));
        M3 jBAng = m3rows(vcross(rBW, jBLin.r[0]), vcross(rBW, jBLin.r[1]), vcross(rBW, jBLin.r[2]));
        M3 K = mdiag(c->penalty.x, c->penalty.y, c->penalty.z);
        V3 C = vadd(vadd(vadd(vadd(vmul(c->C0, 1 - alpha), mvmul(jALin, dqALin)), mvmul(jBLin, dqBLin)),
                         mvmul(jAAng, dqAAng)),
                    mvmul(jBAng, dqBAng));
        V3 F = vadd(mvmul(K, C), c->lambda);
        unsigned short flags = F.x < 0.0f ? 0 : ORACLE_EF_NCLAMP;
        F.x = rmin(F.x, 0.0f);
        float bounds = fabsf(F.x) * m->friction;
        float fs = sqrtf(F.y * F.y + F.z * F.z);
        if (fs > bounds && fs > 0)
        {
            F.y *= bounds / fs;
            F.z *= bounds / fs;
            flags |= ORACLE_EF_CONE;
        }
        if (w->recording)
        {
            const OracleTapeStep *t = &w->tape[w->tapeSteps - 1];
            size_t slot = (size_t)(m - w->man) * 8 + (size_t)i;
            t->flags[((size_t)w->curIter * (size_t)t->nMan * 8 + slot) * 3 + (bodyIsA ? 0 : 1)] = flags;
        }
        M3 jLin = bodyIsA ? jALin : jBLin;
        M3 jAng = bodyIsA ? jAAng : jBAng;
        M3 jLinT = mtrans(jLin), jAngT = mtrans(jAng);
        M3 jAngTk = mmul(jAngT, K);
        s->lhsLin = madd(s->lhsLin, mmul(mmul(jLinT, K), jLin));
        s->lhsAng = madd(s->lhsAng, mmul(jAngTk, jAng));
        s->lhsCross = madd(s->lhsCross, mmul(jAngTk, jLin));
        s->rhsLin = vadd(s->rhsLin, mvmul(jLinT, F));
        s->rhsAng = vadd(s->rhsAng, mvmul(jAngT, F));
    }
}

static M3 gs_ball_socket(int k, V3 v)
{
    float vk = VE(v, k);
    M3 m = mdiag(-vk, -vk, -vk);
    VE(m.r[0], k) += v.x;
    VE(m.r[1], k) += v.y;
    VE(m.r[2], k) += v.z;
    return m;
}

static const M3 M_IDENT = {{{1, 0, 0}, {0, 1, 0}, {0, 0, 1}}};
static const M3 M_NIDENT = {{{-1, 0, 0}, {0, -1, 0}, {0, 0, -1}}};

/* Joint::updatePrimal (joint.cpp:56-123) */
static void joint_primal(const OracleWorld *w, const Joint *j, int bodyIsA, float alpha, System *s)
{
    const Body *B = &w->bodies[j->b];
    const Body *A = j->a >= 0 ? &w->bodies[j->a] : NULL;
    if (vlensq(j->penLin) > 0)
    {
        V3 rAW = A ? qrotate(A->q, j->rA) : v3(0, 0, 0);
        V3 rBW = qrotate(B->q, j->rB);
        M3 K = mdiag(j->penLin.x, j->penLin.y, j->penLin.z);
        V3 C = vsub(A ? vadd(A->pos, rAW) : j->rA, vadd(B->pos, rBW));
        if (isinf(j->stiffLin))
            C = vsub(C, vmul(j->C0Lin, alpha));
        V3 F = vadd(mvmul(K, C), j->lamLin);
        M3 jLin = bodyIsA ? M_IDENT : M_NIDENT;
        M3 jAng = bodyIsA ? mskew(vneg(rAW)) : mskew(rBW);
        M3 jLinT = mtrans(jLin), jAngT = mtrans(jAng);
        M3 jAngTk = mmul(jAngT, K);
        s->lhsLin = madd(s->lhsLin, mmul(mmul(jLinT, K), jLin));
        s->lhsAng = madd(s->lhsAng, mmul(jAngTk, jAng));
        s->lhsCross = madd(s->lhsCross, mmul(jAngTk, jLin));
        V3 r = bodyIsA ? rAW : vneg(rBW);
        M3 H = madd(madd(mscale(gs_ball_socket(0, r), F.x), mscale(gs_ball_socket(1, r), F.y)),
                    mscale(gs_ball_socket(2, r), F.z));
        s->lhsAng = madd(s->lhsAng, mdiagonalize(H));
        s->rhsLin = vadd(s->rhsLin, mvmul(jLinT, F));
        s->rhsAng = vadd(s->rhsAng, mvmul(jAngT, F));
    }
    if (vlensq(j->penAng) > 0)
    {
        M3 K = mdiag(j->penAng.x, j->penAng.y, j->penAng.z);
        V3 C = vmul(qdiff(A ? A->q : q4(0, 0, 0, 1), B->q), j->torqueArm);
        if (isinf(j->stiffAng))
            C = vsub(C, vmul(j->C0Ang, alpha));
        V3 F = vadd(mvmul(K, C), j->lamAng);
        M3 jAng = mscale(bodyIsA ? M_IDENT : M_NIDENT, j->torqueArm);
        s->lhsAng = madd(s->lhsAng, mmul(mmul(mtrans(jAng), K), jAng));
        s->rhsAng = vadd(s->rhsAng, mvmul(mtrans(jAng), F));
    }
}

/* Spring::updatePrimal (spring.cpp:27-69) */
static void spring_primal(const OracleWorld *w, const Spring *sp, int bodyIsA, System *s)
{
    const Body *A = &w->bodies[sp->a], *B = &w->bodies[sp->b];
    V3 pA = xform(A->pos, A->q, sp->rA);
    V3 pB = xform(B->pos, B->q, sp->rB);
    V3 d = vsub(pA, pB);
    float dLen = vlen(d);
    if (dLen <= 1.0e-6f)
        return;
    V3 n = vdiv(d, dLen);
    float C = dLen - sp->rest;
    float f = sp->stiffness * C;
    V3 jLin, jAng;
    if (bodyIsA)
    {
        V3 rW = qrotate(A->q, sp->rA);
        jLin = n;
        jAng = vcross(rW, n);
    }
    else
    {
        V3 rW = qrotate(B->q, sp->rB);
        jLin = vneg(n);
        jAng = vneg(vcross(rW, n));
    }
    V3 F = vmul(jLin, f);
    V3 Tau = vmul(jAng, f);
    s->lhsLin = madd(s->lhsLin, mscale(mouter(jLin, jLin), sp->stiffness));
    s->lhsAng = madd(s->lhsAng, mscale(mouter(jAng, jAng), sp->stiffness));
    s->lhsCross = madd(s->lhsCross, mscale(mouter(jAng, jLin), sp->stiffness));
    s->rhsLin = vadd(s->rhsLin, F);
    s->rhsAng = vadd(s->rhsAng, Tau);
}

static void body_primal(OracleWorld *w, int b)
{
    Body *body = &w->bodies[b];
    float dt = w->p.dt, alpha = w->p.alpha;
    M3 MLin = mdiag(body->mass, body->mass, body->mass);
    M3 MAng = mdiag(body->moment.x, body->moment.y, body->moment.z);
    System s;
    s.lhsLin = mdivs(MLin, dt * dt);
    s.lhsAng = mdivs(MAng, dt * dt);
    s.lhsCross = mdiag(0, 0, 0);
    s.rhsLin = mvmul(mdivs(MLin, dt * dt), vsub(body->pos, body->inertLin));
    s.rhsAng = mvmul(mdivs(MAng, dt * dt), qdiff(body->q, body->inertAng));
    for (int k = w->adjStart[b]; k < w->adjStart[b + 1]; ++k)
    {
        const Incidence *e = &w->inc[k];
        w->counters[6]++;
        if (e->type == ORACLE_FORCE_MANIFOLD)
            manifold_primal(w, &w->man[e->index], e->isA, alpha, &s);
        else if (e->type == ORACLE_FORCE_JOINT)
            joint_primal(w, &w->joints[e->index], e->isA, alpha, &s);
        else if (e->type == ORACLE_FORCE_SPRING)
            spring_primal(w, &w->springs[e->index], e->isA, &s);
    }
    V3 dxLin, dxAng;
    ldl_solve6(s.lhsLin, s.lhsAng, s.lhsCross, vneg(s.rhsLin), vneg(s.rhsAng), &dxLin, &dxAng);
    body->pos = vadd(body->pos, dxLin);
    body->q = qstep(body->q, dxAng);
}

/* Manifold::updateDual (manifold.cpp:231-280) */
static void manifold_dual(OracleWorld *w, Manifold *m, float alpha)
{
    const Body *A = &w->bodies[m->a], *B = &w->bodies[m->b];
    V3 dqALin = vsub(A->pos, A->initLin);
    V3 dqAAng = qdiff(A->q, A->initAng);
    V3 dqBLin = vsub(B->pos, B->initLin);
    V3 dqBAng = qdiff(B->q, B->initAng);
    for (int i = 0; i < m->n; ++i)
    {
        Contact *c = &m->c[i];
        V3 rAW = contact_offset(A, c->rA, m->basis, 1, c->key);
        V3 rBW = contact_offset(B, c->rB, m->basis, 0, c->key);
        M3 jALin = m->basis;
        M3 jBLin = mneg(m->basis);
        M3 jAAng = m3rows(vcross(rAW, jALin.r[0]), vcross(rAW, jALin.r[1]), vcross(rAW, jALin.r[2]));
        M3 jBAng = m3rows(vcross(rBW, jBLin.r[0]), vcross(rBW, jBLin.r[1]), vcross(rBW, jBLin.r[2]));
        M3 K = mdiag(c->penalty.x, c->penalty.y, c->penalty.z);
        V3 C = vadd(vadd(vadd(vadd(vmul(c->C0, 1 - alpha), mvmul(jALin, dqALin)), mvmul(jBLin, dqBLin)),
                         mvmul(jAAng, dqAAng)),
                    mvmul(jBAng, dqBAng));
        V3 F = vadd(mvmul(K, C), c->lambda);
        unsigned short flags = F.x < 0.0f ? 0 : ORACLE_EF_NCLAMP;
        F.x = rmin(F.x, 0.0f);
        float bounds = fabsf(F.x) * m->friction;
        float fs = sqrtf(F.y * F.y + F.z * F.z);
        if (fs > bounds && fs > 0)
        {
            F.y *= bounds / fs;
            F.z *= bounds / fs;
            flags |= ORACLE_EF_CONE;
        }
        if (w->recording)
        {
            if (fs <= bounds)
                flags |= ORACLE_EF_RAMP_T;
            for (int k = 0; k < 3; ++k)
            {
                float ck = VE(C, k);
                if (ck < 0)
                    flags |= (unsigned short)(ORACLE_EF_NEG_X << k);
                else if (ck > 0)
                    flags |= (unsigned short)(ORACLE_EF_POS_X << k);
                int ramps = k == 0 ? F.x < 0 : fs <= bounds;
                if (ramps && !(VE(c->penalty, k) + w->p.betaLin * fabsf(ck) < PENALTY_MAX))
                    flags |= (unsigned short)(ORACLE_EF_CAP_X << k);
            }
            const OracleTapeStep *t = &w->tape[w->tapeSteps - 1];
            size_t slot = (size_t)(m - w->man) * 8 + (size_t)i;
            t->flags[((size_t)w->curIter * (size_t)t->nMan * 8 + slot) * 3 + 2] = flags;
        }
        c->lambda = F;
        if (F.x < 0)
            c->penalty.x = rmin(c->penalty.x + w->p.betaLin * fabsf(C.x), PENALTY_MAX);
        if (fs <= bounds)
        {
            c->penalty.y = rmin(c->penalty.y + w->p.betaLin * fabsf(C.y), PENALTY_MAX);
            c->penalty.z = rmin(c->penalty.z + w->p.betaLin * fabsf(C.z), PENALTY_MAX);
            c->stick = sqrtf(C.y * C.y + C.z * C.z) < STICK_THRESH;
        }
    }
}

/* Joint::updateDual (joint.cpp:125-182) */
static void joint_dual(OracleWorld *w, Joint *j, float alpha)
{
    const Body *B = &w->bodies[j->b];
    const Body *A = j->a >= 0 ? &w->bodies[j->a] : NULL;
    if (vlensq(j->penLin) > 0)
    {
        M3 K = mdiag(j->penLin.x, j->penLin.y, j->penLin.z);
        V3 C = vsub(A ? xform(A->pos, A->q, j->rA) : j->rA, xform(B->pos, B->q, j->rB));
        if (isinf(j->stiffLin))
        {
            C = vsub(C, vmul(j->C0Lin, alpha));
            j->lamLin = vadd(mvmul(K, C), j->lamLin);
        }
        j->penLin = vminf(vadd(j->penLin, vmul(vabs(C), w->p.betaLin)), rmin(j->stiffLin, PENALTY_MAX));
    }
    if (vlensq(j->penAng) > 0)
    {
        M3 K = mdiag(j->penAng.x, j->penAng.y, j->penAng.z);
        V3 C = vmul(qdiff(A ? A->q : q4(0, 0, 0, 1), B->q), j->torqueArm);
        if (isinf(j->stiffAng))
        {
            C = vsub(C, vmul(j->C0Ang, alpha));
            j->lamAng = vadd(mvmul(K, C), j->lamAng);
        }
        j->penAng = vminf(vadd(j->penAng, vmul(vabs(C), w->p.betaAng)), rmin(j->stiffAng, PENALTY_MAX));
    }
    if (vlensq(j->lamAng) > j->fracture * j->fracture)
    {
        j->penLin = v3(0, 0, 0);
        j->penAng = v3(0, 0, 0);
        j->lamLin = v3(0, 0, 0);
        j->lamAng = v3(0, 0, 0);
        j->broken = 1;
    }
}

int oracle_iterate(OracleWorld *w)
{
    for (int it = 0; it < w->p.iterations; ++it)
    {
        w->curIter = it;
        for (int k = 0; k < w->nSolve; ++k)
            body_primal(w, w->solveOrder[k]);
        for (int i = 0; i < w->nMan; ++i)
            manifold_dual(w, &w->man[i], w->p.alpha);
        for (int i = 0; i < w->nJoints; ++i)
            joint_dual(w, &w->joints[i], w->p.alpha);
    }
    return 0;
}

int oracle_finish(OracleWorld *w)
{
    float dt = w->p.dt;
    for (int b = 0; b < w->n; ++b)
    {
        Body *body = &w->bodies[b];
        body->prevVel = body->vel;
        if (body->mass > 0)
        {
            body->vel = vdiv(vsub(body->pos, body->initLin), dt);
            body->angvel = vdiv(qdiff(body->q, body->initAng), dt);
        }
    }
    /* applySphereRollingFriction (solver.cpp:628-662) over the manifolds in the solver's
     * force order (newest first) */
    for (int k = w->nMan - 1; k >= 0; --k)
    {
        const Manifold *m = &w->man[k];
        Body *A = &w->bodies[m->a], *B = &w->bodies[m->b];
        Body *sphere = A->shape == ORACLE_SHAPE_SPHERE ? A : (B->shape == ORACLE_SHAPE_SPHERE ? B : NULL);
        Body *other = sphere == A ? B : A;
        if (!sphere || sphere->mass <= 0.0f || other->mass > 0.0f || m->n <= 0)
            continue;
        float mf = sqrtf(sphere->friction * other->friction);
        if (mf <= 0.0f)
            continue;
        float blend = rclamp(mf * 0.08f, 0.0f, 0.18f);
        for (int i = 0; i < m->n; ++i)
        {
            V3 n = sphere == A ? m->basis.r[0] : vneg(m->basis.r[0]);
            V3 r = vmul(vneg(n), sphere->shapeRadius);
            V3 cv = vadd(sphere->vel, vcross(sphere->angvel, r));
            V3 tv = vsub(cv, vmul(n, vdot(cv, n)));
            sphere->vel = vsub(sphere->vel, vmul(tv, blend));
            V3 desired = vdiv(vcross(n, sphere->vel), sphere->shapeRadius);
            sphere->angvel = vadd(sphere->angvel, vmul(vsub(desired, sphere->angvel), blend));
        }
    }
    return 0;
}

int oracle_step(OracleWorld *w, int nsteps)
{
    for (int s = 0; s < nsteps; ++s)
    {
        oracle_prepare(w);
        oracle_iterate(w);
        oracle_finish(w);
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Construction and queries                                                  */
/* ------------------------------------------------------------------------- */

/* Joint constructor (joint.cpp:25-33): the newest force, zero penalty and lambda. */
static Joint *new_joint(OracleWorld *w, int a, int b, V3 rA, V3 rB, float stiffLin, float stiffAng, float fracture)
{
    w->joints = (Joint *)realloc(w->joints, sizeof(Joint) * (size_t)(w->nJoints + 1));
    Joint *j = &w->joints[w->nJoints++];
    memset(j, 0, sizeof(*j));
    j->a = a;
    j->b = b;
    j->seq = w->nextSeq++;
    j->rA = rA;
    j->rB = rB;
    j->stiffLin = stiffLin;
    j->stiffAng = stiffAng;
    j->fracture = fracture;
    V3 sa = a >= 0 ? w->bodies[a].size : v3(0, 0, 0);
    j->torqueArm = vlensq(vadd(sa, w->bodies[b].size));
    return j;
}

static Joint *joint_by_seq(OracleWorld *w, int64_t seq)
{
    for (int i = 0; i < w->nJoints; ++i)
        if (w->joints[i].seq == seq)
            return &w->joints[i];
    return NULL;
}

int64_t oracle_add_joint(OracleWorld *w, int a, int b, const float *rA3, const float *rB3, float stiffLin,
                         float stiffAng, float fracture)
{
    if (b < 0 || b >= w->n || a >= w->n || a < -1 || a == b)
        return -1;
    Joint *j = new_joint(w, a, b, v3(rA3[0], rA3[1], rA3[2]), v3(rB3[0], rB3[1], rB3[2]), stiffLin, stiffAng,
                         fracture);
    build_adjacency(w);
    return j->seq;
}

int oracle_set_joint_anchor(OracleWorld *w, int64_t seq, const float *rA3)
{
    Joint *j = joint_by_seq(w, seq);
    if (!j)
        return -1;
    j->rA = v3(rA3[0], rA3[1], rA3[2]);
    return 0;
}

int oracle_remove_joint(OracleWorld *w, int64_t seq)
{
    int keep = 0, found = 0;
    for (int i = 0; i < w->nJoints; ++i)
    {
        if (w->joints[i].seq == seq)
        {
            found = 1;
            continue;
        }
        w->joints[keep++] = w->joints[i];
    }
    w->nJoints = keep;
    build_adjacency(w);
    return found ? 0 : -1;
}

OracleWorld *oracle_create(const OracleParams *params, int nBodies, const float *size3, const float *density,
                           const float *friction, const float *pos3, const float *vel3, const float *quat4,
                           int nForces, const int *ftype, const int *fa, const int *fb, const float *frA3,
                           const float *frB3, const float *fparam3)
{
    return oracle_create_shapes(params, nBodies, NULL, NULL, size3, density, friction, pos3, vel3, quat4, nForces,
                                ftype, fa, fb, frA3, frB3, fparam3);
}

/* sphereMass (rigid.cpp:18-21); PI as rigid.cpp:16 */
#define RIGID_PI 3.14159265358979323846f
static float sphere_mass(float r, float density) { return 4.0f / 3.0f * RIGID_PI * r * r * r * density; }

/* Rigid::makeSphere / makeCapsule / makeCylinder (rigid.cpp:44-90): the shape, the
 * constructor's size, then mass, moment and bounding radius. */
static void round_body(Body *b, int shape, float r, float h, float density)
{
    float d = r * 2.0f;
    b->shape = shape;
    b->shapeRadius = r;
    if (shape == ORACLE_SHAPE_SPHERE)
    {
        b->size = v3(d, d, d);
        b->halfLength = 0.0f;
        b->mass = sphere_mass(r, density);
        float inertia = 2.0f / 5.0f * b->mass * r * r;
        b->moment = v3(inertia, inertia, inertia);
        b->radius = r;
    }
    else if (shape == ORACLE_SHAPE_CAPSULE)
    {
        float cylLen = h * 2.0f;
        b->size = v3(d, d, cylLen + d);
        b->halfLength = h;
        float cylMass = RIGID_PI * r * r * cylLen * density;
        float capMass = sphere_mass(r, density);
        b->mass = cylMass + capMass;
        float axial = 0.5f * cylMass * r * r + 2.0f / 5.0f * capMass * r * r;
        float trans = (3.0f * r * r + cylLen * cylLen) / 12.0f * cylMass + 2.0f / 5.0f * capMass * r * r +
                      capMass * h * h;
        b->moment = v3(trans, trans, axial);
        b->radius = h + r;
    }
    else
    {
        float height = h * 2.0f;
        b->size = v3(d, d, height);
        b->halfLength = h;
        b->mass = RIGID_PI * r * r * height * density;
        float axial = 0.5f * b->mass * r * r;
        float trans = (3.0f * r * r + height * height) / 12.0f * b->mass;
        b->moment = v3(trans, trans, axial);
        b->radius = sqrtf(r * r + h * h);
    }
}

OracleWorld *oracle_create_shapes(const OracleParams *params, int nBodies, const int *shape, const float *dim2,
                                  const float *size3, const float *density, const float *friction,
                                  const float *pos3, const float *vel3, const float *quat4, int nForces,
                                  const int *ftype, const int *fa, const int *fb, const float *frA3,
                                  const float *frB3, const float *fparam3)
{
    OracleWorld *w = (OracleWorld *)calloc(1, sizeof(OracleWorld));
    w->p = *params;
    w->n = nBodies;
    w->bodies = (Body *)calloc((size_t)(nBodies > 0 ? nBodies : 1), sizeof(Body));
    w->adjStart = (int *)calloc((size_t)nBodies + 1, sizeof(int));
    w->colour = (int *)calloc((size_t)(nBodies > 0 ? nBodies : 1), sizeof(int));
    w->solveOrder = (int *)calloc((size_t)(nBodies > 0 ? nBodies : 1), sizeof(int));
    /* Rigid constructor (rigid.cpp:24-42); list index = nBodies - 1 - creation index */
    for (int c = 0; c < nBodies; ++c)
    {
        Body *b = &w->bodies[nBodies - 1 - c];
        V3 size = v3(size3[3 * c], size3[3 * c + 1], size3[3 * c + 2]);
        b->pos = v3(pos3[3 * c], pos3[3 * c + 1], pos3[3 * c + 2]);
        b->q = q4(quat4[4 * c], quat4[4 * c + 1], quat4[4 * c + 2], quat4[4 * c + 3]);
        b->vel = v3(vel3[3 * c], vel3[3 * c + 1], vel3[3 * c + 2]);
        b->angvel = v3(0, 0, 0);
        b->prevVel = b->vel;
        b->size = size;
        b->friction = friction[c];
        b->mass = size.x * size.y * size.z * density[c];
        b->moment = v3((size.y * size.y + size.z * size.z) / 12.0f * b->mass,
                       (size.x * size.x + size.z * size.z) / 12.0f * b->mass,
                       (size.x * size.x + size.y * size.y) / 12.0f * b->mass);
        b->radius = vlen(vmul(size, 0.5f));
        b->shape = ORACLE_SHAPE_BOX;
        b->shapeRadius = b->radius;
        b->halfLength = 0.0f;
        if (shape && shape[c] != ORACLE_SHAPE_BOX)
            round_body(b, shape[c], dim2[2 * c], dim2[2 * c + 1], density[c]);
    }
    for (int k = 0; k < nForces; ++k)
    {
        int a = fa[k] >= 0 ? nBodies - 1 - fa[k] : -1;
        int b = nBodies - 1 - fb[k];
        V3 rA = v3(frA3[3 * k], frA3[3 * k + 1], frA3[3 * k + 2]);
        V3 rB = v3(frB3[3 * k], frB3[3 * k + 1], frB3[3 * k + 2]);
        if (ftype[k] == ORACLE_FORCE_JOINT)
        {
            new_joint(w, a, b, rA, rB, fparam3[3 * k], fparam3[3 * k + 1], fparam3[3 * k + 2]);
            continue;
        }
        int64_t seq = w->nextSeq++;
        if (ftype[k] == ORACLE_FORCE_SPRING)
        {
            w->springs = (Spring *)realloc(w->springs, sizeof(Spring) * (size_t)(w->nSprings + 1));
            Spring *s = &w->springs[w->nSprings++];
            s->a = a;
            s->b = b;
            s->seq = seq;
            s->rA = rA;
            s->rB = rB;
            s->stiffness = fparam3[3 * k];
            s->rest = fparam3[3 * k + 1];
            /* spring.cpp:14-25 */
            if (s->rest < 0.0f)
            {
                V3 pA = xform(w->bodies[a].pos, w->bodies[a].q, rA);
                V3 pB = xform(w->bodies[b].pos, w->bodies[b].q, rB);
                s->rest = vlen(vsub(pA, pB));
            }
        }
        else
        {
            w->ignores = (Ignore *)realloc(w->ignores, sizeof(Ignore) * (size_t)(w->nIgnores + 1));
            Ignore *g = &w->ignores[w->nIgnores++];
            g->a = a;
            g->b = b;
            g->seq = seq;
        }
    }
    build_adjacency(w);
    return w;
}

void oracle_destroy(OracleWorld *w)
{
    if (!w)
        return;
    oracle_tape_end(w);
    free(w->bodies);
    free(w->man);
    free(w->joints);
    free(w->springs);
    free(w->ignores);
    free(w->inc);
    free(w->adjStart);
    free(w->colour);
    free(w->solveOrder);
    free(w);
}

void oracle_set_params(OracleWorld *w, const OracleParams *params) { w->p = *params; }

int oracle_num_bodies(const OracleWorld *w) { return w->n; }

void oracle_get_bodies(const OracleWorld *w, float *pos3, float *quat4, float *vel3, float *angvel3, float *prevvel3)
{
    for (int b = 0; b < w->n; ++b)
    {
        const Body *x = &w->bodies[b];
        if (pos3)
            memcpy(pos3 + 3 * b, &x->pos, 12);
        if (quat4)
            memcpy(quat4 + 4 * b, &x->q, 16);
        if (vel3)
            memcpy(vel3 + 3 * b, &x->vel, 12);
        if (angvel3)
            memcpy(angvel3 + 3 * b, &x->angvel, 12);
        if (prevvel3)
            memcpy(prevvel3 + 3 * b, &x->prevVel, 12);
    }
}

void oracle_get_body_aux(const OracleWorld *w, float *initLin3, float *initAng4, float *inertLin3, float *inertAng4)
{
    for (int b = 0; b < w->n; ++b)
    {
        const Body *x = &w->bodies[b];
        if (initLin3)
            memcpy(initLin3 + 3 * b, &x->initLin, 12);
        if (initAng4)
            memcpy(initAng4 + 4 * b, &x->initAng, 16);
        if (inertLin3)
            memcpy(inertLin3 + 3 * b, &x->inertLin, 12);
        if (inertAng4)
            memcpy(inertAng4 + 4 * b, &x->inertAng, 16);
    }
}

void oracle_get_body_props(const OracleWorld *w, float *mass, float *moment3, float *radius, float *size3,
                           float *friction)
{
    for (int b = 0; b < w->n; ++b)
    {
        const Body *x = &w->bodies[b];
        if (mass)
            mass[b] = x->mass;
        if (moment3)
            memcpy(moment3 + 3 * b, &x->moment, 12);
        if (radius)
            radius[b] = x->radius;
        if (size3)
            memcpy(size3 + 3 * b, &x->size, 12);
        if (friction)
            friction[b] = x->friction;
    }
}

void oracle_set_bodies(OracleWorld *w, const float *pos3, const float *quat4, const float *vel3,
                       const float *angvel3, const float *prevvel3)
{
    for (int b = 0; b < w->n; ++b)
    {
        Body *x = &w->bodies[b];
        if (pos3)
            memcpy(&x->pos, pos3 + 3 * b, 12);
        if (quat4)
            memcpy(&x->q, quat4 + 4 * b, 16);
        if (vel3)
            memcpy(&x->vel, vel3 + 3 * b, 12);
        if (angvel3)
            memcpy(&x->angvel, angvel3 + 3 * b, 12);
        if (prevvel3)
            memcpy(&x->prevVel, prevvel3 + 3 * b, 12);
    }
}

int oracle_num_manifolds(const OracleWorld *w) { return w->nMan; }

void oracle_get_manifolds(const OracleWorld *w, int *ab2, int64_t *seq, int *ncontacts, float *basis9,
                          float *friction, int *keys8, float *contact15x8, int *stick8)
{
    for (int i = 0; i < w->nMan; ++i)
    {
        const Manifold *m = &w->man[i];
        if (ab2)
        {
            ab2[2 * i] = m->a;
            ab2[2 * i + 1] = m->b;
        }
        if (seq)
            seq[i] = m->seq;
        if (ncontacts)
            ncontacts[i] = m->n;
        if (basis9)
            memcpy(basis9 + 9 * i, &m->basis, 36);
        if (friction)
            friction[i] = m->friction;
        for (int k = 0; k < 8; ++k)
        {
            const Contact *c = &m->c[k];
            int live = k < m->n;
            if (keys8)
                keys8[8 * i + k] = live ? c->key : 0;
            if (stick8)
                stick8[8 * i + k] = live ? c->stick : 0;
            if (contact15x8)
            {
                float *o = contact15x8 + (size_t)(8 * i + k) * 15;
                if (live)
                {
                    memcpy(o, &c->rA, 12);
                    memcpy(o + 3, &c->rB, 12);
                    memcpy(o + 6, &c->C0, 12);
                    memcpy(o + 9, &c->penalty, 12);
                    memcpy(o + 12, &c->lambda, 12);
                }
                else
                    memset(o, 0, 60);
            }
        }
    }
}

int oracle_num_joints(const OracleWorld *w) { return w->nJoints; }

void oracle_get_joints(const OracleWorld *w, int *ab2, float *state18, int *broken)
{
    for (int i = 0; i < w->nJoints; ++i)
    {
        const Joint *j = &w->joints[i];
        if (ab2)
        {
            ab2[2 * i] = j->a;
            ab2[2 * i + 1] = j->b;
        }
        if (state18)
        {
            float *o = state18 + 18 * i;
            memcpy(o, &j->C0Lin, 12);
            memcpy(o + 3, &j->C0Ang, 12);
            memcpy(o + 6, &j->penLin, 12);
            memcpy(o + 9, &j->penAng, 12);
            memcpy(o + 12, &j->lamLin, 12);
            memcpy(o + 15, &j->lamAng, 12);
        }
        if (broken)
            broken[i] = j->broken;
    }
}

void oracle_get_colours(const OracleWorld *w, int *colour, int *nColours)
{
    if (colour)
        memcpy(colour, w->colour, sizeof(int) * (size_t)w->n);
    if (nColours)
        *nColours = w->nColours;
}

int oracle_get_solve_order(const OracleWorld *w, int *order)
{
    if (order)
        memcpy(order, w->solveOrder, sizeof(int) * (size_t)w->nSolve);
    return w->nSolve;
}

void oracle_get_counters(const OracleWorld *w, int64_t *out9) { memcpy(out9, w->counters, sizeof(w->counters)); }

int oracle_collide_boxes(const float *posA3, const float *quatA4, const float *sizeA3, const float *posB3,
                         const float *quatB4, const float *sizeB3, int *keys8, float *rA3x8, float *rB3x8,
                         float *basis9)
{
    NewContact nc[8];
    memset(nc, 0, sizeof(nc));
    M3 basis;
    memset(&basis, 0, sizeof(basis));
    int n = collide_boxes(v3(posA3[0], posA3[1], posA3[2]), q4(quatA4[0], quatA4[1], quatA4[2], quatA4[3]),
                          v3(sizeA3[0], sizeA3[1], sizeA3[2]), v3(posB3[0], posB3[1], posB3[2]),
                          q4(quatB4[0], quatB4[1], quatB4[2], quatB4[3]), v3(sizeB3[0], sizeB3[1], sizeB3[2]), nc,
                          &basis);
    for (int i = 0; i < 8; ++i)
    {
        keys8[i] = i < n ? nc[i].key : 0;
        memcpy(rA3x8 + 3 * i, i < n ? &nc[i].rA : &(V3){0, 0, 0}, 12);
        memcpy(rB3x8 + 3 * i, i < n ? &nc[i].rB : &(V3){0, 0, 0}, 12);
    }
    memcpy(basis9, &basis, 36);
    return n;
}

void oracle_get_params(const OracleWorld *w, OracleParams *out) { *out = w->p; }

/* ------------------------------------------------------------------------- */
/* Frozen-branch tape                                                        */
/* ------------------------------------------------------------------------- */

static void tape_free_step(OracleTapeStep *t)
{
    free(t->bodyIn);
    free(t->bodyFlags);
    free(t->ab);
    free(t->basis);
    free(t->friction);
    free(t->ncontacts);
    free(t->keys);
    free(t->geo);
    free(t->init);
    free(t->src);
    free(t->initFlags);
    free(t->solveOrder);
    free(t->colourStart);
    free(t->flags);
    memset(t, 0, sizeof(*t));
}

int oracle_tape_begin(OracleWorld *w)
{
    oracle_tape_end(w);
    if (w->nJoints > 0 || w->nSprings > 0)
        return -1;
    w->recording = 1;
    return 0;
}

void oracle_tape_end(OracleWorld *w)
{
    for (int s = 0; s < w->tapeSteps; ++s)
        tape_free_step(&w->tape[s]);
    free(w->tape);
    w->tape = NULL;
    w->tapeSteps = w->tapeCap = 0;
    w->recording = 0;
}

int oracle_tape_steps(const OracleWorld *w) { return w->tapeSteps; }

const OracleTapeStep *oracle_tape_step(const OracleWorld *w, int s)
{
    return s >= 0 && s < w->tapeSteps ? &w->tape[s] : NULL;
}

/* step start: body state before anything of the step runs */
static void tape_begin_step(OracleWorld *w)
{
    if (w->tapeSteps == w->tapeCap)
    {
        w->tapeCap = w->tapeCap ? 2 * w->tapeCap : 64;
        w->tape = (OracleTapeStep *)realloc(w->tape, sizeof(OracleTapeStep) * (size_t)w->tapeCap);
    }
    OracleTapeStep *t = &w->tape[w->tapeSteps++];
    memset(t, 0, sizeof(*t));
    size_t n = (size_t)(w->n > 0 ? w->n : 1);
    t->bodyIn = (float *)calloc(n * 16, sizeof(float));
    t->bodyFlags = (unsigned char *)calloc(n, 1);
    for (int b = 0; b < w->n; ++b)
    {
        const Body *x = &w->bodies[b];
        float *o = t->bodyIn + 16 * (size_t)b;
        memcpy(o, &x->pos, 12);
        memcpy(o + 3, &x->q, 16);
        memcpy(o + 7, &x->vel, 12);
        memcpy(o + 10, &x->angvel, 12);
        memcpy(o + 13, &x->prevVel, 12);
    }
}

/* end of prepare: the step's manifolds, their links to the previous step, the sweep order
 * and room for the iteration flags */
static void tape_record_prepared(OracleWorld *w)
{
    OracleTapeStep *t = &w->tape[w->tapeSteps - 1];
    int M = w->nMan;
    size_t m1 = (size_t)(M > 0 ? M : 1);
    t->nMan = M;
    t->iterations = w->p.iterations;
    t->ab = (int *)calloc(m1 * 2, sizeof(int));
    t->basis = (float *)calloc(m1 * 9, sizeof(float));
    t->friction = (float *)calloc(m1, sizeof(float));
    t->ncontacts = (int *)calloc(m1, sizeof(int));
    t->keys = (int *)calloc(m1 * 8, sizeof(int));
    t->geo = (float *)calloc(m1 * 8 * 6, sizeof(float));
    t->init = (float *)calloc(m1 * 8 * 9, sizeof(float));
    t->src = (int *)calloc(m1 * 8, sizeof(int));
    t->initFlags = (unsigned char *)calloc(m1 * 8, 1);
    for (int i = 0; i < M; ++i)
    {
        const Manifold *m = &w->man[i];
        t->ab[2 * i] = m->a;
        t->ab[2 * i + 1] = m->b;
        memcpy(t->basis + 9 * (size_t)i, &m->basis, 36);
        t->friction[i] = m->friction;
        t->ncontacts[i] = m->n;
        for (int k = 0; k < 8; ++k)
        {
            size_t slot = (size_t)i * 8 + (size_t)k;
            t->src[slot] = -1;
            if (k >= m->n)
                continue;
            const Contact *c = &m->c[k];
            t->keys[slot] = c->key;
            memcpy(t->geo + 6 * slot, &c->rA, 12);
            memcpy(t->geo + 6 * slot + 3, &c->rB, 12);
            memcpy(t->init + 9 * slot, &c->C0, 12);
            memcpy(t->init + 9 * slot + 3, &c->lambda, 12);
            memcpy(t->init + 9 * slot + 6, &c->penalty, 12);
            t->initFlags[slot] = m->iflags[k];
            if (m->oldIndex >= 0 && m->srcSlot[k] >= 0)
                t->src[slot] = m->oldIndex * 8 + m->srcSlot[k];
        }
    }
    t->nSolve = w->nSolve;
    t->nColours = w->nColours;
    t->solveOrder = (int *)calloc((size_t)(w->nSolve > 0 ? w->nSolve : 1), sizeof(int));
    memcpy(t->solveOrder, w->solveOrder, sizeof(int) * (size_t)w->nSolve);
    t->colourStart = (int *)calloc((size_t)w->nColours + 1, sizeof(int));
    if (w->nColours > 0)
    {
        for (int k = 0; k < w->nSolve; ++k)
            t->colourStart[w->colour[w->solveOrder[k]] + 1]++;
        for (int c = 0; c < w->nColours; ++c)
            t->colourStart[c + 1] += t->colourStart[c];
    }
    else
        t->colourStart[0] = w->nSolve;
    t->flags = (unsigned short *)calloc((size_t)w->p.iterations * m1 * 8 * 3, sizeof(unsigned short));
}
