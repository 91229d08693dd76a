// Adjoint of the AVBD step on the GPU (included at the end of avbd_capi.cu, which owns the
// context).
//
// Model. The step with every integer decision of the FP32 run held fixed (avbd_diff.h): a
// smooth map of the initial body state, masses and friction coefficients. Its derivatives
// are evaluated exactly, at the trajectory of that map, in double precision.
//
// avbd_adjoint_forward, per step:
//   1. the ordinary FP32 step (step_once), taping what it decided: the manifolds after
//      initialisation (pairs, basis, body-local anchors), the feature-key links of their
//      contacts to the previous step's list (manifold.cpp:128-160) with the warm-start
//      penalty clamps (manifold.cpp:170), the force lists, the colouring and sweep order,
//      the adaptive warm-start outcome of every body (solver.cpp:1146-1150) and, for every
//      iteration and contact, the branch outcomes of its two primal evaluations and its
//      dual update (manifold.cpp:200-212, 268-278). The outcomes come from the step's own
//      FP32 values: poses and contact state are snapshot at every iteration boundary and
//      re-evaluated with the forward's own eval_contact, so they are bit-for-bit the
//      branches the step took;
//   2. the frozen-branch map replayed in double precision on that tape (the replay
//      kernels below), with a snapshot of the replay state every `every` steps.
// avbd_adjoint_backward walks the checkpoint segments backwards: it restores a segment's
// double-precision snapshot, replays the segment keeping the poses and contact state at
// every iteration boundary, and reverses its steps:
//   finish -> iterations in reverse (dual, then colours in reverse order) -> manifold
//   initialisation (C0, carried lambda / penalty) -> warm start.
// Within one colour no two bodies share a constraint, so a reverse primal launch owns its
// bodies' adjoints and the contact slots it touches; partner bodies (other colours) receive
// their share by atomic addition. A partner's pose adjoint refers to the pose the forward
// saw: partners of an earlier colour are reversed later (their accumulator still holds the
// adjoint of the updated pose), partners of a later colour earlier (it holds the adjoint of
// the pose before their update).
#pragma once

#include "avbd_diff.h"

namespace avbd
{
namespace adjoint
{

namespace ad = avbd_diff;
typedef double D;

// Packed branch outcomes of one contact slot in one iteration: bits 0-11 the dual update
// (EvalFlags), bits 12-13 the primal evaluation for body A, bits 14-15 for body B.
constexpr int PRIMAL_A_SHIFT = 12;
constexpr int PRIMAL_B_SHIFT = 14;

// One taped step (device view).
struct StepTape
{
    int n, nMan;
    const int2 *ab;
    const int *nc;
    const float4 *basis; // 3 per manifold, row0.w = friction
    const float4 *geo;   // 2 per slot: (rA.xyz, rB.x) (rB.yz, -, -)
    const int *src;      // per slot: slot of the previous step's list, -1 = new contact
    const unsigned char *iflags;
    const int *pairIdx; // per manifold: friction pair
    const int *adjStart;
    const unsigned *adj;
    const int *solveList;
    const int *colour;
    const unsigned char *bflags;
    const unsigned short *flags; // iterations x 8 nMan
};

// Double-precision replay state.
struct State64
{
    double4 *p, *q, *v, *w, *vp;        // bodies
    double4 *iLin, *iAng, *tLin, *tAng; // initial (step start) and inertial poses
    double4 *lam, *pen, *c0;            // this step's contact slots
    const double4 *lamPrev, *penPrev;   // the previous step's contact slots
};

// One step of a replayed segment, for the reverse sweep.
struct Snap64
{
    const double4 *bodyIn; // 5n: p, q, v, w, vp at step start
    const double4 *pose;   // per iteration boundary t: 2n (p, q)
    const double4 *lp;     // per iteration boundary t: 16 nMan (lambda of every slot, then penalty)
    const double4 *c0;     // 8 nMan
    const double *ldl;     // per iteration t and body: LDL_STRIDE doubles (D, strict lower L, dx)
};

// A body's 6x6 factorisation and step as the replay computed them: D (6), the strict
// lower triangle of L row by row (15) and dx (6).
constexpr int LDL_STRIDE = 28;

AVBD_DEV void store_ldl(double *o, const ad::Ldl6<D> &f, const D dx[6])
{
    int k = 0;
    for (int i = 0; i < 6; ++i)
        o[k++] = f.D[i];
    for (int i = 1; i < 6; ++i)
        for (int j = 0; j < i; ++j)
            o[k++] = f.L[i][j];
    for (int i = 0; i < 6; ++i)
        o[k++] = dx[i];
}

AVBD_DEV void load_ldl(const double *o, ad::Ldl6<D> &f, D dx[6])
{
    int k = 0;
    for (int i = 0; i < 6; ++i)
        f.D[i] = o[k++];
    for (int i = 1; i < 6; ++i)
        for (int j = 0; j < i; ++j)
            f.L[i][j] = o[k++];
    for (int i = 0; i < 6; ++i)
        dx[i] = o[k++];
}

struct AdjView
{
    double4 *p, *q, *v, *w, *vp;
    double4 *iLin, *iAng, *tLin, *tAng;
    double *m;
    double4 *lam, *pen, *c0;
    double4 *lamPrev, *penPrev;
    double *mu;
};

struct AdjParams
{
    Params P; // FP32, for the branch outcomes
    D dt, g, alpha, beta, gamma;
};

AVBD_DEV ad::V3<D> d3(float4 v) { return ad::v3<D>(v.x, v.y, v.z); }
AVBD_DEV ad::Q4<D> d4(float4 v) { return ad::q4<D>(v.x, v.y, v.z, v.w); }
AVBD_DEV ad::V3<D> ld3(const double4 *p)
{
    double4 v = *p;
    return ad::v3<D>(v.x, v.y, v.z);
}
AVBD_DEV ad::Q4<D> ld4(const double4 *p)
{
    double4 v = *p;
    return ad::q4<D>(v.x, v.y, v.z, v.w);
}
AVBD_DEV void st3(double4 *p, ad::V3<D> v) { *p = make_double4(v.x, v.y, v.z, 0.0); }
AVBD_DEV void st4(double4 *p, ad::Q4<D> v) { *p = make_double4(v.x, v.y, v.z, v.w); }
AVBD_DEV void add3(double4 *p, ad::V3<D> v)
{
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
    atomicAdd(&p->z, v.z);
}
AVBD_DEV void add4(double4 *p, ad::Q4<D> v)
{
    atomicAdd(&p->x, v.x);
    atomicAdd(&p->y, v.y);
    atomicAdd(&p->z, v.z);
    atomicAdd(&p->w, v.w);
}

AVBD_DEV bool dynamic(const DevBodies &B, int b) { return B.massMoment[b].x > 0; }
AVBD_DEV ad::V3<D> shape_of(float4 mm) { return ad::v3<D>((D)mm.y / (D)mm.x, (D)mm.z / (D)mm.x, (D)mm.w / (D)mm.x); }

AVBD_DEV ad::ContactIn<D> contact64(const StepTape &T, int m, int ci, ad::V3<D> C0, ad::V3<D> lam, ad::V3<D> pen)
{
    const float4 *g = T.geo + 2 * ((size_t)m * 8 + ci);
    const float4 *bs = T.basis + 3 * (size_t)m;
    float4 g0 = g[0], g1 = g[1];
    ad::ContactIn<D> c;
    c.rA = ad::v3<D>(g0.x, g0.y, g0.z);
    c.rB = ad::v3<D>(g0.w, g1.x, g1.y);
    c.e[0] = d3(bs[0]);
    c.e[1] = d3(bs[1]);
    c.e[2] = d3(bs[2]);
    c.C0 = C0;
    c.lam = lam;
    c.pen = pen;
    c.mu = (D)bs[0].w;
    return c;
}

AVBD_DEV unsigned primal_bits(unsigned short f, bool isA) { return (f >> (isA ? PRIMAL_A_SHIFT : PRIMAL_B_SHIFT)) & 3u; }
AVBD_DEV unsigned dual_bits(unsigned short f) { return f & 0xFFFu; }

// ---------------------------------------------------------------------------
// Taping the FP32 step
// ---------------------------------------------------------------------------

// Branch outcomes with the forward's FP32 expressions (manifold.cpp:200-212, 268-278)
AVBD_DEV unsigned primal_flags(const ContactEval &e)
{
    unsigned f = 0;
    if (!(e.F.x < 0))
        f |= ad::EF_NCLAMP;
    if (e.fs > e.bounds && e.fs > 0)
        f |= ad::EF_CONE;
    return f;
}

AVBD_DEV unsigned dual_flags(const ContactEval &e, const ContactRec &c, float betaLin)
{
    unsigned f = primal_flags(e);
    bool inCone = e.fs <= e.bounds;
    if (inCone)
        f |= ad::EF_RAMP_T;
    for (int k = 0; k < 3; ++k)
    {
        float ck = comp(e.C, k);
        if (ck < 0)
            f |= ad::EF_NEG_X << k;
        else if (ck > 0)
            f |= ad::EF_POS_X << k;
        bool ramps = k == 0 ? e.F.x < 0 : inCone;
        if (ramps && !(comp(c.pen, k) + betaLin * fabsf(ck) < PENALTY_MAX))
            f |= ad::EF_CAP_X << k;
    }
    return f;
}

// FP32 snapshots of one step being taped.
struct Snap32
{
    int n, nMan;
    const float4 *bodyIn;  // 5n: pos, quat, vel, angvel, prevVel at step start
    const float4 *pose;    // per iteration boundary: 2n
    const float4 *lp;      // per iteration boundary: 16 nMan (contact words 2, 3 of every slot)
    const float4 *contact; // the step's manifolds (words 0, 1 do not change during iterations)
    const float4 *basis;
    const int2 *ab;
    const int *nc;
    const int *colour;
};

AVBD_DEV Pose pose32(const Snap32 &X, int t, int b)
{
    Pose s;
    const float4 *p = X.pose + (size_t)t * 2 * X.n;
    s.p = xyz(p[b]);
    s.q = p[X.n + b];
    s.ip = xyz(X.bodyIn[b]);
    s.iq = X.bodyIn[X.n + b];
    return s;
}

// contact words 2 and 3 (C0.z, penalty; lambda, key | stick) of every slot
__global__ void k_rec_lp(const float4 *contact, int nMan, float4 *out)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= 8 * nMan)
        return;
    int m = s >> 3, ci = s & 7;
    const float4 *c = contact + (size_t)m * 32 + 4 * ci;
    out[2 * s] = c[2];
    out[2 * s + 1] = c[3];
}

// FP32 state at an iteration boundary: body poses and contact words 2, 3 of every slot
__global__ void k_rec_iteration(const float4 *pos, const float4 *quat, int n, const float4 *contact, int nMan,
                                float4 *pose, float4 *lp)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        pose[i] = pos[i];
        pose[n + i] = quat[i];
    }
    if (i < 8 * nMan)
    {
        const float4 *c = contact + (size_t)(i >> 3) * 32 + 4 * (i & 7);
        lp[2 * i] = c[2];
        lp[2 * i + 1] = c[3];
    }
}

// A taped step run by the single-launch iteration kernel: every slice of the per-iteration
// records starts as the state before the first iteration, and the kernel overwrites what each
// iteration changes (the solved bodies' poses, the live slots' multipliers and penalties), so
// the records equal those k_rec_iteration takes between per-colour iterations.
__global__ void k_rec_fill(const float4 *pos, const float4 *quat, int n, const float4 *contact, int nMan,
                           float4 *pose, float4 *lp, int slices)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        const float4 p = pos[i], q = quat[i];
        for (int k = 0; k < slices; ++k)
        {
            pose[(size_t)k * 2 * n + i] = p;
            pose[(size_t)k * 2 * n + n + i] = q;
        }
    }
    if (i < 8ll * nMan)
    {
        const float4 *c = contact + (size_t)(i >> 3) * 32 + 4 * (i & 7);
        const float4 c2 = c[2], c3 = c[3];
        for (int k = 0; k < slices; ++k)
        {
            lp[(size_t)k * 16 * nMan + 2 * i] = c2;
            lp[(size_t)k * 16 * nMan + 2 * i + 1] = c3;
        }
    }
}

// body-local anchors of every slot
__global__ void k_tape_geo(const float4 *contact, int nMan, float4 *geo)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= 8 * nMan)
        return;
    int m = s >> 3, ci = s & 7;
    const float4 *c = contact + (size_t)m * 32 + 4 * ci;
    float4 w1 = c[1];
    geo[2 * s] = c[0];
    geo[2 * s + 1] = make_float4(w1.x, w1.y, 0.0f, 0.0f);
}

// Links of this step's contacts to the previous step's list and the warm-start penalty
// clamp outcomes (manifold.cpp:128-160, 170).
__global__ void k_rec_links(DevManifolds M, int nMan, const unsigned long long *prevSeq, const int *prevN,
                            const float4 *prevLP, int nPrev, float gamma, int *src, unsigned char *iflags)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= 8 * nMan)
        return;
    int m = s >> 3, ci = s & 7;
    src[s] = -1;
    iflags[s] = 0;
    if (ci >= M.n[m])
        return;
    unsigned long long q = M.seq[m];
    int lo = 0, hi = nPrev;
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        if (prevSeq[mid] < q)
            lo = mid + 1;
        else
            hi = mid;
    }
    if (lo >= nPrev || prevSeq[lo] != q)
        return;
    unsigned key = __float_as_uint(M.contact[(size_t)m * 32 + 4 * ci + 3].w) & 0x7FFFFFFFu;
    for (int j = 0; j < prevN[lo]; ++j)
    {
        const float4 *o = prevLP + 2 * ((size_t)lo * 8 + j);
        if ((__float_as_uint(o[1].w) & 0x7FFFFFFFu) == key)
        {
            src[s] = lo * 8 + j;
            float3 pg = mul(f3(o[0].y, o[0].z, o[0].w), gamma);
            unsigned f = 0;
            for (int k = 0; k < 3; ++k)
            {
                float v = comp(pg, k);
                if (v > PENALTY_MAX)
                    f |= ad::IF_HI_X << k;
                else if (v < PENALTY_MIN)
                    f |= ad::IF_LO_X << k;
            }
            iflags[s] = (unsigned char)f;
            return;
        }
    }
}

// Body warm-start outcomes (solver.cpp:1146-1150, 1163-1168) with k_warm_start's FP32
// expressions.
__global__ void k_tape_bflags(DevBodies B, const float4 *bodyIn, const int *adjStart, Params P, unsigned char *out)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    int n = B.n;
    if (b >= n)
        return;
    unsigned f = 0;
    if (B.massMoment[b].x > 0)
        f |= ad::BF_DYNAMIC;
    if (adjStart[b + 1] > adjStart[b])
        f |= ad::BF_FORCES;
    float3 vel = xyz(bodyIn[2 * n + b]);
    float3 pv = xyz(bodyIn[4 * n + b]);
    float3 accel = divs(sub(vel, pv), P.dt);
    float accelExt = accel.z * rsign(P.gravity);
    float raw = accelExt / fabsf(P.gravity);
    float weight = rclamp(raw, 0.0f, 1.0f);
    if (isfinite(weight))
    {
        if (raw > 0.0f && raw < 1.0f)
            f |= ad::BF_ACCEL_IN;
        else if (weight == 1.0f)
            f |= ad::BF_ACCEL_ONE;
    }
    out[b] = (unsigned char)f;
}

// Every contact evaluation of the step: iteration t, slot s. The primal evaluation for body
// A saw A before its update and B after its update if B's colour came first; the dual saw
// both after the primal sweep.
__global__ void k_tape_flags(Snap32 X, Params P, int iterations, unsigned short *flags)
{
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long slots = 8ll * X.nMan;
    if (idx >= slots * iterations)
        return;
    int t = (int)(idx / slots);
    int s = (int)(idx - (long long)t * slots);
    int m = s >> 3, ci = s & 7;
    unsigned short out = 0;
    if (ci < X.nc[m])
    {
        int2 ab = X.ab[m];
        const float4 *cw = X.contact + (size_t)m * 32 + 4 * ci;
        const float4 *l = X.lp + (size_t)t * 16 * X.nMan + 2 * (size_t)s;
        float4 w[4] = {cw[0], cw[1], l[0], l[1]};
        ContactRec c = load_contact(w);
        const float4 *bs = X.basis + 3 * (size_t)m;
        M3 basis = rows(xyz(bs[0]), xyz(bs[1]), xyz(bs[2]));
        int ca = X.colour[ab.x], cb = X.colour[ab.y];
        unsigned f = 0;
        if (ca >= 0)
        {
            Pose A = pose32(X, t, ab.x), B = pose32(X, (cb >= 0 && cb < ca) ? t + 1 : t, ab.y);
            f |= primal_flags(eval_contact(A, B, basis, bs[0].w, c, P.alpha)) << PRIMAL_A_SHIFT;
        }
        if (cb >= 0)
        {
            Pose A = pose32(X, (ca >= 0 && ca < cb) ? t + 1 : t, ab.x), B = pose32(X, t, ab.y);
            f |= primal_flags(eval_contact(A, B, basis, bs[0].w, c, P.alpha)) << PRIMAL_B_SHIFT;
        }
        Pose A = pose32(X, t + 1, ab.x), B = pose32(X, t + 1, ab.y);
        f |= dual_flags(eval_contact(A, B, basis, bs[0].w, c, P.alpha), c, P.betaLin);
        out = (unsigned short)f;
    }
    flags[idx] = out;
}

// (min, max) body pair of every manifold
__global__ void k_pair_keys(const int2 *ab, int nMan, unsigned long long *out)
{
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nMan)
        return;
    int2 p = ab[m];
    unsigned lo = (unsigned)min(p.x, p.y), hi = (unsigned)max(p.x, p.y);
    out[m] = ((unsigned long long)lo << 32) | hi;
}

__global__ void k_pair_index(const int2 *ab, int nMan, const unsigned long long *pairs, int P, int *idx)
{
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= nMan)
        return;
    int2 p = ab[m];
    unsigned long long key = ((unsigned long long)(unsigned)min(p.x, p.y) << 32) | (unsigned)max(p.x, p.y);
    int lo = 0, hi = P;
    while (lo < hi)
    {
        int mid = (lo + hi) >> 1;
        if (pairs[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    idx[m] = (lo < P && pairs[lo] == key) ? lo : -1;
}

// ---------------------------------------------------------------------------
// Double-precision replay of a taped step (the frozen-branch map, avbd_diff.h)
// ---------------------------------------------------------------------------

__global__ void k_state_to_double(DevBodies B, State64 S)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B.n)
        return;
    float4 p = B.pos[b], q = B.quat[b], v = B.vel[b], w = B.angvel[b], vp = B.prevVel[b];
    S.p[b] = make_double4(p.x, p.y, p.z, 0.0);
    S.q[b] = make_double4(q.x, q.y, q.z, q.w);
    S.v[b] = make_double4(v.x, v.y, v.z, 0.0);
    S.w[b] = make_double4(w.x, w.y, w.z, 0.0);
    S.vp[b] = make_double4(vp.x, vp.y, vp.z, 0.0);
}

__global__ void k_lp_to_double(const float4 *contact, int nMan, double4 *lam, double4 *pen)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= 8 * nMan)
        return;
    int m = s >> 3, ci = s & 7;
    const float4 *c = contact + (size_t)m * 32 + 4 * ci;
    float4 k2 = c[2], k3 = c[3];
    pen[s] = make_double4(k2.y, k2.z, k2.w, 0.0);
    lam[s] = make_double4(k3.x, k3.y, k3.z, 0.0);
}

// Manifold::initialize (manifold.cpp:162-171) at the step-start poses
__global__ void k_rep_init(StepTape T, State64 S, AdjParams Q)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= 8 * T.nMan)
        return;
    int m = s >> 3, ci = s & 7;
    if (ci >= T.nc[m])
        return;
    int2 ab = T.ab[m];
    ad::ContactIn<D> c = contact64(T, m, ci, ad::vzero<D>(), ad::vzero<D>(), ad::vzero<D>());
    ad::V3<D> C0 = ad::contact_C0(ld3(S.p + ab.x), ld4(S.q + ab.x), ld3(S.p + ab.y), ld4(S.q + ab.y), c.rA, c.rB, c.e);
    int src = T.src[s];
    ad::V3<D> lp = src >= 0 ? ld3(S.lamPrev + src) : ad::vzero<D>();
    ad::V3<D> pp = src >= 0 ? ld3(S.penPrev + src) : ad::vzero<D>();
    ad::V3<D> lam, pen;
    ad::contact_carry(lp, pp, src >= 0, T.iflags[s], Q.alpha, Q.gamma, lam, pen);
    st3(S.c0 + s, C0);
    st3(S.lam + s, lam);
    st3(S.pen + s, pen);
}

// body warm start (solver.cpp:1134-1169)
__global__ void k_rep_warm(StepTape T, DevBodies B, State64 S, AdjParams Q)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= T.n)
        return;
    ad::V3<D> p0 = ld3(S.p + b);
    ad::Q4<D> q0 = ld4(S.q + b);
    st3(S.iLin + b, p0);
    st4(S.iAng + b, q0);
    if (!dynamic(B, b))
        return;
    ad::WarmOut<D> o = ad::warm_start(p0, q0, ld3(S.v + b), ld3(S.w + b), ld3(S.vp + b), Q.dt, Q.g, T.bflags[b]);
    st3(S.tLin + b, o.inertLin);
    st4(S.tAng + b, o.inertAng);
    st3(S.p + b, o.p);
    st4(S.q + b, o.q);
}

AVBD_DEV ad::Pose<D> pose_state(const State64 &S, int b)
{
    ad::Pose<D> r;
    r.p = ld3(S.p + b);
    r.q = ld4(S.q + b);
    r.pi = ld3(S.iLin + b);
    r.qi = ld4(S.iAng + b);
    return r;
}

// Per-body work is spread over a group of G lanes: the body's contact rows (its manifold
// entries in force order, each contact a row) go round-robin to the lanes, each lane stamps
// its rows into a private 6x6 system, and a butterfly over the group sums them. Every lane
// then holds the same system and factors it, so no lane waits for a broadcast.
constexpr int ADJ_G = 8;
constexpr int ADJ_BLOCK = 64;

template <int G> AVBD_DEV unsigned group_mask()
{
    return G == 32 ? 0xFFFFFFFFu : (((1u << G) - 1u) << ((threadIdx.x & 31) / G * G));
}

template <int G> AVBD_DEV D group_sum(D v, unsigned mask)
{
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1)
        v += __shfl_xor_sync(mask, v, o, G);
    return v;
}

template <int G> AVBD_DEV void group_sum_sys(ad::Sys6<D> &s, unsigned mask)
{
#pragma unroll
    for (int i = 0; i < 6; ++i)
    {
        s.g[i] = group_sum<G>(s.g[i], mask);
#pragma unroll
        for (int j = 0; j < 6; ++j)
            s.H[i][j] = group_sum<G>(s.H[i][j], mask);
    }
}

// body primal for the bodies of one colour (solver.cpp:1177-1242)
__global__ void __launch_bounds__(ADJ_BLOCK) k_rep_primal(StepTape T, DevBodies B, State64 S, AdjParams Q, int t,
                                                          int first, int count, double *ldlOut)
{
    constexpr int G = ADJ_G;
    const int lane = threadIdx.x % G;
    const int gid = blockIdx.x * (ADJ_BLOCK / G) + threadIdx.x / G;
    if (gid >= count)
        return;
    const unsigned mask = group_mask<G>();
    const int b = T.solveList[first + gid];
    float4 mm = B.massMoment[b];
    ad::Pose<D> own = pose_state(S, b);
    const unsigned short *fl = T.flags + (size_t)t * 8 * T.nMan;
    ad::Sys6<D> sys;
    ad::sys_zero(sys);
    int row = 0;
    for (int k = T.adjStart[b]; k < T.adjStart[b + 1]; ++k)
    {
        unsigned e = T.adj[k];
        if (adj_type(e) != ADJ_MANIFOLD)
            continue;
        int m = (int)adj_index(e);
        int nc = T.nc[m];
        int mine = row % G <= lane ? lane - row % G : lane - row % G + G; // first owned contact
        row += nc;
        if (mine >= nc)
            continue;
        bool isA = adj_isA(e) != 0;
        int2 ab = T.ab[m];
        ad::Pose<D> A = isA ? own : pose_state(S, ab.x);
        ad::Pose<D> Bp = isA ? pose_state(S, ab.y) : own;
        for (int ci = mine; ci < nc; ci += G)
        {
            int s = m * 8 + ci;
            ad::ContactIn<D> c = contact64(T, m, ci, ld3(S.c0 + s), ld3(S.lam + s), ld3(S.pen + s));
            ad::stamp_contact(sys, c, ad::contact_forward(A, Bp, c, Q.alpha, primal_bits(fl[s], isA)), isA);
        }
    }
    group_sum_sys<G>(sys, mask);
    ad::stamp_inertia(sys, (D)mm.x, shape_of(mm), own.p, ld3(S.tLin + b), own.q, ld4(S.tAng + b), Q.dt);
    ad::Ldl6<D> f;
    ad::ldl_factor(sys.H, f);
    D dx[6];
    ad::body_dx(f, sys, dx);
    if (lane == 0)
    {
        st3(S.p + b, own.p + ad::v3<D>(dx[0], dx[1], dx[2]));
        st4(S.q + b, ad::qstep(own.q, ad::v3<D>(dx[3], dx[4], dx[5])));
        if (ldlOut)
            store_ldl(ldlOut + ((size_t)t * T.n + b) * LDL_STRIDE, f, dx);
    }
}

// Manifold::updateDual (manifold.cpp:231-279)
__global__ void k_rep_dual(StepTape T, State64 S, AdjParams Q, int t)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= 8 * T.nMan)
        return;
    int m = s >> 3, ci = s & 7;
    if (ci >= T.nc[m])
        return;
    int2 ab = T.ab[m];
    ad::ContactIn<D> c = contact64(T, m, ci, ld3(S.c0 + s), ld3(S.lam + s), ld3(S.pen + s));
    ad::V3<D> lam, pen;
    ad::contact_dual_forward(pose_state(S, ab.x), pose_state(S, ab.y), c, Q.alpha, Q.beta,
                             dual_bits(T.flags[(size_t)t * 8 * T.nMan + s]), lam, pen);
    st3(S.lam + s, lam);
    st3(S.pen + s, pen);
}

// finishStep (solver.cpp:1275-1287)
__global__ void k_rep_finish(StepTape T, DevBodies B, State64 S, AdjParams Q)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= T.n)
        return;
    ad::V3<D> v = ld3(S.v + b);
    st3(S.vp + b, v);
    if (!dynamic(B, b))
        return;
    D idt = D(1) / Q.dt;
    st3(S.v + b, (ld3(S.p + b) - ld3(S.iLin + b)) * idt);
    st3(S.w + b, ad::qdiff(ld4(S.q + b), ld4(S.iAng + b)) * idt);
}

// replay state at an iteration boundary: poses of every body, lambda and penalty of every slot
__global__ void k_snapshot(State64 S, int n, int nMan, double4 *pose, double4 *lp)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        pose[i] = S.p[i];
        pose[n + i] = S.q[i];
    }
    int slots = 8 * nMan;
    if (i < slots)
    {
        lp[i] = S.lam[i];
        lp[slots + i] = S.pen[i];
    }
}

// body state at step start
__global__ void k_snapshot_bodies(State64 S, int n, double4 *out)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n)
        return;
    out[b] = S.p[b];
    out[n + b] = S.q[b];
    out[2 * n + b] = S.v[b];
    out[3 * n + b] = S.w[b];
    out[4 * n + b] = S.vp[b];
}

// ---------------------------------------------------------------------------
// Reverse of one replayed step
// ---------------------------------------------------------------------------

AVBD_DEV ad::Pose<D> pose_snap(const Snap64 &X, int n, int t, int b)
{
    ad::Pose<D> r;
    const double4 *p = X.pose + (size_t)t * 2 * n;
    r.p = ld3(p + b);
    r.q = ld4(p + n + b);
    r.pi = ld3(X.bodyIn + b);
    r.qi = ld4(X.bodyIn + n + b);
    return r;
}

AVBD_DEV ad::ContactIn<D> contact_snap(const StepTape &T, const Snap64 &X, int t, int m, int ci)
{
    size_t s = (size_t)m * 8 + ci;
    const double4 *l = X.lp + (size_t)t * 16 * T.nMan;
    return contact64(T, m, ci, ld3(X.c0 + s), ld3(l + s), ld3(l + 8 * (size_t)T.nMan + s));
}

AVBD_DEV void scatter_pose(const DevBodies &B, AdjView &A, int b, const ad::PoseBar<D> &pb)
{
    if (!dynamic(B, b))
        return;
    add3(A.p + b, pb.p);
    add4(A.q + b, pb.q);
    add3(A.iLin + b, pb.pi);
    add4(A.iAng + b, pb.qi);
}

// finishStep: velocities from the final and initial poses; the previous velocity is the
// step-start velocity.
__global__ void k_adj_finish(StepTape T, Snap64 X, DevBodies B, AdjView A, AdjParams Q, int lastT)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    int n = T.n;
    if (b >= n)
        return;
    ad::V3<D> vb = ld3(A.v + b), wb = ld3(A.w + b), vpb = ld3(A.vp + b);
    ad::V3<D> iLin = ad::vzero<D>();
    ad::Q4<D> iAng = ad::qzero<D>();
    if (dynamic(B, b))
    {
        ad::V3<D> pb = ld3(A.p + b);
        ad::Q4<D> qb = ld4(A.q + b);
        ad::finish_vjp(ld4(X.pose + (size_t)lastT * 2 * n + n + b), ld4(X.bodyIn + n + b), Q.dt, vb, wb, pb, qb,
                       iLin, iAng);
        st3(A.p + b, pb);
        st4(A.q + b, qb);
        st3(A.v + b, vpb);
        st3(A.w + b, ad::vzero<D>());
    }
    else
        st3(A.v + b, vb + vpb);
    st3(A.vp + b, ad::vzero<D>());
    st3(A.iLin + b, iLin);
    st4(A.iAng + b, iAng);
    st3(A.tLin + b, ad::vzero<D>());
    st4(A.tAng + b, ad::qzero<D>());
}

// dual update of iteration t, per contact slot
__global__ void k_adj_dual(StepTape T, Snap64 X, DevBodies B, AdjView A, AdjParams Q, int t)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= 8 * T.nMan)
        return;
    int m = s >> 3, ci = s & 7;
    if (ci >= T.nc[m])
        return;
    int2 ab = T.ab[m];
    ad::ContactIn<D> c = contact_snap(T, X, t, m, ci);
    ad::V3<D> lb = ld3(A.lam + s), pb = ld3(A.pen + s), c0b = ld3(A.c0 + s);
    ad::PoseBar<D> Ab = ad::posebar_zero<D>(), Bb = ad::posebar_zero<D>();
    D mub = 0;
    ad::contact_dual_vjp(pose_snap(X, T.n, t + 1, ab.x), pose_snap(X, T.n, t + 1, ab.y), c, Q.alpha, Q.beta,
                         dual_bits(T.flags[(size_t)t * 8 * T.nMan + s]), lb, pb, Ab, Bb, c0b, mub);
    st3(A.lam + s, lb);
    st3(A.pen + s, pb);
    st3(A.c0 + s, c0b);
    scatter_pose(B, A, ab.x, Ab);
    scatter_pose(B, A, ab.y, Bb);
    if (mub != 0 && T.pairIdx[m] >= 0)
        atomicAdd(A.mu + T.pairIdx[m], mub);
}

// body primal of iteration t for the bodies of colour c, lanes as in k_rep_primal
__global__ void __launch_bounds__(ADJ_BLOCK) k_adj_primal(StepTape T, Snap64 X, DevBodies B, AdjView A, AdjParams Q,
                                                          int t, int c, int first, int count)
{
    constexpr int G = ADJ_G;
    const int lane = threadIdx.x % G;
    const int gid = blockIdx.x * (ADJ_BLOCK / G) + threadIdx.x / G;
    if (gid >= count)
        return;
    const unsigned mask = group_mask<G>();
    const int n = T.n;
    const int b = T.solveList[first + gid];
    auto partner = [&](int x) {
        int cx = T.colour[x];
        return pose_snap(X, n, (cx >= 0 && cx < c) ? t + 1 : t, x);
    };
    const unsigned short *fl = T.flags + (size_t)t * 8 * T.nMan;
    ad::Pose<D> own = pose_snap(X, n, t, b);
    const int start = T.adjStart[b], end = T.adjStart[b + 1];
    float4 mm = B.massMoment[b];
    D mass = mm.x;
    ad::V3<D> shape = shape_of(mm);
    ad::WarmOut<D> wo = ad::warm_start(ld3(X.bodyIn + b), ld4(X.bodyIn + n + b), ld3(X.bodyIn + 2 * n + b),
                                       ld3(X.bodyIn + 3 * n + b), ld3(X.bodyIn + 4 * n + b), Q.dt, Q.g, T.bflags[b]);
    // the factorisation and step the replay stored for this body and iteration
    ad::Ldl6<D> f;
    D dx[6];
    load_ldl(X.ldl + ((size_t)t * n + b) * LDL_STRIDE, f, dx);
    // pose update p += dx_lin, q = q (+) dx_ang
    ad::V3<D> pnew = ld3(A.p + b);
    D dxbar[6] = {pnew.x, pnew.y, pnew.z, 0, 0, 0};
    ad::Q4<D> qbarPre = ad::qzero<D>();
    ad::V3<D> wdx = ad::vzero<D>();
    ad::qstep_vjp(own.q, ad::v3<D>(dx[3], dx[4], dx[5]), ld4(A.q + b), qbarPre, wdx);
    dxbar[3] = wdx.x;
    dxbar[4] = wdx.y;
    dxbar[5] = wdx.z;
    D u[6];
    ad::body_dx_vjp_u(f, dxbar, u);
    // each lane's rows
    ad::PoseBar<D> mineBar = ad::posebar_zero<D>();
    {
        int row = 0;
        for (int k = start; k < end; ++k)
        {
            unsigned e = T.adj[k];
            if (adj_type(e) != ADJ_MANIFOLD)
                continue;
            int m = (int)adj_index(e);
            int nc = T.nc[m];
            int mine = row % G <= lane ? lane - row % G : lane - row % G + G;
            row += nc;
            if (mine >= nc)
                continue;
            bool isA = adj_isA(e) != 0;
            int2 ab = T.ab[m];
            ad::Pose<D> PA = isA ? own : partner(ab.x);
            ad::Pose<D> PB = isA ? partner(ab.y) : own;
            ad::PoseBar<D> Ob = ad::posebar_zero<D>();
            D mub = 0;
            for (int ci = mine; ci < nc; ci += G)
            {
                int s = m * 8 + ci;
                ad::ContactIn<D> cc = contact_snap(T, X, t, m, ci);
                ad::PoseBar<D> Ab = ad::posebar_zero<D>(), Bb = ad::posebar_zero<D>();
                ad::V3<D> lb = ld3(A.lam + s), pnb = ld3(A.pen + s), c0b = ld3(A.c0 + s);
                ad::contact_primal_vjp_outer(PA, PB, cc, Q.alpha, primal_bits(fl[s], isA), isA, u, dx, Ab, Bb, lb,
                                             pnb, c0b, mub);
                st3(A.lam + s, lb);
                st3(A.pen + s, pnb);
                st3(A.c0 + s, c0b);
                const ad::PoseBar<D> &me = isA ? Ab : Bb;
                const ad::PoseBar<D> &them = isA ? Bb : Ab;
                mineBar.p += me.p;
                mineBar.q += me.q;
                mineBar.pi += me.pi;
                mineBar.qi += me.qi;
                Ob.p += them.p;
                Ob.q += them.q;
                Ob.pi += them.pi;
                Ob.qi += them.qi;
            }
            scatter_pose(B, A, isA ? ab.y : ab.x, Ob);
            if (mub != 0 && T.pairIdx[m] >= 0)
                atomicAdd(A.mu + T.pairIdx[m], mub);
        }
    }
    // the body's own share, summed over the group
    D r[14] = {mineBar.p.x, mineBar.p.y, mineBar.p.z, mineBar.q.x, mineBar.q.y, mineBar.q.z, mineBar.q.w,
               mineBar.pi.x, mineBar.pi.y, mineBar.pi.z, mineBar.qi.x, mineBar.qi.y, mineBar.qi.z, mineBar.qi.w};
#pragma unroll
    for (int k = 0; k < 14; ++k)
        r[k] = group_sum<G>(r[k], mask);
    if (lane != 0)
        return;
    ad::V3<D> pbar = pnew + ad::v3<D>(r[0], r[1], r[2]);
    ad::Q4<D> qbar = qbarPre + ad::q4<D>(r[3], r[4], r[5], r[6]);
    D mb = 0;
    ad::V3<D> tLinBar = ad::vzero<D>();
    ad::Q4<D> tAngBar = ad::qzero<D>();
    ad::stamp_inertia_vjp_outer(u, dx, mass, shape, own.p, wo.inertLin, own.q, wo.inertAng, Q.dt, mb, pbar, tLinBar,
                                qbar, tAngBar);
    st3(A.p + b, pbar);
    st4(A.q + b, qbar);
    A.m[b] += mb;
    st3(A.iLin + b, ld3(A.iLin + b) + ad::v3<D>(r[7], r[8], r[9]));
    ad::Q4<D> ia = ld4(A.iAng + b);
    ia += ad::q4<D>(r[10], r[11], r[12], r[13]);
    st4(A.iAng + b, ia);
    st3(A.tLin + b, ld3(A.tLin + b) + tLinBar);
    ad::Q4<D> ta = ld4(A.tAng + b);
    ta += tAngBar;
    st4(A.tAng + b, ta);
}

// Manifold::initialize: C0 from the step-start poses, carried lambda and penalty
__global__ void k_adj_init(StepTape T, Snap64 X, DevBodies B, AdjView A, AdjParams Q)
{
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= 8 * T.nMan)
        return;
    int m = s >> 3, ci = s & 7;
    if (ci >= T.nc[m])
        return;
    int2 ab = T.ab[m];
    const int n = T.n;
    ad::ContactIn<D> c = contact64(T, m, ci, ad::vzero<D>(), ad::vzero<D>(), ad::vzero<D>());
    ad::V3<D> pa = ad::vzero<D>(), pbv = ad::vzero<D>();
    ad::Q4<D> qa = ad::qzero<D>(), qb = ad::qzero<D>();
    ad::contact_C0_vjp(ld4(X.bodyIn + n + ab.x), ld4(X.bodyIn + n + ab.y), c.rA, c.rB, c.e, ld3(A.c0 + s), pa, qa, pbv,
                       qb);
    if (dynamic(B, ab.x))
    {
        add3(A.iLin + ab.x, pa);
        add4(A.iAng + ab.x, qa);
    }
    if (dynamic(B, ab.y))
    {
        add3(A.iLin + ab.y, pbv);
        add4(A.iAng + ab.y, qb);
    }
    int src = T.src[s];
    if (src >= 0)
    {
        ad::V3<D> lp = ad::vzero<D>(), pp = ad::vzero<D>();
        ad::contact_carry_vjp(ld3(A.lam + s), ld3(A.pen + s), T.iflags[s], Q.alpha, Q.gamma, lp, pp);
        add3(A.lamPrev + src, lp);
        add3(A.penPrev + src, pp);
    }
}

// body warm start back to the step-start state
__global__ void k_adj_warm(StepTape T, Snap64 X, DevBodies B, AdjView A, AdjParams Q)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = T.n;
    if (b >= n)
        return;
    ad::V3<D> p0b = ad::vzero<D>(), vb = ld3(A.v + b), wb = ld3(A.w + b), vpb = ld3(A.vp + b);
    ad::Q4<D> q0b = ad::qzero<D>();
    if (dynamic(B, b))
        ad::warm_start_vjp(ld4(X.bodyIn + n + b), ld3(X.bodyIn + 3 * n + b), Q.dt, Q.g, T.bflags[b], ld3(A.p + b),
                           ld4(A.q + b), ld3(A.tLin + b), ld4(A.tAng + b), ld3(A.iLin + b), ld4(A.iAng + b), p0b, q0b,
                           vb, wb, vpb);
    else
    {
        p0b = ld3(A.p + b) + ld3(A.iLin + b);
        q0b = ld4(A.q + b);
        q0b += ld4(A.iAng + b);
    }
    st3(A.p + b, p0b);
    st4(A.q + b, q0b);
    st3(A.v + b, vb);
    st3(A.w + b, wb);
    st3(A.vp + b, vpb);
}

} // namespace adjoint
} // namespace avbd

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

namespace
{

using namespace avbd::adjoint;

struct TapeStep
{
    int nMan = 0, nSolve = 0, iterations = 0;
    std::vector<int> colourStart;
    DArr<int2> ab;
    DArr<int> nc;
    DArr<float4> basis, geo;
    DArr<int> src;
    DArr<unsigned char> iflags;
    DArr<int> pairIdx;
    DArr<int> adjStart;
    DArr<unsigned> adj;
    DArr<int> solveList, colour;
    DArr<unsigned char> bflags;
    DArr<unsigned short> flags;
};

struct Checkpoint64
{
    int nMan = 0;        // contact slots held: 8 nMan
    DArr<double4> body;  // 5n: p, q, v, w, vp
    DArr<double4> lp;    // 16 nMan: lambda of every slot, then penalty
};

struct SegSnap
{
    DArr<double4> bodyIn, pose, lp, c0;
    DArr<double> ldl;
};

} // namespace

struct AdjointState
{
    int steps = 0, every = 0, nMan0 = 0;
    bool ready = false;
    AvbdParams params{}; // the forward's settings; the backward's replay needs the same
    int colourMode = 0;
    std::vector<TapeStep> tape;
    std::vector<Checkpoint64> ck; // replay state before step k * every
    Checkpoint64 last;            // replay state after the last step
    DArr<unsigned long long> keys;
    size_t nKeys = 0;
    DArr<unsigned long long> pairs;
    int P = 0;
    // FP32 scratch of the step being taped
    TapeStep *rec = nullptr;
    int prevMan = 0;
    DArr<unsigned long long> prevSeq;
    DArr<int> prevN;
    DArr<float4> prevLP, bodyIn32, pose32, lp32;
    // double-precision replay state
    DArr<double4> p, q, v, w, vp, iLin, iAng, tLin, tAng;
    DArr<double4> rlam[2], rpen[2], rc0;
    int rcur = 0;
    size_t rCap = 0;
    std::vector<SegSnap> snap; // two sets of `every` steps: replay of one segment, reverse of another
    // The double-precision replay runs on its own stream, overlapping the FP32 steps (forward)
    // and the reverse sweep of the next segment (backward); events order the two.
    cudaStream_t side = nullptr;
    cudaEvent_t evMain = nullptr, evSide = nullptr, evRep[2] = {nullptr, nullptr}, evRev[2] = {nullptr, nullptr};
    // adjoints
    DArr<double4> ap, aq, av, aw, avp, aiLin, aiAng, atLin, atAng;
    DArr<double> am, amu;
    DArr<double4> alam[2], apen[2], ac0;
    int lcur = 0;
    size_t lamCap = 0;
};

namespace
{

template <class T> int copy_d2d(AvbdContext *ctx, T *dst, const T *src, size_t count)
{
    if (count)
        CU(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));
    return AVBD_OK;
}

template <class T> int copy_on(AvbdContext *ctx, cudaStream_t st, T *dst, const T *src, size_t count)
{
    if (count)
        CU(cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyDeviceToDevice, st));
    return AVBD_OK;
}

int side_init(AvbdContext *ctx)
{
    AdjointState *a = ctx->adjoint;
    if (a->side)
        return AVBD_OK;
    CU(cudaStreamCreateWithFlags(&a->side, cudaStreamNonBlocking));
    for (cudaEvent_t *e : {&a->evMain, &a->evSide, &a->evRep[0], &a->evRep[1], &a->evRev[0], &a->evRev[1]})
        CU(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    return AVBD_OK;
}

// the replay stream waits for the work queued so far on the context stream, and back
int side_after_main(AvbdContext *ctx)
{
    AdjointState *a = ctx->adjoint;
    CU(cudaEventRecord(a->evMain, ctx->stream));
    CU(cudaStreamWaitEvent(a->side, a->evMain, 0));
    return AVBD_OK;
}

int main_after_side(AvbdContext *ctx)
{
    AdjointState *a = ctx->adjoint;
    CU(cudaEventRecord(a->evSide, a->side));
    CU(cudaStreamWaitEvent(ctx->stream, a->evSide, 0));
    return AVBD_OK;
}

// Growth of a buffer the replay stream uses: the context stream (which allocates and frees)
// first waits for the replay stream, and the replay stream then waits for the new buffer.
template <class T> int side_reserve(AvbdContext *ctx, DArr<T> &a, size_t count, bool preserve, size_t used = 0)
{
    if (count <= a.cap && a.p)
        return AVBD_OK;
    CHECK(main_after_side(ctx));
    CHECK(reserve(ctx, a, count, preserve, used));
    CHECK(side_after_main(ctx));
    return AVBD_OK;
}

void release_tape(TapeStep &s)
{
    release(s.ab);
    release(s.nc);
    release(s.basis);
    release(s.geo);
    release(s.src);
    release(s.iflags);
    release(s.pairIdx);
    release(s.adjStart);
    release(s.adj);
    release(s.solveList);
    release(s.colour);
    release(s.bflags);
    release(s.flags);
}

void adjoint_release(AvbdContext *ctx)
{
    AdjointState *a = ctx->adjoint;
    if (!a)
        return;
    if (a->side)
    {
        cudaStreamSynchronize(a->side);
        cudaStreamDestroy(a->side);
    }
    for (cudaEvent_t e : {a->evMain, a->evSide, a->evRep[0], a->evRep[1], a->evRev[0], a->evRev[1]})
        if (e)
            cudaEventDestroy(e);
    for (auto &s : a->tape)
        release_tape(s);
    for (auto &c : a->ck)
    {
        release(c.body);
        release(c.lp);
    }
    release(a->last.body);
    release(a->last.lp);
    for (auto &s : a->snap)
    {
        release(s.bodyIn);
        release(s.pose);
        release(s.lp);
        release(s.c0);
        release(s.ldl);
    }
    release(a->keys);
    release(a->pairs);
    release(a->prevSeq);
    release(a->prevN);
    for (DArr<float4> *d : {&a->prevLP, &a->bodyIn32, &a->pose32, &a->lp32})
        release(*d);
    for (DArr<double4> *d : {&a->p, &a->q, &a->v, &a->w, &a->vp, &a->iLin, &a->iAng, &a->tLin, &a->tAng, &a->rlam[0],
                             &a->rlam[1], &a->rpen[0], &a->rpen[1], &a->rc0, &a->ap, &a->aq, &a->av, &a->aw, &a->avp,
                             &a->aiLin, &a->aiAng, &a->atLin, &a->atAng, &a->alam[0], &a->alam[1], &a->apen[0],
                             &a->apen[1], &a->ac0})
        release(*d);
    release(a->am);
    release(a->amu);
    delete a;
    ctx->adjoint = nullptr;
}

void adjoint_invalidate(AvbdContext *ctx)
{
    if (ctx && ctx->adjoint)
        ctx->adjoint->ready = false;
}

// --- taping hooks called from step_once / iterate ---

int rec_step_begin(AvbdContext *ctx)
{
    AdjointState *a = ctx->adjoint;
    int n = ctx->n, M = ctx->nMan;
    CHECK(reserve(ctx, a->bodyIn32, (size_t)5 * std::max(n, 1), false));
    const DArr<float4> *src[5] = {&ctx->pos, &ctx->quat, &ctx->vel, &ctx->angvel, &ctx->prevVel};
    for (int k = 0; k < 5; ++k)
        CHECK(copy_d2d(ctx, a->bodyIn32.p + (size_t)k * n, src[k]->p, n));
    size_t m1 = (size_t)std::max(M, 1);
    CHECK(reserve(ctx, a->prevSeq, m1, false));
    CHECK(reserve(ctx, a->prevN, m1, false));
    CHECK(reserve(ctx, a->prevLP, 16 * m1, false));
    ManBuf &mb = ctx->man[ctx->cur];
    CHECK(copy_d2d(ctx, a->prevSeq.p, mb.seq.p, M));
    CHECK(copy_d2d(ctx, a->prevN.p, mb.n.p, M));
    if (M)
    {
        k_rec_lp<<<grid_for(8ll * M, 256), 256, 0, ctx->stream>>>(mb.contact.p, M, a->prevLP.p);
        LAUNCHED();
    }
    a->prevMan = M;
    return AVBD_OK;
}

int rec_prepared(AvbdContext *ctx)
{
    AdjointState *a = ctx->adjoint;
    TapeStep &s = *a->rec;
    int n = ctx->n, M = ctx->nMan;
    size_t m1 = (size_t)std::max(M, 1);
    ManBuf &mb = ctx->man[ctx->cur];
    s.nMan = M;
    s.iterations = ctx->params.iterations;
    CHECK(reserve(ctx, s.ab, m1, false));
    CHECK(reserve(ctx, s.nc, m1, false));
    CHECK(reserve(ctx, s.basis, 3 * m1, false));
    CHECK(reserve(ctx, s.geo, 16 * m1, false));
    CHECK(reserve(ctx, s.src, 8 * m1, false));
    CHECK(reserve(ctx, s.iflags, 8 * m1, false));
    CHECK(reserve(ctx, s.pairIdx, m1, false));
    CHECK(copy_d2d(ctx, s.ab.p, mb.ab.p, M));
    CHECK(copy_d2d(ctx, s.nc.p, mb.n.p, M));
    CHECK(copy_d2d(ctx, s.basis.p, mb.basis.p, 3 * (size_t)M));
    if (M)
    {
        k_rec_links<<<grid_for(8ll * M, 128), 128, 0, ctx->stream>>>(dev_man(mb), M, a->prevSeq.p, a->prevN.p,
                                                                      a->prevLP.p, a->prevMan, ctx->params.gamma,
                                                                      s.src.p, s.iflags.p);
        LAUNCHED();
    }
    // force lists of this step (n + 1 starts; the entry count is the last start)
    CHECK(reserve(ctx, s.adjStart, (size_t)n + 1, false));
    CHECK(copy_d2d(ctx, s.adjStart.p, ctx->adjStart.p, (size_t)n + 1));
    CU(cudaMemcpyAsync(ctx->hScalars + 2, ctx->adjStart.p + n, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    int nAdj = 0;
    std::memcpy(&nAdj, ctx->hScalars + 2, sizeof(int));
    CHECK(reserve(ctx, s.adj, (size_t)std::max(nAdj, 1), false));
    CHECK(copy_d2d(ctx, s.adj.p, ctx->adj.p, (size_t)nAdj));
    s.nSolve = ctx->nSolve;
    CHECK(reserve(ctx, s.solveList, (size_t)std::max(ctx->nSolve, 1), false));
    CHECK(copy_d2d(ctx, s.solveList.p, ctx->solveList.p, (size_t)ctx->nSolve));
    CHECK(reserve(ctx, s.colour, (size_t)std::max(n, 1), false));
    CHECK(copy_d2d(ctx, s.colour.p, ctx->colour.p, (size_t)n));
    s.colourStart = ctx->hColourStart;
    CHECK(reserve(ctx, s.bflags, (size_t)std::max(n, 1), false));
    k_tape_bflags<<<grid_for(n, 256), 256, 0, ctx->stream>>>(dev_bodies(ctx), a->bodyIn32.p, ctx->adjStart.p,
                                                             dev_params(ctx->params), s.bflags.p);
    LAUNCHED();
    size_t T1 = (size_t)s.iterations + 1;
    CHECK(reserve(ctx, a->pose32, T1 * 2 * (size_t)std::max(n, 1), false));
    CHECK(reserve(ctx, a->lp32, T1 * 16 * m1, false));
    return AVBD_OK;
}

int rec_iteration(AvbdContext *ctx, int it)
{
    AdjointState *a = ctx->adjoint;
    int n = ctx->n, M = ctx->nMan;
    k_rec_iteration<<<grid_for(std::max<long long>(n, 8ll * M), 256), 256, 0, ctx->stream>>>(
        ctx->pos.p, ctx->quat.p, n, ctx->man[ctx->cur].contact.p, M, a->pose32.p + (size_t)it * 2 * n,
        a->lp32.p + (size_t)it * 16 * M);
    LAUNCHED();
    return AVBD_OK;
}

// the records of a step whose iterations run in one launch (k_iterations writes into them)
int rec_tape(AvbdContext *ctx, IterTape *tape)
{
    AdjointState *a = ctx->adjoint;
    int n = ctx->n, M = ctx->nMan, slices = ctx->params.iterations + 1;
    k_rec_fill<<<grid_for(std::max<long long>(n, 8ll * M), 256), 256, 0, ctx->stream>>>(
        ctx->pos.p, ctx->quat.p, n, ctx->man[ctx->cur].contact.p, M, a->pose32.p, a->lp32.p, slices);
    LAUNCHED();
    tape->pose = a->pose32.p;
    tape->lp = a->lp32.p;
    tape->n = n;
    tape->nMan = M;
    return AVBD_OK;
}

// after the FP32 step: anchors and branch outcomes
int rec_finish(AvbdContext *ctx)
{
    AdjointState *a = ctx->adjoint;
    TapeStep &s = *a->rec;
    int M = s.nMan;
    size_t m1 = (size_t)std::max(M, 1);
    CHECK(reserve(ctx, s.flags, (size_t)s.iterations * 8 * m1, false));
    if (!M)
        return AVBD_OK;
    ManBuf &mb = ctx->man[ctx->cur];
    k_tape_geo<<<grid_for(8ll * M, 256), 256, 0, ctx->stream>>>(mb.contact.p, M, s.geo.p);
    LAUNCHED();
    Snap32 X;
    X.n = ctx->n;
    X.nMan = M;
    X.bodyIn = a->bodyIn32.p;
    X.pose = a->pose32.p;
    X.lp = a->lp32.p;
    X.contact = mb.contact.p;
    X.basis = mb.basis.p;
    X.ab = mb.ab.p;
    X.nc = mb.n.p;
    X.colour = s.colour.p;
    long long total = 8ll * M * s.iterations;
    k_tape_flags<<<grid_for(total, 128), 128, 0, ctx->stream>>>(X, dev_params(ctx->params), s.iterations,
                                                                 s.flags.p);
    LAUNCHED();
    return AVBD_OK;
}

StepTape tape_view(AvbdContext *ctx, const TapeStep &s)
{
    StepTape T;
    T.n = ctx->n;
    T.nMan = s.nMan;
    T.ab = s.ab.p;
    T.nc = s.nc.p;
    T.basis = s.basis.p;
    T.geo = s.geo.p;
    T.src = s.src.p;
    T.iflags = s.iflags.p;
    T.pairIdx = s.pairIdx.p;
    T.adjStart = s.adjStart.p;
    T.adj = s.adj.p;
    T.solveList = s.solveList.p;
    T.colour = s.colour.p;
    T.bflags = s.bflags.p;
    T.flags = s.flags.p;
    return T;
}

AdjParams adj_params(AvbdContext *ctx)
{
    AdjParams Q;
    Q.P = dev_params(ctx->params);
    Q.dt = ctx->params.dt;
    Q.g = ctx->params.gravity;
    Q.alpha = ctx->params.alpha;
    Q.beta = ctx->params.betaLin;
    Q.gamma = ctx->params.gamma;
    return Q;
}

// --- double-precision replay ---

int ensure_replay(AvbdContext *ctx, size_t slots)
{
    AdjointState *a = ctx->adjoint;
    if (slots <= a->rCap)
        return AVBD_OK;
    for (int k = 0; k < 2; ++k)
    {
        CHECK(side_reserve(ctx, a->rlam[k], slots, true, a->rCap));
        CHECK(side_reserve(ctx, a->rpen[k], slots, true, a->rCap));
    }
    CHECK(side_reserve(ctx, a->rc0, slots, false));
    a->rCap = std::min({a->rlam[0].cap, a->rlam[1].cap, a->rpen[0].cap, a->rpen[1].cap, a->rc0.cap});
    return AVBD_OK;
}

State64 state_view(AdjointState *a)
{
    State64 S;
    S.p = a->p.p;
    S.q = a->q.p;
    S.v = a->v.p;
    S.w = a->w.p;
    S.vp = a->vp.p;
    S.iLin = a->iLin.p;
    S.iAng = a->iAng.p;
    S.tLin = a->tLin.p;
    S.tAng = a->tAng.p;
    S.lam = a->rlam[a->rcur ^ 1].p;
    S.pen = a->rpen[a->rcur ^ 1].p;
    S.c0 = a->rc0.p;
    S.lamPrev = a->rlam[a->rcur].p;
    S.penPrev = a->rpen[a->rcur].p;
    return S;
}

int prev_man(AdjointState *a, int s) { return s > 0 ? a->tape[s - 1].nMan : a->nMan0; }

// Replays taped step s on the replay stream; with `snap`, keeps what the reverse sweep reads.
int replay_step(AvbdContext *ctx, int s, SegSnap *snap)
{
    AdjointState *a = ctx->adjoint;
    cudaStream_t st = a->side;
    const TapeStep &ts = a->tape[s];
    int n = ctx->n, M = ts.nMan;
    size_t m1 = (size_t)std::max(M, 1);
    CHECK(ensure_replay(ctx, 8 * (size_t)std::max({M, prev_man(a, s), 1})));
    StepTape T = tape_view(ctx, ts);
    State64 S = state_view(a);
    DevBodies B = dev_bodies(ctx);
    AdjParams Q = adj_params(ctx);
    size_t T1 = (size_t)ts.iterations + 1;
    if (snap)
    {
        CHECK(side_reserve(ctx, snap->bodyIn, 5 * (size_t)std::max(n, 1), false));
        CHECK(side_reserve(ctx, snap->pose, T1 * 2 * (size_t)std::max(n, 1), false));
        CHECK(side_reserve(ctx, snap->lp, T1 * 16 * m1, false));
        CHECK(side_reserve(ctx, snap->c0, 8 * m1, false));
        CHECK(side_reserve(ctx, snap->ldl, (size_t)ts.iterations * std::max(n, 1) * LDL_STRIDE, false));
        k_snapshot_bodies<<<grid_for(n, 256), 256, 0, st>>>(S, n, snap->bodyIn.p);
        LAUNCHED();
    }
    if (M)
    {
        k_rep_init<<<grid_for(8ll * M, 128), 128, 0, st>>>(T, S, Q);
        LAUNCHED();
    }
    if (snap)
        CHECK(copy_on(ctx, st, snap->c0.p, (const double4 *)S.c0, 8 * (size_t)M));
    k_rep_warm<<<grid_for(n, 128), 128, 0, st>>>(T, B, S, Q);
    LAUNCHED();
    int C = (int)ts.colourStart.size() - 1;
    auto snapshot = [&](int t) -> int {
        if (!snap)
            return AVBD_OK;
        k_snapshot<<<grid_for(std::max<long long>(n, 8ll * M), 256), 256, 0, st>>>(
            S, n, M, snap->pose.p + (size_t)t * 2 * n, snap->lp.p + (size_t)t * 16 * M);
        LAUNCHED();
        return AVBD_OK;
    };
    for (int t = 0; t < ts.iterations; ++t)
    {
        CHECK(snapshot(t));
        for (int c = 0; c < C; ++c)
        {
            int first = ts.colourStart[c], count = ts.colourStart[c + 1] - first;
            if (count <= 0)
                continue;
            k_rep_primal<<<grid_for(count, ADJ_BLOCK / ADJ_G), ADJ_BLOCK, 0, st>>>(
                T, B, S, Q, t, first, count, snap ? snap->ldl.p : nullptr);
            LAUNCHED();
        }
        if (M)
        {
            k_rep_dual<<<grid_for(8ll * M, 128), 128, 0, st>>>(T, S, Q, t);
            LAUNCHED();
        }
    }
    CHECK(snapshot(ts.iterations));
    k_rep_finish<<<grid_for(n, 128), 128, 0, st>>>(T, B, S, Q);
    LAUNCHED();
    a->rcur ^= 1;
    return AVBD_OK;
}

int save_replay(AvbdContext *ctx, Checkpoint64 &c, int nMan)
{
    AdjointState *a = ctx->adjoint;
    int n = ctx->n;
    CHECK(side_reserve(ctx, c.body, 5 * (size_t)std::max(n, 1), false));
    CHECK(side_reserve(ctx, c.lp, 16 * (size_t)std::max(nMan, 1), false));
    const DArr<double4> *src[5] = {&a->p, &a->q, &a->v, &a->w, &a->vp};
    for (int k = 0; k < 5; ++k)
        CHECK(copy_on(ctx, a->side, c.body.p + (size_t)k * n, (const double4 *)src[k]->p, n));
    CHECK(copy_on(ctx, a->side, c.lp.p, (const double4 *)a->rlam[a->rcur].p, 8 * (size_t)nMan));
    CHECK(copy_on(ctx, a->side, c.lp.p + 8 * (size_t)nMan, (const double4 *)a->rpen[a->rcur].p, 8 * (size_t)nMan));
    c.nMan = nMan;
    return AVBD_OK;
}

int restore_replay(AvbdContext *ctx, const Checkpoint64 &c)
{
    AdjointState *a = ctx->adjoint;
    int n = ctx->n;
    CHECK(ensure_replay(ctx, 8 * (size_t)std::max(c.nMan, 1)));
    DArr<double4> *dst[5] = {&a->p, &a->q, &a->v, &a->w, &a->vp};
    for (int k = 0; k < 5; ++k)
        CHECK(copy_on(ctx, a->side, dst[k]->p, (const double4 *)c.body.p + (size_t)k * n, n));
    CHECK(copy_on(ctx, a->side, a->rlam[a->rcur].p, (const double4 *)c.lp.p, 8 * (size_t)c.nMan));
    CHECK(copy_on(ctx, a->side, a->rpen[a->rcur].p, (const double4 *)c.lp.p + 8 * (size_t)c.nMan, 8 * (size_t)c.nMan));
    return AVBD_OK;
}

// --- reverse sweep ---

AdjView adj_view(AdjointState *a)
{
    AdjView A;
    A.p = a->ap.p;
    A.q = a->aq.p;
    A.v = a->av.p;
    A.w = a->aw.p;
    A.vp = a->avp.p;
    A.iLin = a->aiLin.p;
    A.iAng = a->aiAng.p;
    A.tLin = a->atLin.p;
    A.tAng = a->atAng.p;
    A.m = a->am.p;
    A.lam = a->alam[a->lcur].p;
    A.pen = a->apen[a->lcur].p;
    A.lamPrev = a->alam[a->lcur ^ 1].p;
    A.penPrev = a->apen[a->lcur ^ 1].p;
    A.c0 = a->ac0.p;
    A.mu = a->amu.p;
    return A;
}

int ensure_contact_adjoints(AvbdContext *ctx, size_t slots)
{
    AdjointState *a = ctx->adjoint;
    if (slots <= a->lamCap)
        return AVBD_OK;
    for (int k = 0; k < 2; ++k)
    {
        CHECK(reserve(ctx, a->alam[k], slots, true, a->lamCap));
        CHECK(reserve(ctx, a->apen[k], slots, true, a->lamCap));
    }
    CHECK(reserve(ctx, a->ac0, slots, false));
    a->lamCap = std::min({a->alam[0].cap, a->alam[1].cap, a->apen[0].cap, a->apen[1].cap, a->ac0.cap});
    return AVBD_OK;
}

Snap64 snap_view(const SegSnap &s)
{
    Snap64 X;
    X.bodyIn = s.bodyIn.p;
    X.pose = s.pose.p;
    X.lp = s.lp.p;
    X.c0 = s.c0.p;
    X.ldl = s.ldl.p;
    return X;
}

// On entry the body adjoints refer to the state after step s and the contact adjoints to
// step s's list; on exit to the state before it and the previous step's list.
int reverse_step(AvbdContext *ctx, int s, const SegSnap &snap)
{
    AdjointState *a = ctx->adjoint;
    const TapeStep &ts = a->tape[s];
    int n = ctx->n, M = ts.nMan, Mp = prev_man(a, s);
    CHECK(ensure_contact_adjoints(ctx, 8 * (size_t)std::max({M, Mp, 1})));
    StepTape T = tape_view(ctx, ts);
    Snap64 X = snap_view(snap);
    DevBodies B = dev_bodies(ctx);
    AdjParams Q = adj_params(ctx);
    AdjView A = adj_view(a);
    CU(cudaMemsetAsync(A.c0, 0, sizeof(double4) * 8 * (size_t)std::max(M, 1), ctx->stream));
    k_adj_finish<<<grid_for(n, 128), 128, 0, ctx->stream>>>(T, X, B, A, Q, ts.iterations);
    LAUNCHED();
    int C = (int)ts.colourStart.size() - 1;
    for (int t = ts.iterations - 1; t >= 0; --t)
    {
        if (M)
        {
            k_adj_dual<<<grid_for(8ll * M, 128), 128, 0, ctx->stream>>>(T, X, B, A, Q, t);
            LAUNCHED();
        }
        for (int c = C - 1; c >= 0; --c)
        {
            int first = ts.colourStart[c], count = ts.colourStart[c + 1] - first;
            if (count <= 0)
                continue;
            k_adj_primal<<<grid_for(count, ADJ_BLOCK / ADJ_G), ADJ_BLOCK, 0, ctx->stream>>>(T, X, B, A, Q, t, c,
                                                                                              first, count);
            LAUNCHED();
        }
    }
    CU(cudaMemsetAsync(A.lamPrev, 0, sizeof(double4) * 8 * (size_t)std::max(Mp, 1), ctx->stream));
    CU(cudaMemsetAsync(A.penPrev, 0, sizeof(double4) * 8 * (size_t)std::max(Mp, 1), ctx->stream));
    if (M)
    {
        k_adj_init<<<grid_for(8ll * M, 128), 128, 0, ctx->stream>>>(T, X, B, A, Q);
        LAUNCHED();
    }
    k_adj_warm<<<grid_for(n, 128), 128, 0, ctx->stream>>>(T, X, B, A, Q);
    LAUNCHED();
    a->lcur ^= 1;
    return AVBD_OK;
}

int adjoint_guard(AvbdContext *ctx)
{
    if (!ctx)
        return AVBD_ERR_ARGUMENT;
    if (ctx->errCode)
        return AVBD_ERR_LATCHED;
    if (!ctx->loaded)
        return fail(ctx, AVBD_ERR_STATE, "no world loaded");
    CU(cudaSetDevice(ctx->device));
    return AVBD_OK;
}

int adjoint_ready(AvbdContext *ctx, const char *what)
{
    CHECK(adjoint_guard(ctx));
    AdjointState *a = ctx->adjoint;
    if (!a || !a->ready)
        return fail(ctx, AVBD_ERR_STATE, "%s: run avbd_adjoint_forward first (the world has not changed since)",
                    what);
    return AVBD_OK;
}

} // namespace

extern "C"
{

int avbd_adjoint_forward(AvbdContext *ctx, int32_t nsteps, int32_t checkpoint_every)
{
    SETTLED();
    CHECK(adjoint_guard(ctx));
    if (nsteps < 1 || checkpoint_every < 1)
        return fail(ctx, AVBD_ERR_ARGUMENT, "adjoint_forward: nsteps and checkpoint_every must be positive");
    if (ctx->nJoint > 0 || ctx->nSpring > 0)
        return fail(ctx, AVBD_ERR_ARGUMENT,
                    "adjoint_forward: the differentiable step covers contacts; the world has joints or springs");
    if (ctx->hasShapes)
        return fail(ctx, AVBD_ERR_ARGUMENT,
                    "adjoint_forward: the differentiable step covers boxes; the world has round bodies");
    if (ctx->params.iterations < 1)
        return fail(ctx, AVBD_ERR_ARGUMENT, "adjoint_forward: needs at least one solver iteration");
    if (!ctx->adjoint)
        ctx->adjoint = new AdjointState();
    AdjointState *a = ctx->adjoint;
    a->ready = false;
    a->steps = nsteps;
    a->every = checkpoint_every;
    a->params = ctx->params;
    a->colourMode = ctx->colourMode;
    for (size_t k = nsteps; k < a->tape.size(); ++k)
        release_tape(a->tape[k]);
    a->tape.resize(nsteps);
    int nck = (nsteps + checkpoint_every - 1) / checkpoint_every;
    for (size_t k = nck; k < a->ck.size(); ++k)
    {
        release(a->ck[k].body);
        release(a->ck[k].lp);
    }
    a->ck.resize(nck);
    a->nKeys = 0;
    // the replay starts from the FP32 state
    int n = ctx->n;
    size_t n1 = (size_t)std::max(n, 1);
    for (DArr<double4> *d : {&a->p, &a->q, &a->v, &a->w, &a->vp, &a->iLin, &a->iAng, &a->tLin, &a->tAng})
        CHECK(reserve(ctx, *d, n1, false));
    a->nMan0 = ctx->nMan;
    a->rcur = 0;
    CHECK(side_init(ctx));
    CHECK(ensure_replay(ctx, 8 * (size_t)std::max(ctx->nMan, 1)));
    k_state_to_double<<<grid_for(n, 256), 256, 0, ctx->stream>>>(dev_bodies(ctx), state_view(a));
    LAUNCHED();
    if (ctx->nMan)
    {
        k_lp_to_double<<<grid_for(8ll * ctx->nMan, 256), 256, 0, ctx->stream>>>(
            ctx->man[ctx->cur].contact.p, ctx->nMan, a->rlam[a->rcur].p, a->rpen[a->rcur].p);
        LAUNCHED();
    }
    CHECK(side_after_main(ctx));
    for (int s = 0; s < nsteps; ++s)
    {
        if (s % checkpoint_every == 0)
            CHECK(save_replay(ctx, a->ck[s / checkpoint_every], prev_man(a, s)));
        a->rec = &a->tape[s];
        ctx->recording = true;
        int rc = step_once(ctx);
        ctx->recording = false;
        CHECK(rc);
        CHECK(rec_finish(ctx));
        a->rec = nullptr;
        if (ctx->nMan)
        {
            CHECK(reserve(ctx, a->keys, a->nKeys + ctx->nMan, true, a->nKeys));
            k_pair_keys<<<grid_for(ctx->nMan, 256), 256, 0, ctx->stream>>>(ctx->man[ctx->cur].ab.p, ctx->nMan,
                                                                          a->keys.p + a->nKeys);
            LAUNCHED();
            a->nKeys += ctx->nMan;
        }
        // step s is taped: its replay runs while the next FP32 step proceeds
        CHECK(side_after_main(ctx));
        CHECK(replay_step(ctx, s, nullptr));
    }
    CHECK(save_replay(ctx, a->last, a->tape.back().nMan));
    CHECK(main_after_side(ctx));
    CHECK(prof_collect(ctx));
    // friction pairs: sorted unique (min, max) body pairs of every manifold met
    int P = 0;
    if (a->nKeys)
    {
        DArr<unsigned long long> sorted;
        CHECK(reserve(ctx, sorted, a->nKeys, false));
        CHECK(reserve(ctx, a->pairs, a->nKeys, false));
        CHECK(reserve(ctx, ctx->keepIdx, 2, false));
        int *numOut = ctx->keepIdx.p;
        size_t bytes = 0;
        cub::DeviceRadixSort::SortKeys(nullptr, bytes, a->keys.p, sorted.p, (int)a->nKeys, 0, 64, ctx->stream);
        CHECK(ensure_temp(ctx, bytes));
        CU(cub::DeviceRadixSort::SortKeys(ctx->cubTemp.p, bytes, a->keys.p, sorted.p, (int)a->nKeys, 0, 64,
                                          ctx->stream));
        bytes = 0;
        cub::DeviceSelect::Unique(nullptr, bytes, sorted.p, a->pairs.p, numOut, (int)a->nKeys, ctx->stream);
        CHECK(ensure_temp(ctx, bytes));
        CU(cub::DeviceSelect::Unique(ctx->cubTemp.p, bytes, sorted.p, a->pairs.p, numOut, (int)a->nKeys,
                                     ctx->stream));
        CU(cudaMemcpyAsync(ctx->hScalars + 3, numOut, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        std::memcpy(&P, ctx->hScalars + 3, sizeof(int));
        CU(cudaFreeAsync(sorted.p, ctx->stream));
    }
    a->P = P;
    for (auto &ts : a->tape)
        if (ts.nMan)
        {
            k_pair_index<<<grid_for(ts.nMan, 256), 256, 0, ctx->stream>>>(ts.ab.p, ts.nMan, a->pairs.p, P,
                                                                         ts.pairIdx.p);
            LAUNCHED();
        }
    CU(cudaStreamSynchronize(ctx->stream));
    a->ready = true;
    return AVBD_OK;
}

int avbd_adjoint_num_pairs(AvbdContext *ctx, int32_t *count)
{
    SETTLED();
    CHECK(adjoint_ready(ctx, "adjoint_num_pairs"));
    if (!count)
        return fail(ctx, AVBD_ERR_ARGUMENT, "adjoint_num_pairs: null output");
    *count = ctx->adjoint->P;
    return AVBD_OK;
}

int avbd_adjoint_read_pairs(AvbdContext *ctx, int32_t *lohi2, float *friction)
{
    SETTLED();
    CHECK(adjoint_ready(ctx, "adjoint_read_pairs"));
    AdjointState *a = ctx->adjoint;
    std::vector<unsigned long long> keys(std::max(a->P, 1));
    if (a->P)
        CU(cudaMemcpyAsync(keys.data(), a->pairs.p, sizeof(unsigned long long) * a->P, cudaMemcpyDeviceToHost,
                           ctx->stream));
    std::vector<float> fr(std::max(ctx->n, 1));
    if (ctx->n)
        CU(cudaMemcpyAsync(fr.data(), ctx->friction.p, sizeof(float) * ctx->n, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < a->P; ++i)
    {
        int lo = (int)(keys[i] >> 32), hi = (int)(keys[i] & 0xFFFFFFFFull);
        if (lohi2)
        {
            lohi2[2 * i] = lo;
            lohi2[2 * i + 1] = hi;
        }
        if (friction)
            friction[i] = sqrtf(fr[lo] * fr[hi]); // Manifold::initialize (manifold.cpp:103)
    }
    return AVBD_OK;
}

int avbd_adjoint_replay_state(AvbdContext *ctx, double *position3, double *orientation4, double *velocity3,
                              double *angular_velocity3)
{
    SETTLED();
    CHECK(adjoint_ready(ctx, "adjoint_replay_state"));
    AdjointState *a = ctx->adjoint;
    int n = ctx->n;
    std::vector<double4> h((size_t)5 * std::max(n, 1));
    if (n)
        CU(cudaMemcpyAsync(h.data(), a->last.body.p, sizeof(double4) * 5 * (size_t)n, cudaMemcpyDeviceToHost,
                           ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    double *dst[4] = {position3, orientation4, velocity3, angular_velocity3};
    const int dim[4] = {3, 4, 3, 3};
    const int field[4] = {0, 1, 2, 3}; // p, q, v, w
    for (int k = 0; k < 4; ++k)
    {
        if (!dst[k])
            continue;
        for (int b = 0; b < n; ++b)
        {
            const double4 &x = h[(size_t)field[k] * n + b];
            const double v[4] = {x.x, x.y, x.z, x.w};
            for (int c = 0; c < dim[k]; ++c)
                dst[k][(size_t)dim[k] * b + c] = v[c];
        }
    }
    return AVBD_OK;
}

int avbd_adjoint_tape_step(AvbdContext *ctx, int32_t step, int32_t *num_manifolds, uint16_t *flags,
                           uint8_t *body_flags, int32_t *link)
{
    SETTLED();
    CHECK(adjoint_ready(ctx, "adjoint_tape_step"));
    AdjointState *a = ctx->adjoint;
    if (step < 0 || step >= a->steps)
        return fail(ctx, AVBD_ERR_ARGUMENT, "adjoint_tape_step: step %d outside [0, %d)", step, a->steps);
    const TapeStep &s = a->tape[step];
    if (num_manifolds)
        *num_manifolds = s.nMan;
    if (flags && s.nMan)
        CU(cudaMemcpyAsync(flags, s.flags.p, sizeof(uint16_t) * (size_t)s.iterations * 8 * s.nMan,
                           cudaMemcpyDeviceToHost, ctx->stream));
    if (body_flags && ctx->n)
        CU(cudaMemcpyAsync(body_flags, s.bflags.p, ctx->n, cudaMemcpyDeviceToHost, ctx->stream));
    if (link && s.nMan)
        CU(cudaMemcpyAsync(link, s.src.p, sizeof(int32_t) * 8 * (size_t)s.nMan, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    return AVBD_OK;
}

int avbd_adjoint_backward(AvbdContext *ctx, const double *d_position3, const double *d_orientation4,
                          const double *d_velocity3, const double *d_angular_velocity3, const AvbdAdjointGrad *out)
{
    SETTLED();
    CHECK(adjoint_ready(ctx, "adjoint_backward"));
    AdjointState *a = ctx->adjoint;
    if (!out)
        return fail(ctx, AVBD_ERR_ARGUMENT, "adjoint_backward: null output");
    if (std::memcmp(&a->params, &ctx->params, sizeof(AvbdParams)) != 0 || a->colourMode != ctx->colourMode)
        return fail(ctx, AVBD_ERR_STATE, "adjoint_backward: parameters or colouring changed since adjoint_forward");
    int n = ctx->n;
    size_t n1 = (size_t)std::max(n, 1);
    for (DArr<double4> *d : {&a->ap, &a->aq, &a->av, &a->aw, &a->avp, &a->aiLin, &a->aiAng, &a->atLin, &a->atAng})
        CHECK(reserve(ctx, *d, n1, false));
    CHECK(reserve(ctx, a->am, n1, false));
    CHECK(reserve(ctx, a->amu, (size_t)std::max(a->P, 1), false));
    CU(cudaMemsetAsync(a->am.p, 0, sizeof(double) * n1, ctx->stream));
    CU(cudaMemsetAsync(a->amu.p, 0, sizeof(double) * std::max(a->P, 1), ctx->stream));
    // seed: the adjoint of the final state
    std::vector<double4> h(n1);
    auto seed = [&](DArr<double4> &dst, const double *src, int dim) -> int {
        for (int b = 0; b < n; ++b)
        {
            double x[4] = {0, 0, 0, 0};
            if (src)
                for (int k = 0; k < dim; ++k)
                    x[k] = src[(size_t)dim * b + k];
            h[b] = make_double4(x[0], x[1], x[2], x[3]);
        }
        CU(cudaMemcpyAsync(dst.p, h.data(), sizeof(double4) * n, cudaMemcpyHostToDevice, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        return AVBD_OK;
    };
    CHECK(seed(a->ap, d_position3, 3));
    CHECK(seed(a->aq, d_orientation4, 4));
    CHECK(seed(a->av, d_velocity3, 3));
    CHECK(seed(a->aw, d_angular_velocity3, 3));
    CU(cudaMemsetAsync(a->avp.p, 0, sizeof(double4) * n1, ctx->stream));
    size_t finalSlots = 8 * (size_t)std::max(a->tape.back().nMan, 1);
    CHECK(ensure_contact_adjoints(ctx, finalSlots));
    a->lcur = 0;
    CU(cudaMemsetAsync(a->alam[0].p, 0, sizeof(double4) * finalSlots, ctx->stream));
    CU(cudaMemsetAsync(a->apen[0].p, 0, sizeof(double4) * finalSlots, ctx->stream));

    int every = a->every;
    if ((int)a->snap.size() < 2 * every)
        a->snap.resize(2 * every);
    int nck = (int)a->ck.size();
    CHECK(side_init(ctx));
    CHECK(side_after_main(ctx));
    // Segment k is replayed into snapshot set k % 2 on the replay stream while segment k + 1
    // is reversed on the context stream; a set is refilled only after the reverse that read
    // it has finished.
    auto replay_segment = [&](int seg) -> int {
        int set = seg & 1;
        int s0 = seg * every, s1 = std::min(a->steps, s0 + every);
        CHECK(restore_replay(ctx, a->ck[seg]));
        for (int s = s0; s < s1; ++s)
            CHECK(replay_step(ctx, s, &a->snap[set * every + (s - s0)]));
        CU(cudaEventRecord(a->evRep[set], a->side));
        return AVBD_OK;
    };
    CHECK(replay_segment(nck - 1));
    for (int seg = nck - 1; seg >= 0; --seg)
    {
        int set = seg & 1;
        if (seg > 0)
        {
            if (seg + 1 < nck)
                CU(cudaStreamWaitEvent(a->side, a->evRev[(seg - 1) & 1], 0));
            CHECK(replay_segment(seg - 1));
        }
        CU(cudaStreamWaitEvent(ctx->stream, a->evRep[set], 0));
        int s0 = seg * every, s1 = std::min(a->steps, s0 + every);
        for (int s = s1 - 1; s >= s0; --s)
            CHECK(reverse_step(ctx, s, a->snap[set * every + (s - s0)]));
        CU(cudaEventRecord(a->evRev[set], ctx->stream));
    }
    CHECK(main_after_side(ctx));
    // outputs
    auto fetch = [&](const DArr<double4> &src, double *dst, int dim) -> int {
        if (!dst)
            return AVBD_OK;
        CU(cudaMemcpyAsync(h.data(), src.p, sizeof(double4) * n, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        for (int b = 0; b < n; ++b)
        {
            const double x[4] = {h[b].x, h[b].y, h[b].z, h[b].w};
            for (int k = 0; k < dim; ++k)
                dst[(size_t)dim * b + k] = x[k];
        }
        return AVBD_OK;
    };
    CHECK(fetch(a->ap, out->position, 3));
    CHECK(fetch(a->aq, out->orientation, 4));
    CHECK(fetch(a->av, out->velocity, 3));
    CHECK(fetch(a->aw, out->angular_velocity, 3));
    CHECK(fetch(a->avp, out->prev_velocity, 3));
    if (out->mass && n)
        CU(cudaMemcpyAsync(out->mass, a->am.p, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<double> gmu(std::max(a->P, 1));
    if (a->P)
        CU(cudaMemcpyAsync(gmu.data(), a->amu.p, sizeof(double) * a->P, cudaMemcpyDeviceToHost, ctx->stream));
    CU(cudaStreamSynchronize(ctx->stream));
    if (out->pair_friction && a->P)
        std::memcpy(out->pair_friction, gmu.data(), sizeof(double) * a->P);
    if (out->body_friction)
    {
        // mu = sqrt(mu_a mu_b) (manifold.cpp:103): dmu / dmu_a = mu_b / (2 mu)
        std::vector<unsigned long long> keys(std::max(a->P, 1));
        std::vector<float> fr(n1);
        if (a->P)
            CU(cudaMemcpyAsync(keys.data(), a->pairs.p, sizeof(unsigned long long) * a->P, cudaMemcpyDeviceToHost,
                               ctx->stream));
        if (n)
            CU(cudaMemcpyAsync(fr.data(), ctx->friction.p, sizeof(float) * n, cudaMemcpyDeviceToHost, ctx->stream));
        CU(cudaStreamSynchronize(ctx->stream));
        for (int b = 0; b < n; ++b)
            out->body_friction[b] = 0.0;
        for (int i = 0; i < a->P; ++i)
        {
            int lo = (int)(keys[i] >> 32), hi = (int)(keys[i] & 0xFFFFFFFFull);
            double mu = std::sqrt((double)fr[lo] * (double)fr[hi]);
            if (mu > 0)
            {
                out->body_friction[lo] += gmu[i] * fr[hi] / (2.0 * mu);
                out->body_friction[hi] += gmu[i] * fr[lo] / (2.0 * mu);
            }
        }
    }
    return AVBD_OK;
}

} // extern "C"
