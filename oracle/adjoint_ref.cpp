/*
 * FP64 frozen-branch replay and reference adjoint of the AVBD step -- TEST
 * INFRASTRUCTURE, not part of the product. Only the tests and the benchmark's checks load
 * it (it is linked into oracle/liboracle.so).
 *
 * The oracle (avbd_oracle.c) records, for every step of an FP32 run, the integer decisions
 * the differentiable step holds fixed: the manifolds after Manifold::initialize with their
 * feature-matched links to the previous step (manifold.cpp:119-160), the contact geometry,
 * the primal sweep order, and the branch outcome of every contact evaluation
 * (manifold.cpp:200-212, 268-278), warm-start clamp (manifold.cpp:170) and adaptive
 * warm-start weight (solver.cpp:1146-1150). On that tape:
 *   adjref_loss      replays the step in double precision for any parameter vector
 *                    (initial velocities, masses, per-pair friction) and returns the loss
 *                    |COM(x_T) - target|^2 over the dynamic bodies;
 *   adjref_gradient  the reference adjoint: the exact gradient of that replay, by a serial
 *                    reverse sweep (bodies in reverse sweep order, one at a time, so it does
 *                    not rely on the colouring the CUDA adjoint uses);
 *   adjref_fd        central finite differences of adjref_loss along given directions,
 *                    threaded over the directions.
 * The per-element maps and their VJPs come from avbd_demo3d_b200/csrc/avbd_diff.h.
 *
 * Parity: the reference computes no gradients, so this path is parity unpinned by the
 * reference. The tape comes from the oracle's FP32 run, which is bit-exact to the reference;
 * the gradients are pinned by central finite differences of the double-precision replay
 * (tests/test_adjoint_ref.py, tests/test_gpu_adjoint.py).
 *
 * Parameter vector (list order of bodies, n bodies, P friction pairs):
 *   [ v0 (3n) | w0 (3n) | mass (n) | mu (P) ]
 * v0 is the constructor velocity: it sets the velocity and the previous velocity
 * together (rigid.cpp:24-27); mass scales the moment (rigid.cpp:34-39); mu replaces
 * sqrt(muA muB) (manifold.cpp:103) for every manifold of the pair, pairs ordered by
 * (min(a, b), max(a, b)).
 */
#include "avbd_oracle.h"

#include "../avbd_demo3d_b200/csrc/avbd_diff.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <thread>
#include <vector>

using namespace avbd_diff;
typedef double S;

static_assert((int)ORACLE_EF_NCLAMP == (int)EF_NCLAMP && (int)ORACLE_EF_CONE == (int)EF_CONE &&
                  (int)ORACLE_EF_RAMP_T == (int)EF_RAMP_T && (int)ORACLE_EF_CAP_X == (int)EF_CAP_X &&
                  (int)ORACLE_EF_NEG_X == (int)EF_NEG_X && (int)ORACLE_EF_POS_X == (int)EF_POS_X &&
                  (int)ORACLE_EF_POS_Z == (int)EF_POS_Z,
              "flag layout");
static_assert((int)ORACLE_IF_LO_X == (int)IF_LO_X && (int)ORACLE_IF_HI_Z == (int)IF_HI_Z, "init flag layout");
static_assert((int)ORACLE_BF_DYNAMIC == (int)BF_DYNAMIC && (int)ORACLE_BF_FORCES == (int)BF_FORCES &&
                  (int)ORACLE_BF_ACCEL_IN == (int)BF_ACCEL_IN && (int)ORACLE_BF_ACCEL_ONE == (int)BF_ACCEL_ONE,
              "body flag layout");

namespace
{

struct Problem
{
    OracleParams p{};
    int n = 0, steps = 0, P = 0;
    std::vector<const OracleTapeStep *> st;
    std::vector<S> mass0;
    std::vector<V3<S>> shape;
    std::vector<unsigned long long> pairKeys;      // sorted (lo << 32 | hi)
    std::vector<float> pairMu0;
    std::vector<std::vector<int>> manPair;         // per step, per manifold
    std::vector<std::vector<int>> bodyStart;       // per step: n + 1 ranges into bodyMan
    std::vector<std::vector<int>> bodyMan;         // per step: manifold * 2 + (isA ? 1 : 0)
    V3<S> vel0Offset(int b) const                  // nominal prevVel - vel at step 0
    {
        const float *x = st[0]->bodyIn + 16 * (size_t)b;
        return v3<S>((S)x[13] - (S)x[7], (S)x[14] - (S)x[8], (S)x[15] - (S)x[9]);
    }
};

V3<S> ld3(const float *f) { return v3<S>(f[0], f[1], f[2]); }
Q4<S> ld4(const float *f) { return q4<S>(f[0], f[1], f[2], f[3]); }

bool build_problem(const OracleWorld *w, Problem &pb)
{
    oracle_get_params(w, &pb.p);
    pb.n = oracle_num_bodies(w);
    pb.steps = oracle_tape_steps(w);
    if (pb.steps <= 0)
        return false;
    int n = pb.n;
    std::vector<float> mass(n), moment(3 * (size_t)n);
    oracle_get_body_props(w, mass.data(), moment.data(), nullptr, nullptr, nullptr);
    pb.mass0.resize(n);
    pb.shape.resize(n);
    for (int b = 0; b < n; ++b)
    {
        pb.mass0[b] = mass[b];
        pb.shape[b] = mass[b] > 0 ? v3<S>((S)moment[3 * b] / mass[b], (S)moment[3 * b + 1] / mass[b],
                                          (S)moment[3 * b + 2] / mass[b])
                                  : vzero<S>();
    }
    pb.st.resize(pb.steps);
    std::vector<std::pair<unsigned long long, float>> keys;
    for (int s = 0; s < pb.steps; ++s)
    {
        pb.st[s] = oracle_tape_step(w, s);
        const OracleTapeStep *t = pb.st[s];
        for (int m = 0; m < t->nMan; ++m)
        {
            unsigned a = (unsigned)t->ab[2 * m], b = (unsigned)t->ab[2 * m + 1];
            unsigned lo = std::min(a, b), hi = std::max(a, b);
            keys.push_back({((unsigned long long)lo << 32) | hi, t->friction[m]});
        }
    }
    std::sort(keys.begin(), keys.end(),
              [](const std::pair<unsigned long long, float> &x, const std::pair<unsigned long long, float> &y) {
                  return x.first < y.first;
              });
    for (size_t i = 0; i < keys.size(); ++i)
        if (i == 0 || keys[i].first != keys[i - 1].first)
        {
            pb.pairKeys.push_back(keys[i].first);
            pb.pairMu0.push_back(keys[i].second);
        }
    pb.P = (int)pb.pairKeys.size();
    pb.manPair.resize(pb.steps);
    pb.bodyStart.resize(pb.steps);
    pb.bodyMan.resize(pb.steps);
    for (int s = 0; s < pb.steps; ++s)
    {
        const OracleTapeStep *t = pb.st[s];
        pb.manPair[s].resize(t->nMan);
        std::vector<int> cnt(n + 1, 0);
        for (int m = 0; m < t->nMan; ++m)
        {
            unsigned a = (unsigned)t->ab[2 * m], b = (unsigned)t->ab[2 * m + 1];
            unsigned long long k = ((unsigned long long)std::min(a, b) << 32) | std::max(a, b);
            pb.manPair[s][m] = (int)(std::lower_bound(pb.pairKeys.begin(), pb.pairKeys.end(), k) - pb.pairKeys.begin());
            cnt[a + 1]++;
            cnt[b + 1]++;
        }
        for (int b = 0; b < n; ++b)
            cnt[b + 1] += cnt[b];
        pb.bodyStart[s] = cnt;
        pb.bodyMan[s].assign(cnt[n], 0);
        // each body's rows newest manifold first, the order of the reference's per-body force
        // lists (force.cpp:25-36); manifolds are in creation order
        std::vector<int> fill(cnt.begin(), cnt.end() - 1);
        for (int m = t->nMan - 1; m >= 0; --m)
        {
            pb.bodyMan[s][fill[t->ab[2 * m]]++] = 2 * m + 1;
            pb.bodyMan[s][fill[t->ab[2 * m + 1]]++] = 2 * m;
        }
    }
    return true;
}

int num_params(const Problem &pb) { return 7 * pb.n + pb.P; }

void theta0(const Problem &pb, S *th)
{
    int n = pb.n;
    for (int b = 0; b < n; ++b)
    {
        const float *x = pb.st[0]->bodyIn + 16 * (size_t)b;
        for (int k = 0; k < 3; ++k)
        {
            th[3 * b + k] = x[7 + k];
            th[3 * n + 3 * b + k] = x[10 + k];
        }
        th[6 * n + b] = pb.mass0[b];
    }
    for (int i = 0; i < pb.P; ++i)
        th[7 * n + i] = pb.pairMu0[i];
}

// Dynamic state between steps.
struct State
{
    std::vector<V3<S>> p, v, w, vp;
    std::vector<Q4<S>> q;
    std::vector<V3<S>> lam, pen; // contact slots of the previous step's list
};

// Within one step.
struct StepWork
{
    std::vector<V3<S>> initLin, inertLin;
    std::vector<Q4<S>> initAng, inertAng;
    std::vector<ContactIn<S>> c; // slots of this step's list
};

void initial_state(const Problem &pb, const S *th, State &X)
{
    int n = pb.n;
    X.p.resize(n);
    X.q.resize(n);
    X.v.resize(n);
    X.w.resize(n);
    X.vp.resize(n);
    for (int b = 0; b < n; ++b)
    {
        const float *x = pb.st[0]->bodyIn + 16 * (size_t)b;
        X.p[b] = ld3(x);
        X.q[b] = ld4(x + 3);
        X.v[b] = v3<S>(th[3 * b], th[3 * b + 1], th[3 * b + 2]);
        X.w[b] = v3<S>(th[3 * n + 3 * b], th[3 * n + 3 * b + 1], th[3 * n + 3 * b + 2]);
        X.vp[b] = X.v[b] + pb.vel0Offset(b);
    }
    X.lam.clear();
    X.pen.clear();
}

Pose<S> pose_of(const std::vector<V3<S>> &p, const std::vector<Q4<S>> &q, const StepWork &W, int b)
{
    Pose<S> r;
    r.p = p[b];
    r.q = q[b];
    r.pi = W.initLin[b];
    r.qi = W.initAng[b];
    return r;
}

// Manifold::initialize on the tape and the body warm start.
void prepare(const Problem &pb, int s, const S *th, State &X, StepWork &W)
{
    const OracleTapeStep *t = pb.st[s];
    int n = pb.n;
    S alpha = pb.p.alpha, gamma = pb.p.gamma, dt = pb.p.dt, g = pb.p.gravity;
    W.c.assign((size_t)t->nMan * 8, ContactIn<S>());
    for (int m = 0; m < t->nMan; ++m)
    {
        int a = t->ab[2 * m], b = t->ab[2 * m + 1];
        V3<S> e[3];
        for (int k = 0; k < 3; ++k)
            e[k] = ld3(t->basis + 9 * (size_t)m + 3 * k);
        S mu = th[7 * n + pb.manPair[s][m]];
        for (int k = 0; k < t->ncontacts[m]; ++k)
        {
            size_t slot = (size_t)m * 8 + k;
            ContactIn<S> &c = W.c[slot];
            c.rA = ld3(t->geo + 6 * slot);
            c.rB = ld3(t->geo + 6 * slot + 3);
            for (int r = 0; r < 3; ++r)
                c.e[r] = e[r];
            c.mu = mu;
            c.C0 = contact_C0(X.p[a], X.q[a], X.p[b], X.q[b], c.rA, c.rB, c.e);
            int src = t->src[slot];
            V3<S> lp = src >= 0 ? X.lam[src] : vzero<S>(), pp = src >= 0 ? X.pen[src] : vzero<S>();
            contact_carry(lp, pp, src >= 0, t->initFlags[slot], alpha, gamma, c.lam, c.pen);
        }
    }
    W.initLin = X.p;
    W.initAng = X.q;
    W.inertLin.resize(n);
    W.inertAng.resize(n);
    for (int b = 0; b < n; ++b)
    {
        unsigned bf = t->bodyFlags[b];
        if (!(bf & BF_DYNAMIC))
        {
            W.inertLin[b] = X.p[b] + X.v[b] * dt;
            W.inertAng[b] = qstep(X.q[b], X.w[b] * dt);
            continue;
        }
        WarmOut<S> o = warm_start(X.p[b], X.q[b], X.v[b], X.w[b], X.vp[b], dt, g, bf);
        W.inertLin[b] = o.inertLin;
        W.inertAng[b] = o.inertAng;
        X.p[b] = o.p;
        X.q[b] = o.q;
    }
}

unsigned eval_flags(const OracleTapeStep *t, int it, size_t slot, int which)
{
    return t->flags[((size_t)it * (size_t)t->nMan * 8 + slot) * 3 + which];
}

// system of body b at iteration it with the current poses
void body_system(const Problem &pb, int s, int it, int b, const S *th, const std::vector<V3<S>> &p,
                 const std::vector<Q4<S>> &q, const StepWork &W, Sys6<S> &sys)
{
    const OracleTapeStep *t = pb.st[s];
    S alpha = pb.p.alpha;
    sys_zero(sys);
    stamp_inertia(sys, th[6 * pb.n + b], pb.shape[b], p[b], W.inertLin[b], q[b], W.inertAng[b], (S)pb.p.dt);
    for (int k = pb.bodyStart[s][b]; k < pb.bodyStart[s][b + 1]; ++k)
    {
        int m = pb.bodyMan[s][k] >> 1;
        bool isA = pb.bodyMan[s][k] & 1;
        Pose<S> A = pose_of(p, q, W, t->ab[2 * m]), B = pose_of(p, q, W, t->ab[2 * m + 1]);
        for (int i = 0; i < t->ncontacts[m]; ++i)
        {
            size_t slot = (size_t)m * 8 + i;
            ContactFwd<S> f = contact_forward(A, B, W.c[slot], alpha, eval_flags(t, it, slot, isA ? 0 : 1));
            stamp_contact(sys, W.c[slot], f, isA);
        }
    }
}

void primal_body(const Problem &pb, int s, int it, int b, const S *th, State &X, const StepWork &W)
{
    Sys6<S> sys;
    body_system(pb, s, it, b, th, X.p, X.q, W, sys);
    Ldl6<S> f;
    ldl_factor(sys.H, f);
    S dx[6];
    body_dx(f, sys, dx);
    X.p[b] = X.p[b] + v3(dx[0], dx[1], dx[2]);
    X.q[b] = qstep(X.q[b], v3(dx[3], dx[4], dx[5]));
}

void dual_all(const Problem &pb, int s, int it, State &X, StepWork &W)
{
    const OracleTapeStep *t = pb.st[s];
    for (int m = 0; m < t->nMan; ++m)
    {
        Pose<S> A = pose_of(X.p, X.q, W, t->ab[2 * m]), B = pose_of(X.p, X.q, W, t->ab[2 * m + 1]);
        for (int i = 0; i < t->ncontacts[m]; ++i)
        {
            size_t slot = (size_t)m * 8 + i;
            ContactIn<S> &c = W.c[slot];
            V3<S> lam, pen;
            contact_dual_forward(A, B, c, (S)pb.p.alpha, (S)pb.p.betaLin, eval_flags(t, it, slot, 2), lam, pen);
            c.lam = lam;
            c.pen = pen;
        }
    }
}

void finish(const Problem &pb, int s, State &X, StepWork &W)
{
    const OracleTapeStep *t = pb.st[s];
    S dt = pb.p.dt;
    for (int b = 0; b < pb.n; ++b)
    {
        X.vp[b] = X.v[b];
        if (t->bodyFlags[b] & BF_DYNAMIC)
        {
            X.v[b] = (X.p[b] - W.initLin[b]) * (S(1) / dt);
            X.w[b] = qdiff(X.q[b], W.initAng[b]) * (S(1) / dt);
        }
    }
    size_t ns = W.c.size();
    X.lam.resize(ns);
    X.pen.resize(ns);
    for (size_t i = 0; i < ns; ++i)
    {
        X.lam[i] = W.c[i].lam;
        X.pen[i] = W.c[i].pen;
    }
}

void replay_step(const Problem &pb, int s, const S *th, State &X)
{
    StepWork W;
    prepare(pb, s, th, X, W);
    const OracleTapeStep *t = pb.st[s];
    for (int it = 0; it < t->iterations; ++it)
    {
        for (int k = 0; k < t->nSolve; ++k)
            primal_body(pb, s, it, t->solveOrder[k], th, X, W);
        dual_all(pb, s, it, X, W);
    }
    finish(pb, s, X, W);
}

S com_loss(const Problem &pb, const S *th, const State &X, const S *target, V3<S> *com)
{
    S M = 0;
    V3<S> c = vzero<S>();
    for (int b = 0; b < pb.n; ++b)
        if (pb.st[0]->bodyFlags[b] & BF_DYNAMIC)
        {
            S m = th[6 * pb.n + b];
            M += m;
            c += X.p[b] * m;
        }
    c = c * (S(1) / M);
    if (com)
        *com = c;
    V3<S> d = c - v3<S>(target[0], target[1], target[2]);
    return dot(d, d);
}

S replay_loss(const Problem &pb, const S *th, const S *target, S *finalPos)
{
    State X;
    initial_state(pb, th, X);
    for (int s = 0; s < pb.steps; ++s)
        replay_step(pb, s, th, X);
    if (finalPos)
        for (int b = 0; b < pb.n; ++b)
        {
            finalPos[3 * b] = X.p[b].x;
            finalPos[3 * b + 1] = X.p[b].y;
            finalPos[3 * b + 2] = X.p[b].z;
        }
    return com_loss(pb, th, X, target, nullptr);
}

// Adjoint of the state between steps.
struct Adj
{
    std::vector<V3<S>> p, v, w, vp;
    std::vector<Q4<S>> q;
    std::vector<V3<S>> lam, pen;
};

template <class T> void addto(std::vector<T> &v, int i, T x) { v[i] += x; }

S reference_gradient(const Problem &pb, const S *th, const S *target, S *grad)
{
    int n = pb.n;
    S alpha = pb.p.alpha, beta = pb.p.betaLin, gamma = pb.p.gamma, dt = pb.p.dt, g = pb.p.gravity;
    // forward with a state checkpoint at every step start
    std::vector<State> ck(pb.steps + 1);
    initial_state(pb, th, ck[0]);
    for (int s = 0; s < pb.steps; ++s)
    {
        ck[s + 1] = ck[s];
        replay_step(pb, s, th, ck[s + 1]);
    }
    const State &XT = ck[pb.steps];
    V3<S> com;
    S loss = com_loss(pb, th, XT, target, &com);
    S M = 0;
    for (int b = 0; b < n; ++b)
        if (pb.st[0]->bodyFlags[b] & BF_DYNAMIC)
            M += th[6 * n + b];
    V3<S> dL = (com - v3<S>(target[0], target[1], target[2])) * S(2);

    std::vector<S> gm(n, 0.0), gmu(pb.P, 0.0);
    Adj A;
    A.p.assign(n, vzero<S>());
    A.q.assign(n, qzero<S>());
    A.v.assign(n, vzero<S>());
    A.w.assign(n, vzero<S>());
    A.vp.assign(n, vzero<S>());
    for (int b = 0; b < n; ++b)
        if (pb.st[0]->bodyFlags[b] & BF_DYNAMIC)
        {
            S m = th[6 * n + b];
            A.p[b] = dL * (m / M);
            gm[b] += dot(dL, XT.p[b] - com) / M;
        }
    A.lam.assign(XT.lam.size(), vzero<S>());
    A.pen.assign(XT.pen.size(), vzero<S>());

    for (int s = pb.steps - 1; s >= 0; --s)
    {
        const OracleTapeStep *t = pb.st[s];
        int T = t->iterations;
        // recompute step s with snapshots
        State X = ck[s];
        StepWork W;
        prepare(pb, s, th, X, W);
        std::vector<std::vector<V3<S>>> Pp(T + 1);
        std::vector<std::vector<Q4<S>>> Pq(T + 1);
        std::vector<std::vector<V3<S>>> Lam(T + 1), Pen(T + 1);
        auto snap = [&](int it) {
            Pp[it] = X.p;
            Pq[it] = X.q;
            Lam[it].resize(W.c.size());
            Pen[it].resize(W.c.size());
            for (size_t i = 0; i < W.c.size(); ++i)
            {
                Lam[it][i] = W.c[i].lam;
                Pen[it][i] = W.c[i].pen;
            }
        };
        std::vector<V3<S>> pWarm = X.p;
        std::vector<Q4<S>> qWarm = X.q;
        for (int it = 0; it < T; ++it)
        {
            snap(it);
            for (int k = 0; k < t->nSolve; ++k)
                primal_body(pb, s, it, t->solveOrder[k], th, X, W);
            dual_all(pb, s, it, X, W);
        }
        snap(T);
        (void)pWarm;
        (void)qWarm;

        std::vector<V3<S>> initLinBar(n, vzero<S>()), inertLinBar(n, vzero<S>());
        std::vector<Q4<S>> initAngBar(n, qzero<S>()), inertAngBar(n, qzero<S>());
        std::vector<V3<S>> C0bar(W.c.size(), vzero<S>());
        std::vector<V3<S>> vS(n), wS(n), vpS(n);
        // finish
        for (int b = 0; b < n; ++b)
        {
            if (t->bodyFlags[b] & BF_DYNAMIC)
            {
                finish_vjp(Pq[T][b], W.initAng[b], dt, A.v[b], A.w[b], A.p[b], A.q[b], initLinBar[b], initAngBar[b]);
                vS[b] = A.vp[b];
                wS[b] = vzero<S>();
            }
            else
            {
                vS[b] = A.v[b] + A.vp[b];
                wS[b] = A.w[b];
            }
            vpS[b] = vzero<S>();
        }
        // iterations in reverse
        std::vector<V3<S>> cp = Pp[T];
        std::vector<Q4<S>> cq = Pq[T];
        for (int it = T - 1; it >= 0; --it)
        {
            // contacts as the iteration saw them
            for (size_t i = 0; i < W.c.size(); ++i)
            {
                W.c[i].lam = Lam[it][i];
                W.c[i].pen = Pen[it][i];
            }
            // dual
            for (int m = 0; m < t->nMan; ++m)
            {
                int a = t->ab[2 * m], b = t->ab[2 * m + 1];
                Pose<S> PA = pose_of(cp, cq, W, a), PB = pose_of(cp, cq, W, b);
                for (int i = 0; i < t->ncontacts[m]; ++i)
                {
                    size_t slot = (size_t)m * 8 + i;
                    PoseBar<S> Ab = posebar_zero<S>(), Bb = posebar_zero<S>();
                    contact_dual_vjp(PA, PB, W.c[slot], alpha, beta, eval_flags(t, it, slot, 2), A.lam[slot],
                                     A.pen[slot], Ab, Bb, C0bar[slot], gmu[pb.manPair[s][m]]);
                    A.p[a] += Ab.p;
                    A.q[a] += Ab.q;
                    initLinBar[a] += Ab.pi;
                    initAngBar[a] += Ab.qi;
                    A.p[b] += Bb.p;
                    A.q[b] += Bb.q;
                    initLinBar[b] += Bb.pi;
                    initAngBar[b] += Bb.qi;
                }
            }
            // primal sweep in reverse
            for (int k = t->nSolve - 1; k >= 0; --k)
            {
                int b = t->solveOrder[k];
                cp[b] = Pp[it][b];
                cq[b] = Pq[it][b];
                Sys6<S> sys;
                body_system(pb, s, it, b, th, cp, cq, W, sys);
                Ldl6<S> f;
                ldl_factor(sys.H, f);
                S dx[6];
                body_dx(f, sys, dx);
                S dxbar[6] = {A.p[b].x, A.p[b].y, A.p[b].z, 0, 0, 0};
                Q4<S> qpre = qzero<S>();
                V3<S> wb = vzero<S>();
                qstep_vjp(cq[b], v3(dx[3], dx[4], dx[5]), A.q[b], qpre, wb);
                dxbar[3] = wb.x;
                dxbar[4] = wb.y;
                dxbar[5] = wb.z;
                A.q[b] = qpre;
                Sys6<S> bar;
                body_dx_vjp(f, dx, dxbar, bar);
                stamp_inertia_vjp(bar, th[6 * n + b], pb.shape[b], cp[b], W.inertLin[b], cq[b], W.inertAng[b], dt,
                                  gm[b], A.p[b], inertLinBar[b], A.q[b], inertAngBar[b]);
                for (int e = pb.bodyStart[s][b]; e < pb.bodyStart[s][b + 1]; ++e)
                {
                    int m = pb.bodyMan[s][e] >> 1;
                    bool isA = pb.bodyMan[s][e] & 1;
                    int a = t->ab[2 * m], bb = t->ab[2 * m + 1];
                    Pose<S> PA = pose_of(cp, cq, W, a), PB = pose_of(cp, cq, W, bb);
                    for (int i = 0; i < t->ncontacts[m]; ++i)
                    {
                        size_t slot = (size_t)m * 8 + i;
                        PoseBar<S> Ab = posebar_zero<S>(), Bb = posebar_zero<S>();
                        contact_primal_vjp(PA, PB, W.c[slot], alpha, eval_flags(t, it, slot, isA ? 0 : 1), isA, bar, Ab,
                                           Bb, A.lam[slot], A.pen[slot], C0bar[slot], gmu[pb.manPair[s][m]]);
                        A.p[a] += Ab.p;
                        A.q[a] += Ab.q;
                        initLinBar[a] += Ab.pi;
                        initAngBar[a] += Ab.qi;
                        A.p[bb] += Bb.p;
                        A.q[bb] += Bb.q;
                        initLinBar[bb] += Bb.pi;
                        initAngBar[bb] += Bb.qi;
                    }
                }
            }
        }
        // manifold initialisation: C0 and the carried lambda / penalty
        const State &X0 = ck[s];
        std::vector<V3<S>> lamPrev(X0.lam.size(), vzero<S>()), penPrev(X0.pen.size(), vzero<S>());
        for (int m = 0; m < t->nMan; ++m)
        {
            int a = t->ab[2 * m], b = t->ab[2 * m + 1];
            for (int i = 0; i < t->ncontacts[m]; ++i)
            {
                size_t slot = (size_t)m * 8 + i;
                const ContactIn<S> &c = W.c[slot];
                contact_C0_vjp(X0.q[a], X0.q[b], c.rA, c.rB, c.e, C0bar[slot], initLinBar[a], initAngBar[a],
                               initLinBar[b], initAngBar[b]);
                int src = t->src[slot];
                if (src >= 0)
                    contact_carry_vjp(A.lam[slot], A.pen[slot], t->initFlags[slot], alpha, gamma, lamPrev[src],
                                      penPrev[src]);
            }
        }
        // warm start
        for (int b = 0; b < n; ++b)
        {
            V3<S> p0b = vzero<S>(), vb = vS[b], wb = wS[b], vpb = vpS[b];
            Q4<S> q0b = qzero<S>();
            if (t->bodyFlags[b] & BF_DYNAMIC)
                warm_start_vjp(X0.q[b], X0.w[b], dt, g, t->bodyFlags[b], A.p[b], A.q[b], inertLinBar[b],
                               inertAngBar[b], initLinBar[b], initAngBar[b], p0b, q0b, vb, wb, vpb);
            else
            {
                p0b = A.p[b] + initLinBar[b];
                q0b = A.q[b] + initAngBar[b];
            }
            A.p[b] = p0b;
            A.q[b] = q0b;
            A.v[b] = vb;
            A.w[b] = wb;
            A.vp[b] = vpb;
        }
        A.lam = lamPrev;
        A.pen = penPrev;
    }
    for (int b = 0; b < n; ++b)
    {
        V3<S> gv = A.v[b] + A.vp[b]; // v0 sets velocity and previous velocity
        grad[3 * b] = gv.x;
        grad[3 * b + 1] = gv.y;
        grad[3 * b + 2] = gv.z;
        grad[3 * n + 3 * b] = A.w[b].x;
        grad[3 * n + 3 * b + 1] = A.w[b].y;
        grad[3 * n + 3 * b + 2] = A.w[b].z;
        grad[6 * n + b] = gm[b];
    }
    for (int i = 0; i < pb.P; ++i)
        grad[7 * n + i] = gmu[i];
    return loss;
}

// ---------------------------------------------------------------------------
// VJP self-test: each primitive against central differences of its forward map
// ---------------------------------------------------------------------------

struct Rng
{
    std::mt19937_64 g;
    explicit Rng(unsigned long long s) : g(s) {}
    S u(S lo = -1, S hi = 1) { return std::uniform_real_distribution<S>(lo, hi)(g); }
    V3<S> v(S s = 1) { return v3(u() * s, u() * s, u() * s); }
    Q4<S> q()
    {
        Q4<S> r = q4(u(), u(), u(), u());
        S nn = std::sqrt(qdot(r, r));
        return r * (S(1) / nn);
    }
};

double rel(double a, double b) { return std::fabs(a - b) / std::max(1e-5, std::max(std::fabs(a), std::fabs(b))); }

} // namespace

extern "C"
{

int adjref_num_params(const OracleWorld *w)
{
    Problem pb;
    return build_problem(w, pb) ? num_params(pb) : -1;
}

int adjref_num_pairs(const OracleWorld *w)
{
    Problem pb;
    return build_problem(w, pb) ? pb.P : -1;
}

void adjref_pairs(const OracleWorld *w, int *lohi2, float *mu0)
{
    Problem pb;
    if (!build_problem(w, pb))
        return;
    for (int i = 0; i < pb.P; ++i)
    {
        lohi2[2 * i] = (int)(pb.pairKeys[i] >> 32);
        lohi2[2 * i + 1] = (int)(pb.pairKeys[i] & 0xFFFFFFFFull);
        if (mu0)
            mu0[i] = pb.pairMu0[i];
    }
}

void adjref_theta0(const OracleWorld *w, double *theta)
{
    Problem pb;
    if (build_problem(w, pb))
        theta0(pb, theta);
}

double adjref_loss(const OracleWorld *w, const double *theta, const double *target3, double *finalPos3)
{
    Problem pb;
    if (!build_problem(w, pb))
        return NAN;
    return replay_loss(pb, theta, target3, finalPos3);
}

double adjref_gradient(const OracleWorld *w, const double *theta, const double *target3, double *grad)
{
    Problem pb;
    if (!build_problem(w, pb))
        return NAN;
    return reference_gradient(pb, theta, target3, grad);
}

void adjref_fd(const OracleWorld *w, const double *theta, const double *target3, int nDir, const double *dirs,
               double h, int threads, double *out)
{
    Problem pb;
    if (!build_problem(w, pb))
        return;
    int np = num_params(pb);
    threads = std::max(1, std::min(threads, 2 * nDir));
    std::vector<std::thread> pool;
    for (int tid = 0; tid < threads; ++tid)
        pool.emplace_back([&, tid]() {
            std::vector<S> th(np);
            std::vector<S> lp(nDir, 0.0), lm(nDir, 0.0);
            for (int job = tid; job < 2 * nDir; job += threads)
            {
                int d = job >> 1;
                S sgn = (job & 1) ? S(-1) : S(1);
                for (int i = 0; i < np; ++i)
                    th[i] = theta[i] + sgn * h * dirs[(size_t)d * np + i];
                S l = replay_loss(pb, th.data(), target3, nullptr);
                if (job & 1)
                    out[2 * d + 1] = l;
                else
                    out[2 * d] = l;
            }
        });
    for (auto &t : pool)
        t.join();
    // out[2d], out[2d+1] hold L(+h), L(-h); fold into the derivative in place
    for (int d = 0; d < nDir; ++d)
        out[d] = (out[2 * d] - out[2 * d + 1]) / (2 * h);
}

// Checks each VJP against central differences of its forward map on random inputs;
// returns the largest relative error.
double adjref_selftest(void)
{
    Rng r(12345);
    const S h = 1e-6;
    double worst = 0;
    for (int trial = 0; trial < 20; ++trial)
    {
        // rotate, qdiff, qstep
        Q4<S> q = r.q(), q2 = r.q();
        V3<S> v = r.v(), rb = r.v(), w = r.v(0.2);
        Q4<S> qb = r.q();
        Q4<S> gq = rotate_vjp_q(q, v, rb);
        S gqa[4] = {gq.x, gq.y, gq.z, gq.w};
        for (int k = 0; k < 4; ++k)
        {
            Q4<S> qp = q, qm = q;
            ((S *)&qp)[k] += h;
            ((S *)&qm)[k] -= h;
            S fd = (dot(rotate(qp, v), rb) - dot(rotate(qm, v), rb)) / (2 * h);
            worst = std::max(worst, rel(fd, gqa[k]));
        }
        Q4<S> ab = qzero<S>(), bb = qzero<S>();
        qdiff_vjp(q, q2, rb, ab, bb);
        for (int k = 0; k < 4; ++k)
        {
            Q4<S> p1 = q, m1 = q, p2 = q2, m2 = q2;
            ((S *)&p1)[k] += h;
            ((S *)&m1)[k] -= h;
            ((S *)&p2)[k] += h;
            ((S *)&m2)[k] -= h;
            S fa = (dot(qdiff(p1, q2), rb) - dot(qdiff(m1, q2), rb)) / (2 * h);
            S fb = (dot(qdiff(q, p2), rb) - dot(qdiff(q, m2), rb)) / (2 * h);
            worst = std::max(worst, rel(fa, ((S *)&ab)[k]));
            worst = std::max(worst, rel(fb, ((S *)&bb)[k]));
        }
        Q4<S> qsb = qzero<S>();
        V3<S> wsb = vzero<S>();
        qstep_vjp(q, w, qb, qsb, wsb);
        for (int k = 0; k < 4; ++k)
        {
            Q4<S> qp = q, qm = q;
            ((S *)&qp)[k] += h;
            ((S *)&qm)[k] -= h;
            S fd = (qdot(qstep(qp, w), qb) - qdot(qstep(qm, w), qb)) / (2 * h);
            worst = std::max(worst, rel(fd, ((S *)&qsb)[k]));
        }
        for (int k = 0; k < 3; ++k)
        {
            V3<S> wp = w, wm = w;
            ((S *)&wp)[k] += h;
            ((S *)&wm)[k] -= h;
            S fd = (qdot(qstep(q, wp), qb) - qdot(qstep(q, wm), qb)) / (2 * h);
            worst = std::max(worst, rel(fd, ((S *)&wsb)[k]));
        }
        // one body solve with two contacts, through the pose update, for each flag combination
        unsigned flagSets[4] = {0u, EF_CONE, EF_NCLAMP, EF_NCLAMP | EF_CONE};
        unsigned flags = flagSets[trial % 4];
        Pose<S> A, B;
        A.p = r.v();
        A.pi = A.p + r.v(0.05);
        A.q = r.q();
        A.qi = qstep(A.q, r.v(0.05));
        B.p = r.v();
        B.pi = B.p + r.v(0.05);
        B.q = r.q();
        B.qi = qstep(B.q, r.v(0.05));
        ContactIn<S> c[2];
        for (int i = 0; i < 2; ++i)
        {
            c[i].rA = r.v(0.5);
            c[i].rB = r.v(0.5);
            Q4<S> fr = r.q();
            c[i].e[0] = rotate(fr, v3<S>(1, 0, 0));
            c[i].e[1] = rotate(fr, v3<S>(0, 1, 0));
            c[i].e[2] = rotate(fr, v3<S>(0, 0, 1));
            c[i].C0 = r.v(0.1);
            c[i].lam = v3<S>(-1.0 - r.u(0, 1), r.u(), r.u());
            c[i].pen = v3<S>(r.u(10, 100), r.u(10, 100), r.u(10, 100));
            c[i].mu = r.u(0.2, 0.8);
        }
        S m = r.u(0.5, 2.0), dt = 1.0 / 60.0, alpha = 0.95;
        V3<S> shape = v3<S>(r.u(0.1, 0.3), r.u(0.1, 0.3), r.u(0.1, 0.3));
        V3<S> it = A.p + r.v(0.01);
        Q4<S> iq = qstep(A.q, r.v(0.01));
        V3<S> pbarN = r.v();
        Q4<S> qbarN = r.q();
        // forward: A is the solved body
        auto solve = [&](const Pose<S> &a, const Pose<S> &b, const ContactIn<S> *cc, S mm, V3<S> &pn, Q4<S> &qn) {
            Sys6<S> sys;
            sys_zero(sys);
            stamp_inertia(sys, mm, shape, a.p, it, a.q, iq, dt);
            for (int i = 0; i < 2; ++i)
            {
                ContactFwd<S> f = contact_forward(a, b, cc[i], alpha, flags);
                stamp_contact(sys, cc[i], f, true);
            }
            Ldl6<S> f;
            ldl_factor(sys.H, f);
            S dx[6];
            body_dx(f, sys, dx);
            pn = a.p + v3(dx[0], dx[1], dx[2]);
            qn = qstep(a.q, v3(dx[3], dx[4], dx[5]));
            return dot(pn, pbarN) + qdot(qn, qbarN);
        };
        V3<S> pn;
        Q4<S> qn;
        solve(A, B, c, m, pn, qn);
        // analytic
        Sys6<S> sys;
        sys_zero(sys);
        stamp_inertia(sys, m, shape, A.p, it, A.q, iq, dt);
        for (int i = 0; i < 2; ++i)
            stamp_contact(sys, c[i], contact_forward(A, B, c[i], alpha, flags), true);
        Ldl6<S> f;
        ldl_factor(sys.H, f);
        S dx[6];
        body_dx(f, sys, dx);
        S dxbar[6] = {pbarN.x, pbarN.y, pbarN.z, 0, 0, 0};
        Q4<S> qpre = qzero<S>();
        V3<S> wq = vzero<S>();
        qstep_vjp(A.q, v3(dx[3], dx[4], dx[5]), qbarN, qpre, wq);
        dxbar[3] = wq.x;
        dxbar[4] = wq.y;
        dxbar[5] = wq.z;
        Sys6<S> bar;
        body_dx_vjp(f, dx, dxbar, bar);
        PoseBar<S> Ab = posebar_zero<S>(), Bb = posebar_zero<S>();
        Ab.p = pbarN;
        Ab.q = qpre;
        S mb = 0;
        V3<S> itb = vzero<S>();
        Q4<S> iqb = qzero<S>();
        stamp_inertia_vjp(bar, m, shape, A.p, it, A.q, iq, dt, mb, Ab.p, itb, Ab.q, iqb);
        V3<S> lamb[2] = {vzero<S>(), vzero<S>()}, penb[2] = {vzero<S>(), vzero<S>()},
              c0b[2] = {vzero<S>(), vzero<S>()};
        S mub[2] = {0, 0};
        for (int i = 0; i < 2; ++i)
            contact_primal_vjp(A, B, c[i], alpha, flags, true, bar, Ab, Bb, lamb[i], penb[i], c0b[i], mub[i]);
        auto fd_of = [&](auto mutate) {
            Pose<S> a1 = A, b1 = B, a2 = A, b2 = B;
            ContactIn<S> c1[2] = {c[0], c[1]}, c2[2] = {c[0], c[1]};
            S m1 = m, m2 = m;
            mutate(a1, b1, c1, m1, h);
            mutate(a2, b2, c2, m2, -h);
            V3<S> pp;
            Q4<S> qq;
            S l1 = solve(a1, b1, c1, m1, pp, qq);
            S l2 = solve(a2, b2, c2, m2, pp, qq);
            return (l1 - l2) / (2 * h);
        };
        for (int k = 0; k < 3; ++k)
        {
            worst = std::max(worst, rel(fd_of([&](Pose<S> &a, Pose<S> &, ContactIn<S> *, S &, S d) {
                                            ((S *)&a.p)[k] += d;
                                        }),
                                        ((S *)&Ab.p)[k]));
            worst = std::max(worst, rel(fd_of([&](Pose<S> &, Pose<S> &b, ContactIn<S> *, S &, S d) {
                                            ((S *)&b.p)[k] += d;
                                        }),
                                        ((S *)&Bb.p)[k]));
            worst = std::max(worst, rel(fd_of([&](Pose<S> &a, Pose<S> &, ContactIn<S> *, S &, S d) {
                                            ((S *)&a.pi)[k] += d;
                                        }),
                                        ((S *)&Ab.pi)[k]));
            worst = std::max(worst, rel(fd_of([&](Pose<S> &, Pose<S> &, ContactIn<S> *cc, S &, S d) {
                                            ((S *)&cc[0].lam)[k] += d;
                                        }),
                                        ((S *)&lamb[0])[k]));
            worst = std::max(worst, rel(fd_of([&](Pose<S> &, Pose<S> &, ContactIn<S> *cc, S &, S d) {
                                            ((S *)&cc[1].pen)[k] += d;
                                        }),
                                        ((S *)&penb[1])[k]));
            worst = std::max(worst, rel(fd_of([&](Pose<S> &, Pose<S> &, ContactIn<S> *cc, S &, S d) {
                                            ((S *)&cc[0].C0)[k] += d;
                                        }),
                                        ((S *)&c0b[0])[k]));
        }
        for (int k = 0; k < 4; ++k)
        {
            worst = std::max(worst, rel(fd_of([&](Pose<S> &a, Pose<S> &, ContactIn<S> *, S &, S d) {
                                            ((S *)&a.q)[k] += d;
                                        }),
                                        ((S *)&Ab.q)[k]));
            worst = std::max(worst, rel(fd_of([&](Pose<S> &, Pose<S> &b, ContactIn<S> *, S &, S d) {
                                            ((S *)&b.q)[k] += d;
                                        }),
                                        ((S *)&Bb.q)[k]));
            worst = std::max(worst, rel(fd_of([&](Pose<S> &, Pose<S> &b, ContactIn<S> *, S &, S d) {
                                            ((S *)&b.qi)[k] += d;
                                        }),
                                        ((S *)&Bb.qi)[k]));
        }
        worst = std::max(worst, rel(fd_of([&](Pose<S> &, Pose<S> &, ContactIn<S> *, S &mm, S d) { mm += d; }), mb));
        if (flags & EF_CONE)
            worst = std::max(worst, rel(fd_of([&](Pose<S> &, Pose<S> &, ContactIn<S> *cc, S &, S d) { cc[0].mu += d; }),
                                        mub[0]));
        // rank-one system adjoint forms against the general ones
        {
            S dxr[6], dxbr[6], ur[6];
            for (int k = 0; k < 6; ++k)
            {
                dxr[k] = r.u();
                dxbr[k] = r.u();
            }
            Ldl6<S> fr;
            ldl_factor(sys.H, fr);
            body_dx_vjp_u(fr, dxbr, ur);
            Sys6<S> full;
            body_dx_vjp(fr, dxr, dxbr, full);
            PoseBar<S> A1 = posebar_zero<S>(), B1 = posebar_zero<S>(), A2 = posebar_zero<S>(), B2 = posebar_zero<S>();
            V3<S> l1 = vzero<S>(), l2 = vzero<S>(), p1 = vzero<S>(), p2 = vzero<S>(), z1 = vzero<S>(), z2 = vzero<S>();
            S m1 = 0, m2 = 0;
            contact_primal_vjp(A, B, c[1], alpha, flags, false, full, A1, B1, l1, p1, z1, m1);
            contact_primal_vjp_outer(A, B, c[1], alpha, flags, false, ur, dxr, A2, B2, l2, p2, z2, m2);
            for (int k = 0; k < 3; ++k)
            {
                worst = std::max(worst, rel(((S *)&l1)[k], ((S *)&l2)[k]));
                worst = std::max(worst, rel(((S *)&p1)[k], ((S *)&p2)[k]));
                worst = std::max(worst, rel(((S *)&A1.p)[k], ((S *)&A2.p)[k]));
            }
            for (int k = 0; k < 4; ++k)
                worst = std::max(worst, rel(((S *)&B1.q)[k], ((S *)&B2.q)[k]));
            S mb1 = 0, mb2 = 0;
            V3<S> pb1 = vzero<S>(), pb2 = vzero<S>(), tb1 = vzero<S>(), tb2 = vzero<S>();
            Q4<S> qb1 = qzero<S>(), qb2 = qzero<S>(), qt1 = qzero<S>(), qt2 = qzero<S>();
            stamp_inertia_vjp(full, m, shape, A.p, it, A.q, iq, dt, mb1, pb1, tb1, qb1, qt1);
            stamp_inertia_vjp_outer(ur, dxr, m, shape, A.p, it, A.q, iq, dt, mb2, pb2, tb2, qb2, qt2);
            worst = std::max(worst, rel(mb1, mb2));
            for (int k = 0; k < 4; ++k)
                worst = std::max(worst, rel(((S *)&qb1)[k], ((S *)&qb2)[k]));
        }
        // dual update of contact 0
        unsigned dflags = flags | EF_NEG_X | EF_POS_Y | EF_NEG_Z | ((flags & EF_CONE) ? 0u : EF_RAMP_T);
        V3<S> lbN = r.v(), pbN = r.v();
        auto dual = [&](const Pose<S> &a, const Pose<S> &b, const ContactIn<S> &cc) {
            V3<S> l, p;
            contact_dual_forward(a, b, cc, alpha, S(1000), dflags, l, p);
            return dot(l, lbN) + dot(p, pbN);
        };
        V3<S> lb = lbN, pbb = pbN, c0d = vzero<S>();
        PoseBar<S> Ad = posebar_zero<S>(), Bd = posebar_zero<S>();
        S mud = 0;
        contact_dual_vjp(A, B, c[0], alpha, S(1000), dflags, lb, pbb, Ad, Bd, c0d, mud);
        for (int k = 0; k < 3; ++k)
        {
            Pose<S> a1 = A, a2 = A;
            ((S *)&a1.p)[k] += h;
            ((S *)&a2.p)[k] -= h;
            worst = std::max(worst, rel((dual(a1, B, c[0]) - dual(a2, B, c[0])) / (2 * h), ((S *)&Ad.p)[k]));
            ContactIn<S> c1 = c[0], c2 = c[0];
            ((S *)&c1.pen)[k] += h;
            ((S *)&c2.pen)[k] -= h;
            worst = std::max(worst, rel((dual(A, B, c1) - dual(A, B, c2)) / (2 * h), ((S *)&pbb)[k]));
            c1 = c[0];
            c2 = c[0];
            ((S *)&c1.lam)[k] += h;
            ((S *)&c2.lam)[k] -= h;
            worst = std::max(worst, rel((dual(A, B, c1) - dual(A, B, c2)) / (2 * h), ((S *)&lb)[k]));
        }
        for (int k = 0; k < 4; ++k)
        {
            Pose<S> b1 = B, b2 = B;
            ((S *)&b1.q)[k] += h;
            ((S *)&b2.q)[k] -= h;
            worst = std::max(worst, rel((dual(A, b1, c[0]) - dual(A, b2, c[0])) / (2 * h), ((S *)&Bd.q)[k]));
        }
        // warm start
        unsigned bfs[3] = {BF_DYNAMIC | BF_FORCES | BF_ACCEL_IN, BF_DYNAMIC | BF_FORCES, BF_DYNAMIC};
        unsigned bf = bfs[trial % 3];
        V3<S> v0 = r.v(), w0 = r.v(), vp0 = r.v(), pW = r.v(), iLb = r.v(), itLb = r.v();
        Q4<S> q0 = r.q(), qW = r.q(), iAb = r.q(), itAb = r.q();
        auto warm = [&](V3<S> p, Q4<S> qq, V3<S> vv, V3<S> ww, V3<S> vpp) {
            WarmOut<S> o = warm_start(p, qq, vv, ww, vpp, dt, S(-9.81), bf);
            return dot(o.p, pW) + qdot(o.q, qW) + dot(o.inertLin, itLb) + qdot(o.inertAng, itAb) + dot(p, iLb) +
                   qdot(qq, iAb);
        };
        V3<S> p0b = vzero<S>(), vb = vzero<S>(), wb2 = vzero<S>(), vpb = vzero<S>();
        Q4<S> q0b = qzero<S>();
        warm_start_vjp(q0, w0, dt, S(-9.81), bf, pW, qW, itLb, itAb, iLb, iAb, p0b, q0b, vb, wb2, vpb);
        V3<S> p0 = r.v();
        for (int k = 0; k < 3; ++k)
        {
            V3<S> a1 = v0, a2 = v0;
            ((S *)&a1)[k] += h;
            ((S *)&a2)[k] -= h;
            worst = std::max(worst, rel((warm(p0, q0, a1, w0, vp0) - warm(p0, q0, a2, w0, vp0)) / (2 * h), ((S *)&vb)[k]));
            a1 = vp0;
            a2 = vp0;
            ((S *)&a1)[k] += h;
            ((S *)&a2)[k] -= h;
            worst = std::max(worst, rel((warm(p0, q0, v0, w0, a1) - warm(p0, q0, v0, w0, a2)) / (2 * h) + 1e-300,
                                        ((S *)&vpb)[k] + 1e-300));
            a1 = w0;
            a2 = w0;
            ((S *)&a1)[k] += h;
            ((S *)&a2)[k] -= h;
            worst = std::max(worst, rel((warm(p0, q0, v0, a1, vp0) - warm(p0, q0, v0, a2, vp0)) / (2 * h), ((S *)&wb2)[k]));
            a1 = p0;
            a2 = p0;
            ((S *)&a1)[k] += h;
            ((S *)&a2)[k] -= h;
            worst = std::max(worst, rel((warm(a1, q0, v0, w0, vp0) - warm(a2, q0, v0, w0, vp0)) / (2 * h), ((S *)&p0b)[k]));
        }
        for (int k = 0; k < 4; ++k)
        {
            Q4<S> a1 = q0, a2 = q0;
            ((S *)&a1)[k] += h;
            ((S *)&a2)[k] -= h;
            worst = std::max(worst, rel((warm(p0, a1, v0, w0, vp0) - warm(p0, a2, v0, w0, vp0)) / (2 * h), ((S *)&q0b)[k]));
        }
        // C0
        V3<S> c0w = r.v();
        auto c0f = [&](V3<S> pa, Q4<S> qa, V3<S> pbv, Q4<S> qbv) {
            return dot(contact_C0(pa, qa, pbv, qbv, c[0].rA, c[0].rB, c[0].e), c0w);
        };
        V3<S> pab = vzero<S>(), pbb2 = vzero<S>();
        Q4<S> qab = qzero<S>(), qbb2 = qzero<S>();
        contact_C0_vjp(A.q, B.q, c[0].rA, c[0].rB, c[0].e, c0w, pab, qab, pbb2, qbb2);
        for (int k = 0; k < 4; ++k)
        {
            Q4<S> a1 = A.q, a2 = A.q;
            ((S *)&a1)[k] += h;
            ((S *)&a2)[k] -= h;
            worst = std::max(worst, rel((c0f(A.p, a1, B.p, B.q) - c0f(A.p, a2, B.p, B.q)) / (2 * h), ((S *)&qab)[k]));
        }
    }
    return worst;
}

} // extern "C"
