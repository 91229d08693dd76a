// Differentiable AVBD step: frozen-branch forward pieces and their hand-written
// vector-Jacobian products (VJPs), templated on the scalar type so the same source runs in
// the GPU adjoint kernels (double) and in host code (double: the reference adjoint and the
// finite-difference replay).
//
// What is differentiated. The step of the reference (solver.cpp:1036-1298) with every
// integer decision held at its outcome in the nominal FP32 run:
//   - the contact set and the contact geometry: feature keys, body-local anchors rA / rB and
//     the contact basis from the narrowphase (collide.cpp:898-955, manifold.cpp:119-160);
//   - the colouring (the order of the primal sweep);
//   - the normal-force clamp and the friction-cone scaling (manifold.cpp:200-212);
//   - the penalty ramp conditions, the signs of |C| in the ramp and the PENALTY_MAX caps
//     (manifold.cpp:268-278), and the warm-start penalty clamp (manifold.cpp:170);
//   - the adaptive warm-start weight clamp (solver.cpp:1146-1150).
// Between those decisions the step is a smooth map of the body states, the dual variables,
// the masses and the friction coefficients. C0 (manifold.cpp:164-167) stays a function of
// the poses at step start. The forward functions below are that smooth map; the *_vjp
// functions are its exact vector-Jacobian products.
//
// Conventions follow source/maths.h: quaternions are (x, y, z, w); rotate(q, v) =
// v + w t + u x t with t = 2 u x v; qdiff(a, b) = 2 vec(a * b^-1) (quat - quat);
// qstep(q, w) = normalize(q + (w, 0) * q / 2) (quat + float3). The 6-vectors are
// (linear, angular); the 6x6 systems hold lhsLin, lhsCross, lhsAng of solver.cpp:1189-1232.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define DHD __host__ __device__ __forceinline__
#else
#define DHD inline
#endif

namespace avbd_diff
{

// Solver constants (solver.h:20-24) as the FP32 run sees them.
constexpr double D_PENALTY_MIN = 1.0;
constexpr double D_PENALTY_MAX = 10000000000.0;
constexpr double D_COLLISION_MARGIN = (double)0.01f;

// Branch outcomes of one contact evaluation (primal or dual), from the nominal run.
enum EvalFlags : unsigned
{
    EF_NCLAMP = 1u,  // F.n >= 0: normal force clamped to 0
    EF_CONE = 2u,    // |F.t| > bounds and |F.t| > 0: tangential force scaled onto the cone
    EF_RAMP_T = 4u,  // dual: |F.t| <= bounds, tangential penalties ramp
    EF_CAP_X = 8u,   // dual: a ramped penalty reached PENALTY_MAX
    EF_CAP_Y = 16u,
    EF_CAP_Z = 32u,
    EF_NEG_X = 64u,  // dual: C < 0 (the ramp adds beta * |C|)
    EF_NEG_Y = 128u,
    EF_NEG_Z = 256u,
    EF_POS_X = 512u, // dual: C > 0
    EF_POS_Y = 1024u,
    EF_POS_Z = 2048u
};

// Warm-start penalty clamp of a carried-over contact (manifold.cpp:170).
enum InitFlags : unsigned
{
    IF_LO_X = 1u,
    IF_LO_Y = 2u,
    IF_LO_Z = 4u,
    IF_HI_X = 8u,
    IF_HI_Y = 16u,
    IF_HI_Z = 32u
};

// Per body and step.
enum BodyFlags : unsigned
{
    BF_DYNAMIC = 1u,   // mass > 0
    BF_FORCES = 2u,    // at least one force in the body's list (solver.cpp:1163-1168)
    BF_ACCEL_IN = 4u,  // adaptive weight strictly inside (0, 1)
    BF_ACCEL_ONE = 8u  // adaptive weight clamped at 1
};

template <class S>
struct V3
{
    S x, y, z;
};
template <class S>
struct Q4
{
    S x, y, z, w;
};

template <class S> DHD V3<S> v3(S x, S y, S z) { return V3<S>{x, y, z}; }
template <class S> DHD V3<S> vzero() { return V3<S>{S(0), S(0), S(0)}; }
template <class S> DHD Q4<S> qzero() { return Q4<S>{S(0), S(0), S(0), S(0)}; }
template <class S> DHD V3<S> operator+(V3<S> a, V3<S> b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class S> DHD V3<S> operator-(V3<S> a, V3<S> b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class S> DHD V3<S> operator-(V3<S> a) { return v3(-a.x, -a.y, -a.z); }
template <class S> DHD V3<S> operator*(V3<S> a, S s) { return v3(a.x * s, a.y * s, a.z * s); }
template <class S> DHD V3<S> hadamard(V3<S> a, V3<S> b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
template <class S> DHD V3<S> &operator+=(V3<S> &a, V3<S> b)
{
    a.x += b.x;
    a.y += b.y;
    a.z += b.z;
    return a;
}
template <class S> DHD S dot(V3<S> a, V3<S> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class S> DHD V3<S> cross(V3<S> a, V3<S> b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class S> DHD S comp(V3<S> v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
template <class S> DHD void add_comp(V3<S> &v, int i, S s)
{
    if (i == 0)
        v.x += s;
    else if (i == 1)
        v.y += s;
    else
        v.z += s;
}
template <class S> DHD void set_comp(V3<S> &v, int i, S s)
{
    if (i == 0)
        v.x = s;
    else if (i == 1)
        v.y = s;
    else
        v.z = s;
}

template <class S> DHD Q4<S> q4(S x, S y, S z, S w) { return Q4<S>{x, y, z, w}; }
template <class S> DHD V3<S> vec(Q4<S> q) { return v3(q.x, q.y, q.z); }
template <class S> DHD Q4<S> operator+(Q4<S> a, Q4<S> b) { return q4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
template <class S> DHD Q4<S> operator*(Q4<S> a, S s) { return q4(a.x * s, a.y * s, a.z * s, a.w * s); }
template <class S> DHD Q4<S> &operator+=(Q4<S> &a, Q4<S> b)
{
    a.x += b.x;
    a.y += b.y;
    a.z += b.z;
    a.w += b.w;
    return a;
}
template <class S> DHD S qdot(Q4<S> a, Q4<S> b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
template <class S> DHD Q4<S> qmul(Q4<S> a, Q4<S> b)
{
    return q4(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
              a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}
template <class S> DHD Q4<S> qconj(Q4<S> q) { return q4(-q.x, -q.y, -q.z, q.w); }

// ---------------------------------------------------------------------------
// Rotation and quaternion maps (maths.h:269-277, 417-446) with their VJPs
// ---------------------------------------------------------------------------

template <class S> DHD V3<S> rotate(Q4<S> q, V3<S> v)
{
    V3<S> u = vec(q);
    V3<S> t = cross(u, v) * S(2);
    return (v + t * q.w) + cross(u, t);
}

// q-adjoint of rotate(q, v) for the output adjoint rbar (v fixed)
template <class S> DHD Q4<S> rotate_vjp_q(Q4<S> q, V3<S> v, V3<S> rbar)
{
    V3<S> u = vec(q);
    V3<S> t = cross(u, v) * S(2);
    V3<S> tbar = rbar * q.w + cross(rbar, u);
    V3<S> ubar = cross(t, rbar) + cross(v, tbar) * S(2);
    return q4(ubar.x, ubar.y, ubar.z, dot(rbar, t));
}

// v-adjoint of rotate(q, v)
template <class S> DHD V3<S> rotate_vjp_v(Q4<S> q, V3<S> rbar)
{
    V3<S> u = vec(q);
    V3<S> tbar = rbar * q.w + cross(rbar, u);
    return rbar + cross(tbar, u) * S(2);
}

template <class S> DHD V3<S> qdiff(Q4<S> a, Q4<S> b)
{
    S n2 = qdot(b, b);
    Q4<S> c = qconj(b) * (S(1) / n2);
    return vec(qmul(a, c)) * S(2);
}

template <class S> DHD void qdiff_vjp(Q4<S> a, Q4<S> b, V3<S> rbar, Q4<S> &abar, Q4<S> &bbar)
{
    S n2 = qdot(b, b);
    Q4<S> c = qconj(b) * (S(1) / n2);
    Q4<S> hbar = q4(rbar.x * S(2), rbar.y * S(2), rbar.z * S(2), S(0));
    abar += qmul(hbar, qconj(c));
    Q4<S> cbar = qmul(qconj(a), hbar);
    // c = conj(b) / |b|^2
    S sdot = -cbar.x * b.x - cbar.y * b.y - cbar.z * b.z + cbar.w * b.w;
    S k = S(2) * sdot / (n2 * n2);
    bbar += q4(-cbar.x / n2 - k * b.x, -cbar.y / n2 - k * b.y, -cbar.z / n2 - k * b.z, cbar.w / n2 - k * b.w);
}

template <class S> DHD Q4<S> qstep(Q4<S> q, V3<S> w)
{
    Q4<S> y = q + qmul(q4(w.x, w.y, w.z, S(0)), q) * S(0.5);
    S n = sqrt(qdot(y, y));
    return y * (S(1) / n);
}

template <class S> DHD void qstep_vjp(Q4<S> q, V3<S> w, Q4<S> rbar, Q4<S> &qbar, V3<S> &wbar)
{
    Q4<S> P = q4(w.x, w.y, w.z, S(0));
    Q4<S> y = q + qmul(P, q) * S(0.5);
    S n = sqrt(qdot(y, y));
    Q4<S> r = y * (S(1) / n);
    S rr = qdot(r, rbar);
    Q4<S> ybar =
        q4((rbar.x - r.x * rr) / n, (rbar.y - r.y * rr) / n, (rbar.z - r.z * rr) / n, (rbar.w - r.w * rr) / n);
    qbar += ybar + qmul(qconj(P), ybar) * S(0.5);
    Q4<S> Pbar = qmul(ybar, qconj(q)) * S(0.5);
    wbar += v3(Pbar.x, Pbar.y, Pbar.z);
}

// ---------------------------------------------------------------------------
// Poses and contacts
// ---------------------------------------------------------------------------

// A body's current pose and its pose at step start (Rigid::initial*).
template <class S>
struct Pose
{
    V3<S> p, pi;
    Q4<S> q, qi;
};

template <class S>
struct PoseBar
{
    V3<S> p, pi;
    Q4<S> q, qi;
};

template <class S> DHD PoseBar<S> posebar_zero()
{
    PoseBar<S> b;
    b.p = vzero<S>();
    b.pi = vzero<S>();
    b.q = qzero<S>();
    b.qi = qzero<S>();
    return b;
}

// One contact of a manifold: frozen geometry (rA, rB body-local, basis rows e[0] = normal,
// e[1], e[2] tangents) and the differentiated C0, lambda, penalty and friction.
template <class S>
struct ContactIn
{
    V3<S> rA, rB;
    V3<S> e[3];
    V3<S> C0, lam, pen;
    S mu;
};

template <class S>
struct ContactFwd
{
    V3<S> C, Fpre, F;   // constraint value, force before / after the clamps
    V3<S> jA[3], jB[3]; // angular Jacobian rows of body A and body B
    S fs, bounds;
};

// Manifold::updatePrimal / updateDual front half (manifold.cpp:183-212) on the frozen
// branches: C = C0 (1 - alpha) + J dq, F = K C + lambda, then the recorded clamps.
template <class S> DHD ContactFwd<S> contact_forward(const Pose<S> &A, const Pose<S> &B, const ContactIn<S> &c, S alpha,
                                                     unsigned flags)
{
    ContactFwd<S> f;
    V3<S> dA = A.p - A.pi, dB = B.p - B.pi;
    V3<S> wA = qdiff(A.q, A.qi), wB = qdiff(B.q, B.qi);
    V3<S> rAW = rotate(A.q, c.rA);
    V3<S> rBW = rotate(B.q, c.rB);
    S C[3];
    for (int k = 0; k < 3; ++k)
    {
        f.jA[k] = cross(rAW, c.e[k]);
        f.jB[k] = cross(rBW, -c.e[k]);
        C[k] = comp(c.C0, k) * (S(1) - alpha) + dot(c.e[k], dA) - dot(c.e[k], dB) + dot(f.jA[k], wA) +
               dot(f.jB[k], wB);
    }
    f.C = v3(C[0], C[1], C[2]);
    f.Fpre = v3(c.pen.x * C[0] + c.lam.x, c.pen.y * C[1] + c.lam.y, c.pen.z * C[2] + c.lam.z);
    V3<S> F = f.Fpre;
    // |F.n| with the nominal sign: F.n < 0 whenever it is not clamped
    if (flags & EF_NCLAMP)
    {
        F.x = S(0);
        f.bounds = S(0);
    }
    else
        f.bounds = -F.x * c.mu;
    f.fs = sqrt(F.y * F.y + F.z * F.z);
    if (flags & EF_CONE)
    {
        S s = f.bounds / f.fs;
        F.y = F.y * s;
        F.z = F.z * s;
    }
    f.F = F;
    return f;
}

// Adjoint of the clamped force F to the force before the clamps, and to the friction.
template <class S> DHD V3<S> force_clamp_vjp(const ContactFwd<S> &f, V3<S> Fbar, unsigned flags, S mu, S &mubar)
{
    V3<S> Fpb = Fbar;
    if (flags & EF_CONE)
    {
        S Fy = f.Fpre.y, Fz = f.Fpre.z;
        S s = f.bounds / f.fs;
        S tdot = Fy * Fbar.y + Fz * Fbar.z;
        S k = f.bounds / (f.fs * f.fs * f.fs);
        Fpb.y = s * Fbar.y - k * tdot * Fy;
        Fpb.z = s * Fbar.z - k * tdot * Fz;
        S bbar = tdot / f.fs;
        if (!(flags & EF_NCLAMP))
        {
            // bounds = -F.n * mu
            Fpb.x += -bbar * mu;
            mubar += -bbar * f.Fpre.x;
        }
    }
    if (flags & EF_NCLAMP)
        Fpb.x = S(0);
    return Fpb;
}

// Adjoint of C to both poses, the angular Jacobian rows and C0.
template <class S> DHD void constraint_vjp(const Pose<S> &A, const Pose<S> &B, const ContactIn<S> &c, const ContactFwd<S> &f,
                                           V3<S> Cbar, S alpha, PoseBar<S> &Ab, PoseBar<S> &Bb, V3<S> jAbar[3],
                                           V3<S> jBbar[3], V3<S> &C0bar)
{
    V3<S> wA = qdiff(A.q, A.qi), wB = qdiff(B.q, B.qi);
    V3<S> dAbar = vzero<S>(), wAbar = vzero<S>(), wBbar = vzero<S>();
    for (int k = 0; k < 3; ++k)
    {
        S cb = comp(Cbar, k);
        add_comp(C0bar, k, cb * (S(1) - alpha));
        dAbar += c.e[k] * cb;
        wAbar += f.jA[k] * cb;
        wBbar += f.jB[k] * cb;
        jAbar[k] += wA * cb;
        jBbar[k] += wB * cb;
    }
    Ab.p += dAbar;
    Ab.pi += -dAbar;
    Bb.p += -dAbar;
    Bb.pi += dAbar;
    qdiff_vjp(A.q, A.qi, wAbar, Ab.q, Ab.qi);
    qdiff_vjp(B.q, B.qi, wBbar, Bb.q, Bb.qi);
}

// Jacobian rows jA_k = rAW x e_k, jB_k = rBW x (-e_k) back to the orientations.
template <class S> DHD void jacobian_rows_vjp(const ContactIn<S> &c, const V3<S> jAbar[3], const V3<S> jBbar[3],
                                              const Pose<S> &A, const Pose<S> &B, PoseBar<S> &Ab, PoseBar<S> &Bb)
{
    V3<S> rAb = vzero<S>(), rBb = vzero<S>();
    for (int k = 0; k < 3; ++k)
    {
        rAb += cross(c.e[k], jAbar[k]);
        rBb += cross(-c.e[k], jBbar[k]);
    }
    Ab.q += rotate_vjp_q(A.q, c.rA, rAb);
    Bb.q += rotate_vjp_q(B.q, c.rB, rBb);
}

// ---------------------------------------------------------------------------
// 6x6 systems and the LDL^T solve (maths.h:481-547)
// ---------------------------------------------------------------------------

template <class S>
struct Sys6
{
    S H[6][6];
    S g[6];
};

template <class S> DHD void sys_zero(Sys6<S> &s)
{
    for (int i = 0; i < 6; ++i)
    {
        s.g[i] = S(0);
        for (int j = 0; j < 6; ++j)
            s.H[i][j] = S(0);
    }
}

// Rows of one contact for the updated body: J (3x6) = [+-basis | jA or jB].
template <class S> DHD void contact_rows(const ContactIn<S> &c, const ContactFwd<S> &f, bool isA, S J[3][6])
{
    S sign = isA ? S(1) : S(-1);
    for (int k = 0; k < 3; ++k)
    {
        V3<S> ja = isA ? f.jA[k] : f.jB[k];
        J[k][0] = c.e[k].x * sign;
        J[k][1] = c.e[k].y * sign;
        J[k][2] = c.e[k].z * sign;
        J[k][3] = ja.x;
        J[k][4] = ja.y;
        J[k][5] = ja.z;
    }
}

// H += J^T K J, g += J^T F (manifold.cpp:214-228)
template <class S> DHD void stamp_contact(Sys6<S> &s, const ContactIn<S> &c, const ContactFwd<S> &f, bool isA)
{
    S J[3][6];
    contact_rows(c, f, isA, J);
    S K[3] = {c.pen.x, c.pen.y, c.pen.z};
    S F[3] = {f.F.x, f.F.y, f.F.z};
    for (int i = 0; i < 6; ++i)
    {
        for (int k = 0; k < 3; ++k)
            s.g[i] += J[k][i] * F[k];
        for (int j = 0; j < 6; ++j)
            for (int k = 0; k < 3; ++k)
                s.H[i][j] += J[k][i] * K[k] * J[k][j];
    }
}

// Adjoint of one contact stamp (full-matrix adjoint Hbar and gbar) to F, the penalty
// and the updated body's angular Jacobian rows.
template <class S> DHD void stamp_contact_vjp(const Sys6<S> &bar, const ContactIn<S> &c, const ContactFwd<S> &f, bool isA,
                                              V3<S> &Fbar, V3<S> &penbar, V3<S> jbar[3])
{
    S J[3][6];
    contact_rows(c, f, isA, J);
    S K[3] = {c.pen.x, c.pen.y, c.pen.z};
    S F[3] = {f.F.x, f.F.y, f.F.z};
    for (int k = 0; k < 3; ++k)
    {
        S fb = S(0), kb = S(0);
        S Jb[6];
        for (int i = 0; i < 6; ++i)
        {
            fb += J[k][i] * bar.g[i];
            S hs = S(0), hq = S(0);
            for (int j = 0; j < 6; ++j)
            {
                hs += (bar.H[i][j] + bar.H[j][i]) * J[k][j];
                hq += bar.H[i][j] * J[k][j];
            }
            Jb[i] = bar.g[i] * F[k] + K[k] * hs;
            kb += J[k][i] * hq;
        }
        add_comp(Fbar, k, fb);
        add_comp(penbar, k, kb);
        jbar[k] += v3(Jb[3], Jb[4], Jb[5]);
    }
}

template <class S>
struct Ldl6
{
    S L[6][6];
    S D[6];
};

// Unpivoted LDL^T of a symmetric positive definite 6x6.
template <class S> DHD void ldl_factor(const S H[6][6], Ldl6<S> &f)
{
    for (int j = 0; j < 6; ++j)
    {
        S d = H[j][j];
        for (int k = 0; k < j; ++k)
            d -= f.L[j][k] * f.L[j][k] * f.D[k];
        f.D[j] = d;
        for (int i = j + 1; i < 6; ++i)
        {
            S v = H[i][j];
            for (int k = 0; k < j; ++k)
                v -= f.L[j][k] * f.L[i][k] * f.D[k];
            f.L[i][j] = v / d;
        }
    }
}

template <class S> DHD void ldl_solve(const Ldl6<S> &f, const S b[6], S x[6])
{
    S y[6];
    for (int i = 0; i < 6; ++i)
    {
        S v = b[i];
        for (int k = 0; k < i; ++k)
            v -= f.L[i][k] * y[k];
        y[i] = v;
    }
    for (int i = 5; i >= 0; --i)
    {
        S v = y[i] / f.D[i];
        for (int k = i + 1; k < 6; ++k)
            v -= f.L[k][i] * x[k];
        x[i] = v;
    }
}

// Inertial part (solver.cpp:1189-1198): H0 = diag(m, m, m, I) / dt^2,
// g0 = [m (p - p~); I o qdiff(q, q~)] / dt^2, with I = m * shape (rigid.cpp:34-39).
template <class S> DHD void stamp_inertia(Sys6<S> &s, S m, V3<S> shape, V3<S> p, V3<S> pt, Q4<S> q, Q4<S> qt, S dt)
{
    S idt2 = S(1) / (dt * dt);
    V3<S> d = p - pt, a = qdiff(q, qt);
    V3<S> I = shape * m;
    s.H[0][0] += m * idt2;
    s.H[1][1] += m * idt2;
    s.H[2][2] += m * idt2;
    s.H[3][3] += I.x * idt2;
    s.H[4][4] += I.y * idt2;
    s.H[5][5] += I.z * idt2;
    s.g[0] += m * idt2 * d.x;
    s.g[1] += m * idt2 * d.y;
    s.g[2] += m * idt2 * d.z;
    s.g[3] += I.x * idt2 * a.x;
    s.g[4] += I.y * idt2 * a.y;
    s.g[5] += I.z * idt2 * a.z;
}

template <class S> DHD void stamp_inertia_vjp(const Sys6<S> &bar, S m, V3<S> shape, V3<S> p, V3<S> pt, Q4<S> q, Q4<S> qt,
                                              S dt, S &mbar, V3<S> &pbar, V3<S> &ptbar, Q4<S> &qbar, Q4<S> &qtbar)
{
    S idt2 = S(1) / (dt * dt);
    V3<S> d = p - pt, a = qdiff(q, qt);
    V3<S> I = shape * m;
    mbar += (bar.g[0] * d.x + bar.g[1] * d.y + bar.g[2] * d.z + bar.H[0][0] + bar.H[1][1] + bar.H[2][2]) * idt2;
    mbar += (shape.x * (bar.g[3] * a.x + bar.H[3][3]) + shape.y * (bar.g[4] * a.y + bar.H[4][4]) +
             shape.z * (bar.g[5] * a.z + bar.H[5][5])) *
            idt2;
    V3<S> dbar = v3(bar.g[0], bar.g[1], bar.g[2]) * (m * idt2);
    pbar += dbar;
    ptbar += -dbar;
    V3<S> abar = v3(I.x * bar.g[3], I.y * bar.g[4], I.z * bar.g[5]) * idt2;
    qdiff_vjp(q, qt, abar, qbar, qtbar);
}

// dx = -H^-1 g with the factor of H
template <class S> DHD void body_dx(const Ldl6<S> &f, const Sys6<S> &s, S dx[6])
{
    S b[6];
    for (int i = 0; i < 6; ++i)
        b[i] = -s.g[i];
    ldl_solve(f, b, dx);
}

// Adjoint of dx = -H^-1 g: u = H^-1 dxbar, gbar = -u, Hbar = -u dx^T.
template <class S> DHD void body_dx_vjp(const Ldl6<S> &f, const S dx[6], const S dxbar[6], Sys6<S> &bar)
{
    S u[6];
    ldl_solve(f, dxbar, u);
    for (int i = 0; i < 6; ++i)
    {
        bar.g[i] = -u[i];
        for (int j = 0; j < 6; ++j)
            bar.H[i][j] = -u[i] * dx[j];
    }
}

// The system adjoint of dx = -H^-1 g is rank one: Hbar = -u dx^T, gbar = -u with
// u = H^-1 dxbar. These forms of the stamp VJPs take (u, dx) instead of the 42 entries.
template <class S> DHD void body_dx_vjp_u(const Ldl6<S> &f, const S dxbar[6], S u[6]) { ldl_solve(f, dxbar, u); }

// stamp_contact_vjp for Hbar = -u dx^T, gbar = -u: with a_k = J_k . u and d_k = J_k . dx,
// Fbar_k = -a_k, Kbar_k = -a_k d_k, Jbar_k = -u F_k - K_k (u d_k + dx a_k).
template <class S> DHD void stamp_contact_vjp_outer(const S u[6], const S dx[6], const ContactIn<S> &c,
                                                    const ContactFwd<S> &f, bool isA, V3<S> &Fbar, V3<S> &penbar,
                                                    V3<S> jbar[3])
{
    S J[3][6];
    contact_rows(c, f, isA, J);
    S K[3] = {c.pen.x, c.pen.y, c.pen.z};
    S F[3] = {f.F.x, f.F.y, f.F.z};
    for (int k = 0; k < 3; ++k)
    {
        S a = S(0), d = S(0);
        for (int i = 0; i < 6; ++i)
        {
            a += J[k][i] * u[i];
            d += J[k][i] * dx[i];
        }
        add_comp(Fbar, k, -a);
        add_comp(penbar, k, -a * d);
        S Jb[3];
        for (int i = 3; i < 6; ++i)
            Jb[i - 3] = -u[i] * F[k] - K[k] * (u[i] * d + dx[i] * a);
        jbar[k] += v3(Jb[0], Jb[1], Jb[2]);
    }
}

template <class S> DHD void stamp_inertia_vjp_outer(const S u[6], const S dx[6], S m, V3<S> shape, V3<S> p, V3<S> pt,
                                                    Q4<S> q, Q4<S> qt, S dt, S &mbar, V3<S> &pbar, V3<S> &ptbar,
                                                    Q4<S> &qbar, Q4<S> &qtbar)
{
    Sys6<S> bar;
    for (int i = 0; i < 6; ++i)
    {
        bar.g[i] = -u[i];
        bar.H[i][i] = -u[i] * dx[i];
    }
    // stamp_inertia_vjp reads gbar and the diagonal of Hbar only
    S idt2 = S(1) / (dt * dt);
    V3<S> d = p - pt, a = qdiff(q, qt);
    V3<S> I = shape * m;
    mbar += (bar.g[0] * d.x + bar.g[1] * d.y + bar.g[2] * d.z + bar.H[0][0] + bar.H[1][1] + bar.H[2][2]) * idt2;
    mbar += (shape.x * (bar.g[3] * a.x + bar.H[3][3]) + shape.y * (bar.g[4] * a.y + bar.H[4][4]) +
             shape.z * (bar.g[5] * a.z + bar.H[5][5])) *
            idt2;
    V3<S> dbar = v3(bar.g[0], bar.g[1], bar.g[2]) * (m * idt2);
    pbar += dbar;
    ptbar += -dbar;
    V3<S> abar = v3(I.x * bar.g[3], I.y * bar.g[4], I.z * bar.g[5]) * idt2;
    qdiff_vjp(q, qt, abar, qbar, qtbar);
}

// ---------------------------------------------------------------------------
// Per-contact pieces of the step
// ---------------------------------------------------------------------------

// Rest of a contact row's primal adjoint once the stamp is reversed (Fbar, jb).
template <class S> DHD void contact_row_vjp(const Pose<S> &A, const Pose<S> &B, const ContactIn<S> &c,
                                            const ContactFwd<S> &f, S alpha, unsigned flags, bool isA, V3<S> Fbar,
                                            const V3<S> jb[3], PoseBar<S> &Ab, PoseBar<S> &Bb, V3<S> &lambar,
                                            V3<S> &penbar, V3<S> &C0bar, S &mubar);

// Primal adjoint of one contact row for the body being solved: from the system adjoint to
// both poses, lambda, penalty, C0 and friction.
template <class S> DHD void contact_primal_vjp(const Pose<S> &A, const Pose<S> &B, const ContactIn<S> &c, S alpha,
                                               unsigned flags, bool isA, const Sys6<S> &sysbar, PoseBar<S> &Ab,
                                               PoseBar<S> &Bb, V3<S> &lambar, V3<S> &penbar, V3<S> &C0bar, S &mubar)
{
    ContactFwd<S> f = contact_forward(A, B, c, alpha, flags);
    V3<S> Fbar = vzero<S>();
    V3<S> jb[3] = {vzero<S>(), vzero<S>(), vzero<S>()};
    stamp_contact_vjp(sysbar, c, f, isA, Fbar, penbar, jb);
    contact_row_vjp(A, B, c, f, alpha, flags, isA, Fbar, jb, Ab, Bb, lambar, penbar, C0bar, mubar);
}

// The same with the rank-one system adjoint (u, dx).
template <class S> DHD void contact_primal_vjp_outer(const Pose<S> &A, const Pose<S> &B, const ContactIn<S> &c,
                                                     S alpha, unsigned flags, bool isA, const S u[6], const S dx[6],
                                                     PoseBar<S> &Ab, PoseBar<S> &Bb, V3<S> &lambar, V3<S> &penbar,
                                                     V3<S> &C0bar, S &mubar)
{
    ContactFwd<S> f = contact_forward(A, B, c, alpha, flags);
    V3<S> Fbar = vzero<S>();
    V3<S> jb[3] = {vzero<S>(), vzero<S>(), vzero<S>()};
    stamp_contact_vjp_outer(u, dx, c, f, isA, Fbar, penbar, jb);
    contact_row_vjp(A, B, c, f, alpha, flags, isA, Fbar, jb, Ab, Bb, lambar, penbar, C0bar, mubar);
}

template <class S> DHD void contact_row_vjp(const Pose<S> &A, const Pose<S> &B, const ContactIn<S> &c,
                                            const ContactFwd<S> &f, S alpha, unsigned flags, bool isA, V3<S> Fbar,
                                            const V3<S> jb[3], PoseBar<S> &Ab, PoseBar<S> &Bb, V3<S> &lambar,
                                            V3<S> &penbar, V3<S> &C0bar, S &mubar)
{
    V3<S> Fpb = force_clamp_vjp(f, Fbar, flags, c.mu, mubar);
    lambar += Fpb;
    penbar += hadamard(Fpb, f.C);
    V3<S> Cbar = hadamard(c.pen, Fpb);
    V3<S> jAbar[3] = {vzero<S>(), vzero<S>(), vzero<S>()};
    V3<S> jBbar[3] = {vzero<S>(), vzero<S>(), vzero<S>()};
    for (int k = 0; k < 3; ++k)
    {
        if (isA)
            jAbar[k] = jb[k];
        else
            jBbar[k] = jb[k];
    }
    constraint_vjp(A, B, c, f, Cbar, alpha, Ab, Bb, jAbar, jBbar, C0bar);
    jacobian_rows_vjp(c, jAbar, jBbar, A, B, Ab, Bb);
}

// Manifold::updateDual (manifold.cpp:231-279) on frozen branches: lambda' = F and the
// penalty ramp pen' = min(pen + beta |C|, PENALTY_MAX) where it applies.
template <class S> DHD void contact_dual_forward(const Pose<S> &A, const Pose<S> &B, const ContactIn<S> &c, S alpha,
                                                 S beta, unsigned flags, V3<S> &lamOut, V3<S> &penOut)
{
    ContactFwd<S> f = contact_forward(A, B, c, alpha, flags);
    lamOut = f.F;
    penOut = c.pen;
    const unsigned capBit[3] = {EF_CAP_X, EF_CAP_Y, EF_CAP_Z};
    const unsigned negBit[3] = {EF_NEG_X, EF_NEG_Y, EF_NEG_Z};
    const unsigned posBit[3] = {EF_POS_X, EF_POS_Y, EF_POS_Z};
    for (int k = 0; k < 3; ++k)
    {
        bool ramp = k == 0 ? !(flags & EF_NCLAMP) : (flags & EF_RAMP_T) != 0;
        if (!ramp)
            continue;
        S sgn = (flags & negBit[k]) ? S(-1) : ((flags & posBit[k]) ? S(1) : S(0));
        S v = (flags & capBit[k]) ? S(D_PENALTY_MAX) : comp(c.pen, k) + beta * sgn * comp(f.C, k);
        set_comp(penOut, k, v);
    }
}

// Adjoint of the dual update. lambar / penbar enter as the adjoints of lambda' / pen' and
// leave as those of lambda / pen.
template <class S> DHD void contact_dual_vjp(const Pose<S> &A, const Pose<S> &B, const ContactIn<S> &c, S alpha, S beta,
                                             unsigned flags, V3<S> &lambar, V3<S> &penbar, PoseBar<S> &Ab,
                                             PoseBar<S> &Bb, V3<S> &C0bar, S &mubar)
{
    ContactFwd<S> f = contact_forward(A, B, c, alpha, flags);
    const unsigned capBit[3] = {EF_CAP_X, EF_CAP_Y, EF_CAP_Z};
    const unsigned negBit[3] = {EF_NEG_X, EF_NEG_Y, EF_NEG_Z};
    const unsigned posBit[3] = {EF_POS_X, EF_POS_Y, EF_POS_Z};
    V3<S> Cbar = vzero<S>();
    V3<S> penIn = penbar;
    for (int k = 0; k < 3; ++k)
    {
        bool ramp = k == 0 ? !(flags & EF_NCLAMP) : (flags & EF_RAMP_T) != 0;
        if (!ramp)
            continue;
        S pb = comp(penbar, k);
        if (flags & capBit[k])
            pb = S(0);
        else
        {
            S sgn = (flags & negBit[k]) ? S(-1) : ((flags & posBit[k]) ? S(1) : S(0));
            add_comp(Cbar, k, pb * beta * sgn);
        }
        set_comp(penIn, k, pb);
    }
    V3<S> Fpb = force_clamp_vjp(f, lambar, flags, c.mu, mubar);
    lambar = Fpb;
    penbar = penIn + hadamard(Fpb, f.C);
    Cbar += hadamard(c.pen, Fpb);
    V3<S> jAbar[3] = {vzero<S>(), vzero<S>(), vzero<S>()};
    V3<S> jBbar[3] = {vzero<S>(), vzero<S>(), vzero<S>()};
    constraint_vjp(A, B, c, f, Cbar, alpha, Ab, Bb, jAbar, jBbar, C0bar);
    jacobian_rows_vjp(c, jAbar, jBbar, A, B, Ab, Bb);
}

// Manifold::initialize (manifold.cpp:162-171): C0 = basis (xA - xB) + (margin, 0, 0) at the
// poses of step start.
template <class S> DHD V3<S> contact_C0(V3<S> pA, Q4<S> qA, V3<S> pB, Q4<S> qB, V3<S> rA, V3<S> rB, const V3<S> e[3])
{
    V3<S> d = (pA + rotate(qA, rA)) - (pB + rotate(qB, rB));
    return v3(dot(e[0], d) + S(D_COLLISION_MARGIN), dot(e[1], d), dot(e[2], d));
}

template <class S> DHD void contact_C0_vjp(Q4<S> qA, Q4<S> qB, V3<S> rA, V3<S> rB, const V3<S> e[3], V3<S> C0bar,
                                           V3<S> &pAbar, Q4<S> &qAbar, V3<S> &pBbar, Q4<S> &qBbar)
{
    V3<S> d = e[0] * C0bar.x + e[1] * C0bar.y + e[2] * C0bar.z;
    pAbar += d;
    qAbar += rotate_vjp_q(qA, rA, d);
    pBbar += -d;
    qBbar += rotate_vjp_q(qB, rB, -d);
}

// Carried-over lambda and penalty (manifold.cpp:169-170).
template <class S> DHD void contact_carry(V3<S> lamPrev, V3<S> penPrev, bool hasSrc, unsigned iflags, S alpha, S gamma,
                                          V3<S> &lam, V3<S> &pen)
{
    if (!hasSrc)
    {
        lam = vzero<S>();
        pen = v3(S(D_PENALTY_MIN), S(D_PENALTY_MIN), S(D_PENALTY_MIN));
        return;
    }
    lam = (lamPrev * alpha) * gamma;
    V3<S> p = penPrev * gamma;
    pen.x = (iflags & IF_LO_X) ? S(D_PENALTY_MIN) : ((iflags & IF_HI_X) ? S(D_PENALTY_MAX) : p.x);
    pen.y = (iflags & IF_LO_Y) ? S(D_PENALTY_MIN) : ((iflags & IF_HI_Y) ? S(D_PENALTY_MAX) : p.y);
    pen.z = (iflags & IF_LO_Z) ? S(D_PENALTY_MIN) : ((iflags & IF_HI_Z) ? S(D_PENALTY_MAX) : p.z);
}

template <class S> DHD void contact_carry_vjp(V3<S> lambar, V3<S> penbar, unsigned iflags, S alpha, S gamma,
                                              V3<S> &lamPrevBar, V3<S> &penPrevBar)
{
    lamPrevBar += lambar * (alpha * gamma);
    penPrevBar += v3((iflags & (IF_LO_X | IF_HI_X)) ? S(0) : penbar.x * gamma,
                     (iflags & (IF_LO_Y | IF_HI_Y)) ? S(0) : penbar.y * gamma,
                     (iflags & (IF_LO_Z | IF_HI_Z)) ? S(0) : penbar.z * gamma);
}

// ---------------------------------------------------------------------------
// Per-body pieces of the step
// ---------------------------------------------------------------------------

template <class S>
struct WarmOut
{
    V3<S> p, inertLin;
    Q4<S> q, inertAng;
};

// Body warm start (solver.cpp:1134-1169) for a dynamic body; initial pose = (p0, q0).
template <class S> DHD WarmOut<S> warm_start(V3<S> p0, Q4<S> q0, V3<S> v, V3<S> w, V3<S> vp, S dt, S g, unsigned bflags)
{
    WarmOut<S> o;
    o.inertLin = (p0 + v * dt) + v3(S(0), S(0), g) * (dt * dt);
    o.inertAng = qstep(q0, w * dt);
    S sg = g < S(0) ? S(-1) : (g > S(0) ? S(1) : S(0));
    S ag = g < S(0) ? -g : g;
    S weight = S(0);
    if (bflags & BF_ACCEL_IN)
        weight = ((v.z - vp.z) / dt) * sg / ag;
    else if (bflags & BF_ACCEL_ONE)
        weight = S(1);
    o.p = (p0 + v * dt) + v3(S(0), S(0), g) * (weight * dt * dt);
    o.q = o.inertAng;
    if (!(bflags & BF_FORCES))
        o.p = o.inertLin;
    return o;
}

// Adjoint of the warm start: from the adjoints of the warm-started pose, the inertial
// pose and the initial pose (the latter = the pose at step start) to the step-start state.
template <class S> DHD void warm_start_vjp(Q4<S> q0, V3<S> w, S dt, S g, unsigned bflags, V3<S> pbar, Q4<S> qbar,
                                           V3<S> inertLinBar, Q4<S> inertAngBar, V3<S> initLinBar, Q4<S> initAngBar,
                                           V3<S> &p0bar, Q4<S> &q0bar, V3<S> &vbar, V3<S> &wbar, V3<S> &vpbar)
{
    if (!(bflags & BF_FORCES))
    {
        inertLinBar += pbar;
        pbar = vzero<S>();
    }
    p0bar += pbar + inertLinBar + initLinBar;
    vbar += (pbar + inertLinBar) * dt;
    if (bflags & BF_ACCEL_IN)
    {
        S sg = g < S(0) ? S(-1) : (g > S(0) ? S(1) : S(0));
        S ag = g < S(0) ? -g : g;
        S wb = pbar.z * g * dt * dt;
        S d = wb * sg / (dt * ag);
        vbar.z += d;
        vpbar.z += -d;
    }
    Q4<S> qsum = qbar + inertAngBar;
    V3<S> wsb = vzero<S>();
    qstep_vjp(q0, w * dt, qsum, q0bar, wsb);
    wbar += wsb * dt;
    q0bar += initAngBar;
}

// finishStep (solver.cpp:1275-1287): v = (p - p0) / dt, w = qdiff(q, q0) / dt; the
// previous velocity becomes the step-start velocity (handled by the caller).
template <class S> DHD void finish_vjp(Q4<S> q, Q4<S> q0, S dt, V3<S> vbar, V3<S> wbar, V3<S> &pbar, Q4<S> &qbar,
                                       V3<S> &p0bar, Q4<S> &q0bar)
{
    S idt = S(1) / dt;
    pbar += vbar * idt;
    p0bar += -(vbar * idt);
    qdiff_vjp(q, q0, wbar * idt, qbar, q0bar);
}

} // namespace avbd_diff
