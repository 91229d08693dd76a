// Round shapes (sphere, capsule, cylinder): narrowphase, contact offsets and the sphere
// rolling friction, with the reference's operation order (collide.cpp:435-1176,
// manifold.cpp:16-91, solver.cpp:628-662). Included by avbd_kernels.cuh inside namespace
// avbd, after the box narrowphase, which the cylinder-box fallback reuses.
#pragma once

// RigidShapeType (solver.h:47-53)
constexpr int SHAPE_BOX = 0, SHAPE_SPHERE = 1, SHAPE_CAPSULE = 2, SHAPE_CYLINDER = 3;
constexpr float SAT_EPS = 1.0e-6f; // SAT_AXIS_EPSILON (collide.cpp:20)
constexpr float ROUND_FLAG = 1.0f; // basis row 1 .w of a manifold with a round body

struct BodyShape
{
    int type;
    float radius, halfLength;
};

// Shape of body b; no shape array means every body is a box.
AVBD_DEV BodyShape body_shape(const DevBodies &B, int b)
{
    BodyShape s{SHAPE_BOX, 0.0f, 0.0f};
    if (B.shape)
    {
        float4 v = B.shape[b];
        s.type = (int)v.x;
        s.radius = v.y;
        s.halfLength = v.z;
    }
    return s;
}

// What the narrowphase reads of a body.
struct NpBody
{
    float3 p, v, size;
    float4 q;
    float mass;
    BodyShape s;
};

AVBD_DEV NpBody np_body(const DevBodies &B, int b)
{
    NpBody r;
    r.p = xyz(B.pos[b]);
    r.q = B.quat[b];
    r.v = xyz(B.vel[b]);
    r.size = xyz(B.sizeRad[b]);
    r.mass = B.massMoment[b].x;
    r.s = body_shape(B, b);
    return r;
}

AVBD_DEV bool is_round(const NpBody &b) { return b.s.type == SHAPE_SPHERE || b.s.type == SHAPE_CAPSULE; }
AVBD_DEV bool is_cylinder(const NpBody &b) { return b.s.type == SHAPE_CYLINDER; }
AVBD_DEV void set_comp(float3 &v, int i, float x)
{
    if (i == 0)
        v.x = x;
    else if (i == 1)
        v.y = x;
    else
        v.z = x;
}
AVBD_DEV float3 normalized(float3 v) { return divs(v, len(v)); }

AVBD_DEV float3 obb_closest(const Obb &o, float3 p)
{
    float3 d = sub(p, o.c);
    return add(add(add(o.c, mul(o.ax[0], rclamp(dot(d, o.ax[0]), -o.h.x, o.h.x))),
                   mul(o.ax[1], rclamp(dot(d, o.ax[1]), -o.h.y, o.h.y))),
               mul(o.ax[2], rclamp(dot(d, o.ax[2]), -o.h.z, o.h.z)));
}

AVBD_DEV float3 obb_local(const Obb &o, float3 p)
{
    float3 d = sub(p, o.c);
    return f3(dot(d, o.ax[0]), dot(d, o.ax[1]), dot(d, o.ax[2]));
}

AVBD_DEV bool obb_inside(const Obb &o, float3 p, float3 &local)
{
    local = obb_local(o, p);
    return fabsf(local.x) <= o.h.x && fabsf(local.y) <= o.h.y && fabsf(local.z) <= o.h.z;
}

AVBD_DEV float3 obb_world(const Obb &o, float3 l)
{
    return add(add(add(o.c, mul(o.ax[0], l.x)), mul(o.ax[1], l.y)), mul(o.ax[2], l.z));
}

// capsuleSegment / cylinderSegment (collide.cpp:468-488): a sphere is a point segment
AVBD_DEV void round_segment(const NpBody &b, float3 &a, float3 &c)
{
    if (b.s.type == SHAPE_CAPSULE || b.s.type == SHAPE_CYLINDER)
    {
        float3 axis = rotate(b.q, f3(0.0f, 0.0f, 1.0f));
        a = sub(b.p, mul(axis, b.s.halfLength));
        c = add(b.p, mul(axis, b.s.halfLength));
    }
    else
    {
        a = b.p;
        c = b.p;
    }
}

AVBD_DEV float3 segment_closest(float3 a, float3 b, float3 p)
{
    float3 ab = sub(b, a);
    float denom = lensq(ab);
    if (denom < SAT_EPS)
        return a;
    float t = rclamp(dot(sub(p, a), ab) / denom, 0.0f, 1.0f);
    return add(a, mul(ab, t));
}

// addRoundContact (collide.cpp:500-517)
AVBD_DEV int round_contact(const NpBody &A, const NpBody &Bb, float3 cA, float rA, float3 cB, float rB, int key,
                           NewContact *cs, M3 &basis)
{
    float3 delta = sub(cB, cA);
    float rs = rA + rB;
    float d2 = lensq(delta);
    if (d2 > rs * rs)
        return 0;
    float3 n = d2 > SAT_EPS ? divs(delta, sqrtf(d2)) : f3(1.0f, 0.0f, 0.0f);
    float3 xA = add(cA, mul(n, rA));
    float3 xB = sub(cB, mul(n, rB));
    basis = orthonormal(neg(n));
    int count = 0;
    float3 mids[8];
    add_contact(A.p, A.q, Bb.p, Bb.q, cs, count, mids, xA, xB, key);
    return count;
}

// The thin axis of a static slab and its upward sign, or false (collide.cpp:957-976; the
// same test opens thinStaticBoxTopContactRound and collideThinStaticBoxTopRound).
AVBD_DEV bool slab_frame(const Obb &o, const NpBody &box, int &thin, float &sign)
{
    if (box.mass > 0.0f)
        return false;
    thin = 0;
    if (o.h.y < comp(o.h, thin))
        thin = 1;
    if (o.h.z < comp(o.h, thin))
        thin = 2;
    int a = (thin + 1) % 3, b = (thin + 2) % 3;
    if (comp(o.h, thin) * 4.0f > rmin(comp(o.h, a), comp(o.h, b)))
        return false;
    sign = dot(o.ax[thin], f3(0.0f, 0.0f, 1.0f)) >= 0.0f ? 1.0f : -1.0f;
    return true;
}

// sweptSphereBoxContact (collide.cpp:519-587)
AVBD_DEV bool swept_sphere_box(const Obb &o, const NpBody &sph, const NpBody &box, float dt, float3 &nBoxToSphere,
                               float3 &xBox)
{
    float3 rv = sub(sph.v, box.v);
    if (dt <= 0.0f || lensq(rv) < SAT_EPS)
        return false;
    float3 cur = sph.p;
    float3 prev = sub(cur, mul(rv, dt));
    float3 l0 = obb_local(o, prev), l1 = obb_local(o, cur);
    float3 delta = sub(l1, l0);
    float3 eh = add(o.h, f3(sph.s.radius, sph.s.radius, sph.s.radius));
    float tEnter = 0.0f, tExit = 1.0f, hitSign = 1.0f;
    int hitAxis = -1;
    for (int ax = 0; ax < 3; ++ax)
    {
        float d = comp(delta, ax), s0 = comp(l0, ax), e = comp(eh, ax);
        if (fabsf(d) < SAT_EPS)
        {
            if (s0 < -e || s0 > e)
                return false;
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
            return false;
    }
    if (hitAxis < 0 || tEnter < 0.0f || tEnter > 1.0f)
        return false;
    float3 sl = add(l0, mul(delta, tEnter));
    set_comp(sl, hitAxis, comp(o.h, hitAxis) * hitSign);
    for (int ax = 0; ax < 3; ++ax)
        if (ax != hitAxis)
            set_comp(sl, ax, rclamp(comp(sl, ax), -comp(o.h, ax), comp(o.h, ax)));
    nBoxToSphere = mul(o.ax[hitAxis], hitSign);
    xBox = obb_world(o, sl);
    return true;
}

// Clamp a point of a round body's segment onto a static slab's top face, or false when it
// is beyond the body's radius or off the face (collide.cpp:651-684, 689-708).
AVBD_DEV bool slab_point(const Obb &o, int thin, float sign, float radius, float3 center, float3 &xBox)
{
    float3 l = obb_local(o, center);
    float sd = comp(l, thin) * sign - comp(o.h, thin);
    if (sd > radius)
        return false;
    for (int ax = 0; ax < 3; ++ax)
    {
        if (ax == thin)
            continue;
        if (comp(l, ax) < -comp(o.h, ax) - radius || comp(l, ax) > comp(o.h, ax) + radius)
            return false;
    }
    set_comp(l, thin, comp(o.h, thin) * sign);
    for (int ax = 0; ax < 3; ++ax)
        if (ax != thin)
            set_comp(l, ax, rclamp(comp(l, ax), -comp(o.h, ax), comp(o.h, ax)));
    xBox = obb_world(o, l);
    return true;
}

// collideThinStaticBoxTopRound (collide.cpp:717-754): -1 when not a static slab top
AVBD_DEV int slab_top_round(const Obb &o, const NpBody &rb, const NpBody &box, bool roundIsA, NewContact *cs,
                            M3 &basis)
{
    int thin;
    float sign;
    if (!slab_frame(o, box, thin, sign))
        return -1;
    float3 n = mul(o.ax[thin], sign);
    float3 nAB = roundIsA ? neg(n) : n;
    basis = orthonormal(neg(nAB));
    int count = 0;
    float3 mids[8];
    float3 ends[2];
    int keys[2], nEnds;
    if (rb.s.type == SHAPE_CAPSULE)
    {
        round_segment(rb, ends[0], ends[1]);
        keys[0] = 0x04000000;
        keys[1] = 0x04000001;
        nEnds = 2;
    }
    else
    {
        ends[0] = rb.p;
        keys[0] = 0x02000000;
        nEnds = 1;
    }
    for (int e = 0; e < nEnds; ++e)
    {
        float3 xBox;
        if (!slab_point(o, thin, sign, rb.s.radius, ends[e], xBox))
            continue;
        float3 xRound = sub(ends[e], mul(n, rb.s.radius));
        if (roundIsA)
            add_contact(rb.p, rb.q, box.p, box.q, cs, count, mids, xRound, xBox, keys[e]);
        else
            add_contact(box.p, box.q, rb.p, rb.q, cs, count, mids, xBox, xRound, keys[e]);
    }
    return count > 0 ? count : -1;
}

// collideRoundRound (collide.cpp:756-765)
AVBD_DEV int collide_round_round(const NpBody &A, const NpBody &Bb, NewContact *cs, M3 &basis)
{
    float3 a0, a1, b0, b1, cA, cB;
    round_segment(A, a0, a1);
    round_segment(Bb, b0, b1);
    closest_segments(a0, a1, b0, b1, cA, cB);
    return round_contact(A, Bb, cA, A.s.radius, cB, Bb.s.radius, 0x03000000, cs, basis);
}

// collideRoundBox (collide.cpp:767-896)
AVBD_DEV int collide_round_box(const NpBody &rb, const NpBody &box, bool roundIsA, float dt, NewContact *cs,
                               M3 &basis)
{
    Obb o = make_obb(box.p, box.q, box.size);
    int top = slab_top_round(o, rb, box, roundIsA, cs, basis);
    if (top >= 0)
        return top;

    float3 rc = rb.p;
    if (rb.s.type == SHAPE_CAPSULE)
    {
        float3 sa, sb;
        round_segment(rb, sa, sb);
        float3 ca = obb_closest(o, sa), cb = obb_closest(o, sb);
        rc = lensq(sub(sa, ca)) <= lensq(sub(sb, cb)) ? sa : sb;
    }
    float rr = rb.s.radius;
    float3 closest = obb_closest(o, rc);
    float3 boxToRound = sub(rc, closest);
    float d2 = lensq(boxToRound);

    // thinStaticBoxTopContactRound (collide.cpp:632-685)
    bool onTop = false;
    {
        int thin;
        float sign;
        if (slab_frame(o, box, thin, sign))
        {
            float3 n = mul(o.ax[thin], sign);
            float3 sa, sb;
            round_segment(rb, sa, sb);
            float da = dot(sa, n), db = dot(sb, n);
            float3 topCenter = rb.s.type == SHAPE_CAPSULE && fabsf(da - db) < 1.0e-4f ? segment_closest(sa, sb, rb.p)
                               : da <= db                                             ? sa
                                                                                       : sb;
            float3 xBox;
            if (slab_point(o, thin, sign, rr, topCenter, xBox))
            {
                rc = topCenter;
                boxToRound = n;
                closest = xBox;
                d2 = 1.0f;
                onTop = true;
            }
        }
    }
    float3 local;
    if (onTop)
    {
    }
    else if (obb_inside(o, rc, local))
    {
        float3 sn, sp;
        if (rb.s.type == SHAPE_SPHERE && swept_sphere_box(o, rb, box, dt, sn, sp))
        {
            boxToRound = sn;
            closest = sp;
            d2 = 1.0f;
        }
        else
        {
            int axis = 0;
            float sign = local.x >= 0.0f ? 1.0f : -1.0f;
            float best = o.h.x - fabsf(local.x);
            float3 rv = sub(rb.v, box.v);
            if (box.mass <= 0.0f)
            {
                axis = 0;
                if (o.h.y < comp(o.h, axis))
                    axis = 1;
                if (o.h.z < comp(o.h, axis))
                    axis = 2;
                sign = dot(o.ax[axis], f3(0.0f, 0.0f, 1.0f)) >= 0.0f ? 1.0f : -1.0f;
            }
            else if (lensq(rv) > SAT_EPS)
            {
                float3 against = neg(rv);
                float bestDot = -3.402823466e+38f;
                for (int ca = 0; ca < 3; ++ca)
                    for (int si = 0; si < 2; ++si)
                    {
                        float cs_ = si == 0 ? -1.0f : 1.0f;
                        float d = dot(mul(o.ax[ca], cs_), against);
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
                float dy = o.h.y - fabsf(local.y);
                if (dy < best)
                {
                    axis = 1;
                    sign = local.y >= 0.0f ? 1.0f : -1.0f;
                    best = dy;
                }
                float dz = o.h.z - fabsf(local.z);
                if (dz < best)
                {
                    axis = 2;
                    sign = local.z >= 0.0f ? 1.0f : -1.0f;
                }
            }
            float3 sl = local;
            set_comp(sl, axis, comp(o.h, axis) * sign);
            closest = obb_world(o, sl);
            boxToRound = mul(o.ax[axis], sign);
            d2 = 1.0f;
        }
    }
    else if (d2 > rr * rr)
    {
        float3 sn, sp;
        if (rb.s.type != SHAPE_SPHERE || !swept_sphere_box(o, rb, box, dt, sn, sp))
            return 0;
        boxToRound = sn;
        closest = sp;
        d2 = 1.0f;
    }

    float3 nBR = d2 > SAT_EPS ? divs(boxToRound, sqrtf(d2)) : f3(0.0f, 0.0f, 1.0f);
    float3 nAB = roundIsA ? neg(nBR) : nBR;
    float3 xRound = sub(rc, mul(nBR, rr));
    basis = orthonormal(neg(nAB));
    int count = 0;
    float3 mids[8];
    int key = rb.s.type == SHAPE_CAPSULE ? 0x04000000 : 0x02000000;
    if (roundIsA)
        add_contact(rb.p, rb.q, box.p, box.q, cs, count, mids, xRound, closest, key);
    else
        add_contact(box.p, box.q, rb.p, rb.q, cs, count, mids, closest, xRound, key);
    return count;
}

// addThinStaticBoxTopCylinderContact (collide.cpp:978-1007)
AVBD_DEV void slab_cylinder_point(const Obb &o, const NpBody &cyl, const NpBody &box, bool cylIsA, int thin, float sign,
                                  float3 xCyl, int key, NewContact *cs, int &count, float3 *mids)
{
    float3 l = f3(dot(sub(xCyl, o.c), o.ax[0]), dot(sub(xCyl, o.c), o.ax[1]), dot(sub(xCyl, o.c), o.ax[2]));
    float sd = comp(l, thin) * sign - comp(o.h, thin);
    if (sd > COLLISION_MARGIN)
        return;
    for (int ax = 0; ax < 3; ++ax)
    {
        if (ax == thin)
            continue;
        if (comp(l, ax) < -comp(o.h, ax) - cyl.s.radius || comp(l, ax) > comp(o.h, ax) + cyl.s.radius)
            return;
    }
    set_comp(l, thin, (comp(o.h, thin) + COLLISION_MARGIN) * sign);
    for (int ax = 0; ax < 3; ++ax)
        if (ax != thin)
            set_comp(l, ax, rclamp(comp(l, ax), -comp(o.h, ax), comp(o.h, ax)));
    float3 xBox = obb_world(o, l);
    if (cylIsA)
        add_contact(cyl.p, cyl.q, box.p, box.q, cs, count, mids, xCyl, xBox, key);
    else
        add_contact(box.p, box.q, cyl.p, cyl.q, cs, count, mids, xBox, xCyl, key);
}

// The two unit vectors across an axis (collide.cpp:1030, 1085-1086)
AVBD_DEV void across(float3 a, float3 &u, float3 &v)
{
    u = fabsf(a.x) > fabsf(a.z) ? normalized(f3(-a.y, a.x, 0.0f)) : normalized(f3(0.0f, -a.z, a.y));
    v = normalized(cross(a, u));
}

// collideThinStaticBoxTopCylinder (collide.cpp:1009-1053)
AVBD_DEV int slab_top_cylinder(const Obb &o, const NpBody &cyl, const NpBody &box, bool cylIsA, NewContact *cs,
                               M3 &basis)
{
    int thin;
    float sign;
    if (!slab_frame(o, box, thin, sign))
        return -1;
    float3 n = mul(o.ax[thin], sign);
    float3 nAB = cylIsA ? neg(n) : n;
    basis = orthonormal(neg(nAB));
    float3 axis = rotate(cyl.q, f3(0.0f, 0.0f, 1.0f));
    float ad = dot(axis, n);
    int count = 0;
    float3 mids[8];
    if (fabsf(ad) > 0.65f)
    {
        float as = ad >= 0.0f ? 1.0f : -1.0f;
        float3 cap = sub(cyl.p, mul(axis, cyl.s.halfLength * as));
        float3 u, v;
        across(axis, u, v);
        float3 offs[4] = {mul(u, cyl.s.radius), mul(neg(u), cyl.s.radius), mul(v, cyl.s.radius),
                          mul(neg(v), cyl.s.radius)};
        for (int i = 0; i < 4; ++i)
            slab_cylinder_point(o, cyl, box, cylIsA, thin, sign, add(cap, offs[i]), 0x05000000 | i, cs, count, mids);
    }
    else
    {
        float3 radial = sub(n, mul(axis, ad));
        if (lensq(radial) < SAT_EPS)
            radial = n;
        radial = normalized(radial);
        float3 a = sub(cyl.p, mul(axis, cyl.s.halfLength));
        float3 b = add(cyl.p, mul(axis, cyl.s.halfLength));
        slab_cylinder_point(o, cyl, box, cylIsA, thin, sign, sub(a, mul(radial, cyl.s.radius)), 0x05000100, cs, count,
                            mids);
        slab_cylinder_point(o, cyl, box, cylIsA, thin, sign, sub(b, mul(radial, cyl.s.radius)), 0x05000101, cs, count,
                            mids);
    }
    return count > 0 ? count : -1;
}

// addCylinderCapContacts (collide.cpp:1080-1091)
AVBD_DEV int cylinder_caps(const NpBody &A, const NpBody &Bb, float3 nAB, float3 capA, float3 capB, float radius,
                           NewContact *cs, M3 &basis)
{
    basis = orthonormal(neg(nAB));
    int count = 0;
    float3 mids[8];
    float3 u, v;
    across(nAB, u, v);
    float3 offs[4] = {mul(u, radius), mul(neg(u), radius), mul(v, radius), mul(neg(v), radius)};
    for (int i = 0; i < 4; ++i)
        add_contact(A.p, A.q, Bb.p, Bb.q, cs, count, mids, add(capA, offs[i]), add(capB, offs[i]), 0x06000000 | i);
    return count;
}

// collideCylinders (collide.cpp:1093-1150)
AVBD_DEV int collide_cylinders(const NpBody &A, const NpBody &Bb, NewContact *cs, M3 &basis)
{
    float3 axA = rotate(A.q, f3(0.0f, 0.0f, 1.0f));
    float3 axB = rotate(Bb.q, f3(0.0f, 0.0f, 1.0f));
    float par = dot(axA, axB);
    float3 delta = sub(Bb.p, A.p);
    if (fabsf(par) > 0.95f)
    {
        float axial = dot(delta, axA);
        float3 radial = sub(delta, mul(axA, axial));
        float rl2 = lensq(radial);
        float rs = A.s.radius + Bb.s.radius;
        if (rl2 > rs * rs)
            return 0;
        float overlap = A.s.halfLength + Bb.s.halfLength - fabsf(axial);
        if (overlap < -COLLISION_MARGIN)
            return 0;
        if (fabsf(axial) > (A.s.halfLength + Bb.s.halfLength) * 0.5f)
        {
            float side = axial >= 0.0f ? 1.0f : -1.0f;
            float3 nAB = mul(axA, side);
            float3 capA = add(A.p, mul(nAB, A.s.halfLength));
            float3 capB = sub(Bb.p, mul(nAB, Bb.s.halfLength));
            return cylinder_caps(A, Bb, nAB, capA, capB, rmin(A.s.radius, Bb.s.radius) * 0.85f, cs, basis);
        }
        float3 nAB = rl2 > SAT_EPS ? divs(radial, sqrtf(rl2)) : orthonormal(axA).r1;
        basis = orthonormal(neg(nAB));
        int count = 0;
        float3 mids[8];
        float lo = rmax(-A.s.halfLength, axial - Bb.s.halfLength);
        float hi = rmin(A.s.halfLength, axial + Bb.s.halfLength);
        float vals[2] = {lo, hi};
        for (int i = 0; i < 2; ++i)
        {
            float tA = vals[i];
            float tB = tA - axial;
            float3 xA = add(add(A.p, mul(axA, tA)), mul(nAB, A.s.radius));
            float3 xB = sub(add(Bb.p, mul(axA, tB)), mul(nAB, Bb.s.radius));
            add_contact(A.p, A.q, Bb.p, Bb.q, cs, count, mids, xA, xB, 0x06000100 | i);
        }
        return count;
    }
    float3 a0, a1, b0, b1, cA, cB;
    round_segment(A, a0, a1);
    round_segment(Bb, b0, b1);
    closest_segments(a0, a1, b0, b1, cA, cB);
    return round_contact(A, Bb, cA, A.s.radius, cB, Bb.s.radius, 0x06000200, cs, basis);
}

// collideCylinderRound (collide.cpp:1065-1078)
AVBD_DEV int collide_cylinder_round(const NpBody &cyl, const NpBody &rb, bool cylIsA, NewContact *cs, M3 &basis)
{
    float3 c0, c1, r0, r1, cc, cr;
    round_segment(cyl, c0, c1);
    round_segment(rb, r0, r1);
    closest_segments(c0, c1, r0, r1, cc, cr);
    if (cylIsA)
        return round_contact(cyl, rb, cc, cyl.s.radius, cr, rb.s.radius, 0x07000000, cs, basis);
    return round_contact(rb, cyl, cr, rb.s.radius, cc, cyl.s.radius, 0x07000000, cs, basis);
}

// Manifold::collide (collide.cpp:1154-1176)
AVBD_DEV int collide_shapes(const NpBody &A, const NpBody &Bb, float dt, NewContact *cs, M3 &basis)
{
    if (is_cylinder(A) && is_cylinder(Bb))
        return collide_cylinders(A, Bb, cs, basis);
    if (is_cylinder(A) && is_round(Bb))
        return collide_cylinder_round(A, Bb, true, cs, basis);
    if (is_round(A) && is_cylinder(Bb))
        return collide_cylinder_round(Bb, A, false, cs, basis);
    if (is_cylinder(A) && Bb.s.type == SHAPE_BOX)
    {
        Obb o = make_obb(Bb.p, Bb.q, Bb.size);
        int top = slab_top_cylinder(o, A, Bb, true, cs, basis);
        if (top >= 0)
            return top;
        return collide_boxes(A.p, A.q, A.size, Bb.p, Bb.q, Bb.size, cs, basis);
    }
    if (A.s.type == SHAPE_BOX && is_cylinder(Bb))
    {
        Obb o = make_obb(A.p, A.q, A.size);
        int top = slab_top_cylinder(o, Bb, A, false, cs, basis);
        if (top >= 0)
            return top;
        return collide_boxes(A.p, A.q, A.size, Bb.p, Bb.q, Bb.size, cs, basis);
    }
    if (is_round(A) && is_round(Bb))
        return collide_round_round(A, Bb, cs, basis);
    if (is_round(A) && Bb.s.type == SHAPE_BOX)
        return collide_round_box(A, Bb, true, dt, cs, basis);
    if (A.s.type == SHAPE_BOX && is_round(Bb))
        return collide_round_box(Bb, A, false, dt, cs, basis);
    return collide_boxes(A.p, A.q, A.size, Bb.p, Bb.q, Bb.size, cs, basis);
}

AVBD_DEV bool cylinder_cap_key(int key)
{
    return (key & 0xFFFFFF00) == 0x05000000 || (key & 0xFFFFFF00) == 0x06000000;
}

// contactOffsetWorld (manifold.cpp:28-91): the world offset of a contact point from the
// body's centre, re-derived from the contact basis for round bodies.
AVBD_DEV float3 contact_offset(const BodyShape &s, float4 q, float3 lo, const M3 &basis, bool isA, int key)
{
    if (s.type == SHAPE_SPHERE)
        return mul(basis.r0, isA ? -s.radius : s.radius);
    if (s.type == SHAPE_CAPSULE)
    {
        float3 axis = rotate(q, f3(0.0f, 0.0f, 1.0f));
        float3 n = basis.r0;
        float3 nl = rotate(qconj(q), n);
        float cz = isA ? lo.z + nl.z * s.radius : lo.z - nl.z * s.radius;
        cz = rclamp(cz, -s.halfLength, s.halfLength);
        return add(mul(axis, cz), mul(n, isA ? -s.radius : s.radius));
    }
    if (s.type == SHAPE_CYLINDER)
    {
        float3 sw = mul(basis.r0, isA ? -1.0f : 1.0f);
        float3 sl = rotate(qconj(q), sw);
        float stored = sqrtf(lo.x * lo.x + lo.y * lo.y);
        if (cylinder_cap_key(key))
        {
            float3 l = f3(0.0f, 0.0f, 0.0f);
            if (stored > 1.0e-6f)
            {
                l.x = lo.x / stored * s.radius;
                l.y = lo.y / stored * s.radius;
            }
            float capSign = fabsf(lo.z) > 1.0e-6f ? (lo.z >= 0.0f ? 1.0f : -1.0f) : (sl.z >= 0.0f ? 1.0f : -1.0f);
            l.z = s.halfLength * capSign;
            return rotate(q, l);
        }
        float radialLen = sqrtf(sl.x * sl.x + sl.y * sl.y);
        float z = fabsf(sl.z) > 0.15f ? (sl.z >= 0.0f ? s.halfLength : -s.halfLength)
                                      : rclamp(lo.z, -s.halfLength, s.halfLength);
        float3 l = f3(0.0f, 0.0f, z);
        if (radialLen > 1.0e-6f)
        {
            l.x = sl.x / radialLen * s.radius;
            l.y = sl.y / radialLen * s.radius;
        }
        else if (stored > 1.0e-6f)
        {
            l.x = lo.x / stored * s.radius;
            l.y = lo.y / stored * s.radius;
        }
        return rotate(q, l);
    }
    return rotate(q, lo);
}

// applySphereRollingFriction (solver.cpp:628-662) for every manifold of a dynamic sphere, in
// the solver's force order (the body's list, newest first), after the velocity update.
__global__ void k_rolling_friction(DevBodies B, DevForces F, const int *adjStart, const StepState *st = nullptr)
{
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B.n || !B.shape || step_aborted(st))
        return;
    BodyShape s = body_shape(B, b);
    if (s.type != SHAPE_SPHERE || B.massMoment[b].x <= 0.0f)
        return;
    float3 v = xyz(B.vel[b]), w = xyz(B.angvel[b]);
    bool changed = false;
    for (int k = adjStart[b]; k < adjStart[b + 1]; ++k)
    {
        unsigned e = F.adj[k];
        if (adj_type(e) != ADJ_MANIFOLD)
            continue;
        unsigned m = adj_index(e);
        int2 ab = F.man.ab[m];
        int other = adj_isA(e) ? ab.y : ab.x;
        // the sphere the reference picks is body A when A is a sphere
        bool sphereIsA = body_shape(B, ab.x).type == SHAPE_SPHERE;
        if ((sphereIsA ? ab.x : ab.y) != b)
            continue;
        int nc = F.man.n[m];
        if (B.massMoment[other].x > 0.0f || nc <= 0)
            continue;
        float mf = sqrtf(B.friction[b] * B.friction[other]);
        if (mf <= 0.0f)
            continue;
        float blend = rclamp(mf * 0.08f, 0.0f, 0.18f);
        float3 basis0 = xyz(F.man.basis[3 * (size_t)m]);
        for (int i = 0; i < nc; ++i)
        {
            float3 n = sphereIsA ? basis0 : neg(basis0);
            float3 r = mul(neg(n), s.radius);
            float3 cv = add(v, cross(w, r));
            float3 tv = sub(cv, mul(n, dot(cv, n)));
            v = sub(v, mul(tv, blend));
            float3 desired = divs(cross(n, v), s.radius);
            w = add(w, mul(sub(desired, w), blend));
        }
        changed = true;
    }
    if (changed)
    {
        B.vel[b] = f4(v, 0.0f);
        B.angvel[b] = f4(w, 0.0f);
    }
}
