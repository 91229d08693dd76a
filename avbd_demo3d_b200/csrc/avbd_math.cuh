// Device float math for the AVBD step.
//
// Every routine evaluates the same operations in the same order as the reference's
// source/maths.h (ts-jls/avbd-demo3d): dot = x*x' + y*y' + z*z' left to right, matrix
// products as row-by-column dots, quaternion "difference" 2*vec(a*inverse(b))
// (maths.h:269-272), quaternion "step" normalize(a + (b,0)*a*0.5) (maths.h:274-277),
// rotate (maths.h:441-446) and orthonormal (maths.h:468-474). With --fmad=false and
// IEEE division/sqrt (the nvcc defaults without fast-math) each result is bit-identical
// to the reference compiled for x86-64, which is what makes the GPU trajectory match
// the CPU solver to the last bit instead of drifting after a few steps.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define AVBD_DEV __device__ __forceinline__

namespace avbd
{

struct M3
{
    float3 r0, r1, r2;
};

AVBD_DEV float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
AVBD_DEV float3 xyz(float4 v) { return make_float3(v.x, v.y, v.z); }
AVBD_DEV float4 f4(float3 v, float w) { return make_float4(v.x, v.y, v.z, w); }
AVBD_DEV float comp(float3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

AVBD_DEV float3 add(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
AVBD_DEV float3 sub(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
AVBD_DEV float3 neg(float3 a) { return f3(-a.x, -a.y, -a.z); }
AVBD_DEV float3 mul(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
// A value the compiler cannot see through (an empty asm that may rewrite it).
AVBD_DEV float opaque(float x)
{
    asm("" : "+f"(x));
    return x;
}

// a / s, IEEE round-to-nearest. A zero dividend over a non-zero, non-NaN divisor gives
// the signed zero directly (sign of a xor sign of s, as IEEE 754 defines the quotient).
// Measured on B200: a division whose dividend is zero takes about four times as long as
// one of two normal numbers, in every lane of the warp, and the solver divides many
// exact zeros (the off-diagonals of the mass matrices, quaternion components of unrotated
// bodies, zero couplings of the 6x6 systems). Those lanes divide 1 instead; the dividend
// goes through `opaque`, or the compiler, seeing the quotient unused for a zero dividend,
// would divide the zero after all.
AVBD_DEV float fdiv(float a, float s)
{
    const bool zero = a == 0.0f && s != 0.0f && s == s;
    const float q = opaque(zero ? 1.0f : a) / s;
    return zero ? __int_as_float((__float_as_int(a) ^ __float_as_int(s)) & (int)0x80000000) : q;
}
// 0 / s: the zero with the sign of s for a non-zero, non-NaN s, without dividing (s is
// the same in every lane where this is used, so the branch does not diverge).
AVBD_DEV float zero_over(float s)
{
    if (s != 0.0f && s == s)
        return __int_as_float(__float_as_int(s) & (int)0x80000000);
    return opaque(0.0f) / s;
}
AVBD_DEV float3 divs(float3 a, float s) { return f3(fdiv(a.x, s), fdiv(a.y, s), fdiv(a.z, s)); }
AVBD_DEV float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
AVBD_DEV float lensq(float3 a) { return dot(a, a); }
AVBD_DEV float len(float3 a) { return sqrtf(lensq(a)); }
AVBD_DEV float3 cross(float3 a, float3 b)
{
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
AVBD_DEV float3 absv(float3 a) { return f3(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }

// min/max/clamp with the reference's comparison semantics (maths.h:297-320)
AVBD_DEV float rmin(float a, float b) { return a < b ? a : b; }
AVBD_DEV float rmax(float a, float b) { return a > b ? a : b; }
AVBD_DEV float rclamp(float x, float a, float b) { return rmax(a, rmin(b, x)); }
AVBD_DEV float rsign(float x) { return x < 0 ? -1.0f : (x > 0 ? 1.0f : 0.0f); }
AVBD_DEV float3 minv(float3 a, float b) { return f3(rmin(a.x, b), rmin(a.y, b), rmin(a.z, b)); }
AVBD_DEV float3 clampv(float3 v, float a, float b) { return f3(rclamp(v.x, a, b), rclamp(v.y, a, b), rclamp(v.z, a, b)); }

AVBD_DEV M3 rows(float3 a, float3 b, float3 c)
{
    M3 m;
    m.r0 = a;
    m.r1 = b;
    m.r2 = c;
    return m;
}
AVBD_DEV M3 diag(float a, float b, float c) { return rows(f3(a, 0, 0), f3(0, b, 0), f3(0, 0, c)); }
AVBD_DEV float3 row(const M3 &m, int i) { return i == 0 ? m.r0 : (i == 1 ? m.r1 : m.r2); }
AVBD_DEV float3 col(const M3 &m, int i) { return f3(comp(m.r0, i), comp(m.r1, i), comp(m.r2, i)); }
AVBD_DEV float3 mv(const M3 &a, float3 b) { return f3(dot(a.r0, b), dot(a.r1, b), dot(a.r2, b)); }
AVBD_DEV float3 rowtimes(float3 r, const M3 &b) { return f3(dot(r, col(b, 0)), dot(r, col(b, 1)), dot(r, col(b, 2))); }
AVBD_DEV M3 mm(const M3 &a, const M3 &b) { return rows(rowtimes(a.r0, b), rowtimes(a.r1, b), rowtimes(a.r2, b)); }
AVBD_DEV M3 madd(const M3 &a, const M3 &b) { return rows(add(a.r0, b.r0), add(a.r1, b.r1), add(a.r2, b.r2)); }
AVBD_DEV M3 mscale(const M3 &a, float s) { return rows(mul(a.r0, s), mul(a.r1, s), mul(a.r2, s)); }
AVBD_DEV M3 mdivs(const M3 &a, float s) { return rows(divs(a.r0, s), divs(a.r1, s), divs(a.r2, s)); }
AVBD_DEV M3 mneg(const M3 &a) { return rows(neg(a.r0), neg(a.r1), neg(a.r2)); }
AVBD_DEV M3 trans(const M3 &a) { return rows(col(a, 0), col(a, 1), col(a, 2)); }
AVBD_DEV M3 skew(float3 r) { return rows(f3(0, -r.z, r.y), f3(r.z, 0, -r.x), f3(-r.y, r.x, 0)); }
AVBD_DEV M3 outer(float3 a, float3 b) { return rows(mul(b, a.x), mul(b, a.y), mul(b, a.z)); }
AVBD_DEV M3 diagonalize(const M3 &m) { return diag(len(col(m, 0)), len(col(m, 1)), len(col(m, 2))); }

// quaternions are float4 (x, y, z, w)
AVBD_DEV float4 qmul(float4 a, float4 b)
{
    return make_float4(a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y, a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
                       a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w, a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z);
}
AVBD_DEV float4 qadd(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
AVBD_DEV float4 qscale(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
AVBD_DEV float4 qdivs(float4 a, float s) { return make_float4(fdiv(a.x, s), fdiv(a.y, s), fdiv(a.z, s), fdiv(a.w, s)); }
AVBD_DEV float qlensq(float4 q) { return lensq(xyz(q)) + q.w * q.w; }
AVBD_DEV float4 qnormalize(float4 q) { return qdivs(q, sqrtf(qlensq(q))); }
AVBD_DEV float4 qconj(float4 q) { return make_float4(-q.x, -q.y, -q.z, q.w); }
AVBD_DEV float4 qinverse(float4 q) { return qdivs(qconj(q), qlensq(q)); }
// a - b for orientations: 2 vec(a b^-1)
AVBD_DEV float3 qdiff(float4 a, float4 b) { return mul(xyz(qmul(a, qinverse(b))), 2.0f); }
// qdiff(a, b) given binv = qinverse(b)
AVBD_DEV float3 qdiff_inv(float4 a, float4 binv) { return mul(xyz(qmul(a, binv)), 2.0f); }
// a + w for an orientation and a rotation vector: normalize(a + (w,0) a / 2)
AVBD_DEV float4 qstep(float4 a, float3 w)
{
    return qnormalize(qadd(a, qscale(qmul(make_float4(w.x, w.y, w.z, 0.0f), a), 0.5f)));
}
AVBD_DEV float3 rotate(float4 q, float3 v)
{
    float3 u = xyz(q);
    float3 t = mul(cross(u, v), 2.0f);
    return add(add(v, mul(t, q.w)), cross(u, t));
}
AVBD_DEV float3 xform(float3 p, float4 q, float3 v) { return add(rotate(q, v), p); }
AVBD_DEV M3 orthonormal(float3 n)
{
    float3 t1 = fabsf(n.x) > fabsf(n.z) ? f3(-n.y, n.x, 0) : f3(0, -n.z, n.y);
    t1 = divs(t1, len(t1));
    float3 t2 = cross(n, t1);
    return rows(n, t1, t2);
}

// 6x6 symmetric system in "27-entry" form: the lower triangles of lhsLin and lhsAng,
// all of lhsCross, and the two right-hand sides -- exactly the entries the LDL^T solve
// reads (maths.h:484-489).
enum Entry27
{
    E_LL00 = 0, E_LL10, E_LL11, E_LL20, E_LL21, E_LL22,
    E_LA00 = 6, E_LA10, E_LA11, E_LA20, E_LA21, E_LA22,
    E_LC00 = 12, E_LC01, E_LC02, E_LC10, E_LC11, E_LC12, E_LC20, E_LC21, E_LC22,
    E_RL0 = 21, E_RL1, E_RL2,
    E_RA0 = 24, E_RA1, E_RA2,
    E_COUNT = 27
};

// Unpivoted LDL^T solve of [[aLin, aCross^T],[aCross, aAng]] x = b with the entry
// order and per-entry operation order of maths.h:481-547. `s` holds the 27 entries;
// the right-hand side is negated here (solve(..., -rhsLin, -rhsAng, ...), solver.cpp:1233).
AVBD_DEV void load_sys27(const float *s, float (&A)[6][6])
{
    A[0][0] = s[E_LL00];
    A[1][0] = s[E_LL10];
    A[1][1] = s[E_LL11];
    A[2][0] = s[E_LL20];
    A[2][1] = s[E_LL21];
    A[2][2] = s[E_LL22];
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
            A[3 + r][c] = s[E_LC00 + 3 * r + c];
    A[3][3] = s[E_LA00];
    A[4][3] = s[E_LA10];
    A[4][4] = s[E_LA11];
    A[5][3] = s[E_LA20];
    A[5][4] = s[E_LA21];
    A[5][5] = s[E_LA22];
}

AVBD_DEV void ldl_solve27(const float *s, float3 &xl, float3 &xa)
{
    float A[6][6];
    load_sys27(s, A);
    float L[6][6];
    float D[6];
#pragma unroll
    for (int j = 0; j < 6; ++j)
    {
        if (j == 0)
            D[0] = A[0][0];
        else
        {
            float acc = L[j][0] * L[j][0] * D[0];
#pragma unroll
            for (int k = 1; k < j; ++k)
                acc = acc + L[j][k] * L[j][k] * D[k];
            D[j] = A[j][j] - acc;
        }
#pragma unroll
        for (int i = j + 1; i < 6; ++i)
        {
            float v = A[i][j];
#pragma unroll
            for (int k = 0; k < j; ++k)
                v = v - L[j][k] * L[i][k] * D[k];
            L[i][j] = fdiv(v, D[j]);
        }
    }
    float b[6] = {-s[E_RL0], -s[E_RL1], -s[E_RL2], -s[E_RA0], -s[E_RA1], -s[E_RA2]};
    float y[6], z[6], x[6];
#pragma unroll
    for (int i = 0; i < 6; ++i)
    {
        float v = b[i];
#pragma unroll
        for (int k = 0; k < i; ++k)
            v = v - L[i][k] * y[k];
        y[i] = v;
    }
#pragma unroll
    for (int i = 0; i < 6; ++i)
        z[i] = fdiv(y[i], D[i]);
#pragma unroll
    for (int i = 5; i >= 0; --i)
    {
        float v = z[i];
#pragma unroll
        for (int k = i + 1; k < 6; ++k)
            v = v - L[k][i] * x[k];
        x[i] = v;
    }
    xl = f3(x[0], x[1], x[2]);
    xa = f3(x[3], x[4], x[5]);
}

} // namespace avbd
