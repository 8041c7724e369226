// Soft-step contact solver on the device: constraint preparation, warm
// start, the normal/friction/twist/rolling rows, restitution and the
// impulse store, plus the two integrators and the gyroscopic step.
// Each routine restates the reference's arithmetic in its operand order
// (src/solver.c, lines beside each); graph colouring makes every colour
// a set of constraints with pairwise-disjoint awake dynamic bodies, so
// one thread per constraint inside a colour reproduces the reference's
// serial order bit for bit.
#ifndef M3_SOLVER_CUH
#define M3_SOLVER_CUH

#include "m3_layout.h"

struct m3SoftDev
{
    m3real biasRate;
    m3real massScale;
    m3real impulseScale;
};

// solver.c:30-40
__device__ __forceinline__ m3SoftDev m3MakeSoft(m3real hertz, m3real zeta, m3real h)
{
    m3SoftDev s;
    if (hertz == 0.0f)
    {
        s.biasRate = 0.0f;
        s.massScale = 0.0f;
        s.impulseScale = 0.0f;
        return s;
    }
    m3real omega = 2.0f * M3_PI * hertz;
    m3real a1 = 2.0f * zeta + h * omega;
    m3real a2 = h * omega * a1;
    m3real a3 = 1.0f / (1.0f + a2);
    s.biasRate = omega / a1;
    s.massScale = a2 * a3;
    s.impulseScale = a3;
    return s;
}

struct m3ConstraintPointDev
{
    m3Vec3 rA;
    m3Vec3 rB;
    m3real baseSeparation;
    m3real normalMass;
    m3real leverArm;
    m3real relativeVelocity;
    m3real normalImpulse;
    m3real totalNormalImpulse;
};

// One contact constraint record (the reference's m3ContactConstraint,
// solver.c:66-103, with the body-type tests folded into two flags).
struct m3ContactDev
{
    int32_t bodyA;
    int32_t bodyB;
    int32_t manifoldIndex;
    int32_t pointCount;
    uint8_t dynA;
    uint8_t dynB;
    uint8_t pad[2];
    m3Vec3 normal;
    m3Vec3 t1;
    m3Vec3 t2;
    m3Vec3 originA;
    m3Vec3 originB;
    m3real frictionK11;
    m3real frictionK12;
    m3real frictionK22;
    m3real frictionImpulse1;
    m3real frictionImpulse2;
    m3real twistMass;
    m3real twistImpulse;
    m3real tangentVelocity1;
    m3real tangentVelocity2;
    m3real friction;
    m3real restitution;
    m3real invMassA;
    m3real invMassB;
    m3Mat3 invIA;
    m3Mat3 invIB;
    m3SoftDev softness;
    m3real rollingResistance;
    m3Vec3 rollingImpulse;
    m3Mat3 rollingK;
    m3ConstraintPointDev points[M3_MANIFOLD_MAX_POINTS];
};

// World-space inverse inertia R Il^-1 R^T built column by column
// (solver.c:139-153).
__device__ __forceinline__ m3Mat3 m3WorldInvInertiaDev(const m3WorldView& w, int32_t body)
{
    if (w.btype[body] != M3_BODY_DYNAMIC)
    {
        return m3ZeroMat3();
    }
    m3Quat q = w.xf[body].q;
    m3Mat3 il = w.invI[body];
    m3Mat3 r;
    r.cx = m3RotateVec3(q, m3MulMV3(il, m3InvRotateVec3(q, v3(1.0f, 0.0f, 0.0f))));
    r.cy = m3RotateVec3(q, m3MulMV3(il, m3InvRotateVec3(q, v3(0.0f, 1.0f, 0.0f))));
    r.cz = m3RotateVec3(q, m3MulMV3(il, m3InvRotateVec3(q, v3(0.0f, 0.0f, 1.0f))));
    return r;
}

__device__ __forceinline__ m3Vec3 m3VelocityAt(const m3WorldView& w, int32_t body, m3Vec3 arm)
{
    m3Vec3 v = w.v[body];
    m3Vec3 om = w.w[body];
    return m3Add3(v, m3Cross3(om, arm));
}

// ---------------------------------------------------------------------
// Contact rows in HBM, field-major: word `field` of the row in solve
// slot `slot` sits at base[field * stride + slot].  Slots are the solve
// order (colour by colour), so the threads of a warp working through a
// colour read consecutive words of every field: one 128-byte line per
// field per warp instead of one line per thread.  The fields a pass
// only reads (written once by the preparation kernel) are fetched
// through the read-only path; the impulse accumulators sit in a second
// array and are loaded into registers once per row and written back
// once.
// ---------------------------------------------------------------------
#define M3C_BODY_A 0
#define M3C_BODY_B 1
#define M3C_MANIFOLD 2
#define M3C_POINTS 3
#define M3C_FLAGS 4 // bit 0: side A dynamic, bit 1: side B dynamic
#define M3C_NORMAL 5
#define M3C_T1 8
#define M3C_T2 11
#define M3C_ORIGIN_A 14
#define M3C_ORIGIN_B 17
#define M3C_K11 20
#define M3C_K12 21
#define M3C_K22 22
#define M3C_TWIST_MASS 23
#define M3C_TANGENT_V1 24
#define M3C_TANGENT_V2 25
#define M3C_FRICTION 26
#define M3C_RESTITUTION 27
#define M3C_INV_MASS_A 28
#define M3C_INV_MASS_B 29
#define M3C_SOFT 30 // biasRate, massScale, impulseScale
#define M3C_ROLLING 33
#define M3C_ROLLING_K 34
#define M3C_POINT0 43 // per point: rA, rB, baseSeparation, normalMass, leverArm, relativeVelocity
#define M3C_POINT_WORDS 10
#define M3C_WORDS (M3C_POINT0 + M3C_POINT_WORDS * M3_MANIFOLD_MAX_POINTS)

#define M3A_NORMAL 0 // per point
#define M3A_TOTAL_NORMAL 4 // per point
#define M3A_FRICTION1 8
#define M3A_FRICTION2 9
#define M3A_TWIST 10
#define M3A_ROLLING 11
#define M3A_WORDS 14

struct m3ConRows
{
    float* ro;
    float* acc;
    int32_t stride;
};

// One row of m3ConRows.  f/n/v/m read prepared words through the
// read-only data path: valid only in kernels that never write them.
struct m3ConRef
{
    const float* ro;
    float* acc;
    int32_t stride;

    __device__ __forceinline__ m3real f(int32_t k) const
    {
        return __ldg(ro + (int64_t)k * stride);
    }
    __device__ __forceinline__ int32_t n(int32_t k) const
    {
        return __ldg(reinterpret_cast<const int32_t*>(ro) + (int64_t)k * stride);
    }
    __device__ __forceinline__ m3Vec3 v(int32_t k) const
    {
        return v3(f(k), f(k + 1), f(k + 2));
    }
    __device__ __forceinline__ m3Mat3 m(int32_t k) const
    {
        m3Mat3 r;
        r.cx = v(k);
        r.cy = v(k + 3);
        r.cz = v(k + 6);
        return r;
    }
    __device__ __forceinline__ m3real& a(int32_t k) const
    {
        return acc[(int64_t)k * stride];
    }
};

__device__ __forceinline__ m3ConRef m3ConAt(const m3ConRows& r, int32_t slot)
{
    m3ConRef c;
    c.ro = r.ro + slot;
    c.acc = r.acc + slot;
    c.stride = r.stride;
    return c;
}

// The two bodies of a row and their mass terms, loaded once per row.
// The world-space inverse inertia tensors are not row words: every row
// of a body uses the same prepare-time tensor (m3WorldInvInertiaDev), so
// they come from a per-body table (shared memory in the substep loop),
// read by body index.
struct m3ConBodies
{
    int32_t a;
    int32_t b;
    bool dynA;
    bool dynB;
    m3real mA;
    m3real mB;
    m3Mat3 iA;
    m3Mat3 iB;
};

__device__ __forceinline__ m3ConBodies m3LoadConBodies(const m3ConRef& c, const m3Mat3* invI)
{
    m3ConBodies cb;
    cb.a = c.n(M3C_BODY_A);
    cb.b = c.n(M3C_BODY_B);
    const int32_t flags = c.n(M3C_FLAGS);
    cb.dynA = (flags & 1) != 0;
    cb.dynB = (flags & 2) != 0;
    cb.mA = c.f(M3C_INV_MASS_A);
    cb.mB = c.f(M3C_INV_MASS_B);
    cb.iA = invI[cb.a];
    cb.iB = invI[cb.b];
    return cb;
}

// solver.c:105-121
__device__ __forceinline__ void m3ApplyImpulseRow(const m3WorldView& w, const m3ConBodies& cb,
                                                  m3Vec3 impulse, m3Vec3 rsA, m3Vec3 rsB)
{
    if (cb.dynA)
    {
        w.v[cb.a] = m3Sub3(w.v[cb.a], m3MulSV3(cb.mA, impulse));
        w.w[cb.a] = m3Sub3(w.w[cb.a], m3MulMV3(cb.iA, m3Cross3(rsA, impulse)));
    }
    if (cb.dynB)
    {
        w.v[cb.b] = m3Add3(w.v[cb.b], m3MulSV3(cb.mB, impulse));
        w.w[cb.b] = m3Add3(w.w[cb.b], m3MulMV3(cb.iB, m3Cross3(rsB, impulse)));
    }
}

// solver.c:124-133
__device__ __forceinline__ m3real m3EffectiveMass(const m3ContactDev* c, m3Vec3 rA, m3Vec3 rB,
                                                  m3Vec3 dir)
{
    m3Vec3 arm1 = m3Cross3(rA, dir);
    m3Vec3 arm2 = m3Cross3(rB, dir);
    m3real k = c->invMassA + c->invMassB + m3Dot3(arm1, m3MulMV3(c->invIA, arm1)) +
               m3Dot3(arm2, m3MulMV3(c->invIB, arm2));
    return k > 0.0f ? 1.0f / k : 0.0f;
}

// Per-constraint body of PrepareContacts (solver.c:261-405).
__device__ void m3PrepareContact(const m3WorldView& w, m3ContactDev* c, int32_t pairIndex,
                                 const uint64_t* keys, const m3Manifold* manifolds,
                                 m3SoftDev soft, m3SoftDev staticSoft, const m3Mat3* invI)
{
    const m3Manifold* manifold = &manifolds[pairIndex];
    uint64_t key = keys[pairIndex];
    int32_t shapeA = (int32_t)(key >> 32);
    int32_t shapeB = (int32_t)(key & 0xFFFFFFFFu);
    int32_t bodyA = w.shapeBody[shapeA];
    int32_t bodyB = w.shapeBody[shapeB];
    // Every field a later phase reads is written below (the reference
    // zeroes the whole record first; rollingK is read only when rolling
    // resistance is positive, points only below pointCount).
    c->bodyA = bodyA;
    c->bodyB = bodyB;
    c->manifoldIndex = pairIndex;
    c->pointCount = manifold->pointCount;
    c->dynA = w.btype[bodyA] == M3_BODY_DYNAMIC ? 1 : 0;
    c->dynB = w.btype[bodyB] == M3_BODY_DYNAMIC ? 1 : 0;
    c->normal = manifold->normal;
    m3MakeTangentBasis(c->normal, &c->t1, &c->t2);
    c->invMassA = c->dynA ? w.invMass[bodyA] : 0.0f;
    c->invMassB = c->dynB ? w.invMass[bodyB] : 0.0f;
    c->invIA = invI[bodyA];
    c->invIB = invI[bodyB];
    float fricA = w.friction[shapeA];
    float fricB = w.friction[shapeB];
    float restA = w.restitution[shapeA];
    float restB = w.restitution[shapeB];
    float rollA = w.rolling[shapeA];
    float rollB = w.rolling[shapeB];
    m3Vec3 surfA = w.surfVel[shapeA];
    m3Vec3 surfB = w.surfVel[shapeB];
    c->friction = sqrtf(fricA * fricB);
    c->restitution = m3MaxF(restA, restB);
    c->rollingResistance = m3MaxF(rollA, rollB) * m3MaxF(w.maxExt[bodyA], w.maxExt[bodyB]);
    c->rollingImpulse = manifold->rollingImpulse;
    if (c->rollingResistance > 0.0f)
    {
        m3Mat3 sum = c->invIA;
        sum.cx = m3Add3(sum.cx, c->invIB.cx);
        sum.cy = m3Add3(sum.cy, c->invIB.cy);
        sum.cz = m3Add3(sum.cz, c->invIB.cz);
        c->rollingK = sum;
    }
    c->softness = (c->invMassA == 0.0f || c->invMassB == 0.0f) ? staticSoft : soft;
    for (int32_t k = 0; k < c->pointCount; ++k)
    {
        m3ConstraintPointDev* cp = &c->points[k];
        cp->rA = manifold->points[k].anchorA;
        cp->rB = manifold->points[k].anchorB;
        cp->baseSeparation = manifold->points[k].separation -
                             (m3Dot3(cp->rB, c->normal) - m3Dot3(cp->rA, c->normal));
        cp->normalMass = m3EffectiveMass(c, cp->rA, cp->rB, c->normal);
        cp->relativeVelocity =
            m3Dot3(m3Sub3(m3VelocityAt(w, bodyB, cp->rB), m3VelocityAt(w, bodyA, cp->rA)),
                   c->normal);
        cp->normalImpulse = manifold->points[k].normalImpulse;
        cp->totalNormalImpulse = 0.0f;
    }
    m3Vec3 originA = v3(0.0f, 0.0f, 0.0f);
    m3Vec3 originB = v3(0.0f, 0.0f, 0.0f);
    for (int32_t k = 0; k < c->pointCount; ++k)
    {
        originA = m3Add3(originA, c->points[k].rA);
        originB = m3Add3(originB, c->points[k].rB);
    }
    m3real invCount = 1.0f / (m3real)c->pointCount;
    c->originA = m3MulSV3(invCount, originA);
    c->originB = m3MulSV3(invCount, originB);
    for (int32_t k = 0; k < c->pointCount; ++k)
    {
        c->points[k].leverArm = m3Length3(m3Sub3(c->points[k].rA, c->originA));
    }
    m3Vec3 rtA1 = m3Cross3(c->originA, c->t1);
    m3Vec3 rtA2 = m3Cross3(c->originA, c->t2);
    m3Vec3 rtB1 = m3Cross3(c->originB, c->t1);
    m3Vec3 rtB2 = m3Cross3(c->originB, c->t2);
    m3real k11 = c->invMassA + c->invMassB + m3Dot3(rtA1, m3MulMV3(c->invIA, rtA1)) +
                 m3Dot3(rtB1, m3MulMV3(c->invIB, rtB1));
    m3real k22 = c->invMassA + c->invMassB + m3Dot3(rtA2, m3MulMV3(c->invIA, rtA2)) +
                 m3Dot3(rtB2, m3MulMV3(c->invIB, rtB2));
    m3real k12 = m3Dot3(rtA1, m3MulMV3(c->invIA, rtA2)) + m3Dot3(rtB1, m3MulMV3(c->invIB, rtB2));
    m3real det = k11 * k22 - k12 * k12;
    if (det > 0.0f)
    {
        m3real invDet = 1.0f / det;
        c->frictionK11 = k22 * invDet;
        c->frictionK22 = k11 * invDet;
        c->frictionK12 = -k12 * invDet;
    }
    else
    {
        c->frictionK11 = 0.0f;
        c->frictionK22 = 0.0f;
        c->frictionK12 = 0.0f;
    }
    c->frictionImpulse1 = m3Dot3(manifold->frictionImpulse, c->t1);
    c->frictionImpulse2 = m3Dot3(manifold->frictionImpulse, c->t2);
    m3Vec3 surf = m3Sub3(surfA, surfB);
    c->tangentVelocity1 = m3Dot3(surf, c->t1);
    c->tangentVelocity2 = m3Dot3(surf, c->t2);
    m3Vec3 iSumN = m3Add3(m3MulMV3(c->invIA, c->normal), m3MulMV3(c->invIB, c->normal));
    m3real twistK = m3Dot3(c->normal, iSumN);
    c->twistMass = twistK > 0.0f ? 1.0f / twistK : 0.0f;
    c->twistImpulse = manifold->twistImpulse;
}

// Writes a prepared row into its solve slot: every word a later pass
// reads (points only below the point count, the rolling matrix only
// when rolling resistance is positive) and the starting accumulators.
__device__ void m3WriteContactRow(const m3ConRows& r, int32_t slot, const m3ContactDev& c)
{
    float* ro = r.ro + slot;
    float* acc = r.acc + slot;
    const int64_t st = r.stride;
    auto put = [&](int32_t k, m3real x) { ro[k * st] = x; };
    auto putv = [&](int32_t k, m3Vec3 x) {
        put(k, x.x);
        put(k + 1, x.y);
        put(k + 2, x.z);
    };
    auto putm = [&](int32_t k, const m3Mat3& x) {
        putv(k, x.cx);
        putv(k + 3, x.cy);
        putv(k + 6, x.cz);
    };
    int32_t* ri = reinterpret_cast<int32_t*>(ro);
    ri[M3C_BODY_A * st] = c.bodyA;
    ri[M3C_BODY_B * st] = c.bodyB;
    ri[M3C_MANIFOLD * st] = c.manifoldIndex;
    ri[M3C_POINTS * st] = c.pointCount;
    ri[M3C_FLAGS * st] = (c.dynA ? 1 : 0) | (c.dynB ? 2 : 0);
    putv(M3C_NORMAL, c.normal);
    putv(M3C_T1, c.t1);
    putv(M3C_T2, c.t2);
    putv(M3C_ORIGIN_A, c.originA);
    putv(M3C_ORIGIN_B, c.originB);
    put(M3C_K11, c.frictionK11);
    put(M3C_K12, c.frictionK12);
    put(M3C_K22, c.frictionK22);
    put(M3C_TWIST_MASS, c.twistMass);
    put(M3C_TANGENT_V1, c.tangentVelocity1);
    put(M3C_TANGENT_V2, c.tangentVelocity2);
    put(M3C_FRICTION, c.friction);
    put(M3C_RESTITUTION, c.restitution);
    put(M3C_INV_MASS_A, c.invMassA);
    put(M3C_INV_MASS_B, c.invMassB);
    put(M3C_SOFT, c.softness.biasRate);
    put(M3C_SOFT + 1, c.softness.massScale);
    put(M3C_SOFT + 2, c.softness.impulseScale);
    put(M3C_ROLLING, c.rollingResistance);
    if (c.rollingResistance > 0.0f)
    {
        putm(M3C_ROLLING_K, c.rollingK);
    }
    for (int32_t k = 0; k < c.pointCount; ++k)
    {
        const int32_t p = M3C_POINT0 + M3C_POINT_WORDS * k;
        const m3ConstraintPointDev& cp = c.points[k];
        putv(p, cp.rA);
        putv(p + 3, cp.rB);
        put(p + 6, cp.baseSeparation);
        put(p + 7, cp.normalMass);
        put(p + 8, cp.leverArm);
        put(p + 9, cp.relativeVelocity);
        acc[(M3A_NORMAL + k) * st] = cp.normalImpulse;
        acc[(M3A_TOTAL_NORMAL + k) * st] = cp.totalNormalImpulse;
    }
    acc[M3A_FRICTION1 * st] = c.frictionImpulse1;
    acc[M3A_FRICTION2 * st] = c.frictionImpulse2;
    acc[M3A_TWIST * st] = c.twistImpulse;
    acc[M3A_ROLLING * st] = c.rollingImpulse.x;
    acc[(M3A_ROLLING + 1) * st] = c.rollingImpulse.y;
    acc[(M3A_ROLLING + 2) * st] = c.rollingImpulse.z;
}

// solver.c:408-428
__device__ void m3WarmStartContact(const m3WorldView& w, const m3ConRef& c, const m3Mat3* invI)
{
    const m3ConBodies cb = m3LoadConBodies(c, invI);
    const int32_t pc = c.n(M3C_POINTS);
    const m3Vec3 normal = c.v(M3C_NORMAL);
    m3real imp[M3_MANIFOLD_MAX_POINTS];
#pragma unroll
    for (int32_t k = 0; k < M3_MANIFOLD_MAX_POINTS; ++k)
    {
        imp[k] = k < pc ? c.a(M3A_NORMAL + k) : 0.0f;
    }
    const m3real f1 = c.a(M3A_FRICTION1);
    const m3real f2 = c.a(M3A_FRICTION2);
    const m3real twist = c.a(M3A_TWIST);
    const m3Vec3 rolling = v3(c.a(M3A_ROLLING), c.a(M3A_ROLLING + 1), c.a(M3A_ROLLING + 2));
#pragma unroll
    for (int32_t k = 0; k < M3_MANIFOLD_MAX_POINTS; ++k)
    {
        if (k < pc)
        {
            const int32_t p = M3C_POINT0 + M3C_POINT_WORDS * k;
            m3ApplyImpulseRow(w, cb, m3MulSV3(imp[k], normal), c.v(p), c.v(p + 3));
        }
    }
    m3Vec3 f = m3Add3(m3MulSV3(f1, c.v(M3C_T1)), m3MulSV3(f2, c.v(M3C_T2)));
    m3ApplyImpulseRow(w, cb, f, c.v(M3C_ORIGIN_A), c.v(M3C_ORIGIN_B));
    m3Vec3 tw = m3Add3(m3MulSV3(twist, normal), rolling);
    if (cb.dynA)
    {
        w.w[cb.a] = m3Sub3(w.w[cb.a], m3MulMV3(cb.iA, tw));
    }
    if (cb.dynB)
    {
        w.w[cb.b] = m3Add3(w.w[cb.b], m3MulMV3(cb.iB, tw));
    }
}

// solver.c:430-574
__device__ void m3SolveContact(const m3WorldView& w, const m3ConRef& c, const m3Mat3* invI,
                               const m3Vec3* deltaPos, const m3Quat* deltaRot, m3real invH,
                               m3real pushMaxSpeed, bool useBias)
{
    const m3ConBodies cb = m3LoadConBodies(c, invI);
    const int32_t pc = c.n(M3C_POINTS);
    const m3Vec3 normal = c.v(M3C_NORMAL);
    m3real imp[M3_MANIFOLD_MAX_POINTS];
    m3real tot[M3_MANIFOLD_MAX_POINTS];
#pragma unroll
    for (int32_t k = 0; k < M3_MANIFOLD_MAX_POINTS; ++k)
    {
        imp[k] = k < pc ? c.a(M3A_NORMAL + k) : 0.0f;
        tot[k] = k < pc ? c.a(M3A_TOTAL_NORMAL + k) : 0.0f;
    }
    m3real passNormal = 0.0f;
    m3real twistLimit = 0.0f;
    const m3Quat qA = deltaRot[cb.a];
    const m3Quat qB = deltaRot[cb.b];
    const m3Vec3 dpA = deltaPos[cb.a];
    const m3Vec3 dpB = deltaPos[cb.b];
#pragma unroll
    for (int32_t k = 0; k < M3_MANIFOLD_MAX_POINTS; ++k)
    {
        if (k < pc)
        {
            const int32_t p = M3C_POINT0 + M3C_POINT_WORDS * k;
            const m3Vec3 rA = c.v(p);
            const m3Vec3 rB = c.v(p + 3);
            m3Vec3 rsA = m3RotateVec3(qA, rA);
            m3Vec3 rsB = m3RotateVec3(qB, rB);
            m3Vec3 ds = m3Add3(m3Sub3(dpB, dpA), m3Sub3(rsB, rsA));
            m3real s = c.f(p + 6) + m3Dot3(ds, normal);
            m3real bias = 0.0f;
            m3real massScale = 1.0f;
            m3real impulseScale = 0.0f;
            if (s > 0.0f)
            {
                bias = s * invH;
            }
            else if (useBias)
            {
                bias = m3MaxF(c.f(M3C_SOFT) * s, -pushMaxSpeed);
                massScale = c.f(M3C_SOFT + 1);
                impulseScale = c.f(M3C_SOFT + 2);
            }
            m3real vn = m3Dot3(m3Sub3(m3VelocityAt(w, cb.b, rB), m3VelocityAt(w, cb.a, rA)), normal);
            m3real impulse = -c.f(p + 7) * massScale * (vn + bias) - impulseScale * imp[k];
            m3real newImpulse = m3MaxF(imp[k] + impulse, 0.0f);
            impulse = newImpulse - imp[k];
            imp[k] = newImpulse;
            tot[k] += newImpulse;
            passNormal += newImpulse;
            twistLimit += c.f(p + 8) * newImpulse;
            m3ApplyImpulseRow(w, cb, m3MulSV3(impulse, normal), rA, rB);
        }
    }
#pragma unroll
    for (int32_t k = 0; k < M3_MANIFOLD_MAX_POINTS; ++k)
    {
        if (k < pc)
        {
            c.a(M3A_NORMAL + k) = imp[k];
            c.a(M3A_TOTAL_NORMAL + k) = tot[k];
        }
    }
    if (useBias)
    {
        return;
    }
    const m3real friction = c.f(M3C_FRICTION);
    {
        m3Vec3 wRel = m3Sub3(w.w[cb.b], w.w[cb.a]);
        m3real twistSpeed = m3Dot3(normal, wRel);
        m3real maxTwist = friction * twistLimit;
        m3real delta = -c.f(M3C_TWIST_MASS) * twistSpeed;
        m3real oldTwist = c.a(M3A_TWIST);
        m3real newTwist = oldTwist + delta;
        if (newTwist < -maxTwist)
        {
            newTwist = -maxTwist;
        }
        else if (newTwist > maxTwist)
        {
            newTwist = maxTwist;
        }
        delta = newTwist - oldTwist;
        c.a(M3A_TWIST) = newTwist;
        m3Vec3 tw = m3MulSV3(delta, normal);
        if (cb.dynA)
        {
            w.w[cb.a] = m3Sub3(w.w[cb.a], m3MulMV3(cb.iA, tw));
        }
        if (cb.dynB)
        {
            w.w[cb.b] = m3Add3(w.w[cb.b], m3MulMV3(cb.iB, tw));
        }
    }
    const m3real rollingResistance = c.f(M3C_ROLLING);
    if (rollingResistance > 0.0f)
    {
        // The reference writes both bodies here whatever their type
        // (solver.c:542-545); the step refuses worlds where that would
        // touch a non-dynamic body, so both sides are dynamic here.
        const m3Mat3 rollingK = c.m(M3C_ROLLING_K);
        const m3Vec3 rollingImpulse =
            v3(c.a(M3A_ROLLING), c.a(M3A_ROLLING + 1), c.a(M3A_ROLLING + 2));
        m3Vec3 wRel = m3Sub3(w.w[cb.b], w.w[cb.a]);
        m3Vec3 delta = m3MulSV3(-1.0f, m3Solve3(&rollingK, wRel));
        m3Vec3 accum = m3Add3(rollingImpulse, delta);
        m3real maxRoll = rollingResistance * passNormal;
        m3real mag2 = m3Dot3(accum, accum);
        if (mag2 > maxRoll * maxRoll && mag2 > 0.0f)
        {
            accum = m3MulSV3(maxRoll / sqrtf(mag2), accum);
        }
        delta = m3Sub3(accum, rollingImpulse);
        c.a(M3A_ROLLING) = accum.x;
        c.a(M3A_ROLLING + 1) = accum.y;
        c.a(M3A_ROLLING + 2) = accum.z;
        w.w[cb.a] = m3Sub3(w.w[cb.a], m3MulMV3(cb.iA, delta));
        w.w[cb.b] = m3Add3(w.w[cb.b], m3MulMV3(cb.iB, delta));
    }
    {
        const m3Vec3 t1 = c.v(M3C_T1);
        const m3Vec3 t2 = c.v(M3C_T2);
        const m3Vec3 originA = c.v(M3C_ORIGIN_A);
        const m3Vec3 originB = c.v(M3C_ORIGIN_B);
        const m3real k11 = c.f(M3C_K11);
        const m3real k12 = c.f(M3C_K12);
        const m3real k22 = c.f(M3C_K22);
        const m3real oldF1 = c.a(M3A_FRICTION1);
        const m3real oldF2 = c.a(M3A_FRICTION2);
        m3Vec3 vrel = m3Sub3(m3VelocityAt(w, cb.b, originB), m3VelocityAt(w, cb.a, originA));
        m3real vt1 = m3Dot3(vrel, t1) - c.f(M3C_TANGENT_V1);
        m3real vt2 = m3Dot3(vrel, t2) - c.f(M3C_TANGENT_V2);
        m3real f1 = oldF1 - (k11 * vt1 + k12 * vt2);
        m3real f2 = oldF2 - (k12 * vt1 + k22 * vt2);
        m3real maxFriction = friction * passNormal;
        m3real mag2 = f1 * f1 + f2 * f2;
        if (mag2 > maxFriction * maxFriction)
        {
            m3real mag = sqrtf(mag2);
            m3real scale = mag > 0.0f ? maxFriction / mag : 0.0f;
            f1 *= scale;
            f2 *= scale;
        }
        m3real d1 = f1 - oldF1;
        m3real d2 = f2 - oldF2;
        c.a(M3A_FRICTION1) = f1;
        c.a(M3A_FRICTION2) = f2;
        m3ApplyImpulseRow(w, cb, m3Add3(m3MulSV3(d1, t1), m3MulSV3(d2, t2)), originA, originB);
    }
}

// solver.c:2879-2906 (one constraint's points, in order).
__device__ void m3RestituteContact(const m3WorldView& w, const m3ConRef& c, const m3Mat3* invI,
                                   m3real threshold)
{
    const m3real restitution = c.f(M3C_RESTITUTION);
    if (restitution == 0.0f)
    {
        return;
    }
    const m3ConBodies cb = m3LoadConBodies(c, invI);
    const int32_t pc = c.n(M3C_POINTS);
    const m3Vec3 normal = c.v(M3C_NORMAL);
    for (int32_t k = 0; k < pc; ++k)
    {
        const int32_t p = M3C_POINT0 + M3C_POINT_WORDS * k;
        const m3real relativeVelocity = c.f(p + 9);
        if (relativeVelocity > -threshold || c.a(M3A_TOTAL_NORMAL + k) == 0.0f)
        {
            continue;
        }
        const m3Vec3 rA = c.v(p);
        const m3Vec3 rB = c.v(p + 3);
        m3real vn = m3Dot3(m3Sub3(m3VelocityAt(w, cb.b, rB), m3VelocityAt(w, cb.a, rA)), normal);
        m3real impulse = -c.f(p + 7) * (vn + restitution * relativeVelocity);
        const m3real old = c.a(M3A_NORMAL + k);
        m3real newImpulse = m3MaxF(old + impulse, 0.0f);
        impulse = newImpulse - old;
        c.a(M3A_NORMAL + k) = newImpulse;
        m3ApplyImpulseRow(w, cb, m3MulSV3(impulse, normal), rA, rB);
    }
}

// solver.c:2979-3039 without the hit-event stream (observer only).
__device__ void m3StoreContact(const m3ConRef& c, m3Manifold* manifolds)
{
    m3Manifold* manifold = &manifolds[c.n(M3C_MANIFOLD)];
    const int32_t pc = c.n(M3C_POINTS);
    for (int32_t k = 0; k < pc; ++k)
    {
        manifold->points[k].normalImpulse = c.a(M3A_NORMAL + k);
    }
    manifold->frictionImpulse = m3Add3(m3MulSV3(c.a(M3A_FRICTION1), c.v(M3C_T1)),
                                       m3MulSV3(c.a(M3A_FRICTION2), c.v(M3C_T2)));
    manifold->twistImpulse = c.a(M3A_TWIST);
    manifold->rollingImpulse = v3(c.a(M3A_ROLLING), c.a(M3A_ROLLING + 1), c.a(M3A_ROLLING + 2));
}

// The hit event of one contact constraint (solver.c:2987-3033), if any:
// for a pair with a hit-enabled shape, the fastest-approaching point whose
// approach beat `threshold` and whose impulse fired.  Written after the
// impulses are final and before the continuous phase moves any body, as
// the reference's store does; shape ids carry the world index 0 (the host
// fills it in).  Returns whether there is one.
__device__ bool m3HitCandidate(const m3WorldView& w, const m3ConRef& c, const uint64_t* keys,
                               m3real threshold, m3HitEvent* out)
{
    const uint64_t key = keys[c.n(M3C_MANIFOLD)];
    const int32_t shapeA = (int32_t)(key >> 32);
    const int32_t shapeB = (int32_t)(key & 0xFFFFFFFFu);
    if (w.hitEvents[shapeA] == 0 && w.hitEvents[shapeB] == 0)
    {
        return false;
    }
    const int32_t pc = c.n(M3C_POINTS);
    int32_t best = -1;
    m3real bestSpeed = 0.0f;
    for (int32_t k = 0; k < pc; ++k)
    {
        const m3real rv = c.f(M3C_POINT0 + M3C_POINT_WORDS * k + 9);
        if (rv < -threshold && c.a(M3A_TOTAL_NORMAL + k) > 0.0f && (best < 0 || rv < bestSpeed))
        {
            best = k;
            bestSpeed = rv;
        }
    }
    if (best < 0)
    {
        return false;
    }
    const int32_t bodyA = c.n(M3C_BODY_A);
    const m3Transform xf = w.xf[bodyA];
    const m3Vec3 lcA = m3RotateVec3(xf.q, w.lc[bodyA]);
    const m3Vec3 rA = c.v(M3C_POINT0 + M3C_POINT_WORDS * best);
    m3HitEvent e;
    e.shapeA.index1 = shapeA + 1;
    e.shapeA.world0 = 0;
    e.shapeA.generation = w.shapeGen[shapeA];
    e.shapeB.index1 = shapeB + 1;
    e.shapeB.world0 = 0;
    e.shapeB.generation = w.shapeGen[shapeB];
    e.point.x = xf.p.x + (double)lcA.x + (double)rA.x;
    e.point.y = xf.p.y + (double)lcA.y + (double)rA.y;
    e.point.z = xf.p.z + (double)lcA.z + (double)rA.z;
    e.normal = c.v(M3C_NORMAL);
    e.approachSpeed = -bestSpeed;
    *out = e;
    return true;
}

// Implicit gyroscopic step, one Newton iteration in body coordinates,
// isotropic tensors gated out (solver.c:2933-2977).
__device__ m3Vec3 m3GyroscopicOmega(const m3WorldView& w, int32_t body, m3Vec3 om, m3real h)
{
    const m3Mat3 inertia = w.inertia[body];
    const m3real i00 = inertia.cx.x;
    const m3real i01 = inertia.cy.x;
    const m3real i02 = inertia.cz.x;
    const m3real i11 = inertia.cy.y;
    const m3real i12 = inertia.cz.y;
    const m3real i22 = inertia.cz.z;
    if (i01 == 0.0f && i02 == 0.0f && i12 == 0.0f && i00 == i11 && i11 == i22)
    {
        return om;
    }
    m3Quat q = w.xf[body].q;
    m3Vec3 omega2 = m3InvRotateVec3(q, om);
    const m3real w1 = omega2.x;
    const m3real w2 = omega2.y;
    const m3real w3 = omega2.z;
    const m3real Iw1 = i00 * w1 + i01 * w2 + i02 * w3;
    const m3real Iw2 = i01 * w1 + i11 * w2 + i12 * w3;
    const m3real Iw3 = i02 * w1 + i12 * w2 + i22 * w3;
    m3Vec3 b = v3(h * (w2 * Iw3 - w3 * Iw2), h * (w3 * Iw1 - w1 * Iw3), h * (w1 * Iw2 - w2 * Iw1));
    m3Mat3 J;
    J.cx = v3(i00 + h * (w2 * i02 - w3 * i01), i01 + h * (w3 * i00 - w1 * i02 - Iw3),
              i02 + h * (w1 * i01 - w2 * i00 + Iw2));
    J.cy = v3(i01 + h * (w2 * i12 - w3 * i11 + Iw3), i11 + h * (w3 * i01 - w1 * i12),
              i12 + h * (w1 * i11 - w2 * i01 - Iw1));
    J.cz = v3(i02 + h * (w2 * i22 - w3 * i12 - Iw2), i12 + h * (w3 * i02 - w1 * i22 + Iw1),
              i22 + h * (w1 * i12 - w2 * i02));
    omega2 = m3Sub3(omega2, m3Solve3(&J, b));
    return m3RotateVec3(q, omega2);
}

// One mover's velocity integration (solver.c:4088-4147), water
// volumes absent.
__device__ void m3IntegrateVelocity(const m3WorldView& w, int32_t i, m3real h)
{
    const m3WorldScalars* sc = w.sc;
    m3Vec3 v = w.v[i];
    m3Vec3 om = w.w[i];
    v = m3Add3(v, m3MulSV3(h * w.gravityScale[i], sc->gravity));
    v = m3Add3(v, m3MulSV3(h * w.invMass[i], w.force[i]));
    m3Vec3 tq = w.torque[i];
    if (tq.x != 0.0f || tq.y != 0.0f || tq.z != 0.0f)
    {
        om = m3Add3(om, m3MulSV3(h, m3MulMV3(m3WorldInvInertiaDev(w, i), tq)));
    }
    v = m3MulSV3(1.0f / (1.0f + h * w.linDamp[i]), v);
    om = m3MulSV3(1.0f / (1.0f + h * w.angDamp[i]), om);
    om = m3GyroscopicOmega(w, i, om, h);
    m3real v2 = m3Dot3(v, v);
    m3real cap = sc->maximumLinearSpeed;
    if (v2 > cap * cap)
    {
        v = m3MulSV3(cap / sqrtf(v2), v);
    }
    if ((w.locks[i] & M3_LOCKS_ALLOW_FAST_ROTATION) == 0)
    {
        m3real w2 = m3Dot3(om, om);
        m3real wcap = sc->maximumAngularSpeed;
        if (w2 > wcap * wcap)
        {
            om = m3MulSV3(wcap / sqrtf(w2), om);
        }
    }
    w.v[i] = v;
    w.w[i] = om;
}

// One mover's position integration about the centre of mass and the
// substep delta accumulation (solver.c:4156-4198).
__device__ void m3IntegratePosition(const m3WorldView& w, int32_t i, m3real h, m3Vec3* deltaPos,
                                    m3Quat* deltaRot)
{
    m3Vec3 v = w.v[i];
    m3Vec3 om = w.w[i];
    uint8_t locks = w.locks[i];
    if (locks != 0)
    {
        if (locks & 1u)
            v.x = 0.0f;
        if (locks & 2u)
            v.y = 0.0f;
        if (locks & 4u)
            v.z = 0.0f;
        if (locks & 8u)
            om.x = 0.0f;
        if (locks & 16u)
            om.y = 0.0f;
        if (locks & 32u)
            om.z = 0.0f;
        w.v[i] = v;
        w.w[i] = om;
    }
    m3Vec3 lc = w.lc[i];
    m3Transform xf = w.xf[i];
    m3Vec3 rlcOld = m3RotateVec3(xf.q, lc);
    double cx = xf.p.x + (double)rlcOld.x + (double)(h * v.x);
    double cy = xf.p.y + (double)rlcOld.y + (double)(h * v.y);
    double cz = xf.p.z + (double)rlcOld.z + (double)(h * v.z);
    m3Vec3 dw = m3MulSV3(h, om);
    xf.q = m3IntegrateRotation(xf.q, dw);
    m3Vec3 rlcNew = m3RotateVec3(xf.q, lc);
    xf.p.x = cx - (double)rlcNew.x;
    xf.p.y = cy - (double)rlcNew.y;
    xf.p.z = cz - (double)rlcNew.z;
    w.xf[i] = xf;
    deltaPos[i] = m3Add3(deltaPos[i], m3MulSV3(h, v));
    deltaRot[i] = m3IntegrateRotation(deltaRot[i], dw);
}

#endif // M3_SOLVER_CUH
