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

// solver.c:105-121
__device__ __forceinline__ void m3ApplyImpulseDev(const m3WorldView& w, const m3ContactDev* c,
                                                  m3Vec3 impulse, m3Vec3 rsA, m3Vec3 rsB)
{
    if (c->dynA)
    {
        w.v[c->bodyA] = m3Sub3(w.v[c->bodyA], m3MulSV3(c->invMassA, impulse));
        w.w[c->bodyA] = m3Sub3(w.w[c->bodyA], m3MulMV3(c->invIA, m3Cross3(rsA, impulse)));
    }
    if (c->dynB)
    {
        w.v[c->bodyB] = m3Add3(w.v[c->bodyB], m3MulSV3(c->invMassB, impulse));
        w.w[c->bodyB] = m3Add3(w.w[c->bodyB], m3MulMV3(c->invIB, m3Cross3(rsB, impulse)));
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
                                 m3SoftDev soft, m3SoftDev staticSoft)
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
    c->invIA = m3WorldInvInertiaDev(w, bodyA);
    c->invIB = m3WorldInvInertiaDev(w, bodyB);
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

// solver.c:408-428
__device__ void m3WarmStartContact(const m3WorldView& w, m3ContactDev* c)
{
    for (int32_t k = 0; k < c->pointCount; ++k)
    {
        m3ConstraintPointDev* cp = &c->points[k];
        m3ApplyImpulseDev(w, c, m3MulSV3(cp->normalImpulse, c->normal), cp->rA, cp->rB);
    }
    m3Vec3 f = m3Add3(m3MulSV3(c->frictionImpulse1, c->t1), m3MulSV3(c->frictionImpulse2, c->t2));
    m3ApplyImpulseDev(w, c, f, c->originA, c->originB);
    m3Vec3 tw = m3Add3(m3MulSV3(c->twistImpulse, c->normal), c->rollingImpulse);
    if (c->dynA)
    {
        w.w[c->bodyA] = m3Sub3(w.w[c->bodyA], m3MulMV3(c->invIA, tw));
    }
    if (c->dynB)
    {
        w.w[c->bodyB] = m3Add3(w.w[c->bodyB], m3MulMV3(c->invIB, tw));
    }
}

// solver.c:430-574
__device__ void m3SolveContact(const m3WorldView& w, m3ContactDev* c, const m3Vec3* deltaPos,
                               const m3Quat* deltaRot, m3real invH, m3real pushMaxSpeed,
                               bool useBias)
{
    m3real passNormal = 0.0f;
    m3real twistLimit = 0.0f;
    const m3Quat qA = deltaRot[c->bodyA];
    const m3Quat qB = deltaRot[c->bodyB];
    const m3Vec3 dpA = deltaPos[c->bodyA];
    const m3Vec3 dpB = deltaPos[c->bodyB];
    for (int32_t k = 0; k < c->pointCount; ++k)
    {
        m3ConstraintPointDev* cp = &c->points[k];
        m3Vec3 rsA = m3RotateVec3(qA, cp->rA);
        m3Vec3 rsB = m3RotateVec3(qB, cp->rB);
        m3Vec3 ds = m3Add3(m3Sub3(dpB, dpA), m3Sub3(rsB, rsA));
        m3real s = cp->baseSeparation + m3Dot3(ds, c->normal);
        m3real bias = 0.0f;
        m3real massScale = 1.0f;
        m3real impulseScale = 0.0f;
        if (s > 0.0f)
        {
            bias = s * invH;
        }
        else if (useBias)
        {
            bias = m3MaxF(c->softness.biasRate * s, -pushMaxSpeed);
            massScale = c->softness.massScale;
            impulseScale = c->softness.impulseScale;
        }
        m3real vn = m3Dot3(
            m3Sub3(m3VelocityAt(w, c->bodyB, cp->rB), m3VelocityAt(w, c->bodyA, cp->rA)),
            c->normal);
        m3real impulse = -cp->normalMass * massScale * (vn + bias) - impulseScale * cp->normalImpulse;
        m3real newImpulse = m3MaxF(cp->normalImpulse + impulse, 0.0f);
        impulse = newImpulse - cp->normalImpulse;
        cp->normalImpulse = newImpulse;
        cp->totalNormalImpulse += newImpulse;
        passNormal += newImpulse;
        twistLimit += cp->leverArm * newImpulse;
        m3ApplyImpulseDev(w, c, m3MulSV3(impulse, c->normal), cp->rA, cp->rB);
    }
    if (useBias)
    {
        return;
    }
    {
        m3Vec3 wRel = m3Sub3(w.w[c->bodyB], w.w[c->bodyA]);
        m3real twistSpeed = m3Dot3(c->normal, wRel);
        m3real maxTwist = c->friction * twistLimit;
        m3real delta = -c->twistMass * twistSpeed;
        m3real oldTwist = c->twistImpulse;
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
        c->twistImpulse = newTwist;
        m3Vec3 tw = m3MulSV3(delta, c->normal);
        if (c->dynA)
        {
            w.w[c->bodyA] = m3Sub3(w.w[c->bodyA], m3MulMV3(c->invIA, tw));
        }
        if (c->dynB)
        {
            w.w[c->bodyB] = m3Add3(w.w[c->bodyB], m3MulMV3(c->invIB, tw));
        }
    }
    if (c->rollingResistance > 0.0f)
    {
        // The reference writes both bodies here whatever their type
        // (solver.c:542-545); the step refuses worlds where that would
        // touch a non-dynamic body, so both sides are dynamic here.
        m3Vec3 wRel = m3Sub3(w.w[c->bodyB], w.w[c->bodyA]);
        m3Vec3 delta = m3MulSV3(-1.0f, m3Solve3(&c->rollingK, wRel));
        m3Vec3 accum = m3Add3(c->rollingImpulse, delta);
        m3real maxRoll = c->rollingResistance * passNormal;
        m3real mag2 = m3Dot3(accum, accum);
        if (mag2 > maxRoll * maxRoll && mag2 > 0.0f)
        {
            accum = m3MulSV3(maxRoll / sqrtf(mag2), accum);
        }
        delta = m3Sub3(accum, c->rollingImpulse);
        c->rollingImpulse = accum;
        w.w[c->bodyA] = m3Sub3(w.w[c->bodyA], m3MulMV3(c->invIA, delta));
        w.w[c->bodyB] = m3Add3(w.w[c->bodyB], m3MulMV3(c->invIB, delta));
    }
    {
        m3Vec3 vrel = m3Sub3(m3VelocityAt(w, c->bodyB, c->originB),
                             m3VelocityAt(w, c->bodyA, c->originA));
        m3real vt1 = m3Dot3(vrel, c->t1) - c->tangentVelocity1;
        m3real vt2 = m3Dot3(vrel, c->t2) - c->tangentVelocity2;
        m3real f1 = c->frictionImpulse1 - (c->frictionK11 * vt1 + c->frictionK12 * vt2);
        m3real f2 = c->frictionImpulse2 - (c->frictionK12 * vt1 + c->frictionK22 * vt2);
        m3real maxFriction = c->friction * passNormal;
        m3real mag2 = f1 * f1 + f2 * f2;
        if (mag2 > maxFriction * maxFriction)
        {
            m3real mag = sqrtf(mag2);
            m3real scale = mag > 0.0f ? maxFriction / mag : 0.0f;
            f1 *= scale;
            f2 *= scale;
        }
        m3real d1 = f1 - c->frictionImpulse1;
        m3real d2 = f2 - c->frictionImpulse2;
        c->frictionImpulse1 = f1;
        c->frictionImpulse2 = f2;
        m3ApplyImpulseDev(w, c, m3Add3(m3MulSV3(d1, c->t1), m3MulSV3(d2, c->t2)), c->originA,
                          c->originB);
    }
}

// solver.c:2879-2906 (one constraint's points, in order).
__device__ void m3RestituteContact(const m3WorldView& w, m3ContactDev* c, m3real threshold)
{
    if (c->restitution == 0.0f)
    {
        return;
    }
    for (int32_t k = 0; k < c->pointCount; ++k)
    {
        m3ConstraintPointDev* cp = &c->points[k];
        if (cp->relativeVelocity > -threshold || cp->totalNormalImpulse == 0.0f)
        {
            continue;
        }
        m3real vn = m3Dot3(
            m3Sub3(m3VelocityAt(w, c->bodyB, cp->rB), m3VelocityAt(w, c->bodyA, cp->rA)),
            c->normal);
        m3real impulse = -cp->normalMass * (vn + c->restitution * cp->relativeVelocity);
        m3real newImpulse = m3MaxF(cp->normalImpulse + impulse, 0.0f);
        impulse = newImpulse - cp->normalImpulse;
        cp->normalImpulse = newImpulse;
        m3ApplyImpulseDev(w, c, m3MulSV3(impulse, c->normal), cp->rA, cp->rB);
    }
}

// solver.c:2979-3039 without the hit-event stream (observer only).
__device__ void m3StoreContact(const m3ContactDev* c, m3Manifold* manifolds)
{
    m3Manifold* manifold = &manifolds[c->manifoldIndex];
    for (int32_t k = 0; k < c->pointCount; ++k)
    {
        manifold->points[k].normalImpulse = c->points[k].normalImpulse;
    }
    manifold->frictionImpulse =
        m3Add3(m3MulSV3(c->frictionImpulse1, c->t1), m3MulSV3(c->frictionImpulse2, c->t2));
    manifold->twistImpulse = c->twistImpulse;
    manifold->rollingImpulse = c->rollingImpulse;
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
