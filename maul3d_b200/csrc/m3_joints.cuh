// Joint rows on the device: spherical (point weld), revolute (hinge:
// limits, motor, collinearity lock) and fixed (rotation lock + point
// weld), prepared, warm-started, solved and stored exactly as the
// reference does (src/solver.c:699-1042, :1044-1209, :1211-2702,
// :2704-2730).  The reference runs joints serially in slot order before
// the contact colours; the device groups them into dependency levels (a
// joint's level is one past the last earlier joint sharing a body with
// it), so rows of one level touch disjoint bodies and run on separate
// threads while every body still sees its joints in slot order.
#ifndef M3_JOINTS_CUH
#define M3_JOINTS_CUH

#include "m3_solver.cuh"

struct m3JointDev
{
    int32_t joint;
    uint8_t type;
    uint8_t flags;
    uint8_t pad[2];
    int32_t bodyA;
    int32_t bodyB;
    m3Vec3 rA;
    m3Vec3 rB;
    m3Vec3 deltaCenter;
    m3real invMassA;
    m3real invMassB;
    m3Mat3 invIA;
    m3Mat3 invIB;
    m3SoftDev softness;
    m3Vec3 impulse;
    m3Quat frameQA;
    m3Quat frameQB;
    m3Vec3 rotationAxis;
    m3real axialMass;
    m3Vec3 perpAxisX;
    m3Vec3 perpAxisY;
    m3real perpImpulseX;
    m3real perpImpulseY;
    m3real motorImpulse;
    m3real lowerImpulse;
    m3real upperImpulse;
    m3real motorSpeed;
    m3real maxMotorEffort;
    m3real lowerLimit;
    m3real upperLimit;
    m3Vec3 angularImpulse;
    m3Vec3 springImpulseV;
};
static_assert(sizeof(m3JointDev) % 4 == 0, "joint rows are copied as 32-bit words");

// Half-quaternion rotation of a frame axis (solver.c:690-696).
__device__ __forceinline__ m3Vec3 m3PerpColumn(m3Quat qA, m3Quat relQ, m3Vec3 axis)
{
    m3Vec3 rv = v3(relQ.x, relQ.y, relQ.z);
    m3Vec3 inner = m3Add3(m3MulSV3(relQ.w, axis), m3Cross3(rv, axis));
    return m3MulSV3(0.5f, m3RotateVec3(qA, inner));
}

// Rotation vector of a relative quaternion (solver.c:672-686).
__device__ __forceinline__ m3Vec3 m3QuatToRotationVec(m3Quat relQ)
{
    if (relQ.w < 0.0f)
    {
        relQ = q4(-relQ.x, -relQ.y, -relQ.z, -relQ.w);
    }
    m3Vec3 v = v3(relQ.x, relQ.y, relQ.z);
    m3real len = sqrtf(m3Dot3(v, v));
    if (len < 1.0e-9f)
    {
        return m3MulSV3(2.0f, v);
    }
    m3real angle = 2.0f * m3Atan2(len, relQ.w);
    return m3MulSV3(angle / len, v);
}

// Joint rows the device path covers: spherical without cone or twist
// limits, revolute with limit and motor, fixed, each with or without
// breaking thresholds; no springs.  Returns 0, or a detail code for a
// refused joint.
__device__ __forceinline__ int32_t m3JointRefusal(const m3WorldView& w, int32_t j)
{
    uint8_t type = w.jtype[j];
    uint8_t flags = w.jflags[j];
    if ((flags & 8) != 0 || (type != 0 && type != 1 && type != 3) ||
        (type == 0 && (flags & 5) != 0))
    {
        return 4000 + type;
    }
    return 0;
}

// A joint gets a row when either side is an awake dynamic body
// (solver.c:705-725).
__device__ __forceinline__ bool m3JointActive(const m3WorldView& w, int32_t j)
{
    if (w.jointAlive[j] == 0)
    {
        return false;
    }
    int32_t bodyA = w.jbodyA[j];
    int32_t bodyB = w.jbodyB[j];
    int awakeDynA = w.btype[bodyA] == M3_BODY_DYNAMIC && w.awake[bodyA];
    int awakeDynB = w.btype[bodyB] == M3_BODY_DYNAMIC && w.awake[bodyB];
    return awakeDynA || awakeDynB;
}

// One joint's row, the body of PrepareJoints (solver.c:726-1042) for
// the device joint types.  Every field the store writes back is set:
// the reference zeroes the row first, so a spherical row stores zero
// perpendicular, limit and angular impulses.
__device__ void m3PrepareJoint(const m3WorldView& w, m3JointDev* c, int32_t j, m3real h)
{
    uint8_t type = w.jtype[j];
    uint8_t flags = w.jflags[j];
    int32_t bodyA = w.jbodyA[j];
    int32_t bodyB = w.jbodyB[j];
    c->joint = j;
    c->bodyA = bodyA;
    c->bodyB = bodyB;
    const m3Transform xfA = w.xf[bodyA];
    const m3Transform xfB = w.xf[bodyB];
    c->rA = m3RotateVec3(xfA.q, m3Sub3(w.jlocalA[j], w.lc[bodyA]));
    c->rB = m3RotateVec3(xfB.q, m3Sub3(w.jlocalB[j], w.lc[bodyB]));
    m3Vec3 rlcA = m3RotateVec3(xfA.q, w.lc[bodyA]);
    m3Vec3 rlcB = m3RotateVec3(xfB.q, w.lc[bodyB]);
    c->deltaCenter = v3((m3real)(xfB.p.x + (double)rlcB.x - xfA.p.x - (double)rlcA.x),
                        (m3real)(xfB.p.y + (double)rlcB.y - xfA.p.y - (double)rlcA.y),
                        (m3real)(xfB.p.z + (double)rlcB.z - xfA.p.z - (double)rlcA.z));
    c->invMassA = w.btype[bodyA] == M3_BODY_DYNAMIC ? w.invMass[bodyA] : 0.0f;
    c->invMassB = w.btype[bodyB] == M3_BODY_DYNAMIC ? w.invMass[bodyB] : 0.0f;
    c->invIA = m3WorldInvInertiaDev(w, bodyA);
    c->invIB = m3WorldInvInertiaDev(w, bodyB);
    c->softness = m3MakeSoft(60.0f, 2.0f, h);
    c->impulse = w.jimpulse[j];
    c->type = type;
    c->flags = flags;
    c->springImpulseV = w.jspringImp[j];
    const m3Quat identity = m3IdentityQuat();
    const m3Vec3 zero = v3(0.0f, 0.0f, 0.0f);
    c->frameQA = identity;
    c->frameQB = identity;
    c->rotationAxis = zero;
    c->axialMass = 0.0f;
    c->perpAxisX = zero;
    c->perpAxisY = zero;
    c->perpImpulseX = 0.0f;
    c->perpImpulseY = 0.0f;
    c->motorImpulse = 0.0f;
    c->lowerImpulse = 0.0f;
    c->upperImpulse = 0.0f;
    c->motorSpeed = 0.0f;
    c->maxMotorEffort = 0.0f;
    c->lowerLimit = 0.0f;
    c->upperLimit = 0.0f;
    c->angularImpulse = zero;
    if (type == 1)
    {
        c->frameQA = m3MulQuat(xfA.q, w.jframeA[j]);
        c->frameQB = m3MulQuat(xfB.q, w.jframeB[j]);
        m3Vec3 axis = m3RotateVec3(c->frameQA, v3(0.0f, 0.0f, 1.0f));
        c->rotationAxis = axis;
        m3Vec3 sum = m3Add3(m3MulMV3(c->invIA, axis), m3MulMV3(c->invIB, axis));
        m3real k = m3Dot3(axis, sum);
        c->axialMass = k > 0.0f ? 1.0f / k : 0.0f;
        m3Quat relQ = m3MulQuat(m3Conj(c->frameQA), c->frameQB);
        c->perpAxisX = m3PerpColumn(c->frameQA, relQ, v3(1.0f, 0.0f, 0.0f));
        c->perpAxisY = m3PerpColumn(c->frameQA, relQ, v3(0.0f, 1.0f, 0.0f));
        c->perpImpulseX = w.jperp[j].x;
        c->perpImpulseY = w.jperp[j].y;
        c->motorImpulse = w.jperp[j].z;
        c->lowerImpulse = w.jlimitImp[j].x;
        c->upperImpulse = w.jlimitImp[j].y;
        c->motorSpeed = w.jmotor[j].x;
        c->maxMotorEffort = w.jmotor[j].y;
        c->lowerLimit = w.jlimits[j].x;
        c->upperLimit = w.jlimits[j].y;
        c->angularImpulse = w.jangular[j];
    }
    else if (type == 3)
    {
        c->frameQA = m3MulQuat(xfA.q, w.jframeA[j]);
        c->frameQB = m3MulQuat(xfB.q, w.jframeB[j]);
        c->angularImpulse = w.jangular[j];
    }
}

// One joint's warm start (solver.c:1044-1209 loop body).
__device__ void m3WarmStartJoint(const m3WorldView& w, m3JointDev* c, const m3Quat* deltaRot)
{
    {
        m3Vec3 rA = m3RotateVec3(deltaRot[c->bodyA], c->rA);
        m3Vec3 rB = m3RotateVec3(deltaRot[c->bodyB], c->rB);
        m3Vec3 angularImpulse = v3(0.0f, 0.0f, 0.0f);
        if (c->type == 1)
        {
            m3real axial = c->springImpulseV.x + c->motorImpulse + c->lowerImpulse - c->upperImpulse;
            angularImpulse = m3Add3(m3MulSV3(c->perpImpulseX, c->perpAxisX),
                                    m3MulSV3(c->perpImpulseY, c->perpAxisY));
            angularImpulse = m3Add3(angularImpulse, m3MulSV3(axial, c->rotationAxis));
        }
        else if (c->type == 3)
        {
            angularImpulse = c->angularImpulse;
        }
        m3Vec3 totalLinear = m3Add3(c->impulse, v3(0.0f, 0.0f, 0.0f));
        w.v[c->bodyA] = m3Sub3(w.v[c->bodyA], m3MulSV3(c->invMassA, totalLinear));
        w.w[c->bodyA] = m3Sub3(w.w[c->bodyA],
                               m3MulMV3(c->invIA, m3Add3(m3Cross3(rA, totalLinear), angularImpulse)));
        w.v[c->bodyB] = m3Add3(w.v[c->bodyB], m3MulSV3(c->invMassB, totalLinear));
        w.w[c->bodyB] = m3Add3(w.w[c->bodyB],
                               m3MulMV3(c->invIB, m3Add3(m3Cross3(rB, totalLinear), angularImpulse)));
    }
}

// One-sided angular limit row (solver.c:1374-1430 form).
__device__ __forceinline__ m3real m3LimitRow(m3real cc, m3real cdot, m3real axialMass,
                                             m3real* accum, const m3SoftDev& soft, m3real invH,
                                             bool useBias)
{
    m3real bias = 0.0f;
    m3real massScale = 1.0f;
    m3real impulseScale = 0.0f;
    if (cc > 0.0f)
    {
        bias = cc * invH;
    }
    else if (useBias)
    {
        bias = soft.biasRate * cc;
        massScale = soft.massScale;
        impulseScale = soft.impulseScale;
    }
    m3real old = *accum;
    m3real delta = -massScale * axialMass * (cdot + bias) - impulseScale * old;
    *accum = m3MaxF(old + delta, 0.0f);
    return *accum - old;
}

// One joint's solve (solver.c:1211-2702 loop body) for the device joint
// types.
__device__ void m3SolveJoint(const m3WorldView& w, m3JointDev* c, const m3Vec3* deltaPos,
                             const m3Quat* deltaRot, m3real hSub, m3real invHSub, bool useBias)
{
    {
        m3Vec3 rA = m3RotateVec3(deltaRot[c->bodyA], c->rA);
        m3Vec3 rB = m3RotateVec3(deltaRot[c->bodyB], c->rB);
        m3Vec3 vA = w.v[c->bodyA];
        m3Vec3 wA = w.w[c->bodyA];
        m3Vec3 vB = w.v[c->bodyB];
        m3Vec3 wB = w.w[c->bodyB];
        if (c->type == 1)
        {
            m3Quat quatA = m3MulQuat(deltaRot[c->bodyA], c->frameQA);
            m3Quat quatB = m3MulQuat(deltaRot[c->bodyB], c->frameQB);
            if (quatA.x * quatB.x + quatA.y * quatB.y + quatA.z * quatB.z + quatA.w * quatB.w <
                0.0f)
            {
                quatB = q4(-quatB.x, -quatB.y, -quatB.z, -quatB.w);
            }
            m3Quat relQ = m3MulQuat(m3Conj(quatA), quatB);
            m3Vec3 axis = c->rotationAxis;
            if ((c->flags & 2) != 0)
            {
                m3real cdot = m3Dot3(m3Sub3(wB, wA), axis) - c->motorSpeed;
                m3real delta = -c->axialMass * cdot;
                m3real newImpulse = c->motorImpulse + delta;
                m3real maxImpulse = c->maxMotorEffort * hSub;
                newImpulse = m3MaxF(-maxImpulse, m3MinF(maxImpulse, newImpulse));
                delta = newImpulse - c->motorImpulse;
                c->motorImpulse = newImpulse;
                wA = m3Sub3(wA, m3MulSV3(delta, m3MulMV3(c->invIA, axis)));
                wB = m3Add3(wB, m3MulSV3(delta, m3MulMV3(c->invIB, axis)));
            }
            if ((c->flags & 1) != 0)
            {
                m3real angle = 2.0f * m3Atan2(relQ.z, relQ.w);
                {
                    m3real cdot = m3Dot3(m3Sub3(wB, wA), axis);
                    m3real delta = m3LimitRow(angle - c->lowerLimit, cdot, c->axialMass,
                                              &c->lowerImpulse, c->softness, invHSub, useBias);
                    wA = m3Sub3(wA, m3MulSV3(delta, m3MulMV3(c->invIA, axis)));
                    wB = m3Add3(wB, m3MulSV3(delta, m3MulMV3(c->invIB, axis)));
                }
                {
                    m3real cdot = m3Dot3(m3Sub3(wA, wB), axis);
                    m3real delta = m3LimitRow(c->upperLimit - angle, cdot, c->axialMass,
                                              &c->upperImpulse, c->softness, invHSub, useBias);
                    wA = m3Add3(wA, m3MulSV3(delta, m3MulMV3(c->invIA, axis)));
                    wB = m3Sub3(wB, m3MulSV3(delta, m3MulMV3(c->invIB, axis)));
                }
            }
            {
                m3Vec3 perpX = m3PerpColumn(quatA, relQ, v3(1.0f, 0.0f, 0.0f));
                m3Vec3 perpY = m3PerpColumn(quatA, relQ, v3(0.0f, 1.0f, 0.0f));
                c->perpAxisX = perpX;
                c->perpAxisY = perpY;
                m3real biasX = 0.0f;
                m3real biasY = 0.0f;
                m3real massScale = 1.0f;
                m3real impulseScale = 0.0f;
                if (useBias)
                {
                    biasX = c->softness.biasRate * relQ.x;
                    biasY = c->softness.biasRate * relQ.y;
                    massScale = c->softness.massScale;
                    impulseScale = c->softness.impulseScale;
                }
                m3Vec3 sumX = m3Add3(m3MulMV3(c->invIA, perpX), m3MulMV3(c->invIB, perpX));
                m3Vec3 sumY = m3Add3(m3MulMV3(c->invIA, perpY), m3MulMV3(c->invIB, perpY));
                m3real kxx = m3Dot3(perpX, sumX);
                m3real kyy = m3Dot3(perpY, sumY);
                m3real kxy = m3Dot3(perpX, sumY);
                m3Vec3 wRel = m3Sub3(wB, wA);
                m3real cdotX = m3Dot3(wRel, perpX) + biasX;
                m3real cdotY = m3Dot3(wRel, perpY) + biasY;
                m3real det = kxx * kyy - kxy * kxy;
                m3real solX = 0.0f;
                m3real solY = 0.0f;
                if (det != 0.0f)
                {
                    m3real inv = 1.0f / det;
                    solX = inv * (kyy * cdotX - kxy * cdotY);
                    solY = inv * (kxx * cdotY - kxy * cdotX);
                }
                m3real deltaX = -massScale * solX - impulseScale * c->perpImpulseX;
                m3real deltaY = -massScale * solY - impulseScale * c->perpImpulseY;
                c->perpImpulseX += deltaX;
                c->perpImpulseY += deltaY;
                m3Vec3 angular = m3Add3(m3MulSV3(deltaX, perpX), m3MulSV3(deltaY, perpY));
                wA = m3Sub3(wA, m3MulMV3(c->invIA, angular));
                wB = m3Add3(wB, m3MulMV3(c->invIB, angular));
            }
            w.w[c->bodyA] = wA;
            w.w[c->bodyB] = wB;
            vA = w.v[c->bodyA];
            wA = w.w[c->bodyA];
            vB = w.v[c->bodyB];
            wB = w.w[c->bodyB];
        }
        else if (c->type == 3)
        {
            m3Vec3 bias = v3(0.0f, 0.0f, 0.0f);
            m3real massScale = 1.0f;
            m3real impulseScale = 0.0f;
            if (useBias)
            {
                m3Quat quatA = m3MulQuat(deltaRot[c->bodyA], c->frameQA);
                m3Quat quatB = m3MulQuat(deltaRot[c->bodyB], c->frameQB);
                m3Quat relQ = m3MulQuat(m3Conj(quatA), quatB);
                m3Vec3 rotVec = m3QuatToRotationVec(relQ);
                m3Vec3 cErr = m3RotateVec3(quatA, rotVec);
                bias = m3MulSV3(c->softness.biasRate, cErr);
                massScale = c->softness.massScale;
                impulseScale = c->softness.impulseScale;
            }
            m3Mat3 k;
            k.cx = m3Add3(m3MulMV3(c->invIA, v3(1.0f, 0.0f, 0.0f)),
                          m3MulMV3(c->invIB, v3(1.0f, 0.0f, 0.0f)));
            k.cy = m3Add3(m3MulMV3(c->invIA, v3(0.0f, 1.0f, 0.0f)),
                          m3MulMV3(c->invIB, v3(0.0f, 1.0f, 0.0f)));
            k.cz = m3Add3(m3MulMV3(c->invIA, v3(0.0f, 0.0f, 1.0f)),
                          m3MulMV3(c->invIB, v3(0.0f, 0.0f, 1.0f)));
            m3Vec3 cdotRot = m3Sub3(wB, wA);
            m3Vec3 sol = m3Solve3(&k, m3Add3(cdotRot, bias));
            m3Vec3 delta = m3Sub3(m3MulSV3(-massScale, sol), m3MulSV3(impulseScale, c->angularImpulse));
            c->angularImpulse = m3Add3(c->angularImpulse, delta);
            wA = m3Sub3(wA, m3MulMV3(c->invIA, delta));
            wB = m3Add3(wB, m3MulMV3(c->invIB, delta));
        }

        // The shared point constraint (solver.c:2656-2701).
        m3Vec3 cdot = m3Sub3(m3Add3(vB, m3Cross3(wB, rB)), m3Add3(vA, m3Cross3(wA, rA)));
        m3Vec3 bias = v3(0.0f, 0.0f, 0.0f);
        m3real massScale = 1.0f;
        m3real impulseScale = 0.0f;
        if (useBias)
        {
            m3Vec3 separation =
                m3Add3(m3Add3(m3Sub3(deltaPos[c->bodyB], deltaPos[c->bodyA]), m3Sub3(rB, rA)),
                       c->deltaCenter);
            bias = m3MulSV3(c->softness.biasRate, separation);
            massScale = c->softness.massScale;
            impulseScale = c->softness.impulseScale;
        }
        m3Mat3 k;
        m3Vec3* cols[3] = {&k.cx, &k.cy, &k.cz};
        for (int32_t a = 0; a < 3; ++a)
        {
            m3Vec3 e = v3(a == 0 ? 1.0f : 0.0f, a == 1 ? 1.0f : 0.0f, a == 2 ? 1.0f : 0.0f);
            m3Vec3 tA = m3Cross3(rA, m3MulMV3(c->invIA, m3Cross3(rA, e)));
            m3Vec3 tB = m3Cross3(rB, m3MulMV3(c->invIB, m3Cross3(rB, e)));
            *cols[a] = m3Sub3(m3MulSV3(c->invMassA + c->invMassB, e), m3Add3(tA, tB));
        }
        m3Vec3 b = m3Solve3(&k, m3Add3(cdot, bias));
        m3Vec3 impulse = m3Sub3(m3MulSV3(-massScale, b), m3MulSV3(impulseScale, c->impulse));
        c->impulse = m3Add3(c->impulse, impulse);
        w.v[c->bodyA] = m3Sub3(vA, m3MulSV3(c->invMassA, impulse));
        w.w[c->bodyA] = m3Sub3(wA, m3MulMV3(c->invIA, m3Cross3(rA, impulse)));
        w.v[c->bodyB] = m3Add3(vB, m3MulSV3(c->invMassB, impulse));
        w.w[c->bodyB] = m3Add3(wB, m3MulMV3(c->invIB, m3Cross3(rB, impulse)));
    }
}

// One joint's store (solver.c:2704-2730 loop body).
__device__ void m3StoreJoint(const m3WorldView& w, const m3JointDev* c)
{
    {
        w.jimpulse[c->joint] = c->impulse;
        w.jperp[c->joint] = v3(c->perpImpulseX, c->perpImpulseY, c->motorImpulse);
        w.jlimitImp[c->joint] = v3(c->lowerImpulse, c->upperImpulse, 0.0f);
        w.jangular[c->joint] = c->angularImpulse;
        w.jspringImp[c->joint] = c->springImpulseV;
    }
}

// Reaction magnitudes of a stored joint for the device joint types
// (joint.c:635-711): revolute -- the cross-axis locks, motor and limits
// as torque; spherical -- its twist/swing rows; fixed -- the weld's
// angular impulse; the point impulse as force.  Both scaled by invH.
__device__ __forceinline__ void m3JointReactionDev(const m3WorldView& w, int32_t j, m3real invH,
                                                   m3real* outForce, m3real* outTorque)
{
    const m3Vec3 lin = w.jimpulse[j];
    const m3Vec3 perp = w.jperp[j];
    const m3Vec3 lim = w.jlimitImp[j];
    const m3Vec3 ang = w.jangular[j];
    const m3real force = m3Length3(lin);
    m3real torque;
    if (w.jtype[j] == 1)
    {
        torque = sqrtf(perp.x * perp.x + perp.y * perp.y) + fabsf(perp.z) + fabsf(lim.x) +
                 fabsf(lim.y);
    }
    else if (w.jtype[j] == 0)
    {
        torque = fabsf(lim.x) + fabsf(lim.y) + fabsf(lim.z);
    }
    else
    {
        torque = m3Length3(ang);
    }
    *outForce = force * invH;
    *outTorque = torque * invH;
}

// Removes joint j from one body's joint list (joint.c:324-337).
__device__ __forceinline__ void m3UnlinkJointDev(const m3WorldView& w, int32_t body, int32_t j)
{
    int32_t* cursor = &w.jointHead[body];
    while (*cursor != -1)
    {
        const int32_t k = *cursor;
        if (k == j)
        {
            *cursor = w.jbodyA[k] == body ? w.jnextA[k] : w.jnextB[k];
            return;
        }
        cursor = w.jbodyA[k] == body ? &w.jnextA[k] : &w.jnextB[k];
    }
}

// Joint breakage after the impulse store (solver.c:4228-4257): serially
// in ascending joint order, a joint whose reaction exceeds a set
// threshold is destroyed (joint.c:339-385): unlinked from both bodies,
// which wake, its record reset, its slot freed (generation bumped unless
// retired at 0xFFFF) and queued for the host's free list.
// Whether joint j breaks at the end of this step: alive, breakable and
// its reaction above a threshold (solver.c:4233-4245).  Independent of
// every other joint's fate: the reaction reads only j's own impulses.
__device__ bool m3JointBreaksDev(const m3WorldView& w, int32_t j, m3real invH)
{
    if (w.jointAlive[j] == 0)
    {
        return false;
    }
    const m3real maxForce = w.jbreak[j].x;
    const m3real maxTorque = w.jbreak[j].y;
    if (maxForce == 0.0f && maxTorque == 0.0f)
    {
        return false;
    }
    m3real force;
    m3real torque;
    m3JointReactionDev(w, j, invH, &force, &torque);
    return (maxForce > 0.0f && force > maxForce) || (maxTorque > 0.0f && torque > maxTorque);
}

// Destroys broken joint j (m3DestroyJointInternal, joint.c:339-385):
// unlinks it, wakes its bodies, clears its record and queues the slot.
// Order dependent (the body joint lists, the slot queue): ascending j.
__device__ void m3DestroyBrokenJointDev(const m3WorldView& w, int32_t j)
{
    m3WorldScalars* sc = w.sc;
    const int32_t bodyA = w.jbodyA[j];
    const int32_t bodyB = w.jbodyB[j];
    m3UnlinkJointDev(w, bodyA, j);
    m3UnlinkJointDev(w, bodyB, j);
    if (w.btype[bodyA] == M3_BODY_DYNAMIC && w.bodyAlive[bodyA] != 0)
    {
        w.awake[bodyA] = 1;
        w.sleepTime[bodyA] = 0.0f;
    }
    if (w.btype[bodyB] == M3_BODY_DYNAMIC && w.bodyAlive[bodyB] != 0)
    {
        w.awake[bodyB] = 1;
        w.sleepTime[bodyB] = 0.0f;
    }
    const m3Vec3 zero = v3(0.0f, 0.0f, 0.0f);
    w.jtype[j] = 0;
    w.jbodyA[j] = -1;
    w.jbodyB[j] = -1;
    w.jlocalA[j] = zero;
    w.jlocalB[j] = zero;
    w.jcollide[j] = 0;
    w.jimpulse[j] = zero;
    w.jperp[j] = zero;
    w.jlimitImp[j] = zero;
    w.jangular[j] = zero;
    w.jframeA[j] = m3IdentityQuat();
    w.jframeB[j] = m3IdentityQuat();
    w.jflags[j] = 0;
    w.jmotor[j] = zero;
    w.jbreak[j] = zero;
    w.jspring[j] = zero;
    w.jtargetScalar[j] = 0.0f;
    w.jtargetQ[j] = m3IdentityQuat();
    w.jspringImp[j] = zero;
    w.jlimits[j] = zero;
    w.jnextA[j] = -1;
    w.jnextB[j] = -1;
    w.jointAlive[j] = 0;
    // The host's free queue learns of the slot through the ring:
    // j when freed, -1 - j when retired at generation 0xFFFF.
    int32_t entry = -1 - j;
    if (w.jointGen[j] != 0xFFFF)
    {
        w.jointGen[j] = (uint16_t)(w.jointGen[j] + 1);
        entry = j;
    }
    w.jbroken[sc->brokenCount % sc->jointCap] = entry;
    sc->brokenCount += 1;
}

// Joint breakage of one world on one thread (solver.c:4233-4257):
// reactions against thresholds, broken joints destroyed in ascending
// order.
__device__ void m3BreakJointsDev(const m3WorldView& w, m3real invH)
{
    const int32_t jointMax = w.sc->jointMax;
    for (int32_t j = 0; j < jointMax; ++j)
    {
        if (m3JointBreaksDev(w, j, invH))
        {
            m3DestroyBrokenJointDev(w, j);
        }
    }
}

#endif // M3_JOINTS_CUH
