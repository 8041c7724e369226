// Body commands between steps: forces, torques, impulses and velocity
// sets (body.c:335-418).  One definition serves the host API, the
// journal replay and the device command kernel of the serving path, so
// a command lands on the same bits wherever it is applied.
#ifndef M3_OPS_H
#define M3_OPS_H

#include "m3_layout.h"

// Journal op codes of the commands this path applies (the reference's
// m3JournalOp numbering, world_internal.h:108-147).
enum
{
    M3_OP_STEP = 1,
    M3_OP_SET_LINEAR_VELOCITY = 4,
    M3_OP_SET_ANGULAR_VELOCITY = 5,
    M3_OP_APPLY_FORCE = 26,
    M3_OP_APPLY_TORQUE = 27,
    M3_OP_APPLY_LINEAR_IMPULSE = 28,
    M3_OP_APPLY_ANGULAR_IMPULSE = 29,
    M3_OP_JOINT_SET_BREAK = 55,
    // World settings (world_internal.h:146-175).
    M3_OP_SET_GRAVITY = 39,
    M3_OP_SET_CONTACT_TUNING = 44,
    M3_OP_SET_RESTITUTION_THRESHOLD = 45,
    M3_OP_SET_MAXIMUM_LINEAR_SPEED = 46,
    M3_OP_ENABLE_SLEEPING = 47,
    M3_OP_ENABLE_CONTINUOUS = 48,
    M3_OP_SET_HIT_EVENT_THRESHOLD = 49,
    M3_OP_SET_WIND = 60,
    M3_OP_SET_MAXIMUM_ANGULAR_SPEED = 66,
    // Host-side body commands (world_internal.h:137-174).
    M3_OP_APPLY_FORCE_AT_POINT = 30,
    M3_OP_APPLY_IMPULSE_AT_POINT = 31,
    M3_OP_SET_TRANSFORM = 32,
    M3_OP_SET_TARGET_TRANSFORM = 33,
    M3_OP_SET_TYPE = 34,
    M3_OP_SET_ENABLED = 35,
    M3_OP_SET_MOTION_LOCKS = 36,
    M3_OP_SET_SLEEP_CONTROLS = 37,
    M3_OP_SET_AWAKE = 38,
    M3_OP_SET_ALLOW_FAST_ROTATION = 65,
    M3_OP_SET_BODY_NAME = 68,
    // Shape materials and flags (world_internal.h:146-149, 156-157).
    M3_OP_SET_SHAPE_FRICTION = 40,
    M3_OP_SET_SHAPE_RESTITUTION = 41,
    M3_OP_SET_SHAPE_ROLLING = 42,
    M3_OP_SET_SHAPE_DENSITY = 43,
    M3_OP_ENABLE_SHAPE_HIT_EVENTS = 50,
    M3_OP_ENABLE_SHAPE_PRESOLVE = 51,
    // Joint drives and switches (world_internal.h:158-163).
    M3_OP_JOINT_SET_LIMITS = 52,
    M3_OP_JOINT_SET_MOTOR = 53,
    M3_OP_JOINT_SET_COLLIDE = 54,
    M3_OP_JOINT_SET_SPRING = 56,
    M3_OP_JOINT_SET_TARGET = 57,
};

// One command for the device kernel: `world` indexes the batch, `body`
// the world's body slot.
typedef struct m3BodyOp
{
    int32_t world;
    int32_t op;
    int32_t body;
    m3Vec3 v;
} m3BodyOp;

// World settings: host-side records of the journal (never device ops).
M3_HD bool m3IsWorldSettingOp(int32_t op)
{
    return op == M3_OP_SET_GRAVITY || op == M3_OP_SET_CONTACT_TUNING ||
           op == M3_OP_SET_RESTITUTION_THRESHOLD || op == M3_OP_SET_MAXIMUM_LINEAR_SPEED ||
           op == M3_OP_ENABLE_SLEEPING || op == M3_OP_ENABLE_CONTINUOUS ||
           op == M3_OP_SET_HIT_EVENT_THRESHOLD || op == M3_OP_SET_WIND ||
           op == M3_OP_SET_MAXIMUM_ANGULAR_SPEED;
}

// Body commands applied on the host image only (a world point, a pose,
// lock bits, a type or a flag ride their records): never device ops.
M3_HD bool m3IsHostBodyOp(int32_t op)
{
    return (op >= M3_OP_APPLY_FORCE_AT_POINT && op <= M3_OP_SET_AWAKE) ||
           op == M3_OP_SET_ALLOW_FAST_ROTATION || op == M3_OP_SET_BODY_NAME;
}

// Shape commands applied on the host image only: never device ops.
M3_HD bool m3IsHostShapeOp(int32_t op)
{
    return (op >= M3_OP_SET_SHAPE_FRICTION && op <= M3_OP_SET_SHAPE_DENSITY) ||
           op == M3_OP_ENABLE_SHAPE_HIT_EVENTS || op == M3_OP_ENABLE_SHAPE_PRESOLVE;
}

// Joint commands applied on the host image only: never device ops.
M3_HD bool m3IsHostJointOp(int32_t op)
{
    return (op >= M3_OP_JOINT_SET_LIMITS && op <= M3_OP_JOINT_SET_COLLIDE) ||
           op == M3_OP_JOINT_SET_SPRING || op == M3_OP_JOINT_SET_TARGET;
}

// Joint commands ride the same record: `body` is then the joint slot.
M3_HD bool m3IsJointOp(int32_t op)
{
    return op == M3_OP_JOINT_SET_BREAK;
}

M3_HD bool m3IsBodyOp(int32_t op)
{
    return op == M3_OP_SET_LINEAR_VELOCITY || op == M3_OP_SET_ANGULAR_VELOCITY ||
           op == M3_OP_APPLY_FORCE || op == M3_OP_APPLY_TORQUE ||
           op == M3_OP_APPLY_LINEAR_IMPULSE || op == M3_OP_APPLY_ANGULAR_IMPULSE;
}

// World-space inverse inertia R Il^-1 R^T, column by column
// (solver.c:141-154).
M3_HD m3Mat3 m3WorldInvInertiaHD(const m3WorldView& w, int32_t body)
{
    if (w.btype[body] != M3_BODY_DYNAMIC)
    {
        return m3ZeroMat3();
    }
    const m3Quat q = w.xf[body].q;
    const m3Mat3 il = w.invI[body];
    m3Mat3 r;
    r.cx = m3RotateVec3(q, m3MulMV3(il, m3InvRotateVec3(q, v3(1.0f, 0.0f, 0.0f))));
    r.cy = m3RotateVec3(q, m3MulMV3(il, m3InvRotateVec3(q, v3(0.0f, 1.0f, 0.0f))));
    r.cz = m3RotateVec3(q, m3MulMV3(il, m3InvRotateVec3(q, v3(0.0f, 0.0f, 1.0f))));
    return r;
}

// A nonzero command wakes the body (body.c:342-349).
M3_HD void m3WakeOnCommand(const m3WorldView& w, int32_t body, m3Vec3 a)
{
    if (a.x != 0.0f || a.y != 0.0f || a.z != 0.0f)
    {
        w.awake[body] = 1;
        w.sleepTime[body] = 0.0f;
    }
}

// Applies one command to a live body slot (body.c:351-418).  The
// caller has validated the slot and the vector (and, for the public
// force and impulse entry points, that the body is dynamic with mass).
M3_HD void m3ApplyBodyOp(const m3WorldView& w, int32_t op, int32_t body, m3Vec3 v)
{
    switch (op)
    {
    case M3_OP_SET_LINEAR_VELOCITY:
        w.awake[body] = 1;
        w.sleepTime[body] = 0.0f;
        w.v[body] = v;
        break;
    case M3_OP_SET_ANGULAR_VELOCITY:
        w.awake[body] = 1;
        w.sleepTime[body] = 0.0f;
        w.w[body] = v;
        break;
    case M3_OP_APPLY_FORCE:
        w.force[body] = m3Add3(w.force[body], v);
        m3WakeOnCommand(w, body, v);
        break;
    case M3_OP_APPLY_TORQUE:
        w.torque[body] = m3Add3(w.torque[body], v);
        m3WakeOnCommand(w, body, v);
        break;
    case M3_OP_APPLY_LINEAR_IMPULSE:
        w.v[body] = m3Add3(w.v[body], m3MulSV3(w.invMass[body], v));
        m3WakeOnCommand(w, body, v);
        break;
    case M3_OP_APPLY_ANGULAR_IMPULSE:
        w.w[body] = m3Add3(w.w[body], m3MulMV3(m3WorldInvInertiaHD(w, body), v));
        m3WakeOnCommand(w, body, v);
        break;
    case M3_OP_JOINT_SET_BREAK:
    {
        // joint.c:626-630, 548-560: thresholds (maxForce, maxTorque), then
        // the joint's dynamic bodies wake.
        const int32_t j = body;
        w.jbreak[j] = v3(v.x, v.y, 0.0f);
        const int32_t ends[2] = {w.jbodyA[j], w.jbodyB[j]};
        for (int32_t k = 0; k < 2; ++k)
        {
            if (ends[k] >= 0 && w.btype[ends[k]] == M3_BODY_DYNAMIC)
            {
                w.awake[ends[k]] = 1;
                w.sleepTime[ends[k]] = 0.0f;
            }
        }
        break;
    }
    default:
        break;
    }
}

#endif // M3_OPS_H
