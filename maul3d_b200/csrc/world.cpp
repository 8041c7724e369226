// World creation and the host-side mirror of the reference's creation
// API: worlds, bodies, shapes (sphere, plane, capsule, box hull) and
// joints (spherical, revolute, fixed), with the same validation, the
// same slot allocation, the same hull interning and the same mass
// properties, so a world built here hashes bit-identically to one built
// by the reference from the same calls.  All of this is create-time
// host work; the per-step path is in step.cu.
//
// Reference counterparts: src/world.c:64-460 (world def and create),
// src/body.c:35-103 (body def and create), src/shape.c:31-300 and
// :411-620, :717-830, :1334 (shape defs, mass, create), src/hull.c
// (box hull and half edges, interning), src/joint.c:15-330 (joint def,
// frames, create).

#include "m3_world.h"
#include "m3_ops.h"
#include "m3_tree.h"
#include "m3_hash.h"

#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

// ---------------------------------------------------------------------
// Cookies: a def must come from its m3Default*Def factory
// (world_internal.h:88-93, joint.c:13).  The struct sizes equal the
// reference's, so the cookie values do too.
// ---------------------------------------------------------------------
#define M3_COOKIE 0x4D33u
#define M3_WORLD_COOKIE ((int32_t)(M3_COOKIE ^ ((int32_t)sizeof(m3WorldDef) << 8)))
#define M3_BODY_COOKIE ((int32_t)(M3_COOKIE ^ ((int32_t)sizeof(m3BodyDef) << 8) ^ 1))
#define M3_SHAPE_COOKIE ((int32_t)(M3_COOKIE ^ ((int32_t)sizeof(m3ShapeDef) << 8) ^ 2))
#define M3_JOINT_COOKIE ((int32_t)(M3_COOKIE ^ ((int32_t)sizeof(m3JointDef) << 8) ^ 3))

static_assert(sizeof(m3WorldDef) == 112, "m3WorldDef must match the reference layout");
static_assert(sizeof(m3BodyDef) == 104, "m3BodyDef must match the reference layout");
static_assert(sizeof(m3ShapeDef) == 88, "m3ShapeDef must match the reference layout");
static_assert(sizeof(m3JointDef) == 224, "m3JointDef must match the reference layout");

// Worlds this library can hold at once (ids carry the slot in 16 bits).
#define M3GPU_MAX_WORLDS 65535

static std::vector<m3HostWorld*> s_worlds;
static std::vector<uint16_t> s_worldGenerations;

static bool FiniteF(float x)
{
    return isfinite(x) != 0;
}
static bool FiniteV3(m3Vec3 v)
{
    return FiniteF(v.x) && FiniteF(v.y) && FiniteF(v.z);
}
static bool FiniteQuat(m3Quat q)
{
    return FiniteF(q.x) && FiniteF(q.y) && FiniteF(q.z) && FiniteF(q.w);
}
static bool FinitePos3(m3Pos3 p)
{
    return isfinite(p.x) && isfinite(p.y) && isfinite(p.z);
}

m3HostWorld* m3gpuWorldFromIndex0(uint16_t index0)
{
    return index0 < s_worlds.size() ? s_worlds[index0] : nullptr;
}

m3HostWorld* m3gpuWorldFromId(m3WorldId id)
{
    int32_t slot = id.index1 - 1;
    if (slot < 0 || slot >= (int32_t)s_worlds.size() || s_worlds[slot] == nullptr ||
        s_worlds[slot]->generation != id.generation)
    {
        return nullptr;
    }
    return s_worlds[slot];
}

// ---------------------------------------------------------------------
// Worlds
// ---------------------------------------------------------------------
extern "C" m3WorldDef m3DefaultWorldDef(void)
{
    m3WorldDef def;
    memset(&def, 0, sizeof(def));
    def.gravity = v3(0.0f, -10.0f, 0.0f);
    def.bodyCapacity = 1024;
    def.shapeCapacity = 2048;
    def.meshCapacity = 4;
    def.jointCapacity = 64;
    def.voxelCapacity = 4;
    def.characterCapacity = 4;
    def.vehicleCapacity = 2;
    def.softBodyCapacity = 2;
    def.workerCount = 1;
    def.contactHertz = M3_CONTACT_HERTZ_DEFAULT;
    def.contactDampingRatio = M3_CONTACT_DAMPING_RATIO_DEFAULT;
    def.contactPushMaxSpeed = M3_CONTACT_PUSH_MAX_SPEED_DEFAULT;
    def.restitutionThreshold = M3_RESTITUTION_THRESHOLD_DEFAULT;
    def.maximumLinearSpeed = M3_MAX_LINEAR_SPEED_DEFAULT;
    def.enableSleeping = 1;
    def.enableContinuous = 1;
    def.hitEventThreshold = M3_HIT_EVENT_THRESHOLD_DEFAULT;
    def.internalValue = M3_WORLD_COOKIE;
    return def;
}

// Creation without the world table (world.c:64-460): validation, the
// image and its initial arrays.  It touches only the new world and the
// host memory arena, so it may run on any thread.
m3HostWorld* m3gpuNewWorld(const m3WorldDef* def)
{
    if (def == nullptr || def->internalValue != M3_WORLD_COOKIE || def->bodyCapacity <= 0 ||
        def->shapeCapacity <= 0 || def->meshCapacity <= 0 || def->jointCapacity <= 0 ||
        def->voxelCapacity <= 0 || def->characterCapacity <= 0 || def->vehicleCapacity <= 0 ||
        def->softBodyCapacity <= 0 || def->workerCount <= 0 ||
        (def->enqueueTask == nullptr) != (def->finishTask == nullptr) ||
        !FiniteV3(def->gravity) || !FiniteF(def->contactHertz) || def->contactHertz <= 0.0f ||
        !FiniteF(def->contactDampingRatio) || def->contactDampingRatio <= 0.0f ||
        !FiniteF(def->contactPushMaxSpeed) || def->contactPushMaxSpeed <= 0.0f ||
        !FiniteF(def->restitutionThreshold) || def->restitutionThreshold < 0.0f ||
        !FiniteF(def->maximumLinearSpeed) || def->maximumLinearSpeed <= 0.0f ||
        !FiniteF(def->hitEventThreshold) || def->hitEventThreshold < 0.0f)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateWorld: invalid world def");
        return nullptr;
    }
    m3HostWorld* w = new m3HostWorld();
    w->slot = -1;
    w->bodyCap = def->bodyCapacity;
    w->shapeCap = def->shapeCapacity;
    w->jointCap = def->jointCapacity;
    w->pairCap = 8 * def->shapeCapacity; // world.c:429
    w->meshCap = def->meshCapacity;
    w->voxelCap = def->voxelCapacity;
    w->charCap = def->characterCapacity;
    w->vehicleCap = def->vehicleCapacity;
    w->softCap = def->softBodyCapacity;
    w->bodyFree.Init(w->bodyCap);
    w->shapeFree.Init(w->shapeCap);
    w->hullFree.Init(w->shapeCap);
    w->hullGen.assign((size_t)w->shapeCap, 0);
    w->bodyNames.assign((size_t)w->bodyCap * M3_BODY_NAME_BYTES, 0);
    w->jointFree.Init(w->jointCap);
    w->persistentBytes =
        m3LayoutPersistent(nullptr, nullptr, w->bodyCap, w->shapeCap, w->jointCap, w->pairCap);
    w->image.resize((size_t)w->persistentBytes);
    memset(w->image.data(), 0, (size_t)w->persistentBytes);
    m3LayoutPersistent(&w->hv, w->image.data(), w->bodyCap, w->shapeCap, w->jointCap, w->pairCap);
    w->hv.hulls = nullptr;
    w->hv.scratch = nullptr;
    w->hv.scratchBytes = 0;

    m3WorldScalars* sc = w->hv.sc;
    sc->gravity = def->gravity;
    sc->contactHertz = def->contactHertz;
    sc->contactDampingRatio = def->contactDampingRatio;
    sc->contactPushMaxSpeed = def->contactPushMaxSpeed;
    sc->restitutionThreshold = def->restitutionThreshold;
    sc->maximumLinearSpeed = def->maximumLinearSpeed;
    sc->maximumAngularSpeed = M3_MAX_ANGULAR_SPEED_DEFAULT;
    sc->sleepEnabled = def->enableSleeping != 0 ? 1 : 0;
    sc->continuousEnabled = def->enableContinuous != 0 ? 1 : 0;
    sc->hitEventThreshold = def->hitEventThreshold;
    sc->bodyCap = w->bodyCap;
    sc->shapeCap = w->shapeCap;
    sc->jointCap = w->jointCap;
    sc->pairCap = w->pairCap;
    sc->treeTracked = 1;

    // Array initial values of the reference's create (world.c:160-440):
    // empty list heads and unset slots read -1; joint targets identity.
    for (int32_t i = 0; i < w->bodyCap; ++i)
    {
        w->hv.shapeHead[i] = -1;
        w->hv.jointHead[i] = -1;
    }
    m3TreeInit(m3WorldTree(w->hv));
    for (int32_t i = 0; i < w->shapeCap; ++i)
    {
        w->hv.proxyId[i] = M3_TREE_NULL;
        w->hv.shapeNext[i] = -1;
        w->hv.hullIndex[i] = -1;
        w->hv.hfIndex[i] = -1;
        w->hv.shapeBody[i] = -1;
    }
    for (int32_t i = 0; i < w->jointCap; ++i)
    {
        w->hv.jbodyA[i] = -1;
        w->hv.jbodyB[i] = -1;
        w->hv.jnextA[i] = -1;
        w->hv.jnextB[i] = -1;
    }
    return w;
}

// Enters a world built by m3gpuNewWorld into the world table; when the
// table is full the world is deleted and the null id returned.
m3WorldId m3gpuAttachWorld(m3HostWorld* w)
{
    m3WorldId nullId = {0, 0};
    int32_t slot = -1;
    for (int32_t i = 0; i < (int32_t)s_worlds.size(); ++i)
    {
        if (s_worlds[i] == nullptr)
        {
            slot = i;
            break;
        }
    }
    if (slot < 0)
    {
        if ((int32_t)s_worlds.size() >= M3GPU_MAX_WORLDS)
        {
            delete w;
            m3gpuSetError(M3GPU_ERR_CAPACITY, "m3CreateWorld: world table full");
            return nullId;
        }
        slot = (int32_t)s_worlds.size();
        s_worlds.push_back(nullptr);
        s_worldGenerations.push_back(0);
    }
    w->slot = slot;
    w->generation = s_worldGenerations[slot];
    s_worlds[slot] = w;
    m3WorldId id = {slot + 1, w->generation};
    return id;
}

// A world of m3gpuNewWorld that never entered the table (never resident).
void m3gpuDeleteWorld(m3HostWorld* w)
{
    delete w;
}

extern "C" m3WorldId m3CreateWorld(const m3WorldDef* def)
{
    m3WorldId nullId = {0, 0};
    m3gpuClearError();
    m3HostWorld* w = m3gpuNewWorld(def);
    if (w == nullptr)
    {
        return nullId;
    }
    return m3gpuAttachWorld(w);
}

extern "C" void m3DestroyWorld(m3WorldId worldId)
{
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr)
    {
        return;
    }
    m3gpuRelease(w);
    s_worlds[w->slot] = nullptr;
    s_worldGenerations[w->slot] = (uint16_t)(s_worldGenerations[w->slot] + 1);
    delete w;
}

extern "C" bool m3World_IsValid(m3WorldId worldId)
{
    return m3gpuWorldFromId(worldId) != nullptr;
}

// ---------------------------------------------------------------------
// Bodies (body.c:35-103)
// ---------------------------------------------------------------------
extern "C" m3BodyDef m3DefaultBodyDef(void)
{
    m3BodyDef def;
    memset(&def, 0, sizeof(def));
    def.type = m3_staticBody;
    def.rotation = m3IdentityQuat();
    def.gravityScale = 1.0f;
    def.internalValue = M3_BODY_COOKIE;
    return def;
}

static int32_t BodySlot(const m3HostWorld* w, m3BodyId id)
{
    int32_t index = id.index1 - 1;
    if (w == nullptr || id.world0 != (uint16_t)w->slot || index < 0 ||
        index >= w->hv.sc->bodyMax || w->hv.bodyAlive[index] == 0 ||
        w->hv.bodyGen[index] != id.generation)
    {
        return -1;
    }
    return index;
}

static m3HostWorld* ResolveBody(m3BodyId id, int32_t* index)
{
    m3HostWorld* w = m3gpuWorldFromIndex0(id.world0);
    *index = w != nullptr ? BodySlot(w, id) : -1;
    return *index >= 0 ? w : nullptr;
}

extern "C" m3BodyId m3CreateBody(m3WorldId worldId, const m3BodyDef* def)
{
    m3BodyId nullId = {0, 0, 0};
    m3gpuClearError();
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr || def == nullptr || def->internalValue != M3_BODY_COOKIE)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateBody: stale world or invalid def");
        return nullId;
    }
    m3real qq = def->rotation.x * def->rotation.x + def->rotation.y * def->rotation.y +
                def->rotation.z * def->rotation.z + def->rotation.w * def->rotation.w;
    if ((def->type != m3_staticBody && def->type != m3_kinematicBody &&
         def->type != m3_dynamicBody) ||
        !FinitePos3(def->position) || !FiniteQuat(def->rotation) ||
        !FiniteV3(def->linearVelocity) || !FiniteV3(def->angularVelocity) ||
        !FiniteF(def->gravityScale) || !FiniteF(def->linearDamping) ||
        !FiniteF(def->angularDamping) || def->linearDamping < 0.0f ||
        def->angularDamping < 0.0f || !(qq > 0.98f) || !(qq < 1.02f))
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateBody: invalid body def");
        return nullId;
    }
    if (m3gpuSyncHost(w) != M3GPU_OK)
    {
        return nullId;
    }
    m3WorldView& v = w->hv;
    // Recycled slots first, then a fresh one (allocator.c:178-198).
    int32_t i = -1;
    if (!w->bodyFree.Pop(&i))
    {
        if (v.sc->bodyMax >= w->bodyCap)
        {
            m3gpuSetError(M3GPU_ERR_CAPACITY, "m3CreateBody: body pool exhausted");
            return nullId;
        }
        i = v.sc->bodyMax;
        v.sc->bodyMax += 1;
    }
    v.bodyAlive[i] = 1;
    v.xf[i].p = def->position;
    v.xf[i].q = m3NormalizeQuat(def->rotation);
    v.v[i] = def->linearVelocity;
    v.w[i] = def->angularVelocity;
    v.invMass[i] = def->type == m3_dynamicBody ? 1.0f : 0.0f;
    v.invI[i] = m3ZeroMat3();
    v.inertia[i] = m3ZeroMat3();
    v.awake[i] = 1;
    v.sleepTime[i] = 0.0f;
    v.minExt[i] = 1.0e30f;
    v.maxExt[i] = 0.0f;
    v.lc[i] = v3(0.0f, 0.0f, 0.0f);
    v.gravityScale[i] = def->gravityScale;
    v.linDamp[i] = def->linearDamping;
    v.angDamp[i] = def->angularDamping;
    v.btype[i] = (uint8_t)def->type;
    v.bullet[i] = def->isBullet ? 1 : 0;
    v.userData[i] = def->userData;
    v.enabled[i] = 1;
    v.locks[i] = 0;
    v.sleepThreshold[i] = M3_SLEEP_VELOCITY_DEFAULT;
    v.canSleep[i] = 1;
    v.hasTarget[i] = 0;
    v.target[i].p.x = 0.0;
    v.target[i].p.y = 0.0;
    v.target[i].p.z = 0.0;
    v.target[i].q = m3IdentityQuat();
    v.shapeHead[i] = -1;
    v.jointHead[i] = -1;
    memset(&w->bodyNames[(size_t)i * M3_BODY_NAME_BYTES], 0, M3_BODY_NAME_BYTES);
    w->hostDirty = true;
    m3JournalUnrecordable(w); // creation is not recorded by this path
    w->structure += 1;        // device snapshot slots saved before are void
    m3BodyId id = {i + 1, (uint16_t)w->slot, v.bodyGen[i]};
    return id;
}

extern "C" bool m3Body_IsValid(m3BodyId bodyId)
{
    int32_t index;
    return ResolveBody(bodyId, &index) != nullptr;
}

template <typename T, typename F> static T ReadBody(m3BodyId id, T zero, F get)
{
    int32_t index;
    m3HostWorld* w = ResolveBody(id, &index);
    if (w == nullptr || m3gpuSyncHost(w) != M3GPU_OK)
    {
        return zero;
    }
    return get(w->hv, index);
}

extern "C" m3Pos3 m3Body_GetPosition(m3BodyId bodyId)
{
    m3Pos3 zero = {0.0, 0.0, 0.0};
    return ReadBody(bodyId, zero, [](const m3WorldView& v, int32_t i) { return v.xf[i].p; });
}

extern "C" m3Quat m3Body_GetRotation(m3BodyId bodyId)
{
    return ReadBody(bodyId, m3IdentityQuat(),
                    [](const m3WorldView& v, int32_t i) { return v.xf[i].q; });
}

extern "C" m3Vec3 m3Body_GetLinearVelocity(m3BodyId bodyId)
{
    return ReadBody(bodyId, v3(0.0f, 0.0f, 0.0f),
                    [](const m3WorldView& v, int32_t i) { return v.v[i]; });
}

extern "C" m3Vec3 m3Body_GetAngularVelocity(m3BodyId bodyId)
{
    return ReadBody(bodyId, v3(0.0f, 0.0f, 0.0f),
                    [](const m3WorldView& v, int32_t i) { return v.w[i]; });
}

extern "C" bool m3Body_IsAwake(m3BodyId bodyId)
{
    return ReadBody(bodyId, false, [](const m3WorldView& v, int32_t i) {
        return v.btype[i] != M3_BODY_DYNAMIC || v.awake[i] != 0;
    });
}

// Commands between steps (body.c:818-1014): forces, torques and
// impulses reach dynamic bodies with mass only; velocity sets reach any
// live body.  A stale id or a non-finite vector is a no-op.
static void BodyCommand(m3BodyId id, int32_t op, m3Vec3 v, bool needsMass)
{
    int32_t index;
    m3HostWorld* w = ResolveBody(id, &index);
    if (w == nullptr || !FiniteV3(v) || m3gpuSyncHost(w) != M3GPU_OK)
    {
        return;
    }
    if (needsMass && !(w->hv.btype[index] == M3_BODY_DYNAMIC && w->hv.invMass[index] > 0.0f))
    {
        return;
    }
    struct
    {
        m3BodyId id;
        m3Vec3 v;
    } record = {id, v};
    m3JournalAppend(w, op, &record, (int32_t)sizeof(record));
    m3ApplyBodyOp(w->hv, op, index, v);
    w->hostDirty = true;
}

extern "C" void m3Body_ApplyForce(m3BodyId bodyId, m3Vec3 force)
{
    BodyCommand(bodyId, M3_OP_APPLY_FORCE, force, true);
}

extern "C" void m3Body_ApplyTorque(m3BodyId bodyId, m3Vec3 torque)
{
    BodyCommand(bodyId, M3_OP_APPLY_TORQUE, torque, true);
}

extern "C" void m3Body_ApplyLinearImpulse(m3BodyId bodyId, m3Vec3 impulse)
{
    BodyCommand(bodyId, M3_OP_APPLY_LINEAR_IMPULSE, impulse, true);
}

extern "C" void m3Body_ApplyAngularImpulse(m3BodyId bodyId, m3Vec3 impulse)
{
    BodyCommand(bodyId, M3_OP_APPLY_ANGULAR_IMPULSE, impulse, true);
}

extern "C" void m3Body_SetLinearVelocity(m3BodyId bodyId, m3Vec3 velocity)
{
    BodyCommand(bodyId, M3_OP_SET_LINEAR_VELOCITY, velocity, false);
}

extern "C" void m3Body_SetAngularVelocity(m3BodyId bodyId, m3Vec3 velocity)
{
    BodyCommand(bodyId, M3_OP_SET_ANGULAR_VELOCITY, velocity, false);
}

// ---------------------------------------------------------------------
// Host-side body commands and getters (body.c:170-330, 379-404, 514-823,
// 910-958): forces and impulses at a world point, teleports and kinematic
// targets, type changes, enabling, motion locks, sleep controls, forced
// sleep or wake and the fast-rotation escape.  Each public call checks as
// the reference's, records the reference's journal record and changes the
// host image (the next step uploads it); the journal replay applies the
// same records.
// ---------------------------------------------------------------------
static void RecomputeMass(m3HostWorld* w, int32_t b);

static m3Vec3 ForceArm(const m3WorldView& v, int32_t i, m3Pos3 point)
{
    const m3Transform xf = v.xf[i];
    const m3Vec3 rlc = m3RotateVec3(xf.q, v.lc[i]);
    return v3((m3real)(point.x - xf.p.x) - rlc.x, (m3real)(point.y - xf.p.y) - rlc.y,
              (m3real)(point.z - xf.p.z) - rlc.z);
}

// Wakes every sleeping dynamic body whose position, padded by its largest
// extent and the box margin, overlaps the region around body `i` (its
// position padded by its largest extent and four margins), in ascending
// slots (body.c:170-205).
static void WakeAround(m3WorldView& v, int32_t i)
{
    const double r = (double)v.maxExt[i] + 4.0 * (double)M3_AABB_MARGIN;
    const m3Pos3 c = v.xf[i].p;
    const double lo[3] = {c.x - r, c.y - r, c.z - r};
    const double hi[3] = {c.x + r, c.y + r, c.z + r};
    for (int32_t b = 0; b < v.sc->bodyMax; ++b)
    {
        if (v.bodyAlive[b] == 0 || v.btype[b] != M3_BODY_DYNAMIC || v.awake[b] != 0)
        {
            continue;
        }
        const double pad = (double)v.maxExt[b] + (double)M3_AABB_MARGIN;
        const m3Pos3 p = v.xf[b].p;
        if (p.x - pad <= hi[0] && p.x + pad >= lo[0] && p.y - pad <= hi[1] &&
            p.y + pad >= lo[1] && p.z - pad <= hi[2] && p.z + pad >= lo[2])
        {
            v.awake[b] = 1;
            v.sleepTime[b] = 0.0f;
        }
    }
}

static void Wake(m3WorldView& v, int32_t i)
{
    v.awake[i] = 1;
    v.sleepTime[i] = 0.0f;
}

void m3ApplyHostBodyOp(m3HostWorld* w, const m3JournalRecordView& r)
{
    m3WorldView& v = w->hv;
    const int32_t i = r.body;
    const uint32_t bits = r.bits;
    switch (r.op)
    {
    case M3_OP_APPLY_FORCE_AT_POINT:
        v.force[i] = m3Add3(v.force[i], r.v);
        v.torque[i] = m3Add3(v.torque[i], m3Cross3(ForceArm(v, i, r.point), r.v));
        m3WakeOnCommand(v, i, r.v);
        break;
    case M3_OP_APPLY_IMPULSE_AT_POINT:
        v.v[i] = m3Add3(v.v[i], m3MulSV3(v.invMass[i], r.v));
        v.w[i] = m3Add3(v.w[i], m3MulMV3(m3WorldInvInertiaHD(v, i),
                                         m3Cross3(ForceArm(v, i, r.point), r.v)));
        m3WakeOnCommand(v, i, r.v);
        break;
    case M3_OP_SET_TRANSFORM:
        // The vacated and the arrival neighbourhoods wake (body.c:207-218).
        WakeAround(v, i);
        v.xf[i] = m3Transform{r.point, r.rotation};
        WakeAround(v, i);
        Wake(v, i);
        break;
    case M3_OP_SET_TARGET_TRANSFORM:
        v.hasTarget[i] = 1;
        v.target[i] = m3Transform{r.point, r.rotation};
        Wake(v, i);
        break;
    case M3_OP_SET_TYPE:
    {
        // body.c:228-262: static drops its velocities; kinematic and static
        // keep zero inverse mass; dynamic rebuilds its mass from its shapes.
        const uint8_t type = (uint8_t)bits;
        if (v.btype[i] == type)
        {
            break;
        }
        WakeAround(v, i);
        v.btype[i] = type;
        if (type == M3_BODY_STATIC)
        {
            v.v[i] = v3(0.0f, 0.0f, 0.0f);
            v.w[i] = v3(0.0f, 0.0f, 0.0f);
        }
        if (type == M3_BODY_DYNAMIC)
        {
            RecomputeMass(w, i);
        }
        else
        {
            v.invMass[i] = 0.0f;
            v.invI[i] = m3ZeroMat3();
        }
        Wake(v, i);
        break;
    }
    case M3_OP_SET_ENABLED:
    {
        const uint8_t want = bits != 0 ? 1 : 0;
        if (v.enabled[i] == want)
        {
            break;
        }
        v.enabled[i] = want;
        WakeAround(v, i);
        if (want)
        {
            Wake(v, i);
        }
        break;
    }
    case M3_OP_SET_MOTION_LOCKS:
        // The fast-rotation bit is its own command's (body.c:283-303).
        v.locks[i] = (uint8_t)((v.locks[i] & M3_LOCKS_ALLOW_FAST_ROTATION) | (bits & 0x3Fu));
        if (bits & 1u)
            v.v[i].x = 0.0f;
        if (bits & 2u)
            v.v[i].y = 0.0f;
        if (bits & 4u)
            v.v[i].z = 0.0f;
        if (bits & 8u)
            v.w[i].x = 0.0f;
        if (bits & 16u)
            v.w[i].y = 0.0f;
        if (bits & 32u)
            v.w[i].z = 0.0f;
        break;
    case M3_OP_SET_SLEEP_CONTROLS:
        // body.c:305-314: a non-positive (or NaN) threshold is the default.
        v.sleepThreshold[i] = r.setting[0] > 0.0f ? r.setting[0] : M3_SLEEP_VELOCITY_DEFAULT;
        v.canSleep[i] = bits != 0 ? 1 : 0;
        if (bits == 0)
        {
            Wake(v, i);
        }
        break;
    case M3_OP_SET_AWAKE:
        // body.c:316-330.  The reference also records the frozen body's
        // pairs in its sleeping-pair buffer; that buffer is neither hashed
        // nor saved, and the device finds every pair by its own rule.
        if (bits != 0)
        {
            Wake(v, i);
        }
        else
        {
            v.awake[i] = 0;
            v.v[i] = v3(0.0f, 0.0f, 0.0f);
            v.w[i] = v3(0.0f, 0.0f, 0.0f);
        }
        break;
    case M3_OP_SET_ALLOW_FAST_ROTATION:
        v.locks[i] = bits != 0 ? (uint8_t)(v.locks[i] | M3_LOCKS_ALLOW_FAST_ROTATION)
                               : (uint8_t)(v.locks[i] & ~M3_LOCKS_ALLOW_FAST_ROTATION);
        break;
    case M3_OP_SET_BODY_NAME:
    {
        // Up to the first zero, at most 31 bytes, the rest zeroed
        // (body.c:711-724).
        char* slot = &w->bodyNames[(size_t)i * M3_BODY_NAME_BYTES];
        memset(slot, 0, M3_BODY_NAME_BYTES);
        for (int32_t k = 0; k < M3_BODY_NAME_BYTES - 1 && r.name[k] != 0; ++k)
        {
            slot[k] = r.name[k];
        }
        break;
    }
    default:
        break;
    }
}

// Journals one host body command and applies it: `payload` is the
// reference's record for `r.op`, `r` the command with the body slot.
static void HostCommand(m3HostWorld* w, const m3JournalRecordView& r, const void* payload,
                        int32_t bytes)
{
    m3JournalAppend(w, r.op, payload, bytes);
    m3ApplyHostBodyOp(w, r);
    w->hostDirty = true;
}

static m3JournalRecordView CommandView(int32_t op, int32_t index)
{
    m3JournalRecordView r;
    memset(&r, 0, sizeof(r));
    r.op = op;
    r.body = index;
    return r;
}

// A force or impulse at a world point: {m3BodyId id; m3Vec3 v; m3Pos3 p}.
static void PointCommand(m3BodyId id, int32_t op, m3Vec3 f, m3Pos3 point)
{
    m3gpuClearError();
    int32_t index;
    m3HostWorld* w = ResolveBody(id, &index);
    if (w == nullptr || !FiniteV3(f) || !FinitePos3(point) || m3gpuSyncHost(w) != M3GPU_OK)
    {
        return;
    }
    if (!(w->hv.btype[index] == M3_BODY_DYNAMIC && w->hv.invMass[index] > 0.0f))
    {
        return;
    }
    struct
    {
        m3BodyId id;
        m3Vec3 v;
        m3Pos3 p;
    } record;
    memset(&record, 0, sizeof(record));
    record.id = id;
    record.v = f;
    record.p = point;
    m3JournalRecordView r = CommandView(op, index);
    r.v = f;
    r.point = point;
    HostCommand(w, r, &record, (int32_t)sizeof(record));
}

extern "C" void m3Body_ApplyForceAtPoint(m3BodyId bodyId, m3Vec3 force, m3Pos3 point)
{
    PointCommand(bodyId, M3_OP_APPLY_FORCE_AT_POINT, force, point);
}

extern "C" void m3Body_ApplyLinearImpulseAtPoint(m3BodyId bodyId, m3Vec3 impulse, m3Pos3 point)
{
    PointCommand(bodyId, M3_OP_APPLY_IMPULSE_AT_POINT, impulse, point);
}

// A pose: {m3BodyId id; m3Transform pose}; the rotation must be finite and
// near unit length.  Targets reach kinematic bodies only (body.c:531-583).
static void PoseCommand(m3BodyId id, int32_t op, m3Pos3 position, m3Quat rotation)
{
    m3gpuClearError();
    int32_t index;
    m3HostWorld* w = ResolveBody(id, &index);
    const m3real qq = rotation.x * rotation.x + rotation.y * rotation.y +
                      rotation.z * rotation.z + rotation.w * rotation.w;
    if (w == nullptr || !FinitePos3(position) || !FiniteQuat(rotation) || !(qq > 0.98f) ||
        !(qq < 1.02f) || m3gpuSyncHost(w) != M3GPU_OK)
    {
        return;
    }
    if (op == M3_OP_SET_TARGET_TRANSFORM && w->hv.btype[index] != M3_BODY_KINEMATIC)
    {
        return;
    }
    struct
    {
        m3BodyId id;
        m3Transform pose;
    } record;
    memset(&record, 0, sizeof(record));
    record.id = id;
    record.pose = m3Transform{position, rotation};
    m3JournalRecordView r = CommandView(op, index);
    r.point = position;
    r.rotation = rotation;
    HostCommand(w, r, &record, (int32_t)sizeof(record));
}

extern "C" void m3Body_SetTransform(m3BodyId bodyId, m3Pos3 position, m3Quat rotation)
{
    PoseCommand(bodyId, M3_OP_SET_TRANSFORM, position, rotation);
}

extern "C" void m3Body_SetTargetTransform(m3BodyId bodyId, m3Pos3 position, m3Quat rotation)
{
    PoseCommand(bodyId, M3_OP_SET_TARGET_TRANSFORM, position, rotation);
}

// Lock bits, a type or a flag: {m3BodyId id; uint32 bits}.
static void BitsCommand(m3BodyId id, int32_t op, uint32_t bits)
{
    m3gpuClearError();
    int32_t index;
    m3HostWorld* w = ResolveBody(id, &index);
    if (w == nullptr || m3gpuSyncHost(w) != M3GPU_OK)
    {
        return;
    }
    if (op == M3_OP_SET_AWAKE && w->hv.btype[index] != M3_BODY_DYNAMIC)
    {
        return; // body.c:795-800: dynamic bodies only
    }
    struct
    {
        m3BodyId id;
        uint32_t bits;
    } record;
    memset(&record, 0, sizeof(record));
    record.id = id;
    record.bits = bits;
    m3JournalRecordView r = CommandView(op, index);
    r.bits = bits;
    HostCommand(w, r, &record, (int32_t)sizeof(record));
}

extern "C" void m3Body_SetType(m3BodyId bodyId, m3BodyType type)
{
    if (type != m3_staticBody && type != m3_kinematicBody && type != m3_dynamicBody)
    {
        return;
    }
    BitsCommand(bodyId, M3_OP_SET_TYPE, (uint32_t)type);
}

extern "C" void m3Body_SetEnabled(m3BodyId bodyId, bool enabled)
{
    BitsCommand(bodyId, M3_OP_SET_ENABLED, enabled ? 1u : 0u);
}

extern "C" void m3Body_SetAwake(m3BodyId bodyId, bool awake)
{
    BitsCommand(bodyId, M3_OP_SET_AWAKE, awake ? 1u : 0u);
}

// {m3BodyId id; char name[32]}: the name truncated to 31 bytes and
// zero-filled (body.c:711-756).  Names are saved in snapshots, never hashed.
extern "C" void m3Body_SetName(m3BodyId bodyId, const char* name)
{
    m3gpuClearError();
    int32_t index;
    m3HostWorld* w = ResolveBody(bodyId, &index);
    if (w == nullptr || m3gpuSyncHost(w) != M3GPU_OK)
    {
        return;
    }
    struct
    {
        m3BodyId id;
        char name[M3_BODY_NAME_BYTES];
    } record;
    memset(&record, 0, sizeof(record));
    record.id = bodyId;
    for (int32_t k = 0; name != nullptr && k < M3_BODY_NAME_BYTES - 1 && name[k] != 0; ++k)
    {
        record.name[k] = name[k];
    }
    m3JournalRecordView r = CommandView(M3_OP_SET_BODY_NAME, index);
    memcpy(r.name, record.name, M3_BODY_NAME_BYTES);
    m3JournalAppend(w, M3_OP_SET_BODY_NAME, &record, (int32_t)sizeof(record));
    m3ApplyHostBodyOp(w, r);
}

// The body's name, "" for a stale id; valid until the name changes or the
// world goes.
extern "C" const char* m3Body_GetName(m3BodyId bodyId)
{
    int32_t index;
    m3HostWorld* w = ResolveBody(bodyId, &index);
    if (w == nullptr)
    {
        return "";
    }
    return &w->bodyNames[(size_t)index * M3_BODY_NAME_BYTES];
}

// {m3BodyId id; float threshold; int32 canSleep}; a negative or
// non-finite threshold is refused (body.c:763-786).
extern "C" void m3Body_SetSleepControls(m3BodyId bodyId, float threshold, bool canSleep)
{
    m3gpuClearError();
    int32_t index;
    m3HostWorld* w = ResolveBody(bodyId, &index);
    if (w == nullptr || !isfinite(threshold) || threshold < 0.0f ||
        m3gpuSyncHost(w) != M3GPU_OK)
    {
        return;
    }
    struct
    {
        m3BodyId id;
        float threshold;
        int32_t canSleep;
    } record;
    memset(&record, 0, sizeof(record));
    record.id = bodyId;
    record.threshold = threshold;
    record.canSleep = canSleep ? 1 : 0;
    m3JournalRecordView r = CommandView(M3_OP_SET_SLEEP_CONTROLS, index);
    r.setting[0] = threshold;
    r.bits = canSleep ? 1u : 0u;
    HostCommand(w, r, &record, (int32_t)sizeof(record));
}

extern "C" void m3Body_SetMotionLocks(m3BodyId bodyId, uint32_t locks)
{
    if ((locks & ~0x3Fu) != 0)
    {
        return; // only the six lock bits exist
    }
    BitsCommand(bodyId, M3_OP_SET_MOTION_LOCKS, locks);
}

extern "C" void m3Body_SetAllowFastRotation(m3BodyId bodyId, bool allow)
{
    BitsCommand(bodyId, M3_OP_SET_ALLOW_FAST_ROTATION, allow ? 1u : 0u);
}

extern "C" uint32_t m3Body_GetMotionLocks(m3BodyId bodyId)
{
    return ReadBody(bodyId, 0u, [](const m3WorldView& v, int32_t i) {
        return (uint32_t)(v.locks[i] & 0x3Fu);
    });
}

extern "C" bool m3Body_GetAllowFastRotation(m3BodyId bodyId)
{
    return ReadBody(bodyId, false, [](const m3WorldView& v, int32_t i) {
        return (v.locks[i] & M3_LOCKS_ALLOW_FAST_ROTATION) != 0;
    });
}

extern "C" m3BodyType m3Body_GetType(m3BodyId bodyId)
{
    return ReadBody(bodyId, m3_staticBody,
                    [](const m3WorldView& v, int32_t i) { return (m3BodyType)v.btype[i]; });
}

extern "C" uint64_t m3Body_GetUserData(m3BodyId bodyId)
{
    return ReadBody(bodyId, (uint64_t)0,
                    [](const m3WorldView& v, int32_t i) { return v.userData[i]; });
}

extern "C" bool m3Body_IsEnabled(m3BodyId bodyId)
{
    return ReadBody(bodyId, false,
                    [](const m3WorldView& v, int32_t i) { return v.enabled[i] != 0; });
}

// ---------------------------------------------------------------------
// Mass properties (shape.c:48-300)
// ---------------------------------------------------------------------

// Adjugate inverse of a symmetric 3x3; singular or non-positive gives
// zero (shape.c:48-71).
static m3Mat3 InvertSymmetric(m3Mat3 m)
{
    m3real a = m.cx.x;
    m3real b = m.cy.x;
    m3real c = m.cz.x;
    m3real d = m.cy.y;
    m3real e = m.cz.y;
    m3real f = m.cz.z;
    m3real co00 = d * f - e * e;
    m3real co01 = c * e - b * f;
    m3real co02 = b * e - c * d;
    m3real det = a * co00 + b * co01 + c * co02;
    if (!(det > 0.0f))
    {
        return m3ZeroMat3();
    }
    m3real inv = 1.0f / det;
    m3Mat3 r;
    r.cx = v3(co00 * inv, co01 * inv, co02 * inv);
    r.cy = v3(co01 * inv, (a * f - c * c) * inv, (b * c - a * e) * inv);
    r.cz = v3(co02 * inv, (b * c - a * e) * inv, (a * d - b * b) * inv);
    return r;
}

// Shape frame to body frame: c' = p + R c, I' = R I R^T (shape.c:79-112).
static void ComposeMassProps(const m3WorldView& v, int32_t s, m3Vec3* com, m3Mat3* inertia)
{
    if (v.hasOffset[s] == 0)
    {
        return;
    }
    m3Quat q = v.localRot[s];
    *com = m3Add3(v.localPos[s], m3RotateVec3(q, *com));
    m3Mat3 r;
    r.cx = m3RotateVec3(q, v3(1.0f, 0.0f, 0.0f));
    r.cy = m3RotateVec3(q, v3(0.0f, 1.0f, 0.0f));
    r.cz = m3RotateVec3(q, v3(0.0f, 0.0f, 1.0f));
    const m3Mat3 in = *inertia;
    m3Mat3 t;
    t.cx = v3(in.cx.x * r.cx.x + in.cy.x * r.cx.y + in.cz.x * r.cx.z,
              in.cx.y * r.cx.x + in.cy.y * r.cx.y + in.cz.y * r.cx.z,
              in.cx.z * r.cx.x + in.cy.z * r.cx.y + in.cz.z * r.cx.z);
    t.cy = v3(in.cx.x * r.cy.x + in.cy.x * r.cy.y + in.cz.x * r.cy.z,
              in.cx.y * r.cy.x + in.cy.y * r.cy.y + in.cz.y * r.cy.z,
              in.cx.z * r.cy.x + in.cy.z * r.cy.y + in.cz.z * r.cy.z);
    t.cz = v3(in.cx.x * r.cz.x + in.cy.x * r.cz.y + in.cz.x * r.cz.z,
              in.cx.y * r.cz.x + in.cy.y * r.cz.y + in.cz.y * r.cz.z,
              in.cx.z * r.cz.x + in.cy.z * r.cz.y + in.cz.z * r.cz.z);
    inertia->cx = v3(r.cx.x * t.cx.x + r.cy.x * t.cx.y + r.cz.x * t.cx.z,
                     r.cx.y * t.cx.x + r.cy.y * t.cx.y + r.cz.y * t.cx.z,
                     r.cx.z * t.cx.x + r.cy.z * t.cx.y + r.cz.z * t.cx.z);
    inertia->cy = v3(r.cx.x * t.cy.x + r.cy.x * t.cy.y + r.cz.x * t.cy.z,
                     r.cx.y * t.cy.x + r.cy.y * t.cy.y + r.cz.y * t.cy.z,
                     r.cx.z * t.cy.x + r.cy.z * t.cy.y + r.cz.z * t.cy.z);
    inertia->cz = v3(r.cx.x * t.cz.x + r.cy.x * t.cz.y + r.cz.x * t.cz.z,
                     r.cx.y * t.cz.x + r.cy.y * t.cz.y + r.cz.y * t.cz.z,
                     r.cx.z * t.cz.x + r.cy.z * t.cz.y + r.cz.z * t.cz.z);
}

// Density-scaled mass, centroid and centroid inertia of one shape;
// planes carry none (shape.c:114-180).
static int ShapeMassProps(const m3HostWorld* w, int32_t s, float* massOut, m3Vec3* comOut,
                          m3Mat3* inertiaOut)
{
    const m3WorldView& v = w->hv;
    uint8_t type = v.shapeType[s];
    if (type == M3_SHAPE_SPHERE)
    {
        float r = v.geom[s].s;
        float m = v.density[s] * (4.0f / 3.0f) * M3_PI * r * r * r;
        float ic = 0.4f * m * r * r;
        *massOut = m;
        *comOut = v.geom[s].v;
        *inertiaOut = m3ZeroMat3();
        inertiaOut->cx.x = ic;
        inertiaOut->cy.y = ic;
        inertiaOut->cz.z = ic;
        return 1;
    }
    if (type == M3_SHAPE_CAPSULE)
    {
        // Cylinder plus two hemispheres about the segment midpoint:
        // I = Iperp Id + (Iaxial - Iperp) u u^T.
        m3Vec3 p1 = v.geom[s].v;
        m3Vec3 p2 = v.geom[s].v2;
        float r = v.geom[s].s;
        m3Vec3 axis = m3Sub3(p2, p1);
        float length = sqrtf(m3Dot3(axis, axis));
        m3Vec3 u = length > 0.0f ? m3MulSV3(1.0f / length, axis) : v3(1.0f, 0.0f, 0.0f);
        float density = v.density[s];
        float mCyl = density * M3_PI * r * r * length;
        float mSph = density * (4.0f / 3.0f) * M3_PI * r * r * r;
        float axial = 0.5f * mCyl * r * r + 0.4f * mSph * r * r;
        float perp = mCyl * (length * length / 12.0f + 0.25f * r * r) +
                     mSph * (0.4f * r * r + 0.25f * length * length + 0.375f * length * r);
        *massOut = mCyl + mSph;
        *comOut = m3MulSV3(0.5f, m3Add3(p1, p2));
        m3Mat3 ic2 = m3ZeroMat3();
        float d = axial - perp;
        ic2.cx = v3(perp + d * u.x * u.x, d * u.x * u.y, d * u.x * u.z);
        ic2.cy = v3(d * u.x * u.y, perp + d * u.y * u.y, d * u.y * u.z);
        ic2.cz = v3(d * u.x * u.z, d * u.y * u.z, perp + d * u.z * u.z);
        *inertiaOut = ic2;
        return 1;
    }
    if (type == M3_SHAPE_HULL)
    {
        const m3HullData* hull = &w->hulls[v.hullIndex[s]];
        float density = v.density[s];
        *massOut = density * hull->unitMass;
        *comOut = hull->unitCom;
        m3Mat3 ic = hull->unitInertiaCom;
        ic.cx = m3MulSV3(density, ic.cx);
        ic.cy = m3MulSV3(density, ic.cy);
        ic.cz = m3MulSV3(density, ic.cz);
        *inertiaOut = ic;
        return 1;
    }
    return 0;
}

// Two passes: mass and centre, then the parallel-axis inertia; then the
// continuous-collision extents (shape.c:182-300).
static void RecomputeMass(m3HostWorld* w, int32_t b)
{
    m3WorldView& v = w->hv;
    if (v.btype[b] != M3_BODY_DYNAMIC)
    {
        v.invMass[b] = 0.0f;
        v.invI[b] = m3ZeroMat3();
        v.inertia[b] = m3ZeroMat3();
        v.lc[b] = v3(0.0f, 0.0f, 0.0f);
        v.minExt[b] = 1.0e30f;
        v.maxExt[b] = 0.0f;
        return;
    }
    float mass = 0.0f;
    m3Vec3 center = v3(0.0f, 0.0f, 0.0f);
    for (int32_t s = v.shapeHead[b]; s != -1; s = v.shapeNext[s])
    {
        float m;
        m3Vec3 c;
        m3Mat3 ic;
        if (!ShapeMassProps(w, s, &m, &c, &ic))
        {
            continue;
        }
        ComposeMassProps(v, s, &c, &ic);
        mass += m;
        center = m3Add3(center, m3MulSV3(m, c));
    }
    if (!(mass > 0.0f))
    {
        v.invMass[b] = 1.0f;
        v.invI[b] = m3ZeroMat3();
        v.inertia[b] = m3ZeroMat3();
        v.lc[b] = v3(0.0f, 0.0f, 0.0f);
        v.minExt[b] = 1.0e30f;
        v.maxExt[b] = 0.0f;
        return;
    }
    center = m3MulSV3(1.0f / mass, center);
    m3Mat3 inertia = m3ZeroMat3();
    for (int32_t s = v.shapeHead[b]; s != -1; s = v.shapeNext[s])
    {
        float m;
        m3Vec3 c;
        m3Mat3 ic;
        if (!ShapeMassProps(w, s, &m, &c, &ic))
        {
            continue;
        }
        ComposeMassProps(v, s, &c, &ic);
        m3Vec3 d = m3Sub3(c, center);
        float d2 = m3Dot3(d, d);
        inertia.cx.x += ic.cx.x + m * (d2 - d.x * d.x);
        inertia.cy.y += ic.cy.y + m * (d2 - d.y * d.y);
        inertia.cz.z += ic.cz.z + m * (d2 - d.z * d.z);
        inertia.cy.x += ic.cy.x - m * d.x * d.y;
        inertia.cx.y += ic.cx.y - m * d.x * d.y;
        inertia.cz.x += ic.cz.x - m * d.x * d.z;
        inertia.cx.z += ic.cx.z - m * d.x * d.z;
        inertia.cz.y += ic.cz.y - m * d.y * d.z;
        inertia.cy.z += ic.cy.z - m * d.y * d.z;
    }
    v.invMass[b] = 1.0f / mass;
    v.inertia[b] = inertia;
    v.invI[b] = InvertSymmetric(inertia);

    float minExtent = 1.0e30f;
    float maxExtent = 0.0f;
    for (int32_t s2 = v.shapeHead[b]; s2 != -1; s2 = v.shapeNext[s2])
    {
        uint8_t type = v.shapeType[s2];
        if (type == M3_SHAPE_SPHERE)
        {
            float r = v.geom[s2].s;
            m3Vec3 d = m3Sub3(v.geom[s2].v, center);
            minExtent = m3MinF(minExtent, r);
            maxExtent = m3MaxF(maxExtent, sqrtf(m3Dot3(d, d)) + r);
        }
        else if (type == M3_SHAPE_CAPSULE)
        {
            float r = v.geom[s2].s;
            m3Vec3 d1 = m3Sub3(v.geom[s2].v, center);
            m3Vec3 d2 = m3Sub3(v.geom[s2].v2, center);
            minExtent = m3MinF(minExtent, r);
            maxExtent = m3MaxF(maxExtent, sqrtf(m3MaxF(m3Dot3(d1, d1), m3Dot3(d2, d2))) + r);
        }
        else if (type == M3_SHAPE_HULL)
        {
            const m3HullData* hull = &w->hulls[v.hullIndex[s2]];
            for (int32_t f = 0; f < hull->faceCount; ++f)
            {
                float dist = hull->faceOffsets[f] - m3Dot3(hull->faceNormals[f], center);
                minExtent = m3MinF(minExtent, dist);
            }
            for (int32_t k = 0; k < hull->vertexCount; ++k)
            {
                m3Vec3 d = m3Sub3(hull->vertices[k], center);
                maxExtent = m3MaxF(maxExtent, sqrtf(m3Dot3(d, d)));
            }
        }
    }
    v.minExt[b] = minExtent;
    v.maxExt[b] = maxExtent;
    v.lc[b] = center;
}

// ---------------------------------------------------------------------
// Hulls (hull.c)
// ---------------------------------------------------------------------

// Half-edge adjacency from the face loops, twins at 2k and 2k+1, and
// the vertex centroid (hull.c:71-130).
static void BuildHalfEdges(m3HullData* hull)
{
    int32_t count = 0;
    int32_t dirKey[M3_HULL_MAX_HALF_EDGES];
    int32_t dirSlot[M3_HULL_MAX_HALF_EDGES];
    int32_t dirCount = 0;
    int32_t faceEdgeSlot[M3_HULL_MAX_FACE_INDICES];
    for (int32_t f = 0; f < hull->faceCount; ++f)
    {
        int32_t n = hull->faceVertCounts[f];
        int32_t start = hull->faceVertStart[f];
        for (int32_t k = 0; k < n; ++k)
        {
            int32_t a = hull->faceIndices[start + k];
            int32_t b = hull->faceIndices[start + (k + 1) % n];
            int32_t reverse = b * 256 + a;
            int32_t slot = -1;
            for (int32_t d = 0; d < dirCount; ++d)
            {
                if (dirKey[d] == reverse)
                {
                    slot = dirSlot[d] ^ 1;
                    break;
                }
            }
            if (slot < 0)
            {
                slot = count;
                count += 2;
                dirKey[dirCount] = a * 256 + b;
                dirSlot[dirCount] = slot;
                dirCount += 1;
            }
            hull->edges[slot].origin = (uint8_t)a;
            hull->edges[slot].twin = (uint16_t)(slot ^ 1);
            hull->edges[slot].face = (uint8_t)f;
            faceEdgeSlot[start + k] = slot;
        }
    }
    for (int32_t f = 0; f < hull->faceCount; ++f)
    {
        int32_t n = hull->faceVertCounts[f];
        int32_t start = hull->faceVertStart[f];
        for (int32_t k = 0; k < n; ++k)
        {
            hull->edges[faceEdgeSlot[start + k]].next = (uint16_t)faceEdgeSlot[start + (k + 1) % n];
        }
    }
    hull->edgeCount = count;
    m3Vec3 c = v3(0.0f, 0.0f, 0.0f);
    for (int32_t k = 0; k < hull->vertexCount; ++k)
    {
        c = m3Add3(c, hull->vertices[k]);
    }
    hull->center = m3MulSV3(1.0f / (m3real)hull->vertexCount, c);
}

// Closed-form box: canonical vertex order, six outward CCW faces, unit
// density mass (hull.c:14-64).
static void BuildBoxHull(m3HullData* out, m3Vec3 he)
{
    memset(out, 0, sizeof(*out));
    m3real hx = he.x;
    m3real hy = he.y;
    m3real hz = he.z;
    const m3Vec3 verts[8] = {
        v3(-hx, -hy, -hz), v3(hx, -hy, -hz), v3(hx, hy, -hz), v3(-hx, hy, -hz),
        v3(-hx, -hy, hz),  v3(hx, -hy, hz),  v3(hx, hy, hz),  v3(-hx, hy, hz),
    };
    const m3Vec3 normals[6] = {
        v3(1.0f, 0.0f, 0.0f),  v3(-1.0f, 0.0f, 0.0f), v3(0.0f, 1.0f, 0.0f),
        v3(0.0f, -1.0f, 0.0f), v3(0.0f, 0.0f, 1.0f),  v3(0.0f, 0.0f, -1.0f),
    };
    const m3real offsets[6] = {hx, hx, hy, hy, hz, hz};
    static const uint8_t loops[6][4] = {
        {1, 2, 6, 5}, {0, 4, 7, 3}, {2, 3, 7, 6}, {0, 1, 5, 4}, {4, 5, 6, 7}, {0, 3, 2, 1},
    };
    out->vertexCount = 8;
    out->faceCount = 6;
    out->indexCount = 24;
    memcpy(out->vertices, verts, sizeof(verts));
    memcpy(out->faceNormals, normals, sizeof(normals));
    memcpy(out->faceOffsets, offsets, sizeof(offsets));
    for (int32_t f = 0; f < 6; ++f)
    {
        out->faceVertCounts[f] = 4;
        out->faceVertStart[f] = (uint16_t)(4 * f);
        for (int32_t k = 0; k < 4; ++k)
        {
            out->faceIndices[4 * f + k] = loops[f][k];
        }
    }
    float m = 8.0f * hx * hy * hz;
    out->unitMass = m;
    out->unitCom = v3(0.0f, 0.0f, 0.0f);
    out->unitInertiaCom = m3ZeroMat3();
    out->unitInertiaCom.cx.x = (m / 3.0f) * (hy * hy + hz * hz);
    out->unitInertiaCom.cy.y = (m / 3.0f) * (hx * hx + hz * hz);
    out->unitInertiaCom.cz.z = (m / 3.0f) * (hx * hx + hy * hy);
    BuildHalfEdges(out);
}

uint64_t m3HullKey(const m3HullData* h)
{
    const int32_t nv = h->vertexCount < 0 ? 0
                                          : (h->vertexCount > M3_HULL_MAX_VERTS ? M3_HULL_MAX_VERTS
                                                                                : h->vertexCount);
    uint64_t key = m3Fnv(M3_HASH_INIT, h, (int32_t)offsetof(m3HullData, vertices));
    return m3Fnv(key, h->vertices, 12 * nv);
}

// Content-deduplicated interning in ascending slot order (hull.c:132-152).
// Live slabs are pairwise distinct, so the first match in slot order is
// the only match; a content-hash index finds it without scanning.
static int32_t InternHull(m3HostWorld* w, const m3HullData* data)
{
    m3WorldScalars* sc = w->hv.sc;
    uint64_t key = m3HullKey(data);
    auto range = w->hullIndexByContent.equal_range(key);
    for (auto it = range.first; it != range.second; ++it)
    {
        int32_t i = it->second;
        if (w->hullRefs[i] > 0 && memcmp(&w->hulls[i], data, sizeof(m3HullData)) == 0)
        {
            w->hullRefs[i] += 1;
            return i;
        }
    }
    int32_t index = -1;
    if (w->hullFree.Pop(&index))
    {
        w->hulls[(size_t)index] = *data;
        w->hullRefs[(size_t)index] = 1;
    }
    else
    {
        if (sc->hullMax >= w->shapeCap)
        {
            return -1;
        }
        index = sc->hullMax;
        sc->hullMax += 1;
        w->hulls.push_back(*data);
        w->hullRefs.push_back(1);
    }
    w->hullIndexByContent.emplace(key, index);
    return index;
}

// ---------------------------------------------------------------------
// Shapes (shape.c:411-620, :717-830, :1334)
// ---------------------------------------------------------------------
extern "C" m3ShapeDef m3DefaultShapeDef(void)
{
    m3ShapeDef def;
    memset(&def, 0, sizeof(def));
    def.density = 1.0f;
    def.friction = 0.6f;
    def.restitution = 0.0f;
    def.categoryBits = 1ull;
    def.maskBits = ~0ull;
    def.groupIndex = 0;
    def.localRotation = q4(0.0f, 0.0f, 0.0f, 1.0f);
    def.internalValue = M3_SHAPE_COOKIE;
    return def;
}

static m3ShapeId CreateShapeCommon(m3BodyId bodyId, const m3ShapeDef* def, uint8_t type,
                                   const m3ShapeGeom* geom, const m3HeightFieldDev* grid = nullptr,
                                   const float* heights = nullptr,
                                   const m3HullData* prebuilt = nullptr)
{
    m3ShapeId nullId = {0, 0, 0};
    int32_t b;
    m3HostWorld* w = ResolveBody(bodyId, &b);
    if (w == nullptr || def == nullptr || def->internalValue != M3_SHAPE_COOKIE)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "create shape: stale body or invalid def");
        return nullId;
    }
    float rotLen2 = def->localRotation.x * def->localRotation.x +
                    def->localRotation.y * def->localRotation.y +
                    def->localRotation.z * def->localRotation.z +
                    def->localRotation.w * def->localRotation.w;
    if (!FiniteV3(def->localPosition) || !FiniteQuat(def->localRotation) || rotLen2 < 0.99f ||
        rotLen2 > 1.01f || !FiniteF(def->density) || !(def->density > 0.0f) ||
        !FiniteF(def->friction) || def->friction < 0.0f || !FiniteF(def->restitution) ||
        def->restitution < 0.0f || !FiniteF(def->rollingResistance) ||
        def->rollingResistance < 0.0f)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "create shape: invalid material or offset");
        return nullId;
    }
    if (m3gpuSyncHost(w) != M3GPU_OK)
    {
        return nullId;
    }
    m3WorldView& v = w->hv;
    if (v.sc->shapeMax >= w->shapeCap && w->shapeFree.count == 0)
    {
        m3gpuSetError(M3GPU_ERR_CAPACITY, "create shape: shape pool exhausted");
        return nullId;
    }
    int32_t hullIndex = -1;
    if (type == M3_SHAPE_HULL)
    {
        // A box from its half extents, or a hull built from points.
        m3HullData data;
        if (prebuilt != nullptr)
        {
            data = *prebuilt;
        }
        else
        {
            BuildBoxHull(&data, geom->v);
        }
        hullIndex = InternHull(w, &data);
        if (hullIndex < 0)
        {
            m3gpuSetError(M3GPU_ERR_CAPACITY, "create shape: hull pool exhausted");
            return nullId;
        }
    }
    int32_t s = -1;
    if (!w->shapeFree.Pop(&s))
    {
        s = v.sc->shapeMax;
        v.sc->shapeMax += 1;
    }
    v.shapeAlive[s] = 1;
    v.shapeBody[s] = b;
    v.shapeType[s] = type;
    v.geom[s] = *geom;
    v.density[s] = def->density;
    v.friction[s] = def->friction;
    v.restitution[s] = def->restitution;
    v.rolling[s] = def->rollingResistance;
    v.category[s] = def->categoryBits;
    v.mask[s] = def->maskBits;
    v.group[s] = def->groupIndex;
    v.shapeUserData[s] = def->userData;
    v.sensor[s] = def->isSensor ? 1 : 0;
    v.hitEvents[s] = def->enableHitEvents ? 1 : 0;
    v.preSolve[s] = def->enablePreSolveEvents ? 1 : 0;
    v.surfVel[s] = v3(0.0f, 0.0f, 0.0f);
    v.localPos[s] = def->localPosition;
    v.localRot[s] = def->localRotation;
    v.hasOffset[s] = (def->localPosition.x != 0.0f || def->localPosition.y != 0.0f ||
                      def->localPosition.z != 0.0f || def->localRotation.x != 0.0f ||
                      def->localRotation.y != 0.0f || def->localRotation.z != 0.0f ||
                      def->localRotation.w != 1.0f)
                         ? 1
                         : 0;
    v.shapeNext[s] = v.shapeHead[b];
    v.shapeHead[b] = s;
    v.hullIndex[s] = hullIndex;
    v.hfIndex[s] = -1;
    if (type == M3_SHAPE_HEIGHTFIELD)
    {
        // A fresh heightfield slot holding the caller's samples
        // (shape.c:549-566).
        m3HeightFieldDev slot = *grid;
        slot.sampleStart = (int32_t)w->hfSamples.size();
        v.hfIndex[s] = (int32_t)w->hfHeaders.size();
        w->hfHeaders.push_back(slot);
        w->hfSamples.insert(w->hfSamples.end(), heights, heights + (size_t)grid->nx * grid->nz);
        w->hfVersion += 1;
    }
    // Every shape but a plane enters the broadphase tree with its
    // creation bounds (shape.c:589-606).
    if (type != M3_SHAPE_PLANE)
    {
        m3WorldView tv = v;
        tv.hulls = w->hulls.empty() ? nullptr : w->hulls.data();
        tv.hfs = w->hfHeaders.empty() ? nullptr : w->hfHeaders.data();
        tv.hfSamples = w->hfSamples.empty() ? nullptr : w->hfSamples.data();
        const m3Aabb box = m3ShapeCreationBounds(tv, s);
        v.proxyId[s] =
            m3TreeInsert(m3WorldTree(v), m3TreeArrayStore{v.treeNodes}, box.lo, box.hi, s);
    }
    RecomputeMass(w, b);
    w->hostDirty = true;
    m3JournalUnrecordable(w); // creation is not recorded by this path
    w->structure += 1;        // device snapshot slots saved before are void
    m3ShapeId id = {s + 1, (uint16_t)w->slot, v.shapeGen[s]};
    return id;
}

extern "C" m3ShapeId m3CreateSphereShape(m3BodyId bodyId, const m3ShapeDef* def,
                                         const m3Sphere* sphere)
{
    m3ShapeId nullId = {0, 0, 0};
    m3gpuClearError();
    if (sphere == nullptr || !(sphere->radius > 0.0f) || !FiniteF(sphere->radius) ||
        !FiniteV3(sphere->center))
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateSphereShape: invalid sphere");
        return nullId;
    }
    m3ShapeGeom geom;
    geom.v = sphere->center;
    geom.s = sphere->radius;
    geom.v2 = v3(0.0f, 0.0f, 0.0f);
    geom.s2 = 0.0f;
    return CreateShapeCommon(bodyId, def, M3_SHAPE_SPHERE, &geom);
}

extern "C" m3ShapeId m3CreatePlaneShape(m3BodyId bodyId, const m3ShapeDef* def,
                                        const m3Plane* plane)
{
    m3ShapeId nullId = {0, 0, 0};
    m3gpuClearError();
    if (plane == nullptr || !FiniteV3(plane->normal) || !FiniteF(plane->offset) ||
        !(m3Dot3(plane->normal, plane->normal) > 1.0e-12f))
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreatePlaneShape: invalid plane");
        return nullId;
    }
    int32_t b;
    m3HostWorld* w = ResolveBody(bodyId, &b);
    if (w == nullptr || m3gpuSyncHost(w) != M3GPU_OK || w->hv.btype[b] != M3_BODY_STATIC)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreatePlaneShape: planes need a static body");
        return nullId;
    }
    m3ShapeGeom geom;
    geom.v = m3Normalize3(plane->normal);
    geom.s = plane->offset;
    geom.v2 = v3(0.0f, 0.0f, 0.0f);
    geom.s2 = 0.0f;
    return CreateShapeCommon(bodyId, def, M3_SHAPE_PLANE, &geom);
}

extern "C" m3ShapeId m3CreateCapsuleShape(m3BodyId bodyId, const m3ShapeDef* def,
                                          const m3Capsule* capsule)
{
    m3ShapeId nullId = {0, 0, 0};
    m3gpuClearError();
    if (capsule == nullptr || !(capsule->radius > 0.0f) || !FiniteF(capsule->radius) ||
        !FiniteV3(capsule->point1) || !FiniteV3(capsule->point2))
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateCapsuleShape: invalid capsule");
        return nullId;
    }
    m3Vec3 axis = m3Sub3(capsule->point2, capsule->point1);
    if (!(m3Dot3(axis, axis) > 0.0f))
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateCapsuleShape: zero-length capsule");
        return nullId;
    }
    m3ShapeGeom geom;
    geom.v = capsule->point1;
    geom.s = capsule->radius;
    geom.v2 = capsule->point2;
    geom.s2 = 0.0f;
    return CreateShapeCommon(bodyId, def, M3_SHAPE_CAPSULE, &geom);
}

// shape.c:988-1030 (shape.h:143-149): the convex hull of a point cloud
// (QuickHull, quickhull.cpp), interned like every hull slab.  Null for a
// stale body or def, no points, a non-finite point, or a cloud the hull
// builder refuses (fewer than 4 or more than 256 points, degenerate, over
// the slab's caps).
extern "C" m3ShapeId m3CreateHullShape(m3BodyId bodyId, const m3ShapeDef* def,
                                       const m3Vec3* points, int32_t count)
{
    m3ShapeId nullId = {0, 0, 0};
    m3gpuClearError();
    int32_t b;
    if (ResolveBody(bodyId, &b) == nullptr || def == nullptr ||
        def->internalValue != M3_SHAPE_COOKIE)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateHullShape: stale body or invalid def");
        return nullId;
    }
    if (points == nullptr || count <= 0)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateHullShape: no points");
        return nullId;
    }
    for (int32_t i = 0; i < count; ++i)
    {
        if (!FiniteV3(points[i]))
        {
            m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateHullShape: non-finite point %d", i);
            return nullId;
        }
    }
    m3HullData data;
    if (!m3QuickHull(points, count, &data))
    {
        m3gpuSetError(M3GPU_ERR_INVALID,
                      "m3CreateHullShape: degenerate cloud, or over the hull caps");
        return nullId;
    }
    BuildHalfEdges(&data);
    m3ShapeGeom geom;
    memset(&geom, 0, sizeof(geom));
    return CreateShapeCommon(bodyId, def, M3_SHAPE_HULL, &geom, nullptr, nullptr, &data);
}

extern "C" m3ShapeId m3CreateBoxShape(m3BodyId bodyId, const m3ShapeDef* def, m3Vec3 halfExtents)
{
    m3ShapeId nullId = {0, 0, 0};
    m3gpuClearError();
    if (!(halfExtents.x > 0.0f) || !(halfExtents.y > 0.0f) || !(halfExtents.z > 0.0f) ||
        !FiniteV3(halfExtents))
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateBoxShape: invalid half extents");
        return nullId;
    }
    m3ShapeGeom geom;
    geom.v = halfExtents;
    geom.s = 0.0f;
    geom.v2 = v3(0.0f, 0.0f, 0.0f);
    geom.s2 = 0.0f;
    return CreateShapeCommon(bodyId, def, M3_SHAPE_HULL, &geom);
}

// shape.c:1175-1262: a native heightfield on a static body, an nx x nz
// grid of samples (x fastest) with square cells, its minimum corner at
// the shape's origin.
extern "C" m3ShapeId m3CreateHeightFieldGridShape(m3BodyId bodyId, const m3ShapeDef* def,
                                                  const float* heights, int32_t nx, int32_t nz,
                                                  float cellSize)
{
    m3ShapeId nullId = {0, 0, 0};
    m3gpuClearError();
    int32_t b;
    m3HostWorld* w = ResolveBody(bodyId, &b);
    if (w == nullptr || def == nullptr || def->internalValue != M3_SHAPE_COOKIE ||
        heights == nullptr || m3gpuSyncHost(w) != M3GPU_OK || w->hv.btype[b] != M3_BODY_STATIC)
    {
        m3gpuSetError(M3GPU_ERR_INVALID,
                      "m3CreateHeightFieldGridShape: heightfields need a static body");
        return nullId;
    }
    if (nx < 2 || nx > M3_HEIGHTFIELD_MAX_DIM || nz < 2 || nz > M3_HEIGHTFIELD_MAX_DIM ||
        !FiniteF(cellSize) || !(cellSize > 0.0f))
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateHeightFieldGridShape: invalid grid");
        return nullId;
    }
    float lo = heights[0];
    float hi = heights[0];
    for (int32_t i = 0; i < nx * nz; ++i)
    {
        if (!FiniteF(heights[i]))
        {
            m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateHeightFieldGridShape: non-finite sample");
            return nullId;
        }
        lo = heights[i] < lo ? heights[i] : lo;
        hi = heights[i] > hi ? heights[i] : hi;
    }
    m3HeightFieldDev grid;
    grid.nx = nx;
    grid.nz = nz;
    grid.cellSize = cellSize;
    grid.minHeight = lo;
    grid.maxHeight = hi;
    grid.sampleStart = 0;
    m3ShapeGeom geom;
    memset(&geom, 0, sizeof(geom));
    return CreateShapeCommon(bodyId, def, M3_SHAPE_HEIGHTFIELD, &geom, &grid, heights);
}

extern "C" bool m3Shape_IsValid(m3ShapeId shapeId)
{
    m3HostWorld* w = m3gpuWorldFromIndex0(shapeId.world0);
    int32_t index = shapeId.index1 - 1;
    return w != nullptr && index >= 0 && index < w->hv.sc->shapeMax &&
           w->hv.shapeAlive[index] != 0 && w->hv.shapeGen[index] == shapeId.generation;
}

static m3HostWorld* ResolveShape(m3ShapeId id, int32_t* index)
{
    m3HostWorld* w = m3gpuWorldFromIndex0(id.world0);
    const int32_t i = id.index1 - 1;
    if (w == nullptr || i < 0 || i >= w->hv.sc->shapeMax || w->hv.shapeAlive[i] == 0 ||
        w->hv.shapeGen[i] != id.generation)
    {
        *index = -1;
        return nullptr;
    }
    *index = i;
    return w;
}

extern "C" m3BodyId m3Shape_GetBody(m3ShapeId shapeId)
{
    int32_t index;
    m3HostWorld* w = ResolveShape(shapeId, &index);
    if (w == nullptr)
    {
        return m3BodyId{0, 0, 0};
    }
    const int32_t b = w->hv.shapeBody[index];
    return m3BodyId{b + 1, (uint16_t)w->slot, w->hv.bodyGen[b]};
}

// Shape materials and flags (shape.c:1387-1410, 1463-1600): each public
// call checks as the reference's, records its journal record and changes
// the host image (the next step uploads it); replay applies the same
// records.
void m3ApplyHostShapeOp(m3HostWorld* w, const m3JournalRecordView& r)
{
    m3WorldView& v = w->hv;
    const int32_t s = r.body;
    switch (r.op)
    {
    case M3_OP_SET_SHAPE_FRICTION:
        v.friction[s] = r.setting[0];
        break;
    case M3_OP_SET_SHAPE_RESTITUTION:
        v.restitution[s] = r.setting[0];
        break;
    case M3_OP_SET_SHAPE_ROLLING:
        v.rolling[s] = r.setting[0];
        break;
    case M3_OP_SET_SHAPE_DENSITY:
        v.density[s] = r.setting[0];
        if (r.bits != 0)
        {
            RecomputeMass(w, v.shapeBody[s]);
        }
        break;
    case M3_OP_ENABLE_SHAPE_HIT_EVENTS:
        v.hitEvents[s] = r.bits != 0 ? 1 : 0;
        break;
    case M3_OP_ENABLE_SHAPE_PRESOLVE:
        v.preSolve[s] = r.bits != 0 ? 1 : 0;
        break;
    default:
        break;
    }
}

// {m3ShapeId id; float value} for a material, {m3ShapeId id; float
// density; int32 updateMass} for a density, {m3ShapeId id; int32 on} for
// a flag.
static void ShapeCommand(m3ShapeId id, int32_t op, float value, uint32_t bits)
{
    m3gpuClearError();
    int32_t index;
    m3HostWorld* w = ResolveShape(id, &index);
    if (w == nullptr || m3gpuSyncHost(w) != M3GPU_OK)
    {
        return;
    }
    uint8_t payload[16];
    memset(payload, 0, sizeof(payload));
    memcpy(payload, &id, 8);
    int32_t bytes = 12;
    if (op == M3_OP_ENABLE_SHAPE_HIT_EVENTS || op == M3_OP_ENABLE_SHAPE_PRESOLVE)
    {
        memcpy(payload + 8, &bits, 4);
    }
    else
    {
        memcpy(payload + 8, &value, 4);
        if (op == M3_OP_SET_SHAPE_DENSITY)
        {
            memcpy(payload + 12, &bits, 4);
            bytes = 16;
        }
    }
    m3JournalRecordView r;
    memset(&r, 0, sizeof(r));
    r.op = op;
    r.body = index;
    r.setting[0] = value;
    r.bits = bits;
    m3JournalAppend(w, op, payload, bytes);
    m3ApplyHostShapeOp(w, r);
    w->hostDirty = true;
}

extern "C" void m3Shape_SetFriction(m3ShapeId shapeId, float friction)
{
    if (isfinite(friction) && friction >= 0.0f)
    {
        ShapeCommand(shapeId, M3_OP_SET_SHAPE_FRICTION, friction, 0u);
    }
}

extern "C" void m3Shape_SetRestitution(m3ShapeId shapeId, float restitution)
{
    if (isfinite(restitution) && restitution >= 0.0f)
    {
        ShapeCommand(shapeId, M3_OP_SET_SHAPE_RESTITUTION, restitution, 0u);
    }
}

extern "C" void m3Shape_SetRollingResistance(m3ShapeId shapeId, float value)
{
    if (isfinite(value) && value >= 0.0f)
    {
        ShapeCommand(shapeId, M3_OP_SET_SHAPE_ROLLING, value, 0u);
    }
}

extern "C" void m3Shape_SetDensity(m3ShapeId shapeId, float density, bool updateBodyMass)
{
    if (isfinite(density) && density > 0.0f)
    {
        ShapeCommand(shapeId, M3_OP_SET_SHAPE_DENSITY, density, updateBodyMass ? 1u : 0u);
    }
}

extern "C" void m3Shape_EnableHitEvents(m3ShapeId shapeId, bool flag)
{
    ShapeCommand(shapeId, M3_OP_ENABLE_SHAPE_HIT_EVENTS, 0.0f, flag ? 1u : 0u);
}

extern "C" void m3Shape_EnablePreSolve(m3ShapeId shapeId, bool flag)
{
    ShapeCommand(shapeId, M3_OP_ENABLE_SHAPE_PRESOLVE, 0.0f, flag ? 1u : 0u);
}

template <typename T, typename F> static T ReadShapeField(m3ShapeId id, T zero, F get)
{
    int32_t index;
    m3HostWorld* w = ResolveShape(id, &index);
    if (w == nullptr || m3gpuSyncHost(w) != M3GPU_OK)
    {
        return zero;
    }
    return get(w->hv, index);
}

extern "C" float m3Shape_GetFriction(m3ShapeId shapeId)
{
    return ReadShapeField(shapeId, 0.0f, [](const m3WorldView& v, int32_t s) { return v.friction[s]; });
}

extern "C" float m3Shape_GetRestitution(m3ShapeId shapeId)
{
    return ReadShapeField(shapeId, 0.0f,
                     [](const m3WorldView& v, int32_t s) { return v.restitution[s]; });
}

extern "C" float m3Shape_GetRollingResistance(m3ShapeId shapeId)
{
    return ReadShapeField(shapeId, 0.0f, [](const m3WorldView& v, int32_t s) { return v.rolling[s]; });
}

extern "C" float m3Shape_GetDensity(m3ShapeId shapeId)
{
    return ReadShapeField(shapeId, 0.0f, [](const m3WorldView& v, int32_t s) { return v.density[s]; });
}

extern "C" bool m3Shape_AreHitEventsEnabled(m3ShapeId shapeId)
{
    return ReadShapeField(shapeId, false,
                     [](const m3WorldView& v, int32_t s) { return v.hitEvents[s] != 0; });
}

extern "C" bool m3Shape_IsPreSolveEnabled(m3ShapeId shapeId)
{
    return ReadShapeField(shapeId, false,
                     [](const m3WorldView& v, int32_t s) { return v.preSolve[s] != 0; });
}

// Contact readback (query.c:1330-1409): one entry per manifold with
// points touching the body or shape, in the current pair list's order.
// Points are body A's centre of mass plus the anchor, in f64.
static void FillContact(const m3HostWorld* w, uint64_t key, const m3Manifold& m,
                        m3ContactData* out)
{
    const m3WorldView& v = w->hv;
    const int32_t a = (int32_t)(key >> 32);
    const int32_t b = (int32_t)(key & 0xFFFFFFFFu);
    out->shapeA = m3ShapeId{a + 1, (uint16_t)w->slot, v.shapeGen[a]};
    out->shapeB = m3ShapeId{b + 1, (uint16_t)w->slot, v.shapeGen[b]};
    out->normal = m.normal;
    out->pointCount = m.pointCount;
    const int32_t body = v.shapeBody[a];
    const m3Transform xf = v.xf[body];
    const m3Vec3 rc = m3RotateVec3(xf.q, v.lc[body]);
    for (int32_t k = 0; k < 4; ++k)
    {
        if (k < m.pointCount)
        {
            const m3ManifoldPoint& p = m.points[k];
            out->points[k] = m3Pos3{xf.p.x + (double)(rc.x + p.anchorA.x),
                                    xf.p.y + (double)(rc.y + p.anchorA.y),
                                    xf.p.z + (double)(rc.z + p.anchorA.z)};
            out->separations[k] = p.separation;
            out->normalImpulses[k] = p.normalImpulse;
        }
        else
        {
            out->points[k] = m3Pos3{0.0, 0.0, 0.0};
            out->separations[k] = 0.0f;
            out->normalImpulses[k] = 0.0f;
        }
    }
}

// Walks the current pair list, filling an entry for each manifold with
// points whose shapes pass `touches`.
template <typename F>
static int32_t ReadContacts(m3HostWorld* w, m3ContactData* out, int32_t capacity, F touches)
{
    if (m3gpuSyncHost(w) != M3GPU_OK)
    {
        return 0;
    }
    const m3WorldView& v = w->hv;
    const bool second = v.sc->pairBuf != 0;
    const uint64_t* keys = second ? v.keys1 : v.keys0;
    const m3Manifold* man = second ? v.man1 : v.man0;
    int32_t written = 0;
    for (int32_t i = 0; i < v.sc->pairCount && written < capacity; ++i)
    {
        const int32_t a = (int32_t)(keys[i] >> 32);
        const int32_t b = (int32_t)(keys[i] & 0xFFFFFFFFu);
        if (touches(a, b) && man[i].pointCount > 0)
        {
            FillContact(w, keys[i], man[i], &out[written]);
            written += 1;
        }
    }
    return written;
}

extern "C" int32_t m3Shape_GetContactData(m3ShapeId shapeId, m3ContactData* out, int32_t capacity)
{
    int32_t shape;
    m3HostWorld* w = ResolveShape(shapeId, &shape);
    if (w == nullptr || out == nullptr || capacity <= 0)
    {
        return 0;
    }
    return ReadContacts(w, out, capacity,
                        [shape](int32_t a, int32_t b) { return a == shape || b == shape; });
}

extern "C" int32_t m3Body_GetContactData(m3BodyId bodyId, m3ContactData* out, int32_t capacity)
{
    int32_t body;
    m3HostWorld* w = ResolveBody(bodyId, &body);
    if (w == nullptr || out == nullptr || capacity <= 0)
    {
        return 0;
    }
    const int32_t* shapeBody = w->hv.shapeBody;
    return ReadContacts(w, out, capacity, [body, shapeBody](int32_t a, int32_t b) {
        return shapeBody[a] == body || shapeBody[b] == body;
    });
}

// ---------------------------------------------------------------------
// Joints (joint.c:15-330, :387-520)
// ---------------------------------------------------------------------
extern "C" m3JointDef m3DefaultJointDef(void)
{
    m3JointDef def;
    memset(&def, 0, sizeof(def));
    def.type = m3_sphericalJoint;
    def.localAxisA = v3(0.0f, 0.0f, 1.0f);
    def.localAxisB = v3(0.0f, 0.0f, 1.0f);
    def.genericMotorAxis = 255;
    def.ratio = 1.0f;
    def.internalValue = M3_JOINT_COOKIE;
    return def;
}

// Quaternion of a right-handed column basis, Shepperd's largest-diagonal
// branch (joint.c:30-70).
static m3Quat QuatFromBasis(m3Vec3 t1, m3Vec3 t2, m3Vec3 axis)
{
    m3real m00 = t1.x, m01 = t2.x, m02 = axis.x;
    m3real m10 = t1.y, m11 = t2.y, m12 = axis.y;
    m3real m20 = t1.z, m21 = t2.z, m22 = axis.z;
    m3Quat q;
    m3real trace = m00 + m11 + m22;
    if (trace > 0.0f)
    {
        m3real s = sqrtf(trace + 1.0f) * 2.0f;
        q.w = 0.25f * s;
        q.x = (m21 - m12) / s;
        q.y = (m02 - m20) / s;
        q.z = (m10 - m01) / s;
    }
    else if (m00 > m11 && m00 > m22)
    {
        m3real s = sqrtf(1.0f + m00 - m11 - m22) * 2.0f;
        q.w = (m21 - m12) / s;
        q.x = 0.25f * s;
        q.y = (m01 + m10) / s;
        q.z = (m02 + m20) / s;
    }
    else if (m11 > m22)
    {
        m3real s = sqrtf(1.0f + m11 - m00 - m22) * 2.0f;
        q.w = (m02 - m20) / s;
        q.x = (m01 + m10) / s;
        q.y = 0.25f * s;
        q.z = (m12 + m21) / s;
    }
    else
    {
        m3real s = sqrtf(1.0f + m22 - m00 - m11) * 2.0f;
        q.w = (m10 - m01) / s;
        q.x = (m02 + m20) / s;
        q.y = (m12 + m21) / s;
        q.z = 0.25f * s;
    }
    return m3NormalizeQuat(q);
}

static m3Quat QuatFromAxisZ(m3Vec3 axis)
{
    m3Vec3 t1;
    m3Vec3 t2;
    m3MakeTangentBasis(axis, &t1, &t2);
    return QuatFromBasis(t1, t2, axis);
}

extern "C" m3JointId m3CreateJoint(const m3JointDef* def)
{
    m3JointId nullId = {0, 0, 0};
    m3gpuClearError();
    if (def == nullptr || def->internalValue != M3_JOINT_COOKIE)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateJoint: invalid def");
        return nullId;
    }
    if (def->type != m3_sphericalJoint && def->type != m3_revoluteJoint &&
        def->type != m3_fixedJoint)
    {
        m3gpuSetError(M3GPU_ERR_UNSUPPORTED,
                      "m3CreateJoint: joint type %d is not on the device path", def->type);
        return nullId;
    }
    if (def->type == m3_revoluteJoint && (!(m3Dot3(def->localAxisA, def->localAxisA) > 0.0f) ||
                                          !(m3Dot3(def->localAxisB, def->localAxisB) > 0.0f)))
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateJoint: a hinge needs real axes");
        return nullId;
    }
    if (!FiniteV3(def->localAnchorA) || !FiniteV3(def->localAnchorB) ||
        !FiniteV3(def->localAxisA) || !FiniteV3(def->localAxisB) || !FiniteF(def->lowerLimit) ||
        !FiniteF(def->upperLimit) || !FiniteF(def->motorSpeed) ||
        !FiniteF(def->maxMotorEffort) || !FiniteF(def->coneAngle) ||
        def->maxMotorEffort < 0.0f || (def->enableLimit && def->lowerLimit > def->upperLimit) ||
        (def->enableCone && def->coneAngle < 0.0f))
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateJoint: non-finite or unordered fields");
        return nullId;
    }
    if (def->type == m3_sphericalJoint && (def->enableCone || def->enableLimit))
    {
        m3gpuSetError(M3GPU_ERR_UNSUPPORTED,
                      "m3CreateJoint: spherical cone and twist limits are not on the device path");
        return nullId;
    }
    m3HostWorld* w = m3gpuWorldFromIndex0(def->bodyA.world0);
    if (w == nullptr || def->bodyB.world0 != def->bodyA.world0)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateJoint: bodies must share a world");
        return nullId;
    }
    int32_t a = BodySlot(w, def->bodyA);
    int32_t b = BodySlot(w, def->bodyB);
    if (a < 0 || b < 0 || a == b)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateJoint: stale or identical bodies");
        return nullId;
    }
    if (m3gpuSyncHost(w) != M3GPU_OK)
    {
        return nullId;
    }
    m3WorldView& v = w->hv;
    if (v.btype[a] != M3_BODY_DYNAMIC && v.btype[b] != M3_BODY_DYNAMIC)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3CreateJoint: a joint between immovables");
        return nullId;
    }
    // Recycled slots first, FIFO, then a fresh one (allocator.c:178-198).
    int32_t j = -1;
    if (w->jointFree.Pop(&j))
    {
    }
    else if (v.sc->jointMax < w->jointCap)
    {
        j = v.sc->jointMax;
        v.sc->jointMax += 1;
    }
    else
    {
        m3gpuSetError(M3GPU_ERR_CAPACITY, "m3CreateJoint: joint pool exhausted");
        return nullId;
    }
    v.jointAlive[j] = 1;
    v.jtype[j] = (uint8_t)def->type;
    v.jbodyA[j] = a;
    v.jbodyB[j] = b;
    v.jlocalA[j] = def->localAnchorA;
    v.jlocalB[j] = def->localAnchorB;
    v.jcollide[j] = def->collideConnected ? 1 : 0;
    v.jimpulse[j] = v3(0.0f, 0.0f, 0.0f);
    v.jperp[j] = v3(0.0f, 0.0f, 0.0f);
    v.jlimitImp[j] = v3(0.0f, 0.0f, 0.0f);
    v.jangular[j] = v3(0.0f, 0.0f, 0.0f);
    if (def->type == m3_fixedJoint)
    {
        const m3Transform& xa = v.xf[a];
        const m3Transform& xb = v.xf[b];
        v.jframeA[j] = m3IdentityQuat();
        v.jframeB[j] = m3NormalizeQuat(m3MulQuat(m3Conj(xb.q), xa.q));
    }
    else
    {
        v.jframeA[j] = QuatFromAxisZ(m3Normalize3(def->localAxisA));
        v.jframeB[j] = QuatFromAxisZ(m3Normalize3(def->localAxisB));
    }
    v.jflags[j] = (uint8_t)((def->enableLimit ? 1 : 0) | (def->enableMotor ? 2 : 0) |
                            (def->enableCone ? 4 : 0));
    v.jmotor[j] = v3(def->motorSpeed, def->maxMotorEffort, 0.0f);
    v.jbreak[j] = v3(0.0f, 0.0f, 0.0f);
    v.jspring[j] = v3(0.0f, 0.0f, 0.0f);
    v.jtargetScalar[j] = 0.0f;
    v.jtargetQ[j] = m3IdentityQuat();
    v.jspringImp[j] = v3(0.0f, 0.0f, 0.0f);
    v.jlimits[j] = v3(def->lowerLimit, def->upperLimit, def->coneAngle);
    v.jnextA[j] = v.jointHead[a];
    v.jointHead[a] = j;
    v.jnextB[j] = v.jointHead[b];
    v.jointHead[b] = j;
    if (v.btype[a] == M3_BODY_DYNAMIC)
    {
        v.awake[a] = 1;
        v.sleepTime[a] = 0.0f;
    }
    if (v.btype[b] == M3_BODY_DYNAMIC)
    {
        v.awake[b] = 1;
        v.sleepTime[b] = 0.0f;
    }
    w->hostDirty = true;
    m3JournalUnrecordable(w); // creation is not recorded by this path
    w->structure += 1;        // device snapshot slots saved before are void
    m3JointId id = {j + 1, (uint16_t)w->slot, v.jointGen[j]};
    return id;
}

void m3DrainBrokenJoints(m3HostWorld* w)
{
    const int32_t cap = w->jointCap > 0 ? w->jointCap : 1;
    while (w->brokenDrained < w->hv.sc->brokenCount)
    {
        // Entry j: slot j freed; entry -1 - j: slot j retired (its
        // generation had reached 0xFFFF).
        const int32_t e = w->hv.jbroken[w->brokenDrained % cap];
        if (e >= 0)
        {
            w->jointFree.Push(e);
        }
        else
        {
            w->jointFree.retired += 1;
        }
        w->brokenDrained += 1;
    }
}

// joint.c:914-938 (joint.h:216): breaking thresholds (0 = none); wakes
// the joint's dynamic bodies.  Refuses negative or non-finite values.
extern "C" void m3Joint_SetBreakThresholds(m3JointId jointId, float maxForce, float maxTorque)
{
    m3HostWorld* w = m3gpuWorldFromIndex0(jointId.world0);
    const int32_t j = jointId.index1 - 1;
    if (w == nullptr || !isfinite(maxForce) || maxForce < 0.0f || !isfinite(maxTorque) ||
        maxTorque < 0.0f)
    {
        return;
    }
    if (m3gpuSyncHost(w) != M3GPU_OK)
    {
        return;
    }
    m3WorldView& v = w->hv;
    if (j < 0 || j >= v.sc->jointMax || v.jointAlive[j] == 0 ||
        v.jointGen[j] != jointId.generation)
    {
        return;
    }
    struct
    {
        m3JointId id;
        float maxForce;
        float maxTorque;
    } record = {jointId, maxForce, maxTorque};
    m3JournalAppend(w, M3_OP_JOINT_SET_BREAK, &record, (int32_t)sizeof(record));
    m3ApplyBodyOp(v, M3_OP_JOINT_SET_BREAK, j, v3(maxForce, maxTorque, 0.0f));
    w->hostDirty = true;
}

// ---------------------------------------------------------------------
// Joint drives and switches (joint.c:548-624, 732-1129): limits, motor,
// collide-connected, spring and drive targets.  Each public call checks
// as the reference's, records its journal record and changes the host
// image (the next step uploads it); replay applies the same records.
// ---------------------------------------------------------------------
static m3HostWorld* ResolveJoint(m3JointId id, int32_t* index)
{
    m3HostWorld* w = m3gpuWorldFromIndex0(id.world0);
    const int32_t j = id.index1 - 1;
    if (w == nullptr || j < 0 || j >= w->hv.sc->jointMax || w->hv.jointAlive[j] == 0 ||
        w->hv.jointGen[j] != id.generation)
    {
        *index = -1;
        return nullptr;
    }
    *index = j;
    return w;
}

// The joint's dynamic bodies wake (joint.c:548-560).
static void WakeJointBodies(m3WorldView& v, int32_t j)
{
    const int32_t ends[2] = {v.jbodyA[j], v.jbodyB[j]};
    for (int32_t k = 0; k < 2; ++k)
    {
        if (ends[k] >= 0 && v.btype[ends[k]] == M3_BODY_DYNAMIC)
        {
            Wake(v, ends[k]);
        }
    }
}

void m3ApplyHostJointOp(m3HostWorld* w, const m3JournalRecordView& r)
{
    m3WorldView& v = w->hv;
    const int32_t j = r.body;
    const bool on = r.bits != 0;
    switch (r.op)
    {
    case M3_OP_JOINT_SET_LIMITS:
        // The cone angle rides limits.z and is kept; the lower and upper
        // rows' stored impulses are dropped.
        v.jflags[j] = (uint8_t)((v.jflags[j] & ~1u) | (on ? 1u : 0u));
        v.jlimits[j].x = r.setting[0];
        v.jlimits[j].y = r.setting[1];
        v.jlimitImp[j].x = 0.0f;
        v.jlimitImp[j].y = 0.0f;
        break;
    case M3_OP_JOINT_SET_MOTOR:
        v.jflags[j] = (uint8_t)((v.jflags[j] & ~2u) | (on ? 2u : 0u));
        v.jmotor[j].x = r.setting[0];
        v.jmotor[j].y = r.setting[1];
        if (v.jtype[j] == m3_genericJoint)
        {
            v.jlimitImp[j].y = 0.0f;
        }
        else
        {
            v.jperp[j].z = 0.0f;
        }
        break;
    case M3_OP_JOINT_SET_COLLIDE:
        v.jcollide[j] = on ? 1 : 0;
        break;
    case M3_OP_JOINT_SET_SPRING:
        v.jflags[j] = (uint8_t)((v.jflags[j] & ~8u) | (on ? 8u : 0u));
        v.jspring[j] = v3(r.setting[0], r.setting[1], 0.0f);
        v.jspringImp[j] = v3(0.0f, 0.0f, 0.0f);
        break;
    case M3_OP_JOINT_SET_TARGET:
        v.jtargetScalar[j] = r.setting[0];
        v.jtargetQ[j] = r.rotation;
        break;
    default:
        return;
    }
    WakeJointBodies(v, j);
}

// {m3JointId id; int32 enable; float a; float b} for limits, motor and
// spring, {m3JointId id; int32 on} for collide, {m3JointId id; float
// scalar; m3Quat q} for a target.
static void JointCommand(m3HostWorld* w, m3JointId id, int32_t j, int32_t op, uint32_t bits,
                         float a, float b, m3Quat q)
{
    uint8_t payload[28];
    memset(payload, 0, sizeof(payload));
    memcpy(payload, &id, 8);
    int32_t bytes;
    if (op == M3_OP_JOINT_SET_COLLIDE)
    {
        memcpy(payload + 8, &bits, 4);
        bytes = 12;
    }
    else if (op == M3_OP_JOINT_SET_TARGET)
    {
        memcpy(payload + 8, &a, 4);
        memcpy(payload + 12, &q, 16);
        bytes = 28;
    }
    else
    {
        memcpy(payload + 8, &bits, 4);
        memcpy(payload + 12, &a, 4);
        memcpy(payload + 16, &b, 4);
        bytes = 20;
    }
    m3JournalRecordView r;
    memset(&r, 0, sizeof(r));
    r.op = op;
    r.body = j;
    r.bits = bits;
    r.setting[0] = a;
    r.setting[1] = b;
    r.rotation = q;
    m3JournalAppend(w, op, payload, bytes);
    m3ApplyHostJointOp(w, r);
    w->hostDirty = true;
}

// Resolves a joint and makes its world's host image current.
static m3HostWorld* JointForWrite(m3JointId id, int32_t* j)
{
    m3gpuClearError();
    m3HostWorld* w = ResolveJoint(id, j);
    return w != nullptr && m3gpuSyncHost(w) == M3GPU_OK ? w : nullptr;
}

extern "C" void m3Joint_SetLimits(m3JointId jointId, bool enable, float lower, float upper)
{
    int32_t j;
    m3HostWorld* w = JointForWrite(jointId, &j);
    if (w == nullptr || !isfinite(lower) || !isfinite(upper))
    {
        return;
    }
    // A motor joint's two budgets are independent non-negatives; every
    // other type wants an ordered range.
    if (w->hv.jtype[j] == m3_motorJoint ? (lower < 0.0f || upper < 0.0f) : lower > upper)
    {
        return;
    }
    JointCommand(w, jointId, j, M3_OP_JOINT_SET_LIMITS, enable ? 1u : 0u, lower, upper,
                 m3IdentityQuat());
}

extern "C" void m3Joint_SetMotor(m3JointId jointId, bool enable, float speed, float maxEffort)
{
    int32_t j;
    m3HostWorld* w = JointForWrite(jointId, &j);
    if (w == nullptr || !isfinite(speed) || !isfinite(maxEffort) || maxEffort < 0.0f)
    {
        return;
    }
    JointCommand(w, jointId, j, M3_OP_JOINT_SET_MOTOR, enable ? 1u : 0u, speed, maxEffort,
                 m3IdentityQuat());
}

extern "C" void m3Joint_SetCollideConnected(m3JointId jointId, bool collide)
{
    int32_t j;
    m3HostWorld* w = JointForWrite(jointId, &j);
    if (w != nullptr)
    {
        JointCommand(w, jointId, j, M3_OP_JOINT_SET_COLLIDE, collide ? 1u : 0u, 0.0f, 0.0f,
                     m3IdentityQuat());
    }
}

extern "C" bool m3Joint_GetCollideConnected(m3JointId jointId)
{
    int32_t j;
    m3HostWorld* w = ResolveJoint(jointId, &j);
    return w != nullptr && m3gpuSyncHost(w) == M3GPU_OK && w->hv.jcollide[j] != 0;
}

// The types whose spring drives a target (joint.c:1031-1036).
static bool JointTypeDrives(uint8_t type)
{
    return type == m3_revoluteJoint || type == m3_prismaticJoint || type == m3_sphericalJoint ||
           type == m3_wheelJoint || type == m3_motorJoint;
}

extern "C" void m3Joint_SetSpring(m3JointId jointId, bool enable, float hertz, float dampingRatio)
{
    int32_t j;
    m3HostWorld* w = JointForWrite(jointId, &j);
    if (w == nullptr || !JointTypeDrives(w->hv.jtype[j]) || !isfinite(hertz) || hertz <= 0.0f ||
        !isfinite(dampingRatio) || dampingRatio < 0.0f)
    {
        return;
    }
    JointCommand(w, jointId, j, M3_OP_JOINT_SET_SPRING, enable ? 1u : 0u, hertz, dampingRatio,
                 m3IdentityQuat());
}

extern "C" void m3Joint_SetTargetAngle(m3JointId jointId, float radians)
{
    int32_t j;
    m3HostWorld* w = JointForWrite(jointId, &j);
    if (w == nullptr || w->hv.jtype[j] != m3_revoluteJoint || !isfinite(radians) ||
        radians < -M3_PI || radians > M3_PI)
    {
        return;
    }
    JointCommand(w, jointId, j, M3_OP_JOINT_SET_TARGET, 0u, radians, 0.0f, m3IdentityQuat());
}

extern "C" void m3Joint_SetTargetTranslation(m3JointId jointId, float meters)
{
    int32_t j;
    m3HostWorld* w = JointForWrite(jointId, &j);
    if (w == nullptr ||
        (w->hv.jtype[j] != m3_prismaticJoint && w->hv.jtype[j] != m3_wheelJoint) ||
        !isfinite(meters))
    {
        return;
    }
    JointCommand(w, jointId, j, M3_OP_JOINT_SET_TARGET, 0u, meters, 0.0f, m3IdentityQuat());
}

extern "C" void m3Joint_SetTargetRotation(m3JointId jointId, m3Quat target)
{
    int32_t j;
    m3HostWorld* w = JointForWrite(jointId, &j);
    if (w == nullptr || w->hv.jtype[j] != m3_sphericalJoint || !FiniteQuat(target))
    {
        return;
    }
    const m3real len2 =
        target.x * target.x + target.y * target.y + target.z * target.z + target.w * target.w;
    if (len2 < 0.99f || len2 > 1.01f)
    {
        return;
    }
    JointCommand(w, jointId, j, M3_OP_JOINT_SET_TARGET, 0u, 0.0f, 0.0f, target);
}

// The twist of B's frame about A's frame z, doubled: the revolute (and
// wheel) angle (joint.c:968-983).
extern "C" m3real m3Joint_GetAngle(m3JointId jointId)
{
    int32_t j;
    m3HostWorld* w = ResolveJoint(jointId, &j);
    if (w == nullptr || m3gpuSyncHost(w) != M3GPU_OK ||
        (w->hv.jtype[j] != m3_revoluteJoint && w->hv.jtype[j] != m3_wheelJoint))
    {
        return 0.0f;
    }
    const m3WorldView& v = w->hv;
    const m3Quat qA = m3MulQuat(v.xf[v.jbodyA[j]].q, v.jframeA[j]);
    const m3Quat qB = m3MulQuat(v.xf[v.jbodyB[j]].q, v.jframeB[j]);
    const m3Quat rel = m3MulQuat(m3Quat{-qA.x, -qA.y, -qA.z, qA.w}, qB);
    const m3real twist = rel.w < 0.0f ? m3Atan2(-rel.z, -rel.w) : m3Atan2(rel.z, rel.w);
    return 2.0f * twist;
}

// The anchor separation along the slide axis: frame z for the prismatic,
// frame x for the wheel (joint.c:985-1011).
extern "C" m3real m3Joint_GetTranslation(m3JointId jointId)
{
    int32_t j;
    m3HostWorld* w = ResolveJoint(jointId, &j);
    if (w == nullptr || m3gpuSyncHost(w) != M3GPU_OK ||
        (w->hv.jtype[j] != m3_prismaticJoint && w->hv.jtype[j] != m3_wheelJoint))
    {
        return 0.0f;
    }
    const m3WorldView& v = w->hv;
    const m3Transform xfA = v.xf[v.jbodyA[j]];
    const m3Transform xfB = v.xf[v.jbodyB[j]];
    const m3Vec3 pA = m3RotateVec3(xfA.q, v.jlocalA[j]);
    const m3Vec3 pB = m3RotateVec3(xfB.q, v.jlocalB[j]);
    const m3Vec3 d = v3((m3real)(xfB.p.x + (double)pB.x - xfA.p.x - (double)pA.x),
                        (m3real)(xfB.p.y + (double)pB.y - xfA.p.y - (double)pA.y),
                        (m3real)(xfB.p.z + (double)pB.z - xfA.p.z - (double)pA.z));
    const m3Quat frame = m3MulQuat(xfA.q, v.jframeA[j]);
    const m3Vec3 local = v.jtype[j] == m3_wheelJoint ? v3(1.0f, 0.0f, 0.0f) : v3(0.0f, 0.0f, 1.0f);
    return m3Dot3(d, m3RotateVec3(frame, local));
}

// ---------------------------------------------------------------------
// World settings (world.c:734-1117, world.h:92-176, 288): each public
// setter validates its arguments as the reference's does, records its
// journal record, and changes the world's scalars on the host image (the
// next step uploads them).  The journal replay applies the same records
// through m3ApplyWorldSetting.
// ---------------------------------------------------------------------
void m3ApplyWorldSetting(m3HostWorld* w, int32_t op, const float* f)
{
    m3WorldView& v = w->hv;
    m3WorldScalars* sc = v.sc;
    switch (op)
    {
    case M3_OP_SET_GRAVITY:
        sc->gravity = v3(f[0], f[1], f[2]);
        break;
    case M3_OP_SET_CONTACT_TUNING:
        sc->contactHertz = f[0];
        sc->contactDampingRatio = f[1];
        sc->contactPushMaxSpeed = f[2];
        break;
    case M3_OP_SET_RESTITUTION_THRESHOLD:
        sc->restitutionThreshold = f[0];
        break;
    case M3_OP_SET_MAXIMUM_LINEAR_SPEED:
        sc->maximumLinearSpeed = f[0];
        break;
    case M3_OP_SET_MAXIMUM_ANGULAR_SPEED:
        sc->maximumAngularSpeed = f[0];
        break;
    case M3_OP_SET_HIT_EVENT_THRESHOLD:
        sc->hitEventThreshold = f[0];
        break;
    case M3_OP_ENABLE_SLEEPING:
    case M3_OP_ENABLE_CONTINUOUS:
    {
        int32_t on;
        memcpy(&on, &f[0], sizeof(on));
        if (op == M3_OP_ENABLE_CONTINUOUS)
        {
            sc->continuousEnabled = on != 0 ? 1 : 0;
            break;
        }
        sc->sleepEnabled = on != 0 ? 1 : 0;
        if (on == 0)
        {
            // Sleeping turned off wakes every sleeping dynamic body
            // (world.c:761-778, body.c:316-322).
            for (int32_t i = 0; i < sc->bodyMax; ++i)
            {
                if (v.bodyAlive[i] != 0 && v.awake[i] == 0 && v.btype[i] == M3_BODY_DYNAMIC)
                {
                    v.awake[i] = 1;
                    v.sleepTime[i] = 0.0f;
                }
            }
        }
        break;
    }
    case M3_OP_SET_WIND:
        // The phase survives a retune (world.c:1075-1082).
        sc->windDir = v3(f[0], f[1], f[2]);
        sc->windSpeed = f[3];
        sc->windGustHertz = f[4];
        sc->windGustScale = f[5];
        break;
    default:
        break;
    }
}

// A world whose host image may change: the device's state read back first.
static m3HostWorld* SettingWorld(m3WorldId worldId)
{
    m3gpuClearError();
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr || m3gpuSyncHost(w) != M3GPU_OK)
    {
        return nullptr;
    }
    return w;
}

static void ApplySetting(m3HostWorld* w, int32_t op, const float* words, int32_t count)
{
    m3JournalAppend(w, op, words, (int32_t)sizeof(float) * count);
    m3ApplyWorldSetting(w, op, words);
    w->hostDirty = true;
}

extern "C" void m3World_SetGravity(m3WorldId worldId, m3Vec3 gravity)
{
    if (!FiniteV3(gravity))
    {
        return;
    }
    m3HostWorld* w = SettingWorld(worldId);
    if (w != nullptr)
    {
        const float words[3] = {gravity.x, gravity.y, gravity.z};
        ApplySetting(w, M3_OP_SET_GRAVITY, words, 3);
    }
}

extern "C" m3Vec3 m3World_GetGravity(m3WorldId worldId)
{
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    return w != nullptr ? w->hv.sc->gravity : v3(0.0f, 0.0f, 0.0f);
}

extern "C" void m3World_SetContactTuning(m3WorldId worldId, float hertz, float dampingRatio,
                                         float pushMaxSpeed)
{
    if (!FiniteF(hertz) || hertz <= 0.0f || !FiniteF(dampingRatio) || dampingRatio <= 0.0f ||
        !FiniteF(pushMaxSpeed) || pushMaxSpeed <= 0.0f)
    {
        return;
    }
    m3HostWorld* w = SettingWorld(worldId);
    if (w != nullptr)
    {
        const float words[3] = {hertz, dampingRatio, pushMaxSpeed};
        ApplySetting(w, M3_OP_SET_CONTACT_TUNING, words, 3);
    }
}

// One float setting: `strict` refuses zero as well as negatives.
static void FloatSetting(m3WorldId worldId, int32_t op, float value, bool strict)
{
    if (!FiniteF(value) || value < 0.0f || (strict && value == 0.0f))
    {
        return;
    }
    m3HostWorld* w = SettingWorld(worldId);
    if (w != nullptr)
    {
        ApplySetting(w, op, &value, 1);
    }
}

extern "C" void m3World_SetRestitutionThreshold(m3WorldId worldId, float value)
{
    FloatSetting(worldId, M3_OP_SET_RESTITUTION_THRESHOLD, value, false);
}

extern "C" void m3World_SetMaximumLinearSpeed(m3WorldId worldId, float value)
{
    FloatSetting(worldId, M3_OP_SET_MAXIMUM_LINEAR_SPEED, value, true);
}

extern "C" void m3World_SetMaximumAngularSpeed(m3WorldId worldId, float value)
{
    FloatSetting(worldId, M3_OP_SET_MAXIMUM_ANGULAR_SPEED, value, true);
}

extern "C" void m3World_SetHitEventThreshold(m3WorldId worldId, float value)
{
    FloatSetting(worldId, M3_OP_SET_HIT_EVENT_THRESHOLD, value, false);
}

static void FlagSetting(m3WorldId worldId, int32_t op, bool flag)
{
    m3HostWorld* w = SettingWorld(worldId);
    if (w != nullptr)
    {
        const int32_t on = flag ? 1 : 0;
        float word;
        memcpy(&word, &on, sizeof(word));
        ApplySetting(w, op, &word, 1);
    }
}

extern "C" void m3World_EnableSleeping(m3WorldId worldId, bool flag)
{
    FlagSetting(worldId, M3_OP_ENABLE_SLEEPING, flag);
}

extern "C" bool m3World_IsSleepingEnabled(m3WorldId worldId)
{
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    return w != nullptr && w->hv.sc->sleepEnabled != 0;
}

extern "C" void m3World_EnableContinuous(m3WorldId worldId, bool flag)
{
    FlagSetting(worldId, M3_OP_ENABLE_CONTINUOUS, flag);
}

extern "C" bool m3World_IsContinuousEnabled(m3WorldId worldId)
{
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    return w != nullptr && w->hv.sc->continuousEnabled != 0;
}

extern "C" void m3World_SetWind(m3WorldId worldId, m3Vec3 direction, float speed, float gustHertz,
                                float gustScale)
{
    if (!FiniteV3(direction) || !FiniteF(speed) || speed < 0.0f || !FiniteF(gustHertz) ||
        gustHertz < 0.0f || !FiniteF(gustScale) || gustScale < 0.0f)
    {
        return;
    }
    if (speed > 0.0f)
    {
        // A blowing wind demands a near-unit direction.
        const m3real len2 = m3Dot3(direction, direction);
        if (len2 < 0.99f || len2 > 1.01f)
        {
            return;
        }
    }
    m3HostWorld* w = SettingWorld(worldId);
    if (w != nullptr)
    {
        const float words[6] = {direction.x, direction.y, direction.z, speed, gustHertz, gustScale};
        ApplySetting(w, M3_OP_SET_WIND, words, 6);
    }
}

// White-box hook for the tests: one broadphase tree move on the host
// image, as the step's tree kernel makes it (remove the shape's leaf,
// insert `lo`..`hi`).  Returns the new leaf, or -1.
extern "C" int32_t m3gpu_tree_move(m3WorldId worldId, int32_t shape, const double* lo,
                                   const double* hi)
{
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr || lo == nullptr || hi == nullptr || m3gpuSyncHost(w) != M3GPU_OK)
    {
        return -1;
    }
    m3WorldView& v = w->hv;
    if (shape < 0 || shape >= v.sc->shapeMax || v.proxyId[shape] == M3_TREE_NULL)
    {
        return -1;
    }
    const m3TreeRef tree = m3WorldTree(v);
    const m3TreeArrayStore store{v.treeNodes};
    m3TreeRemove(tree, store, v.proxyId[shape]);
    v.proxyId[shape] = m3TreeInsert(tree, store, lo, hi, shape);
    w->hostDirty = true;
    return v.proxyId[shape];
}

extern "C" bool m3Joint_IsValid(m3JointId jointId)
{
    m3HostWorld* w = m3gpuWorldFromIndex0(jointId.world0);
    int32_t index = jointId.index1 - 1;
    // The step may have broken the joint on the device.
    if (w != nullptr && m3gpuSyncHost(w) != M3GPU_OK)
    {
        return false;
    }
    return w != nullptr && index >= 0 && index < w->hv.sc->jointMax &&
           w->hv.jointAlive[index] != 0 && w->hv.jointGen[index] == jointId.generation;
}
