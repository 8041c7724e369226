/*
 * maul3d_b200 — B200-native step path for the Maul3D rigid-body engine.
 *
 * This header is the drop-in C ABI.  Every function in section 2 keeps the
 * name, signature, argument meaning and error behaviour of the reference
 * engine's public API (the file:line of the declaration it replaces is
 * given beside each one), so a host program written against the
 * reference's include/maul3d/*.h for the features covered here links
 * against libmaul3d_b200.so unchanged.  Section 3 adds the batched and
 * device-management entries the reference has no counterpart for.
 *
 * Value types and definition structs are laid out byte-for-byte like the
 * reference's (include/maul3d/math.h:26-66, base.h:69-106, world.h:43-80,
 * body.h:21-39, shape.h:25-107, joint.h:85-132); the layouts are checked
 * against the reference build by the parity tests.
 *
 * Plain pointers and sizes only; no torch or CUDA types cross this ABI.
 */
#ifndef MAUL3D_B200_H
#define MAUL3D_B200_H

#include <stdbool.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define M3GPU_API __attribute__((visibility("default"))) extern
#else
#define M3GPU_API extern
#endif

/* ---------------------------------------------------------------------
 * 1. Value types (include/maul3d/math.h:26-66, base.h:69-106)
 * ------------------------------------------------------------------- */
typedef float m3real;
#define M3_PI 3.14159265358979323846f
#define M3_HASH_INIT 0xCBF29CE484222325ull

typedef struct m3Vec3 { m3real x, y, z; } m3Vec3;
typedef struct m3Pos3 { double x, y, z; } m3Pos3;
typedef struct m3Quat { m3real x, y, z, w; } m3Quat;
typedef struct m3Transform { m3Pos3 p; m3Quat q; } m3Transform;
typedef struct m3Mat3 { m3Vec3 cx, cy, cz; } m3Mat3;

typedef struct m3WorldId { int32_t index1; uint16_t generation; } m3WorldId;
typedef struct m3BodyId { int32_t index1; uint16_t world0; uint16_t generation; } m3BodyId;
typedef struct m3ShapeId { int32_t index1; uint16_t world0; uint16_t generation; } m3ShapeId;
typedef struct m3JointId { int32_t index1; uint16_t world0; uint16_t generation; } m3JointId;

typedef enum m3BodyType { m3_staticBody = 0, m3_kinematicBody = 1, m3_dynamicBody = 2 } m3BodyType;

typedef enum m3ShapeType {
    m3_sphereShape = 0,
    m3_planeShape = 1,
    m3_hullShape = 2,
    m3_capsuleShape = 3,
    m3_meshShape = 4,
    m3_voxelShape = 5,
    m3_heightFieldShape = 6
} m3ShapeType;

typedef enum m3JointType {
    m3_sphericalJoint = 0,
    m3_revoluteJoint = 1,
    m3_prismaticJoint = 2,
    m3_fixedJoint = 3,
    m3_distanceJoint = 4,
    m3_genericJoint = 5,
    m3_wheelJoint = 6,
    m3_filterJoint = 7,
    m3_parallelJoint = 8,
    m3_motorJoint = 9,
    m3_gearJoint = 10,
    m3_pulleyJoint = 11
} m3JointType;

/* Task hooks (world.h:15-26).  Accepted for ABI compatibility; the device
 * path ignores them (parallelism comes from the GPU, not host threads). */
typedef void m3TaskFn(int32_t startIndex, int32_t endIndex, void* taskContext);
typedef void* m3EnqueueTaskFn(m3TaskFn* task, int32_t itemCount, int32_t minRange,
                              void* taskContext, void* userContext);
typedef void m3FinishTaskFn(void* userTask, void* userContext);

/* world.h:43-80 */
typedef struct m3WorldDef {
    m3Vec3 gravity;
    int32_t bodyCapacity;
    int32_t shapeCapacity;
    int32_t meshCapacity;
    int32_t jointCapacity;
    int32_t voxelCapacity;
    int32_t characterCapacity;
    int32_t vehicleCapacity;
    int32_t softBodyCapacity;
    int32_t workerCount;
    m3EnqueueTaskFn* enqueueTask;
    m3FinishTaskFn* finishTask;
    void* userTaskContext;
    float contactHertz;
    float contactDampingRatio;
    float contactPushMaxSpeed;
    float restitutionThreshold;
    float maximumLinearSpeed;
    int32_t enableSleeping;
    int32_t enableContinuous;
    float hitEventThreshold;
    int32_t internalValue;
} m3WorldDef;

/* body.h:21-39 */
typedef struct m3BodyDef {
    int32_t type;
    m3Pos3 position;
    m3Quat rotation;
    m3Vec3 linearVelocity;
    m3Vec3 angularVelocity;
    float gravityScale;
    float linearDamping;
    float angularDamping;
    uint64_t userData;
    bool isBullet;
    int32_t internalValue;
} m3BodyDef;

/* shape.h:25-38, 102-107 */
typedef struct m3Sphere { m3Vec3 center; m3real radius; } m3Sphere;
typedef struct m3Plane { m3Vec3 normal; m3real offset; } m3Plane;
typedef struct m3Capsule { m3Vec3 point1; m3Vec3 point2; m3real radius; } m3Capsule;

/* shape.h:40-74 */
typedef struct m3ShapeDef {
    float density;
    float friction;
    float restitution;
    uint64_t categoryBits;
    uint64_t maskBits;
    int32_t groupIndex;
    float rollingResistance;
    uint64_t userData;
    bool isSensor;
    bool enableHitEvents;
    bool enablePreSolveEvents;
    m3Vec3 localPosition;
    m3Quat localRotation;
    int32_t internalValue;
} m3ShapeDef;

/* joint.h:85-132 */
typedef struct m3JointDef {
    int32_t type;
    m3BodyId bodyA;
    m3BodyId bodyB;
    m3Vec3 localAnchorA;
    m3Vec3 localAnchorB;
    m3Vec3 localAxisA;
    m3Vec3 localAxisB;
    bool enableLimit;
    m3real lowerLimit;
    m3real upperLimit;
    bool enableMotor;
    m3real motorSpeed;
    m3real maxMotorEffort;
    bool enableCone;
    m3real coneAngle;
    bool collideConnected;
    uint8_t genericLinear[3];
    uint8_t genericAngular[3];
    uint8_t genericMotorAxis;
    uint8_t genericReserved;
    m3real genericLinearLower[3];
    m3real genericLinearUpper[3];
    m3real genericAngularLower[3];
    m3real genericAngularUpper[3];
    m3real ratio;
    m3Pos3 groundAnchorA;
    m3Pos3 groundAnchorB;
    int32_t internalValue;
} m3JointDef;

/* ---------------------------------------------------------------------
 * 2. Drop-in entry points (reference names and semantics)
 * ------------------------------------------------------------------- */

/* core.c:40 (base.h:38): major*10000 + minor*100 + patch of the engine
 * release whose step this library reproduces (1.22.0). */
M3GPU_API int m3GetVersion(void);

/* core.c:46 (base.h:110): FNV-1a 64 over `count` bytes. */
M3GPU_API uint64_t m3Hash64(uint64_t h, const void* bytes, int32_t count);

/* world.c:64 (world.h:88): pinned defaults; gravity (0,-10,0), 1024
 * bodies, 2048 shapes, 64 joints, tuning knobs at the reference values. */
M3GPU_API m3WorldDef m3DefaultWorldDef(void);
/* world.c:90 (world.h:92): null id on an invalid def or a full table. */
M3GPU_API m3WorldId m3CreateWorld(const m3WorldDef* def);
/* world.h:93 */
M3GPU_API void m3DestroyWorld(m3WorldId worldId);
/* world.h:94 */
M3GPU_API bool m3World_IsValid(m3WorldId worldId);

/* World settings (world.h:92, 134-176, 288; world.c:785-1117): the same
 * argument checks (a refused value is a no-op), the same journal records,
 * applied from the next step on.  Turning sleeping off wakes every
 * sleeping body.  A wind that blows needs a near-unit direction. */
M3GPU_API void m3World_SetGravity(m3WorldId worldId, m3Vec3 gravity);
M3GPU_API m3Vec3 m3World_GetGravity(m3WorldId worldId);
M3GPU_API void m3World_SetContactTuning(m3WorldId worldId, float hertz, float dampingRatio,
                                        float pushMaxSpeed);
M3GPU_API void m3World_SetRestitutionThreshold(m3WorldId worldId, float value);
M3GPU_API void m3World_SetMaximumLinearSpeed(m3WorldId worldId, float value);
M3GPU_API void m3World_SetMaximumAngularSpeed(m3WorldId worldId, float value);
M3GPU_API void m3World_EnableSleeping(m3WorldId worldId, bool flag);
M3GPU_API bool m3World_IsSleepingEnabled(m3WorldId worldId);
M3GPU_API void m3World_EnableContinuous(m3WorldId worldId, bool flag);
M3GPU_API bool m3World_IsContinuousEnabled(m3WorldId worldId);
M3GPU_API void m3World_SetHitEventThreshold(m3WorldId worldId, float value);
M3GPU_API void m3World_SetWind(m3WorldId worldId, m3Vec3 direction, float speed, float gustHertz,
                               float gustScale);

/* snapshot.c:603 (world.h:203): the exact byte count m3World_Snapshot
 * writes, -1 for a stale id. */
M3GPU_API int32_t m3World_SnapshotSize(m3WorldId worldId);
/* snapshot.c:613 (world.h:204): writes the world's snapshot (format
 * v54), byte for byte what the reference engine writes for the same
 * world: the persistent state including the broadphase tree and the id
 * pools.  Returns the size, or -1 for a stale id, a null buffer or a
 * capacity below m3World_SnapshotSize. */
M3GPU_API int32_t m3World_Snapshot(m3WorldId worldId, void* out, int32_t capacity);

/* snapshot.c:680 (world.h:205): restores a snapshot (format v54, taken
 * by the reference engine or by this library) into a world created with
 * the same capacities.  False, with the world untouched, on a foreign
 * format or build, mismatched capacities or corrupt content; false with
 * m3gpu_last_error() == M3GPU_ERR_UNSUPPORTED when the snapshot holds
 * content the device path does not model (meshes, voxels, heightfields,
 * characters, vehicles, soft bodies, water volumes). */
M3GPU_API bool m3World_Restore(m3WorldId worldId, const void* data, int32_t size);

/* world.c:1369-1398 (world.h:600-601): journal recording into the
 * caller's buffer: steps, velocity sets, forces, torques, impulses and
 * joint break thresholds are recorded in the reference's record formats.
 * End returns the byte count, or -1 after an overflow or after a call
 * this path does not record (body, shape or joint creation). */
M3GPU_API bool m3World_JournalBegin(m3WorldId worldId, void* buffer, int32_t capacity);
M3GPU_API int32_t m3World_JournalEnd(m3WorldId worldId);

/* world.c:3187 (world.h:606): replays a recorded command stream.  Steps
 * run on the GPU; velocity sets, forces, torques, impulses and joint
 * break thresholds apply between them.  The whole stream is validated first, so a refusal
 * leaves the world untouched; other ops are refused with
 * M3GPU_ERR_UNSUPPORTED. */
M3GPU_API bool m3World_JournalReplay(m3WorldId worldId, const void* data, int32_t size);

/* solver.c:4322 (world.h:195): one step of `dt` seconds in `substeps`
 * substeps, computed on the GPU.  Refuses (no-op) a stale id, dt <= 0 or
 * substeps outside [1, 256], like the reference.  A device-side refusal
 * (a capacity or feature the device path does not cover) is reported by
 * m3gpu_last_error(); the world is then marked failed, its state is
 * unspecified and every later step of it is refused the same way. */
M3GPU_API void m3World_Step(m3WorldId worldId, float dt, int32_t substeps);

/* snapshot.c:932 (world.h:510): FNV-1a over the curated world state,
 * bit-identical to the reference's hash for the same world. 0 for a
 * stale id. */
M3GPU_API uint64_t m3World_Hash(m3WorldId worldId);

/* world.h:531-554 (world.c:917-951): the world's live counts and the
 * last step's solver figures.  colorCount counts the non-empty graph
 * colours of the last step, the overflow colour included (17 when it was
 * used).  scratchPeak and scratchCapacity report the world's device
 * scratch bytes (the device step carves all of it each step);
 * allocCalls/freeCalls count the library's device block allocations and
 * frees.  Zeroes for a stale id. */
typedef struct m3Counters
{
    int32_t bodyCount;
    int32_t shapeCount;
    int32_t jointCount;
    int32_t contactCount;
    int32_t awakeCount;
    int32_t islandCount;
    int32_t colorCount;
    int32_t characterCount;
    int32_t vehicleCount;
    int32_t softBodyCount;
    int32_t voxelChunkCount;
    int32_t hullCount;
    int32_t meshCount;
    int32_t treeHeight;
    int32_t scratchPeak;
    int32_t scratchCapacity;
    int32_t snapshotBytes;
    int64_t allocCalls;
    int64_t freeCalls;
} m3Counters;
M3GPU_API m3Counters m3World_GetCounters(m3WorldId worldId);

/* world.h:578-593 (world.c:955-965): milliseconds of the world's last
 * step by phase, measured on the device with CUDA events around the
 * stages of the batch the world was stepped in: broadphase (bounds and
 * pairs), narrowphase, prepare (islands, colouring, constraint rows),
 * solve (the substep loop, restitution, store) and continuous (the
 * continuous phase and the sleep pass, one kernel); step is their sum.
 * Stages this path does not run report 0.  Zeroes before the first
 * device step and for a stale id. */
typedef struct m3Profile
{
    float step;
    float vehicles;
    float broadphase;
    float narrowphase;
    float events;
    float prepare;
    float solve;
    float continuous;
    float sleep;
    float characters;
    float softBodies;
} m3Profile;
M3GPU_API m3Profile m3World_GetProfile(m3WorldId worldId);

/* world.h:213-224 / world.c:1472-1500: contact begin and end events of the
 * world's LAST step, in the reference's canonical order (ascending pair
 * key over the union of the previous and the current pair lists): begin
 * when a pair's manifold gained points, end when it lost them or the pair
 * vanished; pairs with a sensor go to the sensor streams (world.h:260-263).
 * shapeA is the lower shape index.  Valid until the next step, restore or
 * destruction of the world; a restore clears them.  `count` must be
 * non-null (0 and NULL for a stale world). */
typedef struct m3ContactEvent {
    m3ShapeId shapeA;
    m3ShapeId shapeB;
} m3ContactEvent;
M3GPU_API const m3ContactEvent* m3World_ContactBeginEvents(m3WorldId worldId, int32_t* count);
M3GPU_API const m3ContactEvent* m3World_ContactEndEvents(m3WorldId worldId, int32_t* count);
M3GPU_API const m3ContactEvent* m3World_SensorBeginEvents(m3WorldId worldId, int32_t* count);
M3GPU_API const m3ContactEvent* m3World_SensorEndEvents(m3WorldId worldId, int32_t* count);

/* world.h:302-311 / world.c:1063: the joints the last step broke, in the
 * order it destroyed them (ascending joint index), each with the id it had
 * (already stale when read). */
typedef struct m3JointBreakEvent {
    m3JointId joint;
} m3JointBreakEvent;
M3GPU_API const m3JointBreakEvent* m3World_JointBreakEvents(m3WorldId worldId, int32_t* count);

/* world.h:265-285 / solver.c:2987-3033: hit events of the last step, in
 * contact constraint order: at most one per contact whose shapes include
 * one that enabled hit events, for its fastest-approaching point whose
 * approach beat the world's hit threshold and whose impulse fired.  point
 * is the contact point on shape A's body in world space, normal runs from
 * A to B.  At most the world's pair capacity; the rest are counted by
 * m3World_HitEventsDropped. */
typedef struct m3HitEvent {
    m3ShapeId shapeA;
    m3ShapeId shapeB;
    m3Pos3 point;
    m3Vec3 normal;
    m3real approachSpeed;
} m3HitEvent;
M3GPU_API const m3HitEvent* m3World_HitEvents(m3WorldId worldId, int32_t* count);
M3GPU_API int32_t m3World_HitEventsDropped(m3WorldId worldId);

/* world.h:287-300 / solver.c:4295-4306: one event per body the last step
 * moved (every mover, ascending body index) with its transform after the
 * step; fellAsleep marks the step its island fell asleep. */
typedef struct m3BodyMoveEvent {
    m3BodyId body;
    m3Transform transform;
    bool fellAsleep;
} m3BodyMoveEvent;
M3GPU_API const m3BodyMoveEvent* m3World_BodyMoveEvents(m3WorldId worldId, int32_t* count);

/* body.c:35 (body.h:43) / body.h:49 / body.h:56-59 */
M3GPU_API m3BodyDef m3DefaultBodyDef(void);
M3GPU_API m3BodyId m3CreateBody(m3WorldId worldId, const m3BodyDef* def);
M3GPU_API bool m3Body_IsValid(m3BodyId bodyId);
M3GPU_API m3Pos3 m3Body_GetPosition(m3BodyId bodyId);
M3GPU_API m3Quat m3Body_GetRotation(m3BodyId bodyId);
M3GPU_API m3Vec3 m3Body_GetLinearVelocity(m3BodyId bodyId);
M3GPU_API m3Vec3 m3Body_GetAngularVelocity(m3BodyId bodyId);
/* body.h: awake query (dynamic bodies sleep; others report true) */
M3GPU_API bool m3Body_IsAwake(m3BodyId bodyId);
/* body.c:910-958 (body.h:117-121): a force or impulse at a world point
 * (dynamic bodies with mass only; a non-finite argument is a no-op);
 * body.c:639-703 (body.h:86-94): the six motion-lock bits (others are
 * refused) and the spin-cap escape, each journaled like the reference's;
 * body.c:514-527, 632 (body.h:64-70): type, user data and enabled flag. */
M3GPU_API void m3Body_ApplyForceAtPoint(m3BodyId bodyId, m3Vec3 force, m3Pos3 point);
M3GPU_API void m3Body_ApplyLinearImpulseAtPoint(m3BodyId bodyId, m3Vec3 impulse, m3Pos3 point);
M3GPU_API void m3Body_SetMotionLocks(m3BodyId bodyId, uint32_t locks);
M3GPU_API uint32_t m3Body_GetMotionLocks(m3BodyId bodyId);
M3GPU_API void m3Body_SetAllowFastRotation(m3BodyId bodyId, bool allow);
M3GPU_API bool m3Body_GetAllowFastRotation(m3BodyId bodyId);
M3GPU_API m3BodyType m3Body_GetType(m3BodyId bodyId);
M3GPU_API uint64_t m3Body_GetUserData(m3BodyId bodyId);
M3GPU_API bool m3Body_IsEnabled(m3BodyId bodyId);
/* body.c:170-330, 531-637, 763-823 (body.h:64-106): runtime control,
 * each journaled like the reference's.  A teleport or a pose target needs
 * a finite position and a near-unit rotation (targets: kinematic bodies
 * only); a teleport, a type change or an enable switch wakes the sleeping
 * dynamic bodies around the body; a type change to dynamic rebuilds the
 * mass from the body's shapes; sleep controls refuse a negative or
 * non-finite threshold; forced sleep or wake reaches dynamic bodies only. */
M3GPU_API void m3Body_SetTransform(m3BodyId bodyId, m3Pos3 position, m3Quat rotation);
M3GPU_API void m3Body_SetTargetTransform(m3BodyId bodyId, m3Pos3 position, m3Quat rotation);
M3GPU_API void m3Body_SetType(m3BodyId bodyId, m3BodyType type);
M3GPU_API void m3Body_SetEnabled(m3BodyId bodyId, bool enabled);
M3GPU_API void m3Body_SetSleepControls(m3BodyId bodyId, float threshold, bool canSleep);
M3GPU_API void m3Body_SetAwake(m3BodyId bodyId, bool awake);
/* body.c:711-760 (body.h:95-96): a debug name of at most 31 bytes (longer
 * ones are truncated), journaled and saved in snapshots, never hashed.
 * GetName returns "" for a stale id; the pointer stays valid until the
 * name changes, the world is restored or the world is destroyed. */
M3GPU_API void m3Body_SetName(m3BodyId bodyId, const char* name);
M3GPU_API const char* m3Body_GetName(m3BodyId bodyId);

/* body.h:115-123 (body.c:818-1014): commands between steps.  Forces,
 * torques and impulses act on dynamic bodies with mass; velocity sets on
 * any live body; a nonzero command (any velocity set) wakes the body.
 * Stale ids and non-finite vectors are no-ops. */
M3GPU_API void m3Body_ApplyForce(m3BodyId bodyId, m3Vec3 force);
M3GPU_API void m3Body_ApplyTorque(m3BodyId bodyId, m3Vec3 torque);
M3GPU_API void m3Body_ApplyLinearImpulse(m3BodyId bodyId, m3Vec3 impulse);
M3GPU_API void m3Body_ApplyAngularImpulse(m3BodyId bodyId, m3Vec3 impulse);
M3GPU_API void m3Body_SetLinearVelocity(m3BodyId bodyId, m3Vec3 velocity);
M3GPU_API void m3Body_SetAngularVelocity(m3BodyId bodyId, m3Vec3 velocity);

/* shape.c:31 (shape.h:78) and the creators shape.c:763/782/802/1334 */
M3GPU_API m3ShapeDef m3DefaultShapeDef(void);
M3GPU_API m3ShapeId m3CreateSphereShape(m3BodyId bodyId, const m3ShapeDef* def,
                                        const m3Sphere* sphere);
M3GPU_API m3ShapeId m3CreatePlaneShape(m3BodyId bodyId, const m3ShapeDef* def,
                                       const m3Plane* plane);
M3GPU_API m3ShapeId m3CreateCapsuleShape(m3BodyId bodyId, const m3ShapeDef* def,
                                         const m3Capsule* capsule);
/* shape.c:988-1030 (shape.h:143-149): convex hull of 4-256 points
 * (QuickHull, bit-identical slab to the reference's); null for a stale
 * body or def, no points, a non-finite point or a degenerate cloud. */
M3GPU_API m3ShapeId m3CreateHullShape(m3BodyId bodyId, const m3ShapeDef* def,
                                      const m3Vec3* points, int32_t count);
M3GPU_API m3ShapeId m3CreateBoxShape(m3BodyId bodyId, const m3ShapeDef* def,
                                     m3Vec3 halfExtents);
/* Replaces m3CreateHeightFieldGridShape (include/maul3d/shape.h:194-202,
 * shape.c:1175-1262): a native grid heightfield of nx x nz samples
 * (2..255 each way, x fastest, `cellSize` apart) on a static body, its
 * minimum corner at the shape's origin.  Null id on invalid input. */
M3GPU_API m3ShapeId m3CreateHeightFieldGridShape(m3BodyId bodyId, const m3ShapeDef* def,
                                                 const float* heights, int32_t nx, int32_t nz,
                                                 float cellSize);
M3GPU_API bool m3Shape_IsValid(m3ShapeId shapeId);
/* shape.c:1351-1363 (shape.h:271): the body that carries the shape; a
 * null id for a stale shape. */
M3GPU_API m3BodyId m3Shape_GetBody(m3ShapeId shapeId);
/* Materials and flags (shape.c:1387-1410, 1463-1600; shape.h:286-303),
 * each journaled like the reference's.  Friction, restitution and rolling
 * resistance must be finite and not negative, a density finite and
 * positive (the body's mass is rebuilt from its shapes when asked); a
 * refused value is a no-op.  Getters read 0 (false) for a stale shape. */
M3GPU_API void m3Shape_SetFriction(m3ShapeId shapeId, float friction);
M3GPU_API float m3Shape_GetFriction(m3ShapeId shapeId);
M3GPU_API void m3Shape_SetRestitution(m3ShapeId shapeId, float restitution);
M3GPU_API float m3Shape_GetRestitution(m3ShapeId shapeId);
M3GPU_API void m3Shape_SetRollingResistance(m3ShapeId shapeId, float value);
M3GPU_API float m3Shape_GetRollingResistance(m3ShapeId shapeId);
M3GPU_API void m3Shape_SetDensity(m3ShapeId shapeId, float density, bool updateBodyMass);
M3GPU_API float m3Shape_GetDensity(m3ShapeId shapeId);
M3GPU_API void m3Shape_EnableHitEvents(m3ShapeId shapeId, bool flag);
M3GPU_API bool m3Shape_AreHitEventsEnabled(m3ShapeId shapeId);
M3GPU_API void m3Shape_EnablePreSolve(m3ShapeId shapeId, bool flag);
M3GPU_API bool m3Shape_IsPreSolveEnabled(m3ShapeId shapeId);

/* world.h:512-524 */
typedef struct m3ContactData {
    m3ShapeId shapeA;
    m3ShapeId shapeB;
    m3Vec3 normal; /* from shape A toward shape B */
    int32_t pointCount;
    m3Pos3 points[4];
    float separations[4];
    float normalImpulses[4];
} m3ContactData;
/* query.c:1330-1409 (body.h:99, shape.h:274): up to `capacity` entries,
 * one per manifold with points touching the body or shape, in the
 * current pair list's order; points are body A's centre of mass plus the
 * anchor.  0 for a stale id, a null `out` or a non-positive capacity. */
M3GPU_API int32_t m3Body_GetContactData(m3BodyId bodyId, m3ContactData* out, int32_t capacity);
M3GPU_API int32_t m3Shape_GetContactData(m3ShapeId shapeId, m3ContactData* out, int32_t capacity);

/* joint.c:15 (joint.h:134) and joint.h:136: spherical, revolute and
 * fixed joints are stepped on the device. */
M3GPU_API m3JointDef m3DefaultJointDef(void);
M3GPU_API m3JointId m3CreateJoint(const m3JointDef* def);
/* joint.c:914 (joint.h:216): breaking thresholds in N and N*m (0 = no
 * limit); a joint whose reaction exceeds one is destroyed by the step,
 * in ascending joint order, and its slot is recycled.  Wakes the joint's
 * dynamic bodies.  Negative or non-finite values are refused (no-op). */
M3GPU_API void m3Joint_SetBreakThresholds(m3JointId jointId, float maxForce, float maxTorque);
M3GPU_API bool m3Joint_IsValid(m3JointId jointId);
/* Drives and switches (joint.c:548-624, 732-1129; joint.h:183-248), each
 * journaled like the reference's and waking the joint's dynamic bodies:
 * limits (finite and ordered; a toggled or moved limit drops its stored
 * row impulses), motor (finite speed, finite non-negative effort),
 * collide-connected, spring (revolute, prismatic, spherical, wheel and
 * motor joints; finite positive hertz, finite non-negative damping ratio)
 * and drive targets (an angle in [-pi, pi] for a revolute joint, a
 * translation for a prismatic or wheel joint, a unit rotation for a
 * spherical joint).  A refused value is a no-op.  The angle and
 * translation getters read the current poses (0 for other types). */
M3GPU_API void m3Joint_SetLimits(m3JointId jointId, bool enable, float lower, float upper);
M3GPU_API void m3Joint_SetMotor(m3JointId jointId, bool enable, float speed, float maxEffort);
M3GPU_API void m3Joint_SetCollideConnected(m3JointId jointId, bool collide);
M3GPU_API bool m3Joint_GetCollideConnected(m3JointId jointId);
M3GPU_API void m3Joint_SetSpring(m3JointId jointId, bool enable, float hertz, float dampingRatio);
M3GPU_API void m3Joint_SetTargetAngle(m3JointId jointId, float radians);
M3GPU_API void m3Joint_SetTargetTranslation(m3JointId jointId, float meters);
M3GPU_API void m3Joint_SetTargetRotation(m3JointId jointId, m3Quat target);
M3GPU_API m3real m3Joint_GetAngle(m3JointId jointId);
M3GPU_API m3real m3Joint_GetTranslation(m3JointId jointId);

/* ---------------------------------------------------------------------
 * 3. Device extensions (no reference counterpart)
 * ------------------------------------------------------------------- */

/* Error codes reported by m3gpu_last_error(). */
#define M3GPU_OK 0
#define M3GPU_ERR_INVALID 1      /* bad argument or stale id */
#define M3GPU_ERR_CUDA 2         /* a CUDA call failed (message available) */
#define M3GPU_ERR_CAPACITY 3     /* pair table full: the world stalled */
#define M3GPU_ERR_UNSUPPORTED 4  /* a feature the device path does not cover */
#define M3GPU_ERR_NO_DEVICE 5    /* no CUDA device visible */

/* replay.h:28-62 (replay.c): the M3J1 replay container, a snapshot and
 * the journal recorded after it.  Pure memory codecs, same layout,
 * validation and refusals as the reference's. */
typedef struct m3JournalInfo { int32_t opCount; int32_t stepCount; } m3JournalInfo;
typedef struct m3ReplayView {
    const void* snapshot;
    int32_t snapshotBytes;
    const void* journal;
    int32_t journalBytes;
    uint64_t finalHash;
    m3JournalInfo info;
} m3ReplayView;
M3GPU_API bool m3JournalDescribe(const void* journal, int32_t bytes, m3JournalInfo* out);
M3GPU_API int32_t m3ReplayEncodeSize(int32_t snapshotBytes, int32_t journalBytes);
M3GPU_API int32_t m3ReplayEncode(const void* snapshot, int32_t snapshotBytes, const void* journal,
                                 int32_t journalBytes, uint64_t finalHash, void* out,
                                 int32_t capacity);
M3GPU_API bool m3ReplayDecode(const void* data, int32_t bytes, m3ReplayView* out);

/* Last error raised on the calling thread's most recent m3gpu or drop-in
 * call, and a one-line message for it (never NULL). */
M3GPU_API int32_t m3gpu_last_error(void);
M3GPU_API const char* m3gpu_last_error_message(void);

/* Step `count` independent worlds `steps` times each in ONE batched
 * launch sequence (one CTA per world in the per-world stages, the
 * flattened pairs of every world in the narrowphase).
 * Equivalent, world by world and bit for bit, to calling m3World_Step on
 * each world in turn.  Returns M3GPU_OK or an error code; on error no
 * world is partially stepped past the failing step. */
M3GPU_API int32_t m3gpu_step_worlds(const m3WorldId* worlds, int32_t count, float dt,
                                    int32_t substeps, int32_t steps);

/* World hashes of `count` worlds computed on the device (one block per
 * world), written to out[i].  Same values as m3World_Hash. */
M3GPU_API int32_t m3gpu_hash_worlds(const m3WorldId* worlds, int32_t count, uint64_t* out);

/* Select the CUDA device this library uses in the calling process (one
 * process per GPU).  Call before the first device operation. */
M3GPU_API int32_t m3gpu_set_device(int32_t device);

/* Allocate the HBM slabs of `count` worlds without copying anything, so
 * a later upload or step times only the copies and the work. */
M3GPU_API int32_t m3gpu_reserve_worlds(const m3WorldId* worlds, int32_t count);

/* Copy the host images of `count` worlds to their HBM slabs (worlds
 * whose device copy is already current are skipped). */
M3GPU_API int32_t m3gpu_upload_worlds(const m3WorldId* worlds, int32_t count);

/* Bytes one world's host image occupies (an upload copies the part
 * before the pair buffers, the current pair list and the hulls). */
M3GPU_API int64_t m3gpu_world_image_bytes(m3WorldId world);

/* Host-to-device bytes copied by world uploads since the library was
 * loaded. */
M3GPU_API int64_t m3gpu_uploaded_bytes(void);

/* Allocation-free step of one resident world (no reference counterpart).
 * For callers that must not allocate device memory when they step: a
 * frame loop with a hard deadline (allocating and freeing can stall the
 * whole device), or a host whose device memory belongs to its own pool
 * allocator.  The
 * world must already be resident (m3gpu_reserve_worlds and
 * m3gpu_upload_worlds, called earlier when allocating was allowed); the
 * step then allocates nothing: its scratch lives in a fixed 4 MiB
 * device array (held by every GPU that loads the library until exit).
 * Worlds whose scratch exceeds that, or with more than about 800 bodies,
 * are refused with M3GPU_ERR_CAPACITY before any device work.  The first
 * call on a device looks up that array's address; make it before any
 * stream capture.  The call uses blocking copies on the legacy default
 * stream, so it must not run while any stream of the process is being
 * captured.  Calls share the array: the library serialises the calls of
 * one process, and calls that overlapped on the GPU would race.  Same
 * result, bit for bit, as m3gpu_step_worlds on the same world. */
M3GPU_API int32_t m3gpu_step_world_noalloc(m3WorldId world, float dt, int32_t substeps);

/* The broadphase tree (no reference counterpart): the tree is state only a
 * snapshot reads, so a step records its leaf moves and replays them into
 * the tree later -- once 16 steps have gathered, beside the following
 * steps, or at once when the tree is read (m3World_Snapshot, any readback
 * of the world) or overwritten.  This call replays every recorded move of
 * `count` worlds and waits until the trees are current; m3World_Snapshot
 * does the same for its world by itself. */
M3GPU_API int32_t m3gpu_flush_trees(const m3WorldId* worlds, int32_t count);

/* Wait for all device work of the library to finish. */
M3GPU_API int32_t m3gpu_synchronize(void);

/* Kernel launches the library issued since process start (the evidence
 * a device step really ran), and elapsed device time in milliseconds of
 * the last m3gpu_step_worlds call measured with CUDA events. */
M3GPU_API int64_t m3gpu_launch_count(void);
M3GPU_API float m3gpu_last_step_ms(void);

/* Device time in milliseconds of the last m3gpu_step_worlds call, split
 * by stage and summed over steps: out[0] broadphase (bounds, pairs),
 * out[1] narrowphase, out[2] prepare (islands, colouring, rows), out[3]
 * the substep loop with restitution and store, out[4] continuous and
 * sleep.  `out` holds 5 floats. */
M3GPU_API int32_t m3gpu_kernel_ms(float* out);

/* Wide worlds (no reference counterpart; the reference spreads one
 * world's same-colour constraint batches over host threads, solver.c:
 * 2845-2877).  A step of a single world with at least `shapes` shape
 * slots runs its substep loop over a cooperative grid of many blocks
 * instead of one block, the schedule's levels separated by grid
 * barriers; results are bit-identical either way.  Default 4096; returns
 * the previous value (a value <= 0 only queries). */
M3GPU_API int32_t m3gpu_set_wide_min_shapes(int32_t shapes);

/* Packing of a batch's worlds onto the SMs (no reference counterpart:
 * the reference steps one world per host thread).  The batched step
 * splits its worlds, largest first, into three size classes by shape
 * slots: class 0 holds worlds with at least minShapes[0] slots, class 1
 * those with at least minShapes[1], class 2 the rest.  Each class's
 * per-world kernels run `threads[c]` threads per world (512, 256 or 128:
 * one, two or four worlds resident per SM) with up to `smemBytes[c]`
 * bytes of shared memory per world for its tables (the body cache always
 * fits; 0 keeps every table, body cache included, in global memory).
 * Every packing gives the same bits; only the time differs. */
typedef struct m3gpuPacking
{
    int32_t minShapes[2];
    int32_t threads[3];
    int32_t smemBytes[3];
} m3gpuPacking;

/* The packing in use, and a new one (checked: minShapes[0] >
 * minShapes[1] >= 1, threads 128/256/512, smemBytes 0..204800).  It
 * applies from the next batched step on. */
M3GPU_API int32_t m3gpu_get_packing(m3gpuPacking* out);
M3GPU_API int32_t m3gpu_set_packing(const m3gpuPacking* packing);

/* Autotuner: steps the worlds exactly `steps` times (each a real step,
 * bit for bit m3gpu_step_worlds(worlds, count, dt, substeps, 1), and
 * recorded in an active journal the same way), timing the prepare and
 * substep stages of each step under a candidate packing: candidates
 * alternate with the packing in use, each compared with the mean of the
 * steps beside it, and one that is at least 3 % faster becomes the packing
 * in use, whose neighbours are tried next.  Leaves the fastest packing
 * selected and returns it in `best` (optional) with its stage time per
 * step in `bestMs` (optional).  Fewer than 3 steps only step. */
M3GPU_API int32_t m3gpu_autotune_packing(const m3WorldId* worlds, int32_t count, float dt,
                                         int32_t substeps, int32_t steps, m3gpuPacking* best,
                                         float* bestMs);

/* The last autotuning's trials, in order: each candidate packing, its
 * step's prepare + substep device time, the mean of the two steps beside
 * it under the packing then in use, and whether it was adopted.  Copies
 * at most `cap` trials into `out` (may be null) and returns how many the
 * tuning made. */
typedef struct m3gpuPackingTrial
{
    m3gpuPacking packing;
    float ms;
    float baselineMs;
    int32_t adopted;
} m3gpuPackingTrial;
M3GPU_API int32_t m3gpu_autotune_trials(m3gpuPackingTrial* out, int32_t cap);

/* Work counters of one world accumulated over its device steps:
 * out[0] mover-substeps, out[1] contact-row-substeps, out[2]
 * joint-row-substeps, out[3] candidate pairs, out[4] steps, out[5] the
 * body slot count.  `out` holds 6 values. */
M3GPU_API int32_t m3gpu_world_stats(m3WorldId world, uint64_t* out);

/* Device clock cycles one world's block spent in each step phase,
 * accumulated over its device steps (the device counterpart of the
 * reference's per-phase step profile, world.h:578-593).  `out` holds 16
 * values: islands, prepare, colour+movers, integrate velocities, warm
 * start, bias solve, integrate positions, relax, store, continuous,
 * sleep, bounds, sweep sort, pair count, pair fill, and last the number
 * of broadphase tree leaf moves replayed (a count, not cycles). */
M3GPU_API int32_t m3gpu_world_phase_cycles(m3WorldId world, uint64_t* out);

/* White-box readback for parity tests.  Each copies [0, maxIndex) (or
 * [0, pairCount)) records in the reference's byte layout and returns the
 * record count, or -1 when `cap` is too small or the id is stale. */
M3GPU_API int32_t m3gpu_body_max(m3WorldId world);
M3GPU_API int32_t m3gpu_pair_count(m3WorldId world);
M3GPU_API int32_t m3gpu_copy_bodies(m3WorldId world, void* transforms, void* lin, void* ang,
                                    uint8_t* awake, float* sleepTimes, int32_t cap);
M3GPU_API int32_t m3gpu_copy_mass(m3WorldId world, float* invMass, void* invInertia,
                                  void* inertia, void* localCenters, float* minExt,
                                  float* maxExt, int32_t cap);
M3GPU_API int32_t m3gpu_copy_pairs(m3WorldId world, uint64_t* keys, void* manifolds,
                                   int32_t cap);
M3GPU_API int32_t m3gpu_copy_joints(m3WorldId world, void* impulse, void* perp, void* limit,
                                    void* angular, int32_t cap);

/* Body commands applied on the device before one step of the worlds:
 * each as the reference's m3Body_SetLinearVelocity / SetAngularVelocity /
 * ApplyForce / ApplyTorque / ApplyLinearImpulse / ApplyAngularImpulse
 * call would (a stale body or a non-finite vector is a no-op; forces,
 * torques and impulses reach dynamic bodies with mass only), in list
 * order, without reading the worlds back to the host.  `world` indexes
 * the call's world list; `op` is the command's journal record op (4, 5,
 * 26, 27, 28, 29). */
typedef struct m3gpuBodyCommand
{
    int32_t world;
    int32_t op;
    m3BodyId body;
    m3Vec3 v;
} m3gpuBodyCommand;
M3GPU_API int32_t m3gpu_step_worlds_commands(const m3WorldId* worlds, int32_t count, float dt,
                                             int32_t substeps, const m3gpuBodyCommand* commands,
                                             int32_t commandCount);

/* Device snapshot slots: copies of a world's device state kept in HBM for
 * rollback (save a frame, step on, restore it, step again) without a host
 * snapshot, a restore or an upload.  m3gpu_slots_reserve allocates
 * `slots` slots (0 frees them; either frees the slots held before);
 * m3gpu_slot_save copies the world's state into a slot, after uploading
 * pending host changes; m3gpu_slot_restore copies it back.  A restored
 * world steps, hashes and snapshots exactly as the world did after the
 * save (and as m3World_Restore of a snapshot taken then would).  A slot
 * is void once a body, shape or joint is created in the world or a
 * snapshot is restored into it (M3GPU_ERR_INVALID).  Saves and restores
 * are ordered with the steps on the device and return without waiting. */
M3GPU_API int32_t m3gpu_slots_reserve(m3WorldId world, int32_t slots);
M3GPU_API int32_t m3gpu_slot_save(m3WorldId world, int32_t slot);
M3GPU_API int32_t m3gpu_slot_restore(m3WorldId world, int32_t slot);

/* Serving: replay containers in, final world hashes out.  A server
 * admits queued requests while their device memory fits `deviceBudget`
 * bytes (and at most `maxActive` at once, preparing and active): worker
 * threads restore each into a fresh world and validate its journal whole
 * while the GPU steps the others.  Every m3gpu_serve_tick starts
 * preparing what fits, admits the prepared requests in submission order
 * (waiting for one only when nothing is active), advances every active
 * request by one frame (its body commands and the step that closes them)
 * in one batched launch sequence, and retires the requests whose journal
 * is done with the world hash the reference's m3World_Restore +
 * m3World_JournalReplay would give.  A request's result does not depend
 * on the others in the batch. */
typedef struct m3gpuServer m3gpuServer;
M3GPU_API m3gpuServer* m3gpu_serve_create(int64_t deviceBudget, int32_t maxActive);
M3GPU_API void m3gpu_serve_destroy(m3gpuServer* server);
/* Queues a container (copied); returns its ticket (> 0), or -1 for bytes
 * that are not a valid container.  Any thread may submit, also while
 * another thread ticks; tick, poll, active and stats belong to one
 * thread at a time. */
M3GPU_API int64_t m3gpu_serve_submit(m3gpuServer* server, const void* container, int32_t bytes);
/* Admits, runs one frame, retires; returns the requests still queued or
 * active, or a negative error code. */
M3GPU_API int32_t m3gpu_serve_tick(m3gpuServer* server);
/* Drains up to `capacity` finished requests: ticket, final hash, status
 * (M3GPU_OK, or the refusal: an invalid snapshot or journal, content
 * the device path does not model). */
M3GPU_API int32_t m3gpu_serve_poll(m3gpuServer* server, int64_t* tickets, uint64_t* hashes,
                                   int32_t* status, int32_t capacity);
M3GPU_API int32_t m3gpu_serve_active(const m3gpuServer* server);
/* Counters and host times of a server since its creation.  Device bytes
 * are the allocator's (size-class) bytes of the slab and hull pool of
 * each preparing or active request. */
typedef struct m3gpuServeStats
{
    int64_t submitted, completed, refused, ticks;
    int64_t heldBytes;     /* device bytes of preparing + active requests now */
    int64_t peakHeldBytes; /* the most ever held at once */
    int64_t budget;
    int32_t queued, preparing, active, peakActive, workers, reserved;
    double prepareMs; /* worker time building, restoring and parsing (summed over workers) */
    double admitMs;   /* ticking thread: world table entry and device reservation */
    double stepMs;    /* ticking thread: the batched frames */
    double retireMs;  /* ticking thread: device hashes and world release */
    double waitMs;    /* ticking thread: waiting for a preparation with nothing active */
} m3gpuServeStats;
M3GPU_API int32_t m3gpu_serve_stats(m3gpuServer* server, m3gpuServeStats* out);

/* White-box test hook: one broadphase tree move on the host image (remove
 * the shape's leaf, insert [lo, hi]), as the step's tree refresh makes
 * it; the new leaf or -1. */
M3GPU_API int32_t m3gpu_tree_move(m3WorldId world, int32_t shape, const double* lo,
                                  const double* hi);

#ifdef __cplusplus
}
#endif

#endif /* MAUL3D_B200_H */
