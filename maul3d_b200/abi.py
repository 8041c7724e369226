"""ctypes mirror of the C ABI in include/maul3d_b200.h.

The value types and the drop-in entry points have the reference engine's
names and layouts, so the same declarations bind both this library and a
reference build; `bind_common` declares them on any handle.
"""
from __future__ import annotations

import ctypes as C
import struct

import numpy as np


class m3Vec3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class m3Pos3(C.Structure):
    _fields_ = [("x", C.c_double), ("y", C.c_double), ("z", C.c_double)]


class m3Quat(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float), ("w", C.c_float)]


class m3WorldId(C.Structure):
    _fields_ = [("index1", C.c_int32), ("generation", C.c_uint16)]


class m3BodyId(C.Structure):
    _fields_ = [("index1", C.c_int32), ("world0", C.c_uint16), ("generation", C.c_uint16)]


# Record dtypes in the reference's byte layouts (world_internal.h).
TRANSFORM = np.dtype([("p", "<f8", 3), ("q", "<f4", 4)])  # 40 bytes
VEC3 = np.dtype(("<f4", 3))
MAT3 = np.dtype(("<f4", 9))
MANIFOLD_POINT = np.dtype([("anchorA", "<f4", 3), ("anchorB", "<f4", 3), ("separation", "<f4"),
                           ("normalImpulse", "<f4"), ("id", "<u2"), ("flags", "<u2")])
MANIFOLD = np.dtype([("normal", "<f4", 3), ("pointCount", "<i4"), ("frictionImpulse", "<f4", 3),
                     ("twistImpulse", "<f4"), ("rollingImpulse", "<f4", 3),
                     ("points", MANIFOLD_POINT, 4)])
assert TRANSFORM.itemsize == 40 and MANIFOLD.itemsize == 188

SCENE_SPHERE_PYRAMID = 0
SCENE_BOX_PYRAMID = 1
SCENE_UNEVEN = 2
SCENE_FREEFALL = 3
SCENE_TOWERS = 4
SCENE_TERRAIN = 5
SCENE_SHOTS = 6
SCENE_PLANK = 7
SCENE_BOUNCE = 8
SCENE_CITY = 9
SCENE_RAIN = 10
SCENE_MIXED = 11


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


class m3Counters(C.Structure):
    """world.h:531-552 of the reference."""
    _fields_ = [(name, C.c_int32) for name in (
        "bodyCount", "shapeCount", "jointCount", "contactCount", "awakeCount", "islandCount",
        "colorCount", "characterCount", "vehicleCount", "softBodyCount", "voxelChunkCount",
        "hullCount", "meshCount", "treeHeight", "scratchPeak", "scratchCapacity",
        "snapshotBytes")] + [("allocCalls", C.c_int64), ("freeCalls", C.c_int64)]


class m3Profile(C.Structure):
    """world.h:578-591 of the reference (milliseconds)."""
    _fields_ = [(name, C.c_float) for name in (
        "step", "vehicles", "broadphase", "narrowphase", "events", "prepare", "solve",
        "continuous", "sleep", "characters", "softBodies")]


class m3gpuServeStats(C.Structure):
    """A server's counters and host times (m3gpu_serve_stats)."""
    _fields_ = ([(name, C.c_int64) for name in (
        "submitted", "completed", "refused", "ticks", "heldBytes", "peakHeldBytes", "budget")] +
        [(name, C.c_int32) for name in (
            "queued", "preparing", "active", "peakActive", "workers", "reserved")] +
        [(name, C.c_double) for name in (
            "prepareMs", "admitMs", "stepMs", "retireMs", "waitMs")])


class m3gpuBodyCommand(C.Structure):
    """A body command applied on the device (m3gpu_step_worlds_commands)."""
    _fields_ = [("world", C.c_int32), ("op", C.c_int32), ("body", m3BodyId), ("v", m3Vec3)]


class m3gpuPacking(C.Structure):
    """The batched step's packing of worlds onto SMs (m3gpu_set_packing)."""
    _fields_ = [("minShapes", C.c_int32 * 2), ("threads", C.c_int32 * 3),
                ("smemBytes", C.c_int32 * 3)]

    def as_dict(self) -> dict:
        return {"min_shapes": list(self.minShapes), "threads": list(self.threads),
                "smem_bytes": list(self.smemBytes)}

    @classmethod
    def from_dict(cls, d: dict) -> "m3gpuPacking":
        p = cls()
        p.minShapes[:] = list(d["min_shapes"])
        p.threads[:] = list(d["threads"])
        p.smemBytes[:] = list(d["smem_bytes"])
        return p


class m3gpuPackingTrial(C.Structure):
    """One candidate of the last autotuning (m3gpu_autotune_trials)."""
    _fields_ = [("packing", m3gpuPacking), ("ms", C.c_float), ("baselineMs", C.c_float),
                ("adopted", C.c_int32)]


assert C.sizeof(m3Counters) == 88 and C.sizeof(m3Profile) == 44
assert C.sizeof(m3gpuPacking) == 32 and C.sizeof(m3gpuPackingTrial) == 44
assert C.sizeof(m3gpuServeStats) == 120


def bind_common(lib: C.CDLL) -> C.CDLL:
    """Declare the reference-named entry points shared by both engines."""
    lib.m3World_GetCounters.argtypes = [m3WorldId]
    lib.m3World_GetCounters.restype = m3Counters
    lib.m3World_GetProfile.argtypes = [m3WorldId]
    lib.m3World_GetProfile.restype = m3Profile
    lib.m3World_Step.argtypes = [m3WorldId, C.c_float, C.c_int32]
    lib.m3World_Step.restype = None
    lib.m3World_Hash.argtypes = [m3WorldId]
    lib.m3World_Hash.restype = C.c_uint64
    lib.m3DestroyWorld.argtypes = [m3WorldId]
    lib.m3DestroyWorld.restype = None
    lib.m3World_IsValid.argtypes = [m3WorldId]
    lib.m3World_IsValid.restype = C.c_bool
    lib.m3s_build.argtypes = [C.c_int32, C.c_uint64, C.c_int32]
    lib.m3s_build.restype = m3WorldId
    lib.m3s_uneven_size.argtypes = [C.c_uint64, C.c_int32, C.c_int32, C.c_int32]
    lib.m3s_uneven_size.restype = C.c_int32
    lib.m3Hash64.argtypes = [C.c_uint64, C.c_void_p, C.c_int32]
    lib.m3Hash64.restype = C.c_uint64
    lib.m3GetVersion.argtypes = []
    lib.m3GetVersion.restype = C.c_int
    return lib


# Journal op codes (the reference's m3JournalOp numbering).
OP_STEP = 1
OP_SET_LINEAR_VELOCITY = 4
OP_SET_ANGULAR_VELOCITY = 5
OP_APPLY_FORCE = 26
OP_APPLY_TORQUE = 27
OP_APPLY_LINEAR_IMPULSE = 28
OP_APPLY_ANGULAR_IMPULSE = 29


def journal_step(dt: float, substeps: int) -> bytes:
    """One step record: {float dt; int32 substeps} (world.c:1623)."""
    return struct.pack("<ii", OP_STEP, 8) + struct.pack("<fi", dt, substeps)


def journal_body_command(op: int, index1: int, generation: int, v) -> bytes:
    """One body command record: {m3BodyId id; m3Vec3 v} (world.c:2286)."""
    payload = struct.pack("<iHH3f", index1, 0, generation, *v)
    return struct.pack("<ii", op, len(payload)) + payload


OP_JOINT_SET_BREAK = 55


def journal_record(op: int, payload: bytes) -> bytes:
    """Any record: {int32 op; int32 bytes; payload} (world.c:1348-1366)."""
    return struct.pack("<ii", op, len(payload)) + payload


def journal_joint_break(index1: int, generation: int, max_force: float, max_torque: float) -> bytes:
    """One joint threshold record: {m3JointId id; float maxForce, maxTorque} (world.c:3111)."""
    payload = struct.pack("<iHHff", index1, 0, generation, max_force, max_torque)
    return struct.pack("<ii", OP_JOINT_SET_BREAK, len(payload)) + payload


def bind_snapshot(lib: C.CDLL) -> C.CDLL:
    """Declare the snapshot, restore and journal entry points a handle has."""
    for name, args, res in (("m3World_SnapshotSize", [m3WorldId], C.c_int32),
                            ("m3World_Snapshot", [m3WorldId, C.c_void_p, C.c_int32], C.c_int32),
                            ("m3World_Restore", [m3WorldId, C.c_void_p, C.c_int32], C.c_bool),
                            ("m3World_JournalReplay", [m3WorldId, C.c_void_p, C.c_int32],
                             C.c_bool),
                            ("m3World_JournalBegin", [m3WorldId, C.c_void_p, C.c_int32], C.c_bool),
                            ("m3World_JournalEnd", [m3WorldId], C.c_int32)):
        try:
            fn = getattr(lib, name)
        except AttributeError:
            continue
        fn.argtypes = args
        fn.restype = res
    return lib


class m3JournalInfo(C.Structure):
    _fields_ = [("opCount", C.c_int32), ("stepCount", C.c_int32)]


class m3ReplayView(C.Structure):
    _fields_ = [("snapshot", C.c_void_p), ("snapshotBytes", C.c_int32), ("journal", C.c_void_p),
                ("journalBytes", C.c_int32), ("finalHash", C.c_uint64), ("info", m3JournalInfo)]


def bind_replay(lib: C.CDLL) -> C.CDLL:
    """Declare the M3J1 container codecs (replay.h:34-62)."""
    lib.m3JournalDescribe.argtypes = [C.c_void_p, C.c_int32, C.POINTER(m3JournalInfo)]
    lib.m3JournalDescribe.restype = C.c_bool
    lib.m3ReplayEncodeSize.argtypes = [C.c_int32, C.c_int32]
    lib.m3ReplayEncodeSize.restype = C.c_int32
    lib.m3ReplayEncode.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_uint64,
                                   C.c_void_p, C.c_int32]
    lib.m3ReplayEncode.restype = C.c_int32
    lib.m3ReplayDecode.argtypes = [C.c_void_p, C.c_int32, C.POINTER(m3ReplayView)]
    lib.m3ReplayDecode.restype = C.c_bool
    return lib


def encode_container(lib: C.CDLL, snapshot: bytes, journal: bytes, final_hash: int = 0) -> bytes:
    """An M3J1 container through a library's m3ReplayEncode."""
    n = lib.m3ReplayEncodeSize(len(snapshot), len(journal))
    out = (C.c_uint8 * n)()
    s = (C.c_uint8 * len(snapshot)).from_buffer_copy(snapshot)
    j = (C.c_uint8 * max(len(journal), 1)).from_buffer_copy(journal or b"\0")
    assert lib.m3ReplayEncode(s, len(snapshot), j, len(journal), final_hash, out, n) == n
    return bytes(out)


class WorldState:
    """Readback of one world's per-step state in the reference layouts."""

    def __init__(self, transforms, lin, ang, awake, sleep, keys, manifolds):
        self.transforms = transforms
        self.lin = lin
        self.ang = ang
        self.awake = awake
        self.sleep = sleep
        self.keys = keys
        self.manifolds = manifolds

    def first_difference(self, other: "WorldState") -> str | None:
        """Describe the first field where two states differ, or None."""
        checks = [("pair keys", self.keys, other.keys), ("transforms", self.transforms, other.transforms),
                  ("linear velocity", self.lin, other.lin), ("angular velocity", self.ang, other.ang),
                  ("awake", self.awake, other.awake), ("sleep time", self.sleep, other.sleep),
                  ("manifolds", self.manifolds, other.manifolds)]
        for name, a, b in checks:
            if a.shape != b.shape:
                return f"{name}: shape {a.shape} vs {b.shape}"
            ab = a.view(np.uint8).reshape(len(a), -1) if len(a) else a.view(np.uint8)
            bb = b.view(np.uint8).reshape(len(b), -1) if len(b) else b.view(np.uint8)
            if not np.array_equal(ab, bb):
                rows = np.nonzero((ab != bb).any(axis=1))[0]
                i = int(rows[0])
                return f"{name}: first differing record {i} of {len(a)} ({len(rows)} differ): {a[i]} vs {b[i]}"
        return None


class m3ShapeId(C.Structure):
    _fields_ = [("index1", C.c_int32), ("world0", C.c_uint16), ("generation", C.c_uint16)]


class m3JointId(C.Structure):
    _fields_ = [("index1", C.c_int32), ("world0", C.c_uint16), ("generation", C.c_uint16)]


class m3WorldDef(C.Structure):
    _fields_ = [("gravity", m3Vec3), ("bodyCapacity", C.c_int32), ("shapeCapacity", C.c_int32),
                ("meshCapacity", C.c_int32), ("jointCapacity", C.c_int32),
                ("voxelCapacity", C.c_int32), ("characterCapacity", C.c_int32),
                ("vehicleCapacity", C.c_int32), ("softBodyCapacity", C.c_int32),
                ("workerCount", C.c_int32), ("enqueueTask", C.c_void_p),
                ("finishTask", C.c_void_p), ("userTaskContext", C.c_void_p),
                ("contactHertz", C.c_float), ("contactDampingRatio", C.c_float),
                ("contactPushMaxSpeed", C.c_float), ("restitutionThreshold", C.c_float),
                ("maximumLinearSpeed", C.c_float), ("enableSleeping", C.c_int32),
                ("enableContinuous", C.c_int32), ("hitEventThreshold", C.c_float),
                ("internalValue", C.c_int32)]


class m3BodyDef(C.Structure):
    _fields_ = [("type", C.c_int32), ("position", m3Pos3), ("rotation", m3Quat),
                ("linearVelocity", m3Vec3), ("angularVelocity", m3Vec3),
                ("gravityScale", C.c_float), ("linearDamping", C.c_float),
                ("angularDamping", C.c_float), ("userData", C.c_uint64), ("isBullet", C.c_bool),
                ("internalValue", C.c_int32)]


class m3ShapeDef(C.Structure):
    _fields_ = [("density", C.c_float), ("friction", C.c_float), ("restitution", C.c_float),
                ("categoryBits", C.c_uint64), ("maskBits", C.c_uint64), ("groupIndex", C.c_int32),
                ("rollingResistance", C.c_float), ("userData", C.c_uint64),
                ("isSensor", C.c_bool), ("enableHitEvents", C.c_bool),
                ("enablePreSolveEvents", C.c_bool), ("localPosition", m3Vec3),
                ("localRotation", m3Quat), ("internalValue", C.c_int32)]


class m3Sphere(C.Structure):
    _fields_ = [("center", m3Vec3), ("radius", C.c_float)]


class m3Plane(C.Structure):
    _fields_ = [("normal", m3Vec3), ("offset", C.c_float)]


class m3Capsule(C.Structure):
    _fields_ = [("point1", m3Vec3), ("point2", m3Vec3), ("radius", C.c_float)]


class m3JointDef(C.Structure):
    """joint.h:85-132 of the reference."""
    _fields_ = [("type", C.c_int32), ("bodyA", m3BodyId), ("bodyB", m3BodyId),
                ("localAnchorA", m3Vec3), ("localAnchorB", m3Vec3), ("localAxisA", m3Vec3),
                ("localAxisB", m3Vec3), ("enableLimit", C.c_bool), ("lowerLimit", C.c_float),
                ("upperLimit", C.c_float), ("enableMotor", C.c_bool), ("motorSpeed", C.c_float),
                ("maxMotorEffort", C.c_float), ("enableCone", C.c_bool), ("coneAngle", C.c_float),
                ("collideConnected", C.c_bool), ("genericLinear", C.c_uint8 * 3),
                ("genericAngular", C.c_uint8 * 3), ("genericMotorAxis", C.c_uint8),
                ("genericReserved", C.c_uint8), ("genericLinearLower", C.c_float * 3),
                ("genericLinearUpper", C.c_float * 3), ("genericAngularLower", C.c_float * 3),
                ("genericAngularUpper", C.c_float * 3), ("ratio", C.c_float),
                ("groundAnchorA", m3Pos3), ("groundAnchorB", m3Pos3), ("internalValue", C.c_int32)]


assert C.sizeof(m3WorldDef) == 112 and C.sizeof(m3BodyDef) == 104 and C.sizeof(m3ShapeDef) == 88
assert C.sizeof(m3JointDef) == 224 and m3JointDef.ratio.offset == 160
assert m3JointDef.groundAnchorA.offset == 168 and m3JointDef.internalValue.offset == 216


class m3ContactEvent(C.Structure):
    """world.h:213-217: a pair of shapes, the lower index first."""
    _fields_ = [("shapeA", m3ShapeId), ("shapeB", m3ShapeId)]


class m3JointBreakEvent(C.Structure):
    """world.h:302-305."""
    _fields_ = [("joint", m3JointId)]


class m3Transform(C.Structure):
    _fields_ = [("p", m3Pos3), ("q", m3Quat)]


class m3BodyMoveEvent(C.Structure):
    """world.h:295-300."""
    _fields_ = [("body", m3BodyId), ("transform", m3Transform), ("fellAsleep", C.c_bool)]


class m3HitEvent(C.Structure):
    """world.h:270-277."""
    _fields_ = [("shapeA", m3ShapeId), ("shapeB", m3ShapeId), ("point", m3Pos3),
                ("normal", m3Vec3), ("approachSpeed", C.c_float)]


EVENT_STREAMS = ("m3World_ContactBeginEvents", "m3World_ContactEndEvents",
                 "m3World_SensorBeginEvents", "m3World_SensorEndEvents")


def bind_events(lib: C.CDLL) -> C.CDLL:
    """Declare the reference-named event streams on a handle."""
    for name in EVENT_STREAMS:
        fn = getattr(lib, name)
        fn.argtypes = [m3WorldId, C.POINTER(C.c_int32)]
        fn.restype = C.POINTER(m3ContactEvent)
    lib.m3World_JointBreakEvents.argtypes = [m3WorldId, C.POINTER(C.c_int32)]
    lib.m3World_JointBreakEvents.restype = C.POINTER(m3JointBreakEvent)
    lib.m3World_BodyMoveEvents.argtypes = [m3WorldId, C.POINTER(C.c_int32)]
    lib.m3World_BodyMoveEvents.restype = C.POINTER(m3BodyMoveEvent)
    lib.m3World_HitEvents.argtypes = [m3WorldId, C.POINTER(C.c_int32)]
    lib.m3World_HitEvents.restype = C.POINTER(m3HitEvent)
    lib.m3World_HitEventsDropped.argtypes = [m3WorldId]
    lib.m3World_HitEventsDropped.restype = C.c_int32
    return lib


def read_events(lib: C.CDLL, world: m3WorldId, moves: bool = True) -> dict:
    """Every event stream of a world's last step as lists of (index1,
    generation) tuples (the world index is left out: it is the engine's
    own table slot); body move events add the transform's bytes and the
    fell-asleep flag, hit events the bytes of point, normal and speed."""
    out = {}
    for name in EVENT_STREAMS:
        n = C.c_int32(0)
        ptr = getattr(lib, name)(world, C.byref(n))
        out[name] = [((ptr[i].shapeA.index1, ptr[i].shapeA.generation),
                      (ptr[i].shapeB.index1, ptr[i].shapeB.generation)) for i in range(n.value)]
    n = C.c_int32(0)
    ptr = lib.m3World_JointBreakEvents(world, C.byref(n))
    out["m3World_JointBreakEvents"] = [(ptr[i].joint.index1, ptr[i].joint.generation)
                                       for i in range(n.value)]
    if moves:
        n = C.c_int32(0)
        ptr = lib.m3World_BodyMoveEvents(world, C.byref(n))
        out["m3World_BodyMoveEvents"] = [
            (ptr[i].body.index1, ptr[i].body.generation, bytes(ptr[i].transform),
             bool(ptr[i].fellAsleep)) for i in range(n.value)]
    n = C.c_int32(0)
    ptr = lib.m3World_HitEvents(world, C.byref(n))
    out["m3World_HitEvents"] = [
        ((ptr[i].shapeA.index1, ptr[i].shapeA.generation),
         (ptr[i].shapeB.index1, ptr[i].shapeB.generation),
         bytes(ptr[i].point) + bytes(ptr[i].normal) + bytes(C.c_float(ptr[i].approachSpeed)))
        for i in range(n.value)]
    out["m3World_HitEventsDropped"] = int(lib.m3World_HitEventsDropped(world))
    return out


def bind_settings(lib: C.CDLL) -> C.CDLL:
    """Declare the reference-named world settings on a handle."""
    lib.m3World_SetGravity.argtypes = [m3WorldId, m3Vec3]
    lib.m3World_GetGravity.argtypes = [m3WorldId]
    lib.m3World_GetGravity.restype = m3Vec3
    lib.m3World_SetContactTuning.argtypes = [m3WorldId, C.c_float, C.c_float, C.c_float]
    for name in ("m3World_SetRestitutionThreshold", "m3World_SetMaximumLinearSpeed",
                 "m3World_SetMaximumAngularSpeed", "m3World_SetHitEventThreshold"):
        getattr(lib, name).argtypes = [m3WorldId, C.c_float]
    for name in ("m3World_EnableSleeping", "m3World_EnableContinuous"):
        getattr(lib, name).argtypes = [m3WorldId, C.c_bool]
    for name in ("m3World_IsSleepingEnabled", "m3World_IsContinuousEnabled"):
        getattr(lib, name).argtypes = [m3WorldId]
        getattr(lib, name).restype = C.c_bool
    lib.m3World_SetWind.argtypes = [m3WorldId, m3Vec3, C.c_float, C.c_float, C.c_float]
    for name in ("m3World_SetGravity", "m3World_SetContactTuning",
                 "m3World_SetRestitutionThreshold", "m3World_SetMaximumLinearSpeed",
                 "m3World_SetMaximumAngularSpeed", "m3World_SetHitEventThreshold",
                 "m3World_EnableSleeping", "m3World_EnableContinuous", "m3World_SetWind"):
        getattr(lib, name).restype = None
    return lib


def bind_body_commands(lib: C.CDLL) -> C.CDLL:
    """Declare the reference-named body commands at a world point, the
    runtime controls (teleport, kinematic target, type, enable, motion
    locks, sleep controls, forced sleep or wake, fast rotation) and the
    body getters."""
    for name in ("m3Body_ApplyForceAtPoint", "m3Body_ApplyLinearImpulseAtPoint"):
        getattr(lib, name).argtypes = [m3BodyId, m3Vec3, m3Pos3]
        getattr(lib, name).restype = None
    lib.m3Body_SetMotionLocks.argtypes = [m3BodyId, C.c_uint32]
    lib.m3Body_SetMotionLocks.restype = None
    lib.m3Body_GetMotionLocks.argtypes = [m3BodyId]
    lib.m3Body_GetMotionLocks.restype = C.c_uint32
    lib.m3Body_SetAllowFastRotation.argtypes = [m3BodyId, C.c_bool]
    lib.m3Body_SetAllowFastRotation.restype = None
    for name in ("m3Body_SetTransform", "m3Body_SetTargetTransform"):
        getattr(lib, name).argtypes = [m3BodyId, m3Pos3, m3Quat]
        getattr(lib, name).restype = None
    lib.m3Body_SetType.argtypes = [m3BodyId, C.c_int32]
    lib.m3Body_SetType.restype = None
    for name in ("m3Body_SetEnabled", "m3Body_SetAwake"):
        getattr(lib, name).argtypes = [m3BodyId, C.c_bool]
        getattr(lib, name).restype = None
    lib.m3Body_SetSleepControls.argtypes = [m3BodyId, C.c_float, C.c_bool]
    lib.m3Body_SetSleepControls.restype = None
    lib.m3Body_IsAwake.argtypes = [m3BodyId]
    lib.m3Body_IsAwake.restype = C.c_bool
    lib.m3Body_GetPosition.argtypes = [m3BodyId]
    lib.m3Body_GetPosition.restype = m3Pos3
    lib.m3Body_SetName.argtypes = [m3BodyId, C.c_char_p]
    lib.m3Body_SetName.restype = None
    lib.m3Body_GetName.argtypes = [m3BodyId]
    lib.m3Body_GetName.restype = C.c_char_p
    for name, res in (("m3Body_GetAllowFastRotation", C.c_bool), ("m3Body_GetType", C.c_int32),
                      ("m3Body_GetUserData", C.c_uint64), ("m3Body_IsEnabled", C.c_bool)):
        getattr(lib, name).argtypes = [m3BodyId]
        getattr(lib, name).restype = res
    return lib


def bind_shape_commands(lib: C.CDLL) -> C.CDLL:
    """Declare the reference-named shape materials, flags and getters."""
    for name in ("m3Shape_SetFriction", "m3Shape_SetRestitution", "m3Shape_SetRollingResistance"):
        getattr(lib, name).argtypes = [m3ShapeId, C.c_float]
        getattr(lib, name).restype = None
    lib.m3Shape_SetDensity.argtypes = [m3ShapeId, C.c_float, C.c_bool]
    lib.m3Shape_SetDensity.restype = None
    for name in ("m3Shape_EnableHitEvents", "m3Shape_EnablePreSolve"):
        getattr(lib, name).argtypes = [m3ShapeId, C.c_bool]
        getattr(lib, name).restype = None
    for name, res in (("m3Shape_GetFriction", C.c_float), ("m3Shape_GetRestitution", C.c_float),
                      ("m3Shape_GetRollingResistance", C.c_float),
                      ("m3Shape_GetDensity", C.c_float),
                      ("m3Shape_AreHitEventsEnabled", C.c_bool),
                      ("m3Shape_IsPreSolveEnabled", C.c_bool), ("m3Shape_GetBody", m3BodyId)):
        getattr(lib, name).argtypes = [m3ShapeId]
        getattr(lib, name).restype = res
    return lib


def bind_joint_commands(lib: C.CDLL) -> C.CDLL:
    """Declare the reference-named joint drives, switches and getters."""
    for name in ("m3Joint_SetLimits", "m3Joint_SetMotor", "m3Joint_SetSpring"):
        getattr(lib, name).argtypes = [m3JointId, C.c_bool, C.c_float, C.c_float]
        getattr(lib, name).restype = None
    lib.m3Joint_SetCollideConnected.argtypes = [m3JointId, C.c_bool]
    lib.m3Joint_SetCollideConnected.restype = None
    for name in ("m3Joint_SetTargetAngle", "m3Joint_SetTargetTranslation"):
        getattr(lib, name).argtypes = [m3JointId, C.c_float]
        getattr(lib, name).restype = None
    lib.m3Joint_SetTargetRotation.argtypes = [m3JointId, m3Quat]
    lib.m3Joint_SetTargetRotation.restype = None
    for name, res in (("m3Joint_GetCollideConnected", C.c_bool), ("m3Joint_GetAngle", C.c_float),
                      ("m3Joint_GetTranslation", C.c_float)):
        getattr(lib, name).argtypes = [m3JointId]
        getattr(lib, name).restype = res
    return lib


class m3ContactData(C.Structure):
    _fields_ = [("shapeA", m3ShapeId), ("shapeB", m3ShapeId), ("normal", m3Vec3),
                ("pointCount", C.c_int32), ("points", m3Pos3 * 4),
                ("separations", C.c_float * 4), ("normalImpulses", C.c_float * 4)]


def bind_contact_data(lib: C.CDLL) -> C.CDLL:
    """Declare the reference-named contact readback on a handle."""
    lib.m3Body_GetContactData.argtypes = [m3BodyId, C.c_void_p, C.c_int32]
    lib.m3Body_GetContactData.restype = C.c_int32
    lib.m3Shape_GetContactData.argtypes = [m3ShapeId, C.c_void_p, C.c_int32]
    lib.m3Shape_GetContactData.restype = C.c_int32
    return lib


def bind_create(lib: C.CDLL) -> C.CDLL:
    """Declare the reference-named creation API on a handle."""
    lib.m3DefaultWorldDef.restype = m3WorldDef
    lib.m3CreateWorld.argtypes = [C.POINTER(m3WorldDef)]
    lib.m3CreateWorld.restype = m3WorldId
    lib.m3DefaultBodyDef.restype = m3BodyDef
    lib.m3CreateBody.argtypes = [m3WorldId, C.POINTER(m3BodyDef)]
    lib.m3CreateBody.restype = m3BodyId
    lib.m3DefaultShapeDef.restype = m3ShapeDef
    lib.m3CreateSphereShape.argtypes = [m3BodyId, C.POINTER(m3ShapeDef), C.POINTER(m3Sphere)]
    lib.m3CreateSphereShape.restype = m3ShapeId
    lib.m3CreatePlaneShape.argtypes = [m3BodyId, C.POINTER(m3ShapeDef), C.POINTER(m3Plane)]
    lib.m3CreatePlaneShape.restype = m3ShapeId
    lib.m3CreateCapsuleShape.argtypes = [m3BodyId, C.POINTER(m3ShapeDef), C.POINTER(m3Capsule)]
    lib.m3CreateCapsuleShape.restype = m3ShapeId
    lib.m3CreateBoxShape.argtypes = [m3BodyId, C.POINTER(m3ShapeDef), m3Vec3]
    lib.m3CreateBoxShape.restype = m3ShapeId
    lib.m3CreateHullShape.argtypes = [m3BodyId, C.POINTER(m3ShapeDef), C.POINTER(m3Vec3),
                                      C.c_int32]
    lib.m3CreateHullShape.restype = m3ShapeId
    lib.m3CreateHeightFieldGridShape.argtypes = [m3BodyId, C.POINTER(m3ShapeDef),
                                                 C.POINTER(C.c_float), C.c_int32, C.c_int32,
                                                 C.c_float]
    lib.m3CreateHeightFieldGridShape.restype = m3ShapeId
    lib.m3DefaultJointDef.restype = m3JointDef
    lib.m3CreateJoint.argtypes = [C.POINTER(m3JointDef)]
    lib.m3CreateJoint.restype = m3JointId
    lib.m3Joint_SetBreakThresholds.argtypes = [m3JointId, C.c_float, C.c_float]
    lib.m3Joint_SetBreakThresholds.restype = None
    lib.m3Joint_IsValid.argtypes = [m3JointId]
    lib.m3Joint_IsValid.restype = C.c_bool
    for name in ("m3Body_ApplyForce", "m3Body_ApplyTorque", "m3Body_ApplyLinearImpulse",
                 "m3Body_ApplyAngularImpulse", "m3Body_SetLinearVelocity",
                 "m3Body_SetAngularVelocity"):
        getattr(lib, name).argtypes = [m3BodyId, m3Vec3]
        getattr(lib, name).restype = None
    return lib
