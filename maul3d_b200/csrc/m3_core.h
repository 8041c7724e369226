// Core value types and deterministic math, shared by the host C++ and
// the sm_100a device code.
//
// Every operation is a plain IEEE binary32/binary64 add, subtract,
// multiply, divide or square root, written in the operand order of the
// reference engine's inline math (include/maul3d/math.h:60-230) so that
// the compiled result is bit-identical to the reference's scalar build.
// The device side is compiled with -fmad=false -prec-div=true
// -prec-sqrt=true -ftz=false (no contraction, IEEE division and square
// root, denormals kept); the host side with -ffp-contract=off.  Min and
// max are the pinned ternaries (math.h:83-92), never fminf/fmaxf, whose
// signed-zero and NaN rules differ.
#ifndef M3_CORE_H
#define M3_CORE_H

#include <stdint.h>
#include <string.h>
#include <math.h>

#ifdef __CUDACC__
#define M3_HD __host__ __device__ __forceinline__
#define M3_HD_MEMBER __host__ __device__ __forceinline__
#else
#define M3_HD static inline
#define M3_HD_MEMBER inline
#endif

#ifndef MAUL3D_B200_H
// The public header already defines these when included first.
typedef float m3real;
typedef struct m3Vec3 { m3real x, y, z; } m3Vec3;
typedef struct m3Pos3 { double x, y, z; } m3Pos3;
typedef struct m3Quat { m3real x, y, z, w; } m3Quat;
typedef struct m3Transform { m3Pos3 p; m3Quat q; } m3Transform;
typedef struct m3Mat3 { m3Vec3 cx, cy, cz; } m3Mat3;
#define M3_PI 3.14159265358979323846f
#define M3_HASH_INIT 0xCBF29CE484222325ull
#endif

// ---------------------------------------------------------------------
// Engine constants (src/world_internal.h)
// ---------------------------------------------------------------------
#define M3_AABB_MARGIN (4.0f * 0.005f)            // world_internal.h:97
#define M3_SPECULATIVE_DISTANCE M3_AABB_MARGIN      // manifold.c:16
#define M3_LINEAR_SLOP 0.005f                       // manifold.c:264
#define M3_MAX_SUBSTEPS 256                         // world_internal.h:102
#define M3_MANIFOLD_MAX_POINTS 4                    // world_internal.h:477
#define M3_HULL_MAX_VERTS 64                        // world_internal.h:236
#define M3_HULL_MAX_FACES 124
#define M3_HULL_MAX_FACE_INDICES 372
#define M3_HULL_MAX_HALF_EDGES 372
#define M3_GRAPH_COLORS 16                          // solver.c:2740
#define M3_SLEEP_VELOCITY_DEFAULT 0.05f             // world_internal.h:1113
#define M3_TIME_TO_SLEEP 0.5f                       // solver.c:3624
#define M3_CONTACT_HERTZ_DEFAULT 30.0f              // world_internal.h:1091
#define M3_CONTACT_DAMPING_RATIO_DEFAULT 10.0f
#define M3_CONTACT_PUSH_MAX_SPEED_DEFAULT 3.0f
#define M3_RESTITUTION_THRESHOLD_DEFAULT 1.0f
#define M3_MAX_LINEAR_SPEED_DEFAULT 400.0f
#define M3_MAX_ANGULAR_SPEED_DEFAULT 800.0f
#define M3_HIT_EVENT_THRESHOLD_DEFAULT 1.0f
#define M3_LOCKS_ALLOW_FAST_ROTATION 0x40u
#define M3_SOLVER_REV 21                            // world_internal.h:47

#define M3_BODY_STATIC 0
#define M3_BODY_KINEMATIC 1
#define M3_BODY_DYNAMIC 2

#define M3_SHAPE_SPHERE 0
#define M3_SHAPE_PLANE 1
#define M3_SHAPE_HULL 2
#define M3_SHAPE_CAPSULE 3
#define M3_SHAPE_MESH 4
#define M3_SHAPE_VOXEL 5
#define M3_SHAPE_HEIGHTFIELD 6
#define M3_HEIGHTFIELD_MAX_DIM 255 // samples per grid axis (world_internal.h:305)

// ---------------------------------------------------------------------
// Persistent record layouts (byte-identical to the reference)
// ---------------------------------------------------------------------

// world_internal.h:440-448: 32-byte geometry record interpreted by type.
typedef struct m3ShapeGeom
{
    m3Vec3 v;
    m3real s;
    m3Vec3 v2;
    m3real s2;
} m3ShapeGeom;

// world_internal.h:455-466: one contact point, 36 bytes.
typedef struct m3ManifoldPoint
{
    m3Vec3 anchorA;
    m3Vec3 anchorB;
    m3real separation;
    m3real normalImpulse;
    uint16_t id;
    uint16_t flags;
} m3ManifoldPoint;

// world_internal.h:479-494: 188-byte manifold.
typedef struct m3Manifold
{
    m3Vec3 normal;
    int32_t pointCount;
    m3Vec3 frictionImpulse;
    m3real twistImpulse;
    m3Vec3 rollingImpulse;
    m3ManifoldPoint points[M3_MANIFOLD_MAX_POINTS];
} m3Manifold;

// world_internal.h:222-228
typedef struct m3HullHalfEdge
{
    uint16_t twin;
    uint16_t next;
    uint8_t origin;
    uint8_t face;
} m3HullHalfEdge;

// world_internal.h:229-248: the 5808-byte interned hull slab.
typedef struct m3HullData
{
    int32_t vertexCount;
    int32_t faceCount;
    int32_t indexCount;
    float unitMass;
    m3Vec3 unitCom;
    m3Mat3 unitInertiaCom;
    m3Vec3 vertices[M3_HULL_MAX_VERTS];
    m3Vec3 faceNormals[M3_HULL_MAX_FACES];
    m3real faceOffsets[M3_HULL_MAX_FACES];
    uint8_t faceVertCounts[M3_HULL_MAX_FACES];
    uint16_t faceVertStart[M3_HULL_MAX_FACES];
    uint8_t faceIndices[M3_HULL_MAX_FACE_INDICES];
    int32_t edgeCount;
    m3HullHalfEdge edges[M3_HULL_MAX_HALF_EDGES];
    m3Vec3 center;
} m3HullData;

#ifdef __cplusplus
static_assert(sizeof(m3ShapeGeom) == 32, "shape geom layout");
static_assert(sizeof(m3ManifoldPoint) == 36, "manifold point layout");
static_assert(sizeof(m3Manifold) == 188, "manifold layout");
static_assert(sizeof(m3HullData) == 5808, "hull slab layout");
static_assert(sizeof(m3Transform) == 40, "transform layout");
static_assert(sizeof(m3Mat3) == 36, "mat3 layout");
#endif

// ---------------------------------------------------------------------
// Deterministic math (math.h:60-230, math_functions.c)
// ---------------------------------------------------------------------
M3_HD m3Vec3 v3(m3real x, m3real y, m3real z)
{
    m3Vec3 r;
    r.x = x;
    r.y = y;
    r.z = z;
    return r;
}

M3_HD m3Quat q4(m3real x, m3real y, m3real z, m3real w)
{
    m3Quat r;
    r.x = x;
    r.y = y;
    r.z = z;
    r.w = w;
    return r;
}

M3_HD m3real m3MinF(m3real a, m3real b) { return a < b ? a : b; }
M3_HD m3real m3MaxF(m3real a, m3real b) { return a > b ? a : b; }
M3_HD m3real m3ClampF(m3real a, m3real lo, m3real hi) { return m3MaxF(lo, m3MinF(a, hi)); }
// A float cell coordinate to an integer: NaN parks at `nanPark`, the rest
// clamps to +-2e9 and truncates (world_internal.h:30-35).
M3_HD int32_t m3CellFromF(m3real f, m3real nanPark)
{
    f = f != f ? nanPark : f;
    f = f < -2.0e9f ? -2.0e9f : (f > 2.0e9f ? 2.0e9f : f);
    return (int32_t)f;
}
M3_HD m3real m3AbsF(m3real a) { return a < 0.0f ? -a : a; }

M3_HD m3Vec3 m3Add3(m3Vec3 a, m3Vec3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
M3_HD m3Vec3 m3Sub3(m3Vec3 a, m3Vec3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
M3_HD m3Vec3 m3MulSV3(m3real s, m3Vec3 v) { return v3(s * v.x, s * v.y, s * v.z); }
M3_HD m3Vec3 m3Neg3(m3Vec3 v) { return v3(-v.x, -v.y, -v.z); }
M3_HD m3real m3Dot3(m3Vec3 a, m3Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
M3_HD m3Vec3 m3Cross3(m3Vec3 a, m3Vec3 b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
M3_HD m3real m3Length3(m3Vec3 v) { return sqrtf(v.x * v.x + v.y * v.y + v.z * v.z); }

// Degenerate vectors fall back to +y (math.h:149-158).
M3_HD m3Vec3 m3Normalize3(m3Vec3 v)
{
    m3real length = m3Length3(v);
    if (length < 1.19209290e-7f)
    {
        return v3(0.0f, 1.0f, 0.0f);
    }
    m3real inv = 1.0f / length;
    return v3(inv * v.x, inv * v.y, inv * v.z);
}

M3_HD m3Mat3 m3ZeroMat3(void)
{
    m3Mat3 m;
    m.cx = v3(0.0f, 0.0f, 0.0f);
    m.cy = v3(0.0f, 0.0f, 0.0f);
    m.cz = v3(0.0f, 0.0f, 0.0f);
    return m;
}

// Column-major matrix times vector (math.h:60-66).
M3_HD m3Vec3 m3MulMV3(m3Mat3 m, m3Vec3 v)
{
    return v3(m.cx.x * v.x + m.cy.x * v.y + m.cz.x * v.z, m.cx.y * v.x + m.cy.y * v.y + m.cz.y * v.z,
              m.cx.z * v.x + m.cy.z * v.y + m.cz.z * v.z);
}

M3_HD m3Quat m3IdentityQuat(void) { return q4(0.0f, 0.0f, 0.0f, 1.0f); }

M3_HD m3Quat m3MulQuat(m3Quat a, m3Quat b)
{
    m3Quat q;
    q.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
    q.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
    q.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
    q.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
    return q;
}

M3_HD m3Quat m3Conj(m3Quat q) { return q4(-q.x, -q.y, -q.z, q.w); }

// Identity fallback for a degenerate quaternion (math.h:183-193).
M3_HD m3Quat m3NormalizeQuat(m3Quat q)
{
    m3real mag = sqrtf(q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w);
    if (mag < 1.19209290e-7f)
    {
        return m3IdentityQuat();
    }
    m3real inv = 1.0f / mag;
    return q4(inv * q.x, inv * q.y, inv * q.z, inv * q.w);
}

// v' = v + w t + u x t with t = 2 (u x v) (math.h:196-201).
M3_HD m3Vec3 m3RotateVec3(m3Quat q, m3Vec3 v)
{
    m3Vec3 u = v3(q.x, q.y, q.z);
    m3Vec3 t = m3MulSV3(2.0f, m3Cross3(u, v));
    return m3Add3(m3Add3(v, m3MulSV3(q.w, t)), m3Cross3(u, t));
}

M3_HD m3Vec3 m3InvRotateVec3(m3Quat q, m3Vec3 v) { return m3RotateVec3(m3Conj(q), v); }

// q2 = normalize(q1 + 0.5 (dr, 0) q1) (math.h:214-227).
M3_HD m3Quat m3IntegrateRotation(m3Quat q, m3Vec3 dr)
{
    m3real ax = 0.5f * dr.x;
    m3real ay = 0.5f * dr.y;
    m3real az = 0.5f * dr.z;
    m3Quat qd;
    qd.w = -(ax * q.x + ay * q.y + az * q.z);
    qd.x = ax * q.w + ay * q.z - az * q.y;
    qd.y = -ax * q.z + ay * q.w + az * q.x;
    qd.z = ax * q.y - ay * q.x + az * q.w;
    m3Quat q2 = q4(q.x + qd.x, q.y + qd.y, q.z + qd.z, q.w + qd.w);
    return m3NormalizeQuat(q2);
}

// Minimax atan2 (math_functions.c:14-48); polynomial coefficients are
// the engine's published constants.
M3_HD m3real m3Atan2(m3real y, m3real x)
{
    if (x == 0.0f && y == 0.0f)
    {
        return 0.0f;
    }
    m3real ax = m3AbsF(x);
    m3real ay = m3AbsF(y);
    m3real mx = m3MaxF(ay, ax);
    m3real mn = m3MinF(ay, ax);
    m3real a = mn / mx;
    m3real s = a * a;
    m3real c = s * a;
    m3real q = s * s;
    m3real r = 0.024840285f * q + 0.18681418f;
    m3real t = -0.094097948f * q - 0.33213072f;
    r = r * s + t;
    r = r * c + a;
    if (ay > ax)
    {
        r = 1.57079637f - r;
    }
    if (x < 0.0f)
    {
        r = 3.14159274f - r;
    }
    if (y < 0.0f)
    {
        r = -r;
    }
    return r;
}

// FNV-1a 64 (core.c:46-54).
M3_HD uint64_t m3Fnv(uint64_t h, const void* bytes, int32_t count)
{
    const uint8_t* p = (const uint8_t*)bytes;
    for (int32_t i = 0; i < count; ++i)
    {
        h = (h ^ p[i]) * 0x100000001B3ull;
    }
    return h;
}

// Fixed-rule tangent frame (manifold.c:19-38).
M3_HD void m3MakeTangentBasis(m3Vec3 normal, m3Vec3* t1, m3Vec3* t2)
{
    m3real ax = m3AbsF(normal.x);
    m3real ay = m3AbsF(normal.y);
    m3real az = m3AbsF(normal.z);
    m3Vec3 axis;
    if (ax <= ay && ax <= az)
    {
        axis = v3(1.0f, 0.0f, 0.0f);
    }
    else if (ay <= az)
    {
        axis = v3(0.0f, 1.0f, 0.0f);
    }
    else
    {
        axis = v3(0.0f, 0.0f, 1.0f);
    }
    *t1 = m3Normalize3(m3Cross3(normal, axis));
    *t2 = m3Cross3(normal, *t1);
}

// Cramer's rule 3x3 solve; singular returns zero (solver.c:2909-2925).
M3_HD m3Vec3 m3Solve3(const m3Mat3* J, m3Vec3 b)
{
    m3Vec3 cxy = m3Cross3(J->cy, J->cz);
    m3real det = m3Dot3(J->cx, cxy);
    if (det == 0.0f)
    {
        return v3(0.0f, 0.0f, 0.0f);
    }
    m3real inv = 1.0f / det;
    m3Vec3 x;
    x.x = inv * m3Dot3(b, cxy);
    x.y = inv * m3Dot3(J->cx, m3Cross3(b, J->cz));
    x.z = inv * m3Dot3(J->cx, m3Cross3(J->cy, b));
    return x;
}

#endif // M3_CORE_H
