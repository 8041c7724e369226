// Narrowphase device kernels: one candidate pair in, one manifold out.
//
// Each function follows the reference's collide routine for its pair
// family operation for operation (file:line beside each), so the
// manifold bytes, feature ids and warm-start carry match the reference
// exactly.  They run one pair per thread inside the per-world step
// block (step.cu); hull data is read from the world's hull pool in HBM
// (L1/L2 resident: a scene interns few distinct hulls).
#ifndef M3_NARROW_CUH
#define M3_NARROW_CUH

#include "m3_layout.h"

// Largest clip polygon the device SAT keeps (incident face vertices
// plus one per reference side plane).  A larger polygon is reported as
// unsupported rather than truncated.
#define M3_CLIP_MAX 64

#define M3_NARROW_OK 0
#define M3_NARROW_UNSUPPORTED 1

__device__ __forceinline__ m3Manifold m3EmptyManifold()
{
    m3Manifold m;
    memset(&m, 0, sizeof(m));
    return m;
}

// Shape pose in the world: body pose composed with the compound offset
// (world_internal.h:1276-1290).
__device__ __forceinline__ m3Transform m3ShapeXf(const m3WorldView& w, int32_t shape)
{
    int32_t body = w.shapeBody[shape];
    m3Transform xf = w.xf[body];
    if (w.hasOffset[shape] != 0)
    {
        m3Vec3 r = m3RotateVec3(xf.q, w.localPos[shape]);
        xf.p.x += (double)r.x;
        xf.p.y += (double)r.y;
        xf.p.z += (double)r.z;
        xf.q = m3MulQuat(xf.q, w.localRot[shape]);
    }
    return xf;
}

// World point minus the body's world centre of mass, in float
// (manifold.c:453-460).
__device__ __forceinline__ m3Vec3 m3FromCom(const m3WorldView& w, int32_t body, double px,
                                            double py, double pz)
{
    const m3Transform xf = w.xf[body];
    m3Vec3 rlc = m3RotateVec3(xf.q, w.lc[body]);
    return v3((m3real)(px - xf.p.x - (double)rlc.x), (m3real)(py - xf.p.y - (double)rlc.y),
              (m3real)(pz - xf.p.z - (double)rlc.z));
}

__device__ __forceinline__ void m3SphereCenter(const m3WorldView& w, int32_t shape, double* cx,
                                               double* cy, double* cz)
{
    m3Transform xf = m3ShapeXf(w, shape);
    m3Vec3 r = m3RotateVec3(xf.q, w.geom[shape].v);
    *cx = xf.p.x + (double)r.x;
    *cy = xf.p.y + (double)r.y;
    *cz = xf.p.z + (double)r.z;
}

// manifold.c:41-62
__device__ m3Manifold m3CollideSpheresDev(m3Vec3 d, m3real radiusA, m3real radiusB)
{
    m3Manifold m = m3EmptyManifold();
    m3real distance = m3Length3(d);
    m3real separation = distance - radiusA - radiusB;
    if (separation > M3_SPECULATIVE_DISTANCE)
    {
        return m;
    }
    m3Vec3 normal = m3Normalize3(d);
    m.normal = normal;
    m.pointCount = 1;
    m.points[0].anchorA = m3MulSV3(radiusA, normal);
    m.points[0].anchorB = m3MulSV3(-radiusB, normal);
    m.points[0].separation = separation;
    m.points[0].id = 0;
    return m;
}

// manifold.c:64-84
__device__ m3Manifold m3CollidePlaneSphereDev(m3Vec3 n, m3real dist, m3real radius)
{
    m3Manifold m = m3EmptyManifold();
    m3real separation = dist - radius;
    if (separation > M3_SPECULATIVE_DISTANCE)
    {
        return m;
    }
    m.normal = n;
    m.pointCount = 1;
    m.points[0].anchorB = m3MulSV3(-radius, n);
    m.points[0].separation = separation;
    m.points[0].id = 0;
    return m;
}

// ---------------------------------------------------------------------
// Hull versus hull: face queries, Gauss-map edge query, clip
// (manifold.c:96-437).  Evaluated in A's frame on the float relative
// pose.
// ---------------------------------------------------------------------
struct m3FaceQueryDev
{
    m3real separation;
    int32_t faceIndex;
};

// manifold.c:96-139.  The early break and the separating-face return
// are kept: both are invisible to the result the caller reads.
__device__ m3FaceQueryDev m3QueryFacesDev(const m3HullData* ref, const m3HullData* other, m3Quat q,
                                          m3Vec3 p, int refIsA)
{
    m3FaceQueryDev query;
    query.separation = -3.4e38f;
    query.faceIndex = 0;
    m3Vec3 wv[M3_HULL_MAX_VERTS];
    const int32_t nv = other->vertexCount;
    for (int32_t k = 0; k < nv; ++k)
    {
        wv[k] = refIsA ? m3Add3(m3RotateVec3(q, other->vertices[k]), p)
                       : m3InvRotateVec3(q, m3Sub3(other->vertices[k], p));
    }
    const int32_t nf = ref->faceCount;
    for (int32_t f = 0; f < nf; ++f)
    {
        m3Vec3 n = ref->faceNormals[f];
        m3real off = ref->faceOffsets[f];
        m3real best = 3.4e38f;
        for (int32_t k = 0; k < nv; ++k)
        {
            m3real d = m3Dot3(n, wv[k]) - off;
            best = m3MinF(best, d);
            if (best <= query.separation)
            {
                break;
            }
        }
        if (best > query.separation)
        {
            query.separation = best;
            query.faceIndex = f;
            if (best > M3_SPECULATIVE_DISTANCE)
            {
                return query;
            }
        }
    }
    return query;
}

struct m3EdgeQueryDev
{
    m3real separation;
    int32_t indexA;
    int32_t indexB;
    m3Vec3 axis;
};

// manifold.c:153-228
__device__ m3EdgeQueryDev m3QueryEdgesDev(const m3HullData* hullA, const m3HullData* hullB,
                                          m3Quat q, m3Vec3 p)
{
    m3EdgeQueryDev query;
    query.separation = -3.4e38f;
    query.indexA = -1;
    query.indexB = -1;
    query.axis = v3(0.0f, 1.0f, 0.0f);
    const int32_t ecB = hullB->edgeCount;
    const int32_t ecA = hullA->edgeCount;
    const m3Vec3 centerA = hullA->center;
    for (int32_t ib = 0; ib < ecB; ib += 2)
    {
        const m3HullHalfEdge edgeB = hullB->edges[ib];
        const m3HullHalfEdge twinB = hullB->edges[ib + 1];
        m3Vec3 qB = m3Add3(m3RotateVec3(q, hullB->vertices[twinB.origin]), p);
        m3Vec3 pB = m3Add3(m3RotateVec3(q, hullB->vertices[edgeB.origin]), p);
        m3Vec3 eB = m3Sub3(qB, pB);
        m3Vec3 uB = m3RotateVec3(q, hullB->faceNormals[edgeB.face]);
        m3Vec3 vB = m3RotateVec3(q, hullB->faceNormals[twinB.face]);
        for (int32_t ia = 0; ia < ecA; ia += 2)
        {
            const m3HullHalfEdge edgeA = hullA->edges[ia];
            const m3HullHalfEdge twinA = hullA->edges[ia + 1];
            m3Vec3 pA = hullA->vertices[edgeA.origin];
            m3Vec3 qA = hullA->vertices[twinA.origin];
            m3Vec3 eA = m3Sub3(qA, pA);
            m3Vec3 uA = hullA->faceNormals[edgeA.face];
            m3Vec3 vA = hullA->faceNormals[twinA.face];
            m3real cba = m3Dot3(uB, eA);
            m3real dba = m3Dot3(vB, eA);
            m3real adc = -m3Dot3(uA, eB);
            m3real bdc = -m3Dot3(vA, eB);
            if (!(cba * dba < 0.0f && adc * bdc < 0.0f && cba * bdc > 0.0f))
            {
                continue;
            }
            m3Vec3 axis = m3Cross3(eA, eB);
            m3real len = m3Length3(axis);
            if (len < 1.0e-6f)
            {
                continue;
            }
            axis = m3MulSV3(1.0f / len, axis);
            if (m3Dot3(axis, m3Sub3(pA, centerA)) < 0.0f)
            {
                axis = m3Neg3(axis);
            }
            m3real separation = m3Dot3(axis, m3Sub3(pB, pA));
            if (separation > query.separation)
            {
                query.separation = separation;
                query.indexA = ia;
                query.indexB = ib;
                query.axis = axis;
                if (separation > M3_SPECULATIVE_DISTANCE)
                {
                    return query;
                }
            }
        }
    }
    return query;
}

// manifold.c:231-244
__device__ void m3SegmentClosestDev(m3Vec3 p1, m3Vec3 d1, m3Vec3 p2, m3Vec3 d2, m3Vec3* c1,
                                    m3Vec3* c2)
{
    m3Vec3 r = m3Sub3(p1, p2);
    m3real a = m3Dot3(d1, d1);
    m3real e = m3Dot3(d2, d2);
    m3real f = m3Dot3(d2, r);
    m3real c = m3Dot3(d1, r);
    m3real b = m3Dot3(d1, d2);
    m3real denom = a * e - b * b;
    m3real s = denom > 1.0e-9f ? m3ClampF((b * f - c * e) / denom, 0.0f, 1.0f) : 0.0f;
    m3real t = e > 1.0e-9f ? m3ClampF((b * s + f) / e, 0.0f, 1.0f) : 0.0f;
    s = a > 1.0e-9f ? m3ClampF((b * t - c) / a, 0.0f, 1.0f) : 0.0f;
    *c1 = m3Add3(p1, m3MulSV3(s, d1));
    *c2 = m3Add3(p2, m3MulSV3(t, d2));
}

// manifold.c:246-437.  *status reports a clip polygon above M3_CLIP_MAX.
__device__ m3Manifold m3CollideHullsDev(const m3HullData* hullA, const m3HullData* hullB, m3Quat q,
                                        m3Vec3 p, int32_t* status)
{
    m3Manifold manifold = m3EmptyManifold();
    m3FaceQueryDev faceA = m3QueryFacesDev(hullA, hullB, q, p, 1);
    if (faceA.separation > M3_SPECULATIVE_DISTANCE)
    {
        return manifold;
    }
    m3FaceQueryDev faceB = m3QueryFacesDev(hullB, hullA, q, p, 0);
    if (faceB.separation > M3_SPECULATIVE_DISTANCE)
    {
        return manifold;
    }
    m3EdgeQueryDev edge = m3QueryEdgesDev(hullA, hullB, q, p);
    if (edge.indexA >= 0 && edge.separation > M3_SPECULATIVE_DISTANCE)
    {
        return manifold;
    }
    const m3real linearSlop = M3_LINEAR_SLOP;
    m3real maxFace = m3MaxF(faceA.separation, faceB.separation);
    if (edge.indexA >= 0 && edge.separation > maxFace + 0.1f * linearSlop)
    {
        const m3HullHalfEdge eA = hullA->edges[edge.indexA];
        const m3HullHalfEdge tA = hullA->edges[edge.indexA + 1];
        const m3HullHalfEdge eB = hullB->edges[edge.indexB];
        const m3HullHalfEdge tB = hullB->edges[edge.indexB + 1];
        m3Vec3 pA = hullA->vertices[eA.origin];
        m3Vec3 dA = m3Sub3(hullA->vertices[tA.origin], pA);
        m3Vec3 pB = m3Add3(m3RotateVec3(q, hullB->vertices[eB.origin]), p);
        m3Vec3 dB = m3Sub3(m3Add3(m3RotateVec3(q, hullB->vertices[tB.origin]), p), pB);
        m3Vec3 cA;
        m3Vec3 cB;
        m3SegmentClosestDev(pA, dA, pB, dB, &cA, &cB);
        manifold.normal = edge.axis;
        manifold.pointCount = 1;
        manifold.points[0].anchorA = cA;
        manifold.points[0].anchorB = cB;
        manifold.points[0].separation = edge.separation;
        manifold.points[0].id = (uint16_t)(0x8000u | (((uint32_t)edge.indexA >> 1) << 7) |
                                           ((uint32_t)edge.indexB >> 1));
        return manifold;
    }

    int refIsA = faceB.separation <= faceA.separation + 0.1f * linearSlop ? 1 : 0;
    const m3HullData* ref = refIsA ? hullA : hullB;
    const m3HullData* inc = refIsA ? hullB : hullA;
    int32_t refFace = refIsA ? faceA.faceIndex : faceB.faceIndex;
    m3Vec3 refN = ref->faceNormals[refFace];
    m3real refOff = ref->faceOffsets[refFace];

    m3Vec3 refNInc = refIsA ? m3InvRotateVec3(q, refN) : m3RotateVec3(q, refN);
    int32_t incFace = 0;
    m3real minDot = 3.4e38f;
    for (int32_t f = 0; f < inc->faceCount; ++f)
    {
        m3real d = m3Dot3(refNInc, inc->faceNormals[f]);
        if (d < minDot)
        {
            minDot = d;
            incFace = f;
        }
    }

    m3Vec3 poly[M3_CLIP_MAX];
    uint16_t polyId[M3_CLIP_MAX];
    int32_t polyCount = inc->faceVertCounts[incFace];
    int32_t n = ref->faceVertCounts[refFace];
    if (polyCount + n > M3_CLIP_MAX)
    {
        *status = M3_NARROW_UNSUPPORTED;
        return manifold;
    }
    for (int32_t k = 0; k < polyCount; ++k)
    {
        uint8_t vi = inc->faceIndices[inc->faceVertStart[incFace] + k];
        m3Vec3 vv = inc->vertices[vi];
        poly[k] = refIsA ? m3Add3(m3RotateVec3(q, vv), p) : m3InvRotateVec3(q, m3Sub3(vv, p));
        polyId[k] = vi;
    }

    int32_t start = ref->faceVertStart[refFace];
    for (int32_t e = 0; e < n && polyCount > 0; ++e)
    {
        m3Vec3 v1 = ref->vertices[ref->faceIndices[start + e]];
        m3Vec3 v2 = ref->vertices[ref->faceIndices[start + (e + 1) % n]];
        m3Vec3 tangent = m3Normalize3(m3Sub3(v2, v1));
        m3Vec3 sideN = m3Cross3(tangent, refN);
        m3real sideOff = m3Dot3(sideN, v1);
        m3Vec3 outPoly[M3_CLIP_MAX];
        uint16_t outId[M3_CLIP_MAX];
        int32_t outCount = 0;
        for (int32_t k = 0; k < polyCount; ++k)
        {
            m3Vec3 cur = poly[k];
            m3Vec3 nxt = poly[(k + 1) % polyCount];
            m3real dc = m3Dot3(sideN, cur) - sideOff;
            m3real dn = m3Dot3(sideN, nxt) - sideOff;
            if (dc <= 0.0f)
            {
                outPoly[outCount] = cur;
                outId[outCount] = polyId[k];
                outCount += 1;
            }
            if (dc * dn < 0.0f)
            {
                m3real t = dc / (dc - dn);
                outPoly[outCount] = m3Add3(m3MulSV3(1.0f - t, cur), m3MulSV3(t, nxt));
                outId[outCount] = (uint16_t)(0x4000u | ((uint32_t)e << 8) | polyId[k]);
                outCount += 1;
            }
        }
        for (int32_t k = 0; k < outCount; ++k)
        {
            poly[k] = outPoly[k];
            polyId[k] = outId[k];
        }
        polyCount = outCount;
    }

    // Points below the margin; the deepest four by (separation, id),
    // emitted in ascending id.
    int32_t candIdx[M3_CLIP_MAX];
    m3real candSep[M3_CLIP_MAX];
    int32_t candCount = 0;
    for (int32_t k = 0; k < polyCount; ++k)
    {
        m3real sep = m3Dot3(refN, poly[k]) - refOff;
        if (sep < M3_SPECULATIVE_DISTANCE)
        {
            candIdx[candCount] = k;
            candSep[candCount] = sep;
            candCount += 1;
        }
    }
    int32_t want = candCount < M3_MANIFOLD_MAX_POINTS ? candCount : M3_MANIFOLD_MAX_POINTS;
    uint64_t usedMask = 0;
    int32_t kept[M3_MANIFOLD_MAX_POINTS];
    for (int32_t k = 0; k < want; ++k)
    {
        int32_t best = -1;
        for (int32_t c = 0; c < candCount; ++c)
        {
            if ((usedMask >> c) & 1ull)
            {
                continue;
            }
            if (best < 0 || candSep[c] < candSep[best] ||
                (candSep[c] == candSep[best] && polyId[candIdx[c]] < polyId[candIdx[best]]))
            {
                best = c;
            }
        }
        usedMask |= 1ull << best;
        kept[k] = best;
    }
    for (int32_t a = 0; a < want; ++a)
    {
        for (int32_t b = a + 1; b < want; ++b)
        {
            if (polyId[candIdx[kept[b]]] < polyId[candIdx[kept[a]]])
            {
                int32_t tmp = kept[a];
                kept[a] = kept[b];
                kept[b] = tmp;
            }
        }
    }
    m3Vec3 outN = refIsA ? refN : m3Neg3(m3RotateVec3(q, refN));
    manifold.normal = outN;
    manifold.pointCount = want;
    for (int32_t k = 0; k < want; ++k)
    {
        int32_t c = kept[k];
        m3Vec3 onInc = poly[candIdx[c]];
        m3real sep = candSep[c];
        m3Vec3 onRef = m3Sub3(onInc, m3MulSV3(sep, refN));
        m3Vec3 wInc = refIsA ? onInc : m3Add3(m3RotateVec3(q, onInc), p);
        m3Vec3 wRef = refIsA ? onRef : m3Add3(m3RotateVec3(q, onRef), p);
        manifold.points[k].anchorA = refIsA ? wRef : wInc;
        manifold.points[k].anchorB = refIsA ? wInc : wRef;
        manifold.points[k].separation = sep;
        manifold.points[k].id = (uint16_t)(((uint32_t)refIsA << 15) | ((uint32_t)refFace << 8) |
                                           (polyId[candIdx[c]] & 0xFFu));
    }
    return manifold;
}

#include "m3_distance.cuh"
#include "m3_terrain.cuh"

// GJK proxy of a shape in its own frame (manifold.c:463-499).
__device__ __forceinline__ m3ProxyDev m3MakeProxyDev(const m3WorldView& w, int32_t shape,
                                                     m3Vec3 scratch[2])
{
    m3ProxyDev proxy;
    uint8_t type = w.shapeType[shape];
    if (type == M3_SHAPE_HULL)
    {
        const m3HullData* hull = &w.hulls[w.hullIndex[shape]];
        proxy.points = hull->vertices;
        proxy.count = hull->vertexCount;
        proxy.radius = 0.0f;
        return proxy;
    }
    if (type == M3_SHAPE_CAPSULE)
    {
        scratch[0] = w.geom[shape].v;
        scratch[1] = w.geom[shape].v2;
        proxy.points = scratch;
        proxy.count = 2;
        proxy.radius = w.geom[shape].s;
        return proxy;
    }
    scratch[0] = w.geom[shape].v;
    proxy.points = scratch;
    proxy.count = 1;
    proxy.radius = w.geom[shape].s;
    return proxy;
}

// ---------------------------------------------------------------------
// The pair dispatcher (manifold.c:2357-2911) for the shape families on
// the device path, split by family so that each family runs as its own
// kernel over a bucket of same-family pairs (uniform warps, and each
// kernel only as large as its family's code).  m3PairFamily follows the
// dispatcher's branch order; m3CollideFamily<F> is the branch for family
// F.  A family the device does not cover reports M3_NARROW_UNSUPPORTED
// (the caller stalls the world loudly).
// ---------------------------------------------------------------------
enum
{
    M3F_PLANE_HULL = 0,
    M3F_HULL_HULL = 1,
    M3F_PLANE_CAPSULE = 2,
    M3F_CAPSULE_HULL = 3,
    M3F_ROUND = 4, // hull-sphere, capsule-sphere, capsule-capsule: GJK on the cores
    M3F_PLANE_SPHERE = 5,
    M3F_SPHERE_SPHERE = 6,
    // Heightfield pairs, bucketed by partner so that a warp runs one
    // triangle kernel (any other partner joins the sphere bucket and
    // collides with nothing).
    M3F_TERRAIN_SPHERE = 7,
    M3F_TERRAIN_CAPSULE = 8,
    M3F_TERRAIN_HULL = 9,
    M3F_UNSUPPORTED = 10,
    M3F_COUNT = 11
};

__device__ __forceinline__ int32_t m3PairFamily(uint8_t typeA, uint8_t typeB)
{
    const bool planePair = typeA == M3_SHAPE_PLANE || typeB == M3_SHAPE_PLANE;
    const bool hullPair = typeA == M3_SHAPE_HULL || typeB == M3_SHAPE_HULL;
    const bool capsulePair = typeA == M3_SHAPE_CAPSULE || typeB == M3_SHAPE_CAPSULE;
    // The dispatcher's order: voxel pairs, then heightfield pairs, then
    // mesh pairs (manifold.c:2372-2413).
    if (typeA == M3_SHAPE_VOXEL || typeB == M3_SHAPE_VOXEL)
    {
        return M3F_UNSUPPORTED;
    }
    if (typeA == M3_SHAPE_HEIGHTFIELD || typeB == M3_SHAPE_HEIGHTFIELD)
    {
        const uint8_t other = typeA == M3_SHAPE_HEIGHTFIELD ? typeB : typeA;
        return other == M3_SHAPE_HULL      ? M3F_TERRAIN_HULL
               : other == M3_SHAPE_CAPSULE ? M3F_TERRAIN_CAPSULE
                                           : M3F_TERRAIN_SPHERE;
    }
    if (typeA >= M3_SHAPE_MESH || typeB >= M3_SHAPE_MESH)
    {
        return M3F_UNSUPPORTED;
    }
    if (planePair && hullPair)
    {
        return M3F_PLANE_HULL;
    }
    if (typeA == M3_SHAPE_HULL && typeB == M3_SHAPE_HULL)
    {
        return M3F_HULL_HULL;
    }
    if (planePair && capsulePair)
    {
        return M3F_PLANE_CAPSULE;
    }
    if (hullPair && capsulePair)
    {
        return M3F_CAPSULE_HULL;
    }
    if (hullPair || capsulePair)
    {
        return M3F_ROUND;
    }
    if (planePair)
    {
        return M3F_PLANE_SPHERE;
    }
    return M3F_SPHERE_SPHERE;
}

template <int F>
__device__ int32_t m3CollideFamily(const m3WorldView& w, uint64_t key, m3Manifold* out)
{
    int32_t shapeA = (int32_t)(key >> 32);
    int32_t shapeB = (int32_t)(key & 0xFFFFFFFFu);
    uint8_t typeA = w.shapeType[shapeA];
    uint8_t typeB = w.shapeType[shapeB];
    int hullPair = typeA == M3_SHAPE_HULL || typeB == M3_SHAPE_HULL;
    int32_t status = M3_NARROW_OK;
    m3Manifold fresh = m3EmptyManifold();

    if (F == M3F_UNSUPPORTED)
    {
        *out = fresh;
        return M3_NARROW_UNSUPPORTED;
    }
    if (F == M3F_TERRAIN_SPHERE || F == M3F_TERRAIN_CAPSULE || F == M3F_TERRAIN_HULL)
    {
        // manifold.c:2391-2402: only spheres, capsules and hulls collide
        // with a heightfield; any other partner leaves the manifold empty.
        const int32_t hfShape = typeA == M3_SHAPE_HEIGHTFIELD ? shapeA : shapeB;
        const int32_t otherShape = hfShape == shapeA ? shapeB : shapeA;
        const uint8_t ot = w.shapeType[otherShape];
        if (ot == M3_SHAPE_SPHERE || ot == M3_SHAPE_CAPSULE || ot == M3_SHAPE_HULL)
        {
            m3CollideTerrainDev(w, hfShape, otherShape, hfShape == shapeA, &fresh);
        }
        *out = fresh;
        return status;
    }
    if (F == M3F_PLANE_HULL)
    {
        // Plane versus hull (manifold.c:2415-2520): every vertex inside
        // the margin is a candidate; the four deepest survive (ties to
        // the lower vertex) and emit in ascending vertex order.
        int32_t planeShape = typeA == M3_SHAPE_PLANE ? shapeA : shapeB;
        int32_t hullShape = planeShape == shapeA ? shapeB : shapeA;
        const m3HullData* hull = &w.hulls[w.hullIndex[hullShape]];
        int32_t planeBody = w.shapeBody[planeShape];
        int32_t hullBody = w.shapeBody[hullShape];
        m3Transform xf = m3ShapeXf(w, hullShape);
        m3Vec3 n = w.geom[planeShape].v;
        m3real offset = w.geom[planeShape].s;
        // Selection keeps the four smallest (sep, index) candidates as
        // it scans; equivalent to the reference's repeated argmin over
        // the full candidate list.  The four slots are registers: every
        // index below is a compile-time constant.
        int32_t keepIdx[M3_MANIFOLD_MAX_POINTS];
        m3real keepSep[M3_MANIFOLD_MAX_POINTS];
        double keepW[M3_MANIFOLD_MAX_POINTS][3];
#pragma unroll
        for (int32_t s = 0; s < M3_MANIFOLD_MAX_POINTS; ++s)
        {
            keepIdx[s] = 0;
            keepSep[s] = 0.0f;
            keepW[s][0] = 0.0;
            keepW[s][1] = 0.0;
            keepW[s][2] = 0.0;
        }
        int32_t keepCount = 0;
        const int32_t nv = hull->vertexCount;
        for (int32_t k = 0; k < nv; ++k)
        {
            m3Vec3 r = m3RotateVec3(xf.q, hull->vertices[k]);
            double wx = xf.p.x + (double)r.x;
            double wy = xf.p.y + (double)r.y;
            double wz = xf.p.z + (double)r.z;
            double sep = (double)n.x * wx + (double)n.y * wy + (double)n.z * wz - (double)offset;
            m3real sepF = (m3real)sep;
            if (!(sepF < M3_SPECULATIVE_DISTANCE))
            {
                continue;
            }
            // (sepF, k) goes after every kept entry it does not undercut
            // (indices arrive ascending, so equal separations keep the
            // earlier vertex); entries from there on move down one slot,
            // the last falling off a full list.
            int32_t pos = 0;
#pragma unroll
            for (int32_t s = 0; s < M3_MANIFOLD_MAX_POINTS; ++s)
            {
                pos += (s < keepCount && !(sepF < keepSep[s])) ? 1 : 0;
            }
            if (pos >= M3_MANIFOLD_MAX_POINTS)
            {
                continue;
            }
#pragma unroll
            for (int32_t s = M3_MANIFOLD_MAX_POINTS - 1; s > 0; --s)
            {
                if (s > pos && s <= keepCount)
                {
                    keepIdx[s] = keepIdx[s - 1];
                    keepSep[s] = keepSep[s - 1];
                    keepW[s][0] = keepW[s - 1][0];
                    keepW[s][1] = keepW[s - 1][1];
                    keepW[s][2] = keepW[s - 1][2];
                }
            }
#pragma unroll
            for (int32_t s = 0; s < M3_MANIFOLD_MAX_POINTS; ++s)
            {
                if (s == pos)
                {
                    keepIdx[s] = k;
                    keepSep[s] = sepF;
                    keepW[s][0] = wx;
                    keepW[s][1] = wy;
                    keepW[s][2] = wz;
                }
            }
            if (keepCount < M3_MANIFOLD_MAX_POINTS)
            {
                keepCount += 1;
            }
        }
        // Emit in ascending vertex index: a sorting network over the four
        // slots by index (empty slots carry the largest index and stay
        // last).
#pragma unroll
        for (int32_t s = 0; s < M3_MANIFOLD_MAX_POINTS; ++s)
        {
            keepIdx[s] = s < keepCount ? keepIdx[s] : 0x7FFFFFFF;
        }
        auto order2 = [&](int32_t a, int32_t b) {
            if (keepIdx[b] < keepIdx[a])
            {
                const int32_t ti = keepIdx[a];
                keepIdx[a] = keepIdx[b];
                keepIdx[b] = ti;
                const m3real ts = keepSep[a];
                keepSep[a] = keepSep[b];
                keepSep[b] = ts;
#pragma unroll
                for (int32_t c = 0; c < 3; ++c)
                {
                    const double tw = keepW[a][c];
                    keepW[a][c] = keepW[b][c];
                    keepW[b][c] = tw;
                }
            }
        };
        static_assert(M3_MANIFOLD_MAX_POINTS == 4, "the network sorts four slots");
        order2(0, 1);
        order2(2, 3);
        order2(0, 2);
        order2(1, 3);
        order2(1, 2);
        fresh.normal = n;
        fresh.pointCount = keepCount;
#pragma unroll
        for (int32_t k = 0; k < M3_MANIFOLD_MAX_POINTS; ++k)
        {
            if (k < keepCount)
            {
                double sepD = (double)keepSep[k];
                double px = keepW[k][0] - (double)n.x * sepD;
                double py = keepW[k][1] - (double)n.y * sepD;
                double pz = keepW[k][2] - (double)n.z * sepD;
                fresh.points[k].anchorA = m3FromCom(w, planeBody, px, py, pz);
                fresh.points[k].anchorB =
                    m3FromCom(w, hullBody, keepW[k][0], keepW[k][1], keepW[k][2]);
                fresh.points[k].separation = keepSep[k];
                fresh.points[k].id = (uint16_t)keepIdx[k];
            }
        }
        if (planeShape != shapeA)
        {
            fresh.normal = m3Neg3(fresh.normal);
#pragma unroll
            for (int32_t k = 0; k < M3_MANIFOLD_MAX_POINTS; ++k)
            {
                if (k < keepCount)
                {
                    m3Vec3 tmp = fresh.points[k].anchorA;
                    fresh.points[k].anchorA = fresh.points[k].anchorB;
                    fresh.points[k].anchorB = tmp;
                }
            }
        }
    }
    else if (F == M3F_HULL_HULL)
    {
        // Hull versus hull (manifold.c:2521-2558).
        int32_t bodyA = w.shapeBody[shapeA];
        int32_t bodyB = w.shapeBody[shapeB];
        m3Transform xfA = m3ShapeXf(w, shapeA);
        m3Transform xfB = m3ShapeXf(w, shapeB);
        m3Quat qRel = m3MulQuat(m3Conj(xfA.q), xfB.q);
        m3Vec3 dp = v3((m3real)(xfB.p.x - xfA.p.x), (m3real)(xfB.p.y - xfA.p.y),
                       (m3real)(xfB.p.z - xfA.p.z));
        m3Vec3 pRel = m3InvRotateVec3(xfA.q, dp);
        fresh = m3CollideHullsDev(&w.hulls[w.hullIndex[shapeA]], &w.hulls[w.hullIndex[shapeB]],
                                  qRel, pRel, &status);
        if (fresh.pointCount > 0)
        {
            fresh.normal = m3RotateVec3(xfA.q, fresh.normal);
            for (int32_t k = 0; k < fresh.pointCount; ++k)
            {
                m3Vec3 rA = m3RotateVec3(xfA.q, fresh.points[k].anchorA);
                m3Vec3 rB = m3RotateVec3(xfA.q, fresh.points[k].anchorB);
                fresh.points[k].anchorA = m3FromCom(w, bodyA, xfA.p.x + (double)rA.x,
                                                    xfA.p.y + (double)rA.y, xfA.p.z + (double)rA.z);
                fresh.points[k].anchorB = m3FromCom(w, bodyB, xfA.p.x + (double)rB.x,
                                                    xfA.p.y + (double)rB.y, xfA.p.z + (double)rB.z);
            }
        }
    }
    else if (F == M3F_PLANE_CAPSULE)
    {
        // Plane versus capsule (manifold.c:2559-2616): the two cap
        // centres are the only candidates, in cap order.
        int32_t planeShape = typeA == M3_SHAPE_PLANE ? shapeA : shapeB;
        int32_t capShape = planeShape == shapeA ? shapeB : shapeA;
        int32_t planeBody = w.shapeBody[planeShape];
        int32_t capBody = w.shapeBody[capShape];
        m3Transform xf = m3ShapeXf(w, capShape);
        m3Vec3 n = w.geom[planeShape].v;
        m3real offset = w.geom[planeShape].s;
        m3real radius = w.geom[capShape].s;
        m3Vec3 caps[2] = {w.geom[capShape].v, w.geom[capShape].v2};
        int32_t count = 0;
        for (int32_t k = 0; k < 2; ++k)
        {
            m3Vec3 r = m3RotateVec3(xf.q, caps[k]);
            double wx = xf.p.x + (double)r.x;
            double wy = xf.p.y + (double)r.y;
            double wz = xf.p.z + (double)r.z;
            double centerDist =
                (double)n.x * wx + (double)n.y * wy + (double)n.z * wz - (double)offset;
            m3real sep = (m3real)centerDist - radius;
            if (sep > M3_SPECULATIVE_DISTANCE)
            {
                continue;
            }
            double px = wx - (double)n.x * centerDist;
            double py = wy - (double)n.y * centerDist;
            double pz = wz - (double)n.z * centerDist;
            fresh.points[count].anchorA = m3FromCom(w, planeBody, px, py, pz);
            fresh.points[count].anchorB =
                m3FromCom(w, capBody, wx - (double)(n.x * radius), wy - (double)(n.y * radius),
                          wz - (double)(n.z * radius));
            fresh.points[count].separation = sep;
            fresh.points[count].id = (uint16_t)k;
            count += 1;
        }
        fresh.normal = n;
        fresh.pointCount = count;
        if (count > 0 && planeShape != shapeA)
        {
            fresh.normal = m3Neg3(fresh.normal);
            for (int32_t k = 0; k < count; ++k)
            {
                m3Vec3 tmp = fresh.points[k].anchorA;
                fresh.points[k].anchorA = fresh.points[k].anchorB;
                fresh.points[k].anchorB = tmp;
            }
        }
    }
    else if (F == M3F_CAPSULE_HULL)
    {
        // Capsule versus hull: the segment SAT in the hull frame
        // (manifold.c:2617-2663).
        int32_t hullShape = typeA == M3_SHAPE_HULL ? shapeA : shapeB;
        int32_t capShape = hullShape == shapeA ? shapeB : shapeA;
        int32_t hullBody = w.shapeBody[hullShape];
        int32_t capBody = w.shapeBody[capShape];
        m3Transform xfH = m3ShapeXf(w, hullShape);
        m3Transform xfC = m3ShapeXf(w, capShape);
        m3Quat qRel = m3MulQuat(m3Conj(xfH.q), xfC.q);
        m3Vec3 dp = v3((m3real)(xfC.p.x - xfH.p.x), (m3real)(xfC.p.y - xfH.p.y),
                       (m3real)(xfC.p.z - xfH.p.z));
        m3Vec3 pRel = m3InvRotateVec3(xfH.q, dp);
        m3Vec3 s1 = m3Add3(m3RotateVec3(qRel, w.geom[capShape].v), pRel);
        m3Vec3 s2 = m3Add3(m3RotateVec3(qRel, w.geom[capShape].v2), pRel);
        const m3HullData* hull = &w.hulls[w.hullIndex[hullShape]];
        m3Manifold local = m3CollideSegmentHullDev(hull, s1, s2, w.geom[capShape].s);
        if (local.pointCount > 0)
        {
            m3Vec3 nWorld = m3RotateVec3(xfH.q, local.normal);
            fresh.normal = hullShape == shapeA ? nWorld : m3Neg3(nWorld);
            fresh.pointCount = local.pointCount;
            for (int32_t k = 0; k < local.pointCount; ++k)
            {
                m3Vec3 rH = m3RotateVec3(xfH.q, local.points[k].anchorA);
                m3Vec3 rC = m3RotateVec3(xfH.q, local.points[k].anchorB);
                m3Vec3 aHull = m3FromCom(w, hullBody, xfH.p.x + (double)rH.x,
                                         xfH.p.y + (double)rH.y, xfH.p.z + (double)rH.z);
                m3Vec3 aCap = m3FromCom(w, capBody, xfH.p.x + (double)rC.x,
                                        xfH.p.y + (double)rC.y, xfH.p.z + (double)rC.z);
                fresh.points[k].anchorA = hullShape == shapeA ? aHull : aCap;
                fresh.points[k].anchorB = hullShape == shapeA ? aCap : aHull;
                fresh.points[k].separation = local.points[k].separation;
                fresh.points[k].id = local.points[k].id;
            }
        }
    }
    else if (F == M3F_ROUND)
    {
        // Hull-sphere, capsule-sphere, capsule-capsule: GJK on the
        // cores in A's frame, radii applied analytically, one point,
        // feature id 0; exact answers for a deep core overlap
        // (manifold.c:2664-2807).
        int32_t bodyA = w.shapeBody[shapeA];
        int32_t bodyB = w.shapeBody[shapeB];
        m3Transform xfA = m3ShapeXf(w, shapeA);
        m3Transform xfB = m3ShapeXf(w, shapeB);
        m3Quat qIn = m3MulQuat(m3Conj(xfA.q), xfB.q);
        m3Vec3 dp = v3((m3real)(xfB.p.x - xfA.p.x), (m3real)(xfB.p.y - xfA.p.y),
                       (m3real)(xfB.p.z - xfA.p.z));
        m3Vec3 pIn = m3InvRotateVec3(xfA.q, dp);
        m3Vec3 pointsA[2];
        m3Vec3 pointsB[2];
        m3ProxyDev proxyA = m3MakeProxyDev(w, shapeA, pointsA);
        m3ProxyDev proxyB = m3MakeProxyDev(w, shapeB, pointsB);
        m3DistanceOutDev dout = m3ShapeDistanceDev(proxyA, proxyB, qIn, pIn);
        m3real rA = proxyA.radius;
        m3real rB = proxyB.radius;
        m3real sep = dout.distance - rA - rB;
        if (sep <= M3_SPECULATIVE_DISTANCE)
        {
            m3Vec3 nLocal;
            m3Vec3 pALocal;
            m3Vec3 pBLocal;
            if (dout.distance > 0.0f)
            {
                nLocal = dout.normal;
                pALocal = m3Add3(dout.pointA, m3MulSV3(rA, nLocal));
                pBLocal = m3Sub3(dout.pointB, m3MulSV3(rB, nLocal));
            }
            else if (hullPair)
            {
                int hullIsA = typeA == M3_SHAPE_HULL;
                const m3HullData* hull = &w.hulls[w.hullIndex[hullIsA ? shapeA : shapeB]];
                const m3ProxyDev& round = hullIsA ? proxyB : proxyA;
                m3Vec3 core = hullIsA ? m3Add3(m3RotateVec3(qIn, round.points[0]), pIn)
                                      : m3InvRotateVec3(qIn, m3Sub3(round.points[0], pIn));
                m3Vec3 nHull;
                m3real coreSep;
                m3Vec3 onHull;
                m3DeepPointInHull(hull, core, &nHull, &coreSep, &onHull);
                m3real rRound = round.radius;
                sep = coreSep - rRound;
                if (hullIsA)
                {
                    nLocal = nHull;
                    pALocal = onHull;
                    pBLocal = m3Sub3(core, m3MulSV3(rRound, nHull));
                }
                else
                {
                    m3Vec3 nA = m3RotateVec3(qIn, nHull);
                    nLocal = m3Neg3(nA);
                    pALocal = m3Sub3(m3Add3(m3RotateVec3(qIn, core), pIn), m3MulSV3(rRound, nA));
                    pBLocal = m3Add3(m3RotateVec3(qIn, onHull), pIn);
                }
            }
            else
            {
                m3Vec3 axis;
                m3Vec3 cA;
                m3Vec3 cB;
                if (proxyA.count == 2 && proxyB.count == 2)
                {
                    m3Vec3 dirA = m3Sub3(pointsA[1], pointsA[0]);
                    m3Vec3 dirB = m3RotateVec3(qIn, m3Sub3(pointsB[1], pointsB[0]));
                    axis = m3Cross3(dirA, dirB);
                    cA = m3MulSV3(0.5f, m3Add3(pointsA[0], pointsA[1]));
                    cB = m3Add3(m3RotateVec3(qIn, m3MulSV3(0.5f, m3Add3(pointsB[0], pointsB[1]))),
                                pIn);
                    if (m3Dot3(axis, axis) < 1.0e-10f)
                    {
                        axis = m3Sub3(cB, cA);
                    }
                }
                else
                {
                    m3Vec3 dir = proxyA.count == 2
                                     ? m3Sub3(pointsA[1], pointsA[0])
                                     : m3RotateVec3(qIn, m3Sub3(pointsB[1], pointsB[0]));
                    m3Vec3 t1;
                    m3Vec3 t2;
                    m3MakeTangentBasis(m3Normalize3(dir), &t1, &t2);
                    axis = t1;
                    cA = proxyA.count == 1 ? pointsA[0]
                                           : m3MulSV3(0.5f, m3Add3(pointsA[0], pointsA[1]));
                    cB = proxyB.count == 1
                             ? m3Add3(m3RotateVec3(qIn, pointsB[0]), pIn)
                             : m3Add3(m3RotateVec3(qIn, m3MulSV3(0.5f, m3Add3(pointsB[0], pointsB[1]))),
                                      pIn);
                }
                nLocal = m3Normalize3(axis);
                if (m3Dot3(nLocal, m3Sub3(cB, cA)) < 0.0f)
                {
                    nLocal = m3Neg3(nLocal);
                }
                m3Vec3 mid = m3MulSV3(0.5f, m3Add3(cA, cB));
                pALocal = mid;
                pBLocal = mid;
                sep = -(rA + rB);
            }
            fresh.normal = m3RotateVec3(xfA.q, nLocal);
            m3Vec3 wA = m3RotateVec3(xfA.q, pALocal);
            m3Vec3 wB = m3RotateVec3(xfA.q, pBLocal);
            fresh.points[0].anchorA = m3FromCom(w, bodyA, xfA.p.x + (double)wA.x,
                                                xfA.p.y + (double)wA.y, xfA.p.z + (double)wA.z);
            fresh.points[0].anchorB = m3FromCom(w, bodyB, xfA.p.x + (double)wB.x,
                                                xfA.p.y + (double)wB.y, xfA.p.z + (double)wB.z);
            fresh.points[0].separation = sep;
            fresh.points[0].id = 0;
            fresh.pointCount = 1;
        }
    }
    else if (F == M3F_PLANE_SPHERE)
    {
        // Plane versus sphere (manifold.c:2808-2844).
        int32_t planeShape = typeA == M3_SHAPE_PLANE ? shapeA : shapeB;
        int32_t sphereShape = planeShape == shapeA ? shapeB : shapeA;
        m3Vec3 n = w.geom[planeShape].v;
        m3real offset = w.geom[planeShape].s;
        double cx, cy, cz;
        m3SphereCenter(w, sphereShape, &cx, &cy, &cz);
        double distD = (double)n.x * cx + (double)n.y * cy + (double)n.z * cz - (double)offset;
        fresh = m3CollidePlaneSphereDev(n, (m3real)distD, w.geom[sphereShape].s);
        if (fresh.pointCount > 0)
        {
            int32_t planeBody = w.shapeBody[planeShape];
            int32_t ballBody = w.shapeBody[sphereShape];
            double px = cx - (double)(fresh.normal.x * (m3real)distD);
            double py = cy - (double)(fresh.normal.y * (m3real)distD);
            double pz = cz - (double)(fresh.normal.z * (m3real)distD);
            fresh.points[0].anchorA = m3FromCom(w, planeBody, px, py, pz);
            fresh.points[0].anchorB =
                m3Add3(m3FromCom(w, ballBody, cx, cy, cz), fresh.points[0].anchorB);
            if (planeShape != shapeA)
            {
                m3Vec3 tmp = fresh.points[0].anchorA;
                fresh.points[0].anchorA = fresh.points[0].anchorB;
                fresh.points[0].anchorB = tmp;
                fresh.normal = m3Neg3(fresh.normal);
            }
        }
    }
    else if (F == M3F_SPHERE_SPHERE)
    {
        // Sphere versus sphere (manifold.c:2845-2866).
        double ax, ay, az, bx, by, bz;
        m3SphereCenter(w, shapeA, &ax, &ay, &az);
        m3SphereCenter(w, shapeB, &bx, &by, &bz);
        m3Vec3 d = v3((m3real)(bx - ax), (m3real)(by - ay), (m3real)(bz - az));
        fresh = m3CollideSpheresDev(d, w.geom[shapeA].s, w.geom[shapeB].s);
        if (fresh.pointCount > 0)
        {
            fresh.points[0].anchorA =
                m3Add3(m3FromCom(w, w.shapeBody[shapeA], ax, ay, az), fresh.points[0].anchorA);
            fresh.points[0].anchorB =
                m3Add3(m3FromCom(w, w.shapeBody[shapeB], bx, by, bz), fresh.points[0].anchorB);
        }
    }
    *out = fresh;
    return status;
}

// All families through one entry (the allocation-free single-world path
// and any caller without buckets).
__device__ int32_t m3CollidePair(const m3WorldView& w, uint64_t key, m3Manifold* out)
{
    const uint8_t typeA = w.shapeType[(int32_t)(key >> 32)];
    const uint8_t typeB = w.shapeType[(int32_t)(key & 0xFFFFFFFFu)];
    switch (m3PairFamily(typeA, typeB))
    {
    case M3F_PLANE_HULL:
        return m3CollideFamily<M3F_PLANE_HULL>(w, key, out);
    case M3F_HULL_HULL:
        return m3CollideFamily<M3F_HULL_HULL>(w, key, out);
    case M3F_PLANE_CAPSULE:
        return m3CollideFamily<M3F_PLANE_CAPSULE>(w, key, out);
    case M3F_CAPSULE_HULL:
        return m3CollideFamily<M3F_CAPSULE_HULL>(w, key, out);
    case M3F_ROUND:
        return m3CollideFamily<M3F_ROUND>(w, key, out);
    case M3F_PLANE_SPHERE:
        return m3CollideFamily<M3F_PLANE_SPHERE>(w, key, out);
    case M3F_SPHERE_SPHERE:
        return m3CollideFamily<M3F_SPHERE_SPHERE>(w, key, out);
    case M3F_TERRAIN_SPHERE:
        return m3CollideFamily<M3F_TERRAIN_SPHERE>(w, key, out);
    case M3F_TERRAIN_CAPSULE:
        return m3CollideFamily<M3F_TERRAIN_CAPSULE>(w, key, out);
    case M3F_TERRAIN_HULL:
        return m3CollideFamily<M3F_TERRAIN_HULL>(w, key, out);
    default:
        return m3CollideFamily<M3F_UNSUPPORTED>(w, key, out);
    }
}

// Index of `key` in keys[0, n) (sorted ascending, unique), or -1.  The
// search starts at `hint` (the pair's index in this step's list; pair
// lists change little between steps, so the key is usually there or a
// few slots away) and gallops outwards before bisecting what is left:
// a handful of dependent loads instead of a full bisection's log2(n).
// Keys are unique, so the answer is the same as any exact search's.
__device__ __forceinline__ int32_t m3FindPairKey(const uint64_t* keys, int32_t n, uint64_t key,
                                                 int32_t hint)
{
    if (n <= 0)
    {
        return -1;
    }
    const int32_t i = hint < 0 ? 0 : (hint < n ? hint : n - 1);
    const uint64_t ki = keys[i];
    if (ki == key)
    {
        return i;
    }
    int32_t lo;
    int32_t hi;
    if (ki < key)
    {
        lo = i + 1;
        hi = n - 1;
        for (int32_t step = 1; i + step < n; step <<= 1)
        {
            const uint64_t kj = keys[i + step];
            if (kj == key)
            {
                return i + step;
            }
            if (kj > key)
            {
                hi = i + step - 1;
                break;
            }
            lo = i + step + 1;
        }
    }
    else
    {
        lo = 0;
        hi = i - 1;
        for (int32_t step = 1; i - step >= 0; step <<= 1)
        {
            const uint64_t kj = keys[i - step];
            if (kj == key)
            {
                return i - step;
            }
            if (kj < key)
            {
                lo = i - step + 1;
                break;
            }
            hi = i - step - 1;
        }
    }
    while (lo <= hi)
    {
        const int32_t mid = (lo + hi) / 2;
        const uint64_t k = keys[mid];
        if (k == key)
        {
            return mid;
        }
        if (k < key)
        {
            lo = mid + 1;
        }
        else
        {
            hi = mid - 1;
        }
    }
    return -1;
}

// Warm-start carry (manifold.c:2868-2908): the previous step's manifold
// of the same key, pair-level friction payload, per-point impulse by
// feature id.  `hint` is the pair's index in this step's sorted list.
// The point loop runs over fixed slots so the manifold stays in
// registers.
__device__ __forceinline__ void m3WarmCarry(m3Manifold* fresh, uint64_t key,
                                            const uint64_t* oldKeys, const m3Manifold* oldMan,
                                            int32_t oldCount, int32_t hint)
{
    if (fresh->pointCount <= 0 || oldCount <= 0)
    {
        return;
    }
    const int32_t at = m3FindPairKey(oldKeys, oldCount, key, hint);
    if (at < 0)
    {
        return;
    }
    const m3Manifold* previous = &oldMan[at];
    fresh->frictionImpulse = previous->frictionImpulse;
    fresh->twistImpulse = previous->twistImpulse;
    fresh->rollingImpulse = previous->rollingImpulse;
    const int32_t pc = previous->pointCount;
    const int32_t fc = fresh->pointCount;
#pragma unroll
    for (int32_t a = 0; a < M3_MANIFOLD_MAX_POINTS; ++a)
    {
        if (a < fc)
        {
            for (int32_t o = 0; o < pc; ++o)
            {
                if (previous->points[o].id == fresh->points[a].id)
                {
                    fresh->points[a].normalImpulse = previous->points[o].normalImpulse;
                    fresh->points[a].flags |= 1;
                    break;
                }
            }
        }
    }
}

#endif // M3_NARROW_CUH
