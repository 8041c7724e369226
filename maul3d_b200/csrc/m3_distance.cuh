// GJK distance between convex cores on the device (src/distance.c:1-711)
// and the capsule-versus-hull segment SAT (src/manifold.c:534-692), plus
// the deep-point face query (manifold.c:503-532).  Same Voronoi region
// tests, same barycentric divisors, same 32-iteration cap and the same
// duplicate-support termination, so the witness points and the normal
// come out bit-identical to the reference's.
#ifndef M3_DISTANCE_CUH
#define M3_DISTANCE_CUH

#include "m3_layout.h"

#define M3_MAX_GJK_ITERATIONS 32 // world_internal.h:1301
#define M3_FLT_EPSILON 1.19209290e-7f
#define M3_FLT_MIN 1.17549435e-38f
#define M3_FLT_MAX 3.40282347e+38f

struct m3ProxyDev
{
    const m3Vec3* points;
    int32_t count;
    m3real radius;
};

struct m3SimplexVertexDev
{
    m3Vec3 wA;
    m3Vec3 wB;
    m3Vec3 w;
    m3real a;
    int32_t indexA;
    int32_t indexB;
};

struct m3SimplexDev
{
    m3SimplexVertexDev v[4];
    int32_t count;
};

struct m3DistanceOutDev
{
    m3Vec3 pointA;
    m3Vec3 pointB;
    m3Vec3 normal;
    m3real distance;
};

__device__ __forceinline__ m3real m3Triple(m3Vec3 a, m3Vec3 b, m3Vec3 c)
{
    return m3Dot3(a, m3Cross3(b, c));
}

__device__ __forceinline__ m3Vec3 m3Blend2(m3real a, m3Vec3 wa, m3real b, m3Vec3 wb)
{
    return v3(a * wa.x + b * wb.x, a * wa.y + b * wb.y, a * wa.z + b * wb.z);
}

__device__ __forceinline__ m3Vec3 m3Blend3(m3real a, m3Vec3 wa, m3real b, m3Vec3 wb, m3real c,
                                           m3Vec3 wc)
{
    return v3(a * wa.x + b * wb.x + c * wc.x, a * wa.y + b * wb.y + c * wc.y,
              a * wa.z + b * wb.z + c * wc.z);
}

// Farthest point along the axis, measured from the first point.
__device__ __forceinline__ int32_t m3Support(const m3ProxyDev& proxy, m3Vec3 axis)
{
    m3Vec3 origin = proxy.points[0];
    int32_t maxIndex = 0;
    m3real maxProjection = 0.0f;
    for (int32_t i = 1; i < proxy.count; ++i)
    {
        m3real projection = m3Dot3(axis, m3Sub3(proxy.points[i], origin));
        if (projection > maxProjection)
        {
            maxIndex = i;
            maxProjection = projection;
        }
    }
    return maxIndex;
}

__device__ __forceinline__ void m3BaryEdge(m3real out[3], m3Vec3 a, m3Vec3 b)
{
    m3Vec3 ab = m3Sub3(b, a);
    out[0] = m3Dot3(b, ab);
    out[1] = -m3Dot3(a, ab);
    out[2] = m3Dot3(ab, ab);
}

__device__ __forceinline__ void m3BaryTri(m3real out[4], m3Vec3 a, m3Vec3 b, m3Vec3 c)
{
    m3Vec3 ab = m3Sub3(b, a);
    m3Vec3 ac = m3Sub3(c, a);
    m3Vec3 n = m3Cross3(ab, ac);
    out[0] = m3Dot3(m3Cross3(b, c), n);
    out[1] = m3Dot3(m3Cross3(c, a), n);
    out[2] = m3Dot3(m3Cross3(a, b), n);
    out[3] = m3Dot3(n, n);
}

__device__ __forceinline__ void m3BaryTet(m3real out[5], m3Vec3 a, m3Vec3 b, m3Vec3 c, m3Vec3 d)
{
    m3Vec3 ab = m3Sub3(b, a);
    m3Vec3 ac = m3Sub3(c, a);
    m3Vec3 ad = m3Sub3(d, a);
    m3real divisor = m3Triple(ab, ac, ad);
    m3real sign = divisor < 0.0f ? -1.0f : 1.0f;
    out[0] = sign * m3Triple(b, c, d);
    out[1] = sign * m3Triple(a, d, c);
    out[2] = sign * m3Triple(a, b, d);
    out[3] = sign * m3Triple(a, c, b);
    out[4] = sign * divisor;
}

// Simplex reductions (distance.c:134-471): keep the Voronoi feature
// nearest the origin, in the reference's region test order.
__device__ bool m3SolveSimplex2(m3SimplexDev* s)
{
    m3SimplexVertexDev* vs = s->v;
    m3Vec3 a = vs[0].w;
    m3Vec3 b = vs[1].w;
    m3Vec3 ab = m3Sub3(b, a);
    m3real divisor = m3Dot3(ab, ab);
    m3real u = m3Dot3(b, ab);
    m3real v = -m3Dot3(a, ab);
    if (v <= 0.0f)
    {
        s->count = 1;
        vs[0].a = 1.0f;
        return true;
    }
    if (u <= 0.0f)
    {
        s->count = 1;
        vs[0] = vs[1];
        vs[0].a = 1.0f;
        return true;
    }
    if (divisor <= 0.0f)
    {
        return false;
    }
    m3real denominator = 1.0f / divisor;
    vs[0].a = denominator * u;
    vs[1].a = denominator * v;
    return true;
}

__device__ __forceinline__ bool m3Keep1(m3SimplexDev* s, const m3SimplexVertexDev& a)
{
    s->count = 1;
    s->v[0] = a;
    s->v[0].a = 1.0f;
    return true;
}

__device__ __forceinline__ bool m3Keep2(m3SimplexDev* s, const m3SimplexVertexDev& a,
                                        const m3SimplexVertexDev& b, const m3real w[3])
{
    s->count = 2;
    s->v[0] = a;
    s->v[1] = b;
    if (w[2] <= 0.0f)
    {
        return false;
    }
    s->v[0].a = w[0] / w[2];
    s->v[1].a = w[1] / w[2];
    return true;
}

__device__ __forceinline__ bool m3Keep3(m3SimplexDev* s, const m3SimplexVertexDev& a,
                                        const m3SimplexVertexDev& b, const m3SimplexVertexDev& c,
                                        const m3real w[4])
{
    s->count = 3;
    s->v[0] = a;
    s->v[1] = b;
    s->v[2] = c;
    if (w[3] <= 0.0f)
    {
        return false;
    }
    s->v[0].a = w[0] / w[3];
    s->v[1].a = w[1] / w[3];
    s->v[2].a = w[2] / w[3];
    return true;
}

__device__ bool m3SolveSimplex3(m3SimplexDev* s)
{
    const m3SimplexVertexDev v1 = s->v[0];
    const m3SimplexVertexDev v2 = s->v[1];
    const m3SimplexVertexDev v3v = s->v[2];
    m3real wAB[3];
    m3real wBC[3];
    m3real wCA[3];
    m3BaryEdge(wAB, v1.w, v2.w);
    m3BaryEdge(wBC, v2.w, v3v.w);
    m3BaryEdge(wCA, v3v.w, v1.w);
    if (wAB[1] <= 0.0f && wCA[0] <= 0.0f)
    {
        return m3Keep1(s, v1);
    }
    if (wBC[1] <= 0.0f && wAB[0] <= 0.0f)
    {
        return m3Keep1(s, v2);
    }
    if (wCA[1] <= 0.0f && wBC[0] <= 0.0f)
    {
        return m3Keep1(s, v3v);
    }
    m3real wABC[4];
    m3BaryTri(wABC, v1.w, v2.w, v3v.w);
    if (wABC[2] <= 0.0f && wAB[0] > 0.0f && wAB[1] > 0.0f)
    {
        return m3Keep2(s, v1, v2, wAB);
    }
    if (wABC[0] <= 0.0f && wBC[0] > 0.0f && wBC[1] > 0.0f)
    {
        return m3Keep2(s, v2, v3v, wBC);
    }
    if (wABC[1] <= 0.0f && wCA[0] > 0.0f && wCA[1] > 0.0f)
    {
        return m3Keep2(s, v3v, v1, wCA);
    }
    if (wABC[3] <= 0.0f)
    {
        return false;
    }
    s->v[0].a = wABC[0] / wABC[3];
    s->v[1].a = wABC[1] / wABC[3];
    s->v[2].a = wABC[2] / wABC[3];
    return true;
}

__device__ bool m3SolveSimplex4(m3SimplexDev* s)
{
    const m3SimplexVertexDev vA = s->v[0];
    const m3SimplexVertexDev vB = s->v[1];
    const m3SimplexVertexDev vC = s->v[2];
    const m3SimplexVertexDev vD = s->v[3];
    m3real wAB[3], wAC[3], wAD[3], wBC[3], wCD[3], wDB[3];
    m3BaryEdge(wAB, vA.w, vB.w);
    m3BaryEdge(wAC, vA.w, vC.w);
    m3BaryEdge(wAD, vA.w, vD.w);
    m3BaryEdge(wBC, vB.w, vC.w);
    m3BaryEdge(wCD, vC.w, vD.w);
    m3BaryEdge(wDB, vD.w, vB.w);
    if (wAB[1] <= 0.0f && wAC[1] <= 0.0f && wAD[1] <= 0.0f)
    {
        return m3Keep1(s, vA);
    }
    if (wAB[0] <= 0.0f && wDB[0] <= 0.0f && wBC[1] <= 0.0f)
    {
        return m3Keep1(s, vB);
    }
    if (wAC[0] <= 0.0f && wBC[0] <= 0.0f && wCD[1] <= 0.0f)
    {
        return m3Keep1(s, vC);
    }
    if (wAD[0] <= 0.0f && wCD[0] <= 0.0f && wDB[1] <= 0.0f)
    {
        return m3Keep1(s, vD);
    }
    m3real wACB[4], wABD[4], wADC[4], wBCD[4];
    m3BaryTri(wACB, vA.w, vC.w, vB.w);
    m3BaryTri(wABD, vA.w, vB.w, vD.w);
    m3BaryTri(wADC, vA.w, vD.w, vC.w);
    m3BaryTri(wBCD, vB.w, vC.w, vD.w);
    if (wABD[2] <= 0.0f && wACB[1] <= 0.0f && wAB[0] > 0.0f && wAB[1] > 0.0f)
    {
        return m3Keep2(s, vA, vB, wAB);
    }
    if (wACB[2] <= 0.0f && wADC[1] <= 0.0f && wAC[0] > 0.0f && wAC[1] > 0.0f)
    {
        return m3Keep2(s, vA, vC, wAC);
    }
    if (wADC[2] <= 0.0f && wABD[1] <= 0.0f && wAD[0] > 0.0f && wAD[1] > 0.0f)
    {
        return m3Keep2(s, vA, vD, wAD);
    }
    if (wACB[0] <= 0.0f && wBCD[2] <= 0.0f && wBC[0] > 0.0f && wBC[1] > 0.0f)
    {
        return m3Keep2(s, vB, vC, wBC);
    }
    if (wADC[0] <= 0.0f && wBCD[0] <= 0.0f && wCD[0] > 0.0f && wCD[1] > 0.0f)
    {
        return m3Keep2(s, vC, vD, wCD);
    }
    if (wABD[0] <= 0.0f && wBCD[1] <= 0.0f && wDB[0] > 0.0f && wDB[1] > 0.0f)
    {
        return m3Keep2(s, vD, vB, wDB);
    }
    m3real wABCD[5];
    m3BaryTet(wABCD, vA.w, vB.w, vC.w, vD.w);
    if (wABCD[3] < 0.0f && wACB[0] > 0.0f && wACB[1] > 0.0f && wACB[2] > 0.0f)
    {
        return m3Keep3(s, vA, vC, vB, wACB);
    }
    if (wABCD[2] < 0.0f && wABD[0] > 0.0f && wABD[1] > 0.0f && wABD[2] > 0.0f)
    {
        return m3Keep3(s, vA, vB, vD, wABD);
    }
    if (wABCD[1] < 0.0f && wADC[0] > 0.0f && wADC[1] > 0.0f && wADC[2] > 0.0f)
    {
        return m3Keep3(s, vA, vD, vC, wADC);
    }
    if (wABCD[0] < 0.0f && wBCD[0] > 0.0f && wBCD[1] > 0.0f && wBCD[2] > 0.0f)
    {
        return m3Keep3(s, vB, vC, vD, wBCD);
    }
    if (wABCD[4] <= 0.0f)
    {
        return false;
    }
    s->v[0].a = wABCD[0] / wABCD[4];
    s->v[1].a = wABCD[1] / wABCD[4];
    s->v[2].a = wABCD[2] / wABCD[4];
    s->v[3].a = wABCD[3] / wABCD[4];
    return true;
}

__device__ void m3Witness(const m3SimplexDev* s, m3Vec3* pointA, m3Vec3* pointB)
{
    const m3SimplexVertexDev* vs = s->v;
    switch (s->count)
    {
    case 1:
        *pointA = vs[0].wA;
        *pointB = vs[0].wB;
        break;
    case 2:
        *pointA = m3Blend2(vs[0].a, vs[0].wA, vs[1].a, vs[1].wA);
        *pointB = m3Blend2(vs[0].a, vs[0].wB, vs[1].a, vs[1].wB);
        break;
    case 3:
        *pointA = m3Blend3(vs[0].a, vs[0].wA, vs[1].a, vs[1].wA, vs[2].a, vs[2].wA);
        *pointB = m3Blend3(vs[0].a, vs[0].wB, vs[1].a, vs[1].wB, vs[2].a, vs[2].wB);
        break;
    case 4:
    {
        m3Vec3 sum = m3Add3(m3Blend2(vs[0].a, vs[0].wA, vs[1].a, vs[1].wA),
                            m3Blend2(vs[2].a, vs[2].wA, vs[3].a, vs[3].wA));
        *pointA = sum;
        *pointB = sum;
        break;
    }
    default:
        *pointA = v3(0.0f, 0.0f, 0.0f);
        *pointB = v3(0.0f, 0.0f, 0.0f);
        break;
    }
}

// The simplex cache (distance.c:60-132): the vertex indices of the last
// simplex and its size metric.
struct m3SimplexCacheDev
{
    int32_t count;
    m3real metric;
    uint8_t indexA[4];
    uint8_t indexB[4];
};

// distance.c:100-121
__device__ __forceinline__ m3real m3SimplexMetric(const m3SimplexDev& s)
{
    const m3SimplexVertexDev* vs = s.v;
    switch (s.count)
    {
    case 2:
        return m3Length3(m3Sub3(vs[1].w, vs[0].w));
    case 3:
        return 0.5f * m3Length3(m3Cross3(m3Sub3(vs[1].w, vs[0].w), m3Sub3(vs[2].w, vs[0].w)));
    case 4:
        return m3Triple(m3Sub3(vs[1].w, vs[0].w), m3Sub3(vs[2].w, vs[0].w),
                        m3Sub3(vs[3].w, vs[0].w)) /
               6.0f;
    default:
        return 0.0f;
    }
}

// The A indices of a cache written back, as a bit mask over at most its
// first three vertices (the triangle kernels' feature).
__device__ __forceinline__ int32_t m3CacheMaskA(const m3SimplexCacheDev& c)
{
    int32_t mask = 0;
    for (int32_t i = 0; i < c.count && i < 3; ++i)
    {
        mask |= 1 << c.indexA[i];
    }
    return mask;
}

// m3ShapeDistance with useRadii = false (distance.c:505-709).  B's pose
// in A's frame is (q, p).  Without a cache the simplex starts from
// vertex pair (0, 0), the form the narrowphase calls (manifold.c:2664-
// 2700); with one it starts from the cached simplex unless the metric
// moved (flushed then), and the regular exit writes the final simplex
// back (the two early exits leave the cache as it was).
__device__ m3DistanceOutDev m3ShapeDistanceDev(const m3ProxyDev& proxyA, const m3ProxyDev& proxyB,
                                               m3Quat q, m3Vec3 p,
                                               m3SimplexCacheDev* cache = nullptr)
{
    m3DistanceOutDev output;
    output.pointA = v3(0.0f, 0.0f, 0.0f);
    output.pointB = v3(0.0f, 0.0f, 0.0f);
    output.normal = v3(0.0f, 0.0f, 0.0f);
    output.distance = 0.0f;
    m3SimplexDev simplex;
    memset(&simplex, 0, sizeof(simplex));
    m3SimplexVertexDev* vs = simplex.v;
    simplex.count = 0;
    if (cache != nullptr)
    {
        simplex.count = cache->count <= 4 ? cache->count : 0;
        for (int32_t i = 0; i < simplex.count; ++i)
        {
            const int32_t indexA = cache->indexA[i];
            const int32_t indexB = cache->indexB[i];
            if (indexA >= proxyA.count || indexB >= proxyB.count)
            {
                simplex.count = 0;
                break;
            }
            vs[i].indexA = indexA;
            vs[i].indexB = indexB;
            vs[i].wA = proxyA.points[indexA];
            vs[i].wB = m3Add3(m3RotateVec3(q, proxyB.points[indexB]), p);
            vs[i].w = m3Sub3(vs[i].wB, vs[i].wA);
            vs[i].a = 0.0f;
        }
        if (simplex.count > 0)
        {
            const m3real metric1 = cache->metric;
            const m3real metric2 = m3SimplexMetric(simplex);
            if (2.0f * metric1 < metric2 || metric2 < 0.5f * metric1 || metric2 < M3_FLT_EPSILON)
            {
                simplex.count = 0;
            }
        }
    }
    if (simplex.count == 0)
    {
        simplex.count = 1;
        vs[0].indexA = 0;
        vs[0].indexB = 0;
        vs[0].wA = proxyA.points[0];
        vs[0].wB = m3Add3(m3RotateVec3(q, proxyB.points[0]), p);
        vs[0].w = m3Sub3(vs[0].wB, vs[0].wA);
        vs[0].a = 0.0f;
    }

    m3SimplexDev backup;
    memset(&backup, 0, sizeof(backup));
    m3real distanceSq = M3_FLT_MAX;
    m3Vec3 normal = v3(0.0f, 0.0f, 0.0f);
    for (int32_t iteration = 0; iteration < M3_MAX_GJK_ITERATIONS; ++iteration)
    {
        bool solved = false;
        switch (simplex.count)
        {
        case 1:
            vs[0].a = 1.0f;
            solved = true;
            break;
        case 2:
            solved = m3SolveSimplex2(&simplex);
            break;
        case 3:
            solved = m3SolveSimplex3(&simplex);
            break;
        case 4:
            solved = m3SolveSimplex4(&simplex);
            break;
        default:
            break;
        }
        if (!solved)
        {
            if (backup.count == 0)
            {
                break;
            }
            simplex = backup;
            break;
        }
        if (simplex.count == 4)
        {
            m3Witness(&simplex, &output.pointA, &output.pointB);
            return output;
        }
        m3real oldDistanceSq = distanceSq;
        m3Vec3 closest;
        switch (simplex.count)
        {
        case 1:
            closest = vs[0].w;
            break;
        case 2:
            closest = m3Blend2(vs[0].a, vs[0].w, vs[1].a, vs[1].w);
            break;
        default:
            closest = m3Blend3(vs[0].a, vs[0].w, vs[1].a, vs[1].w, vs[2].a, vs[2].w);
            break;
        }
        distanceSq = m3Dot3(closest, closest);
        if (distanceSq >= oldDistanceSq)
        {
            if (backup.count != 0)
            {
                simplex = backup;
            }
            break;
        }
        m3Vec3 search;
        switch (simplex.count)
        {
        case 1:
            search = m3Neg3(vs[0].w);
            break;
        case 2:
        {
            m3Vec3 ab = m3Sub3(vs[1].w, vs[0].w);
            search = m3Cross3(m3Cross3(ab, m3Neg3(vs[0].w)), ab);
            break;
        }
        default:
        {
            m3Vec3 ab = m3Sub3(vs[1].w, vs[0].w);
            m3Vec3 ac = m3Sub3(vs[2].w, vs[0].w);
            m3Vec3 n = m3Cross3(ab, ac);
            search = m3Dot3(n, vs[0].w) < 0.0f ? n : m3Neg3(n);
            break;
        }
        }
        if (m3Dot3(search, search) < 1000.0f * M3_FLT_MIN)
        {
            m3Witness(&simplex, &output.pointA, &output.pointB);
            return output;
        }
        normal = m3Neg3(search);
        int32_t indexA = m3Support(proxyA, m3Neg3(search));
        m3Vec3 supportA = proxyA.points[indexA];
        int32_t indexB = m3Support(proxyB, m3InvRotateVec3(q, search));
        m3Vec3 supportB = m3Add3(m3RotateVec3(q, proxyB.points[indexB]), p);
        backup = simplex;
        bool duplicate = false;
        for (int32_t i = 0; i < simplex.count; ++i)
        {
            if (vs[i].indexA == indexA && vs[i].indexB == indexB)
            {
                duplicate = true;
                break;
            }
        }
        if (duplicate)
        {
            break;
        }
        vs[simplex.count].indexA = indexA;
        vs[simplex.count].indexB = indexB;
        vs[simplex.count].wA = supportA;
        vs[simplex.count].wB = supportB;
        vs[simplex.count].w = m3Sub3(supportB, supportA);
        simplex.count += 1;
    }
    normal = m3Normalize3(normal);
    m3Vec3 pointA;
    m3Vec3 pointB;
    m3Witness(&simplex, &pointA, &pointB);
    if (cache != nullptr)
    {
        cache->metric = m3SimplexMetric(simplex);
        cache->count = simplex.count;
        for (int32_t i = 0; i < simplex.count; ++i)
        {
            cache->indexA[i] = (uint8_t)vs[i].indexA;
            cache->indexB[i] = (uint8_t)vs[i].indexB;
        }
    }
    output.pointA = pointA;
    output.pointB = pointB;
    output.distance = m3Length3(m3Sub3(pointA, pointB));
    output.normal = normal;
    return output;
}

// The least-deep face of a hull for a point inside it (manifold.c:511-532).
__device__ void m3DeepPointInHull(const m3HullData* hull, m3Vec3 q, m3Vec3* normalOut,
                                  m3real* coreSepOut, m3Vec3* onHullOut)
{
    int32_t best = 0;
    m3real bestD = -3.4e38f;
    for (int32_t f = 0; f < hull->faceCount; ++f)
    {
        m3real d = m3Dot3(hull->faceNormals[f], q) - hull->faceOffsets[f];
        if (d > bestD)
        {
            bestD = d;
            best = f;
        }
    }
    *normalOut = hull->faceNormals[best];
    *coreSepOut = bestD;
    *onHullOut = m3Sub3(q, m3MulSV3(bestD, hull->faceNormals[best]));
}

// Capsule segment versus hull in the hull frame (manifold.c:534-692):
// anchorA on the hull, anchorB on the capsule skin, normal hull to
// capsule.
__device__ m3Manifold m3CollideSegmentHullDev(const m3HullData* hull, m3Vec3 p1, m3Vec3 p2,
                                              m3real radius)
{
    const m3real linearSlop = M3_LINEAR_SLOP;
    m3Manifold manifold;
    memset(&manifold, 0, sizeof(manifold));
    int32_t bestFace = 0;
    m3real bestFaceSep = -3.4e38f;
    for (int32_t f = 0; f < hull->faceCount; ++f)
    {
        m3real d1 = m3Dot3(hull->faceNormals[f], p1) - hull->faceOffsets[f];
        m3real d2 = m3Dot3(hull->faceNormals[f], p2) - hull->faceOffsets[f];
        m3real sep = m3MinF(d1, d2);
        if (sep > bestFaceSep)
        {
            bestFaceSep = sep;
            bestFace = f;
        }
    }
    m3Vec3 segDir = m3Sub3(p2, p1);
    m3Vec3 bestEdgeAxis = v3(0.0f, 1.0f, 0.0f);
    m3real bestEdgeSep = -3.4e38f;
    int32_t bestEdge = -1;
    for (int32_t e = 0; e < hull->edgeCount; e += 2)
    {
        m3Vec3 a = hull->vertices[hull->edges[e].origin];
        m3Vec3 b = hull->vertices[hull->edges[e + 1].origin];
        m3Vec3 axis = m3Cross3(m3Sub3(b, a), segDir);
        m3real len2 = m3Dot3(axis, axis);
        if (len2 < 1.0e-10f)
        {
            continue;
        }
        axis = m3MulSV3(1.0f / sqrtf(len2), axis);
        if (m3Dot3(axis, m3Sub3(a, hull->center)) < 0.0f)
        {
            axis = m3Neg3(axis);
        }
        m3real hullMax = -3.4e38f;
        for (int32_t v = 0; v < hull->vertexCount; ++v)
        {
            m3real proj = m3Dot3(axis, hull->vertices[v]);
            if (proj > hullMax)
            {
                hullMax = proj;
            }
        }
        m3real sep = m3MinF(m3Dot3(axis, p1), m3Dot3(axis, p2)) - hullMax;
        if (sep > bestEdgeSep)
        {
            bestEdgeSep = sep;
            bestEdgeAxis = axis;
            bestEdge = e;
        }
    }
    int edgeWins = bestEdge >= 0 && bestEdgeSep > bestFaceSep + 0.1f * linearSlop;
    m3real coreSep = edgeWins ? bestEdgeSep : bestFaceSep;
    if (coreSep - radius > M3_SPECULATIVE_DISTANCE)
    {
        return manifold;
    }
    if (edgeWins)
    {
        m3Vec3 a = hull->vertices[hull->edges[bestEdge].origin];
        m3Vec3 b = hull->vertices[hull->edges[bestEdge + 1].origin];
        m3Vec3 cSeg;
        m3Vec3 cEdge;
        m3SegmentClosestDev(p1, segDir, a, m3Sub3(b, a), &cSeg, &cEdge);
        manifold.normal = bestEdgeAxis;
        manifold.pointCount = 1;
        manifold.points[0].anchorA = cEdge;
        manifold.points[0].anchorB = m3Sub3(cSeg, m3MulSV3(radius, bestEdgeAxis));
        manifold.points[0].separation = bestEdgeSep - radius;
        manifold.points[0].id = (uint16_t)(0x8000u | (uint32_t)bestEdge);
        return manifold;
    }
    m3Vec3 n = hull->faceNormals[bestFace];
    m3real off = hull->faceOffsets[bestFace];
    int32_t count = hull->faceVertCounts[bestFace];
    int32_t startIdx = hull->faceVertStart[bestFace];
    m3Vec3 centroid = v3(0.0f, 0.0f, 0.0f);
    for (int32_t k = 0; k < count; ++k)
    {
        centroid = m3Add3(centroid, hull->vertices[hull->faceIndices[startIdx + k]]);
    }
    centroid = m3MulSV3(1.0f / (m3real)count, centroid);
    m3real t0 = 0.0f;
    m3real t1 = 1.0f;
    int emptySlab = 0;
    for (int32_t k = 0; k < count; ++k)
    {
        m3Vec3 a = hull->vertices[hull->faceIndices[startIdx + k]];
        m3Vec3 b = hull->vertices[hull->faceIndices[startIdx + (k + 1) % count]];
        m3Vec3 sideN = m3Cross3(m3Sub3(b, a), n);
        if (m3Dot3(sideN, m3Sub3(centroid, a)) < 0.0f)
        {
            sideN = m3Neg3(sideN);
        }
        m3real c0 = m3Dot3(sideN, m3Sub3(p1, a));
        m3real cd = m3Dot3(sideN, segDir);
        if (cd > -1.0e-9f && cd < 1.0e-9f)
        {
            if (c0 < 0.0f)
            {
                emptySlab = 1;
                break;
            }
            continue;
        }
        m3real tc = -c0 / cd;
        if (cd > 0.0f)
        {
            t0 = m3MaxF(t0, tc);
        }
        else
        {
            t1 = m3MinF(t1, tc);
        }
    }
    if (emptySlab || t0 > t1)
    {
        m3real tm = 0.5f * (t0 + t1);
        tm = m3MaxF(0.0f, m3MinF(1.0f, tm));
        t0 = tm;
        t1 = tm;
    }
    int32_t emitted = 0;
    for (int32_t k = 0; k < 2; ++k)
    {
        if (k == 1 && !(t1 > t0))
        {
            break;
        }
        m3real t = k == 0 ? t0 : t1;
        m3Vec3 pt = m3Add3(p1, m3MulSV3(t, segDir));
        m3real d = m3Dot3(n, pt) - off;
        m3real sepK = d - radius;
        if (sepK > M3_SPECULATIVE_DISTANCE)
        {
            continue;
        }
        manifold.points[emitted].anchorA = m3Sub3(pt, m3MulSV3(d, n));
        manifold.points[emitted].anchorB = m3Sub3(pt, m3MulSV3(radius, n));
        manifold.points[emitted].separation = sepK;
        manifold.points[emitted].id = (uint16_t)k;
        emitted += 1;
    }
    manifold.normal = n;
    manifold.pointCount = emitted;
    return manifold;
}

#endif // M3_DISTANCE_CUH
