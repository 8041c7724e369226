// Time of impact on the device (distance.c:711-1215): conservative
// advancement of two swept convex proxies with the separating-axis root
// finder, the form the continuous phase calls against static targets
// (solver.c:3081-3274).  Same sweeps, same separation functions, same
// iteration caps and the same simplex cache between the GJK calls, so the
// fraction and the state come out bit-identical to the reference's.
#ifndef M3_TOI_CUH
#define M3_TOI_CUH

#include "m3_distance.cuh"

// A body's motion over the step, relative to a base point
// (world_internal.h m3Sweep).
struct m3SweepDev
{
    m3Vec3 localCenter;
    m3Vec3 c1;
    m3Vec3 c2;
    m3Quat q1;
    m3Quat q2;
};

// distance.c:711-730: normalised lerp with the hemisphere guard.
__device__ __forceinline__ m3Transform m3SweepAt(const m3SweepDev& sweep, m3real time)
{
    m3Quat q2 = sweep.q2;
    if (sweep.q1.x * q2.x + sweep.q1.y * q2.y + sweep.q1.z * q2.z + sweep.q1.w * q2.w < 0.0f)
    {
        q2 = q4(-q2.x, -q2.y, -q2.z, -q2.w);
    }
    const m3Quat q = q4(sweep.q1.x + time * (q2.x - sweep.q1.x),
                        sweep.q1.y + time * (q2.y - sweep.q1.y),
                        sweep.q1.z + time * (q2.z - sweep.q1.z),
                        sweep.q1.w + time * (q2.w - sweep.q1.w));
    m3Transform xf;
    xf.q = m3NormalizeQuat(q);
    const m3Vec3 c = m3Add3(sweep.c1, m3MulSV3(time, m3Sub3(sweep.c2, sweep.c1)));
    const m3Vec3 r = m3RotateVec3(xf.q, sweep.localCenter);
    xf.p.x = (double)(c.x - r.x);
    xf.p.y = (double)(c.y - r.y);
    xf.p.z = (double)(c.z - r.z);
    return xf;
}

// distance.c:734-738
__device__ __forceinline__ m3Vec3 m3ToiPoint(const m3Transform& xf, m3Vec3 p)
{
    const m3Vec3 r = m3RotateVec3(xf.q, p);
    return v3((m3real)xf.p.x + r.x, (m3real)xf.p.y + r.y, (m3real)xf.p.z + r.z);
}

// distance.c:740-760
__device__ __forceinline__ int32_t m3ToiUniqueCount(int32_t count, const int32_t v[3])
{
    if (count == 1)
    {
        return 1;
    }
    if (count == 2)
    {
        return v[0] != v[1] ? 2 : 1;
    }
    if (v[0] != v[1] && v[0] != v[2] && v[1] != v[2])
    {
        return 3;
    }
    if (v[0] == v[1] && v[0] == v[2])
    {
        return 1;
    }
    return 2;
}

// distance.c:763-777: first vertex of greatest projection.
__device__ __forceinline__ int32_t m3ToiSupport(const m3ProxyDev& proxy, m3Vec3 d)
{
    int32_t best = 0;
    m3real bestDot = m3Dot3(proxy.points[0], d);
    for (int32_t i = 1; i < proxy.count; ++i)
    {
        const m3real x = m3Dot3(proxy.points[i], d);
        if (x > bestDot)
        {
            bestDot = x;
            best = i;
        }
    }
    return best;
}

enum
{
    M3_SEP_VERTICES = 0,
    M3_SEP_EDGES = 1,
    M3_SEP_FACE_A = 2,
    M3_SEP_FACE_B = 3,
};

struct m3SeparationDev
{
    const m3ProxyDev* proxyA;
    const m3ProxyDev* proxyB;
    const m3SweepDev* sweepA;
    const m3SweepDev* sweepB;
    m3Vec3 witness1;
    m3Vec3 witness2;
    int32_t type;
};

// distance.c:781-791
__device__ __forceinline__ bool m3ToiFastEdges(const m3SweepDev& sweepA, const m3SweepDev& sweepB,
                                               m3Vec3 localEdgeA, m3Vec3 localEdgeB, m3Vec3 axis0)
{
    const m3Transform xfA = m3SweepAt(sweepA, 1.0f);
    const m3Transform xfB = m3SweepAt(sweepB, 1.0f);
    const m3Vec3 edgeA = m3RotateVec3(xfA.q, localEdgeA);
    const m3Vec3 edgeB = m3RotateVec3(xfB.q, localEdgeB);
    const m3Vec3 axis = m3Cross3(edgeA, edgeB);
    return m3Dot3(axis, axis0) < 0.0f;
}

// distance.c:812-937
__device__ m3SeparationDev m3ToiMakeSeparation(const m3SimplexCacheDev& cache,
                                               const m3ProxyDev* proxyA,
                                               const m3SweepDev* sweepA,
                                               const m3ProxyDev* proxyB,
                                               const m3SweepDev* sweepB, m3Vec3 worldNormal,
                                               m3real t1)
{
    m3SeparationDev fcn;
    fcn.proxyA = proxyA;
    fcn.proxyB = proxyB;
    fcn.sweepA = sweepA;
    fcn.sweepB = sweepB;
    fcn.witness1 = worldNormal;
    fcn.witness2 = v3(0.0f, 0.0f, 0.0f);
    fcn.type = M3_SEP_VERTICES;

    const int32_t indexA[3] = {cache.indexA[0], cache.indexA[1], cache.indexA[2]};
    const int32_t indexB[3] = {cache.indexB[0], cache.indexB[1], cache.indexB[2]};
    const int32_t count = cache.count < 3 ? cache.count : 3;
    const int32_t uniqueA = m3ToiUniqueCount(count, indexA);
    const int32_t uniqueB = m3ToiUniqueCount(count, indexB);

    const m3Transform xfA1 = m3SweepAt(*sweepA, t1);
    const m3Transform xfB1 = m3SweepAt(*sweepB, t1);
    const m3Vec3 deltaP = v3((m3real)(xfB1.p.x - xfA1.p.x), (m3real)(xfB1.p.y - xfA1.p.y),
                             (m3real)(xfB1.p.z - xfA1.p.z));

    if (count == 2 || (count == 3 && uniqueA <= 2 && uniqueB <= 2))
    {
        int32_t ia[2];
        int32_t ib[2];
        if (count == 2 && uniqueA == 2 && uniqueB == 2)
        {
            ia[0] = indexA[0];
            ia[1] = indexA[1];
            ib[0] = indexB[0];
            ib[1] = indexB[1];
        }
        else if (count == 3 && uniqueA == 2 && uniqueB == 2)
        {
            ia[0] = indexA[0];
            ia[1] = indexA[0] != indexA[1] ? indexA[1] : indexA[2];
            ib[0] = indexB[0];
            ib[1] = indexB[0] != indexB[1] ? indexB[1] : indexB[2];
        }
        else
        {
            return fcn; // vertex versus edge: the world axis
        }
        const m3Vec3 vA1 = proxyA->points[ia[0]];
        const m3Vec3 localEdgeA = m3Normalize3(m3Sub3(proxyA->points[ia[1]], vA1));
        const m3Vec3 edgeA = m3RotateVec3(xfA1.q, localEdgeA);
        const m3Vec3 vB1 = proxyB->points[ib[0]];
        m3Vec3 localEdgeB = m3Normalize3(m3Sub3(proxyB->points[ib[1]], vB1));
        const m3Vec3 edgeB = m3RotateVec3(xfB1.q, localEdgeB);
        m3Vec3 axis = m3Cross3(edgeA, edgeB);
        const m3real len2 = m3Dot3(axis, axis);
        const m3real tolerance2 = count == 2 ? 0.05f * 0.05f : 0.005f * 0.005f;
        if (len2 < tolerance2)
        {
            return fcn; // near parallel: the world axis
        }
        const m3Vec3 delta =
            m3Add3(m3Sub3(m3RotateVec3(xfB1.q, vB1), m3RotateVec3(xfA1.q, vA1)), deltaP);
        if (m3Dot3(delta, axis) < 0.0f)
        {
            axis = m3Neg3(axis);
            localEdgeB = m3Neg3(localEdgeB);
        }
        if (m3ToiFastEdges(*sweepA, *sweepB, localEdgeA, localEdgeB, axis))
        {
            fcn.witness1 = m3Normalize3(axis); // unsafe: a fixed world axis
            return fcn;
        }
        fcn.type = M3_SEP_EDGES;
        fcn.witness1 = localEdgeA;
        fcn.witness2 = localEdgeB;
        return fcn;
    }

    if (count == 3 && uniqueA == 3)
    {
        const m3Vec3 vA1 = proxyA->points[indexA[0]];
        const m3Vec3 vA2 = proxyA->points[indexA[1]];
        const m3Vec3 vA3 = proxyA->points[indexA[2]];
        m3Vec3 localAxisA = m3Normalize3(m3Cross3(m3Sub3(vA2, vA1), m3Sub3(vA3, vA1)));
        const m3Vec3 axisA = m3RotateVec3(xfA1.q, localAxisA);
        const m3Vec3 localPointA = m3MulSV3(1.0f / 3.0f, m3Add3(m3Add3(vA1, vA2), vA3));
        const m3Vec3 localPointB = proxyB->points[indexB[0]];
        const m3Vec3 delta = m3Add3(
            m3Sub3(m3RotateVec3(xfB1.q, localPointB), m3RotateVec3(xfA1.q, localPointA)), deltaP);
        if (m3Dot3(delta, axisA) < 0.0f)
        {
            localAxisA = m3Neg3(localAxisA);
        }
        fcn.type = M3_SEP_FACE_A;
        fcn.witness1 = localAxisA;
        fcn.witness2 = localPointA;
        return fcn;
    }
    if (count == 3 && uniqueB == 3)
    {
        const m3Vec3 vB1 = proxyB->points[indexB[0]];
        const m3Vec3 vB2 = proxyB->points[indexB[1]];
        const m3Vec3 vB3 = proxyB->points[indexB[2]];
        m3Vec3 localAxisB = m3Normalize3(m3Cross3(m3Sub3(vB2, vB1), m3Sub3(vB3, vB1)));
        const m3Vec3 axisB = m3RotateVec3(xfB1.q, localAxisB);
        const m3Vec3 localPointA = proxyA->points[indexA[0]];
        const m3Vec3 localPointB = m3MulSV3(1.0f / 3.0f, m3Add3(m3Add3(vB1, vB2), vB3));
        const m3Vec3 delta = m3Sub3(
            m3Sub3(m3RotateVec3(xfA1.q, localPointA), m3RotateVec3(xfB1.q, localPointB)), deltaP);
        if (m3Dot3(delta, axisB) < 0.0f)
        {
            localAxisB = m3Neg3(localAxisB);
        }
        fcn.type = M3_SEP_FACE_B;
        fcn.witness1 = localAxisB;
        fcn.witness2 = localPointB;
        return fcn;
    }
    return fcn;
}

// distance.c:939-994
__device__ m3real m3ToiFindMinSeparation(const m3SeparationDev& f, int32_t* indexA,
                                         int32_t* indexB, m3real t)
{
    const m3Transform xfA = m3SweepAt(*f.sweepA, t);
    const m3Transform xfB = m3SweepAt(*f.sweepB, t);
    const m3Vec3 deltaP = v3((m3real)(xfB.p.x - xfA.p.x), (m3real)(xfB.p.y - xfA.p.y),
                             (m3real)(xfB.p.z - xfA.p.z));
    switch (f.type)
    {
    case M3_SEP_VERTICES:
    {
        const m3Vec3 axis = f.witness1;
        *indexA = m3ToiSupport(*f.proxyA, m3InvRotateVec3(xfA.q, axis));
        *indexB = m3ToiSupport(*f.proxyB, m3InvRotateVec3(xfB.q, m3Neg3(axis)));
        const m3Vec3 delta = m3Add3(m3Sub3(m3RotateVec3(xfB.q, f.proxyB->points[*indexB]),
                                           m3RotateVec3(xfA.q, f.proxyA->points[*indexA])),
                                    deltaP);
        return m3Dot3(delta, axis);
    }
    case M3_SEP_EDGES:
    {
        const m3Vec3 edgeA = m3RotateVec3(xfA.q, f.witness1);
        const m3Vec3 edgeB = m3RotateVec3(xfB.q, f.witness2);
        const m3Vec3 axis = m3Normalize3(m3Cross3(edgeA, edgeB));
        *indexA = m3ToiSupport(*f.proxyA, m3InvRotateVec3(xfA.q, axis));
        *indexB = m3ToiSupport(*f.proxyB, m3InvRotateVec3(xfB.q, m3Neg3(axis)));
        const m3Vec3 delta = m3Add3(m3Sub3(m3RotateVec3(xfB.q, f.proxyB->points[*indexB]),
                                           m3RotateVec3(xfA.q, f.proxyA->points[*indexA])),
                                    deltaP);
        return m3Dot3(delta, axis);
    }
    case M3_SEP_FACE_A:
    {
        const m3Vec3 normal = m3RotateVec3(xfA.q, f.witness1);
        *indexA = -1;
        const m3Vec3 pointA = m3ToiPoint(xfA, f.witness2);
        *indexB = m3ToiSupport(*f.proxyB, m3InvRotateVec3(xfB.q, m3Neg3(normal)));
        const m3Vec3 pointB = m3ToiPoint(xfB, f.proxyB->points[*indexB]);
        return m3Dot3(m3Sub3(pointB, pointA), normal);
    }
    default:
    {
        const m3Vec3 normal = m3RotateVec3(xfB.q, f.witness1);
        *indexA = m3ToiSupport(*f.proxyA, m3InvRotateVec3(xfA.q, m3Neg3(normal)));
        const m3Vec3 pointA = m3ToiPoint(xfA, f.proxyA->points[*indexA]);
        *indexB = -1;
        const m3Vec3 pointB = m3ToiPoint(xfB, f.witness2);
        return m3Dot3(m3Sub3(pointA, pointB), normal);
    }
    }
}

// distance.c:996-1036
__device__ m3real m3ToiEvaluateSeparation(const m3SeparationDev& f, int32_t indexA,
                                          int32_t indexB, m3real t)
{
    const m3Transform xfA = m3SweepAt(*f.sweepA, t);
    const m3Transform xfB = m3SweepAt(*f.sweepB, t);
    switch (f.type)
    {
    case M3_SEP_VERTICES:
    {
        const m3Vec3 pointA = m3ToiPoint(xfA, f.proxyA->points[indexA]);
        const m3Vec3 pointB = m3ToiPoint(xfB, f.proxyB->points[indexB]);
        return m3Dot3(m3Sub3(pointB, pointA), f.witness1);
    }
    case M3_SEP_EDGES:
    {
        const m3Vec3 edgeA = m3RotateVec3(xfA.q, f.witness1);
        const m3Vec3 edgeB = m3RotateVec3(xfB.q, f.witness2);
        const m3Vec3 axis = m3Normalize3(m3Cross3(edgeA, edgeB));
        const m3Vec3 pointA = m3ToiPoint(xfA, f.proxyA->points[indexA]);
        const m3Vec3 pointB = m3ToiPoint(xfB, f.proxyB->points[indexB]);
        return m3Dot3(m3Sub3(pointB, pointA), axis);
    }
    case M3_SEP_FACE_A:
    {
        const m3Vec3 axis = m3RotateVec3(xfA.q, f.witness1);
        const m3Vec3 pointA = m3ToiPoint(xfA, f.witness2);
        const m3Vec3 pointB = m3ToiPoint(xfB, f.proxyB->points[indexB]);
        return m3Dot3(m3Sub3(pointB, pointA), axis);
    }
    default:
    {
        const m3Vec3 axis = m3RotateVec3(xfB.q, f.witness1);
        const m3Vec3 pointA = m3ToiPoint(xfA, f.proxyA->points[indexA]);
        const m3Vec3 pointB = m3ToiPoint(xfB, f.witness2);
        return m3Dot3(m3Sub3(pointA, pointB), axis);
    }
    }
}

// distance.c:1026-1036
__device__ __forceinline__ void m3ToiForceFixedAxis(m3SeparationDev* f, m3real t)
{
    const m3Transform xfA = m3SweepAt(*f->sweepA, t);
    const m3Transform xfB = m3SweepAt(*f->sweepB, t);
    const m3Vec3 edgeA = m3RotateVec3(xfA.q, f->witness1);
    const m3Vec3 edgeB = m3RotateVec3(xfB.q, f->witness2);
    f->witness1 = m3Normalize3(m3Cross3(edgeA, edgeB));
    f->witness2 = v3(0.0f, 0.0f, 0.0f);
    f->type = M3_SEP_VERTICES;
}

enum
{
    M3_TOI_UNKNOWN = 0,
    M3_TOI_FAILED = 1,
    M3_TOI_OVERLAPPED = 2,
    M3_TOI_HIT = 3,
    M3_TOI_SEPARATED = 4,
};

// distance.c:1039-1215: the fraction of the sweep at which the proxies
// first come within the target distance; `state` one of M3_TOI_*.
__device__ __noinline__ m3real m3TimeOfImpactDev(const m3ProxyDev& proxyA, m3SweepDev sweepA,
                                    const m3ProxyDev& proxyB, m3SweepDev sweepB,
                                    m3real maxFraction, int32_t* state)
{
    *state = M3_TOI_UNKNOWN;
    m3real fraction = maxFraction;

    // Both sweeps shifted so that A starts at the origin.
    const m3Vec3 origin = sweepA.c1;
    sweepA.c1 = m3Sub3(sweepA.c1, origin);
    sweepA.c2 = m3Sub3(sweepA.c2, origin);
    sweepB.c1 = m3Sub3(sweepB.c1, origin);
    sweepB.c2 = m3Sub3(sweepB.c2, origin);

    const m3real linearSlop = 0.005f;
    const m3real totalRadius = proxyA.radius + proxyB.radius;
    const m3real target = m3MaxF(linearSlop, totalRadius - linearSlop);
    const m3real tolerance = 0.25f * linearSlop;
    const m3real tMax = maxFraction;
    const int32_t maxPushBackIterations = proxyA.count + proxyB.count;
    m3real t1 = 0.0f;
    const int32_t maxIterations = 25;
    int32_t distanceIterations = 0;

    m3SimplexCacheDev cache;
    cache.count = 0;
    cache.metric = 0.0f;

    for (;;)
    {
        const m3Transform xfA = m3SweepAt(sweepA, t1);
        const m3Transform xfB = m3SweepAt(sweepB, t1);
        const m3Quat conjA = q4(-xfA.q.x, -xfA.q.y, -xfA.q.z, xfA.q.w);
        const m3Quat q = m3MulQuat(conjA, xfB.q);
        const m3Vec3 dp = v3((m3real)(xfB.p.x - xfA.p.x), (m3real)(xfB.p.y - xfA.p.y),
                             (m3real)(xfB.p.z - xfA.p.z));
        const m3Vec3 p = m3InvRotateVec3(xfA.q, dp);
        const m3DistanceOutDev out = m3ShapeDistanceDev(proxyA, proxyB, q, p, &cache);
        distanceIterations += 1;

        if (out.distance <= 0.0f)
        {
            *state = M3_TOI_OVERLAPPED;
            fraction = 0.0f;
            break;
        }
        if (out.distance <= target + tolerance)
        {
            *state = M3_TOI_HIT;
            fraction = t1;
            break;
        }
        if (distanceIterations == maxIterations)
        {
            *state = M3_TOI_FAILED;
            fraction = t1;
            break;
        }

        const m3Vec3 worldNormal = m3RotateVec3(xfA.q, out.normal);
        m3SeparationDev function =
            m3ToiMakeSeparation(cache, &proxyA, &sweepA, &proxyB, &sweepB, worldNormal, t1);

        bool done = false;
        m3real t2 = tMax;
        int32_t pushBackIterations = 0;
        for (;;)
        {
            int32_t indexA;
            int32_t indexB;
            m3real s2 = m3ToiFindMinSeparation(function, &indexA, &indexB, t2);
            if (s2 - target > tolerance)
            {
                *state = M3_TOI_SEPARATED;
                fraction = tMax;
                done = true;
                break;
            }
            if (s2 >= target - tolerance)
            {
                t1 = t2;
                break;
            }
            m3real s1 = m3ToiEvaluateSeparation(function, indexA, indexB, t1);
            if (s1 < target - tolerance)
            {
                *state = M3_TOI_FAILED;
                fraction = t1;
                done = true;
                break;
            }
            if (s1 <= target + tolerance)
            {
                *state = M3_TOI_HIT;
                fraction = t1;
                done = true;
                break;
            }

            // Root of s(t) = target: false position and bisection in turn.
            int32_t rootIterationCount = 0;
            const int32_t maxRootIterations = 50;
            m3real a1 = t1;
            m3real a2 = t2;
            for (;;)
            {
                m3real t;
                if (rootIterationCount & 1)
                {
                    t = a1 + (target - s1) * (a2 - a1) / (s2 - s1);
                }
                else
                {
                    t = 0.5f * (a1 + a2);
                }
                rootIterationCount += 1;
                const m3real sv = m3ToiEvaluateSeparation(function, indexA, indexB, t);
                const m3real err = sv - target;
                if ((err < 0.0f ? -err : err) <= tolerance)
                {
                    t2 = t;
                    break;
                }
                if (sv > target)
                {
                    a1 = t;
                    s1 = sv;
                }
                else
                {
                    a2 = t;
                    s2 = sv;
                }
                if (rootIterationCount == maxRootIterations)
                {
                    break;
                }
            }
            if (rootIterationCount == maxRootIterations - 1 && function.type == M3_SEP_EDGES)
            {
                t2 = tMax;
                m3ToiForceFixedAxis(&function, t1);
            }
            pushBackIterations += 1;
            if (pushBackIterations == maxPushBackIterations)
            {
                break;
            }
        }
        if (done)
        {
            break;
        }
    }
    return fraction;
}

#endif // M3_TOI_CUH
