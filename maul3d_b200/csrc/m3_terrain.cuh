// Heightfield versus convex narrowphase on the device (manifold.c:693-
// 2071): the convex's reach picks a window of grid cells (one halo cell
// each way, at most 16 per axis), the window is read as a triangle mesh
// in the heightfield's frame, every window triangle runs the sphere,
// capsule or hull triangle kernel, and the welded acceptance keeps face
// contacts first and then the edge and vertex contacts whose features
// are still unclaimed.  The accepted contacts cluster around the deepest
// one's normal and the deepest four points of the cluster become the
// pair's manifold.
//
// Same arithmetic as the reference, different bookkeeping, chosen for a
// thread that owns one pair:
//   * the window mesh is never built: a triangle's vertices and indices
//     come straight from the grid (the reference's triangulation rule,
//     alternating diagonals by cell parity);
//   * the edge convexity flags (shape.c:304-348) are computed only for
//     the triangles that need them, and the neighbour across an edge is
//     found among the (at most two) triangles of the cells beside that
//     edge instead of by a search of the whole window: in a grid every
//     edge has at most one other triangle, so this is the triangle the
//     search finds;
//   * candidates keep 12 bytes (squared distance, deepest separation,
//     triangle, feature) and a triangle's contact is recomputed when its
//     points are needed (the same inputs give the same bits);
//   * claimed edges and vertices are bits over the window's vertices;
//     at most 64 accepted triangles claim at most 192 of each, which is
//     the reference's list capacity, so no claim is ever dropped there;
//   * the deepest four points are kept while the cluster streams by (the
//     reference's repeated minimum over (separation, id) selects the same
//     four: ids are unique within a pair).
#ifndef M3_TERRAIN_CUH
#define M3_TERRAIN_CUH

#include "m3_distance.cuh"

#define M3_HF_WINDOW 16         // cells per axis, halo included (manifold.c:1922)
#define M3_MESH_CANDIDATE_CAP 64 // manifold.c:1457
#define M3_MESH_CLIP_CAP 16      // manifold.c:1073
#define M3_TRI_FEATURE_HULL_FACE 8
#define M3_HF_MAX_VERTS ((M3_HF_WINDOW + 1) * (M3_HF_WINDOW + 1))

// One triangle's contact in the heightfield frame (manifold.c:769-781).
struct m3TriManifoldDev
{
    m3Vec3 normal;
    m3Vec3 triNormal;
    m3real dist2;
    int32_t pointCount;
    int32_t feature; // vertex bit mask, 7 = face interior, 8 = hull face
    m3Vec3 point[4];
    m3real separation[4];
    uint16_t localId[4];
};

// manifold.c:716-761: closest point on triangle abc to q and its Voronoi
// feature (vertex bit mask, 7 = interior).
__device__ __forceinline__ m3Vec3 m3ClosestOnTriangle(m3Vec3 a, m3Vec3 b, m3Vec3 c, m3Vec3 q,
                                                      int32_t* feature)
{
    const m3Vec3 ab = m3Sub3(b, a);
    const m3Vec3 ac = m3Sub3(c, a);
    const m3Vec3 aq = m3Sub3(q, a);
    const m3real d1 = m3Dot3(ab, aq);
    const m3real d2 = m3Dot3(ac, aq);
    if (d1 <= 0.0f && d2 <= 0.0f)
    {
        *feature = 1;
        return a;
    }
    const m3Vec3 bq = m3Sub3(q, b);
    const m3real d3 = m3Dot3(ab, bq);
    const m3real d4 = m3Dot3(ac, bq);
    if (d3 > 0.0f && d4 <= d3)
    {
        *feature = 2;
        return b;
    }
    const m3real vc = d1 * d4 - d3 * d2;
    if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f)
    {
        const m3real t = d1 / (d1 - d3);
        *feature = 1 | 2;
        return m3Add3(a, m3MulSV3(t, ab));
    }
    const m3Vec3 cq = m3Sub3(q, c);
    const m3real d5 = m3Dot3(ab, cq);
    const m3real d6 = m3Dot3(ac, cq);
    if (d6 >= 0.0f && d5 <= d6)
    {
        *feature = 4;
        return c;
    }
    const m3real vb = d5 * d2 - d1 * d6;
    if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f)
    {
        const m3real t = d2 / (d2 - d6);
        *feature = 1 | 4;
        return m3Add3(a, m3MulSV3(t, ac));
    }
    const m3real va = d3 * d6 - d5 * d4;
    if (va <= 0.0f && d4 >= d3 && d5 >= d6)
    {
        const m3real t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        *feature = 2 | 4;
        return m3Add3(b, m3MulSV3(t, m3Sub3(c, b)));
    }
    const m3real t1 = vb / (va + vb + vc);
    const m3real t2 = vc / (va + vb + vc);
    *feature = 7;
    return m3Add3(a, m3Add3(m3MulSV3(t1, ab), m3MulSV3(t2, ac)));
}

// manifold.c:783-811
__device__ void m3SphereTriangleDev(m3TriManifoldDev* out, m3Vec3 center, m3real radius,
                                    const m3Vec3 tri[3])
{
    out->pointCount = 0;
    const m3Vec3 triN = m3Cross3(m3Sub3(tri[1], tri[0]), m3Sub3(tri[2], tri[0]));
    if (m3Dot3(triN, m3Sub3(center, tri[0])) < 0.0f)
    {
        return; // back side
    }
    int32_t feature;
    const m3Vec3 closest = m3ClosestOnTriangle(tri[0], tri[1], tri[2], center, &feature);
    const m3Vec3 d = m3Sub3(center, closest);
    const m3real dist2 = m3Dot3(d, d);
    const m3real reach = radius + M3_SPECULATIVE_DISTANCE;
    if (dist2 > reach * reach)
    {
        return;
    }
    const m3real dist = sqrtf(dist2);
    const m3Vec3 normal =
        dist2 > 1000.0f * M3_FLT_MIN ? m3MulSV3(1.0f / dist, d) : m3Normalize3(triN);
    out->normal = normal;
    out->triNormal = m3Normalize3(triN);
    out->dist2 = dist2;
    out->feature = feature;
    out->pointCount = 1;
    out->separation[0] = dist - radius;
    out->point[0] = m3MulSV3(0.5f, m3Add3(m3Sub3(center, m3MulSV3(radius, normal)), closest));
    out->localId[0] = 0;
}

// manifold.c:814-851: the segment clipped to the triangle's side planes;
// false when fewer than two points survive a plane.
__device__ bool m3ClipSegmentToTriFace(m3Vec3 segment[2], const m3Vec3 tri[3], m3Vec3 faceNormal)
{
    m3Vec3 vertex1 = tri[2];
    for (int32_t i = 0; i < 3; ++i)
    {
        const m3Vec3 vertex2 = tri[i];
        const m3Vec3 tangent = m3Normalize3(m3Sub3(vertex2, vertex1));
        const m3Vec3 binormal = m3Cross3(tangent, faceNormal);
        const m3real planeOff = m3Dot3(binormal, vertex1);
        const m3Vec3 p1 = segment[0];
        const m3Vec3 p2 = segment[1];
        const m3real distance1 = m3Dot3(binormal, p1) - planeOff;
        const m3real distance2 = m3Dot3(binormal, p2) - planeOff;
        int32_t vertexCount = 0;
        m3Vec3 kept[3];
        if (distance1 <= 0.0f)
        {
            kept[vertexCount++] = p1;
        }
        if (distance2 <= 0.0f)
        {
            kept[vertexCount++] = p2;
        }
        if (distance1 * distance2 < 0.0f)
        {
            const m3real t = distance1 / (distance1 - distance2);
            kept[vertexCount++] = m3Add3(p1, m3MulSV3(t, m3Sub3(p2, p1)));
        }
        if (vertexCount != 2)
        {
            return false;
        }
        segment[0] = kept[0];
        segment[1] = kept[1];
        vertex1 = vertex2;
    }
    return true;
}

// manifold.c:854-873: closest points of two infinite lines, as fractions.
__device__ __forceinline__ void m3LineClosest(m3Vec3 p1, m3Vec3 d1, m3Vec3 p2, m3Vec3 d2,
                                              m3real* f1, m3real* f2)
{
    const m3real a11 = m3Dot3(d1, d1);
    const m3real a12 = -m3Dot3(d1, d2);
    const m3real a21 = m3Dot3(d2, d1);
    const m3real a22 = -m3Dot3(d2, d2);
    const m3Vec3 w = m3Sub3(p1, p2);
    const m3real b1 = -m3Dot3(d1, w);
    const m3real b2 = -m3Dot3(d2, w);
    const m3real det = a11 * a22 - a12 * a21;
    if (det * det < 1000.0f * M3_FLT_MIN)
    {
        *f1 = a11 > 0.0f ? m3Dot3(m3Sub3(p2, p1), d1) / a11 : 0.0f;
        *f2 = 0.0f;
        return;
    }
    *f1 = (a22 * b1 - a12 * b2) / det;
    *f2 = (a11 * b2 - a21 * b1) / det;
}

// manifold.c:876-907: edge-edge separation with the orientation guard.
__device__ __forceinline__ m3real m3EdgeEdgeSepDev(m3Vec3 p1, m3Vec3 e1, m3Vec3 c1, m3Vec3 p2,
                                                   m3Vec3 e2, m3Vec3 c2)
{
    const m3Vec3 u = m3Cross3(e1, e2);
    const m3real length2 = m3Dot3(u, u);
    const m3real scale2 = m3Dot3(e1, e1) * m3Dot3(e2, e2);
    if (length2 < 0.005f * 0.005f * scale2 || length2 < 1000.0f * M3_FLT_MIN)
    {
        return -3.4e38f;
    }
    m3Vec3 n = m3MulSV3(1.0f / sqrtf(length2), u);
    const m3real sign1 = m3Dot3(n, m3Sub3(p1, c1));
    const m3real sign2 = m3Dot3(n, m3Sub3(p2, c2));
    const m3real a1 = sign1 < 0.0f ? -sign1 : sign1;
    const m3real a2 = sign2 < 0.0f ? -sign2 : sign2;
    if (a1 > a2)
    {
        if (sign1 < 0.0f)
        {
            n = m3Neg3(n);
        }
    }
    else
    {
        if (sign2 > 0.0f)
        {
            n = m3Neg3(n);
        }
    }
    return m3Dot3(n, m3Sub3(p2, p1));
}

// manifold.c:911-1071: capsule versus one triangle.
__device__ void m3CapsuleTriangleDev(m3TriManifoldDev* out, m3Vec3 c1, m3Vec3 c2, m3real radius,
                                     const m3Vec3 tri[3])
{
    out->pointCount = 0;
    const m3Vec3 triN = m3Normalize3(m3Cross3(m3Sub3(tri[1], tri[0]), m3Sub3(tri[2], tri[0])));
    const m3real triOff = m3Dot3(triN, tri[0]);
    const m3Vec3 mid = m3MulSV3(0.5f, m3Add3(c1, c2));
    if (m3Dot3(triN, mid) - triOff < 0.0f)
    {
        return; // back side
    }
    out->triNormal = triN;

    const m3Vec3 segPts[2] = {c1, c2};
    m3ProxyDev proxyA;
    proxyA.points = tri;
    proxyA.count = 3;
    proxyA.radius = 0.0f;
    m3ProxyDev proxyB;
    proxyB.points = segPts;
    proxyB.count = 2;
    proxyB.radius = 0.0f;
    m3SimplexCacheDev cache;
    cache.count = 0;
    cache.metric = 0.0f;
    const m3DistanceOutDev dOut = m3ShapeDistanceDev(proxyA, proxyB, q4(0.0f, 0.0f, 0.0f, 1.0f),
                                                     v3(0.0f, 0.0f, 0.0f), &cache);
    const int32_t cacheMask = m3CacheMaskA(cache);
    if (dOut.distance > radius + M3_SPECULATIVE_DISTANCE)
    {
        return;
    }

    if (dOut.distance > 100.0f * M3_FLT_EPSILON)
    {
        const m3Vec3 delta = m3Normalize3(m3Sub3(dOut.pointB, dOut.pointA));
        m3real cosAngle = m3Dot3(triN, delta);
        cosAngle = cosAngle < 0.0f ? -cosAngle : cosAngle;
        if (cosAngle > 0.2f)
        {
            m3Vec3 segment[2] = {c1, c2};
            if (m3ClipSegmentToTriFace(segment, tri, triN))
            {
                out->normal = triN;
                out->dist2 = dOut.distance * dOut.distance;
                out->feature = 7;
                out->pointCount = 2;
                for (int32_t k = 0; k < 2; ++k)
                {
                    const m3real d = m3Dot3(triN, segment[k]) - triOff;
                    out->separation[k] = d - radius;
                    out->point[k] = m3Sub3(segment[k], m3MulSV3(0.5f * (radius + d), triN));
                    out->localId[k] = (uint16_t)k;
                }
                return;
            }
        }
        out->normal = delta;
        out->dist2 = dOut.distance * dOut.distance;
        out->feature = cacheMask == 0 ? 7 : cacheMask;
        out->pointCount = 1;
        out->separation[0] = dOut.distance - radius;
        out->point[0] =
            m3MulSV3(0.5f, m3Add3(dOut.pointA, m3Sub3(dOut.pointB, m3MulSV3(radius, delta))));
        out->localId[0] = 0;
        return;
    }

    // Deep: face query versus edge query.
    const m3real sep1 = m3Dot3(triN, c1) - triOff;
    const m3real sep2 = m3Dot3(triN, c2) - triOff;
    const m3real faceQuerySep = m3MinF(sep1, sep2);
    if (faceQuerySep > radius)
    {
        return;
    }
    const m3Vec3 capDir = m3Sub3(c2, c1);
    const m3Vec3 triCenter = m3MulSV3(1.0f / 3.0f, m3Add3(tri[0], m3Add3(tri[1], tri[2])));
    m3real bestEdgeSep = -3.4e38f;
    int32_t bestEdge = 0;
    for (int32_t k = 0; k < 3; ++k)
    {
        const m3Vec3 v1 = tri[k];
        const m3Vec3 e = m3Sub3(tri[(k + 1) % 3], v1);
        const m3real sep = m3EdgeEdgeSepDev(v1, e, triCenter, c1, capDir, mid);
        if (sep > bestEdgeSep)
        {
            bestEdgeSep = sep;
            bestEdge = k;
        }
    }
    if (bestEdgeSep > radius)
    {
        return;
    }

    m3real faceSeparation = faceQuerySep - radius;
    m3Vec3 segment[2] = {c1, c2};
    if (m3ClipSegmentToTriFace(segment, tri, triN))
    {
        out->normal = triN;
        out->dist2 = 0.0f;
        out->feature = 7;
        out->pointCount = 2;
        m3real minSep = 3.4e38f;
        for (int32_t k = 0; k < 2; ++k)
        {
            const m3real d = m3Dot3(triN, segment[k]) - triOff;
            out->separation[k] = d - radius;
            minSep = m3MinF(minSep, out->separation[k]);
            out->point[k] = m3Sub3(segment[k], m3MulSV3(0.5f * (radius + d), triN));
            out->localId[k] = (uint16_t)k;
        }
        faceSeparation = minSep;
    }

    const m3real edgeSeparation = bestEdgeSep - radius;
    if (out->pointCount == 0 || edgeSeparation > 0.5f * faceSeparation + 0.005f)
    {
        const m3Vec3 v1 = tri[bestEdge];
        const m3Vec3 triEdge = m3Sub3(tri[(bestEdge + 1) % 3], v1);
        m3Vec3 normal = m3Normalize3(m3Cross3(capDir, triEdge));
        if (m3Dot3(normal, m3Sub3(v1, triCenter)) < 0.0f)
        {
            normal = m3Neg3(normal);
        }
        m3real f1;
        m3real f2;
        m3LineClosest(v1, triEdge, c1, capDir, &f1, &f2);
        if (f1 < 0.0f || f1 > 1.0f || f2 < 0.0f || f2 > 1.0f)
        {
            return;
        }
        const m3Vec3 onTriEdge = m3Add3(v1, m3MulSV3(f1, triEdge));
        const m3Vec3 onCapCore = m3Add3(c1, m3MulSV3(f2, capDir));
        const m3real separation = m3Dot3(normal, m3Sub3(onCapCore, onTriEdge));
        out->normal = normal;
        out->dist2 = separation > 0.0f ? separation * separation : 0.0f;
        out->feature = (1 << bestEdge) | (1 << ((bestEdge + 1) % 3));
        out->pointCount = 1;
        out->separation[0] = separation - radius;
        out->point[0] =
            m3MulSV3(0.5f, m3Add3(m3Sub3(onCapCore, m3MulSV3(radius, normal)), onTriEdge));
        out->localId[0] = 0;
    }
}

struct m3MeshClipVertexDev
{
    m3Vec3 position;
    m3real separation;
};

// manifold.c:1083-1111: one Sutherland-Hodgman step, separations taken
// against the reference plane for the new points.
__device__ int32_t m3MeshClipPolygonDev(m3MeshClipVertexDev* out, const m3MeshClipVertexDev* in,
                                        int32_t count, m3Vec3 clipNormal, m3real clipOffset,
                                        m3Vec3 refNormal, m3real refOffset)
{
    int32_t outCount = 0;
    m3MeshClipVertexDev prev = in[count - 1];
    m3real prevDist = m3Dot3(clipNormal, prev.position) - clipOffset;
    for (int32_t i = 0; i < count; ++i)
    {
        const m3MeshClipVertexDev curr = in[i];
        const m3real currDist = m3Dot3(clipNormal, curr.position) - clipOffset;
        if (prevDist <= 0.0f)
        {
            out[outCount++] = prev;
        }
        if (prevDist * currDist < 0.0f)
        {
            const m3real t = prevDist / (prevDist - currDist);
            const m3Vec3 p =
                m3Add3(prev.position, m3MulSV3(t, m3Sub3(curr.position, prev.position)));
            out[outCount].position = p;
            out[outCount].separation = m3Dot3(refNormal, p) - refOffset;
            outCount += 1;
        }
        prev = curr;
        prevDist = currDist;
    }
    return outCount;
}

// manifold.c:1114-1165: the deepest four clip points (ties to the lower
// slot) in ascending slot order, those within the margin emitted.
__device__ void m3KeepDeepestClipDev(m3TriManifoldDev* out, const m3MeshClipVertexDev* points,
                                     int32_t count)
{
    int32_t kept[4];
    int32_t keptCount = 0;
    uint32_t used = 0;
    const int32_t want = count < 4 ? count : 4;
    for (int32_t k = 0; k < want; ++k)
    {
        int32_t best = -1;
        for (int32_t c = 0; c < count; ++c)
        {
            if ((used >> c) & 1u)
            {
                continue;
            }
            if (best < 0 || points[c].separation < points[best].separation)
            {
                best = c;
            }
        }
        used |= 1u << best;
        kept[keptCount++] = best;
    }
    for (int32_t a = 0; a < keptCount; ++a)
    {
        for (int32_t b = a + 1; b < keptCount; ++b)
        {
            if (kept[b] < kept[a])
            {
                const int32_t tmp = kept[a];
                kept[a] = kept[b];
                kept[b] = tmp;
            }
        }
    }
    out->pointCount = 0;
    for (int32_t k = 0; k < keptCount; ++k)
    {
        const int32_t c = kept[k];
        if (points[c].separation > M3_SPECULATIVE_DISTANCE)
        {
            continue;
        }
        const int32_t slot = out->pointCount;
        out->point[slot] =
            m3Sub3(points[c].position, m3MulSV3(0.5f * points[c].separation, out->normal));
        out->separation[slot] = points[c].separation;
        out->localId[slot] = (uint16_t)slot;
        out->pointCount += 1;
    }
}

// The first half-edge of a hull face, or -1.
__device__ __forceinline__ int32_t m3HullFaceEdge(const m3HullData* hull, int32_t face)
{
    for (int32_t e = 0; e < hull->edgeCount; ++e)
    {
        if (hull->edges[e].face == (uint8_t)face)
        {
            return e;
        }
    }
    return -1;
}

// manifold.c:1172-1455: hull versus one triangle, in the hull's frame.
__device__ void m3HullTriangleDev(m3TriManifoldDev* out, const m3HullData* hull,
                                  const m3Vec3 tri[3])
{
    out->pointCount = 0;
    const m3real linearSlop = 0.005f;
    const m3Vec3 triN = m3Normalize3(m3Cross3(m3Sub3(tri[1], tri[0]), m3Sub3(tri[2], tri[0])));
    const m3real triOff = m3Dot3(triN, tri[0]);
    out->triNormal = triN;
    if (m3Dot3(triN, hull->center) - triOff < -linearSlop)
    {
        return; // back side
    }
    const m3Vec3 triCenter = m3MulSV3(1.0f / 3.0f, m3Add3(tri[0], m3Add3(tri[1], tri[2])));
    const m3Vec3 triEdge[3] = {m3Sub3(tri[1], tri[0]), m3Sub3(tri[2], tri[1]),
                               m3Sub3(tri[0], tri[2])};

    // Face query A: the triangle's face against the hull's support.
    m3real sepA = 3.4e38f;
    for (int32_t v = 0; v < hull->vertexCount; ++v)
    {
        sepA = m3MinF(sepA, m3Dot3(triN, hull->vertices[v]) - triOff);
    }
    if (sepA > M3_SPECULATIVE_DISTANCE)
    {
        return;
    }

    // Face query B: every hull face against the triangle's support.
    int32_t faceB = 0;
    m3real sepB = -3.4e38f;
    for (int32_t f = 0; f < hull->faceCount; ++f)
    {
        const m3Vec3 n = hull->faceNormals[f];
        m3real best = 3.4e38f;
        for (int32_t k = 0; k < 3; ++k)
        {
            best = m3MinF(best, m3Dot3(n, tri[k]) - hull->faceOffsets[f]);
        }
        if (best > sepB)
        {
            sepB = best;
            faceB = f;
        }
    }
    if (sepB > M3_SPECULATIVE_DISTANCE)
    {
        return;
    }

    // Edge query, gated by the Gauss-map test.
    m3real edgeSep = -3.4e38f;
    int32_t edgeTri = -1;
    int32_t edgeHull = -1;
    for (int32_t e = 0; e < hull->edgeCount; e += 2)
    {
        const m3Vec3 hp = hull->vertices[hull->edges[e].origin];
        const m3Vec3 he = m3Sub3(hull->vertices[hull->edges[e + 1].origin], hp);
        const m3Vec3 hn1 = hull->faceNormals[hull->edges[e].face];
        const m3Vec3 hn2 = hull->faceNormals[hull->edges[e + 1].face];
        for (int32_t j = 0; j < 3; ++j)
        {
            const m3real cab = m3Dot3(hn1, triEdge[j]);
            const m3real dab = m3Dot3(hn2, triEdge[j]);
            const m3real bcd = m3Dot3(triN, he);
            if (cab * dab >= 0.0f || cab * bcd <= 0.0f)
            {
                continue;
            }
            const m3real sep =
                m3EdgeEdgeSepDev(tri[j], triEdge[j], triCenter, hp, he, hull->center);
            if (sep > edgeSep)
            {
                edgeSep = sep;
                edgeTri = j;
                edgeHull = e;
            }
        }
    }
    if (edgeSep > M3_SPECULATIVE_DISTANCE)
    {
        return;
    }

    m3real clippedSep = 3.4e38f;
    const m3Vec3 hullFaceN = hull->faceNormals[faceB];
    const bool pushingUp = m3Dot3(hullFaceN, triN) < 0.0f;
    m3MeshClipVertexDev buf1[M3_MESH_CLIP_CAP];
    m3MeshClipVertexDev buf2[M3_MESH_CLIP_CAP];
    if (sepB > sepA + linearSlop && pushingUp)
    {
        // The hull face is the reference: clip the triangle by its sides.
        const m3real refOff = hull->faceOffsets[faceB];
        for (int32_t k = 0; k < 3; ++k)
        {
            buf1[k].position = tri[k];
            buf1[k].separation = m3Dot3(hullFaceN, tri[k]) - refOff;
        }
        int32_t count = 3;
        m3MeshClipVertexDev* input = buf1;
        m3MeshClipVertexDev* output = buf2;
        const int32_t startEdge = m3HullFaceEdge(hull, faceB);
        int32_t edgeIndex = startEdge;
        int32_t guard = 0;
        if (startEdge < 0)
        {
            count = 0;
        }
        while (count > 0)
        {
            const int32_t nextIndex = hull->edges[edgeIndex].next;
            const m3Vec3 vertex1 = hull->vertices[hull->edges[edgeIndex].origin];
            const m3Vec3 vertex2 = hull->vertices[hull->edges[nextIndex].origin];
            const m3Vec3 tangent = m3Normalize3(m3Sub3(vertex2, vertex1));
            const m3Vec3 binormal = m3Cross3(tangent, hullFaceN);
            count = m3MeshClipPolygonDev(output, input, count, binormal, m3Dot3(binormal, vertex1),
                                         hullFaceN, refOff);
            if (count < 3 || count > M3_MESH_CLIP_CAP - 2)
            {
                count = 0;
                break;
            }
            m3MeshClipVertexDev* tmp = input;
            input = output;
            output = tmp;
            edgeIndex = nextIndex;
            if (edgeIndex == startEdge)
            {
                break;
            }
            if (++guard > hull->edgeCount)
            {
                count = 0; // not a closed face loop: no valid hull has one
                break;
            }
        }
        if (count > 0)
        {
            out->normal = m3Neg3(hullFaceN);
            out->feature = M3_TRI_FEATURE_HULL_FACE;
            m3KeepDeepestClipDev(out, input, count);
            clippedSep = 3.4e38f;
            for (int32_t k = 0; k < out->pointCount; ++k)
            {
                clippedSep = m3MinF(clippedSep, out->separation[k]);
            }
        }
    }
    else
    {
        // The triangle is the reference: clip the hull's most
        // anti-parallel face by the triangle's sides.
        int32_t incFace = 0;
        m3real minDot = 3.4e38f;
        for (int32_t f = 0; f < hull->faceCount; ++f)
        {
            const m3real d = m3Dot3(triN, hull->faceNormals[f]);
            if (d < minDot)
            {
                minDot = d;
                incFace = f;
            }
        }
        int32_t count = 0;
        const int32_t startEdge = m3HullFaceEdge(hull, incFace);
        if (startEdge >= 0)
        {
            int32_t edgeIndex = startEdge;
            do
            {
                const m3Vec3 p = hull->vertices[hull->edges[edgeIndex].origin];
                buf1[count].position = p;
                buf1[count].separation = m3Dot3(triN, p) - triOff;
                count += 1;
                edgeIndex = hull->edges[edgeIndex].next;
            } while (edgeIndex != startEdge && count < M3_MESH_CLIP_CAP - 2);
        }
        m3MeshClipVertexDev* input = buf1;
        m3MeshClipVertexDev* output = buf2;
        for (int32_t j = 0; j < 3 && count > 0; ++j)
        {
            const m3Vec3 sideN = m3Normalize3(m3Cross3(triEdge[j], triN));
            count = m3MeshClipPolygonDev(output, input, count, sideN, m3Dot3(sideN, tri[j]), triN,
                                         triOff);
            if (count > M3_MESH_CLIP_CAP - 2)
            {
                count = 0;
                break;
            }
            m3MeshClipVertexDev* tmp = input;
            input = output;
            output = tmp;
        }
        if (count > 0)
        {
            out->normal = triN;
            out->feature = 7;
            m3KeepDeepestClipDev(out, input, count);
            clippedSep = 3.4e38f;
            for (int32_t k = 0; k < out->pointCount; ++k)
            {
                clippedSep = m3MinF(clippedSep, out->separation[k]);
            }
        }
    }

    // The edge axis takes over when it is genuinely better.
    if (edgeTri >= 0)
    {
        const m3real maxFaceSep = m3MaxF(sepA, sepB);
        if ((out->pointCount == 0 && edgeSep > maxFaceSep) ||
            (out->pointCount == 1 && edgeSep > clippedSep + linearSlop))
        {
            const m3Vec3 hp = hull->vertices[hull->edges[edgeHull].origin];
            const m3Vec3 he = m3Sub3(hull->vertices[hull->edges[edgeHull + 1].origin], hp);
            m3Vec3 normal = m3Normalize3(m3Cross3(triEdge[edgeTri], he));
            const m3real outwardA = m3Dot3(normal, m3Sub3(tri[edgeTri], triCenter));
            const m3real outwardB = m3Dot3(normal, m3Sub3(hull->center, hp));
            const m3real aA = outwardA < 0.0f ? -outwardA : outwardA;
            const m3real aB = outwardB < 0.0f ? -outwardB : outwardB;
            if (aA > aB ? outwardA < 0.0f : outwardB < 0.0f)
            {
                normal = m3Neg3(normal);
            }
            m3real f1;
            m3real f2;
            m3LineClosest(tri[edgeTri], triEdge[edgeTri], hp, he, &f1, &f2);
            if (f1 >= 0.0f && f1 <= 1.0f && f2 >= 0.0f && f2 <= 1.0f)
            {
                const m3Vec3 onTri = m3Add3(tri[edgeTri], m3MulSV3(f1, triEdge[edgeTri]));
                const m3Vec3 onHull = m3Add3(hp, m3MulSV3(f2, he));
                const m3real separation = m3Dot3(normal, m3Sub3(onHull, onTri));
                out->pointCount = 1;
                out->normal = normal;
                out->feature = (1 << edgeTri) | (1 << ((edgeTri + 1) % 3));
                out->dist2 = separation > 0.0f ? separation * separation : 0.0f;
                out->point[0] = m3MulSV3(0.5f, m3Add3(onTri, onHull));
                out->separation[0] = separation;
                out->localId[0] = 0;
            }
        }
    }

    // GJK fallback: one witness for a nearby pair the SAT left empty.
    if (out->pointCount == 0)
    {
        m3ProxyDev proxyA;
        proxyA.points = tri;
        proxyA.count = 3;
        proxyA.radius = 0.0f;
        m3ProxyDev proxyB;
        proxyB.points = hull->vertices;
        proxyB.count = hull->vertexCount;
        proxyB.radius = 0.0f;
        m3SimplexCacheDev cache;
        cache.count = 0;
        cache.metric = 0.0f;
        const m3DistanceOutDev dOut = m3ShapeDistanceDev(
            proxyA, proxyB, q4(0.0f, 0.0f, 0.0f, 1.0f), v3(0.0f, 0.0f, 0.0f), &cache);
        const int32_t cacheMask = m3CacheMaskA(cache);
        if (dOut.distance > 0.0f && dOut.distance <= M3_SPECULATIVE_DISTANCE)
        {
            out->pointCount = 1;
            out->normal = dOut.normal;
            out->feature = cacheMask == 0 ? 7 : cacheMask;
            out->dist2 = dOut.distance * dOut.distance;
            out->point[0] = m3MulSV3(0.5f, m3Add3(dOut.pointA, dOut.pointB));
            out->separation[0] = dOut.distance;
            out->localId[0] = 0;
        }
        return;
    }
    out->dist2 = clippedSep > 0.0f ? clippedSep * clippedSep : 0.0f;
}

// ---------------------------------------------------------------------
// The window and the welded pipeline (manifold.c:1513-1906, 1924-2071).
// ---------------------------------------------------------------------

// The pair, localised into the heightfield's frame, and its window.
struct m3TerrainCtx
{
    const float* heights;
    int32_t nx;
    m3real cell;
    int32_t cx0;
    int32_t cz0;
    int32_t wx; // window corners per axis
    int32_t wz;
    uint8_t otherType;
    m3real radius;
    m3Vec3 s1;
    m3Vec3 s2;
    const m3HullData* hull;
    m3Quat qRel; // other shape -> heightfield frame
    m3Vec3 pRel;
    m3Quat qHull; // heightfield frame -> hull frame
    m3Vec3 pHull;
};

// Window vertex v (row-major, x fastest) in the heightfield's frame.
__device__ __forceinline__ m3Vec3 m3HfVertex(const m3TerrainCtx& c, int32_t v)
{
    const int32_t gx = c.cx0 + v % c.wx;
    const int32_t gz = c.cz0 + v / c.wx;
    return v3((m3real)gx * c.cell, c.heights[gz * c.nx + gx], (m3real)gz * c.cell);
}

// Window triangle t's vertex indices: two per cell in row-major cell
// order, the diagonal alternating with the grid cell's parity.
__device__ __forceinline__ void m3HfTriangle(const m3TerrainCtx& c, int32_t t, int32_t idx[3])
{
    const int32_t cellIndex = t >> 1;
    const int32_t x = cellIndex % (c.wx - 1);
    const int32_t z = cellIndex / (c.wx - 1);
    const int32_t a = z * c.wx + x;
    const int32_t b = a + 1;
    const int32_t cc = (z + 1) * c.wx + x + 1;
    const int32_t d = (z + 1) * c.wx + x;
    const bool even = ((c.cx0 + x) + (c.cz0 + z)) % 2 == 0;
    const bool second = (t & 1) != 0;
    if (even)
    {
        idx[0] = a;
        idx[1] = second ? d : cc;
        idx[2] = second ? cc : b;
    }
    else
    {
        idx[0] = b;
        idx[1] = second ? d : a;
        idx[2] = second ? cc : d;
    }
}

// The vertex opposite edge (v1, v2) in the other triangle holding that
// edge, or -1 on the window's boundary.
__device__ int32_t m3HfOpposite(const m3TerrainCtx& c, int32_t t, int32_t v1, int32_t v2)
{
    const int32_t x1 = v1 % c.wx;
    const int32_t z1 = v1 / c.wx;
    const int32_t x2 = v2 % c.wx;
    const int32_t z2 = v2 / c.wx;
    const int32_t xm = x1 < x2 ? x1 : x2;
    const int32_t zm = z1 < z2 ? z1 : z2;
    int32_t cellX[2];
    int32_t cellZ[2];
    int32_t cells = 0;
    if (z1 == z2)
    {
        cellX[0] = xm;
        cellZ[0] = zm - 1;
        cellX[1] = xm;
        cellZ[1] = zm;
        cells = 2;
    }
    else if (x1 == x2)
    {
        cellX[0] = xm - 1;
        cellZ[0] = zm;
        cellX[1] = xm;
        cellZ[1] = zm;
        cells = 2;
    }
    else
    {
        cellX[0] = xm;
        cellZ[0] = zm;
        cells = 1;
    }
    for (int32_t k = 0; k < cells; ++k)
    {
        if (cellX[k] < 0 || cellX[k] > c.wx - 2 || cellZ[k] < 0 || cellZ[k] > c.wz - 2)
        {
            continue;
        }
        for (int32_t h = 0; h < 2; ++h)
        {
            const int32_t u = 2 * (cellZ[k] * (c.wx - 1) + cellX[k]) + h;
            if (u == t)
            {
                continue;
            }
            int32_t idx[3];
            m3HfTriangle(c, u, idx);
            for (int32_t j = 0; j < 3; ++j)
            {
                const int32_t w1 = idx[j];
                const int32_t w2 = idx[(j + 1) % 3];
                if ((w1 == v2 && w2 == v1) || (w1 == v1 && w2 == v2))
                {
                    return idx[(j + 2) % 3];
                }
            }
        }
    }
    return -1;
}

// shape.c:304-348 for one window triangle: bit k marks edge k (vertex k
// to k + 1) as a real feature, a boundary or a convex ridge.
__device__ uint8_t m3HfEdgeFlags(const m3TerrainCtx& c, int32_t t)
{
    int32_t idx[3];
    m3HfTriangle(c, t, idx);
    const m3Vec3 a = m3HfVertex(c, idx[0]);
    const m3Vec3 b = m3HfVertex(c, idx[1]);
    const m3Vec3 cc = m3HfVertex(c, idx[2]);
    const m3Vec3 n = m3Normalize3(m3Cross3(m3Sub3(b, a), m3Sub3(cc, a)));
    const m3real off = m3Dot3(n, a);
    uint8_t flags = 0;
    for (int32_t k = 0; k < 3; ++k)
    {
        const int32_t opp = m3HfOpposite(c, t, idx[k], idx[(k + 1) % 3]);
        if (opp < 0)
        {
            flags |= (uint8_t)(1 << k);
            continue;
        }
        const m3real d = m3Dot3(n, m3HfVertex(c, opp)) - off;
        if (d < -0.005f)
        {
            flags |= (uint8_t)(1 << k);
        }
    }
    return flags;
}

// Window triangle t's contact with the convex (manifold.c:1640-1672),
// in the heightfield's frame.
__device__ void m3HfCollideTriangle(const m3TerrainCtx& c, const m3Vec3 tri[3],
                                    m3TriManifoldDev* local)
{
    memset(local, 0, sizeof(*local));
    if (c.otherType == M3_SHAPE_SPHERE)
    {
        m3SphereTriangleDev(local, c.s1, c.radius, tri);
        return;
    }
    if (c.otherType == M3_SHAPE_CAPSULE)
    {
        m3CapsuleTriangleDev(local, c.s1, c.s2, c.radius, tri);
        return;
    }
    m3Vec3 triH[3];
    for (int32_t k = 0; k < 3; ++k)
    {
        triH[k] = m3Add3(m3RotateVec3(c.qHull, tri[k]), c.pHull);
    }
    m3HullTriangleDev(local, c.hull, triH);
    if (local->pointCount > 0)
    {
        local->normal = m3RotateVec3(c.qRel, local->normal);
        local->triNormal = m3RotateVec3(c.qRel, local->triNormal);
        for (int32_t k = 0; k < local->pointCount; ++k)
        {
            local->point[k] = m3Add3(m3RotateVec3(c.qRel, local->point[k]), c.pRel);
        }
    }
}

__device__ __forceinline__ void m3HfTriangleVerts(const m3TerrainCtx& c, int32_t t, m3Vec3 tri[3])
{
    int32_t idx[3];
    m3HfTriangle(c, t, idx);
    tri[0] = m3HfVertex(c, idx[0]);
    tri[1] = m3HfVertex(c, idx[1]);
    tri[2] = m3HfVertex(c, idx[2]);
}

// A candidate triangle: what the acceptance and the clustering read.
struct m3HfCandidate
{
    m3real dist2;
    m3real minSep;
    uint16_t tri;
    uint8_t feature;
    uint8_t pad;
};

// Claimed window edges and vertices (manifold.c:1458-1510).
struct m3HfClaims
{
    uint32_t verts[(M3_HF_MAX_VERTS + 31) / 32];
    uint32_t edges[(4 * M3_HF_MAX_VERTS + 31) / 32];
};

__device__ __forceinline__ bool m3HfClaimBit(uint32_t* bits, int32_t i)
{
    const uint32_t m = 1u << (i & 31);
    const bool fresh = (bits[i >> 5] & m) == 0;
    bits[i >> 5] |= m;
    return fresh;
}

// An undirected window edge as lower vertex x 4 + the step to the upper
// one (along x, along z, or one of the two diagonals).
__device__ __forceinline__ bool m3HfClaimEdge(m3HfClaims* set, int32_t wx, int32_t v1, int32_t v2)
{
    const int32_t lo = v1 < v2 ? v1 : v2;
    const int32_t hi = v1 < v2 ? v2 : v1;
    const int32_t step = hi - lo;
    const int32_t code = step == 1 ? 0 : step == wx ? 1 : step == wx + 1 ? 2 : 3;
    return m3HfClaimBit(set->edges, 4 * lo + code);
}

// Heightfield versus sphere, capsule or hull (manifold.c:1924-2071 and
// the core it feeds, :1513-1906).  `fresh` arrives empty.
__device__ __noinline__ void m3CollideTerrainDev(const m3WorldView& w, int32_t hfShape,
                                                 int32_t otherShape, bool hfIsA,
                                                 m3Manifold* fresh)
{
    const m3HeightFieldDev hf = w.hfs[w.hfIndex[hfShape]];
    const m3Transform xfH = m3ShapeXf(w, hfShape);
    const m3Transform xfO = m3ShapeXf(w, otherShape);
    m3TerrainCtx c;
    c.heights = w.hfSamples + hf.sampleStart;
    c.nx = hf.nx;
    c.cell = hf.cellSize;
    const m3Quat conjH = q4(-xfH.q.x, -xfH.q.y, -xfH.q.z, xfH.q.w);
    c.qRel = m3MulQuat(conjH, xfO.q);
    const m3Vec3 dp = v3((m3real)(xfO.p.x - xfH.p.x), (m3real)(xfO.p.y - xfH.p.y),
                         (m3real)(xfO.p.z - xfH.p.z));
    c.pRel = m3InvRotateVec3(xfH.q, dp);
    c.otherType = w.shapeType[otherShape];
    c.radius = w.geom[otherShape].s;
    c.s1 = v3(0.0f, 0.0f, 0.0f);
    c.s2 = v3(0.0f, 0.0f, 0.0f);
    c.hull = nullptr;
    c.qHull = q4(0.0f, 0.0f, 0.0f, 1.0f);
    c.pHull = v3(0.0f, 0.0f, 0.0f);

    // The convex's bounds in the heightfield's frame.
    m3Vec3 boundLo;
    m3Vec3 boundHi;
    if (c.otherType == M3_SHAPE_HULL)
    {
        c.hull = &w.hulls[w.hullIndex[otherShape]];
        c.qHull = q4(-c.qRel.x, -c.qRel.y, -c.qRel.z, c.qRel.w);
        c.pHull = m3Neg3(m3InvRotateVec3(c.qRel, c.pRel));
        boundLo = v3(3.4e38f, 3.4e38f, 3.4e38f);
        boundHi = v3(-3.4e38f, -3.4e38f, -3.4e38f);
        for (int32_t v = 0; v < c.hull->vertexCount; ++v)
        {
            const m3Vec3 p = m3Add3(m3RotateVec3(c.qRel, c.hull->vertices[v]), c.pRel);
            boundLo.x = m3MinF(boundLo.x, p.x);
            boundLo.y = m3MinF(boundLo.y, p.y);
            boundLo.z = m3MinF(boundLo.z, p.z);
            boundHi.x = m3MaxF(boundHi.x, p.x);
            boundHi.y = m3MaxF(boundHi.y, p.y);
            boundHi.z = m3MaxF(boundHi.z, p.z);
        }
        c.radius = 0.0f;
    }
    else if (c.otherType == M3_SHAPE_SPHERE)
    {
        c.s1 = m3Add3(m3RotateVec3(c.qRel, w.geom[otherShape].v), c.pRel);
        boundLo = c.s1;
        boundHi = c.s1;
    }
    else
    {
        c.s1 = m3Add3(m3RotateVec3(c.qRel, w.geom[otherShape].v), c.pRel);
        c.s2 = m3Add3(m3RotateVec3(c.qRel, w.geom[otherShape].v2), c.pRel);
        boundLo = v3(m3MinF(c.s1.x, c.s2.x), m3MinF(c.s1.y, c.s2.y), m3MinF(c.s1.z, c.s2.z));
        boundHi = v3(m3MaxF(c.s1.x, c.s2.x), m3MaxF(c.s1.y, c.s2.y), m3MaxF(c.s1.z, c.s2.z));
    }
    const m3real reach = c.radius + M3_SPECULATIVE_DISTANCE;

    // The cell window: the reach plus a halo cell, clipped to the grid
    // and to the window bound (world_internal.h:30-35 for the cell
    // conversion).
    const m3real inv = 1.0f / hf.cellSize;
    int32_t cx0 = m3CellFromF(floorf((boundLo.x - reach) * inv), 2.0e9f) - 1;
    int32_t cx1 = m3CellFromF(floorf((boundHi.x + reach) * inv), -2.0e9f) + 1;
    int32_t cz0 = m3CellFromF(floorf((boundLo.z - reach) * inv), 2.0e9f) - 1;
    int32_t cz1 = m3CellFromF(floorf((boundHi.z + reach) * inv), -2.0e9f) + 1;
    cx0 = cx0 < 0 ? 0 : cx0;
    cz0 = cz0 < 0 ? 0 : cz0;
    cx1 = cx1 > hf.nx - 2 ? hf.nx - 2 : cx1;
    cz1 = cz1 > hf.nz - 2 ? hf.nz - 2 : cz1;
    if (cx1 < cx0 || cz1 < cz0)
    {
        return; // off the grid
    }
    if (cx1 - cx0 + 1 > M3_HF_WINDOW)
    {
        cx1 = cx0 + M3_HF_WINDOW - 1;
    }
    if (cz1 - cz0 + 1 > M3_HF_WINDOW)
    {
        cz1 = cz0 + M3_HF_WINDOW - 1;
    }
    c.cx0 = cx0;
    c.cz0 = cz0;
    c.wx = cx1 - cx0 + 2;
    c.wz = cz1 - cz0 + 2;
    const int32_t triCount = 2 * (c.wx - 1) * (c.wz - 1);

    // Every window triangle in ascending order: face contacts accepted
    // at once, the rest tentative (manifold.c:1604-1703).
    m3HfCandidate faceAccepted[M3_MESH_CANDIDATE_CAP];
    int32_t faceCount = 0;
    m3HfCandidate tentative[M3_MESH_CANDIDATE_CAP];
    int32_t tentativeCount = 0;
    m3TriManifoldDev local;
    for (int32_t t = 0; t < triCount; ++t)
    {
        if (faceCount >= M3_MESH_CANDIDATE_CAP || tentativeCount >= M3_MESH_CANDIDATE_CAP)
        {
            break;
        }
        m3Vec3 tri[3];
        m3HfTriangleVerts(c, t, tri);
        const m3real lox = m3MinF(tri[0].x, m3MinF(tri[1].x, tri[2].x)) - reach;
        const m3real hix = m3MaxF(tri[0].x, m3MaxF(tri[1].x, tri[2].x)) + reach;
        const m3real loy = m3MinF(tri[0].y, m3MinF(tri[1].y, tri[2].y)) - reach;
        const m3real hiy = m3MaxF(tri[0].y, m3MaxF(tri[1].y, tri[2].y)) + reach;
        const m3real loz = m3MinF(tri[0].z, m3MinF(tri[1].z, tri[2].z)) - reach;
        const m3real hiz = m3MaxF(tri[0].z, m3MaxF(tri[1].z, tri[2].z)) + reach;
        if (boundHi.x < lox || boundLo.x > hix || boundHi.y < loy || boundLo.y > hiy ||
            boundHi.z < loz || boundLo.z > hiz)
        {
            continue;
        }
        m3HfCollideTriangle(c, tri, &local);
        if (local.pointCount == 0)
        {
            continue;
        }
        m3HfCandidate cand;
        cand.dist2 = local.dist2;
        cand.minSep = 3.4e38f;
        for (int32_t k = 0; k < local.pointCount; ++k)
        {
            cand.minSep = m3MinF(cand.minSep, local.separation[k]);
        }
        cand.tri = (uint16_t)t;
        cand.feature = (uint8_t)local.feature;
        cand.pad = 0;
        if (local.feature == 7)
        {
            faceAccepted[faceCount++] = cand;
        }
        else if (local.feature == M3_TRI_FEATURE_HULL_FACE)
        {
            const m3real cosAngle = m3Dot3(local.triNormal, local.normal);
            if (cosAngle > 0.5f || cand.minSep < -2.0f * 0.005f)
            {
                faceAccepted[faceCount++] = cand;
            }
            else
            {
                tentative[tentativeCount++] = cand;
            }
        }
        else
        {
            tentative[tentativeCount++] = cand;
        }
    }

    // Face contacts claim their features first, in triangle order.
    m3HfClaims set;
    memset(&set, 0, sizeof(set));
    for (int32_t k = 0; k < faceCount; ++k)
    {
        int32_t idx[3];
        m3HfTriangle(c, faceAccepted[k].tri, idx);
        (void)m3HfClaimEdge(&set, c.wx, idx[0], idx[1]);
        (void)m3HfClaimEdge(&set, c.wx, idx[1], idx[2]);
        (void)m3HfClaimEdge(&set, c.wx, idx[2], idx[0]);
        (void)m3HfClaimBit(set.verts, idx[0]);
        (void)m3HfClaimBit(set.verts, idx[1]);
        (void)m3HfClaimBit(set.verts, idx[2]);
    }

    // Tentatives by ascending distance, ties to the lower triangle (the
    // reference's selection sort, step for step).
    for (int32_t a = 0; a < tentativeCount; ++a)
    {
        int32_t best = a;
        for (int32_t b = a + 1; b < tentativeCount; ++b)
        {
            if (tentative[b].dist2 < tentative[best].dist2 ||
                (tentative[b].dist2 == tentative[best].dist2 &&
                 tentative[b].tri < tentative[best].tri))
            {
                best = b;
            }
        }
        const m3HfCandidate tmp = tentative[a];
        tentative[a] = tentative[best];
        tentative[best] = tmp;
    }

    // A tentative survives on an unclaimed feature, or on a real edge.
    for (int32_t k = 0; k < tentativeCount && faceCount < M3_MESH_CANDIDATE_CAP; ++k)
    {
        const int32_t t = tentative[k].tri;
        int32_t idx[3];
        m3HfTriangle(c, t, idx);
        const bool newEdge1 = m3HfClaimEdge(&set, c.wx, idx[0], idx[1]);
        const bool newEdge2 = m3HfClaimEdge(&set, c.wx, idx[1], idx[2]);
        const bool newEdge3 = m3HfClaimEdge(&set, c.wx, idx[2], idx[0]);
        const bool newVert1 = m3HfClaimBit(set.verts, idx[0]);
        const bool newVert2 = m3HfClaimBit(set.verts, idx[1]);
        const bool newVert3 = m3HfClaimBit(set.verts, idx[2]);
        const uint8_t convex = m3HfEdgeFlags(c, t);
        bool shouldCollide = false;
        switch (tentative[k].feature)
        {
        case 1 | 2:
            shouldCollide = (convex & 1) != 0 || newEdge1;
            break;
        case 2 | 4:
            shouldCollide = (convex & 2) != 0 || newEdge2;
            break;
        case 1 | 4:
            shouldCollide = (convex & 4) != 0 || newEdge3;
            break;
        case 1:
            shouldCollide = newVert1;
            break;
        case 2:
            shouldCollide = newVert2;
            break;
        case 4:
            shouldCollide = newVert3;
            break;
        case M3_TRI_FEATURE_HULL_FACE:
            shouldCollide = convex != 0 ||
                            (newEdge1 && newEdge2 && newEdge3 && newVert1 && newVert2 && newVert3);
            break;
        default:
            break;
        }
        if (shouldCollide)
        {
            faceAccepted[faceCount++] = tentative[k];
        }
    }
    if (faceCount == 0)
    {
        return;
    }

    // The deepest accepted contact (ties to the lower triangle) sets the
    // cluster's normal (manifold.c:1803-1818).
    int32_t repIndex = 0;
    m3real repSep = 3.4e38f;
    for (int32_t k = 0; k < faceCount; ++k)
    {
        const m3real sep = faceAccepted[k].minSep;
        if (sep < repSep ||
            (sep == repSep && faceAccepted[k].tri < faceAccepted[repIndex].tri))
        {
            repSep = sep;
            repIndex = k;
        }
    }
    m3Vec3 tri[3];
    m3HfTriangleVerts(c, faceAccepted[repIndex].tri, tri);
    m3HfCollideTriangle(c, tri, &local);
    const m3Vec3 repNormal = local.normal;

    // The cluster's points stream through; the deepest four by
    // (separation, id) stay, sorted by (separation, id).
    m3Vec3 keptPoint[4];
    m3real keptSep[4];
    uint16_t keptId[4];
    int32_t keptCount = 0;
    int32_t gCount = 0;
    for (int32_t k = 0; k < faceCount && gCount < 2 * M3_MESH_CANDIDATE_CAP; ++k)
    {
        m3HfTriangleVerts(c, faceAccepted[k].tri, tri);
        m3HfCollideTriangle(c, tri, &local);
        if (m3Dot3(local.normal, repNormal) < 0.99f)
        {
            continue;
        }
        for (int32_t p = 0; p < local.pointCount && gCount < 2 * M3_MESH_CANDIDATE_CAP; ++p)
        {
            gCount += 1;
            const m3real sep = local.separation[p];
            const uint16_t id = (uint16_t)((faceAccepted[k].tri << 2) | local.localId[p]);
            int32_t at = keptCount;
            while (at > 0 && (sep < keptSep[at - 1] || (sep == keptSep[at - 1] && id < keptId[at - 1])))
            {
                at -= 1;
            }
            if (at >= 4)
            {
                continue;
            }
            const int32_t last = keptCount < 4 ? keptCount : 3;
            for (int32_t j = last; j > at; --j)
            {
                keptPoint[j] = keptPoint[j - 1];
                keptSep[j] = keptSep[j - 1];
                keptId[j] = keptId[j - 1];
            }
            keptPoint[at] = local.point[p];
            keptSep[at] = sep;
            keptId[at] = id;
            keptCount = keptCount < 4 ? keptCount + 1 : 4;
        }
    }
    // Ascending id (the canonical point order).
    for (int32_t a = 0; a < keptCount; ++a)
    {
        for (int32_t b = a + 1; b < keptCount; ++b)
        {
            if (keptId[b] < keptId[a])
            {
                const m3Vec3 tp = keptPoint[a];
                keptPoint[a] = keptPoint[b];
                keptPoint[b] = tp;
                const m3real ts = keptSep[a];
                keptSep[a] = keptSep[b];
                keptSep[b] = ts;
                const uint16_t ti = keptId[a];
                keptId[a] = keptId[b];
                keptId[b] = ti;
            }
        }
    }

    // Emit: each point splits into both anchors along the normal.
    const int32_t meshBody = w.shapeBody[hfShape];
    const int32_t otherBody = w.shapeBody[otherShape];
    const m3Vec3 nWorld = m3RotateVec3(xfH.q, repNormal);
    fresh->normal = hfIsA ? nWorld : m3Neg3(nWorld);
    fresh->pointCount = keptCount;
    for (int32_t k = 0; k < keptCount; ++k)
    {
        const m3Vec3 pw = m3RotateVec3(xfH.q, keptPoint[k]);
        const double px = xfH.p.x + (double)pw.x;
        const double py = xfH.p.y + (double)pw.y;
        const double pz = xfH.p.z + (double)pw.z;
        const m3real half = 0.5f * keptSep[k];
        const m3Vec3 anchorMesh =
            m3FromCom(w, meshBody, px - (double)(nWorld.x * half), py - (double)(nWorld.y * half),
                      pz - (double)(nWorld.z * half));
        const m3Vec3 anchorOther =
            m3FromCom(w, otherBody, px + (double)(nWorld.x * half), py + (double)(nWorld.y * half),
                      pz + (double)(nWorld.z * half));
        fresh->points[k].anchorA = hfIsA ? anchorMesh : anchorOther;
        fresh->points[k].anchorB = hfIsA ? anchorOther : anchorMesh;
        fresh->points[k].separation = keptSep[k];
        fresh->points[k].id = keptId[k];
        fresh->points[k].flags = 0;
    }
}

#endif // M3_TERRAIN_CUH
