// Convex hulls from point clouds for m3CreateHullShape (shape.h:143-149,
// shape.c:988-1030): QuickHull as the reference builds it
// (src/quickhull.c:1-1216) -- a scaled tolerance, the four-point seed,
// per-face conflict lists with a cached farthest point, the horizon found
// by an explicit-stack walk, the cone of new triangles, then three merge
// passes (flipped, concave, coplanar) -- emitted into the fixed hull slab
// with unit-density mass properties and the half-edge table.
//
// The hull's bytes are interned and hashed world state, so every
// floating-point expression, list order and tie rule follows the
// reference (strict improvements keep the earliest candidate; lists are
// walked in construction order).  The storage is this file's own: pools
// indexed by integers, doubly linked lists over a shared node space with
// one sentinel per list, free lists as index stacks.
#include "m3_world.h"

#include <float.h>
#include <string.h>

#include <memory>

namespace
{
constexpr int32_t kNone = -1;
constexpr int32_t kMaxInput = 256; // world_internal.h:217
constexpr int32_t kVertexCap = kMaxInput + 4;
constexpr int32_t kEdgeCap = 24 * M3_HULL_MAX_VERTS - 48;
constexpr int32_t kFaceCap = 5 * M3_HULL_MAX_VERTS - 10;
constexpr int32_t kRingCap = 3 * M3_HULL_MAX_VERTS - 6;
constexpr int32_t kMergeCap = 2 * M3_HULL_MAX_VERTS - 4;
constexpr int32_t kVisible = 0;
constexpr int32_t kDeleted = 1;

// Vertex list nodes: vertices 0..kVertexCap-1, then the orphan list's
// sentinel, the hull vertex list's sentinel, then one conflict-list
// sentinel per face.
constexpr int32_t kOrphans = kVertexCap;
constexpr int32_t kHullVerts = kVertexCap + 1;
constexpr int32_t kConflict0 = kVertexCap + 2;
constexpr int32_t kVertexNodes = kConflict0 + kFaceCap;
// Face list nodes: faces 0..kFaceCap-1, then the hull face list's sentinel.
constexpr int32_t kHullFaces = kFaceCap;
constexpr int32_t kFaceNodes = kFaceCap + 1;

struct Edge
{
    int32_t prev; // ring around the owning face
    int32_t next;
    int32_t origin;
    int32_t face;
    int32_t twin;
};

struct Face
{
    int32_t edge;
    int32_t mark;
    m3real area;
    m3Vec3 normal; // unit plane normal: dot(normal, x) = offset on the face
    m3real offset;
    m3Vec3 centroid;
    m3real maxConflictDistance;
    int32_t maxConflict;
    int32_t flipped;
};

struct Frame
{
    int32_t face;
    int32_t startEdge;
    int32_t edge;
    int32_t started;
};

struct Links
{
    int32_t prev;
    int32_t next;
};

class Builder
{
public:
    bool Build(const m3Vec3* points, int32_t count, m3HullData* out);

private:
    // Lists ------------------------------------------------------------
    void InitList(Links* links, int32_t head) { links[head] = Links{head, head}; }
    static bool InList(const Links* links, int32_t node) { return links[node].prev != kNone; }
    void Remove(Links* links, int32_t node)
    {
        links[links[node].prev].next = links[node].next;
        links[links[node].next].prev = links[node].prev;
        links[node] = Links{kNone, kNone};
    }
    void PushBack(Links* links, int32_t head, int32_t node)
    {
        links[node].prev = links[head].prev;
        links[node].next = head;
        links[links[head].prev].next = node;
        links[head].prev = node;
    }

    // Pools ------------------------------------------------------------
    int32_t NewVertex(m3Vec3 position);
    int32_t NewEdge();
    void RetireEdge(int32_t e) { edgeFree_[edgeFreeCount_++] = e; }
    int32_t NewFace(int32_t va, int32_t vb, int32_t vc);
    void RetireFace(int32_t f);

    m3real Separation(int32_t f, m3Vec3 p) const
    {
        return m3Dot3(face_[f].normal, p) - face_[f].offset;
    }
    bool EdgeConvex(int32_t e, m3real tol) const
    {
        return Separation(edge_[e].face, face_[edge_[edge_[e].twin].face].centroid) < -tol;
    }
    bool EdgeConcave(int32_t e, m3real tol) const
    {
        return Separation(edge_[e].face, face_[edge_[edge_[e].twin].face].centroid) > tol;
    }
    int32_t FaceVertexCount(int32_t f) const;
    int32_t EdgeAt(int32_t f, int32_t index) const;
    void Twin(int32_t a, int32_t b)
    {
        edge_[a].twin = b;
        edge_[b].twin = a;
    }
    void NewellPlane(int32_t f);
    void Recache(int32_t f);
    void DrainConflicts(int32_t f);

    // Stages -----------------------------------------------------------
    void Tolerance(int32_t count, const m3Vec3* p);
    bool Seed(int32_t count, const m3Vec3* p);
    int32_t NextConflict() const;
    void EnterHorizonFace(int32_t f, int32_t entry, Frame* frame);
    bool Horizon(int32_t apex, int32_t seed);
    bool Cone(int32_t apex);
    void DestroyEdges(int32_t begin, int32_t end);
    void ConnectEdges(int32_t prev, int32_t next);
    void Absorb(int32_t f);
    void ConnectFaces(int32_t e);
    bool MergeConcave(int32_t f);
    bool MergeCoplanar(int32_t f);
    void MergeFaces();
    void ResolveVertices();
    void ResolveFaces();
    bool AddVertex(int32_t v);
    void Clean();

    m3real tolerance_ = 0.0f;
    m3real minRadius_ = 0.0f;
    m3real minOutside_ = 0.0f;
    m3Vec3 interior_ = {0.0f, 0.0f, 0.0f};
    bool overflow_ = false;

    m3Vec3 position_[kVertexCap];
    int32_t conflictFace_[kVertexCap];
    int32_t finalIndex_[kVertexCap];
    int32_t reachable_[kVertexCap];
    int32_t vertexCount_ = 0;
    Links vlink_[kVertexNodes];

    Edge edge_[kEdgeCap];
    int32_t edgeCount_ = 0;
    int32_t edgeFree_[kEdgeCap];
    int32_t edgeFreeCount_ = 0;

    Face face_[kFaceCap];
    int32_t faceCount_ = 0;
    int32_t faceFree_[kFaceCap];
    int32_t faceFreeCount_ = 0;
    Links flink_[kFaceNodes];

    int32_t horizon_[kRingCap];
    int32_t horizonCount_ = 0;
    int32_t cone_[kRingCap];
    int32_t coneCount_ = 0;
    int32_t merged_[kMergeCap];
    int32_t mergedCount_ = 0;
    Frame stack_[kMergeCap];

    int32_t finalVertices_ = 0;
    int32_t finalHalfEdges_ = 0;
    int32_t finalFaces_ = 0;
    m3Vec3 shifted_[kMaxInput];
};

int32_t Builder::NewVertex(m3Vec3 position)
{
    if (vertexCount_ >= kVertexCap)
    {
        overflow_ = true;
        return kNone;
    }
    const int32_t v = vertexCount_++;
    vlink_[v] = Links{kNone, kNone};
    conflictFace_[v] = kNone;
    position_[v] = position;
    finalIndex_[v] = kNone;
    reachable_[v] = 0;
    return v;
}

int32_t Builder::NewEdge()
{
    if (edgeFreeCount_ > 0)
    {
        return edgeFree_[--edgeFreeCount_];
    }
    if (edgeCount_ >= kEdgeCap)
    {
        overflow_ = true;
        return kNone;
    }
    return edgeCount_++;
}

// quickhull.c:189-243: a triangle (va, vb, vc) with its plane, area and
// centroid; flipped when the interior point lies in front of it.
int32_t Builder::NewFace(int32_t va, int32_t vb, int32_t vc)
{
    int32_t f;
    if (faceFreeCount_ > 0)
    {
        f = faceFree_[--faceFreeCount_];
    }
    else if (faceCount_ < kFaceCap)
    {
        f = faceCount_++;
    }
    else
    {
        overflow_ = true;
        return kNone;
    }
    flink_[f] = Links{kNone, kNone};
    Face& face = face_[f];
    face.maxConflict = kNone;
    face.maxConflictDistance = 0.0f;
    const int32_t e1 = NewEdge();
    const int32_t e2 = NewEdge();
    const int32_t e3 = NewEdge();
    if (e1 == kNone || e2 == kNone || e3 == kNone)
    {
        return kNone;
    }
    const m3Vec3 p1 = position_[va];
    const m3Vec3 p2 = position_[vb];
    const m3Vec3 p3 = position_[vc];
    m3Vec3 normal = m3Cross3(m3Sub3(p2, p1), m3Sub3(p3, p1));
    const m3real length = sqrtf(m3Dot3(normal, normal));
    normal = length > 0.0f ? m3MulSV3(1.0f / length, normal) : v3(0.0f, 1.0f, 0.0f);
    face.edge = e1;
    face.mark = kVisible;
    face.area = 0.5f * length;
    face.centroid = m3MulSV3(1.0f / 3.0f, m3Add3(p1, m3Add3(p2, p3)));
    face.normal = normal;
    face.offset = m3Dot3(normal, p1);
    face.flipped = Separation(f, interior_) > 0.0f ? 1 : 0;
    InitList(vlink_, kConflict0 + f);
    edge_[e1] = Edge{e3, e2, va, f, kNone};
    edge_[e2] = Edge{e1, e3, vb, f, kNone};
    edge_[e3] = Edge{e2, e1, vc, f, kNone};
    return f;
}

void Builder::RetireFace(int32_t f)
{
    if (InList(flink_, f))
    {
        Remove(flink_, f);
    }
    face_[f].edge = kNone;
    faceFree_[faceFreeCount_++] = f;
}

int32_t Builder::FaceVertexCount(int32_t f) const
{
    int32_t count = 0;
    int32_t e = face_[f].edge;
    do
    {
        count++;
        e = edge_[e].next;
    } while (e != face_[f].edge);
    return count;
}

int32_t Builder::EdgeAt(int32_t f, int32_t index) const
{
    int32_t e = face_[f].edge;
    while (index-- > 0)
    {
        e = edge_[e].next;
    }
    return e;
}

// quickhull.c:307-333: Newell normal and centroid of an n-gon, the first
// vertex as local origin.
void Builder::NewellPlane(int32_t f)
{
    int32_t count = 0;
    m3Vec3 centroid = v3(0.0f, 0.0f, 0.0f);
    m3Vec3 normal = v3(0.0f, 0.0f, 0.0f);
    int32_t e = face_[f].edge;
    const m3Vec3 origin = position_[edge_[e].origin];
    do
    {
        const m3Vec3 a = m3Sub3(position_[edge_[e].origin], origin);
        const m3Vec3 b = m3Sub3(position_[edge_[edge_[e].twin].origin], origin);
        count++;
        centroid = m3Add3(centroid, a);
        normal.x += (a.y - b.y) * (a.z + b.z);
        normal.y += (a.z - b.z) * (a.x + b.x);
        normal.z += (a.x - b.x) * (a.y + b.y);
        e = edge_[e].next;
    } while (e != face_[f].edge);
    centroid = m3Add3(m3MulSV3(1.0f / (m3real)count, centroid), origin);
    const m3real length = sqrtf(m3Dot3(normal, normal));
    normal = length > 0.0f ? m3MulSV3(1.0f / length, normal) : v3(0.0f, 1.0f, 0.0f);
    face_[f].centroid = centroid;
    face_[f].normal = normal;
    face_[f].offset = m3Dot3(normal, centroid);
    face_[f].area = 0.5f * length;
}

// quickhull.c:578-595: the face's farthest conflict after its plane moved.
void Builder::Recache(int32_t f)
{
    int32_t best = kNone;
    m3real bestDistance = minOutside_;
    const int32_t head = kConflict0 + f;
    for (int32_t n = vlink_[head].next; n != head; n = vlink_[n].next)
    {
        const m3real d = Separation(f, position_[n]);
        if (d > bestDistance)
        {
            bestDistance = d;
            best = n;
        }
    }
    face_[f].maxConflict = best;
    face_[f].maxConflictDistance = bestDistance;
}

void Builder::DrainConflicts(int32_t f)
{
    const int32_t head = kConflict0 + f;
    int32_t n = vlink_[head].next;
    while (n != head)
    {
        const int32_t orphan = n;
        n = vlink_[n].next;
        conflictFace_[orphan] = kNone;
        Remove(vlink_, orphan);
        PushBack(vlink_, kOrphans, orphan);
    }
}

// quickhull.c:335-360: tolerance scaled by the cloud's extent.
void Builder::Tolerance(int32_t count, const m3Vec3* p)
{
    m3Vec3 lo = p[0];
    m3Vec3 hi = p[0];
    for (int32_t i = 1; i < count; ++i)
    {
        lo.x = m3MinF(lo.x, p[i].x);
        lo.y = m3MinF(lo.y, p[i].y);
        lo.z = m3MinF(lo.z, p[i].z);
        hi.x = m3MaxF(hi.x, p[i].x);
        hi.y = m3MaxF(hi.y, p[i].y);
        hi.z = m3MaxF(hi.z, p[i].z);
    }
    m3Vec3 maxAbs;
    maxAbs.x = m3MaxF(lo.x < 0.0f ? -lo.x : lo.x, hi.x < 0.0f ? -hi.x : hi.x);
    maxAbs.y = m3MaxF(lo.y < 0.0f ? -lo.y : lo.y, hi.y < 0.0f ? -hi.y : hi.y);
    maxAbs.z = m3MaxF(lo.z < 0.0f ? -lo.z : lo.z, hi.z < 0.0f ? -hi.z : hi.z);
    const m3real maxSum = maxAbs.x + maxAbs.y + maxAbs.z;
    const m3real maxCoord = m3MaxF(maxAbs.x, m3MaxF(maxAbs.y, maxAbs.z));
    const m3real maxDistance = m3MinF(1.7320508f * maxCoord, maxSum);
    tolerance_ = (3.0f * maxDistance * 1.01f + maxCoord) * FLT_EPSILON;
    minRadius_ = 4.0f * tolerance_;
    minOutside_ = 2.0f * minRadius_;
}

// quickhull.c:362-576: the extreme pair along the widest axis, the point
// farthest from their line, the point farthest from that plane; the
// tetrahedron (wound outward) and every other point to the face it is
// farthest in front of.
bool Builder::Seed(int32_t count, const m3Vec3* p)
{
    // Widest axis.
    m3Vec3 minPt[3] = {p[0], p[0], p[0]};
    m3Vec3 maxPt[3] = {p[0], p[0], p[0]};
    int32_t minIndex[3] = {0, 0, 0};
    int32_t maxIndex[3] = {0, 0, 0};
    for (int32_t i = 1; i < count; ++i)
    {
        const m3Vec3 v = p[i];
        if (v.x < minPt[0].x)
        {
            minPt[0] = v;
            minIndex[0] = i;
        }
        else if (v.x > maxPt[0].x)
        {
            maxPt[0] = v;
            maxIndex[0] = i;
        }
        if (v.y < minPt[1].y)
        {
            minPt[1] = v;
            minIndex[1] = i;
        }
        else if (v.y > maxPt[1].y)
        {
            maxPt[1] = v;
            maxIndex[1] = i;
        }
        if (v.z < minPt[2].z)
        {
            minPt[2] = v;
            minIndex[2] = i;
        }
        else if (v.z > maxPt[2].z)
        {
            maxPt[2] = v;
            maxIndex[2] = i;
        }
    }
    const m3real span[3] = {maxPt[0].x - minPt[0].x, maxPt[1].y - minPt[1].y,
                            maxPt[2].z - minPt[2].z};
    int32_t axis = 0;
    if (span[1] > span[axis])
    {
        axis = 1;
    }
    if (span[2] > span[axis])
    {
        axis = 2;
    }
    if (!(span[axis] > 2.0f * tolerance_))
    {
        return false;
    }
    const int32_t i1 = minIndex[axis];
    int32_t i2 = maxIndex[axis];
    // Farthest from the line (i1, i2).
    int32_t i3 = kNone;
    {
        const m3Vec3 a = p[i1];
        const m3Vec3 ab = m3Sub3(p[i2], a);
        const m3real abLen2 = m3Dot3(ab, ab);
        if (!(abLen2 > 0.0f))
        {
            return false;
        }
        const m3real invAbLen2 = 1.0f / abLen2;
        m3real best = 4.0f * tolerance_ * tolerance_;
        for (int32_t i = 0; i < count; ++i)
        {
            if (i == i1 || i == i2)
            {
                continue;
            }
            const m3Vec3 c = m3Cross3(m3Sub3(p[i], a), ab);
            const m3real d2 = m3Dot3(c, c) * invAbLen2;
            if (d2 > best)
            {
                best = d2;
                i3 = i;
            }
        }
        if (i3 == kNone)
        {
            return false;
        }
    }
    // Farthest from the plane (i1, i2, i3).
    int32_t i4 = kNone;
    {
        const m3Vec3 a = p[i1];
        m3Vec3 n = m3Cross3(m3Sub3(p[i2], a), m3Sub3(p[i3], a));
        const m3real len = sqrtf(m3Dot3(n, n));
        if (!(len > 0.0f))
        {
            return false;
        }
        n = m3MulSV3(1.0f / len, n);
        const m3real off = m3Dot3(n, a);
        m3real best = 2.0f * tolerance_;
        for (int32_t i = 0; i < count; ++i)
        {
            if (i == i1 || i == i2 || i == i3)
            {
                continue;
            }
            m3real d = m3Dot3(n, p[i]) - off;
            d = d < 0.0f ? -d : d;
            if (d > best)
            {
                best = d;
                i4 = i;
            }
        }
        if (i4 == kNone)
        {
            return false;
        }
    }
    const m3Vec3 w1 = m3Sub3(p[i1], p[i4]);
    const m3Vec3 w2 = m3Sub3(p[i2], p[i4]);
    const m3Vec3 w3 = m3Sub3(p[i3], p[i4]);
    if (m3Dot3(w1, m3Cross3(w2, w3)) < 0.0f)
    {
        const int32_t t = i2;
        i2 = i3;
        i3 = t;
    }
    interior_ = m3MulSV3(0.25f, m3Add3(m3Add3(p[i1], p[i2]), m3Add3(p[i3], p[i4])));
    const int32_t a = NewVertex(p[i1]);
    PushBack(vlink_, kHullVerts, a);
    const int32_t b = NewVertex(p[i2]);
    PushBack(vlink_, kHullVerts, b);
    const int32_t c = NewVertex(p[i3]);
    PushBack(vlink_, kHullVerts, c);
    const int32_t d = NewVertex(p[i4]);
    PushBack(vlink_, kHullVerts, d);
    const int32_t f1 = NewFace(a, b, c);
    PushBack(flink_, kHullFaces, f1);
    const int32_t f2 = NewFace(d, b, a);
    PushBack(flink_, kHullFaces, f2);
    const int32_t f3 = NewFace(d, c, b);
    PushBack(flink_, kHullFaces, f3);
    const int32_t f4 = NewFace(d, a, c);
    PushBack(flink_, kHullFaces, f4);
    Twin(EdgeAt(f1, 0), EdgeAt(f2, 1));
    Twin(EdgeAt(f1, 1), EdgeAt(f3, 1));
    Twin(EdgeAt(f1, 2), EdgeAt(f4, 1));
    Twin(EdgeAt(f2, 0), EdgeAt(f3, 2));
    Twin(EdgeAt(f3, 0), EdgeAt(f4, 2));
    Twin(EdgeAt(f4, 0), EdgeAt(f2, 2));
    for (int32_t index = 0; index < count; ++index)
    {
        if (index == i1 || index == i2 || index == i3 || index == i4)
        {
            continue;
        }
        const m3Vec3 point = p[index];
        m3real best = minOutside_;
        int32_t bestFace = kNone;
        for (int32_t f = flink_[kHullFaces].next; f != kHullFaces; f = flink_[f].next)
        {
            const m3real dist = Separation(f, point);
            if (dist > best)
            {
                best = dist;
                bestFace = f;
            }
        }
        if (bestFace != kNone)
        {
            const int32_t v = NewVertex(point);
            if (v == kNone)
            {
                return false;
            }
            conflictFace_[v] = bestFace;
            PushBack(vlink_, kConflict0 + bestFace, v);
            if (best > face_[bestFace].maxConflictDistance)
            {
                face_[bestFace].maxConflictDistance = best;
                face_[bestFace].maxConflict = v;
            }
        }
    }
    return !overflow_;
}

// quickhull.c:597-612: the farthest conflict over every face.
int32_t Builder::NextConflict() const
{
    int32_t best = kNone;
    m3real bestDistance = minOutside_;
    for (int32_t f = flink_[kHullFaces].next; f != kHullFaces; f = flink_[f].next)
    {
        if (face_[f].maxConflict != kNone && face_[f].maxConflictDistance > bestDistance)
        {
            bestDistance = face_[f].maxConflictDistance;
            best = face_[f].maxConflict;
        }
    }
    return best;
}

void Builder::EnterHorizonFace(int32_t f, int32_t entry, Frame* frame)
{
    face_[f].mark = kDeleted;
    DrainConflicts(f);
    frame->face = f;
    frame->started = 0;
    if (entry != kNone)
    {
        frame->startEdge = entry;
        frame->edge = edge_[entry].next;
    }
    else
    {
        frame->startEdge = face_[f].edge;
        frame->edge = face_[f].edge;
    }
}

// quickhull.c:646-678: depth-first over the faces the apex sees; the
// horizon is the ring of edges whose far face it does not see.
bool Builder::Horizon(int32_t apex, int32_t seed)
{
    int32_t top = 0;
    EnterHorizonFace(seed, kNone, &stack_[top++]);
    while (top > 0)
    {
        Frame* fr = &stack_[top - 1];
        if (fr->started && fr->edge == fr->startEdge)
        {
            top--;
            continue;
        }
        fr->started = 1;
        const int32_t e = fr->edge;
        const int32_t twin = edge_[e].twin;
        fr->edge = edge_[e].next;
        if (face_[edge_[twin].face].mark != kVisible)
        {
            continue;
        }
        const m3real dist = Separation(edge_[twin].face, position_[apex]);
        if (dist > minRadius_)
        {
            if (top >= kMergeCap)
            {
                return false;
            }
            EnterHorizonFace(edge_[twin].face, twin, &stack_[top++]);
        }
        else
        {
            if (horizonCount_ >= kRingCap)
            {
                return false;
            }
            horizon_[horizonCount_++] = e;
        }
    }
    return true;
}

// quickhull.c:680-697: a triangle from the apex over each horizon edge,
// linked to the far face and to its cone neighbours.
bool Builder::Cone(int32_t apex)
{
    for (int32_t i = 0; i < horizonCount_; ++i)
    {
        const int32_t e = horizon_[i];
        const int32_t f = NewFace(apex, edge_[e].origin, edge_[edge_[e].twin].origin);
        if (f == kNone || coneCount_ >= kRingCap)
        {
            return false;
        }
        cone_[coneCount_++] = f;
        Twin(EdgeAt(f, 1), edge_[e].twin);
    }
    int32_t f1 = cone_[coneCount_ - 1];
    for (int32_t i = 0; i < coneCount_; ++i)
    {
        const int32_t f2 = cone_[i];
        Twin(EdgeAt(f1, 2), EdgeAt(f2, 0));
        f1 = f2;
    }
    return true;
}

void Builder::DestroyEdges(int32_t begin, int32_t end)
{
    int32_t e = begin;
    while (e != end)
    {
        const int32_t next = edge_[e].next;
        RetireEdge(e);
        e = next;
    }
}

// quickhull.c:714-768: splices `prev` to `next`; when both face the same
// opposing face, the redundant edge is dissolved (and a triangle left
// with two edges on this face is absorbed).
void Builder::ConnectEdges(int32_t prev, int32_t next)
{
    Edge* E = edge_;
    if (E[E[prev].twin].face == E[E[next].twin].face)
    {
        if (face_[E[next].face].edge == next)
        {
            face_[E[next].face].edge = prev;
        }
        int32_t twin;
        if (FaceVertexCount(E[E[prev].twin].face) == 3)
        {
            const int32_t dead0 = E[prev].twin;
            const int32_t dead1 = E[next].twin;
            const int32_t dead2 = E[E[next].twin].prev;
            twin = E[dead2].twin;
            const int32_t opposing = E[E[prev].twin].face;
            face_[opposing].mark = kDeleted;
            if (mergedCount_ >= kMergeCap)
            {
                overflow_ = true;
                return;
            }
            merged_[mergedCount_++] = opposing;
            E[prev].next = E[next].next;
            E[E[prev].next].prev = prev;
            E[prev].twin = twin;
            E[twin].twin = prev;
            Remove(vlink_, E[next].origin);
            RetireEdge(dead0);
            RetireEdge(dead1);
            RetireEdge(dead2);
        }
        else
        {
            twin = E[next].twin;
            if (face_[E[twin].face].edge == E[prev].twin)
            {
                face_[E[twin].face].edge = twin;
            }
            E[twin].next = E[E[prev].twin].next;
            E[E[twin].next].prev = twin;
            RetireEdge(E[prev].twin);
            E[prev].next = E[next].next;
            E[E[prev].next].prev = prev;
            E[prev].twin = twin;
            E[twin].twin = prev;
            Remove(vlink_, E[next].origin);
        }
        NewellPlane(E[twin].face);
        Recache(E[twin].face);
    }
    else
    {
        E[prev].next = next;
        E[next].prev = prev;
    }
}

// quickhull.c:770-803: the merged faces' conflicts move to `f` (or are
// orphaned) and the merged faces are retired.
void Builder::Absorb(int32_t f)
{
    for (int32_t i = 0; i < mergedCount_; ++i)
    {
        const int32_t head = kConflict0 + merged_[i];
        int32_t n = vlink_[head].next;
        while (n != head)
        {
            const int32_t v = n;
            n = vlink_[n].next;
            Remove(vlink_, v);
            const m3real dist = Separation(f, position_[v]);
            if (dist > minOutside_)
            {
                PushBack(vlink_, kConflict0 + f, v);
                conflictFace_[v] = f;
                if (dist > face_[f].maxConflictDistance)
                {
                    face_[f].maxConflictDistance = dist;
                    face_[f].maxConflict = v;
                }
            }
            else
            {
                PushBack(vlink_, kOrphans, v);
                conflictFace_[v] = kNone;
            }
        }
        RetireFace(merged_[i]);
    }
}

// quickhull.c:805-845: merges the face across `e` into e's face.
void Builder::ConnectFaces(int32_t e)
{
    Edge* E = edge_;
    const int32_t f = E[e].face;
    const int32_t twin = E[e].twin;
    const int32_t twinFace = E[twin].face;
    int32_t edgePrev = E[e].prev;
    int32_t edgeNext = E[e].next;
    int32_t twinPrev = E[twin].prev;
    int32_t twinNext = E[twin].next;
    while (E[E[edgePrev].twin].face == twinFace)
    {
        edgePrev = E[edgePrev].prev;
        twinNext = E[twinNext].next;
    }
    while (E[E[edgeNext].twin].face == twinFace)
    {
        edgeNext = E[edgeNext].next;
        twinPrev = E[twinPrev].prev;
    }
    face_[f].edge = edgePrev;
    mergedCount_ = 0;
    merged_[mergedCount_++] = twinFace;
    face_[twinFace].mark = kDeleted;
    face_[twinFace].edge = kNone;
    for (int32_t a = twinNext; a != E[twinPrev].next; a = E[a].next)
    {
        E[a].face = f;
    }
    DestroyEdges(E[edgePrev].next, edgeNext);
    DestroyEdges(E[twinPrev].next, twinNext);
    ConnectEdges(edgePrev, twinNext);
    ConnectEdges(twinPrev, edgeNext);
    NewellPlane(f);
    Recache(f);
    Absorb(f);
}

bool Builder::MergeConcave(int32_t f)
{
    int32_t e = face_[f].edge;
    do
    {
        if (EdgeConcave(e, minRadius_) || EdgeConcave(edge_[e].twin, minRadius_))
        {
            ConnectFaces(e);
            return !overflow_;
        }
        e = edge_[e].next;
    } while (e != face_[f].edge);
    return false;
}

bool Builder::MergeCoplanar(int32_t f)
{
    int32_t e = face_[f].edge;
    do
    {
        if (!EdgeConvex(e, minRadius_) || !EdgeConvex(edge_[e].twin, minRadius_))
        {
            ConnectFaces(e);
            return !overflow_;
        }
        e = edge_[e].next;
    } while (e != face_[f].edge);
    return false;
}

// quickhull.c:877-924: flipped cone faces into their largest neighbour,
// then concave repair, then coplanar cleanup.
void Builder::MergeFaces()
{
    for (int32_t i = 0; i < coneCount_ && !overflow_; ++i)
    {
        const int32_t f = cone_[i];
        if (face_[f].mark == kVisible && face_[f].flipped)
        {
            face_[f].flipped = 0;
            m3real bestArea = 0.0f;
            int32_t bestEdge = kNone;
            int32_t e = face_[f].edge;
            do
            {
                const m3real area = face_[edge_[edge_[e].twin].face].area;
                if (area > bestArea)
                {
                    bestArea = area;
                    bestEdge = e;
                }
                e = edge_[e].next;
            } while (e != face_[f].edge);
            if (bestEdge == kNone)
            {
                overflow_ = true;
                return;
            }
            ConnectFaces(bestEdge);
        }
    }
    for (int32_t i = 0; i < coneCount_ && !overflow_; ++i)
    {
        const int32_t f = cone_[i];
        if (face_[f].mark == kVisible)
        {
            while (MergeConcave(f))
            {
            }
        }
    }
    for (int32_t i = 0; i < coneCount_ && !overflow_; ++i)
    {
        const int32_t f = cone_[i];
        if (face_[f].mark == kVisible)
        {
            while (MergeCoplanar(f))
            {
            }
        }
    }
}

// quickhull.c:926-960: orphans to the visible cone face they are farthest
// in front of; the rest are inside.
void Builder::ResolveVertices()
{
    int32_t n = vlink_[kOrphans].next;
    while (n != kOrphans)
    {
        const int32_t v = n;
        n = vlink_[n].next;
        Remove(vlink_, v);
        m3real best = minOutside_;
        int32_t bestFace = kNone;
        for (int32_t i = 0; i < coneCount_; ++i)
        {
            if (face_[cone_[i]].mark == kVisible)
            {
                const m3real dist = Separation(cone_[i], position_[v]);
                if (dist > best)
                {
                    best = dist;
                    bestFace = cone_[i];
                }
            }
        }
        if (bestFace != kNone)
        {
            PushBack(vlink_, kConflict0 + bestFace, v);
            conflictFace_[v] = bestFace;
            if (best > face_[bestFace].maxConflictDistance)
            {
                face_[bestFace].maxConflictDistance = best;
                face_[bestFace].maxConflict = v;
            }
        }
    }
}

// quickhull.c:962-983: deleted faces leave the hull list, the surviving
// cone faces join its end in cone order.
void Builder::ResolveFaces()
{
    int32_t n = flink_[kHullFaces].next;
    while (n != kHullFaces)
    {
        const int32_t f = n;
        n = flink_[n].next;
        if (face_[f].mark == kDeleted && InList(flink_, f))
        {
            Remove(flink_, f);
        }
    }
    for (int32_t i = 0; i < coneCount_; ++i)
    {
        if (face_[cone_[i]].mark == kDeleted)
        {
            continue;
        }
        PushBack(flink_, kHullFaces, cone_[i]);
    }
}

bool Builder::AddVertex(int32_t v)
{
    const int32_t f = conflictFace_[v];
    conflictFace_[v] = kNone;
    Remove(vlink_, v);
    PushBack(vlink_, kHullVerts, v);
    horizonCount_ = 0;
    if (!Horizon(v, f))
    {
        return false;
    }
    coneCount_ = 0;
    if (!Cone(v))
    {
        return false;
    }
    MergeFaces();
    if (overflow_)
    {
        return false;
    }
    ResolveVertices();
    ResolveFaces();
    return true;
}

// quickhull.c:1001-1039: unreachable vertices leave the list; counts.
void Builder::Clean()
{
    int32_t faces = 0;
    int32_t halfEdges = 0;
    for (int32_t f = flink_[kHullFaces].next; f != kHullFaces; f = flink_[f].next)
    {
        int32_t e = face_[f].edge;
        do
        {
            reachable_[edge_[e].origin] = 1;
            e = edge_[e].next;
            halfEdges++;
        } while (e != face_[f].edge);
        faces++;
    }
    int32_t vertices = 0;
    int32_t n = vlink_[kHullVerts].next;
    while (n != kHullVerts)
    {
        const int32_t v = n;
        n = vlink_[n].next;
        if (!reachable_[v])
        {
            Remove(vlink_, v);
        }
        else
        {
            vertices++;
        }
    }
    finalVertices_ = vertices;
    finalHalfEdges_ = halfEdges;
    finalFaces_ = faces;
}

bool Builder::Build(const m3Vec3* points, int32_t count, m3HullData* out)
{
    InitList(vlink_, kOrphans);
    InitList(vlink_, kHullVerts);
    InitList(flink_, kHullFaces);
    // Shift by the first point to reduce round-off.
    const m3Vec3 origin = points[0];
    for (int32_t i = 0; i < count; ++i)
    {
        shifted_[i] = m3Sub3(points[i], origin);
    }
    Tolerance(count, shifted_);
    if (!Seed(count, shifted_))
    {
        return false;
    }
    int32_t budget = M3_HULL_MAX_VERTS - 4;
    int32_t v = NextConflict();
    while (v != kNone && budget > 0)
    {
        if (!AddVertex(v))
        {
            return false;
        }
        v = NextConflict();
        budget -= 1;
    }
    Clean();
    // Euler's identity and the slab's caps gate the emit.
    const int32_t nv = finalVertices_;
    const int32_t ne = finalHalfEdges_ / 2;
    const int32_t nf = finalFaces_;
    if (nv - ne + nf != 2 || nf < 4 || nv > M3_HULL_MAX_VERTS || nf > M3_HULL_MAX_FACES ||
        finalHalfEdges_ > M3_HULL_MAX_FACE_INDICES)
    {
        return false;
    }
    memset(out, 0, sizeof(*out));
    int32_t vertexCount = 0;
    for (int32_t n = vlink_[kHullVerts].next; n != kHullVerts; n = vlink_[n].next)
    {
        finalIndex_[n] = vertexCount;
        out->vertices[vertexCount] = m3Add3(position_[n], origin);
        vertexCount += 1;
    }
    int32_t faceCount = 0;
    int32_t indexCount = 0;
    for (int32_t f = flink_[kHullFaces].next; f != kHullFaces; f = flink_[f].next)
    {
        out->faceNormals[faceCount] = face_[f].normal;
        out->faceOffsets[faceCount] = face_[f].offset + m3Dot3(face_[f].normal, origin);
        out->faceVertStart[faceCount] = (uint16_t)indexCount;
        int32_t k = 0;
        int32_t e = face_[f].edge;
        do
        {
            out->faceIndices[indexCount++] = (uint8_t)finalIndex_[edge_[e].origin];
            k += 1;
            e = edge_[e].next;
        } while (e != face_[f].edge);
        out->faceVertCounts[faceCount] = (uint8_t)k;
        faceCount += 1;
    }
    out->vertexCount = vertexCount;
    out->faceCount = faceCount;
    out->indexCount = indexCount;
    return true;
}

// quickhull.c:1041-1108: unit-density volume, centre and central inertia
// by the divergence theorem, fanning each face against the first vertex.
bool HullMassProperties(m3HullData* hull)
{
    const m3Vec3 origin = hull->vertices[0];
    m3real volume = 0.0f;
    m3Vec3 center = v3(0.0f, 0.0f, 0.0f);
    m3real xx = 0.0f;
    m3real yy = 0.0f;
    m3real zz = 0.0f;
    m3real xy = 0.0f;
    m3real xz = 0.0f;
    m3real yz = 0.0f;
    for (int32_t f = 0; f < hull->faceCount; ++f)
    {
        const int32_t n = hull->faceVertCounts[f];
        const int32_t start = hull->faceVertStart[f];
        const m3Vec3 a = m3Sub3(hull->vertices[hull->faceIndices[start]], origin);
        for (int32_t k = 1; k + 1 < n; ++k)
        {
            const m3Vec3 b = m3Sub3(hull->vertices[hull->faceIndices[start + k]], origin);
            const m3Vec3 c = m3Sub3(hull->vertices[hull->faceIndices[start + k + 1]], origin);
            const m3real det = m3Dot3(a, m3Cross3(b, c));
            volume += det;
            const m3Vec3 d = m3Add3(a, m3Add3(b, c));
            center = m3Add3(center, m3MulSV3(det, d));
            xx += det * (a.x * a.x + b.x * b.x + c.x * c.x + d.x * d.x);
            yy += det * (a.y * a.y + b.y * b.y + c.y * c.y + d.y * d.y);
            zz += det * (a.z * a.z + b.z * b.z + c.z * c.z + d.z * d.z);
            xy += det * (a.x * a.y + b.x * b.y + c.x * c.y + d.x * d.y);
            xz += det * (a.x * a.z + b.x * b.z + c.x * c.z + d.x * d.z);
            yz += det * (a.y * a.z + b.y * b.z + c.y * c.z + d.y * d.z);
        }
    }
    if (!(volume > 0.0f))
    {
        return false;
    }
    const m3Vec3 localCenter = m3MulSV3(0.25f / volume, center);
    const m3real mass = volume / 6.0f;
    m3Mat3 inertia;
    inertia.cx = v3(yy + zz, -xy, -xz);
    inertia.cy = v3(-xy, xx + zz, -yz);
    inertia.cz = v3(-xz, -yz, xx + yy);
    const m3real scale = 1.0f / 120.0f;
    inertia.cx = m3MulSV3(scale, inertia.cx);
    inertia.cy = m3MulSV3(scale, inertia.cy);
    inertia.cz = m3MulSV3(scale, inertia.cz);
    // Parallel axes: from the fan origin to the centre of mass.
    const m3Vec3 c = localCenter;
    const m3real c2 = m3Dot3(c, c);
    inertia.cx.x -= mass * (c2 - c.x * c.x);
    inertia.cy.y -= mass * (c2 - c.y * c.y);
    inertia.cz.z -= mass * (c2 - c.z * c.z);
    inertia.cy.x += mass * c.x * c.y;
    inertia.cx.y += mass * c.x * c.y;
    inertia.cz.x += mass * c.x * c.z;
    inertia.cx.z += mass * c.x * c.z;
    inertia.cz.y += mass * c.y * c.z;
    inertia.cy.z += mass * c.y * c.z;
    hull->unitMass = mass;
    hull->unitCom = m3Add3(localCenter, origin);
    hull->unitInertiaCom = inertia;
    return true;
}
} // namespace

// quickhull.c:1110-1216 (m3ComputeHull): false for fewer than 4 or more
// than 256 points, a non-finite or huge coordinate, a degenerate cloud,
// a hull over the slab's caps or without positive volume.  The
// half-edge table is left to the caller (m3HullBuildHalfEdges).
bool m3QuickHull(const m3Vec3* points, int32_t count, m3HullData* out)
{
    if (points == nullptr || out == nullptr || count < 4 || count > kMaxInput)
    {
        return false;
    }
    for (int32_t i = 0; i < count; ++i)
    {
        const m3Vec3 p = points[i];
        if (!(p.x == p.x) || !(p.y == p.y) || !(p.z == p.z) || p.x > 1.0e18f || p.x < -1.0e18f ||
            p.y > 1.0e18f || p.y < -1.0e18f || p.z > 1.0e18f || p.z < -1.0e18f)
        {
            return false;
        }
    }
    std::unique_ptr<Builder> b(new (std::nothrow) Builder());
    if (!b || !b->Build(points, count, out))
    {
        return false;
    }
    if (!HullMassProperties(out))
    {
        memset(out, 0, sizeof(*out));
        return false;
    }
    return true;
}
