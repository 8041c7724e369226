// The broadphase tree the reference keeps as world state (its nodes and
// proxy ids are snapshot bytes, snapshot.c:245-247): a dynamic AABB tree
// of fat shape bounds, grown by surface-area-heuristic descent and kept
// balanced by AVL-style rotations (dynamic_tree.c:16-363).  This path
// does not query it (candidate pairs come from a sort-and-sweep over
// fresh bounds, the same set); it maintains it so a snapshot carries the
// reference's tree byte for byte.  Every bound is a double and every
// decision a strict comparison, so the same sequence of inserts and
// removes gives the same nodes on the host (shape creation) and on the
// device (the per-step refresh).
#ifndef M3_TREE_H
#define M3_TREE_H

#include "m3_layout.h"

#define M3_TREE_NULL (-1)

typedef struct m3Aabb
{
    double lo[3];
    double hi[3];
} m3Aabb;

// A tree over a node array of fixed capacity; root and free-list head
// live in the world scalars.
typedef struct m3TreeRef
{
    m3TreeNode* nodes;
    int32_t capacity;
    int32_t* root;
    int32_t* freeList;
} m3TreeRef;

M3_HD m3TreeRef m3WorldTree(const m3WorldView& w)
{
    m3TreeRef t;
    t.nodes = w.treeNodes;
    t.capacity = 2 * w.sc->shapeCap;
    t.root = &w.sc->treeRoot;
    t.freeList = &w.sc->treeFreeList;
    return t;
}

// An empty tree: every node free, chained in index order
// (dynamic_tree.c:41-55).
M3_HD void m3TreeInit(m3TreeRef t)
{
    for (int32_t i = 0; i < t.capacity; ++i)
    {
        m3TreeNode n;
        for (int32_t k = 0; k < 3; ++k)
        {
            n.lo[k] = 0.0;
            n.hi[k] = 0.0;
        }
        n.parent = i + 1 < t.capacity ? i + 1 : M3_TREE_NULL;
        n.child1 = 0;
        n.child2 = 0;
        n.userData = 0;
        n.height = -1;
        n.pad = 0;
        t.nodes[i] = n;
    }
    *t.root = M3_TREE_NULL;
    *t.freeList = t.capacity > 0 ? 0 : M3_TREE_NULL;
}

M3_HD double m3TreeArea(const double lo[3], const double hi[3])
{
    const double dx = hi[0] - lo[0];
    const double dy = hi[1] - lo[1];
    const double dz = hi[2] - lo[2];
    return 2.0 * (dx * dy + dy * dz + dz * dx);
}

M3_HD void m3TreeUnion(const double aLo[3], const double aHi[3], const double bLo[3],
                       const double bHi[3], double outLo[3], double outHi[3])
{
    for (int32_t k = 0; k < 3; ++k)
    {
        outLo[k] = aLo[k] < bLo[k] ? aLo[k] : bLo[k];
        outHi[k] = aHi[k] > bHi[k] ? aHi[k] : bHi[k];
    }
}

// Node storage the tree operations go through, one whole record at a
// time: the plain node array (host), or the array behind a cache in
// shared memory (the device's tree kernel, m3TreeCachedStore).
struct m3TreeArrayStore
{
    m3TreeNode* nodes;
    M3_HD_MEMBER m3TreeNode Get(int32_t i) const { return nodes[i]; }
    M3_HD_MEMBER void Put(int32_t i, const m3TreeNode& n) const { nodes[i] = n; }
};

template <class Store> M3_HD int32_t m3TreeTakeNode(m3TreeRef t, const Store& st)
{
    const int32_t id = *t.freeList;
    if (id == M3_TREE_NULL)
    {
        return M3_TREE_NULL;
    }
    m3TreeNode n = st.Get(id);
    *t.freeList = n.parent;
    n.parent = M3_TREE_NULL;
    n.child1 = M3_TREE_NULL;
    n.child2 = M3_TREE_NULL;
    n.height = 0;
    n.userData = -1;
    n.pad = 0;
    st.Put(id, n);
    return id;
}

// A freed node is zeroed and pushed on the free chain (dynamic_tree.c:83-90).
template <class Store> M3_HD void m3TreeGiveNode(m3TreeRef t, const Store& st, int32_t id)
{
    m3TreeNode n;
    for (int32_t k = 0; k < 3; ++k)
    {
        n.lo[k] = 0.0;
        n.hi[k] = 0.0;
    }
    n.child1 = 0;
    n.child2 = 0;
    n.userData = 0;
    n.pad = 0;
    n.parent = *t.freeList;
    n.height = -1;
    st.Put(id, n);
    *t.freeList = id;
}

M3_HD int32_t m3TreeMaxI(int32_t a, int32_t b)
{
    return a > b ? a : b;
}

// Re-links `child` under `parent` in place of `old` (or as the root).
template <class Store>
M3_HD void m3TreeReplaceChild(m3TreeRef t, const Store& st, int32_t parent, int32_t old,
                              int32_t child)
{
    if (parent != M3_TREE_NULL)
    {
        m3TreeNode n = st.Get(parent);
        if (n.child1 == old)
        {
            n.child1 = child;
        }
        else
        {
            n.child2 = child;
        }
        st.Put(parent, n);
    }
    else
    {
        *t.root = child;
    }
}

// Rotates the subtree at a (record A, children records B and C) whose
// children's heights differ by more than one: the taller child (p)
// rises, a becomes its child, and a keeps the shorter of p's children
// while p keeps the taller one (dynamic_tree.c:92-203).  Writes a, p and
// the moved grandchild; returns p's record (bounds and height final).
template <class Store>
M3_HD m3TreeNode m3TreeRotate(m3TreeRef t, const Store& st, int32_t a, m3TreeNode A,
                              const m3TreeNode& B, const m3TreeNode& C, int32_t* newRoot)
{
    const int32_t b = A.child1;
    const int32_t c = A.child2;
    const bool right = C.height - B.height > 1;
    const int32_t p = right ? c : b;
    m3TreeNode P = right ? C : B;
    const m3TreeNode& Q = right ? B : C;
    const int32_t p1 = P.child1;
    const int32_t p2 = P.child2;
    const m3TreeNode P1 = st.Get(p1);
    const m3TreeNode P2 = st.Get(p2);
    P.child1 = a;
    P.parent = A.parent;
    A.parent = p;
    m3TreeReplaceChild(t, st, P.parent, a, p);
    // keep: p's taller child stays with p; move: the other goes to a.
    const bool firstTaller = P1.height > P2.height;
    const int32_t keep = firstTaller ? p1 : p2;
    const int32_t move = firstTaller ? p2 : p1;
    const m3TreeNode& K = firstTaller ? P1 : P2;
    m3TreeNode M = firstTaller ? P2 : P1;
    P.child2 = keep;
    if (right)
    {
        A.child2 = move;
    }
    else
    {
        A.child1 = move;
    }
    M.parent = a;
    m3TreeUnion(Q.lo, Q.hi, M.lo, M.hi, A.lo, A.hi);
    m3TreeUnion(A.lo, A.hi, K.lo, K.hi, P.lo, P.hi);
    A.height = 1 + m3TreeMaxI(Q.height, M.height);
    P.height = 1 + m3TreeMaxI(A.height, K.height);
    st.Put(move, M);
    st.Put(a, A);
    st.Put(p, P);
    *newRoot = p;
    return P;
}

// Walks from `index` to the root, rebalancing and refitting heights and
// bounds (dynamic_tree.c:205-219).  The balance test reads the node's
// stored height, as the reference's does before its refit; after a
// rotation the risen node's height and bounds are already what the
// refit would compute (the union of its two children, in order).
// `from`, when not M3_TREE_NULL, is a child of `index` whose current
// record is `fromRec`: the walk carries each level's record up to the
// next instead of reading it again, and asks for the parent's record
// before the level's arithmetic, so a level waits on one load (the
// other child).  A walk longer than the node count can only come from a
// malformed tree; it stops there.
template <class Store>
M3_HD void m3TreeRefit(m3TreeRef t, const Store& st, int32_t index, int32_t from,
                       m3TreeNode fromRec)
{
    if (index == M3_TREE_NULL)
    {
        return;
    }
    m3TreeNode n = st.Get(index);
    for (int32_t guard = 0; guard < t.capacity; ++guard)
    {
        m3TreeNode c1;
        m3TreeNode c2;
        if (n.child1 == from)
        {
            c1 = fromRec;
            c2 = st.Get(n.child2);
        }
        else if (n.child2 == from)
        {
            c1 = st.Get(n.child1);
            c2 = fromRec;
        }
        else
        {
            c1 = st.Get(n.child1);
            c2 = st.Get(n.child2);
        }
        const int32_t up = n.parent;
        m3TreeNode upRec = n;
        if (up != M3_TREE_NULL)
        {
            upRec = st.Get(up);
        }
        const int32_t balance = c2.height - c1.height;
        if (n.height >= 2 && n.child1 != M3_TREE_NULL && (balance > 1 || balance < -1))
        {
            int32_t root = index;
            const m3TreeNode risen = m3TreeRotate(t, st, index, n, c1, c2, &root);
            if (risen.parent == M3_TREE_NULL)
            {
                return;
            }
            // The rotation re-linked the parent's child: read it again.
            from = root;
            fromRec = risen;
            index = risen.parent;
            n = st.Get(index);
            continue;
        }
        n.height = 1 + m3TreeMaxI(c1.height, c2.height);
        m3TreeUnion(c1.lo, c1.hi, c2.lo, c2.hi, n.lo, n.hi);
        st.Put(index, n);
        if (up == M3_TREE_NULL)
        {
            return;
        }
        from = index;
        fromRec = n;
        index = up;
        n = upRec;
    }
}

// Inserts a leaf for `userData` with bounds [lo, hi]; returns its node or
// M3_TREE_NULL when the node pool is exhausted (dynamic_tree.c:221-322).
template <class Store>
M3_HD int32_t m3TreeInsert(m3TreeRef t, const Store& st, const double lo[3], const double hi[3],
                           int32_t userData)
{
    const int32_t leaf = m3TreeTakeNode(t, st);
    if (leaf == M3_TREE_NULL)
    {
        return M3_TREE_NULL;
    }
    m3TreeNode L = st.Get(leaf);
    for (int32_t k = 0; k < 3; ++k)
    {
        L.lo[k] = lo[k];
        L.hi[k] = hi[k];
    }
    L.userData = userData;
    L.height = 0;
    if (*t.root == M3_TREE_NULL)
    {
        st.Put(leaf, L);
        *t.root = leaf;
        return leaf;
    }
    // Descend while a child is cheaper than pairing here (at most one
    // level per node: a longer descent means a malformed tree).  The
    // chosen child's record, its own area and the area of its union
    // with the new box (both computed for its cost) are carried down,
    // so each level loads and measures only the two children.  (Asking
    // for the grandchildren before choosing hid the loads but doubled the
    // instructions, and the walk runs beside the step's own kernels,
    // where instructions cost more than latency.)
    int32_t index = *t.root;
    m3TreeNode cur = st.Get(index);
    double curUnion;
    double curArea;
    {
        double ulo[3];
        double uhi[3];
        m3TreeUnion(cur.lo, cur.hi, lo, hi, ulo, uhi);
        curUnion = m3TreeArea(ulo, uhi);
        curArea = m3TreeArea(cur.lo, cur.hi);
    }
    for (int32_t guard = 0; cur.height > 0; ++guard)
    {
        if (guard >= t.capacity)
        {
            return M3_TREE_NULL;
        }
        const int32_t c1 = cur.child1;
        const int32_t c2 = cur.child2;
        const m3TreeNode n1 = st.Get(c1);
        const m3TreeNode n2 = st.Get(c2);
        const double here = 2.0 * curUnion;
        const double inherited = 2.0 * (curUnion - curArea);
        double ulo[3];
        double uhi[3];
        m3TreeUnion(n1.lo, n1.hi, lo, hi, ulo, uhi);
        const double union1 = m3TreeArea(ulo, uhi);
        const double area1 = n1.height == 0 ? 0.0 : m3TreeArea(n1.lo, n1.hi);
        m3TreeUnion(n2.lo, n2.hi, lo, hi, ulo, uhi);
        const double union2 = m3TreeArea(ulo, uhi);
        const double area2 = n2.height == 0 ? 0.0 : m3TreeArea(n2.lo, n2.hi);
        // dynamic_tree.c:245-273: a leaf child's cost is its union's area
        // plus the inherited cost; an internal child's subtracts its own
        // area.
        const double cost1 = n1.height == 0 ? union1 + inherited : union1 - area1 + inherited;
        const double cost2 = n2.height == 0 ? union2 + inherited : union2 - area2 + inherited;
        if (here < cost1 && here < cost2)
        {
            break;
        }
        if (cost1 < cost2)
        {
            index = c1;
            cur = n1;
            curUnion = union1;
            curArea = area1; // a leaf ends the descent: its area is not read
        }
        else
        {
            index = c2;
            cur = n2;
            curUnion = union2;
            curArea = area2;
        }
    }
    // A new parent takes the sibling's place; sibling and leaf hang
    // under it in that order.
    const int32_t sibling = index;
    m3TreeNode S = cur;
    const int32_t oldParent = S.parent;
    const int32_t parent = m3TreeTakeNode(t, st);
    if (parent == M3_TREE_NULL)
    {
        m3TreeGiveNode(t, st, leaf);
        return M3_TREE_NULL;
    }
    m3TreeNode N = st.Get(parent);
    N.parent = oldParent;
    N.userData = -1;
    m3TreeUnion(lo, hi, S.lo, S.hi, N.lo, N.hi);
    N.height = S.height + 1;
    m3TreeReplaceChild(t, st, oldParent, sibling, parent);
    N.child1 = sibling;
    N.child2 = leaf;
    S.parent = parent;
    L.parent = parent;
    st.Put(parent, N);
    st.Put(sibling, S);
    st.Put(leaf, L);
    m3TreeRefit(t, st, parent, leaf, L);
    return leaf;
}

// Removes a leaf; its parent is freed and the sibling takes the parent's
// place (dynamic_tree.c:324-358).
template <class Store> M3_HD void m3TreeRemove(m3TreeRef t, const Store& st, int32_t leaf)
{
    if (leaf == *t.root)
    {
        *t.root = M3_TREE_NULL;
        m3TreeGiveNode(t, st, leaf);
        return;
    }
    const int32_t parent = st.Get(leaf).parent;
    const m3TreeNode P = st.Get(parent);
    const int32_t grand = P.parent;
    const int32_t sibling = P.child1 == leaf ? P.child2 : P.child1;
    m3TreeNode S = st.Get(sibling);
    if (grand != M3_TREE_NULL)
    {
        m3TreeReplaceChild(t, st, grand, parent, sibling);
        S.parent = grand;
        st.Put(sibling, S);
        m3TreeGiveNode(t, st, parent);
        m3TreeRefit(t, st, grand, sibling, S);
    }
    else
    {
        *t.root = sibling;
        S.parent = M3_TREE_NULL;
        st.Put(sibling, S);
        m3TreeGiveNode(t, st, parent);
    }
    m3TreeGiveNode(t, st, leaf);
}

M3_HD bool m3TreeContains(const m3TreeNode& n, const m3Aabb& b)
{
    return n.lo[0] <= b.lo[0] && n.lo[1] <= b.lo[1] && n.lo[2] <= b.lo[2] && b.hi[0] <= n.hi[0] &&
           b.hi[1] <= n.hi[1] && b.hi[2] <= n.hi[2];
}

// Shape pose in the world: body pose composed with the compound offset
// (world_internal.h:1276-1290).
M3_HD m3Transform m3ShapePose(const m3WorldView& w, int32_t shape)
{
    const int32_t body = w.shapeBody[shape];
    m3Transform xf = w.xf[body];
    if (w.hasOffset[shape] != 0)
    {
        const m3Vec3 r = m3RotateVec3(xf.q, w.localPos[shape]);
        xf.p.x += (double)r.x;
        xf.p.y += (double)r.y;
        xf.p.z += (double)r.z;
        xf.q = m3MulQuat(xf.q, w.localRot[shape]);
    }
    return xf;
}

// Fresh bounds of one non-plane shape, tight plus the margin
// (broad_phase.c:22-135): hull vertices rotated out, capsule cap
// centres, sphere centre, min and max in double.
M3_HD m3Aabb m3ShapeFreshBounds(const m3WorldView& w, int32_t shape)
{
    const m3Transform xf = m3ShapePose(w, shape);
    m3Aabb box;
    const uint8_t type = w.shapeType[shape];
    if (type == M3_SHAPE_HULL)
    {
        const m3HullData* hull = &w.hulls[w.hullIndex[shape]];
        for (int32_t k = 0; k < 3; ++k)
        {
            box.lo[k] = 1.0e30;
            box.hi[k] = -1.0e30;
        }
        const int32_t nv = hull->vertexCount;
        for (int32_t v = 0; v < nv; ++v)
        {
            const m3Vec3 r = m3RotateVec3(xf.q, hull->vertices[v]);
            const double p[3] = {xf.p.x + (double)r.x, xf.p.y + (double)r.y,
                                 xf.p.z + (double)r.z};
            for (int32_t k = 0; k < 3; ++k)
            {
                box.lo[k] = p[k] < box.lo[k] ? p[k] : box.lo[k];
                box.hi[k] = p[k] > box.hi[k] ? p[k] : box.hi[k];
            }
        }
        for (int32_t k = 0; k < 3; ++k)
        {
            box.lo[k] -= (double)M3_AABB_MARGIN;
            box.hi[k] += (double)M3_AABB_MARGIN;
        }
        return box;
    }
    if (type == M3_SHAPE_HEIGHTFIELD)
    {
        // The grid's box from the shape's origin and the baked sample
        // extremes, rotation ignored (broad_phase.c:52-67).
        const m3HeightFieldDev hf = w.hfs[w.hfIndex[shape]];
        box.lo[0] = xf.p.x;
        box.lo[1] = xf.p.y + (double)hf.minHeight;
        box.lo[2] = xf.p.z;
        box.hi[0] = xf.p.x + (double)((float)(hf.nx - 1) * hf.cellSize);
        box.hi[1] = xf.p.y + (double)hf.maxHeight;
        box.hi[2] = xf.p.z + (double)((float)(hf.nz - 1) * hf.cellSize);
        for (int32_t k = 0; k < 3; ++k)
        {
            box.lo[k] -= (double)M3_AABB_MARGIN;
            box.hi[k] += (double)M3_AABB_MARGIN;
        }
        return box;
    }
    if (type == M3_SHAPE_CAPSULE)
    {
        const m3Vec3 r1 = m3RotateVec3(xf.q, w.geom[shape].v);
        const m3Vec3 r2 = m3RotateVec3(xf.q, w.geom[shape].v2);
        const double c1[3] = {xf.p.x + (double)r1.x, xf.p.y + (double)r1.y, xf.p.z + (double)r1.z};
        const double c2[3] = {xf.p.x + (double)r2.x, xf.p.y + (double)r2.y, xf.p.z + (double)r2.z};
        const double fat = (double)(w.geom[shape].s + M3_AABB_MARGIN);
        for (int32_t k = 0; k < 3; ++k)
        {
            box.lo[k] = (c1[k] < c2[k] ? c1[k] : c2[k]) - fat;
            box.hi[k] = (c1[k] > c2[k] ? c1[k] : c2[k]) + fat;
        }
        return box;
    }
    const m3Vec3 r = m3RotateVec3(xf.q, w.geom[shape].v);
    const double c[3] = {xf.p.x + (double)r.x, xf.p.y + (double)r.y, xf.p.z + (double)r.z};
    const double fat = (double)(w.geom[shape].s + M3_AABB_MARGIN);
    for (int32_t k = 0; k < 3; ++k)
    {
        box.lo[k] = c[k] - fat;
        box.hi[k] = c[k] + fat;
    }
    return box;
}

// The box a shape enters the tree with at creation (broad_phase.c:
// 149-173): the fresh bounds, except for a heightfield, whose box hangs
// from its BODY's origin with a fixed 0.1 margin.
M3_HD m3Aabb m3ShapeCreationBounds(const m3WorldView& w, int32_t shape)
{
    if (w.shapeType[shape] != M3_SHAPE_HEIGHTFIELD)
    {
        return m3ShapeFreshBounds(w, shape);
    }
    const m3HeightFieldDev hf = w.hfs[w.hfIndex[shape]];
    const m3Transform xf = w.xf[w.shapeBody[shape]];
    const double margin = 0.1;
    m3Aabb box;
    box.lo[0] = xf.p.x - margin;
    box.lo[1] = xf.p.y + (double)hf.minHeight - margin;
    box.lo[2] = xf.p.z - margin;
    box.hi[0] = xf.p.x + (double)((float)(hf.nx - 1) * hf.cellSize) + margin;
    box.hi[1] = xf.p.y + (double)hf.maxHeight + margin;
    box.hi[2] = xf.p.z + (double)((float)(hf.nz - 1) * hf.cellSize) + margin;
    return box;
}

#ifndef __CUDACC__
#include <vector>

// Structural check of a tree read from outside (a restored snapshot):
// every link in range, parents and children agreeing, heights and
// bounds as the tree keeps them, no node reached twice, the free chain
// of free nodes only, together covering every node, and each live
// non-plane shape's proxy a leaf naming it.  The device trusts a tree
// that passed.
static inline bool m3TreeValid(const m3TreeNode* nodes, int32_t capacity, int32_t root,
                               int32_t freeList, const int32_t* proxyId, const uint8_t* alive,
                               const uint8_t* type, int32_t shapeMax)
{
    std::vector<uint8_t> seen((size_t)capacity, 0);
    int32_t reached = 0;
    std::vector<int32_t> stack;
    if (root != M3_TREE_NULL)
    {
        if (root < 0 || root >= capacity || nodes[root].parent != M3_TREE_NULL)
        {
            return false;
        }
        stack.push_back(root);
    }
    while (!stack.empty())
    {
        const int32_t i = stack.back();
        stack.pop_back();
        if (seen[(size_t)i] != 0)
        {
            return false;
        }
        seen[(size_t)i] = 1;
        reached += 1;
        const m3TreeNode& n = nodes[i];
        if (n.height == 0)
        {
            if (n.userData < 0 || n.userData >= shapeMax || proxyId[n.userData] != i)
            {
                return false;
            }
            continue;
        }
        if (n.height < 0)
        {
            return false;
        }
        const int32_t c[2] = {n.child1, n.child2};
        for (int32_t k = 0; k < 2; ++k)
        {
            if (c[k] < 0 || c[k] >= capacity || nodes[c[k]].parent != i)
            {
                return false;
            }
            stack.push_back(c[k]);
        }
        if (n.height != 1 + m3TreeMaxI(nodes[c[0]].height, nodes[c[1]].height))
        {
            return false;
        }
    }
    for (int32_t i = freeList, guard = 0; i != M3_TREE_NULL; i = nodes[i].parent, ++guard)
    {
        if (i < 0 || i >= capacity || guard >= capacity || seen[(size_t)i] != 0 ||
            nodes[i].height != -1)
        {
            return false;
        }
        seen[(size_t)i] = 1;
        reached += 1;
    }
    if (reached != capacity)
    {
        return false;
    }
    for (int32_t s = 0; s < shapeMax; ++s)
    {
        const int32_t leaf = proxyId[s];
        const bool wantsLeaf = alive[s] != 0 && type[s] != M3_SHAPE_PLANE;
        if (leaf == M3_TREE_NULL)
        {
            if (wantsLeaf)
            {
                return false;
            }
            continue;
        }
        if (leaf < 0 || leaf >= capacity || nodes[leaf].height != 0 || nodes[leaf].userData != s)
        {
            return false;
        }
    }
    return true;
}
#endif

#endif // M3_TREE_H
