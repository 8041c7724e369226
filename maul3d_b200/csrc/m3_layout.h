// One world's memory image: a single slab holding every persistent SoA
// array the step reads or writes, followed (on the device only) by the
// step's scratch arrays.  The host keeps a byte-identical copy of the
// persistent part, so moving a world between host and HBM is one copy
// each way and a batch of thousands of worlds is thousands of slabs
// addressed through one descriptor table.
//
// Field lists are X-macros so the offsets, the host view and the
// device view are generated from a single declaration.  Every array is
// sized by the world's capacity (bodies, shapes, joints, pairs) like
// the reference's persistent arrays (src/world.c:160-440), and aligned
// to 256 bytes so warp accesses start on a sector boundary.
#ifndef M3_LAYOUT_H
#define M3_LAYOUT_H

#include "maul3d_b200.h"
#include "m3_core.h"

// World-global scalars (the m3World header fields the step touches).
typedef struct m3WorldScalars
{
    m3Vec3 gravity;
    float contactHertz;
    float contactDampingRatio;
    float contactPushMaxSpeed;
    float restitutionThreshold;
    float maximumLinearSpeed;
    float maximumAngularSpeed;
    float hitEventThreshold;
    uint8_t sleepEnabled;
    uint8_t continuousEnabled;
    uint8_t pad0[2];
    m3Vec3 windDir;
    float windSpeed;
    float windGustHertz;
    float windGustScale;
    float windPhase;
    float lastInvH;
    uint64_t stepCount;
    int32_t bodyCap;
    int32_t shapeCap;
    int32_t jointCap;
    int32_t pairCap;
    int32_t bodyMax;
    int32_t shapeMax;
    int32_t jointMax;
    int32_t hullMax;
    int32_t pairCount;
    int32_t pairBuf;    // which of the two pair buffers is current
    int32_t status;     // M3GPU_* code of the last device step (0 = ok)
    int32_t statusDetail;
    int32_t lastColorCount;
    int32_t lastIslandCount;
    int32_t constraintCount;
    int32_t moverCount;
    int32_t jointConstraintCount;
    int32_t newPairCount; // pair list the running step is building
    // The previous step's pair count (the other pair buffer) and where the
    // ring of broken joints stood when the last step began: the last
    // step's event streams are read from them.
    int32_t prevPairCount;
    int32_t stepBrokenStart;
    // Joints the device destroyed (breakage), as a ring over jbroken:
    // the host drains entries [drained, brokenCount) into its free queue.
    int32_t brokenCount;
    // The broadphase tree's root and free-list head (nodes: treeNodes).
    int32_t treeRoot;
    int32_t treeFreeList;
    // Whether the step keeps the broadphase tree (snapshot state).  Off
    // only for worlds nobody can snapshot (the serving path's own).
    int32_t treeTracked;
    // Cursors of the ring of per-step tree move lists (device scratch):
    // the broadphase writes slot treeHead % depth and advances treeHead,
    // the tree kernel replays slot treeTail % depth and advances
    // treeTail.  Equal whenever no tree work is pending.
    int32_t treeHead;
    int32_t treeTail;
    // Work counters accumulated over every device step (observer only,
    // never hashed): the algorithmic-byte model of the roofline reads
    // them.  [0] movers x substeps, [1] contact rows x substeps,
    // [2] joint rows x substeps, [3] candidate pairs, [4] steps.
    uint64_t work[5];
    // Device clock cycles spent per step phase by the world's block,
    // accumulated over steps (observer only, never hashed; the index
    // list is M3_PHASE_* in step.cu).
    uint64_t phase[16];
} m3WorldScalars;

// One broadphase tree node, the reference's 72-byte record
// (dynamic_tree.h:18-28): bounds, links (parent doubles as the free-list
// next), the shape index on leaves, height (-1 free, 0 leaf).
typedef struct m3TreeNode
{
    double lo[3];
    double hi[3];
    int32_t parent;
    int32_t child1;
    int32_t child2;
    int32_t userData;
    int32_t height;
    int32_t pad;
} m3TreeNode;

// One heightfield slot (world_internal.h:307-315): an nx x nz grid of
// samples, row-major with x fastest, starting at `sampleStart` in the
// world's sample pool; the sample extremes are baked at creation.
typedef struct m3HeightFieldDev
{
    int32_t nx;
    int32_t nz;
    float cellSize;
    float minHeight;
    float maxHeight;
    int32_t sampleStart;
} m3HeightFieldDev;

// Per-body persistent arrays (capacity = bodyCap).
#define M3_BODY_FIELDS(X)                                                                          \
    X(m3Transform, xf)                                                                             \
    X(m3Vec3, v)                                                                                   \
    X(m3Vec3, w)                                                                                   \
    X(float, invMass)                                                                              \
    X(m3Mat3, invI)                                                                                \
    X(m3Mat3, inertia)                                                                             \
    X(m3Vec3, lc)                                                                                  \
    X(float, gravityScale)                                                                         \
    X(float, linDamp)                                                                              \
    X(float, angDamp)                                                                              \
    X(uint8_t, btype)                                                                              \
    X(uint8_t, awake)                                                                              \
    X(float, sleepTime)                                                                            \
    X(uint8_t, bullet)                                                                             \
    X(float, minExt)                                                                               \
    X(float, maxExt)                                                                               \
    X(m3Vec3, force)                                                                               \
    X(m3Vec3, torque)                                                                              \
    X(uint8_t, enabled)                                                                            \
    X(uint8_t, locks)                                                                              \
    X(float, sleepThreshold)                                                                       \
    X(uint8_t, canSleep)                                                                           \
    X(uint8_t, hasTarget)                                                                          \
    X(m3Transform, target)                                                                         \
    X(int32_t, shapeHead)                                                                          \
    X(int32_t, jointHead)                                                                          \
    X(uint8_t, bodyAlive)                                                                          \
    X(uint16_t, bodyGen)                                                                           \
    X(uint64_t, userData)

// Per-shape persistent arrays (capacity = shapeCap).
#define M3_SHAPE_FIELDS(X)                                                                         \
    X(int32_t, shapeBody)                                                                          \
    X(uint8_t, shapeType)                                                                          \
    X(m3ShapeGeom, geom)                                                                           \
    X(float, density)                                                                              \
    X(float, friction)                                                                             \
    X(float, restitution)                                                                          \
    X(float, rolling)                                                                              \
    X(uint8_t, sensor)                                                                             \
    X(uint8_t, hitEvents)                                                                          \
    X(uint8_t, preSolve)                                                                           \
    X(m3Vec3, surfVel)                                                                             \
    X(m3Vec3, localPos)                                                                            \
    X(m3Quat, localRot)                                                                            \
    X(uint8_t, hasOffset)                                                                          \
    X(uint64_t, category)                                                                          \
    X(uint64_t, mask)                                                                              \
    X(int32_t, group)                                                                              \
    X(int32_t, shapeNext)                                                                          \
    X(int32_t, proxyId)                                                                            \
    X(int32_t, hullIndex)                                                                          \
    X(int32_t, hfIndex)                                                                            \
    X(uint8_t, shapeAlive)                                                                         \
    X(uint16_t, shapeGen)                                                                          \
    X(uint64_t, shapeUserData)

// Per-joint persistent arrays (capacity = jointCap).
#define M3_JOINT_FIELDS(X)                                                                         \
    X(uint8_t, jtype)                                                                              \
    X(int32_t, jbodyA)                                                                             \
    X(int32_t, jbodyB)                                                                             \
    X(m3Vec3, jlocalA)                                                                             \
    X(m3Vec3, jlocalB)                                                                             \
    X(uint8_t, jcollide)                                                                           \
    X(m3Vec3, jimpulse)                                                                            \
    X(m3Vec3, jperp)                                                                               \
    X(m3Vec3, jlimitImp)                                                                           \
    X(m3Vec3, jangular)                                                                            \
    X(m3Quat, jframeA)                                                                             \
    X(m3Quat, jframeB)                                                                             \
    X(uint8_t, jflags)                                                                             \
    X(m3Vec3, jmotor)                                                                              \
    X(m3Vec3, jbreak)                                                                              \
    X(m3Vec3, jspring)                                                                             \
    X(float, jtargetScalar)                                                                        \
    X(m3Quat, jtargetQ)                                                                            \
    X(m3Vec3, jspringImp)                                                                          \
    X(m3Vec3, jlimits)                                                                             \
    X(int32_t, jnextA)                                                                             \
    X(int32_t, jnextB)                                                                             \
    X(uint8_t, jointAlive)                                                                         \
    X(uint16_t, jointGen)                                                                          \
    X(int32_t, jbroken)

// Broadphase tree nodes (capacity = 2 * shapeCap).
#define M3_TREE_FIELDS(X) X(m3TreeNode, treeNodes)

// Candidate pairs and manifolds, double-buffered: the step reads the
// previous step's lists for the warm-start carry while it writes the
// new ones (capacity = pairCap each).
#define M3_PAIR_FIELDS(X)                                                                          \
    X(uint64_t, keys0)                                                                             \
    X(uint64_t, keys1)                                                                             \
    X(m3Manifold, man0)                                                                            \
    X(m3Manifold, man1)

// Pointers into one slab (host or device address space).
typedef struct m3WorldView
{
    m3WorldScalars* sc;
#define M3_X_PTR(T, name) T* name;
    M3_BODY_FIELDS(M3_X_PTR)
    M3_SHAPE_FIELDS(M3_X_PTR)
    M3_JOINT_FIELDS(M3_X_PTR)
    M3_TREE_FIELDS(M3_X_PTR)
    M3_PAIR_FIELDS(M3_X_PTR)
#undef M3_X_PTR
    // Interned hull slabs (count-derived pool, outside the slab).
    m3HullData* hulls;
    // Heightfield slots and their samples (count-derived, outside the
    // slab; null in a world without heightfields).
    const m3HeightFieldDev* hfs;
    const float* hfSamples;
    // Device-only scratch (null in host views), laid out by the step
    // module which owns its record types.
    uint8_t* scratch;
    int64_t scratchBytes;
} m3WorldView;

#define M3_SLAB_ALIGN 256
#define M3_PAIR_SECTION_ALIGN 4096

M3_HD int64_t m3AlignUp(int64_t x, int64_t a)
{
    return (x + a - 1) / a * a;
}

// Assign offsets for the persistent part; returns its byte size.
// `base` may be null to only measure.
static inline int64_t m3LayoutPersistent(m3WorldView* view, uint8_t* base, int32_t bodyCap,
                                         int32_t shapeCap, int32_t jointCap, int32_t pairCap)
{
    int64_t off = 0;
    if (view)
    {
        view->sc = (m3WorldScalars*)(base ? base + off : 0);
    }
    off = m3AlignUp(off + (int64_t)sizeof(m3WorldScalars), M3_SLAB_ALIGN);
#define M3_X_OFF(T, name, n)                                                                       \
    if (view)                                                                                      \
    {                                                                                              \
        view->name = (T*)(base ? base + off : 0);                                                  \
    }                                                                                              \
    off = m3AlignUp(off + (int64_t)sizeof(T) * (int64_t)(n), M3_SLAB_ALIGN);
#define M3_X_BODY(T, name) M3_X_OFF(T, name, bodyCap)
#define M3_X_SHAPE(T, name) M3_X_OFF(T, name, shapeCap)
#define M3_X_JOINT(T, name) M3_X_OFF(T, name, jointCap)
#define M3_X_PAIR(T, name) M3_X_OFF(T, name, pairCap)
#define M3_X_TREE(T, name) M3_X_OFF(T, name, 2 * (int64_t)shapeCap)
    M3_BODY_FIELDS(M3_X_BODY)
    M3_SHAPE_FIELDS(M3_X_SHAPE)
    M3_JOINT_FIELDS(M3_X_JOINT)
    M3_TREE_FIELDS(M3_X_TREE)
    // The pair buffers start on a fresh 4 KiB page: the host pages before
    // them are page-locked for uploads, and a copy must not straddle the
    // locked and unlocked parts.
    off = m3AlignUp(off, M3_PAIR_SECTION_ALIGN);
    M3_PAIR_FIELDS(M3_X_PAIR)
#undef M3_X_BODY
#undef M3_X_SHAPE
#undef M3_X_JOINT
#undef M3_X_PAIR
#undef M3_X_TREE
#undef M3_X_OFF
    return off;
}

// Bytes of device scratch one world needs (implemented by the step
// module, which owns the scratch record layouts).
#ifdef __cplusplus
extern "C" {
#endif
int64_t m3gpuScratchBytes(int32_t bodyCap, int32_t shapeCap, int32_t jointCap, int32_t pairCap);
#ifdef __cplusplus
}
#endif

#endif // M3_LAYOUT_H
