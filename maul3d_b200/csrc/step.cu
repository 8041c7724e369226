// The device step: m3StepInternal (src/solver.c:3662-4320) for a batch
// of independent worlds, one thread block per world.
//
// Launches per step:
//   m3BroadKernel        one block per world: fresh bounds, sort-and-sweep
//                        and the canonical (sorted) pair list;
//   m3PairOffsetsKernel  prefix of the worlds' pair counts;
//   m3FamilyCount/ScatterKernel  bucket the batch's flattened pairs by
//                        pair family;
//   m3NarrowFamilyKernel<F>  one per covered family, one thread per pair
//                        of its bucket: the narrowphase with the
//                        warm-start carry (m3NarrowKernel, all families
//                        in one, serves the single-world path);
//   m3PrepareKernel      one block per world: islands and wake, contact
//                        selection, graph colouring, contact rows written
//                        into their solve slots, joint rows and their
//                        dependency levels, movers;
//   m3SubstepKernel      one block per world: the substep loop (integrate,
//                        warm start, colour-by-colour solve, integrate
//                        positions, relax) with body velocities in shared
//                        memory, restitution and the impulse store;
//   m3FinishKernel       one block per world: the continuous pass against
//                        planes, the sleep pass and the step counter.
// Block barriers separate every dependent phase, so inside a world the
// order of every write is the reference's; across worlds nothing is
// shared.  Worlds are ordered largest first so the long worlds start
// first (greedy longest-processing-time packing onto the SMs).
//
// Refusals: a world that needs something this path does not implement
// (a pair family, rolling resistance on a static contact, a bullet, a
// breakable joint, ...) or whose pair list would exceed its capacity gets
// its status word set and is skipped by every later kernel; the host
// reports it and the world stays failed.

#include "m3_world.h"
#include "m3_hash.h"
#include "m3_narrow.cuh"
#include "m3_solver.cuh"
#include "m3_joints.cuh"
#include "m3_tree.h"
#include "m3_ops.h"
#include "m3_toi.cuh"

#include <cuda_runtime.h>

#include <string.h>

#include <algorithm>
#include <vector>

#define M3_BLOCK 256
// Planes a world may hold (the broadphase enumerates their pairs
// directly; more are refused).
#define M3_MAX_PLANES 16
// The wide kernels' grid: at most this many blocks, and the layout of the
// wide prepare kernel's grid-shared words.
#define M3_WIDE_MAX_BLOCKS 512
#define M3_WW_FLAG 0        // 3 words: the colouring rounds' pending flags (round % 3)
#define M3_WW_LEVELS 3      // joint levels
#define M3_WW_CLEVELS 4     // contact levels
#define M3_WW_JFLAG 5       // 3 words: the joint-level rounds' change flags (round % 3)
#define M3_WW_BROKEN 8      // broken joints this step
#define M3_WW_PART 32       // M3_WIDE_MAX_BLOCKS + 1 words: the grid scan's block totals
#define M3_WW_BLOCKCOLOR (M3_WW_PART + M3_WIDE_MAX_BLOCKS + 1)
#define M3_WW_WORDS (M3_WW_BLOCKCOLOR + M3_WIDE_MAX_BLOCKS * (M3_GRAPH_COLORS + 1))
// Colouring: the marker of a constraint not coloured yet, and the
// parallel rounds before the serial finish (one block per world; a wide
// world's grid affords many more rounds).
#define M3_COLOR_PENDING 0xFF
#define M3_COLOR_ROUNDS 64
#define M3_WIDE_COLOR_ROUNDS 4096
// Rounds of the wide joint-level relaxation before the serial walk.
#define M3_WIDE_JOINT_ROUNDS 4096

// Step phases timed with the SM clock by thread 0 of each world's block
// right after the barrier that closes the phase.
enum
{
    M3_PHASE_ISLANDS = 0,
    M3_PHASE_PREPARE = 1,
    M3_PHASE_COLOR = 2,
    M3_PHASE_INTEGRATE_V = 3,
    M3_PHASE_WARM = 4,
    M3_PHASE_SOLVE = 5,
    M3_PHASE_INTEGRATE_P = 6,
    M3_PHASE_RELAX = 7,
    M3_PHASE_STORE = 8,
    M3_PHASE_CONTINUOUS = 9,
    M3_PHASE_SLEEP = 10,
    M3_PHASE_BOUNDS = 11,
    M3_PHASE_SORT = 12,
    M3_PHASE_COUNT = 13,
    M3_PHASE_FILL = 14,
};

#define M3_PHASE_MARK(k)                                                                           \
    if (threadIdx.x == 0)                                                                          \
    {                                                                                              \
        long long now_ = clock64();                                                                \
        sc->phase[k] += (uint64_t)(now_ - t_phase);                                                \
        t_phase = now_;                                                                            \
    }

// ---------------------------------------------------------------------
// Scratch layout (device only)
// ---------------------------------------------------------------------
// What the preparation kernel hands the substep and finish kernels.
struct m3StepPlan
{
    int32_t constraintCount;
    int32_t jointCount;
    int32_t jointLevels;
    int32_t moverCount;
    int32_t anyRestitution;
    int32_t levels; // joint/contact schedule levels; levelStart[levels] starts the overflow
    int32_t starts[M3_GRAPH_COLORS + 2]; // colour sizes (as offsets) of the colouring
};

struct m3Scratch
{
    m3Aabb* aabb;          // per shape
    int32_t* rowCount;     // per shape: pair count, then row offsets
    int32_t* rowFill;      // per shape: row fill cursor
    int32_t* planeFlag;    // per shape: plane row scan
    uint64_t* sortKey;     // sweep order keys (power-of-two padded)
    int32_t* sortIdx;      // sweep order shape indices
    uint64_t* sweepPairs;  // per pair: the sweep's pair keys, in discovery order
    m3Pos3* com0;          // per body
    m3Quat* rot0;          // per body
    int32_t* parent;       // per body (island union-find)
    int32_t* forced;       // per body
    int32_t* forcedRoot;   // per body
    int32_t* ready;        // per body
    m3Vec3* deltaPos;      // per body
    m3Quat* deltaRot;      // per body
    m3Mat3* bodyInvI;      // per body: prepare-time world inverse inertia
    int32_t* movers;       // per body
    int32_t* moverFlag;    // per body
    uint32_t* bodyMask;    // per body
    int32_t* colorMin;     // 2 per body: colouring round claims
    m3StepPlan* plan;      // counts and offsets handed between the step kernels
    m3ConRows rows;        // contact rows, field-major, one slot per constraint
    int32_t* conPairIndex; // per constraint: its pair
    int32_t* conSlot;      // per constraint: its solve slot
    int32_t* conLevel;     // per constraint: its level in the joint/contact schedule
    int32_t* levelStart;   // level offsets into the solve slots (+ the overflow bucket)
    int32_t* levelFill;    // level fill cursors
    int32_t* pairFlag;     // per pair (compaction)
    uint8_t* colors;       // per pair
    int2* conPair;         // per pair: colouring body pair
    int32_t* lists;        // per pair
    int32_t* starts;       // M3_GRAPH_COLORS + 2
    m3JointDev* joints;    // per joint row
    int32_t* jointFlag;    // per joint (selection scan)
    int32_t* jointLevel;   // per joint row: dependency level
    int32_t* jointOrder;   // joint rows grouped by level
    int32_t* jointLevelStart; // level offsets into jointOrder
    int32_t* treeMove;     // per shape: leaf-escape flags, then their scan
    m3Aabb* leafBox;       // per shape: its tree leaf's bounds (kept by the broadphase)
    int32_t* hasLeaf;      // per shape: whether it has a tree leaf
    int32_t* treeMoveCount; // M3_TREE_LAG: moves of each step in the ring
    int32_t* treeMoveShape; // M3_TREE_LAG x shapeCap: a step's moves (shapes, ascending)
    m3Aabb* treeMoveBox;   // M3_TREE_LAG x shapeCap: the fat bounds they are inserted with
    uint32_t* gridBar;     // 4 words: the wide kernels' grid barrier (count, generation, error)
    int32_t* staticList;   // per shape: static-target flags, then their scan
    int32_t* targetList;   // the continuous phase's static targets, ascending
    int2* jointBodies;     // per joint row: its two bodies (the level walk's compact input)
    int32_t* broadState;   // 20 words: a wide world's broadphase between its kernels
    int32_t* wideWork;     // the wide prepare kernel's grid-shared words (M3_WW_*)
    int32_t* jointAdj;     // 2 per joint row: rows by body (the wide joint levels)
    int2* jointPrev;       // per joint row: the previous row on each of its bodies
    uint8_t* hitFlag;      // per contact constraint: whether the step left a hit event
    m3HitEvent* hits;      // per contact constraint: that event (world index 0)
    m3Transform* xfPre;    // per body: its end pose before a continuous pull-back
    uint8_t* pulled;       // per body: whether the continuous phase pulled it back
};

static __host__ __device__ inline int64_t NextPow2(int64_t n)
{
    int64_t p = 1;
    while (p < n)
    {
        p <<= 1;
    }
    return p;
}

// The ring of tree move lists comes last and is `treeLag` steps deep:
// only the kernels that touch it need the depth the scratch was sized
// with; for every other array the offsets do not depend on it.
static __host__ __device__ inline int64_t ScratchCarve(m3Scratch* s, uint8_t* base, int32_t bodyCap,
                                                     int32_t shapeCap, int32_t jointCap,
                                                     int32_t pairCap, int32_t treeLag = 1)
{
    int64_t off = 0;
#define M3_CARVE(field, T, n)                                                                      \
    if (s)                                                                                         \
    {                                                                                              \
        s->field = (T*)(base + off);                                                               \
    }                                                                                              \
    off = m3AlignUp(off + (int64_t)sizeof(T) * (int64_t)(n), M3_SLAB_ALIGN);
    M3_CARVE(aabb, m3Aabb, shapeCap)
    M3_CARVE(rowCount, int32_t, shapeCap + 1)
    M3_CARVE(rowFill, int32_t, shapeCap + 1)
    M3_CARVE(planeFlag, int32_t, shapeCap + 1)
    M3_CARVE(sortKey, uint64_t, NextPow2(shapeCap))
    M3_CARVE(sortIdx, int32_t, NextPow2(shapeCap))
    M3_CARVE(sweepPairs, uint64_t, pairCap)
    M3_CARVE(com0, m3Pos3, bodyCap)
    M3_CARVE(rot0, m3Quat, bodyCap)
    M3_CARVE(parent, int32_t, bodyCap)
    M3_CARVE(forced, int32_t, bodyCap)
    M3_CARVE(forcedRoot, int32_t, bodyCap)
    M3_CARVE(ready, int32_t, bodyCap)
    M3_CARVE(deltaPos, m3Vec3, bodyCap)
    M3_CARVE(deltaRot, m3Quat, bodyCap)
    M3_CARVE(bodyInvI, m3Mat3, bodyCap)
    M3_CARVE(movers, int32_t, bodyCap)
    M3_CARVE(moverFlag, int32_t, bodyCap + 1)
    M3_CARVE(bodyMask, uint32_t, bodyCap)
    M3_CARVE(colorMin, int32_t, 2 * (int64_t)bodyCap)
    M3_CARVE(plan, m3StepPlan, 1)
    const int32_t rowStride = (int32_t)m3AlignUp(pairCap, 32);
    if (s)
    {
        s->rows.stride = rowStride;
    }
    M3_CARVE(rows.ro, float, (int64_t)M3C_WORDS * rowStride)
    M3_CARVE(rows.acc, float, (int64_t)M3A_WORDS * rowStride)
    M3_CARVE(conPairIndex, int32_t, pairCap)
    M3_CARVE(conSlot, int32_t, pairCap)
    M3_CARVE(conLevel, int32_t, pairCap)
    M3_CARVE(levelStart, int32_t, (int64_t)jointCap + M3_GRAPH_COLORS + 3)
    M3_CARVE(levelFill, int32_t, (int64_t)jointCap + M3_GRAPH_COLORS + 3)
    M3_CARVE(pairFlag, int32_t, pairCap + 1)
    M3_CARVE(colors, uint8_t, pairCap)
    M3_CARVE(conPair, int2, pairCap)
    M3_CARVE(lists, int32_t, pairCap)
    M3_CARVE(starts, int32_t, M3_GRAPH_COLORS + 2)
    M3_CARVE(joints, m3JointDev, jointCap)
    M3_CARVE(jointFlag, int32_t, jointCap + 1)
    M3_CARVE(jointLevel, int32_t, jointCap)
    M3_CARVE(jointOrder, int32_t, jointCap)
    M3_CARVE(jointLevelStart, int32_t, jointCap + 2)
    M3_CARVE(treeMove, int32_t, shapeCap + 1)
    M3_CARVE(leafBox, m3Aabb, shapeCap)
    M3_CARVE(hasLeaf, int32_t, shapeCap)
    M3_CARVE(treeMoveCount, int32_t, M3_TREE_LAG)
    M3_CARVE(gridBar, uint32_t, 4)
    M3_CARVE(staticList, int32_t, shapeCap + 1)
    M3_CARVE(targetList, int32_t, shapeCap)
    M3_CARVE(jointBodies, int2, jointCap)
    M3_CARVE(broadState, int32_t, 4 + M3_MAX_PLANES)
    M3_CARVE(wideWork, int32_t, M3_WW_WORDS)
    M3_CARVE(jointAdj, int32_t, 2 * (int64_t)jointCap)
    M3_CARVE(jointPrev, int2, jointCap)
    M3_CARVE(hitFlag, uint8_t, pairCap)
    M3_CARVE(hits, m3HitEvent, pairCap)
    M3_CARVE(xfPre, m3Transform, bodyCap)
    M3_CARVE(pulled, uint8_t, bodyCap)
    M3_CARVE(treeMoveBox, m3Aabb, (int64_t)treeLag * shapeCap)
    M3_CARVE(treeMoveShape, int32_t, (int64_t)treeLag * shapeCap)
#undef M3_CARVE
    return off;
}

extern "C" int64_t m3gpuScratchBytes(int32_t bodyCap, int32_t shapeCap, int32_t jointCap,
                                     int32_t pairCap)
{
    return ScratchCarve(nullptr, nullptr, bodyCap, shapeCap, jointCap, pairCap, M3_TREE_LAG);
}

// ---------------------------------------------------------------------
// Block utilities
// ---------------------------------------------------------------------

// Exclusive prefix sum of a[0, n) in place; returns the total.  Each
// thread scans a contiguous chunk, chunk totals are scanned in shared
// memory.  Must be called by every thread of the block.
template <int NT> __device__ int32_t BlockExclusiveScan(int32_t* a, int32_t n)
{
    __shared__ int32_t warpSums[NT / 32];
    __shared__ int32_t total;
    const int32_t t = threadIdx.x;
    const int32_t lane = t & 31;
    const int32_t warp = t >> 5;
    const int32_t chunk = (n + NT - 1) / NT;
    const int32_t lo = t * chunk < n ? t * chunk : n;
    const int32_t hi = lo + chunk < n ? lo + chunk : n;
    int32_t sum = 0;
    for (int32_t i = lo; i < hi; ++i)
    {
        sum += a[i];
    }
    // Inclusive scan of the chunk sums across the warp, then across the
    // warps' totals.
    int32_t x = sum;
    for (int32_t o = 1; o < 32; o <<= 1)
    {
        int32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o)
        {
            x += y;
        }
    }
    if (lane == 31)
    {
        warpSums[warp] = x;
    }
    __syncthreads();
    if (warp == 0)
    {
        int32_t v = lane < NT / 32 ? warpSums[lane] : 0;
        int32_t inc = v;
        for (int32_t o = 1; o < 32; o <<= 1)
        {
            int32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
            if (lane >= o)
            {
                inc += y;
            }
        }
        if (lane < NT / 32)
        {
            warpSums[lane] = inc - v;
        }
        if (lane == NT / 32 - 1)
        {
            total = inc;
        }
    }
    __syncthreads();
    int32_t run = warpSums[warp] + (x - sum);
    for (int32_t i = lo; i < hi; ++i)
    {
        int32_t y = a[i];
        a[i] = run;
        run += y;
    }
    __syncthreads();
    return total;
}

// ---------------------------------------------------------------------
// Broadphase (broad_phase.c:22-215, :641-681)
// ---------------------------------------------------------------------

// Fresh bounds of one shape, tight plus the margin (broad_phase.c:22-135).
__device__ __forceinline__ m3Aabb ShapeBounds(const m3WorldView& w, int32_t shape)
{
    return m3ShapeFreshBounds(w, shape);
}

__device__ __forceinline__ bool Overlap(const m3Aabb& a, const m3Aabb& b)
{
    return a.lo[0] <= b.hi[0] && b.lo[0] <= a.hi[0] && a.lo[1] <= b.hi[1] && b.lo[1] <= a.hi[1] &&
           a.lo[2] <= b.hi[2] && b.lo[2] <= a.hi[2];
}

// The shared pair filter (broad_phase.c:182-230).
__device__ bool PairAllowed(const m3WorldView& w, int32_t i, int32_t j)
{
    int32_t bodyI = w.shapeBody[i];
    int32_t bodyJ = w.shapeBody[j];
    if (bodyI == bodyJ)
    {
        return false;
    }
    if (w.enabled[bodyI] == 0 || w.enabled[bodyJ] == 0)
    {
        return false;
    }
    if (w.btype[bodyI] == M3_BODY_STATIC && w.btype[bodyJ] == M3_BODY_STATIC)
    {
        return false;
    }
    if (w.sensor[i] != 0 && w.sensor[j] != 0)
    {
        return false;
    }
    int32_t gi = w.group[i];
    if (gi != 0 && gi == w.group[j])
    {
        if (gi < 0)
        {
            return false;
        }
    }
    else if (!((w.category[i] & w.mask[j]) != 0 && (w.category[j] & w.mask[i]) != 0))
    {
        return false;
    }
    for (int32_t jt = w.jointHead[bodyI]; jt != -1;
         jt = w.jbodyA[jt] == bodyI ? w.jnextA[jt] : w.jnextB[jt])
    {
        int32_t other = w.jbodyA[jt] == bodyI ? w.jbodyB[jt] : w.jbodyA[jt];
        if (other == bodyJ && w.jcollide[jt] == 0)
        {
            return false;
        }
    }
    return true;
}

// ---------------------------------------------------------------------
// Kernel 1: fresh bounds and the canonical pair list (one block per
// world).  Sort-and-sweep on the x lower bound finds every overlapping
// non-plane pair exactly once; plane pairs are enumerated directly.
// Each pair lands in the row of its smaller shape index; rows are then
// ordered by the larger index, which yields the reference's ascending
// key order (broad_phase.c:632-637) without a global sort.
// ---------------------------------------------------------------------

// Total order on doubles as unsigned integers (negative values flipped).
__device__ __forceinline__ uint64_t OrderKey(double x)
{
    uint64_t b = (uint64_t)__double_as_longlong(x);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}


// The broadphase tree's leaves as the broadphase reads them: each
// shape's leaf bounds, copied out of the tree once per batch; the
// broadphase keeps the copy current as it moves leaves, so its
// containment tests never wait for the tree kernel.
__global__ void __launch_bounds__(M3_BLOCK) m3LeafBoxKernel(const m3WorldView* views,
                                                           int32_t count)
{
    const m3WorldView& w = views[blockIdx.x];
    const m3WorldScalars* sc = w.sc;
    m3Scratch s;
    ScratchCarve(&s, w.scratch, sc->bodyCap, sc->shapeCap, sc->jointCap, sc->pairCap);
    const int32_t shapeMax = sc->shapeMax;
    for (int32_t i = threadIdx.x; i < shapeMax; i += blockDim.x)
    {
        const int32_t leaf = w.proxyId[i];
        s.hasLeaf[i] = leaf != M3_TREE_NULL ? 1 : 0;
        if (leaf != M3_TREE_NULL)
        {
            const m3TreeNode& n = w.treeNodes[leaf];
            m3Aabb b;
            for (int32_t k = 0; k < 3; ++k)
            {
                b.lo[k] = n.lo[k];
                b.hi[k] = n.hi[k];
            }
            s.leafBox[i] = b;
        }
    }
}

// Broadphase tree refresh, second half (broad_phase.c:516-538): one warp
// per world replays one step's moves in ascending shape order, each a
// leaf removal and the insertion of its fat bounds; the warp's lanes
// prefetch the world's nodes into L2, lane 0 walks.  (One lane per world,
// 32 worlds to a warp, measured several times slower: the worlds' walks
// diverge and their dependent loads serialise.)  The tree is state only a
// snapshot reads, so this runs on its own stream beside the following
// steps, each world up to M3_TREE_LAG steps behind (the move lists sit in
// a ring of that depth).
// One step's leaf moves of one world, replayed by lane 0 (the lanes
// have prefetched the world's nodes).
__device__ void m3ReplayTreeStep(const m3WorldView& w, const m3Scratch& s, int32_t slot,
                                 int32_t moves)
{
    m3WorldScalars* sc = w.sc;
    const m3TreeRef tree = m3WorldTree(w);
    // Observer only: leaf moves replayed, in the phase counters' spare
    // slot (a count, not cycles).
    sc->phase[15] += (uint64_t)moves;
    const m3TreeArrayStore store{w.treeNodes};
    const int32_t* shapes = s.treeMoveShape + (int64_t)slot * sc->shapeCap;
    const m3Aabb* boxes = s.treeMoveBox + (int64_t)slot * sc->shapeCap;
    const int32_t shapeMax = sc->shapeMax;
    const int32_t nodeCap = 2 * sc->shapeCap;
    for (int32_t m = 0; m < moves; ++m)
    {
        const int32_t shape = shapes[m];
        const m3Aabb box = boxes[m];
        const int32_t old = shape >= 0 && shape < shapeMax ? w.proxyId[shape] : M3_TREE_NULL;
        if (old == M3_TREE_NULL || old < 0 || old >= nodeCap)
        {
            // Only shapes with a leaf are ever recorded as moves.
            atomicExch(&sc->status, M3GPU_ERR_INVALID);
            sc->statusDetail = 6001;
            return;
        }
        m3TreeRemove(tree, store, old);
        const int32_t leaf = m3TreeInsert(tree, store, box.lo, box.hi, shape);
        w.proxyId[shape] = leaf;
        if (leaf == M3_TREE_NULL)
        {
            // The reference's pair update refuses with m3_errorCapacity.
            atomicExch(&sc->status, M3GPU_ERR_CAPACITY);
            return;
        }
    }
}

// The replay of each world's oldest `steps[world]` recorded steps (the
// world's index in `views`), in the order the broadphase recorded them.
__global__ void __launch_bounds__(32)
    m3TreeKernel(const m3WorldView* views, const int32_t* order, int32_t count, int32_t treeLag,
                 const int32_t* steps)
{
    const int32_t k = blockIdx.x;
    const int32_t lane = (int32_t)threadIdx.x;
    if (k >= count)
    {
        return;
    }
    const int32_t wi = order[k];
    const int32_t n = steps[wi];
    const m3WorldView& w = views[wi];
    m3WorldScalars* sc = w.sc;
    if (sc->treeTracked == 0 || n <= 0)
    {
        return;
    }
    m3Scratch s;
    ScratchCarve(&s, w.scratch, sc->bodyCap, sc->shapeCap, sc->jointCap, sc->pairCap, treeLag);
    const int32_t tail = sc->treeTail;
    __syncwarp();
    if (lane == 0)
    {
        sc->treeTail = tail + n;
    }
    // A refused world's tree is not kept (its state is unspecified after
    // a refusal).
    if (sc->status != 0)
    {
        return;
    }
    // The walk below is a chain of dependent loads: bring the world's
    // nodes into L2 first, one bulk prefetch per 64 KiB piece (the array
    // is 256-byte aligned and 144 bytes a shape, so every piece is a
    // multiple of 16 bytes).
    {
        const int64_t bytes = (int64_t)sizeof(m3TreeNode) * 2 * sc->shapeCap;
        const uint8_t* base = (const uint8_t*)w.treeNodes;
        for (int64_t off = (int64_t)lane << 16; off < bytes; off += (int64_t)32 << 16)
        {
            const int64_t left = bytes - off;
            const uint32_t piece = (uint32_t)(left < 65536 ? left : 65536);
            asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(base + off), "r"(piece)
                         : "memory");
        }
    }
    if (lane != 0)
    {
        return;
    }
    for (int32_t i = 0; i < n; ++i)
    {
        const int32_t slot = (int32_t)((uint32_t)(tail + i) % (uint32_t)treeLag);
        const int32_t moves = s.treeMoveCount[slot];
        // A move count above the shape slots cannot come from this
        // world's broadphase.
        if (moves > 0 && moves <= sc->shapeMax)
        {
            m3ReplayTreeStep(w, s, slot, moves);
        }
        if (sc->status != 0)
        {
            return;
        }
    }
}

// Visit every non-plane pair (a < b) whose fresh bounds overlap and that
// the filter allows, from the sweep position `p` of the sorted order.
template <typename F>
__device__ __forceinline__ void SweepFrom(const m3WorldView& w, const m3Scratch& s, int32_t p,
                                          int32_t n, F&& visit)
{
    const int32_t a = s.sortIdx[p];
    const m3Aabb boxA = s.aabb[a];
    for (int32_t q = p + 1; q < n; ++q)
    {
        const int32_t b = s.sortIdx[q];
        const m3Aabb& boxB = s.aabb[b];
        if (!(boxB.lo[0] <= boxA.hi[0]))
        {
            break;
        }
        if (Overlap(boxA, boxB))
        {
            int32_t lo = a < b ? a : b;
            int32_t hi = a < b ? b : a;
            if (PairAllowed(w, lo, hi))
            {
                visit(lo, hi);
            }
        }
    }
}

// Rows longer than this are ordered by the whole block (at most
// M3_LONG_ROWS of them per world per step; any further ones by their
// thread).
#define M3_LONG_ROW 64
#define M3_LONG_ROWS 16

// PART 0 is the whole broadphase of one world per block.  A wide world
// splits it around the sweep: PART 1 (bounds, tree moves, sort; one
// block) leaves the plane list and the sweep count in s.broadState,
// m3WideSweepKernel counts and records the pairs over the whole grid,
// PART 2 (scan, fill, row order; one block) finishes.
#define M3_BS_PLANES 0
#define M3_BS_SWEEP 1
#define M3_BS_PAIRS 2
#define M3_BS_PLANE0 4
template <int NT, int MIN_BLOCKS, int PART = 0>
__global__ void __launch_bounds__(NT, MIN_BLOCKS) m3BroadKernel(const m3WorldView* views,
                                                          const int32_t* order, int32_t count,
                                                          int32_t treeLag)
{
    const int32_t wi = order[blockIdx.x];
    const m3WorldView& w = views[wi];
    m3WorldScalars* sc = w.sc;
    m3Scratch s;
    ScratchCarve(&s, w.scratch, sc->bodyCap, sc->shapeCap, sc->jointCap, sc->pairCap, treeLag);
    const int32_t tid = threadIdx.x;
    __shared__ int32_t s_status;
    __shared__ int32_t s_planes[M3_MAX_PLANES];
    __shared__ int32_t s_planeCount;
    __shared__ int32_t s_sweepCount;
    __shared__ int32_t s_sweepPairs;
    __shared__ int32_t s_treeSlot;
    if (tid == 0)
    {
        s_status = sc->status;
        s_planeCount = 0;
        s_sweepCount = 0;
        s_sweepPairs = 0;
        // A world that keeps the tree records one ring slot per step, read
        // back by exactly one tree launch.  No moves are recorded unless
        // this step reaches the containment tests below: the tree kernel
        // must never replay a slot (or scratch shared with another world)
        // left by an older step.
        int32_t slot = 0;
        if (PART != 2 && sc->treeTracked != 0)
        {
            slot = (int32_t)((uint32_t)sc->treeHead % (uint32_t)treeLag);
            sc->treeHead += 1;
            s.treeMoveCount[slot] = 0;
        }
        s_treeSlot = slot;
        if (PART == 1)
        {
            // The wide kernels of this step start their grid barrier
            // with no arrivals and no error.
            s.gridBar[0] = 0;
            s.gridBar[2] = 0;
        }
        if (PART == 2 && s_status == 0)
        {
            s_planeCount = s.broadState[M3_BS_PLANES];
            s_sweepPairs = s.broadState[M3_BS_PAIRS];
            for (int32_t k = 0; k < s_planeCount && k < M3_MAX_PLANES; ++k)
            {
                s_planes[k] = s.broadState[M3_BS_PLANE0 + k];
            }
        }
    }
    __syncthreads();
    const int32_t treeSlot = s_treeSlot;
    if (s_status != 0)
    {
        return;
    }
    long long t_phase = clock64();
    const int32_t shapeMax = sc->shapeMax;
    if (PART != 2)
    {

    // Fresh bounds once per shape; the sweep set and the plane list.
    for (int32_t i = tid; i < shapeMax; i += NT)
    {
        s.rowCount[i] = 0;
        s.rowFill[i] = 0;
        if (w.shapeAlive[i] == 0)
        {
            continue;
        }
        if (w.shapeType[i] == M3_SHAPE_PLANE)
        {
            int32_t k = atomicAdd(&s_planeCount, 1);
            if (k < M3_MAX_PLANES)
            {
                s_planes[k] = i;
            }
            continue;
        }
        s.aabb[i] = ShapeBounds(w, i);
        int32_t k = atomicAdd(&s_sweepCount, 1);
        s.sortIdx[k] = i;
    }
    __syncthreads();
    if (s_planeCount > M3_MAX_PLANES)
    {
        if (tid == 0)
        {
            sc->status = M3GPU_ERR_UNSUPPORTED;
            sc->statusDetail = 5001;
        }
        return;
    }
    // Broadphase tree refresh, first half (broad_phase.c:500-539): the
    // awake shapes whose fresh bounds left their leaf, ascending, with
    // the fat bounds they are reinserted with.  A leaf moves only when
    // its own shape is reinserted, so every containment test can run
    // here at once; m3TreeKernel replays the moves in order.
    const bool tracked = sc->treeTracked != 0;
    for (int32_t i = tid; i < shapeMax; i += NT)
    {
        int32_t move = 0;
        if (tracked && w.shapeAlive[i] != 0 && s.hasLeaf[i] != 0 && w.awake[w.shapeBody[i]] != 0)
        {
            const m3Aabb& leaf = s.leafBox[i];
            const m3Aabb& b = s.aabb[i];
            move = leaf.lo[0] <= b.lo[0] && leaf.lo[1] <= b.lo[1] && leaf.lo[2] <= b.lo[2] &&
                           b.hi[0] <= leaf.hi[0] && b.hi[1] <= leaf.hi[1] && b.hi[2] <= leaf.hi[2]
                       ? 0
                       : 1;
        }
        s.treeMove[i] = move;
    }
    __syncthreads();
    const int32_t treeMoves = BlockExclusiveScan<NT>(s.treeMove, shapeMax);
    int32_t* moveShape = s.treeMoveShape + (int64_t)treeSlot * sc->shapeCap;
    m3Aabb* moveBox = s.treeMoveBox + (int64_t)treeSlot * sc->shapeCap;
    for (int32_t i = tid; i < shapeMax; i += NT)
    {
        const int32_t at = s.treeMove[i];
        const int32_t next = i + 1 < shapeMax ? s.treeMove[i + 1] : treeMoves;
        if (next != at)
        {
            m3Aabb fat = s.aabb[i];
            for (int32_t k = 0; k < 3; ++k)
            {
                fat.lo[k] -= (double)M3_AABB_MARGIN;
                fat.hi[k] += (double)M3_AABB_MARGIN;
            }
            moveShape[at] = i;
            moveBox[at] = fat;
            s.leafBox[i] = fat;
        }
    }
    if (tid == 0)
    {
        s.treeMoveCount[treeSlot] = treeMoves;
    }
    M3_PHASE_MARK(M3_PHASE_BOUNDS)
    const int32_t n = s_sweepCount;
    int32_t pow2 = 1;
    while (pow2 < n)
    {
        pow2 <<= 1;
    }
    for (int32_t i = tid; i < pow2; i += NT)
    {
        if (i < n)
        {
            s.sortKey[i] = OrderKey(s.aabb[s.sortIdx[i]].lo[0]);
        }
        else
        {
            s.sortKey[i] = ~0ull;
            s.sortIdx[i] = 0x7FFFFFFF;
        }
    }
    __syncthreads();
    // Bitonic sort by (x lower bound, shape index).
    for (int32_t k = 2; k <= pow2; k <<= 1)
    {
        for (int32_t j = k >> 1; j > 0; j >>= 1)
        {
            for (int32_t i = tid; i < pow2; i += NT)
            {
                int32_t ixj = i ^ j;
                if (ixj > i)
                {
                    uint64_t ka = s.sortKey[i];
                    uint64_t kb = s.sortKey[ixj];
                    int32_t ia = s.sortIdx[i];
                    int32_t ib = s.sortIdx[ixj];
                    bool greater = ka > kb || (ka == kb && ia > ib);
                    bool ascending = (i & k) == 0;
                    if (greater == ascending)
                    {
                        s.sortKey[i] = kb;
                        s.sortKey[ixj] = ka;
                        s.sortIdx[i] = ib;
                        s.sortIdx[ixj] = ia;
                    }
                }
            }
            __syncthreads();
        }
    }

    M3_PHASE_MARK(M3_PHASE_SORT)
    if (PART == 1)
    {
        if (tid == 0)
        {
            s.broadState[M3_BS_PLANES] = s_planeCount;
            s.broadState[M3_BS_SWEEP] = n;
            s.broadState[M3_BS_PAIRS] = 0;
            for (int32_t k = 0; k < s_planeCount; ++k)
            {
                s.broadState[M3_BS_PLANE0 + k] = s_planes[k];
            }
        }
        return;
    }
    // Count every row's pairs; the sweep's pairs are recorded on the way
    // so the fill below need not sweep again.
    const int32_t planeCount = s_planeCount;
    const int32_t pairCap = sc->pairCap;
    for (int32_t p = tid; p < n; p += NT)
    {
        SweepFrom(w, s, p, n, [&](int32_t lo, int32_t hi) {
            atomicAdd(&s.rowCount[lo], 1);
            const int32_t r = atomicAdd(&s_sweepPairs, 1);
            if (r < pairCap)
            {
                s.sweepPairs[r] = ((uint64_t)(uint32_t)lo << 32) | (uint64_t)(uint32_t)hi;
            }
        });
    }
    for (int32_t i = tid; i < shapeMax; i += NT)
    {
        if (w.shapeAlive[i] == 0 || w.shapeType[i] == M3_SHAPE_PLANE)
        {
            continue;
        }
        for (int32_t k = 0; k < planeCount; ++k)
        {
            int32_t pl = s_planes[k];
            int32_t lo = pl < i ? pl : i;
            int32_t hi = pl < i ? i : pl;
            if (PairAllowed(w, lo, hi))
            {
                atomicAdd(&s.rowCount[lo], 1);
            }
        }
    }
    __syncthreads();
    }
    const int32_t planeCount = s_planeCount;
    const int32_t total = BlockExclusiveScan<NT>(s.rowCount, shapeMax);
    if (total > sc->pairCap)
    {
        // The reference's m3UpdatePairs refuses with m3_errorCapacity
        // and the step stalls (broad_phase.c:257-260, solver.c:3722).
        if (tid == 0)
        {
            sc->status = M3GPU_ERR_CAPACITY;
            sc->statusDetail = total;
        }
        return;
    }
    const int32_t cur = sc->pairBuf;
    uint64_t* newKeys = cur == 0 ? w.keys1 : w.keys0;
    {
        // The reference keeps one pair array: past the new list it still
        // holds what longer lists of earlier steps left there, and a
        // snapshot carries those bytes.  The old buffer agrees with it
        // past the old list and holds the old list itself, so the new
        // buffer takes [total, old count) from it.
        const int32_t oldCount = sc->pairCount;
        const uint64_t* oldKeys = cur == 0 ? w.keys0 : w.keys1;
        const m3Manifold* oldMan = cur == 0 ? w.man0 : w.man1;
        m3Manifold* newMan = cur == 0 ? w.man1 : w.man0;
        for (int32_t i = total + tid; i < oldCount; i += NT)
        {
            newKeys[i] = oldKeys[i];
            newMan[i] = oldMan[i];
        }
    }

    M3_PHASE_MARK(M3_PHASE_COUNT)
    // Fill rows: sweep pairs through per-row cursors, then each plane's
    // own row in ascending partner order by a scan.
    const int32_t swept = s_sweepPairs;
    for (int32_t r = tid; r < swept; r += NT)
    {
        const uint64_t key = s.sweepPairs[r];
        const int32_t lo = (int32_t)(key >> 32);
        const int32_t slot = atomicAdd(&s.rowFill[lo], 1);
        newKeys[s.rowCount[lo] + slot] = key;
    }
    for (int32_t i = tid; i < shapeMax; i += NT)
    {
        if (w.shapeAlive[i] == 0 || w.shapeType[i] == M3_SHAPE_PLANE)
        {
            continue;
        }
        for (int32_t k = 0; k < planeCount; ++k)
        {
            int32_t pl = s_planes[k];
            if (pl < i || !PairAllowed(w, i, pl))
            {
                continue;
            }
            int32_t slot = atomicAdd(&s.rowFill[i], 1);
            newKeys[s.rowCount[i] + slot] = ((uint64_t)(uint32_t)i << 32) | (uint64_t)(uint32_t)pl;
        }
    }
    for (int32_t k = 0; k < planeCount; ++k)
    {
        const int32_t pl = s_planes[k];
        __syncthreads();
        for (int32_t i = tid; i < shapeMax; i += NT)
        {
            s.planeFlag[i] = (i > pl && w.shapeAlive[i] != 0 && w.shapeType[i] != M3_SHAPE_PLANE &&
                              PairAllowed(w, pl, i))
                                 ? 1
                                 : 0;
        }
        __syncthreads();
        BlockExclusiveScan<NT>(s.planeFlag, shapeMax);
        const int32_t base = s.rowCount[pl];
        for (int32_t i = tid; i < shapeMax; i += NT)
        {
            int32_t next = i + 1 < shapeMax ? s.planeFlag[i + 1] : -1;
            bool flagged = i + 1 < shapeMax ? next != s.planeFlag[i]
                                            : (i > pl && w.shapeAlive[i] != 0 &&
                                               w.shapeType[i] != M3_SHAPE_PLANE &&
                                               PairAllowed(w, pl, i));
            if (flagged)
            {
                newKeys[base + s.planeFlag[i]] =
                    ((uint64_t)(uint32_t)pl << 32) | (uint64_t)(uint32_t)i;
            }
        }
    }
    // Order each non-plane row by partner index: a short row by one
    // thread's insertion sort; a long one (a heightfield's, or a large
    // static shape's, pairs with much of the world) by the whole block,
    // each key written at its rank (keys in a row are distinct).
    __shared__ int32_t s_longRows[M3_LONG_ROWS];
    __shared__ int32_t s_longCount;
    if (tid == 0)
    {
        s_longCount = 0;
    }
    __syncthreads();
    for (int32_t i = tid; i < shapeMax; i += NT)
    {
        if (w.shapeAlive[i] == 0 || w.shapeType[i] == M3_SHAPE_PLANE)
        {
            continue;
        }
        const int32_t a = s.rowCount[i];
        const int32_t c = s.rowFill[i];
        if (c > M3_LONG_ROW)
        {
            const int32_t slot = atomicAdd(&s_longCount, 1);
            if (slot < M3_LONG_ROWS)
            {
                s_longRows[slot] = i;
                continue;
            }
        }
        for (int32_t x = a + 1; x < a + c; ++x)
        {
            uint64_t key = newKeys[x];
            int32_t y = x - 1;
            while (y >= a && newKeys[y] > key)
            {
                newKeys[y + 1] = newKeys[y];
                y -= 1;
            }
            newKeys[y + 1] = key;
        }
    }
    __syncthreads();
    // The long rows; the sweep's pair list is spent and holds each row's
    // sorted copy (a row is no longer than the pair capacity).
    const int32_t longRows = s_longCount < M3_LONG_ROWS ? s_longCount : M3_LONG_ROWS;
    for (int32_t r = 0; r < longRows; ++r)
    {
        const int32_t a = s.rowCount[s_longRows[r]];
        const int32_t c = s.rowFill[s_longRows[r]];
        for (int32_t x = tid; x < c; x += NT)
        {
            const uint64_t key = newKeys[a + x];
            int32_t rank = 0;
            for (int32_t y = 0; y < c; ++y)
            {
                rank += newKeys[a + y] < key ? 1 : 0;
            }
            s.sweepPairs[rank] = key;
        }
        __syncthreads();
        for (int32_t x = tid; x < c; x += NT)
        {
            newKeys[a + x] = s.sweepPairs[x];
        }
        __syncthreads();
    }
    M3_PHASE_MARK(M3_PHASE_FILL)
    if (tid == 0)
    {
        sc->newPairCount = total;
    }
}

// A wide world's sweep (between m3BroadKernel PART 1 and PART 2): every
// sorted position sweeps its own candidates, as the per-world kernel's
// threads do, over the whole grid; row counts and the recorded pairs go
// through global atomics (the fill orders each row afterwards).
__global__ void __launch_bounds__(256) m3WideSweepKernel(const m3WorldView* views,
                                                        const int32_t* order)
{
    const m3WorldView& w = views[order[0]];
    m3WorldScalars* sc = w.sc;
    if (sc->status != 0)
    {
        return;
    }
    m3Scratch s;
    ScratchCarve(&s, w.scratch, sc->bodyCap, sc->shapeCap, sc->jointCap, sc->pairCap);
    const int32_t n = s.broadState[M3_BS_SWEEP];
    const int32_t planeCount = s.broadState[M3_BS_PLANES];
    const int32_t pairCap = sc->pairCap;
    const int32_t shapeMax = sc->shapeMax;
    const int32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int32_t gstride = gridDim.x * blockDim.x;
    int32_t* recorded = &s.broadState[M3_BS_PAIRS];
    for (int32_t p = gtid; p < n; p += gstride)
    {
        SweepFrom(w, s, p, n, [&](int32_t lo, int32_t hi) {
            atomicAdd(&s.rowCount[lo], 1);
            const int32_t r = atomicAdd(recorded, 1);
            if (r < pairCap)
            {
                s.sweepPairs[r] = ((uint64_t)(uint32_t)lo << 32) | (uint64_t)(uint32_t)hi;
            }
        });
    }
    for (int32_t i = gtid; i < shapeMax; i += gstride)
    {
        if (w.shapeAlive[i] == 0 || w.shapeType[i] == M3_SHAPE_PLANE)
        {
            continue;
        }
        for (int32_t k = 0; k < planeCount; ++k)
        {
            const int32_t pl = s.broadState[M3_BS_PLANE0 + k];
            const int32_t lo = pl < i ? pl : i;
            const int32_t hi = pl < i ? i : pl;
            if (PairAllowed(w, lo, hi))
            {
                atomicAdd(&s.rowCount[lo], 1);
            }
        }
    }
}

// Exclusive offsets of every world's new pair count, in batch order
// (one block; the narrowphase grid strides over the flattened pairs).
__global__ void m3PairOffsetsKernel(const m3WorldView* views, int32_t count, int32_t* offsets)
{
    __shared__ int32_t partial[M3_BLOCK];
    const int32_t t = threadIdx.x;
    const int32_t chunk = (count + M3_BLOCK - 1) / M3_BLOCK;
    const int32_t lo = t * chunk < count ? t * chunk : count;
    const int32_t hi = lo + chunk < count ? lo + chunk : count;
    int32_t sum = 0;
    for (int32_t i = lo; i < hi; ++i)
    {
        const m3WorldScalars* sc = views[i].sc;
        sum += sc->status == 0 ? sc->newPairCount : 0;
    }
    partial[t] = sum;
    __syncthreads();
    if (t == 0)
    {
        int32_t run = 0;
        for (int32_t k = 0; k < M3_BLOCK; ++k)
        {
            int32_t x = partial[k];
            partial[k] = run;
            run += x;
        }
        offsets[count] = run;
    }
    __syncthreads();
    int32_t run = partial[t];
    for (int32_t i = lo; i < hi; ++i)
    {
        offsets[i] = run;
        const m3WorldScalars* sc = views[i].sc;
        run += sc->status == 0 ? sc->newPairCount : 0;
    }
}

// ---------------------------------------------------------------------
// Kernel 2: the narrowphase and warm-start carry over the flattened
// pairs of every world of the batch, one thread per pair.
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(128) m3NarrowKernel(const m3WorldView* views,
                                                      const int32_t* offsets, int32_t count)
{
    const int32_t total = offsets[count];
    for (int32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < total;
         g += gridDim.x * blockDim.x)
    {
        // The world owning flattened pair g: last offset <= g.
        int32_t lo = 0;
        int32_t hi = count - 1;
        while (lo < hi)
        {
            int32_t mid = (lo + hi + 1) >> 1;
            if (offsets[mid] <= g)
            {
                lo = mid;
            }
            else
            {
                hi = mid - 1;
            }
        }
        const m3WorldView& w = views[lo];
        m3WorldScalars* sc = w.sc;
        const int32_t k = g - offsets[lo];
        const int32_t cur = sc->pairBuf;
        const uint64_t* oldKeys = cur == 0 ? w.keys0 : w.keys1;
        const m3Manifold* oldMan = cur == 0 ? w.man0 : w.man1;
        const uint64_t* newKeys = cur == 0 ? w.keys1 : w.keys0;
        m3Manifold* newMan = cur == 0 ? w.man1 : w.man0;
        const uint64_t key = newKeys[k];
        m3Manifold fresh;
        int32_t st = m3CollidePair(w, key, &fresh);
        if (st != M3_NARROW_OK)
        {
            atomicMax(&sc->status, M3GPU_ERR_UNSUPPORTED);
            sc->statusDetail = 1000 + (int32_t)w.shapeType[(int32_t)(key >> 32)] * 10 +
                               (int32_t)w.shapeType[(int32_t)(key & 0xFFFFFFFFu)];
        }
        m3WarmCarry(&fresh, key, oldKeys, oldMan, sc->pairCount, k);
        newMan[k] = fresh;
    }
}

// ---------------------------------------------------------------------
// Kernels 2b-2c: the batch's flattened pairs bucketed by pair family
// (m3PairFamily), so that each family's narrowphase runs as its own
// kernel over same-family warps.  A two-pass partition without global
// atomics: each block counts the families of a contiguous range of the
// flattened pairs, then scatters that range in order behind the counts
// of all earlier blocks; the buckets hold flattened pair indices.
// ---------------------------------------------------------------------
#define M3_FAMILY_BLOCKS 592
#define M3_FAMILY_THREADS 256

// The world owning flattened pair g: the last world whose offset <= g.
__device__ __forceinline__ int32_t FlatWorld(const int32_t* offsets, int32_t count, int32_t g)
{
    int32_t lo = 0;
    int32_t hi = count - 1;
    while (lo < hi)
    {
        const int32_t mid = (lo + hi + 1) >> 1;
        if (offsets[mid] <= g)
        {
            lo = mid;
        }
        else
        {
            hi = mid - 1;
        }
    }
    return lo;
}

__device__ __forceinline__ int32_t FlatFamily(const m3WorldView* views, const int32_t* offsets,
                                              int32_t count, int32_t g, int32_t* world)
{
    const int32_t wi = FlatWorld(offsets, count, g);
    const m3WorldView& w = views[wi];
    const uint64_t* newKeys = w.sc->pairBuf == 0 ? w.keys1 : w.keys0;
    const uint64_t key = newKeys[g - offsets[wi]];
    *world = wi;
    return m3PairFamily(w.shapeType[(int32_t)(key >> 32)],
                        w.shapeType[(int32_t)(key & 0xFFFFFFFFu)]);
}

__device__ __forceinline__ void FamilyRange(int32_t total, int32_t* lo, int32_t* hi)
{
    const int32_t chunk = (total + (int32_t)gridDim.x - 1) / (int32_t)gridDim.x;
    const int32_t a = (int32_t)blockIdx.x * chunk;
    *lo = a < total ? a : total;
    *hi = a + chunk < total ? a + chunk : total;
}

__global__ void __launch_bounds__(M3_FAMILY_THREADS)
    m3FamilyCountKernel(const m3WorldView* views, const int32_t* offsets, int32_t count,
                        int32_t* blockHist)
{
    __shared__ int32_t hist[M3F_COUNT];
    const int32_t tid = threadIdx.x;
    if (tid < M3F_COUNT)
    {
        hist[tid] = 0;
    }
    __syncthreads();
    int32_t lo;
    int32_t hi;
    FamilyRange(offsets[count], &lo, &hi);
    for (int32_t g = lo + tid; g < hi; g += M3_FAMILY_THREADS)
    {
        int32_t wi;
        const int32_t f = FlatFamily(views, offsets, count, g, &wi);
        if (f == M3F_UNSUPPORTED)
        {
            // A pair family the device does not cover: the world stalls.
            const m3WorldView& w = views[wi];
            const uint64_t* newKeys = w.sc->pairBuf == 0 ? w.keys1 : w.keys0;
            const uint64_t key = newKeys[g - offsets[wi]];
            atomicMax(&w.sc->status, M3GPU_ERR_UNSUPPORTED);
            w.sc->statusDetail = 1000 + (int32_t)w.shapeType[(int32_t)(key >> 32)] * 10 +
                                 (int32_t)w.shapeType[(int32_t)(key & 0xFFFFFFFFu)];
        }
        atomicAdd(&hist[f], 1);
    }
    __syncthreads();
    if (tid < M3F_COUNT)
    {
        blockHist[blockIdx.x * M3F_COUNT + tid] = hist[tid];
    }
}

__global__ void __launch_bounds__(M3_FAMILY_THREADS)
    m3FamilyScatterKernel(const m3WorldView* views, const int32_t* offsets, int32_t count,
                          const int32_t* blockHist, int32_t* famStart, int32_t* bucket)
{
    __shared__ int32_t base[M3F_COUNT];
    __shared__ int32_t total[M3F_COUNT];
    __shared__ int32_t warpCount[M3_FAMILY_THREADS / 32][M3F_COUNT];
    const int32_t tid = threadIdx.x;
    const int32_t lane = tid & 31;
    const int32_t warp = tid >> 5;
    if (tid < M3F_COUNT)
    {
        // Family totals over all blocks, and this family's pairs in the
        // blocks before this one.
        int32_t before = 0;
        int32_t all = 0;
        for (int32_t b = 0; b < (int32_t)gridDim.x; ++b)
        {
            const int32_t v = blockHist[b * M3F_COUNT + tid];
            before += b < (int32_t)blockIdx.x ? v : 0;
            all += v;
        }
        total[tid] = all;
        base[tid] = before;
    }
    __syncthreads();
    if (tid == 0)
    {
        int32_t start = 0;
        for (int32_t f = 0; f < M3F_COUNT; ++f)
        {
            if (blockIdx.x == 0)
            {
                famStart[f] = start;
            }
            base[f] += start;
            start += total[f];
        }
        if (blockIdx.x == 0)
        {
            famStart[M3F_COUNT] = start;
        }
    }
    __syncthreads();
    int32_t lo;
    int32_t hi;
    FamilyRange(offsets[count], &lo, &hi);
    const uint32_t ltMask = (1u << lane) - 1u;
    for (int32_t t0 = lo; t0 < hi; t0 += M3_FAMILY_THREADS)
    {
        const int32_t g = t0 + tid;
        int32_t f = M3F_COUNT; // past the range: no family
        if (g < hi)
        {
            int32_t wi;
            f = FlatFamily(views, offsets, count, g, &wi);
        }
        int32_t rank = 0;
#pragma unroll
        for (int32_t k = 0; k < M3F_COUNT; ++k)
        {
            const uint32_t b = __ballot_sync(0xFFFFFFFFu, f == k);
            if (f == k)
            {
                rank = __popc(b & ltMask);
            }
            if (lane == 0)
            {
                warpCount[warp][k] = __popc(b);
            }
        }
        __syncthreads();
        if (f < M3F_COUNT)
        {
            int32_t pos = base[f] + rank;
            for (int32_t k = 0; k < warp; ++k)
            {
                pos += warpCount[k][f];
            }
            bucket[pos] = g;
        }
        __syncthreads();
        if (tid < M3F_COUNT)
        {
            int32_t add = 0;
            for (int32_t k = 0; k < M3_FAMILY_THREADS / 32; ++k)
            {
                add += warpCount[k][tid];
            }
            base[tid] += add;
        }
        __syncthreads();
    }
}

// Kernel 2d: the narrowphase of one pair family over its bucket, with
// the warm-start carry.
template <int F>
__global__ void __launch_bounds__(128)
    m3NarrowFamilyKernel(const m3WorldView* views, const int32_t* offsets, int32_t count,
                         const int32_t* famStart, const int32_t* bucket)
{
    const int32_t end = famStart[F + 1];
    for (int32_t idx = famStart[F] + blockIdx.x * blockDim.x + threadIdx.x; idx < end;
         idx += gridDim.x * blockDim.x)
    {
        const int32_t g = bucket[idx];
        const int32_t wi = FlatWorld(offsets, count, g);
        const m3WorldView& w = views[wi];
        m3WorldScalars* sc = w.sc;
        const int32_t k = g - offsets[wi];
        const int32_t cur = sc->pairBuf;
        const uint64_t* oldKeys = cur == 0 ? w.keys0 : w.keys1;
        const m3Manifold* oldMan = cur == 0 ? w.man0 : w.man1;
        const uint64_t* newKeys = cur == 0 ? w.keys1 : w.keys0;
        m3Manifold* newMan = cur == 0 ? w.man1 : w.man0;
        const uint64_t key = newKeys[k];
        m3Manifold fresh;
        if (m3CollideFamily<F>(w, key, &fresh) != M3_NARROW_OK)
        {
            // A clip polygon beyond the device's bound: the world stalls.
            atomicMax(&sc->status, M3GPU_ERR_UNSUPPORTED);
            sc->statusDetail = 1000 + (int32_t)w.shapeType[(int32_t)(key >> 32)] * 10 +
                               (int32_t)w.shapeType[(int32_t)(key & 0xFFFFFFFFu)];
        }
        m3WarmCarry(&fresh, key, oldKeys, oldMan, sc->pairCount, k);
        newMan[k] = fresh;
    }
}

// ---------------------------------------------------------------------
// Islands (solver.c:3437-3578): a lock-free union-find whose links
// always point a root at a smaller root, so each component's final
// root is its smallest body index, the reference's "lower root wins".
// ---------------------------------------------------------------------
__device__ __forceinline__ int32_t IslandFind(int32_t* parent, int32_t i)
{
    while (true)
    {
        int32_t p = parent[i];
        if (p == i)
        {
            return i;
        }
        int32_t gp = parent[p];
        if (gp != p)
        {
            parent[i] = gp; // halving: gp is an ancestor of i
        }
        i = p;
    }
}

__device__ void IslandUnion(int32_t* parent, int32_t a, int32_t b)
{
    while (true)
    {
        a = IslandFind(parent, a);
        b = IslandFind(parent, b);
        if (a == b)
        {
            return;
        }
        if (a > b)
        {
            int32_t t = a;
            a = b;
            b = t;
        }
        int32_t old = atomicCAS(&parent[b], b, a);
        if (old == b)
        {
            return;
        }
        b = old;
    }
}

__device__ __forceinline__ void MarkKinematicContact(const m3WorldView& w, const m3Scratch& s,
                                                     int32_t bodyA, int32_t bodyB)
{
    int dynA = w.btype[bodyA] == M3_BODY_DYNAMIC;
    int dynB = w.btype[bodyB] == M3_BODY_DYNAMIC;
    if (dynA && dynB)
    {
        IslandUnion(s.parent, bodyA, bodyB);
    }
    else if (dynA || dynB)
    {
        int32_t kin = dynA ? bodyB : bodyA;
        int32_t dyn = dynA ? bodyA : bodyB;
        if (w.btype[kin] == M3_BODY_KINEMATIC)
        {
            m3Vec3 v = w.v[kin];
            m3Vec3 om = w.w[kin];
            if (m3Dot3(v, v) > 0.0f || m3Dot3(om, om) > 0.0f)
            {
                s.forced[dyn] = 1;
            }
        }
    }
}

// Continuous collision against planes for one fast non-bullet body
// (solver.c:3286-3347, the plane arm of SolveContinuousPhase :3349-3425).
__device__ m3Transform SweepTransform(const m3Vec3& lc, const m3Vec3& c1, const m3Vec3& c2,
                                      const m3Quat& q1, m3Quat q2, m3real time)
{
    m3Transform xf;
    if (q1.x * q2.x + q1.y * q2.y + q1.z * q2.z + q1.w * q2.w < 0.0f)
    {
        q2 = q4(-q2.x, -q2.y, -q2.z, -q2.w);
    }
    m3Quat q = q4(q1.x + time * (q2.x - q1.x), q1.y + time * (q2.y - q1.y),
                  q1.z + time * (q2.z - q1.z), q1.w + time * (q2.w - q1.w));
    xf.q = m3NormalizeQuat(q);
    m3Vec3 c = m3Add3(c1, m3MulSV3(time, m3Sub3(c2, c1)));
    m3Vec3 r = m3RotateVec3(xf.q, lc);
    xf.p.x = (double)(c.x - r.x);
    xf.p.y = (double)(c.y - r.y);
    xf.p.z = (double)(c.z - r.z);
    return xf;
}

// Support points of the fast shape's distance proxy (manifold.c:463-499).
__device__ __forceinline__ int32_t ProxyPoints(const m3WorldView& w, int32_t shape,
                                               const m3Vec3** pts, m3Vec3 scratch[2],
                                               m3real* radius)
{
    uint8_t type = w.shapeType[shape];
    if (type == M3_SHAPE_HULL)
    {
        const m3HullData* hull = &w.hulls[w.hullIndex[shape]];
        *pts = hull->vertices;
        *radius = 0.0f;
        return hull->vertexCount;
    }
    if (type == M3_SHAPE_CAPSULE)
    {
        scratch[0] = w.geom[shape].v;
        scratch[1] = w.geom[shape].v2;
        *pts = scratch;
        *radius = w.geom[shape].s;
        return 2;
    }
    scratch[0] = w.geom[shape].v;
    *pts = scratch;
    *radius = w.geom[shape].s;
    return 1;
}

__device__ void ContinuousVersusPlane(const m3WorldView& w, int32_t body, int32_t fastShape,
                                      int32_t planeShape, const m3Pos3& base, const m3Vec3& lc,
                                      const m3Vec3& c1, const m3Vec3& c2, const m3Quat& q1,
                                      const m3Quat& q2, m3real* fraction)
{
    m3Vec3 n = w.geom[planeShape].v;
    m3real offset = w.geom[planeShape].s -
                    (m3real)((double)n.x * base.x + (double)n.y * base.y + (double)n.z * base.z);
    m3Vec3 scratch[2];
    const m3Vec3* pts;
    m3real radius;
    int32_t count = ProxyPoints(w, fastShape, &pts, scratch, &radius);
    const m3real linearSlop = M3_LINEAR_SLOP;
    m3real target = m3MaxF(linearSlop, radius - linearSlop);
    m3real tolerance = 0.25f * linearSlop;
    m3Vec3 travel = m3Sub3(c2, c1);
    m3Quat dq = m3MulQuat(q2, q4(-q1.x, -q1.y, -q1.z, q1.w));
    m3real arc = 2.0f * sqrtf(dq.x * dq.x + dq.y * dq.y + dq.z * dq.z) * w.maxExt[body];
    m3real rate = sqrtf(m3Dot3(travel, travel)) + arc;
    if (!(rate > 0.0f))
    {
        return;
    }
    m3real t = 0.0f;
    for (int32_t iter = 0; iter < 25; ++iter)
    {
        m3Transform xf = SweepTransform(lc, c1, c2, q1, q2, t);
        m3real minD = 3.4e38f;
        for (int32_t k = 0; k < count; ++k)
        {
            m3Vec3 r = m3RotateVec3(xf.q, pts[k]);
            m3real d = n.x * ((m3real)xf.p.x + r.x) + n.y * ((m3real)xf.p.y + r.y) +
                       n.z * ((m3real)xf.p.z + r.z);
            minD = m3MinF(minD, d);
        }
        m3real sep = minD - offset;
        if (sep <= 0.0f)
        {
            return;
        }
        if (sep <= target + tolerance)
        {
            if (t > 0.0f && t < *fraction)
            {
                *fraction = t;
            }
            return;
        }
        t += (sep - target) / rate;
        if (t >= *fraction)
        {
            return;
        }
    }
}

// ---------------------------------------------------------------------
// Kernel 2: islands and wake, contact selection, colouring, row
// preparation, joint rows and their levels, movers
// ---------------------------------------------------------------------
// Shared-memory bytes per body of the substep-loop cache: v, w, the
// position delta (12 B each) and the rotation delta (16 B).
#define M3_BODY_CACHE_BYTES 52
// Velocities alone (linear and angular).
#define M3_BODY_VELOCITY_BYTES 24
// Dynamic shared memory per block that still lets two 256-thread blocks
// share an SM (228 KB per SM, 1 KB reserved per block, static arrays).
#define M3_TWO_BLOCK_SMEM (110 * 1024)

template <int NT, int MIN_BLOCKS>
__global__ void __launch_bounds__(NT, MIN_BLOCKS) m3PrepareKernel(const m3WorldView* views,
                                                            const int32_t* order, int32_t count,
                                                            float dt, int32_t substeps,
                                                            int32_t cacheBytes, int32_t wide = 0)
{
    const int32_t wi = order[blockIdx.x];
    const m3WorldView& w = views[wi];
    m3WorldScalars* sc = w.sc;
    m3Scratch s;
    ScratchCarve(&s, w.scratch, sc->bodyCap, sc->shapeCap, sc->jointCap, sc->pairCap);
    const int32_t tid = threadIdx.x;
    __shared__ int32_t s_status;
    __shared__ int32_t s_anyRestitution;
    __shared__ int32_t s_starts[M3_GRAPH_COLORS + 2];
    __shared__ int32_t s_jointLevels;
    __shared__ int32_t s_contactLevels;
    __shared__ int32_t s_totalLevels;
    if (tid == 0)
    {
        s_status = sc->status;
        s_anyRestitution = 0;
        // A wide substep kernel may follow: its grid barrier starts with
        // no arrivals and no error.
        s.gridBar[0] = 0;
        s.gridBar[2] = 0;
        if (s_status == 0)
        {
            // The pair list and manifolds built by the collide kernels
            // become the current ones.
            sc->pairBuf = 1 - sc->pairBuf;
            sc->prevPairCount = sc->pairCount;
            sc->pairCount = sc->newPairCount;
            sc->stepBrokenStart = sc->brokenCount;
        }
    }
    __syncthreads();
    if (s_status != 0)
    {
        return;
    }
    long long t_phase = clock64();
    const int32_t bodyMax = sc->bodyMax;
    const int32_t jointMax = sc->jointMax;
    const int32_t pairCount = sc->pairCount;
    const uint64_t* keys = sc->pairBuf == 0 ? w.keys0 : w.keys1;
    m3Manifold* man = sc->pairBuf == 0 ? w.man0 : w.man1;

    // Begin-of-step centres and rotations (solver.c:3866-3877); island
    // arrays reset.
    for (int32_t i = tid; i < bodyMax; i += NT)
    {
        s.parent[i] = i;
        s.forced[i] = 0;
        s.forcedRoot[i] = 0;
        if (w.bodyAlive[i] == 0)
        {
            s.bodyInvI[i] = m3ZeroMat3();
            continue;
        }
        const m3Transform xf = w.xf[i];
        m3Vec3 rlc = m3RotateVec3(xf.q, w.lc[i]);
        m3Pos3 c;
        c.x = xf.p.x + (double)rlc.x;
        c.y = xf.p.y + (double)rlc.y;
        c.z = xf.p.z + (double)rlc.z;
        s.com0[i] = c;
        s.rot0[i] = xf.q;
        // The contact rows' world-space inverse inertia, once per body
        // (the transforms do not change before the rows are prepared).
        s.bodyInvI[i] = m3WorldInvInertiaDev(w, i);
    }
    __syncthreads();

    // Island wake pass (solver.c:3468-3578).
    for (int32_t k = tid; k < pairCount; k += NT)
    {
        if (man[k].pointCount == 0)
        {
            continue;
        }
        uint64_t key = keys[k];
        int32_t shapeA = (int32_t)(key >> 32);
        int32_t shapeB = (int32_t)(key & 0xFFFFFFFFu);
        if (w.sensor[shapeA] != 0 || w.sensor[shapeB] != 0)
        {
            continue;
        }
        MarkKinematicContact(w, s, w.shapeBody[shapeA], w.shapeBody[shapeB]);
    }
    for (int32_t j = tid; j < jointMax; j += NT)
    {
        if (w.jointAlive[j] != 0)
        {
            MarkKinematicContact(w, s, w.jbodyA[j], w.jbodyB[j]);
        }
    }
    __syncthreads();
    for (int32_t i = tid; i < bodyMax; i += NT)
    {
        if (w.bodyAlive[i] == 0 || w.btype[i] != M3_BODY_DYNAMIC)
        {
            continue;
        }
        if (w.awake[i] != 0 || s.forced[i] != 0)
        {
            s.forcedRoot[IslandFind(s.parent, i)] = 1;
        }
    }
    __syncthreads();
    for (int32_t i = tid; i < bodyMax; i += NT)
    {
        if (w.bodyAlive[i] == 0 || w.btype[i] != M3_BODY_DYNAMIC)
        {
            continue;
        }
        if (w.awake[i] == 0 && s.forcedRoot[IslandFind(s.parent, i)] != 0)
        {
            w.awake[i] = 1;
            w.sleepTime[i] = 0.0f;
        }
    }
    for (int32_t i = tid; i < bodyMax; i += NT)
    {
        s.deltaPos[i] = v3(0.0f, 0.0f, 0.0f);
        s.deltaRot[i] = m3IdentityQuat();
    }
    __syncthreads();

    M3_PHASE_MARK(M3_PHASE_ISLANDS)
    // Contact selection and preparation (solver.c:156-405).
    const m3real h = dt / (m3real)substeps;
    const m3SoftDev soft = m3MakeSoft(sc->contactHertz, sc->contactDampingRatio, h);
    const m3SoftDev staticSoft = m3MakeSoft(2.0f * sc->contactHertz, sc->contactDampingRatio, h);
    for (int32_t k = tid; k < pairCount; k += NT)
    {
        int32_t flag = 0;
        if (man[k].pointCount != 0)
        {
            uint64_t key = keys[k];
            int32_t shapeA = (int32_t)(key >> 32);
            int32_t shapeB = (int32_t)(key & 0xFFFFFFFFu);
            int32_t bodyA = w.shapeBody[shapeA];
            int32_t bodyB = w.shapeBody[shapeB];
            int awakeDynA = w.btype[bodyA] == M3_BODY_DYNAMIC && w.awake[bodyA] != 0;
            int awakeDynB = w.btype[bodyB] == M3_BODY_DYNAMIC && w.awake[bodyB] != 0;
            if ((awakeDynA || awakeDynB) && w.sensor[shapeA] == 0 && w.sensor[shapeB] == 0)
            {
                flag = 1;
            }
        }
        s.pairFlag[k] = flag;
    }
    __syncthreads();
    const int32_t constraintCount = BlockExclusiveScan<NT>(s.pairFlag, pairCount);
    for (int32_t k = tid; k < pairCount; k += NT)
    {
        int32_t next = k + 1 < pairCount ? s.pairFlag[k + 1] : constraintCount;
        if (next != s.pairFlag[k])
        {
            s.conPairIndex[s.pairFlag[k]] = k;
        }
    }
    // Joint rows (solver.c:699-1042): selection in slot order, rows
    // prepared in parallel, then grouped into dependency levels.  A
    // joint's level is one past the latest earlier joint sharing either
    // of its bodies (any body, static ones included), so the joints of
    // one level touch disjoint bodies and solving level by level, each
    // level in parallel, reproduces the reference's serial slot order.
    for (int32_t j = tid; j < jointMax; j += NT)
    {
        int32_t flag = 0;
        if (w.jointAlive[j] != 0)
        {
            int32_t refusal = m3JointRefusal(w, j);
            if (refusal != 0)
            {
                s_status = M3GPU_ERR_UNSUPPORTED;
                sc->statusDetail = refusal;
            }
            else if (m3JointActive(w, j))
            {
                flag = 1;
            }
        }
        s.jointFlag[j] = flag;
    }
    __syncthreads();
    const int32_t jointCount = BlockExclusiveScan<NT>(s.jointFlag, jointMax);
    for (int32_t j = tid; j < jointMax; j += NT)
    {
        int32_t next = j + 1 < jointMax ? s.jointFlag[j + 1] : jointCount;
        if (next != s.jointFlag[j])
        {
            const int32_t r = s.jointFlag[j];
            m3PrepareJoint(w, &s.joints[r], j, h);
            s.jointBodies[r] = make_int2(s.joints[r].bodyA, s.joints[r].bodyB);
        }
    }
    for (int32_t i = tid; i < bodyMax; i += NT)
    {
        s.ready[i] = -1;
    }
    __syncthreads();
    // The levels follow the slot order: one thread walks the rows' body
    // pairs (a compact array, read ahead of the walk's own dependences).
    if (tid == 0)
    {
        int32_t levels = 0;
        for (int32_t r = 0; r < jointCount; ++r)
        {
            const int2 ab = s.jointBodies[r];
            const int32_t la = s.ready[ab.x];
            const int32_t lb = s.ready[ab.y];
            const int32_t level = 1 + (la > lb ? la : lb);
            s.ready[ab.x] = level;
            s.ready[ab.y] = level;
            s.jointLevel[r] = level;
            levels = level + 1 > levels ? level + 1 : levels;
        }
        s_jointLevels = levels;
        sc->jointConstraintCount = jointCount;
    }
    __syncthreads();
    // Rows grouped by level (any order inside a level: its rows touch
    // disjoint bodies).
    const int32_t jointLevelCount = s_jointLevels;
    for (int32_t k = tid; k <= jointLevelCount; k += NT)
    {
        s.jointLevelStart[k] = 0;
    }
    __syncthreads();
    for (int32_t r = tid; r < jointCount; r += NT)
    {
        atomicAdd(&s.jointLevelStart[s.jointLevel[r] + 1], 1);
    }
    __syncthreads();
    if (tid == 0)
    {
        for (int32_t k = 0; k < jointLevelCount; ++k)
        {
            s.jointLevelStart[k + 1] += s.jointLevelStart[k];
        }
    }
    __syncthreads();
    for (int32_t k = tid; k <= jointLevelCount; k += NT)
    {
        s.levelFill[k] = s.jointLevelStart[k];
    }
    __syncthreads();
    for (int32_t r = tid; r < jointCount; r += NT)
    {
        s.jointOrder[atomicAdd(&s.levelFill[s.jointLevel[r]], 1)] = r;
    }
    __syncthreads();
    if (s_status != 0)
    {
        if (tid == 0)
        {
            sc->status = s_status;
        }
        return;
    }

    M3_PHASE_MARK(M3_PHASE_PREPARE)
    // Greedy 16-colour first-free-bit colouring in constraint order, the
    // overflow bucket last (solver.c:2750-2810), computed in rounds.  In
    // the serial walk a constraint's colour depends only on the colours
    // of the earlier constraints that share one of its (awake dynamic)
    // bodies.  So in each round every uncoloured constraint that is the
    // earliest uncoloured one on each of its bodies takes its colour at
    // once: exactly the masks the serial walk would see, and no two
    // constraints of a round touch the same body.  Each round colours
    // at least the earliest uncoloured constraint; after M3_COLOR_ROUNDS
    // rounds thread 0 finishes any rest in order.  Slots are then
    // assigned colour by colour in constraint order (a stable counting
    // sort), as the serial list fill does.
    extern __shared__ __align__(16) uint8_t s_colorStage[];
    const int64_t bodyWords = ((int64_t)bodyMax + 1) & ~1LL;
    const int64_t stageBytes = 12 * bodyWords + 9 * (int64_t)constraintCount;
    const bool staged = stageBytes <= (int64_t)cacheBytes;
    uint32_t* cMask = staged ? (uint32_t*)s_colorStage : s.bodyMask;
    int32_t* cMin0 = staged ? (int32_t*)(cMask + bodyWords) : s.colorMin;
    int32_t* cMin1 = cMin0 + (staged ? bodyWords : (int64_t)sc->bodyCap);
    int2* cPair = staged ? (int2*)(s_colorStage + 12 * bodyWords) : s.conPair;
    uint8_t* cColor = staged ? (uint8_t*)(cPair + constraintCount) : s.colors;
    for (int32_t i = tid; i < bodyMax; i += NT)
    {
        cMask[i] = 0u;
        cMin0[i] = INT32_MAX;
        cMin1[i] = INT32_MAX;
    }
    for (int32_t i = tid; i < constraintCount; i += NT)
    {
        const uint64_t key = keys[s.conPairIndex[i]];
        const int32_t bodyA = w.shapeBody[(int32_t)(key >> 32)];
        const int32_t bodyB = w.shapeBody[(int32_t)(key & 0xFFFFFFFFu)];
        int32_t a = w.btype[bodyA] == M3_BODY_DYNAMIC && w.awake[bodyA] ? bodyA : -1;
        int32_t b = w.btype[bodyB] == M3_BODY_DYNAMIC && w.awake[bodyB] ? bodyB : -1;
        cPair[i] = make_int2(a, b);
        cColor[i] = M3_COLOR_PENDING;
    }
    __syncthreads();
    bool pendingLeft = constraintCount > 0;
    for (int32_t round = 0; pendingLeft && round < M3_COLOR_ROUNDS; ++round)
    {
        int32_t* cur = (round & 1) ? cMin1 : cMin0;
        int32_t* nxt = (round & 1) ? cMin0 : cMin1;
        for (int32_t i = tid; i < constraintCount; i += NT)
        {
            if (cColor[i] == M3_COLOR_PENDING)
            {
                const int2 p = cPair[i];
                if (p.x >= 0)
                {
                    atomicMin(&cur[p.x], i);
                }
                if (p.y >= 0)
                {
                    atomicMin(&cur[p.y], i);
                }
            }
        }
        __syncthreads();
        int32_t waiting = 0;
        for (int32_t i = tid; i < constraintCount; i += NT)
        {
            if (cColor[i] != M3_COLOR_PENDING)
            {
                continue;
            }
            const int2 p = cPair[i];
            const bool ready = (p.x < 0 || cur[p.x] == i) && (p.y < 0 || cur[p.y] == i);
            // The next round's claims start from empty on every body a
            // pending constraint may touch.
            if (p.x >= 0)
            {
                nxt[p.x] = INT32_MAX;
            }
            if (p.y >= 0)
            {
                nxt[p.y] = INT32_MAX;
            }
            if (!ready)
            {
                waiting = 1;
                continue;
            }
            const uint32_t mask = (p.x >= 0 ? cMask[p.x] : 0u) | (p.y >= 0 ? cMask[p.y] : 0u);
            // First clear bit among the 16 colours; 16 = overflow.
            int32_t color = __ffs((int)~mask) - 1;
            color = color < M3_GRAPH_COLORS ? color : M3_GRAPH_COLORS;
            cColor[i] = (uint8_t)color;
            if (color < M3_GRAPH_COLORS)
            {
                const uint32_t bit = 1u << color;
                if (p.x >= 0)
                {
                    cMask[p.x] |= bit;
                }
                if (p.y >= 0)
                {
                    cMask[p.y] |= bit;
                }
            }
        }
        pendingLeft = __syncthreads_or(waiting) != 0;
    }
    if (pendingLeft && tid == 0)
    {
        // Long dependency chains: the rest in constraint order.
        for (int32_t i = 0; i < constraintCount; ++i)
        {
            if (cColor[i] != M3_COLOR_PENDING)
            {
                continue;
            }
            const int2 p = cPair[i];
            const uint32_t mask = (p.x >= 0 ? cMask[p.x] : 0u) | (p.y >= 0 ? cMask[p.y] : 0u);
            int32_t color = __ffs((int)~mask) - 1;
            color = color < M3_GRAPH_COLORS ? color : M3_GRAPH_COLORS;
            cColor[i] = (uint8_t)color;
            if (color < M3_GRAPH_COLORS)
            {
                const uint32_t bit = 1u << color;
                if (p.x >= 0)
                {
                    cMask[p.x] |= bit;
                }
                if (p.y >= 0)
                {
                    cMask[p.y] |= bit;
                }
            }
        }
    }
    // Colour sizes and offsets.
    __shared__ int32_t s_colorFill[M3_GRAPH_COLORS + 1];
    __shared__ int32_t s_warpColor[NT / 32][M3_GRAPH_COLORS + 1];
    if (tid <= M3_GRAPH_COLORS)
    {
        s_colorFill[tid] = 0;
    }
    __syncthreads();
    for (int32_t i = tid; i < constraintCount; i += NT)
    {
        atomicAdd(&s_colorFill[cColor[i]], 1);
    }
    __syncthreads();
    if (tid == 0)
    {
        int32_t cursor = 0;
        int32_t used = 0;
        for (int32_t c = 0; c <= M3_GRAPH_COLORS; ++c)
        {
            const int32_t n = s_colorFill[c];
            s_starts[c] = cursor;
            s_colorFill[c] = cursor;
            cursor += n;
            used += n > 0 ? 1 : 0;
        }
        s_starts[M3_GRAPH_COLORS + 1] = cursor;
        sc->lastColorCount = used;
        sc->constraintCount = constraintCount;
    }
    __syncthreads();
    // Slots: colour by colour, constraint order inside a colour.
    {
        const int32_t lane = tid & 31;
        const int32_t warp = tid >> 5;
        const uint32_t ltMask = (1u << lane) - 1u;
        for (int32_t c0 = 0; c0 < constraintCount; c0 += NT)
        {
            const int32_t i = c0 + tid;
            const int32_t color = i < constraintCount ? (int32_t)cColor[i] : M3_GRAPH_COLORS + 1;
            for (int32_t k = tid; k < (NT / 32) * (M3_GRAPH_COLORS + 1); k += NT)
            {
                (&s_warpColor[0][0])[k] = 0;
            }
            __syncthreads();
            const uint32_t peers = __match_any_sync(0xFFFFFFFFu, color);
            const int32_t rank = __popc(peers & ltMask);
            if (rank == 0 && color <= M3_GRAPH_COLORS)
            {
                s_warpColor[warp][color] = __popc(peers);
            }
            __syncthreads();
            if (color <= M3_GRAPH_COLORS)
            {
                int32_t slot = s_colorFill[color] + rank;
                for (int32_t k = 0; k < warp; ++k)
                {
                    slot += s_warpColor[k][color];
                }
                s.lists[slot] = i;
                s.conSlot[i] = slot;
            }
            __syncthreads();
            if (tid <= M3_GRAPH_COLORS)
            {
                int32_t add = 0;
                for (int32_t k = 0; k < NT / 32; ++k)
                {
                    add += s_warpColor[k][tid];
                }
                s_colorFill[tid] += add;
            }
            __syncthreads();
        }
    }
    __syncthreads();
    // One schedule for joints and contacts.  Per body, the reference
    // applies its joints (slot order) and then its contacts (colour
    // order) in each pass.  A contact's level is therefore at least one
    // past the last joint level on either of its awake dynamic bodies and
    // one past the level of the previous contact on either of them; the
    // substep loop then runs level by level, joint rows and contact rows
    // of a level together, so contacts away from the joint chains no
    // longer wait for them.  The overflow colour stays last and serial.
    // Contacts are re-slotted by level (any order inside a level: its
    // rows touch disjoint bodies).
    {
        int32_t* cLast = cMin0; // per body: first level free for its next contact
        for (int32_t i = tid; i < bodyMax; i += NT)
        {
            cLast[i] = jointCount > 0 ? s.ready[i] + 1 : 0;
        }
        if (tid == 0)
        {
            s_contactLevels = 0;
        }
        __syncthreads();
        for (int32_t color = 0; color < M3_GRAPH_COLORS; ++color)
        {
            for (int32_t k = s_starts[color] + tid; k < s_starts[color + 1]; k += NT)
            {
                const int32_t i = s.lists[k];
                const int2 p = cPair[i];
                int32_t level = 0;
                if (p.x >= 0)
                {
                    level = cLast[p.x] > level ? cLast[p.x] : level;
                }
                if (p.y >= 0)
                {
                    level = cLast[p.y] > level ? cLast[p.y] : level;
                }
                s.conLevel[i] = level;
                if (p.x >= 0)
                {
                    cLast[p.x] = level + 1;
                }
                if (p.y >= 0)
                {
                    cLast[p.y] = level + 1;
                }
                atomicMax(&s_contactLevels, level + 1);
            }
            __syncthreads();
        }
        const int32_t levels = s_contactLevels > s_jointLevels ? s_contactLevels : s_jointLevels;
        // Counts per level (the overflow colour is bucket `levels`),
        // offsets, then each constraint claims a slot in its level.
        for (int32_t k = tid; k <= levels + 1; k += NT)
        {
            s.levelStart[k] = 0;
        }
        __syncthreads();
        for (int32_t i = tid; i < constraintCount; i += NT)
        {
            const int32_t level = cColor[i] == M3_GRAPH_COLORS ? levels : s.conLevel[i];
            s.conLevel[i] = level;
            atomicAdd(&s.levelStart[level + 1], 1);
        }
        __syncthreads();
        if (tid == 0)
        {
            for (int32_t k = 0; k <= levels; ++k)
            {
                s.levelStart[k + 1] += s.levelStart[k];
            }
            s_totalLevels = levels;
        }
        __syncthreads();
        for (int32_t k = tid; k <= levels; k += NT)
        {
            s.levelFill[k] = s.levelStart[k];
        }
        __syncthreads();
        // The overflow bucket keeps constraint order (it runs serially).
        for (int32_t i = tid; i < constraintCount; i += NT)
        {
            const int32_t level = s.conLevel[i];
            if (level < levels)
            {
                const int32_t slot = atomicAdd(&s.levelFill[level], 1);
                s.lists[slot] = i;
                s.conSlot[i] = slot;
            }
        }
        if (tid == 0 && s.levelStart[levels + 1] > s.levelStart[levels])
        {
            int32_t slot = s.levelStart[levels];
            for (int32_t i = 0; i < constraintCount; ++i)
            {
                if (s.conLevel[i] == levels)
                {
                    s.lists[slot] = i;
                    s.conSlot[i] = slot;
                    slot += 1;
                }
            }
        }
    }
    __syncthreads();
    M3_PHASE_MARK(M3_PHASE_COLOR)
    // Contact rows (solver.c:261-405), prepared straight into their
    // solve slots; consecutive threads write consecutive slots.  A wide
    // world's rows are prepared over the whole grid instead
    // (m3WideRowsKernel, right after this kernel).
    for (int32_t slot = tid; slot < constraintCount && wide == 0; slot += NT)
    {
        m3ContactDev c;
        m3PrepareContact(w, &c, s.conPairIndex[s.lists[slot]], keys, man, soft, staticSoft,
                         s.bodyInvI);
        m3WriteContactRow(s.rows, slot, c);
        if (c.restitution != 0.0f)
        {
            s_anyRestitution = 1;
        }
        if (c.rollingResistance > 0.0f && (!c.dynA || !c.dynB))
        {
            s_status = M3GPU_ERR_UNSUPPORTED;
            sc->statusDetail = 2001;
        }
    }
    __syncthreads();
    if (s_status != 0)
    {
        if (tid == 0)
        {
            sc->status = s_status;
        }
        return;
    }
    M3_PHASE_MARK(M3_PHASE_PREPARE)

    // Movers: alive, enabled, kinematic or awake dynamic, ascending
    // (solver.c:3945-3983), with the kinematic servo.
    for (int32_t i = tid; i < bodyMax; i += NT)
    {
        int32_t flag = 0;
        if (w.bodyAlive[i] != 0 && w.enabled[i] != 0)
        {
            uint8_t type = w.btype[i];
            if (type == M3_BODY_KINEMATIC || (type == M3_BODY_DYNAMIC && w.awake[i] != 0))
            {
                flag = 1;
            }
            if (type == M3_BODY_KINEMATIC && w.hasTarget[i] != 0)
            {
                m3real servoInvDt = 1.0f / dt;
                const m3Transform now = w.xf[i];
                const m3Transform want = w.target[i];
                w.v[i] = v3((m3real)(want.p.x - now.p.x) * servoInvDt,
                            (m3real)(want.p.y - now.p.y) * servoInvDt,
                            (m3real)(want.p.z - now.p.z) * servoInvDt);
                m3Quat dq = m3MulQuat(want.q, q4(-now.q.x, -now.q.y, -now.q.z, now.q.w));
                if (dq.w < 0.0f)
                {
                    dq = q4(-dq.x, -dq.y, -dq.z, -dq.w);
                }
                w.w[i] = m3MulSV3(2.0f * servoInvDt, v3(dq.x, dq.y, dq.z));
                w.hasTarget[i] = 0;
            }
        }
        s.moverFlag[i] = flag;
    }
    __syncthreads();
    const int32_t moverCount = BlockExclusiveScan<NT>(s.moverFlag, bodyMax);
    for (int32_t i = tid; i < bodyMax; i += NT)
    {
        int32_t next = i + 1 < bodyMax ? s.moverFlag[i + 1] : moverCount;
        if (next != s.moverFlag[i])
        {
            s.movers[s.moverFlag[i]] = i;
        }
    }
    __syncthreads();
    M3_PHASE_MARK(M3_PHASE_COLOR)
    if (tid == 0)
    {
        m3StepPlan* plan = s.plan;
        plan->constraintCount = constraintCount;
        plan->jointCount = sc->jointConstraintCount;
        plan->jointLevels = s_jointLevels;
        plan->moverCount = moverCount;
        plan->anyRestitution = s_anyRestitution;
        plan->levels = s_totalLevels;
        for (int32_t c = 0; c < M3_GRAPH_COLORS + 2; ++c)
        {
            plan->starts[c] = s_starts[c];
        }
    }
}

// ---------------------------------------------------------------------
// Kernel 3: the substep loop, restitution and the impulse store
// ---------------------------------------------------------------------
// NT threads per world (one of the size classes below); MIN_BLOCKS keeps
// the register budget at 128 per thread for every class.
template <int NT, int MIN_BLOCKS>
__global__ void __launch_bounds__(NT, MIN_BLOCKS) m3SubstepKernel(const m3WorldView* views,
                                                            const int32_t* order, int32_t count,
                                                            float dt, int32_t substeps,
                                                            int32_t cacheBytes)
{
    const int32_t wi = order[blockIdx.x];
    const m3WorldView& w = views[wi];
    m3WorldScalars* sc = w.sc;
    if (sc->status != 0)
    {
        return;
    }
    long long t_phase = clock64();
    m3Scratch s;
    ScratchCarve(&s, w.scratch, sc->bodyCap, sc->shapeCap, sc->jointCap, sc->pairCap);
    const int32_t tid = threadIdx.x;
    __shared__ int32_t s_starts[M3_GRAPH_COLORS + 2];
    if (tid < M3_GRAPH_COLORS + 2)
    {
        s_starts[tid] = s.plan->starts[tid];
    }
    const int32_t bodyMax = sc->bodyMax;
    const int32_t constraintCount = s.plan->constraintCount;
    const int32_t jointCount = s.plan->jointCount;
    const int32_t jointLevels = s.plan->jointLevels;
    const int32_t moverCount = s.plan->moverCount;
    const bool anyRestitution = s.plan->anyRestitution != 0;
    m3Manifold* man = sc->pairBuf == 0 ? w.man0 : w.man1;
    const m3real h = dt / (m3real)substeps;
    const m3real invH = h > 0.0f ? 1.0f / h : 0.0f;
    const m3real pushMax = sc->contactPushMaxSpeed;

    // Body velocities and the substep deltas live in shared memory for
    // the whole substep loop when the world fits: every solve row then
    // reads and writes its two bodies at shared-memory latency.  One
    // copy in here, one copy out after restitution; the arithmetic is
    // unchanged.
    extern __shared__ __align__(16) uint8_t s_bodyCache[];
    m3WorldView wl = w;
    m3Vec3* dP = s.deltaPos;
    m3Quat* dQ = s.deltaRot;
    const bool cached = (int64_t)bodyMax * M3_BODY_CACHE_BYTES <= (int64_t)cacheBytes;
    // A world too large for the whole cache keeps at least its velocities
    // there (the rows' read-modify-write chain); the substep deltas, which
    // rows only read, stay in global memory.
    const bool cachedV =
        !cached && (int64_t)bodyMax * M3_BODY_VELOCITY_BYTES <= (int64_t)cacheBytes;
    if (cachedV)
    {
        m3Vec3* cv = (m3Vec3*)s_bodyCache;
        m3Vec3* cw = cv + bodyMax;
        for (int32_t i = tid; i < bodyMax; i += NT)
        {
            cv[i] = w.v[i];
            cw[i] = w.w[i];
        }
        wl.v = cv;
        wl.w = cw;
    }
    if (cached)
    {
        m3Quat* cq = (m3Quat*)s_bodyCache;
        m3Vec3* cv = (m3Vec3*)(cq + bodyMax);
        m3Vec3* cw = cv + bodyMax;
        m3Vec3* cp = cw + bodyMax;
        for (int32_t i = tid; i < bodyMax; i += NT)
        {
            cv[i] = w.v[i];
            cw[i] = w.w[i];
            cp[i] = v3(0.0f, 0.0f, 0.0f);
            cq[i] = m3IdentityQuat();
        }
        wl.v = cv;
        wl.w = cw;
        dP = cp;
        dQ = cq;
    }
    // Then the per-body inverse inertia table of the contact rows, when
    // the world fits, and the joint rows when it leaves room: a joint
    // dependency chain is a sequence of single-thread row solves, each
    // bound by the latency of its row reads.
    const m3Mat3* invI = s.bodyInvI;
    int64_t smemUsed = m3AlignUp(cached    ? (int64_t)bodyMax * M3_BODY_CACHE_BYTES
                                 : cachedV ? (int64_t)bodyMax * M3_BODY_VELOCITY_BYTES
                                           : 0,
                                 16);
    if ((cached || cachedV) &&
        smemUsed + (int64_t)bodyMax * (int64_t)sizeof(m3Mat3) <= (int64_t)cacheBytes)
    {
        m3Mat3* table = (m3Mat3*)(s_bodyCache + smemUsed);
        const int32_t words = bodyMax * (int32_t)(sizeof(m3Mat3) / 4);
        for (int32_t k = tid; k < words; k += NT)
        {
            ((uint32_t*)table)[k] = ((const uint32_t*)s.bodyInvI)[k];
        }
        invI = table;
        smemUsed = m3AlignUp(smemUsed + (int64_t)bodyMax * (int64_t)sizeof(m3Mat3), 16);
    }
    m3JointDev* jrows = s.joints;
    const int64_t jointOff = smemUsed;
    if (jointCount > 0 &&
        jointOff + (int64_t)jointCount * (int64_t)sizeof(m3JointDev) <= (int64_t)cacheBytes)
    {
        jrows = (m3JointDev*)(s_bodyCache + jointOff);
        const int32_t words = jointCount * (int32_t)(sizeof(m3JointDev) / 4);
        for (int32_t k = tid; k < words; k += NT)
        {
            ((uint32_t*)jrows)[k] = ((const uint32_t*)s.joints)[k];
        }
    }
    __syncthreads();
    // One pass over the joint/contact schedule (pass 0 warm start, 1 the
    // biased solve, 2 relax): level by level, the level's joint rows on
    // the first warps and its contact rows on the remaining warps (whole
    // warps apart, so the two kinds of row never diverge inside a warp),
    // then the overflow colour serially.
    const int32_t levels = s.plan->levels;
    auto mergedPass = [&](int32_t pass) {
        for (int32_t level = 0; level < levels; ++level)
        {
            int32_t jointThreads = 0;
            if (level < jointLevels)
            {
                const int32_t j0 = s.jointLevelStart[level];
                const int32_t j1 = s.jointLevelStart[level + 1];
                const int32_t warps = (j1 - j0 + 31) / 32;
                jointThreads = 32 * (warps < NT / 32 - 1 ? warps : NT / 32 - 1);
                for (int32_t k = j0 + tid; tid < jointThreads && k < j1; k += jointThreads)
                {
                    m3JointDev* row = &jrows[s.jointOrder[k]];
                    if (pass == 0)
                    {
                        m3WarmStartJoint(wl, row, dQ);
                    }
                    else
                    {
                        m3SolveJoint(wl, row, dP, dQ, h, invH, pass == 1);
                    }
                }
            }
            const int32_t c1 = s.levelStart[level + 1];
            const int32_t contactThreads = NT - jointThreads;
            for (int32_t k = s.levelStart[level] + tid - jointThreads;
                 tid >= jointThreads && k < c1; k += contactThreads)
            {
                if (pass == 0)
                {
                    m3WarmStartContact(wl, m3ConAt(s.rows, k), invI);
                }
                else
                {
                    m3SolveContact(wl, m3ConAt(s.rows, k), invI, dP, dQ, invH, pushMax,
                                   pass == 1);
                }
            }
            __syncthreads();
        }
        if (tid == 0)
        {
            for (int32_t k = s.levelStart[levels]; k < s.levelStart[levels + 1]; ++k)
            {
                if (pass == 0)
                {
                    m3WarmStartContact(wl, m3ConAt(s.rows, k), invI);
                }
                else
                {
                    m3SolveContact(wl, m3ConAt(s.rows, k), invI, dP, dQ, invH, pushMax,
                                   pass == 1);
                }
            }
        }
        __syncthreads();
    };
    // The substep loop (solver.c:4085-4203).
    for (int32_t sub = 0; sub < substeps; ++sub)
    {
        for (int32_t m = tid; m < moverCount; m += NT)
        {
            int32_t i = s.movers[m];
            if (w.btype[i] == M3_BODY_DYNAMIC)
            {
                m3IntegrateVelocity(wl, i, h);
            }
        }
        __syncthreads();
        M3_PHASE_MARK(M3_PHASE_INTEGRATE_V)
        mergedPass(0); // warm start
        M3_PHASE_MARK(M3_PHASE_WARM)
        mergedPass(1); // solve with bias
        M3_PHASE_MARK(M3_PHASE_SOLVE)
        for (int32_t m = tid; m < moverCount; m += NT)
        {
            m3IntegratePosition(wl, s.movers[m], h, dP, dQ);
        }
        __syncthreads();
        M3_PHASE_MARK(M3_PHASE_INTEGRATE_P)
        mergedPass(2); // relax
        M3_PHASE_MARK(M3_PHASE_RELAX)
    }

    // Forces live one step (solver.c:4207-4211).
    for (int32_t m = tid; m < moverCount; m += NT)
    {
        int32_t i = s.movers[m];
        w.force[i] = v3(0.0f, 0.0f, 0.0f);
        w.torque[i] = v3(0.0f, 0.0f, 0.0f);
    }
    // Restitution is serial in constraint order (solver.c:2879-2906).
    if (tid == 0 && anyRestitution)
    {
        const m3real threshold = sc->restitutionThreshold;
        for (int32_t i = 0; i < constraintCount; ++i)
        {
            m3RestituteContact(wl, m3ConAt(s.rows, s.conSlot[i]), invI, threshold);
        }
    }
    __syncthreads();
    if (cached || cachedV)
    {
        for (int32_t i = tid; i < bodyMax; i += NT)
        {
            w.v[i] = wl.v[i];
            w.w[i] = wl.w[i];
        }
    }
    __syncthreads();
    for (int32_t i = tid; i < constraintCount; i += NT)
    {
        m3StoreContact(m3ConAt(s.rows, i), man);
    }
    // Hit events, per constraint in constraint order (solver.c:2987-3033).
    {
        const uint64_t* keys = sc->pairBuf == 0 ? w.keys0 : w.keys1;
        const m3real hitThreshold = sc->hitEventThreshold;
        for (int32_t i = tid; i < constraintCount; i += NT)
        {
            s.hitFlag[i] = m3HitCandidate(w, m3ConAt(s.rows, s.conSlot[i]), keys, hitThreshold,
                                          &s.hits[i])
                               ? 1
                               : 0;
        }
    }
    for (int32_t r = tid; r < jointCount; r += NT)
    {
        m3StoreJoint(w, &jrows[r]);
    }
    __syncthreads(); // breakage reads the stored joint impulses
    if (tid == 0)
    {
        sc->lastInvH = invH;
        // Wind phase (solver.c:4220-4229).
        if (sc->windGustHertz > 0.0f)
        {
            sc->windPhase += 2.0f * M3_PI * sc->windGustHertz * dt;
            if (sc->windPhase > 2.0f * M3_PI)
            {
                sc->windPhase -=
                    2.0f * M3_PI * (m3real)(int32_t)(sc->windPhase / (2.0f * M3_PI));
            }
        }
        if (sc->jointMax > 0)
        {
            m3BreakJointsDev(w, invH);
        }
    }
    M3_PHASE_MARK(M3_PHASE_STORE)
}

// ---------------------------------------------------------------------
// Wide worlds: one world across the whole grid
// ---------------------------------------------------------------------
// A world of tens of thousands of bodies gets one thread block, and so
// one SM, in the per-world kernels above.  Its substep loop instead runs
// here over a cooperative grid of many blocks: the rows of one schedule
// level (disjoint awake dynamic bodies, the reference's same-colour
// batches that RunColored fans out to host threads, solver.c:2845-2877)
// are spread over every thread of the grid, and a grid barrier separates
// the levels, as the reference's barrier between colours does.  The
// serial parts (the overflow colour, restitution, the destruction of
// broken joints) run on one thread between barriers.  Body state stays
// in global memory (L2), every row's arithmetic is the per-world
// kernel's.

// Grid barrier over `blocks` co-resident blocks (a cooperative launch).
// Thread 0 of each block arrives on a counter; the last arrival resets it
// and advances the generation the others wait on.  A wait that lasts
// longer than `limitNs` (a block that never arrives) sets the error word
// instead of spinning on: every block then leaves the kernel at its next
// barrier, and the host reports the world as failed.
#define M3_GRID_WAIT_NS (4000000000ull)

__device__ __forceinline__ uint64_t m3GlobalTimerNs()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ bool m3GridSync(uint32_t* bar, uint32_t blocks)
{
    __shared__ uint32_t s_ok;
    __syncthreads();
    if (threadIdx.x == 0)
    {
        volatile uint32_t* vbar = bar;
        const uint32_t gen = vbar[1];
        __threadfence();
        if (atomicAdd(&bar[0], 1u) == blocks - 1)
        {
            bar[0] = 0;
            __threadfence();
            atomicAdd(&bar[1], 1u);
        }
        else
        {
            const uint64_t start = m3GlobalTimerNs();
            while (vbar[1] == gen && vbar[2] == 0)
            {
                __nanosleep(64);
                if (m3GlobalTimerNs() - start > M3_GRID_WAIT_NS)
                {
                    atomicExch(&bar[2], 1u);
                    break;
                }
            }
        }
        __threadfence();
        s_ok = vbar[2] == 0 ? 1u : 0u;
    }
    __syncthreads();
    return s_ok != 0;
}

// Exclusive prefix sum of a[0, n) over a cooperative grid: each block
// scans its contiguous chunk, the chunks' totals (ww[M3_WW_PART..])
// give each block its offset.  Every thread of the grid calls it;
// returns the total, or -1 when a barrier gave up.
template <int NT>
__device__ int32_t GridExclusiveScan(int32_t* a, int32_t n, int32_t* ww, uint32_t* bar)
{
    __shared__ int32_t s_offset;
    __shared__ int32_t s_total;
    const int32_t blocks = (int32_t)gridDim.x;
    const int32_t chunk = (n + blocks - 1) / blocks;
    const int32_t lo = (int32_t)blockIdx.x * chunk < n ? (int32_t)blockIdx.x * chunk : n;
    const int32_t hi = lo + chunk < n ? lo + chunk : n;
    const int32_t t = BlockExclusiveScan<NT>(a + lo, hi - lo);
    if (threadIdx.x == 0)
    {
        ww[M3_WW_PART + blockIdx.x] = t;
    }
    if (!m3GridSync(bar, (uint32_t)blocks))
    {
        return -1;
    }
    if (threadIdx.x == 0)
    {
        int32_t off = 0;
        int32_t total = 0;
        for (int32_t b = 0; b < blocks; ++b)
        {
            const int32_t v = ((volatile int32_t*)ww)[M3_WW_PART + b];
            off += b < (int32_t)blockIdx.x ? v : 0;
            total += v;
        }
        s_offset = off;
        s_total = total;
    }
    __syncthreads();
    for (int32_t i = lo + (int32_t)threadIdx.x; i < hi; i += NT)
    {
        a[i] += s_offset;
    }
    const int32_t total = s_total;
    if (!m3GridSync(bar, (uint32_t)blocks))
    {
        return -1;
    }
    return total;
}

// The preparation of one wide world over a cooperative grid: the same
// stages, in the same order and with the same arithmetic, as
// m3PrepareKernel's (islands and wake, contact and joint selection, joint
// rows and their levels, the greedy colouring in rounds, solve slots,
// the joint/contact level schedule, movers), with grid barriers where the
// per-world kernel has block barriers.  The walks that are serial there
// (the joint levels, the colouring's finish after its rounds, the
// overflow bucket's fill) are serial here too, on one thread.  The
// contact rows are left to m3WideRowsKernel.
template <int NT>
__global__ void __launch_bounds__(NT, 2) m3WidePrepareKernel(const m3WorldView* views,
                                                           const int32_t* order, float dt,
                                                           int32_t substeps)
{
    const m3WorldView& w = views[order[0]];
    m3WorldScalars* sc = w.sc;
    if (sc->status != 0)
    {
        return;
    }
    m3Scratch s;
    ScratchCarve(&s, w.scratch, sc->bodyCap, sc->shapeCap, sc->jointCap, sc->pairCap);
    uint32_t* bar = s.gridBar;
    int32_t* ww = s.wideWork;
    volatile int32_t* vww = ww;
    volatile int32_t* vstatus = &sc->status;
    const uint32_t blocks = gridDim.x;
    const int32_t tid = threadIdx.x;
    const int32_t gtid = (int32_t)blockIdx.x * NT + tid;
    const int32_t gstride = (int32_t)blocks * NT;
    const bool lead = blockIdx.x == 0 && tid == 0;
    long long t_phase = clock64();
#define M3_WIDE_MARK(k)                                                                            \
    if (lead)                                                                                      \
    {                                                                                              \
        long long now_ = clock64();                                                                \
        sc->phase[k] += (uint64_t)(now_ - t_phase);                                                \
        t_phase = now_;                                                                            \
    }
#define M3_GSYNC()                                                                                 \
    if (!m3GridSync(bar, blocks))                                                                  \
    {                                                                                              \
        return;                                                                                    \
    }
    // The pair list and manifolds built by the collide kernels become
    // the current ones.
    if (lead)
    {
        sc->pairBuf = 1 - sc->pairBuf;
        sc->prevPairCount = sc->pairCount;
        sc->pairCount = sc->newPairCount;
        sc->stepBrokenStart = sc->brokenCount;
    }
    M3_GSYNC()
    const int32_t bodyMax = sc->bodyMax;
    const int32_t jointMax = sc->jointMax;
    const int32_t pairCount = ((volatile int32_t*)&sc->pairCount)[0];
    const int32_t pairBuf = ((volatile int32_t*)&sc->pairBuf)[0];
    const uint64_t* keys = pairBuf == 0 ? w.keys0 : w.keys1;
    m3Manifold* man = pairBuf == 0 ? w.man0 : w.man1;

    // Begin-of-step centres and rotations (solver.c:3866-3877); island
    // arrays reset; the rows' world inverse inertia.
    for (int32_t i = gtid; i < bodyMax; i += gstride)
    {
        s.parent[i] = i;
        s.forced[i] = 0;
        s.forcedRoot[i] = 0;
        if (w.bodyAlive[i] == 0)
        {
            s.bodyInvI[i] = m3ZeroMat3();
            continue;
        }
        const m3Transform xf = w.xf[i];
        m3Vec3 rlc = m3RotateVec3(xf.q, w.lc[i]);
        m3Pos3 c;
        c.x = xf.p.x + (double)rlc.x;
        c.y = xf.p.y + (double)rlc.y;
        c.z = xf.p.z + (double)rlc.z;
        s.com0[i] = c;
        s.rot0[i] = xf.q;
        s.bodyInvI[i] = m3WorldInvInertiaDev(w, i);
    }
    M3_GSYNC()
    // Island wake pass (solver.c:3468-3578).
    for (int32_t k = gtid; k < pairCount; k += gstride)
    {
        if (man[k].pointCount == 0)
        {
            continue;
        }
        const uint64_t key = keys[k];
        const int32_t shapeA = (int32_t)(key >> 32);
        const int32_t shapeB = (int32_t)(key & 0xFFFFFFFFu);
        if (w.sensor[shapeA] != 0 || w.sensor[shapeB] != 0)
        {
            continue;
        }
        MarkKinematicContact(w, s, w.shapeBody[shapeA], w.shapeBody[shapeB]);
    }
    for (int32_t j = gtid; j < jointMax; j += gstride)
    {
        if (w.jointAlive[j] != 0)
        {
            MarkKinematicContact(w, s, w.jbodyA[j], w.jbodyB[j]);
        }
    }
    M3_GSYNC()
    for (int32_t i = gtid; i < bodyMax; i += gstride)
    {
        if (w.bodyAlive[i] == 0 || w.btype[i] != M3_BODY_DYNAMIC)
        {
            continue;
        }
        if (w.awake[i] != 0 || s.forced[i] != 0)
        {
            s.forcedRoot[IslandFind(s.parent, i)] = 1;
        }
    }
    M3_GSYNC()
    for (int32_t i = gtid; i < bodyMax; i += gstride)
    {
        s.deltaPos[i] = v3(0.0f, 0.0f, 0.0f);
        s.deltaRot[i] = m3IdentityQuat();
        if (w.bodyAlive[i] == 0 || w.btype[i] != M3_BODY_DYNAMIC)
        {
            continue;
        }
        if (w.awake[i] == 0 && s.forcedRoot[IslandFind(s.parent, i)] != 0)
        {
            w.awake[i] = 1;
            w.sleepTime[i] = 0.0f;
        }
    }
    M3_GSYNC()
    M3_WIDE_MARK(M3_PHASE_ISLANDS)

    // Contact selection (solver.c:156-405).
    const m3real h = dt / (m3real)substeps;
    for (int32_t k = gtid; k < pairCount; k += gstride)
    {
        int32_t flag = 0;
        if (man[k].pointCount != 0)
        {
            const uint64_t key = keys[k];
            const int32_t shapeA = (int32_t)(key >> 32);
            const int32_t shapeB = (int32_t)(key & 0xFFFFFFFFu);
            const int32_t bodyA = w.shapeBody[shapeA];
            const int32_t bodyB = w.shapeBody[shapeB];
            const int awakeDynA = w.btype[bodyA] == M3_BODY_DYNAMIC && w.awake[bodyA] != 0;
            const int awakeDynB = w.btype[bodyB] == M3_BODY_DYNAMIC && w.awake[bodyB] != 0;
            if ((awakeDynA || awakeDynB) && w.sensor[shapeA] == 0 && w.sensor[shapeB] == 0)
            {
                flag = 1;
            }
        }
        s.pairFlag[k] = flag;
    }
    // Joint selection in slot order.
    for (int32_t j = gtid; j < jointMax; j += gstride)
    {
        int32_t flag = 0;
        if (w.jointAlive[j] != 0)
        {
            const int32_t refusal = m3JointRefusal(w, j);
            if (refusal != 0)
            {
                atomicExch(&sc->status, M3GPU_ERR_UNSUPPORTED);
                sc->statusDetail = refusal;
            }
            else if (m3JointActive(w, j))
            {
                flag = 1;
            }
        }
        s.jointFlag[j] = flag;
    }
    M3_GSYNC()
    const int32_t constraintCount = GridExclusiveScan<NT>(s.pairFlag, pairCount, ww, bar);
    if (constraintCount < 0)
    {
        return;
    }
    const int32_t jointCount = GridExclusiveScan<NT>(s.jointFlag, jointMax, ww, bar);
    if (jointCount < 0 || *vstatus != 0)
    {
        return;
    }
    for (int32_t k = gtid; k < pairCount; k += gstride)
    {
        const int32_t next = k + 1 < pairCount ? s.pairFlag[k + 1] : constraintCount;
        if (next != s.pairFlag[k])
        {
            s.conPairIndex[s.pairFlag[k]] = k;
        }
    }
    // Joint rows (solver.c:699-1042), then their dependency levels.
    for (int32_t j = gtid; j < jointMax; j += gstride)
    {
        const int32_t next = j + 1 < jointMax ? s.jointFlag[j + 1] : jointCount;
        if (next != s.jointFlag[j])
        {
            const int32_t r = s.jointFlag[j];
            m3PrepareJoint(w, &s.joints[r], j, h);
            s.jointBodies[r] = make_int2(s.joints[r].bodyA, s.joints[r].bodyB);
        }
    }
    // Joint levels: a row's level is one past the latest earlier row on
    // either of its bodies (the serial walk's rule).  Each row finds that
    // previous row on each body from the body's rows, then every row
    // relaxes level = 1 + max(previous levels) until nothing changes;
    // a row's value is exact once its whole chain of previous rows is,
    // so the rounds needed are the longest chain.  Past the round cap the
    // serial walk decides (same result).
    int32_t* adjCount = s.colorMin;                 // per body, then offsets
    int32_t* adjFill = s.colorMin + sc->bodyCap;    // per body: fill cursors
    for (int32_t i = gtid; i < bodyMax; i += gstride)
    {
        adjCount[i] = 0;
        s.ready[i] = -1;
    }
    if (lead)
    {
        ww[M3_WW_JFLAG] = 0;
        ww[M3_WW_JFLAG + 1] = 0;
        ww[M3_WW_JFLAG + 2] = 0;
    }
    M3_GSYNC()
    for (int32_t r = gtid; r < jointCount; r += gstride)
    {
        const int2 ab = s.jointBodies[r];
        atomicAdd(&adjCount[ab.x], 1);
        if (ab.y != ab.x)
        {
            atomicAdd(&adjCount[ab.y], 1);
        }
    }
    M3_GSYNC()
    if (GridExclusiveScan<NT>(adjCount, bodyMax, ww, bar) < 0)
    {
        return;
    }
    for (int32_t i = gtid; i < bodyMax; i += gstride)
    {
        adjFill[i] = adjCount[i];
    }
    M3_GSYNC()
    for (int32_t r = gtid; r < jointCount; r += gstride)
    {
        const int2 ab = s.jointBodies[r];
        s.jointAdj[atomicAdd(&adjFill[ab.x], 1)] = r;
        if (ab.y != ab.x)
        {
            s.jointAdj[atomicAdd(&adjFill[ab.y], 1)] = r;
        }
    }
    M3_GSYNC()
    for (int32_t r = gtid; r < jointCount; r += gstride)
    {
        const int2 ab = s.jointBodies[r];
        int32_t pa = -1;
        for (int32_t k = adjCount[ab.x]; k < adjFill[ab.x]; ++k)
        {
            const int32_t o = s.jointAdj[k];
            pa = o < r && o > pa ? o : pa;
        }
        int32_t pb = -1;
        for (int32_t k = adjCount[ab.y]; k < adjFill[ab.y]; ++k)
        {
            const int32_t o = s.jointAdj[k];
            pb = o < r && o > pb ? o : pb;
        }
        s.jointPrev[r] = make_int2(pa, pb);
        s.jointLevel[r] = 0;
    }
    M3_GSYNC()
    bool changed = jointCount > 0;
    int32_t jround = 0;
    for (; changed && jround < M3_WIDE_JOINT_ROUNDS; ++jround)
    {
        if (lead)
        {
            ww[M3_WW_JFLAG + (jround + 1) % 3] = 0;
        }
        bool mine = false;
        for (int32_t r = gtid; r < jointCount; r += gstride)
        {
            const int2 pr = s.jointPrev[r];
            const int32_t la = pr.x >= 0 ? ((volatile int32_t*)s.jointLevel)[pr.x] : -1;
            const int32_t lb = pr.y >= 0 ? ((volatile int32_t*)s.jointLevel)[pr.y] : -1;
            const int32_t level = 1 + (la > lb ? la : lb);
            if (level != s.jointLevel[r])
            {
                s.jointLevel[r] = level;
                mine = true;
            }
        }
        if (mine)
        {
            ww[M3_WW_JFLAG + jround % 3] = 1;
        }
        M3_GSYNC()
        changed = vww[M3_WW_JFLAG + jround % 3] != 0;
    }
    if (lead)
    {
        int32_t levels = 0;
        if (changed)
        {
            // Chains longer than the round cap: the serial walk.
            for (int32_t r = 0; r < jointCount; ++r)
            {
                const int2 ab = s.jointBodies[r];
                const int32_t la = s.ready[ab.x];
                const int32_t lb = s.ready[ab.y];
                const int32_t level = 1 + (la > lb ? la : lb);
                s.ready[ab.x] = level;
                s.ready[ab.y] = level;
                s.jointLevel[r] = level;
            }
        }
        ww[M3_WW_LEVELS] = 0;
        sc->jointConstraintCount = jointCount;
        (void)levels;
    }
    M3_GSYNC()
    // The levels' count, and each body's last joint level (its latest
    // row's: levels grow along a body's rows).
    for (int32_t r = gtid; r < jointCount; r += gstride)
    {
        const int32_t level = s.jointLevel[r];
        atomicMax(&ww[M3_WW_LEVELS], level + 1);
        const int2 ab = s.jointBodies[r];
        atomicMax(&s.ready[ab.x], level);
        atomicMax(&s.ready[ab.y], level);
    }
    M3_GSYNC()
    const int32_t jointLevels = vww[M3_WW_LEVELS];
    for (int32_t k = gtid; k <= jointLevels; k += gstride)
    {
        s.jointLevelStart[k] = 0;
    }
    M3_GSYNC()
    for (int32_t r = gtid; r < jointCount; r += gstride)
    {
        atomicAdd(&s.jointLevelStart[s.jointLevel[r] + 1], 1);
    }
    M3_GSYNC()
    if (lead)
    {
        for (int32_t k = 0; k < jointLevels; ++k)
        {
            s.jointLevelStart[k + 1] += s.jointLevelStart[k];
        }
    }
    M3_GSYNC()
    for (int32_t k = gtid; k <= jointLevels; k += gstride)
    {
        s.levelFill[k] = s.jointLevelStart[k];
    }
    M3_GSYNC()
    for (int32_t r = gtid; r < jointCount; r += gstride)
    {
        s.jointOrder[atomicAdd(&s.levelFill[s.jointLevel[r]], 1)] = r;
    }
    M3_GSYNC()
    M3_WIDE_MARK(M3_PHASE_PREPARE)

    // Greedy 16-colour first-free-bit colouring in constraint order, the
    // overflow bucket last (solver.c:2750-2810), in rounds: each round
    // colours every uncoloured constraint that is the earliest
    // uncoloured one on each of its awake dynamic bodies (exactly the
    // masks the serial walk sees); after M3_COLOR_ROUNDS rounds one
    // thread finishes the rest in order.
    uint32_t* cMask = s.bodyMask;
    int32_t* cMin0 = s.colorMin;
    int32_t* cMin1 = s.colorMin + sc->bodyCap;
    int2* cPair = s.conPair;
    uint8_t* cColor = s.colors;
    for (int32_t i = gtid; i < bodyMax; i += gstride)
    {
        cMask[i] = 0u;
        cMin0[i] = INT32_MAX;
        cMin1[i] = INT32_MAX;
    }
    for (int32_t i = gtid; i < constraintCount; i += gstride)
    {
        const uint64_t key = keys[s.conPairIndex[i]];
        const int32_t bodyA = w.shapeBody[(int32_t)(key >> 32)];
        const int32_t bodyB = w.shapeBody[(int32_t)(key & 0xFFFFFFFFu)];
        const int32_t a = w.btype[bodyA] == M3_BODY_DYNAMIC && w.awake[bodyA] ? bodyA : -1;
        const int32_t b = w.btype[bodyB] == M3_BODY_DYNAMIC && w.awake[bodyB] ? bodyB : -1;
        cPair[i] = make_int2(a, b);
        cColor[i] = M3_COLOR_PENDING;
    }
    if (lead)
    {
        ww[M3_WW_FLAG] = 0;
        ww[M3_WW_FLAG + 1] = 0;
        ww[M3_WW_FLAG + 2] = 0;
    }
    M3_GSYNC()
    // Round r raises flag r % 3 and every block reads it after the round's
    // last barrier; it is cleared again at the start of round r + 2, after
    // two more barriers, when no block can still be reading it.
    bool pendingLeft = constraintCount > 0;
    for (int32_t round = 0; pendingLeft && round < M3_WIDE_COLOR_ROUNDS; ++round)
    {
        int32_t* cur = (round & 1) ? cMin1 : cMin0;
        int32_t* nxt = (round & 1) ? cMin0 : cMin1;
        if (lead)
        {
            ww[M3_WW_FLAG + (round + 1) % 3] = 0; // the next round's flag
        }
        for (int32_t i = gtid; i < constraintCount; i += gstride)
        {
            if (cColor[i] == M3_COLOR_PENDING)
            {
                const int2 p = cPair[i];
                if (p.x >= 0)
                {
                    atomicMin(&cur[p.x], i);
                }
                if (p.y >= 0)
                {
                    atomicMin(&cur[p.y], i);
                }
            }
        }
        M3_GSYNC()
        bool waiting = false;
        for (int32_t i = gtid; i < constraintCount; i += gstride)
        {
            if (cColor[i] != M3_COLOR_PENDING)
            {
                continue;
            }
            const int2 p = cPair[i];
            const bool ready = (p.x < 0 || cur[p.x] == i) && (p.y < 0 || cur[p.y] == i);
            if (p.x >= 0)
            {
                nxt[p.x] = INT32_MAX;
            }
            if (p.y >= 0)
            {
                nxt[p.y] = INT32_MAX;
            }
            if (!ready)
            {
                waiting = true;
                continue;
            }
            const uint32_t mask = (p.x >= 0 ? cMask[p.x] : 0u) | (p.y >= 0 ? cMask[p.y] : 0u);
            int32_t color = __ffs((int)~mask) - 1;
            color = color < M3_GRAPH_COLORS ? color : M3_GRAPH_COLORS;
            cColor[i] = (uint8_t)color;
            if (color < M3_GRAPH_COLORS)
            {
                const uint32_t bit = 1u << color;
                if (p.x >= 0)
                {
                    cMask[p.x] |= bit;
                }
                if (p.y >= 0)
                {
                    cMask[p.y] |= bit;
                }
            }
        }
        if (waiting)
        {
            ww[M3_WW_FLAG + round % 3] = 1;
        }
        M3_GSYNC()
        pendingLeft = vww[M3_WW_FLAG + round % 3] != 0;
    }
    if (pendingLeft)
    {
        if (lead)
        {
            for (int32_t i = 0; i < constraintCount; ++i)
            {
                if (cColor[i] != M3_COLOR_PENDING)
                {
                    continue;
                }
                const int2 p = cPair[i];
                const uint32_t mask =
                    (p.x >= 0 ? cMask[p.x] : 0u) | (p.y >= 0 ? cMask[p.y] : 0u);
                int32_t color = __ffs((int)~mask) - 1;
                color = color < M3_GRAPH_COLORS ? color : M3_GRAPH_COLORS;
                cColor[i] = (uint8_t)color;
                if (color < M3_GRAPH_COLORS)
                {
                    const uint32_t bit = 1u << color;
                    if (p.x >= 0)
                    {
                        cMask[p.x] |= bit;
                    }
                    if (p.y >= 0)
                    {
                        cMask[p.y] |= bit;
                    }
                }
            }
        }
        M3_GSYNC()
    }
    // Slots: colour by colour, constraint order inside a colour (a stable
    // counting sort).  Each block owns a contiguous range of constraints:
    // its count per colour, then its first slot per colour, then its
    // slots in order, chunk by chunk.
    __shared__ int32_t s_colorFill[M3_GRAPH_COLORS + 1];
    __shared__ int32_t s_warpColor[NT / 32][M3_GRAPH_COLORS + 1];
    const int32_t chunk = (constraintCount + (int32_t)blocks - 1) / (int32_t)blocks;
    const int32_t cLo = (int32_t)blockIdx.x * chunk < constraintCount ? (int32_t)blockIdx.x * chunk
                                                                      : constraintCount;
    const int32_t cHi = cLo + chunk < constraintCount ? cLo + chunk : constraintCount;
    if (tid <= M3_GRAPH_COLORS)
    {
        s_colorFill[tid] = 0;
    }
    __syncthreads();
    for (int32_t i = cLo + tid; i < cHi; i += NT)
    {
        atomicAdd(&s_colorFill[cColor[i]], 1);
    }
    __syncthreads();
    if (tid <= M3_GRAPH_COLORS)
    {
        ww[M3_WW_BLOCKCOLOR + blockIdx.x * (M3_GRAPH_COLORS + 1) + tid] = s_colorFill[tid];
    }
    M3_GSYNC()
    if (lead)
    {
        // Colour offsets, then each block's first slot per colour.
        int32_t cursor = 0;
        int32_t used = 0;
        for (int32_t c = 0; c <= M3_GRAPH_COLORS; ++c)
        {
            int32_t n = 0;
            for (uint32_t b = 0; b < blocks; ++b)
            {
                int32_t* cell = &ww[M3_WW_BLOCKCOLOR + b * (M3_GRAPH_COLORS + 1) + c];
                const int32_t v = *cell;
                *cell = cursor + n;
                n += v;
            }
            s.plan->starts[c] = cursor;
            cursor += n;
            used += n > 0 ? 1 : 0;
        }
        s.plan->starts[M3_GRAPH_COLORS + 1] = cursor;
        sc->lastColorCount = used;
        sc->constraintCount = constraintCount;
    }
    M3_GSYNC()
    if (tid <= M3_GRAPH_COLORS)
    {
        s_colorFill[tid] = vww[M3_WW_BLOCKCOLOR + blockIdx.x * (M3_GRAPH_COLORS + 1) + tid];
    }
    __syncthreads();
    {
        const int32_t lane = tid & 31;
        const int32_t warp = tid >> 5;
        const uint32_t ltMask = (1u << lane) - 1u;
        for (int32_t c0 = cLo; c0 < cHi; c0 += NT)
        {
            const int32_t i = c0 + tid;
            const int32_t color = i < cHi ? (int32_t)cColor[i] : M3_GRAPH_COLORS + 1;
            for (int32_t k = tid; k < (NT / 32) * (M3_GRAPH_COLORS + 1); k += NT)
            {
                (&s_warpColor[0][0])[k] = 0;
            }
            __syncthreads();
            const uint32_t peers = __match_any_sync(0xFFFFFFFFu, color);
            const int32_t rank = __popc(peers & ltMask);
            if (rank == 0 && color <= M3_GRAPH_COLORS)
            {
                s_warpColor[warp][color] = __popc(peers);
            }
            __syncthreads();
            if (color <= M3_GRAPH_COLORS)
            {
                int32_t slot = s_colorFill[color] + rank;
                for (int32_t k = 0; k < warp; ++k)
                {
                    slot += s_warpColor[k][color];
                }
                s.lists[slot] = i;
                s.conSlot[i] = slot;
            }
            __syncthreads();
            if (tid <= M3_GRAPH_COLORS)
            {
                int32_t add = 0;
                for (int32_t k = 0; k < NT / 32; ++k)
                {
                    add += s_warpColor[k][tid];
                }
                s_colorFill[tid] += add;
            }
            __syncthreads();
        }
    }
    // The joint/contact schedule: a contact's level is at least one past
    // the last joint level on either of its awake dynamic bodies and one
    // past the level of the previous contact (colour order) on either of
    // them; the overflow colour stays last and serial.
    int32_t* cLast = cMin0;
    for (int32_t i = gtid; i < bodyMax; i += gstride)
    {
        cLast[i] = jointCount > 0 ? s.ready[i] + 1 : 0;
    }
    if (lead)
    {
        ww[M3_WW_CLEVELS] = 0;
    }
    M3_GSYNC()
    for (int32_t color = 0; color < M3_GRAPH_COLORS; ++color)
    {
        const int32_t k0 = s.plan->starts[color];
        const int32_t k1 = s.plan->starts[color + 1];
        for (int32_t k = k0 + gtid; k < k1; k += gstride)
        {
            const int32_t i = s.lists[k];
            const int2 p = cPair[i];
            int32_t level = 0;
            if (p.x >= 0)
            {
                level = cLast[p.x] > level ? cLast[p.x] : level;
            }
            if (p.y >= 0)
            {
                level = cLast[p.y] > level ? cLast[p.y] : level;
            }
            s.conLevel[i] = level;
            if (p.x >= 0)
            {
                cLast[p.x] = level + 1;
            }
            if (p.y >= 0)
            {
                cLast[p.y] = level + 1;
            }
            atomicMax(&ww[M3_WW_CLEVELS], level + 1);
        }
        if (k1 > k0)
        {
            M3_GSYNC()
        }
    }
    const int32_t contactLevels = vww[M3_WW_CLEVELS];
    const int32_t levels = contactLevels > jointLevels ? contactLevels : jointLevels;
    for (int32_t k = gtid; k <= levels + 1; k += gstride)
    {
        s.levelStart[k] = 0;
    }
    M3_GSYNC()
    for (int32_t i = gtid; i < constraintCount; i += gstride)
    {
        const int32_t level = cColor[i] == M3_GRAPH_COLORS ? levels : s.conLevel[i];
        s.conLevel[i] = level;
        atomicAdd(&s.levelStart[level + 1], 1);
    }
    M3_GSYNC()
    if (lead)
    {
        for (int32_t k = 0; k <= levels; ++k)
        {
            s.levelStart[k + 1] += s.levelStart[k];
        }
    }
    M3_GSYNC()
    for (int32_t k = gtid; k <= levels; k += gstride)
    {
        s.levelFill[k] = s.levelStart[k];
    }
    M3_GSYNC()
    for (int32_t i = gtid; i < constraintCount; i += gstride)
    {
        const int32_t level = s.conLevel[i];
        if (level < levels)
        {
            const int32_t slot = atomicAdd(&s.levelFill[level], 1);
            s.lists[slot] = i;
            s.conSlot[i] = slot;
        }
    }
    if (lead && s.levelStart[levels + 1] > s.levelStart[levels])
    {
        // The overflow bucket keeps constraint order (it runs serially).
        int32_t slot = s.levelStart[levels];
        for (int32_t i = 0; i < constraintCount; ++i)
        {
            if (s.conLevel[i] == levels)
            {
                s.lists[slot] = i;
                s.conSlot[i] = slot;
                slot += 1;
            }
        }
    }
    M3_GSYNC()
    M3_WIDE_MARK(M3_PHASE_COLOR)

    // Movers: alive, enabled, kinematic or awake dynamic, ascending
    // (solver.c:3945-3983), with the kinematic servo.
    for (int32_t i = gtid; i < bodyMax; i += gstride)
    {
        int32_t flag = 0;
        if (w.bodyAlive[i] != 0 && w.enabled[i] != 0)
        {
            const uint8_t type = w.btype[i];
            if (type == M3_BODY_KINEMATIC || (type == M3_BODY_DYNAMIC && w.awake[i] != 0))
            {
                flag = 1;
            }
            if (type == M3_BODY_KINEMATIC && w.hasTarget[i] != 0)
            {
                m3real servoInvDt = 1.0f / dt;
                const m3Transform now = w.xf[i];
                const m3Transform want = w.target[i];
                w.v[i] = v3((m3real)(want.p.x - now.p.x) * servoInvDt,
                            (m3real)(want.p.y - now.p.y) * servoInvDt,
                            (m3real)(want.p.z - now.p.z) * servoInvDt);
                m3Quat dq = m3MulQuat(want.q, q4(-now.q.x, -now.q.y, -now.q.z, now.q.w));
                if (dq.w < 0.0f)
                {
                    dq = q4(-dq.x, -dq.y, -dq.z, -dq.w);
                }
                w.w[i] = m3MulSV3(2.0f * servoInvDt, v3(dq.x, dq.y, dq.z));
                w.hasTarget[i] = 0;
            }
        }
        s.moverFlag[i] = flag;
    }
    M3_GSYNC()
    const int32_t moverCount = GridExclusiveScan<NT>(s.moverFlag, bodyMax, ww, bar);
    if (moverCount < 0)
    {
        return;
    }
    for (int32_t i = gtid; i < bodyMax; i += gstride)
    {
        const int32_t next = i + 1 < bodyMax ? s.moverFlag[i + 1] : moverCount;
        if (next != s.moverFlag[i])
        {
            s.movers[s.moverFlag[i]] = i;
        }
    }
    if (lead)
    {
        m3StepPlan* plan = s.plan;
        plan->constraintCount = constraintCount;
        plan->jointCount = jointCount;
        plan->jointLevels = jointLevels;
        plan->moverCount = moverCount;
        plan->anyRestitution = 0; // the rows kernel raises it
        plan->levels = levels;
    }
    M3_WIDE_MARK(M3_PHASE_COLOR)
#undef M3_GSYNC
#undef M3_WIDE_MARK
}

template <int NT>
__global__ void __launch_bounds__(NT, 2) m3WideSubstepKernel(const m3WorldView* views,
                                                           const int32_t* order, float dt,
                                                           int32_t substeps)
{
    const m3WorldView& w = views[order[0]];
    m3WorldScalars* sc = w.sc;
    if (sc->status != 0)
    {
        return;
    }
    m3Scratch s;
    ScratchCarve(&s, w.scratch, sc->bodyCap, sc->shapeCap, sc->jointCap, sc->pairCap);
    uint32_t* bar = s.gridBar;
    const uint32_t blocks = gridDim.x;
    const int32_t tid = threadIdx.x;
    const int32_t gtid = (int32_t)blockIdx.x * NT + tid;
    const int32_t gstride = (int32_t)blocks * NT;
    const bool lead = blockIdx.x == 0 && tid == 0;
    const int32_t constraintCount = s.plan->constraintCount;
    const int32_t jointCount = s.plan->jointCount;
    const int32_t jointLevels = s.plan->jointLevels;
    const int32_t moverCount = s.plan->moverCount;
    const int32_t levels = s.plan->levels;
    const bool anyRestitution = s.plan->anyRestitution != 0;
    m3Manifold* man = sc->pairBuf == 0 ? w.man0 : w.man1;
    const m3real h = dt / (m3real)substeps;
    const m3real invH = h > 0.0f ? 1.0f / h : 0.0f;
    const m3real pushMax = sc->contactPushMaxSpeed;
    m3Vec3* dP = s.deltaPos;
    m3Quat* dQ = s.deltaRot;
    const m3Mat3* invI = s.bodyInvI;
    m3JointDev* jrows = s.joints;
    long long t_phase = clock64();
#define M3_WIDE_MARK(k)                                                                            \
    if (lead)                                                                                      \
    {                                                                                              \
        long long now_ = clock64();                                                                \
        sc->phase[k] += (uint64_t)(now_ - t_phase);                                                \
        t_phase = now_;                                                                            \
    }
    // (The substep deltas were cleared by the prepare kernel.)
    // One pass over the joint/contact schedule: per level, the level's
    // joint rows then its contact rows, over the whole grid; the overflow
    // colour serially.
    auto pass = [&](int32_t which) -> bool {
        for (int32_t level = 0; level < levels; ++level)
        {
            int32_t j0 = 0;
            int32_t nj = 0;
            if (level < jointLevels)
            {
                j0 = s.jointLevelStart[level];
                nj = s.jointLevelStart[level + 1] - j0;
            }
            const int32_t c0 = s.levelStart[level];
            const int32_t nc = s.levelStart[level + 1] - c0;
            for (int32_t r = gtid; r < nj + nc; r += gstride)
            {
                if (r < nj)
                {
                    m3JointDev* row = &jrows[s.jointOrder[j0 + r]];
                    if (which == 0)
                    {
                        m3WarmStartJoint(w, row, dQ);
                    }
                    else
                    {
                        m3SolveJoint(w, row, dP, dQ, h, invH, which == 1);
                    }
                }
                else
                {
                    const m3ConRef c = m3ConAt(s.rows, c0 + (r - nj));
                    if (which == 0)
                    {
                        m3WarmStartContact(w, c, invI);
                    }
                    else
                    {
                        m3SolveContact(w, c, invI, dP, dQ, invH, pushMax, which == 1);
                    }
                }
            }
            if (!m3GridSync(bar, blocks))
            {
                return false;
            }
        }
        const int32_t o0 = s.levelStart[levels];
        const int32_t o1 = s.levelStart[levels + 1];
        if (o1 > o0)
        {
            if (lead)
            {
                for (int32_t k = o0; k < o1; ++k)
                {
                    if (which == 0)
                    {
                        m3WarmStartContact(w, m3ConAt(s.rows, k), invI);
                    }
                    else
                    {
                        m3SolveContact(w, m3ConAt(s.rows, k), invI, dP, dQ, invH, pushMax,
                                       which == 1);
                    }
                }
            }
            if (!m3GridSync(bar, blocks))
            {
                return false;
            }
        }
        return true;
    };
    // The substep loop (solver.c:4085-4203).
    for (int32_t sub = 0; sub < substeps; ++sub)
    {
        for (int32_t m = gtid; m < moverCount; m += gstride)
        {
            const int32_t i = s.movers[m];
            if (w.btype[i] == M3_BODY_DYNAMIC)
            {
                m3IntegrateVelocity(w, i, h);
            }
        }
        if (!m3GridSync(bar, blocks))
        {
            return;
        }
        M3_WIDE_MARK(M3_PHASE_INTEGRATE_V)
        if (!pass(0))
        {
            return;
        }
        M3_WIDE_MARK(M3_PHASE_WARM)
        if (!pass(1))
        {
            return;
        }
        M3_WIDE_MARK(M3_PHASE_SOLVE)
        for (int32_t m = gtid; m < moverCount; m += gstride)
        {
            m3IntegratePosition(w, s.movers[m], h, dP, dQ);
        }
        if (!m3GridSync(bar, blocks))
        {
            return;
        }
        M3_WIDE_MARK(M3_PHASE_INTEGRATE_P)
        if (!pass(2))
        {
            return;
        }
        M3_WIDE_MARK(M3_PHASE_RELAX)
    }
    // Forces live one step (solver.c:4207-4211).
    for (int32_t m = gtid; m < moverCount; m += gstride)
    {
        const int32_t i = s.movers[m];
        w.force[i] = v3(0.0f, 0.0f, 0.0f);
        w.torque[i] = v3(0.0f, 0.0f, 0.0f);
    }
    // Restitution is serial in constraint order (solver.c:2879-2906).
    if (anyRestitution)
    {
        if (lead)
        {
            const m3real threshold = sc->restitutionThreshold;
            for (int32_t i = 0; i < constraintCount; ++i)
            {
                m3RestituteContact(w, m3ConAt(s.rows, s.conSlot[i]), invI, threshold);
            }
        }
        if (!m3GridSync(bar, blocks))
        {
            return;
        }
    }
    for (int32_t i = gtid; i < constraintCount; i += gstride)
    {
        m3StoreContact(m3ConAt(s.rows, i), man);
    }
    {
        const uint64_t* keys = ((volatile int32_t*)&sc->pairBuf)[0] == 0 ? w.keys0 : w.keys1;
        const m3real hitThreshold = sc->hitEventThreshold;
        for (int32_t i = gtid; i < constraintCount; i += gstride)
        {
            s.hitFlag[i] = m3HitCandidate(w, m3ConAt(s.rows, s.conSlot[i]), keys, hitThreshold,
                                          &s.hits[i])
                               ? 1
                               : 0;
        }
    }
    for (int32_t r = gtid; r < jointCount; r += gstride)
    {
        m3StoreJoint(w, &jrows[r]);
    }
    if (!m3GridSync(bar, blocks)) // breakage reads the stored joint impulses
    {
        return;
    }
    // Breakage: each joint's test alone over the grid, the broken ones
    // listed in ascending order (a grid scan of the flags), then destroyed
    // in that order on one thread.
    const int32_t jointMax = sc->jointMax;
    for (int32_t j = gtid; j < jointMax; j += gstride)
    {
        s.jointFlag[j] = m3JointBreaksDev(w, j, invH) ? 1 : 0;
    }
    if (!m3GridSync(bar, blocks))
    {
        return;
    }
    int32_t* ww = s.wideWork;
    const int32_t brokenCount = GridExclusiveScan<NT>(s.jointFlag, jointMax, ww, bar);
    if (brokenCount < 0)
    {
        return;
    }
    for (int32_t j = gtid; j < jointMax; j += gstride)
    {
        const int32_t next = j + 1 < jointMax ? s.jointFlag[j + 1] : brokenCount;
        if (next != s.jointFlag[j])
        {
            s.jointOrder[s.jointFlag[j]] = j;
        }
    }
    if (!m3GridSync(bar, blocks))
    {
        return;
    }
    if (lead)
    {
        sc->lastInvH = invH;
        // Wind phase (solver.c:4220-4229).
        if (sc->windGustHertz > 0.0f)
        {
            sc->windPhase += 2.0f * M3_PI * sc->windGustHertz * dt;
            if (sc->windPhase > 2.0f * M3_PI)
            {
                sc->windPhase -=
                    2.0f * M3_PI * (m3real)(int32_t)(sc->windPhase / (2.0f * M3_PI));
            }
        }
        for (int32_t k = 0; k < brokenCount; ++k)
        {
            m3DestroyBrokenJointDev(w, s.jointOrder[k]);
        }
    }
    M3_WIDE_MARK(M3_PHASE_STORE)
#undef M3_WIDE_MARK
}

// A wide world's contact rows (solver.c:261-405), one per thread over
// the whole grid, straight into the solve slots the prepare kernel
// assigned: the same arithmetic as the per-world kernel's row loop.
__global__ void __launch_bounds__(256) m3WideRowsKernel(const m3WorldView* views,
                                                       const int32_t* order, float dt,
                                                       int32_t substeps)
{
    const m3WorldView& w = views[order[0]];
    m3WorldScalars* sc = w.sc;
    if (sc->status != 0)
    {
        return;
    }
    m3Scratch s;
    ScratchCarve(&s, w.scratch, sc->bodyCap, sc->shapeCap, sc->jointCap, sc->pairCap);
    const uint64_t* keys = sc->pairBuf == 0 ? w.keys0 : w.keys1;
    m3Manifold* man = sc->pairBuf == 0 ? w.man0 : w.man1;
    const m3real h = dt / (m3real)substeps;
    const m3SoftDev soft = m3MakeSoft(sc->contactHertz, sc->contactDampingRatio, h);
    const m3SoftDev staticSoft = m3MakeSoft(2.0f * sc->contactHertz, sc->contactDampingRatio, h);
    const int32_t constraintCount = s.plan->constraintCount;
    for (int32_t slot = blockIdx.x * blockDim.x + threadIdx.x; slot < constraintCount;
         slot += gridDim.x * blockDim.x)
    {
        m3ContactDev c;
        m3PrepareContact(w, &c, s.conPairIndex[s.lists[slot]], keys, man, soft, staticSoft,
                         s.bodyInvI);
        m3WriteContactRow(s.rows, slot, c);
        if (c.restitution != 0.0f)
        {
            atomicOr(&s.plan->anyRestitution, 1);
        }
        if (c.rollingResistance > 0.0f && (!c.dynA || !c.dynB))
        {
            atomicExch(&sc->status, M3GPU_ERR_UNSUPPORTED);
            sc->statusDetail = 2001;
        }
    }
}

// A barrier that gave up marks the world failed (after the wide kernel,
// one thread).
__global__ void m3WideStatusKernel(const m3WorldView* views, const int32_t* order)
{
    const m3WorldView& w = views[order[0]];
    m3Scratch s;
    ScratchCarve(&s, w.scratch, w.sc->bodyCap, w.sc->shapeCap, w.sc->jointCap, w.sc->pairCap);
    if (s.gridBar[2] != 0 && w.sc->status == 0)
    {
        w.sc->status = M3GPU_ERR_CUDA;
        w.sc->statusDetail = 7001;
    }
}

// A bullet's sweep against the moving bodies (solver.c:3237-3270 with
// the non-static branch): every alive, enabled, non-bullet, non-sensor
// shape of another non-static body whose current tree leaf (the
// broadphase's copy, refreshed this step) touches the swept box
// [lo, hi] and that the filters let through, swept with the target's own
// motion.  The reference visits bodies in ascending order, so a target
// below the bullet shows its pose after its own pull-back and one above
// it its pose before; bullets never sweep against bullets.  Counts the
// hits below `limit` like SweepStaticTargets and leaves the last one's
// fraction in *hitFraction.
__device__ __noinline__ int32_t SweepMovingTargets(const m3WorldView& w, const m3Scratch& s,
                                                   int32_t bullet, int32_t sh, const double* lo,
                                                   const double* hi, const m3Pos3& base,
                                                   const m3ProxyDev& proxyB,
                                                   const m3SweepDev& fastSweep, m3real limit,
                                                   m3real* hitFraction)
{
    int32_t hits = 0;
    const int32_t shapeMax = w.sc->shapeMax;
    for (int32_t o = 0; o < shapeMax; ++o)
    {
        if (w.shapeAlive[o] == 0 || w.shapeType[o] == M3_SHAPE_PLANE || o == sh ||
            s.hasLeaf[o] == 0 || w.sensor[o] != 0)
        {
            continue;
        }
        const int32_t ob = w.shapeBody[o];
        if (ob == bullet || w.btype[ob] == M3_BODY_STATIC || w.enabled[ob] == 0 ||
            w.bullet[ob] != 0)
        {
            continue;
        }
        const m3Aabb& leaf = s.leafBox[o];
        if (!(leaf.lo[0] <= hi[0] && lo[0] <= leaf.hi[0] && leaf.lo[1] <= hi[1] &&
              lo[1] <= leaf.hi[1] && leaf.lo[2] <= hi[2] && lo[2] <= leaf.hi[2]))
        {
            continue;
        }
        const int32_t gi = w.group[o];
        if (gi != 0 && gi == w.group[sh])
        {
            if (gi < 0)
            {
                continue;
            }
        }
        else if (!((w.category[o] & w.mask[sh]) != 0 && (w.category[sh] & w.mask[o]) != 0))
        {
            continue;
        }
        m3Vec3 scratchA[2];
        m3ProxyDev proxyA;
        proxyA.count = ProxyPoints(w, o, &proxyA.points, scratchA, &proxyA.radius);
        const m3Pos3 oc0 = s.com0[ob];
        const m3Transform oxf = (ob > bullet && s.pulled[ob] != 0) ? s.xfPre[ob] : w.xf[ob];
        const m3Vec3 orlc = m3RotateVec3(oxf.q, w.lc[ob]);
        m3SweepDev sweepA;
        sweepA.localCenter = w.lc[ob];
        sweepA.c1 = v3((m3real)(oc0.x - base.x), (m3real)(oc0.y - base.y),
                       (m3real)(oc0.z - base.z));
        sweepA.c2 = v3((m3real)(oxf.p.x + (double)orlc.x - base.x),
                       (m3real)(oxf.p.y + (double)orlc.y - base.y),
                       (m3real)(oxf.p.z + (double)orlc.z - base.z));
        sweepA.q1 = s.rot0[ob];
        sweepA.q2 = oxf.q;
        int32_t state;
        const m3real t = m3TimeOfImpactDev(proxyA, sweepA, proxyB, fastSweep, limit, &state);
        if (state == M3_TOI_HIT && 0.0f < t && t < limit)
        {
            hits += 1;
            *hitFraction = t;
        }
    }
    return hits;
}

// ---------------------------------------------------------------------
// The tree arm of the continuous phase for one shape of a fast body
// (solver.c:3081-3274): every static target whose tree leaf touches the
// swept box [lo, hi], swept by the time of impact bounded by `*fraction`.
// Returns how many targets hit before `*fraction`; with exactly one,
// `*fraction` becomes its fraction.  `*refusal` is set for a mesh or
// voxel target.
__device__ __noinline__ int32_t SweepStaticTargets(const m3WorldView& w, const m3Pos3* com0,
                                                   const m3Quat* rot0, int32_t i, int32_t sh,
                                                   const int32_t* targets, int32_t targetCount,
                                                   const double* lo,
                                                   const double* hi, const m3Pos3& base,
                                                   const m3ProxyDev& proxyB,
                                                   const m3SweepDev& fastSweep, m3real* fraction,
                                                   int32_t* refusal)
{
    const m3real limit = *fraction;
    int32_t hits = 0;
    m3real hitFraction = limit;
    // `targets` lists, ascending, the alive non-plane shapes of static
    // bodies: the only shapes the checks below can let through.
    for (int32_t n = 0; n < targetCount; ++n)
    {
        const int32_t o = targets[n];
        if (w.shapeAlive[o] == 0 || w.shapeType[o] == M3_SHAPE_PLANE || o == sh ||
            w.proxyId[o] == M3_TREE_NULL)
        {
            continue;
        }
        const int32_t ob = w.shapeBody[o];
        if (ob == i || w.enabled[ob] == 0 || w.bullet[ob] != 0 || w.sensor[o] != 0)
        {
            continue;
        }
        // Only bullets sweep against moving bodies.  (The reference tests
        // this after the mesh and voxel cases; those shapes live on static
        // bodies only, so testing it first, before the leaf is read,
        // changes nothing.)
        if (w.btype[ob] != M3_BODY_STATIC)
        {
            continue;
        }
        const m3TreeNode& leaf = w.treeNodes[w.proxyId[o]];
        if (!(leaf.lo[0] <= hi[0] && lo[0] <= leaf.hi[0] && leaf.lo[1] <= hi[1] &&
              lo[1] <= leaf.hi[1] && leaf.lo[2] <= hi[2] && lo[2] <= leaf.hi[2]))
        {
            continue;
        }
        if (w.shapeType[o] == M3_SHAPE_MESH || w.shapeType[o] == M3_SHAPE_VOXEL)
        {
            *refusal = 3003;
            continue;
        }
        const int32_t gi = w.group[o];
        if (gi != 0 && gi == w.group[sh])
        {
            if (gi < 0)
            {
                continue;
            }
        }
        else if (!((w.category[o] & w.mask[sh]) != 0 &&
                   (w.category[sh] & w.mask[o]) != 0))
        {
            continue;
        }
        m3Vec3 scratchA[2];
        m3ProxyDev proxyA;
        proxyA.count = ProxyPoints(w, o, &proxyA.points, scratchA, &proxyA.radius);
        // The target's sweep relative to the fast body's base
        // (solver.c:3065-3079).
        const m3Pos3 oc0 = com0[ob];
        const m3Transform oxf = w.xf[ob];
        const m3Vec3 orlc = m3RotateVec3(oxf.q, w.lc[ob]);
        m3SweepDev sweepA;
        sweepA.localCenter = w.lc[ob];
        sweepA.c1 = v3((m3real)(oc0.x - base.x), (m3real)(oc0.y - base.y),
                       (m3real)(oc0.z - base.z));
        sweepA.c2 = v3((m3real)(oxf.p.x + (double)orlc.x - base.x),
                       (m3real)(oxf.p.y + (double)orlc.y - base.y),
                       (m3real)(oxf.p.z + (double)orlc.z - base.z));
        sweepA.q1 = rot0[ob];
        sweepA.q2 = oxf.q;
        int32_t state;
        const m3real t =
            m3TimeOfImpactDev(proxyA, sweepA, proxyB, fastSweep, limit, &state);
        if (state == M3_TOI_HIT && 0.0f < t && t < limit)
        {
            hits += 1;
            hitFraction = t;
        }
    }
    if (hits == 1)
    {
        *fraction = hitFraction;
    }
    return hits;
}

// Kernel 4: continuous collision against planes and the sleep pass
// ---------------------------------------------------------------------
__global__ void __launch_bounds__(M3_BLOCK, 2) m3FinishKernel(const m3WorldView* views,
                                                           const int32_t* order, int32_t count,
                                                           float dt, int32_t substeps)
{
    const int32_t wi = order[blockIdx.x];
    const m3WorldView& w = views[wi];
    m3WorldScalars* sc = w.sc;
    if (sc->status != 0)
    {
        return;
    }
    long long t_phase = clock64();
    m3Scratch s;
    ScratchCarve(&s, w.scratch, sc->bodyCap, sc->shapeCap, sc->jointCap, sc->pairCap);
    const int32_t tid = threadIdx.x;
    __shared__ int32_t s_status;
    if (tid == 0)
    {
        s_status = 0;
    }
    __syncthreads();
    const int32_t bodyMax = sc->bodyMax;
    const int32_t shapeMax = sc->shapeMax;
    const int32_t pairCount = sc->pairCount;
    const int32_t constraintCount = s.plan->constraintCount;
    const int32_t moverCount = s.plan->moverCount;
    // Continuous phase (solver.c:3349-3425).  A non-bullet fast body
    // sweeps only against static targets, and a pull-back moves only the
    // fast body itself, so those bodies are independent and run in
    // parallel.  Bullets follow, also in parallel (they never sweep
    // against one another), each seeing every moving target as the
    // reference's ascending walk would.  Tree targets and then planes are
    // swept per shape; a mesh or voxel target, or two tree hits for one
    // shape (whose order would matter), are refused.
    if (sc->continuousEnabled != 0)
    {
        // The targets, once per step and ascending: the static non-plane
        // shapes (the tree arm's only candidates) and the planes (at most
        // M3_MAX_PLANES: the broadphase refuses more).  Without a static
        // target the tree arm finds nothing, and fast bodies meet only
        // planes.
        __shared__ int32_t s_planeList[M3_MAX_PLANES];
        __shared__ int32_t s_planeCount;
        if (tid == 0)
        {
            s_planeCount = 0;
        }
        __syncthreads();
        for (int32_t o = tid; o < shapeMax; o += M3_BLOCK)
        {
            int32_t flag = 0;
            if (w.shapeAlive[o] != 0)
            {
                if (w.shapeType[o] == M3_SHAPE_PLANE)
                {
                    const int32_t k = atomicAdd(&s_planeCount, 1);
                    if (k < M3_MAX_PLANES)
                    {
                        s_planeList[k] = o;
                    }
                }
                else if (w.btype[w.shapeBody[o]] == M3_BODY_STATIC)
                {
                    flag = 1;
                }
            }
            s.staticList[o] = flag;
        }
        __syncthreads();
        if (tid == 0)
        {
            // Planes in ascending shape order (the reference's scan).
            const int32_t n = s_planeCount < M3_MAX_PLANES ? s_planeCount : M3_MAX_PLANES;
            for (int32_t a = 1; a < n; ++a)
            {
                const int32_t v = s_planeList[a];
                int32_t b = a - 1;
                while (b >= 0 && s_planeList[b] > v)
                {
                    s_planeList[b + 1] = s_planeList[b];
                    b -= 1;
                }
                s_planeList[b + 1] = v;
            }
            s_planeCount = n;
        }
        const int32_t targetCount = BlockExclusiveScan<M3_BLOCK>(s.staticList, shapeMax);
        int32_t* targets = s.targetList;
        for (int32_t o = tid; o < shapeMax; o += M3_BLOCK)
        {
            const int32_t next = o + 1 < shapeMax ? s.staticList[o + 1] : targetCount;
            if (next != s.staticList[o])
            {
                targets[s.staticList[o]] = o;
            }
        }
        __syncthreads();
        const bool staticTargets = targetCount > 0;
        const int32_t planeCount = s_planeCount;
        for (int32_t i = tid; i < bodyMax; i += M3_BLOCK)
        {
            s.pulled[i] = 0;
        }
        __syncthreads();
        // Two passes: the non-bullets (independent of one another), then
        // the bullets, which also sweep against moving bodies and must see
        // each target as the reference's ascending walk leaves it.
        for (int32_t pass = 0; pass < 2; ++pass)
        {
            if (pass == 1)
            {
                __syncthreads();
            }
            for (int32_t i = tid; i < bodyMax; i += M3_BLOCK)
            {
                if (w.bodyAlive[i] == 0 || w.btype[i] != M3_BODY_DYNAMIC ||
                    (w.bullet[i] != 0) != (pass == 1))
                {
                    continue;
                }
                const m3Transform xfEnd = w.xf[i];
                m3Vec3 rlc = m3RotateVec3(xfEnd.q, w.lc[i]);
                double cx = xfEnd.p.x + (double)rlc.x;
                double cy = xfEnd.p.y + (double)rlc.y;
                double cz = xfEnd.p.z + (double)rlc.z;
                const m3Pos3 c0 = s.com0[i];
                m3Vec3 dc = v3((m3real)(cx - c0.x), (m3real)(cy - c0.y), (m3real)(cz - c0.z));
                m3Quat q0 = s.rot0[i];
                m3Quat dq = m3MulQuat(xfEnd.q, q4(-q0.x, -q0.y, -q0.z, q0.w));
                m3real arc = 2.0f * sqrtf(dq.x * dq.x + dq.y * dq.y + dq.z * dq.z) * w.maxExt[i];
                m3real maxMotion = sqrtf(m3Dot3(dc, dc)) + arc;
                if (!(maxMotion > 0.5f * w.minExt[i]))
                {
                    continue;
                }
                if (pass == 1 && sc->treeTracked == 0)
                {
                    // A world that keeps no tree keeps no leaf boxes to query.
                    s_status = M3GPU_ERR_UNSUPPORTED;
                    sc->statusDetail = 3001;
                    continue;
                }
                // Relative sweep about the begin centre (MakeRelativeSweep).
                const m3Pos3 base = c0;
                const m3Vec3 lc = w.lc[i];
                const m3Vec3 sc1 = v3((m3real)(c0.x - base.x), (m3real)(c0.y - base.y),
                                      (m3real)(c0.z - base.z));
                const m3Vec3 sc2 = v3((m3real)(xfEnd.p.x + (double)rlc.x - base.x),
                                      (m3real)(xfEnd.p.y + (double)rlc.y - base.y),
                                      (m3real)(xfEnd.p.z + (double)rlc.z - base.z));
                m3real fraction = 1.0f;
                double pad = (double)(w.maxExt[i] + M3_AABB_MARGIN);
                double lo[3] = {(c0.x < cx ? c0.x : cx) - pad, (c0.y < cy ? c0.y : cy) - pad,
                                (c0.z < cz ? c0.z : cz) - pad};
                double hi[3] = {(c0.x > cx ? c0.x : cx) + pad, (c0.y > cy ? c0.y : cy) + pad,
                                (c0.z > cz ? c0.z : cz) + pad};
                m3SweepDev fastSweep;
                fastSweep.localCenter = lc;
                fastSweep.c1 = sc1;
                fastSweep.c2 = sc2;
                fastSweep.q1 = q0;
                fastSweep.q2 = xfEnd.q;
                for (int32_t sh = w.shapeHead[i]; sh != -1; sh = w.shapeNext[sh])
                {
                    if (w.sensor[sh] != 0)
                    {
                        continue;
                    }
                    // The tree query (solver.c:3081-3274): static targets whose
                    // tree leaf touches the swept box, each swept by the time
                    // of impact.  Static leaves never move, so their boxes are
                    // read straight from the tree.  The reference visits them
                    // in tree order, each call bounded by the fraction so far;
                    // with one hit the order does not matter (every target
                    // sees the fraction of the earlier shapes), with two or
                    // more it would, and the world is refused.
                    m3Vec3 scratchB[2];
                    m3ProxyDev proxyB;
                    proxyB.count = ProxyPoints(w, sh, &proxyB.points, scratchB, &proxyB.radius);
                    int32_t refusal = 0;
                    const m3real entry = fraction;
                    int32_t hits =
                        staticTargets ? SweepStaticTargets(w, s.com0, s.rot0, i, sh, targets,
                                                           targetCount, lo, hi, base, proxyB,
                                                           fastSweep, &fraction, &refusal)
                                      : 0;
                    if (pass == 1)
                    {
                        // A bullet's moving targets, bounded by the same entry
                        // fraction: with one hit in all, the order is moot.
                        m3real moving = entry;
                        const int32_t movingHits = SweepMovingTargets(w, s, i, sh, lo, hi, base,
                                                                      proxyB, fastSweep, entry,
                                                                      &moving);
                        if (movingHits == 1 && hits == 0)
                        {
                            fraction = moving;
                        }
                        hits += movingHits;
                    }
                    if (refusal != 0)
                    {
                        s_status = M3GPU_ERR_UNSUPPORTED;
                        sc->statusDetail = refusal;
                    }
                    if (hits > 1)
                    {
                        s_status = M3GPU_ERR_UNSUPPORTED;
                        sc->statusDetail = 3002;
                    }
                    for (int32_t k = 0; k < planeCount; ++k)
                    {
                        ContinuousVersusPlane(w, i, sh, s_planeList[k], base, lc, sc1, sc2, q0,
                                              xfEnd.q, &fraction);
                    }
                }
                if (fraction < 1.0f)
                {
                    m3Transform xf = SweepTransform(lc, sc1, sc2, q0, xfEnd.q, fraction);
                    m3Transform out;
                    out.q = xf.q;
                    out.p.x = base.x + xf.p.x;
                    out.p.y = base.y + xf.p.y;
                    out.p.z = base.z + xf.p.z;
                    s.xfPre[i] = xfEnd;
                    s.pulled[i] = 1;
                    w.xf[i] = out;
                }
            }
        }
        __syncthreads();
        if (s_status != 0)
        {
            if (tid == 0)
            {
                sc->status = s_status;
            }
            return;
        }
    }

    M3_PHASE_MARK(M3_PHASE_CONTINUOUS)
    // Sleep pass (solver.c:3582-3660).
    if (sc->sleepEnabled != 0)
    {
        const m3real invDt = dt > 0.0f ? 1.0f / dt : 0.0f;
        for (int32_t i = tid; i < bodyMax; i += M3_BLOCK)
        {
            s.ready[i] = 1;
            if (w.bodyAlive[i] == 0 || w.btype[i] != M3_BODY_DYNAMIC || w.awake[i] == 0)
            {
                continue;
            }
            m3Vec3 v = w.v[i];
            m3Vec3 om = w.w[i];
            m3real velocity = sqrtf(m3Dot3(v, v)) + sqrtf(m3Dot3(om, om)) * w.maxExt[i];
            const m3Transform xf = w.xf[i];
            m3Vec3 rlc = m3RotateVec3(xf.q, w.lc[i]);
            const m3Pos3 c0 = s.com0[i];
            m3Vec3 dc = v3((m3real)(xf.p.x + (double)rlc.x - c0.x),
                           (m3real)(xf.p.y + (double)rlc.y - c0.y),
                           (m3real)(xf.p.z + (double)rlc.z - c0.z));
            m3Quat q0 = s.rot0[i];
            m3Quat dq = m3MulQuat(xf.q, q4(-q0.x, -q0.y, -q0.z, q0.w));
            m3real motion = sqrtf(m3Dot3(dc, dc)) +
                            2.0f * sqrtf(dq.x * dq.x + dq.y * dq.y + dq.z * dq.z) * w.maxExt[i];
            m3real sleepVelocity = m3MaxF(velocity, 0.5f * invDt * motion);
            if (w.canSleep[i] == 0)
            {
                sleepVelocity = 3.4e38f;
            }
            if (sleepVelocity < w.sleepThreshold[i])
            {
                w.sleepTime[i] += dt;
            }
            else
            {
                w.sleepTime[i] = 0.0f;
            }
        }
        __syncthreads();
        for (int32_t i = tid; i < bodyMax; i += M3_BLOCK)
        {
            if (w.bodyAlive[i] == 0 || w.btype[i] != M3_BODY_DYNAMIC || w.awake[i] == 0)
            {
                continue;
            }
            if (w.sleepTime[i] < M3_TIME_TO_SLEEP)
            {
                s.ready[IslandFind(s.parent, i)] = 0;
            }
        }
        __syncthreads();
        for (int32_t i = tid; i < bodyMax; i += M3_BLOCK)
        {
            if (w.bodyAlive[i] == 0 || w.btype[i] != M3_BODY_DYNAMIC || w.awake[i] == 0)
            {
                continue;
            }
            if (s.ready[IslandFind(s.parent, i)] != 0)
            {
                w.awake[i] = 0;
                w.v[i] = v3(0.0f, 0.0f, 0.0f);
                w.w[i] = v3(0.0f, 0.0f, 0.0f);
            }
        }
        __syncthreads();
    }
    if (tid == 0)
    {
        M3_PHASE_MARK(M3_PHASE_SLEEP)
        sc->moverCount = moverCount;
        sc->stepCount += 1;
        sc->work[0] += (uint64_t)moverCount * (uint64_t)substeps;
        sc->work[1] += (uint64_t)constraintCount * (uint64_t)substeps;
        sc->work[2] += (uint64_t)sc->jointConstraintCount * (uint64_t)substeps;
        sc->work[3] += (uint64_t)pairCount;
        sc->work[4] += 1;
    }
}

// Largest status word over the batch (0 when every world stepped).
__global__ void m3StatusKernel(const m3WorldView* views, int32_t count, int32_t* out)
{
    int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count)
    {
        int32_t st = views[i].sc->status;
        if (st != 0)
        {
            atomicMax(out, st);
        }
    }
}

// ---------------------------------------------------------------------
// Host launch
// ---------------------------------------------------------------------
static int64_t s_launches = 0;
static float s_lastStepMs = 0.0f;

extern "C" int64_t m3gpu_launch_count(void)
{
    return s_launches;
}

extern "C" float m3gpu_last_step_ms(void)
{
    return s_lastStepMs;
}

extern "C" int32_t m3gpu_synchronize(void)
{
    M3_DEVICE_GUARD;
    if (m3gpuEnsureDevice() != M3GPU_OK)
    {
        return m3gpu_last_error();
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
    {
        return m3gpuSetError(M3GPU_ERR_CUDA, "synchronize: %s", cudaGetErrorString(e));
    }
    return M3GPU_OK;
}

// Device copies of the world views and the largest-first launch order,
// cached across calls while the batch stays the same.
struct m3BatchCache
{
    std::vector<m3HostWorld*> worlds;
    uint64_t epoch = 0;
    int32_t cacheBytes = 0;
    m3WorldView* dviews = nullptr;
    int32_t* dorder = nullptr;
    int32_t* doffsets = nullptr;
    uint64_t* dhash = nullptr;
    int32_t cap = 0;
    // Pair-family buckets of the flattened pairs: per-block counts and
    // family offsets, and the bucket array (capacity: the batch's total
    // pair capacity).
    int32_t* dfamily = nullptr; // blockHist[M3_FAMILY_BLOCKS * M3F_COUNT], famStart[M3F_COUNT + 1]
    int32_t* dbucket = nullptr;
    int64_t bucketCap = 0;
    // Substep size classes: order[classFirst[c] .. classFirst[c + 1]) and
    // each class's dynamic shared memory.
    int32_t classFirst[4] = {0, 0, 0, 0};
    int32_t classCache[3] = {0, 0, 0};
    // Each class's kernel variant (0: 512 threads, 1: 256, 2: 128), the
    // largest-first order on the host, and the packing they came from.
    int32_t classVariant[3] = {0, 1, 2};
    std::vector<int32_t> horder;
    uint64_t packingSeq = 0;
};
static m3BatchCache s_batch;

static int32_t Check(cudaError_t e, const char* what)
{
    if (e != cudaSuccess)
    {
        return m3gpuSetError(M3GPU_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    }
    return M3GPU_OK;
}

// Substep size classes: a world's threads follow its size (shape slots;
// the batch order is by shape slots, largest first, so each class is a
// contiguous run of the order).  By default large worlds get 512
// threads: twice the rows per colour in flight and half as many worlds
// resident at once, whose rows then stay in L2 across the passes.  Small
// worlds get 128: four worlds share an SM instead of two, hiding each
// other's joint chains, with one warp for a level's joint rows and three
// for its contact rows.  Every variant keeps 128 registers per thread.
// The split, each class's variant and its shared-memory budget form the
// packing (m3gpu_set_packing, m3gpu_autotune_packing).
#define M3_CLASSES 3
static m3gpuPacking s_packing = {{769, 161},
                                 {512, 256, 128},
                                 {200 * 1024, M3_TWO_BLOCK_SMEM, 54 * 1024}};
// Bumped by every change of the packing: a prepared batch then splits
// its classes again before its next step.
static uint64_t s_packingSeq = 1;

static int32_t VariantOfThreads(int32_t threads)
{
    return threads >= 512 ? 0 : threads >= 256 ? 1 : 2;
}

// One variant's prepare (stage 0) or substep (stage 1) kernel: variant 0
// runs 512 threads per world, 1 runs 256, 2 runs 128.
static void LaunchClass(int32_t stage, int32_t c, cudaStream_t stream, const m3WorldView* views,
                        const int32_t* order, int32_t count, float dt, int32_t substeps,
                        int32_t cacheBytes)
{
    if (count <= 0)
    {
        return;
    }
#define M3_LAUNCH_CLASS(NT, MB)                                                                    \
    if (stage == 0)                                                                                \
    {                                                                                              \
        m3PrepareKernel<NT, MB><<<count, NT, cacheBytes, stream>>>(views, order, count, dt,       \
                                                                   substeps, cacheBytes);          \
    }                                                                                              \
    else                                                                                           \
    {                                                                                              \
        m3SubstepKernel<NT, MB><<<count, NT, cacheBytes, stream>>>(views, order, count, dt,       \
                                                                   substeps, cacheBytes);          \
    }
    if (c == 0)
    {
        M3_LAUNCH_CLASS(512, 1)
    }
    else if (c == 1)
    {
        M3_LAUNCH_CLASS(256, 2)
    }
    else
    {
        M3_LAUNCH_CLASS(128, 4)
    }
#undef M3_LAUNCH_CLASS
}

// The dynamic shared memory each variant's kernels were last allowed
// (0: never set, the default of 48 KB for static and dynamic together).
static int32_t s_classSmemSet[M3_CLASSES] = {0, 0, 0};

static int32_t SetClassSmem(int32_t c, int32_t bytes)
{
    cudaError_t e = cudaSuccess;
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if (c == 0)
    {
        e = cudaFuncSetAttribute(m3PrepareKernel<512, 1>, a, bytes);
        if (e == cudaSuccess)
        {
            e = cudaFuncSetAttribute(m3SubstepKernel<512, 1>, a, bytes);
        }
    }
    else if (c == 1)
    {
        e = cudaFuncSetAttribute(m3PrepareKernel<256, 2>, a, bytes);
        if (e == cudaSuccess)
        {
            e = cudaFuncSetAttribute(m3SubstepKernel<256, 2>, a, bytes);
        }
    }
    else
    {
        e = cudaFuncSetAttribute(m3PrepareKernel<128, 4>, a, bytes);
        if (e == cudaSuccess)
        {
            e = cudaFuncSetAttribute(m3SubstepKernel<128, 4>, a, bytes);
        }
    }
    if (e != cudaSuccess)
    {
        return m3gpuSetError(M3GPU_ERR_CUDA, "cudaFuncSetAttribute(class smem): %s",
                             cudaGetErrorString(e));
    }
    s_classSmemSet[c] = bytes;
    return M3GPU_OK;
}

// Allows a class's kernels `bytes` of dynamic shared memory, raising the
// limit when a launch needs more than it was last set to.  Always set,
// never left to the default: the default's 48 KB covers the kernels'
// static shared memory too, so a launch just under 48 KB of dynamic
// shared memory would not fit it.
static int32_t EnsureClassSmem(int32_t c, int32_t bytes)
{
    return bytes > s_classSmemSet[c] ? SetClassSmem(c, bytes) : M3GPU_OK;
}

// Streams for the classes (they run side by side), and the events that
// fork them off the default stream after the prepare kernel and join
// them back before the finish kernel.
struct m3ClassStreams
{
    int device = -1;
    cudaStream_t stream[M3_CLASSES] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[M3_CLASSES] = {};
    // The broadphase tree's stream (its launches' events are a ring by
    // launch, below).
    cudaStream_t tree = nullptr;
};
static m3ClassStreams s_classStreams;

static int32_t EnsureClassStreams()
{
    int device = 0;
    cudaGetDevice(&device);
    if (s_classStreams.device == device)
    {
        return M3GPU_OK;
    }
    cudaError_t e = cudaEventCreateWithFlags(&s_classStreams.fork, cudaEventDisableTiming);
    for (int32_t c = 0; e == cudaSuccess && c < M3_CLASSES; ++c)
    {
        e = cudaStreamCreateWithFlags(&s_classStreams.stream[c], cudaStreamNonBlocking);
        if (e == cudaSuccess)
        {
            e = cudaEventCreateWithFlags(&s_classStreams.join[c], cudaEventDisableTiming);
        }
    }
    if (e == cudaSuccess)
    {
        // Default priority: the tree's blocks then take SMs as the step's
        // kernels free them instead of waiting for idle SMs, which a busy
        // batch never leaves.
        e = cudaStreamCreateWithFlags(&s_classStreams.tree, cudaStreamNonBlocking);
    }
    if (e != cudaSuccess)
    {
        return m3gpuSetError(M3GPU_ERR_CUDA, "class streams: %s", cudaGetErrorString(e));
    }
    s_classStreams.device = device;
    return M3GPU_OK;
}

// Size classes over the batch's largest-first order under the packing in
// use, and each class's shared memory: its largest body cache, plus the
// inverse inertia table and the joint rows within the class's budget
// (the default budgets keep one 512-thread block, two 256-thread blocks
// or four 128-thread blocks per SM); a budget of 0 keeps every table in
// global memory.
static int32_t ClassifyBatch()
{
    const int64_t limit = 200 * 1024;
    const int32_t count = (int32_t)s_batch.worlds.size();
    const std::vector<int32_t>& order = s_batch.horder;
    m3HostWorld* const* worlds = s_batch.worlds.data();
    const int32_t minShapes[M3_CLASSES] = {s_packing.minShapes[0], s_packing.minShapes[1], 0};
    int32_t c = 0;
    s_batch.classFirst[0] = 0;
    for (int32_t k = 0; k < count; ++k)
    {
        const int32_t shapes = worlds[order[(size_t)k]]->hv.sc->shapeMax;
        while (c < M3_CLASSES - 1 && shapes < minShapes[c])
        {
            s_batch.classFirst[++c] = k;
        }
    }
    while (c < M3_CLASSES)
    {
        s_batch.classFirst[++c] = count;
    }
    int32_t rc = M3GPU_OK;
    for (int32_t k = 0; rc == M3GPU_OK && k < M3_CLASSES; ++k)
    {
        int64_t cBodies = 0;
        int64_t cWant = 0;
        for (int32_t j = s_batch.classFirst[k]; j < s_batch.classFirst[k + 1]; ++j)
        {
            const m3WorldScalars* sc = worlds[order[(size_t)j]]->hv.sc;
            const int64_t bodies = (int64_t)sc->bodyMax * M3_BODY_CACHE_BYTES;
            const int64_t withTables =
                m3AlignUp(m3AlignUp(bodies, 16) + (int64_t)sc->bodyMax * (int64_t)sizeof(m3Mat3),
                          16) +
                (int64_t)sc->jointMax * (int64_t)sizeof(m3JointDev);
            cBodies = bodies > cBodies ? bodies : cBodies;
            cWant = withTables > cWant ? withTables : cWant;
        }
        const int64_t budget = s_packing.smemBytes[k];
        const int64_t cap = cBodies > budget ? cBodies : budget;
        cWant = cWant < cap ? cWant : cap;
        cWant = cWant < limit ? cWant : limit;
        cWant = budget == 0 ? 0 : cWant;
        const int32_t variant = VariantOfThreads(s_packing.threads[k]);
        s_batch.classCache[k] = (int32_t)cWant;
        s_batch.classVariant[k] = variant;
        rc = EnsureClassSmem(variant, (int32_t)cWant);
    }
    if (rc == M3GPU_OK)
    {
        s_batch.packingSeq = s_packingSeq;
    }
    return rc;
}

static int32_t PrepareBatch(m3HostWorld** worlds, int32_t count)
{
    std::vector<m3HostWorld*> dirty;
    for (int32_t i = 0; i < count; ++i)
    {
        m3HostWorld* w = worlds[i];
        if (w->hostDirty || w->dslab == nullptr)
        {
            w->hv.sc->status = 0;
            dirty.push_back(w);
        }
    }
    if (!dirty.empty())
    {
        int32_t rc = m3gpuUploadBatch(dirty.data(), (int32_t)dirty.size());
        if (rc != M3GPU_OK)
        {
            return rc;
        }
    }
    bool same = s_batch.dviews != nullptr && s_batch.epoch == g_m3ResidencyEpoch &&
                (int32_t)s_batch.worlds.size() == count;
    for (int32_t i = 0; same && i < count; ++i)
    {
        same = s_batch.worlds[(size_t)i] == worlds[i];
    }
    if (same)
    {
        // The same batch: split again only under a new packing.
        return s_batch.packingSeq == s_packingSeq ? M3GPU_OK : ClassifyBatch();
    }
    if (count > s_batch.cap)
    {
        cudaFree(s_batch.dviews);
        cudaFree(s_batch.dorder);
        cudaFree(s_batch.dhash);
        cudaFree(s_batch.doffsets);
        s_batch.doffsets = nullptr;
        s_batch.dviews = nullptr;
        s_batch.dorder = nullptr;
        s_batch.dhash = nullptr;
        int32_t rc = Check(cudaMalloc((void**)&s_batch.dviews, sizeof(m3WorldView) * (size_t)count),
                           "cudaMalloc(views)");
        if (rc == M3GPU_OK)
        {
            rc = Check(cudaMalloc((void**)&s_batch.dorder, sizeof(int32_t) * (size_t)count),
                       "cudaMalloc(order)");
        }
        if (rc == M3GPU_OK)
        {
            rc = Check(cudaMalloc((void**)&s_batch.dhash, sizeof(uint64_t) * (size_t)count),
                       "cudaMalloc(hash)");
        }
        if (rc == M3GPU_OK)
        {
            rc = Check(cudaMalloc((void**)&s_batch.doffsets, sizeof(int32_t) * (size_t)(count + 1)),
                       "cudaMalloc(offsets)");
        }
        if (rc != M3GPU_OK)
        {
            s_batch.cap = 0;
            return rc;
        }
        s_batch.cap = count;
    }
    std::vector<m3WorldView> views((size_t)count);
    std::vector<int32_t> order((size_t)count);
    for (int32_t i = 0; i < count; ++i)
    {
        m3AttachDevicePools(worlds[i], &worlds[i]->dv);
        views[(size_t)i] = worlds[i]->dv;
        order[(size_t)i] = i;
    }
    // Largest first: the per-world work grows with bodies and pairs.
    std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
        return worlds[a]->hv.sc->shapeMax > worlds[b]->hv.sc->shapeMax;
    });
    int32_t rc = Check(cudaMemcpy(s_batch.dviews, views.data(), sizeof(m3WorldView) * (size_t)count,
                                  cudaMemcpyHostToDevice),
                       "upload views");
    if (rc == M3GPU_OK)
    {
        rc = Check(cudaMemcpy(s_batch.dorder, order.data(), sizeof(int32_t) * (size_t)count,
                              cudaMemcpyHostToDevice),
                   "upload order");
    }
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    int64_t pairTotal = 0;
    for (int32_t i = 0; i < count; ++i)
    {
        pairTotal += worlds[i]->pairCap;
    }
    if (s_batch.dfamily == nullptr)
    {
        rc = Check(cudaMalloc((void**)&s_batch.dfamily,
                              sizeof(int32_t) * (size_t)(M3_FAMILY_BLOCKS * M3F_COUNT + M3F_COUNT + 1)),
                   "cudaMalloc(family counts)");
        if (rc != M3GPU_OK)
        {
            s_batch.dfamily = nullptr;
            return rc;
        }
    }
    if (pairTotal > s_batch.bucketCap)
    {
        cudaFree(s_batch.dbucket);
        s_batch.dbucket = nullptr;
        s_batch.bucketCap = 0;
        rc = Check(cudaMalloc((void**)&s_batch.dbucket, sizeof(int32_t) * (size_t)pairTotal),
                   "cudaMalloc(pair buckets)");
        if (rc != M3GPU_OK)
        {
            s_batch.dbucket = nullptr;
            return rc;
        }
        s_batch.bucketCap = pairTotal;
    }
    s_batch.worlds.assign(worlds, worlds + count);
    s_batch.epoch = g_m3ResidencyEpoch;
    // Shared memory for the substep kernel: the body cache of the
    // largest world and, room permitting, each world's joint rows.  The
    // joint rows never push a block past M3_TWO_BLOCK_SMEM (two blocks
    // per SM); the body cache alone may go up to the per-block limit.
    int64_t bodyOnly = 0;
    int64_t want = 0;
    for (int32_t i = 0; i < count; ++i)
    {
        const m3WorldScalars* sc = worlds[i]->hv.sc;
        const int64_t bodies = (int64_t)sc->bodyMax * M3_BODY_CACHE_BYTES;
        const int64_t withJoints =
            m3AlignUp(bodies, 16) + (int64_t)sc->jointMax * (int64_t)sizeof(m3JointDev);
        bodyOnly = bodies > bodyOnly ? bodies : bodyOnly;
        want = withJoints > want ? withJoints : want;
    }
    const int64_t jointCap = bodyOnly > M3_TWO_BLOCK_SMEM ? bodyOnly : M3_TWO_BLOCK_SMEM;
    want = want < jointCap ? want : jointCap;
    const int64_t limit = 200 * 1024;
    s_batch.cacheBytes = (int32_t)(want < limit ? want : limit);
    s_batch.horder = order;
    return ClassifyBatch();
}

// Narrowphase grid: enough 128-thread blocks to fill every SM several
// times; the kernels stride over their pairs.
static int32_t s_narrowGrid = 148 * 16;

// The narrowphase of one step: family count and scatter, then one
// kernel per covered family over its bucket.
#define M3_NARROW_LAUNCHES (2 + M3F_TERRAIN_SPHERE)
#define M3_TERRAIN_LAUNCHES 3
// Batches of at most this many worlds take the single narrowphase kernel.
#define M3_NARROW_SMALL_BATCH 4

static void LaunchNarrow(const m3WorldView* views, const int32_t* offsets, int32_t count,
                         bool terrain)
{
    if (count <= M3_NARROW_SMALL_BATCH)
    {
        // A handful of worlds: one kernel over every family beats the
        // bucketing's nine launches.
        m3NarrowKernel<<<148, 128>>>(views, offsets, count);
        return;
    }
    int32_t* blockHist = s_batch.dfamily;
    int32_t* famStart = s_batch.dfamily + M3_FAMILY_BLOCKS * M3F_COUNT;
    const int32_t* bucket = s_batch.dbucket;
    m3FamilyCountKernel<<<M3_FAMILY_BLOCKS, M3_FAMILY_THREADS>>>(views, offsets, count, blockHist);
    m3FamilyScatterKernel<<<M3_FAMILY_BLOCKS, M3_FAMILY_THREADS>>>(views, offsets, count,
                                                                   blockHist, famStart,
                                                                   s_batch.dbucket);
    m3NarrowFamilyKernel<M3F_PLANE_HULL>
        <<<s_narrowGrid, 128>>>(views, offsets, count, famStart, bucket);
    m3NarrowFamilyKernel<M3F_HULL_HULL>
        <<<s_narrowGrid, 128>>>(views, offsets, count, famStart, bucket);
    m3NarrowFamilyKernel<M3F_PLANE_CAPSULE>
        <<<s_narrowGrid, 128>>>(views, offsets, count, famStart, bucket);
    m3NarrowFamilyKernel<M3F_CAPSULE_HULL>
        <<<s_narrowGrid, 128>>>(views, offsets, count, famStart, bucket);
    m3NarrowFamilyKernel<M3F_ROUND><<<s_narrowGrid, 128>>>(views, offsets, count, famStart, bucket);
    m3NarrowFamilyKernel<M3F_PLANE_SPHERE>
        <<<s_narrowGrid, 128>>>(views, offsets, count, famStart, bucket);
    m3NarrowFamilyKernel<M3F_SPHERE_SPHERE>
        <<<s_narrowGrid, 128>>>(views, offsets, count, famStart, bucket);
    if (terrain)
    {
        // Heightfield pairs, only in batches holding a heightfield.
        m3NarrowFamilyKernel<M3F_TERRAIN_SPHERE>
            <<<s_narrowGrid, 128>>>(views, offsets, count, famStart, bucket);
        m3NarrowFamilyKernel<M3F_TERRAIN_CAPSULE>
            <<<s_narrowGrid, 128>>>(views, offsets, count, famStart, bucket);
        m3NarrowFamilyKernel<M3F_TERRAIN_HULL>
            <<<s_narrowGrid, 128>>>(views, offsets, count, famStart, bucket);
    }
}

// The three per-world solve kernels of one step, in order on the current
// stream.  `marks`, when given, receives an event after the first two.
// The three per-world solve kernels of one step on the default stream.
// With `classFirst` (classFirst[c] .. classFirst[c + 1] index `order`)
// the prepare and substep stages run per size class on the class
// streams, forked off and joined back to the default stream around each
// stage; without it (one world, the allocation-free path) every kernel
// runs at 256 threads.  `marks`, when given, receives an event after the
// prepare and after the substep stage.
static void ClassStage(int32_t stage, const m3WorldView* views, const int32_t* order, float dt,
                       int32_t substeps, const int32_t* classFirst, const int32_t* classCache)
{
    cudaEventRecord(s_classStreams.fork, 0);
    for (int32_t c = 0; c < M3_CLASSES; ++c)
    {
        const int32_t n = classFirst[c + 1] - classFirst[c];
        if (n <= 0)
        {
            continue;
        }
        cudaStreamWaitEvent(s_classStreams.stream[c], s_classStreams.fork, 0);
        LaunchClass(stage, s_batch.classVariant[c], s_classStreams.stream[c], views,
                    order + classFirst[c], n, dt, substeps, classCache[c]);
        cudaEventRecord(s_classStreams.join[c], s_classStreams.stream[c]);
        cudaStreamWaitEvent(0, s_classStreams.join[c], 0);
    }
}

// Wide worlds: a single world with at least this many shape slots steps
// its substep loop over a cooperative grid (m3WideSubstepKernel).
static int32_t s_wideMinShapes = 4096;
static int32_t s_smCount = 148;

extern "C" int32_t m3gpu_set_wide_min_shapes(int32_t shapes)
{
    M3_DEVICE_GUARD;
    const int32_t previous = s_wideMinShapes;
    if (shapes > 0)
    {
        s_wideMinShapes = shapes;
    }
    return previous;
}

const int32_t* m3gpuDeviceMovers(const m3HostWorld* w)
{
    m3Scratch s;
    ScratchCarve(&s, w->dv.scratch, w->bodyCap, w->shapeCap, w->jointCap, w->pairCap);
    return s.movers;
}

void m3gpuDeviceHits(const m3HostWorld* w, const uint8_t** flags, const m3HitEvent** hits)
{
    m3Scratch s;
    ScratchCarve(&s, w->dv.scratch, w->bodyCap, w->shapeCap, w->jointCap, w->pairCap);
    *flags = s.hitFlag;
    *hits = s.hits;
}

extern "C" int32_t m3gpu_get_packing(m3gpuPacking* out)
{
    M3_DEVICE_GUARD;
    m3gpuClearError();
    if (out == nullptr)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "null packing");
    }
    *out = s_packing;
    return M3GPU_OK;
}

extern "C" int32_t m3gpu_set_packing(const m3gpuPacking* p)
{
    M3_DEVICE_GUARD;
    m3gpuClearError();
    if (p == nullptr)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "null packing");
    }
    if (!(p->minShapes[1] >= 1 && p->minShapes[0] > p->minShapes[1]))
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "class bounds %d, %d: need %d > %d >= 1",
                             p->minShapes[0], p->minShapes[1], p->minShapes[0], p->minShapes[1]);
    }
    for (int32_t c = 0; c < M3_CLASSES; ++c)
    {
        const int32_t t = p->threads[c];
        if (t != 128 && t != 256 && t != 512)
        {
            return m3gpuSetError(M3GPU_ERR_INVALID, "class %d: %d threads (128, 256 or 512)", c, t);
        }
        if (p->smemBytes[c] < 0 || p->smemBytes[c] > 200 * 1024)
        {
            return m3gpuSetError(M3GPU_ERR_INVALID, "class %d: %d bytes of shared memory "
                                 "(0 to 204800)", c, p->smemBytes[c]);
        }
    }
    if (memcmp(p, &s_packing, sizeof(s_packing)) != 0)
    {
        s_packing = *p;
        s_packingSeq += 1;
    }
    return M3GPU_OK;
}

// Blocks of the wide grid for a world: enough to give each level's rows
// a thread or so (about one block per 512 shape slots), at least 8, and
// never more than can be resident at once (a cooperative launch).
static int32_t WideBlocks(const m3HostWorld* w)
{
    static int32_t maxResident = 0;
    const int32_t shapes = w->hv.sc->shapeMax;
    if (shapes < s_wideMinShapes)
    {
        return 0;
    }
    if (maxResident == 0)
    {
        int device = 0;
        int sms = 0;
        int perSm = 0;
        cudaGetDevice(&device);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        s_smCount = sms;
        int perSmPrepare = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, m3WideSubstepKernel<256>, 256, 0);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSmPrepare, m3WidePrepareKernel<256>, 256,
                                                      0);
        perSm = perSm < perSmPrepare ? perSm : perSmPrepare;
        maxResident = sms * perSm;
        if (maxResident <= 0)
        {
            maxResident = -1; // cooperative launch impossible: never wide
        }
    }
    if (maxResident < 0)
    {
        return 0;
    }
    // At most one block per SM: the other half of each SM stays free for
    // the tree walks running beside the step on their own stream.
    int32_t blocks = shapes / 512;
    blocks = blocks < 8 ? 8 : blocks;
    blocks = blocks < s_smCount ? blocks : s_smCount;
    blocks = blocks < M3_WIDE_MAX_BLOCKS ? blocks : M3_WIDE_MAX_BLOCKS;
    return blocks < maxResident ? blocks : maxResident;
}

static void LaunchWideSubstep(const m3WorldView* views, const int32_t* order, float dt,
                              int32_t substeps, int32_t blocks)
{
    m3WideRowsKernel<<<4 * s_smCount, 256>>>(views, order, dt, substeps);
    void* args[] = {(void*)&views, (void*)&order, (void*)&dt, (void*)&substeps};
    cudaLaunchCooperativeKernel((const void*)m3WideSubstepKernel<256>, dim3(blocks), dim3(256),
                                args, 0, 0);
    m3WideStatusKernel<<<1, 1>>>(views, order);
}

static void LaunchSolve(const m3WorldView* views, const int32_t* order, int32_t count, float dt,
                        int32_t substeps, int32_t cacheBytes, const cudaEvent_t* marks,
                        const int32_t* classFirst = nullptr, const int32_t* classCache = nullptr,
                        int32_t wideBlocks = 0)
{
    if (wideBlocks > 0)
    {
        // One world: its preparation over the whole grid, then its rows.
        void* args[] = {(void*)&views, (void*)&order, (void*)&dt, (void*)&substeps};
        cudaLaunchCooperativeKernel((const void*)m3WidePrepareKernel<256>, dim3(wideBlocks),
                                    dim3(256), args, 0, 0);
        m3WideStatusKernel<<<1, 1>>>(views, order);
    }
    else if (classFirst == nullptr)
    {
        m3PrepareKernel<256, 2><<<count, 256, cacheBytes>>>(views, order, count, dt, substeps,
                                                            cacheBytes);
    }
    else
    {
        ClassStage(0, views, order, dt, substeps, classFirst, classCache);
    }
    if (marks != nullptr)
    {
        cudaEventRecord(marks[0]);
    }
    if (wideBlocks > 0)
    {
        LaunchWideSubstep(views, order, dt, substeps, wideBlocks);
    }
    else if (classFirst == nullptr)
    {
        m3SubstepKernel<256, 2><<<count, 256, cacheBytes>>>(views, order, count, dt, substeps,
                                                            cacheBytes);
    }
    else
    {
        ClassStage(1, views, order, dt, substeps, classFirst, classCache);
    }
    if (marks != nullptr)
    {
        cudaEventRecord(marks[1]);
    }
    m3FinishKernel<<<count, M3_BLOCK>>>(views, order, count, dt, substeps);
}

// Device milliseconds of the last batched call per stage: broadphase
// (bounds, pairs), narrowphase, prepare, substeps, finish.
#define M3_STAGES 5
static float s_kernelMs[M3_STAGES] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
static std::vector<cudaEvent_t> s_events;
static int32_t* s_dstatus = nullptr;

extern "C" int32_t m3gpu_kernel_ms(float* out)
{
    M3_DEVICE_GUARD;
    if (out == nullptr)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "null output");
    }
    for (int32_t k = 0; k < M3_STAGES; ++k)
    {
        out[k] = s_kernelMs[k];
    }
    return M3GPU_OK;
}

extern "C" int32_t m3gpu_world_stats(m3WorldId world, uint64_t* out)
{
    M3_DEVICE_GUARD;
    m3HostWorld* w = m3gpuWorldFromId(world);
    if (w == nullptr || out == nullptr)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "stale world or null output");
    }
    // The counters alone, read from the device's scalars when the device
    // is ahead (no tree replay, no download of the world).
    decltype(w->hv.sc->work) work;
    memcpy(work, w->hv.sc->work, sizeof(work));
    if (w->deviceAhead && w->dslab != nullptr)
    {
        const int32_t rc = Check(cudaMemcpy(work, w->dv.sc->work, sizeof(work),
                                            cudaMemcpyDeviceToHost),
                                 "work counters");
        if (rc != M3GPU_OK)
        {
            return rc;
        }
    }
    for (int32_t k = 0; k < 5; ++k)
    {
        out[k] = work[k];
    }
    out[5] = (uint64_t)w->hv.sc->bodyMax;
    return M3GPU_OK;
}

extern "C" int32_t m3gpu_world_phase_cycles(m3WorldId world, uint64_t* out)
{
    M3_DEVICE_GUARD;
    m3HostWorld* w = m3gpuWorldFromId(world);
    if (w == nullptr || out == nullptr)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "stale world or null output");
    }
    if (m3gpuSyncHost(w) != M3GPU_OK)
    {
        return m3gpu_last_error();
    }
    for (int32_t k = 0; k < 16; ++k)
    {
        out[k] = w->hv.sc->phase[k];
    }
    return M3GPU_OK;
}

// Body commands between steps (body.c:351-418), for the serving path:
// one thread per world applies its commands in order.
__global__ void __launch_bounds__(M3_BLOCK) m3BodyOpKernel(const m3WorldView* views, int32_t count,
                                                          const m3BodyOp* ops,
                                                          const int32_t* offsets)
{
    const int32_t wi = blockIdx.x * blockDim.x + threadIdx.x;
    if (wi >= count)
    {
        return;
    }
    const m3WorldView& w = views[wi];
    if (w.sc->status != 0)
    {
        return;
    }
    for (int32_t k = offsets[wi]; k < offsets[wi + 1]; ++k)
    {
        const m3BodyOp o = ops[k];
        const int32_t slots = m3IsJointOp(o.op) ? w.sc->jointMax : w.sc->bodyMax;
        if (o.body >= 0 && o.body < slots)
        {
            m3ApplyBodyOp(w, o.op, o.body, o.v);
        }
    }
}

// Page-locked staging and device copies of a batch's body commands.
struct m3OpStaging
{
    uint8_t* host = nullptr;
    uint8_t* dev = nullptr;
    int64_t cap = 0;
};
static m3OpStaging s_ops;

static int32_t LaunchBodyOps(int32_t count, const m3BodyOp* ops, int32_t opCount)
{
    // Ops sorted by world (stable), and each world's range.
    std::vector<int32_t> offsets((size_t)count + 1, 0);
    for (int32_t k = 0; k < opCount; ++k)
    {
        if (ops[k].world < 0 || ops[k].world >= count)
        {
            return m3gpuSetError(M3GPU_ERR_INVALID, "body command names world %d of %d",
                                 ops[k].world, count);
        }
        offsets[(size_t)ops[k].world + 1] += 1;
    }
    for (int32_t i = 0; i < count; ++i)
    {
        offsets[(size_t)i + 1] += offsets[(size_t)i];
    }
    std::vector<int32_t> fill(offsets.begin(), offsets.end() - 1);
    std::vector<m3BodyOp> sorted((size_t)opCount);
    for (int32_t k = 0; k < opCount; ++k)
    {
        sorted[(size_t)fill[(size_t)ops[k].world]++] = ops[k];
    }
    const int64_t opBytes = (int64_t)sizeof(m3BodyOp) * opCount;
    const int64_t offBytes = (int64_t)sizeof(int32_t) * (count + 1);
    const int64_t need = m3AlignUp(opBytes, 256) + offBytes;
    if (need > s_ops.cap)
    {
        cudaDeviceSynchronize();
        cudaFreeHost(s_ops.host);
        cudaFree(s_ops.dev);
        s_ops = m3OpStaging{};
        int32_t rc = Check(cudaMallocHost((void**)&s_ops.host, (size_t)need), "op staging");
        if (rc == M3GPU_OK)
        {
            rc = Check(cudaMalloc((void**)&s_ops.dev, (size_t)need), "op staging");
        }
        if (rc != M3GPU_OK)
        {
            return rc;
        }
        s_ops.cap = need;
    }
    memcpy(s_ops.host, sorted.data(), (size_t)opBytes);
    memcpy(s_ops.host + m3AlignUp(opBytes, 256), offsets.data(), (size_t)offBytes);
    int32_t rc = Check(cudaMemcpyAsync(s_ops.dev, s_ops.host, (size_t)need, cudaMemcpyHostToDevice, 0),
                       "upload body commands");
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    m3BodyOpKernel<<<(count + M3_BLOCK - 1) / M3_BLOCK, M3_BLOCK>>>(
        s_batch.dviews, count, (const m3BodyOp*)s_ops.dev,
        (const int32_t*)(s_ops.dev + m3AlignUp(opBytes, 256)));
    s_launches += 1;
    return Check(cudaGetLastError(), "body command kernel");
}

// Every tree launch gets a sequence number (from 1) and an event in a
// ring; waiting for launch q waits on its event, or, once the ring has
// moved past it, on the oldest event still in the ring (the tree stream
// runs its launches in order, so a later launch done means q is done).
#define M3_TREE_EVENTS 64
static cudaEvent_t s_treeEvents[M3_TREE_EVENTS] = {};
static uint64_t s_treeSeq = 0;

static cudaEvent_t TreeEventFor(uint64_t q)
{
    if (s_treeSeq - q >= M3_TREE_EVENTS)
    {
        q = s_treeSeq - M3_TREE_EVENTS + 1;
    }
    return s_treeEvents[q % M3_TREE_EVENTS];
}

static uint64_t RecordTreeLaunch(cudaStream_t stream)
{
    const uint64_t q = s_treeSeq + 1;
    cudaEvent_t& e = s_treeEvents[q % M3_TREE_EVENTS];
    if (e == nullptr)
    {
        cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
    }
    cudaEventRecord(e, stream);
    s_treeSeq = q;
    return q;
}

// The tree launches of a call read their own copy of the call's world
// table: they finish behind the call, after the next call may have
// rebuilt the batch table.  A copy is reused (oldest first) once the
// last launch reading it is done.
#define M3_TREE_TABLES 8
struct m3TreeTable
{
    m3WorldView* views = nullptr;
    int32_t* order = nullptr;
    int32_t* steps = nullptr;     // per world: recorded steps to replay
    int32_t* hostSteps = nullptr; // page-locked staging of `steps`
    int32_t cap = 0;
    uint64_t lastSeq = 0;
};
static m3TreeTable s_treeTables[M3_TREE_TABLES];
static int32_t s_treeTableNext = 0;

static int32_t TakeTreeTable(int32_t count, m3TreeTable** out)
{
    m3TreeTable& t = s_treeTables[s_treeTableNext];
    s_treeTableNext = (s_treeTableNext + 1) % M3_TREE_TABLES;
    if (t.lastSeq != 0)
    {
        const cudaError_t e = cudaEventSynchronize(TreeEventFor(t.lastSeq));
        if (e != cudaSuccess)
        {
            return m3gpuSetError(M3GPU_ERR_CUDA, "tree table: %s", cudaGetErrorString(e));
        }
        t.lastSeq = 0;
    }
    if (count > t.cap)
    {
        cudaFree(t.views);
        cudaFree(t.order);
        cudaFree(t.steps);
        cudaFreeHost(t.hostSteps);
        t.views = nullptr;
        t.order = nullptr;
        t.steps = nullptr;
        t.hostSteps = nullptr;
        t.cap = 0;
        cudaError_t e = cudaMalloc((void**)&t.views, sizeof(m3WorldView) * (size_t)count);
        if (e == cudaSuccess)
        {
            e = cudaMalloc((void**)&t.order, sizeof(int32_t) * (size_t)count);
        }
        if (e == cudaSuccess)
        {
            e = cudaMalloc((void**)&t.steps, sizeof(int32_t) * (size_t)count);
        }
        if (e == cudaSuccess)
        {
            e = cudaMallocHost((void**)&t.hostSteps, sizeof(int32_t) * (size_t)count);
        }
        if (e != cudaSuccess)
        {
            return m3gpuSetError(M3GPU_ERR_CUDA, "tree table: %s", cudaGetErrorString(e));
        }
        t.cap = count;
    }
    // Ordered on the default stream after the batch table's upload and
    // before the broadphase the tree launches wait for.
    cudaError_t e = cudaMemcpyAsync(t.views, s_batch.dviews, sizeof(m3WorldView) * (size_t)count,
                                    cudaMemcpyDeviceToDevice, 0);
    if (e == cudaSuccess)
    {
        e = cudaMemcpyAsync(t.order, s_batch.dorder, sizeof(int32_t) * (size_t)count,
                            cudaMemcpyDeviceToDevice, 0);
    }
    if (e != cudaSuccess)
    {
        return m3gpuSetError(M3GPU_ERR_CUDA, "tree table: %s", cudaGetErrorString(e));
    }
    *out = &t;
    return M3GPU_OK;
}

// Launches the replay of every recorded step no launch covers yet, for
// the worlds of `table` (views index i = worlds[i]), on `stream` after the
// events it already waits for; the covered steps take the launch's
// sequence number.
static void LaunchTreeReplay(m3TreeTable* table, m3HostWorld** worlds, int32_t count,
                             cudaStream_t stream)
{
    for (int32_t i = 0; i < count; ++i)
    {
        table->hostSteps[i] = worlds[i]->hv.sc->treeTracked != 0 ? worlds[i]->treeUnlaunched : 0;
    }
    cudaMemcpyAsync(table->steps, table->hostSteps, sizeof(int32_t) * (size_t)count,
                    cudaMemcpyHostToDevice, stream);
    m3TreeKernel<<<count, 32, 0, stream>>>(table->views, table->order, count, M3_TREE_LAG,
                                           table->steps);
    const uint64_t q = RecordTreeLaunch(stream);
    table->lastSeq = q;
    s_launches += 1;
    for (int32_t i = 0; i < count; ++i)
    {
        m3HostWorld* w = worlds[i];
        for (int32_t k = w->treeCount - w->treeUnlaunched; k < w->treeCount; ++k)
        {
            w->treeSlotSeq[(w->treeFirst + k) % M3_TREE_LAG] = q;
        }
        w->treeUnlaunched = 0;
    }
}

// A replay of the batch's unlaunched steps with its own copy of the
// batch table, on the tree's stream after everything the default stream
// holds so far (the steps' broadphases included).
static int32_t ReplayBatch(m3HostWorld** worlds, int32_t count, cudaStream_t treeStream)
{
    static cudaEvent_t fork = nullptr;
    if (fork == nullptr && cudaEventCreateWithFlags(&fork, cudaEventDisableTiming) != cudaSuccess)
    {
        fork = nullptr;
        return m3gpuSetError(M3GPU_ERR_CUDA, "tree replay event");
    }
    m3TreeTable* table = nullptr;
    const int32_t rc = TakeTreeTable(count, &table);
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    cudaEventRecord(fork, 0);
    cudaStreamWaitEvent(treeStream, fork, 0);
    LaunchTreeReplay(table, worlds, count, treeStream);
    return M3GPU_OK;
}

// One world's replay table (views and order of one entry), for readers
// of a single world's tree.
static m3WorldView* s_oneView = nullptr;
static int32_t* s_oneOrder = nullptr;
static int32_t* s_oneSteps = nullptr;

void m3gpuWaitTree(m3HostWorld* w)
{
    M3_DEVICE_GUARD;
    if (w->treeCount == 0)
    {
        return;
    }
    // Launches already covering some of its steps come first.
    uint64_t last = 0;
    for (int32_t k = 0; k < w->treeCount; ++k)
    {
        const uint64_t q = w->treeSlotSeq[(w->treeFirst + k) % M3_TREE_LAG];
        last = q > last ? q : last;
    }
    if (last != 0)
    {
        cudaStreamWaitEvent(0, TreeEventFor(last), 0);
    }
    if (w->treeUnlaunched > 0 && w->dslab != nullptr)
    {
        // The rest replayed here, on the default stream, before the
        // reader's own work.
        if (s_oneView == nullptr)
        {
            cudaMalloc((void**)&s_oneView, sizeof(m3WorldView));
            cudaMalloc((void**)&s_oneOrder, 2 * sizeof(int32_t));
            s_oneSteps = s_oneOrder + 1;
        }
        m3WorldView view = w->dv;
        m3AttachDevicePools(w, &view);
        const int32_t table[2] = {0, w->treeUnlaunched};
        cudaMemcpy(s_oneView, &view, sizeof(view), cudaMemcpyHostToDevice);
        cudaMemcpy(s_oneOrder, table, sizeof(table), cudaMemcpyHostToDevice);
        m3TreeKernel<<<1, 32>>>(s_oneView, s_oneOrder, 1, M3_TREE_LAG, s_oneSteps);
        s_launches += 1;
    }
    w->treeCount = 0;
    w->treeFirst = 0;
    w->treeUnlaunched = 0;
}

// Every recorded move of the worlds replayed into their trees, and the
// trees finished (the tree stream's work done).
extern "C" int32_t m3gpu_flush_trees(const m3WorldId* worldIds, int32_t count)
{
    M3_DEVICE_GUARD;
    m3gpuClearError();
    if (worldIds == nullptr || count <= 0)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "empty world list");
    }
    std::vector<m3HostWorld*> ws((size_t)count);
    for (int32_t i = 0; i < count; ++i)
    {
        ws[(size_t)i] = m3gpuWorldFromId(worldIds[i]);
        if (ws[(size_t)i] == nullptr)
        {
            return m3gpuSetError(M3GPU_ERR_INVALID, "stale world id at position %d", i);
        }
    }
    int32_t rc = m3gpuEnsureDevice();
    if (rc == M3GPU_OK)
    {
        rc = EnsureClassStreams();
    }
    bool unlaunched = false;
    for (m3HostWorld* w : ws)
    {
        unlaunched = unlaunched || (w->treeUnlaunched > 0 && w->dslab != nullptr &&
                                    !w->hostDirty && w->hv.sc->treeTracked != 0);
    }
    if (rc == M3GPU_OK && unlaunched)
    {
        // Every world's unlaunched steps in one launch, one warp a world.
        rc = PrepareBatch(ws.data(), count);
        if (rc == M3GPU_OK)
        {
            rc = ReplayBatch(ws.data(), count, s_classStreams.tree);
        }
    }
    if (rc == M3GPU_OK)
    {
        rc = Check(cudaDeviceSynchronize(), "flush trees");
    }
    if (rc == M3GPU_OK)
    {
        for (m3HostWorld* w : ws)
        {
            m3gpuWaitTree(w); // nothing left to replay: clears the ring's record
        }
    }
    return rc;
}

int32_t m3gpuStepBatch(m3HostWorld** worlds, int32_t count, float dt, int32_t substeps,
                       int32_t steps, const m3BodyOp* ops, int32_t opCount)
{
    M3_DEVICE_GUARD;
    int32_t rc = m3gpuEnsureDevice();
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    rc = PrepareBatch(worlds, count);
    if (rc == M3GPU_OK)
    {
        rc = EnsureClassStreams();
    }
    if (rc == M3GPU_OK && opCount > 0)
    {
        // The staging buffer is reused by the next call only after this
        // one synchronised (below, reading the status).
        rc = LaunchBodyOps(count, ops, opCount);
    }
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    // Events: one before the batch, then per step one after the collide
    // kernels and one after each solve kernel, so the stages' device
    // times are separable.
    size_t needEvents = (size_t)(M3_STAGES * steps + 1);
    while (s_events.size() < needEvents)
    {
        cudaEvent_t e;
        rc = Check(cudaEventCreate(&e), "cudaEventCreate");
        if (rc != M3GPU_OK)
        {
            return rc;
        }
        s_events.push_back(e);
    }
    if (s_dstatus == nullptr)
    {
        rc = Check(cudaMalloc((void**)&s_dstatus, sizeof(int32_t)), "cudaMalloc(status)");
        if (rc != M3GPU_OK)
        {
            return rc;
        }
    }
    cudaEventRecord(s_events[0]);
    // The broadphase tree: the leaves' bounds once per fresh slab, then
    // per step the tree kernel on its own stream, each world at most
    // M3_TREE_LAG steps behind its own step (the move lists sit in a ring
    // of that depth in its scratch), across calls.  Batches of worlds
    // that keep no tree skip both.
    bool anyTracked = false;
    bool anyTerrain = false;
    bool leafBoxes = false;
    std::vector<m3HostWorld*> tracked;
    for (int32_t i = 0; i < count; ++i)
    {
        if (worlds[i]->hv.sc->treeTracked != 0)
        {
            anyTracked = true;
            tracked.push_back(worlds[i]);
            leafBoxes = leafBoxes || !worlds[i]->leafBoxValid;
        }
        anyTerrain = anyTerrain || !worlds[i]->hfHeaders.empty();
    }
    if (leafBoxes)
    {
        // Fresh slabs: copy every leaf's bounds out of the (finished)
        // trees once; the broadphase keeps the copy current afterwards.
        for (m3HostWorld* w : tracked)
        {
            m3gpuWaitTree(w);
        }
        m3LeafBoxKernel<<<count, M3_BLOCK>>>(s_batch.dviews, count);
        s_launches += 1;
        for (m3HostWorld* w : tracked)
        {
            w->leafBoxValid = true;
        }
    }
    const cudaStream_t treeStream = s_classStreams.tree;
    // One large world alone: its substep loop over the whole grid.
    const int32_t wideBlocks = count == 1 ? WideBlocks(worlds[0]) : 0;
    for (int32_t step = 0; step < steps; ++step)
    {
        const cudaEvent_t* ev = &s_events[(size_t)(M3_STAGES * step)];
        if (anyTracked)
        {
            // The step records into each world's oldest ring slot once the
            // ring is full: the launch replaying that slot must be done
            // (and launched first, if none covers it yet).
            bool unlaunchedFull = false;
            for (m3HostWorld* w : tracked)
            {
                unlaunchedFull = unlaunchedFull ||
                                 (w->treeCount == M3_TREE_LAG && w->treeUnlaunched == M3_TREE_LAG);
            }
            if (unlaunchedFull)
            {
                rc = ReplayBatch(worlds, count, treeStream);
                if (rc != M3GPU_OK)
                {
                    return rc;
                }
            }
            uint64_t need = 0;
            for (m3HostWorld* w : tracked)
            {
                if (w->treeCount == M3_TREE_LAG)
                {
                    const uint64_t q = w->treeSlotSeq[w->treeFirst];
                    need = q > need ? q : need;
                    w->treeFirst = (w->treeFirst + 1) % M3_TREE_LAG;
                    w->treeCount -= 1;
                }
            }
            if (need != 0)
            {
                cudaStreamWaitEvent(0, TreeEventFor(need), 0);
            }
        }
        if (wideBlocks > 0)
        {
            // One large world: its sweep over the whole grid between the
            // head and the tail of its broadphase.
            m3BroadKernel<512, 1, 1><<<1, 512>>>(s_batch.dviews, s_batch.dorder, count,
                                                  M3_TREE_LAG);
            m3WideSweepKernel<<<4 * s_smCount, 256>>>(s_batch.dviews, s_batch.dorder);
            m3BroadKernel<512, 1, 2><<<1, 512>>>(s_batch.dviews, s_batch.dorder, count,
                                                  M3_TREE_LAG);
            s_launches += 2;
        }
        else
        {
            m3BroadKernel<M3_BLOCK, 2><<<count, M3_BLOCK>>>(s_batch.dviews, s_batch.dorder, count,
                                                            M3_TREE_LAG);
        }
        cudaEventRecord(ev[1]);
        if (anyTracked)
        {
            // The step's moves are recorded; once M3_TREE_REPLAY_AT steps
            // wait in a world's ring, the batch's recorded steps are
            // replayed on the tree's stream beside the following steps.
            bool replay = false;
            for (m3HostWorld* w : tracked)
            {
                w->treeSlotSeq[(w->treeFirst + w->treeCount) % M3_TREE_LAG] = 0;
                w->treeCount += 1;
                w->treeUnlaunched += 1;
                replay = replay || w->treeUnlaunched >= M3_TREE_REPLAY_AT;
            }
            if (replay)
            {
                rc = ReplayBatch(worlds, count, treeStream);
                if (rc != M3GPU_OK)
                {
                    return rc;
                }
            }
        }
        m3PairOffsetsKernel<<<1, M3_BLOCK>>>(s_batch.dviews, count, s_batch.doffsets);
        LaunchNarrow(s_batch.dviews, s_batch.doffsets, count, anyTerrain);
        cudaEventRecord(ev[2]);
        LaunchSolve(s_batch.dviews, s_batch.dorder, count, dt, substeps, s_batch.cacheBytes,
                    ev + 3, s_batch.classFirst, s_batch.classCache, wideBlocks);
        cudaEventRecord(ev[5]);
        s_launches += 5 + (count <= M3_NARROW_SMALL_BATCH ? 1 : M3_NARROW_LAUNCHES + (anyTerrain ? M3_TERRAIN_LAUNCHES : 0));
    }
    // The trees catch up later: replays already launched finish on their
    // own stream, recorded steps not yet launched wait in the ring; a
    // later step waits only for a ring slot it reuses, and anything that
    // reads or overwrites a world's tree first replays the world's
    // recorded steps (m3gpuWaitTree, m3gpu_flush_trees).
    cudaMemsetAsync(s_dstatus, 0, sizeof(int32_t));
    m3StatusKernel<<<(count + 255) / 256, 256>>>(s_batch.dviews, count, s_dstatus);
    s_launches += 1;
    rc = Check(cudaGetLastError(), "step launch");
    int32_t status = 0;
    if (rc == M3GPU_OK)
    {
        rc = Check(cudaMemcpy(&status, s_dstatus, sizeof(int32_t), cudaMemcpyDeviceToHost),
                   "step");
    }
    for (int32_t i = 0; i < count; ++i)
    {
        worlds[i]->deviceAhead = true;
        worlds[i]->pairTailsOnDevice = true;
        if (rc == M3GPU_OK && steps > 0)
        {
            m3MarkEventEpoch(worlds[i], true);
        }
    }
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    float total = 0.0f;
    cudaEventElapsedTime(&total, s_events[0], s_events[(size_t)(M3_STAGES * steps)]);
    for (int32_t k = 0; k < M3_STAGES; ++k)
    {
        s_kernelMs[k] = 0.0f;
    }
    float last[M3_STAGES] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    for (int32_t step = 0; step < steps; ++step)
    {
        const cudaEvent_t* ev = &s_events[(size_t)(M3_STAGES * step)];
        for (int32_t k = 0; k < M3_STAGES; ++k)
        {
            float ms = 0.0f;
            cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
            s_kernelMs[k] += ms;
            last[k] = ms;
        }
    }
    s_lastStepMs = total;
    // Every world's profile (m3World_GetProfile) is its batch's last
    // step: the device runs the batch's worlds together, stage by stage.
    if (steps > 0)
    {
        float stepMs = 0.0f;
        for (int32_t k = 0; k < M3_STAGES; ++k)
        {
            stepMs += last[k];
        }
        for (int32_t i = 0; i < count; ++i)
        {
            m3StepProfile& p = worlds[i]->profile;
            p.step = stepMs;
            p.broadphase = last[0];
            p.narrowphase = last[1];
            p.prepare = last[2];
            p.solve = last[3];
            p.finish = last[4];
            p.valid = true;
        }
    }
    if (status != 0)
    {
        // Name the first refusing world and its detail code.
        for (int32_t i = 0; i < count; ++i)
        {
            int32_t st = 0;
            int32_t detail = 0;
            cudaMemcpy(&st, &worlds[i]->dv.sc->status, sizeof(int32_t), cudaMemcpyDeviceToHost);
            if (st != 0)
            {
                cudaMemcpy(&detail, &worlds[i]->dv.sc->statusDetail, sizeof(int32_t),
                           cudaMemcpyDeviceToHost);
                return m3gpuSetError(st, "world %d stalled on the device (status %d, detail %d)",
                                     worlds[i]->slot, st, detail);
            }
        }
        return m3gpuSetError(status, "a world stalled on the device (status %d)", status);
    }
    return M3GPU_OK;
}

int32_t m3gpuHashBatch(m3HostWorld** worlds, int32_t count, uint64_t* out)
{
    M3_DEVICE_GUARD;
    int32_t rc = m3gpuEnsureDevice();
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    rc = PrepareBatch(worlds, count);
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    rc = m3gpuLaunchHash(s_batch.dviews, s_batch.dorder, count, s_batch.dhash);
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    s_launches += 1;
    rc = Check(cudaGetLastError(), "hash launch");
    if (rc == M3GPU_OK)
    {
        rc = Check(cudaMemcpy(out, s_batch.dhash, sizeof(uint64_t) * (size_t)count,
                              cudaMemcpyDeviceToHost),
                   "hash readback");
    }
    return rc;
}

// ---------------------------------------------------------------------
// Allocation-free single-world step.
//
// Some callers cannot allocate device memory at the moment they need a
// step: a frame loop with a hard deadline (cudaMalloc and cudaFree can
// synchronise the whole device), or a host whose device memory is owned
// entirely by its own pool allocator.  For them m3gpu_step_world_noalloc
// steps one world
// that is already resident in HBM (reserved and uploaded earlier, when
// allocating was allowed) without allocating anything: the step's
// scratch, the one-world launch table and the status word live in
// file-scope __device__ arrays of fixed size instead of the world's own
// slab scratch and the batch tables.
//
// Limits: the world's scratch need (bodies, shapes, joints and 8 pairs
// per shape of the reference's pair capacity) must fit in
// M3_NOALLOC_SCRATCH_BYTES (4 MiB, about 800 shape slots), and its
// body-velocity cache in 48 KiB of shared memory (800 bodies); larger
// worlds are refused with M3GPU_ERR_CAPACITY before any device work.
// Every GPU that loads the library holds these arrays until exit.
//
// The first call on a device looks up the arrays' device addresses
// (cudaGetSymbolAddress) with that device current and caches them; make
// that first call before any stream capture.  The call itself copies the
// launch table and reads the status with blocking copies on the legacy
// default stream, so it must not run while any stream of the process is
// being captured.  All calls share the arrays and leave the last call's
// contents behind (every field the step reads is rewritten first, and
// the tree's move count is zeroed before anything can return early), so
// calls that overlap on the GPU race: the library's lock serialises the
// calls of one process; callers in several processes sharing a GPU each
// hold their own copy of the arrays.
// ---------------------------------------------------------------------
#define M3_NOALLOC_SCRATCH_BYTES (4 * 1024 * 1024)
#define M3_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) uint8_t g_noallocScratch[M3_NOALLOC_SCRATCH_BYTES];
static __device__ __align__(256) m3WorldView g_noallocView;
static __device__ __align__(256) int32_t g_noallocTable[4]; // order[1], offsets[2], tree steps[1]

struct m3NoallocSymbols
{
    uint8_t* scratch;
    m3WorldView* view;
    int32_t* table;
};
static m3NoallocSymbols s_noalloc[M3_NOALLOC_MAX_DEVICES];

static int32_t NoallocSetup(int32_t device, m3NoallocSymbols* out)
{
    if (device < 0 || device >= M3_NOALLOC_MAX_DEVICES)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "device %d beyond the supported range", device);
    }
    m3NoallocSymbols& sym = s_noalloc[device];
    if (sym.scratch == nullptr)
    {
        int32_t rc = Check(cudaGetSymbolAddress((void**)&sym.scratch, g_noallocScratch),
                           "cudaGetSymbolAddress(scratch)");
        if (rc == M3GPU_OK)
        {
            rc = Check(cudaGetSymbolAddress((void**)&sym.view, g_noallocView),
                       "cudaGetSymbolAddress(view)");
        }
        if (rc == M3GPU_OK)
        {
            rc = Check(cudaGetSymbolAddress((void**)&sym.table, g_noallocTable),
                       "cudaGetSymbolAddress(table)");
        }
        if (rc != M3GPU_OK)
        {
            sym.scratch = nullptr;
            return rc;
        }
    }
    *out = sym;
    return M3GPU_OK;
}

extern "C" int32_t m3gpu_step_world_noalloc(m3WorldId worldId, float dt, int32_t substeps)
{
    M3_DEVICE_GUARD;
    m3gpuClearError();
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr || !(dt > 0.0f) || substeps < 1 || substeps > M3_MAX_SUBSTEPS)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "stale world or invalid dt/substeps");
    }
    if (w->dslab == nullptr || w->hostDirty)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID,
                             "world is not resident on the device: reserve and upload it first "
                             "(m3gpu_reserve_worlds, m3gpu_upload_worlds)");
    }
    // One slot of tree moves: this path runs the tree kernel in order.
    const int64_t need =
        ScratchCarve(nullptr, nullptr, w->bodyCap, w->shapeCap, w->jointCap, w->pairCap, 1);
    const int64_t cache = (int64_t)w->hv.sc->bodyMax * M3_BODY_CACHE_BYTES;
    if (need > M3_NOALLOC_SCRATCH_BYTES || cache > 48 * 1024)
    {
        return m3gpuSetError(M3GPU_ERR_CAPACITY,
                             "world needs %lld scratch bytes and %lld cache bytes; the "
                             "allocation-free step holds %d and %d",
                             (long long)need, (long long)cache, M3_NOALLOC_SCRATCH_BYTES,
                             48 * 1024);
    }
    // The library's device, made current for this thread (the world's
    // slab lives there); the static arrays are looked up on it.
    int32_t rc = m3gpuEnsureDevice();
    int device = 0;
    if (rc == M3GPU_OK)
    {
        rc = Check(cudaGetDevice(&device), "cudaGetDevice");
    }
    m3NoallocSymbols sym;
    if (rc == M3GPU_OK)
    {
        rc = NoallocSetup(device, &sym);
    }
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    // The one-world launch table: the world's view with its scratch
    // redirected to the static array, order {0}.
    m3WorldView view = w->dv;
    m3AttachDevicePools(w, &view);
    view.scratch = sym.scratch;
    view.scratchBytes = M3_NOALLOC_SCRATCH_BYTES;
    // Launch table: order {0}, then two words for the pair offsets, then
    // the one step the tree replays.
    const int32_t table[4] = {0, 0, 0, 1};
    rc = Check(cudaMemcpy(sym.view, &view, sizeof(view), cudaMemcpyHostToDevice), "noalloc view");
    if (rc == M3GPU_OK)
    {
        rc = Check(cudaMemcpy(sym.table, table, sizeof(table), cudaMemcpyHostToDevice),
                   "noalloc order");
    }
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    int32_t* order = sym.table;
    int32_t* offsets = sym.table + 1;
    const int32_t cacheBytes = (int32_t)cache;
    // The 256-thread kernels (size class 1) run this world.
    rc = EnsureClassSmem(1, cacheBytes);
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    // Tree replays of earlier regular steps first; this call replays its
    // own moves in order on the default stream, and moves leaves the
    // slab scratch's copy of their bounds does not see.
    m3gpuWaitTree(w);
    w->leafBoxValid = false;
    m3LeafBoxKernel<<<1, M3_BLOCK>>>(sym.view, 1);
    m3BroadKernel<M3_BLOCK, 1><<<1, M3_BLOCK>>>(sym.view, order, 1, 1);
    m3TreeKernel<<<1, 32>>>(sym.view, order, 1, 1, sym.table + 3);
    m3PairOffsetsKernel<<<1, M3_BLOCK>>>(sym.view, 1, offsets);
    m3NarrowKernel<<<148, 128>>>(sym.view, offsets, 1);
    LaunchSolve(sym.view, order, 1, dt, substeps, cacheBytes, nullptr);
    s_launches += 8;
    rc = Check(cudaGetLastError(), "noalloc step launch");
    int32_t status = 0;
    if (rc == M3GPU_OK)
    {
        rc = Check(cudaMemcpy(&status, &w->dv.sc->status, sizeof(int32_t), cudaMemcpyDeviceToHost),
                   "noalloc step");
    }
    w->deviceAhead = true;
    w->pairTailsOnDevice = true;
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    m3MarkEventEpoch(w, true);
    if (status == 0)
    {
        // The step's mover list (its body move events) into the world's
        // own scratch: the static array belongs to every call.
        m3Scratch from;
        m3Scratch to;
        ScratchCarve(&from, sym.scratch, w->bodyCap, w->shapeCap, w->jointCap, w->pairCap);
        ScratchCarve(&to, w->dv.scratch, w->bodyCap, w->shapeCap, w->jointCap, w->pairCap);
        rc = Check(cudaMemcpy(to.movers, from.movers,
                              sizeof(int32_t) * (size_t)w->hv.sc->bodyMax,
                              cudaMemcpyDeviceToDevice),
                   "noalloc movers");
        // And its hit events.
        if (rc == M3GPU_OK)
        {
            rc = Check(cudaMemcpy(to.hitFlag, from.hitFlag, (size_t)w->pairCap,
                                  cudaMemcpyDeviceToDevice),
                       "noalloc hit flags");
        }
        if (rc == M3GPU_OK)
        {
            rc = Check(cudaMemcpy(to.hits, from.hits, sizeof(m3HitEvent) * (size_t)w->pairCap,
                                  cudaMemcpyDeviceToDevice),
                       "noalloc hit events");
        }
        if (rc != M3GPU_OK)
        {
            return rc;
        }
    }
    if (status != 0)
    {
        int32_t detail = 0;
        cudaMemcpy(&detail, &w->dv.sc->statusDetail, sizeof(int32_t), cudaMemcpyDeviceToHost);
        return m3gpuSetError(status, "world %d stalled on the device (status %d, detail %d)",
                             w->slot, status, detail);
    }
    return M3GPU_OK;
}
