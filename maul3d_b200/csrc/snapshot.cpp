// Snapshots and journal replay at the reference's byte formats:
// m3World_SnapshotSize / m3World_Snapshot write snapshot v54
// (snapshot.c:603-678), m3World_Restore reads it (snapshot.c:680-931),
// and m3World_JournalReplay applies a recorded command stream
// (world.c:1505-3218) whose steps run on the GPU.  Restore and replay
// are the ingestion side of serving: a request is a snapshot plus the
// journal of the frames to simulate.
//
// A snapshot is a 192-byte header and the persistent arrays as
// canonical blocks in one fixed order, then a count-derived tail (mesh,
// hull and heightfield content).  One walk over the blocks serves every
// direction: it measures, checks an input, reads it into a world, or
// writes a world out.  Blocks of state this path keeps map onto the
// world image.  Blocks of pools it does not model (voxels, heightfields,
// characters, vehicles, soft bodies, meshes, water volumes, generic and
// pulley joint fields, debug names) must describe no live object on
// restore; their bytes are carried verbatim, so a restored world writes
// them back unchanged, and a world built here writes the values a fresh
// reference world holds.
#include "m3_world.h"
#include "m3_ops.h"
#include "m3_tree.h"

#include <math.h>
#include <string.h>

#include <vector>

namespace
{
constexpr uint32_t kSnapshotMagic = 0x4D33534Eu; // 'M3SN'
constexpr uint32_t kSnapshotVersion = 54u;
constexpr int32_t kSolverRevision = 21;

// Sizes of the reference's fixed records and caps that size its blocks
// (world_internal.h): debug name bytes per body, voxel chunk, vehicle
// wheels / engine curve points / gears, soft-body tets / particles /
// edges / anchors, water volumes, mesh caps and material table.
constexpr int32_t kBodyNameBytes = M3_BODY_NAME_BYTES;
constexpr int32_t kVoxelChunkBytes = 12808;
constexpr int32_t kVehicleWheels = 8;
constexpr int32_t kEngineCurve = 8;
constexpr int32_t kGears = 6;
constexpr int32_t kSoftTets = 1024;
constexpr int32_t kSoftParticles = 512;
constexpr int32_t kSoftEdges = 5120;
constexpr int32_t kSoftAnchors = 32;
constexpr int32_t kWaterVolumes = 8;
constexpr int32_t kMeshMaxVerts = 65535;
constexpr int32_t kMeshMaxTris = 65535;
constexpr int32_t kMeshMaterialBytes = 8 * 24;
constexpr int32_t kHeightFieldMaxDim = M3_HEIGHTFIELD_MAX_DIM;

#pragma pack(push, 1)
struct SnapshotHeader // snapshot.c:88-127
{
    uint32_t magic;
    uint32_t formatVersion;
    uint64_t configHash;
    uint64_t stepCount;
    int32_t bodyCapacity, maxIndex, freeHead, freeCount, retiredCount;
    int32_t shapeCapacity, shapeMaxIndex, shapeFreeHead, shapeFreeCount, shapeRetiredCount;
    int32_t pairCount, treeRoot, treeFreeList;
    int32_t hullMaxIndex, hullFreeHead, hullFreeCount, hullRetiredCount;
    int32_t meshCapacity, meshMaxIndex, meshFreeHead, meshFreeCount, meshRetiredCount;
    int32_t jointCapacity, jointMaxIndex, jointFreeHead, jointFreeCount, jointRetiredCount;
    int32_t voxelCapacity, voxelMaxIndex, voxelFreeHead, voxelFreeCount, voxelRetiredCount;
    int32_t charCapacity, charMaxIndex, charFreeHead, charFreeCount, charRetiredCount;
    int32_t reserved[2];
    m3Vec3 gravity;
};
#pragma pack(pop)
static_assert(sizeof(SnapshotHeader) == 192, "snapshot header layout");

// What the bytes mean: engine version, solver revision, real and
// position sizes and the floating-point policy (snapshot.c:131-147).
uint64_t ConfigHash()
{
    uint64_t h = M3_HASH_INIT;
    const int32_t version = m3GetVersion();
    const int32_t rev = kSolverRevision;
    const int32_t realSize = (int32_t)sizeof(m3real);
    const int32_t posSize = (int32_t)sizeof(double);
    const char* policy = "contract-off;no-fast-math;no-fuse-4wide";
    h = m3Fnv(h, &version, 4);
    h = m3Fnv(h, &rev, 4);
    h = m3Fnv(h, &realSize, 4);
    h = m3Fnv(h, &posSize, 4);
    h = m3Fnv(h, policy, (int32_t)strlen(policy));
    return h;
}

bool PoolSane(int32_t mx, int32_t fh, int32_t fc, int32_t rc, int32_t cap)
{
    return mx >= 0 && mx <= cap && fh >= -1 && fh < cap && fc >= 0 && fc <= cap && rc >= 0 &&
           rc <= cap && (fc == 0 || fh >= 0);
}

bool AllZero(const uint8_t* p, int64_t n)
{
    for (int64_t i = 0; i < n; ++i)
    {
        if (p[i] != 0)
        {
            return false;
        }
    }
    return true;
}

int32_t ReadI32(const uint8_t* p)
{
    int32_t x;
    memcpy(&x, p, 4);
    return x;
}

enum class Mode
{
    kMeasure, // sum the block sizes
    kCheck,   // validate an input, write nothing
    kRead,    // input -> world
    kWrite,   // world -> output
};

// Canonical content of a carried block in a world built here: zeros, or
// -1 in every 32-bit word (unset slot indices).
enum class Fill
{
    kZero,
    kMinusOne,
};

// One pass over the fixed blocks, in the reference's order
// (snapshot.c:161-474).
class BlockWalk
{
public:
    BlockWalk(Mode mode, const uint8_t* in, uint8_t* out, std::vector<uint8_t>* carry)
        : mode_(mode), in_(in), out_(out), carry_(carry)
    {
    }

    // A block this path keeps in the world.
    void Keep(void* field, int64_t bytes)
    {
        if (mode_ == Mode::kRead)
        {
            memcpy(field, in_ + cursor_, (size_t)bytes);
        }
        else if (mode_ == Mode::kWrite)
        {
            memcpy(out_ + cursor_, field, (size_t)bytes);
        }
        cursor_ += bytes;
    }
    // A block this path carries: read into the carry, written back from
    // it (or canonically for a world built here).
    void Carry(int64_t bytes, Fill fill)
    {
        if (mode_ == Mode::kRead)
        {
            carry_->insert(carry_->end(), in_ + cursor_, in_ + cursor_ + bytes);
        }
        else if (mode_ == Mode::kWrite)
        {
            uint8_t* dst = out_ + cursor_;
            if (carry_ != nullptr && !carry_->empty())
            {
                memcpy(dst, carry_->data() + carried_, (size_t)bytes);
                carried_ += bytes;
            }
            else if (fill == Fill::kZero)
            {
                memset(dst, 0, (size_t)bytes);
            }
            else
            {
                memset(dst, 0xFF, (size_t)bytes);
            }
        }
        cursor_ += bytes;
    }
    // The liveness array of a pool this path does not model: on restore
    // it must describe no live object.
    void Empty(int64_t bytes, const char* what)
    {
        if (mode_ == Mode::kCheck && unsupported_ == nullptr && !AllZero(in_ + cursor_, bytes))
        {
            unsupported_ = what;
        }
        Carry(bytes, Fill::kZero);
    }
    // Where the next block starts in the input (check pass only).
    const uint8_t* Here() const { return mode_ == Mode::kCheck ? in_ + cursor_ : nullptr; }
    int64_t cursor() const { return cursor_; }
    const char* unsupported() const { return unsupported_; }
    // Writing a world built here (no restored bytes to carry).
    bool WritesOwn() const
    {
        return mode_ == Mode::kWrite && (carry_ == nullptr || carry_->empty());
    }

private:
    Mode mode_;
    const uint8_t* in_;
    uint8_t* out_;
    std::vector<uint8_t>* carry_;
    int64_t cursor_ = 0;
    int64_t carried_ = 0;
    const char* unsupported_ = nullptr;
};

// Pool data the walk moves that lives outside the image: the hull
// pool's counts, generations and liveness, the free-queue rings, and
// (check pass) where the shape type and liveness blocks sit in the input.
struct PoolBlocks
{
    std::vector<int32_t> hullRefs;
    std::vector<uint16_t> hullGens;
    std::vector<uint8_t> hullAlive;
    std::vector<int32_t> bodyQueue;
    std::vector<int32_t> shapeQueue;
    std::vector<int32_t> hullQueue;
    std::vector<int32_t> jointQueue;
    // The heightfield pool of a world built here (shape.c:549-566): slots
    // 0 .. count-1 live, reference count 1, generation 0, queue empty.
    std::vector<int32_t> hfRefs;
    std::vector<uint16_t> hfGens;
    std::vector<uint8_t> hfAlive;
    std::vector<int32_t> hfQueue;
    std::vector<char> names;
    const uint8_t* shapeType = nullptr;
    const uint8_t* shapeAlive = nullptr;
    const uint8_t* hfIndex = nullptr;
    const uint8_t* proxyId = nullptr;
    const uint8_t* treeNodes = nullptr;

    void Size(const m3HostWorld* w)
    {
        hullRefs.assign((size_t)w->shapeCap, 0);
        hullGens.assign((size_t)w->shapeCap, 0);
        hullAlive.assign((size_t)w->shapeCap, 0);
        bodyQueue.assign((size_t)w->bodyCap, 0);
        shapeQueue.assign((size_t)w->shapeCap, 0);
        hullQueue.assign((size_t)w->shapeCap, 0);
        jointQueue.assign((size_t)w->jointCap, 0);
        hfRefs.assign((size_t)w->shapeCap, 0);
        hfGens.assign((size_t)w->shapeCap, 0);
        hfAlive.assign((size_t)w->shapeCap, 0);
        hfQueue.assign((size_t)w->shapeCap, 0);
        names.assign((size_t)w->bodyCap * kBodyNameBytes, 0);
    }
    // The world's pools as the walk writes them.
    void From(const m3HostWorld* w)
    {
        Size(w);
        for (size_t h = 0; h < w->hullRefs.size(); ++h)
        {
            hullRefs[h] = w->hullRefs[h];
            hullAlive[h] = w->hullRefs[h] > 0 ? 1 : 0;
        }
        hullGens = w->hullGen;
        bodyQueue = w->bodyFree.queue;
        if (w->bodyNames.size() == names.size())
        {
            names = w->bodyNames;
        }
        shapeQueue = w->shapeFree.queue;
        hullQueue = w->hullFree.queue;
        jointQueue = w->jointFree.queue;
        for (size_t f = 0; f < w->hfHeaders.size(); ++f)
        {
            hfRefs[f] = 1;
            hfAlive[f] = 1;
        }
    }
};

void WalkFixed(BlockWalk& b, const m3HostWorld* w, const m3WorldView& v, PoolBlocks& pb)
{
    m3WorldScalars* sc = v.sc;
    const int64_t nb = w->bodyCap;
    const int64_t ns = w->shapeCap;
    const int64_t nj = w->jointCap;
    const int64_t np = w->pairCap;
    const int64_t nv = w->voxelCap;
    const int64_t nc = w->charCap;
    const int64_t nh = w->vehicleCap;
    const int64_t nf = w->softCap;
    const int64_t nm = w->meshCap;
    const int64_t W = kVehicleWheels;

    // Bodies.
    b.Keep(v.xf, 40 * nb);
    b.Keep(v.v, 12 * nb);
    b.Keep(v.w, 12 * nb);
    b.Keep(v.invMass, 4 * nb);
    b.Keep(v.invI, 36 * nb);
    b.Keep(v.inertia, 36 * nb);
    b.Keep(v.lc, 12 * nb);
    b.Keep(v.gravityScale, 4 * nb);
    b.Keep(v.linDamp, 4 * nb);
    b.Keep(v.angDamp, 4 * nb);
    b.Keep(v.btype, nb);
    b.Keep(v.awake, nb);
    b.Keep(v.sleepTime, 4 * nb);
    b.Keep(v.bullet, nb);
    b.Keep(v.minExt, 4 * nb);
    b.Keep(v.maxExt, 4 * nb);
    b.Keep(v.userData, 8 * nb);
    b.Keep(pb.names.data(), kBodyNameBytes * nb); // debug names, never hashed
    b.Keep(v.force, 12 * nb);
    b.Keep(v.torque, 12 * nb);
    b.Keep(v.enabled, nb);
    b.Keep(v.locks, nb);
    b.Keep(v.sleepThreshold, 4 * nb);
    b.Keep(v.canSleep, nb);
    b.Keep(v.hasTarget, nb);
    b.Keep(v.target, 40 * nb);
    // World tuning and wind.
    b.Keep(&sc->contactHertz, 4);
    b.Keep(&sc->contactDampingRatio, 4);
    b.Keep(&sc->contactPushMaxSpeed, 4);
    b.Keep(&sc->restitutionThreshold, 4);
    b.Keep(&sc->maximumLinearSpeed, 4);
    b.Keep(&sc->maximumAngularSpeed, 4);
    b.Keep(&sc->sleepEnabled, 1);
    b.Keep(&sc->continuousEnabled, 1);
    b.Keep(&sc->hitEventThreshold, 4);
    b.Keep(&sc->windDir, 12);
    b.Keep(&sc->windSpeed, 4);
    b.Keep(&sc->windGustHertz, 4);
    b.Keep(&sc->windGustScale, 4);
    b.Keep(&sc->windPhase, 4);
    // Body pool.
    b.Keep(v.bodyGen, 2 * nb);
    b.Keep(v.bodyAlive, nb);
    b.Keep(pb.bodyQueue.data(), 4 * nb);
    b.Keep(v.shapeHead, 4 * nb);

    // Shapes.
    b.Keep(v.shapeBody, 4 * ns);
    pb.shapeType = b.Here();
    b.Keep(v.shapeType, ns);
    b.Keep(v.geom, 32 * ns);
    b.Keep(v.density, 4 * ns);
    b.Keep(v.friction, 4 * ns);
    b.Keep(v.restitution, 4 * ns);
    b.Keep(v.shapeUserData, 8 * ns);
    b.Keep(v.shapeNext, 4 * ns);
    b.Keep(v.shapeGen, 2 * ns);
    pb.shapeAlive = b.Here();
    b.Keep(v.shapeAlive, ns);
    b.Keep(pb.shapeQueue.data(), 4 * ns);

    b.Keep(v.keys0, 8 * np);
    // The broadphase: proxy ids and tree nodes.
    pb.proxyId = b.Here();
    b.Keep(v.proxyId, 4 * ns);
    pb.treeNodes = b.Here();
    b.Keep(v.treeNodes, (int64_t)sizeof(m3TreeNode) * 2 * ns);
    b.Keep(v.hullIndex, 4 * ns);
    // Hull reference counts and pool.
    b.Keep(pb.hullRefs.data(), 4 * ns);
    b.Keep(pb.hullGens.data(), 2 * ns);
    b.Keep(pb.hullAlive.data(), ns);
    b.Keep(pb.hullQueue.data(), 4 * ns);
    b.Carry(4 * ns, Fill::kMinusOne); // mesh index per shape
    b.Keep(v.sensor, ns);
    b.Keep(v.rolling, 4 * ns);
    b.Keep(v.hitEvents, ns);
    b.Keep(v.preSolve, ns);
    b.Keep(v.surfVel, 12 * ns);
    b.Keep(v.localPos, 12 * ns);
    b.Keep(v.localRot, 16 * ns);
    b.Keep(v.hasOffset, ns);
    b.Keep(v.category, 8 * ns);
    b.Keep(v.mask, 8 * ns);
    b.Keep(v.group, 4 * ns);

    // Voxel chunks and heightfield pools.
    b.Carry(kVoxelChunkBytes * nv + 4 * nv + 2 * nv, Fill::kZero);
    b.Empty(nv, "voxel chunks");
    b.Carry(4 * nv, Fill::kZero);
    b.Carry(4 * ns, Fill::kMinusOne); // voxel index per shape
    pb.hfIndex = b.Here();
    b.Keep(v.hfIndex, 4 * ns); // heightfield index per shape
    if (b.WritesOwn() && !w->hfHeaders.empty())
    {
        // The heightfield pool of a world built here.
        b.Keep(pb.hfRefs.data(), 4 * ns);
        b.Keep(pb.hfGens.data(), 2 * ns);
        b.Keep(pb.hfAlive.data(), ns);
        b.Keep(pb.hfQueue.data(), 4 * ns);
    }
    else
    {
        // As restored (or a fresh world's empty pool): reference counts,
        // generations, liveness, free queue.
        b.Carry(4 * ns + 2 * ns + ns + 4 * ns, Fill::kZero);
    }
    // Characters.
    b.Carry(4 * nc, Fill::kMinusOne); // body
    b.Carry(nc * (4 * 6 + 1 + 12 + 4 + 4 + 4 + 2 + 2), Fill::kZero);
    b.Empty(nc, "characters");
    b.Carry(4 * nc, Fill::kZero);
    // Vehicles.
    b.Carry(4 * nh, Fill::kMinusOne); // chassis
    b.Carry(nh * (2 + 4 + 4 + 4 + 4 + 8), Fill::kZero);
    b.Carry(nh * W * (12 + 12 + 4 + 4 + 4 + 4 + 4 + 1 + 4), Fill::kZero);
    b.Carry(nh * (1 + 4 + 4 + 4), Fill::kZero);
    b.Carry(nh * W * (4 + 1), Fill::kZero);
    b.Carry(nh * (4 + 4 + 4 + 4), Fill::kZero);
    b.Carry(nh * W * 4, Fill::kZero);
    b.Carry(nh * (1 + 4 + 4 * kEngineCurve + 4 * kEngineCurve + 4 + 4 * kGears + 4 + 4 + 4 + 4),
            Fill::kZero);
    b.Carry(nh * W * 4, Fill::kZero);
    b.Carry(nh * (4 + 4 + 4 + 1 + 1 + 4 + 4), Fill::kZero);
    b.Carry(2 * nh, Fill::kZero);
    b.Empty(nh, "vehicles");
    b.Carry(4 * nh, Fill::kZero);
    // Soft bodies.
    b.Carry(nf * (4 + 4 + 4 + 4 + 4 + 2 + 2 + 2 + 4 + 4 + 4), Fill::kZero);
    b.Carry(nf * kSoftTets * (2 * 4 + 4), Fill::kZero);
    b.Carry(nf * kSoftParticles * 24, Fill::kZero);
    b.Carry(nf * (4 + 4 + 4 + 8), Fill::kZero);
    b.Carry(nf * kSoftParticles * (24 + 24 + 4 + 12), Fill::kZero);
    b.Carry(nf * kSoftEdges * (2 + 2 + 4), Fill::kZero);
    b.Carry(nf * 4, Fill::kZero);
    b.Carry(nf * kSoftAnchors * (4 + 4 + 2 + 12), Fill::kZero);
    b.Carry(nf * 4, Fill::kZero);
    b.Carry(nf * kSoftAnchors * (4 + 4 + 2 + 4), Fill::kZero);
    b.Carry(2 * nf, Fill::kZero);
    b.Empty(nf, "soft bodies");
    b.Carry(4 * nf, Fill::kZero);
    // Mesh pool.
    b.Carry(4 * nm + 2 * nm, Fill::kZero);
    b.Empty(nm, "meshes");
    b.Carry(4 * nm, Fill::kZero);

    // Joints.
    b.Keep(v.jtype, nj);
    b.Keep(v.jbodyA, 4 * nj);
    b.Keep(v.jbodyB, 4 * nj);
    b.Keep(v.jlocalA, 12 * nj);
    b.Keep(v.jlocalB, 12 * nj);
    b.Keep(v.jcollide, nj);
    b.Keep(v.jimpulse, 12 * nj);
    b.Keep(v.jperp, 12 * nj);
    b.Keep(v.jlimitImp, 12 * nj);
    b.Keep(v.jangular, 12 * nj);
    b.Keep(v.jframeA, 16 * nj);
    b.Keep(v.jframeB, 16 * nj);
    b.Keep(v.jflags, nj);
    b.Keep(v.jmotor, 12 * nj);
    b.Keep(v.jbreak, 12 * nj);
    b.Keep(v.jspring, 12 * nj);
    b.Keep(v.jtargetScalar, 4 * nj);
    b.Keep(v.jtargetQ, 16 * nj);
    b.Keep(v.jspringImp, 12 * nj);
    b.Keep(v.jlimits, 12 * nj);
    // Generic-joint modes and ranges, pulley anchors: joint types the
    // step refuses, carried.
    b.Carry(2 * nj + 12 * nj * 4 + 24 * nj * 2, Fill::kZero);
    // Water volumes.
    b.Carry(kWaterVolumes * (24 + 24 + 4 + 4 + 4 + 12 + 2), Fill::kZero);
    b.Empty(kWaterVolumes, "water volumes");
    b.Carry(4 * kWaterVolumes, Fill::kZero);
    b.Keep(v.jnextA, 4 * nj);
    b.Keep(v.jnextB, 4 * nj);
    b.Keep(v.jointHead, 4 * nb);
    b.Keep(v.jointGen, 2 * nj);
    b.Keep(v.jointAlive, nj);
    b.Keep(pb.jointQueue.data(), 4 * nj);
    b.Keep(v.man0, (int64_t)sizeof(m3Manifold) * np);
}

// Bytes of one hull slot's content in the tail (snapshot.c:513-528).
int64_t HullContentBytes(int32_t vc, int32_t fc, int32_t ic, int32_t ec)
{
    return 4 + 12 + 36 + 12 + 12LL * vc + (int64_t)fc * (12 + 4 + 1 + 2) + ic + 6LL * ec;
}

// Moves one hull slot's content between a slab and the tail, in the
// tail's field order; `toSlab` reads the tail.
void HullContent(uint8_t* p, m3HullData* h, bool toSlab)
{
    auto move = [&p, toSlab](void* field, int64_t n) {
        if (toSlab)
        {
            memcpy(field, p, (size_t)n);
        }
        else
        {
            memcpy(p, field, (size_t)n);
        }
        p += n;
    };
    const int32_t vc = h->vertexCount;
    const int32_t fc = h->faceCount;
    move(&h->unitMass, 4);
    move(&h->unitCom, 12);
    move(&h->unitInertiaCom, 36);
    move(&h->center, 12);
    move(h->vertices, 12LL * vc);
    move(h->faceNormals, 12LL * fc);
    move(h->faceOffsets, 4LL * fc);
    move(h->faceVertCounts, fc);
    move(h->faceVertStart, 2LL * fc);
    move(h->faceIndices, h->indexCount);
    move(h->edges, 6LL * h->edgeCount);
}

void SetRing(m3FreeRing& ring, std::vector<int32_t>& queue, int32_t head, int32_t count,
             int32_t retired)
{
    ring.queue.swap(queue);
    ring.head = head < 0 ? 0 : head;
    ring.count = count;
    ring.retired = retired;
}

int64_t FixedBytes(const m3HostWorld* w)
{
    PoolBlocks none;
    BlockWalk measure(Mode::kMeasure, nullptr, nullptr, nullptr);
    WalkFixed(measure, w, w->hv, none);
    return measure.cursor();
}

// Tail bytes of a world as this library writes it: empty mesh slots,
// the hull slots' counts and content, empty heightfield slots.
int64_t TailBytes(const m3HostWorld* w)
{
    int64_t n = 8LL * w->meshCap + 12LL * w->shapeCap;
    for (const m3HeightFieldDev& hf : w->hfHeaders)
    {
        n += hf.nx > 0 ? 8 + 4LL * hf.nx * hf.nz : 0;
    }
    for (int32_t h = 0; h < w->shapeCap; ++h)
    {
        n += 16;
        if (h < (int32_t)w->hulls.size() && w->hulls[(size_t)h].vertexCount > 0)
        {
            const m3HullData& d = w->hulls[(size_t)h];
            n += HullContentBytes(d.vertexCount, d.faceCount, d.indexCount, d.edgeCount);
        }
    }
    return n;
}
} // namespace

// snapshot.c:603-611 (world.h:203): the exact size m3World_Snapshot
// writes; -1 for a stale id.
extern "C" int32_t m3World_SnapshotSize(m3WorldId worldId)
{
    m3gpuClearError();
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr || m3gpuSyncHost(w) != M3GPU_OK)
    {
        return -1;
    }
    return (int32_t)((int64_t)sizeof(SnapshotHeader) + FixedBytes(w) + TailBytes(w));
}

// snapshot.c:613-678 (world.h:204): writes the world's snapshot, byte
// for byte what the reference writes for the same world; returns the
// size, or -1 for a stale id, a null buffer or too small a capacity.
extern "C" int32_t m3World_Snapshot(m3WorldId worldId, void* out, int32_t capacity)
{
    m3gpuClearError();
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr || out == nullptr || m3gpuSyncHost(w) != M3GPU_OK ||
        m3gpuDownloadPairTails(w) != M3GPU_OK)
    {
        return -1;
    }
    if (w->hv.sc->treeTracked == 0)
    {
        m3gpuSetError(M3GPU_ERR_UNSUPPORTED, "m3World_Snapshot: the world keeps no tree");
        return -1;
    }
    if (w->hfHeaders.size() != w->hfAtRestore && !w->snapshotCarry.empty())
    {
        m3gpuSetError(M3GPU_ERR_UNSUPPORTED,
                      "m3World_Snapshot: heightfields created after a restore");
        return -1;
    }
    const int64_t fixed = FixedBytes(w);
    const int64_t size = (int64_t)sizeof(SnapshotHeader) + fixed + TailBytes(w);
    if (capacity < size)
    {
        return -1;
    }
    uint8_t* bytes = (uint8_t*)out;
    const m3WorldScalars* sc = w->hv.sc;
    SnapshotHeader hd;
    memset(&hd, 0, sizeof(hd));
    if (w->snapshotHeaderCarry.size() == sizeof(hd))
    {
        // Cursors of the pools this path does not model, as restored.
        memcpy(&hd, w->snapshotHeaderCarry.data(), sizeof(hd));
    }
    hd.magic = kSnapshotMagic;
    hd.formatVersion = kSnapshotVersion;
    hd.configHash = ConfigHash();
    hd.stepCount = sc->stepCount;
    hd.bodyCapacity = w->bodyCap;
    hd.maxIndex = sc->bodyMax;
    hd.freeHead = w->bodyFree.head;
    hd.freeCount = w->bodyFree.count;
    hd.retiredCount = w->bodyFree.retired;
    hd.shapeCapacity = w->shapeCap;
    hd.shapeMaxIndex = sc->shapeMax;
    hd.shapeFreeHead = w->shapeFree.head;
    hd.shapeFreeCount = w->shapeFree.count;
    hd.shapeRetiredCount = w->shapeFree.retired;
    hd.pairCount = sc->pairCount;
    hd.treeRoot = sc->treeRoot;
    hd.treeFreeList = sc->treeFreeList;
    hd.hullMaxIndex = sc->hullMax;
    hd.hullFreeHead = w->hullFree.head;
    hd.hullFreeCount = w->hullFree.count;
    hd.hullRetiredCount = w->hullFree.retired;
    hd.reserved[0] = 0;
    hd.reserved[1] = 0;
    hd.meshCapacity = w->meshCap;
    hd.jointCapacity = w->jointCap;
    hd.jointMaxIndex = sc->jointMax;
    hd.jointFreeHead = w->jointFree.head;
    hd.jointFreeCount = w->jointFree.count;
    hd.jointRetiredCount = w->jointFree.retired;
    hd.charCapacity = w->charCap;
    hd.voxelCapacity = w->voxelCap;
    hd.gravity = sc->gravity;
    memcpy(bytes, &hd, sizeof(hd));

    // The current pair buffer is the one the snapshot's blocks name.
    m3WorldView v = w->hv;
    if (sc->pairBuf != 0)
    {
        v.keys0 = w->hv.keys1;
        v.man0 = w->hv.man1;
    }
    PoolBlocks pb;
    pb.From(w);
    std::vector<uint8_t> carry = w->snapshotCarry;
    BlockWalk write(Mode::kWrite, nullptr, bytes + sizeof(hd), &carry);
    WalkFixed(write, w, v, pb);

    uint8_t* p = bytes + sizeof(hd) + fixed;
    memset(p, 0, 8 * (size_t)w->meshCap);
    p += 8 * (size_t)w->meshCap;
    m3HullData empty;
    memset(&empty, 0, sizeof(empty));
    for (int32_t h = 0; h < w->shapeCap; ++h)
    {
        m3HullData* d = h < (int32_t)w->hulls.size() ? &w->hulls[(size_t)h] : &empty;
        const int32_t counts[4] = {d->vertexCount, d->faceCount, d->indexCount, d->edgeCount};
        memcpy(p, counts, 16);
        p += 16;
        if (d->vertexCount > 0)
        {
            HullContent(p, d, false);
            p += HullContentBytes(d->vertexCount, d->faceCount, d->indexCount, d->edgeCount);
        }
    }
    for (int32_t f = 0; f < w->shapeCap; ++f)
    {
        if (f < (int32_t)w->hfHeaders.size() && w->hfHeaders[(size_t)f].nx > 0)
        {
            // A heightfield: counts, cell, extremes, samples.
            const m3HeightFieldDev& hf = w->hfHeaders[(size_t)f];
            memcpy(p, &hf.nx, 4);
            memcpy(p + 4, &hf.nz, 4);
            memcpy(p + 8, &hf.cellSize, 4);
            memcpy(p + 12, &hf.minHeight, 4);
            memcpy(p + 16, &hf.maxHeight, 4);
            const size_t samples = (size_t)hf.nx * (size_t)hf.nz;
            memcpy(p + 20, w->hfSamples.data() + hf.sampleStart, 4 * samples);
            p += 20 + 4 * samples;
            continue;
        }
        // An empty heightfield slot: no samples, its cell size as carried.
        memset(p, 0, 12);
        if (w->heightFieldCellCarry.size() == (size_t)w->shapeCap)
        {
            memcpy(p + 8, &w->heightFieldCellCarry[(size_t)f], 4);
        }
        p += 12;
    }
    return (int32_t)size;
}

// snapshot.c:680-931 (world.h:205): restores a snapshot taken by the
// reference (or by this library) into a world created with the same
// capacities.  Refuses, leaving the world untouched, on a foreign format
// or build, mismatched capacities, corrupt pool cursors or counts, a
// size that does not match the content, and (reported as
// M3GPU_ERR_UNSUPPORTED) on content this path does not model: meshes,
// voxels, heightfields, characters, vehicles, soft bodies, water
// volumes.
extern "C" bool m3World_Restore(m3WorldId worldId, const void* data, int32_t size)
{
    m3gpuClearError();
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: stale world or short buffer");
        return false;
    }
    return m3gpuRestoreWorld(w, data, size);
}

// The restore itself, on a world object (one of the table's, or one
// built by m3gpuNewWorld on a serving thread).
bool m3gpuRestoreWorld(m3HostWorld* w, const void* data, int32_t size)
{
    if (data == nullptr || size < (int32_t)sizeof(SnapshotHeader))
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: stale world or short buffer");
        return false;
    }
    const uint8_t* raw = (const uint8_t*)data;
    SnapshotHeader hd;
    memcpy(&hd, raw, sizeof(hd));
    if (hd.magic != kSnapshotMagic || hd.formatVersion != kSnapshotVersion ||
        hd.configHash != ConfigHash() || hd.bodyCapacity != w->bodyCap ||
        hd.shapeCapacity != w->shapeCap || hd.meshCapacity != w->meshCap ||
        hd.jointCapacity != w->jointCap || hd.voxelCapacity != w->voxelCap ||
        hd.charCapacity != w->charCap)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: foreign format or world shape");
        return false;
    }
    if (!PoolSane(hd.maxIndex, hd.freeHead, hd.freeCount, hd.retiredCount, w->bodyCap) ||
        !PoolSane(hd.shapeMaxIndex, hd.shapeFreeHead, hd.shapeFreeCount, hd.shapeRetiredCount,
                  w->shapeCap) ||
        !PoolSane(hd.hullMaxIndex, hd.hullFreeHead, hd.hullFreeCount, hd.hullRetiredCount,
                  w->shapeCap) ||
        !PoolSane(hd.jointMaxIndex, hd.jointFreeHead, hd.jointFreeCount, hd.jointRetiredCount,
                  w->jointCap) ||
        !PoolSane(hd.meshMaxIndex, hd.meshFreeHead, hd.meshFreeCount, hd.meshRetiredCount,
                  w->meshCap) ||
        !PoolSane(hd.voxelMaxIndex, hd.voxelFreeHead, hd.voxelFreeCount, hd.voxelRetiredCount,
                  w->voxelCap) ||
        !PoolSane(hd.charMaxIndex, hd.charFreeHead, hd.charFreeCount, hd.charRetiredCount,
                  w->charCap) ||
        hd.pairCount < 0 || hd.pairCount > w->pairCap || hd.treeRoot < -1 ||
        hd.treeRoot >= 2 * w->shapeCap || hd.treeFreeList < -1 ||
        hd.treeFreeList >= 2 * w->shapeCap)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: corrupt pool cursors");
        return false;
    }

    // Sizes first: the fixed blocks, then the count-derived tail parsed
    // straight from the buffer (snapshot.c:725-826).
    int64_t cursor = (int64_t)sizeof(SnapshotHeader) + FixedBytes(w);
    const char* unsupported = nullptr;
    for (int32_t m = 0; m < w->meshCap; ++m)
    {
        if (size - cursor < 8)
        {
            m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: truncated mesh section");
            return false;
        }
        const int32_t vc = ReadI32(raw + cursor);
        const int32_t tc = ReadI32(raw + cursor + 4);
        cursor += 8;
        if (vc < 0 || vc > kMeshMaxVerts || tc < 0 || tc > kMeshMaxTris || (vc == 0) != (tc == 0))
        {
            m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: corrupt mesh counts");
            return false;
        }
        if (tc > 0)
        {
            const int64_t content = 12LL * vc + 6LL * tc + tc + 4 + kMeshMaterialBytes + tc;
            if (size - cursor < content)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: truncated mesh content");
                return false;
            }
            cursor += content;
            unsupported = "meshes";
        }
    }
    std::vector<int64_t> hullAt((size_t)w->shapeCap, -1);
    for (int32_t h = 0; h < w->shapeCap; ++h)
    {
        if (size - cursor < 16)
        {
            m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: truncated hull section");
            return false;
        }
        const int32_t vc = ReadI32(raw + cursor);
        const int32_t fc = ReadI32(raw + cursor + 4);
        const int32_t ic = ReadI32(raw + cursor + 8);
        const int32_t ec = ReadI32(raw + cursor + 12);
        if (vc < 0 || vc > M3_HULL_MAX_VERTS || fc < 0 || fc > M3_HULL_MAX_FACES || ic < 0 ||
            ic > M3_HULL_MAX_FACE_INDICES || ec < 0 || ec > M3_HULL_MAX_HALF_EDGES ||
            (vc == 0 && (fc | ic | ec) != 0))
        {
            m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: corrupt hull counts");
            return false;
        }
        hullAt[(size_t)h] = cursor;
        cursor += 16;
        if (vc > 0)
        {
            const int64_t content = HullContentBytes(vc, fc, ic, ec);
            if (size - cursor < content)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: truncated hull content");
                return false;
            }
            if (h >= hd.hullMaxIndex)
            {
                unsupported = "hull content past the hull pool's end";
            }
            cursor += content;
        }
    }
    std::vector<m3HeightFieldDev> hfSlots; // nx == 0: an empty slot
    std::vector<float> hfCells((size_t)w->shapeCap, 0.0f);
    for (int32_t f = 0; f < w->shapeCap; ++f)
    {
        if (size - cursor < 12)
        {
            m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: truncated heightfield section");
            return false;
        }
        const int32_t nx = ReadI32(raw + cursor);
        const int32_t nz = ReadI32(raw + cursor + 4);
        memcpy(&hfCells[(size_t)f], raw + cursor + 8, 4);
        cursor += 12;
        if (nx < 0 || nx > kHeightFieldMaxDim || nz < 0 || nz > kHeightFieldMaxDim ||
            (nx == 0) != (nz == 0) || (nx > 0 && (nx < 2 || nz < 2)))
        {
            m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: corrupt heightfield counts");
            return false;
        }
        if (nx > 0)
        {
            const int64_t content = 8 + 4LL * nx * nz;
            if (size - cursor < content)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: truncated heightfield");
                return false;
            }
            m3HeightFieldDev hf;
            hf.nx = nx;
            hf.nz = nz;
            memcpy(&hf.cellSize, raw + cursor - 4, 4);
            memcpy(&hf.minHeight, raw + cursor, 4);
            memcpy(&hf.maxHeight, raw + cursor + 4, 4);
            hf.sampleStart = (int32_t)(cursor + 8); // byte offset, rebased at commit
            if (!(hf.cellSize > 0.0f) || !(hf.cellSize < 3.4e38f))
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: corrupt heightfield cell");
                return false;
            }
            hfSlots.resize((size_t)f + 1);
            hfSlots[(size_t)f] = hf;
            cursor += content;
        }
    }
    if (cursor != size)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: size does not match the content");
        return false;
    }

    // Check pass: nothing is written yet.
    PoolBlocks pb;
    pb.Size(w);
    BlockWalk check(Mode::kCheck, raw + sizeof(SnapshotHeader), nullptr, nullptr);
    WalkFixed(check, w, w->hv, pb);
    if (unsupported == nullptr)
    {
        unsupported = check.unsupported();
    }
    for (int32_t s = 0; s < hd.shapeMaxIndex && unsupported == nullptr; ++s)
    {
        const uint8_t t = pb.shapeType[s];
        if (pb.shapeAlive[s] != 0 && t != M3_SHAPE_SPHERE && t != M3_SHAPE_PLANE &&
            t != M3_SHAPE_HULL && t != M3_SHAPE_CAPSULE && t != M3_SHAPE_HEIGHTFIELD)
        {
            unsupported = "mesh or voxel shapes";
        }
        if (pb.shapeAlive[s] != 0 && t == M3_SHAPE_HEIGHTFIELD)
        {
            // A live heightfield shape names a slot holding samples.
            const int32_t f = ReadI32(pb.hfIndex + 4LL * s);
            if (f < 0 || f >= (int32_t)hfSlots.size() || hfSlots[(size_t)f].nx == 0)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: corrupt heightfield index");
                return false;
            }
        }
    }
    if (unsupported != nullptr)
    {
        m3gpuSetError(M3GPU_ERR_UNSUPPORTED, "m3World_Restore: %s are not on the device path",
                      unsupported);
        return false;
    }
    {
        // The broadphase tree must be well formed before the device
        // walks it (copied out of the input: it may be unaligned).
        const int32_t cap = 2 * w->shapeCap;
        std::vector<m3TreeNode> nodes((size_t)cap);
        std::vector<int32_t> proxy((size_t)w->shapeCap);
        memcpy(nodes.data(), pb.treeNodes, sizeof(m3TreeNode) * (size_t)cap);
        memcpy(proxy.data(), pb.proxyId, 4 * (size_t)w->shapeCap);
        if (!m3TreeValid(nodes.data(), cap, hd.treeRoot, hd.treeFreeList, proxy.data(),
                         pb.shapeAlive, pb.shapeType, hd.shapeMaxIndex))
        {
            m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Restore: malformed broadphase tree");
            return false;
        }
    }

    // Read pass.
    std::vector<uint8_t> carry;
    BlockWalk read(Mode::kRead, raw + sizeof(SnapshotHeader), nullptr, &carry);
    WalkFixed(read, w, w->hv, pb);
    m3WorldScalars* sc = w->hv.sc;
    sc->stepCount = hd.stepCount;
    sc->gravity = hd.gravity;
    sc->bodyMax = hd.maxIndex;
    sc->shapeMax = hd.shapeMaxIndex;
    sc->jointMax = hd.jointMaxIndex;
    sc->hullMax = hd.hullMaxIndex;
    sc->pairCount = hd.pairCount;
    sc->pairBuf = 0;
    sc->treeRoot = hd.treeRoot;
    sc->treeFreeList = hd.treeFreeList;
    sc->lastInvH = 0.0f;
    sc->status = M3GPU_OK;
    sc->statusDetail = 0;
    sc->brokenCount = 0;
    w->brokenDrained = 0;
    // Both pair buffers hold the restored arrays: the step writes the
    // new list into the other one, and the parts of the arrays past the
    // live pairs must read the same from either.
    memcpy(w->hv.keys1, w->hv.keys0, sizeof(uint64_t) * (size_t)w->pairCap);
    memcpy(w->hv.man1, w->hv.man0, sizeof(m3Manifold) * (size_t)w->pairCap);
    SetRing(w->bodyFree, pb.bodyQueue, hd.freeHead, hd.freeCount, hd.retiredCount);
    SetRing(w->shapeFree, pb.shapeQueue, hd.shapeFreeHead, hd.shapeFreeCount,
            hd.shapeRetiredCount);
    SetRing(w->jointFree, pb.jointQueue, hd.jointFreeHead, hd.jointFreeCount,
            hd.jointRetiredCount);
    SetRing(w->hullFree, pb.hullQueue, hd.hullFreeHead, hd.hullFreeCount, hd.hullRetiredCount);
    w->hullGen = pb.hullGens;
    w->hulls.resize((size_t)hd.hullMaxIndex);
    if (hd.hullMaxIndex > 0)
    {
        memset(w->hulls.data(), 0, sizeof(m3HullData) * (size_t)hd.hullMaxIndex);
    }
    w->hullRefs.assign(pb.hullRefs.begin(), pb.hullRefs.begin() + hd.hullMaxIndex);
    w->hullIndexByContent.clear();
    for (int32_t h = 0; h < hd.hullMaxIndex; ++h)
    {
        m3HullData* d = &w->hulls[(size_t)h]; // zeroed by the assign above
        const uint8_t* p = raw + hullAt[(size_t)h];
        d->vertexCount = ReadI32(p);
        d->faceCount = ReadI32(p + 4);
        d->indexCount = ReadI32(p + 8);
        d->edgeCount = ReadI32(p + 12);
        if (d->vertexCount > 0)
        {
            HullContent((uint8_t*)p + 16, d, true);
        }
        if (w->hullRefs[(size_t)h] > 0)
        {
            w->hullIndexByContent.emplace(m3HullKey(d), h);
        }
    }
    w->snapshotCarry.swap(carry);
    w->bodyNames.swap(pb.names);
    w->snapshotHeaderCarry.assign(raw, raw + sizeof(SnapshotHeader));
    w->heightFieldCellCarry = hfCells;
    // The heightfield slots and samples (the index per shape came with
    // the fixed blocks).
    w->hfHeaders.clear();
    w->hfSamples.clear();
    for (m3HeightFieldDev hf : hfSlots)
    {
        if (hf.nx > 0)
        {
            const size_t samples = (size_t)hf.nx * (size_t)hf.nz;
            const size_t at = w->hfSamples.size();
            w->hfSamples.resize(at + samples);
            memcpy(w->hfSamples.data() + at, raw + hf.sampleStart, 4 * samples);
            hf.sampleStart = (int32_t)at;
        }
        else
        {
            memset(&hf, 0, sizeof(hf));
        }
        w->hfHeaders.push_back(hf);
    }
    w->hfVersion += 1;
    w->hfAtRestore = w->hfHeaders.size();
    // The image on the host is now the world; the next step uploads it,
    // the pair arrays in full.  Device snapshot slots saved before are
    // void.
    w->structure += 1;
    w->deviceAhead = false;
    w->hostDirty = true;
    w->pairTailsToDevice = true;
    w->pairTailsOnDevice = false;
    // Events are observations of a step, never state (snapshot.c:867-879).
    m3MarkEventEpoch(w, false);
    return true;
}

// world.c:3187-3218 (world.h:606): replays a recorded command stream:
// records of (op, payload bytes, payload).  Covered ops: steps (run on
// the GPU), velocity sets, forces, torques and impulses (also at a world
// point), motion locks, the fast-rotation flag, joint break thresholds and
// the world settings.  The stream is
// validated whole before anything is applied (framing, op, payload
// size, body ids, finite vectors, step arguments), so a refusal leaves
// the world untouched, as the reference's snapshot-backed rollback does.
// An op outside that set is refused with M3GPU_ERR_UNSUPPORTED.
extern "C" bool m3World_JournalReplay(m3WorldId worldId, const void* data, int32_t size)
{
    m3gpuClearError();
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr || data == nullptr || size < 0)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3World_JournalReplay: stale world or bad buffer");
        return false;
    }
    if (m3gpuSyncHost(w) != M3GPU_OK)
    {
        return false;
    }
    std::vector<m3JournalRecordView> records;
    if (!m3ParseJournal(w, (const uint8_t*)data, size, &records))
    {
        return false;
    }
    for (const m3JournalRecordView& r : records)
    {
        if (r.op == M3_OP_STEP)
        {
            if (m3gpuStepBatch(&w, 1, r.dt, r.substeps, 1) != M3GPU_OK)
            {
                return false;
            }
            continue;
        }
        if (m3gpuSyncHost(w) != M3GPU_OK)
        {
            return false;
        }
        if (m3IsWorldSettingOp(r.op))
        {
            m3ApplyWorldSetting(w, r.op, r.setting);
        }
        else if (m3IsHostBodyOp(r.op))
        {
            m3ApplyHostBodyOp(w, r);
        }
        else if (m3IsHostShapeOp(r.op))
        {
            m3ApplyHostShapeOp(w, r);
        }
        else if (m3IsHostJointOp(r.op))
        {
            m3ApplyHostJointOp(w, r);
        }
        else
        {
            m3ApplyBodyOp(w->hv, r.op, r.body, r.v);
        }
        w->hostDirty = true;
    }
    return true;
}

bool m3ParseJournal(const m3HostWorld* w, const uint8_t* stream, int32_t size,
                    std::vector<m3JournalRecordView>* out)
{
    out->clear();
    int64_t cursor = 0;
    while (cursor < size)
    {
        if (size - cursor < 8)
        {
            m3gpuSetError(M3GPU_ERR_INVALID, "journal: truncated record header");
            return false;
        }
        const int32_t op = ReadI32(stream + cursor);
        const int32_t bytes = ReadI32(stream + cursor + 4);
        cursor += 8;
        if (bytes < 0 || bytes > size - cursor)
        {
            m3gpuSetError(M3GPU_ERR_INVALID, "journal: truncated payload");
            return false;
        }
        const uint8_t* payload = stream + cursor;
        cursor += bytes;
        m3JournalRecordView r{};
        r.op = op;
        if (op == M3_OP_STEP)
        {
            // world.c:1623-1641: {float dt; int32 substeps}.
            if (bytes != 8)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "journal: bad step record");
                return false;
            }
            memcpy(&r.dt, payload, 4);
            memcpy(&r.substeps, payload + 4, 4);
            if (!(r.dt > 0.0f) || r.substeps < 1 || r.substeps > M3_MAX_SUBSTEPS)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "journal: bad step arguments");
                return false;
            }
        }
        else if (m3IsBodyOp(op))
        {
            // world.c:1571-1611, 2283-2321: {m3BodyId id; m3Vec3 v}; the
            // id is retargeted to this world.
            if (bytes != 20)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "journal: bad body command record");
                return false;
            }
            m3BodyId id;
            memcpy(&id, payload, 8);
            memcpy(&r.v, payload + 8, 12);
            const int32_t index = id.index1 - 1;
            if (index < 0 || index >= w->hv.sc->bodyMax || w->hv.bodyAlive[index] == 0 ||
                w->hv.bodyGen[index] != id.generation || !isfinite(r.v.x) || !isfinite(r.v.y) ||
                !isfinite(r.v.z))
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "journal: stale body or non-finite command");
                return false;
            }
            r.body = index;
        }
        else if (op == M3_OP_JOINT_SET_BREAK)
        {
            // world.c:3111-3133: {m3JointId id; float maxForce, maxTorque}.
            if (bytes != 16)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "journal: bad joint break record");
                return false;
            }
            m3JointId id;
            memcpy(&id, payload, 8);
            memcpy(&r.v.x, payload + 8, 4);
            memcpy(&r.v.y, payload + 12, 4);
            const int32_t j = id.index1 - 1;
            if (j < 0 || j >= w->hv.sc->jointMax || w->hv.jointAlive[j] == 0 ||
                w->hv.jointGen[j] != id.generation || !isfinite(r.v.x) || !isfinite(r.v.y) ||
                r.v.x < 0.0f || r.v.y < 0.0f)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "journal: stale joint or bad thresholds");
                return false;
            }
            r.body = j;
            r.generation = id.generation;
        }
        else if (m3IsHostBodyOp(op))
        {
            // world.c:2323-2465, 2904-2928: forces and impulses at a world
            // point {m3BodyId; m3Vec3; m3Pos3}, poses {m3BodyId;
            // m3Transform}, sleep controls {m3BodyId; float; int32}, and
            // locks, types and flags {m3BodyId; uint32}; the id is
            // retargeted to this world.
            const bool point =
                op == M3_OP_APPLY_FORCE_AT_POINT || op == M3_OP_APPLY_IMPULSE_AT_POINT;
            const bool pose = op == M3_OP_SET_TRANSFORM || op == M3_OP_SET_TARGET_TRANSFORM;
            const int32_t want = point || pose                     ? 48
                                 : op == M3_OP_SET_BODY_NAME         ? 8 + M3_BODY_NAME_BYTES
                                 : op == M3_OP_SET_SLEEP_CONTROLS    ? 16
                                                                     : 12;
            if (bytes != want)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "journal: bad body record (op %d)", op);
                return false;
            }
            m3BodyId id;
            memcpy(&id, payload, 8);
            const int32_t index = id.index1 - 1;
            bool ok = index >= 0 && index < w->hv.sc->bodyMax && w->hv.bodyAlive[index] != 0 &&
                      w->hv.bodyGen[index] == id.generation;
            if (point)
            {
                memcpy(&r.v, payload + 8, 12);
                memcpy(&r.point, payload + 24, 24);
                ok = ok && isfinite(r.v.x) && isfinite(r.v.y) && isfinite(r.v.z) &&
                     isfinite(r.point.x) && isfinite(r.point.y) && isfinite(r.point.z);
            }
            else if (pose)
            {
                memcpy(&r.point, payload + 8, 24);
                memcpy(&r.rotation, payload + 32, 16);
                const m3Quat q = r.rotation;
                const float qq = q.x * q.x + q.y * q.y + q.z * q.z + q.w * q.w;
                ok = ok && isfinite(r.point.x) && isfinite(r.point.y) && isfinite(r.point.z) &&
                     isfinite(q.x) && isfinite(q.y) && isfinite(q.z) && isfinite(q.w) &&
                     qq > 0.98f && qq < 1.02f;
            }
            else if (op == M3_OP_SET_BODY_NAME)
            {
                // Any bytes; the last is forced to the terminator
                // (world.c:2620-2641).
                memcpy(r.name, payload + 8, M3_BODY_NAME_BYTES);
                r.name[M3_BODY_NAME_BYTES - 1] = 0;
            }
            else if (op == M3_OP_SET_SLEEP_CONTROLS)
            {
                // Any threshold: a non-positive or NaN one is the default.
                memcpy(&r.setting[0], payload + 8, 4);
                int32_t canSleep;
                memcpy(&canSleep, payload + 12, 4);
                r.bits = canSleep != 0 ? 1u : 0u;
            }
            else
            {
                memcpy(&r.bits, payload + 8, 4);
                ok = ok && (op != M3_OP_SET_ALLOW_FAST_ROTATION || r.bits <= 1u);
                if (op == M3_OP_SET_TYPE)
                {
                    // The reference keeps the low byte whatever it holds;
                    // a byte that names no body type is refused here.
                    r.bits &= 0xFFu;
                    ok = ok && r.bits <= (uint32_t)M3_BODY_DYNAMIC;
                }
            }
            if (!ok)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "journal: stale body or bad values (op %d)", op);
                return false;
            }
            r.body = index;
        }
        else if (m3IsHostJointOp(op))
        {
            // world.c:3050-3179: limits and motor {m3JointId; int32; float;
            // float} (finite; limits ordered, a motor joint's budgets not
            // negative), collide {m3JointId; int32}, spring {m3JointId;
            // int32; float; float} (hertz finite and positive, damping
            // finite and not negative), target {m3JointId; float; m3Quat}
            // (finite); the id is retargeted to this world.
            const int32_t want = op == M3_OP_JOINT_SET_COLLIDE  ? 12
                                 : op == M3_OP_JOINT_SET_TARGET ? 28
                                                                : 20;
            if (bytes != want)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "journal: bad joint record (op %d)", op);
                return false;
            }
            m3JointId id;
            memcpy(&id, payload, 8);
            const int32_t j = id.index1 - 1;
            bool ok = j >= 0 && j < w->hv.sc->jointMax && w->hv.jointAlive[j] != 0 &&
                      w->hv.jointGen[j] == id.generation;
            int32_t enable = 0;
            if (op == M3_OP_JOINT_SET_TARGET)
            {
                memcpy(&r.setting[0], payload + 8, 4);
                memcpy(&r.rotation, payload + 12, 16);
                const m3Quat q = r.rotation;
                ok = ok && isfinite(r.setting[0]) && isfinite(q.x) && isfinite(q.y) &&
                     isfinite(q.z) && isfinite(q.w);
            }
            else
            {
                memcpy(&enable, payload + 8, 4);
                if (op != M3_OP_JOINT_SET_COLLIDE)
                {
                    memcpy(&r.setting[0], payload + 12, 8);
                    const float a = r.setting[0];
                    const float b = r.setting[1];
                    ok = ok && isfinite(a) && isfinite(b);
                    if (ok && op == M3_OP_JOINT_SET_LIMITS)
                    {
                        ok = w->hv.jtype[j] == m3_motorJoint ? a >= 0.0f && b >= 0.0f : a <= b;
                    }
                    if (op == M3_OP_JOINT_SET_SPRING)
                    {
                        ok = ok && a > 0.0f && b >= 0.0f;
                    }
                }
            }
            if (!ok)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "journal: stale joint or bad values (op %d)", op);
                return false;
            }
            r.bits = enable != 0 ? 1u : 0u;
            r.body = j;
        }
        else if (m3IsHostShapeOp(op))
        {
            // world.c:2500-2555, 3021-3049: materials {m3ShapeId; float}
            // (finite, not negative), densities {m3ShapeId; float; int32}
            // (finite, positive), flags {m3ShapeId; int32}; the id is
            // retargeted to this world.
            const bool flag =
                op == M3_OP_ENABLE_SHAPE_HIT_EVENTS || op == M3_OP_ENABLE_SHAPE_PRESOLVE;
            if (bytes != (op == M3_OP_SET_SHAPE_DENSITY ? 16 : 12))
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "journal: bad shape record (op %d)", op);
                return false;
            }
            m3ShapeId id;
            memcpy(&id, payload, 8);
            const int32_t index = id.index1 - 1;
            bool ok = index >= 0 && index < w->hv.sc->shapeMax && w->hv.shapeAlive[index] != 0 &&
                      w->hv.shapeGen[index] == id.generation;
            if (flag)
            {
                int32_t on;
                memcpy(&on, payload + 8, 4);
                r.bits = on != 0 ? 1u : 0u;
            }
            else
            {
                memcpy(&r.setting[0], payload + 8, 4);
                const float value = r.setting[0];
                ok = ok && isfinite(value) &&
                     (op == M3_OP_SET_SHAPE_DENSITY ? value > 0.0f : value >= 0.0f);
                if (op == M3_OP_SET_SHAPE_DENSITY)
                {
                    int32_t update;
                    memcpy(&update, payload + 12, 4);
                    r.bits = update != 0 ? 1u : 0u;
                }
            }
            if (!ok)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "journal: stale shape or bad value (op %d)", op);
                return false;
            }
            r.body = index;
        }
        else if (m3IsWorldSettingOp(op))
        {
            // world.c:2485-2620, 2943-2990, 3006-3020: the settings'
            // records, their payloads checked as the reference's replay
            // checks them (hostile bytes fail loudly).
            const int32_t want = op == M3_OP_SET_WIND                                   ? 24
                                 : op == M3_OP_SET_GRAVITY || op == M3_OP_SET_CONTACT_TUNING ? 12
                                                                                       : 4;
            if (bytes != want)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "journal: bad setting record (op %d)", op);
                return false;
            }
            memset(r.setting, 0, sizeof(r.setting));
            memcpy(r.setting, payload, (size_t)bytes);
            const float* f = r.setting;
            bool ok = true;
            switch (op)
            {
            case M3_OP_SET_GRAVITY:
                ok = isfinite(f[0]) && isfinite(f[1]) && isfinite(f[2]);
                break;
            case M3_OP_SET_CONTACT_TUNING:
                ok = isfinite(f[0]) && f[0] > 0.0f && isfinite(f[1]) && f[1] > 0.0f &&
                     isfinite(f[2]) && f[2] > 0.0f;
                break;
            case M3_OP_SET_RESTITUTION_THRESHOLD:
            case M3_OP_SET_HIT_EVENT_THRESHOLD:
                ok = isfinite(f[0]) && f[0] >= 0.0f;
                break;
            case M3_OP_SET_MAXIMUM_LINEAR_SPEED:
            case M3_OP_SET_MAXIMUM_ANGULAR_SPEED:
                ok = isfinite(f[0]) && f[0] > 0.0f;
                break;
            case M3_OP_SET_WIND:
                ok = isfinite(f[0]) && isfinite(f[1]) && isfinite(f[2]) && isfinite(f[3]) &&
                     f[3] >= 0.0f && isfinite(f[4]) && f[4] >= 0.0f && isfinite(f[5]) &&
                     f[5] >= 0.0f;
                break;
            default: // the sleeping and continuous flags: any value
                break;
            }
            if (!ok)
            {
                m3gpuSetError(M3GPU_ERR_INVALID, "journal: bad setting values (op %d)", op);
                return false;
            }
        }
        else if (op <= 0)
        {
            m3gpuSetError(M3GPU_ERR_INVALID, "journal: unknown op %d", op);
            return false;
        }
        else
        {
            m3gpuSetError(M3GPU_ERR_UNSUPPORTED, "journal: op %d is not on the device path", op);
            return false;
        }
        out->push_back(r);
    }
    return true;
}

void m3JournalAppend(m3HostWorld* w, int32_t op, const void* payload, int32_t bytes)
{
    if (!w->journalActive)
    {
        return;
    }
    const int64_t need = 8 + (int64_t)bytes;
    if (w->journalCursor + need > w->journalCapacity)
    {
        w->journalOverflow = true;
        w->journalActive = false;
        return;
    }
    uint8_t* out = w->journalBuffer + w->journalCursor;
    memcpy(out, &op, 4);
    memcpy(out + 4, &bytes, 4);
    memcpy(out + 8, payload, (size_t)bytes);
    w->journalCursor += (int32_t)need;
}

void m3JournalUnrecordable(m3HostWorld* w)
{
    if (w->journalActive)
    {
        w->journalOverflow = true;
        w->journalActive = false;
    }
}

// world.c:1369-1382 (world.h:600): starts recording into the caller's
// buffer; false for a stale id, a null or tiny buffer, or a session
// already running.
extern "C" bool m3World_JournalBegin(m3WorldId worldId, void* buffer, int32_t capacity)
{
    m3gpuClearError();
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr || buffer == nullptr || capacity < 8 || w->journalActive)
    {
        return false;
    }
    w->journalBuffer = (uint8_t*)buffer;
    w->journalCapacity = capacity;
    w->journalCursor = 0;
    w->journalActive = true;
    w->journalOverflow = false;
    return true;
}

// world.c:1384-1398 (world.h:601): ends the session; the recorded byte
// count, or -1 after an overflow (or, here, after a call this path does
// not record: world, body, shape or joint creation).
extern "C" int32_t m3World_JournalEnd(m3WorldId worldId)
{
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr)
    {
        return -1;
    }
    const int32_t bytes = w->journalOverflow ? -1 : w->journalCursor;
    w->journalBuffer = nullptr;
    w->journalCapacity = 0;
    w->journalCursor = 0;
    w->journalActive = false;
    w->journalOverflow = false;
    return bytes;
}
