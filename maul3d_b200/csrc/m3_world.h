// Host-side world object: the persistent slab image (m3_layout.h), the
// interned hull store, and the device residency bookkeeping.  Internal
// to the library; the public surface is include/maul3d_b200.h.
#ifndef M3_WORLD_H
#define M3_WORLD_H

#include "m3_layout.h"

#include <stdint.h>
#include <stdlib.h>
#include <new>
#include <unordered_map>
#include <mutex>
#include <vector>

// Host memory for world images and hull buffers (hostmem.cpp): page-
// granular blocks from large mappings, page-locked chunk by chunk when a
// world becomes device-resident, so uploads are asynchronous DMA copies.
#define M3_HOST_PAGE 4096
// Bytes of one body's debug name, terminator included (world_internal.h:197).
#define M3_BODY_NAME_BYTES 32

// Size classes of the host and device block allocators: `bytes` in
// granules, rounded up to m * 2^k granules with 8 <= m < 16 (at most an
// eighth over), so that freed blocks of worlds of similar size serve the
// next ones instead of fresh memory.
inline size_t m3SizeClass(size_t bytes, size_t granule)
{
    const size_t n = bytes == 0 ? 1 : (bytes + granule - 1) / granule;
    if (n <= 16)
    {
        return n * granule;
    }
    const int k = 63 - __builtin_clzll((unsigned long long)n) - 3;
    const size_t m = (n + ((size_t)1 << k) - 1) >> k;
    return (m << k) * granule;
}
void* m3HostAlloc(size_t bytes);
void m3HostFree(void* p, size_t bytes);
// Page-lock every chunk not locked yet (one driver call per chunk).
int32_t m3HostLockAll(void);
// The library's device once it is up (page-locking host memory on any
// thread), else -1 (device.cpp).
int m3gpuLockDevice(void);
// Whether [p, p + bytes) lies in a locked chunk.
bool m3HostIsLocked(const void* p, size_t bytes);
// The device's address of [p, p + bytes) when it lies in a locked (and
// mapped) chunk, else null.
const uint8_t* m3HostDevicePointer(const void* p, size_t bytes);

// One copy of a batched upload, done on the GPU from page-locked, mapped
// host memory (upload.cu): `bytes` raw bytes, or, when `hulls` > 0, that
// many interned hull slabs of which only the parts their counts use.
struct m3UploadItem
{
    const uint8_t* src;
    uint8_t* dst;
    int64_t bytes;
    int32_t hulls;
    int32_t pad;
};
int32_t m3gpuLaunchUpload(const m3UploadItem* items, int32_t count);
// Bytes of one hull slab an upload copies (the parts its counts use).
int64_t m3HullUsedBytes(const m3HullData* h);
// Content key of an interned hull slab for the dedup index: FNV-1a over
// its counts and used vertices (equal slabs give equal keys; lookups
// confirm with a full compare).
uint64_t m3HullKey(const m3HullData* h);


template <class T> struct m3PageAllocator
{
    using value_type = T;
    m3PageAllocator() = default;
    template <class U> m3PageAllocator(const m3PageAllocator<U>&)
    {
    }
    T* allocate(size_t n)
    {
        return (T*)m3HostAlloc(n * sizeof(T));
    }
    void deallocate(T* p, size_t n)
    {
        m3HostFree(p, n * sizeof(T));
    }
    // Elements are default-initialised (no zeroing on resize): the owners
    // clear what they allocate with one memset.
    template <class U> void construct(U* p)
    {
        ::new ((void*)p) U;
    }
    template <class U, class... Args> void construct(U* p, Args&&... args)
    {
        ::new ((void*)p) U(static_cast<Args&&>(args)...);
    }
    template <class U> bool operator==(const m3PageAllocator<U>&) const
    {
        return true;
    }
    template <class U> bool operator!=(const m3PageAllocator<U>&) const
    {
        return false;
    }
};

// A slot pool's free queue as the reference keeps it (allocator.c:178-
// 218): a ring over `capacity` entries read from `head`, so a snapshot
// carries it byte for byte.  Slots whose generation reached 0xFFFF are
// retired instead of queued.
struct m3FreeRing
{
    std::vector<int32_t> queue;
    int32_t head = 0;
    int32_t count = 0;
    int32_t retired = 0;

    void Init(int32_t capacity)
    {
        queue.assign((size_t)capacity, 0);
        head = 0;
        count = 0;
        retired = 0;
    }
    bool Pop(int32_t* index)
    {
        if (count <= 0)
        {
            return false;
        }
        *index = queue[(size_t)head];
        head = (head + 1) % (int32_t)queue.size();
        count -= 1;
        return true;
    }
    void Push(int32_t index)
    {
        queue[(size_t)((head + count) % (int32_t)queue.size())] = index;
        count += 1;
    }
};

// Device milliseconds of a world's last step, per stage (the batch it
// was stepped in), for m3World_GetProfile.
struct m3StepProfile
{
    float step = 0.0f;
    float broadphase = 0.0f;
    float narrowphase = 0.0f;
    float prepare = 0.0f;
    float solve = 0.0f;
    float finish = 0.0f; // continuous phase and sleep
    bool valid = false;
};

// The broadphase tree is state only snapshots read: each step records
// its leaf moves in a ring of this many per-step lists in the world's
// scratch, and the moves are replayed into the tree later -- once
// M3_TREE_REPLAY_AT steps have gathered (on the tree's own stream, beside
// the following steps), when the ring would overflow, or at once when
// something reads or overwrites the tree.
#define M3_TREE_LAG 32
#define M3_TREE_REPLAY_AT 16

struct m3HostWorld
{
    int32_t slot = -1;
    uint16_t generation = 0;
    int32_t bodyCap = 0;
    int32_t shapeCap = 0;
    int32_t jointCap = 0;
    int32_t pairCap = 0;

    // Persistent image (host copy) and its view.
    std::vector<uint8_t, m3PageAllocator<uint8_t>> image;
    int64_t persistentBytes = 0;
    m3WorldView hv{};

    // Interned hull slabs live outside the fixed-capacity image: the
    // pool is sized by the hulls actually interned (count-derived, as
    // the reference's snapshot treats them).
    std::vector<m3HullData, m3PageAllocator<m3HullData>> hulls;
    // Recycled slots of each pool, reused first (FIFO).  The device's
    // joint breakage appends to jointFree through the jbroken ring,
    // drained up to `brokenDrained` at each download.
    m3FreeRing bodyFree;
    m3FreeRing shapeFree;
    m3FreeRing hullFree;
    m3FreeRing jointFree;
    int32_t brokenDrained = 0;
    // Hull slot generations (the pool's liveness is the reference count).
    std::vector<uint16_t> hullGen;
    // Snapshot bytes of the state this path does not model, as the last
    // restore read them, written back by the next snapshot (empty for a
    // world built here: it writes a fresh world's values).
    std::vector<uint8_t> snapshotCarry;
    std::vector<uint8_t> snapshotHeaderCarry;
    // Debug names, M3_BODY_NAME_BYTES a body slot (body.c:711-760): saved
    // in snapshots, never hashed, never on the device.
    std::vector<char> bodyNames;
    std::vector<float> heightFieldCellCarry;
    // Event streams of the world's last step (world.h:207-313): computed
    // on the first read after a step from the device's two pair lists and
    // its ring of broken joints.  stepEpoch counts device step calls and
    // restores; the streams are current when eventsEpoch equals it.
    uint64_t stepEpoch = 0;
    bool lastEpochIsStep = false;
    uint64_t eventsEpoch = 0;
    std::vector<m3ContactEvent> beginEvents;
    std::vector<m3ContactEvent> endEvents;
    std::vector<m3ContactEvent> sensorBeginEvents;
    std::vector<m3ContactEvent> sensorEndEvents;
    std::vector<m3JointBreakEvent> jointBreakEvents;
    // Body move events, built on their own first read (they copy every
    // body's transform back).
    uint64_t moveEventsEpoch = 0;
    std::vector<m3BodyMoveEvent> moveEvents;
    // Hit events, likewise built on their own first read.
    uint64_t hitEventsEpoch = 0;
    std::vector<m3HitEvent> hitEvents;
    int32_t hitEventsDropped = 0;
    // Journal recording (world.c:1348-1398): records appended to the
    // caller's buffer while active; overflow latches and ends it.
    uint8_t* journalBuffer = nullptr;
    int32_t journalCapacity = 0;
    int32_t journalCursor = 0;
    bool journalActive = false;
    bool journalOverflow = false;
    // Capacities of the pools this path does not model; they size the
    // snapshot's blocks (snapshot.c:161-600).
    int32_t meshCap = 0;
    int32_t voxelCap = 0;
    int32_t charCap = 0;
    int32_t vehicleCap = 0;
    int32_t softCap = 0;
    std::vector<int32_t> hullRefs;
    std::unordered_multimap<uint64_t, int32_t> hullIndexByContent;
    // Heightfield slots (hfMax in use) and their samples; hfVersion
    // counts content changes, so the device copy is refreshed only then.
    std::vector<m3HeightFieldDev> hfHeaders;
    std::vector<float> hfSamples;
    uint64_t hfVersion = 0;
    size_t hfAtRestore = 0; // slots the last restore left

    // Device residency.
    uint8_t* dslab = nullptr;        // persistent + scratch
    int64_t dslabBytes = 0;
    int64_t scratchBytes = 0;
    m3HullData* dhulls = nullptr;    // device hull pool
    int32_t dhullCap = 0;
    uint8_t* dhf = nullptr;          // device heightfield slots + samples
    size_t dhfBytes = 0;
    uint64_t dhfVersion = 0;
    m3WorldView dv{};                // device view (device addresses)
    bool hostDirty = true;           // host image newer than device
    bool deviceAhead = false;        // device newer than host image
    // The pair arrays past the live list are snapshot bytes (what longer
    // lists of earlier steps left there).  A restore sets them on the
    // host, and the next upload copies the whole current buffer; a step
    // changes them on the device, and a snapshot downloads them.
    bool pairTailsToDevice = false;
    bool pairTailsOnDevice = false;
    m3StepProfile profile;

    // Device snapshot slots (m3gpu_slots_reserve): `slotCount` copies of
    // the slab's persistent part, one after another from `dslots`, and
    // per slot the host state a step can change (joint slots freed by
    // breakage and drained into the free queue) and the structure it
    // belongs to.  `structure` counts the host's structural changes:
    // bodies, shapes and joints created, snapshots restored.
    struct DeviceSlot
    {
        bool valid = false;
        uint64_t structure = 0;
        m3FreeRing jointFree;
        int32_t brokenDrained = 0;
    };
    uint8_t* dslots = nullptr;
    int32_t slotCount = 0;
    std::vector<DeviceSlot> slots;
    uint64_t structure = 0;
    // The steps whose moves sit in the ring, oldest first: for each, the
    // sequence number of the tree launch replaying it (0 while no launch
    // covers it yet; those are the newest `treeUnlaunched` entries); and
    // whether the scratch's copy of the tree leaves' bounds is current
    // (it is kept by the broadphase once made).
    uint64_t treeSlotSeq[M3_TREE_LAG] = {};
    int32_t treeFirst = 0;
    int32_t treeCount = 0;
    int32_t treeUnlaunched = 0;
    bool leafBoxValid = false;
};

// Points a device view at the world's pools outside the slab.
inline void m3AttachDevicePools(m3HostWorld* w, m3WorldView* view)
{
    view->hulls = w->dhulls;
    const size_t headers = m3AlignUp((int64_t)(w->hfHeaders.size() * sizeof(m3HeightFieldDev)), 16);
    view->hfs = w->dhf != nullptr ? (const m3HeightFieldDev*)w->dhf : nullptr;
    view->hfSamples = w->dhf != nullptr ? (const float*)(w->dhf + headers) : nullptr;
}

// Convex hull of a point cloud into a hull slab (quickhull.cpp): the
// reference's QuickHull with unit-density mass properties; the half-edge
// table is the caller's to build.
bool m3QuickHull(const m3Vec3* points, int32_t count, m3HullData* out);

// Registry (world.cpp).
m3HostWorld* m3gpuWorldFromId(m3WorldId id);
m3HostWorld* m3gpuWorldFromIndex0(uint16_t index0);

// The library's shared device state (the selected device, the batch
// tables, streams, events, staging buffers, the device chunk allocator
// and every world's residency) sits behind one process-wide recursive
// lock, taken by each internal entry below that touches it.  Distinct
// worlds may therefore be stepped, hashed, snapshotted and restored from
// distinct host threads (the reference's threading contract): their
// device work is serialised, each call's result is the one it gets alone.
std::recursive_mutex& m3gpuDeviceMutex();
#define M3_DEVICE_GUARD std::lock_guard<std::recursive_mutex> m3DeviceGuard_(m3gpuDeviceMutex())

// Residency (device.cpp).
extern uint64_t g_m3ResidencyEpoch;
// Host-to-device bytes copied by uploads (device.cpp).
extern int64_t g_m3UploadedBytes;
// Device blocks allocated and freed (device.cpp).
extern int64_t g_m3DevAllocCalls;
extern int64_t g_m3DevFreeCalls;
int32_t m3gpuEnsureDevice(void);
int32_t m3gpuReserve(m3HostWorld* w);
int32_t m3gpuUpload(m3HostWorld* w);
// Upload many worlds with one kernel where their host memory allows; the
// rest one world at a time.
int32_t m3gpuUploadBatch(m3HostWorld** worlds, int32_t count);
int32_t m3gpuDownload(m3HostWorld* w);
// The world's step status word (M3GPU_OK or its refusal), read from the
// device when it is resident.
int32_t m3gpuWorldStatus(m3HostWorld* w);
// The current pair buffer in full, device to host (for a snapshot).
int32_t m3gpuDownloadPairTails(m3HostWorld* w);
void m3gpuRelease(m3HostWorld* w);
// Make the host image current before a host read or write.
int32_t m3gpuSyncHost(m3HostWorld* w);
// One validated journal record (snapshot.cpp): a step or a body command.
struct m3JournalRecordView
{
    int32_t op;
    int32_t body; // body slot, or joint slot for a joint record
    m3Vec3 v;     // command vector, or (maxForce, maxTorque) of a joint record
    float dt;
    int32_t substeps;
    uint16_t generation; // joint records
    float setting[6];    // world-setting records: their payload's words
    m3Pos3 point;        // force and impulse at a point: the world point; a pose's position
    m3Quat rotation;     // a pose's rotation
    uint32_t bits;       // motion locks, a type, a flag (canSleep for sleep controls)
    char name[M3_BODY_NAME_BYTES]; // a body name, zero-filled past its terminator
};
// Applies a validated world-setting record (world.c:734-783, 1013-1082)
// to the host image: the setting's fields, and for sleeping turned off
// every sleeping dynamic body woken.  world.cpp.
void m3ApplyWorldSetting(m3HostWorld* w, int32_t op, const float* words);
// Applies a validated host-side body command (body.c:170-330, 379-404,
// 663-703) to the host image, the body slot in `r.body`: `v` a force or
// impulse with its world `point`; a pose (`point`, `rotation`); `bits`
// the lock bits, type or flag; `setting[0]` a sleep threshold.  world.cpp.
void m3ApplyHostBodyOp(m3HostWorld* w, const m3JournalRecordView& r);
// Applies a validated shape command (shape.c:1387-1410, 1557-1565) to the
// host image, the shape slot in `r.body`: `setting[0]` the friction,
// restitution, rolling resistance or density; `bits` the flag, or for a
// density whether the body's mass is rebuilt.  world.cpp.
void m3ApplyHostShapeOp(m3HostWorld* w, const m3JournalRecordView& r);
// Applies a validated joint command (joint.c:562-590, 620-624, 1014-1029)
// to the host image, the joint slot in `r.body`: `bits` the enable or
// collide switch; `setting[0..1]` the limits, the motor's speed and
// effort or the spring's hertz and damping ratio; `setting[0]` with
// `rotation` a drive target.  world.cpp.
void m3ApplyHostJointOp(m3HostWorld* w, const m3JournalRecordView& r);
// Parses and validates a whole journal against a world's bodies; false
// (with the error set) on the first bad or unsupported record.
// Worlds outside the world table (world.cpp): built on any thread,
// entered into the table later (the null id and the world deleted when
// the table is full), or deleted without ever entering it.
m3HostWorld* m3gpuNewWorld(const m3WorldDef* def);
m3WorldId m3gpuAttachWorld(m3HostWorld* w);
void m3gpuDeleteWorld(m3HostWorld* w);
// m3World_Restore on a world object (snapshot.cpp).
bool m3gpuRestoreWorld(m3HostWorld* w, const void* data, int32_t size);

bool m3ParseJournal(const m3HostWorld* w, const uint8_t* stream, int32_t size,
                    std::vector<m3JournalRecordView>* out);

// Appends one record to the world's active journal (snapshot.cpp).
void m3JournalAppend(m3HostWorld* w, int32_t op, const void* payload, int32_t bytes);
// Ends an active journal as unrecordable: a call this path cannot record
// happened during the session (snapshot.cpp).
void m3JournalUnrecordable(m3HostWorld* w);

// Queue the joint slots the device freed since the last call (world.cpp).
void m3DrainBrokenJoints(m3HostWorld* w);

// A world's event streams start over: a step just ran on the device
// (`stepped`), or a restore replaced its state (no events until the next
// step).
inline void m3MarkEventEpoch(m3HostWorld* w, bool stepped)
{
    w->stepEpoch += 1;
    w->lastEpochIsStep = stepped;
}

// The device address of the last step's mover list (ascending body
// indices; its length is the scalars' moverCount) in a world's slab
// scratch (step.cu).
const int32_t* m3gpuDeviceMovers(const m3HostWorld* w);
// The device addresses of the last step's per-constraint hit flags and
// hit events (constraint order; the scalars' constraintCount entries).
void m3gpuDeviceHits(const m3HostWorld* w, const uint8_t** flags, const m3HitEvent** hits);

// Step and hash entry points (step.cu).
// `ops` (optional) are body commands applied on the device before the
// first step: m3BodyOp.world indexes `worlds`; per world they apply in
// array order.
int32_t m3gpuStepBatch(m3HostWorld** worlds, int32_t count, float dt, int32_t substeps,
                       int32_t steps, const struct m3BodyOp* ops = nullptr, int32_t opCount = 0);
int32_t m3gpuHashBatch(m3HostWorld** worlds, int32_t count, uint64_t* out);
// Orders the default stream after every tree launch still pending for
// the world (step.cu): anything that reads or overwrites its tree or its
// scratch on the default stream calls this first.
void m3gpuWaitTree(m3HostWorld* w);
// The parallel world hash (hash.cu): one block per world, blocks in
// `order`, out[world] = that world's m3WorldHashView.
int32_t m3gpuLaunchHash(const m3WorldView* views, const int32_t* order, int32_t count,
                        uint64_t* out);

// Error reporting (capi.cpp).
int32_t m3gpuSetError(int32_t code, const char* fmt, ...);
void m3gpuClearError(void);

#endif // M3_WORLD_H
