// The exported C ABI glue: error state, the drop-in step and hash
// entries (solver.c:4322-4355, snapshot.c:932), the batched device
// entries and the white-box readbacks the parity tests use.

#include "m3_world.h"
#include "m3_hash.h"
#include "m3_ops.h"
#include "m3_tree.h"

#include <cuda_runtime.h>

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <vector>

static thread_local int32_t t_error = M3GPU_OK;
static thread_local char t_message[512] = "ok";

int32_t m3gpuSetError(int32_t code, const char* fmt, ...)
{
    t_error = code;
    va_list args;
    va_start(args, fmt);
    vsnprintf(t_message, sizeof(t_message), fmt, args);
    va_end(args);
    return code;
}

void m3gpuClearError(void)
{
    t_error = M3GPU_OK;
    strcpy(t_message, "ok");
}

extern "C" int32_t m3gpu_last_error(void)
{
    return t_error;
}

extern "C" const char* m3gpu_last_error_message(void)
{
    return t_message;
}

extern "C" int m3GetVersion(void)
{
    return 1 * 10000 + 22 * 100 + 0;
}

extern "C" uint64_t m3Hash64(uint64_t h, const void* bytes, int32_t count)
{
    return m3Fnv(h, bytes, count);
}

// solver.c:4332-4354: a step is recorded after it ran ({dt, substeps}).
static void RecordSteps(m3HostWorld* w, float dt, int32_t substeps, int32_t steps)
{
    struct
    {
        float dt;
        int32_t substeps;
    } record = {dt, substeps};
    for (int32_t k = 0; k < steps && w->journalActive; ++k)
    {
        m3JournalAppend(w, M3_OP_STEP, &record, (int32_t)sizeof(record));
    }
}

extern "C" void m3World_Step(m3WorldId worldId, float dt, int32_t substeps)
{
    m3gpuClearError();
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr || !(dt > 0.0f) || substeps < 1 || substeps > M3_MAX_SUBSTEPS)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3World_Step: stale world or invalid dt/substeps");
        return;
    }
    if (m3gpuStepBatch(&w, 1, dt, substeps, 1) == M3GPU_OK)
    {
        RecordSteps(w, dt, substeps, 1);
    }
}

extern "C" uint64_t m3World_Hash(m3WorldId worldId)
{
    m3gpuClearError();
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr)
    {
        return 0;
    }
    if (w->deviceAhead)
    {
        uint64_t h = 0;
        if (m3gpuHashBatch(&w, 1, &h) == M3GPU_OK)
        {
            return h;
        }
        return 0;
    }
    m3WorldView view = w->hv;
    view.hulls = w->hulls.empty() ? nullptr : w->hulls.data();
    return m3WorldHashView(&view);
}

// world.c:917-951: live counts from the (synced) host image, the last
// step's island and colour counts from the device's scalars.
extern "C" m3Counters m3World_GetCounters(m3WorldId worldId)
{
    m3Counters c;
    memset(&c, 0, sizeof(c));
    m3gpuClearError();
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr || m3gpuSyncHost(w) != M3GPU_OK)
    {
        return c;
    }
    const m3WorldView& v = w->hv;
    const m3WorldScalars* sc = v.sc;
    for (int32_t i = 0; i < sc->bodyMax; ++i)
    {
        if (v.bodyAlive[i] != 0)
        {
            c.bodyCount += 1;
            if (v.btype[i] == M3_BODY_DYNAMIC && v.awake[i] != 0)
            {
                c.awakeCount += 1;
            }
        }
    }
    for (int32_t i = 0; i < sc->shapeMax; ++i)
    {
        c.shapeCount += v.shapeAlive[i] != 0 ? 1 : 0;
    }
    for (int32_t i = 0; i < sc->jointMax; ++i)
    {
        c.jointCount += v.jointAlive[i] != 0 ? 1 : 0;
    }
    for (int32_t r : w->hullRefs)
    {
        c.hullCount += r > 0 ? 1 : 0;
    }
    c.contactCount = sc->pairCount;
    c.islandCount = sc->lastIslandCount;
    c.colorCount = sc->lastColorCount;
    c.treeHeight = sc->treeRoot != M3_TREE_NULL ? v.treeNodes[sc->treeRoot].height : 0;
    const int64_t scratch =
        w->scratchBytes > 0 ? w->scratchBytes
                            : m3gpuScratchBytes(w->bodyCap, w->shapeCap, w->jointCap, w->pairCap);
    c.scratchCapacity = scratch > INT32_MAX ? INT32_MAX : (int32_t)scratch;
    c.scratchPeak = c.scratchCapacity;
    c.snapshotBytes = m3World_SnapshotSize(worldId);
    c.allocCalls = g_m3DevAllocCalls;
    c.freeCalls = g_m3DevFreeCalls;
    return c;
}

// world.c:955-965: the last device step's stage times.
extern "C" m3Profile m3World_GetProfile(m3WorldId worldId)
{
    m3Profile p;
    memset(&p, 0, sizeof(p));
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr || !w->profile.valid)
    {
        return p;
    }
    p.step = w->profile.step;
    p.broadphase = w->profile.broadphase;
    p.narrowphase = w->profile.narrowphase;
    p.prepare = w->profile.prepare;
    p.solve = w->profile.solve;
    p.continuous = w->profile.finish;
    return p;
}

static int32_t Resolve(const m3WorldId* ids, int32_t count, std::vector<m3HostWorld*>& out)
{
    if (ids == nullptr || count <= 0)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "empty world list");
    }
    out.resize((size_t)count);
    for (int32_t i = 0; i < count; ++i)
    {
        out[(size_t)i] = m3gpuWorldFromId(ids[i]);
        if (out[(size_t)i] == nullptr)
        {
            return m3gpuSetError(M3GPU_ERR_INVALID, "stale world id at position %d", i);
        }
    }
    return M3GPU_OK;
}

extern "C" int32_t m3gpu_step_worlds(const m3WorldId* worlds, int32_t count, float dt,
                                     int32_t substeps, int32_t steps)
{
    m3gpuClearError();
    if (!(dt > 0.0f) || substeps < 1 || substeps > M3_MAX_SUBSTEPS || steps < 0)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "invalid dt, substeps or steps");
    }
    std::vector<m3HostWorld*> ws;
    int32_t rc = Resolve(worlds, count, ws);
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    if (steps == 0)
    {
        return M3GPU_OK;
    }
    rc = m3gpuStepBatch(ws.data(), count, dt, substeps, steps);
    if (rc == M3GPU_OK)
    {
        for (m3HostWorld* w : ws)
        {
            RecordSteps(w, dt, substeps, steps);
        }
    }
    return rc;
}

// Body commands on the device, then one step (body.c:818-1014 for the
// commands' rules, as m3Body_Apply* / m3Body_Set*Velocity give them): a
// stale body or a non-finite vector is a no-op; forces, torques and
// impulses reach dynamic bodies with mass only.  Recorded in an active
// journal like the calls they replace.
extern "C" int32_t m3gpu_step_worlds_commands(const m3WorldId* worlds, int32_t count, float dt,
                                              int32_t substeps, const m3gpuBodyCommand* commands,
                                              int32_t commandCount)
{
    m3gpuClearError();
    if (!(dt > 0.0f) || substeps < 1 || substeps > M3_MAX_SUBSTEPS || commandCount < 0 ||
        (commandCount > 0 && commands == nullptr))
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "invalid dt, substeps or commands");
    }
    std::vector<m3HostWorld*> ws;
    int32_t rc = Resolve(worlds, count, ws);
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    std::vector<m3BodyOp> ops;
    ops.reserve((size_t)commandCount);
    for (int32_t k = 0; k < commandCount; ++k)
    {
        const m3gpuBodyCommand& c = commands[k];
        if (c.world < 0 || c.world >= count || !m3IsBodyOp(c.op))
        {
            return m3gpuSetError(M3GPU_ERR_INVALID, "command %d: bad world index or op", k);
        }
        m3HostWorld* w = ws[(size_t)c.world];
        // Liveness, type and mass change only through host calls: the
        // host image has them current even while the device is ahead.
        const int32_t index = c.body.index1 - 1;
        if (c.body.world0 != (uint16_t)w->slot || index < 0 || index >= w->hv.sc->bodyMax ||
            w->hv.bodyAlive[index] == 0 || w->hv.bodyGen[index] != c.body.generation ||
            !isfinite(c.v.x) || !isfinite(c.v.y) || !isfinite(c.v.z))
        {
            continue;
        }
        const bool needsMass = c.op != M3_OP_SET_LINEAR_VELOCITY && c.op != M3_OP_SET_ANGULAR_VELOCITY;
        if (needsMass && !(w->hv.btype[index] == M3_BODY_DYNAMIC && w->hv.invMass[index] > 0.0f))
        {
            continue;
        }
        struct
        {
            m3BodyId id;
            m3Vec3 v;
        } record = {c.body, c.v};
        m3JournalAppend(w, c.op, &record, (int32_t)sizeof(record));
        ops.push_back(m3BodyOp{c.world, c.op, index, c.v});
    }
    rc = m3gpuStepBatch(ws.data(), count, dt, substeps, 1, ops.data(), (int32_t)ops.size());
    if (rc == M3GPU_OK)
    {
        for (m3HostWorld* w : ws)
        {
            RecordSteps(w, dt, substeps, 1);
        }
    }
    return rc;
}

// ---------------------------------------------------------------------
// Packing autotuner.  Every packing steps the worlds to the same bits, so
// the tuner times candidates on live steps instead of on copies: each of
// its steps is a real step of the batch.  Candidates are the neighbours of
// the packing in use (each class bound scaled down and up, each class's
// threads per world switched, the two larger classes' shared-memory
// budgets switched, the largest class at two worlds per SM); a
// candidate's step sits between two steps of the packing in use and is
// compared with their mean, so the slow drift of a settling batch
// cancels.  A candidate at least 3 % faster is adopted and its own
// neighbours are tried next.
// ---------------------------------------------------------------------
namespace
{

bool SamePacking(const m3gpuPacking& a, const m3gpuPacking& b)
{
    return memcmp(&a, &b, sizeof(a)) == 0;
}

std::vector<m3gpuPacking> PackingNeighbours(const m3gpuPacking& p)
{
    std::vector<m3gpuPacking> out;
    auto push = [&](const m3gpuPacking& q) {
        if (!(q.minShapes[1] >= 1 && q.minShapes[0] > q.minShapes[1]) || SamePacking(q, p))
        {
            return;
        }
        for (const m3gpuPacking& o : out)
        {
            if (SamePacking(o, q))
            {
                return;
            }
        }
        out.push_back(q);
    };
    m3gpuPacking q = p;
    q.minShapes[0] = p.minShapes[0] * 2 / 3;
    push(q);
    q = p;
    q.minShapes[0] = p.minShapes[0] * 3 / 2;
    push(q);
    q = p;
    q.minShapes[1] = p.minShapes[1] / 2;
    push(q);
    q = p;
    q.minShapes[1] = p.minShapes[1] * 2;
    push(q);
    q = p;
    q.threads[0] = p.threads[0] == 512 ? 256 : 512;
    push(q);
    q = p;
    q.threads[1] = p.threads[1] == 256 ? 128 : 256;
    push(q);
    q = p;
    q.threads[2] = p.threads[2] == 128 ? 256 : 128;
    push(q);
    // The largest class at two worlds per SM: the most shared memory two
    // blocks can have (a 2048-body world's body cache and joint rows fit;
    // its inverse-inertia table stays in global memory), alone and with
    // 256 threads a world (the register file then holds two).
    const int32_t twoPerSm = 113664;
    q = p;
    q.smemBytes[0] = p.smemBytes[0] > twoPerSm ? twoPerSm : 200 * 1024;
    push(q);
    q = p;
    q.threads[0] = 256;
    q.smemBytes[0] = twoPerSm;
    push(q);
    q = p;
    q.smemBytes[1] = p.smemBytes[1] > 54 * 1024 ? 54 * 1024 : 110 * 1024;
    push(q);
    return out;
}

// The last tuning's trials (m3gpu_autotune_trials); guarded by the
// device lock like the tuning itself.
std::vector<m3gpuPackingTrial> g_trials;

} // namespace

extern "C" int32_t m3gpu_autotune_trials(m3gpuPackingTrial* out, int32_t cap)
{
    M3_DEVICE_GUARD;
    m3gpuClearError();
    const int32_t n = (int32_t)g_trials.size();
    for (int32_t i = 0; out != nullptr && i < n && i < cap; ++i)
    {
        out[i] = g_trials[(size_t)i];
    }
    return n;
}

extern "C" int32_t m3gpu_autotune_packing(const m3WorldId* worlds, int32_t count, float dt,
                                          int32_t substeps, int32_t steps, m3gpuPacking* best,
                                          float* bestMs)
{
    M3_DEVICE_GUARD;
    m3gpuClearError();
    if (!(dt > 0.0f) || substeps < 1 || substeps > M3_MAX_SUBSTEPS || steps < 0)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "invalid dt, substeps or steps");
    }
    std::vector<m3HostWorld*> ws;
    int32_t rc = Resolve(worlds, count, ws);
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    m3gpuPacking cur;
    rc = m3gpu_get_packing(&cur);
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    int32_t done = 0;
    // One real step under packing `p`; its prepare and substep stages'
    // device time in *ms.  The broadphase trees' pending moves are
    // replayed first, untimed: a replay launched beside the step (every
    // 16 steps) would share the SMs with it and slow the stages timed.
    auto measure = [&](const m3gpuPacking& p, float* ms) -> int32_t {
        int32_t r = m3gpu_flush_trees(worlds, count);
        if (r == M3GPU_OK)
        {
            r = m3gpu_set_packing(&p);
        }
        if (r == M3GPU_OK)
        {
            r = m3gpuStepBatch(ws.data(), count, dt, substeps, 1);
        }
        if (r != M3GPU_OK)
        {
            return r;
        }
        for (m3HostWorld* w : ws)
        {
            RecordSteps(w, dt, substeps, 1);
        }
        float stage[5];
        r = m3gpu_kernel_ms(stage);
        *ms = stage[2] + stage[3];
        done += 1;
        return r;
    };
    float base = 0.0f;
    g_trials.clear();
    if (steps >= 3)
    {
        rc = measure(cur, &base);
        std::vector<m3gpuPacking> tried(1, cur);
        std::vector<m3gpuPacking> queue = PackingNeighbours(cur);
        size_t next = 0;
        while (rc == M3GPU_OK && done + 2 <= steps && next < queue.size())
        {
            const m3gpuPacking cand = queue[next++];
            bool seen = false;
            for (const m3gpuPacking& t : tried)
            {
                seen = seen || SamePacking(t, cand);
            }
            if (seen)
            {
                continue;
            }
            tried.push_back(cand);
            float candMs = 0.0f;
            float after = 0.0f;
            rc = measure(cand, &candMs);
            if (rc == M3GPU_OK)
            {
                rc = measure(cur, &after);
            }
            if (rc != M3GPU_OK)
            {
                break;
            }
            const float mean = 0.5f * (base + after);
            base = after;
            const bool adopt = mean > 0.0f && candMs < 0.97f * mean;
            g_trials.push_back(m3gpuPackingTrial{cand, candMs, mean, adopt ? 1 : 0});
            if (adopt)
            {
                // Adopted: the next steps use it, and its neighbours
                // come next.
                cur = cand;
                base = candMs;
                queue = PackingNeighbours(cur);
                next = 0;
            }
        }
    }
    // The remaining steps under the packing chosen.
    while (rc == M3GPU_OK && done < steps)
    {
        rc = measure(cur, &base);
    }
    if (rc == M3GPU_OK)
    {
        rc = m3gpu_set_packing(&cur);
    }
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    if (best != nullptr)
    {
        *best = cur;
    }
    if (bestMs != nullptr)
    {
        *bestMs = base;
    }
    return M3GPU_OK;
}

extern "C" int32_t m3gpu_hash_worlds(const m3WorldId* worlds, int32_t count, uint64_t* out)
{
    m3gpuClearError();
    std::vector<m3HostWorld*> ws;
    int32_t rc = Resolve(worlds, count, ws);
    if (rc != M3GPU_OK || out == nullptr)
    {
        return rc != M3GPU_OK ? rc : m3gpuSetError(M3GPU_ERR_INVALID, "null output");
    }
    return m3gpuHashBatch(ws.data(), count, out);
}

// ----------------------------------------------------------------------
// White-box readbacks
// ----------------------------------------------------------------------
static m3HostWorld* Synced(m3WorldId id)
{
    m3HostWorld* w = m3gpuWorldFromId(id);
    if (w == nullptr)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "stale world id");
        return nullptr;
    }
    if (m3gpuSyncHost(w) != M3GPU_OK)
    {
        return nullptr; // the error is set by the failing copy
    }
    return w;
}

extern "C" int32_t m3gpu_body_max(m3WorldId world)
{
    m3HostWorld* w = m3gpuWorldFromId(world);
    return w ? w->hv.sc->bodyMax : -1;
}

extern "C" int32_t m3gpu_pair_count(m3WorldId world)
{
    m3HostWorld* w = Synced(world);
    return w ? w->hv.sc->pairCount : -1;
}

extern "C" int32_t m3gpu_copy_bodies(m3WorldId world, void* transforms, void* lin, void* ang,
                                     uint8_t* awake, float* sleepTimes, int32_t cap)
{
    m3HostWorld* w = Synced(world);
    if (w == nullptr)
    {
        return -1;
    }
    if (cap < w->hv.sc->bodyMax)
    {
        m3gpuSetError(M3GPU_ERR_CAPACITY, "readback room %d below %d body slots", cap,
                      w->hv.sc->bodyMax);
        return -1;
    }
    int32_t n = w->hv.sc->bodyMax;
    memcpy(transforms, w->hv.xf, (size_t)n * sizeof(m3Transform));
    memcpy(lin, w->hv.v, (size_t)n * sizeof(m3Vec3));
    memcpy(ang, w->hv.w, (size_t)n * sizeof(m3Vec3));
    memcpy(awake, w->hv.awake, (size_t)n);
    memcpy(sleepTimes, w->hv.sleepTime, (size_t)n * sizeof(float));
    return n;
}

extern "C" int32_t m3gpu_copy_mass(m3WorldId world, float* invMass, void* invInertia,
                                   void* inertia, void* localCenters, float* minExt,
                                   float* maxExt, int32_t cap)
{
    m3HostWorld* w = Synced(world);
    if (w == nullptr || cap < w->hv.sc->bodyMax)
    {
        return -1;
    }
    int32_t n = w->hv.sc->bodyMax;
    memcpy(invMass, w->hv.invMass, (size_t)n * sizeof(float));
    memcpy(invInertia, w->hv.invI, (size_t)n * sizeof(m3Mat3));
    memcpy(inertia, w->hv.inertia, (size_t)n * sizeof(m3Mat3));
    memcpy(localCenters, w->hv.lc, (size_t)n * sizeof(m3Vec3));
    memcpy(minExt, w->hv.minExt, (size_t)n * sizeof(float));
    memcpy(maxExt, w->hv.maxExt, (size_t)n * sizeof(float));
    return n;
}

extern "C" int32_t m3gpu_copy_pairs(m3WorldId world, uint64_t* keys, void* manifolds, int32_t cap)
{
    m3HostWorld* w = Synced(world);
    if (w == nullptr || cap < w->hv.sc->pairCount)
    {
        return -1;
    }
    int32_t n = w->hv.sc->pairCount;
    const uint64_t* k = w->hv.sc->pairBuf == 0 ? w->hv.keys0 : w->hv.keys1;
    const m3Manifold* m = w->hv.sc->pairBuf == 0 ? w->hv.man0 : w->hv.man1;
    memcpy(keys, k, (size_t)n * sizeof(uint64_t));
    memcpy(manifolds, m, (size_t)n * sizeof(m3Manifold));
    return n;
}

extern "C" int32_t m3gpu_copy_joints(m3WorldId world, void* impulse, void* perp, void* limit,
                                     void* angular, int32_t cap)
{
    m3HostWorld* w = Synced(world);
    if (w == nullptr || cap < w->hv.sc->jointMax)
    {
        return -1;
    }
    int32_t n = w->hv.sc->jointMax;
    memcpy(impulse, w->hv.jimpulse, (size_t)n * sizeof(m3Vec3));
    memcpy(perp, w->hv.jperp, (size_t)n * sizeof(m3Vec3));
    memcpy(limit, w->hv.jlimitImp, (size_t)n * sizeof(m3Vec3));
    memcpy(angular, w->hv.jangular, (size_t)n * sizeof(m3Vec3));
    return n;
}

extern "C" int32_t m3gpu_reserve_worlds(const m3WorldId* worlds, int32_t count)
{
    m3gpuClearError();
    std::vector<m3HostWorld*> ws;
    int32_t rc = Resolve(worlds, count, ws);
    for (int32_t i = 0; rc == M3GPU_OK && i < count; ++i)
    {
        rc = m3gpuReserve(ws[(size_t)i]);
    }
    return rc;
}

extern "C" int32_t m3gpu_upload_worlds(const m3WorldId* worlds, int32_t count)
{
    m3gpuClearError();
    std::vector<m3HostWorld*> ws;
    int32_t rc = Resolve(worlds, count, ws);
    std::vector<m3HostWorld*> dirty;
    for (int32_t i = 0; rc == M3GPU_OK && i < count; ++i)
    {
        m3HostWorld* w = ws[(size_t)i];
        if (w->hostDirty || w->dslab == nullptr)
        {
            w->hv.sc->status = 0;
            dirty.push_back(w);
        }
    }
    if (rc == M3GPU_OK && !dirty.empty())
    {
        rc = m3gpuUploadBatch(dirty.data(), (int32_t)dirty.size());
    }
    // Uploads from page-locked images are asynchronous: the images must
    // not change under the copies, so return only once they are done.
    const cudaError_t e = cudaStreamSynchronize(0);
    if (rc == M3GPU_OK && e != cudaSuccess)
    {
        rc = m3gpuSetError(M3GPU_ERR_CUDA, "upload: %s", cudaGetErrorString(e));
    }
    return rc;
}

extern "C" int64_t m3gpu_uploaded_bytes(void)
{
    return g_m3UploadedBytes;
}

extern "C" int64_t m3gpu_world_image_bytes(m3WorldId world)
{
    m3HostWorld* w = m3gpuWorldFromId(world);
    if (w == nullptr)
    {
        return -1;
    }
    return w->persistentBytes + (int64_t)w->hulls.size() * (int64_t)sizeof(m3HullData);
}
