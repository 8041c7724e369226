// Serving: many short rollback/verification sessions at once.  A request
// is the reference's replay container (M3J1: a snapshot and the journal
// recorded after it, replay.c:15-136); its answer is the world hash at
// the end of the journal, what a verifier compares against the
// container's recorded final hash.
//
// The server keeps a queue and a set of active requests.  Each tick it
// admits queued requests while their device memory fits the budget
// (restore into a fresh world, journal parsed and validated whole), then
// advances every active request by one frame: the frame's body commands
// and its step run for all active worlds in one batched launch sequence
// (worlds grouped by step arguments), the commands applied by a device
// kernel.  Requests whose journal is done are hashed on the device and
// retired.  A request's result does not depend on what else is in the
// batch: worlds never interact.
#include "m3_world.h"
#include "m3_ops.h"

#include <string.h>

#include <algorithm>
#include <atomic>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <utility>
#include <vector>

namespace
{
constexpr uint32_t kReplayMagic = 0x314A334Du; // "M3J1" little-endian
constexpr uint32_t kReplayVersion = 1u;
constexpr int32_t kReplayHeaderBytes = 32;

int32_t ReadI32(const uint8_t* p)
{
    int32_t x;
    memcpy(&x, p, 4);
    return x;
}
} // namespace

// replay.c:15-49 (replay.h:34): record and step counts of a journal;
// false on malformed framing.
extern "C" bool m3JournalDescribe(const void* journal, int32_t bytes, m3JournalInfo* out)
{
    if (journal == nullptr || bytes < 0 || out == nullptr)
    {
        return false;
    }
    const uint8_t* p = (const uint8_t*)journal;
    int32_t cursor = 0;
    int32_t ops = 0;
    int32_t steps = 0;
    while (cursor < bytes)
    {
        if (bytes - cursor < 8)
        {
            return false;
        }
        const int32_t op = ReadI32(p + cursor);
        const int32_t payload = ReadI32(p + cursor + 4);
        if (op <= 0 || payload < 0 || payload > bytes - cursor - 8)
        {
            return false;
        }
        ops += 1;
        steps += op == M3_OP_STEP ? 1 : 0;
        cursor += 8 + payload;
    }
    out->opCount = ops;
    out->stepCount = steps;
    return true;
}

// replay.c:51-58 (replay.h:43).
extern "C" int32_t m3ReplayEncodeSize(int32_t snapshotBytes, int32_t journalBytes)
{
    if (snapshotBytes <= 0 || journalBytes < 0)
    {
        return 0;
    }
    return kReplayHeaderBytes + snapshotBytes + journalBytes;
}

// replay.c:60-92 (replay.h:50): 0 on refusal.
extern "C" int32_t m3ReplayEncode(const void* snapshot, int32_t snapshotBytes, const void* journal,
                                  int32_t journalBytes, uint64_t finalHash, void* out,
                                  int32_t capacity)
{
    const int32_t need = m3ReplayEncodeSize(snapshotBytes, journalBytes);
    m3JournalInfo info;
    if (need == 0 || snapshot == nullptr || (journal == nullptr && journalBytes > 0) ||
        out == nullptr || capacity < need ||
        !m3JournalDescribe(journalBytes > 0 ? journal : "", journalBytes, &info))
    {
        return 0;
    }
    uint8_t* p = (uint8_t*)out;
    const uint32_t magic = kReplayMagic;
    const uint32_t version = kReplayVersion;
    memcpy(p, &magic, 4);
    memcpy(p + 4, &version, 4);
    memcpy(p + 8, &snapshotBytes, 4);
    memcpy(p + 12, &journalBytes, 4);
    memcpy(p + 16, &info.stepCount, 4);
    memcpy(p + 20, &info.opCount, 4);
    memcpy(p + 24, &finalHash, 8);
    memcpy(p + kReplayHeaderBytes, snapshot, (size_t)snapshotBytes);
    if (journalBytes > 0)
    {
        memcpy(p + kReplayHeaderBytes + snapshotBytes, journal, (size_t)journalBytes);
    }
    return need;
}

// replay.c:94-136 (replay.h:62): validates the framing; the view aliases
// the input.
extern "C" bool m3ReplayDecode(const void* data, int32_t bytes, m3ReplayView* out)
{
    if (data == nullptr || bytes < kReplayHeaderBytes || out == nullptr)
    {
        return false;
    }
    const uint8_t* p = (const uint8_t*)data;
    uint32_t magic;
    uint32_t version;
    memcpy(&magic, p, 4);
    memcpy(&version, p + 4, 4);
    const int32_t snapshotBytes = ReadI32(p + 8);
    const int32_t journalBytes = ReadI32(p + 12);
    const int32_t stepCount = ReadI32(p + 16);
    const int32_t opCount = ReadI32(p + 20);
    uint64_t finalHash;
    memcpy(&finalHash, p + 24, 8);
    if (magic != kReplayMagic || version != kReplayVersion || snapshotBytes <= 0 ||
        journalBytes < 0 ||
        (int64_t)kReplayHeaderBytes + snapshotBytes + journalBytes != (int64_t)bytes)
    {
        return false;
    }
    m3JournalInfo info;
    const uint8_t* journal = p + kReplayHeaderBytes + snapshotBytes;
    if (!m3JournalDescribe(journal, journalBytes, &info) || info.stepCount != stepCount ||
        info.opCount != opCount)
    {
        return false;
    }
    out->snapshot = p + kReplayHeaderBytes;
    out->snapshotBytes = snapshotBytes;
    out->journal = journal;
    out->journalBytes = journalBytes;
    out->finalHash = finalHash;
    out->info = info;
    return true;
}

namespace
{
struct Request
{
    int64_t ticket = 0;
    std::vector<uint8_t> snapshot;
    std::vector<uint8_t> journal;
    m3WorldId world{0, 0};
    m3HostWorld* host = nullptr;
    std::vector<m3JournalRecordView> records;
    size_t next = 0;
    int64_t deviceBytes = 0;
};

struct Completion
{
    int64_t ticket;
    uint64_t hash;
    int32_t status;
};

// Capacities the snapshot header names (snapshot.c:88-127): body, shape,
// mesh, joint, voxel and character pools.
struct SnapshotShape
{
    int32_t body, shape, mesh, joint, voxel, character, hulls;
};

bool ReadShape(const std::vector<uint8_t>& snap, SnapshotShape* out)
{
    if (snap.size() < 192)
    {
        return false;
    }
    const uint8_t* p = snap.data();
    out->body = ReadI32(p + 24);
    out->shape = ReadI32(p + 44);
    out->hulls = ReadI32(p + 76);
    out->mesh = ReadI32(p + 92);
    out->joint = ReadI32(p + 112);
    out->voxel = ReadI32(p + 132);
    out->character = ReadI32(p + 152);
    return out->body > 0 && out->shape > 0 && out->mesh > 0 && out->joint > 0 &&
           out->voxel > 0 && out->character > 0 && out->hulls >= 0;
}

// Device bytes of a world of that shape: the slab (persistent image and
// step scratch) and the interned hull pool.
int64_t DeviceBytes(const SnapshotShape& s)
{
    const int32_t pairCap = 8 * s.shape;
    return m3LayoutPersistent(nullptr, nullptr, s.body, s.shape, s.joint, pairCap) +
           m3gpuScratchBytes(s.body, s.shape, s.joint, pairCap) +
           (int64_t)(s.hulls < 4 ? 4 : s.hulls) * (int64_t)sizeof(m3HullData);
}
} // namespace

struct m3gpuServer
{
    int64_t budget = 0;
    int32_t maxActive = 0;
    int64_t nextTicket = 1;
    int64_t activeBytes = 0;
    std::deque<std::unique_ptr<Request>> queue;
    std::vector<std::unique_ptr<Request>> active;
    std::deque<Completion> done;
};

namespace
{
void Retire(m3gpuServer* s, std::unique_ptr<Request>& r, uint64_t hash, int32_t status)
{
    s->done.push_back(Completion{r->ticket, hash, status});
    if (r->host != nullptr)
    {
        m3DestroyWorld(r->world);
        r->host = nullptr;
    }
}

// Admits queued requests while they fit; refused ones retire at once
// with their error code.  Worlds are created in order (the world table
// is shared), restored and their journals parsed on host threads (each
// touches only its own world), then reserved on the device in order.
void Admit(m3gpuServer* s)
{
    std::vector<std::unique_ptr<Request>> batch;
    int64_t bytes = s->activeBytes;
    while (!s->queue.empty() && (int32_t)(s->active.size() + batch.size()) < s->maxActive)
    {
        std::unique_ptr<Request>& front = s->queue.front();
        SnapshotShape shape;
        if (!ReadShape(front->snapshot, &shape))
        {
            Retire(s, front, 0, M3GPU_ERR_INVALID);
            s->queue.pop_front();
            continue;
        }
        if (front->deviceBytes == 0)
        {
            front->deviceBytes = DeviceBytes(shape);
        }
        if (!(s->active.empty() && batch.empty()) && bytes + front->deviceBytes > s->budget)
        {
            break; // the memory budget is full: wait for retirements
        }
        std::unique_ptr<Request> r = std::move(front);
        s->queue.pop_front();
        m3WorldDef def = m3DefaultWorldDef();
        def.bodyCapacity = shape.body;
        def.shapeCapacity = shape.shape;
        def.meshCapacity = shape.mesh;
        def.jointCapacity = shape.joint;
        def.voxelCapacity = shape.voxel;
        def.characterCapacity = shape.character;
        r->world = m3CreateWorld(&def);
        r->host = m3gpuWorldFromId(r->world);
        if (r->host == nullptr)
        {
            const int32_t code = m3gpu_last_error();
            Retire(s, r, 0, code != M3GPU_OK ? code : M3GPU_ERR_INVALID);
            continue;
        }
        bytes += r->deviceBytes;
        batch.push_back(std::move(r));
    }
    if (batch.empty())
    {
        return;
    }
    std::vector<int32_t> codes(batch.size(), M3GPU_OK);
    std::atomic<size_t> nextJob{0};
    auto work = [&]() {
        for (size_t i = nextJob.fetch_add(1); i < batch.size(); i = nextJob.fetch_add(1))
        {
            Request& r = *batch[i];
            if (!m3World_Restore(r.world, r.snapshot.data(), (int32_t)r.snapshot.size()) ||
                !m3ParseJournal(r.host, r.journal.data(), (int32_t)r.journal.size(), &r.records))
            {
                const int32_t code = m3gpu_last_error();
                codes[i] = code != M3GPU_OK ? code : M3GPU_ERR_INVALID;
            }
        }
    };
    const size_t threads =
        std::min<size_t>(batch.size(), std::max(1u, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (size_t t = 1; t < threads; ++t)
    {
        pool.emplace_back(work);
    }
    work();
    for (std::thread& t : pool)
    {
        t.join();
    }
    for (size_t i = 0; i < batch.size(); ++i)
    {
        std::unique_ptr<Request>& r = batch[i];
        if (codes[i] == M3GPU_OK && m3gpuReserve(r->host) != M3GPU_OK)
        {
            codes[i] = m3gpu_last_error();
        }
        if (codes[i] != M3GPU_OK)
        {
            Retire(s, r, 0, codes[i]);
            continue;
        }
        // Nobody can snapshot a served world: it keeps no broadphase tree.
        r->host->hv.sc->treeTracked = 0;
        // The inputs live on in the world; the request keeps only its
        // parsed records.
        std::vector<uint8_t>().swap(r->snapshot);
        std::vector<uint8_t>().swap(r->journal);
        s->activeBytes += r->deviceBytes;
        s->active.push_back(std::move(r));
    }
}
} // namespace

extern "C" m3gpuServer* m3gpu_serve_create(int64_t deviceBudgetBytes, int32_t maxActive)
{
    m3gpuClearError();
    if (deviceBudgetBytes <= 0 || maxActive <= 0)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3gpu_serve_create: budget and active limit must be > 0");
        return nullptr;
    }
    m3gpuServer* s = new m3gpuServer();
    s->budget = deviceBudgetBytes;
    s->maxActive = maxActive;
    return s;
}

extern "C" void m3gpu_serve_destroy(m3gpuServer* s)
{
    if (s == nullptr)
    {
        return;
    }
    for (std::unique_ptr<Request>& r : s->active)
    {
        if (r->host != nullptr)
        {
            m3DestroyWorld(r->world);
        }
    }
    delete s;
}

extern "C" int64_t m3gpu_serve_submit(m3gpuServer* s, const void* container, int32_t bytes)
{
    m3gpuClearError();
    m3ReplayView view;
    if (s == nullptr || !m3ReplayDecode(container, bytes, &view))
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "m3gpu_serve_submit: not a replay container");
        return -1;
    }
    std::unique_ptr<Request> r(new Request());
    r->ticket = s->nextTicket++;
    const uint8_t* snap = (const uint8_t*)view.snapshot;
    const uint8_t* jour = (const uint8_t*)view.journal;
    r->snapshot.assign(snap, snap + view.snapshotBytes);
    r->journal.assign(jour, jour + view.journalBytes);
    const int64_t ticket = r->ticket;
    s->queue.push_back(std::move(r));
    return ticket;
}

extern "C" int32_t m3gpu_serve_tick(m3gpuServer* s)
{
    m3gpuClearError();
    if (s == nullptr)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "m3gpu_serve_tick: null server");
    }
    Admit(s);

    // One frame of every active request: its commands up to and including
    // the next step, batched by step arguments.
    std::map<std::pair<float, int32_t>, std::vector<size_t>> groups;
    for (size_t i = 0; i < s->active.size(); ++i)
    {
        Request& r = *s->active[i];
        size_t k = r.next;
        while (k < r.records.size() && r.records[k].op != M3_OP_STEP)
        {
            ++k;
        }
        if (k < r.records.size())
        {
            groups[{r.records[k].dt, r.records[k].substeps}].push_back(i);
        }
        else if (r.next < r.records.size())
        {
            // Commands after the last step apply on the host.
            if (m3gpuSyncHost(r.host) == M3GPU_OK)
            {
                for (size_t j = r.next; j < r.records.size(); ++j)
                {
                    m3ApplyBodyOp(r.host->hv, r.records[j].op, r.records[j].body, r.records[j].v);
                }
                r.host->hostDirty = true;
            }
            r.next = r.records.size();
        }
    }
    std::vector<m3HostWorld*> worlds;
    std::vector<m3BodyOp> ops;
    for (auto& g : groups)
    {
        worlds.clear();
        ops.clear();
        for (size_t i : g.second)
        {
            Request& r = *s->active[i];
            const int32_t wi = (int32_t)worlds.size();
            worlds.push_back(r.host);
            while (r.records[r.next].op != M3_OP_STEP)
            {
                const m3JournalRecordView& rec = r.records[r.next];
                ops.push_back(m3BodyOp{wi, rec.op, rec.body, rec.v});
                ++r.next;
            }
            ++r.next; // the step
        }
        const int32_t rc = m3gpuStepBatch(worlds.data(), (int32_t)worlds.size(), g.first.first,
                                          g.first.second, 1, ops.data(), (int32_t)ops.size());
        if (rc != M3GPU_OK && rc != M3GPU_ERR_UNSUPPORTED && rc != M3GPU_ERR_CAPACITY)
        {
            return rc;
        }
    }

    // Retire finished requests: device hash of the finished worlds (a
    // world the device refused reports its refusal instead).
    std::vector<m3HostWorld*> finished;
    std::vector<size_t> finishedAt;
    for (size_t i = 0; i < s->active.size(); ++i)
    {
        if (s->active[i]->next >= s->active[i]->records.size())
        {
            finished.push_back(s->active[i]->host);
            finishedAt.push_back(i);
        }
    }
    if (!finished.empty())
    {
        std::vector<uint64_t> hashes(finished.size(), 0);
        const int32_t rc = m3gpuHashBatch(finished.data(), (int32_t)finished.size(), hashes.data());
        if (rc != M3GPU_OK)
        {
            return rc;
        }
        for (size_t f = 0; f < finished.size(); ++f)
        {
            std::unique_ptr<Request>& r = s->active[finishedAt[f]];
            const int32_t status = m3gpuWorldStatus(finished[f]);
            s->activeBytes -= r->deviceBytes;
            Retire(s, r, status == M3GPU_OK ? hashes[f] : 0, status);
        }
        std::vector<std::unique_ptr<Request>> keep;
        keep.reserve(s->active.size());
        for (std::unique_ptr<Request>& r : s->active)
        {
            if (r->host != nullptr)
            {
                keep.push_back(std::move(r));
            }
        }
        s->active.swap(keep);
    }
    return (int32_t)(s->active.size() + s->queue.size());
}

extern "C" int32_t m3gpu_serve_poll(m3gpuServer* s, int64_t* tickets, uint64_t* hashes,
                                    int32_t* status, int32_t capacity)
{
    if (s == nullptr || capacity < 0 || (capacity > 0 && (tickets == nullptr || hashes == nullptr ||
                                                          status == nullptr)))
    {
        return -1;
    }
    int32_t n = 0;
    while (n < capacity && !s->done.empty())
    {
        const Completion c = s->done.front();
        s->done.pop_front();
        tickets[n] = c.ticket;
        hashes[n] = c.hash;
        status[n] = c.status;
        ++n;
    }
    return n;
}

extern "C" int32_t m3gpu_serve_active(const m3gpuServer* s)
{
    return s == nullptr ? -1 : (int32_t)s->active.size();
}
