// Serving: many short rollback/verification sessions at once.  A request
// is the reference's replay container (M3J1: a snapshot and the journal
// recorded after it, replay.c:15-136); its answer is the world hash at
// the end of the journal, what a verifier compares against the
// container's recorded final hash.
//
// Clients submit from any thread (the container is copied on theirs);
// one thread ticks.  A request moves through three sets.  Queued:
// submitted, waiting for room.  Preparing: its device memory counted against the budget, a
// worker thread builds its world off the world table, restores the
// snapshot into it and parses and validates the journal whole.
// Active: entered into the world table and reserved on the device.  Each
// tick starts preparing queued requests while they fit the budget and
// the active limit, admits the prepared ones in submission order, and
// advances every active request by one frame: the frame's body commands
// and its step run for all active worlds in one batched launch sequence
// (worlds grouped by step arguments), the commands applied by a device
// kernel.  The workers keep preparing while the frame runs on the GPU.
// Requests whose journal is done are hashed on the device and retired.
// A request's result does not depend on what else is in the batch:
// worlds never interact.
#include "m3_world.h"
#include "m3_ops.h"

#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
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
    m3HostWorld* host = nullptr;  // in the world table: active
    m3HostWorld* built = nullptr; // prepared off the table, not yet admitted
    std::vector<m3JournalRecordView> records;
    size_t next = 0;
    int64_t deviceBytes = 0;
    int32_t code = M3GPU_OK; // the preparation's refusal
    bool ready = false;      // prepared (under the server's mutex)
    bool suspect = false;    // a step of its batch reported a refusal
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
    const int64_t slab = m3LayoutPersistent(nullptr, nullptr, s.body, s.shape, s.joint, pairCap) +
                         m3gpuScratchBytes(s.body, s.shape, s.joint, pairCap);
    const int64_t hulls = (int64_t)(s.hulls < 4 ? 4 : s.hulls) * (int64_t)sizeof(m3HullData);
    // What the device allocator hands out: its size classes.
    return (int64_t)m3SizeClass((size_t)slab, M3_SLAB_ALIGN) +
           (int64_t)m3SizeClass((size_t)hulls, M3_SLAB_ALIGN);
}

double MsSince(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}
} // namespace

struct m3gpuServer
{
    int64_t budget = 0;
    int32_t maxActive = 0;
    // Submissions, from any thread: tickets and the inbox under inboxMu;
    // each tick moves the inbox to the queue.
    std::mutex inboxMu;
    int64_t nextTicket = 1;
    std::deque<std::unique_ptr<Request>> inbox;
    int64_t heldBytes = 0; // device bytes of preparing and active requests
    std::deque<std::unique_ptr<Request>> queue;
    std::deque<std::unique_ptr<Request>> preparing; // submission order
    std::vector<std::unique_ptr<Request>> active;
    std::deque<Completion> done;
    m3gpuServeStats stats{};

    // Preparation workers: `jobs` holds requests of `preparing` not yet
    // taken; a worker marks its request ready under `mu`.
    std::mutex mu;
    std::condition_variable jobReady;
    std::condition_variable prepared;
    std::deque<Request*> jobs;
    std::vector<std::thread> workers;
    bool stopping = false;
    std::atomic<int64_t> prepareUs{0};
};

namespace
{
void Retire(m3gpuServer* s, std::unique_ptr<Request>& r, uint64_t hash, int32_t status)
{
    s->done.push_back(Completion{r->ticket, hash, status});
    if (status == M3GPU_OK)
    {
        s->stats.completed += 1;
    }
    else
    {
        s->stats.refused += 1;
    }
    if (r->host != nullptr)
    {
        m3DestroyWorld(r->world);
        r->host = nullptr;
    }
    if (r->built != nullptr)
    {
        m3gpuDeleteWorld(r->built);
        r->built = nullptr;
    }
}

// Served journals carry body and joint commands and steps: the frames run
// as device ops in a batched step.  A record that only the host applies
// (a world setting, a force at a point, motion locks) is refused.
bool NoSettings(const std::vector<m3JournalRecordView>& records)
{
    for (const m3JournalRecordView& rec : records)
    {
        if (m3IsWorldSettingOp(rec.op) || m3IsHostBodyOp(rec.op) || m3IsHostShapeOp(rec.op) ||
            m3IsHostJointOp(rec.op))
        {
            m3gpuSetError(M3GPU_ERR_UNSUPPORTED, "served journal: host-side op %d", rec.op);
            return false;
        }
    }
    return true;
}

// A worker's preparation of one request: its world built off the world
// table with the snapshot's capacities, the snapshot restored into it and
// the journal parsed and validated whole.  Touches only the request.
void Prepare(Request& r)
{
    SnapshotShape shape;
    ReadShape(r.snapshot, &shape); // checked when the request started
    m3WorldDef def = m3DefaultWorldDef();
    def.bodyCapacity = shape.body;
    def.shapeCapacity = shape.shape;
    def.meshCapacity = shape.mesh;
    def.jointCapacity = shape.joint;
    def.voxelCapacity = shape.voxel;
    def.characterCapacity = shape.character;
    m3HostWorld* w = m3gpuNewWorld(&def);
    int32_t code = M3GPU_OK;
    if (w == nullptr ||
        !m3gpuRestoreWorld(w, r.snapshot.data(), (int32_t)r.snapshot.size()) ||
        !m3ParseJournal(w, r.journal.data(), (int32_t)r.journal.size(), &r.records) ||
        !NoSettings(r.records))
    {
        code = m3gpu_last_error();
        code = code != M3GPU_OK ? code : M3GPU_ERR_INVALID;
        if (w != nullptr)
        {
            m3gpuDeleteWorld(w);
            w = nullptr;
        }
    }
    if (w != nullptr)
    {
        // Nobody can snapshot a served world: it keeps no broadphase tree,
        // and its pair arrays past the live pairs (which only a snapshot
        // reads; the step and the hash read the live pairs) stay on the
        // host: the upload carries the live pairs alone, in the batched
        // upload with the other admitted worlds.
        w->hv.sc->treeTracked = 0;
        w->pairTailsToDevice = false;
    }
    // The inputs live on in the world; the request keeps only its parsed
    // records.
    std::vector<uint8_t>().swap(r.snapshot);
    std::vector<uint8_t>().swap(r.journal);
    r.built = w;
    r.code = code;
}

void WorkerLoop(m3gpuServer* s)
{
    for (;;)
    {
        Request* r = nullptr;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            s->jobReady.wait(lock, [s] { return s->stopping || !s->jobs.empty(); });
            if (s->stopping && s->jobs.empty())
            {
                return;
            }
            r = s->jobs.front();
            s->jobs.pop_front();
        }
        const auto t0 = std::chrono::steady_clock::now();
        Prepare(*r);
        s->prepareUs += (int64_t)(MsSince(t0) * 1000.0);
        {
            std::lock_guard<std::mutex> lock(s->mu);
            r->ready = true;
        }
        s->prepared.notify_all();
    }
}

// Starts preparing queued requests while they fit: at most `maxActive`
// preparing and active, their device bytes within the budget (a request
// alone is always let in, so that one larger than the budget still
// runs).  A container whose snapshot header is unreadable retires at once.
void Start(m3gpuServer* s)
{
    int32_t started = 0;
    while (!s->queue.empty() &&
           (int32_t)(s->active.size() + s->preparing.size()) < s->maxActive)
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
        const bool alone = s->active.empty() && s->preparing.empty();
        if (!alone && s->heldBytes + front->deviceBytes > s->budget)
        {
            break; // the memory budget is full: wait for retirements
        }
        s->heldBytes += front->deviceBytes;
        s->stats.peakHeldBytes = std::max(s->stats.peakHeldBytes, s->heldBytes);
        Request* job = front.get();
        s->preparing.push_back(std::move(front));
        s->queue.pop_front();
        {
            std::lock_guard<std::mutex> lock(s->mu);
            s->jobs.push_back(job);
        }
        started += 1;
    }
    if (started > 0)
    {
        s->jobReady.notify_all();
    }
}

// Admits every prepared request (in submission order among them; one
// still being prepared holds up nobody behind it, and with nothing active
// the oldest is waited for): each enters the world table and is reserved
// on the device.  Results do not depend on the order of admission.
void Admit(m3gpuServer* s)
{
    std::vector<std::unique_ptr<Request>> ready;
    {
        std::unique_lock<std::mutex> lock(s->mu);
        if (s->active.empty() && !s->preparing.empty() && !s->preparing.front()->ready)
        {
            const auto t0 = std::chrono::steady_clock::now();
            Request* front = s->preparing.front().get();
            s->prepared.wait(lock, [front] { return front->ready; });
            s->stats.waitMs += MsSince(t0);
        }
        std::deque<std::unique_ptr<Request>> waiting;
        for (std::unique_ptr<Request>& r : s->preparing)
        {
            if (r->ready)
            {
                ready.push_back(std::move(r));
            }
            else
            {
                waiting.push_back(std::move(r));
            }
        }
        s->preparing.swap(waiting);
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (std::unique_ptr<Request>& r : ready)
    {
        int32_t code = r->code;
        if (code == M3GPU_OK)
        {
            m3HostWorld* w = r->built;
            r->built = nullptr;
            r->world = m3gpuAttachWorld(w); // deletes the world when the table is full
            r->host = m3gpuWorldFromId(r->world);
            if (r->host == nullptr)
            {
                code = m3gpu_last_error();
                code = code != M3GPU_OK ? code : M3GPU_ERR_CAPACITY;
            }
            else if (m3gpuReserve(r->host) != M3GPU_OK)
            {
                code = m3gpu_last_error();
            }
        }
        if (code != M3GPU_OK)
        {
            s->heldBytes -= r->deviceBytes;
            Retire(s, r, 0, code);
        }
        else
        {
            s->active.push_back(std::move(r));
        }
    }
    s->stats.admitMs += MsSince(t0);
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
    // Preparation workers: the host's threads but the ticking one.
    const unsigned hw = std::max(2u, std::thread::hardware_concurrency());
    const unsigned workers = std::min(32u, hw - 1);
    for (unsigned t = 0; t < workers; ++t)
    {
        s->workers.emplace_back(WorkerLoop, s);
    }
    return s;
}

extern "C" void m3gpu_serve_destroy(m3gpuServer* s)
{
    if (s == nullptr)
    {
        return;
    }
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stopping = true;
        s->jobs.clear(); // requests not yet taken are dropped
    }
    s->jobReady.notify_all();
    for (std::thread& t : s->workers)
    {
        t.join();
    }
    for (std::unique_ptr<Request>& r : s->preparing)
    {
        if (r->built != nullptr)
        {
            m3gpuDeleteWorld(r->built);
        }
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
    // The copy happens on the caller's thread, outside the server's locks.
    std::unique_ptr<Request> r(new Request());
    const uint8_t* snap = (const uint8_t*)view.snapshot;
    const uint8_t* jour = (const uint8_t*)view.journal;
    r->snapshot.assign(snap, snap + view.snapshotBytes);
    r->journal.assign(jour, jour + view.journalBytes);
    std::lock_guard<std::mutex> lock(s->inboxMu);
    r->ticket = s->nextTicket++;
    const int64_t ticket = r->ticket;
    s->inbox.push_back(std::move(r));
    return ticket;
}

extern "C" int32_t m3gpu_serve_tick(m3gpuServer* s)
{
    m3gpuClearError();
    if (s == nullptr)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "m3gpu_serve_tick: null server");
    }
    s->stats.ticks += 1;
    {
        // Requests submitted since the last tick, from any thread.
        std::lock_guard<std::mutex> lock(s->inboxMu);
        s->stats.submitted += (int64_t)s->inbox.size();
        for (std::unique_ptr<Request>& r : s->inbox)
        {
            s->queue.push_back(std::move(r));
        }
        s->inbox.clear();
    }
    Start(s);
    Admit(s);
    Start(s); // room freed by refusals
    s->stats.peakActive = std::max(s->stats.peakActive, (int32_t)s->active.size());
    const auto tStep = std::chrono::steady_clock::now();

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
        if (rc != M3GPU_OK)
        {
            // Some world of the batch refused: its requests read their
            // own status when they retire (the others are known good).
            for (size_t i : g.second)
            {
                s->active[i]->suspect = true;
            }
        }
    }

    s->stats.stepMs += MsSince(tStep);
    const auto tRetire = std::chrono::steady_clock::now();

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
            const int32_t status = r->suspect ? m3gpuWorldStatus(finished[f]) : M3GPU_OK;
            s->heldBytes -= r->deviceBytes;
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
    s->stats.retireMs += MsSince(tRetire);
    std::lock_guard<std::mutex> lock(s->inboxMu);
    return (int32_t)(s->active.size() + s->preparing.size() + s->queue.size() + s->inbox.size());
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

extern "C" int32_t m3gpu_serve_stats(m3gpuServer* s, m3gpuServeStats* out)
{
    if (s == nullptr || out == nullptr)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "m3gpu_serve_stats: null argument");
    }
    *out = s->stats;
    out->heldBytes = s->heldBytes;
    out->budget = s->budget;
    {
        std::lock_guard<std::mutex> lock(s->inboxMu);
        out->queued = (int32_t)(s->queue.size() + s->inbox.size());
    }
    out->preparing = (int32_t)s->preparing.size();
    out->active = (int32_t)s->active.size();
    out->workers = (int32_t)s->workers.size();
    out->prepareMs = (double)s->prepareUs.load() / 1000.0;
    return M3GPU_OK;
}
