// Event streams of a world's last step (world.h:207-313): contact and
// sensor begin/end events, joint-break, body move and hit events.
//
// The device step keeps the previous step's pair list and manifolds in
// the second pair buffer (the two buffers swap every step), records the
// previous pair count, and appends every joint it breaks to a ring with
// the ring's position at the start of the step.  So the last step's
// events need no work inside the step: the first read after a step
// copies the two key lists, the manifolds' point counts and the step's
// ring entries back and walks them as the reference's step does
// (solver.c:3747-3815 for contacts, solver.c:4233-4257 for breaks); the
// move events read the step's mover list (still in the world's scratch)
// and the bodies' transforms; the hit events, which need each contact's
// impulses and its body's transform before the continuous phase moves
// it, are the one stream the step writes itself (a flag and a record per
// contact constraint, in the world's scratch).
// Shape liveness and generations come from the host image, which this
// path never changes behind the host's back (the device destroys joints
// only, never shapes).
#include "m3_world.h"

#include <cuda_runtime.h>

#include <stddef.h>
#include <string.h>

#include <type_traits>
#include <vector>

namespace
{

int32_t Cuda(cudaError_t e, const char* what)
{
    if (e != cudaSuccess)
    {
        return m3gpuSetError(M3GPU_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    }
    return M3GPU_OK;
}

// Keys [0, n) of a device pair buffer and each manifold's point count.
int32_t ReadPairs(const uint64_t* dkeys, const m3Manifold* dman, int32_t n,
                  std::vector<uint64_t>& keys, std::vector<int32_t>& points)
{
    keys.resize((size_t)n);
    points.resize((size_t)n);
    if (n == 0)
    {
        return M3GPU_OK;
    }
    int32_t rc = Cuda(cudaMemcpy(keys.data(), dkeys, sizeof(uint64_t) * (size_t)n,
                                 cudaMemcpyDeviceToHost),
                      "event pair keys");
    if (rc == M3GPU_OK)
    {
        rc = Cuda(cudaMemcpy2D(points.data(), sizeof(int32_t),
                               (const char*)dman + offsetof(m3Manifold, pointCount),
                               sizeof(m3Manifold), sizeof(int32_t), (size_t)n,
                               cudaMemcpyDeviceToHost),
                  "event point counts");
    }
    return rc;
}

void ClearEvents(m3HostWorld* w)
{
    w->beginEvents.clear();
    w->endEvents.clear();
    w->sensorBeginEvents.clear();
    w->sensorEndEvents.clear();
    w->jointBreakEvents.clear();
}

// The streams of the last step, built once per step.
int32_t EnsureEvents(m3HostWorld* w)
{
    if (w->eventsEpoch == w->stepEpoch)
    {
        return M3GPU_OK;
    }
    ClearEvents(w);
    if (!w->lastEpochIsStep || w->dslab == nullptr)
    {
        w->eventsEpoch = w->stepEpoch;
        return M3GPU_OK;
    }
    m3WorldScalars sc;
    int32_t rc = Cuda(cudaMemcpy(&sc, w->dv.sc, sizeof(sc), cudaMemcpyDeviceToHost),
                      "event scalars");
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    if (sc.status != 0)
    {
        // A refused step has no events (the world is marked failed).
        w->eventsEpoch = w->stepEpoch;
        return M3GPU_OK;
    }
    const bool curIs0 = sc.pairBuf == 0;
    auto clampCount = [&](int32_t n) { return n < 0 ? 0 : (n < sc.pairCap ? n : sc.pairCap); };
    const int32_t newCount = clampCount(sc.pairCount);
    const int32_t oldCount = clampCount(sc.prevPairCount);
    std::vector<uint64_t> newKeys;
    std::vector<uint64_t> oldKeys;
    std::vector<int32_t> newPoints;
    std::vector<int32_t> oldPoints;
    rc = ReadPairs(curIs0 ? w->dv.keys0 : w->dv.keys1, curIs0 ? w->dv.man0 : w->dv.man1, newCount,
                   newKeys, newPoints);
    if (rc == M3GPU_OK)
    {
        rc = ReadPairs(curIs0 ? w->dv.keys1 : w->dv.keys0, curIs0 ? w->dv.man1 : w->dv.man0,
                       oldCount, oldKeys, oldPoints);
    }
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    // The merge walk over both sorted key lists (solver.c:3747-3815).
    const m3WorldView& v = w->hv;
    const size_t cap = (size_t)sc.pairCap;
    const uint16_t world0 = (uint16_t)w->slot;
    int32_t iNew = 0;
    int32_t iOld = 0;
    while (iNew < newCount || iOld < oldCount)
    {
        const uint64_t keyNew = iNew < newCount ? newKeys[(size_t)iNew] : UINT64_MAX;
        const uint64_t keyOld = iOld < oldCount ? oldKeys[(size_t)iOld] : UINT64_MAX;
        bool touchNew = false;
        bool touchOld = false;
        uint64_t key;
        if (keyNew < keyOld)
        {
            key = keyNew;
            touchNew = newPoints[(size_t)iNew] > 0;
            iNew += 1;
        }
        else if (keyOld < keyNew)
        {
            key = keyOld;
            touchOld = oldPoints[(size_t)iOld] > 0;
            iOld += 1;
        }
        else
        {
            key = keyNew;
            touchNew = newPoints[(size_t)iNew] > 0;
            touchOld = oldPoints[(size_t)iOld] > 0;
            iNew += 1;
            iOld += 1;
        }
        if (touchNew == touchOld)
        {
            continue;
        }
        const int32_t sA = (int32_t)(key >> 32);
        const int32_t sB = (int32_t)(key & 0xFFFFFFFFu);
        if (sA < 0 || sB < 0 || sA >= w->shapeCap || sB >= w->shapeCap || v.shapeAlive[sA] == 0 ||
            v.shapeAlive[sB] == 0)
        {
            continue;
        }
        m3ContactEvent event;
        event.shapeA = m3ShapeId{sA + 1, world0, v.shapeGen[sA]};
        event.shapeB = m3ShapeId{sB + 1, world0, v.shapeGen[sB]};
        const bool sensorPair = v.sensor[sA] != 0 || v.sensor[sB] != 0;
        std::vector<m3ContactEvent>& out =
            sensorPair ? (touchNew ? w->sensorBeginEvents : w->sensorEndEvents)
                       : (touchNew ? w->beginEvents : w->endEvents);
        if (out.size() < cap)
        {
            out.push_back(event);
        }
    }
    // Joint breaks: the step's entries of the ring, in destruction order;
    // each joint's generation before its destruction (a retired slot
    // keeps 0xFFFF).
    const int32_t jointCap = sc.jointCap > 0 ? sc.jointCap : 1;
    const int32_t breaks = sc.brokenCount - sc.stepBrokenStart;
    if (breaks > 0 && breaks <= jointCap)
    {
        std::vector<int32_t> ring((size_t)jointCap);
        std::vector<uint16_t> gens((size_t)jointCap);
        rc = Cuda(cudaMemcpy(ring.data(), w->dv.jbroken, sizeof(int32_t) * (size_t)jointCap,
                             cudaMemcpyDeviceToHost),
                  "event joint ring");
        if (rc == M3GPU_OK)
        {
            rc = Cuda(cudaMemcpy(gens.data(), w->dv.jointGen, sizeof(uint16_t) * (size_t)jointCap,
                                 cudaMemcpyDeviceToHost),
                      "event joint generations");
        }
        if (rc != M3GPU_OK)
        {
            return rc;
        }
        for (int32_t k = 0; k < breaks; ++k)
        {
            const int32_t e = ring[(size_t)((sc.stepBrokenStart + k) % jointCap)];
            const int32_t j = e >= 0 ? e : -1 - e;
            if (j < 0 || j >= jointCap)
            {
                continue;
            }
            const uint16_t gen = e >= 0 ? (uint16_t)(gens[(size_t)j] - 1) : (uint16_t)0xFFFF;
            w->jointBreakEvents.push_back(m3JointBreakEvent{m3JointId{j + 1, world0, gen}});
        }
    }
    w->eventsEpoch = w->stepEpoch;
    return M3GPU_OK;
}

// Body move events of the last step (solver.c:4295-4306): the step's
// movers in ascending order, each with its transform after the step and
// whether its island fell asleep on this step.
int32_t EnsureMoveEvents(m3HostWorld* w)
{
    if (w->moveEventsEpoch == w->stepEpoch)
    {
        return M3GPU_OK;
    }
    w->moveEvents.clear();
    if (!w->lastEpochIsStep || w->dslab == nullptr)
    {
        w->moveEventsEpoch = w->stepEpoch;
        return M3GPU_OK;
    }
    m3WorldScalars sc;
    int32_t rc = Cuda(cudaMemcpy(&sc, w->dv.sc, sizeof(sc), cudaMemcpyDeviceToHost),
                      "event scalars");
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    const int32_t bodies = sc.bodyMax;
    const int32_t movers = sc.moverCount;
    if (sc.status != 0 || movers <= 0 || movers > bodies)
    {
        w->moveEventsEpoch = w->stepEpoch;
        return M3GPU_OK;
    }
    std::vector<int32_t> list((size_t)movers);
    std::vector<m3Transform> xf((size_t)bodies);
    std::vector<uint8_t> type((size_t)bodies);
    std::vector<uint8_t> awake((size_t)bodies);
    rc = Cuda(cudaMemcpy(list.data(), m3gpuDeviceMovers(w), sizeof(int32_t) * (size_t)movers,
                         cudaMemcpyDeviceToHost),
              "event movers");
    if (rc == M3GPU_OK)
    {
        rc = Cuda(cudaMemcpy(xf.data(), w->dv.xf, sizeof(m3Transform) * (size_t)bodies,
                             cudaMemcpyDeviceToHost),
                  "event transforms");
    }
    if (rc == M3GPU_OK)
    {
        rc = Cuda(cudaMemcpy(type.data(), w->dv.btype, (size_t)bodies, cudaMemcpyDeviceToHost),
                  "event body types");
    }
    if (rc == M3GPU_OK)
    {
        rc = Cuda(cudaMemcpy(awake.data(), w->dv.awake, (size_t)bodies, cudaMemcpyDeviceToHost),
                  "event awake flags");
    }
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    const uint16_t world0 = (uint16_t)w->slot;
    w->moveEvents.reserve((size_t)movers);
    for (int32_t m = 0; m < movers; ++m)
    {
        const int32_t i = list[(size_t)m];
        if (i < 0 || i >= bodies)
        {
            continue;
        }
        m3BodyMoveEvent e;
        memset(&e, 0, sizeof(e));
        e.body = m3BodyId{i + 1, world0, w->hv.bodyGen[i]};
        e.transform = xf[(size_t)i];
        e.fellAsleep = type[(size_t)i] == M3_BODY_DYNAMIC && awake[(size_t)i] == 0;
        w->moveEvents.push_back(e);
    }
    w->moveEventsEpoch = w->stepEpoch;
    return M3GPU_OK;
}

// Hit events of the last step (solver.c:2987-3033): the step left one
// flag and, where set, one event per contact constraint in constraint
// order; the first pair-capacity events are kept, the rest counted.
int32_t EnsureHitEvents(m3HostWorld* w)
{
    if (w->hitEventsEpoch == w->stepEpoch)
    {
        return M3GPU_OK;
    }
    w->hitEvents.clear();
    w->hitEventsDropped = 0;
    if (!w->lastEpochIsStep || w->dslab == nullptr)
    {
        w->hitEventsEpoch = w->stepEpoch;
        return M3GPU_OK;
    }
    m3WorldScalars sc;
    int32_t rc = Cuda(cudaMemcpy(&sc, w->dv.sc, sizeof(sc), cudaMemcpyDeviceToHost),
                      "event scalars");
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    const int32_t n = sc.constraintCount;
    if (sc.status != 0 || n <= 0 || n > sc.pairCap)
    {
        w->hitEventsEpoch = w->stepEpoch;
        return M3GPU_OK;
    }
    const uint8_t* dflags = nullptr;
    const m3HitEvent* dhits = nullptr;
    m3gpuDeviceHits(w, &dflags, &dhits);
    std::vector<uint8_t> flags((size_t)n);
    rc = Cuda(cudaMemcpy(flags.data(), dflags, (size_t)n, cudaMemcpyDeviceToHost), "hit flags");
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    int32_t last = -1;
    for (int32_t i = 0; i < n; ++i)
    {
        last = flags[(size_t)i] != 0 ? i : last;
    }
    std::vector<m3HitEvent> records((size_t)(last + 1));
    if (last >= 0)
    {
        rc = Cuda(cudaMemcpy(records.data(), dhits, sizeof(m3HitEvent) * (size_t)(last + 1),
                             cudaMemcpyDeviceToHost),
                  "hit events");
        if (rc != M3GPU_OK)
        {
            return rc;
        }
    }
    const uint16_t world0 = (uint16_t)w->slot;
    const size_t cap = (size_t)sc.pairCap;
    for (int32_t i = 0; i <= last; ++i)
    {
        if (flags[(size_t)i] == 0)
        {
            continue;
        }
        if (w->hitEvents.size() >= cap)
        {
            w->hitEventsDropped += 1;
            continue;
        }
        m3HitEvent e = records[(size_t)i];
        e.shapeA.world0 = world0;
        e.shapeB.world0 = world0;
        w->hitEvents.push_back(e);
    }
    w->hitEventsEpoch = w->stepEpoch;
    return M3GPU_OK;
}

template <class T>
const T* Stream(m3WorldId worldId, int32_t* count, std::vector<T> m3HostWorld::*member)
{
    M3_DEVICE_GUARD;
    m3gpuClearError();
    if (count == nullptr)
    {
        return nullptr;
    }
    *count = 0;
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    int32_t rc = M3GPU_OK;
    if (w != nullptr)
    {
        rc = std::is_same<T, m3BodyMoveEvent>::value ? EnsureMoveEvents(w)
             : std::is_same<T, m3HitEvent>::value    ? EnsureHitEvents(w)
                                                     : EnsureEvents(w);
    }
    if (w == nullptr || rc != M3GPU_OK)
    {
        return nullptr;
    }
    const std::vector<T>& v = w->*member;
    *count = (int32_t)v.size();
    return v.empty() ? nullptr : v.data();
}

} // namespace

extern "C" const m3ContactEvent* m3World_ContactBeginEvents(m3WorldId worldId, int32_t* count)
{
    return Stream(worldId, count, &m3HostWorld::beginEvents);
}

extern "C" const m3ContactEvent* m3World_ContactEndEvents(m3WorldId worldId, int32_t* count)
{
    return Stream(worldId, count, &m3HostWorld::endEvents);
}

extern "C" const m3ContactEvent* m3World_SensorBeginEvents(m3WorldId worldId, int32_t* count)
{
    return Stream(worldId, count, &m3HostWorld::sensorBeginEvents);
}

extern "C" const m3ContactEvent* m3World_SensorEndEvents(m3WorldId worldId, int32_t* count)
{
    return Stream(worldId, count, &m3HostWorld::sensorEndEvents);
}

extern "C" const m3JointBreakEvent* m3World_JointBreakEvents(m3WorldId worldId, int32_t* count)
{
    return Stream(worldId, count, &m3HostWorld::jointBreakEvents);
}

extern "C" const m3BodyMoveEvent* m3World_BodyMoveEvents(m3WorldId worldId, int32_t* count)
{
    return Stream(worldId, count, &m3HostWorld::moveEvents);
}

extern "C" const m3HitEvent* m3World_HitEvents(m3WorldId worldId, int32_t* count)
{
    return Stream(worldId, count, &m3HostWorld::hitEvents);
}

extern "C" int32_t m3World_HitEventsDropped(m3WorldId worldId)
{
    M3_DEVICE_GUARD;
    m3gpuClearError();
    m3HostWorld* w = m3gpuWorldFromId(worldId);
    if (w == nullptr || EnsureHitEvents(w) != M3GPU_OK)
    {
        return 0;
    }
    return w->hitEventsDropped;
}
