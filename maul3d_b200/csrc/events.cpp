// Event streams of a world's last step (world.h:207-313): contact and
// sensor begin/end events and joint-break events.
//
// The device step keeps the previous step's pair list and manifolds in
// the second pair buffer (the two buffers swap every step), records the
// previous pair count, and appends every joint it breaks to a ring with
// the ring's position at the start of the step.  So the last step's
// events need no work inside the step: the first read after a step
// copies the two key lists, the manifolds' point counts and the step's
// ring entries back and walks them as the reference's step does
// (solver.c:3747-3815 for contacts, solver.c:4233-4257 for breaks).
// Shape liveness and generations come from the host image, which this
// path never changes behind the host's back (the device destroys joints
// only, never shapes).
#include "m3_world.h"

#include <cuda_runtime.h>

#include <stddef.h>

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
    const int32_t newCount = sc.pairCount < 0 ? 0 : (sc.pairCount < sc.pairCap ? sc.pairCount : sc.pairCap);
    const int32_t oldCount =
        sc.prevPairCount < 0 ? 0 : (sc.prevPairCount < sc.pairCap ? sc.prevPairCount : sc.pairCap);
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
    if (w == nullptr || EnsureEvents(w) != M3GPU_OK)
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
