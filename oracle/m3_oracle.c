// Oracle capture harness (test infrastructure, never shipped).
//
// White-box accessors over the reference engine compiled from its own
// sources (oracle/Makefile).  The parity tests drive the reference
// through its public API (m3World_Step, m3World_Hash, m3World_Snapshot)
// and read the internal SoA arrays through these functions so that a
// hash mismatch can be localised to the first differing body, pair or
// manifold.  Internal layout: src/world_internal.h:583-999 (m3World),
// :492-508 (m3Manifold, 188 bytes).

#include "world_internal.h"

#include <string.h>

#define M3O_API __attribute__((visibility("default")))

static const m3World* W(m3WorldId id)
{
    return m3WorldFromId(id);
}

M3O_API int32_t m3o_body_max(m3WorldId id)
{
    const m3World* w = W(id);
    return w ? w->bodyPool.maxIndex : -1;
}

M3O_API int32_t m3o_shape_max(m3WorldId id)
{
    const m3World* w = W(id);
    return w ? w->shapePool.maxIndex : -1;
}

M3O_API int32_t m3o_joint_max(m3WorldId id)
{
    const m3World* w = W(id);
    return w ? w->jointPool.maxIndex : -1;
}

M3O_API int32_t m3o_pair_count(m3WorldId id)
{
    const m3World* w = W(id);
    return w ? w->pairCount : -1;
}

M3O_API int32_t m3o_pair_capacity(m3WorldId id)
{
    const m3World* w = W(id);
    return w ? w->pairCapacity : -1;
}

M3O_API uint64_t m3o_step_count(m3WorldId id)
{
    const m3World* w = W(id);
    return w ? w->stepCount : 0;
}

M3O_API int32_t m3o_scratch_overflow(m3WorldId id)
{
    const m3World* w = W(id);
    return w ? w->scratch.overflow : -1;
}

M3O_API int32_t m3o_last_color_count(m3WorldId id)
{
    const m3World* w = W(id);
    return w ? w->lastColorCount : -1;
}

// Pair keys (u64) and manifolds (188-byte records) for [0, pairCount).
M3O_API int32_t m3o_copy_pairs(m3WorldId id, uint64_t* keys, void* manifolds, int32_t cap)
{
    const m3World* w = W(id);
    if (w == NULL || cap < w->pairCount)
    {
        return -1;
    }
    memcpy(keys, w->pairKeys, (size_t)w->pairCount * sizeof(uint64_t));
    memcpy(manifolds, w->manifolds, (size_t)w->pairCount * sizeof(m3Manifold));
    return w->pairCount;
}

// Per-body dynamic state for [0, maxIndex): transforms (40 B), linear
// and angular velocity (12 B each), awake flags and sleep timers.
M3O_API int32_t m3o_copy_bodies(m3WorldId id, void* transforms, void* lin, void* ang,
                                uint8_t* awake, float* sleepTimes, int32_t cap)
{
    const m3World* w = W(id);
    if (w == NULL || cap < w->bodyPool.maxIndex)
    {
        return -1;
    }
    int32_t n = w->bodyPool.maxIndex;
    memcpy(transforms, w->transforms, (size_t)n * sizeof(m3Transform));
    memcpy(lin, w->linearVelocities, (size_t)n * sizeof(m3Vec3));
    memcpy(ang, w->angularVelocities, (size_t)n * sizeof(m3Vec3));
    memcpy(awake, w->awake, (size_t)n);
    memcpy(sleepTimes, w->sleepTimes, (size_t)n * sizeof(float));
    return n;
}

// Creation-time body properties the hash covers (mass, inertia, centre).
M3O_API int32_t m3o_copy_mass(m3WorldId id, float* invMass, void* invInertia, void* inertia,
                              void* localCenters, float* minExt, float* maxExt, int32_t cap)
{
    const m3World* w = W(id);
    if (w == NULL || cap < w->bodyPool.maxIndex)
    {
        return -1;
    }
    int32_t n = w->bodyPool.maxIndex;
    memcpy(invMass, w->invMass, (size_t)n * sizeof(float));
    memcpy(invInertia, w->invInertiaLocal, (size_t)n * sizeof(m3Mat3));
    memcpy(inertia, w->inertiaLocal, (size_t)n * sizeof(m3Mat3));
    memcpy(localCenters, w->localCenters, (size_t)n * sizeof(m3Vec3));
    memcpy(minExt, w->minExtents, (size_t)n * sizeof(float));
    memcpy(maxExt, w->maxExtents, (size_t)n * sizeof(float));
    return n;
}

// Joint warm-start state for [0, jointMaxIndex).
M3O_API int32_t m3o_copy_joints(m3WorldId id, void* impulse, void* perp, void* limit,
                                void* angular, int32_t cap)
{
    const m3World* w = W(id);
    if (w == NULL || cap < w->jointPool.maxIndex)
    {
        return -1;
    }
    int32_t n = w->jointPool.maxIndex;
    memcpy(impulse, w->jointImpulse, (size_t)n * sizeof(m3Vec3));
    memcpy(perp, w->jointPerpImpulse, (size_t)n * sizeof(m3Vec3));
    memcpy(limit, w->jointLimitImpulse, (size_t)n * sizeof(m3Vec3));
    memcpy(angular, w->jointAngularImpulse, (size_t)n * sizeof(m3Vec3));
    return n;
}

// Hull slab of one interned hull slot (5808 bytes, padding-free).
M3O_API int32_t m3o_copy_hull(m3WorldId id, int32_t slot, void* out)
{
    const m3World* w = W(id);
    if (w == NULL || slot < 0 || slot >= w->hullPool.maxIndex)
    {
        return -1;
    }
    memcpy(out, &w->hullData[slot], sizeof(m3HullData));
    return (int32_t)sizeof(m3HullData);
}

// Step `steps` times and record the world hash after every step: the
// per-step parity trace the device path is compared against.
M3O_API void m3o_step_trace(m3WorldId id, float dt, int32_t substeps, int32_t steps,
                            uint64_t* hashes)
{
    for (int32_t s = 0; s < steps; ++s)
    {
        m3World_Step(id, dt, substeps);
        if (hashes != NULL)
        {
            hashes[s] = m3World_Hash(id);
        }
    }
}

M3O_API int32_t m3o_sizeof_manifold(void)
{
    return (int32_t)sizeof(m3Manifold);
}

M3O_API int32_t m3o_sizeof_hull(void)
{
    return (int32_t)sizeof(m3HullData);
}
