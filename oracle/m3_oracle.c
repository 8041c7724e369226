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

// ---------------------------------------------------------------------
// Host task pool for timing the reference with threads: the reference's
// own task interface (include/maul3d/world.h:15-26), the pattern of its
// determinism test (test/test_determinism.c:34-135), with persistent
// workers instead of a thread per range.  An enqueued task is split into
// at most `workers` ranges of at least minRange items; the calling
// thread runs the first, the workers the rest; finish waits for them.
// The reference's results do not depend on the split (parallel phases
// write disjoint slots), which the hashes confirm.
// ---------------------------------------------------------------------
#include <pthread.h>

#define M3O_POOL_MAX 64

typedef struct m3oPool
{
    pthread_mutex_t mu;
    pthread_cond_t work;
    pthread_cond_t done;
    pthread_t threads[M3O_POOL_MAX];
    int32_t workers;
    // The current task: ranges [1, rangeCount) are the workers'.
    m3TaskFn* task;
    void* context;
    int32_t starts[M3O_POOL_MAX + 1];
    int32_t rangeCount;
    int32_t nextRange;
    int32_t pending;
    uint64_t generation;
    int32_t quit;
} m3oPool;

static m3oPool s_pool;
static int32_t s_poolReady = 0;

static void* m3oPoolMain(void* arg)
{
    (void)arg;
    pthread_mutex_lock(&s_pool.mu);
    for (;;)
    {
        while (!s_pool.quit && s_pool.nextRange >= s_pool.rangeCount)
        {
            pthread_cond_wait(&s_pool.work, &s_pool.mu);
        }
        if (s_pool.quit)
        {
            break;
        }
        const int32_t r = s_pool.nextRange++;
        m3TaskFn* task = s_pool.task;
        void* context = s_pool.context;
        const int32_t a = s_pool.starts[r];
        const int32_t b = s_pool.starts[r + 1];
        pthread_mutex_unlock(&s_pool.mu);
        task(a, b, context);
        pthread_mutex_lock(&s_pool.mu);
        s_pool.pending -= 1;
        if (s_pool.pending == 0)
        {
            pthread_cond_signal(&s_pool.done);
        }
    }
    pthread_mutex_unlock(&s_pool.mu);
    return NULL;
}

static void* m3oPoolEnqueue(m3TaskFn* task, int32_t itemCount, int32_t minRange,
                            void* taskContext, void* userContext)
{
    (void)userContext;
    const int32_t parts = s_pool.workers + 1;
    int32_t grain = (itemCount + parts - 1) / parts;
    grain = grain < minRange ? minRange : grain;
    grain = grain < 1 ? 1 : grain;
    pthread_mutex_lock(&s_pool.mu);
    int32_t n = 0;
    for (int32_t start = 0; start < itemCount && n < parts; start += grain)
    {
        s_pool.starts[n++] = start;
    }
    s_pool.starts[n] = itemCount;
    s_pool.task = task;
    s_pool.context = taskContext;
    s_pool.rangeCount = n;
    s_pool.nextRange = 1;
    s_pool.pending = n > 0 ? n - 1 : 0;
    s_pool.generation += 1;
    pthread_cond_broadcast(&s_pool.work);
    pthread_mutex_unlock(&s_pool.mu);
    if (n > 0)
    {
        task(s_pool.starts[0], s_pool.starts[1], taskContext);
    }
    return &s_pool;
}

static void m3oPoolFinish(void* userTask, void* userContext)
{
    (void)userTask;
    (void)userContext;
    pthread_mutex_lock(&s_pool.mu);
    while (s_pool.pending > 0)
    {
        pthread_cond_wait(&s_pool.done, &s_pool.mu);
    }
    s_pool.rangeCount = 0;
    s_pool.nextRange = 0;
    pthread_mutex_unlock(&s_pool.mu);
}

// Gives the world the pool's hooks with `threads` threads in all (the
// caller's included); 1 or less takes them away (serial).  One pool per
// process, sized by its first use.  Returns the threads in use.
M3O_API int32_t m3o_use_task_pool(m3WorldId id, int32_t threads)
{
    m3World* w = m3WorldFromId(id);
    if (w == NULL)
    {
        return -1;
    }
    if (threads <= 1)
    {
        w->workerCount = 1;
        w->enqueueTask = NULL;
        w->finishTask = NULL;
        w->userTaskContext = NULL;
        return 1;
    }
    if (!s_poolReady)
    {
        const int32_t workers = threads - 1 < M3O_POOL_MAX ? threads - 1 : M3O_POOL_MAX;
        pthread_mutex_init(&s_pool.mu, NULL);
        pthread_cond_init(&s_pool.work, NULL);
        pthread_cond_init(&s_pool.done, NULL);
        s_pool.workers = workers;
        for (int32_t k = 0; k < workers; ++k)
        {
            pthread_create(&s_pool.threads[k], NULL, m3oPoolMain, NULL);
        }
        s_poolReady = 1;
    }
    w->workerCount = s_pool.workers + 1;
    w->enqueueTask = m3oPoolEnqueue;
    w->finishTask = m3oPoolFinish;
    w->userTaskContext = NULL;
    return s_pool.workers + 1;
}
