// Host-side world object: the persistent slab image (m3_layout.h), the
// interned hull store, and the device residency bookkeeping.  Internal
// to the library; the public surface is include/maul3d_b200.h.
#ifndef M3_WORLD_H
#define M3_WORLD_H

#include "m3_layout.h"

#include <stdint.h>
#include <unordered_map>
#include <vector>

struct m3HostWorld
{
    int32_t slot = -1;
    uint16_t generation = 0;
    int32_t bodyCap = 0;
    int32_t shapeCap = 0;
    int32_t jointCap = 0;
    int32_t pairCap = 0;

    // Persistent image (host copy) and its view.
    std::vector<uint8_t> image;
    int64_t persistentBytes = 0;
    m3WorldView hv{};

    // Interned hull slabs live outside the fixed-capacity image: the
    // pool is sized by the hulls actually interned (count-derived, as
    // the reference's snapshot treats them).
    std::vector<m3HullData> hulls;
    std::vector<int32_t> hullRefs;
    std::unordered_multimap<uint64_t, int32_t> hullIndexByContent;

    // Device residency.
    uint8_t* dslab = nullptr;        // persistent + scratch
    int64_t dslabBytes = 0;
    int64_t scratchBytes = 0;
    m3HullData* dhulls = nullptr;    // device hull pool
    int32_t dhullCap = 0;
    m3WorldView dv{};                // device view (device addresses)
    bool hostDirty = true;           // host image newer than device
    bool deviceAhead = false;        // device newer than host image
};

// Registry (world.cpp).
m3HostWorld* m3gpuWorldFromId(m3WorldId id);
m3HostWorld* m3gpuWorldFromIndex0(uint16_t index0);

// Residency (device.cpp).
extern uint64_t g_m3ResidencyEpoch;
// Host-to-device bytes copied by uploads (device.cpp).
extern int64_t g_m3UploadedBytes;
int32_t m3gpuEnsureDevice(void);
int32_t m3gpuReserve(m3HostWorld* w);
int32_t m3gpuUpload(m3HostWorld* w);
int32_t m3gpuDownload(m3HostWorld* w);
void m3gpuRelease(m3HostWorld* w);
// Make the host image current before a host read or write.
int32_t m3gpuSyncHost(m3HostWorld* w);

// Step and hash entry points (step.cu).
int32_t m3gpuStepBatch(m3HostWorld** worlds, int32_t count, float dt, int32_t substeps,
                       int32_t steps);
int32_t m3gpuHashBatch(m3HostWorld** worlds, int32_t count, uint64_t* out);
// The parallel world hash (hash.cu): one block per world, blocks in
// `order`, out[world] = that world's m3WorldHashView.
int32_t m3gpuLaunchHash(const m3WorldView* views, const int32_t* order, int32_t count,
                        uint64_t* out);

// Error reporting (capi.cpp).
int32_t m3gpuSetError(int32_t code, const char* fmt, ...);
void m3gpuClearError(void);

#endif // M3_WORLD_H
