// Device residency of worlds: one HBM slab per world (persistent image
// followed by the step's scratch), one device hull pool per world, and
// the host<->device copies that keep the host image and the slab in
// agreement.  A world is uploaded whole before its first device step
// after any host-side change; the host image is refreshed lazily, only
// the sections a step can change (bodies, joints, the current pair
// lists, the scalars).

#include "m3_world.h"

#include <cuda_runtime.h>

#include <string.h>

#include <atomic>
#include <map>
#include <utility>
#include <vector>

static int s_deviceState = 0; // 0 unknown, 1 ready, -1 absent
static int s_device = 0;
// The device for page-locking host memory, readable from any thread
// without the device lock: -1 until the device is ready.
static std::atomic<int> s_lockDevice{-1};

int m3gpuLockDevice(void)
{
    return s_lockDevice.load(std::memory_order_acquire);
}

// Bumped whenever any world's device allocations change (slab or hull
// pool allocated, released): cached device views of a batch are valid
// only for the epoch they were built in.
uint64_t g_m3ResidencyEpoch = 1;
int64_t g_m3UploadedBytes = 0;

std::recursive_mutex& m3gpuDeviceMutex()
{
    static std::recursive_mutex* mu = new std::recursive_mutex(); // lives until exit
    return *mu;
}

extern "C" int32_t m3gpu_set_device(int32_t device)
{
    M3_DEVICE_GUARD;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
    {
        cudaGetLastError();
        return m3gpuSetError(M3GPU_ERR_INVALID, "device %d is not visible", device);
    }
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess)
    {
        return m3gpuSetError(M3GPU_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
    }
    s_device = device;
    s_deviceState = 1;
    s_lockDevice.store(device, std::memory_order_release);
    return M3GPU_OK;
}

// The current device is a property of the calling host thread: every
// entry makes the library's device current for its caller, so a thread
// other than the one that selected it launches on the same GPU.
int32_t m3gpuEnsureDevice(void)
{
    M3_DEVICE_GUARD;
    if (s_deviceState == 1)
    {
        const cudaError_t e = cudaSetDevice(s_device);
        if (e != cudaSuccess)
        {
            return m3gpuSetError(M3GPU_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
        }
        return M3GPU_OK;
    }
    if (s_deviceState == -1)
    {
        return m3gpuSetError(M3GPU_ERR_NO_DEVICE, "no CUDA device is visible");
    }
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count <= 0)
    {
        s_deviceState = -1;
        cudaGetLastError();
        return m3gpuSetError(M3GPU_ERR_NO_DEVICE, "no CUDA device is visible (%s)",
                             cudaGetErrorString(e));
    }
    s_deviceState = 1;
    cudaSetDevice(s_device);
    s_lockDevice.store(s_device, std::memory_order_release);
    return M3GPU_OK;
}

// Device memory for slabs and hull pools: blocks carved from large
// cudaMalloc chunks of the current device and reused through free lists
// per size class (m3SizeClass; cudaMalloc is a slow driver call: one per
// 512 MiB instead of two per world).  Chunks stay allocated until the
// process exits.
namespace
{
constexpr size_t kDevChunkBytes = (size_t)512 << 20;

struct DevChunk
{
    int device;
    uint8_t* base;
    size_t bytes;
    size_t used;
};

struct DevArena
{
    std::vector<DevChunk> chunks;
    std::map<std::pair<int, size_t>, std::vector<void*>> freeBlocks;
};

DevArena& TheDevArena()
{
    static DevArena* arena = new DevArena();
    return *arena;
}

size_t RoundDev(size_t bytes)
{
    return m3SizeClass(bytes, M3_SLAB_ALIGN);
}
} // namespace

int64_t g_m3DevAllocCalls = 0;
int64_t g_m3DevFreeCalls = 0;

static cudaError_t DevAlloc(void** out, size_t bytes)
{
    DevArena& a = TheDevArena();
    g_m3DevAllocCalls += 1;
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess)
    {
        return e;
    }
    const size_t size = RoundDev(bytes);
    auto it = a.freeBlocks.find(std::make_pair(device, size));
    if (it != a.freeBlocks.end() && !it->second.empty())
    {
        *out = it->second.back();
        it->second.pop_back();
        return cudaSuccess;
    }
    for (auto c = a.chunks.rbegin(); c != a.chunks.rend(); ++c)
    {
        if (c->device != device)
        {
            continue;
        }
        if (c->bytes - c->used >= size)
        {
            *out = c->base + c->used;
            c->used += size;
            return cudaSuccess;
        }
        break; // only the device's newest chunk is bumped
    }
    size_t chunkBytes = size > kDevChunkBytes ? size : kDevChunkBytes;
    void* base = nullptr;
    e = cudaMalloc(&base, chunkBytes);
    if (e != cudaSuccess && chunkBytes > size)
    {
        cudaGetLastError();
        chunkBytes = size; // memory is short: just this block
        e = cudaMalloc(&base, chunkBytes);
    }
    if (e != cudaSuccess)
    {
        return e;
    }
    a.chunks.push_back(DevChunk{device, (uint8_t*)base, chunkBytes, size});
    *out = base;
    return cudaSuccess;
}

static void DevFree(void* p, size_t bytes)
{
    if (p == nullptr)
    {
        return;
    }
    g_m3DevFreeCalls += 1;
    DevArena& a = TheDevArena();
    for (const DevChunk& c : a.chunks)
    {
        if ((uint8_t*)p >= c.base && (uint8_t*)p < c.base + c.bytes)
        {
            a.freeBlocks[std::make_pair(c.device, RoundDev(bytes))].push_back(p);
            return;
        }
    }
}

static int32_t CudaCheck(cudaError_t e, const char* what)
{
    if (e != cudaSuccess)
    {
        return m3gpuSetError(M3GPU_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
    }
    return M3GPU_OK;
}

// Offsets of a field inside the host image.
static int64_t Offset(const m3HostWorld* w, const void* hostPtr)
{
    return (int64_t)((const uint8_t*)hostPtr - w->image.data());
}

static void BuildDeviceView(m3HostWorld* w)
{
    m3LayoutPersistent(&w->dv, w->dslab, w->bodyCap, w->shapeCap, w->jointCap, w->pairCap);
    m3AttachDevicePools(w, &w->dv);
    w->dv.scratch = w->dslab + w->persistentBytes;
    w->dv.scratchBytes = w->scratchBytes;
}

// The heightfield slots and samples, copied whole when their content
// changed since the last copy (heightfields are static: in practice
// once, before the first step).
static int32_t UploadHeightFields(m3HostWorld* w)
{
    if (w->hfHeaders.empty() || (w->dhf != nullptr && w->dhfVersion == w->hfVersion))
    {
        return M3GPU_OK;
    }
    const size_t headers = (size_t)m3AlignUp(
        (int64_t)(w->hfHeaders.size() * sizeof(m3HeightFieldDev)), 16);
    const size_t bytes = headers + w->hfSamples.size() * sizeof(float);
    if (w->dhf != nullptr && w->dhfBytes < bytes)
    {
        cudaDeviceSynchronize();
        DevFree(w->dhf, w->dhfBytes);
        w->dhf = nullptr;
        w->dhfBytes = 0;
    }
    int32_t rc = M3GPU_OK;
    if (w->dhf == nullptr)
    {
        g_m3ResidencyEpoch += 1;
        rc = CudaCheck(DevAlloc((void**)&w->dhf, bytes), "allocate heightfields");
        if (rc != M3GPU_OK)
        {
            w->dhf = nullptr;
            return rc;
        }
        w->dhfBytes = bytes;
    }
    std::vector<uint8_t> blob(bytes, 0);
    memcpy(blob.data(), w->hfHeaders.data(), w->hfHeaders.size() * sizeof(m3HeightFieldDev));
    memcpy(blob.data() + headers, w->hfSamples.data(), w->hfSamples.size() * sizeof(float));
    rc = CudaCheck(cudaMemcpy(w->dhf, blob.data(), bytes, cudaMemcpyHostToDevice),
                   "upload heightfields");
    if (rc == M3GPU_OK)
    {
        w->dhfVersion = w->hfVersion;
    }
    return rc;
}

int32_t m3gpuReserve(m3HostWorld* w)
{
    M3_DEVICE_GUARD;
    int32_t rc = m3gpuEnsureDevice();
    if (rc != M3GPU_OK || w->dslab != nullptr)
    {
        return rc;
    }
    w->scratchBytes = m3gpuScratchBytes(w->bodyCap, w->shapeCap, w->jointCap, w->pairCap);
    w->dslabBytes = w->persistentBytes + w->scratchBytes;
    rc = CudaCheck(DevAlloc((void**)&w->dslab, (size_t)w->dslabBytes), "allocate slab");
    if (rc != M3GPU_OK)
    {
        w->dslab = nullptr;
    }
    // Both pair buffers start as the host's do at creation: zero (the
    // step keeps their parts past the live list equal to the reference's
    // single array, which starts zeroed).
    if (rc == M3GPU_OK)
    {
        const int64_t pairs = Offset(w, w->hv.keys0);
        rc = CudaCheck(cudaMemsetAsync(w->dslab + pairs, 0, (size_t)(w->persistentBytes - pairs), 0),
                       "clear pair buffers");
    }
    // Page-lock the host memory of the images (chunk by chunk, see
    // hostmem.cpp), so uploads are DMA copies straight from it.
    if (rc == M3GPU_OK)
    {
        m3HostLockAll();
    }
    // The hull pool too, sized for the hulls interned so far, so that the
    // upload itself allocates nothing.
    const int32_t hullCount = (int32_t)w->hulls.size();
    if (rc == M3GPU_OK && w->dhulls == nullptr)
    {
        const int32_t cap = hullCount < 4 ? 4 : hullCount;
        rc = CudaCheck(DevAlloc((void**)&w->dhulls, (size_t)cap * sizeof(m3HullData)),
                       "allocate hull pool");
        w->dhullCap = rc == M3GPU_OK ? cap : 0;
        if (rc != M3GPU_OK)
        {
            w->dhulls = nullptr;
        }
    }
    if (rc == M3GPU_OK)
    {
        rc = UploadHeightFields(w);
    }
    g_m3ResidencyEpoch += 1;
    return rc;
}

// Device allocations and the device view for an upload.
static int32_t UploadPrepare(m3HostWorld* w)
{
    int32_t rc = m3gpuEnsureDevice();
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    // The upload overwrites the device tree: no replay of the old one may
    // still be running.  The scratch's leaf bounds are then stale.
    m3gpuWaitTree(w);
    w->leafBoxValid = false;
    if (w->dslab == nullptr)
    {
        w->scratchBytes = m3gpuScratchBytes(w->bodyCap, w->shapeCap, w->jointCap, w->pairCap);
        w->dslabBytes = w->persistentBytes + w->scratchBytes;
        rc = CudaCheck(DevAlloc((void**)&w->dslab, (size_t)w->dslabBytes), "allocate slab");
        g_m3ResidencyEpoch += 1;
        if (rc != M3GPU_OK)
        {
            w->dslab = nullptr;
            return rc;
        }
        const int64_t pairs = Offset(w, w->hv.keys0);
        rc = CudaCheck(cudaMemsetAsync(w->dslab + pairs, 0, (size_t)(w->persistentBytes - pairs), 0),
                       "clear pair buffers");
        if (rc != M3GPU_OK)
        {
            return rc;
        }
    }
    int32_t hullCount = (int32_t)w->hulls.size();
    if (hullCount > w->dhullCap)
    {
        if (w->dhulls != nullptr)
        {
            // Steps in flight may still read the old pool; its block goes
            // back to the free lists only once they are done.
            cudaDeviceSynchronize();
            DevFree(w->dhulls, (size_t)w->dhullCap * sizeof(m3HullData));
            w->dhulls = nullptr;
        }
        g_m3ResidencyEpoch += 1;
        int32_t cap = hullCount < 4 ? 4 : hullCount;
        rc = CudaCheck(DevAlloc((void**)&w->dhulls, (size_t)cap * sizeof(m3HullData)),
                       "allocate hull pool");
        if (rc != M3GPU_OK)
        {
            w->dhullCap = 0;
            return rc;
        }
        w->dhullCap = cap;
    }
    if (w->dhulls == nullptr)
    {
        g_m3ResidencyEpoch += 1;
        rc = CudaCheck(DevAlloc((void**)&w->dhulls, 4 * sizeof(m3HullData)), "allocate hull pool");
        if (rc != M3GPU_OK)
        {
            return rc;
        }
        w->dhullCap = 4;
    }
    rc = UploadHeightFields(w);
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    BuildDeviceView(w);
    return M3GPU_OK;
}

// The copies of one world's upload, one call per part.
static int32_t UploadCopies(m3HostWorld* w)
{
    int32_t rc = M3GPU_OK;
    const int32_t hullCount = (int32_t)w->hulls.size();
    // Everything before the pair buffers, then the current pair list up
    // to its count: the other buffer and the unused tails are written by
    // the step before anything reads them.
    const int64_t head = Offset(w, w->hv.keys0);
    if (m3HostIsLocked(w->image.data(), (size_t)head))
    {
        // Page-locked: an asynchronous DMA on the default stream, ordered
        // before any later kernel; callers that return to the host
        // synchronise first.
        rc = CudaCheck(cudaMemcpyAsync(w->dslab, w->image.data(), (size_t)head,
                                       cudaMemcpyHostToDevice, 0),
                       "upload world image");
    }
    else
    {
        rc = CudaCheck(cudaMemcpy(w->dslab, w->image.data(), (size_t)head,
                                  cudaMemcpyHostToDevice),
                       "upload world image");
    }
    int64_t bytes = head;
    const int32_t n = w->pairTailsToDevice ? w->pairCap : w->hv.sc->pairCount;
    if (rc == M3GPU_OK && w->pairTailsToDevice)
    {
        // A restore set the whole arrays: both device buffers take the
        // host's current one.
        // Asynchronous on the default stream (ordered before any later
        // kernel) when the image is page-locked, as the head copy above.
        const int32_t buf = w->hv.sc->pairBuf;
        const size_t kb = (size_t)w->pairCap * sizeof(uint64_t);
        const size_t mb = (size_t)w->pairCap * sizeof(m3Manifold);
        const uint64_t* hk = buf == 0 ? w->hv.keys0 : w->hv.keys1;
        const m3Manifold* hm = buf == 0 ? w->hv.man0 : w->hv.man1;
        const bool locked = m3HostIsLocked(hk, kb) && m3HostIsLocked(hm, mb);
        auto copy = [locked](void* dst, const void* src, size_t n, cudaMemcpyKind kind) {
            return locked ? cudaMemcpyAsync(dst, src, n, kind, 0) : cudaMemcpy(dst, src, n, kind);
        };
        rc = CudaCheck(copy(w->dv.keys0, hk, kb, cudaMemcpyHostToDevice), "upload pair arrays");
        if (rc == M3GPU_OK)
        {
            rc = CudaCheck(copy(w->dv.man0, hm, mb, cudaMemcpyHostToDevice), "upload pair arrays");
        }
        if (rc == M3GPU_OK)
        {
            rc = CudaCheck(cudaMemcpyAsync(w->dv.keys1, w->dv.keys0, kb, cudaMemcpyDeviceToDevice, 0),
                           "copy pair arrays");
        }
        if (rc == M3GPU_OK)
        {
            rc = CudaCheck(cudaMemcpyAsync(w->dv.man1, w->dv.man0, mb, cudaMemcpyDeviceToDevice, 0),
                           "copy pair arrays");
        }
        bytes += (int64_t)(kb + mb);
        if (rc == M3GPU_OK)
        {
            w->pairTailsToDevice = false;
            w->pairTailsOnDevice = false;
        }
    }
    else if (rc == M3GPU_OK && n > 0)
    {
        const int32_t buf = w->hv.sc->pairBuf;
        rc = CudaCheck(cudaMemcpy(buf == 0 ? w->dv.keys0 : w->dv.keys1,
                                  buf == 0 ? w->hv.keys0 : w->hv.keys1,
                                  (size_t)n * sizeof(uint64_t), cudaMemcpyHostToDevice),
                       "upload pair keys");
        if (rc == M3GPU_OK)
        {
            rc = CudaCheck(cudaMemcpy(buf == 0 ? w->dv.man0 : w->dv.man1,
                                      buf == 0 ? w->hv.man0 : w->hv.man1,
                                      (size_t)n * sizeof(m3Manifold), cudaMemcpyHostToDevice),
                           "upload manifolds");
        }
        bytes += (int64_t)n * (int64_t)(sizeof(uint64_t) + sizeof(m3Manifold));
    }
    if (rc == M3GPU_OK && hullCount > 0)
    {
        const size_t hullBytes = (size_t)hullCount * sizeof(m3HullData);
        if (m3HostIsLocked(w->hulls.data(), hullBytes))
        {
            rc = CudaCheck(cudaMemcpyAsync(w->dhulls, w->hulls.data(), hullBytes,
                                           cudaMemcpyHostToDevice, 0),
                           "upload hulls");
        }
        else
        {
            rc = CudaCheck(cudaMemcpy(w->dhulls, w->hulls.data(), hullBytes,
                                      cudaMemcpyHostToDevice),
                           "upload hulls");
        }
        bytes += (int64_t)hullBytes;
    }
    g_m3UploadedBytes += bytes;
    if (rc == M3GPU_OK)
    {
        w->hostDirty = false;
    }
    return rc;
}

int32_t m3gpuUpload(m3HostWorld* w)
{
    M3_DEVICE_GUARD;
    int32_t rc = UploadPrepare(w);
    return rc == M3GPU_OK ? UploadCopies(w) : rc;
}

// Batched upload: worlds whose host memory the GPU can read (page-locked,
// mapped chunks) become items of one upload kernel; the others copy one
// call per part.  The item table goes through a page-locked staging
// buffer; callers synchronise before returning to the host, so a later
// call finds the staging free.
static m3UploadItem* s_itemHost = nullptr;
static m3UploadItem* s_itemDev = nullptr;
static int32_t s_itemCap = 0;

int32_t m3gpuUploadBatch(m3HostWorld** worlds, int32_t count)
{
    M3_DEVICE_GUARD;
    std::vector<m3UploadItem> items;
    std::vector<m3HostWorld*> batched;
    int64_t bytes = 0;
    for (int32_t i = 0; i < count; ++i)
    {
        m3HostWorld* w = worlds[i];
        int32_t rc = UploadPrepare(w);
        if (rc != M3GPU_OK)
        {
            return rc;
        }
        const int64_t head = Offset(w, w->hv.keys0);
        const int32_t n = w->hv.sc->pairCount;
        const int32_t buf = w->hv.sc->pairBuf;
        const uint64_t* hk = buf == 0 ? w->hv.keys0 : w->hv.keys1;
        const m3Manifold* hm = buf == 0 ? w->hv.man0 : w->hv.man1;
        const int32_t hullCount = (int32_t)w->hulls.size();
        if (w->pairTailsToDevice)
        {
            rc = UploadCopies(w);
            if (rc != M3GPU_OK)
            {
                return rc;
            }
            continue;
        }
        const uint8_t* srcHead = m3HostDevicePointer(w->image.data(), (size_t)head);
        const uint8_t* srcKeys = n > 0 ? m3HostDevicePointer(hk, (size_t)n * sizeof(uint64_t)) : nullptr;
        const uint8_t* srcMan = n > 0 ? m3HostDevicePointer(hm, (size_t)n * sizeof(m3Manifold)) : nullptr;
        const uint8_t* srcHulls =
            hullCount > 0 ? m3HostDevicePointer(w->hulls.data(), (size_t)hullCount * sizeof(m3HullData))
                          : nullptr;
        if (srcHead == nullptr || (n > 0 && (srcKeys == nullptr || srcMan == nullptr)) ||
            (hullCount > 0 && srcHulls == nullptr))
        {
            rc = UploadCopies(w);
            if (rc != M3GPU_OK)
            {
                return rc;
            }
            continue;
        }
        items.push_back(m3UploadItem{srcHead, w->dslab, head, 0, 0});
        bytes += head;
        if (n > 0)
        {
            items.push_back(m3UploadItem{srcKeys, (uint8_t*)(buf == 0 ? w->dv.keys0 : w->dv.keys1),
                                         (int64_t)n * (int64_t)sizeof(uint64_t), 0, 0});
            items.push_back(m3UploadItem{srcMan, (uint8_t*)(buf == 0 ? w->dv.man0 : w->dv.man1),
                                         (int64_t)n * (int64_t)sizeof(m3Manifold), 0, 0});
            bytes += (int64_t)n * (int64_t)(sizeof(uint64_t) + sizeof(m3Manifold));
        }
        if (hullCount > 0)
        {
            items.push_back(m3UploadItem{srcHulls, (uint8_t*)w->dhulls, 0, hullCount, 0});
            for (int32_t h = 0; h < hullCount; ++h)
            {
                bytes += m3HullUsedBytes(&w->hulls[(size_t)h]);
            }
        }
        batched.push_back(w);
    }
    const int32_t n = (int32_t)items.size();
    if (n == 0)
    {
        return M3GPU_OK;
    }
    if (n > s_itemCap)
    {
        cudaDeviceSynchronize();
        cudaFreeHost(s_itemHost);
        cudaFree(s_itemDev);
        s_itemHost = nullptr;
        s_itemDev = nullptr;
        s_itemCap = 0;
        int32_t rc = CudaCheck(cudaMallocHost((void**)&s_itemHost, sizeof(m3UploadItem) * (size_t)n),
                               "allocate upload table");
        if (rc == M3GPU_OK)
        {
            rc = CudaCheck(cudaMalloc((void**)&s_itemDev, sizeof(m3UploadItem) * (size_t)n),
                           "allocate upload table");
        }
        if (rc != M3GPU_OK)
        {
            return rc;
        }
        s_itemCap = n;
    }
    memcpy(s_itemHost, items.data(), sizeof(m3UploadItem) * (size_t)n);
    int32_t rc = CudaCheck(cudaMemcpyAsync(s_itemDev, s_itemHost, sizeof(m3UploadItem) * (size_t)n,
                                           cudaMemcpyHostToDevice, 0),
                           "upload table");
    if (rc == M3GPU_OK)
    {
        m3gpuLaunchUpload(s_itemDev, n);
        rc = CudaCheck(cudaGetLastError(), "upload kernel");
    }
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    for (m3HostWorld* w : batched)
    {
        w->hostDirty = false;
    }
    g_m3UploadedBytes += bytes;
    return M3GPU_OK;
}

int32_t m3gpuDownload(m3HostWorld* w)
{
    M3_DEVICE_GUARD;
    if (w->dslab == nullptr)
    {
        return M3GPU_OK;
    }
    int32_t rc0 = m3gpuEnsureDevice();
    if (rc0 != M3GPU_OK)
    {
        return rc0;
    }
    // The tree nodes are in the joint section below: its pending
    // replays first.
    m3gpuWaitTree(w);
    // Scalars first: they say which pair buffer is current and how long.
    int32_t rc = CudaCheck(cudaMemcpy(w->hv.sc, w->dv.sc, sizeof(m3WorldScalars),
                                      cudaMemcpyDeviceToHost),
                           "download scalars");
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    // Body section: [xf, shapeBody).
    int64_t b0 = Offset(w, w->hv.xf);
    int64_t b1 = Offset(w, w->hv.shapeBody);
    rc = CudaCheck(cudaMemcpy(w->image.data() + b0, w->dslab + b0, (size_t)(b1 - b0),
                              cudaMemcpyDeviceToHost),
                   "download bodies");
    // Joint section: [jtype, keys0).
    int64_t j0 = Offset(w, w->hv.jtype);
    int64_t j1 = Offset(w, w->hv.keys0);
    if (rc == M3GPU_OK)
    {
        rc = CudaCheck(cudaMemcpy(w->image.data() + j0, w->dslab + j0, (size_t)(j1 - j0),
                                  cudaMemcpyDeviceToHost),
                       "download joints");
    }
    // The current pair lists up to pairCount.
    int32_t n = w->hv.sc->pairCount;
    if (rc == M3GPU_OK && n > 0)
    {
        uint64_t* hk = w->hv.sc->pairBuf == 0 ? w->hv.keys0 : w->hv.keys1;
        uint64_t* dk = w->hv.sc->pairBuf == 0 ? w->dv.keys0 : w->dv.keys1;
        m3Manifold* hm = w->hv.sc->pairBuf == 0 ? w->hv.man0 : w->hv.man1;
        m3Manifold* dm = w->hv.sc->pairBuf == 0 ? w->dv.man0 : w->dv.man1;
        rc = CudaCheck(cudaMemcpy(hk, dk, (size_t)n * sizeof(uint64_t), cudaMemcpyDeviceToHost),
                       "download pair keys");
        if (rc == M3GPU_OK)
        {
            rc = CudaCheck(
                cudaMemcpy(hm, dm, (size_t)n * sizeof(m3Manifold), cudaMemcpyDeviceToHost),
                "download manifolds");
        }
    }
    if (rc == M3GPU_OK)
    {
        w->deviceAhead = false;
        m3DrainBrokenJoints(w);
    }
    return rc;
}

int32_t m3gpuWorldStatus(m3HostWorld* w)
{
    M3_DEVICE_GUARD;
    if (w->dslab == nullptr || !w->deviceAhead)
    {
        return w->hv.sc->status;
    }
    if (m3gpuEnsureDevice() != M3GPU_OK)
    {
        return m3gpu_last_error();
    }
    int32_t status = 0;
    if (CudaCheck(cudaMemcpy(&status, &w->dv.sc->status, sizeof(int32_t), cudaMemcpyDeviceToHost),
                  "read status") != M3GPU_OK)
    {
        return M3GPU_ERR_CUDA;
    }
    return status;
}

int32_t m3gpuDownloadPairTails(m3HostWorld* w)
{
    M3_DEVICE_GUARD;
    if (w->dslab == nullptr || !w->pairTailsOnDevice)
    {
        return M3GPU_OK;
    }
    if (m3gpuEnsureDevice() != M3GPU_OK)
    {
        return m3gpu_last_error();
    }
    const int32_t buf = w->hv.sc->pairBuf;
    int32_t rc = CudaCheck(cudaMemcpy(buf == 0 ? w->hv.keys0 : w->hv.keys1,
                                      buf == 0 ? w->dv.keys0 : w->dv.keys1,
                                      (size_t)w->pairCap * sizeof(uint64_t),
                                      cudaMemcpyDeviceToHost),
                           "download pair arrays");
    if (rc == M3GPU_OK)
    {
        rc = CudaCheck(cudaMemcpy(buf == 0 ? w->hv.man0 : w->hv.man1,
                                  buf == 0 ? w->dv.man0 : w->dv.man1,
                                  (size_t)w->pairCap * sizeof(m3Manifold), cudaMemcpyDeviceToHost),
                       "download pair arrays");
    }
    if (rc == M3GPU_OK)
    {
        w->pairTailsOnDevice = false;
    }
    return rc;
}

int32_t m3gpuSyncHost(m3HostWorld* w)
{
    M3_DEVICE_GUARD;
    if (!w->deviceAhead)
    {
        return M3GPU_OK;
    }
    return m3gpuDownload(w);
}

static void FreeSlots(m3HostWorld* w)
{
    if (w->dslots != nullptr)
    {
        DevFree(w->dslots, (size_t)w->persistentBytes * (size_t)w->slotCount);
        w->dslots = nullptr;
    }
    w->slotCount = 0;
    w->slots.clear();
}

void m3gpuRelease(m3HostWorld* w)
{
    M3_DEVICE_GUARD;
    g_m3ResidencyEpoch += 1;
    if (w->dslab != nullptr || w->dhulls != nullptr || w->dhf != nullptr)
    {
        // No copy from the host image may be in flight when it is freed.
        m3gpuEnsureDevice();
        cudaDeviceSynchronize();
    }
    w->treeCount = 0;
    w->treeFirst = 0;
    w->treeUnlaunched = 0;
    w->leafBoxValid = false;
    if (w->dslab != nullptr)
    {
        DevFree(w->dslab, (size_t)w->dslabBytes);
        w->dslab = nullptr;
    }
    if (w->dhulls != nullptr)
    {
        DevFree(w->dhulls, (size_t)w->dhullCap * sizeof(m3HullData));
        w->dhulls = nullptr;
    }
    w->dhullCap = 0;
    if (w->dhf != nullptr)
    {
        DevFree(w->dhf, w->dhfBytes);
        w->dhf = nullptr;
    }
    w->dhfBytes = 0;
    w->dhfVersion = 0;
    FreeSlots(w);
    w->hostDirty = true;
    w->deviceAhead = false;
}

// ---------------------------------------------------------------------
// Device snapshot slots: the slab's persistent part (everything a step
// reads and writes that outlives the step) copied within HBM, with the
// host state a step can change beside it.  The step's scratch needs no
// copy: a step rebuilds it, but for the tree's pending moves (replayed
// before a save and before a restore) and the leaves' bounds (rebuilt
// after a restore).
// ---------------------------------------------------------------------
static m3HostWorld* SlotWorld(m3WorldId world, int32_t slot, const char* what)
{
    m3HostWorld* w = m3gpuWorldFromId(world);
    if (w == nullptr || slot < 0 || slot >= w->slotCount)
    {
        m3gpuSetError(M3GPU_ERR_INVALID, "%s: stale world or slot out of range", what);
        return nullptr;
    }
    return w;
}

extern "C" int32_t m3gpu_slots_reserve(m3WorldId world, int32_t slots)
{
    M3_DEVICE_GUARD;
    m3gpuClearError();
    m3HostWorld* w = m3gpuWorldFromId(world);
    if (w == nullptr || slots < 0)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID, "m3gpu_slots_reserve: stale world or bad count");
    }
    int32_t rc = m3gpuEnsureDevice();
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    if (w->dslots != nullptr)
    {
        cudaDeviceSynchronize(); // no save or restore may still use them
        FreeSlots(w);
    }
    if (slots == 0)
    {
        return M3GPU_OK;
    }
    rc = CudaCheck(DevAlloc((void**)&w->dslots, (size_t)w->persistentBytes * (size_t)slots),
                   "allocate device snapshot slots");
    if (rc != M3GPU_OK)
    {
        w->dslots = nullptr;
        return rc;
    }
    w->slotCount = slots;
    w->slots.assign((size_t)slots, m3HostWorld::DeviceSlot());
    return M3GPU_OK;
}

extern "C" int32_t m3gpu_slot_save(m3WorldId world, int32_t slot)
{
    M3_DEVICE_GUARD;
    m3gpuClearError();
    m3HostWorld* w = SlotWorld(world, slot, "m3gpu_slot_save");
    if (w == nullptr)
    {
        return M3GPU_ERR_INVALID;
    }
    int32_t rc = m3gpuEnsureDevice();
    // The device copy must be the world: host changes uploaded, the
    // tree's recorded moves replayed.
    if (rc == M3GPU_OK && (w->dslab == nullptr || w->hostDirty))
    {
        rc = m3gpuUpload(w);
    }
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    m3gpuWaitTree(w);
    const size_t bytes = (size_t)w->persistentBytes;
    rc = CudaCheck(cudaMemcpyAsync(w->dslots + bytes * (size_t)slot, w->dslab, bytes,
                                   cudaMemcpyDeviceToDevice, 0),
                   "save device snapshot slot");
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    m3HostWorld::DeviceSlot& d = w->slots[(size_t)slot];
    d.valid = true;
    d.structure = w->structure;
    d.jointFree = w->jointFree;
    d.brokenDrained = w->brokenDrained;
    return M3GPU_OK;
}

extern "C" int32_t m3gpu_slot_restore(m3WorldId world, int32_t slot)
{
    M3_DEVICE_GUARD;
    m3gpuClearError();
    m3HostWorld* w = SlotWorld(world, slot, "m3gpu_slot_restore");
    if (w == nullptr)
    {
        return M3GPU_ERR_INVALID;
    }
    const m3HostWorld::DeviceSlot& d = w->slots[(size_t)slot];
    if (!d.valid || d.structure != w->structure || w->dslab == nullptr)
    {
        return m3gpuSetError(M3GPU_ERR_INVALID,
                             "m3gpu_slot_restore: slot %d is empty, or the world was built on "
                             "or restored since it was saved",
                             slot);
    }
    int32_t rc = m3gpuEnsureDevice();
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    // Replays of the current timeline write the slab: they finish first.
    m3gpuWaitTree(w);
    const size_t bytes = (size_t)w->persistentBytes;
    rc = CudaCheck(cudaMemcpyAsync(w->dslab, w->dslots + bytes * (size_t)slot, bytes,
                                   cudaMemcpyDeviceToDevice, 0),
                   "restore device snapshot slot");
    if (rc != M3GPU_OK)
    {
        return rc;
    }
    w->jointFree = d.jointFree;
    w->brokenDrained = d.brokenDrained;
    // The device holds the world now; the host image is read back when
    // needed, the pair arrays whole.
    w->deviceAhead = true;
    w->hostDirty = false;
    w->pairTailsToDevice = false;
    w->pairTailsOnDevice = true;
    w->leafBoxValid = false;
    m3JournalUnrecordable(w); // a rewind is not a command of the journal
    m3MarkEventEpoch(w, false);  // like a restore: no events until a step
    return M3GPU_OK;
}
