// Host memory for world images and hull buffers: page-granular blocks
// carved from large anonymous mappings ("chunks").  A world that becomes
// device-resident page-locks the chunks (cudaHostRegister, once per
// chunk, never per world: registering is a slow driver call, so one call
// per 64 MiB instead of two per world).  Uploads from a locked chunk are
// plain asynchronous DMA copies.
//
// Blocks are reused through free lists per size class (m3SizeClass);
// chunks stay mapped (and, once locked, locked) until the process exits.
#include "m3_world.h"

#include <cuda_runtime.h>
#include <sys/mman.h>

#include <map>
#include <mutex>
#include <new>
#include <vector>

namespace
{
constexpr size_t kChunkBytes = (size_t)64 << 20;

struct Chunk
{
    uint8_t* base;
    size_t bytes;
    size_t used;
    bool locked;
    uint8_t* deviceBase; // the chunk as the GPU addresses it (locked chunks)
};

struct Arena
{
    std::mutex mu;
    std::vector<Chunk> chunks;
    std::map<size_t, std::vector<void*>> freeBlocks; // by size class
};

Arena& TheArena()
{
    static Arena* arena = new Arena(); // lives until exit, like the mappings
    return *arena;
}

size_t RoundPages(size_t bytes)
{
    return m3SizeClass(bytes, M3_HOST_PAGE);
}
} // namespace

void* m3HostAlloc(size_t bytes)
{
    Arena& a = TheArena();
    const size_t size = RoundPages(bytes);
    std::lock_guard<std::mutex> lock(a.mu);
    auto it = a.freeBlocks.find(size);
    if (it != a.freeBlocks.end() && !it->second.empty())
    {
        void* p = it->second.back();
        it->second.pop_back();
        return p;
    }
    // Bump allocation in the newest chunk (older chunks' space comes back
    // through the free lists); a block larger than a chunk gets a chunk
    // of its own.
    if (!a.chunks.empty())
    {
        Chunk& c = a.chunks.back();
        if (c.bytes - c.used >= size)
        {
            void* p = c.base + c.used;
            c.used += size;
            return p;
        }
    }
    const size_t chunkBytes = size > kChunkBytes ? size : kChunkBytes;
    void* m = mmap(nullptr, chunkBytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
    if (m == MAP_FAILED)
    {
        throw std::bad_alloc();
    }
    Chunk c{(uint8_t*)m, chunkBytes, size, false, nullptr};
    a.chunks.push_back(c);
    return m;
}

void m3HostFree(void* p, size_t bytes)
{
    if (p == nullptr)
    {
        return;
    }
    Arena& a = TheArena();
    std::lock_guard<std::mutex> lock(a.mu);
    a.freeBlocks[RoundPages(bytes)].push_back(p);
}

int32_t m3HostLockAll(void)
{
    Arena& a = TheArena();
    std::lock_guard<std::mutex> lock(a.mu);
    for (Chunk& c : a.chunks)
    {
        if (c.locked)
        {
            continue;
        }
        // Mapped too: the upload kernel reads the images straight from here.
        if (cudaHostRegister(c.base, c.bytes, cudaHostRegisterMapped | cudaHostRegisterPortable) ==
            cudaSuccess)
        {
            c.locked = true;
            void* dev = nullptr;
            if (cudaHostGetDevicePointer(&dev, c.base, 0) == cudaSuccess)
            {
                c.deviceBase = (uint8_t*)dev;
            }
            else
            {
                cudaGetLastError();
            }
        }
        else
        {
            cudaGetLastError(); // not fatal: uploads from it stay synchronous
        }
    }
    return M3GPU_OK;
}

bool m3HostIsLocked(const void* p, size_t bytes)
{
    Arena& a = TheArena();
    std::lock_guard<std::mutex> lock(a.mu);
    const uint8_t* q = (const uint8_t*)p;
    for (const Chunk& c : a.chunks)
    {
        if (q >= c.base && q + bytes <= c.base + c.bytes)
        {
            return c.locked;
        }
    }
    return false;
}

const uint8_t* m3HostDevicePointer(const void* p, size_t bytes)
{
    Arena& a = TheArena();
    std::lock_guard<std::mutex> lock(a.mu);
    const uint8_t* q = (const uint8_t*)p;
    for (const Chunk& c : a.chunks)
    {
        if (q >= c.base && q + bytes <= c.base + c.bytes)
        {
            return c.locked && c.deviceBase != nullptr ? c.deviceBase + (q - c.base) : nullptr;
        }
    }
    return nullptr;
}
