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
    std::mutex mu;     // chunks and free lists
    std::mutex growMu; // held while a new chunk is made
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

// Page-locks a chunk for the library's device (mapped too: the upload
// kernel reads the images straight from there); false when no device is
// up yet or the driver refuses (uploads from it then stay synchronous).
static bool LockChunk(Chunk& c, int device)
{
    if (device < 0 || cudaSetDevice(device) != cudaSuccess ||
        cudaHostRegister(c.base, c.bytes, cudaHostRegisterMapped | cudaHostRegisterPortable) !=
            cudaSuccess)
    {
        cudaGetLastError();
        return false;
    }
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
    return true;
}

// The free list of the block's size class, else a bump in the newest
// chunk; null when neither has room.  Under the arena's mutex.
static void* TakeBlock(Arena& a, size_t size)
{
    auto it = a.freeBlocks.find(size);
    if (it != a.freeBlocks.end() && !it->second.empty())
    {
        void* p = it->second.back();
        it->second.pop_back();
        return p;
    }
    // Older chunks' space comes back through the free lists.
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
    return nullptr;
}

void* m3HostAlloc(size_t bytes)
{
    Arena& a = TheArena();
    const size_t size = RoundPages(bytes);
    {
        std::lock_guard<std::mutex> lock(a.mu);
        if (void* p = TakeBlock(a, size))
        {
            return p;
        }
    }
    // A new chunk, one thread at a time (the others that need one wait
    // for it and then bump from it), made outside the arena's mutex so
    // that allocations with room keep going meanwhile; a block larger
    // than a chunk gets a chunk of its own.  Once the library's device
    // is up the chunk is page-locked here, on the allocating thread,
    // rather than by the next device reservation.
    std::lock_guard<std::mutex> grow(a.growMu);
    {
        std::lock_guard<std::mutex> lock(a.mu);
        if (void* p = TakeBlock(a, size))
        {
            return p;
        }
    }
    const size_t chunkBytes = size > kChunkBytes ? size : kChunkBytes;
    void* m = mmap(nullptr, chunkBytes, PROT_READ | PROT_WRITE, MAP_PRIVATE | MAP_ANONYMOUS, -1, 0);
    if (m == MAP_FAILED)
    {
        throw std::bad_alloc();
    }
    // Huge pages where the kernel offers them: a 2 MiB page is faulted
    // in once instead of 512 times.
    madvise(m, chunkBytes, MADV_HUGEPAGE);
    Chunk c{(uint8_t*)m, chunkBytes, size, false, nullptr};
    LockChunk(c, m3gpuLockDevice());
    std::lock_guard<std::mutex> lock(a.mu);
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
    const int device = m3gpuLockDevice();
    std::lock_guard<std::mutex> lock(a.mu);
    for (Chunk& c : a.chunks)
    {
        if (!c.locked)
        {
            LockChunk(c, device);
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
