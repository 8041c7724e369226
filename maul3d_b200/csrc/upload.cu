// Batched world upload: one kernel copies every world's image parts (the
// part before the pair buffers, the current pair list) and interned hull
// slabs straight from page-locked, mapped host memory into the worlds'
// HBM slabs and hull pools.  One launch replaces thousands of small
// copy calls, and a hull slab (5808 bytes, sized for the largest hull)
// moves only the parts its counts use: about 460 bytes for a box.
#include "m3_world.h"

#include <cuda_runtime.h>

#include <stddef.h>

namespace
{
// Copies `bytes` (a multiple of 4) with the block's threads.
__device__ __forceinline__ void BlockCopy(uint8_t* dst, const uint8_t* src, int64_t bytes)
{
    if ((((uintptr_t)dst | (uintptr_t)src) & 15u) == 0)
    {
        const int64_t vecs = bytes / 16;
        const uint4* s4 = (const uint4*)src;
        uint4* d4 = (uint4*)dst;
        for (int64_t k = threadIdx.x; k < vecs; k += blockDim.x)
        {
            d4[k] = s4[k];
        }
        const int64_t done = vecs * 16;
        for (int64_t k = done / 4 + threadIdx.x; k < bytes / 4; k += blockDim.x)
        {
            ((uint32_t*)dst)[k] = ((const uint32_t*)src)[k];
        }
        return;
    }
    for (int64_t k = threadIdx.x; k < bytes / 4; k += blockDim.x)
    {
        ((uint32_t*)dst)[k] = ((const uint32_t*)src)[k];
    }
}

__host__ __device__ __forceinline__ int64_t RoundUp4(int64_t x)
{
    return (x + 3) & ~(int64_t)3;
}

// The used parts of one hull slab: [offset, offset + bytes) pairs, each a
// multiple of 4 bytes and inside its array (the arrays' sizes are
// multiples of 4 bytes, so rounding up stays inside them).
__host__ __device__ __forceinline__ int32_t HullRanges(int32_t nv, int32_t nf, int32_t ni,
                                                       int32_t ne, int64_t off[8], int64_t len[8])
{
    // Counts past the slab's arrays cannot come from the creation code;
    // clamp them anyway, so no range leaves the slab.
    nv = nv < 0 ? 0 : (nv > M3_HULL_MAX_VERTS ? M3_HULL_MAX_VERTS : nv);
    nf = nf < 0 ? 0 : (nf > M3_HULL_MAX_FACES ? M3_HULL_MAX_FACES : nf);
    ni = ni < 0 ? 0 : (ni > M3_HULL_MAX_FACE_INDICES ? M3_HULL_MAX_FACE_INDICES : ni);
    ne = ne < 0 ? 0 : (ne > M3_HULL_MAX_HALF_EDGES ? M3_HULL_MAX_HALF_EDGES : ne);
    off[0] = 0;
    len[0] = (int64_t)offsetof(m3HullData, vertices) + 12 * (int64_t)nv;
    off[1] = (int64_t)offsetof(m3HullData, faceNormals);
    len[1] = 12 * (int64_t)nf;
    off[2] = (int64_t)offsetof(m3HullData, faceOffsets);
    len[2] = 4 * (int64_t)nf;
    off[3] = (int64_t)offsetof(m3HullData, faceVertCounts);
    len[3] = RoundUp4(nf);
    off[4] = (int64_t)offsetof(m3HullData, faceVertStart);
    len[4] = RoundUp4(2 * (int64_t)nf);
    off[5] = (int64_t)offsetof(m3HullData, faceIndices);
    len[5] = RoundUp4(ni);
    off[6] = (int64_t)offsetof(m3HullData, edgeCount);
    len[6] = 4 + RoundUp4(6 * (int64_t)ne);
    off[7] = (int64_t)offsetof(m3HullData, center);
    len[7] = 12;
    return 8;
}

static_assert(offsetof(m3HullData, faceVertCounts) % 4 == 0, "word-aligned hull arrays");
static_assert(offsetof(m3HullData, faceVertStart) % 4 == 0, "word-aligned hull arrays");
static_assert(offsetof(m3HullData, faceIndices) % 4 == 0, "word-aligned hull arrays");
static_assert(offsetof(m3HullData, edgeCount) % 4 == 0, "word-aligned hull arrays");
static_assert(offsetof(m3HullData, edges) == offsetof(m3HullData, edgeCount) + 4,
              "edges follow the edge count");
static_assert((M3_HULL_MAX_FACES % 4) == 0 && (M3_HULL_MAX_FACE_INDICES % 4) == 0 &&
                  ((6 * M3_HULL_MAX_HALF_EDGES) % 4) == 0,
              "rounded-up ranges stay inside their arrays");

// Copies `bytes` (a multiple of 4) with the lanes of one warp.
__device__ __forceinline__ void WarpCopy(uint8_t* dst, const uint8_t* src, int64_t bytes,
                                         int32_t lane)
{
    for (int64_t k = lane; k < bytes / 4; k += 32)
    {
        ((uint32_t*)dst)[k] = ((const uint32_t*)src)[k];
    }
}

// One block per item; a hull item's slabs go one per warp.
__global__ void __launch_bounds__(256) m3UploadKernel(const m3UploadItem* items, int32_t count)
{
    const m3UploadItem it = items[blockIdx.x];
    if (it.hulls == 0)
    {
        BlockCopy(it.dst, it.src, it.bytes);
        return;
    }
    const int32_t lane = threadIdx.x & 31;
    const int32_t warps = blockDim.x >> 5;
    for (int32_t h = threadIdx.x >> 5; h < it.hulls; h += warps)
    {
        const uint8_t* src = it.src + (int64_t)h * (int64_t)sizeof(m3HullData);
        uint8_t* dst = it.dst + (int64_t)h * (int64_t)sizeof(m3HullData);
        int32_t c = 0;
        if (lane < 4)
        {
            const m3HullData* hs = (const m3HullData*)src;
            c = lane == 0 ? hs->vertexCount
                          : (lane == 1 ? hs->faceCount : (lane == 2 ? hs->indexCount : hs->edgeCount));
        }
        const int32_t nv = __shfl_sync(0xFFFFFFFFu, c, 0);
        const int32_t nf = __shfl_sync(0xFFFFFFFFu, c, 1);
        const int32_t ni = __shfl_sync(0xFFFFFFFFu, c, 2);
        const int32_t ne = __shfl_sync(0xFFFFFFFFu, c, 3);
        int64_t off[8];
        int64_t len[8];
        const int32_t n = HullRanges(nv, nf, ni, ne, off, len);
        for (int32_t r = 0; r < n; ++r)
        {
            WarpCopy(dst + off[r], src + off[r], len[r], lane);
        }
    }
}
} // namespace

int64_t m3HullUsedBytes(const m3HullData* h)
{
    int64_t off[8];
    int64_t len[8];
    const int32_t n = HullRanges(h->vertexCount, h->faceCount, h->indexCount, h->edgeCount, off,
                                 len);
    int64_t total = 0;
    for (int32_t r = 0; r < n; ++r)
    {
        total += len[r];
    }
    return total;
}

int32_t m3gpuLaunchUpload(const m3UploadItem* items, int32_t count)
{
    if (count > 0)
    {
        m3UploadKernel<<<count, 256>>>(items, count);
    }
    return M3GPU_OK;
}
