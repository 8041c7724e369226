// World hash on the device, one thread block per world, the byte stream
// hashed in parallel.
//
// FNV-1a 64 folds one byte at a time, h = (h ^ b) * P with
// P = 2^40 + 435, which is a chain of dependent multiplies: folded by one
// thread it runs at the multiply latency per byte, several milliseconds
// for a world of a few thousand bodies.  The block instead splits the
// stream into 32-byte chunks, one per thread, and uses three facts about
// the recurrence (all arithmetic mod 2^32, on the two 32-bit halves
// lo/hi of h):
//
//  1. The low byte s of lo evolves on its own: s' = ((s ^ b) * 435) & 255.
//     Multiplication by an odd constant and XOR are triangular in the
//     bits (bit j of the result depends on bits <= j only), and bit j of
//     s' is bit j of s XOR a function of b and the bits below j.  So bit j
//     of s over the whole stream is an exclusive prefix XOR, computable
//     by a block-wide scan once bits 0..j-1 are known: eight rounds, one
//     per bit, each a bit-sliced update of 32 bytes per thread plus a
//     ballot-and-popcount XOR scan across the block.
//  2. With s known at every byte, lo ^ b = lo + ((s ^ b) - s), so
//     lo' = 435 * (lo + d) is affine in lo: each chunk is one map
//     x -> A x + C, and an ordered scan of those maps gives every chunk's
//     starting lo.
//  3. hi' = 435 * hi + umulhi(x, 435) + (x << 8) with x = lo ^ b is affine
//     in hi once the lo sequence is known: one more ordered composition
//     gives the block's final hi.
//
// The stream itself is the record sequence of m3_hash.h (header, bodies,
// shapes, joints, pair count, pairs).  Each round of the outer loop
// stages up to one record per thread of the block's first half into
// shared memory (lengths by a counting pass and a block scan, then the
// bytes) and hashes the staged bytes tile by tile, carrying (lo, hi)
// across tiles and rounds.  The
// result is bit-identical to m3WorldHashView.
#include "m3_world.h"
#include "m3_hash.h"

#include <cuda_runtime.h>

#define M3H_BLOCK 256
#define M3H_WARPS (M3H_BLOCK / 32)
#define M3H_RECORD_MAX 256 // longest record of the stream (a body: 197 bytes)
// Records staged per round: half the block, so that the stage (32 KB)
// lets four blocks share an SM (the registers allow four; a 64 KB stage
// allowed three).
#define M3H_ROUND_RECORDS (M3H_BLOCK / 2)
#define M3H_STAGE_BYTES (M3H_ROUND_RECORDS * M3H_RECORD_MAX)
#define M3H_CHUNK 32
#define M3H_TILE (M3H_BLOCK * M3H_CHUNK)
#define M3H_MUL 435u // P = 2^40 + 435

static_assert(M3H_STAGE_BYTES % M3H_TILE == 0, "tiles must cover the stage exactly");

// Writes emitted bytes into the shared-memory stage at a running offset.
struct m3StageSink
{
    uint8_t* dst;
    int32_t off;
    __device__ void put(const void* p, int32_t n)
    {
        const uint8_t* s = (const uint8_t*)p;
        uint8_t* d = dst + off;
        int32_t k = 0;
        if (((uintptr_t)s & 3u) == 0)
        {
            for (; k + 4 <= n; k += 4)
            {
                const uint32_t v = *(const uint32_t*)(s + k);
                d[k] = (uint8_t)v;
                d[k + 1] = (uint8_t)(v >> 8);
                d[k + 2] = (uint8_t)(v >> 16);
                d[k + 3] = (uint8_t)(v >> 24);
            }
        }
        for (; k < n; ++k)
        {
            d[k] = s[k];
        }
        off += n;
    }
};

struct m3HashShared
{
    uint32_t warpBits[8][M3H_WARPS];
    uint32_t warpA[M3H_WARPS];
    uint32_t warpC[M3H_WARPS];
    int32_t warpSum[M3H_WARPS];
    uint32_t pow435[M3H_CHUNK + 1];
    int32_t bad;
};

// Transpose of an 8x8 bit matrix held in a 64-bit word, rows = bytes:
// bit c of byte r moves to bit r of byte c.
__device__ __forceinline__ uint64_t Transpose8(uint64_t x)
{
    uint64_t t = (x ^ (x >> 7)) & 0x00AA00AA00AA00AAull;
    x = x ^ t ^ (t << 7);
    t = (x ^ (x >> 14)) & 0x0000CCCC0000CCCCull;
    x = x ^ t ^ (t << 14);
    t = (x ^ (x >> 28)) & 0x00000000F0F0F0F0ull;
    x = x ^ t ^ (t << 28);
    return x;
}

// Exclusive block scan of one int per thread; every thread gets its
// offset and the total.
__device__ int32_t HashBlockScan(int32_t v, int32_t* total, m3HashShared& sh)
{
    const int32_t lane = threadIdx.x & 31;
    const int32_t warp = threadIdx.x >> 5;
    int32_t x = v;
    for (int32_t o = 1; o < 32; o <<= 1)
    {
        const int32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o)
        {
            x += y;
        }
    }
    if (lane == 31)
    {
        sh.warpSum[warp] = x;
    }
    __syncthreads();
    int32_t before = 0;
    int32_t all = 0;
    for (int32_t k = 0; k < M3H_WARPS; ++k)
    {
        const int32_t s = sh.warpSum[k];
        before += k < warp ? s : 0;
        all += s;
    }
    __syncthreads();
    *total = all;
    return before + x - v;
}

// Ordered composition of the threads' affine maps x -> A x + C (thread 0
// first).  Returns, per thread, the composition of all earlier threads'
// maps (exA, exC) and, to every thread, the composition of all of them.
__device__ void AffineBlockScan(uint32_t A, uint32_t C, uint32_t* exA, uint32_t* exC,
                                uint32_t* totA, uint32_t* totC, m3HashShared& sh)
{
    const int32_t lane = threadIdx.x & 31;
    const int32_t warp = threadIdx.x >> 5;
    uint32_t iA = A;
    uint32_t iC = C;
    for (int32_t o = 1; o < 32; o <<= 1)
    {
        const uint32_t a2 = __shfl_up_sync(0xFFFFFFFFu, iA, o);
        const uint32_t c2 = __shfl_up_sync(0xFFFFFFFFu, iC, o);
        if (lane >= o)
        {
            // Earlier map first, then this one.
            iC = iA * c2 + iC;
            iA = iA * a2;
        }
    }
    uint32_t eA = __shfl_up_sync(0xFFFFFFFFu, iA, 1);
    uint32_t eC = __shfl_up_sync(0xFFFFFFFFu, iC, 1);
    if (lane == 0)
    {
        eA = 1u;
        eC = 0u;
    }
    if (lane == 31)
    {
        sh.warpA[warp] = iA;
        sh.warpC[warp] = iC;
    }
    __syncthreads();
    uint32_t pA = 1u;
    uint32_t pC = 0u;
    uint32_t tA = 1u;
    uint32_t tC = 0u;
    for (int32_t k = 0; k < M3H_WARPS; ++k)
    {
        const uint32_t a2 = sh.warpA[k];
        const uint32_t c2 = sh.warpC[k];
        if (k < warp)
        {
            pC = a2 * pC + c2;
            pA = a2 * pA;
        }
        tC = a2 * tC + c2;
        tA = a2 * tA;
    }
    __syncthreads();
    *exC = eA * pC + eC;
    *exA = eA * pA;
    *totA = tA;
    *totC = tC;
}

// Folds tile[0, n) (n <= M3H_TILE) into (lo, hi); every thread of the
// block calls it with the same arguments and gets the same result.
__device__ void FnvTile(const uint8_t* tile, int32_t n, uint32_t& lo, uint32_t& hi,
                        m3HashShared& sh)
{
    const int32_t tid = threadIdx.x;
    const int32_t lane = tid & 31;
    const int32_t warp = tid >> 5;
    int32_t cnt = n - tid * M3H_CHUNK;
    cnt = cnt < 0 ? 0 : (cnt > M3H_CHUNK ? M3H_CHUNK : cnt);
    const uint32_t valid = cnt >= 32 ? 0xFFFFFFFFu : ((1u << cnt) - 1u);

    uint32_t wd[8];
    if (cnt > 0)
    {
        const uint4* src = (const uint4*)(tile + tid * M3H_CHUNK);
        const uint4 q0 = src[0];
        const uint4 q1 = src[1];
        wd[0] = q0.x;
        wd[1] = q0.y;
        wd[2] = q0.z;
        wd[3] = q0.w;
        wd[4] = q1.x;
        wd[5] = q1.y;
        wd[6] = q1.z;
        wd[7] = q1.w;
    }
    else
    {
#pragma unroll
        for (int32_t k = 0; k < 8; ++k)
        {
            wd[k] = 0u;
        }
    }
    // Bit planes: bit i of B[j] = bit j of byte i of the chunk.
    uint32_t B[8];
#pragma unroll
    for (int32_t j = 0; j < 8; ++j)
    {
        B[j] = 0u;
    }
#pragma unroll
    for (int32_t g = 0; g < 4; ++g)
    {
        const uint64_t y = Transpose8((uint64_t)wd[2 * g] | ((uint64_t)wd[2 * g + 1] << 32));
#pragma unroll
        for (int32_t j = 0; j < 8; ++j)
        {
            B[j] |= (uint32_t)((y >> (8 * j)) & 0xFFu) << (8 * g);
        }
    }

    // Round j: bit j of the low byte s before every byte of the tile.
    // acc holds, bit-sliced, ((s ^ b) mod 2^j) * 435 mod 256 for every
    // byte, i.e. the part of the product known from the lower bits.
    uint32_t acc[8];
    uint32_t S[8];
#pragma unroll
    for (int32_t j = 0; j < 8; ++j)
    {
        acc[j] = 0u;
    }
    const uint32_t s0 = lo & 0xFFu;
    const uint32_t ltMask = (1u << lane) - 1u;
#pragma unroll
    for (int32_t j = 0; j < 8; ++j)
    {
        // s'_j = s_j ^ b_j ^ acc_j: the toggles, prefix-XORed.
        const uint32_t T = (B[j] ^ acc[j]) & valid;
        uint32_t Q = T << 1;
        Q ^= Q << 1;
        Q ^= Q << 2;
        Q ^= Q << 4;
        Q ^= Q << 8;
        Q ^= Q << 16;
        const uint32_t ballot = __ballot_sync(0xFFFFFFFFu, (__popc(T) & 1) != 0);
        if (lane == 0)
        {
            sh.warpBits[j][warp] = (uint32_t)(__popc(ballot) & 1);
        }
        __syncthreads();
        uint32_t carry = ((s0 >> j) & 1u) ^ ((uint32_t)__popc(ballot & ltMask) & 1u);
        for (int32_t k = 0; k < warp; ++k)
        {
            carry ^= sh.warpBits[j][k];
        }
        S[j] = Q ^ (0u - carry);
        // Add x_j * 435 * 2^j (435 = 0b110110011 = 256 + 179; mod 256 the
        // multiplier is 179 = 2^7 + 2^5 + 2^4 + 2^1 + 2^0).
        const uint32_t X = S[j] ^ B[j];
#pragma unroll
        for (int32_t o = 0; o < 8; ++o)
        {
            if (((179 >> o) & 1) == 0 || j + o >= 8)
            {
                continue;
            }
            uint32_t c = X;
#pragma unroll
            for (int32_t q = j + o; q < 8; ++q)
            {
                const uint32_t t2 = acc[q] & c;
                acc[q] ^= c;
                c = t2;
            }
        }
    }
    // Low bytes back to byte order.
    uint32_t sw[8];
#pragma unroll
    for (int32_t g = 0; g < 4; ++g)
    {
        uint64_t z = 0;
#pragma unroll
        for (int32_t j = 0; j < 8; ++j)
        {
            z |= (uint64_t)((S[j] >> (8 * g)) & 0xFFu) << (8 * j);
        }
        const uint64_t y = Transpose8(z);
        sw[2 * g] = (uint32_t)y;
        sw[2 * g + 1] = (uint32_t)(y >> 32);
    }
    // lo: lo' = 435 * (lo + ((s ^ b) - s)), one affine map per chunk.
    uint32_t C = 0u;
#pragma unroll
    for (int32_t k = 0; k < M3H_CHUNK; ++k)
    {
        if (k < cnt)
        {
            const uint32_t s = (sw[k >> 2] >> (8 * (k & 3))) & 0xFFu;
            const uint32_t b = (wd[k >> 2] >> (8 * (k & 3))) & 0xFFu;
            C = M3H_MUL * (C + ((s ^ b) - s));
        }
    }
    const uint32_t A = sh.pow435[cnt];
    uint32_t exA;
    uint32_t exC;
    uint32_t totA;
    uint32_t totC;
    AffineBlockScan(A, C, &exA, &exC, &totA, &totC, sh);
    uint32_t l = exA * lo + exC;
    const uint32_t loEnd = totA * lo + totC;
    // hi: hi' = 435 * hi + umulhi(x, 435) + (x << 8), x = lo ^ b.
    uint32_t H = 0u;
#pragma unroll
    for (int32_t k = 0; k < M3H_CHUNK; ++k)
    {
        if (k < cnt)
        {
            const uint32_t b = (wd[k >> 2] >> (8 * (k & 3))) & 0xFFu;
            const uint32_t x = l ^ b;
            H = M3H_MUL * H + (__umulhi(x, M3H_MUL) + (x << 8));
            l = x * M3H_MUL;
        }
    }
    uint32_t hA;
    uint32_t hC;
    AffineBlockScan(A, H, &exA, &exC, &hA, &hC, sh);
    lo = loEnd;
    hi = hA * hi + hC;
}

__global__ void __launch_bounds__(M3H_BLOCK, 5) m3HashKernel(const m3WorldView* views,
                                                          const int32_t* order, int32_t count,
                                                          uint64_t* out)
{
    const int32_t wi = order[blockIdx.x];
    const m3WorldView* w = &views[wi];
    extern __shared__ __align__(16) uint8_t s_stage[];
    __shared__ m3HashShared sh;
    const int32_t tid = threadIdx.x;
    if (tid <= M3H_CHUNK)
    {
        uint32_t p = 1u;
        for (int32_t k = 0; k < tid; ++k)
        {
            p *= M3H_MUL;
        }
        sh.pow435[tid] = p;
    }
    if (tid == 0)
    {
        sh.bad = 0;
    }
    __syncthreads();
    const int32_t records = m3HashRecordCount(w);
    uint32_t lo = (uint32_t)M3_HASH_INIT;
    uint32_t hi = (uint32_t)(M3_HASH_INIT >> 32);
    for (int32_t r0 = 0; r0 < records; r0 += M3H_ROUND_RECORDS)
    {
        const int32_t r = r0 + tid;
        int32_t len = 0;
        if (tid < M3H_ROUND_RECORDS && r < records)
        {
            m3CountSink c{0};
            m3HashRecord(w, r, c);
            len = c.n;
            if (len > M3H_RECORD_MAX)
            {
                // Cannot happen with this record set; never overrun the stage.
                sh.bad = 1;
                len = 0;
            }
        }
        int32_t total = 0;
        const int32_t off = HashBlockScan(len, &total, sh);
        if (len > 0)
        {
            m3StageSink k{s_stage, off};
            m3HashRecord(w, r, k);
        }
        __syncthreads();
        for (int32_t base = 0; base < total; base += M3H_TILE)
        {
            const int32_t n = total - base < M3H_TILE ? total - base : M3H_TILE;
            FnvTile(s_stage + base, n, lo, hi, sh);
        }
        __syncthreads();
    }
    if (tid == 0)
    {
        out[wi] = sh.bad != 0 ? 0ull : (((uint64_t)hi << 32) | lo);
    }
}

int32_t m3gpuLaunchHash(const m3WorldView* views, const int32_t* order, int32_t count,
                        uint64_t* out)
{
    static int s_configured = -1;
    int device = 0;
    cudaGetDevice(&device);
    if (s_configured != device)
    {
        cudaError_t e = cudaFuncSetAttribute(
            m3HashKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, M3H_STAGE_BYTES);
        if (e != cudaSuccess)
        {
            return m3gpuSetError(M3GPU_ERR_CUDA, "cudaFuncSetAttribute(hash smem): %s",
                                 cudaGetErrorString(e));
        }
        s_configured = device;
    }
    if (count > 0)
    {
        m3HashKernel<<<count, M3H_BLOCK, M3H_STAGE_BYTES>>>(views, order, count, out);
    }
    return M3GPU_OK;
}
