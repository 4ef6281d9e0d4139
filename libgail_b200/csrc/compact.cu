// Tier-1 output compaction: per-block results from the fixed-stride device tables into
// the packed Tier1Frame form the host codec consumes (Josephur/libgail
// core/tier1_types.h:12-28): CblkInfo per block, pass lengths and distortions back to
// back, codewords back to back on 4-byte boundaries.
//
// Three launches: the sums of tiles of 1024 blocks; per tile one CTA that adds up the
// sums of the tiles before it, scans its own blocks in shared memory and writes the
// CblkInfo records as contiguous words and each block's offsets to a device table; then
// a warp per block copies the pass tables and the codeword. Nothing is read from the
// output buffers, which may be mapped host memory.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "compact.cuh"
#include "hull.cuh"

namespace gb {

namespace {

constexpr int TILE = 1024;
constexpr int INFO_WORDS = 5;

__device__ __forceinline__ uint32_t warpInclusive(uint32_t v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__device__ __forceinline__ uint32_t warpTotal(uint32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// Codeword bytes rounded to whole words, and passes, of block i (zero past the end).
__device__ __forceinline__ void blockCounts(const CompactArgs& a, uint32_t i, uint32_t& bytes, uint32_t& passes) {
    bytes = passes = 0;
    if (i < a.n) {
        const uint4 in = reinterpret_cast<const uint4*>(a.info)[i];
        bytes = (in.w + 3u) & ~3u;
        passes = in.y;
    }
}

__global__ void __launch_bounds__(TILE) tileSumKernel(CompactArgs a) {
    __shared__ uint32_t sB[32], sP[32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    uint32_t b, p;
    blockCounts(a, blockIdx.x * TILE + tid, b, p);
    b = warpTotal(b);
    p = warpTotal(p);
    if (lane == 0) {
        sB[wid] = b;
        sP[wid] = p;
    }
    __syncthreads();
    if (wid == 0) {
        b = warpTotal(sB[lane]);
        p = warpTotal(sP[lane]);
        if (lane == 0) {
            a.scratch[2 * blockIdx.x] = b;
            a.scratch[2 * blockIdx.x + 1] = p;
        }
    }
}

__global__ void __launch_bounds__(TILE) scanKernel(CompactArgs a) {
    __shared__ uint32_t sRec[TILE * INFO_WORDS];
    __shared__ uint32_t sB[32], sP[32], sBase[2];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const uint32_t tile = blockIdx.x, first = tile * TILE;
    const uint32_t count = min((uint32_t)TILE, a.n - first);

    // offsets of this tile: the sums of the tiles before it
    if (wid == 0) {
        uint32_t b = 0, p = 0;
        for (uint32_t t = lane; t < tile; t += 32) {
            b += a.scratch[2 * t];
            p += a.scratch[2 * t + 1];
        }
        b = warpTotal(b);
        p = warpTotal(p);
        if (lane == 0) {
            sBase[0] = b;
            sBase[1] = p;
        }
    }
    // exclusive scan of the tile's blocks
    const uint32_t i = first + tid;
    uint32_t bytes, passes;
    blockCounts(a, i, bytes, passes);
    const uint32_t ib = warpInclusive(bytes, lane), ip = warpInclusive(passes, lane);
    if (lane == 31) {
        sB[wid] = ib;
        sP[wid] = ip;
    }
    __syncthreads();
    if (wid == 0) {
        const uint32_t vb = sB[lane], vp = sP[lane];
        const uint32_t xb = warpInclusive(vb, lane), xp = warpInclusive(vp, lane);
        sB[lane] = xb - vb;
        sP[lane] = xp - vp;
        if (tile == gridDim.x - 1 && lane == 31) {
            a.tot[0] = sBase[0] + xb;
            a.tot[1] = sBase[1] + xp;
        }
    }
    __syncthreads();
    const uint32_t dOff = sBase[0] + sB[wid] + ib - bytes, pOff = sBase[1] + sP[wid] + ip - passes;
    if ((uint32_t)tid < count) {
        uint32_t* r = sRec + INFO_WORDS * tid;
        r[0] = a.info[4 * (size_t)i];
        r[1] = passes;
        r[2] = dOff;
        r[3] = a.info[4 * (size_t)i + 3];
        r[4] = pOff;
        a.offsets[i] = make_uint2(dOff, pOff);
    }
    __syncthreads();
    // the CblkInfo records, contiguous words
    uint32_t* outInfo = a.outInfo + (size_t)INFO_WORDS * first;
    for (uint32_t k = tid; k < count * INFO_WORDS; k += TILE) outInfo[k] = sRec[k];
}

// A warp per block: its pass tables and codeword to their packed places.
__global__ void __launch_bounds__(256) copyKernel(CompactArgs a) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x >> 5);
    bool over = false;
    for (uint32_t blk = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); blk < a.n; blk += warps) {
        const uint2 o = a.offsets[blk];
        const uint4 in = reinterpret_cast<const uint4*>(a.info)[blk];
        const uint32_t np = in.y, len = in.w;
        const size_t src = (size_t)blk * kMaxPasses;
        for (uint32_t q = lane; q < np; q += 32) {
            a.outPassLen[o.y + q] = a.passLen[src + q];
            if (a.outPassDist) a.outPassDist[o.y + q] = a.passDist[src + q];
        }
        if (a.outHullPasses)
            for (uint32_t q = lane; q < np; q += 32) {
                a.outHullPasses[o.y + q] = a.hullPasses[src + q];
                a.outHullSlope[o.y + q] = a.hullSlope[src + q];
            }
        const uint32_t words = (len + 3u) >> 2;
        if ((uint64_t)o.x + words * 4ull > a.dataCap) {
            over = true;
            continue;
        }
        const uint32_t* cw = reinterpret_cast<const uint32_t*>(a.jobs[blk].cw);
        uint32_t* dst = reinterpret_cast<uint32_t*>(a.outData + o.x);
        // the bytes past the codeword in its last word are zeroed so that the packed frame
        // does not depend on what the region held before
        const uint32_t tailMask = (len & 3u) ? (1u << (8 * (len & 3u))) - 1u : 0xFFFFFFFFu;
        uint32_t w = lane;
        for (; w + 97 < words; w += 128) {  // four loads in flight per lane, never the last word
            const uint32_t v0 = cw[w], v1 = cw[w + 32], v2 = cw[w + 64], v3 = cw[w + 96];
            dst[w] = v0;
            dst[w + 32] = v1;
            dst[w + 64] = v2;
            dst[w + 96] = v3;
        }
        for (; w < words; w += 32) dst[w] = w == words - 1 ? cw[w] & tailMask : cw[w];
    }
    if (__any_sync(kFull, over) && lane == 0) a.tot[2] = 1u;
}

// PCRD hull points, a thread per block, from the fixed-stride pass tables.
__global__ void __launch_bounds__(HULL_THREADS) hullKernel(CompactArgs a) {
    __shared__ HullStack st;
    const int t = threadIdx.x;
    const uint32_t blk = blockIdx.x * HULL_THREADS + t;
    if (blk >= a.n) return;
    const uint4 in = reinterpret_cast<const uint4*>(a.info)[blk];
    const size_t o = (size_t)blk * kMaxPasses;
    hullOfBlock(st, t, (int)in.x, min((int)in.y, kMaxPasses), a.scale[blk], a.passLen + o, a.passDist + o,
                a.hullPasses + o, a.hullSlope + o);
}

}  // namespace

void compactTier1(const CompactArgs& a, cudaStream_t st) {
    if (a.n == 0) return;
    const uint32_t tiles = divUp(a.n, (uint32_t)TILE);
    tileSumKernel<<<tiles, TILE, 0, st>>>(a);
    scanKernel<<<tiles, TILE, 0, st>>>(a);
    if (a.scale) hullKernel<<<divUp(a.n, (uint32_t)HULL_THREADS), HULL_THREADS, 0, st>>>(a);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // into host memory the copy is bound by the bus: a third of the SMs keep it busy and
    // leave the rest to the kernels of other streams
    const uint32_t cap = a.hostOut ? (uint32_t)std::max(1, sms / 3) : (uint32_t)sms * 8;
    copyKernel<<<std::min(divUp(a.n, 8u), cap), 256, 0, st>>>(a);
    GB_CHECK(cudaGetLastError());
}

}  // namespace gb
