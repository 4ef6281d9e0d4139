// Device rate control and Tier-2 (rate_gpu.h).
//
// Per frame: the range of the hull slopes (one reduction), the slope histogram (a thread
// per block, 32-bit atomic sums of whole bytes and blocks, exact in any order), then per
// measurement of the threshold search one launch of the packet coder (a warp per packet:
// its lanes select the passes of the packet's blocks from their hull points, fetch their
// lengths and make each block's header bits in parallel, and one lane applies the bit
// stuffing) and a read-back of the tile-parts' sizes; with it, the packets at the same
// thresholds are placed by a scan and written, the warp copying the codewords.
#include "rate_gpu.h"

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstring>
#include <stdexcept>

#include "capi_util.h"
#include <math_constants.h>

#include "common.cuh"
#include "encoder.h"
#include "hull.cuh"
#include "rate_search.h"

namespace gb {

namespace {

constexpr int kPacketBlocks = 64;     // blocks of one packet the device coder holds (DCI: 48)
constexpr uint32_t kMaxAmbiguous = 4096;
constexpr double kBinMargin = 1e-7;   // bin units from an edge within which the host bins

struct PlanArgs {
    const int4* segs;       // x: first block, y: blocks across the band, z: ncbx | ncby << 16, w: Mb | comp << 8
    const int32_t* pkSeg;   // segments of packet p: [pkSeg[p], pkSeg[p + 1])
    const uint8_t* pkTp;    // tile-part of each packet
    const uint8_t* comp;    // component of each block
    uint32_t numPackets, numBlocks;
};

struct FrameArgs {
    const GbCblkInfo* info;
    const uint32_t* passLen;
    const uint8_t* data;
    const uint8_t* hp;
    const double* hs;
};

__device__ __forceinline__ int floorLog2(uint32_t v) { return 31 - __clz(v); }  // v > 0

// Passes of a block at threshold t: its hull points down to the first flatter one.
__device__ __forceinline__ uint32_t passesAt(const FrameArgs& f, const GbCblkInfo& ci, double t) {
    uint32_t np = 0;
    for (uint32_t q = 0; q < ci.numPasses; ++q) {
        const uint32_t k = f.hp[ci.passBase + q];
        if (k == 0 || f.hs[ci.passBase + q] < t) break;
        np = k;
    }
    return np;
}

// ---------------------------------------------------------- packet-header bits
// A packet header (B.10) is, after its first bit, each block's bits in packet order: its
// inclusion tag-tree bits, and for an included block its zero-bit-plane tag-tree bits, the
// pass-count code (Table B.4) and its length with the Lblock increment (B.10.7). Bit
// stuffing (B.10.1: the byte after an 0xFF carries 7 bits) applies to the concatenation.
//
// A tag-tree node sends bits only the first time a coding walk passes it: zeros from its
// parent's value (capped at the threshold) up to its own, then a 1 when its value is below
// the threshold; later walks find it known or at the threshold and send nothing. The first
// walk through a node of the inclusion tree is that of the first leaf in raster order of its
// rectangle (every block is coded, in raster order); through a node of the zero-bit-plane
// tree, that of the first included leaf of its rectangle. So each block's bits follow from
// its rectangles alone: a lane per block makes them, a scan places them, and one lane walks
// the bytes for the stuffing.

constexpr int kPacketSegs = 8;            // precinct-bands of one packet (DCI: 3)
constexpr int kRawWords = 2 * kPacketBlocks * 4 + 8;  // raw header bits, 115 at most per block

// A bit string of up to 128 bits, right-aligned in (hi, lo), first bit most significant.
struct BitStr {
    unsigned long long hi = 0, lo = 0;
    int n = 0;
    __device__ void put(uint32_t v, int k) {  // the k (<= 32) low bits of v
        if (k == 0) return;
        const unsigned long long x = (unsigned long long)(v & (k == 32 ? 0xFFFFFFFFu : ((1u << k) - 1u)));
        hi = (hi << k) | (lo >> (64 - k));
        lo = (lo << k) | x;
        n += k;
    }
    __device__ void zeros(int k) {
        for (; k > 32; k -= 32) put(0, 32);
        put(0, k);
    }
    // bits [from, from + k) counted from the least significant end, k <= 32
    __device__ uint32_t take(int from, int k) const {
        unsigned long long x;
        if (from >= 64) x = hi >> (from - 64);
        else if (from == 0) x = lo;
        else x = (lo >> from) | (hi << (64 - from));
        return (uint32_t)(x & (k == 32 ? 0xFFFFFFFFull : ((1ull << k) - 1ull)));
    }
};

// One warp's packet: its blocks in packet order (passes, planes, lengths, codeword offsets,
// segment), its segments (first block, geometry) and the raw header bits.
struct WarpPacket {
    uint8_t np[kPacketBlocks], nbps[kPacketBlocks], seg[kPacketBlocks];
    uint32_t len[kPacketBlocks], dataOff[kPacketBlocks];
    int segBase[kPacketSegs], segW[kPacketSegs], segH[kPacketSegs], segMb[kPacketSegs];
    uint32_t raw[kRawWords];
};

// Over the leaves of the rectangle of node (l, nx, ny) of a segment's tag trees: whether
// any is included, the least zero-bit-plane count, the raster index of the first included.
__device__ __forceinline__ void rectOf(const WarpPacket& W, int base, int w, int h, int Mb, int l, int nx, int ny,
                                       bool& any, int& minMsb, int& firstIncl) {
    const int x0 = nx << l, y0 = ny << l, x1 = min(w, (nx + 1) << l), y1 = min(h, (ny + 1) << l);
    any = false;
    minMsb = 1 << 30;
    firstIncl = -1;
    for (int y = y0; y < y1; ++y)
        for (int x = x0; x < x1; ++x) {
            const int k = y * w + x;
            minMsb = min(minMsb, Mb - (int)W.nbps[base + k]);
            if (W.np[base + k] && !any) {
                any = true;
                firstIncl = k;
            }
        }
}

// The header bits of block k of the packet (without the packet's first bit).
__device__ BitStr blockBits(const WarpPacket& W, int k) {
    const int s = W.seg[k], base = W.segBase[s], w = W.segW[s], h = W.segH[s], Mb = W.segMb[s];
    const int kk = k - base, x = kk % w, y = kk / w;
    int levels = 1;
    while (((w - 1) >> (levels - 1)) > 0 || ((h - 1) >> (levels - 1)) > 0) ++levels;
    BitStr b;
    // inclusion (threshold 1: a node's value is 0 when its rectangle has an included leaf)
    for (int l = levels - 1; l >= 0; --l) {
        const int nx = x >> l, ny = y >> l;
        if (x != (nx << l) || y != (ny << l)) continue;  // not the rectangle's first leaf
        bool any, anyP = true;
        int mm, fi;
        rectOf(W, base, w, h, Mb, l, nx, ny, any, mm, fi);
        if (l < levels - 1) rectOf(W, base, w, h, Mb, l + 1, nx >> 1, ny >> 1, anyP, mm, fi);
        const int v = any ? 0 : 1, vp = anyP ? 0 : 1;  // the root's floor is 0
        b.zeros(v - vp);
        if (v == 0) b.put(1, 1);
    }
    const int np = W.np[k];
    if (!np) return b;
    // zero bit-planes (no threshold is reached: every first visit ends with a 1)
    for (int l = levels - 1; l >= 0; --l) {
        const int nx = x >> l, ny = y >> l;
        bool any;
        int v, fi, vp = 0;
        rectOf(W, base, w, h, Mb, l, nx, ny, any, v, fi);
        if (fi != kk) continue;  // an earlier included leaf passed this node
        if (l < levels - 1) rectOf(W, base, w, h, Mb, l + 1, nx >> 1, ny >> 1, any, vp, fi);
        b.zeros(v - vp);
        b.put(1, 1);
    }
    // the pass count (Table B.4)
    if (np == 1) b.put(0, 1);
    else if (np == 2) b.put(0x2, 2);
    else if (np <= 5) b.put(0xC | (uint32_t)(np - 3), 4);
    else if (np <= 36) b.put(0x1E0 | (uint32_t)(np - 6), 9);
    else b.put(0xFF80 | (uint32_t)(np - 37), 16);
    // Lblock starts at 3; the length takes Lblock + floor(log2 passes) bits
    const uint32_t len = W.len[k];
    const int extra = floorLog2((uint32_t)np);
    const int need = len ? floorLog2(len) + 1 : 1;
    const int incr = max(0, need - (3 + extra));
    b.put(((1u << incr) - 1u) << 1, incr + 1);  // incr ones and a zero
    b.put(len, 3 + incr + extra);
    return b;
}

// Ors bit string b into the raw bits from bit position pos on.
__device__ __forceinline__ void orBits(uint32_t* raw, uint32_t pos, const BitStr& b) {
    int rem = b.n;
    while (rem > 0) {
        const int k = min(32 - (int)(pos & 31), rem);
        const uint32_t v = b.take(rem - k, k);
        atomicOr(&raw[pos >> 5], v << (32 - (int)(pos & 31) - k));
        pos += k;
        rem -= k;
    }
}

// The header bytes from `bits` raw bits (one lane): each byte takes 8 bits, or 7 after an
// 0xFF byte; the last is padded with zeros, and an 0xFF at the end is followed by 0x00.
// out null: count only.
__device__ uint32_t stuffBytes(const uint32_t* raw, uint32_t bits, uint8_t* out) {
    uint32_t pos = 0, bytes = 0, last = 0;
    while (pos < bits) {
        const int room = last == 0xFFu ? 7 : 8;
        const int k = (int)min((uint32_t)room, bits - pos);
        const unsigned long long win = ((unsigned long long)raw[pos >> 5] << 32) | raw[(pos >> 5) + 1];
        const uint32_t v = (uint32_t)((win << (pos & 31)) >> (64 - k));
        last = v << (room - k);
        if (out) out[bytes] = (uint8_t)last;
        ++bytes;
        pos += k;
    }
    if (last == 0xFFu) {
        if (out) out[bytes] = 0;
        ++bytes;
    }
    return bytes;
}

// Control words of one frame's device rate control.
struct RcCtl {
    unsigned long long range[2];  // max of ~bits (the smallest slope), max of bits (the largest)
    double lo, hi;                // the search bounds, log2 of the range widened by an octave
    int nb;                       // slope bins
    uint32_t flags;               // kFlagBins: the bins did not fit; kFlagBody: the body did not
};
constexpr uint32_t kFlagBins = 1u, kFlagBody = 2u;

// Copies a codeword of len bytes from src (on a 4-byte boundary, the codeword padded with
// zeros to whole words, as the packed frame keeps it) to dst (any alignment): the bytes up to
// dst's next word boundary, whole words each made from two source words by a funnel shift,
// then the rest. Lanes lane, lane + step, ... share the work.
__device__ __forceinline__ void copyCodeword(uint8_t* dst, const uint8_t* src, uint32_t len, uint32_t lane,
                                             uint32_t step) {
    const uint32_t head = min(len, (uint32_t)((4u - ((uint32_t)(uintptr_t)dst & 3u)) & 3u));
    for (uint32_t i = lane; i < head; i += step) dst[i] = src[i];
    const uint32_t words = (len - head) >> 2, sh = 8 * head;
    const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
    uint32_t* d = reinterpret_cast<uint32_t*>(dst + head);
    for (uint32_t j = lane; j < words; j += step) d[j] = head ? __funnelshift_r(s[j], s[j + 1], sh) : s[j];
    for (uint32_t i = head + 4 * words + lane; i < len; i += step) dst[i] = src[i];
}

// A warp (the whole CTA) per packet: small CTAs fit beside the resident Tier-1 kernels.
// WRITE false: the packet's size into pkBytes and its tile-part's total; WRITE true: the
// packet at body + pkOff[p] (when it fits in bodyCap) and its blocks' passes.
template <bool WRITE>
__global__ void __launch_bounds__(32) t2Kernel(PlanArgs P, FrameArgs F, double l0, double l1, double l2,
                                               uint32_t* pkBytes, unsigned long long* tpBytes, const uint32_t* pkOff,
                                               uint8_t* body, uint64_t bodyCap, uint8_t* passesOut, RcCtl* ctl) {
    __shared__ WarpPacket W;
    const int lane = threadIdx.x;
    const uint32_t p = blockIdx.x;
    if (p >= P.numPackets) return;
    const int s0 = P.pkSeg[p], s1 = P.pkSeg[p + 1];
    const double lam[3] = {l0, l1, l2};
    // the packet's blocks, a lane each
    bool any = false;
    int nb = 0;
    uint32_t bodyBytes = 0;
    for (int s = s0; s < s1; ++s) {
        const int4 g = P.segs[s];
        const int ncbx = g.z & 0xFFFF, ncby = g.z >> 16, nl = ncbx * ncby;
        if (lane == 0) {
            W.segBase[s - s0] = nb;
            W.segW[s - s0] = ncbx;
            W.segH[s - s0] = ncby;
            W.segMb[s - s0] = g.w & 0xFF;
        }
        const double t = lam[(g.w >> 8) & 3];
        for (int k = lane; k < nl; k += 32) {
            const uint32_t blk = (uint32_t)(g.x + (k / ncbx) * g.y + k % ncbx);
            const GbCblkInfo ci = F.info[blk];
            const uint32_t np = passesAt(F, ci, t);
            const uint32_t len = np ? F.passLen[ci.passBase + np - 1] : 0u;
            W.np[nb + k] = (uint8_t)np;
            W.nbps[nb + k] = (uint8_t)ci.nbps;
            W.seg[nb + k] = (uint8_t)(s - s0);
            W.len[nb + k] = len;
            W.dataOff[nb + k] = ci.dataOffset;
            any = any || np != 0;
            bodyBytes += len;
            if (WRITE) passesOut[blk] = (uint8_t)np;
        }
        nb += nl;
    }
    for (int i = lane; i < kRawWords; i += 32) W.raw[i] = 0;
    any = __any_sync(kFull, any);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) bodyBytes += __shfl_xor_sync(kFull, bodyBytes, o);
    __syncwarp();
    if (WRITE && (uint64_t)pkOff[p] + pkBytes[p] > bodyCap) {  // sized by the measurement before
        if (lane == 0) atomicOr(&ctl->flags, kFlagBody);
        return;
    }
    // the header: the packet's bit, then each block's bits at its place
    uint32_t bits = 1;
    if (any) {
        BitStr b0, b1;
        if (lane < nb) b0 = blockBits(W, lane);
        if (lane + 32 < nb) b1 = blockBits(W, lane + 32);
        uint32_t x0 = (uint32_t)b0.n, x1 = (uint32_t)b1.n;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t0 = __shfl_up_sync(kFull, x0, o), t1 = __shfl_up_sync(kFull, x1, o);
            if (lane >= o) {
                x0 += t0;
                x1 += t1;
            }
        }
        const uint32_t tot0 = __shfl_sync(kFull, x0, 31), tot1 = __shfl_sync(kFull, x1, 31);
        if (lane == 0) atomicOr(&W.raw[0], 0x80000000u);  // the packet is not empty
        orBits(W.raw, 1 + x0 - (uint32_t)b0.n, b0);
        orBits(W.raw, 1 + tot0 + x1 - (uint32_t)b1.n, b1);
        bits = 1 + tot0 + tot1;
    }
    __syncwarp();
    uint32_t hdr = 0;
    if (lane == 0) hdr = stuffBytes(W.raw, bits, WRITE ? body + pkOff[p] : nullptr);
    hdr = __shfl_sync(kFull, hdr, 0);
    if (!any) bodyBytes = 0;
    if (!WRITE) {
        if (lane == 0) {
            pkBytes[p] = hdr + bodyBytes;
            atomicAdd(&tpBytes[P.pkTp[p]], (unsigned long long)(hdr + bodyBytes));
        }
        return;
    }
    __syncwarp();
    // the codewords after the header: short ones each by its own lane, long ones by the warp
    const uint32_t len0 = lane < nb ? W.len[lane] : 0u, len1 = lane + 32 < nb ? W.len[lane + 32] : 0u;
    uint32_t x0 = len0, x1 = len1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t0 = __shfl_up_sync(kFull, x0, o), t1 = __shfl_up_sync(kFull, x1, o);
        if (lane >= o) {
            x0 += t0;
            x1 += t1;
        }
    }
    const uint32_t off0 = x0 - len0, off1 = __shfl_sync(kFull, x0, 31) + x1 - len1;
    uint8_t* dst = body + pkOff[p] + hdr;
    constexpr uint32_t kShort = 256;
    if (len0 && len0 <= kShort) copyCodeword(dst + off0, F.data + W.dataOff[lane], len0, 0, 1);
    if (len1 && len1 <= kShort) copyCodeword(dst + off1, F.data + W.dataOff[lane + 32], len1, 0, 1);
    for (int k = 0; k < nb; ++k) {
        const uint32_t len = W.len[k];
        if (len <= kShort) continue;
        const uint32_t off = __shfl_sync(kFull, k < 32 ? off0 : off1, k & 31);
        copyCodeword(dst + off, F.data + W.dataOff[k], len, (uint32_t)lane, 32);
    }
}

// Packet offsets in the codestream body: the packets before, and 14 bytes (SOT segment
// and SOD) before each tile-part's packets. One warp.
__global__ void __launch_bounds__(32) offsetsKernel(PlanArgs P, const uint32_t* pkBytes, uint32_t* pkOff) {
    const int lane = threadIdx.x;
    uint32_t carry = 0;
    for (uint32_t base = 0; base < P.numPackets; base += 32) {
        const uint32_t i = base + lane;
        const uint32_t v = i < P.numPackets ? pkBytes[i] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += t;
        }
        if (i < P.numPackets) pkOff[i] = carry + x - v + 14u * (P.pkTp[i] + 1u);
        carry += __shfl_sync(kFull, x, 31);
    }
}

// The range of the finite positive hull slopes into ctl->range; positive doubles order as
// their bit patterns.
__global__ void __launch_bounds__(64) rangeKernel(FrameArgs F, uint32_t n, RcCtl* ctl) {
    unsigned long long lo = 0, hi = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const GbCblkInfo ci = F.info[i];
        for (uint32_t q = 0; q < ci.numPasses && F.hp[ci.passBase + q] != 0; ++q) {
            const double s = F.hs[ci.passBase + q];
            if (isfinite(s) && s > 0) {
                const unsigned long long b = (unsigned long long)__double_as_longlong(s);
                lo = max(lo, ~b);
                hi = max(hi, b);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        lo = max(lo, __shfl_xor_sync(kFull, lo, o));
        hi = max(hi, __shfl_xor_sync(kFull, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (lo) atomicMax(&ctl->range[0], lo);
        if (hi) atomicMax(&ctl->range[1], hi);
    }
}

// The search bounds and bin count from the range, as the host forms them but with the
// device's log2; the host compares them with its own before it takes the bins.
__global__ void boundsKernel(RcCtl* ctl) {
    const unsigned long long r0 = ctl->range[0], r1 = ctl->range[1];
    double mn = r0 ? __longlong_as_double((long long)~r0) : CUDART_INF;
    double mx = r1 ? __longlong_as_double((long long)r1) : 0.0;
    if (mx == 0) mx = mn = 1;
    const double lo = log2(mn) - 1, hi = log2(mx) + 1;
    ctl->lo = lo;
    ctl->hi = hi;
    ctl->nb = max(16, (int)ceil((hi - lo) * 1024.0) + 2);
}

// The slope histogram: per component, bytes (each point's rate step) and blocks (a
// block's first point) by bin; bins is [bytes c0, c1, c2, blocks c0, c1, c2] x cap, for
// ctl->nb <= cap bins from ctl->lo (else only the flag). A point whose bin value lies within
// kBinMargin of an edge goes to amb (count, then per point: comp | first << 8, bytes,
// slope as two words) for the host to bin.
__global__ void __launch_bounds__(64) binsKernel(PlanArgs P, FrameArgs F, const RcCtl* ctlIn, RcCtl* ctl, int cap,
                                                 uint32_t* bins, uint32_t* amb) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const double lo = ctlIn->lo;
    const int nb = ctlIn->nb;
    if (nb > cap) {
        if (i == 0) atomicOr(&ctl->flags, kFlagBins);
        return;
    }
    if (i >= P.numBlocks) return;
    const GbCblkInfo ci = F.info[i];
    const int c = P.comp[i];
    uint32_t prev = 0;
    bool first = true;
    for (uint32_t q = 0; q < ci.numPasses; ++q) {
        const uint32_t k = F.hp[ci.passBase + q];
        if (k == 0) break;
        const uint32_t rate = F.passLen[ci.passBase + k - 1];
        const double s = F.hs[ci.passBase + q];
        int b = nb - 1;
        bool sure = true;
        if (isfinite(s)) {
            const double v = (log2(s) - lo) * 1024.0;
            const double fl = floor(v), fr = v - fl;
            sure = fr >= kBinMargin && fr <= 1.0 - kBinMargin;
            b = (int)fmin(fmax(fl, 0.0), (double)(nb - 1));
        }
        if (sure) {
            atomicAdd(&bins[(size_t)c * cap + b], rate - prev);
            if (first) atomicAdd(&bins[(size_t)(3 + c) * cap + b], 1u);
        } else {
            const uint32_t slot = atomicAdd(amb, 1u);
            if (slot < kMaxAmbiguous) {
                uint32_t* e = amb + 1 + 4 * slot;
                const unsigned long long bits = (unsigned long long)__double_as_longlong(s);
                e[0] = (uint32_t)c | (first ? 256u : 0u);
                e[1] = rate - prev;
                e[2] = (uint32_t)bits;
                e[3] = (uint32_t)(bits >> 32);
            }
        }
        prev = rate;
        first = false;
    }
}

// Hull points of a packed frame (pass tables at each block's passBase).
__global__ void __launch_bounds__(HULL_THREADS) packedHullKernel(const GbCblkInfo* info, const uint32_t* passLen,
                                                                 const int32_t* passDist, const double* scale,
                                                                 uint32_t n, uint8_t* hp, double* hs) {
    __shared__ HullStack st;
    const int t = threadIdx.x;
    const uint32_t blk = blockIdx.x * HULL_THREADS + t;
    if (blk >= n) return;
    const GbCblkInfo ci = info[blk];
    hullOfBlock(st, t, (int)ci.nbps, (int)ci.numPasses, scale[blk], passLen + ci.passBase, passDist + ci.passBase,
                hp + ci.passBase, hs + ci.passBase);
}

double asDouble(unsigned long long bits) {
    double d;
    std::memcpy(&d, &bits, 8);
    return d;
}

template <class T>
struct DevBuf {  // a growable device buffer
    T* p = nullptr;
    size_t cap = 0;
    void ensure(size_t n) {
        if (n <= cap) return;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        check(cudaMalloc((void**)&p, std::max<size_t>(n, 16) * sizeof(T)), "device memory for rate control");
        cap = n;
    }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

template <class T>
struct HostBuf {  // a growable pinned host buffer
    T* p = nullptr;
    size_t cap = 0;
    void ensure(size_t n) {
        if (n <= cap) return;
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        check(cudaHostAlloc((void**)&p, std::max<size_t>(n, 16) * sizeof(T), cudaHostAllocDefault),
              "pinned host memory for rate control");
        cap = n;
    }
    ~HostBuf() {
        if (p) cudaFreeHost(p);
    }
};

}  // namespace

// The control words, tile-part totals and edge points of one frame, one block of device
// memory so that each round trip clears and reads back one range.
struct RcState {
    RcCtl ctl;
    unsigned long long tp[8];
    uint32_t amb[1 + 4 * kMaxAmbiguous];
};
constexpr uint32_t kFirstAmb = 64;  // edge points read back with the first copy
constexpr size_t kHeadBytes = offsetof(RcState, amb) + 4;                  // ctl, tp, edge count
constexpr size_t kFirstBytes = offsetof(RcState, amb) + (1 + 4 * kFirstAmb) * 4;
constexpr size_t kFlagsAt = offsetof(RcState, ctl) + offsetof(RcCtl, flags);
constexpr size_t kMeasureBytes = offsetof(RcState, amb);                   // ctl and tp

struct DeviceRateControl::Impl {
    int dev;
    CodestreamWriter w;
    PlanArgs plan{};
    int ntp = 0;
    uint32_t n = 0, nPad = 0;  // blocks; the passes' bytes at the head of the output buffer
    DevBuf<int4> segs;
    DevBuf<int32_t> pkSeg;
    DevBuf<uint8_t> pkTp, comp;
    DevBuf<double> scale;
    // per frame, sized once
    DevBuf<RcState> state;
    DevBuf<RcCtl> ctl2;  // the host's bounds, for a second histogram
    DevBuf<uint32_t> bins, pk, pkOff;
    DevBuf<uint8_t> outBuf;  // passes (nPad bytes), then the codestream body
    HostBuf<RcState> hState;
    HostBuf<RcCtl> hCtl2;
    HostBuf<uint32_t> hBins;
    HostBuf<uint8_t> hOut;
    int binsCap = 1 << 16;   // bins per array the histogram holds
    int nbGuess = 48 << 10;  // bins read back with the first copy (the last frame's count)
    // frames uploaded from host memory
    DevBuf<GbCblkInfo> upInfo;
    DevBuf<uint32_t> upLen;
    DevBuf<int32_t> upDist;
    DevBuf<uint8_t> upData, upHp;
    DevBuf<double> upHs;

    Impl(int device, const Layout& L, const std::string& label, size_t bodyHint) : dev(device), w(L, label) {
        GB_CHECK(cudaSetDevice(dev));
        const auto& sg = w.segments();
        const auto& ps = w.packetSegments();
        const auto& tps = w.tilePartPackets();
        ntp = w.numTileParts();
        if (ntp > 8) throw std::logic_error("more tile-parts than the device rate control counts");
        std::vector<int4> hs(sg.size());
        for (size_t s = 0; s < sg.size(); ++s) {
            const auto& g = sg[s];
            const GbSubband& b = L.bands[(size_t)g.band];
            if (g.ncbx * g.ncby > 16 || g.ncbx > 16 || g.ncby > 16)
                throw std::logic_error("precinct-band too large for the device Tier-2 (at most 4 x 4 code-blocks)");
            hs[s] = make_int4(b.cblkBase + g.cby0 * b.ncbx + g.cbx0, b.ncbx, g.ncbx | (g.ncby << 16), b.Mb | (b.comp << 8));
        }
        std::vector<uint8_t> tpOf((size_t)w.numPackets());
        for (int t = 0; t < ntp; ++t)
            for (int p = tps[(size_t)t]; p < tps[(size_t)t + 1]; ++p) tpOf[(size_t)p] = (uint8_t)t;
        for (int p = 0; p < w.numPackets(); ++p) {
            int blocks = 0;
            for (int s = ps[(size_t)p]; s < ps[(size_t)p + 1]; ++s) blocks += sg[(size_t)s].ncbx * sg[(size_t)s].ncby;
            if (blocks > kPacketBlocks) throw std::logic_error("packet with too many code-blocks for the device Tier-2");
            if (ps[(size_t)p + 1] - ps[(size_t)p] > kPacketSegs)
                throw std::logic_error("packet with too many precinct-bands for the device Tier-2");
        }
        n = (uint32_t)L.numCblks();
        nPad = (n + 15u) & ~15u;
        std::vector<uint8_t> cmp(n);
        for (uint32_t i = 0; i < n; ++i) cmp[i] = (uint8_t)L.bands[L.cblks[i].band].comp;
        const std::vector<double> sc = blockScales(L);
        segs.ensure(hs.size());
        pkSeg.ensure(ps.size());
        pkTp.ensure(tpOf.size());
        comp.ensure(cmp.size());
        scale.ensure(sc.size());
        GB_CHECK(cudaMemcpy(segs.p, hs.data(), hs.size() * sizeof(int4), cudaMemcpyHostToDevice));
        GB_CHECK(cudaMemcpy(pkSeg.p, ps.data(), ps.size() * 4, cudaMemcpyHostToDevice));
        GB_CHECK(cudaMemcpy(pkTp.p, tpOf.data(), tpOf.size(), cudaMemcpyHostToDevice));
        GB_CHECK(cudaMemcpy(comp.p, cmp.data(), cmp.size(), cudaMemcpyHostToDevice));
        GB_CHECK(cudaMemcpy(scale.p, sc.data(), sc.size() * 8, cudaMemcpyHostToDevice));
        plan = {segs.p, pkSeg.p, pkTp.p, comp.p, (uint32_t)w.numPackets(), n};
        state.ensure(1);
        ctl2.ensure(1);
        hState.ensure(1);
        hCtl2.ensure(1);
        pk.ensure((size_t)w.numPackets());
        pkOff.ensure((size_t)w.numPackets());
        bins.ensure((size_t)6 * binsCap);
        hBins.ensure((size_t)6 * binsCap);
        outBuf.ensure(nPad + bodyHint);
        hOut.ensure(nPad + bodyHint);
    }

    // The tile-parts' sizes of the last measurement as CodestreamWriter::measure() reports them.
    CodestreamSizes sizesOf(const unsigned long long* tpb) {
        CodestreamSizes sz;
        sz.numTileParts = ntp;
        size_t total = w.longestHeaderBytes();
        for (int t = 0; t < ntp; ++t) {
            const size_t bytes = 14 + tpb[t];
            sz.tilePart[t] = bytes;
            sz.comp[t % 3] += bytes;
            total += bytes;
        }
        sz.total = total + 2;
        return sz;
    }

    uint64_t bodyBytesOf(const unsigned long long* tpb) const {
        uint64_t b = 0;
        for (int t = 0; t < ntp; ++t) b += 14 + tpb[t];
        return b;
    }

    // Reads back `count` bins of each of the six histogram arrays into hBins (the same
    // layout, stride binsCap), from entry `from` on.
    void copyBins(int from, int count, cudaStream_t st, RateResult& res) {
        if (count <= 0) return;
        GB_CHECK(cudaMemcpy2DAsync(hBins.p + from, (size_t)binsCap * 4, bins.p + from, (size_t)binsCap * 4,
                                   (size_t)count * 4, 6, cudaMemcpyDeviceToHost, st));
        res.d2hBytes += (size_t)6 * count * 4;
    }

    // The packets at thresholds l into outBuf (passes, then the body from nPad), with the
    // offsets from the sizes in pk.
    void enqueueWrite(const FrameArgs& F, const double l[3], cudaStream_t st) {
        offsetsKernel<<<1, 32, 0, st>>>(plan, pk.p, pkOff.p);
        t2Kernel<true><<<plan.numPackets, 32, 0, st>>>(plan, F, l[0], l[1], l[2], pk.p, nullptr, pkOff.p, outBuf.p + nPad,
                                                       outBuf.cap - nPad, outBuf.p, &state.p->ctl);
    }

    // Round trips to the device per frame: one for the slope range, bounds, histogram and the
    // size with every pass; one per further size measurement, each of which also writes the
    // packets at its thresholds and reads them back (the last one is the codestream's).
    RateResult run(const DeviceTier1& d, const RateLimits& lim, const std::string& tag, std::vector<uint8_t>& out,
                   cudaStream_t st) {
        GB_CHECK(cudaSetDevice(dev));
        const FrameArgs F{d.info, d.passLen, d.data, d.hullPasses, d.hullSlope};
        const uint32_t np = plan.numPackets;
        RcState* S = state.p;
        RcState& H = *hState.p;
        hOut.ensure(outBuf.cap);
        RateResult res;
        // (1) range, bounds, histogram, the size with every pass
        GB_CHECK(cudaMemsetAsync(S, 0, kHeadBytes, st));
        GB_CHECK(cudaMemsetAsync(bins.p, 0, (size_t)6 * binsCap * 4, st));
        rangeKernel<<<std::min(divUp(n, 64u), 592u), 64, 0, st>>>(F, n, &S->ctl);
        boundsKernel<<<1, 1, 0, st>>>(&S->ctl);
        binsKernel<<<divUp(n, 64u), 64, 0, st>>>(plan, F, &S->ctl, &S->ctl, binsCap, bins.p, S->amb);
        t2Kernel<false><<<np, 32, 0, st>>>(plan, F, 0.0, 0.0, 0.0, pk.p, S->tp, nullptr, nullptr, 0, nullptr, &S->ctl);
        GB_CHECK(cudaMemcpyAsync(&H, S, kFirstBytes, cudaMemcpyDeviceToHost, st));
        const int guess = std::min(nbGuess, binsCap);
        copyBins(0, guess, st, res);
        GB_CHECK(cudaStreamSynchronize(st));
        GB_CHECK(cudaGetLastError());
        res.launches += 4;
        res.d2hBytes += kFirstBytes;
        const CodestreamSizes size0 = sizesOf(H.tp);
        const uint64_t body0 = bodyBytesOf(H.tp);
        // the host's own bounds from the exact range; the device's bins count only if its
        // bounds are the same
        double minSlope = H.ctl.range[0] ? asDouble(~H.ctl.range[0]) : INFINITY;
        double maxSlope = H.ctl.range[1] ? asDouble(H.ctl.range[1]) : 0.0;
        double lo, hi;
        slopeBounds(minSlope, maxSlope, lo, hi);
        SlopeBins sb(lo, hi);
        const int nb = sb.size();
        // The device's bins are the host's when the bin counts agree and the lower bounds
        // differ by at most kLoTolerance (the two log2s may differ in the last place): such a
        // shift moves a point's bin value by ~1e-9 bin, so only points within the edge
        // margin could change bins, and those are binned here with the host's own bounds.
        constexpr double kLoTolerance = 1e-12;
        const bool same = H.ctl.nb == nb && std::fabs(H.ctl.lo - lo) <= kLoTolerance && !(H.ctl.flags & kFlagBins);
        if (!same) {  // a histogram at the host's bounds, in a larger buffer if need be
            if (nb > binsCap) {
                binsCap = nb + 4096;
                bins.ensure((size_t)6 * binsCap);
                hBins.ensure((size_t)6 * binsCap);
            }
            *hCtl2.p = RcCtl{};
            hCtl2.p->lo = lo;
            hCtl2.p->hi = hi;
            hCtl2.p->nb = nb;
            GB_CHECK(cudaMemcpyAsync(ctl2.p, hCtl2.p, sizeof(RcCtl), cudaMemcpyHostToDevice, st));
            GB_CHECK(cudaMemsetAsync(bins.p, 0, (size_t)6 * binsCap * 4, st));
            GB_CHECK(cudaMemsetAsync(S->amb, 0, 4, st));
            binsKernel<<<divUp(n, 64u), 64, 0, st>>>(plan, F, ctl2.p, &S->ctl, binsCap, bins.p, S->amb);
            GB_CHECK(cudaMemcpyAsync(H.amb, S->amb, (1 + 4 * kFirstAmb) * 4, cudaMemcpyDeviceToHost, st));
            copyBins(0, nb, st, res);
            GB_CHECK(cudaStreamSynchronize(st));
            GB_CHECK(cudaGetLastError());
            res.launches += 1;
            res.d2hBytes += (1 + 4 * kFirstAmb) * 4;
        } else if (nb > guess) {
            copyBins(guess, nb - guess, st, res);
            GB_CHECK(cudaStreamSynchronize(st));
        }
        nbGuess = nb + 4096;
        for (int c = 0; c < 3; ++c)
            for (int b = 0; b < nb; ++b) {
                const uint32_t by = hBins.p[(size_t)c * binsCap + b], bl = hBins.p[(size_t)(3 + c) * binsCap + b];
                if (by | bl) sb.add(c, b, (double)by, (double)bl);
            }
        const uint32_t na = H.amb[0];
        if (na > kMaxAmbiguous) throw std::runtime_error("too many hull slopes on slope-bin edges");
        if (na > kFirstAmb) {
            const size_t more = 4 * (size_t)(na - kFirstAmb) * 4;
            GB_CHECK(cudaMemcpyAsync(H.amb + 1 + 4 * kFirstAmb, S->amb + 1 + 4 * kFirstAmb, more, cudaMemcpyDeviceToHost,
                                     st));
            GB_CHECK(cudaStreamSynchronize(st));
            res.d2hBytes += more;
        }
        for (uint32_t a = 0; a < na; ++a) {
            const uint32_t* e = H.amb + 1 + 4 * a;
            const double sl = asDouble((unsigned long long)e[2] | ((unsigned long long)e[3] << 32));
            sb.add((int)(e[0] & 255u), sb.bin(sl), (double)e[1], (e[0] & 256u) ? 1.0 : 0.0);
        }
        sb.finish();
        // (2) the threshold search; each measurement also writes its packets and reads back
        // as much of them as a codestream under the limit can hold
        const uint64_t bodyCopy = std::min<uint64_t>(outBuf.cap - nPad, (uint64_t)lim.maxTotal + 65536);
        bool zeroPending = true;  // the first measurement (every pass) is the one above
        bool written = false;     // the last measurement's packets are in hOut
        auto measureWrite = [&](const double l[3]) {
            ++res.iterations;
            if (zeroPending && l[0] == 0 && l[1] == 0 && l[2] == 0) {
                zeroPending = false;
                written = false;
                return size0;
            }
            zeroPending = false;
            GB_CHECK(cudaMemsetAsync(reinterpret_cast<uint8_t*>(S) + kFlagsAt, 0, kMeasureBytes - kFlagsAt, st));
            t2Kernel<false><<<np, 32, 0, st>>>(plan, F, l[0], l[1], l[2], pk.p, S->tp, nullptr, nullptr, 0, nullptr,
                                               &S->ctl);
            enqueueWrite(F, l, st);
            GB_CHECK(cudaMemcpyAsync(&H, S, kMeasureBytes, cudaMemcpyDeviceToHost, st));
            GB_CHECK(cudaMemcpyAsync(hOut.p, outBuf.p, nPad + bodyCopy, cudaMemcpyDeviceToHost, st));
            GB_CHECK(cudaStreamSynchronize(st));
            GB_CHECK(cudaGetLastError());
            res.launches += 3;
            res.d2hBytes += kMeasureBytes + nPad + bodyCopy;
            written = !(H.ctl.flags & kFlagBody) && bodyBytesOf(H.tp) <= bodyCopy;
            return sizesOf(H.tp);
        };
        double lam[3] = {0, 0, 0};
        CodestreamSizes sz;
        rateSearch(lim, minSlope, maxSlope, lo, hi, sb, measureWrite, lam, sz);
        const uint64_t body = bodyBytesOf(H.tp);
        if (!written) {  // the frame fits with every pass, or its packets outgrew the buffer or the copy
            if (body > body0) throw std::logic_error("codestream body larger than with every pass");
            if (nPad + body > outBuf.cap) outBuf.ensure(nPad + body + 65536);
            hOut.ensure(nPad + body);
            GB_CHECK(cudaMemsetAsync(reinterpret_cast<uint8_t*>(S) + kFlagsAt, 0, 4, st));
            enqueueWrite(F, lam, st);
            GB_CHECK(cudaMemcpyAsync(&H.ctl, &S->ctl, sizeof(RcCtl), cudaMemcpyDeviceToHost, st));
            GB_CHECK(cudaMemcpyAsync(hOut.p, outBuf.p, nPad + body, cudaMemcpyDeviceToHost, st));
            GB_CHECK(cudaStreamSynchronize(st));
            GB_CHECK(cudaGetLastError());
            if (H.ctl.flags & kFlagBody) throw std::logic_error("codestream body outgrew its buffer");
            res.launches += 2;
            res.d2hBytes += sizeof(RcCtl) + nPad + body;
        }
        uint64_t tpBytes[8] = {};
        for (int t = 0; t < ntp; ++t) tpBytes[t] = 14 + H.tp[t];
        const CodestreamSizes made = w.assemble(hOut.p + nPad, tpBytes, tag, out);
        if (made.total != sz.total) throw std::logic_error("device codestream size differs from its measurement");
        res.passes.assign(hOut.p, hOut.p + n);
        res.lambda = std::max({lam[0], lam[1], lam[2]});
        for (int c = 0; c < 3; ++c) res.lambdaComp[c] = lam[c];
        res.distortion = NAN;
        res.sizes = sz;
        return res;
    }

    RateResult runHost(const Tier1View& t1, const RateLimits& lim, const std::string& tag, std::vector<uint8_t>& out,
                       cudaStream_t st) {
        GB_CHECK(cudaSetDevice(dev));
        if (t1.numInfo != n) throw std::logic_error("Tier-1 frame and layout have different code-block counts");
        for (uint32_t i = 0; i < n; ++i) {
            const GbCblkInfo& c = t1.info[i];
            if (c.numPasses > (uint32_t)kMaxPasses) throw std::logic_error("more coding passes than the device holds");
            for (uint32_t k = 1; k < c.numPasses; ++k)
                if (t1.passLen[c.passBase + k] < t1.passLen[c.passBase + k - 1])
                    throw std::logic_error("pass lengths that decrease");
        }
        // the codewords on 4-byte boundaries, zero-padded to whole words, as the device's packed
        // frames hold them (the packet writer copies them by words)
        std::vector<GbCblkInfo> info(t1.info, t1.info + n);
        size_t total = 0;
        for (const GbCblkInfo& c : info) total += (c.dataLen + 3u) & ~3u;
        std::vector<uint8_t> data(std::max<size_t>(total, 16), 0);
        size_t at = 0;
        for (uint32_t i = 0; i < n; ++i) {
            if (info[i].dataLen) std::memcpy(data.data() + at, t1.data + t1.info[i].dataOffset, info[i].dataLen);
            info[i].dataOffset = (uint32_t)at;
            at += (info[i].dataLen + 3u) & ~3u;
        }
        const size_t npass = std::max<size_t>(t1.numPasses, 1), nd = data.size();
        upInfo.ensure(n);
        upLen.ensure(npass);
        upDist.ensure(npass);
        upData.ensure(nd);
        upHp.ensure(npass);
        upHs.ensure(npass);
        GB_CHECK(cudaMemcpyAsync(upInfo.p, info.data(), (size_t)n * sizeof(GbCblkInfo), cudaMemcpyHostToDevice, st));
        if (t1.numPasses) {
            GB_CHECK(cudaMemcpyAsync(upLen.p, t1.passLen, (size_t)t1.numPasses * 4, cudaMemcpyHostToDevice, st));
            GB_CHECK(cudaMemcpyAsync(upDist.p, t1.passDist, (size_t)t1.numPasses * 4, cudaMemcpyHostToDevice, st));
        }
        GB_CHECK(cudaMemcpyAsync(upData.p, data.data(), nd, cudaMemcpyHostToDevice, st));
        packedHullKernel<<<divUp(n, (uint32_t)HULL_THREADS), HULL_THREADS, 0, st>>>(upInfo.p, upLen.p, upDist.p, scale.p,
                                                                                   n, upHp.p, upHs.p);
        GB_CHECK(cudaGetLastError());
        DeviceTier1 d{upInfo.p, upLen.p, upData.p, upHp.p, upHs.p};
        RateResult r = run(d, lim, tag, out, st);
        r.launches += 1;
        return r;
    }
};

DeviceRateControl::DeviceRateControl(int device, const Layout& L, const std::string& label, size_t bodyHint)
    : p_(std::make_unique<Impl>(device, L, label, bodyHint)) {}
DeviceRateControl::~DeviceRateControl() = default;

RateResult DeviceRateControl::run(const DeviceTier1& f, const RateLimits& lim, const std::string& tag,
                                  std::vector<uint8_t>& out, cudaStream_t st) {
    return p_->run(f, lim, tag, out, st);
}

RateResult DeviceRateControl::runHost(const Tier1View& t1, const RateLimits& lim, const std::string& tag,
                                      std::vector<uint8_t>& out, cudaStream_t st) {
    return p_->runHost(t1, lim, tag, out, st);
}

const Layout& DeviceRateControl::layout() const { return p_->w.layout(); }
size_t DeviceRateControl::emptyBytes() { return p_->w.emptyBytes(); }

}  // namespace gb
