// EBCOT Tier-1 encoder for sm_100a.
//
// Stage 1, context modelling (t1CmKernel): one warp per code-block. Lane x owns column x
// of the block and keeps its state as 32-bit row masks (bit r = row r): significance,
// sign, refined-before, coded-in-this-plane. A stripe (4 rows) of one pass is done by all
// lanes at once. The only sequential dependency of the scan order (columns left to right,
// rows top down) that matters is significance propagation, where a sample that becomes
// significant makes later samples eligible; it is solved as a least fixpoint over the
// warp (shuffle the left column's new significance, recompute, until no lane changes),
// which is the causal result because the dependency graph runs strictly left to right
// and top down. Each lane then emits its column's decisions in scan order and a warp
// prefix sum places them; a plane's decisions are staged in shared memory and copied out
// with coalesced stores. Per-pass symbol counts and distortion reductions are written.
//
// Stage 2, ordering (t1OrderKernel): counting sort of the blocks by decision count, most
// first, so the longest serial MQ chains start first.
//
// Stage 3, MQ coding (t1MqKernel): one lane per code-block. Lanes pull blocks from a
// device queue one at a time, so a lane that finishes early takes the next block
// instead of idling while its warp-mates finish. The coder is in branch-free
// select form (both MPS and LPS take the same instruction path until renormalisation),
// its contexts live in shared memory, and its input is prefetched 16 decisions ahead.
// The MQ state at each pass's end is recorded.
//
// Stage 4, truncation lengths (t1TruncKernel): a warp per block, a lane per pass; each
// pass's length is found from its recorded MQ state and the final codeword bytes. Kept
// out of the MQ kernel, whose lanes would otherwise stall on these byte reads one block
// end at a time while their warp-mates code.
//
// Semantics restated from ISO/IEC 15444-1 Annexes C and D as the reference coder applies
// them (Josephur/libgail core/t1_ref.cpp:52-292, kernels/mq_encoder.h:48-169,
// kernels/t1_common.h:20-53); bit-exact with it for every block.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "common.cuh"
#include "t1_encode.cuh"
#include "capi_util.h"
#include "t1_tables.h"
#include "tuning.h"

namespace gb {

namespace {

constexpr int CM_WARPS = 4;          // warps (code-blocks in flight) per CTA
constexpr int CM_THREADS = CM_WARPS * 32;
// Staging bytes per warp: one plane's decisions. A sample takes one refinement decision
// or at most two (zero coding and sign) in a plane, and a run-length stripe column adds at
// most two more (run, two position decisions, sign, in place of one zero-coding decision):
// 2 * 1024 + 2 * 256 = 2560 for a 32x32 block.
constexpr int STAGE = 2560 + 64;
constexpr int MQ_THREADS = 128;
constexpr int ORDER_BUCKETS = 128;

__constant__ uint8_t c_zc[4 * 45];   // zero-coding context by orient, h + 3 v + 9 d
__constant__ uint8_t c_sc[9];        // sign context | xor bit << 5, by (hc+1) * 3 + (vc+1)
__constant__ uint32_t c_mq[47];      // Qe | switch << 17 | NMPS << 18 | NLPS << 24

__device__ __forceinline__ uint32_t bit(uint32_t m, int r) { return (m >> r) & 1u; }
// A neighbour's contribution to the sign context: 0 when insignificant, else -1 / +1 by sign.
__device__ __forceinline__ int chiBits(int sig, int sgn) { return sig ? (sgn ? -1 : 1) : 0; }
__device__ __forceinline__ int clamp1(int v) { return v < -1 ? -1 : (v > 1 ? 1 : v); }
__device__ __forceinline__ int32_t distSig(uint32_t w) { return 192 * (int32_t)w - 9216; }
__device__ __forceinline__ int32_t distRef(uint32_t w) { return w >= 64u ? 64 * (int32_t)w - 5120 : 3072 - 64 * (int32_t)w; }

// Neighbourhood of one column for one stripe, all as row masks.
struct Nbr {
    uint32_t L;    // left column, current (includes its new significance in this stripe)
    uint32_t R;    // right column, as before this stripe (it is visited later)
    uint32_t S;    // own column as before this stripe
};

// Per 4-bit group of x, its number of set bits.
__device__ __forceinline__ uint32_t nibbleCounts(uint32_t x) {
    x = x - ((x >> 1) & 0x55555555u);
    return (x & 0x33333333u) + ((x >> 2) & 0x33333333u);
}

// Per stripe s of a row mask, at bit 4s: any of its four rows set; the row above it (4s - 1)
// set; the row below it (4s + 4) set.
__device__ __forceinline__ uint32_t nibbleAny(uint32_t m) { return (m | (m >> 1) | (m >> 2) | (m >> 3)) & 0x11111111u; }
__device__ __forceinline__ uint32_t rowAbove(uint32_t m) { return (m << 1) & 0x11111111u; }
__device__ __forceinline__ uint32_t rowBelow(uint32_t m) { return (m >> 4) & 0x11111111u; }

// Warp-inclusive prefix sum.
__device__ __forceinline__ uint32_t warpScan(uint32_t v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(kFull, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__device__ __forceinline__ int32_t warpSum(int32_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

__device__ __forceinline__ uint32_t shUp(uint32_t v, int lane) {
    const uint32_t t = __shfl_up_sync(kFull, v, 1);
    return lane == 0 ? 0u : t;
}
__device__ __forceinline__ uint32_t shDown(uint32_t v, int lane) {
    const uint32_t t = __shfl_down_sync(kFull, v, 1);
    return lane == 31 ? 0u : t;
}

// The contexts as tables of a sample's neighbour bits. Zero coding, per orientation, by
// bits 0-2: left column rows r-1..r+1, 3-5: right column rows r-1..r+1, 6: row above,
// 7: row below (all significance). Sign coding, the whole decision byte (context << 1 |
// coded bit), by bits 1, 4, 6, 7 as in the zero-coding key (left, right, above, below
// significant) and 0: sign of the row above, 2: the sample's own sign, 3: sign of the row
// below, 5: sign of the left neighbour, 8: sign of the right neighbour.
__device__ __forceinline__ void cmTables(uint8_t* s_zk, uint8_t* s_sk) {
    for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) {
        const int o = i >> 8, k = i & 255;
        const int h = ((k >> 1) & 1) + ((k >> 4) & 1);
        const int v = ((k >> 6) & 1) + ((k >> 7) & 1);
        const int d = (k & 1) + ((k >> 2) & 1) + ((k >> 3) & 1) + ((k >> 5) & 1);
        s_zk[i] = c_zc[45 * o + h + 3 * v + 9 * d];
    }
    for (int k = threadIdx.x; k < 512; k += blockDim.x) {
        const int hc = clamp1(chiBits((k >> 1) & 1, (k >> 5) & 1) + chiBits((k >> 4) & 1, (k >> 8) & 1));
        const int vc = clamp1(chiBits((k >> 6) & 1, k & 1) + chiBits((k >> 7) & 1, (k >> 3) & 1));
        const uint32_t t = c_sc[(hc + 1) * 3 + (vc + 1)];
        s_sk[k] = (uint8_t)(((t & 31u) << 1) | (((uint32_t)k >> 2 & 1u) ^ (t >> 5)));
    }
}

// Four rows' fields of a stripe side by side, one byte per row (row i of the stripe in
// byte i), by one multiply: the four shifted copies of x land in disjoint bit ranges.
// spread1: bit i of x (x < 16) to bit 0 of byte i; spread3: bits i..i+2 of x (x < 64) to
// bits 0-2 of byte i.
__device__ __forceinline__ uint32_t spread1(uint32_t x) { return (x * 0x00204081u) & 0x01010101u; }
__device__ __forceinline__ uint32_t spread3(uint32_t x) { return (x * 0x00204081u) & 0x07070707u; }
__device__ __forceinline__ uint32_t byteOf(uint32_t packed, int i) { return (packed >> (8 * i)) & 0xFFu; }

// Context modelling of block `job` by one warp: its decisions to its symbol region, its
// pass table and info words. mag: the warp's 32 x 32 magnitudes, buf: its plane staging,
// hist: its 19 context counters (zero between blocks). Returns the block's decisions
// (the same on every lane).
__device__ __forceinline__ uint32_t cmJob(const T1Launch& P, uint32_t job, uint32_t (*mag)[32], uint8_t* buf,
                                          uint32_t* hist, const uint8_t* s_zk, const uint8_t* s_sk, int lane) {
    uint32_t* status = P.ctl + 1;
    {
        const T1Job J = P.jobs[job];
        const int w = (J.geom & 31u) + 1, h = ((J.geom >> 5) & 31u) + 1, orient = (J.geom >> 10) & 3u;
        const int maxPasses = (J.geom >> 12) & 127u;
        const float slope = P.slope ? P.slope[J.slope] : 0.f;
        const uint8_t* zk = s_zk + 256 * orient;

        // Load: the block's 4 KB into the warp's rows as 16-byte vectors, each lane's loads
        // all in flight at once; then lane x reads column x. The words keep their sign bit
        // (bit 31): no magnitude read below reaches it but the early-termination estimate,
        // which masks it. Words outside w x h are zeroed here.
        {
            const uint4* src = reinterpret_cast<const uint4*>(J.coeffs);
            uint4* dst = reinterpret_cast<uint4*>(&mag[0][0]);
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                uint4 v[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) v[k] = src[(4 * half + k) * 32 + lane];
#pragma unroll
                for (int k = 0; k < 4; ++k) dst[(4 * half + k) * 32 + lane] = v[k];
            }
        }
        __syncwarp();
        if (w < 32 || h < 32)
            for (int r = 0; r < 32; ++r)
                if (lane >= w || r >= h) mag[r][lane] = 0u;
        uint32_t sgn = 0, colMax = 0;
#pragma unroll 8
        for (int r = 0; r < 32; ++r) {
            const uint32_t v = mag[r][lane];
            sgn |= (v >> 31) << r;
            colMax = max(colMax, v & 0x7FFFFFFFu);
        }
        uint32_t mx = colMax;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(kFull, mx, o));
        const uint32_t top = mx >> kFracBits;
        const int nbps = top ? 32 - __clz(top) : 0;
        uint32_t* info = P.info + 4 * (size_t)job;
        if (nbps == 0 || 3 * nbps - 2 > kMaxPasses) {
            if (lane == 0) {
                info[0] = nbps > 0 ? (uint32_t)nbps : 0u;
                info[1] = 0;
                info[2] = 0;
                info[3] = 0;
                if (nbps) atomicOr(status, kErrTooManyPlanes);
            }
            __syncwarp();
            return 0u;
        }
        if (lane < 19) hist[lane] = 0;
        __syncwarp();

        const uint32_t valid = lane < w ? (h >= 32 ? kFull : ((1u << h) - 1u)) : 0u;
        const uint32_t sgnL = shUp(sgn, lane), sgnR = shDown(sgn, lane);
        uint32_t sig = 0, refined = 0, symTotal = 0;
        int np = 0;
        const int nstripes = (h + 3) >> 2;
        uint8_t* gsym = J.sym;

        for (int p = nbps - 1; p >= 0 && np < maxPasses; --p) {
            uint32_t Bp = 0;
            for (int r = 0; r < h; ++r) Bp |= ((mag[r][lane] >> (p + kFracBits)) & 1u) << r;
            const uint32_t sig0 = sig;
            uint32_t vis = 0, count = 0;
            // the plane's decisions are staged at the alignment their region has in global
            // memory, so that they go out as 16-byte vectors
            uint8_t* const pb = buf + (symTotal & 15u);
            int32_t planeDist = 0;
            for (int type = (p == nbps - 1 ? 2 : 0); type < 3 && np < maxPasses; ++type) {
                // (1) the pass's row masks: E = rows coded, NEW = rows that become significant
                const uint32_t Spass = sig;
                uint32_t E = 0, NEW = 0;
                if (type == 0) {
                    // significance propagation: eligible = insignificant with a significant
                    // neighbour in scan order; stripes in order, each a warp fixpoint
#pragma unroll 1
                    for (int s = 0; s < nstripes; ++s) {
                        const int r0 = 4 * s;
                        const uint32_t S = sig, SL = shUp(S, lane), R = shDown(S, lane);
                        const uint32_t cand = (0xFu << r0) & valid & ~S;
                        // what makes a row eligible apart from the left column: the right
                        // column (rows r-1..r+1) and the own column's rows above and below,
                        // as before this stripe
                        const uint32_t fixed = R | (R << 1) | (R >> 1) | (S << 1) | (S >> 1);
                        if (!__any_sync(kFull, cand & (SL | (SL << 1) | (SL >> 1) | fixed))) continue;
                        // rows that turn significant once they are eligible
                        const uint32_t grow = cand & Bp;
                        // from nn = 0 upwards; done when the left columns' new significance
                        // makes no further sample eligible (the right column, the row below
                        // and the in-column chain do not change between iterations)
                        uint32_t nn = 0, ee = 0, L = SL;
#pragma unroll 1
                        for (int it = 0; it < 34; ++it) {
                            // eligible without the rows above turning significant in this
                            // pass; those that turn significant (seed); then down the column,
                            // a row below a new one is eligible and turns significant when
                            // its bit is set: a chain of at most three more rows
                            const uint32_t a = cand & (L | (L << 1) | (L >> 1) | fixed);
                            const uint32_t seed = a & Bp;
                            uint32_t n = seed | (grow & (seed << 1));
                            n = seed | (grow & (n << 1));
                            n = seed | (grow & (n << 1));
                            nn = n;
                            ee = a | (cand & (n << 1));
                            const uint32_t Ln = SL | shUp(nn, lane);
                            if (!__any_sync(kFull, cand & ~ee & (Ln | (Ln << 1) | (Ln >> 1)))) break;
                            L = Ln;
                        }
                        E |= ee;
                        NEW |= nn;
                        sig = S | nn;
                    }
                    vis |= E;
                } else if (type == 1) {
                    E = sig0 & valid;  // refinement of what was significant before this plane
                } else {
                    E = valid & ~Spass & ~vis;  // cleanup: everything else
                    NEW = E & Bp;
                    sig = Spass | NEW;
                }
                int32_t dist = 0;
                if (__any_sync(kFull, E)) {
                    // (2) neighbourhoods as the scan order sees them, per stripe s with rows
                    //     Q and the rows before it P: left column current up to the stripe,
                    //     right column and own column as before the stripe
                    const uint32_t SLp = shUp(Spass, lane), SRp = shDown(Spass, lane);
                    const uint32_t NL = shUp(NEW, lane), NR = shDown(NEW, lane);
                    const uint32_t nAny = (Spass << 1) | (Spass >> 1) | SLp | (SLp << 1) | (SLp >> 1) | SRp | (SRp << 1) |
                                          (SRp >> 1);
                    // cleanup run-length mode per stripe (bit 4s)
                    uint32_t runs = 0;
                    // (3) decisions per stripe, 10-bit fields, three stripes per word
                    uint32_t w0 = 0, w1 = 0, w2 = 0;
                    if (type != 2) {
                        // one decision per coded row, and a sign decision per new one: the
                        // popcounts of the 4-row groups, all stripes at once
                        const uint32_t c = nibbleCounts(E) + (type == 0 ? nibbleCounts(NEW) : 0u);
                        w0 = (c & 0xFu) | (((c >> 4) & 0xFu) << 10) | (((c >> 8) & 0xFu) << 20);
                        w1 = ((c >> 12) & 0xFu) | (((c >> 16) & 0xFu) << 10) | (((c >> 20) & 0xFu) << 20);
                        w2 = ((c >> 24) & 0xFu) | (((c >> 28) & 0xFu) << 10);
                    } else {
                        // all stripes at once, one bit (4s) or one nibble per stripe s. Run-length
                        // mode: all four rows in cleanup and no significant sample in the window
                        // rows r0-1 .. r0+4 of the left column (new ones up to the stripe's end),
                        // the right column and the own column (new ones above the stripe only).
                        const uint32_t full = E & (E >> 1) & (E >> 2) & (E >> 3) & 0x11111111u;
                        const uint32_t blocked = nibbleAny(SLp) | rowAbove(SLp) | rowBelow(SLp) | nibbleAny(NL) |
                                                 rowAbove(NL) | nibbleAny(SRp) | rowAbove(SRp) | rowBelow(SRp) |
                                                 rowAbove(NR) | nibbleAny(Spass) | rowAbove(Spass) | rowBelow(Spass) |
                                                 rowAbove(NEW);
                        runs = full & ~blocked;
                        const uint32_t runRows = runs * 0xFu;
                        // a run stripe: one decision when nothing in it turns significant, else
                        // the run decision, two position decisions, and the first new sample's
                        // sign, then the rows after it with their signs: 6 - first + new ones
                        const uint32_t N = NEW & runRows;
                        const uint32_t fill = N | ((N << 1) & 0xEEEEEEEEu) | ((N << 2) & 0xCCCCCCCCu) | ((N << 3) & 0x88888888u);
                        const uint32_t newRun = nibbleAny(N);
                        const uint32_t c = nibbleCounts(E & ~runRows) + nibbleCounts(NEW & ~runRows) + nibbleCounts(fill) +
                                           nibbleCounts(N) + (newRun << 1) + (runs & ~newRun);
                        w0 = (c & 0xFu) | (((c >> 4) & 0xFu) << 10) | (((c >> 8) & 0xFu) << 20);
                        w1 = ((c >> 12) & 0xFu) | (((c >> 16) & 0xFu) << 10) | (((c >> 20) & 0xFu) << 20);
                        w2 = ((c >> 24) & 0xFu) | (((c >> 28) & 0xFu) << 10);
                    }
                    const uint32_t i0 = warpScan(w0, lane), i1 = warpScan(w1, lane), i2 = warpScan(w2, lane);
                    const uint32_t t0 = __shfl_sync(kFull, i0, 31), t1 = __shfl_sync(kFull, i1, 31),
                                   t2 = __shfl_sync(kFull, i2, 31);
                    const uint32_t x0 = i0 - w0, x1 = i1 - w1, x2 = i2 - w2;
                    // (4) every lane writes its decisions for every stripe at its place
                    uint32_t sbase = count;
#pragma unroll 1
                    for (int s = 0; s < nstripes; ++s) {
                        const int r0 = 4 * s;
                        const int sh = 10 * (s % 3);
                        uint32_t pos = sbase + (((s < 3 ? x0 : (s < 6 ? x1 : x2)) >> sh) & 1023u);
                        sbase += ((s < 3 ? t0 : (s < 6 ? t1 : t2)) >> sh) & 1023u;
                        const uint32_t Q = 0xFu << r0, P = (1u << r0) - 1u;
                        uint32_t rows = E & Q;
                        if (!rows) continue;
                        if (type == 1) {
                            // the stripe's four decision bytes: context 16 (refined before),
                            // 15 (a significant neighbour) or 14, and the bit
                            const uint32_t rf = spread1((refined >> r0) & 0xFu);
                            const uint32_t dec = 0x1C1C1C1Cu + ((rf << 2) | ((spread1((nAny >> r0) & 0xFu) & ~rf) << 1) |
                                                                spread1((Bp >> r0) & 0xFu));
#pragma unroll 1
                            for (; rows; rows &= rows - 1) {
                                const int r = __ffs(rows) - 1;
                                pb[pos++] = (uint8_t)byteOf(dec, r - r0);
                                dist += distRef((mag[r][lane] >> p) & 0x7Fu);
                            }
                            continue;
                        }
                        uint32_t skip = 0;  // the row whose zero-coding decision the run decisions replace
                        if ((runs >> r0) & 1u) {
                            const uint32_t nb = (NEW >> r0) & 0xFu;
                            pb[pos++] = (uint8_t)((17u << 1) | (nb != 0));
                            if (nb == 0) continue;
                            const uint32_t first = __ffs(nb) - 1;
                            pb[pos++] = (uint8_t)((18u << 1) | (first >> 1));
                            pb[pos++] = (uint8_t)((18u << 1) | (first & 1u));
                            skip = 1u << (r0 + first);
                            rows &= ~(skip - 1u);
                        }
                        Nbr q;
                        q.L = SLp | (NL & (P | Q));
                        q.R = SRp | (NR & P);
                        q.S = Spass | (NEW & P);
                        const uint32_t SN = q.S | (NEW & Q);
                        // neighbour windows of the stripe, bit i about row r0 + i: left / right
                        // columns and own signs at rows r-1..r+1 from bit i, the row above (final:
                        // SN) at bit i, the row below (before the stripe) at bit i + 1; the
                        // neighbouring columns' signs are read at row r itself
                        const uint32_t wL = (uint32_t)(((unsigned long long)q.L << 1) >> r0);
                        const uint32_t wR = (uint32_t)(((unsigned long long)q.R << 1) >> r0);
                        const uint32_t wU = (uint32_t)(((unsigned long long)SN << 1) >> r0);
                        const uint32_t wS = q.S >> r0;
                        const uint32_t wG = (uint32_t)(((unsigned long long)sgn << 1) >> r0);
                        // the four rows' zero-coding keys, byte i for row r0 + i
                        const uint32_t zkeys = spread3(wL & 0x3Fu) | (spread3(wR & 0x3Fu) << 3) | (spread1(wU & 0xFu) << 6) |
                                               (spread1((wS >> 1) & 0xFu) << 7);
                        // and the sign bits of their sign-coding keys: own signs of rows r-1, r,
                        // r+1 to bits 0, 2, 3, the left neighbour's to bit 5
                        const uint32_t g3 = spread3(wG & 0x3Fu);
                        const uint32_t skeys = (g3 & 0x01010101u) | ((g3 & 0x06060606u) << 1) |
                                               (spread1((sgnL >> r0) & 0xFu) << 5);
#pragma unroll 1
                        for (; rows; rows &= rows - 1) {
                            const int r = __ffs(rows) - 1, i = r - r0;
                            const uint32_t zkey = byteOf(zkeys, i);
                            if (!((skip >> r) & 1u)) pb[pos++] = (uint8_t)((zk[zkey] << 1) | bit(Bp, r));
                            if (bit(NEW, r)) {
                                const uint32_t key = (zkey & 0xD2u) | (byteOf(skeys, i) & 0x2Du) | (((sgnR >> r) & 1u) << 8);
                                pb[pos++] = s_sk[key];
                                dist += distSig((mag[r][lane] >> p) & 0x7Fu);
                            }
                        }
                    }
                    count = sbase;
                }
                if (type == 1) refined |= sig0;
                const int32_t total = warpSum(dist);
                if (lane == 0) {
                    P.passEnd[(size_t)job * kMaxPasses + np] = symTotal + min(count, (uint32_t)STAGE);
                    P.passDist[(size_t)job * kMaxPasses + np] = total;
                }
                ++np;
                planeDist += total;
            }
            // the plane's decisions to the block's region
            count = min(count, (uint32_t)STAGE);
            __syncwarp();
            if (symTotal + count <= J.cap) {
                const uint32_t head = min(count, (16u - (symTotal & 15u)) & 15u);
                if ((uint32_t)lane < head) gsym[symTotal + lane] = pb[lane];
                const uint32_t nv = (count - head) >> 4;
                const uint4* s4 = reinterpret_cast<const uint4*>(pb + head);
                uint4* d4 = reinterpret_cast<uint4*>(gsym + symTotal + head);
                for (uint32_t i = lane; i < nv; i += 32) d4[i] = s4[i];
                const uint32_t done = head + 16u * nv;
                if ((uint32_t)lane < count - done) gsym[symTotal + done + lane] = pb[done + lane];
            } else if (lane == 0) {
                atomicOr(status, kErrSymbolSpace);
            }
            bool stop = false;
            if (slope > 0.f) {
                // early termination (the reference's stopAfterPlane, core/t1_ref.cpp:115-162),
                // with every float operation in the CPU's order
                for (uint32_t i = lane; i < count; i += 32) {
                    const uint32_t s = pb[i];
                    atomicAdd(&hist[s >> 1], (s & 1u) ? 0x10000u : 1u);
                }
                __syncwarp();
                if (lane == 0) {
                    float bits = 0.f;
                    for (int cx = 0; cx < 19; ++cx) {
                        const uint32_t hv = hist[cx];
                        const float n0 = (float)(hv & 0xFFFFu), n1 = (float)(hv >> 16), n = __fadd_rn(n0, n1);
                        if (n > 0.f) {
                            const float l0 = log2f(__fdiv_rn(fmaxf(n0, 0.5f), n));
                            const float l1 = log2f(__fdiv_rn(fmaxf(n1, 0.5f), n));
                            const float t = __fadd_rn(__fmul_rn(n0, l0), __fmul_rn(n1, l1));
                            bits = __fadd_rn(bits, __fadd_rn(-t, 2.f));
                        }
                    }
                    const float bytes = __fadd_rn(__fmul_rn(bits, 0.125f), 1.f);
                    if (p > 0) {
                        const float lim = __fmul_rn(slope, bytes);
                        const float dabs =
                            __fmul_rn(__fmul_rn(__fmul_rn((float)planeDist, exp2f((float)(2 * p))), 1.f / 4096.f), J.dscale);
                        if (dabs < lim) {
                            float e = 0.f;
                            const float step = exp2f((float)p);
                            for (int y = 0; y < h; ++y)
                                for (int x = 0; x < w; ++x) {
                                    const uint32_t m = mag[y][x] & 0x7FFFFFFFu;
                                    const float v = __fmul_rn((float)m, 1.f / 64.f);
                                    const uint32_t qq = m >> (p + kFracBits);
                                    const float rec = qq == 0 ? 0.f : __fmul_rn(__fadd_rn((float)qq, 0.5f), step);
                                    const float d = __fsub_rn(v, rec);
                                    e = __fadd_rn(e, __fmul_rn(d, d));
                                }
                            stop = __fmul_rn(e, J.dscale) < lim;
                        }
                    }
                }
                __syncwarp();
                if (lane < 19) hist[lane] = 0;
                stop = __shfl_sync(kFull, stop, 0);
            }
            symTotal += count;
            __syncwarp();
            if (stop) break;
        }
        if (lane == 0) {
            info[0] = (uint32_t)nbps;
            info[1] = (uint32_t)np;
            info[2] = symTotal;
            info[3] = 0;
            atomicAdd(P.ctl + 2, symTotal);
        }
        __syncwarp();
        return symTotal;
    }
}

__global__ void __launch_bounds__(CM_THREADS, 7) t1CmKernel(T1Launch P) {
    __shared__ __align__(16) uint32_t s_mag[CM_WARPS][32][32];  // 16-byte rows: filled by vector stores
    __shared__ __align__(16) uint8_t s_stage[CM_WARPS][STAGE];
    __shared__ uint8_t s_zk[4 * 256];
    __shared__ uint8_t s_sk[512];
    __shared__ uint32_t s_hist[CM_WARPS][19];
    cmTables(s_zk, s_sk);
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (uint32_t job = blockIdx.x * CM_WARPS + wid; job < P.n; job += gridDim.x * CM_WARPS)
        cmJob(P, job, s_mag[wid], s_stage[wid], s_hist[wid], s_zk, s_sk, lane);
}

// ---------------------------------------------------------------------------- ordering
__device__ __forceinline__ uint32_t orderBucket(uint32_t s) {
    // log-spaced classes, four per octave; the most decisions first
    if (s < 4) return ORDER_BUCKETS - 1;
    const uint32_t l = 31 - __clz(s);
    const uint32_t cls = min(4 * l + ((s >> (l - 2)) & 3u), (uint32_t)ORDER_BUCKETS - 1);
    return ORDER_BUCKETS - 1 - cls;
}

// Blocks with at least P.soloDecisions decisions are MQ-coded alone in a warp (its lane 0),
// at most one per warp for half the launch's warps: the longest serial chains, which would
// otherwise run beside 31 divergent neighbours. A power of two, so that they are exactly
// the first blocks of the order.
__global__ void __launch_bounds__(1024) t1OrderKernel(T1Launch P, uint32_t maxSolo) {
    __shared__ uint32_t hist[ORDER_BUCKETS];
    __shared__ uint32_t solo;
    for (int i = threadIdx.x; i < ORDER_BUCKETS; i += blockDim.x) hist[i] = 0;
    if (threadIdx.x == 0) solo = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < P.n; i += blockDim.x) {
        const uint32_t d = P.info[4 * (size_t)i + 2];
        atomicAdd(&hist[orderBucket(d)], 1u);
        if (d >= P.soloDecisions) atomicAdd(&solo, 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) P.ctl[3] = min(solo, maxSolo);
    if (threadIdx.x < 32) {
        // exclusive scan of 128 counters by one warp, four per lane
        const int lane = threadIdx.x;
        uint32_t v[4], s = 0;
        for (int k = 0; k < 4; ++k) {
            v[k] = hist[4 * lane + k];
            s += v[k];
        }
        const uint32_t incl = warpScan(s, lane);
        uint32_t run = incl - s;
        for (int k = 0; k < 4; ++k) {
            hist[4 * lane + k] = run;
            run += v[k];
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < P.n; i += blockDim.x)
        P.perm[atomicAdd(&hist[orderBucket(P.info[4 * (size_t)i + 2])], 1u)] = i;
}

// Words of a launch's work area the wide ordering uses (those of the persistent launch's
// solo count and bucket histogram: a launch is one or the other).
constexpr uint32_t kWSoloWide = 2, kWHistWide = 16;

// The same ordering over the whole GPU, for launches with a work area (the histogram and the
// solo count in its words kWHist / kWSolo, zeroed before): per-CTA histograms summed into
// the work area, one warp's exclusive scan of it, then a scatter through the bucket cursors.
// Blocks within a bucket land in any order, as in the one-CTA form (the order only decides
// which lane codes a block when, never its bytes).
__global__ void __launch_bounds__(256) t1OrderCountKernel(T1Launch P) {
    __shared__ uint32_t hist[ORDER_BUCKETS];
    __shared__ uint32_t solo;
    for (int i = threadIdx.x; i < ORDER_BUCKETS; i += blockDim.x) hist[i] = 0;
    if (threadIdx.x == 0) solo = 0;
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x) {
        const uint32_t d = P.info[4 * (size_t)i + 2];
        atomicAdd(&hist[orderBucket(d)], 1u);
        if (d >= P.soloDecisions) atomicAdd(&solo, 1u);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < ORDER_BUCKETS; b += blockDim.x)
        if (hist[b]) atomicAdd(P.work + kWHistWide + b, hist[b]);
    if (threadIdx.x == 0 && solo) atomicAdd(P.work + kWSoloWide, solo);
}

__global__ void __launch_bounds__(32) t1OrderScanKernel(T1Launch P, uint32_t maxSolo) {
    const int lane = threadIdx.x;
    uint32_t* hist = P.work + kWHistWide;
    uint32_t v[4], s = 0;
    for (int k = 0; k < 4; ++k) {
        v[k] = hist[4 * lane + k];
        s += v[k];
    }
    const uint32_t incl = warpScan(s, lane);
    uint32_t run = incl - s;
    for (int k = 0; k < 4; ++k) {
        hist[4 * lane + k] = run;
        run += v[k];
    }
    if (lane == 0) P.ctl[3] = min(P.work[kWSoloWide], maxSolo);
}

__global__ void __launch_bounds__(256) t1OrderScatterKernel(T1Launch P) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < P.n; i += gridDim.x * blockDim.x)
        P.perm[atomicAdd(P.work + kWHistWide + orderBucket(P.info[4 * (size_t)i + 2]), 1u)] = i;
}

// ---------------------------------------------------------------------------- MQ coding
// Context state word: Qe | MPS << 16 | state index << 17. nextStateEntry(k), k = state
// index << 2 | MPS << 1 | LPS: the state word after a renormalising decision; the coder keeps
// the two entries of each (state, MPS) side by side.
__device__ __forceinline__ uint32_t nextStateEntry(uint32_t k) {
    const uint32_t idx = k >> 2, mps = (k >> 1) & 1u, lps = k & 1u, e = c_mq[idx];
    const uint32_t nidx = lps ? (e >> 24) & 63u : (e >> 18) & 63u;
    const uint32_t nm = mps ^ (lps ? (e >> 17) & 1u : 0u);
    return (c_mq[nidx] & 0xFFFFu) | (nm << 16) | (nidx << 17);
}
__device__ __forceinline__ uint32_t initialState(uint32_t idx) { return (c_mq[idx] & 0xFFFFu) | (idx << 17); }

struct Coder {
    uint32_t A, C, B;
    int CT, bp;
    uint8_t* out;
    uint32_t cap;
    bool overflow;

    // Annex C BYTEOUT with its three cases as selects: after 0xFF a stuffed bit (7 bits
    // next); otherwise a carry into the pending byte, which may make it 0xFF.
    __device__ __forceinline__ void byteout() {
        const bool carry = B != 0xFFu && C >= 0x8000000u;
        B += carry ? 1u : 0u;
        C &= carry ? 0x7FFFFFFu : 0xFFFFFFFFu;
        const bool stuff = B == 0xFFu;
        if (bp >= 0) {
            if ((uint32_t)bp < cap) out[bp] = (uint8_t)B;
            else overflow = true;
        }
        ++bp;
        B = (C >> (stuff ? 20 : 19)) & 0xFFu;
        C &= stuff ? 0xFFFFFu : 0x7FFFFu;
        CT = stuff ? 7 : 8;
    }
    // One decision in context state t; returns the context's next state. Renormalisation
    // shifts by clz(A) - 16, which is 0 when A stayed at or above 0x8000; the byte-out is the
    // only branch. next[t >> 16] holds both successors of the state (after an MPS that
    // renormalises, after an LPS), so the load does not wait for the decision's outcome.
    __device__ __forceinline__ uint32_t encode(uint32_t t, uint32_t d, const uint2* next) {
        const uint2 succ = next[t >> 16];
        const uint32_t qe = t & 0xFFFFu;
        const uint32_t a = A - qe;
        const bool lps = ((d ^ (t >> 16)) & 1u) != 0;
        const bool upper = (a >= qe) != lps;  // which sub-interval the decision takes
        C += upper ? qe : 0u;
        A = upper ? a : qe;
        const bool rn = lps || !(a & 0x8000u);
        const uint32_t nt = lps ? succ.y : succ.x;
        int n = __clz(A) - 16;
        A <<= n;
        for (;;) {
            const int sh = min(n, CT);
            C <<= sh;
            CT -= sh;
            n -= sh;
            if (CT != 0) break;
            byteout();
            if (n == 0) break;
        }
        return rn ? nt : t;
    }
    __device__ __forceinline__ uint32_t flush() {
        const uint32_t tempc = C + A;
        C |= 0xFFFFu;
        if (C >= tempc) C -= 0x8000u;
        C <<= CT;
        byteout();
        C <<= CT;
        byteout();
        if (B != 0xFFu) {
            if ((uint32_t)bp < cap) out[bp] = (uint8_t)B;
            else overflow = true;
            return (uint32_t)(bp + 1);
        }
        return (uint32_t)bp;
    }
};

// Control words of a persistent launch (T1Launch::work, zeroed before it), then the
// order's bucket counters (offsets once scanned), then the list of blocks whose MQ coding
// is done, in the order they finished (block + 1; 0 = not yet written).
enum : uint32_t {
    kWCmHead = 0,      // next block to model
    kWCmDone = 1,      // blocks modelled
    kWSolo = 2,        // blocks of soloDecisions decisions or more
    kWScanDone = 3,    // the order's bucket offsets are ready
    kWScatHead = 4,    // next chunk of the order's scatter
    kWScatDone = 5,
    kWSoloHead = 6,    // next solo block to claim
    kWTruncTail = 7,   // entries in the list
    kWTruncHead = 8,   // next entry to take for truncation lengths
    kWHist = 16,
    kWList = 16 + ORDER_BUCKETS,
};
static_assert(kWList == kT1WorkHead, "work layout");
static_assert(kWSoloWide == kWSolo && kWHistWide == kWHist, "the wide ordering's words");

// Loads of what other warps of a persistent launch wrote during the launch, into lines an
// SM may have read before (the info words, MQ states and codewords that truncation reads)
// go around L1, which SMs do not keep coherent with one another; the separate kernels load
// normally.
template <bool PERS, class T>
__device__ __forceinline__ T ldx(const T* p) {
    if constexpr (PERS) return __ldcg(p);
    else return *p;
}

// Shortest prefix >= minLen that a decoder reading 1-bits past the end decodes exactly
// up to the snapshot, never ending on 0xFF. Same arithmetic as the oracle's mq_trunc.
template <bool PERS>
__device__ uint32_t truncLen(uint4 s, const uint8_t* buf, uint32_t len, uint32_t minLen) {
    const int bp = (int)s.x;
    const uint32_t C = s.y, A = s.z & 0xFFFFu, B = s.w;
    const int CT = (int)(s.z >> 16);
    const int base = 43 - CT;
    const unsigned long long low = ((unsigned long long)B << base) + ((unsigned long long)C << 16);
    const unsigned long long high = low + ((unsigned long long)A << 16);
    unsigned long long acc = 0;
    int used = 0;
    for (int i = bp; i < (int)len; ++i) {
        const uint32_t byte = i >= 0 ? ldx<PERS>(buf + i) : 0u;
        const int sh = base - used;
        if (sh < 0) break;
        acc += (unsigned long long)byte << sh;
        const unsigned long long tail = 1ull << sh;
        const uint32_t l = (uint32_t)(i + 1);
        if (l >= minLen && byte != 0xFFu && acc + tail <= high && acc + tail > low) return l;
        used += byte == 0xFFu ? 7 : 8;
    }
    return len;
}

__device__ __forceinline__ void mqTables(uint2* s_next, uint32_t* s_init) {
    for (int i = threadIdx.x; i < 2 * 47; i += blockDim.x)
        s_next[i] = make_uint2(nextStateEntry(2 * i), nextStateEntry(2 * i + 1));
    if (threadIdx.x == 0) {
        s_init[0] = initialState(0);
        s_init[1] = initialState(4);
        s_init[2] = initialState(3);
        s_init[3] = initialState(46);
    }
}

// MQ coding, a lane per block, until the queue is empty. ctx: the lane's 19 context states,
// CS words apart. warpId: the warp's place among the solo warps of a separate MQ launch.
// PERS (a persistent launch): the solo blocks go to the first warps to get here, and each
// block, coded or empty, is listed for its truncation lengths when it is done.
template <int CS, bool PERS>
__device__ __forceinline__ void mqRun(const T1Launch& P, uint32_t* ctx, const uint2* s_next, const uint32_t* s_init,
                                      uint32_t warpId) {
    uint32_t* status = P.ctl + 1;
    const int lane = threadIdx.x & 31;

    // Per-lane state of the block in hand. Invariant between decisions: s is the decision
    // at pos and t the state of its context; nxt holds the decisions from pos on.
    uint32_t job = 0, pos = 0, nsym = 0, np = 0, k = 0, nextEnd = 0, stop = 0, s = 0, t = 0;
    uint32_t laterEnd = 0;  // the pass end after nextEnd, loaded one pass ahead
    const uint8_t* sym = nullptr;
    uint4 nxt = make_uint4(0, 0, 0, 0);
    Coder e;
    e.cap = 0;
    bool have = false;

    auto listed = [&](uint32_t j) {
        if constexpr (PERS) {
            __threadfence();  // the block's results before its list entry
            const uint32_t slot = atomicAdd(P.work + kWTruncTail, 1u);
            atomicExch(P.work + kWList + slot, j + 1);
        }
    };
    // starts block j; false when it has no coding pass (nothing to code)
    auto begin = [&](uint32_t j) {
        job = j;
        np = ldx<false>(P.info + 4 * (size_t)job + 1);
        nsym = ldx<false>(P.info + 4 * (size_t)job + 2);
        if (np == 0) {
            P.info[4 * (size_t)job + 3] = 0;
            listed(job);
            return false;
        }
        const T1Job J = P.jobs[job];
        sym = J.sym;
        e.out = J.cw;
        e.cap = J.cap;
        e.A = 0x8000u;
        e.C = 0;
        e.CT = 12;
        e.bp = -1;
        e.B = 0;
        e.overflow = false;
        // initial states, Table D.7: ZC context 0 state 4, run-length 3, uniform 46
#pragma unroll
        for (int c = 0; c < 19; ++c) ctx[c * CS] = s_init[0];
        ctx[0] = s_init[1];
        ctx[17 * CS] = s_init[2];
        ctx[18 * CS] = s_init[3];
        pos = 0;
        k = 0;
        nextEnd = ldx<false>(P.passEnd + (size_t)job * kMaxPasses);
        laterEnd = np > 1 ? ldx<false>(P.passEnd + (size_t)job * kMaxPasses + 1) : 0xFFFFFFFFu;
        stop = min(nsym, nextEnd);
        nxt = nsym ? ldx<false>(reinterpret_cast<const uint4*>(sym)) : make_uint4(0, 0, 0, 0);
        s = nxt.x & 0xFFu;
        t = ctx[(s >> 1) * CS];
        have = true;
        return true;
    };

    // A solo warp first codes its solo block (perm[0 .. solo)) on its lane 0 while the other
    // lanes wait. Then the warp takes the next 32 blocks of the order at once, a lane each,
    // and codes them until the last of them is done: the order is largest first in narrow
    // size classes, so the 32 are about the same length, and the lanes start, run and end
    // their blocks together instead of each claiming its next block at its own time (which
    // left a third of the lanes of a warp idle at any moment).
    const uint32_t solo = ldx<false>(P.ctl + 3);
    uint32_t mine = warpId;
    if constexpr (PERS) {
        if (lane == 0) mine = atomicAdd(P.work + kWSoloHead, 1u);
        mine = __shfl_sync(kFull, mine, 0);
    }
    // end of the block in hand: remaining pass ends, flush, the codeword's length (the
    // truncation lengths are found afterwards, a warp per block)
    auto endBlock = [&] {
        while (k < np) {
            P.snaps[(size_t)job * kMaxPasses + k] = make_uint4((uint32_t)e.bp, e.C, e.A | ((uint32_t)e.CT << 16), e.B);
            ++k;
        }
        const uint32_t len = e.flush();
        if (e.overflow) atomicOr(status, kErrCodewordSpace);
        P.info[4 * (size_t)job + 3] = e.overflow ? 0u : len;
        listed(job);
        have = false;
    };
    // one aligned chunk of 16 decisions of the block in hand (fewer at its end)
    auto chunk = [&] {
        // one aligned chunk of 16 decisions (fewer at the block's end): a word of four
        // decisions unrolled at a time, the next decision's context state read ahead, off
        // the serial chain of the coder
        const uint4 v = nxt;
        nxt = (pos + 16 < nsym) ? ldx<false>(reinterpret_cast<const uint4*>(sym + pos + 16)) : make_uint4(0, 0, 0, 0);
        uint32_t w0 = v.x, w1 = v.y, w2 = v.z, w3 = v.w;
        const uint32_t w4 = nxt.x;
        // one decision: s (context and bit) in state t; sn the next decision
        auto one = [&](uint32_t sn) {
            // the byte past the block's last decision is not a decision: the clamp keeps its
            // look-ahead read inside the lane's 19 contexts
            const uint32_t cn = min(sn >> 1, 18u), cx = s >> 1;
            const uint32_t tn = ctx[cn * CS];
            const uint32_t tNew = e.encode(t, s & 1u, s_next);
            ctx[cx * CS] = tNew;
            t = cn == cx ? tNew : tn;
            s = sn;
            ++pos;
        };
        bool done = false;
#pragma unroll 1
        for (int q = 0; q < 4 && !done; ++q) {
            const uint32_t cur = w0;
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                if (pos >= stop) {
                    if (pos >= nsym) {
                        done = true;
                        break;
                    }
                    while (pos == nextEnd && k < np) {  // pass ends before this decision
                        P.snaps[(size_t)job * kMaxPasses + k] =
                            make_uint4((uint32_t)e.bp, e.C, e.A | ((uint32_t)e.CT << 16), e.B);
                        ++k;
                        nextEnd = laterEnd;  // loaded a pass ago: no wait here
                        laterEnd = k + 1 < np ? ldx<false>(P.passEnd + (size_t)job * kMaxPasses + k + 1) : 0xFFFFFFFFu;
                    }
                    stop = min(nsym, nextEnd);
                }
                one(b < 3 ? (cur >> (8 * (b + 1))) & 0xFFu : w1 & 0xFFu);
            }
            w0 = w1;
            w1 = w2;
            w2 = w3;
            w3 = w4;
        }
    };
    if (mine < solo) {  // warp-uniform
        if (lane == 0) have = begin(ldx<false>(P.perm + mine));
        while (__shfl_sync(kFull, (int)have, 0)) {
            if (lane == 0) {
                if (pos >= nsym) endBlock();
                else chunk();
            }
        }
    }
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(P.ctl, 32u);
        base = __shfl_sync(kFull, base, 0);
        if (solo + base >= P.n) break;  // warp-uniform
        const uint32_t qi = solo + base + lane;
        have = qi < P.n && begin(ldx<false>(P.perm + qi));
        while (__any_sync(kFull, have)) {
            if (have) {
                if (pos >= nsym) endBlock();
                else chunk();
            }
        }
    }
}

// MINB: CTAs per SM the registers must allow. A launch of a frame or two has fewer lanes
// than the GPU holds and runs uncapped; wide batched launches run at 10 CTAs per SM (the
// registers that allows need no spill; measured faster on B200 than 12 with a spill).
template <int MINB>
__global__ void __launch_bounds__(MQ_THREADS, MINB) t1MqKernel(T1Launch P) {
    __shared__ uint2 s_next[2 * 47];  // by (state, MPS): next state after an MPS renormalisation, after an LPS
    __shared__ uint32_t s_init[4];
    __shared__ uint32_t s_ctx[19 * MQ_THREADS];
    mqTables(s_next, s_init);
    __syncthreads();
    mqRun<MQ_THREADS, false>(P, s_ctx + threadIdx.x, s_next, s_init,
                             blockIdx.x * (MQ_THREADS / 32) + (threadIdx.x >> 5));
}

// Truncation lengths of one block by one warp: lane q finds the shortest prefix for pass q
// from the MQ state recorded at its end, as if no earlier pass constrained it; lane 0 then
// walks the passes in order and, where a pass's shortest prefix is shorter than an earlier
// pass's length, searches again from that length (the lengths of a block never decrease).
// The last pass takes the whole codeword.
template <bool PERS>
__device__ __forceinline__ void truncJob(const T1Launch& P, uint32_t job, int lane) {
    const uint32_t np = ldx<PERS>(P.info + 4 * (size_t)job + 1), len = ldx<PERS>(P.info + 4 * (size_t)job + 3);
    if (np == 0 || len == 0) return;  // nothing coded, or an overflow already reported
    const uint8_t* cw = P.jobs[job].cw;
    const size_t base = (size_t)job * kMaxPasses;
    uint32_t c0 = 0, c1 = 0;  // the unconstrained lengths of passes lane and lane + 32
    if ((uint32_t)lane + 1 < np) c0 = truncLen<PERS>(ldx<PERS>(P.snaps + base + lane), cw, len, 1);
    if ((uint32_t)lane + 33 < np) c1 = truncLen<PERS>(ldx<PERS>(P.snaps + base + lane + 32), cw, len, 1);
    uint32_t prev = 1, mine0 = 0, mine1 = 0;
    for (uint32_t q = 0; q < np; ++q) {
        const uint32_t c = __shfl_sync(kFull, q < 32 ? c0 : c1, q & 31);
        uint32_t L = len;
        if (q + 1 < np) {
            L = c;
            if (L < prev && lane == 0) L = truncLen<PERS>(ldx<PERS>(P.snaps + base + q), cw, len, prev);
            L = __shfl_sync(kFull, L, 0);
        }
        if ((q & 31) == (uint32_t)lane) (q < 32 ? mine0 : mine1) = L;
        prev = max(prev, L);
    }
    if ((uint32_t)lane < np) P.passLen[base + lane] = mine0;
    if ((uint32_t)lane + 32 < np) P.passLen[base + lane + 32] = mine1;
}

// Kept out of the MQ kernel, whose lanes would otherwise stall on these byte reads one
// block end at a time while their warp-mates code.
constexpr int TRUNC_THREADS = 256;

__global__ void __launch_bounds__(TRUNC_THREADS) t1TruncKernel(T1Launch P) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (TRUNC_THREADS / 32);
    for (uint32_t job = blockIdx.x * (TRUNC_THREADS / 32) + (threadIdx.x >> 5); job < P.n; job += warps)
        truncJob<false>(P, job, lane);
}

// ---------------------------------------------------------------------------- one launch
__device__ __forceinline__ uint32_t ldAcquire(const uint32_t* p) {
    uint32_t x;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(x) : "l"(p) : "memory");
    return x;
}

__device__ __forceinline__ uint32_t ldRelaxed(const uint32_t* p) {
    uint32_t x;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(x) : "l"(p) : "memory");
    return x;
}

constexpr uint64_t kQueueWaitNs = 2000000000ull;  // a persistent launch's longest wait

// Waits until *p >= v (polling with relaxed loads, backing off from 0.25 to 8 us so that
// thousands of waiting warps leave L2 to the working ones; the caller acquires once it
// holds); gives up after limitNs (2 s in the launches) with kErrQueueWait set, so that a
// launch whose other warps stopped returns.
__device__ bool waitFor(const uint32_t* p, uint32_t v, uint32_t* status, uint64_t limitNs = kQueueWaitNs) {
    uint64_t t0, t1;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    uint32_t nap = 256;
    for (uint32_t it = 0; it < (1u << 26); ++it) {
        if (ldRelaxed(p) >= v) return true;
        __nanosleep(nap);
        nap = min(nap * 2, 8192u);
        if ((it & 63u) == 63u) {
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
            if (t1 - t0 > limitNs) break;
        }
    }
    atomicOr(status, kErrQueueWait);
    return false;
}

// Lane 0 waits until *p >= v, then every lane makes its own acquire load of *p: the memory
// model orders later loads after the writes that preceded the release only for the thread
// that performs the acquire, not for lanes that hear of the value from lane 0 by shuffle.
// Returns *p as every lane read it, 0 when the wait gave up (warp-uniform).
__device__ __forceinline__ uint32_t warpWaitFor(const uint32_t* p, uint32_t v, uint32_t* status, int lane,
                                                uint64_t limitNs = kQueueWaitNs) {
    const bool ok = lane == 0 ? waitFor(p, v, status, limitNs) : true;
    if (!__shfl_sync(kFull, ok, 0)) return 0u;
    return ldAcquire(p);
}

constexpr uint32_t SCAT_CHUNK = 256;  // blocks per claim of the order's scatter

// The whole Tier-1 stage in one launch, every warp through the same phases, each fed by a
// device queue: (1) context modelling, a block per claim; (2) the order (counting sort by
// decision count, most first: the warp that models the last block scans the bucket
// counters the modelling filled, every warp scatters chunks of blocks); (3) MQ coding, a
// lane per block, the heaviest blocks alone in the first warps to arrive; (4) truncation
// lengths, a warp per block in the order the blocks finished MQ coding, by every warp done
// with MQ coding. A warp waits only for work that a running warp has claimed (it reaches
// the wait after the queue it drew from ran dry), so the launch cannot deadlock whatever
// its grid and whatever runs beside it; every wait is bounded all the same. A lane reads
// what other warps wrote only after its own acquire load of the word that announced it.
// Each warp's context-modelling memory holds its lanes' MQ contexts afterwards.
__global__ void __launch_bounds__(CM_THREADS, 7) t1PersistentKernel(T1Launch P, uint32_t maxSolo) {
    struct WarpCm {
        uint32_t mag[32][32];
        uint8_t stage[STAGE];
    };
    union WarpMem {
        WarpCm cm;
        uint32_t ctx[19 * 32];
    };
    __shared__ __align__(16) WarpMem s_w[CM_WARPS];
    __shared__ uint8_t s_zk[4 * 256];
    __shared__ uint8_t s_sk[512];
    __shared__ uint32_t s_hist[CM_WARPS][19];
    __shared__ uint2 s_next[2 * 47];
    __shared__ uint32_t s_init[4];
    cmTables(s_zk, s_sk);
    mqTables(s_next, s_init);
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t* work = P.work;
    uint32_t* status = P.ctl + 1;

    // (1) context modelling
    for (;;) {
        uint32_t job = 0;
        if (lane == 0) job = atomicAdd(work + kWCmHead, 1u);
        job = __shfl_sync(kFull, job, 0);
        if (job >= P.n) break;
        const uint32_t nsym = cmJob(P, job, s_w[wid].cm.mag, s_w[wid].cm.stage, s_hist[wid], s_zk, s_sk, lane);
        if (lane == 0) {
            atomicAdd(work + kWHist + orderBucket(nsym), 1u);
            if (nsym >= P.soloDecisions) atomicAdd(work + kWSolo, 1u);
        }
        __threadfence();  // the block's decisions and tables before it counts as done
        __syncwarp();
        uint32_t done = 0;
        if (lane == 0) done = atomicAdd(work + kWCmDone, 1u);
        // (2) the order: bucket offsets by the warp that modelled the last block
        if (__shfl_sync(kFull, done, 0) != P.n - 1) continue;
        ldAcquire(work + kWCmDone);
        uint32_t v[4], sum = 0;
        for (int q = 0; q < 4; ++q) {
            v[q] = __ldcg(work + kWHist + 4 * lane + q);
            sum += v[q];
        }
        uint32_t run = warpScan(sum, lane) - sum;
        for (int q = 0; q < 4; ++q) {
            work[kWHist + 4 * lane + q] = run;
            run += v[q];
        }
        if (lane == 0) P.ctl[3] = min(__ldcg(work + kWSolo), maxSolo);
        __threadfence();
        __syncwarp();
        if (lane == 0) atomicExch(work + kWScanDone, 1u);
    }
    if (!warpWaitFor(work + kWScanDone, 1u, status, lane)) return;
    const uint32_t chunks = divUp(P.n, SCAT_CHUNK);
    for (;;) {
        uint32_t c = 0;
        if (lane == 0) c = atomicAdd(work + kWScatHead, 1u);
        c = __shfl_sync(kFull, c, 0);
        if (c >= chunks) break;
        const uint32_t end = min(P.n, (c + 1) * SCAT_CHUNK);
        for (uint32_t i = c * SCAT_CHUNK + lane; i < end; i += 32)
            P.perm[atomicAdd(work + kWHist + orderBucket(__ldcg(P.info + 4 * (size_t)i + 2)), 1u)] = i;
        __threadfence();
        __syncwarp();
        if (lane == 0) atomicAdd(work + kWScatDone, 1u);
    }
    if (!warpWaitFor(work + kWScatDone, chunks, status, lane)) return;
    // (3) MQ coding, the lanes' contexts in the warp's modelling memory
    __syncwarp();
    mqRun<32, true>(P, s_w[wid].ctx + lane, s_next, s_init, 0);
    __syncwarp();
    // (4) truncation lengths, the list's entries in turn (an entry not yet written belongs
    // to a block whose MQ coding a running lane holds)
    for (;;) {
        uint32_t i = 0;
        if (lane == 0) i = atomicAdd(work + kWTruncHead, 1u);
        i = __shfl_sync(kFull, i, 0);
        if (i >= P.n) break;
        const uint32_t j = warpWaitFor(work + kWList + i, 1u, status, lane);
        if (j == 0) return;
        truncJob<true>(P, j - 1, lane);
    }
}

// One warp waits, as the persistent launch's warps wait, on a flag nothing sets: the
// failure-detection path of that launch (a partner warp that never announces its work)
// made to run out without a fault.
__global__ void waitSelftestKernel(const uint32_t* flag, uint32_t* status, uint64_t limitNs) {
    warpWaitFor(flag, 1u, status, (int)(threadIdx.x & 31), limitNs);
}

}  // namespace

uint32_t t1WaitSelftest(uint32_t limitMs, float* elapsedMs) {
    uint32_t* d = nullptr;  // [0] the flag, [1] the status word
    cudaEvent_t e[2] = {nullptr, nullptr};
    uint32_t h[2] = {0, 0};
    auto release = [&] {
        for (auto& x : e)
            if (x) cudaEventDestroy(x);
        if (d) cudaFree(d);
    };
    try {
        GB_CHECK(cudaMalloc(&d, 8));
        GB_CHECK(cudaMemset(d, 0, 8));
        for (auto& x : e) GB_CHECK(cudaEventCreate(&x));
        GB_CHECK(cudaEventRecord(e[0], 0));
        waitSelftestKernel<<<1, 32>>>(d, d + 1, (uint64_t)limitMs * 1000000ull);
        GB_CHECK(cudaGetLastError());
        GB_CHECK(cudaEventRecord(e[1], 0));
        GB_CHECK(cudaMemcpy(h, d, 8, cudaMemcpyDeviceToHost));
        if (elapsedMs) GB_CHECK(cudaEventElapsedTime(elapsedMs, e[0], e[1]));
    } catch (...) {
        release();
        throw;
    }
    release();
    return h[1];
}

cudaError_t kernelsLoadable() {
    cudaFuncAttributes attr;
    return cudaFuncGetAttributes(&attr, t1OrderKernel);
}

void t1Init() {
    uint8_t zc[4 * 45], sc[9];
    uint32_t mq[47];
    t1BuildTables(zc, sc, mq);
    GB_CHECK(cudaMemcpyToSymbol(c_zc, zc, sizeof zc));
    GB_CHECK(cudaMemcpyToSymbol(c_sc, sc, sizeof sc));
    GB_CHECK(cudaMemcpyToSymbol(c_mq, mq, sizeof mq));
}

// Resident CTAs per SM of the persistent kernel, queried once per device index (devices
// of different kinds in one process each get their own figure).
static int persistentOccupancy(int dev) {
    constexpr int kMaxDevices = 64;
    static std::mutex mutex;
    static int occ[kMaxDevices] = {};
    if (dev < 0 || dev >= kMaxDevices) dev = 0;
    std::lock_guard<std::mutex> lock(mutex);
    if (!occ[dev]) {
        int o = 0;
        GB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, t1PersistentKernel, CM_THREADS, 0));
        occ[dev] = max(o, 1);
    }
    return occ[dev];
}

void t1Encode(const T1Launch& launch, cudaStream_t st, cudaEvent_t* marks) {
    if (launch.n == 0) return;
    T1Launch L = launch;
    const Tuning def = defaultTuning();
    if (!L.soloDecisions) L.soloDecisions = def.soloDecisions;
    if (!L.cmCtasPerSm) L.cmCtasPerSm = (uint16_t)def.cmCtasPerSm;
    if (!L.mqCtasPerSm) L.mqCtasPerSm = (uint16_t)def.mqCtasPerSm;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (L.persistent && L.work) {
        // one CTA per resident slot (the kernel is correct with any grid; more would only wait)
        const int occ = persistentOccupancy(dev);
        const uint32_t grid = min(divUp(L.n, CM_WARPS), (uint32_t)(sms * occ));
        GB_CHECK(cudaMemsetAsync(L.work, 0, t1WorkWords(L.n) * 4, st));
        t1PersistentKernel<<<grid, CM_THREADS, 0, st>>>(L, grid * CM_WARPS / 2);
        GB_CHECK(cudaGetLastError());
        if (marks) {
            GB_CHECK(cudaEventRecord(marks[0], st));
            GB_CHECK(cudaEventRecord(marks[1], st));
        }
        return;
    }
    const uint32_t cmBlocks = min(divUp(L.n, CM_WARPS), (uint32_t)sms * L.cmCtasPerSm);
    t1CmKernel<<<cmBlocks, CM_THREADS, 0, st>>>(L);
    if (marks) GB_CHECK(cudaEventRecord(marks[0], st));
    // a wide (batched) launch gives each lane two blocks on average, so that lanes whose
    // blocks end early take more from the queue
    const bool wide = divUp(L.n, MQ_THREADS) > (uint32_t)sms * 4u;
    const uint32_t mqBlocks = min(divUp(L.n, MQ_THREADS * (wide ? 2u : 1u)), (uint32_t)sms * L.mqCtasPerSm);
    const uint32_t maxSolo = mqBlocks * (MQ_THREADS / 32) / 2;
    if (L.work) {  // over the whole GPU: a batch of frames has 100,000 blocks and more
        const uint32_t og = min(divUp(L.n, 256u), (uint32_t)sms * 2u);
        GB_CHECK(cudaMemsetAsync(L.work, 0, kT1WorkHead * 4, st));
        t1OrderCountKernel<<<og, 256, 0, st>>>(L);
        t1OrderScanKernel<<<1, 32, 0, st>>>(L, maxSolo);
        t1OrderScatterKernel<<<og, 256, 0, st>>>(L);
    } else {
        t1OrderKernel<<<1, 1024, 0, st>>>(L, maxSolo);
    }
    if (marks) GB_CHECK(cudaEventRecord(marks[1], st));
    if (!wide) t1MqKernel<1><<<mqBlocks, MQ_THREADS, 0, st>>>(L);
    else t1MqKernel<10><<<mqBlocks, MQ_THREADS, 0, st>>>(L);
    t1TruncKernel<<<min(divUp(L.n, (uint32_t)(TRUNC_THREADS / 32)), (uint32_t)sms * 8u), TRUNC_THREADS, 0, st>>>(L);
    GB_CHECK(cudaGetLastError());
}

}  // namespace gb
