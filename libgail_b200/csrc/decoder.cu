// Decoder on sm_100a: Tier-1 decoding with dequantisation, inverse 9/7 wavelet, inverse
// ICT and 12-bit packing.
//
// Tier-1 (decodeKernel): one code-block per warp at a time, decoded by its lane 0 (the
// decode's control flow depends on every decoded bit, so lanes of one warp decoding
// different blocks would only run one after another); up to 32 such warps per SM pull
// blocks from a device queue ordered longest codeword first (orderKernel), the heaviest
// on SMs of their own. A block's state is kept as row masks in shared memory
// (significance and sign for rows -1..32, coded-this-plane and refined); the scan visits
// only columns that have something to code (bit scans over candidate masks) with the rows
// above, at and below the sample in registers (one shared load per sample), zero-coding
// and sign contexts come from shared tables keyed by the neighbour bits, the refinement
// pass keeps its three contexts in registers, and the decoded words (sign, twice the
// magnitude plus the mid-point of the planes not decoded) are built in shared memory and
// written to the wavelet plane as floats (word * step / 2) when the block is done. The
// decoding lane is a serial chain of dependent instructions, so its length in
// instructions is its time, and the code is kept compact: the instruction cache holds it
// (the same loops unrolled to keep whole stripes in registers ran 1.6x slower). Untrusted
// input: bytes past the codeword read as 0xFF, a block whose bytes lie outside the
// codestream decodes as zero, and nothing outside the block's own samples is written.
//
// Inverse wavelet (invLevelKernel): per level, 64 x 64 output tiles with a 4-sample halo
// in the interleaved domain, rows then columns (the reference's order), whole-sample
// symmetric mirror at the edges. The last level carries the inverse ICT, the rounding
// and clamping to 12 bits and the interleaved 16-bit store.
//
// Semantics restated from Josephur/libgail core/t1_dec.cpp:45-179,
// kernels/mq_decoder.h:46-114, core/cpu_decode_backend.cpp:36-99 and
// core/dwt_cpu.cpp:96-133, 213-240; bit-identical to the CPU decoder.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <stdexcept>
#include <string>

#include "common.cuh"
#include "decoder.h"
#include "pool.h"
#include "t1_tables.h"
#include "tuning.h"

namespace gb {

namespace {

// One code-block per warp: its lane 0 decodes it (the decode of a block is a serial chain
// whose control flow depends on every decoded bit, so lanes of one warp decoding different
// blocks would run one after another anyway); up to 32 such warps per SM keep the
// schedulers busy.
constexpr int DEC_THREADS = 32;
constexpr int ORDER_BUCKETS = 128;

__constant__ uint8_t c_zc[4 * 45];
__constant__ uint8_t c_sc[9];
__constant__ uint32_t c_mq[47];

// Heavy blocks: the longest codewords, decoded on SMs of their own (at most four per SM, one
// per scheduler) instead of beside 31 other decoding warps, where a block of a thousand
// bytes or more takes the whole launch's time.
constexpr uint32_t kMaxReserveSms = 32;
constexpr uint32_t kMaxHeavy = 4 * kMaxReserveSms;
// Control words: [0] queue head, [1] status, [2] wanted blocks, [3] heavy blocks, [4] the
// wanted blocks' codeword bytes; from kCtlArrive a counter per reserved SM, from kCtlClaim a
// claim flag per heavy block.
constexpr uint32_t kCtlArrive = 16, kCtlClaim = kCtlArrive + kMaxReserveSms;
constexpr uint32_t kCtlWords = kCtlClaim + kMaxHeavy;

struct DecArgs {
    const uint8_t* bytes;
    uint64_t size;
    const GbCblkCode* codes;
    const DecBlock* blocks;
    uint32_t n;
    const float* half;  // per band: step / 2
    uint32_t* planes;   // float planes seen as words while decoding
    uint32_t W;
    uint32_t* perm;
    uint32_t* ctl;      // kCtlWords control words, zeroed before the launch
    uint32_t slots;     // the decode launch's warps
    uint32_t heavyPct;  // heavy: codeword bytes above heavyPct % of the mean per warp (0: none)
};

__device__ __forceinline__ uint32_t lenBucket(uint32_t len) {
    if (len < 4) return ORDER_BUCKETS - 1;
    const uint32_t l = 31 - __clz(len);
    return ORDER_BUCKETS - 1 - min(4 * l + ((len >> (l - 2)) & 3u), (uint32_t)ORDER_BUCKETS - 1);
}

__global__ void __launch_bounds__(1024) orderKernel(DecArgs a) {
    __shared__ uint32_t hist[ORDER_BUCKETS];
    __shared__ uint32_t total, bytes, heavy;
    for (int i = threadIdx.x; i < ORDER_BUCKETS; i += blockDim.x) hist[i] = 0;
    if (threadIdx.x == 0) total = bytes = heavy = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < a.n; i += blockDim.x)
        if (a.blocks[i].wanted) {
            const uint32_t len = a.codes[i].len;
            atomicAdd(&hist[lenBucket(len)], 1u);
            atomicAdd(&total, 1u);
            atomicAdd(&bytes, min(len, 1u << 20));
        }
    __syncthreads();
    // heavy blocks: above heavyPct % of the mean codeword bytes per decoding warp
    const uint64_t limit = (uint64_t)bytes * a.heavyPct / (100ull * max(a.slots, 1u));
    for (uint32_t i = threadIdx.x; i < a.n; i += blockDim.x)
        if (a.heavyPct && a.blocks[i].wanted && a.codes[i].len > limit) atomicAdd(&heavy, 1u);
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int b = 0; b < ORDER_BUCKETS; ++b) {
            const uint32_t c = hist[b];
            hist[b] = run;
            run += c;
        }
        a.ctl[2] = total;
        a.ctl[4] = bytes;
    }
    __syncthreads();
    if (threadIdx.x == 0) a.ctl[3] = min(heavy, kMaxHeavy);  // the first ones of the order
    for (uint32_t i = threadIdx.x; i < a.n; i += blockDim.x)
        if (a.blocks[i].wanted) a.perm[atomicAdd(&hist[lenBucket(a.codes[i].len)], 1u)] = i;
}

// A block's first kCwCache codeword bytes are copied into shared memory before it is decoded.
constexpr uint32_t kCwCache = 2048;

// MQ decoder (ISO/IEC 15444-1 C.3) over one codeword; bytes past its end read as 0xFF. The
// first `cached` bytes come from the shared-memory copy, so that a byte-in on the serial chain
// does not wait for global memory.
struct MqDecoder {
    uint32_t A, C, bp, end, cached;
    int CT;
    const uint8_t* in;
    const uint8_t* cache;

    __device__ __forceinline__ uint32_t at(uint32_t i) const {
        return i < cached ? (uint32_t)cache[i] : (i < end ? (uint32_t)in[i] : 0xFFu);
    }
    // The decision in context state t when it is its context's MPS, 0, with no renormalisation:
    // then only the interval changes (the context keeps its state), and it is made here; false
    // (nothing changed) otherwise.
    __device__ __forceinline__ bool fastZero(uint32_t t) {
        const uint32_t qe = t & 0xFFFFu;
        if ((t >> 16) & 1u) return false;
        if ((C >> 16) < qe) return false;
        const uint32_t a = A - qe;
        if (!(a & 0x8000u)) return false;
        A = a;
        C -= qe << 16;
        return true;
    }
    __device__ __forceinline__ void bytein() {
        const uint32_t b = at(bp), b1 = at(bp + 1);
        if (b == 0xFFu) {
            if (b1 > 0x8Fu) {  // a marker: not consumed, ones from here on
                C += 0xFF00u;
                CT = 8;
            } else {
                ++bp;
                C += b1 << 9;
                CT = 7;
            }
        } else {
            ++bp;
            C += b1 << 8;
            CT = 8;
        }
    }
    __device__ __forceinline__ void init(const uint8_t* data, uint32_t len, const uint8_t* copy, uint32_t copied) {
        in = data;
        end = len;
        cache = copy;
        cached = copied;
        bp = 0;
        C = at(0) << 16;
        bytein();
        C <<= 7;
        CT -= 7;
        A = 0x8000u;
    }
    __device__ __forceinline__ void renorm() {
        int n = __clz(A) - 16;
        if (n <= CT) {  // the usual case: the bits are already in C
            A <<= n;
            C <<= n;
            CT -= n;
            return;
        }
        do {
            if (CT == 0) bytein();
            const int s = min(n, CT);
            A <<= s;
            C <<= s;
            CT -= s;
            n -= s;
        } while (n > 0);
    }
    // One decision in the context whose state word t a register holds (updated in place).
    __device__ __forceinline__ uint32_t decodeIn(uint32_t& t, const uint32_t* tab) {
        const uint32_t qe = t & 0xFFFFu, mps = (t >> 16) & 1u;
        A -= qe;
        bool lps;
        if ((C >> 16) < qe) {
            lps = A >= qe;
            A = qe;
        } else {
            C -= qe << 16;
            if (A & 0x8000u) return mps;
            lps = A < qe;
        }
        const uint32_t nidx = lps ? (t >> 24) & 63u : (t >> 18) & 63u;
        const uint32_t nm = mps ^ (lps ? (t >> 17) & 1u : 0u);
        t = tab[nidx] | (nm << 16);
        renorm();
        return lps ? mps ^ 1u : mps;
    }
    // One decision in context cx (state word: table entry | mps << 16).
    __device__ __forceinline__ uint32_t decode(uint32_t* ctx, int cx, const uint32_t* tab) {
        uint32_t t = ctx[cx];
        const uint32_t qe = t & 0xFFFFu, mps = (t >> 16) & 1u;
        A -= qe;
        bool lps;
        if ((C >> 16) < qe) {
            lps = A >= qe;  // conditional exchange in the lower sub-interval
            A = qe;
        } else {
            C -= qe << 16;
            if (A & 0x8000u) return mps;
            lps = A < qe;
        }
        const uint32_t nidx = lps ? (t >> 24) & 63u : (t >> 18) & 63u;
        const uint32_t nm = mps ^ (lps ? (t >> 17) & 1u : 0u);
        ctx[cx] = tab[nidx] | (nm << 16);
        renorm();
        return lps ? mps ^ 1u : mps;
    }
};

__device__ __forceinline__ uint32_t bt(uint32_t m, int x) { return (m >> x) & 1u; }
// Row bits x-1, x, x+1 of a 32-column row mask at bits 0..2 (zero outside the block).
__device__ __forceinline__ uint32_t win3(uint32_t row, int x) { return __funnelshift_r(row << 1, row >> 31, x) & 7u; }
// Neighbour key of sample (x, row M) from the rows above (U) and below (D): bits 0-2 row
// above columns x-1..x+1, 3 and 5 same row columns x-1 and x+1, 6-8 row below.
__device__ __forceinline__ uint32_t nbKey(uint32_t U, uint32_t M, uint32_t D, int x) {
    return win3(U, x) | ((win3(M, x) & 5u) << 3) | (win3(D, x) << 6);
}

struct BlockCtx {
    uint32_t* sig;  // significance rows -1..32 at index y + 1
    uint32_t* sgn;  // sign rows, the same indexing
    uint32_t* words;  // the block's decoded words, 32 per row (shared memory)
    const uint8_t* zk;  // zero-coding context by neighbour key, this block's orientation
    const uint8_t* sk;  // sign context | xor bit << 5 by the sign key
    const uint32_t* tab;
    uint32_t* ctx;
    MqDecoder mq;

    // Sample (x, y) with significance rows U, M, D (y - 1, y, y + 1) has its first 1-bit
    // in plane p: decode its sign, set its significance (M too) and write sign, bit and
    // mid-point.
    __device__ __forceinline__ void becomeSig(uint32_t U, uint32_t& M, uint32_t D, int x, int y, int p) {
        const uint32_t GU = sgn[y], GM = sgn[y + 1], GD = sgn[y + 2];
        const uint32_t key = (win3(M, x) & 5u) | ((win3(GM, x) & 5u) << 1) | (bt(U, x) << 4) | (bt(GU, x) << 5) |
                             (bt(D, x) << 6) | (bt(GD, x) << 7);
        const uint32_t c = sk[key];
        const uint32_t neg = mq.decode(ctx, c & 31u, tab) ^ (c >> 5);
        M |= 1u << x;
        sig[y + 1] = M;
        sgn[y + 1] = GM | (neg << x);
        words[y * 32 + x] = (neg << 31) | (3u << p);
    }
};

__global__ void __launch_bounds__(DEC_THREADS) decodeKernel(DecArgs a) {
    // per block: significance and sign of rows -1..32, coded-this-plane and refined rows 0..31
    __shared__ uint32_t s_sig[34], s_sgn[34], s_vis[32], s_ref[32];
    // the block's decoded words (sign, twice the magnitude plus the mid-point of the planes
    // not decoded), kept here and turned into floats in the plane when the block is done:
    // each refinement updates its word, and a global read-modify-write per refinement put a
    // memory round trip on the decoder's serial chain. Only significant samples' words are
    // ever read, and each is written when its sample becomes significant.
    __shared__ uint32_t s_word[32 * 32];
    __shared__ uint32_t s_ctx[19];
    __shared__ uint32_t s_tab[48];
    __shared__ uint8_t s_cw[kCwCache];  // the block's codeword, its first kCwCache bytes
    __shared__ uint8_t s_zc[4 * 45], s_sc[16];
    // zero coding by orientation and neighbour key (nbKey); sign coding by the sign key:
    // bits 0/1 left neighbour significant/negative, 2/3 right, 4/5 above, 6/7 below
    __shared__ uint8_t s_zk[4 * 512], s_sk[256];
    for (int i = threadIdx.x; i < 47; i += blockDim.x) s_tab[i] = c_mq[i];
    for (int i = threadIdx.x; i < 4 * 45; i += blockDim.x) s_zc[i] = c_zc[i];
    if (threadIdx.x < 9) s_sc[threadIdx.x] = c_sc[threadIdx.x];
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * 512; i += blockDim.x) {
        const int o = i >> 9, k = i & 511;
        const int h = ((k >> 3) & 1) + ((k >> 5) & 1);
        const int v = ((k >> 1) & 1) + ((k >> 7) & 1);
        const int d = (k & 1) + ((k >> 2) & 1) + ((k >> 6) & 1) + ((k >> 8) & 1);
        s_zk[i] = s_zc[45 * o + h + 3 * v + 9 * d];
    }
    for (int k = threadIdx.x; k < 256; k += blockDim.x) {
        auto chi = [&](int bit) { return ((k >> bit) & 1) ? (((k >> (bit + 1)) & 1) ? -1 : 1) : 0; };
        const int hc = max(-1, min(1, chi(0) + chi(2)));
        const int vc = max(-1, min(1, chi(4) + chi(6)));
        s_sk[k] = s_sc[(hc + 1) * 3 + (vc + 1)];
    }
    __syncthreads();
    const uint32_t lane = threadIdx.x;
    BlockCtx b;
    b.sig = s_sig;
    b.sgn = s_sgn;
    b.sk = s_sk;
    b.tab = s_tab;
    b.ctx = s_ctx;
    const uint32_t count = a.ctl[2], heavy = a.ctl[3];
    auto decodeBlock = [&](uint32_t j) {
        const DecBlock blk = a.blocks[j];
        const GbCblkCode code = a.codes[j];
        const int w = blk.w, h = blk.h;
        uint32_t* out = a.planes + blk.dst;  // zeroed before the launch: only significant samples are written
        const int nbps = code.nbps;
        const bool valid = code.passes > 0 && nbps >= 1 && nbps <= 30 && (uint64_t)code.offset + code.len <= a.size;
        if (!valid) return;
        b.words = s_word;
        b.zk = s_zk + 512 * blk.orient;
        for (int i = 0; i < 34; ++i) s_sig[i] = s_sgn[i] = 0;
        for (int i = 0; i < 32; ++i) s_vis[i] = s_ref[i] = 0;
        for (int c = 0; c < 19; ++c) s_ctx[c] = s_tab[0];
        s_ctx[0] = s_tab[4];
        s_ctx[17] = s_tab[3];
        s_ctx[18] = s_tab[46];
        b.mq.init(a.bytes + code.offset, code.len, s_cw, min(code.len, kCwCache));
        const uint32_t wmask = w >= 32 ? 0xFFFFFFFFu : (1u << w) - 1u;
        int done = 0;
        const int passes = code.passes;
        for (int p = nbps - 1; p >= 0 && done < passes; --p) {
            for (int type = (p == nbps - 1 ? 2 : 0); type < 3 && done < passes; ++type, ++done) {
                // the refinement pass keeps its three contexts (14-16) in registers
                uint32_t t14 = 0, t15 = 0, t16 = 0;
                if (type == 1) {
                    t14 = s_ctx[14];
                    t15 = s_ctx[15];
                    t16 = s_ctx[16];
                }
                // stripes of four rows from y0; rows y0-1..y0+4 lie in -1..32 (y0 <= 28) and
                // rows at or past h are zero. Each column is scanned top to bottom with the
                // rows above, at and below the sample in U, M, D.
                for (int y0 = 0; y0 < h; y0 += 4) {
                    const int n = min(4, h - y0);
                    if (type == 0) {  // significance propagation
                        uint32_t cm = 0;
                        for (int k = 0; k < n; ++k) {
                            const uint32_t U = s_sig[y0 + k], M = s_sig[y0 + k + 1], D = s_sig[y0 + k + 2];
                            cm |= (U | (U << 1) | (U >> 1) | (M << 1) | (M >> 1) | D | (D << 1) | (D >> 1)) & ~M;
                        }
                        cm &= wmask;
                        while (cm) {
                            const int x = __ffs(cm) - 1;
                            cm &= cm - 1;
                            uint32_t U = s_sig[y0], M = s_sig[y0 + 1];
                            for (int k = 0; k < n; ++k) {
                                const int y = y0 + k;
                                const uint32_t D = s_sig[y + 2];
                                if (!bt(M, x)) {
                                    const uint32_t key = nbKey(U, M, D, x);
                                    if (key) {
                                        const uint32_t bit = b.mq.decode(s_ctx, b.zk[key], s_tab);
                                        s_vis[y] |= 1u << x;
                                        if (bit) {
                                            b.becomeSig(U, M, D, x, y, p);
                                            cm |= (2u << x) & wmask;  // the next column may now be eligible
                                        }
                                    }
                                }
                                U = M;
                                M = D;
                            }
                        }
                    } else if (type == 1) {  // magnitude refinement
                        // nothing changes significance in this pass, so every sample's context
                        // is known before it: per row of the stripe, the samples to refine
                        // (significant before this plane, not coded in it), those refined
                        // before (context 16) and those with a significant neighbour (15,
                        // else 14); per column their four rows as nibbles
                        uint32_t e4[4] = {0, 0, 0, 0}, r4[4] = {0, 0, 0, 0}, n4[4] = {0, 0, 0, 0};
                        uint32_t cm = 0;
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            if (k >= n) break;
                            const uint32_t U = s_sig[y0 + k], M = s_sig[y0 + k + 1], D = s_sig[y0 + k + 2];
                            e4[k] = M & ~s_vis[y0 + k];
                            r4[k] = s_ref[y0 + k];
                            n4[k] = U | (U << 1) | (U >> 1) | (M << 1) | (M >> 1) | D | (D << 1) | (D >> 1);
                            cm |= e4[k];
                        }
                        while (cm) {
                            const int x = __ffs(cm) - 1;
                            cm &= cm - 1;
                            const uint32_t ec = bt(e4[0], x) | bt(e4[1], x) << 1 | bt(e4[2], x) << 2 | bt(e4[3], x) << 3;
                            const uint32_t rc = bt(r4[0], x) | bt(r4[1], x) << 1 | bt(r4[2], x) << 2 | bt(r4[3], x) << 3;
                            const uint32_t nc = bt(n4[0], x) | bt(n4[1], x) << 1 | bt(n4[2], x) << 2 | bt(n4[3], x) << 3;
                            for (uint32_t m = ec; m; m &= m - 1) {
                                const int k = __ffs(m) - 1;
                                const bool c16 = bt(rc, k), c15 = bt(nc, k);
                                uint32_t t = c16 ? t16 : (c15 ? t15 : t14);
                                const uint32_t bit = b.mq.decodeIn(t, s_tab);
                                if (c16) t16 = t;
                                else if (c15) t15 = t;
                                else t14 = t;
                                uint32_t& word = s_word[(y0 + k) * 32 + x];
                                word = bit ? word + (1u << p) : word - (1u << p);
                            }
                        }
                        // every sample refined here counts as refined from now on
#pragma unroll
                        for (int k = 0; k < 4; ++k)
                            if (k < n) s_ref[y0 + k] = r4[k] | e4[k];
                    } else {  // cleanup, with run-length coding of quiet columns
                        uint32_t cm = 0, any = s_sig[y0], vis = 0;
                        for (int k = 0; k < n; ++k) {
                            const uint32_t M = s_sig[y0 + k + 1], V = s_vis[y0 + k];
                            cm |= ~M & ~V;
                            any |= M;
                            vis |= V;
                        }
                        any |= s_sig[y0 + n + 1];
                        cm &= wmask;
                        while (cm) {
                            int x = __ffs(cm) - 1;
                            if (n == 4) {
                                // quiet columns whose run-length decision is a 0 that is its
                                // context's MPS and needs no renormalisation: nothing in them,
                                // and only the interval changes
                                const uint32_t t17 = s_ctx[17];
                                while (!win3(any, x) && !bt(vis, x) && b.mq.fastZero(t17)) {
                                    cm &= cm - 1;
                                    if (!cm) break;
                                    x = __ffs(cm) - 1;
                                }
                                if (!cm) break;
                            }
                            cm &= cm - 1;
                            int r = 0;
                            // quiet column: nothing significant in rows y0-1..y0+4 around it and
                            // nothing coded in this plane in it
                            if (n == 4 && !win3(any, x) && !bt(vis, x)) {
                                if (!b.mq.decode(s_ctx, 17, s_tab)) continue;
                                int first = (int)b.mq.decode(s_ctx, 18, s_tab) << 1;
                                first |= (int)b.mq.decode(s_ctx, 18, s_tab);
                                uint32_t M = s_sig[y0 + first + 1];
                                b.becomeSig(s_sig[y0 + first], M, s_sig[y0 + first + 2], x, y0 + first, p);
                                any |= 1u << x;
                                r = first + 1;
                            }
                            uint32_t U = s_sig[y0 + r], M = s_sig[y0 + r + 1];
                            for (int k = r; k < n; ++k) {
                                const int y = y0 + k;
                                const uint32_t D = s_sig[y + 2];
                                if (!bt(M | s_vis[y], x)) {
                                    const uint32_t bit = b.mq.decode(s_ctx, b.zk[nbKey(U, M, D, x)], s_tab);
                                    if (bit) {
                                        b.becomeSig(U, M, D, x, y, p);
                                        any |= 1u << x;
                                    }
                                }
                                U = M;
                                M = D;
                            }
                        }
                    }
                }
                if (type == 1) {
                    s_ctx[14] = t14;
                    s_ctx[15] = t15;
                    s_ctx[16] = t16;
                }
            }
            for (int i = 0; i < 32; ++i) s_vis[i] = 0;
        }
        // dequantise into the plane, the significant samples only (every other sample
        // is 0, which is 0.0f): word * step / 2, sign from bit 31
        const float half = a.half[blk.band];
        float* f = reinterpret_cast<float*>(out);
        for (int y = 0; y < h; ++y)
            for (uint32_t m = s_sig[y + 1] & wmask; m; m &= m - 1) {
                const int x = __ffs(m) - 1;
                const uint32_t v = s_word[y * 32 + x];
                const float mag = (float)(v & 0x7FFFFFFFu) * half;
                f[(size_t)y * a.W + x] = (v & 0x80000000u) ? -mag : mag;
            }
    };

    // Every lane stays: lane 0 picks each block and decodes it, the others first copy its
    // codeword into shared memory with it. The heavy blocks (the first of the order): on a
    // reserved SM (%smid below the reserved count), the first four warps to arrive take one
    // each and every other warp leaves, so that the SM runs their serial chains alone; the
    // other warps take blocks from the queue, then any heavy block no reserved SM's warp took
    // (a grid that did not reach every reserved SM).
    uint32_t smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    const uint32_t reserved = (heavy + 3) / 4;
    int phase = smid < reserved ? 0 : 1;  // 0 reserved SM, 1 queue, 2 unclaimed heavy blocks, 3 done
    uint32_t fb = 0;
    for (;;) {
        uint32_t j = 0xFFFFFFFFu;
        if (lane == 0) {
            if (phase == 0) {
                const uint32_t k = atomicAdd(a.ctl + kCtlArrive + smid, 1u), hi = 4 * smid + k;
                if (k < 4 && hi < heavy && atomicExch(a.ctl + kCtlClaim + hi, 1u) == 0) j = a.perm[hi];
                phase = 3;
            } else if (phase == 1) {
                const uint32_t q = heavy + atomicAdd(a.ctl, 1u);  // longest codewords first
                if (q < count) j = a.perm[q];
                else phase = 2;
            }
            if (phase == 2) {
                while (fb < heavy && atomicExch(a.ctl + kCtlClaim + fb, 1u) != 0) ++fb;
                if (fb < heavy) j = a.perm[fb++];
                else phase = 3;
            }
        }
        j = __shfl_sync(kFull, j, 0);
        if (j == 0xFFFFFFFFu) break;
        const GbCblkCode code = a.codes[j];
        if ((uint64_t)code.offset + code.len <= a.size) {
            const uint8_t* src = a.bytes + code.offset;
            for (uint32_t i = lane; i < min(code.len, kCwCache); i += 32) s_cw[i] = src[i];
        }
        __syncwarp();
        if (lane == 0) decodeBlock(j);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------- inverse DWT
constexpr int TS = 64, HALO = 4, TW = TS + 2 * HALO, TP = TW + 1;
constexpr int IV_THREADS = 256;
__constant__ float kUnlift[4] = {-(float)0.443506852043971, -(float)0.882911075530934, -(float)-0.052980118572961,
                              -(float)-1.586134342059924};  // -delta, -gamma, -beta, -alpha
constexpr float kK = (float)1.230174104914001;
constexpr float kInvK = (float)(1.0 / 1.230174104914001);

__device__ __forceinline__ int mirror(int i, int n) {
    if (n == 1) return 0;
    const int period = 2 * (n - 1);
    i %= period;
    if (i < 0) i += period;
    return i < n ? i : period - i;
}

struct InvArgs {
    int w, h;            // this level's output (interleaved) size
    int snx, sny;        // low-band sizes
    const float* A;      // Mallat planes (high bands of this level; LL too at the top level)
    uint64_t aComp;
    int aStride;
    const float* ll;     // LL of this level (the previous inverse output), or NULL: take it from A
    uint64_t llComp;
    int llStride;
    float* out;          // LL of the level below (interleaved), or NULL at the last level
    uint64_t outComp;
    int outStride;
    uint16_t* pix;       // last level: interleaved 12-bit X'Y'Z' output
    int shift;
};

__device__ __forceinline__ float coeffAt(const InvArgs& a, int comp, int gy, int gx) {
    const bool ly = !(gy & 1), lx = !(gx & 1);
    if (ly && lx) {
        if (a.ll) return a.ll[comp * a.llComp + (size_t)(gy >> 1) * a.llStride + (gx >> 1)];
        return a.A[comp * a.aComp + (size_t)(gy >> 1) * a.aStride + (gx >> 1)];
    }
    const int row = ly ? (gy >> 1) : a.sny + (gy >> 1), col = lx ? (gx >> 1) : a.snx + (gx >> 1);
    return a.A[comp * a.aComp + (size_t)row * a.aStride + col];
}

template <bool LAST>
__global__ void __launch_bounds__(IV_THREADS) invLevelKernel(InvArgs a) {
    extern __shared__ float smem[];
    constexpr int NC = LAST ? 3 : 1;
    const int tid = threadIdx.x, tx = blockIdx.x, ty = blockIdx.y;
    const int x0 = tx * TS - HALO, y0 = ty * TS - HALO;
    const int w = a.w, h = a.h;
    for (int k = 0; k < NC; ++k) {
        const int comp = LAST ? k : (int)blockIdx.z;
        float* t = smem + k * TW * TP;
        for (int idx = tid; idx < TW * TW; idx += IV_THREADS) {
            const int ly = idx / TW, lx = idx % TW;
            t[ly * TP + lx] = coeffAt(a, comp, mirror(y0 + ly, h), mirror(x0 + lx, w));
        }
    }
    __syncthreads();
    for (int k = 0; k < NC; ++k) {
        float* t = smem + k * TW * TP;
        if (w >= 2) {  // rows: scale, then the lifting steps undone in reverse
            for (int idx = tid; idx < TW * TW; idx += IV_THREADS) {
                const int r = idx % TW, col = idx / TW;
                t[r * TP + col] *= (col & 1) ? kInvK : kK;
            }
            __syncthreads();
#pragma unroll 1
            for (int s = 0; s < 4; ++s) {
                const int first = (s & 1) ? 1 : 2;  // -delta, -beta: even; -gamma, -alpha: odd
                const float c = kUnlift[s];
                for (int idx = tid; idx < TW * 35; idx += IV_THREADS) {
                    const int r = idx % TW, i = first + 2 * (idx / TW);
                    float* x = t + r * TP + i;
                    x[0] += c * (x[-1] + x[1]);
                }
                __syncthreads();
            }
        }
        if (h >= 2) {  // then columns
            for (int idx = tid; idx < TW * TS; idx += IV_THREADS) {
                const int col = HALO + idx % TS, r = idx / TS;
                t[r * TP + col] *= (r & 1) ? kInvK : kK;
            }
            __syncthreads();
#pragma unroll 1
            for (int s = 0; s < 4; ++s) {
                const int first = (s & 1) ? 1 : 2;
                const float c = kUnlift[s];
                for (int idx = tid; idx < TS * 35; idx += IV_THREADS) {
                    const int col = HALO + idx % TS, i = first + 2 * (idx / TS);
                    float* x = t + i * TP + col;
                    x[0] += c * (x[-TP] + x[TP]);
                }
                __syncthreads();
            }
        }
    }
    for (int idx = tid; idx < TS * TS; idx += IV_THREADS) {
        const int ly = HALO + idx / TS, lx = HALO + idx % TS;
        const int gy = y0 + ly, gx = x0 + lx;
        if (gy >= h || gx >= w) continue;
        if (LAST) {
            const float y0v = smem[ly * TP + lx], y1v = smem[TW * TP + ly * TP + lx], y2v = smem[2 * TW * TP + ly * TP + lx];
            const float v[3] = {y0v + (float)1.402 * y2v, y0v + (float)(-0.34413) * y1v + (float)(-0.71414) * y2v,
                                y0v + (float)1.772 * y1v};
            uint16_t* o = a.pix + ((size_t)gy * w + gx) * 3;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const int code = (int)floorf(v[c] + 2048.5f);
                o[c] = (uint16_t)(min(max(code, 0), 4095) << a.shift);
            }
        } else {
            a.out[blockIdx.z * a.outComp + (size_t)gy * a.outStride + gx] = smem[ly * TP + lx];
        }
    }
}

// reduce == levels: the picture is the LL band as it is.
__global__ void colorOutKernel(const float* A, uint64_t comp, int stride, int w, int h, uint16_t* pix, int shift) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= w || y >= h) return;
    const size_t i = (size_t)y * stride + x;
    const float y0 = A[i], y1 = A[comp + i], y2 = A[2 * comp + i];
    const float v[3] = {y0 + (float)1.402 * y2, y0 + (float)(-0.34413) * y1 + (float)(-0.71414) * y2, y0 + (float)1.772 * y1};
    uint16_t* o = pix + ((size_t)y * w + x) * 3;
    for (int c = 0; c < 3; ++c) {
        const int code = (int)floorf(v[c] + 2048.5f);
        o[c] = (uint16_t)(min(max(code, 0), 4095) << shift);
    }
}

constexpr size_t kInvSmemLast = (size_t)3 * TW * TP * 4;
constexpr size_t kInvSmem = (size_t)TW * TP * 4;


}  // namespace

void decoderInit() {
    uint8_t zc[4 * 45], sc[9];
    uint32_t mq[47];
    t1BuildTables(zc, sc, mq);
    GB_CHECK(cudaMemcpyToSymbol(c_zc, zc, sizeof zc));
    GB_CHECK(cudaMemcpyToSymbol(c_sc, sc, sizeof sc));
    GB_CHECK(cudaMemcpyToSymbol(c_mq, mq, sizeof mq));
    GB_CHECK(cudaFuncSetAttribute(invLevelKernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kInvSmemLast));
}

uint64_t decoderSlotBytes(const Layout& L, const GailCudaDecodeSettings& s) {
    const uint64_t npix = (uint64_t)L.width * L.height, ll = (uint64_t)L.levelW(1) * L.levelH(1);
    const uint64_t out = (uint64_t)L.levelW(s.reduce) * L.levelH(s.reduce) * 6;
    return npix * 12 + 2 * ll * 12 + out + (uint64_t)L.numCblks() * (12 + 12 + 4) + (4ull << 20);
}

DecoderSlot::DecoderSlot(int device, const Layout& L, const GailCudaDecodeSettings& s, bool heavySms) : dev_(device), L_(L), s_(s) {
    heavySms_ = heavySms;
    if (s.reduce < 0 || s.reduce > L.levels) throw std::runtime_error("more resolution levels left out than the stream has");
    outW_ = L.levelW(s.reduce);
    outH_ = L.levelH(s.reduce);
    try {
        GB_CHECK(cudaSetDevice(dev_));
        GB_CHECK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
        for (auto& e : ev_) GB_CHECK(cudaEventCreate(&e));
        for (auto& e : bandEv_) GB_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        const uint64_t npix = (uint64_t)L.width * L.height, ll = (uint64_t)L.levelW(1) * L.levelH(1);
        const uint64_t n = (uint64_t)L.numCblks();
        auto alloc = [&](auto*& p, uint64_t bytes) {
            void* q = nullptr;
            check(cudaMalloc(&q, std::max<uint64_t>(bytes, 16)), "device memory for a decoder slot");
            allocs_.push_back(q);
            p = static_cast<std::remove_reference_t<decltype(p)>>(q);
        };
        alloc(dPlanes_, npix * 12);
        alloc(dLL_[0], ll * 12);
        alloc(dLL_[1], ll * 12);
        alloc(dHalf_, L.bands.size() * 4);
        alloc(dCodes_, n * sizeof(GbCblkCode));
        alloc(dBlocks_, n * sizeof(DecBlock));
        alloc(dPerm_, n * 4);
        alloc(dCtl_, kCtlWords * 4);
        alloc(dOut_, (uint64_t)outW_ * outH_ * 6);
        check(cudaHostAlloc((void**)&hOut_, std::max<uint64_t>(16, (uint64_t)outW_ * outH_ * 6), cudaHostAllocDefault),
              "pinned host memory");
        check(cudaHostAlloc((void**)&hCodes_, std::max<uint64_t>(16, n * sizeof(GbCblkCode)), cudaHostAllocDefault),
              "pinned host memory");
        check(cudaHostAlloc((void**)&hHalf_, L.bands.size() * 4 + 16, cudaHostAllocDefault), "pinned host memory");
        check(cudaHostAlloc((void**)&hCtl_, 64, cudaHostAllocDefault), "pinned host memory");
        capBytes_ = 1500000;
        alloc(dBytes_, capBytes_);
        check(cudaHostAlloc((void**)&hBytes_, capBytes_, cudaHostAllocDefault), "pinned host memory");
        std::vector<DecBlock> blocks(n);
        const int maxRes = L.levels - s.reduce;
        for (uint64_t i = 0; i < n; ++i) {
            const CodeBlock& cb = L.cblks[i];
            const GbSubband& b = L.bands[cb.band];
            blocks[i] = {(uint32_t)((uint64_t)b.comp * npix + (uint64_t)(b.py0 + cb.y0) * L.width + b.px0 + cb.x0),
                         (uint16_t)cb.w, (uint16_t)cb.h, (uint8_t)b.orient, (uint8_t)cb.band,
                         (uint8_t)(b.res <= maxRes ? 1 : 0), 0};
        }
        GB_CHECK(cudaMemcpy(dBlocks_, blocks.data(), n * sizeof(DecBlock), cudaMemcpyHostToDevice));
    } catch (...) {
        release();
        throw;
    }
}

DecoderSlot::~DecoderSlot() { release(); }

void DecoderSlot::release() {
    cudaSetDevice(dev_);
    if (st_) cudaStreamSynchronize(st_);
    for (void* p : allocs_) cudaFree(p);
    allocs_.clear();
    for (void* p : {(void*)hOut_, (void*)hCodes_, (void*)hHalf_, (void*)hCtl_, (void*)hBytes_})
        if (p) cudaFreeHost(p);
    hOut_ = nullptr;
    hCodes_ = nullptr;
    hHalf_ = nullptr;
    hCtl_ = nullptr;
    hBytes_ = nullptr;
    for (auto& e : ev_)
        if (e) {
            cudaEventDestroy(e);
            e = nullptr;
        }
    for (auto& e : bandEv_)
        if (e) {
            cudaEventDestroy(e);
            e = nullptr;
        }
    if (st_) cudaStreamDestroy(st_);
    st_ = nullptr;
    cudaGetLastError();
}

void DecoderSlot::decode(const Layout& frame, const uint8_t* data, size_t size, const GbCblkCode* blocks, size_t numBlocks,
                         void* dst, ptrdiff_t strideBytes, GailCudaDecodeTimings* tm) {
    const uint64_t rowBytes = (uint64_t)outW_ * 6;
    // page-locked caller rows (a serving layer's pinned buffers): the picture goes there
    // from the device directly
    cudaPointerAttributes at{};
    const bool pinned = cudaPointerGetAttributes(&at, dst) == cudaSuccess && at.type == cudaMemoryTypeHost &&
                        strideBytes >= (ptrdiff_t)rowBytes;
    cudaGetLastError();
    if (pinned) {
        enqueue(frame, data, size, blocks, numBlocks, tm && tm->wantWavelet, dst, strideBytes);
        finish(tm);
        return;
    }
    // pageable rows: the picture comes back in bands, and the host pool copies each band
    // into the caller's rows as soon as it has arrived, while the next bands are in flight
    // (52 MB at 4K: copied after the whole download it added its full time to the decode)
    enqueue(frame, data, size, blocks, numBlocks, tm && tm->wantWavelet, nullptr, 0, kBands);
    parallelFor(kBands, [&](int k) {
        GB_CHECK(cudaSetDevice(dev_));
        GB_CHECK(cudaEventSynchronize(bandEv_[k]));
        const int y0 = (int)((int64_t)outH_ * k / kBands), y1 = (int)((int64_t)outH_ * (k + 1) / kBands);
        const uint8_t* src = (const uint8_t*)hOut_ + (uint64_t)y0 * rowBytes;
        uint8_t* out = (uint8_t*)dst + (ptrdiff_t)y0 * strideBytes;
        if (strideBytes == (ptrdiff_t)rowBytes) {
            std::memcpy(out, src, rowBytes * (uint64_t)(y1 - y0));
        } else {
            for (int y = y0; y < y1; ++y, src += rowBytes, out += strideBytes) std::memcpy(out, src, rowBytes);
        }
    });
    finish(tm);
}

void DecoderSlot::enqueue(const Layout& frame, const uint8_t* data, size_t size, const GbCblkCode* blocks,
                          size_t numBlocks, bool wantWavelet, void* pinnedDst, ptrdiff_t dstStride, int bands) {
    if (bands < 1 || bands > kBands) throw std::logic_error("picture bands out of range");
    t0_ = std::chrono::steady_clock::now();
    if (frame.width != L_.width || frame.height != L_.height || frame.levels != L_.levels ||
        frame.bands.size() != L_.bands.size() || (int)numBlocks != L_.numCblks())
        throw std::logic_error("frame does not match the layout the slot was made for");
    if (size > 0xFFFFFFFFull) throw std::runtime_error("codestream too large");
    GB_CHECK(cudaSetDevice(dev_));
    const cudaStream_t st = st_;
    const uint64_t npix = (uint64_t)L_.width * L_.height, n = numBlocks;
    GB_CHECK(cudaStreamSynchronize(st));  // the slot's pinned buffers are free again
    if (size > capBytes_) {
        cudaFree(dBytes_);
        allocs_.erase(std::find(allocs_.begin(), allocs_.end(), (void*)dBytes_));
        cudaFreeHost(hBytes_);
        dBytes_ = nullptr;
        hBytes_ = nullptr;
        capBytes_ = size + size / 2;
        void* q = nullptr;
        check(cudaMalloc(&q, capBytes_), "device memory for a decoder slot");
        dBytes_ = (uint8_t*)q;
        allocs_.push_back(q);
        check(cudaHostAlloc((void**)&hBytes_, capBytes_, cudaHostAllocDefault), "pinned host memory");
    }
    std::memcpy(hBytes_, data, size);
    std::memcpy(hCodes_, blocks, n * sizeof(GbCblkCode));
    for (size_t i = 0; i < frame.bands.size(); ++i) hHalf_[i] = 0.5f * frame.bands[i].delta;
    wantWavelet_ = wantWavelet;

    GB_CHECK(cudaEventRecord(ev_[0], st));
    GB_CHECK(cudaMemcpyAsync(dBytes_, hBytes_, size, cudaMemcpyHostToDevice, st));
    GB_CHECK(cudaMemcpyAsync(dCodes_, hCodes_, n * sizeof(GbCblkCode), cudaMemcpyHostToDevice, st));
    GB_CHECK(cudaMemcpyAsync(dHalf_, hHalf_, frame.bands.size() * 4, cudaMemcpyHostToDevice, st));
    GB_CHECK(cudaMemsetAsync(dCtl_, 0, kCtlWords * 4, st));
    GB_CHECK(cudaMemsetAsync(dPlanes_, 0, npix * 12, st));  // coefficients of uncoded samples
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev_);
    const Tuning tu = tuningFor(L_.profile);
    const uint32_t grid = std::min<uint32_t>((uint32_t)n, (uint32_t)(sms * tu.decCtasPerSm));
    DecArgs da{dBytes_, size, dCodes_, dBlocks_, (uint32_t)n, dHalf_, (uint32_t*)dPlanes_, (uint32_t)L_.width, dPerm_, dCtl_,
               grid, heavySms_ ? (uint32_t)tu.decHeavyPct : 0u};
    orderKernel<<<1, 1024, 0, st>>>(da);
    decodeKernel<<<grid, DEC_THREADS, 0, st>>>(da);
    GB_CHECK(cudaGetLastError());
    GB_CHECK(cudaEventRecord(ev_[1], st));
    // inverse wavelet, levels top down; the last one writes the picture (the planes are only
    // read, so the wavelet tap can still be copied out after it)
    const int stop = s_.reduce;
    const int llStride = L_.levelW(1);
    const uint64_t llComp = (uint64_t)L_.levelW(1) * L_.levelH(1);
    const int shift = s_.highBits ? 4 : 0;
    if (stop == L_.levels) {
        colorOutKernel<<<dim3(divUp(outW_, 256), outH_), 256, 0, st>>>(dPlanes_, npix, L_.width, outW_, outH_, dOut_, shift);
    }
    for (int l = L_.levels; l > stop; --l) {
        InvArgs a{};
        a.w = L_.levelW(l - 1);
        a.h = L_.levelH(l - 1);
        a.snx = L_.levelW(l);
        a.sny = L_.levelH(l);
        a.A = dPlanes_;
        a.aComp = npix;
        a.aStride = L_.width;
        a.ll = l == L_.levels ? nullptr : dLL_[l & 1];
        a.llComp = llComp;
        a.llStride = llStride;
        const bool last = l - 1 == stop;
        a.out = last ? nullptr : dLL_[(l - 1) & 1];
        a.outComp = llComp;
        a.outStride = llStride;
        a.pix = dOut_;
        a.shift = shift;
        if (last)
            invLevelKernel<true><<<dim3(divUp(a.w, TS), divUp(a.h, TS), 1), IV_THREADS, kInvSmemLast, st>>>(a);
        else
            invLevelKernel<false><<<dim3(divUp(a.w, TS), divUp(a.h, TS), 3), IV_THREADS, kInvSmem, st>>>(a);
    }
    GB_CHECK(cudaGetLastError());
    GB_CHECK(cudaEventRecord(ev_[2], st));
    const uint64_t rowBytes = (uint64_t)outW_ * 6;
    if (pinnedDst) {
        GB_CHECK(cudaMemcpy2DAsync(pinnedDst, (size_t)dstStride, dOut_, rowBytes, rowBytes, (size_t)outH_,
                                   cudaMemcpyDeviceToHost, st));
    } else {
        for (int k = 0; k < bands; ++k) {
            const uint64_t y0 = (uint64_t)outH_ * k / bands, y1 = (uint64_t)outH_ * (k + 1) / bands;
            GB_CHECK(cudaMemcpyAsync((uint8_t*)hOut_ + y0 * rowBytes, (const uint8_t*)dOut_ + y0 * rowBytes,
                                     (y1 - y0) * rowBytes, cudaMemcpyDeviceToHost, st));
            if (bands > 1) GB_CHECK(cudaEventRecord(bandEv_[k], st));
        }
    }
    GB_CHECK(cudaMemcpyAsync(hCtl_, dCtl_, 64, cudaMemcpyDeviceToHost, st));
    GB_CHECK(cudaEventRecord(ev_[3], st));
}

const uint16_t* DecoderSlot::finish(GailCudaDecodeTimings* tm) {
    GB_CHECK(cudaSetDevice(dev_));
    GB_CHECK(cudaStreamSynchronize(st_));
    GB_CHECK(cudaGetLastError());
    const uint64_t npix = (uint64_t)L_.width * L_.height;
    if (wantWavelet_)
        for (int c = 0; c < 3; ++c) {
            wavelet_[c].resize(npix);
            GB_CHECK(cudaMemcpy(wavelet_[c].data(), dPlanes_ + c * npix, npix * 4, cudaMemcpyDeviceToHost));
        }
    if (tm) {
        float a = 0, b = 0, c = 0;
        cudaEventElapsedTime(&a, ev_[0], ev_[1]);
        cudaEventElapsedTime(&b, ev_[1], ev_[2]);
        cudaEventElapsedTime(&c, ev_[2], ev_[3]);
        tm->t1 = a;
        tm->dwt = b;
        tm->color = c;
        tm->total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0_).count();
        tm->numWavelet = wantWavelet_ ? npix : 0;
        for (int k = 0; k < 3; ++k) tm->wavelet[k] = wantWavelet_ ? wavelet_[k].data() : nullptr;
    }
    return hOut_;
}

}  // namespace gb
