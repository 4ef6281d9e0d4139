// Encoder front end: colour -> 9/7 DWT -> dead-zone quantisation, one kernel per level.
//
// Each CTA owns a tile of the level's input (64 x 64 by default; 128 x 64 or 64 x 128 by the
// tuning knobs dwtTile1 / dwtTileN), all three components at level 1, one later, and loads
// it with a 4-sample halo (whole-sample symmetric mirror at the image edges) into shared
// memory. It lifts the columns, then the rows (the order of the reference, Annex F.4.2):
// one thread per line, in registers, the four lifting steps applied in streaming order
// (alpha at j-1, beta at j-2, gamma at j-3, delta at j-4 as sample j arrives), which gives
// every sample the same operands as step-by-step lifting, so every tile shape gives the
// same coefficients. Then it writes the subband pieces it produced. Because tiles are
// 64-aligned, each piece is whole code-blocks of its band, so the high bands (and the LL
// band at the last level) are quantised in registers and stored straight into the
// code-block-major layout Tier-1 reads: 32 consecutive words per row, zero outside the
// band. The LL piece of an intermediate level goes to a float plane for the next level.
//
// Level 1 also does the colour conversion in its tile loads (the frame is read once,
// never written back as planes): R'G'B' from interleaved 16-bit or planar Y'CbCr,
// EOTF lookup, 3x3 to XYZ, the 12-bit DCI encoding as the count of 4096 host-built
// thresholds at or below the value (a fast power gives the first guess, the thresholds
// decide), DC shift and forward ICT. Two more routes are instantiations of their own, so
// the common one keeps its registers: the managed route puts a tone map (shoulder or
// BT.2390, on luminance, max(R,G,B) or each target channel) and a soft gamut compression
// between the 3x3 and the encoding; the LUT route maps R'G'B' through an application 3D
// LUT (trilinear) straight to codes.
//
// Float arithmetic is compiled without contraction and written in the reference's
// operation order (Josephur/libgail core/dwt_cpu.cpp:24-93, core/color.cpp:142-189,
// kernels/color_math.h:25-179, core/quant.h:20-25), so coefficients are bit-identical
// to the CPU path's; the managed route's powers are taken in double precision and rounded
// once to float, as the host's C library powf rounds them but for rare near-ties.
#include <cuda_runtime.h>

#include <stdexcept>

#include "common.cuh"
#include "frontend.cuh"

namespace gb {

namespace {

constexpr int HALO = 4;
// lifting coefficients alpha, beta, gamma, delta
__device__ __forceinline__ constexpr float liftCoef(int s) {
    return s == 0 ? (float)-1.586134342059924
                  : s == 1 ? (float)-0.052980118572961 : s == 2 ? (float)0.882911075530934 : (float)0.443506852043971;
}
constexpr float kLowScale = (float)(1.0 / 1.230174104914001);
constexpr float kHighScale = (float)1.230174104914001;

__device__ __forceinline__ int mirror(int i, int n) {
    if ((unsigned)i < (unsigned)n) return i;
    if (n == 1) return 0;
    const int period = 2 * (n - 1);
    i %= period;
    if (i < 0) i += period;
    return i < n ? i : period - i;
}

__device__ __forceinline__ uint32_t quantize(float v, float inv, uint32_t maxMag) {
    const float a = fabsf(v);
    const float q = a * inv * 64.0f;
    const uint32_t m = q >= (float)maxMag ? maxMag : (uint32_t)q;
    return m | ((v < 0.f && m >= 64u) ? 0x80000000u : 0u);
}

__device__ __forceinline__ float sampleAt(const void* src, int bits, size_t i) {
    return bits > 8 ? (float)((const uint16_t*)src)[i] : (float)((const uint8_t*)src)[i];
}

__device__ __forceinline__ uint32_t round16(float v) {
    const int r = (int)v;
    return (uint32_t)(r + ((v - (float)r) >= 0.5f ? 1 : 0));
}

__device__ __forceinline__ float clamp01(float v) { return fminf(fmaxf(v, 0.f), 1.f); }

// R'G'B' 16-bit codes of container pixel (x, y) of a planar frame (black outside the
// active picture).
__device__ void planarRgb(const void* src, const PlanarParams& p, int x, int y, uint32_t rgb[3]) {
    const int ax = x - p.ox, ay = y - p.oy;
    if (ax < 0 || ay < 0 || ax >= p.aw || ay >= p.ah) {
        rgb[0] = rgb[1] = rgb[2] = 0;
        return;
    }
    float cyp = !p.sy ? (float)ay : p.chroma == 2 ? ay * 0.5f : (ay - 0.5f) * 0.5f;
    cyp = fminf(fmaxf(cyp, 0.f), (float)(p.ch - 1));
    const int y0 = (int)cyp, y1 = min(y0 + 1, p.ch - 1);
    const float fy = cyp - y0;
    float cxp = !p.sx ? (float)ax : p.chroma == 1 ? (ax - 0.5f) * 0.5f : ax * 0.5f;
    cxp = fminf(fmaxf(cxp, 0.f), (float)(p.cw - 1));
    const int x0 = (int)cxp, x1 = min(x0 + 1, p.cw - 1);
    const float fx = cxp - x0;
    const size_t uOff = (size_t)p.aw * p.ah, vOff = uOff + (size_t)p.cw * p.ch;
    // all four neighbours of both chroma planes and the luma sample are loaded at once (x1,
    // y1 are in the plane); a weight of exactly zero multiplies a finite sample >= 0 to +0,
    // and adding +0 changes nothing, so the result is the interpolation's whatever the weights
    float s[9];
    {
        const size_t r0 = (size_t)y0 * p.cw, r1 = (size_t)y1 * p.cw;
        const size_t at[9] = {uOff + r0 + x0, uOff + r0 + x1, uOff + r1 + x0, uOff + r1 + x1,
                              vOff + r0 + x0, vOff + r0 + x1, vOff + r1 + x0, vOff + r1 + x1,
                              (size_t)ay * p.aw + ax};
#pragma unroll
        for (int i = 0; i < 9; ++i) s[i] = sampleAt(src, p.bits, at[i]);
    }
    float uv[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const float* q = s + 4 * k;
        const float top = q[0] * (1 - fx) + q[1] * fx;
        const float bot = q[2] * (1 - fx) + q[3] * fx;
        uv[k] = top * (1 - fy) + bot * fy;
    }
    float Y = s[8], U = uv[0], V = uv[1];
    float v[3];
    if (p.rgb) {  // planes G', B', R'
        v[0] = V / p.maxv;
        v[1] = Y / p.maxv;
        v[2] = U / p.maxv;
    } else {
        if (p.fullRange) {
            Y /= p.maxv;
            U = (U - 128.f * p.scale) / p.maxv;
            V = (V - 128.f * p.scale) / p.maxv;
        } else {
            Y = (Y - 16.f * p.scale) / (219.f * p.scale);
            U = (U - 128.f * p.scale) / (224.f * p.scale);
            V = (V - 128.f * p.scale) / (224.f * p.scale);
        }
        v[0] = Y + p.crR * V;
        v[1] = Y - p.cbG * U - p.crG * V;
        v[2] = Y + p.cbB * U;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) rgb[c] = round16(clamp01(v[c]) * 65535.f);
}

// 12-bit code: the number of thresholds at or below n (thr[0] = 0, thr ascending). A
// fast power gives a guess within a code or two; four neighbouring thresholds, loaded at
// once, decide among the guess and the codes either side of it, and a walk (then a binary
// search) takes the rare guess further off.
__device__ __noinline__ int dciCodeSearch(const float* __restrict__ thr, float n, int k) {
#pragma unroll 1
    for (int it = 0; it < 8; ++it) {
        if (k < 4095 && __ldg(thr + k + 1) <= n) {
            ++k;
        } else if (k > 0 && __ldg(thr + k) > n) {
            --k;
        } else {
            return k;
        }
    }
    k = 0;
#pragma unroll 1
    for (int step = 2048; step > 0; step >>= 1)
        if (k + step <= 4095 && __ldg(thr + k + step) <= n) k += step;
    return k;
}
__device__ __forceinline__ int dciCode(const float* __restrict__ thr, float n) {
    const int k = (int)(4095.f * __powf(n, 1.f / 2.6f) + 0.5f);
    const int b = min(max(k, 1), 4093);
    const float t0 = __ldg(thr + b - 1), t1 = __ldg(thr + b), t2 = __ldg(thr + b + 1), t3 = __ldg(thr + b + 2);
    if (t0 <= n && t3 > n) return b - 1 + (t1 <= n ? 1 : 0) + (t2 <= n ? 1 : 0);
    return dciCodeSearch(thr, n, b);
}

// ---- the managed and LUT routes (kernels/color_math.h:25-179) ----
// a power as the host's powf gives it: in double precision, rounded once to float
__device__ __forceinline__ float powHost(float a, float b) { return (float)pow((double)a, (double)b); }

// SMPTE ST 2084 constants (exact in float)
constexpr float kPqM1 = 2610.0f / 16384.0f, kPqM2 = 2523.0f / 4096.0f * 128.0f, kPqC1 = 3424.0f / 4096.0f,
                kPqC2 = 2413.0f / 4096.0f * 32.0f, kPqC3 = 2392.0f / 4096.0f * 32.0f;

__device__ float pqToNits(float e) {
    const float p = powHost(fminf(fmaxf(e, 0.0f), 1.0f), 1.0f / kPqM2);
    return 10000.0f * powHost(fmaxf(p - kPqC1, 0.0f) / (kPqC2 - kPqC3 * p), 1.0f / kPqM1);
}

__device__ float nitsToPq(float nits) {
    const float y = powHost(fminf(fmaxf(nits / 10000.0f, 0.0f), 1.0f), kPqM1);
    return powHost((kPqC1 + kPqC2 * y) / (1.0f + kPqC3 * y), kPqM2);
}

// Target luminance (cd/m^2) for source luminance y.
__device__ float toneCurve(const ToneParams& t, float y) {
    if (y <= 0.0f) return 0.0f;
    if (t.tone == 2) {
        // BT.2390 EETF: identity below the knee ks (in PQ relative to the source peak), a
        // Hermite segment from there to the target peak
        const float e1 = nitsToPq(y) / t.pqSrcMax;
        if (e1 < t.pqKs) return y;
        const float s = (fminf(e1, 1.0f) - t.pqKs) / (1.0f - t.pqKs);
        const float s2 = s * s, s3 = s2 * s;
        const float e2 = (2.0f * s3 - 3.0f * s2 + 1.0f) * t.pqKs + (s3 - 2.0f * s2 + s) * (1.0f - t.pqKs) +
                         (-2.0f * s3 + 3.0f * s2) * t.pqMaxLum;
        return pqToNits(e2 * t.pqSrcMax);
    }
    // shoulder: linear up to the knee, then an extended-Reinhard segment that meets the
    // target peak at the source peak
    float v = t.gain * y / t.srcRef;
    if (v > t.knee) {
        const float u = (v - t.knee) / (1.0f - t.knee);
        v = t.knee + (1.0f - t.knee) * fminf(u * (1.0f + u / (t.shoulderT * t.shoulderT)) / (1.0f + u), 1.0f);
    }
    return v * t.peak;
}

__device__ __forceinline__ void mul3(const float* A, float a, float b, float c, float o[3]) {
    o[0] = A[0] * a + A[1] * b + A[2] * c;
    o[1] = A[3] * a + A[4] * b + A[5] * c;
    o[2] = A[6] * a + A[7] * b + A[8] * c;
}

// Moves XYZ toward the neutral of the same luminance until every target channel is in
// [0, 1], compressing smoothly beyond gamutThresh of the way to the gamut edge.
__device__ void compressGamut(const ToneParams& t, float xyz[3]) {
    float c[3];
    mul3(t.toTarget, xyz[0], xyz[1], xyz[2], c);
    const float n = xyz[1] / t.peak;
    if (n >= 1.0f) {
        c[0] = c[1] = c[2] = 1.0f;
    } else {
        float amax = 1.0f, d[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            d[k] = c[k] - n;
            if (d[k] > 0.0f) amax = fminf(amax, (1.0f - n) / d[k]);
            if (d[k] < 0.0f) amax = fminf(amax, -n / d[k]);
        }
        const float dist = 1.0f / fmaxf(amax, 1e-6f), th = t.gamutThresh;
        float alpha = 1.0f;
        if (dist > th) {
            const float x = (dist - th) / (1.0f - th);
            const float y = x / (1.0f + x);
            alpha = (th + (1.0f - th) * y) / dist;
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) c[k] = n + alpha * d[k];
    }
    mul3(t.fromTarget, c[0], c[1], c[2], xyz);
}

// XYZ (cd/m^2) of linear R, G, B with the tone map and the gamut compression applied.
__device__ void managedXyz(const ColorArgs& c, float R, float G, float B, float xyz[3]) {
    mul3(c.m, R, G, B, xyz);
    const ToneParams& t = c.tone;
    if (t.tone != 0 && xyz[1] > 0.0f) {
        float tg[3];
        mul3(t.toTarget, xyz[0], xyz[1], xyz[2], tg);
        const float pk = t.peak;
        if (t.norm == 2) {
            // each target channel on its own; negative (out-of-gamut) channels scaled as the
            // brightest one is
            const float mx = fmaxf(tg[0], fmaxf(tg[1], tg[2])) * pk;
            const float sneg = mx > 0.0f ? toneCurve(t, mx) / mx : 1.0f;
#pragma unroll
            for (int k = 0; k < 3; ++k) tg[k] = tg[k] > 0.0f ? toneCurve(t, tg[k] * pk) / pk : tg[k] * sneg;
            mul3(t.fromTarget, tg[0], tg[1], tg[2], xyz);
        } else {
            const float m = t.norm == 1 ? fmaxf(xyz[1], fmaxf(tg[0], fmaxf(tg[1], tg[2])) * pk) : xyz[1];
            const float s = toneCurve(t, m) / m;
#pragma unroll
            for (int k = 0; k < 3; ++k) xyz[k] *= s;
        }
    }
    if (t.gamut) compressGamut(t, xyz);
}

// X'Y'Z' codes of 16-bit R'G'B' through the application 3D LUT.
__device__ void lutCodes(const ColorArgs& c, const uint32_t rgb[3], int code[3]) {
    const int n = c.lutN;
    const float top = (float)(n - 1);
    int i0[3];
    float w[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float f = fminf(fmaxf((float)rgb[k] / 65535.f, 0.0f), 1.0f) * top;
        i0[k] = min((int)f, n - 2);
        w[k] = f - (float)i0[k];
    }
    // the eight surrounding nodes, three floats each
    const float* q[2][2][2];
#pragma unroll
    for (int db = 0; db < 2; ++db)
#pragma unroll
        for (int dg = 0; dg < 2; ++dg)
#pragma unroll
            for (int dr = 0; dr < 2; ++dr)
                q[db][dg][dr] = c.lut3 + ((size_t)((i0[2] + db) * n + i0[1] + dg) * n + i0[0] + dr) * 3;
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        float e[2][2];
#pragma unroll
        for (int db = 0; db < 2; ++db)
#pragma unroll
            for (int dg = 0; dg < 2; ++dg)
                e[db][dg] = __ldg(q[db][dg][0] + ch) * (1.0f - w[0]) + __ldg(q[db][dg][1] + ch) * w[0];
        const float v = (e[0][0] * (1.0f - w[1]) + e[0][1] * w[1]) * (1.0f - w[2]) +
                        (e[1][0] * (1.0f - w[1]) + e[1][1] * w[1]) * w[2];
        code[ch] = (int)floorf(fminf(fmaxf(v, 0.0f), 1.0f) * 4095.0f + 0.5f);
    }
}

// The three 12-bit codes of a pixel by the route MODE (1 direct, 2 managed, 3 LUT).
template <int MODE>
__device__ __forceinline__ void pixelCodes(const ColorArgs& c, const uint32_t rgb[3], int code[3]) {
    if (MODE == 3) {
        lutCodes(c, rgb, code);
        return;
    }
    // the EOTF table index floor(clamp(code / 65535) * 65535 + 0.5) is the code
    // itself for every 16-bit code (checked exhaustively in float32)
    const float R = __ldg(c.eotf + rgb[0]), G = __ldg(c.eotf + rgb[1]), B = __ldg(c.eotf + rgb[2]);
    float xyz[3];
    if (MODE == 2) managedXyz(c, R, G, B, xyz);
    else mul3(c.m, R, G, B, xyz);
#pragma unroll
    for (int k = 0; k < 3; ++k) code[k] = dciCode(c.thr, clamp01(xyz[k] / 52.37f));
}

// Tile shapes (the knob dwtTile1 / dwtTileN): 0 = 64 x 64, 1 = 128 x 64 (wide), 2 = 64 x 128
// (tall) samples of the level's input, each with a 4-sample halo. A tile's band pieces
// are whole code-blocks: CBX x CBY of them per band.
template <int SHAPE>
struct Tile {
    static constexpr int X = SHAPE == 1 ? 128 : 64, Y = SHAPE == 2 ? 128 : 64;
    static constexpr int WX = X + 2 * HALO, WY = Y + 2 * HALO, P = WX + 1;  // P: row pitch
    static constexpr int CBX = X / 64, CBY = Y / 64;
};

// One line of N samples of a tile, `step` floats between samples: the four lifting steps
// (x[i] += c * (x[i-1] + x[i+1]) on odd 1..N-3, even 2..N-2, odd, even), then the scaling
// of the N - 8 samples the tile outputs, written back in place. Sample k is final once
// delta has passed k + 1, so it is stored five samples behind the loads.
template <int N>
__device__ __forceinline__ void liftLine(float* t, int step) {
    float x[N];
#pragma unroll
    for (int j = 0; j < N + 5; ++j) {
        if (j < N) x[j] = t[j * step];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const int i = j - 1 - s;
            const bool odd = !(s & 1);
            if (i >= (odd ? 1 : 2) && i <= (odd ? N - 3 : N - 2) && (i & 1) == (odd ? 1 : 0))
                x[i] = x[i] + liftCoef(s) * (x[i - 1] + x[i + 1]);
        }
        const int k = j - 5;
        if (k >= HALO && k < N - HALO) t[k * step] = x[k] * ((k & 1) ? kHighScale : kLowScale);
    }
}

// The tile's outputs for component comp: its code-blocks of each band (and LL floats).
template <int THREADS, int SHAPE>
__device__ void writeOutputs(const LevelArgs& a, const float* t, int comp, int tx, int ty, int tid) {
    using T = Tile<SHAPE>;
    if constexpr (T::CBX == 1 && T::CBY == 1) {  // the 64 x 64 tile
        // one 32 x 32 code-block per band: a thread keeps one column of the block (lane =
        // column, so the rows go out coalesced) and steps down its rows; the band's sample
        // (column i, row j of the block) sits at tile column HALO + 2 i + (o & 1) and row
        // HALO + 2 j + (o >> 1)
        static_assert(THREADS % 32 == 0, "whole warps");
        const int i = tid & 31;
        for (int o = 0; o < 4; ++o) {
            const BandOut& b = a.band[comp][o];
            if (tx >= b.ncbx || ty >= b.ncby) continue;
            const bool quant = o != 0 || a.last;
            const int bx = tx * 32 + i;
            const bool inx = bx < b.w;
            const float* col = t + (HALO + (o >> 1)) * T::P + HALO + 2 * i + (o & 1);
            uint32_t* blk = a.coeffs + ((size_t)b.cblkBase + (size_t)ty * b.ncbx + tx) * kCblkArea;
            for (int j = tid >> 5; j < 32; j += THREADS / 32) {
                const int by = ty * 32 + j;
                const bool in = inx && by < b.h;
                const float v = in ? col[2 * j * T::P] : 0.f;
                if (quant) {
                    blk[j * 32 + i] = in ? quantize(v, b.invDelta, b.maxMag) : 0u;
                    if (in && a.tap) a.tap[comp * a.tapComp + (size_t)(b.py0 + by) * a.tapStride + b.px0 + bx] = v;
                } else if (in) {
                    a.ll[comp * a.llComp + (size_t)by * a.llStride + bx] = v;
                }
            }
        }
    } else {
        const int x0 = tx * T::X - HALO, y0 = ty * T::Y - HALO;
        for (int o = 0; o < 4; ++o) {
            const BandOut& b = a.band[comp][o];
            const bool quant = o != 0 || a.last;
            for (int idx = tid; idx < T::CBX * T::CBY * kCblkArea; idx += THREADS) {
                const int cb = idx >> 10, e = idx & (kCblkArea - 1);
                const int cbx = tx * T::CBX + cb % T::CBX, cby = ty * T::CBY + cb / T::CBX;
                if (cbx >= b.ncbx || cby >= b.ncby) continue;
                const int i = e & 31, j = e >> 5;
                const int bx = cbx * 32 + i, by = cby * 32 + j;
                const bool in = bx < b.w && by < b.h;
                float v = 0.f;
                if (in) {
                    const int gx = 2 * bx + (o & 1), gy = 2 * by + (o >> 1);
                    v = t[(gy - y0) * T::P + (gx - x0)];
                }
                if (quant) {
                    uint32_t* blk = a.coeffs + ((size_t)b.cblkBase + (size_t)cby * b.ncbx + cbx) * kCblkArea;
                    blk[e] = in ? quantize(v, b.invDelta, b.maxMag) : 0u;
                    if (in && a.tap) a.tap[comp * a.tapComp + (size_t)(b.py0 + by) * a.tapStride + b.px0 + bx] = v;
                } else if (in) {
                    a.ll[comp * a.llComp + (size_t)by * a.llStride + bx] = v;
                }
            }
        }
    }
}

// Threads of a CTA: level 1 holds the three components of a tile, later levels one; enough
// for a thread per column of every component and per output row.
template <int MODE, int SHAPE>
__host__ __device__ constexpr int feThreads() {
    using T = Tile<SHAPE>;
    constexpr int nc = MODE ? 3 : 1;
    constexpr int need = (nc * T::WX > nc * T::Y ? nc * T::WX : nc * T::Y);
    constexpr int base = MODE ? 384 : 128;
    return ((need > base ? need : base) + 31) / 32 * 32;
}
template <int MODE, int SHAPE>
__host__ __device__ constexpr size_t feSmem() {
    using T = Tile<SHAPE>;
    return (size_t)(MODE ? 3 : 1) * T::WY * T::P * 4;
}
// CTAs per SM the launch bounds ask for: as many as the shared memory allows (up to 8).
template <int MODE, int SHAPE>
__host__ __device__ constexpr int feMinCtas() {
    constexpr size_t per = feSmem<MODE, SHAPE>() + 1024;
    constexpr int fit = (int)((size_t)227 * 1024 / per);
    constexpr int cap = MODE == 0 ? 8 : MODE == 1 ? 3 : 2;
    return fit < 1 ? 1 : (fit < cap ? fit : cap);
}

// MODE 0: a later level from the previous LL planes; 1..3: level 1 with the colour route
// of pixelCodes. SHAPE: the tile shape.
template <int MODE, int SHAPE>
__global__ void __launch_bounds__(feThreads<MODE, SHAPE>(), feMinCtas<MODE, SHAPE>())
    levelKernel(ColorArgs c, LevelArgs a) {
    extern __shared__ float smem[];
    using T = Tile<SHAPE>;
    constexpr bool COLOR = MODE != 0;
    constexpr int THREADS = feThreads<MODE, SHAPE>();
    constexpr int NC = COLOR ? 3 : 1;
    constexpr int PLANE = T::WY * T::P;
    const int tid = threadIdx.x, tx = blockIdx.x, ty = blockIdx.y;
    const int x0 = tx * T::X - HALO, y0 = ty * T::Y - HALO;
    const int w = a.w, h = a.h;
    if (COLOR) {
        for (int idx = tid; idx < T::WX * T::WY; idx += THREADS) {
            const int ly = idx / T::WX, lx = idx % T::WX;
            const int gy = mirror(y0 + ly, h), gx = mirror(x0 + lx, w);
            uint32_t rgb[3];
            if (c.kind == 0) {
                const uint16_t* p = (const uint16_t*)c.src + ((size_t)gy * w + gx) * 3;
                rgb[0] = p[0];
                rgb[1] = p[1];
                rgb[2] = p[2];
            } else {
                planarRgb(c.src, c.pp, gx, gy, rgb);
            }
            int code[3];
            pixelCodes<MODE>(c, rgb, code);
            const int cx = code[0], cy = code[1], cz = code[2];
            if (c.xyz && lx >= HALO && lx < HALO + T::X && ly >= HALO && ly < HALO + T::Y && x0 + lx < w &&
                y0 + ly < h) {
                uint16_t* o = c.xyz + ((size_t)(y0 + ly) * w + (x0 + lx)) * 3;
                o[0] = (uint16_t)cx;
                o[1] = (uint16_t)cy;
                o[2] = (uint16_t)cz;
            }
            const float fx = (float)(cx - 2048), fy = (float)(cy - 2048), fz = (float)(cz - 2048);
            smem[0 * PLANE + ly * T::P + lx] = (float)0.299 * fx + (float)0.587 * fy + (float)0.114 * fz;
            smem[1 * PLANE + ly * T::P + lx] = (float)(-0.16875) * fx + (float)(-0.33126) * fy + (float)0.5 * fz;
            smem[2 * PLANE + ly * T::P + lx] = (float)0.5 * fx + (float)(-0.41869) * fy + (float)(-0.08131) * fz;
        }
    } else {
        const float* src = a.src + blockIdx.z * a.srcComp;
        // a thread's loads of the tile, several in flight at once (the later levels' grids
        // are small: each CTA's load latency is most of its time)
#pragma unroll 4
        for (int idx = tid; idx < T::WX * T::WY; idx += THREADS) {
            const int ly = idx / T::WX, lx = idx % T::WX;
            smem[ly * T::P + lx] = __ldg(src + (size_t)mirror(y0 + ly, h) * a.srcStride + mirror(x0 + lx, w));
        }
    }
    __syncthreads();
    // columns: one thread per (component, column), every column of the tile and its halo
    if (h >= 2 && tid < NC * T::WX) {
        const int comp = tid / T::WX, col = tid - comp * T::WX;
        liftLine<T::WY>(smem + comp * PLANE + col, T::P);
    }
    __syncthreads();
    // rows: one thread per (component, output row)
    if (w >= 2 && tid < NC * T::Y) {
        const int comp = tid / T::Y, r = HALO + (tid - comp * T::Y);
        liftLine<T::WX>(smem + comp * PLANE + r * T::P, 1);
    }
    __syncthreads();
    for (int k = 0; k < NC; ++k)
        writeOutputs<THREADS, SHAPE>(a, smem + k * PLANE, COLOR ? k : (int)blockIdx.z, tx, ty, tid);
}

template <int MODE, int SHAPE>
void optIn() {
    GB_CHECK(cudaFuncSetAttribute(levelKernel<MODE, SHAPE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)feSmem<MODE, SHAPE>()));
}

template <int MODE, int SHAPE>
void launch(const ColorArgs& c, const LevelArgs& a, int comps, cudaStream_t st) {
    using T = Tile<SHAPE>;
    const dim3 grid(divUp(a.w, T::X), divUp(a.h, T::Y), comps);
    levelKernel<MODE, SHAPE><<<grid, feThreads<MODE, SHAPE>(), feSmem<MODE, SHAPE>(), st>>>(c, a);
}

}  // namespace

void frontendInit() {
    optIn<1, 0>();
    optIn<1, 1>();
    optIn<1, 2>();
    optIn<2, 0>();
    optIn<3, 0>();
    optIn<0, 0>();
    optIn<0, 1>();
    optIn<0, 2>();
}

void launchLevel1(const ColorArgs& c, const LevelArgs& a, int shape, cudaStream_t st) {
    if (shape < 0 || shape > 2) throw std::logic_error("tile shape must be 0, 1 or 2");
    if (c.route == kRouteLut) {
        if (!c.lut3 || c.lutN < 2) throw std::logic_error("LUT route without a LUT");
        launch<3, 0>(c, a, 1, st);  // the rarer routes keep the 64 x 64 tile
    } else if (c.route == kRouteManaged) {
        launch<2, 0>(c, a, 1, st);
    } else if (shape == 1) {
        launch<1, 1>(c, a, 1, st);
    } else if (shape == 2) {
        launch<1, 2>(c, a, 1, st);
    } else {
        launch<1, 0>(c, a, 1, st);
    }
    GB_CHECK(cudaGetLastError());
}

void launchLevel(const LevelArgs& a, int shape, cudaStream_t st) {
    if (shape < 0 || shape > 2) throw std::logic_error("tile shape must be 0, 1 or 2");
    if (shape == 1) launch<0, 1>(ColorArgs{}, a, 3, st);
    else if (shape == 2) launch<0, 2>(ColorArgs{}, a, 3, st);
    else launch<0, 0>(ColorArgs{}, a, 3, st);
    GB_CHECK(cudaGetLastError());
}

}  // namespace gb
