// PCRD hull points of one code-block on the device: the lower convex hull of its
// (truncation length, accumulated weighted distortion reduction) points, by the same
// sequence of IEEE double operations as the host rate control (the hull construction of
// Josephur/libgail src/core/rate_control.cpp:38-86), each written with an explicit
// round-to-nearest intrinsic so that nothing is contracted or reordered: the points and
// slopes are bit-identical to the host's.
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>

#include <cstdint>

#include "common.cuh"

namespace gb {

constexpr int HULL_THREADS = 32;            // threads (blocks) per CTA of a hull kernel
constexpr int HULL_DEPTH = kMaxPasses + 1;  // the origin and one point per pass

// The hull stack of a CTA's threads, one column per thread.
struct HullStack {
    double D[HULL_DEPTH][HULL_THREADS];
    uint32_t R[HULL_DEPTH][HULL_THREADS];
    uint8_t K[HULL_DEPTH][HULL_THREADS];
};

// Block with nbps planes and np passes (len / dist: its pass tables), distortion weight
// scale: its points to hp / hs (coding passes, slope from the previous point), then zeros
// up to np. t: the calling thread's column of the stack.
__device__ __forceinline__ void hullOfBlock(HullStack& st, int t, int nbps, int np, double scale, const uint32_t* len,
                                            const int32_t* dist, uint8_t* hp, double* hs) {
    // slope from stack point m - 1 to point m, as the host computes it when m is pushed
    // (its inputs stay unchanged while m is on the stack, so recomputing it is exact)
    auto slopeAt = [&](int m) {
        const uint32_t r1 = st.R[m][t], r0 = st.R[m - 1][t];
        return r1 == r0 ? CUDART_INF : __ddiv_rn(__dsub_rn(st.D[m][t], st.D[m - 1][t]), (double)(r1 - r0));
    };
    int m = 0;
    st.D[0][t] = 0.0;
    st.R[0][t] = 0;
    st.K[0][t] = 0;
    double acc = 0.0;
    for (int k = 0; k < np; ++k) {
        // the plane pass k codes and its weight 4^plane / 4096 (shift counts taken mod 64,
        // as the host's shift instruction does)
        const int plane = k == 0 ? nbps - 1 : nbps - 2 - (k - 1) / 3;
        const double ps = (double)(1ull << ((2 * plane) & 63)) / 4096.0;
        acc = __dadd_rn(acc, __dmul_rn(__dmul_rn((double)dist[k], ps), scale));
        const uint32_t r = len[k];
        if (acc <= st.D[m][t]) continue;  // no gain: never a hull point
        while (m >= 1) {  // drop the points the new one makes concave
            const uint32_t rm = st.R[m][t];
            const double sNew = r == rm ? CUDART_INF : __ddiv_rn(__dsub_rn(acc, st.D[m][t]), (double)(r - rm));
            if (sNew < slopeAt(m)) break;
            --m;
        }
        ++m;
        st.R[m][t] = r;
        st.D[m][t] = acc;
        st.K[m][t] = (uint8_t)(k + 1);
    }
    for (int q = 1; q <= m; ++q) {
        const double dr = __dsub_rn((double)st.R[q][t], (double)st.R[q - 1][t]);
        hp[q - 1] = st.K[q][t];
        hs[q - 1] = dr <= 0 ? CUDART_INF : __ddiv_rn(__dsub_rn(st.D[q][t], st.D[q - 1][t]), dr);
    }
    for (int q = m; q < np; ++q) {
        hp[q] = 0;
        hs[q] = 0.0;
    }
}

}  // namespace gb
