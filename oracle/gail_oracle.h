/* CPU oracle for the JPEG 2000 encode/decode hot path: test infrastructure only.
 *
 * A plain-C restatement of the reference CPU path (Josephur/libgail, src/core and
 * src/kernels) used as the checker for the CUDA kernels. Nothing in the product links or
 * calls this code: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * load it. Every function cites the reference file:line whose behaviour it restates.
 *
 * Parity of this restatement is pinned against the reference itself, built from its own
 * sources by oracle/Makefile into oracle/_ref/ (see tests/test_oracle_vs_ref.py), and
 * against the committed fixtures in tests/golden/.
 */
#ifndef GAIL_ORACLE_H
#define GAIL_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OR_CBLK 32
#define OR_CBLK_AREA 1024
#define OR_FRAC_BITS 6
#define OR_MAX_PASSES 64

/* One coded block: the reference's T1Result (core/t1_ref.h:13-19). */
typedef struct {
    int32_t nbps;
    int32_t num_passes;
    uint32_t data_len;
    uint32_t num_symbols;           /* MQ decisions coded (for throughput accounting) */
    uint32_t pass_len[OR_MAX_PASSES];
    int32_t pass_dist[OR_MAX_PASSES];
} or_t1_result;

/* Tier-1 encode of one 32x32 block of sign-magnitude words (t1EncodeRef,
 * core/t1_ref.cpp:288-292). buf receives the codeword; buf_cap must be at least
 * 4096 * nbps + 64 bytes (20 * 4096 + 64 always suffices). slope_thresh 0 codes every
 * pass; otherwise the early-termination rule of core/t1_ref.cpp:128-162 applies.
 * Returns 0, or -1 when the block needs more than 64 passes. */
int or_t1_encode(const uint32_t* coeffs, int w, int h, int orient, int max_passes, float slope_thresh,
                 float dist_scale, uint8_t* buf, size_t buf_cap, or_t1_result* out);

/* Dead-zone quantiser, quantizeCoeff (core/quant.h:20-25). */
uint32_t or_quantize(float v, float inv_delta, uint32_t max_mag);

/* Forward / inverse irreversible 9/7 transform of one plane in place (fdwt97_2d,
 * core/dwt_cpu.cpp:184-206; idwt97_2d, :213-240). stride in floats. */
void or_fdwt97_2d(float* plane, int stride, int width, int height, int levels);
void or_idwt97_2d(float* plane, int stride, int width, int height, int levels, int skip);
/* One-dimensional double-precision inverse (idwt97_1d, core/dwt_cpu.cpp:140-155). */
void or_idwt97_1d_f64(const double* in, double* out, int n);

/* ---- frame geometry (core/layout.cpp:77-210) ---- */
typedef struct {
    int32_t comp, res, level, orient;
    int32_t px0, py0, w, h, ncbx, ncby, cblk_base;
    int32_t eps, mu, mb;
    float delta;
    double weight;
} or_band;

typedef struct {
    int32_t band, x0, y0, w, h;
} or_cblk;

/* Number of bands and code-blocks of a frame (for sizing the arrays below). */
void or_geometry_counts(int width, int height, int levels, int* num_bands, int* num_cblks);
/* makeLayout: geometry plus step sizes from base_step. Returns 0, or -1 on a step size
 * that does not fit (more than 22 bit-planes). */
int or_make_layout(int width, int height, int fourk, double base_step, or_band* bands, or_cblk* cblks);
double or_synthesis_norm(int level, int orient);

/* ---- colour (core/color.cpp, kernels/color_math.h) ---- */
enum { OR_TF_BT1886 = 0, OR_TF_SRGB = 1, OR_TF_PQ = 2, OR_TF_HLG = 3, OR_TF_LINEAR = 4, OR_TF_GAMMA26 = 5 };
enum { OR_PRI_BT709 = 0, OR_PRI_BT2020 = 1, OR_PRI_P3D65 = 2, OR_PRI_DCIP3 = 3, OR_PRI_XYZ = 4 };

/* The managed colour route without tone map, gamut compression or 3D LUT (the routes the
 * benchmark inputs use): 64K-entry EOTF table and the RGB->XYZ matrix (ColorConverter,
 * core/color.cpp:296-372). */
typedef struct {
    float eotf[65536];
    float m[9];
} or_color;
void or_color_init(or_color* c, int transfer, int primaries, double sdr_white);
/* R'G'B' 16-bit codes -> 12-bit X'Y'Z' codes (cm_rgb_to_xyz12, color_math.h:117-179). */
void or_color_xyz12(const or_color* c, uint16_t r, uint16_t g, uint16_t b, int out[3]);
/* ICT of DC-shifted codes (ictForward, core/color.h:136-140). */
void or_ict_forward(int x, int y, int z, float out[3]);

/* Planar Y'CbCr (or G'B'R') frame -> container-size interleaved R'G'B' 16-bit
 * (planarToRgb48Row, core/color.cpp:142-204). */
typedef struct {
    int32_t width, height, active_w, active_h, ox, oy, sx, sy, rgb, bits, full_range, chroma;
    double kr, kb;
} or_planar;
void or_planar_to_rgb48(const or_planar* f, const void* src, uint16_t* rgb);

/* Whole encoder front end: R'G'B' 16-bit interleaved frame -> three ICT planes. */
void or_color_frame(const or_color* c, const uint16_t* rgb, int npix, float* p0, float* p1, float* p2, uint16_t* xyz12);

/* ---- decoder (core/t1_dec.cpp, core/cpu_decode_backend.cpp) ---- */
/* Decodes `passes` passes of a block (t1DecodeBlock, core/t1_dec.cpp:176-179). out: 32x32
 * words, bit 31 sign, low bits twice the magnitude plus the mid-point. */
void or_t1_decode(const uint8_t* data, uint32_t len, int w, int h, int orient, int nbps, int passes, uint32_t* out);
/* Inverse ICT + level shift + 12-bit clamp of one sample triple (cpu_decode_backend.cpp:77-91). */
void or_ict_inverse_pack(float y0, float y1, float y2, int shift, uint16_t out[3]);

/* Batch forms for the tests: or_t1_encode over n blocks (same arguments as the
 * library's gb_t1_encode_blocks), quantisation of whole Mallat planes into
 * code-block-major words, and the 12-bit encoding of one normalised value. */
int or_t1_encode_many(const uint32_t* coeffs, const int32_t* geom4, uint32_t n, float slope, const float* dscale,
                      uint32_t* info4, uint32_t* pass_len, int32_t* pass_dist, uint8_t* data, uint32_t stride);
void or_quantize_frame(const float* planes, int width, int height, const or_band* bands, const or_cblk* cblks, int nc,
                       uint32_t* out);
int or_dci_code(float n);

/* 12-bit code -> 16-bit signal as the public API fills X'Y'Z' frames (gail_api.cpp:389-394). */
uint16_t or_xyz12_to_16(uint32_t v);

#ifdef __cplusplus
}
#endif

#endif
