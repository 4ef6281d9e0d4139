/* The GAIL CUDA plugin interface, as plain C: the function table libgail reaches a CUDA
 * backend through, and every structure that crosses it, member for member.
 *
 * This is the boundary gail_b200 is a drop-in behind. It restates the reference's
 * src/cuda/cuda_plugin.h:36-191 (Josephur/libgail) and the library structures that pass
 * through it unchanged (gail::Subband, src/core/layout.h:29-42; gail::CblkInfo,
 * src/core/tier1_types.h:12-18; gail::CblkCode, src/core/t2_parse.h:17-22;
 * gail::FrameFormat, src/core/color.h:47-73; gail::FrameTimings, src/core/backend.h:33-37).
 * The layouts must match byte for byte: libgail compares `size` and `layout` (a hash of
 * the structure sizes, gb_plugin_layout_hash()) before it uses a plugin.
 */
#ifndef GAIL_CUDA_PLUGIN_ABI_H
#define GAIL_CUDA_PLUGIN_ABI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GAIL_CUDA_PLUGIN_ABI 1u
#define GAIL_CUDA_PLUGIN_ENTRY "gail_cuda_plugin_get"

enum GailCudaStatus {
    GAIL_CUDA_OK = 0,
    GAIL_CUDA_ERROR = 1,
    GAIL_CUDA_DEVICE_MEMORY = 2, /* the device stays usable */
    GAIL_CUDA_HOST_MEMORY = 3,
    GAIL_CUDA_MISUSE = 4,
    GAIL_CUDA_NO_CODE = 5 /* device_usable: no code for this device, ever */
};

/* ---- library structures carried as they are --------------------------------------- */
typedef struct GbSubband {
    int32_t comp, res, level, orient; /* orient: 0 LL, 1 HL, 2 LH, 3 HH */
    int32_t px0, py0;                 /* top-left in the Mallat-layout plane */
    int32_t w, h;
    int32_t ncbx, ncby;               /* code-block grid */
    int32_t cblkBase;                 /* global index of its first code-block */
    int32_t eps, mu;                  /* signalled step (exponent, mantissa) */
    int32_t Mb;                       /* magnitude bit-planes */
    float delta;                      /* quantisation step */
    double weight;                    /* squared-error weight */
} GbSubband;

typedef struct GbCblkInfo {
    uint32_t nbps, numPasses, dataOffset, dataLen, passBase;
} GbCblkInfo;

typedef struct GbCblkCode {
    uint32_t offset, len;
    uint8_t passes, nbps;
} GbCblkCode;

enum { GB_FRAME_RGB48 = 0, GB_FRAME_PLANAR = 1 };
enum { GB_CHROMA_LEFT = 0, GB_CHROMA_CENTER = 1, GB_CHROMA_TOPLEFT = 2 };

typedef struct GbFrameFormat {
    int32_t kind;   /* GB_FRAME_* */
    int32_t chroma; /* GB_CHROMA_* */
    int32_t width, height;
    int32_t activeW, activeH, ox, oy;
    int32_t sx, sy;
    uint8_t rgb; /* C++ bool */
    int32_t bits;
    uint8_t fullRange; /* C++ bool */
    double kr, kb;
} GbFrameFormat;

typedef struct GbFrameTimings {
    double upload, color, dwt, quant, t1, t1cm, t1mq, download, gpu, total;
    double symbols, codedBytes;
} GbFrameTimings;

/* ---- the plugin's own structures --------------------------------------------------- */
typedef void (*GailCudaLog)(void* user, int level, const char* message);
typedef struct GailCudaDevice GailCudaDevice;
typedef struct GailCudaEncoder GailCudaEncoder;
typedef struct GailCudaDecoder GailCudaDecoder;

typedef struct GailCudaDeviceDesc {
    int32_t index;
    int32_t smMajor, smMinor;
    uint64_t memoryBytes;
    char name[256];
    char uuid[48];
    char pciBusId[32];
} GailCudaDeviceDesc;

typedef struct GailCudaLayout {
    int32_t profile, width, height, levels, guardBits; /* profile: 0 2K, 1 4K */
    int32_t numBands, numCblks;
    double baseStep;
    const GbSubband* bands;
} GailCudaLayout;

/* transfer: 0 BT.1886, 1 sRGB, 2 PQ, 3 HLG, 4 linear, 5 gamma 2.6; primaries: 0 BT.709,
 * 1 BT.2020, 2 P3-D65, 3 DCI-P3, 4 XYZ; toneMap: 0 signal, 1 shoulder, 2 BT.2390, 3 none;
 * toneNorm: 0 channel, 1 maxRGB, 2 luminance; gamut: 0 P3-D65, 1 DCI-P3, 2 none. */
typedef struct GailCudaColor {
    int32_t transfer, primaries, toneMap, toneNorm, gamut, lut3dSize;
    double sdrWhite, hdrPeak, cinemaPeak, hdrRefWhite, cinemaRefWhite, knee, gamutThreshold;
    const char* lut3d;
    const float* lut3dData;
    uint64_t lut3dCount;
} GailCudaColor;

typedef struct GailCudaEncodeSettings {
    int32_t profile, width, height;
    double baseStep, slopeFactor, bitsPerSymbol;
    GbFrameFormat input;
    GailCudaColor color;
} GailCudaEncodeSettings;

typedef struct GailCudaDecodeSettings {
    int32_t reduce, highBits;
} GailCudaDecodeSettings;

typedef struct GailCudaMemory {
    uint64_t total, available;
    int32_t budgeted;
} GailCudaMemory;

typedef struct GailCudaTier1 {
    const GbCblkInfo* info;
    const uint32_t* passLen;
    const int32_t* passDist;
    const uint8_t* data;
    uint64_t numInfo, numPasses, numData;
} GailCudaTier1;

typedef struct GailCudaDebug {
    int32_t full;
    const uint16_t* xyz12;
    const uint32_t* coeffs;
    const float* wavelet;
    uint64_t numXyz12, numCoeffs, numWavelet;
} GailCudaDebug;

typedef struct GailCudaDecodeTimings {
    double t1, dwt, color, total;
    int32_t wantWavelet;
    const float* wavelet[3];
    uint64_t numWavelet;
} GailCudaDecodeTimings;

typedef struct GailCudaPlugin {
    uint32_t abi;
    uint32_t size;
    uint64_t layout;
    const char* name;
    const char* toolkit;
    const char* archs;
    const char* (*last_error)(void);
    int (*device_count)(void);
    int (*device_desc)(int index, GailCudaDeviceDesc* out);
    int (*device_usable)(int index);
    int (*device_create)(int index, GailCudaLog log, void* user, GailCudaDevice** out);
    void (*device_destroy)(GailCudaDevice* d);
    const char* (*device_name)(GailCudaDevice* d);
    int (*device_memory)(GailCudaDevice* d, GailCudaMemory* out);
    uint64_t (*encoder_bytes)(GailCudaDevice* d, const GailCudaLayout* layout, const GailCudaEncodeSettings* settings);
    int (*encoder_create)(GailCudaDevice* d, const GailCudaLayout* layout, const GailCudaEncodeSettings* settings,
                          GailCudaEncoder** out);
    void (*encoder_destroy)(GailCudaEncoder* e);
    void* (*encoder_input)(GailCudaEncoder* e);
    void (*encoder_set_slope)(GailCudaEncoder* e, double threshold);
    int (*encoder_encode)(GailCudaEncoder* e, const void* frame, GailCudaTier1* out, GbFrameTimings* timings,
                          GailCudaDebug* debug);
    uint64_t (*decoder_bytes)(GailCudaDevice* d, const GailCudaLayout* layout, const GailCudaDecodeSettings* settings);
    int (*decoder_create)(GailCudaDevice* d, const GailCudaLayout* layout, const GailCudaDecodeSettings* settings,
                          GailCudaDecoder** out);
    void (*decoder_destroy)(GailCudaDecoder* d);
    int (*decoder_decode)(GailCudaDecoder* d, const GailCudaLayout* frame, const uint8_t* data, size_t size,
                          const GbCblkCode* blocks, size_t numBlocks, void* dst, ptrdiff_t strideBytes,
                          GailCudaDecodeTimings* timings);
} GailCudaPlugin;

/* The one symbol a GAIL CUDA plugin exports: the table, or NULL for another ABI. */
#if defined(_WIN32)
__declspec(dllexport)
#else
__attribute__((visibility("default")))
#endif
const GailCudaPlugin* gail_cuda_plugin_get(uint32_t abi);

#ifdef __cplusplus
}
#endif

#endif
