/* gail_b200: B200-native (sm_100a) JPEG 2000 encode/decode hot path behind GAIL's
 * CUDA plugin ABI.
 *
 * The library libgail_cuda13.so exports exactly two kinds of entry point:
 *
 *  1. gail_cuda_plugin_get(), the one symbol a GAIL CUDA plugin exports, returning the
 *     GailCudaPlugin function table (declared in gail_cuda_plugin_abi.h). It replaces the
 *     reference plugin's entry point, Josephur/libgail src/cuda/cuda_plugin.h:195 and
 *     src/cuda/cuda_plugin.cpp:249, so that libgail loads this library as its
 *     gail_cuda13 backend.
 *
 *  2. The gb_* functions below: the stages of that path over plain buffers, for callers
 *     that hold code-blocks, codestreams or Tier-1 frames rather than whole pictures.
 *     Each names the reference interface it replaces.
 *
 * Every function that can fail returns a GailCudaStatus value (0 = OK) and leaves its
 * message for the calling thread in gb_last_error(). Host pointers everywhere; no
 * function keeps a pointer it was given after it returns.
 */
#ifndef GAIL_B200_H
#define GAIL_B200_H

#include <stddef.h>
#include <stdint.h>

#include "gail_cuda_plugin_abi.h"

#if defined(_WIN32)
#define GB_API __declspec(dllexport)
#else
#define GB_API __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Message of the calling thread's most recent failed call (never NULL). Replaces the
 * plugin table's last_error, src/cuda/cuda_plugin.h:151. */
GB_API const char* gb_last_error(void);

/* Tier-1 encode of n quantised code-blocks on the current CUDA device. Replaces
 * t1EncodeRef (src/core/t1_ref.h:39-40) applied to each block.
 *   coeffs     n x 1024 sign-magnitude words (bit 31 sign, 6 fractional magnitude bits),
 *              32 x 32 row-major per block, zero outside the block's w x h
 *   geom4      n x {w (1..32), h (1..32), orient (0 LL, 1 HL, 2 LH, 3 HH), maxPasses (0..64)}
 *   slope      early-termination threshold (0: code every pass)
 *   distScale  per-block distortion scale of that rule (NULL: 1)
 *   info4      out: n x {nbps, passes, MQ decisions, codeword bytes}
 *   passLen    out: n x 64 truncation lengths; passDist: n x 64 distortion reductions
 *   data       out: codeword of block i at data + i * dataStride */
GB_API int gb_t1_encode_blocks(const uint32_t* coeffs, const int32_t* geom4, uint32_t n, float slope,
                               const float* distScale, uint32_t* info4, uint32_t* passLen, int32_t* passDist,
                               uint8_t* data, uint32_t dataStride);

/* gb_t1_encode_blocks without any allocation. No counterpart in the reference: it is for
 * callers that must not allocate device memory themselves, such as a real-time frame
 * thread (cudaMalloc may wait for the whole device and stall it) or a process whose
 * device memory is budgeted up front. Same arguments and results as gb_t1_encode_blocks,
 * but every call works in one static device array of 7.6 MB that this library reserves on
 * each GPU it is loaded on, for the life of the process:
 *   - at most 64 code-blocks per call; more is refused with GAIL_CUDA_MISUSE;
 *   - the first call on a device looks up the array's device address and loads the
 *     kernels' tables there; make that first call before any stream capture;
 *   - calls share the array: two calls whose work overlaps on the GPU (other threads,
 *     other streams) race and corrupt each other's results, so serialise them;
 *   - the work runs on a non-blocking stream the library makes for the device at the
 *     first call, and the call waits for that stream alone before it returns;
 *   - each codeword is copied into its row of data exactly (info4[4i+3] bytes); the row's
 *     bytes after it are left untouched;
 *   - cudaDeviceReset on a device after the first call there is not supported (the array's
 *     address and the stream are kept for the life of the process). */
GB_API int gb_t1_encode_blocks_noalloc(const uint32_t* coeffs, const int32_t* geom4, uint32_t n, float slope,
                                       const float* distScale, uint32_t* info4, uint32_t* passLen, int32_t* passDist,
                                       uint8_t* data, uint32_t dataStride);

/* Failure detection of the persistent Tier-1 launch (GbTuning.t1Persistent), exercised
 * without a fault: one warp waits on a device flag that nothing sets, as the launch's warps
 * wait for a partner's announced work, with its limit lowered to limitMs (1..2000; the
 * launch uses 2000) and returns. *status gets the device status bits it left (16: the wait
 * gave up) and *elapsedMs (may be NULL) the launch's duration; the device stays usable.
 * No counterpart in the reference (its kernels do not wait on one another). */
GB_API int gb_t1_wait_selftest(uint32_t limitMs, uint32_t* status, float* elapsedMs);

/* The DCI frame layout: subbands (with their quantisation steps) in the plugin ABI's
 * form, for callers that build GailCudaLayout themselves. Replaces makeLayout
 * (src/core/layout.h:87 with Profile::Cinema2K / Cinema4K). maxBands >= 3 * 19 + 3. */
GB_API int gb_make_layout(int width, int height, int fourk, double baseStep, GbSubband* bands, int maxBands,
                          int* numBands, int* numCblks);

/* The colour tables the encoder uploads for a colour setting: the 65536-entry EOTF, the
 * RGB->XYZ matrix and the 4096 thresholds of the 12-bit DCI encoding. Replaces
 * ColorConverter's lut()/params() (src/core/color.h:105-108). Any pointer may be NULL. */
GB_API int gb_color_tables(const GailCudaColor* color, float* eotf65536, float* matrix9, float* thresholds4096);

/* The colour route of a setting (0 direct, 1 tone map and / or gamut compression, 2 3D
 * LUT), its constants in the positions of the reference's 48-float parameter block
 * (src/kernels/color_params.h; ColorConverter::params(), src/core/color.h:106) and the LUT's
 * nodes per axis (0 without one). A LUT given by path is read. route and lutN may be NULL. */
GB_API int gb_color_route(const GailCudaColor* color, float* params48, int32_t* route, int32_t* lutN);

/* Launch tuning per frame profile (0 = 2K, 1 = 4K), read by every launch of that profile
 * made after the call (plain encoders and decoders, engine batches). No counterpart in the
 * reference, whose launch shapes are fixed; libgail_b200/autotune.py measures candidates
 * on the GPU and keeps the fastest. gb_set_tuning(profile, NULL) restores the defaults.
 *   soloDecisions  MQ coding: blocks with at least this many decisions are coded alone in
 *                  a warp first (rounded down to a power of two; default 16384)
 *   cmCtasPerSm, mqCtasPerSm, decCtasPerSm  grid caps in CTAs per SM of context modelling,
 *                  MQ coding and Tier-1 decoding (defaults 16, 16, 32; 1..64)
 *   t1Persistent   1: Tier-1 encoding as one persistent launch whose warps take context
 *                  modelling, the order, MQ coding and truncation lengths from device
 *                  queues in turn; 0 (default): four launches. Same results either way. */
typedef struct GbTuning {
    uint32_t soloDecisions;
    int32_t cmCtasPerSm, mqCtasPerSm, decCtasPerSm;
    int32_t t1Persistent;
    int32_t decHeavyPct;  /* Tier-1 decode: blocks whose codeword exceeds this % of the mean bytes per
                             decoding warp run on SMs of their own, four per SM (0: none) */
    int32_t dwtTile1, dwtTileN;  /* encoder front-end tile at level 1 and at levels 2..: 0 = 64 x 64,
                                    1 = 128 x 64, 2 = 64 x 128 (same coefficients; read when an
                                    encoder or engine frame slot is made) */
} GbTuning;
GB_API int gb_set_tuning(int profile, const GbTuning* t);
GB_API int gb_get_tuning(int profile, GbTuning* t);

/* Frames already in device memory (a serving layer that keeps them resident). The
 * encoder is one made by the plugin table's encoder_create; these replace the upload half
 * of encoder_encode (the reference's CudaSlot::encodeView, src/cuda/cuda_backend.cu:870-977).
 *   gb_encoder_stream          the encoder's CUDA stream (cudaStream_t), for ordering and
 *                              timing the caller's own work against it
 *   gb_encoder_enqueue_device  enqueue front end, Tier-1 and packing of the frame at dFrame
 *                              (device memory, the encoder's input format) on that stream;
 *                              returns at once; dFrame must stay valid until it is done
 *   gb_encoder_finish          wait for the enqueued work and check the kernels' status */
GB_API void* gb_encoder_stream(GailCudaEncoder* e);
GB_API int gb_encoder_enqueue_device(GailCudaEncoder* e, const void* dFrame);
GB_API int gb_encoder_finish(GailCudaEncoder* e);

/* Per-stage device time of gb_encoder_enqueue_device (the reference's FrameTimings stage
 * split, src/core/backend.h:33-37): gb_encoder_stage_timing(e, 1) makes every enqueue
 * record CUDA events between its stages; gb_encoder_stage_times waits for the stream and
 * returns in ms5 the summed durations of {front end (colour, wavelet, quantisation),
 * Tier-1 context modelling, Tier-1 ordering, MQ coding, packing} over the enqueues since
 * the last call (at most 512), and their number in count. */
GB_API int gb_encoder_stage_timing(GailCudaEncoder* e, int on);
GB_API int gb_encoder_stage_times(GailCudaEncoder* e, double* ms5, int* count);

/* The batched, served encoder: many frames (of any registered layouts) in flight on one
 * GPU, their Tier-1 work batched into shared launches as they become ready (continuous
 * batching), admission against an HBM budget. No counterpart in the reference, whose
 * per-frame slots (src/cuda/cuda_backend.cu:870-977, driven by src/core/pipeline.cpp:170-249)
 * each launch their own kernels; the results are the same Tier1Frame views, bit-identical.
 *   gb_engine_create       maxBatch: most frames per Tier-1 launch; hbmBudget: device bytes for
 *                          frames in flight (0: 90 % of the free memory)
 *   gb_engine_add_encoder  a frame class (layout, input format, colour); frameBytes: its
 *                          device footprint per frame in flight
 *   gb_engine_reserve      make frame slots for a class now, until it has `slots` of them (or
 *                          the budget is spent; *have: how many it has): capacity set up
 *                          before serving. Otherwise a slot is made when a frame finds none
 *                          free, by a thread of the engine's own, while fewer frames than
 *                          eight batches are in progress (making one takes tens of ms)
 *   gb_engine_submit       queue one frame (host memory, pinned for speed, or device memory
 *                          with onDevice); the frame must stay valid until it is released
 *   gb_engine_wait         the next finished frame (id -1 after timeoutMs without one), its
 *                          Tier-1 view (valid until release), submit-to-finish latency and
 *                          status
 *   gb_engine_release      give the frame's slot back
 *   gb_engine_stats        frames, batches, frames in batches, slots, slot bytes
 *   gb_engine_set_codestream  from now on, every frame also gets its DCI codestream, driven
 *                          by `threads` host workers: gb_rate_and_build's rate control and
 *                          codestream (fps, maxMbps, compMbps, label, tag), then with check
 *                          the DCI check; the frame is handed out by gb_engine_wait once its
 *                          codestream is made (the latency includes it). flags 0: rate control
 *                          and Tier-2 on the device (gb_device_rate_and_build's path; the
 *                          Tier-1 frame stays in device memory and gb_engine_wait hands out an
 *                          empty Tier-1 view); GB_CS_HOST: on the host workers from the Tier-1
 *                          frame in host memory, with the hull points computed on the GPU
 *                          (gb_rate_and_build_hull's path); GB_CS_TIER1: the Tier-1 frame and
 *                          its hull points also in host memory, as without codestreams
 *   gb_engine_set_slope_factor  Tier-1 early termination as libgail's pipeline drives it
 *                          (src/core/pipeline.cpp:194-217; gail.h's encoder forces 0.25,
 *                          src/api/gail_api.cpp:607): each encode admitted from now on stops
 *                          coding a block's bit-planes below lastLambda x factor, lastLambda the
 *                          smallest per-component slope threshold of the last finished frame's
 *                          rate control (0 at first: every pass); a frame whose own threshold
 *                          comes out below the one it was coded with is coded again with every
 *                          pass. 0 turns it off. Needs codestreams on
 *   gb_engine_frame_info   a finished encode's first early-termination threshold and whether
 *                          it was coded again with every pass
 *   gb_engine_counters     for the engine's encodes so far: host-to-device and device-to-host
 *                          bytes copied (frames in; Tier-1 frames, rate-control read-backs and
 *                          codestreams out) and kernels launched (any pointer may be NULL)
 *   gb_engine_codestream   a handed-out frame's codestream (valid until release) and its
 *                          DCI verdict (1, 0, or -1 when not checked)
 *   gb_engine_add_decoder  a decode class (layout, decode settings as decoder_create takes
 *                          them); frameBytes: its device footprint per decode in flight
 *   gb_engine_submit_decode  queue a codestream (copied) for decoding: host workers parse it
 *                          (gb_parse_codestream) and decode it on a decoder slot of its class
 *                          (decoder_decode's stages, each slot on its own stream, sharing the
 *                          HBM budget); handed out by gb_engine_wait like an encode (its Tier-1
 *                          view empty)
 *   gb_engine_picture      a handed-out decode's picture (valid until release): height rows
 *                          of width x 3 codes
 *   gb_engine_hull         a handed-out encode's PCRD hull points, computed on the GPU after
 *                          Tier-1 (valid until release; the layout of gb_tier1_hull, over the
 *                          frame's numPasses slots); its codestream's rate control takes them
 *   gb_engine_open_loop    an open-loop load, driven natively: request i (kind 0: encode of
 *                          the frame item[i] of class classId[i], on the device when
 *                          onDevice[i]; kind 1: decode of the codestream item[i] of size[i]
 *                          bytes) is submitted arrivalSec[i] seconds after the call starts
 *                          (non-decreasing), whether or not earlier ones have finished; a
 *                          second thread waits for each and releases it. Out: each request's
 *                          latency (submit to finish, as gb_engine_wait reports it) and
 *                          status, and the time from the start to the last finish. For
 *                          latency under Poisson arrivals without the caller's own threads
 *                          in the way
 *   gb_engine_decode_times for the engine's decode requests since the last reset: ms3 = host
 *                          time waiting for a free decoder slot, parsing, and in the slot
 *                          (upload, device stages, picture back); counts2 = decodes, decoder
 *                          slots made after their class was added (each allocates device and
 *                          pinned host memory); reset 1 zeroes them
 *   gb_engine_stage_timing per-stage timing of the served path on (1) or off (0): CUDA events
 *                          around each frame's front-end graph and each Tier-1 batch's stages,
 *                          host wall time of each frame's device rate control
 *   gb_engine_stage_times  the totals since the last reset: ms6 = front end, context
 *                          modelling, ordering, MQ coding with truncation lengths, packing
 *                          (elapsed on the batch stream), rate control and Tier-2 round trips;
 *                          counts4 = frames timed in the front end, batches timed, frames in
 *                          them, frames timed in rate control; reset 1 zeroes them */
typedef struct GbEngine GbEngine;
GB_API int gb_engine_create(int device, uint64_t hbmBudget, int maxBatch, GbEngine** out);
GB_API void gb_engine_destroy(GbEngine* e);
GB_API int gb_engine_add_encoder(GbEngine* e, const GailCudaLayout* layout, const GailCudaEncodeSettings* settings,
                                 int* classId, uint64_t* frameBytes);
GB_API int gb_engine_reserve(GbEngine* e, int classId, int slots, int* have);
GB_API int gb_engine_submit(GbEngine* e, int classId, const void* frame, int onDevice, double slope, int64_t* id);
GB_API int gb_engine_wait(GbEngine* e, int timeoutMs, int64_t* id, GailCudaTier1* out, double* latencyMs,
                          int* frameStatus);
GB_API int gb_engine_release(GbEngine* e, int64_t id);
GB_API int gb_engine_stats(GbEngine* e, uint64_t* out5);
GB_API int gb_engine_stage_timing(GbEngine* e, int on);
GB_API int gb_engine_decode_times(GbEngine* e, int reset, double* ms3, uint64_t* counts2);
GB_API int gb_engine_open_loop(GbEngine* e, uint32_t n, const int* classId, const int* kind, const void* const* item,
                               const uint64_t* size, const int* onDevice, const double* arrivalSec, double* latencyMs,
                               int* status, double* elapsedSec);
GB_API int gb_engine_stage_times(GbEngine* e, int reset, double* ms6, uint64_t* counts4);
/* Batch policy: at most maxBatch frames per Tier-1 launch; while another batch keeps the GPU
 * busy, a batch waits to gather minBatchPct % of maxBatch ready frames, but not past
 * maxWaitMs after its oldest frame (defaults: the create call's maxBatch, 25 %, 2 ms). */
GB_API int gb_engine_set_policy(GbEngine* e, int maxBatch, int minBatchPct, double maxWaitMs);
enum { GB_CS_HOST = 1, GB_CS_TIER1 = 2 };
GB_API int gb_engine_set_codestream(GbEngine* e, double fps, double maxMbps, double compMbps, const char* label,
                                    const char* tag, int threads, int check, int flags);
GB_API int gb_engine_counters(GbEngine* e, uint64_t* h2d, uint64_t* d2h, uint64_t* launches);
GB_API int gb_engine_set_slope_factor(GbEngine* e, double factor);
GB_API int gb_engine_frame_info(GbEngine* e, int64_t id, double* threshold, int* recoded);
GB_API int gb_engine_codestream(GbEngine* e, int64_t id, const uint8_t** data, uint64_t* size, int* dciOk);
GB_API int gb_engine_add_decoder(GbEngine* e, const GailCudaLayout* layout, const GailCudaDecodeSettings* settings,
                                 int* classId, uint64_t* frameBytes);
GB_API int gb_engine_submit_decode(GbEngine* e, int classId, const uint8_t* data, uint64_t size, int64_t* id);
GB_API int gb_engine_picture(GbEngine* e, int64_t id, const uint16_t** pix, int* width, int* height);
GB_API int gb_engine_hull(GbEngine* e, int64_t id, const uint8_t** passes, const double** slope);

/* The host codec around a Tier-1 frame, byte-identical to libgail's core for the same
 * frame. Thread-safe across threads (each keeps its own writer per layout and label).
 *   gb_dci_limits              DCI byte budgets at fps: whole frame under maxMbps (the
 *                              reference's rate target is 230) and each component under
 *                              compMbps (200); replaces dciLimits (src/core/rate_control.h:30)
 *   gb_empty_codestream_bytes  the codestream with no pass: the smallest budget that can be
 *                              met (emptyCodestreamBytes, src/core/t2.h:47)
 *   gb_build_codestream        Tier-2 packets and the DCI codestream with passes[i] coding
 *                              passes of block i (buildCodestream, src/core/t2.h:41); label +
 *                              " " + tag (tag at most 9 bytes, none when empty) is the COM text
 *   gb_rate_and_build          PCRD rate control under gb_dci_limits(fps, maxMbps, compMbps),
 *                              then the codestream (allocateRate, src/core/rate_control.h:32,
 *                              followed by buildCodestream, as src/core/pipeline.cpp:210-219);
 *                              passesOut: one byte per block; out may be NULL to get the size
 *   gb_rate_and_build_hull     gb_rate_and_build taking each block's PCRD hull points instead of
 *                              computing them (the convex hull of buildHull,
 *                              src/core/rate_control.cpp:38-86): hullPasses/hullSlope as
 *                              gb_tier1_hull lays them out, e.g. from gb_engine_hull; the
 *                              result is the same as gb_rate_and_build's
 *   gb_device_rate_and_build   gb_rate_and_build on a GPU: the Tier-1 frame (host memory) is
 *                              uploaded; its hull points, slope histogram, every size
 *                              measurement of the threshold search and the final packets are
 *                              computed there (the host runs only the search over a few numbers
 *                              per measurement); the same codestream, passes and lambda
 *   gb_tier1_hull              the hull points on the host: per pass slot of the Tier-1 frame
 *                              (numPasses entries), block i's points from its passBase on, in
 *                              order, each the coding passes at the point and the slope from
 *                              the previous point (distortion reduction per byte, +inf for no
 *                              added bytes); a block's points end at its pass count or at the
 *                              first entry with passes 0
 *   gb_check_dci               DCI compliance of a codestream at fps: *ok 1 or 0, msg the COM
 *                              text or the first error (checkDciCodestream,
 *                              src/core/codestream_check.h:33)
 *   gb_parse_codestream        a DCI codestream read back for decoder_decode: its bands
 *                              (geometry and signalled steps) and per-block code
 *                              (parseCodestream + parsePackets, src/core/codestream_parse.h:53,
 *                              src/core/t2_parse.h:27); arrays may be NULL to get the counts */
GB_API int gb_dci_limits(double fps, double maxMbps, double compMbps, uint64_t* total, uint64_t* comp);
GB_API int gb_empty_codestream_bytes(const GailCudaLayout* layout, const char* label, uint64_t* bytes);
GB_API int gb_build_codestream(const GailCudaLayout* layout, const GailCudaTier1* t1, const uint8_t* passes,
                               const char* label, const char* tag, uint8_t* out, uint64_t cap, uint64_t* size);
GB_API int gb_rate_and_build(const GailCudaLayout* layout, const GailCudaTier1* t1, double fps, double maxMbps,
                             double compMbps, const char* label, const char* tag, uint8_t* passesOut, uint8_t* out,
                             uint64_t cap, uint64_t* size, double* lambda);
GB_API int gb_rate_and_build_hull(const GailCudaLayout* layout, const GailCudaTier1* t1, const uint8_t* hullPasses,
                                  const double* hullSlope, double fps, double maxMbps, double compMbps,
                                  const char* label, const char* tag, uint8_t* passesOut, uint8_t* out, uint64_t cap,
                                  uint64_t* size, double* lambda);
GB_API int gb_device_rate_and_build(int device, const GailCudaLayout* layout, const GailCudaTier1* t1, double fps,
                                    double maxMbps, double compMbps, const char* label, const char* tag,
                                    uint8_t* passesOut, uint8_t* out, uint64_t cap, uint64_t* size, double* lambda);
GB_API int gb_tier1_hull(const GailCudaLayout* layout, const GailCudaTier1* t1, uint8_t* passes, double* slope);
GB_API int gb_check_dci(const uint8_t* data, uint64_t size, double fps, char* msg, uint64_t msgCap, int* ok);
GB_API int gb_parse_codestream(const uint8_t* data, uint64_t size, GbSubband* bands, int maxBands, int* numBands,
                               GbCblkCode* blocks, uint64_t maxBlocks, uint64_t* numBlocks, int* width, int* height,
                               int* profile);

/* FNV hash of the ABI structure sizes, as the plugin table's `layout` field carries it
 * (cudaPluginLayout, src/cuda/cuda_plugin.h:208-217). */
GB_API uint64_t gb_plugin_layout_hash(void);

#ifdef __cplusplus
}
#endif

#endif
