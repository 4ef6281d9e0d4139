// The batched, served encode path: frames of any number of profiles in flight on one GPU,
// continuous batching of their Tier-1 work. No counterpart in the reference (whose
// per-frame slots each run their own launches); it sits beside the plain path of
// encoder.h, which stays the drop-in and the comparison.
//
// A request's life: submit() queues it; the engine thread admits it into a frame slot
// when one is free or the HBM budget allows a new one; the slot's front end (upload,
// colour, wavelet, quantisation) runs as one CUDA graph on the front stream; every frame
// whose front end has finished joins the next Tier-1 batch, one launch of the Tier-1
// kernels over all their code-blocks (largest first across frames), with two batches in
// flight so that one batch's serial MQ tail overlaps the next batch's work; packing
// writes each frame's Tier1Frame straight into mapped host memory. With codestreams on,
// a pool of host workers then makes each frame's DCI codestream (PCRD rate control,
// Tier-2, optionally the DCI check) while the GPU carries on with later frames. wait()
// hands out finished frames, release() frees their slots.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "color.h"
#include "decoder.h"
#include "encoder.h"
#include "gail_cuda_plugin_abi.h"
#include "layout.h"
#include "t1_encode.cuh"

namespace gb {

class EncodeEngine {
public:
    // maxBatch: most frames per Tier-1 launch; hbmBudget: device bytes the engine's frame
    // slots may take (0: 90 % of what is free when the engine starts).
    EncodeEngine(int device, uint64_t hbmBudget, int maxBatch);
    // Batch policy: at most maxBatch frames per Tier-1 launch; while another batch keeps the
    // GPU busy, a batch waits to gather minBatchPct % of maxBatch ready frames, but not longer
    // than maxWaitMs after its oldest frame arrived (defaults 25 % and 2 ms).
    void setPolicy(int maxBatch, int minBatchPct, double maxWaitMs);
    ~EncodeEngine();
    EncodeEngine(const EncodeEngine&) = delete;
    EncodeEngine& operator=(const EncodeEngine&) = delete;

    // A frame class: one layout, input format and colour setting. Returns its id and the
    // device bytes one of its frames in flight takes.
    int addClass(const GailCudaLayout& layout, const GailCudaEncodeSettings& s, uint64_t* frameBytes);
    // Makes frame slots for class cls now, on the calling thread, until it has n (or the
    // budget is spent); returns how many it has. Slots asked for while serving are made by
    // the slot thread instead, one at a time.
    int reserve(int cls, int n);
    // Queues a frame of class cls: frame is host memory (pinned for a fast upload) or,
    // with onDevice, device memory; it must stay valid until the frame is released.
    int64_t submit(int cls, const void* frame, bool onDevice, double slope);
    // Waits up to timeoutMs for a finished frame. Returns false on timeout. latency: ms
    // from submit() to the end of its packing; status: 0 or a GailCudaStatus.
    bool wait(int timeoutMs, int64_t* id, GailCudaTier1* out, double* latencyMs, int* status);
    void release(int64_t id);

    // Codestreams for every frame from now on: rate control to the DCI budgets at fps
    // (whole frame under maxMbps, each component under compMbps), the COM text label +
    // " " + tag, the DCI check when check is set, on `threads` host workers.
    // onDevice: rate control and Tier-2 on the device (the Tier-1 frame stays there; only
    // the codestream and a few numbers per size measurement come back), else on the host
    // workers from the Tier-1 frame in host memory; tier1: the Tier-1 frame (and its hull
    // points) also in host memory for wait() / hull() (always so on the host path).
    struct CodestreamConfig {
        double fps = 24.0, maxMbps = 230.0, compMbps = 200.0;
        std::string label, tag;
        bool check = true;
        int threads = 4;
        bool onDevice = true, tier1 = false;
    };
    void setCodestream(const CodestreamConfig& c);
    // Tier-1 early termination as libgail's pipeline drives it (src/core/pipeline.cpp:194-217):
    // with factor > 0 each encode admitted from now on stops coding a block's bit-planes
    // below the threshold lastLambda x factor, lastLambda being the smallest per-component
    // slope threshold of the rate control of the frame finished last (0 at first: every
    // pass); a frame whose own threshold comes out below the one it was coded with is coded
    // again with every pass before its codestream is made. Needs codestreams on.
    void setSlopeFactor(double factor);
    // The early-termination threshold a finished encode was first coded with, and whether
    // it was coded again with every pass.
    bool frameInfo(int64_t id, double* threshold, int* recoded);
    // The codestream of a finished frame (valid until release): its bytes and whether it
    // passed the DCI check (-1 when not checked). False when codestreams are off.
    bool codestream(int64_t id, const uint8_t** data, uint64_t* size, int* dciOk);

    // Decode requests beside the encodes. A decode class is a layout and decode settings;
    // its frames in flight take decoder slots from the same HBM budget. A decode request
    // (the codestream is copied on submit) is parsed, decoded and handed out by the host
    // workers (those of setCodestream, or four started with the first decode class), each
    // slot on its own stream, so decodes overlap each other and the encode batches. The
    // class's slots (three per worker, as the budget allows) are made when it is added and
    // none while serving: a decode waits for a slot whose picture was released, so a caller
    // that keeps more pictures than that unreleased holds the workers up.
    int addDecodeClass(const GailCudaLayout& layout, const GailCudaDecodeSettings& s, uint64_t* frameBytes);
    int64_t submitDecode(int cls, const uint8_t* data, uint64_t size);
    // The picture of a finished decode (valid until release): height rows of width x 3
    // codes. False for an encode request.
    bool picture(int64_t id, const uint16_t** pix, int* width, int* height);
    // The PCRD hull points of a finished encode (valid until release), computed on the GPU
    // after Tier-1, in the HullView layout over its Tier-1 frame. False for a decode.
    bool hull(int64_t id, const uint8_t** passes, const double** slope);

    struct Stats {
        uint64_t frames = 0, batches = 0, batchFrames = 0, slots = 0, slotBytes = 0;
        uint64_t h2dBytes = 0, d2hBytes = 0;  // bytes copied between host and device for encodes
        uint64_t launches = 0;                // kernels launched for encodes
    };
    Stats stats() const;

    // Per-stage times of the served path while on (CUDA events on the streams the work runs
    // on; a little overhead, so off by default): each frame's front end (its CUDA graph:
    // colour, wavelet, quantisation; the upload before it not included), and per Tier-1
    // batch its context modelling, ordering, MQ coding with truncation lengths, and packing
    // (elapsed on the batch stream: the two batches in flight and the front ends share the
    // GPU meanwhile). Rate control and Tier-2 on the device: host wall time of each frame's
    // round trips on its worker.
    struct StageTimes {
        double frontMs = 0, cmMs = 0, orderMs = 0, mqMs = 0, packMs = 0, rcMs = 0;
        uint64_t frontFrames = 0, batches = 0, batchFrames = 0, rcFrames = 0;
    };
    void setStageTiming(bool on);
    StageTimes stageTimes(bool reset);
    // Decode requests, always counted: host ms spent waiting for a free decoder slot,
    // parsing, and in the slot (enqueue to finish: upload, device stages, picture back);
    // decodes done; decoder slots made after their class was added (each one allocates).
    struct DecodeTimes {
        double waitMs = 0, parseMs = 0, runMs = 0;
        uint64_t decodes = 0, slotsMadeLater = 0;
    };
    DecodeTimes decodeTimes(bool reset);

private:
    struct Class;
    struct Slot;
    struct Request;
    struct Batch;
    struct DecClass;
    struct DecSlot;

    void run();
    void codestreamWorker(int id);
    void decodeJob(Request* r);
    void startWorkers(int n);
    void prepareRc();
    bool admit();
    bool launchBatch(Batch& b);
    bool collect(Batch& b);
    Slot* newSlot(int cls);
    void slotMaker();
    DecSlot* newDecSlot(int cls);
    void sizeBatches();
    void growBatch(Batch& b, uint64_t blocks, uint64_t poolBytes);
    static uint64_t poolShare(uint64_t arena);
    uint64_t budgetLocked();  // under budgetM_

    int dev_;
    uint64_t budget_ = 0, used_ = 0;  // used_ under budgetM_
    bool budgetAuto_ = false;        // budget_ set when the first slot is made
    std::mutex budgetM_;
    std::mutex tablesM_;             // the batches' tables and pools while they are set up
    int maxBatch_;
    int minBatchPct_ = 25;
    double maxWaitMs_ = 2.0;
    // front ends on two streams, a slot on the one its index picks, so that two frames'
    // front ends can run at once (each stream has its own LL scratch planes per class)
    static constexpr int kFronts = 2;
    cudaStream_t front_[kFronts] = {};
    cudaStream_t copy_ = nullptr;  // frame uploads
    std::vector<std::unique_ptr<Class>> classes_;
    std::vector<std::unique_ptr<Slot>> slots_;
    std::vector<std::unique_ptr<Batch>> batches_;
    float* dSlope_ = nullptr;  // per slot
    float* hSlope_ = nullptr;
    std::vector<std::unique_ptr<Request>> requests_;  // owned; index = id - base
    int64_t nextId_ = 0;

    mutable std::mutex m_;
    std::condition_variable cvDone_, cvWork_;
    std::deque<Request*> pending_;    // submitted, not admitted
    int encActive_ = 0;               // encode requests admitted and not yet finished
    // frame slots are made on a thread of their own: device memory, pinned host memory and a
    // graph take tens of milliseconds, in which the serving thread would launch nothing
    std::thread maker_;
    std::condition_variable cvMake_;
    std::deque<int> makeQ_;           // classes a slot is wanted for
    std::vector<int> making_;         // per class: slots asked for, not yet made
    bool slotsFull_ = false;          // a slot could not be made (budget or memory): ask no more
    int nextSlotIndex_ = 0;           // a slot's index into the per-slot arrays (under m_)
    std::vector<Request*> front_q_;   // front end enqueued, not yet in a batch
    std::deque<Request*> done_;       // finished, not yet handed out
    std::atomic<bool> stop_{false};
    std::atomic<double> slopeFactor_{0.0}, lastLambda_{0.0};
    float* hZero_ = nullptr;  // a pinned 0 threshold for frames coded again
    std::string error_;
    Stats stats_;
    std::atomic<bool> timing_{false};
    StageTimes times_;  // under m_
    DecodeTimes decTimes_;  // under m_
    std::thread worker_;
    // codestream stage
    CodestreamConfig cs_;
    bool csOn_ = false;
    std::deque<Request*> csq_;  // Tier-1 done, codestream to make; or a decode to run
    std::condition_variable cvCs_;
    std::vector<std::thread> csWorkers_;
    // per worker: its stream and a device rate control per frame class, made before any
    // frame needs them (their buffers are allocated once, not while frames are served)
    struct WorkerRc;
    std::vector<std::unique_ptr<WorkerRc>> workerRc_;
    // decode requests
    std::vector<std::unique_ptr<DecClass>> decClasses_;
    std::vector<std::unique_ptr<DecSlot>> decSlots_;
    std::condition_variable cvDecSlot_;
};

}  // namespace gb
