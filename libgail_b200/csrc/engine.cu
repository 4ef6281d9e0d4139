// The batched, served encode engine (see engine.h).
#include "engine.h"

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>

#include "capi_util.h"
#include "codestream.h"
#include "common.cuh"
#include "compact.cuh"
#include "frontend.cuh"
#include "rate_gpu.h"
#include "tuning.h"

namespace gb {

namespace {

using Clock = std::chrono::steady_clock;

// A frame's Tier-1 jobs into a batch: the decision and codeword regions, stored as offsets,
// become pointers into the frame's share of the batch's pools.
__global__ void placeJobsKernel(const T1Job* src, T1Job* dst, uint32_t n, uint8_t* sym, uint8_t* cw) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T1Job j = src[i];
    j.sym = sym + reinterpret_cast<uintptr_t>(j.sym);
    j.cw = cw + reinterpret_cast<uintptr_t>(j.cw);
    dst[i] = j;
}

void placeJobs(const T1Job* src, T1Job* dst, uint32_t n, uint8_t* sym, uint8_t* cw, cudaStream_t st) {
    if (!n) return;
    placeJobsKernel<<<(n + 255) / 256, 256, 0, st>>>(src, dst, n, sym, cw);
    GB_CHECK(cudaGetLastError());
}

double msBetween(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

constexpr uint32_t kBatchSoloFloor = 16384;  // MQ solo threshold of batched launches, at least
constexpr int kMaxSlots = 1024;               // frame slots an engine makes at most (per-slot arrays)

struct EncodeEngine::Class {
    Layout L;
    GailCudaEncodeSettings s;
    SlotSizes z;
    ColorTables color;
    ColorArgs colorArgs{};
    float* dEotf = nullptr;
    float* dThr = nullptr;
    float* dLut = nullptr;  // the application 3D LUT, if the colour route takes one
    float* dLL[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // per front stream
    double* dScale = nullptr;  // per block: the hull's distortion weight
    uint64_t slotBytes = 0, dataCap = 0;
    std::vector<Slot*> free;
    std::vector<void*> dev;
};

struct EncodeEngine::Slot {
    int cls = 0, index = 0;
    uint8_t* dIn = nullptr;
    uint32_t* dCoeffs = nullptr;
    // its blocks' Tier-1 jobs; their decision and codeword regions are offsets into the
    // frame's share of a batch's pools, made pointers when the frame joins a batch
    T1Job* dJobs = nullptr;
    uint32_t n = 0;
    // the packed Tier-1 frame, written by the device straight into mapped host memory
    uint32_t *hInfo = nullptr, *hLen = nullptr, *hTot = nullptr;
    int32_t* hDist = nullptr;
    uint8_t* hData = nullptr;
    uint8_t* hHullPasses = nullptr;  // the PCRD hull points, packed like hLen
    double* hHullSlope = nullptr;
    // the packed Tier-1 frame and hull points in device memory, for device rate control
    uint32_t *dInfoP = nullptr, *dLenP = nullptr;
    uint8_t *dDataP = nullptr, *dHullP = nullptr;
    double* dHullS = nullptr;
    uint64_t dataCap = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graphKernels = 0;  // kernel launches one front-end graph makes
    cudaEvent_t frontDone = nullptr;
    cudaEvent_t upDone = nullptr;  // the frame's upload (on the copy stream) is done
    cudaEvent_t frontT[2] = {};    // stage timing: around the front-end graph
    std::vector<void*> dev, host;
};

struct EncodeEngine::Request {
    int64_t id = 0;
    int cls = 0;
    const void* frame = nullptr;
    bool onDevice = false;
    double slope = 0;
    Clock::time_point t0;
    double latency = 0;
    Slot* slot = nullptr;
    uint32_t jobBase = 0;
    int status = 0;
    double thr = 0;         // the early-termination threshold it was first coded with
    bool recoded = false;   // coded again with every pass
    bool tier1 = true;      // the Tier-1 frame was packed into host memory
    bool devFrame = false;  // ... and into the slot's device buffers
    bool frontTimed = false;  // its front end was bracketed by the slot's timing events
    std::vector<uint8_t> cs;  // the codestream, when the engine makes them
    int dciOk = -1;
    // decode requests
    bool decode = false;
    std::vector<uint8_t> input;  // the codestream to decode
    DecSlot* dslot = nullptr;
    const uint16_t* pix = nullptr;
};

struct EncodeEngine::DecClass {
    Layout L;
    GailCudaDecodeSettings s;
    uint64_t slotBytes = 0;
    std::vector<DecSlot*> free;
};

struct EncodeEngine::DecSlot {
    int cls = 0;
    std::unique_ptr<DecoderSlot> slot;
};

struct EncodeEngine::WorkerRc {
    cudaStream_t st = nullptr;
    std::vector<std::unique_ptr<DeviceRateControl>> rc;  // by frame class
    ~WorkerRc() {
        rc.clear();
        if (st) cudaStreamDestroy(st);
    }
};

struct EncodeEngine::Batch {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    T1Job* dJobs = nullptr;
    uint32_t *info = nullptr, *end = nullptr, *len = nullptr, *perm = nullptr, *ctl = nullptr, *hCtl = nullptr,
             *work = nullptr;
    int32_t* dist = nullptr;
    uint4* snaps = nullptr;
    uint2* offs = nullptr;
    uint8_t* hullPasses = nullptr;
    double* hullSlope = nullptr;
    uint32_t cap = 0;
    // the decision and codeword regions of every frame in the batch, each frame's at the
    // offset its jobs were given (worst case of its blocks, as the arenas of a plain encoder)
    uint8_t *symPool = nullptr, *cwPool = nullptr;
    uint64_t poolCap = 0;
    std::vector<Request*> frames;
    bool busy = false;
    std::vector<void*> dev, pools;
    // stage timing: start, after context modelling, after ordering, after MQ and
    // truncation lengths, after packing
    cudaEvent_t t[5] = {};
    bool timed = false;
};

EncodeEngine::EncodeEngine(int device, uint64_t hbmBudget, int maxBatch) : dev_(device), maxBatch_(std::max(1, maxBatch)) {
    GB_CHECK(cudaSetDevice(dev_));
    ensureDevice();
    // 0: 90 % of what is free when the first slot is made (after the batches' pools, which
    // the classes size)
    budgetAuto_ = hbmBudget == 0;
    budget_ = hbmBudget;
    for (auto& f : front_) GB_CHECK(cudaStreamCreateWithFlags(&f, cudaStreamNonBlocking));
    GB_CHECK(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
    check(cudaMalloc(&dSlope_, kMaxSlots * 4), "device memory for the engine");
    check(cudaHostAlloc((void**)&hSlope_, kMaxSlots * 4, cudaHostAllocDefault), "pinned host memory");
    check(cudaHostAlloc((void**)&hZero_, 16, cudaHostAllocDefault), "pinned host memory");
    *hZero_ = 0.f;
    for (int i = 0; i < 2; ++i) batches_.push_back(std::make_unique<Batch>());
    for (auto& b : batches_) {
        GB_CHECK(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking));
        GB_CHECK(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
        for (auto& e : b->t) GB_CHECK(cudaEventCreate(&e));
        check(cudaHostAlloc((void**)&b->hCtl, 64, cudaHostAllocDefault), "pinned host memory");
    }
    worker_ = std::thread([this] { run(); });
    maker_ = std::thread([this] { slotMaker(); });
}

EncodeEngine::~EncodeEngine() {
    {
        std::lock_guard<std::mutex> lock(m_);  // so that no worker misses the wake-up
        stop_ = true;
    }
    cvWork_.notify_all();
    cvMake_.notify_all();
    if (maker_.joinable()) maker_.join();
    if (worker_.joinable()) worker_.join();
    cvCs_.notify_all();
    for (auto& t : csWorkers_)
        if (t.joinable()) t.join();
    cudaSetDevice(dev_);
    cudaDeviceSynchronize();
    workerRc_.clear();
    for (auto& s : slots_) {
        if (s->exec) cudaGraphExecDestroy(s->exec);
        if (s->graph) cudaGraphDestroy(s->graph);
        if (s->frontDone) cudaEventDestroy(s->frontDone);
        if (s->upDone) cudaEventDestroy(s->upDone);
        for (auto e : s->frontT)
            if (e) cudaEventDestroy(e);
        for (void* p : s->dev) cudaFree(p);
        for (void* p : s->host) cudaFreeHost(p);
    }
    for (auto& c : classes_)
        for (void* p : c->dev) cudaFree(p);
    for (auto& b : batches_) {
        for (void* p : b->dev) cudaFree(p);
        for (void* p : b->pools) cudaFree(p);
        if (b->hCtl) cudaFreeHost(b->hCtl);
        if (b->done) cudaEventDestroy(b->done);
        for (auto e : b->t)
            if (e) cudaEventDestroy(e);
        if (b->st) cudaStreamDestroy(b->st);
    }
    if (dSlope_) cudaFree(dSlope_);
    if (hSlope_) cudaFreeHost(hSlope_);
    if (hZero_) cudaFreeHost(hZero_);
    for (auto f : front_)
        if (f) cudaStreamDestroy(f);
    if (copy_) cudaStreamDestroy(copy_);
    cudaGetLastError();
}

int EncodeEngine::addClass(const GailCudaLayout& layout, const GailCudaEncodeSettings& s, uint64_t* frameBytes) {
    GB_CHECK(cudaSetDevice(dev_));
    auto c = std::make_unique<Class>();
    layoutFromAbi(layout, c->L);
    if (c->L.levels < 1) throw std::logic_error("the encoder needs at least one decomposition level");
    if (s.input.width != c->L.width || s.input.height != c->L.height)
        throw std::logic_error("input frame size differs from the layout");
    c->s = s;
    c->z = slotSizes(c->L, s.input);
    c->color = buildColorTables(s.color);
    auto alloc = [&](auto*& p, uint64_t bytes) {
        void* q = nullptr;
        check(cudaMalloc(&q, std::max<uint64_t>(bytes, 16)), "device memory for the engine");
        c->dev.push_back(q);
        p = static_cast<std::remove_reference_t<decltype(p)>>(q);
    };
    alloc(c->dEotf, 65536 * 4);
    alloc(c->dThr, 4096 * 4);
    alloc(c->dLut, c->color.lut3.size() * 4);
    for (auto& ll : c->dLL) {
        alloc(ll[0], c->z.llFloats * 12);
        alloc(ll[1], c->z.llFloats * 12);
    }
    alloc(c->dScale, c->z.n * 8);
    const std::vector<double> scales = blockScales(c->L);
    GB_CHECK(cudaMemcpy(c->dScale, scales.data(), scales.size() * 8, cudaMemcpyHostToDevice));
    GB_CHECK(cudaMemcpy(c->dEotf, c->color.eotf.data(), 65536 * 4, cudaMemcpyHostToDevice));
    GB_CHECK(cudaMemcpy(c->dThr, c->color.thr.data(), 4096 * 4, cudaMemcpyHostToDevice));
    if (!c->color.lut3.empty())
        GB_CHECK(cudaMemcpy(c->dLut, c->color.lut3.data(), c->color.lut3.size() * 4, cudaMemcpyHostToDevice));
    ColorArgs& a = c->colorArgs;
    a.kind = s.input.kind == GB_FRAME_PLANAR ? 1 : 0;
    a.pp = planarParams(s.input);
    a.eotf = c->dEotf;
    a.thr = c->dThr;
    std::memcpy(a.m, c->color.m, sizeof a.m);
    a.xyz = nullptr;
    a.route = c->color.route;
    a.tone = c->color.tone;
    a.lut3 = c->dLut;
    a.lutN = c->color.lutN;
    const uint64_t n = c->z.n, npix = c->z.npix;
    c->dataCap = c->z.outCap;
    c->slotBytes = c->z.inBytes + n * kCblkArea * 4 + n * sizeof(T1Job) + n * 20 + n * kMaxPasses * (4 + 1 + 8) +
                   c->dataCap;
    if (frameBytes) *frameBytes = c->slotBytes;
    int id;
    {
        std::lock_guard<std::mutex> lock(m_);
        classes_.push_back(std::move(c));
        making_.push_back(0);
        if (csOn_ && cs_.onDevice) prepareRc();
        id = (int)classes_.size() - 1;
    }
    sizeBatches();
    return id;
}

// Tier-1 batch tables and pools for maxBatch frames of the largest class (each pool at most
// kPoolBytes, at least one frame: 8 frames of 4K), made while the batches are idle (at
// set-up), so that serving does not allocate.
constexpr uint64_t kPoolBytes = 8ull << 30;
void EncodeEngine::sizeBatches() {
    uint64_t blocks = 0, pool = 0;
    int mb;
    {
        std::lock_guard<std::mutex> lock(m_);
        for (auto& c : classes_) {
            blocks = std::max<uint64_t>(blocks, c->z.n);
            pool = std::max<uint64_t>(pool, poolShare(c->z.arena));
        }
        mb = maxBatch_;
    }
    if (!blocks) return;
    std::lock_guard<std::mutex> lock(tablesM_);
    for (auto& b : batches_) {
        {
            std::lock_guard<std::mutex> l2(m_);
            if (b->busy) continue;  // sized by launchBatch when it next needs more
        }
        growBatch(*b, blocks * (uint64_t)mb, std::min<uint64_t>(pool * (uint64_t)mb, std::max<uint64_t>(pool, kPoolBytes)));
    }
}

uint64_t EncodeEngine::poolShare(uint64_t arena) { return (arena + 255) & ~(uint64_t)255; }

void EncodeEngine::growBatch(Batch& b, uint64_t blocks, uint64_t poolBytes) {
    if (blocks > b.cap) {
        for (void* p : b.dev) cudaFree(p);
        b.dev.clear();
        b.cap = 0;
        const uint64_t cap = blocks;
        auto alloc = [&](auto*& p, uint64_t bytes) {
            void* q = nullptr;
            check(cudaMalloc(&q, std::max<uint64_t>(bytes, 16)), "device memory for a Tier-1 batch");
            b.dev.push_back(q);
            p = static_cast<std::remove_reference_t<decltype(p)>>(q);
        };
        alloc(b.dJobs, cap * sizeof(T1Job));
        alloc(b.info, cap * 16);
        alloc(b.end, cap * kMaxPasses * 4);
        alloc(b.len, cap * kMaxPasses * 4);
        alloc(b.dist, cap * kMaxPasses * 4);
        alloc(b.snaps, cap * kMaxPasses * 16);
        alloc(b.perm, cap * 4);
        alloc(b.work, t1WorkWords((uint32_t)cap) * 4);
        alloc(b.offs, cap * 8);
        alloc(b.hullPasses, cap * kMaxPasses);
        alloc(b.hullSlope, cap * kMaxPasses * 8);
        alloc(b.ctl, 64);
        b.cap = (uint32_t)cap;
    }
    if (poolBytes > b.poolCap) {
        for (void* p : b.pools) cudaFree(p);
        b.pools.clear();
        b.poolCap = 0;
        b.symPool = b.cwPool = nullptr;
        void* q = nullptr;
        check(cudaMalloc(&q, poolBytes), "device memory for a Tier-1 batch's decision pool");
        b.pools.push_back(q);
        b.symPool = static_cast<uint8_t*>(q);
        check(cudaMalloc(&q, poolBytes), "device memory for a Tier-1 batch's codeword pool");
        b.pools.push_back(q);
        b.cwPool = static_cast<uint8_t*>(q);
        b.poolCap = poolBytes;
    }
}

uint64_t EncodeEngine::budgetLocked() {
    if (budgetAuto_) {
        size_t f = 0, t = 0;
        GB_CHECK(cudaMemGetInfo(&f, &t));
        budget_ = used_ + (uint64_t)(f * 0.9);
        budgetAuto_ = false;
    }
    return budget_;
}

int EncodeEngine::reserve(int cls, int n) {
    int have;
    {
        std::lock_guard<std::mutex> lock(m_);
        if (cls < 0 || cls >= (int)classes_.size()) throw std::logic_error("unknown frame class");
        have = 0;
        for (auto& s : slots_) have += s->cls == cls;
    }
    while (have < n) {
        Slot* s = newSlot(cls);
        if (!s) break;
        std::lock_guard<std::mutex> lock(m_);
        classes_[cls]->free.push_back(s);
        ++have;
        cvWork_.notify_all();
    }
    return have;
}

// Makes the frame slots admit() asks for, one at a time, and hands each to its class.
void EncodeEngine::slotMaker() {
    try {
        GB_CHECK(cudaSetDevice(dev_));
        for (;;) {
            int cls;
            {
                std::unique_lock<std::mutex> lock(m_);
                cvMake_.wait(lock, [&] { return stop_.load() || !makeQ_.empty(); });
                if (stop_) return;
                cls = makeQ_.front();
                makeQ_.pop_front();
            }
            Slot* s = newSlot(cls);
            std::lock_guard<std::mutex> lock(m_);
            --making_[cls];
            if (s) classes_[cls]->free.push_back(s);
            else slotsFull_ = true;
            cvWork_.notify_all();
        }
    } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lock(m_);
        if (error_.empty()) error_ = e.what();
        cvDone_.notify_all();
    }
}

EncodeEngine::Slot* EncodeEngine::newSlot(int cls) {
    Class* cp;
    {
        std::lock_guard<std::mutex> lock(m_);
        cp = classes_[cls].get();
    }
    Class& c = *cp;
    {
        std::lock_guard<std::mutex> lock(budgetM_);
        if (used_ + c.slotBytes > budgetLocked()) return nullptr;
        used_ += c.slotBytes;  // reserved now, given back if the slot cannot be made
    }
    // the slot's index into the per-slot arrays, taken only once the budget allows the slot
    // (the slot thread and reserve() may make slots at once)
    int index;
    {
        std::lock_guard<std::mutex> lock(m_);
        index = nextSlotIndex_ < kMaxSlots ? nextSlotIndex_++ : -1;
    }
    if (index < 0) {
        std::lock_guard<std::mutex> lock(budgetM_);
        used_ -= c.slotBytes;
        return nullptr;
    }
    auto s = std::make_unique<Slot>();
    s->cls = cls;
    s->index = index;
    s->n = (uint32_t)c.z.n;
    auto alloc = [&](auto*& p, uint64_t bytes) {
        void* q = nullptr;
        check(cudaMalloc(&q, std::max<uint64_t>(bytes, 16)), "device memory for a frame slot");
        s->dev.push_back(q);
        p = static_cast<std::remove_reference_t<decltype(p)>>(q);
    };
    auto mapped = [&](auto*& p, uint64_t bytes) {
        void* q = nullptr;
        check(cudaHostAlloc(&q, std::max<uint64_t>(bytes, 16), cudaHostAllocMapped | cudaHostAllocPortable),
              "pinned host memory for a frame slot");
        s->host.push_back(q);
        p = static_cast<std::remove_reference_t<decltype(p)>>(q);
    };
    try {
        alloc(s->dIn, c.z.inBytes);
        alloc(s->dCoeffs, (uint64_t)s->n * kCblkArea * 4);
        alloc(s->dJobs, (uint64_t)s->n * sizeof(T1Job));
        alloc(s->dInfoP, (uint64_t)s->n * 20);
        alloc(s->dLenP, (uint64_t)s->n * kMaxPasses * 4);
        alloc(s->dHullP, (uint64_t)s->n * kMaxPasses);
        alloc(s->dHullS, (uint64_t)s->n * kMaxPasses * 8);
        alloc(s->dDataP, c.dataCap);
        mapped(s->hInfo, (uint64_t)s->n * 20);
        mapped(s->hLen, (uint64_t)s->n * kMaxPasses * 4);
        mapped(s->hDist, (uint64_t)s->n * kMaxPasses * 4);
        mapped(s->hData, c.dataCap);
        mapped(s->hHullPasses, (uint64_t)s->n * kMaxPasses);
        mapped(s->hHullSlope, (uint64_t)s->n * kMaxPasses * 8);
        mapped(s->hTot, 64);
        s->dataCap = c.dataCap;
        std::vector<T1Job> jobs;
        buildJobOffsets(c.L, s->dCoeffs, (uint32_t)s->index, jobs);
        GB_CHECK(cudaMemcpy(s->dJobs, jobs.data(), jobs.size() * sizeof(T1Job), cudaMemcpyHostToDevice));
        GB_CHECK(cudaEventCreateWithFlags(&s->frontDone, cudaEventDisableTiming));
        GB_CHECK(cudaEventCreateWithFlags(&s->upDone, cudaEventDisableTiming));
        for (auto& e : s->frontT) GB_CHECK(cudaEventCreate(&e));
        // the slot's front end as one graph: it always reads the slot's input buffer and
        // writes the slot's coefficient buffer
        cudaStream_t cap;
        GB_CHECK(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
        ColorArgs a = c.colorArgs;
        a.src = s->dIn;
        GB_CHECK(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        const int fs = s->index % kFronts;  // the front stream this slot's frames take
        launchFrontEnd(c.L, a, c.dLL[fs][0], c.dLL[fs][1], c.z.llFloats, s->dCoeffs, nullptr, cap);
        GB_CHECK(cudaStreamEndCapture(cap, &s->graph));
        GB_CHECK(cudaStreamDestroy(cap));
        size_t nodes = 0;
        GB_CHECK(cudaGraphGetNodes(s->graph, nullptr, &nodes));
        std::vector<cudaGraphNode_t> nv(nodes);
        if (nodes) GB_CHECK(cudaGraphGetNodes(s->graph, nv.data(), &nodes));
        for (cudaGraphNode_t nd : nv) {
            cudaGraphNodeType ty;
            GB_CHECK(cudaGraphNodeGetType(nd, &ty));
            if (ty == cudaGraphNodeTypeKernel) ++s->graphKernels;
        }
        GB_CHECK(cudaGraphInstantiate(&s->exec, s->graph, 0));
    } catch (...) {
        for (void* p : s->dev) cudaFree(p);
        for (void* p : s->host) cudaFreeHost(p);
        if (s->exec) cudaGraphExecDestroy(s->exec);
        if (s->graph) cudaGraphDestroy(s->graph);
        if (s->frontDone) cudaEventDestroy(s->frontDone);
        if (s->upDone) cudaEventDestroy(s->upDone);
        for (auto e : s->frontT)
            if (e) cudaEventDestroy(e);
        cudaGetLastError();
        std::lock_guard<std::mutex> lock(budgetM_);
        used_ -= c.slotBytes;
        return nullptr;  // out of memory now: the request waits for a slot to free up
    }
    Slot* raw = s.get();
    uint64_t used;
    {
        std::lock_guard<std::mutex> lock(budgetM_);
        used = used_;
    }
    std::lock_guard<std::mutex> lock(m_);
    slots_.push_back(std::move(s));
    stats_.slots = slots_.size();
    stats_.slotBytes = used;
    return raw;
}

int64_t EncodeEngine::submit(int cls, const void* frame, bool onDevice, double slope) {
    if (!frame) throw std::logic_error("no frame");
    std::lock_guard<std::mutex> lock(m_);
    if (cls < 0 || cls >= (int)classes_.size()) throw std::logic_error("unknown frame class");
    if (!error_.empty()) throw std::runtime_error(error_);
    auto r = std::make_unique<Request>();
    r->id = nextId_++;
    r->cls = cls;
    r->frame = frame;
    r->onDevice = onDevice;
    r->slope = slope;
    r->t0 = Clock::now();
    pending_.push_back(r.get());
    requests_.push_back(std::move(r));
    cvWork_.notify_one();
    return requests_.back()->id;
}

bool EncodeEngine::wait(int timeoutMs, int64_t* id, GailCudaTier1* out, double* latencyMs, int* status) {
    std::unique_lock<std::mutex> lock(m_);
    if (!cvDone_.wait_for(lock, std::chrono::milliseconds(timeoutMs), [&] { return !done_.empty() || !error_.empty(); }))
        return false;
    if (done_.empty()) throw std::runtime_error(error_);
    Request* r = done_.front();
    done_.pop_front();
    *id = r->id;
    *latencyMs = r->latency;
    *status = r->status;
    const Slot* s = r->slot;
    if (r->decode || !s || !r->tier1) *out = GailCudaTier1{};
    else *out = {reinterpret_cast<const GbCblkInfo*>(s->hInfo), s->hLen, s->hDist, s->hData, s->n, s->hTot[1], s->hTot[0]};
    return true;
}

void EncodeEngine::release(int64_t id) {
    std::lock_guard<std::mutex> lock(m_);
    if (id < 0 || id >= (int64_t)requests_.size() || !requests_[id]) throw std::logic_error("unknown request");
    Request* r = requests_[id].get();
    if (r->decode) {
        if (r->dslot) {
            decClasses_[r->cls]->free.push_back(r->dslot);
            cvDecSlot_.notify_all();
        }
        requests_[id].reset();
        return;
    }
    if (!r->slot) throw std::logic_error("request not finished");
    classes_[r->cls]->free.push_back(r->slot);
    requests_[id].reset();
    cvWork_.notify_one();
}

void EncodeEngine::setPolicy(int maxBatch, int minBatchPct, double maxWaitMs) {
    if (maxBatch < 1 || maxBatch > 1024 || minBatchPct < 0 || minBatchPct > 100 || !(maxWaitMs >= 0) || maxWaitMs > 1000)
        throw std::logic_error("batch policy out of range");
    {
        std::lock_guard<std::mutex> lock(m_);
        maxBatch_ = maxBatch;
        minBatchPct_ = minBatchPct;
        maxWaitMs_ = maxWaitMs;
    }
    sizeBatches();
}

void EncodeEngine::setCodestream(const CodestreamConfig& c) {
    if (c.threads < 1 || c.threads > 256) throw std::logic_error("codestream workers out of range");
    if (c.tag.size() > kMaxDeviceTagBytes) throw std::logic_error("device tag too long");
    const RateLimits lim = dciLimits(c.fps, c.maxMbps, c.compMbps);
    for (auto& cl : classes_) {
        CodestreamWriter w(cl->L, c.label);
        if (w.emptyBytes() > lim.maxTotal) throw std::logic_error("the frame budget is below the smallest codestream");
    }
    std::lock_guard<std::mutex> lock(m_);
    if (csOn_) throw std::logic_error("codestreams are already on");
    cs_ = c;
    startWorkers(c.threads);
    if (c.onDevice) prepareRc();
    csOn_ = true;
}

// Grows the pool of host workers to at least n (m_ held).
void EncodeEngine::startWorkers(int n) {
    while ((int)csWorkers_.size() < n) {
        const int id = (int)csWorkers_.size();
        csWorkers_.emplace_back([this, id] { codestreamWorker(id); });
    }
}

// A stream and a device rate control per frame class for every worker (m_ held).
void EncodeEngine::prepareRc() {
    GB_CHECK(cudaSetDevice(dev_));
    const RateLimits lim = dciLimits(cs_.fps, cs_.maxMbps, cs_.compMbps);
    const size_t hint = 2 * lim.maxTotal + (64u << 10);
    while (workerRc_.size() < csWorkers_.size()) workerRc_.push_back(std::make_unique<WorkerRc>());
    for (auto& w : workerRc_) {
        if (!w->st) {
            int lo = 0, hi = 0;
            GB_CHECK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
            GB_CHECK(cudaStreamCreateWithPriority(&w->st, cudaStreamNonBlocking, hi));
        }
        while (w->rc.size() < classes_.size())
            w->rc.push_back(std::make_unique<DeviceRateControl>(dev_, classes_[w->rc.size()]->L, cs_.label, hint));
    }
}

int EncodeEngine::addDecodeClass(const GailCudaLayout& layout, const GailCudaDecodeSettings& s, uint64_t* frameBytes) {
    GB_CHECK(cudaSetDevice(dev_));
    auto c = std::make_unique<DecClass>();
    layoutFromAbi(layout, c->L);
    if (s.reduce < 0 || s.reduce > c->L.levels) throw std::logic_error("more resolution levels left out than the layout has");
    c->s = s;
    c->slotBytes = decoderSlotBytes(c->L, s);
    if (frameBytes) *frameBytes = c->slotBytes;
    int cls, workers;
    {
        std::lock_guard<std::mutex> lock(m_);
        decClasses_.push_back(std::move(c));
        startWorkers(4);
        if (csOn_ && cs_.onDevice) prepareRc();
        cls = (int)decClasses_.size() - 1;
        workers = (int)csWorkers_.size();
    }
    // three slots per host worker now (one decoding, up to two holding pictures not yet
    // released), while the HBM budget has room: making one while serving (device memory,
    // pinned host memory) stalls its worker and the device, so decodes wait for a released
    // slot instead, and only a class left without any slot makes one later
    for (int i = 0; i < 3 * workers; ++i) {
        DecSlot* ds = nullptr;
        try {
            ds = newDecSlot(cls);
        } catch (const std::exception&) {  // out of memory now: slots are made on demand
            cudaGetLastError();
        }
        if (!ds) break;
        std::lock_guard<std::mutex> lock(m_);
        decClasses_[cls]->free.push_back(ds);
    }
    return cls;
}

// A new decoder slot of decode class cls, or NULL when the HBM budget has no room.
EncodeEngine::DecSlot* EncodeEngine::newDecSlot(int cls) {
    DecClass* c;
    {
        std::lock_guard<std::mutex> lock(m_);
        c = decClasses_[cls].get();
    }
    {
        std::lock_guard<std::mutex> lock(budgetM_);
        if (used_ + c->slotBytes > budgetLocked()) return nullptr;
        used_ += c->slotBytes;
    }
    auto d = std::make_unique<DecSlot>();
    d->cls = cls;
    try {
        d->slot = std::make_unique<DecoderSlot>(dev_, c->L, c->s, false);  // several decode at once
    } catch (...) {
        std::lock_guard<std::mutex> lock(budgetM_);
        used_ -= c->slotBytes;
        throw;
    }
    DecSlot* ds = d.get();
    std::lock_guard<std::mutex> lock(m_);
    decSlots_.push_back(std::move(d));
    return ds;
}

int64_t EncodeEngine::submitDecode(int cls, const uint8_t* data, uint64_t size) {
    if (!data || size == 0) throw std::logic_error("no codestream");
    auto r = std::make_unique<Request>();
    r->decode = true;
    r->cls = cls;
    r->input.assign(data, data + size);
    r->t0 = Clock::now();
    std::lock_guard<std::mutex> lock(m_);
    if (cls < 0 || cls >= (int)decClasses_.size()) throw std::logic_error("unknown decode class");
    if (!error_.empty()) throw std::runtime_error(error_);
    r->id = nextId_++;
    csq_.push_back(r.get());
    requests_.push_back(std::move(r));
    cvCs_.notify_one();
    return requests_.back()->id;
}

bool EncodeEngine::picture(int64_t id, const uint16_t** pix, int* width, int* height) {
    std::lock_guard<std::mutex> lock(m_);
    if (id < 0 || id >= (int64_t)requests_.size() || !requests_[id]) throw std::logic_error("unknown request");
    const Request* r = requests_[id].get();
    if (!r->decode) return false;
    *pix = r->pix;
    *width = r->dslot ? r->dslot->slot->outW() : 0;
    *height = r->dslot ? r->dslot->slot->outH() : 0;
    return true;
}

bool EncodeEngine::hull(int64_t id, const uint8_t** passes, const double** slope) {
    std::lock_guard<std::mutex> lock(m_);
    if (id < 0 || id >= (int64_t)requests_.size() || !requests_[id]) throw std::logic_error("unknown request");
    const Request* r = requests_[id].get();
    if (r->decode || !r->slot || !r->tier1) return false;
    *passes = r->slot->hHullPasses;
    *slope = r->slot->hHullSlope;
    return true;
}

// A decode request on a worker: parse, a decoder slot of its class (made when the budget
// allows, else the next one released), decode on the slot's stream, hand out.
void EncodeEngine::decodeJob(Request* r) {
    DecClass* c;
    {
        std::lock_guard<std::mutex> lock(m_);
        c = decClasses_[r->cls].get();
    }
    Layout frame;
    std::vector<GbCblkCode> blocks;
    const auto t0 = Clock::now();
    auto t1 = t0, t2 = t0;
    bool made = false;
    try {
        parseCodestream(r->input.data(), r->input.size(), frame, blocks);
        if (frame.width != c->L.width || frame.height != c->L.height || frame.levels != c->L.levels)
            throw std::runtime_error("codestream of another frame size than its decode class");
        t1 = Clock::now();
        DecSlot* ds = nullptr;
        for (;;) {
            {
                std::unique_lock<std::mutex> lock(m_);
                if (!c->free.empty()) {
                    ds = c->free.back();
                    c->free.pop_back();
                    break;
                }
            }
            bool none;
            {
                std::lock_guard<std::mutex> lock(m_);
                none = std::none_of(decSlots_.begin(), decSlots_.end(), [&](auto& d) { return d->cls == r->cls; });
            }
            if (none) {
                ds = newDecSlot(r->cls);
                if (ds) {
                    made = true;
                    break;
                }
            }
            std::unique_lock<std::mutex> lock(m_);  // no room: the next released slot
            cvDecSlot_.wait_for(lock, std::chrono::milliseconds(50), [&] { return !c->free.empty() || stop_.load(); });
            if (stop_) throw std::runtime_error("engine stopping");
        }
        t2 = Clock::now();
        r->dslot = ds;
        ds->slot->enqueue(frame, r->input.data(), r->input.size(), blocks.data(), blocks.size(), false);
        r->pix = ds->slot->finish(nullptr);
        r->status = kOk;
    } catch (const std::exception&) {
        r->status = kError;
    }
    const auto t3 = Clock::now();
    std::lock_guard<std::mutex> lock(m_);
    decTimes_.parseMs += msBetween(t0, t1);
    decTimes_.waitMs += msBetween(t1, t2);
    decTimes_.runMs += msBetween(t2, t3);
    decTimes_.decodes++;
    if (made) decTimes_.slotsMadeLater++;
}

bool EncodeEngine::codestream(int64_t id, const uint8_t** data, uint64_t* size, int* dciOk) {
    std::lock_guard<std::mutex> lock(m_);
    if (id < 0 || id >= (int64_t)requests_.size() || !requests_[id]) throw std::logic_error("unknown request");
    const Request* r = requests_[id].get();
    if (!csOn_) return false;
    *data = r->cs.data();
    *size = r->cs.size();
    *dciOk = r->dciOk;
    return true;
}

void EncodeEngine::codestreamWorker(int id) {
    cudaSetDevice(dev_);
    // one writer per frame class on this worker for the host path (the packet order is
    // flattened once); the device path uses the worker's device rate controls, on its own
    // stream at the highest priority, so that their short launches go ahead of the Tier-1
    // batches
    std::vector<std::unique_ptr<CodestreamWriter>> writers;
    for (;;) {
        Request* r;
        const Class* c = nullptr;
        DeviceRateControl* rc = nullptr;
        cudaStream_t st = nullptr;
        {
            std::unique_lock<std::mutex> lock(m_);
            cvCs_.wait(lock, [&] { return stop_.load() || !csq_.empty(); });
            if (csq_.empty()) return;
            r = csq_.front();
            csq_.pop_front();
            if (!r->decode) {
                c = classes_[r->cls].get();
                if (writers.size() < classes_.size()) writers.resize(classes_.size());
                if (r->devFrame && (size_t)id < workerRc_.size() && (size_t)r->cls < workerRc_[id]->rc.size()) {
                    rc = workerRc_[id]->rc[r->cls].get();
                    st = workerRc_[id]->st;
                }
            }
        }
        if (r->decode) {
            decodeJob(r);
            const auto now = Clock::now();
            std::lock_guard<std::mutex> lock(m_);
            r->latency = msBetween(r->t0, now);
            done_.push_back(r);
            stats_.frames++;
            cvDone_.notify_all();
            continue;
        }
        Slot* s = r->slot;
        const RateLimits lim = dciLimits(cs_.fps, cs_.maxMbps, cs_.compMbps);
        uint64_t d2h = r->tier1 ? (uint64_t)s->n * 20 + (uint64_t)s->hTot[1] * 17 + s->hTot[0] : 0, launches = 0;
        bool again = false;  // coded with early termination past what rate control keeps: code again
        if (r->status == kOk) {
            try {
                double lam = 0;  // the smallest per-component slope threshold of the rate control
                auto minComp = [](const RateResult& rr) {
                    return std::min({rr.lambdaComp[0], rr.lambdaComp[1], rr.lambdaComp[2]});
                };
                if (r->devFrame) {
                    if (!rc) throw std::logic_error("no device rate control for this worker and class");
                    const DeviceTier1 f{reinterpret_cast<const GbCblkInfo*>(s->dInfoP), s->dLenP, s->dDataP, s->dHullP,
                                        s->dHullS};
                    const auto rc0 = Clock::now();
                    const RateResult rr = rc->run(f, lim, cs_.tag, r->cs, st);
                    if (timing_.load()) {
                        const double ms = msBetween(rc0, Clock::now());
                        std::lock_guard<std::mutex> lock(m_);
                        times_.rcMs += ms;
                        times_.rcFrames++;
                    }
                    d2h += rr.d2hBytes;
                    launches = (uint64_t)rr.launches;
                    lam = minComp(rr);
                    again = r->thr > 0 && !r->recoded && lam < r->thr;
                } else {
                    auto& w = writers[r->cls];
                    if (!w) w = std::make_unique<CodestreamWriter>(c->L, cs_.label);
                    Tier1View v;
                    v.info = reinterpret_cast<const GbCblkInfo*>(s->hInfo);
                    v.passLen = s->hLen;
                    v.passDist = s->hDist;
                    v.data = s->hData;
                    v.numInfo = s->n;
                    v.numPasses = s->hTot[1];
                    v.numData = s->hTot[0];
                    const HullView hull{s->hHullPasses, s->hHullSlope};  // computed on the GPU
                    const RateResult rr = allocateRate(*w, v, lim, &hull);
                    lam = minComp(rr);
                    again = r->thr > 0 && !r->recoded && lam < r->thr;
                    if (!again) w->build(v, rr.passes.data(), &r->cs, cs_.tag);
                }
                if (!again) {
                    lastLambda_.store(lam);
                    if (cs_.check) r->dciOk = checkDci(r->cs.data(), r->cs.size(), cs_.fps).ok ? 1 : 0;
                } else {
                    // the frame is easier than the one its threshold came from: passes the rate
                    // control now keeps may have been left out; its Tier-1 again, every pass
                    // (the coefficients are still in its slot)
                    r->recoded = true;
                    r->cs.clear();
                    GB_CHECK(cudaMemcpyAsync(dSlope_ + s->index, hZero_, 4, cudaMemcpyHostToDevice, copy_));
                    GB_CHECK(cudaEventRecord(s->frontDone, copy_));
                }
            } catch (const std::exception&) {
                r->status = kError;
                again = false;
            }
        }
        std::lock_guard<std::mutex> lock(m_);
        stats_.d2hBytes += d2h;
        stats_.launches += launches;
        if (again) {
            front_q_.push_back(r);
            cvWork_.notify_all();
            continue;
        }
        r->latency = msBetween(r->t0, Clock::now());
        done_.push_back(r);
        --encActive_;
        stats_.frames++;
        cvDone_.notify_all();
    }
}

void EncodeEngine::setSlopeFactor(double factor) {
    if (!(factor >= 0)) throw std::logic_error("slope factor must be 0 or more");
    if (factor > 0) {
        std::lock_guard<std::mutex> lock(m_);
        if (!csOn_) throw std::logic_error("early termination needs codestreams on (its thresholds come from them)");
    }
    slopeFactor_.store(factor);
}

bool EncodeEngine::frameInfo(int64_t id, double* threshold, int* recoded) {
    std::lock_guard<std::mutex> lock(m_);
    if (id < 0 || id >= (int64_t)requests_.size() || !requests_[id]) throw std::logic_error("unknown request");
    const Request* r = requests_[id].get();
    if (r->decode) return false;
    *threshold = r->thr;
    *recoded = r->recoded ? 1 : 0;
    return true;
}

EncodeEngine::Stats EncodeEngine::stats() const {
    std::lock_guard<std::mutex> lock(m_);
    return stats_;
}

void EncodeEngine::setStageTiming(bool on) { timing_.store(on); }

EncodeEngine::DecodeTimes EncodeEngine::decodeTimes(bool reset) {
    std::lock_guard<std::mutex> lock(m_);
    const DecodeTimes t = decTimes_;
    if (reset) decTimes_ = DecodeTimes{};
    return t;
}

EncodeEngine::StageTimes EncodeEngine::stageTimes(bool reset) {
    std::lock_guard<std::mutex> lock(m_);
    const StageTimes t = times_;
    if (reset) times_ = StageTimes{};
    return t;
}

bool EncodeEngine::admit() {
    bool progress = false;
    for (;;) {
        Request* r;
        Slot* s = nullptr;
        {
            std::lock_guard<std::mutex> lock(m_);
            if (pending_.empty()) break;
            r = pending_.front();
            Class& c = *classes_[r->cls];
            if (!c.free.empty()) {
                s = c.free.back();
                c.free.pop_back();
            } else if (!slotsFull_ && making_[r->cls] == 0 && encActive_ < std::max(32, 8 * maxBatch_)) {
                // a new slot, made by the slot thread while this one keeps serving; only
                // while fewer frames than the pipeline's depth are in progress (eight
                // batches: two in Tier-1, the next ones' front ends, the frames whose
                // codestreams the host workers are making): more would only wait, and
                // finished frames whose results the caller still holds do not count
                ++making_[r->cls];
                makeQ_.push_back(r->cls);
                cvMake_.notify_one();
            }
        }
        if (!s) break;  // first in, first admitted: later requests wait too
        {
            std::lock_guard<std::mutex> lock(m_);
            pending_.pop_front();
            ++encActive_;
        }
        Class& c = *classes_[r->cls];
        r->slot = s;
        const double factor = slopeFactor_.load();
        if (factor > 0) r->slope = lastLambda_.load() * factor;  // as libgail's pipeline
        r->thr = r->slope;
        hSlope_[s->index] = (float)r->slope;
        // the upload on the copy stream, so that it overlaps the front ends of the frames
        // before; the front end waits for it
        GB_CHECK(cudaMemcpyAsync(dSlope_ + s->index, hSlope_ + s->index, 4, cudaMemcpyHostToDevice, copy_));
        GB_CHECK(cudaMemcpyAsync(s->dIn, r->frame, c.z.inBytes, r->onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                 copy_));
        GB_CHECK(cudaEventRecord(s->upDone, copy_));
        const cudaStream_t fst = front_[s->index % kFronts];
        GB_CHECK(cudaStreamWaitEvent(fst, s->upDone, 0));
        r->frontTimed = timing_.load() && s->frontT[0];
        if (r->frontTimed) GB_CHECK(cudaEventRecord(s->frontT[0], fst));
        GB_CHECK(cudaGraphLaunch(s->exec, fst));
        if (r->frontTimed) GB_CHECK(cudaEventRecord(s->frontT[1], fst));
        GB_CHECK(cudaEventRecord(s->frontDone, fst));
        std::lock_guard<std::mutex> lock(m_);
        if (!r->onDevice) stats_.h2dBytes += c.z.inBytes;
        stats_.launches += (uint64_t)s->graphKernels;
        front_q_.push_back(r);
        progress = true;
    }
    return progress;
}

bool EncodeEngine::launchBatch(Batch& b) {
    std::vector<Request*> sel;
    std::vector<uint64_t> shares;  // each frame's share of the batch's pools
    {
        std::lock_guard<std::mutex> lock(m_);
        if (front_q_.empty()) return false;
        const bool otherBusy = std::any_of(batches_.begin(), batches_.end(), [&](auto& x) { return x.get() != &b && x->busy; });
        uint64_t pool = 0;
        for (Request* r : front_q_) {
            if ((int)sel.size() >= maxBatch_) break;
            const uint64_t share = poolShare(classes_[r->cls]->z.arena);
            if (!sel.empty() && pool + share > b.poolCap) break;  // the batch's pools are full
            if (cudaEventQuery(r->slot->frontDone) != cudaSuccess) break;  // in order: later ones are not done either
            sel.push_back(r);
            shares.push_back(share);
            pool += share;
        }
        // while the other batch keeps the GPU busy, let small batches grow a little
        if (sel.empty() || (otherBusy && (int)sel.size() < std::max(1, maxBatch_ * minBatchPct_ / 100) &&
                            msBetween(front_q_.front()->t0, Clock::now()) < maxWaitMs_ && sel.size() < front_q_.size()))
            return false;
        front_q_.erase(front_q_.begin(), front_q_.begin() + (long)sel.size());
    }
    std::lock_guard<std::mutex> tables(tablesM_);
    uint64_t total = 0, pool = 0;
    for (size_t i = 0; i < sel.size(); ++i) {
        total += sel[i]->slot->n;
        pool += shares[i];
    }
    if (total > b.cap || pool > b.poolCap)  // a batch larger than set-up foresaw
        growBatch(b, std::max<uint64_t>(total, (uint64_t)b.cap), std::max<uint64_t>(pool, b.poolCap));
    uint32_t base = 0;
    uint64_t poolOff = 0;
    for (size_t i = 0; i < sel.size(); ++i) {
        Request* r = sel[i];
        GB_CHECK(cudaStreamWaitEvent(b.st, r->slot->frontDone, 0));
        // the frame's jobs into the batch, their regions in its share of the pools
        placeJobs(r->slot->dJobs, b.dJobs + base, r->slot->n, b.symPool + poolOff, b.cwPool + poolOff, b.st);
        r->jobBase = base;
        base += r->slot->n;
        poolOff += shares[i];
    }
    GB_CHECK(cudaMemsetAsync(b.ctl, 0, 64, b.st));
    b.timed = timing_.load() && b.t[0];
    if (b.timed) GB_CHECK(cudaEventRecord(b.t[0], b.st));
    T1Launch L{b.dJobs, (uint32_t)total, b.info, b.end, b.len, b.dist, b.snaps, b.perm, b.ctl, dSlope_};
    bool any4k = false;  // a batch with a 4K frame is launched with the 4K tuning
    for (Request* r : sel) any4k = any4k || classes_[r->cls]->L.profile == 1;
    const Tuning tu = tuningFor(any4k ? 1 : 0);
    // the solo threshold is tuned on one-frame launches, where the longest blocks' chains set
    // the time; a batch of frames has enough other blocks to hide them behind, and taking
    // warps for solo blocks below 16,384 decisions cost it throughput (4K served codestreams:
    // 560 per second at 16,384, 530 at 8,192, on B200)
    L.soloDecisions = std::max<uint32_t>(tu.soloDecisions, kBatchSoloFloor);
    L.cmCtasPerSm = (uint16_t)tu.cmCtasPerSm;
    L.mqCtasPerSm = (uint16_t)tu.mqCtasPerSm;
    L.persistent = (uint16_t)tu.t1Persistent;
    L.work = b.work;
    t1Encode(L, b.st, b.timed ? &b.t[1] : nullptr);
    if (b.timed) GB_CHECK(cudaEventRecord(b.t[3], b.st));
    // context modelling, ordering, MQ coding, truncation lengths: four launches or one
    uint64_t launches = tu.t1Persistent ? 1 : 4;
    bool onDevice, tier1;
    {
        std::lock_guard<std::mutex> lock(m_);
        onDevice = csOn_ && cs_.onDevice;
        tier1 = !onDevice || cs_.tier1;
    }
    for (Request* r : sel) {
        Slot* s = r->slot;
        std::memset(s->hTot, 0, 64);
        const uint32_t j = r->jobBase;
        const Class& c = *classes_[r->cls];
        uint8_t* hp = b.hullPasses + (uint64_t)kMaxPasses * j;
        double* hs = b.hullSlope + (uint64_t)kMaxPasses * j;
        if (onDevice) {  // packed into the slot's device buffers, for the device rate control
            CompactArgs ca{s->n, b.info + 4 * (uint64_t)j, b.len + (uint64_t)kMaxPasses * j, b.dist + (uint64_t)kMaxPasses * j,
                           b.dJobs + j, s->dInfoP, s->dLenP, nullptr, s->dDataP, s->hTot, s->dataCap, b.perm, b.offs, 0,
                           c.dScale, hp, hs, s->dHullP, s->dHullS};
            compactTier1(ca, b.st);
            launches += 4;  // tile sums, scan, hull points, copy
        }
        if (tier1) {  // packed straight into mapped host memory
            // (after a device compaction the hull points are computed already)
            CompactArgs ca{s->n, b.info + 4 * (uint64_t)j, b.len + (uint64_t)kMaxPasses * j, b.dist + (uint64_t)kMaxPasses * j,
                           b.dJobs + j, s->hInfo, s->hLen, s->hDist, s->hData, s->hTot, s->dataCap, b.perm, b.offs, 1,
                           onDevice ? nullptr : c.dScale, hp, hs, s->hHullPasses, s->hHullSlope};
            compactTier1(ca, b.st);
            launches += onDevice ? 3 : 4;
        }
        r->tier1 = tier1;
        r->devFrame = onDevice;
    }
    if (b.timed) GB_CHECK(cudaEventRecord(b.t[4], b.st));
    GB_CHECK(cudaMemcpyAsync(b.hCtl, b.ctl, 64, cudaMemcpyDeviceToHost, b.st));
    GB_CHECK(cudaEventRecord(b.done, b.st));
    b.frames = std::move(sel);
    b.busy = true;
    std::lock_guard<std::mutex> lock(m_);
    stats_.batches++;
    stats_.batchFrames += b.frames.size();
    stats_.launches += launches;
    return true;
}

bool EncodeEngine::collect(Batch& b) {
    if (!b.busy) return false;
    const cudaError_t e = cudaEventQuery(b.done);
    if (e == cudaErrorNotReady) return false;
    GB_CHECK(e);
    const auto now = Clock::now();
    const uint32_t status = b.hCtl[1];
    float ms[4] = {0, 0, 0, 0};
    if (b.timed)
        for (int k = 0; k < 4; ++k) GB_CHECK(cudaEventElapsedTime(&ms[k], b.t[k], b.t[k + 1]));
    std::vector<float> front;
    for (Request* r : b.frames)
        if (r->frontTimed) {
            float f = 0;
            GB_CHECK(cudaEventElapsedTime(&f, r->slot->frontT[0], r->slot->frontT[1]));
            front.push_back(f);
            r->frontTimed = false;
        }
    std::lock_guard<std::mutex> lock(m_);
    if (b.timed) {
        times_.cmMs += ms[0];
        times_.orderMs += ms[1];
        times_.mqMs += ms[2];
        times_.packMs += ms[3];
        times_.batches++;
        times_.batchFrames += b.frames.size();
    }
    for (float f : front) {
        times_.frontMs += f;
        times_.frontFrames++;
    }
    for (Request* r : b.frames) {
        r->latency = msBetween(r->t0, now);
        r->status = (status || r->slot->hTot[2]) ? kError : kOk;
        if (csOn_) {
            csq_.push_back(r);
        } else {
            done_.push_back(r);
            --encActive_;
            stats_.frames++;
            const Slot* s = r->slot;
            stats_.d2hBytes += (uint64_t)s->n * 20 + (uint64_t)s->hTot[1] * 17 + s->hTot[0];
        }
    }
    if (csOn_) cvCs_.notify_all();
    b.frames.clear();
    b.busy = false;
    return true;
}

void EncodeEngine::run() {
    try {
        GB_CHECK(cudaSetDevice(dev_));
        while (!stop_) {
            bool did = admit();
            bool finished = false;
            for (auto& b : batches_) finished |= collect(*b);
            for (auto& b : batches_)
                if (!b->busy) did |= launchBatch(*b);
            if (finished) cvDone_.notify_all();
            if (!did && !finished) {
                std::unique_lock<std::mutex> lock(m_);
                cvWork_.wait_for(lock, std::chrono::microseconds(50));
            }
        }
    } catch (const std::exception& ex) {
        std::lock_guard<std::mutex> lock(m_);
        error_ = ex.what();
        cvDone_.notify_all();
    }
}

}  // namespace gb
