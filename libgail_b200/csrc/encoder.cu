// The plain per-frame encoder slot.
#include "encoder.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <stdexcept>
#include <string>

#include "common.cuh"
#include "frontend.cuh"
#include "tuning.h"

namespace gb {

namespace {

uint64_t page(uint64_t b) { return (b + (2ull << 20) - 1) & ~((2ull << 20) - 1); }

BandOut bandOut(const GbSubband& b) {
    BandOut o{};
    o.cblkBase = (uint32_t)b.cblkBase;
    o.ncbx = b.ncbx;
    o.ncby = b.ncby;
    o.w = b.w;
    o.h = b.h;
    o.px0 = b.px0;
    o.py0 = b.py0;
    o.invDelta = 1.0f / b.delta;
    o.maxMag = ((1u << b.Mb) << kFracBits) - 1u;
    return o;
}

}  // namespace

uint64_t SlotSizes::deviceBytes() const {
    const uint64_t sizes[] = {inBytes,     65536 * 4,   4096 * 4,    2 * llFloats * 4 * 3, n * kCblkArea * 4,
                              n * 48,      arena,       arena,       n * 16,               n * kMaxPasses * 4 * 3,
                              n * kMaxPasses * 16,      n * 4,       t1WorkWords((uint32_t)n) * 4, 64, n * 20,
                              n * 8,                    n * kMaxPasses * 8,       outCap};
    uint64_t t = 0;
    for (uint64_t b : sizes) t += page(b);
    return t;
}

uint64_t buildJobs(const Layout& L, const uint32_t* coeffs, uint8_t* sym, uint8_t* cw, uint32_t slope,
                   std::vector<T1Job>& jobs) {
    uint64_t region = 0;
    for (int i = 0; i < L.numCblks(); ++i) {
        const CodeBlock& cb = L.cblks[i];
        const GbSubband& b = L.bands[cb.band];
        const uint32_t cap = t1SymbolBound(cb.w, cb.h, std::max(1, std::min(b.Mb, kMaxPlanes)));
        const float dscale = (float)((double)b.delta * b.delta * b.weight);
        jobs.push_back({coeffs ? coeffs + (size_t)i * kCblkArea : nullptr, sym ? sym + region : nullptr,
                        cw ? cw + region : nullptr, cap, t1Geom(cb.w, cb.h, b.orient, kMaxPasses), dscale, slope, {0, 0}});
        region += cap;
    }
    return region;
}

uint64_t buildJobOffsets(const Layout& L, const uint32_t* coeffs, uint32_t slope, std::vector<T1Job>& jobs) {
    const size_t first = jobs.size();
    const uint64_t arena = buildJobs(L, coeffs, nullptr, nullptr, slope, jobs);
    uint64_t region = 0;
    for (size_t i = first; i < jobs.size(); ++i) {
        jobs[i].sym = reinterpret_cast<uint8_t*>(static_cast<uintptr_t>(region));
        jobs[i].cw = reinterpret_cast<uint8_t*>(static_cast<uintptr_t>(region));
        region += jobs[i].cap;
    }
    return arena;
}

std::vector<double> blockScales(const Layout& L) {
    std::vector<double> v((size_t)L.numCblks());
    for (int i = 0; i < L.numCblks(); ++i) {
        const GbSubband& b = L.bands[L.cblks[(size_t)i].band];
        v[(size_t)i] = (double)b.delta * b.delta * b.weight;
    }
    return v;
}

void launchFrontEnd(const Layout& L, const ColorArgs& c, float* ll0, float* ll1, uint64_t llFloats, uint32_t* coeffs,
                    float* tap, cudaStream_t st) {
    const int NL = L.levels;
    const Tuning tu = tuningFor(L.profile);
    float* llBuf[2] = {ll0, ll1};
    for (int l = 1; l <= NL; ++l) {
        LevelArgs a{};
        a.w = L.levelW(l - 1);
        a.h = L.levelH(l - 1);
        a.src = l == 1 ? nullptr : llBuf[(l - 1) & 1];
        a.srcStride = L.levelW(1);
        a.srcComp = llFloats;
        a.last = l == NL;
        a.ll = a.last ? nullptr : llBuf[l & 1];
        a.llStride = L.levelW(1);
        a.llComp = llFloats;
        a.coeffs = coeffs;
        a.tap = tap;
        a.tapStride = L.width;
        a.tapComp = (uint64_t)L.width * L.height;
        const int r = NL - l + 1;
        for (int comp = 0; comp < 3; ++comp) {
            for (int o = 1; o <= 3; ++o) a.band[comp][o] = bandOut(L.bands[L.bandIndex(comp, r, o)]);
            if (a.last) {
                a.band[comp][0] = bandOut(L.bands[L.bandIndex(comp, 0, 0)]);
            } else {
                BandOut& b = a.band[comp][0];
                b = BandOut{};
                b.w = L.levelW(l);
                b.h = L.levelH(l);
                b.ncbx = (b.w + 31) / 32;
                b.ncby = (b.h + 31) / 32;
            }
        }
        if (l == 1) launchLevel1(c, a, tu.dwtTile1, st);
        else launchLevel(a, tu.dwtTileN, st);
    }
}

SlotSizes slotSizes(const Layout& L, const GbFrameFormat& in) {
    SlotSizes z;
    z.npix = (uint64_t)L.width * L.height;
    z.n = (uint64_t)L.numCblks();
    z.inBytes = frameBytes(in);
    std::vector<T1Job> jobs;
    z.arena = buildJobs(L, nullptr, nullptr, nullptr, 0, jobs);
    z.llFloats = (uint64_t)L.levelW(1) * L.levelH(1);
    z.outCap = std::min<uint64_t>(z.arena, z.npix * 6 + (64u << 10));
    return z;
}

EncoderSlot::EncoderSlot(int device, const Layout& L, const GailCudaEncodeSettings& s) : dev_(device), L_(L), s_(s) {
    if (L.levels < 1) throw std::logic_error("the encoder needs at least one decomposition level");
    if (s.input.width != L.width || s.input.height != L.height)
        throw std::logic_error("input frame size differs from the layout");
    if (s.input.kind == GB_FRAME_PLANAR &&
        (s.input.activeW < 1 || s.input.activeH < 1 || s.input.ox < 0 || s.input.oy < 0 ||
         s.input.ox + s.input.activeW > L.width || s.input.oy + s.input.activeH > L.height || s.input.bits < 8 ||
         s.input.bits > 16 || s.input.sx < 0 || s.input.sx > 1 || s.input.sy < 0 || s.input.sy > 1))
        throw std::logic_error("planar input format out of range");
    color_ = buildColorTables(s.color);
    std::memcpy(m_, color_.m, sizeof m_);
    z_ = slotSizes(L, s.input);
    try {
        GB_CHECK(cudaSetDevice(dev_));
        GB_CHECK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
        for (auto& e : ev_) GB_CHECK(cudaEventCreate(&e));
        auto alloc = [&](auto*& p, uint64_t bytes) {
            void* q = nullptr;
            check(cudaMalloc(&q, std::max<uint64_t>(bytes, 16)), "device memory for an encoder slot");
            dev_allocs_.push_back(q);
            p = static_cast<std::remove_reference_t<decltype(p)>>(q);
        };
        const uint64_t n = z_.n;
        alloc(dIn_, z_.inBytes);
        alloc(dEotf_, 65536 * 4);
        alloc(dThr_, 4096 * 4);
        alloc(dLut_, color_.lut3.size() * 4);
        alloc(dLL_[0], z_.llFloats * 4 * 3);
        alloc(dLL_[1], z_.llFloats * 4 * 3);
        alloc(dCoeffs_, n * kCblkArea * 4);
        alloc(dJobs_, n * sizeof(T1Job));
        alloc(dSym_, z_.arena);
        alloc(dCw_, z_.arena);
        alloc(dInfo_, n * 16);
        alloc(dEnd_, n * kMaxPasses * 4);
        alloc(dLen_, n * kMaxPasses * 4);
        alloc(dDist_, n * kMaxPasses * 4);
        alloc(dSnaps_, n * kMaxPasses * 16);
        alloc(dPerm_, n * 4);
        alloc(dWork_, t1WorkWords((uint32_t)n) * 4);
        alloc(dCtl_, 64);
        alloc(dSlope_, 16);
        alloc(dOutInfo_, n * 20);
        alloc(dOffsets_, n * 8);
        alloc(dOutLen_, n * kMaxPasses * 4);
        alloc(dOutDist_, n * kMaxPasses * 4);
        alloc(dOutData_, z_.outCap);
        jobs_.clear();
        buildJobs(L_, dCoeffs_, dSym_, dCw_, 0, jobs_);
        auto pinned = [&](auto*& p, uint64_t bytes) {
            void* q = nullptr;
            check(cudaHostAlloc(&q, std::max<uint64_t>(bytes, 16), cudaHostAllocDefault), "pinned host memory");
            p = static_cast<std::remove_reference_t<decltype(p)>>(q);
        };
        pinned(hIn_, z_.inBytes);
        pinned(hInfo_, n * 20);
        pinned(hLen_, n * kMaxPasses * 4);
        pinned(hDist_, n * kMaxPasses * 4);
        pinned(hSmall_, 64);
        pinned(hSlope_, 16);
        hDataCap_ = std::min<uint64_t>(z_.arena, std::max<uint64_t>(64ull << 20, n * 2048));
        pinned(hData_, hDataCap_);
        uploadStatic();
    } catch (...) {
        release();
        throw;
    }
}

EncoderSlot::~EncoderSlot() { release(); }

void EncoderSlot::release() {
    cudaSetDevice(dev_);
    if (st_) cudaStreamSynchronize(st_);
    for (void* p : dev_allocs_) cudaFree(p);
    dev_allocs_.clear();
    for (void* p : {(void*)hIn_, (void*)hInfo_, (void*)hLen_, (void*)hDist_, (void*)hSmall_, (void*)hSlope_, (void*)hData_})
        if (p) cudaFreeHost(p);
    hIn_ = nullptr;
    hInfo_ = hLen_ = hSmall_ = nullptr;
    hDist_ = nullptr;
    hSlope_ = nullptr;
    hData_ = nullptr;
    if (dXyz_) cudaFree(dXyz_);
    if (dTap_) cudaFree(dTap_);
    dXyz_ = nullptr;
    dTap_ = nullptr;
    for (auto& e : ev_)
        if (e) {
            cudaEventDestroy(e);
            e = nullptr;
        }
    for (auto& e : ring_)
        if (e) cudaEventDestroy(e);
    ring_.clear();
    if (st_) cudaStreamDestroy(st_);
    st_ = nullptr;
    cudaGetLastError();
}

void EncoderSlot::uploadStatic() {
    GB_CHECK(cudaMemcpy(dEotf_, color_.eotf.data(), 65536 * 4, cudaMemcpyHostToDevice));
    GB_CHECK(cudaMemcpy(dThr_, color_.thr.data(), 4096 * 4, cudaMemcpyHostToDevice));
    if (!color_.lut3.empty())
        GB_CHECK(cudaMemcpy(dLut_, color_.lut3.data(), color_.lut3.size() * 4, cudaMemcpyHostToDevice));
    GB_CHECK(cudaMemcpy(dJobs_, jobs_.data(), jobs_.size() * sizeof(T1Job), cudaMemcpyHostToDevice));
}

void EncoderSlot::enqueueStages(const void* dFrame, bool taps, bool full) {
    const cudaStream_t st = st_;
    const uint64_t npix = z_.npix;
    // control words: all but the status word (ctl[1]), which collects every frame's
    // status until finish() or encode() reads it
    GB_CHECK(cudaMemsetAsync(dCtl_, 0, 4, st));
    GB_CHECK(cudaMemsetAsync(dCtl_ + 2, 0, 56, st));
    cudaEvent_t* mark = nullptr;
    if (timing_) {
        if (ring_.empty()) {
            ring_.resize((size_t)kTimingRing * 6);
            for (auto& e : ring_) GB_CHECK(cudaEventCreate(&e));
        }
        mark = &ring_[(size_t)ringNext_ * 6];
        ringNext_ = (ringNext_ + 1) % kTimingRing;
        ringCount_ = std::min(ringCount_ + 1, kTimingRing);
        GB_CHECK(cudaEventRecord(mark[0], st));
    }
    // front end: colour + level 1, then one kernel per level
    ColorArgs c{};
    c.kind = s_.input.kind == GB_FRAME_PLANAR ? 1 : 0;
    c.src = dFrame;
    c.pp = planarParams(s_.input);
    c.eotf = dEotf_;
    c.thr = dThr_;
    std::memcpy(c.m, m_, sizeof m_);
    c.route = color_.route;
    c.tone = color_.tone;
    c.lut3 = dLut_;
    c.lutN = color_.lutN;
    c.xyz = taps ? dXyz_ : nullptr;
    launchFrontEnd(L_, c, dLL_[0], dLL_[1], z_.llFloats, dCoeffs_, full ? dTap_ : nullptr, st);
    GB_CHECK(cudaEventRecord(ev_[2], st));
    if (mark) GB_CHECK(cudaEventRecord(mark[1], st));
    const uint64_t n = z_.n;
    T1Launch t{dJobs_, (uint32_t)n, dInfo_, dEnd_, dLen_, dDist_, dSnaps_, dPerm_, dCtl_, dSlope_};
    const Tuning tu = tuningFor(L_.profile);
    t.soloDecisions = tu.soloDecisions;
    t.cmCtasPerSm = (uint16_t)tu.cmCtasPerSm;
    t.mqCtasPerSm = (uint16_t)tu.mqCtasPerSm;
    t.persistent = (uint16_t)tu.t1Persistent;
    t.work = dWork_;
    t1Encode(t, st, mark ? mark + 2 : nullptr);
    GB_CHECK(cudaEventRecord(ev_[3], st));
    if (mark) GB_CHECK(cudaEventRecord(mark[4], st));
    CompactArgs ca{(uint32_t)n, dInfo_,    dLen_,      dDist_,   dJobs_,    dOutInfo_, dOutLen_,
                   dOutDist_,   dOutData_, dCtl_ + 8, z_.outCap, dPerm_,    dOffsets_, 0};
    compactTier1(ca, st);
    if (mark) GB_CHECK(cudaEventRecord(mark[5], st));
}

void EncoderSlot::enqueue(const void* dFrame) {
    GB_CHECK(cudaSetDevice(dev_));
    *hSlope_ = slope_;
    GB_CHECK(cudaMemcpyAsync(dSlope_, hSlope_, 4, cudaMemcpyHostToDevice, st_));
    enqueueStages(dFrame ? dFrame : dIn_, false, false);
}

void EncoderSlot::finish() {
    GB_CHECK(cudaSetDevice(dev_));
    GB_CHECK(cudaMemcpyAsync(hSmall_, dCtl_, 64, cudaMemcpyDeviceToHost, st_));
    GB_CHECK(cudaStreamSynchronize(st_));
    GB_CHECK(cudaGetLastError());
    const uint32_t status = hSmall_[1];
    GB_CHECK(cudaMemsetAsync(dCtl_ + 1, 0, 4, st_));
    if (status) throw std::runtime_error("Tier-1 kernels reported status " + std::to_string(status));
}

int EncoderSlot::stageTimes(double ms[5]) {
    for (int k = 0; k < 5; ++k) ms[k] = 0;
    GB_CHECK(cudaStreamSynchronize(st_));
    const int count = ringCount_;
    for (int i = 0; i < count; ++i) {
        cudaEvent_t* e = &ring_[(size_t)((ringNext_ - 1 - i + kTimingRing) % kTimingRing) * 6];
        for (int k = 0; k < 5; ++k) {
            float t = 0;
            GB_CHECK(cudaEventElapsedTime(&t, e[k], e[k + 1]));
            ms[k] += t;
        }
    }
    ringCount_ = 0;
    return count;
}

void EncoderSlot::encode(const void* frame, GailCudaTier1* out, GbFrameTimings* tm, GailCudaDebug* dbg) {
    const auto t0 = std::chrono::steady_clock::now();
    GB_CHECK(cudaSetDevice(dev_));
    if (!frame) throw std::logic_error("no frame");
    const bool full = dbg && dbg->full;
    const uint64_t npix = z_.npix, n = z_.n;
    if (dbg && !dXyz_) check(cudaMalloc(&dXyz_, npix * 6), "device memory for the debug taps");
    if (full && !dTap_) check(cudaMalloc(&dTap_, npix * 12), "device memory for the debug taps");
    if (frame != hIn_) std::memcpy(hIn_, frame, z_.inBytes);
    *hSlope_ = slope_;
    const cudaStream_t st = st_;
    GB_CHECK(cudaEventRecord(ev_[0], st));
    GB_CHECK(cudaMemcpyAsync(dIn_, hIn_, z_.inBytes, cudaMemcpyHostToDevice, st));
    GB_CHECK(cudaMemcpyAsync(dSlope_, hSlope_, 4, cudaMemcpyHostToDevice, st));
    GB_CHECK(cudaMemsetAsync(dCtl_ + 1, 0, 4, st));
    GB_CHECK(cudaEventRecord(ev_[1], st));
    enqueueStages(dIn_, dbg != nullptr, full);
    GB_CHECK(cudaMemcpyAsync(hSmall_, dCtl_, 64, cudaMemcpyDeviceToHost, st));
    GB_CHECK(cudaStreamSynchronize(st));
    const uint32_t status = hSmall_[1], totData = hSmall_[8], totPasses = hSmall_[9];
    if (status) throw std::runtime_error("Tier-1 kernels reported status " + std::to_string(status));
    if (totData > hDataCap_) {
        cudaFreeHost(hData_);
        hData_ = nullptr;
        hDataCap_ = (uint64_t)totData + totData / 2;
        check(cudaHostAlloc((void**)&hData_, hDataCap_, cudaHostAllocDefault), "pinned host memory");
    }
    GB_CHECK(cudaMemcpyAsync(hInfo_, dOutInfo_, n * 20, cudaMemcpyDeviceToHost, st));
    GB_CHECK(cudaMemcpyAsync(hLen_, dOutLen_, (uint64_t)totPasses * 4, cudaMemcpyDeviceToHost, st));
    GB_CHECK(cudaMemcpyAsync(hDist_, dOutDist_, (uint64_t)totPasses * 4, cudaMemcpyDeviceToHost, st));
    GB_CHECK(cudaMemcpyAsync(hData_, dOutData_, totData, cudaMemcpyDeviceToHost, st));
    GB_CHECK(cudaEventRecord(ev_[4], st));
    GB_CHECK(cudaStreamSynchronize(st));
    GB_CHECK(cudaGetLastError());

    *out = {reinterpret_cast<const GbCblkInfo*>(hInfo_), hLen_, hDist_, hData_, n, totPasses, totData};
    if (dbg) {
        xyz_.resize(npix * 3);
        GB_CHECK(cudaMemcpy(xyz_.data(), dXyz_, npix * 6, cudaMemcpyDeviceToHost));
        if (full) {
            coeffs_.resize(n * kCblkArea);
            GB_CHECK(cudaMemcpy(coeffs_.data(), dCoeffs_, n * kCblkArea * 4, cudaMemcpyDeviceToHost));
            wavelet_.resize(npix * 3);
            GB_CHECK(cudaMemcpy(wavelet_.data(), dTap_, npix * 12, cudaMemcpyDeviceToHost));
        }
        *dbg = {dbg->full, xyz_.data(), full ? coeffs_.data() : nullptr, full ? wavelet_.data() : nullptr,
                xyz_.size(), full ? coeffs_.size() : 0, full ? wavelet_.size() : 0};
    }
    if (tm) {
        float ms[4];
        for (int i = 0; i < 4; ++i) cudaEventElapsedTime(&ms[i], ev_[i], ev_[i + 1]);
        *tm = GbFrameTimings{};
        tm->upload = ms[0];
        tm->color = 0;  // folded into the first wavelet level
        tm->dwt = ms[1];
        tm->quant = 0;  // folded into the wavelet's output
        tm->t1 = ms[2];
        tm->t1cm = ms[2];
        tm->t1mq = 0;
        tm->download = ms[3];
        float g = 0;
        cudaEventElapsedTime(&g, ev_[0], ev_[4]);
        tm->gpu = g;
        tm->symbols = hSmall_[2];
        tm->codedBytes = totData;
        tm->total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
}

}  // namespace gb
