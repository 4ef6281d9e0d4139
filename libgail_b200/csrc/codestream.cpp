// Host codec around the Tier-1 frame (see codestream.h).
//
// What has to match the reference byte for byte, and so follows its steps: the packet
// order (CPRL, B.12.1.5, with the DCI 4K POC: resolutions 0..NL-1, then NL; progression.h),
// the packet-header syntax (B.10: inclusion and zero-bit-plane tag trees, the pass-count
// code of Table B.4, Lblock, bit stuffing; t2.cpp:19-122, tagtree.h, bitio.h), the main
// header the reference writes (t2.cpp:133-190), the hull and slope-threshold search of the
// rate control (rate_control.cpp:36-279, same floating-point operations in the same order
// so that the same passes are chosen), and the DCI rules of its checker
// (codestream_check.cpp:43-280).
#include "codestream.h"
#include "rate_search.h"

#include "pool.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace gb {

namespace {

enum : uint32_t {
    kSOC = 0xFF4F, kCAP = 0xFF50, kSIZ = 0xFF51, kCOD = 0xFF52, kCOC = 0xFF53, kTLM = 0xFF55, kPLM = 0xFF57,
    kPLT = 0xFF58, kQCD = 0xFF5C, kQCC = 0xFF5D, kRGN = 0xFF5E, kPOC = 0xFF5F, kPPM = 0xFF60, kCRG = 0xFF63,
    kCOM = 0xFF64, kSOT = 0xFF90, kSOP = 0xFF91, kEPH = 0xFF92, kSOD = 0xFF93, kEOC = 0xFFD9,
};
constexpr int kCblkLog2 = 5;

int floorLog2(uint32_t v) { return 31 - __builtin_clz(v); }  // v > 0

constexpr int kChunks = 16;  // work items per parallel phase
template <class F> void forChunks(int n, F&& f) {  // f(begin, end) over [0, n) in chunks
    if (n <= 0) return;
    if (n < 2 * kChunks) {  // too little to share out
        f(0, n);
        return;
    }
    const int per = (n + kChunks - 1) / kChunks;
    parallelFor(kChunks, [&](int c) {
        const int b = c * per, e = std::min(n, b + per);
        if (b < e) f(b, e);
    });
}


// ------------------------------------------------------------------ packet-header bits
// B.10.1: bits fill each byte from the top; the byte after an 0xFF byte carries only 7
// (its top bit is the stuffed 0). With no output it only counts.
class HeaderBits {
public:
    explicit HeaderBits(std::vector<uint8_t>* out) : out_(out) {}
    void put(uint32_t v, int n) {  // the n (<= 32) low bits of v, most significant first
        while (n > 0) {
            const int k = std::min(n, room_ - fill_);
            n -= k;
            cur_ = (cur_ << k) | ((v >> n) & ((1u << k) - 1u));
            fill_ += k;
            if (fill_ == room_) push();
        }
    }
    void bit(uint32_t b) { put(b, 1); }
    void zeros(int n) {
        for (; n > 8; n -= 8) put(0, 8);
        put(0, n);
    }
    // Pads the byte in progress with zeros; a header that ends on 0xFF owes the byte its
    // stuffing promised (0x00); a header with no bits is one 0x00. Returns its bytes.
    size_t end() {
        if (fill_ > 0 || bytes_ == 0) {
            cur_ <<= room_ - fill_;
            push();
        }
        if (last_ == 0xFFu) push();
        return bytes_;
    }

private:
    void push() {
        last_ = cur_ & 0xFFu;
        if (out_) out_->push_back((uint8_t)last_);
        ++bytes_;
        room_ = last_ == 0xFFu ? 7 : 8;
        cur_ = 0;
        fill_ = 0;
    }
    std::vector<uint8_t>* out_;
    uint32_t cur_ = 0, last_ = 0;
    int fill_ = 0, room_ = 8;
    size_t bytes_ = 0;
};

// The reading side: after an 0xFF byte the next carries 7 bits; reading past the end
// gives zeros and marks the overrun.
class HeaderReader {
public:
    HeaderReader(const uint8_t* p, size_t n) : p_(p), n_(n) {}
    uint32_t bit() {
        if (left_ == 0) next();
        return (cur_ >> --left_) & 1u;
    }
    uint32_t get(int n) {
        uint32_t v = 0;
        while (n-- > 0) v = (v << 1) | bit();
        return v;
    }
    // Where the header ends: the rest of the byte is padding, a final 0xFF has its
    // stuffed byte after it, and a header with no bits read is one byte.
    size_t end() {
        if (pos_ == 0) next();
        if (last_ == 0xFFu) next();
        left_ = 0;
        return pos_;
    }
    bool overrun() const { return over_; }

private:
    void next() {
        const bool stuffed = last_ == 0xFFu;
        cur_ = pos_ < n_ ? p_[pos_] : 0u;
        over_ = over_ || pos_ >= n_;
        ++pos_;
        last_ = cur_;
        left_ = stuffed ? 7 : 8;
    }
    const uint8_t* p_;
    size_t n_, pos_ = 0;
    uint32_t cur_ = 0, last_ = 0;
    int left_ = 0;
    bool over_ = false;
};

// ------------------------------------------------------------------------ tag trees
// B.10.2 over a w x h grid of leaves (a precinct-band's code-blocks, at most 4 x 4 in
// DCI; up to 64 x 64 here). A node's value is the minimum of its children's; coding a
// leaf against a threshold walks from the root: each node sends a 0 per unit its value
// is known to exceed (from where it stopped before, and at least its parent's bound) up
// to the threshold, and a 1 when its value is reached below the threshold.
class TagTree {
public:
    void shape(int w, int h) {
        if (w != w_ || h != h_) {
            if (w < 1 || h < 1 || w > 64 || h > 64) throw std::runtime_error("tag tree shape out of range");
            w_ = w;
            h_ = h;
            n_ = 0;
            int lw = w, lh = h, base = 0;
            for (;;) {
                const int nb = base + lw * lh, pw = (lw + 1) / 2;
                for (int y = 0; y < lh; ++y)
                    for (int x = 0; x < lw; ++x) parent_[base + y * lw + x] = (lw == 1 && lh == 1) ? -1 : nb + (y / 2) * pw + x / 2;
                n_ = nb;
                if (lw == 1 && lh == 1) break;
                base = nb;
                lw = pw;
                lh = (lh + 1) / 2;
            }
        }
        for (int i = 0; i < n_; ++i) {
            low_[i] = 0;
            known_[i] = 0;
        }
    }
    void leaf(int i, int v) { value_[i] = v; }
    void close() {  // internal nodes: the minimum of their children
        const int leaves = w_ * h_;
        for (int i = leaves; i < n_; ++i) value_[i] = 1 << 30;
        for (int i = 0; i < n_; ++i)
            if (parent_[i] >= 0) value_[parent_[i]] = std::min(value_[parent_[i]], value_[i]);
    }
    void encode(HeaderBits& hb, int leafIndex, int threshold) {
        int path[16], d = 0;
        for (int i = leafIndex; i >= 0; i = parent_[i]) path[d++] = i;
        int floorv = 0;
        while (d > 0) {
            const int i = path[--d];
            int lo = std::max(low_[i], floorv);
            const int to = std::min(value_[i], threshold);
            if (to > lo) {
                hb.zeros(to - lo);
                lo = to;
            }
            low_[i] = lo;
            if (lo >= value_[i] && lo < threshold && !known_[i]) {
                hb.bit(1);
                known_[i] = 1;
            }
            floorv = lo;
        }
    }
    bool decode(HeaderReader& hr, int leafIndex, int threshold) {
        int path[16], d = 0;
        for (int i = leafIndex; i >= 0; i = parent_[i]) path[d++] = i;
        int floorv = 0;
        while (d > 0) {
            const int i = path[--d];
            int lo = std::max(low_[i], floorv);
            while (!known_[i] && lo < threshold) {
                if (hr.bit()) {
                    known_[i] = 1;
                    value_[i] = lo;
                } else {
                    ++lo;
                }
            }
            low_[i] = lo;
            floorv = lo;
        }
        return known_[leafIndex] && value_[leafIndex] < threshold;
    }
    int value(int i) const { return value_[i]; }

private:
    static constexpr int kMax = 64 * 64 * 2;
    int w_ = -1, h_ = -1, n_ = 0;
    int parent_[kMax], value_[kMax], low_[kMax];
    uint8_t known_[kMax];
};

// The packets of component comp in resolutions [rs, re), CPRL order (B.12.1.5): precinct
// positions on the reference grid row by row, and at each the resolutions whose precinct
// grid has a corner there.
template <class F> void forEachPacket(const Layout& L, int rs, int re, int comp, F&& f) {
    const int NL = L.levels;
    int xstep = 1 << 30, ystep = 1 << 30;
    for (int r = rs; r < re; ++r) {
        const Resolution& R = L.resolution(0, r);
        xstep = std::min(xstep, 1 << (R.ppx + NL - r));
        ystep = std::min(ystep, 1 << (R.ppy + NL - r));
    }
    for (int y = 0; y < L.height; y += ystep)
        for (int x = 0; x < L.width; x += xstep)
            for (int r = rs; r < re; ++r) {
                const Resolution& R = L.resolution(comp, r);
                const int xr = 1 << (R.ppx + NL - r), yr = 1 << (R.ppy + NL - r);
                if ((x & (xr - 1)) || (y & (yr - 1))) continue;
                const int px = x / xr, py = y / yr;
                if (px < R.npx && py < R.npy) f(r, py * R.npx + px);
            }
}

// The DCI progression volumes: all resolutions at 2K; at 4K the POC's two, the 2K
// resolutions first.
int dciVolumes(const Layout& L, int rs[2], int re[2]) {
    const int NL = L.levels;
    if (L.profile == 1) {
        rs[0] = 0;
        re[0] = NL;
        rs[1] = NL;
        re[1] = NL + 1;
        return 2;
    }
    rs[0] = 0;
    re[0] = NL + 1;
    return 1;
}

void put16(std::vector<uint8_t>& v, uint32_t x) {
    v.push_back((uint8_t)(x >> 8));
    v.push_back((uint8_t)x);
}
void put32(std::vector<uint8_t>& v, uint32_t x) {
    put16(v, x >> 16);
    put16(v, x & 0xFFFFu);
}

// The pass-count code of Table B.4.
void putPasses(HeaderBits& hb, int n) {
    if (n == 1) hb.put(0, 1);
    else if (n == 2) hb.put(0x2, 2);
    else if (n <= 5) hb.put(0xC | (uint32_t)(n - 3), 4);
    else if (n <= 36) hb.put(0x1E0 | (uint32_t)(n - 6), 9);
    else if (n <= 164) hb.put(0xFF80 | (uint32_t)(n - 37), 16);
    else throw std::runtime_error("more than 164 coding passes in a code-block");
}
int getPasses(HeaderReader& hr) {
    if (!hr.bit()) return 1;
    if (!hr.bit()) return 2;
    uint32_t v = hr.get(2);
    if (v != 3) return 3 + (int)v;
    v = hr.get(5);
    if (v != 31) return 6 + (int)v;
    return 37 + (int)hr.get(7);
}

thread_local TagTree t_incl, t_msb;

}  // namespace

// ------------------------------------------------------------------ codestream writer
CodestreamWriter::CodestreamWriter(const Layout& L, std::string label) : L_(L), label_(std::move(label)) {
    int rs[2], re[2];
    const int nv = dciVolumes(L_, rs, re);
    ntp_ = 3 * nv;
    blockPacket_.assign((size_t)L_.numCblks(), -1);
    for (int v = 0; v < nv; ++v)
        for (int c = 0; c < kNumComps; ++c) {
            tpStart_.push_back((int32_t)pkStart_.size());
            forEachPacket(L_, rs[v], re[v], c, [&](int r, int prec) {
                const int p = (int)pkStart_.size();
                pkStart_.push_back((int32_t)segs_.size());
                const Precinct& P = L_.resolution(c, r).precincts[prec];
                for (int k = 0; k < P.nb; ++k) {
                    const PrecinctBand& pb = P.bands[k];
                    if (pb.ncbx <= 0 || pb.ncby <= 0) continue;
                    segs_.push_back({pb.band, pb.cbx0, pb.cby0, pb.ncbx, pb.ncby});
                    const GbSubband& b = L_.bands[pb.band];
                    for (int j = 0; j < pb.ncby; ++j)
                        for (int i = 0; i < pb.ncbx; ++i) blockPacket_[b.cblkBase + (pb.cby0 + j) * b.ncbx + pb.cbx0 + i] = p;
                }
            });
        }
    tpStart_.push_back((int32_t)pkStart_.size());
    pkStart_.push_back((int32_t)segs_.size());
    for (int32_t p : blockPacket_)
        if (p < 0) throw std::logic_error("a code-block belongs to no packet");
}

void CodestreamWriter::mainHeader(std::vector<uint8_t>& v, const std::string& comment) const {
    const bool fourk = L_.profile == 1;
    const int nres = L_.numRes();
    put16(v, kSOC);
    put16(v, kSIZ);
    put16(v, 38 + 3 * kNumComps);
    put16(v, fourk ? 4 : 3);  // Rsiz: CINEMA4K, CINEMA2K
    put32(v, (uint32_t)L_.width);
    put32(v, (uint32_t)L_.height);
    put32(v, 0);
    put32(v, 0);
    put32(v, (uint32_t)L_.width);  // a single tile
    put32(v, (uint32_t)L_.height);
    put32(v, 0);
    put32(v, 0);
    put16(v, kNumComps);
    for (int c = 0; c < kNumComps; ++c) {
        v.push_back(kBitDepth - 1);
        v.push_back(1);
        v.push_back(1);
    }
    put16(v, kCOD);
    put16(v, 12 + nres);
    v.push_back(0x01);  // precincts given, no SOP, no EPH
    v.push_back(4);     // CPRL
    put16(v, 1);        // one layer
    v.push_back(1);     // ICT
    v.push_back((uint8_t)L_.levels);
    v.push_back(kCblkLog2 - 2);
    v.push_back(kCblkLog2 - 2);
    v.push_back(0);  // no mode switches
    v.push_back(0);  // 9/7
    for (int r = 0; r < nres; ++r) v.push_back(r == 0 ? 0x77 : 0x88);
    put16(v, kQCD);
    const int nb = L_.bandsPerComp();
    put16(v, 3 + 2 * nb);
    v.push_back((uint8_t)((L_.guardBits << 5) | 2));  // scalar expounded
    for (int i = 0; i < nb; ++i) put16(v, (uint32_t)((L_.bands[i].eps << 11) | L_.bands[i].mu));
    if (fourk) {
        put16(v, kPOC);
        put16(v, 2 + 7 * 2);
        const uint8_t NL = (uint8_t)L_.levels;
        const uint8_t e[14] = {0, 0, 0, 1, NL, 3, 4, NL, 0, 0, 1, (uint8_t)(NL + 1), 3, 4};
        v.insert(v.end(), e, e + 14);
    }
    put16(v, kCOM);
    put16(v, (uint32_t)(4 + comment.size()));
    put16(v, 1);  // Latin-1 text
    v.insert(v.end(), comment.begin(), comment.end());
    put16(v, kTLM);  // one entry per tile-part, lengths filled in as they are written
    put16(v, 4 + 5 * ntp_);
    v.push_back(0);     // Ztlm
    v.push_back(0x50);  // Stlm: 8-bit tile index, 32-bit lengths
    for (int i = 0; i < ntp_; ++i) {
        v.push_back(0);
        put32(v, 0);
    }
}

size_t CodestreamWriter::packet(int p, const Tier1View& t1, const uint8_t* passes, std::vector<uint8_t>* out) {
    const int s0 = pkStart_[p], s1 = pkStart_[p + 1];
    bool any = false;
    for (int s = s0; s < s1 && !any; ++s) {
        const Seg& g = segs_[s];
        const GbSubband& b = L_.bands[g.band];
        for (int j = 0; j < g.ncby && !any; ++j) {
            const uint8_t* row = passes + b.cblkBase + (g.cby0 + j) * b.ncbx + g.cbx0;
            for (int i = 0; i < g.ncbx; ++i)
                if (row[i]) {
                    any = true;
                    break;
                }
        }
    }
    HeaderBits hb(out);
    if (!any) {
        hb.bit(0);
        return hb.end();
    }
    hb.bit(1);
    size_t body = 0;
    TagTree& incl = t_incl;
    TagTree& msbTree = t_msb;
    for (int s = s0; s < s1; ++s) {
        const Seg& g = segs_[s];
        const GbSubband& b = L_.bands[g.band];
        incl.shape(g.ncbx, g.ncby);
        msbTree.shape(g.ncbx, g.ncby);
        for (int j = 0; j < g.ncby; ++j)
            for (int i = 0; i < g.ncbx; ++i) {
                const int ci = b.cblkBase + (g.cby0 + j) * b.ncbx + g.cbx0 + i;
                incl.leaf(j * g.ncbx + i, passes[ci] ? 0 : 1);
                msbTree.leaf(j * g.ncbx + i, b.Mb - (int)t1.info[ci].nbps);
            }
        incl.close();
        msbTree.close();
        for (int j = 0; j < g.ncby; ++j)
            for (int i = 0; i < g.ncbx; ++i) {
                const int leaf = j * g.ncbx + i;
                const int ci = b.cblkBase + (g.cby0 + j) * b.ncbx + g.cbx0 + i;
                incl.encode(hb, leaf, 1);
                const int np = passes[ci];
                if (!np) continue;
                msbTree.encode(hb, leaf, 999);
                putPasses(hb, np);
                const uint32_t len = t1.len(ci, np - 1);
                // Lblock starts at 3; the length takes Lblock + floor(log2 passes) bits
                const int extra = floorLog2((uint32_t)np);
                const int need = len ? floorLog2(len) + 1 : 1;
                const int incr = std::max(0, need - (3 + extra));
                hb.put(((1u << incr) - 1u) << 1, incr + 1);  // incr ones and a zero
                hb.put(len, 3 + incr + extra);
                body += len;
            }
    }
    const size_t hdr = hb.end();
    if (out) {
        size_t at = out->size();
        out->resize(at + body);
        uint8_t* dst = out->data();
        for (int s = s0; s < s1; ++s) {
            const Seg& g = segs_[s];
            const GbSubband& b = L_.bands[g.band];
            for (int j = 0; j < g.ncby; ++j)
                for (int i = 0; i < g.ncbx; ++i) {
                    const int ci = b.cblkBase + (g.cby0 + j) * b.ncbx + g.cbx0 + i;
                    const int np = passes[ci];
                    if (!np) continue;
                    const uint32_t len = t1.len(ci, np - 1);
                    std::memcpy(dst + at, t1.data + t1.info[ci].dataOffset, len);
                    at += len;
                }
        }
    }
    return hdr + body;
}

CodestreamSizes CodestreamWriter::build(const Tier1View& t1, const uint8_t* passes, std::vector<uint8_t>* out,
                                        const std::string& tag) {
    if (tag.size() > kMaxDeviceTagBytes) throw std::logic_error("device tag \"" + tag + "\" is too long");
    const std::string comment = tag.empty() ? label_ : label_ + " " + tag;
    const size_t slack = label_.size() + 1 + kMaxDeviceTagBytes - comment.size();
    std::vector<uint8_t> hdr;
    mainHeader(hdr, comment);
    const size_t tlmAt = hdr.size() - 5 * (size_t)ntp_;
    // every packet's size, in parallel
    const int np = numPackets();
    std::vector<uint32_t> pk((size_t)np);
    forChunks(np, [&](int b, int e) {
        for (int p = b; p < e; ++p) pk[(size_t)p] = (uint32_t)packet(p, t1, passes, nullptr);
    });
    CodestreamSizes sz;
    sz.numTileParts = ntp_;
    size_t total = hdr.size();
    std::vector<size_t> at((size_t)np);  // each packet's offset in the codestream
    for (int tp = 0; tp < ntp_; ++tp) {
        size_t bytes = 14;  // SOT segment and SOD
        for (int p = tpStart_[tp]; p < tpStart_[tp + 1]; ++p) {
            at[(size_t)p] = total + bytes;
            bytes += pk[(size_t)p];
        }
        sz.tilePart[tp] = bytes;
        sz.comp[tp % 3] += bytes;
        total += bytes;
    }
    sz.total = total + slack + 2;
    if (out) {
        out->assign(total + 2, 0);
        uint8_t* d = out->data();
        std::memcpy(d, hdr.data(), hdr.size());
        size_t pos = hdr.size();
        for (int tp = 0; tp < ntp_; ++tp) {
            const uint32_t psot = (uint32_t)sz.tilePart[tp];
            const uint8_t sot[14] = {0xFF, 0x90, 0, 10, 0, 0, (uint8_t)(psot >> 24), (uint8_t)(psot >> 16),
                                     (uint8_t)(psot >> 8), (uint8_t)psot, (uint8_t)tp, (uint8_t)ntp_, 0xFF, 0x93};
            std::memcpy(d + pos, sot, 14);
            for (int k = 0; k < 4; ++k) d[tlmAt + 5 * tp + 1 + k] = (uint8_t)(psot >> (24 - 8 * k));
            pos += psot;
        }
        d[total] = 0xFF;  // EOC
        d[total + 1] = 0xD9;
        // the packets into their places, in parallel
        std::atomic<bool> mismatch{false};
        forChunks(np, [&](int b, int e) {
            thread_local std::vector<uint8_t> tmp;
            for (int p = b; p < e; ++p) {
                tmp.clear();
                packet(p, t1, passes, &tmp);
                if (tmp.size() != pk[(size_t)p]) {
                    mismatch.store(true);
                    continue;
                }
                std::memcpy(d + at[(size_t)p], tmp.data(), tmp.size());
            }
        });
        if (mismatch.load()) throw std::logic_error("packet size mismatch");
        if (out->size() + slack != sz.total) throw std::logic_error("codestream size mismatch");
    }
    return sz;
}

CodestreamSizes CodestreamWriter::measure(const Tier1View& t1, const uint8_t* passes) {
    const int np = numPackets(), n = L_.numCblks();
    if (!measured_) {
        pkBytes_.assign((size_t)np, 0);
        forChunks(np, [&](int b, int e) {
            for (int p = b; p < e; ++p) pkBytes_[(size_t)p] = (uint32_t)packet(p, t1, passes, nullptr);
        });
        lastPasses_.assign(passes, passes + n);
        dirty_.assign((size_t)np, 0);
        measured_ = true;
    } else {
        for (int i = 0; i < n; ++i)
            if (passes[i] != lastPasses_[(size_t)i]) {
                dirty_[(size_t)blockPacket_[(size_t)i]] = 1;
                lastPasses_[(size_t)i] = passes[i];
            }
        std::vector<int> todo;
        for (int p = 0; p < np; ++p)
            if (dirty_[(size_t)p]) {
                todo.push_back(p);
                dirty_[(size_t)p] = 0;
            }
        forChunks((int)todo.size(), [&](int b, int e) {
            for (int q = b; q < e; ++q) pkBytes_[(size_t)todo[(size_t)q]] = (uint32_t)packet(todo[(size_t)q], t1, passes, nullptr);
        });
    }
    CodestreamSizes sz;
    sz.numTileParts = ntp_;
    size_t total = longestHeaderBytes();
    for (int tp = 0; tp < ntp_; ++tp) {
        size_t bytes = 14;
        for (int p = tpStart_[tp]; p < tpStart_[tp + 1]; ++p) bytes += pkBytes_[(size_t)p];
        sz.tilePart[tp] = bytes;
        sz.comp[tp % 3] += bytes;
        total += bytes;
    }
    sz.total = total + 2;
    return sz;
}

size_t CodestreamWriter::longestHeaderBytes() {
    if (!hdrLongest_) {
        std::vector<uint8_t> hdr;
        mainHeader(hdr, label_ + std::string(1 + kMaxDeviceTagBytes, ' '));
        hdrLongest_ = hdr.size();
    }
    return hdrLongest_;
}

CodestreamSizes CodestreamWriter::assemble(const uint8_t* body, const uint64_t* tpBytes, const std::string& tag,
                                           std::vector<uint8_t>& out) const {
    if (tag.size() > kMaxDeviceTagBytes) throw std::logic_error("device tag \"" + tag + "\" is too long");
    const std::string comment = tag.empty() ? label_ : label_ + " " + tag;
    const size_t slack = label_.size() + 1 + kMaxDeviceTagBytes - comment.size();
    out.clear();
    mainHeader(out, comment);
    const size_t hdr = out.size(), tlmAt = hdr - 5 * (size_t)ntp_;
    CodestreamSizes sz;
    sz.numTileParts = ntp_;
    size_t body_ = 0;
    for (int tp = 0; tp < ntp_; ++tp) {
        if (tpBytes[tp] < 14 || tpBytes[tp] > 0xFFFFFFFFull) throw std::logic_error("tile-part size out of range");
        sz.tilePart[tp] = tpBytes[tp];
        sz.comp[tp % 3] += tpBytes[tp];
        body_ += tpBytes[tp];
    }
    out.resize(hdr + body_ + 2);
    uint8_t* d = out.data();
    std::memcpy(d + hdr, body, body_);
    size_t pos = hdr;
    for (int tp = 0; tp < ntp_; ++tp) {
        const uint32_t psot = (uint32_t)tpBytes[tp];
        const uint8_t sot[14] = {0xFF, 0x90, 0, 10, 0, 0, (uint8_t)(psot >> 24), (uint8_t)(psot >> 16),
                                 (uint8_t)(psot >> 8), (uint8_t)psot, (uint8_t)tp, (uint8_t)ntp_, 0xFF, 0x93};
        std::memcpy(d + pos, sot, 14);
        for (int k = 0; k < 4; ++k) d[tlmAt + 5 * tp + 1 + k] = (uint8_t)(psot >> (24 - 8 * k));
        pos += psot;
    }
    d[hdr + body_] = 0xFF;  // EOC
    d[hdr + body_ + 1] = 0xD9;
    sz.total = out.size() + slack;
    return sz;
}

size_t CodestreamWriter::emptyBytes() {
    std::vector<GbCblkInfo> info((size_t)L_.numCblks(), GbCblkInfo{});
    const std::vector<uint8_t> none((size_t)L_.numCblks(), 0);
    Tier1View t1;
    t1.info = info.data();
    t1.numInfo = (uint32_t)info.size();
    return build(t1, none.data(), nullptr).total;
}

// ------------------------------------------------------------------------ rate control
RateLimits dciLimits(double fps, double maxMbps, double compMbps) {
    // strictly below the limit libdcp checks (size > rint(Mbps * 1e6 / (8 fps))); a budget
    // that cannot be positive is 0, which no frame meets
    auto budget = [fps](double mbps) {
        const double b = std::floor(mbps * 1e6 / (8.0 * fps)) - 16;
        return std::isfinite(b) && b > 0 ? (size_t)b : (size_t)0;
    };
    return {budget(maxMbps), budget(compMbps)};
}

namespace {

// Per block, the points of the lower convex hull of its (rate, distortion reduction)
// curve: passes, rate, slope to the previous point, distortion gained from it. A block has
// at most as many points as passes, so block i's points sit at its pass offset:
// [first[i], first[i] + count[i]) (the arrays have gaps between blocks).
struct Hull {
    std::vector<uint32_t> first, count;
    std::vector<uint32_t> rate;
    std::vector<double> gain;  // empty for a hull that came precomputed
    const uint8_t* passes = nullptr;
    const double* slope = nullptr;
    size_t slots = 0;
    std::vector<uint8_t> ownPasses;  // the storage of a hull computed here
    std::vector<double> ownSlope;
    uint32_t end(size_t i) const { return first[i] + count[i]; }
};

constexpr int kMaxHull = 165;  // the origin and up to 164 passes

// Distortion units of pass k of a block with nbps planes: the plane it codes, as 4^plane /
// 4096 (the Tier-1 distortions are in 1/4096 of a plane's squared step).
double planeScale(int nbps, int k) {
    const int plane = k == 0 ? nbps - 1 : nbps - 2 - (k - 1) / 3;
    return (double)(1ull << (2 * plane)) / 4096.0;
}

// The hull points of blocks [b, e), written at their blocks' pass offsets: passes, slope,
// and where given, rate and gain; first/count where given.
struct HullOut {
    uint8_t* passes;
    double* slope;
    uint32_t* rate;
    double* gain;
    uint32_t* first;
    uint32_t* count;
};

void hullRange(const Layout& L, const Tier1View& t1, int b, int e, const HullOut& H) {
    uint32_t R[kMaxHull];
    double D[kMaxHull], S[kMaxHull];  // S[m]: slope from point m - 1 to point m
    int K[kMaxHull];
    double planes[64];  // 4^plane / 4096, exact powers of two
    for (int p = 0; p < 64; ++p) planes[p] = p < 32 ? (double)(1ull << (2 * p)) / 4096.0 : 0.0;
    for (int i = b; i < e; ++i) {
        const GbCblkInfo& ci = t1.info[i];
        const int np = (int)ci.numPasses;
        if (H.first) H.first[(size_t)i] = ci.passBase;
        if (H.count) H.count[(size_t)i] = 0;
        if (np == 0) continue;
        const GbSubband& band = L.bands[L.cblks[(size_t)i].band];
        const double scale = (double)band.delta * band.delta * band.weight;
        const uint32_t* len = t1.passLen + ci.passBase;
        const int32_t* dist = t1.passDist + ci.passBase;
        int m = 0;  // top of the hull stack; point 0 is the origin
        R[0] = 0;
        D[0] = 0.0;
        K[0] = 0;
        double acc = 0;
        const int nbps = (int)ci.nbps;
        for (int k = 0; k < np; ++k) {
            const int plane = k == 0 ? nbps - 1 : nbps - 2 - (k - 1) / 3;
            acc += dist[k] * (plane >= 0 && plane < 32 ? planes[plane] : planeScale(nbps, k)) * scale;
            const uint32_t r = len[k];
            if (acc <= D[m]) continue;  // no gain: never a hull point
            // drop the points the new one makes concave
            while (m >= 1) {
                const double sNew = r == R[m] ? INFINITY : (acc - D[m]) / (double)(r - R[m]);
                if (sNew < S[m]) break;
                --m;
            }
            ++m;
            R[m] = r;
            D[m] = acc;
            K[m] = k + 1;
            S[m] = R[m] == R[m - 1] ? INFINITY : (D[m] - D[m - 1]) / (double)(R[m] - R[m - 1]);
        }
        const size_t o = ci.passBase;
        for (int q = 1; q <= m; ++q) {
            H.passes[o + q - 1] = (uint8_t)K[q];
            const double dr = (double)R[q] - (double)R[q - 1];
            H.slope[o + q - 1] = dr <= 0 ? INFINITY : (D[q] - D[q - 1]) / dr;
            if (H.rate) H.rate[o + q - 1] = R[q];
            if (H.gain) H.gain[o + q - 1] = D[q] - D[q - 1];
        }
        if (H.count) H.count[(size_t)i] = (uint32_t)m;
        for (int q = m; q < np; ++q) {  // the rest of the block's entries: the end mark
            H.passes[o + q] = 0;
            H.slope[o + q] = 0;
        }
    }
}

Hull buildHull(const Layout& L, const Tier1View& t1) {
    const int n = L.numCblks();
    Hull H;
    H.first.assign((size_t)n, 0);
    H.count.assign((size_t)n, 0);
    H.ownPasses.resize(t1.numPasses);
    H.ownSlope.resize(t1.numPasses);
    H.rate.resize(t1.numPasses);
    H.gain.resize(t1.numPasses);
    H.passes = H.ownPasses.data();
    H.slope = H.ownSlope.data();
    H.slots = t1.numPasses;
    const HullOut out{H.ownPasses.data(), H.ownSlope.data(), H.rate.data(), H.gain.data(), H.first.data(),
                      H.count.data()};
    forChunks(n, [&](int b, int e) { hullRange(L, t1, b, e, out); });
    return H;
}

// A hull computed elsewhere (the GPU), in the HullView layout: its points are checked to
// be well formed (strictly increasing pass counts within the block's passes) and their
// rates looked up in the pass tables.
Hull hullFromView(const Layout& L, const Tier1View& t1, const HullView& v) {
    const int n = L.numCblks();
    Hull H;
    H.first.assign((size_t)n, 0);
    H.count.assign((size_t)n, 0);
    H.rate.resize(t1.numPasses);
    H.passes = v.passes;
    H.slope = v.slope;
    H.slots = t1.numPasses;
    std::atomic<bool> bad{false};
    forChunks(n, [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            const GbCblkInfo& ci = t1.info[i];
            const uint32_t o = ci.passBase, np = ci.numPasses;
            H.first[(size_t)i] = o;
            uint32_t m = 0, prev = 0;
            for (; m < np && v.passes[o + m] != 0; ++m) {
                const uint32_t k = v.passes[o + m];
                if (k <= prev || k > np) {
                    bad = true;
                    break;
                }
                H.rate[o + m] = t1.passLen[o + k - 1];
                prev = k;
            }
            H.count[(size_t)i] = m;
        }
    });
    if (bad) throw std::runtime_error("malformed hull points");
    return H;
}

// The hull points into the bins: the bin of every point in parallel (the log2 is the
// cost), then the sums of integer-valued doubles, exact in any order.
void binHull(const Layout& L, const Hull& H, SlopeBins& bins) {
    std::vector<int> binOf(H.slots);
    forChunks(L.numCblks(), [&](int b, int e) {
        for (int i = b; i < e; ++i)
            for (uint32_t h = H.first[(size_t)i]; h < H.end((size_t)i); ++h) binOf[h] = bins.bin(H.slope[h]);
    });
    for (int i = 0; i < L.numCblks(); ++i) {
        const int c = L.bands[L.cblks[(size_t)i].band].comp;
        uint32_t prev = 0;
        for (uint32_t h = H.first[(size_t)i]; h < H.end((size_t)i); ++h) {
            bins.add(c, binOf[h], (double)H.rate[h] - prev, h == H.first[(size_t)i] ? 1.0 : 0.0);
            prev = H.rate[h];
        }
    }
    bins.finish();
}

}  // namespace

SlopeBins::SlopeBins(double lo, double hi) : lo_(lo) {
    nb_ = std::max(16, (int)std::ceil((hi - lo) * kPerOctave) + 2);
    for (int c = 0; c < 3; ++c) {
        bytes_[c].assign((size_t)nb_ + 1, 0.0);
        blocks_[c].assign((size_t)nb_ + 1, 0.0);
    }
}

int SlopeBins::bin(double slope) const {
    if (!std::isfinite(slope)) return nb_ - 1;
    const int b = (int)std::floor((std::log2(slope) - lo_) * kPerOctave);
    return std::clamp(b, 0, nb_ - 1);
}

void SlopeBins::finish() {
    for (int c = 0; c < 3; ++c)
        for (int b = nb_ - 1; b >= 0; --b) {
            bytes_[c][(size_t)b] += bytes_[c][(size_t)b + 1];
            blocks_[c][(size_t)b] += blocks_[c][(size_t)b + 1];
        }
}

void SlopeBins::at(const double lam[3], double bytes[3], double blocks[3]) const {
    for (int c = 0; c < 3; ++c) {
        const int b = lam[c] <= 0 ? 0 : std::min(nb_, bin(lam[c]));
        bytes[c] = bytes_[c][(size_t)b];
        blocks[c] = blocks_[c][(size_t)b];
    }
}

void slopeBounds(double& minSlope, double& maxSlope, double& lo, double& hi) {
    if (maxSlope == 0) maxSlope = minSlope = 1;
    lo = std::log2(minSlope) - 1;
    hi = std::log2(maxSlope) + 1;
}

void rateSearch(const RateLimits& lim, double minSlope, double maxSlope, double loBound, double hiBound,
                const SlopeBins& bins, const MeasureFn& measure, double lam[3], CodestreamSizes& sz) {
    sz = measure(lam);
    // size model per component: header bytes ~ calibrated + beta * (blocks included - calibrated)
    double hdrCal[3], blkCal[3], beta[3];
    auto calibrate = [&](const double l[3], const CodestreamSizes& ex) {
        double bytes[3], blocks[3];
        bins.at(l, bytes, blocks);
        for (int c = 0; c < 3; ++c) {
            hdrCal[c] = (double)ex.comp[c] - bytes[c];
            blkCal[c] = blocks[c];
            beta[c] = blocks[c] > 0 ? std::max(1.0, std::min(8.0, hdrCal[c] / blocks[c])) : 3.0;
        }
    };
    auto model = [&](const double l[3], double comp[3]) {
        double bytes[3], blocks[3];
        bins.at(l, bytes, blocks);
        double tot = (double)(sz.total - sz.comp[0] - sz.comp[1] - sz.comp[2]);  // main header, EOC
        for (int c = 0; c < 3; ++c) {
            comp[c] = bytes[c] + hdrCal[c] + beta[c] * (blocks[c] - blkCal[c]);
            tot += comp[c];
        }
        return tot;
    };
    // the smallest log2 threshold in [lo, hi] for which fits() holds, by bisection
    auto search = [](auto fits, double lo, double hi) {
        for (int it = 0; it < 48 && hi - lo > 1e-5; ++it) {
            const double mid = 0.5 * (lo + hi);
            if (fits(mid)) hi = mid;
            else lo = mid;
        }
        return hi;
    };

    if (sz.total > lim.maxTotal) {
        calibrate(lam, sz);
        const double target = (double)lim.maxTotal;
        for (int round = 0; round < 6; ++round) {
            const double lg = search(
                [&](double m) {
                    const double l = std::exp2(m), ll[3] = {l, l, l};
                    double comp[3];
                    return model(ll, comp) <= target;
                },
                loBound, hiBound);
            lam[0] = lam[1] = lam[2] = std::exp2(lg);
            sz = measure(lam);
            if (sz.total <= lim.maxTotal && sz.total + lim.maxTotal / 500 >= lim.maxTotal) break;
            calibrate(lam, sz);
        }
        // raise the thresholds in small steps until the exact size fits; past the steepest
        // slope nothing more can be dropped
        while (sz.total > lim.maxTotal && lam[0] <= maxSlope) {
            for (int c = 0; c < 3; ++c) lam[c] = lam[c] > 0 ? lam[c] * 1.002 : minSlope;
            sz = measure(lam);
        }
    }
    for (int c = 0; c < kNumComps; ++c) {  // each component under its own cap
        if (sz.comp[c] <= lim.maxComp) continue;
        calibrate(lam, sz);
        for (int round = 0; round < 6; ++round) {
            const double lg = search(
                [&](double m) {
                    double ll[3] = {lam[0], lam[1], lam[2]};
                    ll[c] = std::exp2(m);
                    double comp[3];
                    model(ll, comp);
                    return comp[c] <= (double)lim.maxComp;
                },
                std::log2(std::max(lam[c], minSlope)), hiBound);
            lam[c] = std::exp2(lg);
            sz = measure(lam);
            if (sz.comp[c] <= lim.maxComp && sz.comp[c] + lim.maxComp / 500 >= lim.maxComp) break;
            calibrate(lam, sz);
        }
        while (sz.comp[c] > lim.maxComp && lam[c] <= maxSlope) {
            lam[c] = lam[c] > 0 ? lam[c] * 1.002 : minSlope;
            sz = measure(lam);
        }
    }
}

void computeHull(const Layout& L, const Tier1View& t1, uint8_t* passes, double* slope) {
    const HullOut out{passes, slope, nullptr, nullptr, nullptr, nullptr};
    forChunks(L.numCblks(), [&](int b, int e) { hullRange(L, t1, b, e, out); });
}

RateResult allocateRate(CodestreamWriter& w, const Tier1View& t1, const RateLimits& lim, const HullView* hull) {
    const Layout& L = w.layout();
    const int n = L.numCblks();
    const Hull H = hull ? hullFromView(L, t1, *hull) : buildHull(L, t1);
    RateResult res;
    res.passes.assign((size_t)n, 0);
    double lam[3] = {0, 0, 0};
    std::vector<int> compOf((size_t)n);
    for (int i = 0; i < n; ++i) compOf[(size_t)i] = L.bands[L.cblks[(size_t)i].band].comp;

    // every block's passes at the thresholds: its hull points down to the first flatter one
    auto select = [&](const double l[3]) {
        forChunks(n, [&](int b, int e) {
            for (int i = b; i < e; ++i) {
                const double t = l[compOf[(size_t)i]];
                uint8_t np = 0;
                for (uint32_t h = H.first[(size_t)i]; h < H.end((size_t)i); ++h) {
                    if (H.slope[h] < t) break;
                    np = H.passes[h];
                }
                res.passes[(size_t)i] = np;
            }
        });
    };
    w.restart();
    auto measure = [&](const double l[3]) {
        select(l);
        ++res.iterations;
        return w.measure(t1, res.passes.data());
    };

    double maxSlope = 0, minSlope = INFINITY;
    {
        double mx[kChunks], mn[kChunks];
        std::fill(mx, mx + kChunks, 0.0);
        std::fill(mn, mn + kChunks, INFINITY);
        const int per = (n + kChunks - 1) / kChunks;
        parallelFor(kChunks, [&](int c) {
            double hi = 0, lo = INFINITY;  // in registers: one store per chunk
            for (int i = c * per; i < std::min(n, (c + 1) * per); ++i)
                for (uint32_t h = H.first[(size_t)i]; h < H.end((size_t)i); ++h) {
                    const double s = H.slope[h];
                    if (std::isfinite(s) && s > 0) {
                        hi = std::max(hi, s);
                        lo = std::min(lo, s);
                    }
                }
            mx[c] = hi;
            mn[c] = lo;
        });
        for (int c = 0; c < kChunks; ++c) {
            maxSlope = std::max(maxSlope, mx[c]);
            minSlope = std::min(minSlope, mn[c]);
        }
    }
    double loBound, hiBound;
    slopeBounds(minSlope, maxSlope, loBound, hiBound);
    SlopeBins bins(loBound, hiBound);
    binHull(L, H, bins);

    CodestreamSizes sz;
    rateSearch(lim, minSlope, maxSlope, loBound, hiBound, bins, measure, lam, sz);
    res.lambda = std::max({lam[0], lam[1], lam[2]});
    for (int c = 0; c < 3; ++c) res.lambdaComp[c] = lam[c];
    double dist = H.gain.empty() ? NAN : 0.0;
    if (!H.gain.empty())
        for (int i = 0; i < n; ++i)  // in block order, as the sum is not exact in any other
            for (uint32_t h = H.first[(size_t)i]; h < H.end((size_t)i); ++h)
                if (H.passes[h] > res.passes[(size_t)i]) dist += H.gain[h];
    res.distortion = dist;
    res.sizes = sz;
    return res;
}

// --------------------------------------------------------------- big-endian reading
namespace {

// Reads that set fail, and give 0, once they run past the end.
struct Bytes {
    const uint8_t* p;
    const uint8_t* end;
    bool fail = false;
    uint32_t u8() {
        if (p >= end) {
            fail = true;
            return 0;
        }
        return *p++;
    }
    uint32_t u16() {
        const uint32_t a = u8();
        return (a << 8) | u8();
    }
    uint32_t u32() {
        const uint32_t a = u16();
        return (a << 16) | u16();
    }
};

std::string hexOf(uint32_t v) {
    char b[16];
    std::snprintf(b, sizeof b, "0x%X", v);
    return b;
}

}  // namespace

// ---------------------------------------------------------------------------- reading
void parseCodestream(const uint8_t* data, size_t size, Layout& L, std::vector<GbCblkCode>& blocks) {
    auto bad = [](const std::string& s) { throw std::runtime_error("codestream: " + s); };
    Bytes in{data, data + size};
    if (in.u16() != kSOC) bad("no SOC");
    if (in.u16() != kSIZ) bad("no SIZ after SOC");
    auto segment = [&](Bytes& seg) {
        const uint32_t len = in.u16();
        if (in.fail || len < 2 || (size_t)(in.end - in.p) < (size_t)len - 2) bad("a marker segment runs past the end");
        seg = Bytes{in.p, in.p + len - 2};
        in.p += len - 2;
    };
    Bytes seg{nullptr, nullptr};
    segment(seg);
    const uint32_t rsiz = seg.u16(), xs = seg.u32(), ys = seg.u32(), xo = seg.u32(), yo = seg.u32();
    const uint32_t xt = seg.u32(), yt = seg.u32(), xto = seg.u32(), yto = seg.u32(), csiz = seg.u16();
    if (seg.fail) bad("short SIZ");
    if (rsiz != 3 && rsiz != 4) bad("not a DCI cinema profile");
    if (csiz != 3 || xo || yo || xto || yto || xt < xs || yt < ys) bad("not a single-tile three-component frame");
    for (uint32_t c = 0; c < csiz; ++c)
        if (seg.u8() != 11 || seg.u8() != 1 || seg.u8() != 1) bad("components are not 12-bit, 1x1");
    const bool fourk = rsiz == 4;
    const int width = (int)xs, height = (int)ys;
    if (width < 64 || height < 64 || (fourk ? (width > 4096 || height > 2160) : (width > 2048 || height > 1080)))
        bad("size outside the DCI container");

    int levels = -1, guard = -1;
    bool sop = false, eph = false;
    int eps[3][3 * 32 + 1] = {}, mu[3][3 * 32 + 1] = {};
    bool qcc[3] = {false, false, false}, haveQcd = false;
    std::vector<int> volRs, volRe;
    uint32_t m = 0;
    auto readSteps = [&](Bytes& s, int* e, int* u, int& g) {
        const uint32_t sq = s.u8();
        g = (int)(sq >> 5);
        const int style = (int)(sq & 31), nb = 3 * levels + 1;
        if (style == 2) {
            for (int i = 0; i < nb; ++i) {
                const uint32_t v = s.u16();
                e[i] = (int)(v >> 11);
                u[i] = (int)(v & 0x7FF);
            }
        } else if (style == 1) {  // derived from the LL pair by level
            const uint32_t v = s.u16();
            for (int i = 0; i < nb; ++i) {
                const int lev = i == 0 ? levels : levels - (1 + (i - 1) / 3) + 1;
                e[i] = (int)(v >> 11) - levels + lev;
                u[i] = (int)(v & 0x7FF);
                if (e[i] < 0) bad("derived step exponent below zero");
            }
        } else {
            bad("quantisation style " + std::to_string(style));
        }
        if (s.fail) bad("short quantisation segment");
    };
    for (;;) {
        if (in.end - in.p < 2) bad("ends inside the main header");
        m = in.u16();
        if (m == kSOT) break;
        if ((m >> 8) != 0xFF) bad("no marker in the main header");
        if (m == kEOC || m == kSOC || m == kSOD) bad("marker out of place in the main header");
        segment(seg);
        if (m == kCOD) {
            const uint32_t scod = seg.u8(), prog = seg.u8(), layers = seg.u16(), mct = seg.u8();
            levels = (int)seg.u8();
            const uint32_t xcb = seg.u8(), ycb = seg.u8(), style = seg.u8(), xform = seg.u8();
            sop = (scod & 2) != 0;
            eph = (scod & 4) != 0;
            if (prog != 4 || layers != 1 || mct != 1 || xcb != 3 || ycb != 3 || style != 0 || xform != 0 || !(scod & 1))
                bad("coding style outside DCI (CPRL, one layer, ICT, 32x32, no mode switches, 9/7, precincts)");
            if (levels < 1 || levels > (fourk ? 6 : 5)) bad("decomposition levels");
            for (int r = 0; r <= levels; ++r)
                if (seg.u8() != (r == 0 ? 0x77u : 0x88u)) bad("precincts other than the DCI ones");
            if (seg.fail) bad("short COD");
        } else if (m == kQCD) {
            if (levels < 0) bad("QCD before COD");
            readSteps(seg, eps[0], mu[0], guard);
            haveQcd = true;
        } else if (m == kQCC) {
            if (levels < 0) bad("QCC before COD");
            const uint32_t c = seg.u8();
            int g = 0;
            if (c >= 3) bad("QCC of a fourth component");
            readSteps(seg, eps[c], mu[c], g);
            qcc[c] = true;
            if (haveQcd && g != guard) bad("per-component guard bits");
        } else if (m == kPOC) {
            while (seg.end - seg.p >= 7) {
                const uint32_t rs = seg.u8(), cs = seg.u8(), lye = seg.u16(), re = seg.u8(), ce = seg.u8(), order = seg.u8();
                if (order != 4 || cs != 0 || (ce != 0 && ce < 3) || lye < 1) bad("progression change other than by resolution");
                volRs.push_back((int)rs);
                volRe.push_back((int)re);
            }
        } else if (m == kCOC || m == kRGN || m == kPPM || m == kCAP) {
            bad("marker " + hexOf(m) + " (not taken by this decoder)");
        }  // TLM, PLM, CRG, COM: nothing needed
    }
    if (levels < 0 || !haveQcd) bad("no COD or QCD");
    for (int c = 1; c < 3; ++c)
        if (!qcc[c]) {
            std::memcpy(eps[c], eps[0], sizeof eps[0]);
            std::memcpy(mu[c], mu[0], sizeof mu[0]);
        }
    L = makeGeometry(width, height, fourk ? 1 : 0, levels, guard);
    for (int c = 0; c < 3; ++c) setSignalledSteps(L, c, eps[c], mu[c]);
    if (volRs.empty()) {
        volRs.push_back(0);
        volRe.push_back(levels + 1);
    }
    for (size_t v = 0, next = 0; v < volRs.size(); ++v) {  // the volumes follow on from each other
        volRe[v] = std::min(volRe[v], levels + 1);
        if (volRs[v] != (int)next || volRe[v] <= volRs[v]) bad("progression volumes do not follow on");
        next = (size_t)volRe[v];
        if (v + 1 == volRs.size() && next != (size_t)levels + 1) bad("progression volumes leave resolutions out");
    }

    // tile-parts: the packets of each lie from after its SOD to its end
    struct Span {
        size_t b, e;
    };
    std::vector<Span> parts;
    while (m == kSOT) {
        const size_t sot = (size_t)(in.p - data) - 2;
        const uint32_t lsot = in.u16(), isot = in.u16(), psot = in.u32(), tp = in.u8();
        in.u8();
        if (in.fail || lsot != 10 || isot != 0 || tp != parts.size()) bad("tile-part header");
        size_t end;
        if (psot == 0) end = size >= 2 && data[size - 2] == 0xFF && data[size - 1] == 0xD9 ? size - 2 : size;
        else if (psot < 14 || size - sot < psot) bad("tile-part runs past the end");
        else end = sot + psot;
        for (;;) {
            if ((size_t)(in.p - data) + 2 > end) bad("tile-part without SOD");
            const uint32_t t = in.u16();
            if (t == kSOD) break;
            if ((t >> 8) != 0xFF) bad("no marker in a tile-part header");
            segment(seg);
            if ((size_t)(in.p - data) > end) bad("tile-part header runs past its tile-part");
            if (t != kPLT && t != kCOM) bad("marker " + hexOf(t) + " in a tile-part header");
        }
        parts.push_back({(size_t)(in.p - data), end});
        in.p = data + end;
        if (in.p == in.end) break;
        if (in.end - in.p < 2) bad("stray byte after the last tile-part");
        m = in.u16();
        if (m != kSOT && m != kEOC) bad("neither SOT nor EOC after a tile-part");
    }
    if (parts.empty()) bad("no tile-parts");

    // packets. One packet from pos (within [pos, end)); returns where the next one starts.
    blocks.assign((size_t)L.numCblks(), GbCblkCode{});
    auto parsePacket = [&](int c, int r, int prec, size_t pos, size_t end) {
        TagTree& incl = t_incl;
        TagTree& msbTree = t_msb;
        if (sop && end - pos >= 6 && data[pos] == 0xFF && data[pos + 1] == (kSOP & 0xFF)) pos += 6;
        const Precinct& P = L.resolution(c, r).precincts[(size_t)prec];
        HeaderReader hr(data + pos, end - pos);
        size_t body = 0;
        const bool present = hr.bit() != 0;
        for (int k = 0; present && k < P.nb; ++k) {
            const PrecinctBand& pb = P.bands[k];
            if (pb.ncbx <= 0 || pb.ncby <= 0) continue;
            const GbSubband& b = L.bands[pb.band];
            incl.shape(pb.ncbx, pb.ncby);
            msbTree.shape(pb.ncbx, pb.ncby);
            for (int j = 0; j < pb.ncby; ++j)
                for (int i = 0; i < pb.ncbx; ++i) {
                    const int leaf = j * pb.ncbx + i;
                    if (!incl.decode(hr, leaf, 1)) continue;
                    if (!msbTree.decode(hr, leaf, b.Mb + 1)) bad("more missing bit-planes than the band has");
                    const int nbps = b.Mb - msbTree.value(leaf);
                    const int np = getPasses(hr);
                    int lblock = 3;
                    while (hr.bit())
                        if (++lblock > 24) bad("code-block length field too wide");
                    const uint32_t len = hr.get(lblock + floorLog2((uint32_t)np));
                    if (hr.overrun()) bad("packet header runs past its tile-part");
                    if (nbps < 1 || np > 3 * nbps - 2) bad("more coding passes than bit-planes allow");
                    GbCblkCode& cb = blocks[(size_t)(b.cblkBase + (pb.cby0 + j) * b.ncbx + pb.cbx0 + i)];
                    cb.len = len;
                    cb.passes = (uint8_t)np;
                    cb.nbps = (uint8_t)nbps;
                    body += len;
                }
        }
        const size_t hdr = hr.end();
        if (hr.overrun() || hdr > end - pos) bad("packet header runs past its tile-part");
        pos += hdr;
        if (eph && end - pos >= 2 && data[pos] == 0xFF && data[pos + 1] == (kEPH & 0xFF)) pos += 2;
        if (body > end - pos) bad("code-block data runs past its tile-part");
        for (int k = 0; present && k < P.nb; ++k) {
            const PrecinctBand& pb = P.bands[k];
            if (pb.ncbx <= 0 || pb.ncby <= 0) continue;
            const GbSubband& b = L.bands[pb.band];
            for (int j = 0; j < pb.ncby; ++j)
                for (int i = 0; i < pb.ncbx; ++i) {
                    GbCblkCode& cb = blocks[(size_t)(b.cblkBase + (pb.cby0 + j) * b.ncbx + pb.cbx0 + i)];
                    if (!cb.passes) continue;
                    cb.offset = (uint32_t)pos;
                    pos += cb.len;
                }
        }
        return pos;
    };
    // The DCI organisation: tile-part g holds exactly the packets of (volume g / 3,
    // component g % 3), so the tile-parts are read in parallel. Any other organisation
    // (packets spilling over tile-part boundaries) is read in order below.
    struct NotOneGroupPerPart {};
    bool done = false;
    if (parts.size() == volRs.size() * 3) {
        try {
            parallelFor((int)parts.size(), [&](int g) {
                const int v = g / 3, c = g % 3;
                size_t pos = parts[(size_t)g].b;
                const size_t end = parts[(size_t)g].e;
                forEachPacket(L, volRs[(size_t)v], volRe[(size_t)v], c, [&](int r, int prec) {
                    if (pos >= end) throw NotOneGroupPerPart{};
                    pos = parsePacket(c, r, prec, pos, end);
                });
                if (pos != end) throw NotOneGroupPerPart{};
            });
            done = true;
        } catch (const NotOneGroupPerPart&) {
            blocks.assign((size_t)L.numCblks(), GbCblkCode{});
        }
    }
    if (!done) {
        size_t tp = 0, pos = parts[0].b, end = parts[0].e;
        for (size_t v = 0; v < volRs.size(); ++v)
            for (int c = 0; c < kNumComps; ++c)
                forEachPacket(L, volRs[v], volRe[v], c, [&](int r, int prec) {
                    while (pos >= end) {
                        if (++tp >= parts.size()) bad("the tile-parts end before the last packet");
                        pos = parts[tp].b;
                        end = parts[tp].e;
                    }
                    pos = parsePacket(c, r, prec, pos, end);
                });
    }
}

}  // namespace gb
