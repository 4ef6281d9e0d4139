// DCI codestream compliance: checkDci.
//
// Gives the verdict of the reference's checker (checkDciCodestream,
// src/core/codestream_check.cpp:43-280) on the DCI rules it enforces, from a design of its
// own, in three steps:
//
//   1. a segment walker splits the codestream into marker segments (bare markers, segments
//      with a length, tile-parts) and stops at the first structural fault: a missing marker,
//      a segment that runs past the data, an unusable Psot, a marker DCI does not allow;
//   2. each segment is checked against the rule of its marker: where it may stand (main
//      header or between tile-parts), its length, and its fields against a table of
//      expected values (fixed, or per profile, or the image size);
//   3. rules over the whole frame: how many of each marker, the tile-part sequence, the
//      TLM lengths against the tile-parts, and the byte caps of the frame, of each
//      tile-part and of each component at the frame rate.
//
// The rules are the DCI profile's (SMPTE ST 429-4 with the 2K / 4K cinema profiles of
// ISO/IEC 15444-1 Amd. 1, and the 250 / 200 Mbit/s limits): Rsiz 3 or 4, one tile, three
// 12-bit unsubsampled components, CPRL, one layer, the component transform, 5 or 6 levels,
// 32x32 code-blocks without mode switches, the 9/7 wavelet, 128/256 precincts, scalar
// expounded quantisation with 1 or 2 guard bits, the 4K progression order change, TLM, 3 or
// 6 tile-parts (one per component, and per resolution group at 4K), no marker codes in the
// packet data. The byte caps round as the reference rounds them (the frame and 230 Mbit/s
// caps to the nearest byte, the 200 Mbit/s cap down), so that the verdict agrees at every
// frame rate.
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "codestream.h"

namespace gb {

namespace {

// marker codes (ISO/IEC 15444-1 Table A.2)
enum : uint16_t {
    M_SOC = 0xFF4F, M_SIZ = 0xFF51, M_COD = 0xFF52, M_COC = 0xFF53, M_TLM = 0xFF55, M_QCD = 0xFF5C,
    M_QCC = 0xFF5D, M_POC = 0xFF5F, M_COM = 0xFF64, M_SOT = 0xFF90, M_SOD = 0xFF93, M_EOC = 0xFFD9,
};

std::string hex(uint32_t v) {
    char b[16];
    std::snprintf(b, sizeof b, "0x%X", v);
    return b;
}

// Big-endian reads inside one segment's body; a read past the body yields 0 and marks the
// segment short.
struct Body {
    const uint8_t* p = nullptr;
    size_t n = 0;
    mutable bool shortRead = false;
    uint32_t at(size_t off, int width) const {
        if (off + (size_t)width > n) {
            shortRead = true;
            return 0;
        }
        uint32_t v = 0;
        for (int i = 0; i < width; ++i) v = (v << 8) | p[off + (size_t)i];
        return v;
    }
};

struct Segment {
    uint16_t code;
    size_t offset;      // of the marker
    bool mainHeader;    // before the first SOT
    Body body;          // after the length field (segments with a length)
    size_t tilePartEnd; // SOT: offset just past the tile-part
};

// ---- step 1: the segment walker ------------------------------------------------------

enum class Shape { Bare, Sized, TilePart };

Shape shapeOf(uint16_t code) {
    switch (code) {
        case M_SOC:
        case M_EOC:
            return Shape::Bare;
        case M_SOT:
            return Shape::TilePart;
        default:
            return Shape::Sized;
    }
}

bool allowedInDci(uint16_t code) {
    switch (code) {
        case M_SIZ: case M_COD: case M_COC: case M_TLM: case M_QCD: case M_QCC: case M_POC: case M_COM:
        case M_SOT: case M_EOC:
            return true;
        default:
            return false;
    }
}

struct Walk {
    std::vector<Segment> segments;
    bool broken = false;  // the walk stopped at a structural fault
};

Walk walkSegments(const uint8_t* d, size_t size, DciReport& r) {
    Walk w;
    auto fault = [&](std::string s) {
        r.error(std::move(s));
        w.broken = true;
    };
    auto marker = [&](size_t at) -> int { return at + 2 <= size ? (d[at] << 8) | d[at + 1] : -1; };
    if (marker(0) != M_SOC) {
        fault("the codestream does not open with SOC");
        return w;
    }
    w.segments.push_back({M_SOC, 0, true, {}, 0});
    if (marker(2) != M_SIZ) {
        fault("SOC is not followed by SIZ");
        return w;
    }
    size_t at = 2;
    bool main = true;
    while (at < size) {
        const int m = marker(at);
        if (m < 0 || (m >> 8) != 0xFF) {
            fault("expected a marker at byte " + std::to_string(at));
            break;
        }
        const uint16_t code = (uint16_t)m;
        if (!allowedInDci(code)) {
            fault("marker " + hex(code) + " at byte " + std::to_string(at) + " is not allowed in a DCI codestream");
            break;
        }
        Segment s{code, at, main, {}, 0};
        const Shape shape = shapeOf(code);
        if (shape == Shape::Bare) {  // EOC: the last two bytes
            w.segments.push_back(s);
            at += 2;
            if (at != size) r.error("bytes follow EOC");
            break;
        }
        const size_t len = at + 4 <= size ? ((size_t)d[at + 2] << 8 | d[at + 3]) : 0;
        if (len < 2 || at + 2 + len > size) {
            fault("segment " + hex(code) + " at byte " + std::to_string(at) + " runs past the data");
            break;
        }
        s.body = {d + at + 4, len - 2};
        if (shape == Shape::TilePart) {
            main = false;
            s.mainHeader = false;
            const uint32_t psot = s.body.at(2, 4);
            if (psot < 14 || psot > size - at) {
                w.segments.push_back(s);
                fault("tile-part at byte " + std::to_string(at) + " has an unusable length (Psot " +
                      std::to_string(psot) + ")");
                break;
            }
            s.tilePartEnd = at + psot;
            w.segments.push_back(s);
            at += psot;
        } else {
            w.segments.push_back(s);
            at += 2 + len;
        }
    }
    return w;
}

// ---- step 2: per-marker rules --------------------------------------------------------

struct Frame {
    bool fourk = false;
    int width = 0, height = 0;
    int levels() const { return fourk ? 6 : 5; }
    int resolutions() const { return levels() + 1; }
    int tilePartsWanted() const { return fourk ? 6 : 3; }
};

// An expected field value: a constant, one per profile, or the image width / height.
struct Expect {
    enum Kind { Const, Profile, Width, Height } kind;
    uint32_t a, b;  // Const: a; Profile: a (2K) / b (4K)
    uint32_t value(const Frame& f) const {
        switch (kind) {
            case Profile: return f.fourk ? b : a;
            case Width: return (uint32_t)f.width;
            case Height: return (uint32_t)f.height;
            default: return a;
        }
    }
};

struct FieldRule {
    uint16_t offset;  // in the segment body (after the length field)
    uint8_t width;    // bytes
    uint8_t shift;    // bits the value is shifted down by
    uint32_t mask;    // of the shifted value
    Expect expect;
    const char* what;
};

constexpr uint32_t ALL = 0xFFFFFFFFu;

// SIZ body: Rsiz, Xsiz, Ysiz, XOsiz, YOsiz, XTsiz, YTsiz, XTOsiz, YTOsiz, Csiz, then
// Ssiz / XRsiz / YRsiz per component
const FieldRule kSizRules[] = {
    {0, 2, 0, ALL, {Expect::Profile, 3, 4}, "Rsiz is not the cinema profile of the image size"},
    {10, 4, 0, ALL, {Expect::Const, 0, 0}, "image x offset"},
    {14, 4, 0, ALL, {Expect::Const, 0, 0}, "image y offset"},
    {18, 4, 0, ALL, {Expect::Width, 0, 0}, "tile width is not the image width (one tile)"},
    {22, 4, 0, ALL, {Expect::Height, 0, 0}, "tile height is not the image height (one tile)"},
    {26, 4, 0, ALL, {Expect::Const, 0, 0}, "tile x offset"},
    {30, 4, 0, ALL, {Expect::Const, 0, 0}, "tile y offset"},
    {34, 2, 0, ALL, {Expect::Const, 3, 3}, "component count is not 3"},
};
const FieldRule kSizComponentRules[] = {
    {36, 1, 0, ALL, {Expect::Const, 11, 11}, "component is not 12-bit unsigned"},
    {37, 1, 0, ALL, {Expect::Const, 1, 1}, "component is subsampled horizontally"},
    {38, 1, 0, ALL, {Expect::Const, 1, 1}, "component is subsampled vertically"},
};

// COD body: Scod, progression, layers, MCT, levels, xcb, ycb, style, transform, precincts
const FieldRule kCodRules[] = {
    {0, 1, 0, ALL, {Expect::Const, 1, 1}, "Scod: precincts must be signalled, without SOP / EPH"},
    {1, 1, 0, ALL, {Expect::Const, 4, 4}, "progression order is not CPRL"},
    {2, 2, 0, ALL, {Expect::Const, 1, 1}, "more than one quality layer"},
    {4, 1, 0, ALL, {Expect::Const, 1, 1}, "no multiple component transform"},
    {5, 1, 0, ALL, {Expect::Profile, 5, 6}, "decomposition levels are not the profile's"},
    {6, 1, 0, ALL, {Expect::Const, 3, 3}, "code-block width is not 32"},
    {7, 1, 0, ALL, {Expect::Const, 3, 3}, "code-block height is not 32"},
    {8, 1, 0, ALL, {Expect::Const, 0, 0}, "code-block mode switches"},
    {9, 1, 0, ALL, {Expect::Const, 0, 0}, "wavelet is not the irreversible 9/7"},
};

// QCD body: Sqcd (style in the low 5 bits, guard bits in the high 3), then 16-bit SPqcd
const FieldRule kQcdRules[] = {
    {0, 1, 0, 0x1F, {Expect::Const, 2, 2}, "quantisation is not scalar expounded"},
    {0, 1, 5, 0x07, {Expect::Profile, 1, 2}, "guard bits are not the profile's"},
};

// POC body: two progression changes (RSpoc CSpoc LYEpoc REpoc CEpoc Ppoc), the 4K profile's
// 2K-resolutions-first order: resolutions 0-5 of every component, then resolution 6
const FieldRule kPocRules[] = {
    {0, 1, 0, ALL, {Expect::Const, 0, 0}, "POC"},  {1, 1, 0, ALL, {Expect::Const, 0, 0}, "POC"},
    {2, 2, 0, ALL, {Expect::Const, 1, 1}, "POC"},  {4, 1, 0, ALL, {Expect::Const, 6, 6}, "POC"},
    {5, 1, 0, ALL, {Expect::Const, 3, 3}, "POC"},  {6, 1, 0, ALL, {Expect::Const, 4, 4}, "POC"},
    {7, 1, 0, ALL, {Expect::Const, 6, 6}, "POC"},  {8, 1, 0, ALL, {Expect::Const, 0, 0}, "POC"},
    {9, 2, 0, ALL, {Expect::Const, 1, 1}, "POC"},  {11, 1, 0, ALL, {Expect::Const, 7, 7}, "POC"},
    {12, 1, 0, ALL, {Expect::Const, 3, 3}, "POC"}, {13, 1, 0, ALL, {Expect::Const, 4, 4}, "POC"},
};

template <size_t N>
void applyFields(const FieldRule (&rules)[N], const Body& b, const Frame& f, DciReport& r, size_t base = 0,
                 const std::string& prefix = "") {
    for (const FieldRule& fr : rules) {
        const uint32_t v = (b.at(base + fr.offset, fr.width) >> fr.shift) & fr.mask;
        if (v != fr.expect.value(f)) r.error(prefix + fr.what + " (" + std::to_string(v) + ")");
    }
}

// What the frame-level rules need from the segments.
struct Tally {
    int cod = 0, qcd = 0, pocMain = 0, pocLater = 0, tlm = 0;
    std::vector<uint32_t> tlmLengths;  // Ptlm entries in order
    std::vector<uint32_t> partLengths; // Psot of each tile-part in order
    bool eoc = false;
};

void checkSiz(const Segment& s, Frame& f, DciReport& r) {
    const Body& b = s.body;
    if (b.n + 2 != 47) r.error("Lsiz is " + std::to_string(b.n + 2) + " (47 for three components)");
    r.rsiz = (int)b.at(0, 2);
    f.width = r.width = (int)b.at(2, 4);
    f.height = r.height = (int)b.at(6, 4);
    f.fourk = f.width > 2048;
    const int maxW = f.fourk ? 4096 : 2048, maxH = f.fourk ? 2160 : 1080;
    if (f.width > maxW || f.height > maxH) r.error("image larger than the DCI container of its profile");
    applyFields(kSizRules, b, f, r);
    const int comps = (int)b.at(34, 2);
    for (int c = 0; c < comps && c < 3; ++c)
        applyFields(kSizComponentRules, b, f, r, 3 * (size_t)c, "component " + std::to_string(c) + ": ");
    if (b.shortRead) r.error("SIZ is shorter than its fields");
}

void checkCod(const Segment& s, const Frame& f, DciReport& r) {
    const Body& b = s.body;
    if (!s.mainHeader) r.error("COD outside the main header");
    r.levels = (int)b.at(5, 1);
    applyFields(kCodRules, b, f, r);
    const int nres = f.resolutions();
    if (b.n != (size_t)(10 + nres)) r.error("Lcod is " + std::to_string(b.n + 2));
    // precinct sizes, lowest resolution first: 2^7 x 2^7 there, 2^8 x 2^8 above
    for (int i = 0; i < nres && (size_t)(10 + i) < b.n; ++i)
        if (b.at(10 + (size_t)i, 1) != (i == 0 ? 0x77u : 0x88u)) {
            r.error("precinct size of resolution " + std::to_string(i));
            break;
        }
}

void checkQcd(const Segment& s, const Frame& f, DciReport& r) {
    const Body& b = s.body;
    applyFields(kQcdRules, b, f, r);
    const int bands = 3 * f.levels() + 1;
    if (b.n != (size_t)(1 + 2 * bands)) r.error("Lqcd is " + std::to_string(b.n + 2));
    const int guard = (int)(b.at(0, 1) >> 5);
    // magnitude bit-planes of each band: guard bits + exponent - 1, at most 30 (the bits a
    // 32-bit sign-magnitude coefficient word holds beside its fraction)
    for (size_t i = 0; i < (size_t)bands && 3 + 2 * i <= b.n; ++i) {
        const int exponent = (int)(b.at(1 + 2 * i, 2) >> 11);
        if (guard + exponent - 1 > 30) r.error("band " + std::to_string(i) + " signals over 30 bit-planes");
    }
}

void checkPoc(const Segment& s, const Frame& f, DciReport& r) {
    if (s.body.n != 14) {
        r.error("Lpoc is " + std::to_string(s.body.n + 2));
        return;
    }
    DciReport one;
    applyFields(kPocRules, s.body, f, one);
    if (!one.ok) r.error("POC is not the DCI 4K progression");
}

void readTlm(const Segment& s, Tally& t) {
    const Body& b = s.body;
    const uint32_t stlm = b.at(1, 1);
    const int st = (int)((stlm >> 4) & 3);
    const int tileIndexBytes = st == 3 ? 0 : st;      // ST = 3 is reserved: read as none
    const int lengthBytes = (stlm >> 6) & 1 ? 4 : 2;  // SP
    const size_t entry = (size_t)(tileIndexBytes + lengthBytes);
    for (size_t off = 2; off + entry <= b.n; off += entry) t.tlmLengths.push_back(b.at(off + tileIndexBytes, lengthBytes));
}

void checkTilePart(const uint8_t* d, const Segment& s, const Frame& f, double partCap, Tally& t, DciReport& r) {
    const Body& b = s.body;
    if (b.n != 8) r.error("Lsot is " + std::to_string(b.n + 2));
    const uint32_t isot = b.at(0, 2), psot = b.at(2, 4), tpsot = b.at(6, 1), tnsot = b.at(7, 1);
    if (isot != 0) r.error("tile index " + std::to_string(isot) + " (one tile)");
    if ((int)tnsot != f.tilePartsWanted())
        r.error("TNsot " + std::to_string(tnsot) + " (the profile has " + std::to_string(f.tilePartsWanted()) + ")");
    if ((int)tpsot != (int)t.partLengths.size())
        r.error("tile-part " + std::to_string(tpsot) + " where " + std::to_string(t.partLengths.size()) + " belongs");
    t.partLengths.push_back(psot);
    // tile-part k holds component k mod 3 (one tile-part per component, per resolution
    // group at 4K)
    r.compBytes[tpsot % 3] += psot;
    if ((double)psot > partCap)
        r.error("tile-part " + std::to_string(tpsot) + " is " + std::to_string(psot) + " bytes, over the 200 Mbit/s cap");
    // SOD closes the tile-part header (Lsot 10: the header is SOT alone)
    const size_t sod = s.offset + 12;
    if (sod + 2 > s.tilePartEnd || ((d[sod] << 8) | d[sod + 1]) != M_SOD) r.error("SOT is not followed by SOD");
    // packet data: no two-byte sequence in the marker range 0xFF90-0xFFFF
    for (size_t q = sod + 2; q + 1 < s.tilePartEnd; ++q)
        if (d[q] == 0xFF && d[q + 1] >= 0x90) {
            r.error("marker code " + hex((uint32_t)(0xFF00 | d[q + 1])) + " inside packet data at byte " +
                    std::to_string(q));
            break;
        }
}

// The byte caps at a frame rate: the 250 Mbit/s frame cap and the 230 Mbit/s level to the
// nearest byte, the 200 Mbit/s tile-part and component cap rounded down.
struct Caps {
    double frame, nearFrame, part;
};

double bytesAt(double mbits, double fps) { return mbits * 1e6 / (8.0 * fps); }

Caps capsAt(double fps) {
    return {std::nearbyint(bytesAt(250.0, fps)), std::nearbyint(bytesAt(230.0, fps)), std::floor(bytesAt(200.0, fps))};
}

}  // namespace

DciReport checkDci(const uint8_t* data, size_t size, double fps) {
    DciReport r;
    r.totalBytes = size;
    const Walk walk = walkSegments(data, size, r);
    const Caps caps = capsAt(fps);
    Frame f;
    Tally t;
    for (const Segment& s : walk.segments) {
        switch (s.code) {
            case M_SIZ: checkSiz(s, f, r); break;
            case M_COD: ++t.cod; checkCod(s, f, r); break;
            case M_QCD: ++t.qcd; checkQcd(s, f, r); break;
            case M_POC: ++(s.mainHeader ? t.pocMain : t.pocLater); checkPoc(s, f, r); break;
            case M_TLM: ++t.tlm; readTlm(s, t); break;
            case M_COC: r.warnings.push_back("COC marker"); break;
            case M_COM:
                // Rcom 1: Latin text, kept from the main header
                if (s.mainHeader && s.body.n >= 2 && s.body.at(0, 2) == 1)
                    r.comment.assign((const char*)s.body.p + 2, s.body.n - 2);
                break;
            case M_SOT:
                if (s.tilePartEnd) checkTilePart(data, s, f, caps.part, t, r);
                break;
            case M_EOC: t.eoc = true; break;
            default: break;  // SOC, QCC: nothing to check
        }
    }
    r.tileParts = (int)t.partLengths.size();

    // ---- step 3: rules over the whole frame ----
    struct FrameRule {
        bool holds;
        std::string what;
    };
    const FrameRule rules[] = {
        {!walk.broken, "the codestream is truncated or malformed"},
        {t.eoc, "no EOC"},
        {t.cod == 1, "COD appears " + std::to_string(t.cod) + " times (once)"},
        {t.qcd == 1, "QCD appears " + std::to_string(t.qcd) + " times (once)"},
        {t.pocMain == (f.fourk ? 1 : 0), f.fourk ? "a 4K codestream needs one POC in its main header"
                                                 : "POC in a 2K codestream"},
        {t.pocLater == 0, "POC outside the main header"},
        {t.tlm > 0, "no TLM"},
        {(int)t.partLengths.size() == f.tilePartsWanted(),
         std::to_string(t.partLengths.size()) + " tile-parts (the profile has " + std::to_string(f.tilePartsWanted()) +
             ")"},
        {t.tlm == 0 || t.tlmLengths == t.partLengths, "TLM lengths do not match the tile-parts"},
        {(double)r.compBytes[0] <= caps.part, "component 0 over the 200 Mbit/s cap"},
        {(double)r.compBytes[1] <= caps.part, "component 1 over the 200 Mbit/s cap"},
        {(double)r.compBytes[2] <= caps.part, "component 2 over the 200 Mbit/s cap"},
        {(double)size <= caps.frame, "frame of " + std::to_string(size) + " bytes over the 250 Mbit/s cap"},
    };
    for (const FrameRule& fr : rules)
        if (!fr.holds) r.error(fr.what);
    if ((double)size <= caps.frame && (double)size > caps.nearFrame) r.warnings.push_back("frame above 230 Mbit/s");
    return r;
}

}  // namespace gb
