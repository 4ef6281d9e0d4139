// Host codec around the Tier-1 frame: PCRD rate control under the DCI byte limits, Tier-2
// packets (tag trees, CPRL with the DCI 4K progression order change), the codestream
// (main header, one tile in 3 or 6 tile-parts with TLM), the DCI compliance check, and
// the reading of a codestream back into per-block code for the decoder.
//
// The reference does these on the CPU in libgail's core (src/core/rate_control.cpp,
// t2.cpp, tagtree.h, bitio.h, progression.h, codestream_check.cpp,
// codestream_parse.cpp, t2_parse.cpp); the results here are byte-identical for the
// same Tier-1 frame. Built for throughput on a host feeding a B200: the packet order is
// flattened once per layout, and rate control re-measures only the packets whose
// code-blocks changed their pass count since the previous measurement.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "gail_cuda_plugin_abi.h"
#include "layout.h"

namespace gb {

// A Tier-1 frame as the plugin hands it out (GailCudaTier1).
struct Tier1View {
    const GbCblkInfo* info = nullptr;
    const uint32_t* passLen = nullptr;
    const int32_t* passDist = nullptr;
    const uint8_t* data = nullptr;
    uint32_t numInfo = 0, numPasses = 0;
    uint64_t numData = 0;
    uint32_t len(int i, int k) const { return passLen[info[i].passBase + k]; }
    int32_t dist(int i, int k) const { return passDist[info[i].passBase + k]; }
};

struct CodestreamSizes {
    size_t total = 0;
    size_t comp[3] = {0, 0, 0};  // each component's tile-parts, SOT and SOD included
    int numTileParts = 0;
    size_t tilePart[6] = {};
};

// The longest device tag a codestream comment carries after its label ("cuda99.99").
constexpr size_t kMaxDeviceTagBytes = 9;

// The packets of one layout in codestream order, and the writer of its codestreams.
// Not thread-safe: one per worker thread.
class CodestreamWriter {
public:
    // label: the first part of the COM text (the encoder's name and version); the sizes
    // it reports budget for label + " " + the longest device tag, so the coded data do not
    // depend on the tag.
    CodestreamWriter(const Layout& L, std::string label);

    // Measures (out == nullptr) or writes the codestream with passes[i] coding passes of
    // block i; tag is appended to the label after a space (none when empty).
    CodestreamSizes build(const Tier1View& t1, const uint8_t* passes, std::vector<uint8_t>* out,
                          const std::string& tag = std::string());
    // Measurement that re-codes only the packets with a block whose pass count differs
    // from the previous call's since restart() (after it, every packet). Same sizes as
    // build(); the Tier-1 frame must stay the same between restarts.
    void restart() { measured_ = false; }
    CodestreamSizes measure(const Tier1View& t1, const uint8_t* passes);
    // The size with no coding pass at all: the smallest frame the layout can give.
    size_t emptyBytes();

    const Layout& layout() const { return L_; }
    const std::string& label() const { return label_; }
    int numPackets() const { return (int)pkStart_.size() - 1; }

    // The packet structure, for writers elsewhere (the device Tier-2): the segments (one
    // precinct-band each) of packet p are [packetSegments()[p], packetSegments()[p + 1]);
    // the packets of tile-part t are [tilePartPackets()[t], tilePartPackets()[t + 1]).
    struct Seg {  // one precinct-band of a packet
        int32_t band, cbx0, cby0, ncbx, ncby;
    };
    const std::vector<Seg>& segments() const { return segs_; }
    const std::vector<int32_t>& packetSegments() const { return pkStart_; }
    const std::vector<int32_t>& tilePartPackets() const { return tpStart_; }
    int numTileParts() const { return ntp_; }
    // The main header with the longest comment the label allows (what sizes budget for).
    size_t longestHeaderBytes();
    // The codestream around packets written elsewhere. body: the tile-parts back to back,
    // each 14 bytes of room for its SOT segment and SOD, then its packets; tpBytes: each
    // tile-part's bytes (those 14 included). Returns the sizes as build() reports them.
    CodestreamSizes assemble(const uint8_t* body, const uint64_t* tpBytes, const std::string& tag,
                             std::vector<uint8_t>& out) const;

private:
    size_t packet(int p, const Tier1View& t1, const uint8_t* passes, std::vector<uint8_t>* out);
    void mainHeader(std::vector<uint8_t>& v, const std::string& comment) const;

    Layout L_;
    std::string label_;
    int ntp_ = 0;
    std::vector<int32_t> tpStart_;   // packets of tile-part t: [tpStart_[t], tpStart_[t + 1])
    std::vector<int32_t> pkStart_;   // segments of packet p: [pkStart_[p], pkStart_[p + 1])
    std::vector<Seg> segs_;
    std::vector<int32_t> blockPacket_;  // the packet that carries block i
    // incremental measurement state
    std::vector<uint8_t> lastPasses_;
    std::vector<uint32_t> pkBytes_;
    std::vector<uint8_t> dirty_;
    bool measured_ = false;
    size_t hdrLongest_ = 0;  // the main header with the longest comment
};

struct RateLimits {
    size_t maxTotal = 0;  // bytes per frame, the whole codestream
    size_t maxComp = 0;   // bytes per component (its tile-parts)
};

// The DCI budgets at a frame rate, strictly below maxMbps and compMbps.
RateLimits dciLimits(double fps, double maxMbps = 230.0, double compMbps = 200.0);

struct RateResult {
    std::vector<uint8_t> passes;  // passes included per block
    double lambda = 0;            // the final slope threshold (largest of the components')
    double lambdaComp[3] = {0, 0, 0};
    double distortion = 0;        // estimated remaining weighted squared error (NaN when
                                  // the hull came precomputed, without the gains)
    CodestreamSizes sizes;
    int iterations = 0;           // exact measurements taken
    size_t d2hBytes = 0;          // device-to-host bytes the device rate control read back
    int launches = 0;             // kernels the device rate control launched
};

// Per block, the points of the lower convex hull of its (truncation length, weighted
// distortion reduction) curve, laid out like the Tier-1 pass tables: block i's points at
// its passBase, in order, ending at its pass count or at the first entry with passes 0.
// passes: coding passes at the point; slope: distortion reduction per byte from the
// previous point (+inf for no added bytes).
struct HullView {
    const uint8_t* passes = nullptr;
    const double* slope = nullptr;
};

// The hull points of every block into passes/slope (t1.numPasses entries each), by the
// arithmetic allocateRate uses.
void computeHull(const Layout& L, const Tier1View& t1, uint8_t* passes, double* slope);

// PCRD-opt: per block the convex hull of (rate, weighted distortion reduction) over its
// truncation points, one slope threshold per component, the largest set of passes whose
// codestream fits the limits. With hull, its points are taken instead of computed (they
// must be those computeHull gives; a malformed hull throws).
RateResult allocateRate(CodestreamWriter& w, const Tier1View& t1, const RateLimits& lim,
                        const HullView* hull = nullptr);

struct DciReport {
    bool ok = true;
    std::vector<std::string> errors;
    std::vector<std::string> warnings;
    int rsiz = 0, width = 0, height = 0, levels = 0, tileParts = 0;
    size_t totalBytes = 0, compBytes[3] = {0, 0, 0};
    std::string comment;
    void error(std::string s) {
        ok = false;
        errors.push_back(std::move(s));
    }
};

// DCI compliance (SMPTE ST 429-4 cinema profiles with the 250 Mbit/s frame and 200 Mbit/s
// component limits at fps, as libdcp checks them).
DciReport checkDci(const uint8_t* data, size_t size, double fps);

// Reads a codestream back for the decoder: its layout (geometry and the signalled steps)
// and each block's code (offset and length into the codestream, passes, coded
// bit-planes), in layout order. Throws std::runtime_error on a codestream this decoder
// does not take (not single-tile DCI, not one layer, ...) or one that is damaged.
void parseCodestream(const uint8_t* data, size_t size, Layout& L, std::vector<GbCblkCode>& blocks);

}  // namespace gb
