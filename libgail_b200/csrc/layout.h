// Frame geometry of a single-tile DCI JPEG 2000 frame: subbands in Mallat layout,
// code-blocks, precincts and quantisation steps. Same numbering as the reference
// (Josephur/libgail src/core/layout.h:29-84, layout.cpp:77-210), which the plugin ABI
// carries unchanged: bands component-major then resolution (QCD order), code-blocks
// raster within each band, precincts 4 x 4 code-blocks in band coordinates.
#pragma once
#include <cstdint>
#include <vector>

#include "gail_cuda_plugin_abi.h"

namespace gb {

constexpr int kNumComps = 3;
constexpr int kBitDepth = 12;

struct CodeBlock {
    int band, x0, y0, w, h;  // position inside the band
};

struct PrecinctBand {
    int band = -1, cbx0 = 0, cby0 = 0, ncbx = 0, ncby = 0;
};

struct Precinct {
    int nb = 0;
    PrecinctBand bands[3];
};

struct Resolution {
    int comp = 0, res = 0, w = 0, h = 0, ppx = 0, ppy = 0, npx = 0, npy = 0;
    std::vector<Precinct> precincts;
};

struct Layout {
    int profile = 0;  // 0 2K, 1 4K
    int width = 0, height = 0, levels = 0, guardBits = 0;
    double baseStep = 1.0;
    std::vector<GbSubband> bands;
    std::vector<CodeBlock> cblks;
    std::vector<Resolution> resolutions;  // comp * (levels + 1) + res

    int numRes() const { return levels + 1; }
    int bandsPerComp() const { return 3 * levels + 1; }
    int bandIndex(int comp, int res, int orient) const {
        return comp * bandsPerComp() + (res == 0 ? 0 : 1 + 3 * (res - 1) + (orient - 1));
    }
    const Resolution& resolution(int comp, int res) const { return resolutions[(size_t)comp * numRes() + res]; }
    int numCblks() const { return (int)cblks.size(); }
    // widths / heights of the LL region after l levels
    int levelW(int l) const;
    int levelH(int l) const;
};

// Subbands, code-blocks and precincts of a frame; steps left unset.
Layout makeGeometry(int width, int height, int profile, int levels, int guardBits);
// The DCI layout: 5 levels and 1 guard bit at 2K, 6 and 2 at 4K; per-band steps for equal
// image-domain error from baseStep. Throws std::runtime_error on sizes outside the profile.
Layout makeLayout(int width, int height, int profile, double baseStep);
// Rebuilds the geometry from a plugin-ABI layout and takes its bands (steps) as given.
// Throws std::logic_error when the bands do not have the geometry of the size and levels.
void layoutFromAbi(const GailCudaLayout& p, Layout& L);
GailCudaLayout layoutToAbi(const Layout& L);
// The steps of component comp's bands from a QCD's (eps, mu) pairs, in QCD band order.
// Throws std::runtime_error on a step that needs more than 22 magnitude bit-planes.
void setSignalledSteps(Layout& L, int comp, const int* eps, const int* mu);

double synthesisNorm(int level, int orient);
double ictSynthesisNorm(int comp);

}  // namespace gb
