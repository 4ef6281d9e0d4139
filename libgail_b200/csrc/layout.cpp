// Frame geometry and quantisation steps (restates Josephur/libgail core/layout.cpp:77-210).
#include "layout.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>

namespace gb {

namespace {

constexpr double kK97 = 1.230174104914001;  // ISO/IEC 15444-1 Table F.4
constexpr double kLift[4] = {-1.586134342059924, -0.052980118572961, 0.882911075530934, 0.443506852043971};

// Inverse 9/7 of one line in double precision (scale, then undo the four lifting steps
// with the whole-sample symmetric mirror at the ends).
void inverseLine(const std::vector<double>& in, std::vector<double>& out, int n) {
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    const int sn = (n + 1) / 2;
    for (int i = 0; i < sn; ++i) out[2 * i] = in[i] * kK97;
    for (int i = 0; i < n / 2; ++i) out[2 * i + 1] = in[sn + i] * (1.0 / kK97);
    for (int s = 3; s >= 0; --s) {
        const int parity = (s & 1) ? 0 : 1;  // delta, beta touch even samples; gamma, alpha odd
        const double c = -kLift[s];
        for (int i = parity; i < n; i += 2) {
            const double l = i > 0 ? out[i - 1] : out[1];
            const double r = i + 1 < n ? out[i + 1] : out[n - 2];
            out[i] += c * (l + r);
        }
    }
}

// L2 norm of the 1-D synthesis basis of a low or high band at `level`.
double synth1d(int level, bool high) {
    const int n = 64 << level;
    std::vector<double> sig(n, 0.0), tmp(n, 0.0);
    const int band = n >> level;
    sig[high ? band + band / 2 : band / 2] = 1.0;
    for (int l = level; l >= 1; --l) {
        const int len = n >> (l - 1);
        inverseLine(sig, tmp, len);
        std::copy(tmp.begin(), tmp.begin() + len, sig.begin());
    }
    double e = 0;
    for (double v : sig) e += v * v;
    return std::sqrt(e);
}

int nominalRange(int orient) { return kBitDepth + (orient == 0 ? 0 : (orient == 3 ? 2 : 1)); }

void applyStep(GbSubband& b, int guardBits, int eps, int mu) {
    b.eps = eps;
    b.mu = mu;
    b.delta = (float)(std::ldexp(1.0, nominalRange(b.orient) - eps) * (1.0 + mu / 2048.0));
    b.Mb = guardBits + eps - 1;
    if (b.Mb > 22) throw std::runtime_error("quantization step too fine (more than 22 bitplanes)");
}

}  // namespace

double synthesisNorm(int level, int orient) {
    static std::mutex m;
    static std::map<std::pair<int, int>, double> cache;
    std::lock_guard<std::mutex> lock(m);
    const auto key = std::make_pair(level, orient);
    const auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    const bool hx = orient == 1 || orient == 3, hy = orient == 2 || orient == 3;
    const double v = synth1d(level, hx) * synth1d(level, hy);
    cache[key] = v;
    return v;
}

double ictSynthesisNorm(int comp) {
    // columns of the inverse ICT (ISO/IEC 15444-1 G.3)
    static const double cols[3][3] = {{1, 1, 1}, {0, -0.34413, 1.772}, {1.402, -0.71414, 0}};
    double e = 0;
    for (int i = 0; i < 3; ++i) e += cols[comp][i] * cols[comp][i];
    return std::sqrt(e);
}

int Layout::levelW(int l) const {
    int w = width;
    for (int i = 0; i < l; ++i) w = (w + 1) / 2;
    return w;
}
int Layout::levelH(int l) const {
    int h = height;
    for (int i = 0; i < l; ++i) h = (h + 1) / 2;
    return h;
}

Layout makeGeometry(int width, int height, int profile, int levels, int guardBits) {
    if (width < 1 || height < 1 || levels < 0 || levels > 32) throw std::logic_error("frame geometry out of range");
    Layout L;
    L.profile = profile;
    L.width = width;
    L.height = height;
    L.levels = levels;
    L.guardBits = guardBits;
    std::vector<int> ws(levels + 1), hs(levels + 1);
    ws[0] = width;
    hs[0] = height;
    for (int l = 1; l <= levels; ++l) {
        ws[l] = (ws[l - 1] + 1) / 2;
        hs[l] = (hs[l - 1] + 1) / 2;
    }
    int count = 0;
    for (int c = 0; c < kNumComps; ++c)
        for (int r = 0; r <= levels; ++r)
            for (int o = 0; o < (r == 0 ? 1 : 3); ++o) {
                GbSubband b{};
                b.comp = c;
                b.res = r;
                b.orient = r == 0 ? 0 : o + 1;
                b.level = r == 0 ? levels : levels - r + 1;
                const int n = b.level;
                const bool hx = b.orient == 1 || b.orient == 3, hy = b.orient == 2 || b.orient == 3;
                b.px0 = hx ? ws[n] : 0;
                b.py0 = hy ? hs[n] : 0;
                b.w = hx ? ws[n - 1] - ws[n] : ws[n];
                b.h = hy ? hs[n - 1] - hs[n] : hs[n];
                b.ncbx = (b.w + 31) / 32;
                b.ncby = (b.h + 31) / 32;
                b.cblkBase = count;
                b.delta = 1.f;
                b.weight = 1.0;
                count += b.ncbx * b.ncby;
                L.bands.push_back(b);
            }
    L.cblks.resize(count);
    for (int bi = 0; bi < (int)L.bands.size(); ++bi) {
        const GbSubband& b = L.bands[bi];
        for (int cy = 0; cy < b.ncby; ++cy)
            for (int cx = 0; cx < b.ncbx; ++cx)
                L.cblks[b.cblkBase + cy * b.ncbx + cx] = {bi, cx * 32, cy * 32, std::min(32, b.w - cx * 32),
                                                          std::min(32, b.h - cy * 32)};
    }
    // precincts: 2^7 at resolution 0, 2^8 above (DCI); 4 x 4 code-blocks in band coordinates
    for (int c = 0; c < kNumComps; ++c)
        for (int r = 0; r <= levels; ++r) {
            Resolution R;
            R.comp = c;
            R.res = r;
            R.w = ws[levels - r];
            R.h = hs[levels - r];
            R.ppx = R.ppy = r == 0 ? 7 : 8;
            R.npx = (R.w + (1 << R.ppx) - 1) >> R.ppx;
            R.npy = (R.h + (1 << R.ppy) - 1) >> R.ppy;
            const int cbPerPrec = 1 << ((r == 0 ? R.ppx : R.ppx - 1) - 5);
            R.precincts.resize((size_t)R.npx * R.npy);
            for (int py = 0; py < R.npy; ++py)
                for (int px = 0; px < R.npx; ++px) {
                    Precinct& P = R.precincts[(size_t)py * R.npx + px];
                    P.nb = r == 0 ? 1 : 3;
                    for (int k = 0; k < P.nb; ++k) {
                        const int bi = L.bandIndex(c, r, r == 0 ? 0 : k + 1);
                        const GbSubband& b = L.bands[bi];
                        PrecinctBand& pb = P.bands[k];
                        pb.band = bi;
                        pb.cbx0 = px * cbPerPrec;
                        pb.cby0 = py * cbPerPrec;
                        pb.ncbx = std::max(0, std::min(cbPerPrec, b.ncbx - pb.cbx0));
                        pb.ncby = std::max(0, std::min(cbPerPrec, b.ncby - pb.cby0));
                        if (pb.ncbx == 0 || pb.ncby == 0) pb.ncbx = pb.ncby = 0;
                    }
                }
            L.resolutions.push_back(std::move(R));
        }
    return L;
}

Layout makeLayout(int width, int height, int profile, double baseStep) {
    const bool fourk = profile == 1;
    if (fourk ? (width > 4096 || height > 2160) : (width > 2048 || height > 1080))
        throw std::runtime_error("image size exceeds the DCI container for this profile");
    if (width < 64 || height < 64) throw std::runtime_error("image too small");
    Layout L = makeGeometry(width, height, profile, fourk ? 6 : 5, fourk ? 2 : 1);
    L.baseStep = baseStep;
    for (GbSubband& b : L.bands) {
        // equal image-domain error per coefficient: step = baseStep / synthesis norm,
        // signalled as 2^(Rb - eps) (1 + mu / 2^11)
        const double norm = synthesisNorm(b.level, b.orient);
        const double x = (baseStep / norm) / std::ldexp(1.0, nominalRange(b.orient));
        int eps = (int)std::ceil(-std::log2(x));
        if (std::ldexp(x, eps) < 1.0) ++eps;
        if (std::ldexp(x, eps) >= 2.0) --eps;
        int mu = (int)std::lround((std::ldexp(x, eps) - 1.0) * 2048.0);
        if (mu >= 2048) {
            mu = 0;
            --eps;
        }
        if (eps < 0 || eps > 31) throw std::runtime_error("quantization step out of range");
        applyStep(b, L.guardBits, eps, mu);
        const double wc = ictSynthesisNorm(b.comp);
        b.weight = norm * norm * wc * wc;
    }
    return L;
}

void setSignalledSteps(Layout& L, int comp, const int* eps, const int* mu) {
    for (GbSubband& b : L.bands) {
        if (b.comp != comp) continue;
        const int i = b.res == 0 ? 0 : 1 + 3 * (b.res - 1) + (b.orient - 1);
        applyStep(b, L.guardBits, eps[i], mu[i]);
        b.weight = 0.0;  // only the encoder's rate control uses it
    }
}

void layoutFromAbi(const GailCudaLayout& p, Layout& L) {
    if (p.numBands < 0 || p.numCblks < 0 || !p.bands) throw std::logic_error("frame layout is empty");
    if (L.profile != p.profile || L.width != p.width || L.height != p.height || L.levels != p.levels ||
        L.guardBits != p.guardBits || (int)L.bands.size() != p.numBands)
        L = makeGeometry(p.width, p.height, p.profile, p.levels, p.guardBits);
    if ((int)L.bands.size() != p.numBands || L.numCblks() != p.numCblks)
        throw std::logic_error("frame layout does not have the geometry of its size and levels");
    for (int i = 0; i < p.numBands; ++i) {
        const GbSubband& a = p.bands[i];
        const GbSubband& g = L.bands[i];
        if (a.comp != g.comp || a.orient != g.orient || a.px0 != g.px0 || a.py0 != g.py0 || a.w != g.w || a.h != g.h ||
            a.cblkBase != g.cblkBase)
            throw std::logic_error("frame layout band " + std::to_string(i) + " does not match its geometry");
        if (a.Mb < 0 || a.Mb > 22 || !(a.delta > 0.f)) throw std::logic_error("band step out of range");
    }
    L.baseStep = p.baseStep;
    L.bands.assign(p.bands, p.bands + p.numBands);
}

GailCudaLayout layoutToAbi(const Layout& L) {
    return {L.profile, L.width, L.height, L.levels, L.guardBits, (int32_t)L.bands.size(), (int32_t)L.cblks.size(),
            L.baseStep, L.bands.data()};
}

}  // namespace gb
