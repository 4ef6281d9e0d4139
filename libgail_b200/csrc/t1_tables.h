// Context and probability tables of EBCOT Tier-1 (ISO/IEC 15444-1 Tables C.2, D.1 and
// D.3), built on the host in the packed forms the kernels index.
#pragma once
#include <cstdint>

namespace gb {

// Zero-coding context from the counts of significant horizontal (h, 0..2), vertical
// (v, 0..2) and diagonal (d, 0..4) neighbours; orient 0 LL, 1 HL, 2 LH, 3 HH (Table D.1).
inline int zcContext(int h, int v, int d, int orient) {
    if (orient == 3) {
        const int hv = h + v;
        if (d >= 3) return 8;
        if (d == 2) return hv >= 1 ? 7 : 6;
        if (d == 1) return hv >= 2 ? 5 : (hv == 1 ? 4 : 3);
        return hv >= 2 ? 2 : hv;
    }
    if (orient == 1) {  // the horizontally high-pass band swaps the roles of h and v
        const int t = h;
        h = v;
        v = t;
    }
    if (h == 2) return 8;
    if (h == 1) return v >= 1 ? 7 : (d >= 1 ? 6 : 5);
    if (v == 2) return 4;
    if (v == 1) return 3;
    return d >= 2 ? 2 : d;
}

// Sign-coding context and XOR bit from the clamped horizontal and vertical sign
// contributions hc, vc in -1..1 (Table D.3).
inline void scContext(int hc, int vc, int& cx, int& xorbit) {
    if (hc == 0) {
        cx = vc == 0 ? 9 : 10;
        xorbit = vc < 0 ? 1 : 0;
        return;
    }
    const int v = hc > 0 ? vc : -vc;  // the table is symmetric under negating both
    cx = v > 0 ? 13 : (v == 0 ? 12 : 11);
    xorbit = hc < 0 ? 1 : 0;
}

// MQ probability states (Table C.2): Qe, next index after an MPS / LPS, and the switch.
struct MqState {
    uint16_t qe;
    uint8_t nmps, nlps, sw;
};
inline const MqState* mqStates() {
    static const MqState t[47] = {
        {0x5601, 1, 1, 1},   {0x3401, 2, 6, 0},   {0x1801, 3, 9, 0},   {0x0AC1, 4, 12, 0},  {0x0521, 5, 29, 0},
        {0x0221, 38, 33, 0}, {0x5601, 7, 6, 1},   {0x5401, 8, 14, 0},  {0x4801, 9, 14, 0},  {0x3801, 10, 14, 0},
        {0x3001, 11, 17, 0}, {0x2401, 12, 18, 0}, {0x1C01, 13, 20, 0}, {0x1601, 29, 21, 0}, {0x5601, 15, 14, 1},
        {0x5401, 16, 14, 0}, {0x5101, 17, 15, 0}, {0x4801, 18, 16, 0}, {0x3801, 19, 17, 0}, {0x3401, 20, 18, 0},
        {0x3001, 21, 19, 0}, {0x2801, 22, 19, 0}, {0x2401, 23, 20, 0}, {0x2201, 24, 21, 0}, {0x1C01, 25, 22, 0},
        {0x1801, 26, 23, 0}, {0x1601, 27, 24, 0}, {0x1401, 28, 25, 0}, {0x1201, 29, 26, 0}, {0x1101, 30, 27, 0},
        {0x0AC1, 31, 28, 0}, {0x09C1, 32, 29, 0}, {0x08A1, 33, 30, 0}, {0x0521, 34, 31, 0}, {0x0441, 35, 32, 0},
        {0x02A1, 36, 33, 0}, {0x0221, 37, 34, 0}, {0x0141, 38, 35, 0}, {0x0111, 39, 36, 0}, {0x0085, 40, 37, 0},
        {0x0049, 41, 38, 0}, {0x0025, 42, 39, 0}, {0x0015, 43, 40, 0}, {0x0009, 44, 41, 0}, {0x0005, 45, 42, 0},
        {0x0001, 45, 43, 0}, {0x5601, 46, 46, 0},
    };
    return t;
}

// zc: 4 x 45 bytes indexed by orient * 45 + h + 3 v + 9 d; sc: 9 bytes indexed by
// (hc + 1) * 3 + (vc + 1), context | xor << 5; mq: 47 words Qe | switch << 17 |
// NMPS << 18 | NLPS << 24 (bit 16 is left for the context's MPS).
inline void t1BuildTables(uint8_t* zc, uint8_t* sc, uint32_t* mq) {
    for (int o = 0; o < 4; ++o)
        for (int d = 0; d <= 4; ++d)
            for (int v = 0; v <= 2; ++v)
                for (int h = 0; h <= 2; ++h) zc[o * 45 + h + 3 * v + 9 * d] = (uint8_t)zcContext(h, v, d, o);
    for (int hc = -1; hc <= 1; ++hc)
        for (int vc = -1; vc <= 1; ++vc) {
            int cx, x;
            scContext(hc, vc, cx, x);
            sc[(hc + 1) * 3 + (vc + 1)] = (uint8_t)(cx | (x << 5));
        }
    const MqState* s = mqStates();
    for (int i = 0; i < 47; ++i)
        mq[i] = (uint32_t)s[i].qe | ((uint32_t)s[i].sw << 17) | ((uint32_t)s[i].nmps << 18) | ((uint32_t)s[i].nlps << 24);
}

}  // namespace gb
