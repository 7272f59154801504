// rt_jpeg.cpp - baseline JPEG textures without an image library.
//
// The reference loads textures with stb_image (core/src/Scene.cpp:181-189),
// which reads JPEG files.  This decoder follows ITU-T T.81 for the baseline
// sequential process (SOF0/SOF1, 8-bit samples, Huffman coding): canonical
// Huffman tables (DHT), quantisation tables (DQT), interleaved or single-
// component scans with restart intervals, a separable floating-point inverse
// DCT, chroma upsampling by linear interpolation between sample centres (for
// 2x factors the 3/4 - 1/4 "triangle" filter), and the JFIF YCbCr to RGB
// transform.  Progressive and arithmetic-coded files are rejected.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "rt_image.h"

namespace rti {
namespace {

constexpr double kPi = 3.14159265358979323846;

const uint8_t kZigzag[64] = {0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33, 40, 48,
                             41, 34, 27, 20, 13, 6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23,
                             30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

struct HuffTable {
    bool present = false;
    uint8_t count[17] = {0};  // codes of each length 1..16
    uint8_t symbol[256] = {0};
    int first_code[17] = {0}, first_index[17] = {0};
    void prepare() {
        int code = 0, index = 0;
        for (int len = 1; len <= 16; len++) {
            first_code[len] = code;
            first_index[len] = index;
            code = (code + count[len]) << 1;
            index += count[len];
        }
    }
};

struct Component {
    int id, h, v, tq;
    int td = 0, ta = 0;  // DC / AC table of the scan
    int pred = 0;        // DC predictor
    int bw = 0, bh = 0;  // blocks across / down, padded to whole MCUs
    std::vector<uint8_t> pixels;
};

struct Reader {
    const uint8_t* p;
    size_t n, pos = 0;
    uint32_t buf = 0;
    int cnt = 0;
    bool marker_hit = false;  // a marker ended the entropy-coded data
    int bit() {
        if (cnt == 0) {
            uint8_t b = 0;
            if (!marker_hit && pos < n) {
                b = p[pos];
                if (b == 0xFF) {
                    const uint8_t nx = pos + 1 < n ? p[pos + 1] : 0;
                    if (nx == 0x00) {
                        pos += 2;  // stuffed byte
                    } else {
                        marker_hit = true;  // feed zeros until the decoder resynchronises
                        b = 0;
                    }
                } else {
                    pos++;
                }
            }
            buf = b;
            cnt = 8;
        }
        cnt--;
        return int((buf >> cnt) & 1u);
    }
    int bits(int k) {
        int v = 0;
        for (int i = 0; i < k; i++) v = (v << 1) | bit();
        return v;
    }
    void reset_bits() { cnt = 0; }
};

int decode_huff(Reader& r, const HuffTable& t) {
    int code = 0;
    for (int len = 1; len <= 16; len++) {
        code = (code << 1) | r.bit();
        const int k = code - t.first_code[len];
        if (k >= 0 && k < t.count[len]) return t.symbol[t.first_index[len] + k];
    }
    return -1;
}

// the magnitude category `s` and its bits -> signed value (T.81 F.2.2.1)
int extend(int v, int s) { return (s > 0 && v < (1 << (s - 1))) ? v - (1 << s) + 1 : v; }

void idct8x8(const float in[64], uint8_t* out, int stride) {
    static float cosines[8][8];
    static bool ready = false;
    if (!ready) {
        for (int x = 0; x < 8; x++)
            for (int u = 0; u < 8; u++)
                cosines[x][u] = float((u == 0 ? std::sqrt(0.5) : 1.0) * std::cos((2 * x + 1) * u * kPi / 16.0));
        ready = true;
    }
    float tmp[64];
    for (int y = 0; y < 8; y++)  // rows of coefficients v -> columns
        for (int u = 0; u < 8; u++) {
            float s = 0.f;
            for (int v = 0; v < 8; v++) s += cosines[y][v] * in[v * 8 + u];
            tmp[y * 8 + u] = s;
        }
    for (int y = 0; y < 8; y++)
        for (int x = 0; x < 8; x++) {
            float s = 0.f;
            for (int u = 0; u < 8; u++) s += cosines[x][u] * tmp[y * 8 + u];
            const float v = s * 0.25f + 128.0f;
            out[y * stride + x] = uint8_t(v < 0.f ? 0 : (v > 255.f ? 255 : int(v + 0.5f)));
        }
}

uint16_t be16(const uint8_t* p) { return uint16_t((p[0] << 8) | p[1]); }

}  // namespace

bool read_jpeg(const std::string& file, std::vector<uint8_t>& rgba, int& w, int& h, std::string& err) {
    const uint8_t* p = reinterpret_cast<const uint8_t*>(file.data());
    const size_t n = file.size();
    if (n < 4 || p[0] != 0xFF || p[1] != 0xD8) {
        err = "not a JPEG file";
        return false;
    }
    float qt[4][64];
    bool have_qt[4] = {false, false, false, false};
    HuffTable dc[4], ac[4];
    std::vector<Component> comps;
    int hmax = 1, vmax = 1, restart = 0;
    bool have_frame = false, done = false;
    size_t pos = 2;
    while (pos + 4 <= n && !done) {
        if (p[pos] != 0xFF) {
            err = "marker expected";
            return false;
        }
        const uint8_t m = p[pos + 1];
        if (m == 0xFF) {  // fill byte
            pos++;
            continue;
        }
        if (m == 0xD9) break;  // EOI
        const size_t len = be16(p + pos + 2);
        if (len < 2 || pos + 2 + len > n) {
            err = "truncated segment";
            return false;
        }
        const uint8_t* s = p + pos + 4;
        const size_t sl = len - 2;
        if (m == 0xDB) {  // DQT
            size_t o = 0;
            while (o < sl) {
                const int pq = s[o] >> 4, tq = s[o] & 15;
                if (tq > 3 || o + 1 + 64 * (pq + 1) > sl) {
                    err = "bad DQT";
                    return false;
                }
                for (int k = 0; k < 64; k++)
                    qt[tq][kZigzag[k]] = pq ? float(be16(s + o + 1 + 2 * k)) : float(s[o + 1 + k]);
                have_qt[tq] = true;
                o += 1 + size_t(64) * (pq + 1);
            }
        } else if (m == 0xC4) {  // DHT
            size_t o = 0;
            while (o < sl) {
                if (o + 17 > sl) {
                    err = "bad DHT";
                    return false;
                }
                const int tc = s[o] >> 4, th = s[o] & 15;
                if (tc > 1 || th > 3) {
                    err = "bad DHT";
                    return false;
                }
                HuffTable& t = tc ? ac[th] : dc[th];
                int total = 0;
                for (int l = 1; l <= 16; l++) total += (t.count[l] = s[o + l]);
                if (total > 256 || o + 17 + size_t(total) > sl) {
                    err = "bad DHT";
                    return false;
                }
                std::memcpy(t.symbol, s + o + 17, size_t(total));
                t.prepare();
                t.present = true;
                o += 17 + size_t(total);
            }
        } else if (m == 0xDD) {  // DRI
            restart = be16(s);
        } else if (m == 0xC0 || m == 0xC1) {  // baseline / extended sequential, Huffman
            if (sl < 6 || s[0] != 8) {
                err = "only 8-bit JPEG is supported";
                return false;
            }
            h = be16(s + 1);
            w = be16(s + 3);
            const int nc = s[5];
            if (w <= 0 || h <= 0 || int64_t(w) * h > (int64_t(1) << 28) || (nc != 1 && nc != 3) ||
                sl < size_t(6 + 3 * nc)) {
                err = "bad frame header";
                return false;
            }
            for (int c = 0; c < nc; c++) {
                Component k;
                k.id = s[6 + 3 * c];
                k.h = s[7 + 3 * c] >> 4;
                k.v = s[7 + 3 * c] & 15;
                k.tq = s[8 + 3 * c];
                if (k.h < 1 || k.h > 4 || k.v < 1 || k.v > 4 || k.tq > 3) {
                    err = "bad component";
                    return false;
                }
                hmax = std::max(hmax, k.h);
                vmax = std::max(vmax, k.v);
                comps.push_back(k);
            }
            have_frame = true;
        } else if ((m >= 0xC2 && m <= 0xC3) || (m >= 0xC5 && m <= 0xCF && m != 0xC8 && m != 0xCC)) {
            err = "progressive, lossless or arithmetic-coded JPEG is not supported";
            return false;
        } else if (m == 0xDA) {  // SOS: one scan holding all components
            if (!have_frame) {
                err = "scan before frame header";
                return false;
            }
            const int ns = s[0];
            if (ns != int(comps.size())) {
                err = "non-interleaved multi-scan JPEG is not supported";
                return false;
            }
            for (int i = 0; i < ns; i++) {
                const int id = s[1 + 2 * i], t = s[2 + 2 * i];
                bool found = false;
                for (Component& k : comps)
                    if (k.id == id) {
                        k.td = t >> 4;
                        k.ta = t & 15;
                        found = true;
                    }
                if (!found) {
                    err = "scan names an unknown component";
                    return false;
                }
            }
            for (const Component& k : comps)
                if (k.td > 3 || k.ta > 3 || !dc[k.td].present || !ac[k.ta].present || !have_qt[k.tq]) {
                    err = "missing Huffman or quantisation table";
                    return false;
                }
            // decode the entropy-coded data that follows
            const int mcux = (w + 8 * hmax - 1) / (8 * hmax), mcuy = (h + 8 * vmax - 1) / (8 * vmax);
            const bool single = comps.size() == 1;
            for (Component& k : comps) {
                k.bw = single ? (w + 7) / 8 : mcux * k.h;
                k.bh = single ? (h + 7) / 8 : mcuy * k.v;
                k.pixels.assign(size_t(k.bw) * 8 * size_t(k.bh) * 8, 0);
                k.pred = 0;
            }
            Reader r{p, n, pos + 2 + len};
            const int units = single ? comps[0].bw * comps[0].bh : mcux * mcuy;
            float coef[64];
            for (int u = 0; u < units; u++) {
                if (restart && u > 0 && u % restart == 0) {  // RSTn: byte-align, skip the marker, reset predictors
                    r.reset_bits();
                    r.marker_hit = false;
                    while (r.pos + 1 < n && !(p[r.pos] == 0xFF && p[r.pos + 1] >= 0xD0 && p[r.pos + 1] <= 0xD7)) r.pos++;
                    r.pos += 2;
                    for (Component& k : comps) k.pred = 0;
                }
                for (Component& k : comps) {
                    const int nby = single ? 1 : k.v, nbx = single ? 1 : k.h;
                    for (int by = 0; by < nby; by++)
                        for (int bx = 0; bx < nbx; bx++) {
                            std::memset(coef, 0, sizeof(coef));
                            const int t = decode_huff(r, dc[k.td]);
                            if (t < 0 || t > 11) {
                                err = "bad DC code";
                                return false;
                            }
                            k.pred += extend(r.bits(t), t);
                            coef[0] = float(k.pred) * qt[k.tq][0];
                            for (int i = 1; i < 64;) {
                                const int rs = decode_huff(r, ac[k.ta]);
                                if (rs < 0) {
                                    err = "bad AC code";
                                    return false;
                                }
                                const int run = rs >> 4, sz = rs & 15;
                                if (sz == 0) {
                                    if (run != 15) break;  // end of block
                                    i += 16;
                                    continue;
                                }
                                i += run;
                                if (i > 63) {
                                    err = "AC coefficients past the block";
                                    return false;
                                }
                                const int zz = kZigzag[i];
                                coef[zz] = float(extend(r.bits(sz), sz)) * qt[k.tq][zz];
                                i++;
                            }
                            const int bxx = single ? u % k.bw : (u % mcux) * k.h + bx;
                            const int byy = single ? u / k.bw : (u / mcux) * k.v + by;
                            const int stride = k.bw * 8;
                            idct8x8(coef, k.pixels.data() + size_t(byy) * 8 * size_t(stride) + size_t(bxx) * 8, stride);
                        }
                }
            }
            done = true;
            break;
        }
        pos += 2 + len;
    }
    if (!done) {
        err = "no image data";
        return false;
    }
    // colour conversion and upsampling; output row 0 = bottom (stbi's flip)
    rgba.assign(size_t(w) * size_t(h) * 4, 255);
    const bool single = comps.size() == 1;
    auto sample = [&](const Component& k, int x, int y) -> float {
        if (single || (k.h == hmax && k.v == vmax)) return float(k.pixels[size_t(y) * size_t(k.bw) * 8 + size_t(x)]);
        // centre of output pixel x in the component's sample grid, clamped to its valid samples
        const int cw = (w * k.h + hmax - 1) / hmax, ch = (h * k.v + vmax - 1) / vmax;
        const float fx = (float(x) + 0.5f) * float(k.h) / float(hmax) - 0.5f;
        const float fy = (float(y) + 0.5f) * float(k.v) / float(vmax) - 0.5f;
        const int x0 = int(std::floor(fx)), y0 = int(std::floor(fy));
        const float ax = fx - float(x0), ay = fy - float(y0);
        auto at = [&](int xx, int yy) {
            xx = std::min(std::max(xx, 0), cw - 1);
            yy = std::min(std::max(yy, 0), ch - 1);
            return float(k.pixels[size_t(yy) * size_t(k.bw) * 8 + size_t(xx)]);
        };
        return (1.f - ay) * ((1.f - ax) * at(x0, y0) + ax * at(x0 + 1, y0)) +
               ay * ((1.f - ax) * at(x0, y0 + 1) + ax * at(x0 + 1, y0 + 1));
    };
    for (int y = 0; y < h; y++) {
        uint8_t* dst = rgba.data() + size_t(h - 1 - y) * size_t(w) * 4;
        for (int x = 0; x < w; x++) {
            float c[3];
            for (size_t ci = 0; ci < comps.size(); ci++) c[ci] = sample(comps[ci], x, y);
            uint8_t* o = dst + size_t(x) * 4;
            if (single) {
                o[0] = o[1] = o[2] = uint8_t(c[0]);
            } else {  // JFIF YCbCr -> RGB
                const float Y = c[0], cb = c[1] - 128.f, cr = c[2] - 128.f;
                const float rgb[3] = {Y + 1.402f * cr, Y - 0.344136f * cb - 0.714136f * cr, Y + 1.772f * cb};
                for (int k = 0; k < 3; k++) o[k] = uint8_t(rgb[k] < 0.f ? 0 : (rgb[k] > 255.f ? 255 : int(rgb[k] + 0.5f)));
            }
        }
    }
    return true;
}

}  // namespace rti
