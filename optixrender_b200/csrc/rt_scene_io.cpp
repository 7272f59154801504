// rt_scene_io.cpp - on-disk scene formats: the JSON scene description of the
// reference (models/test.json; SceneParser, core/src/SceneParser.cpp:3-46),
// Wavefront OBJ meshes (TriangleMesh::LoadMesh, core/src/Scene.cpp:83-179) and
// Radiance RGBE environment images (HdrTexture, core/src/Scene.cpp:197-206).
#include <cmath>
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "rt_image.h"
#include "rt_internal.h"

using namespace rti;

namespace {

// ------------------------------------------------------------------ JSON
struct Json {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    bool b = false;
    double n = 0.0;
    std::string s;
    std::vector<Json> a;
    std::vector<std::pair<std::string, Json>> o;
    const Json* get(const char* key) const {
        if (kind != Obj) return nullptr;
        for (auto& kv : o)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
};

struct JsonParser {
    const char* p;
    const char* end;
    std::string err;
    void ws() {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) p++;
    }
    bool fail(const char* m) {
        if (err.empty()) err = m;
        return false;
    }
    bool value(Json& v, int depth) {
        if (depth > 64) return fail("nesting too deep");
        ws();
        if (p >= end) return fail("unexpected end of input");
        char c = *p;
        if (c == '{') {
            v.kind = Json::Obj;
            p++;
            ws();
            if (p < end && *p == '}') {
                p++;
                return true;
            }
            while (true) {
                ws();
                Json k;
                if (p >= end || *p != '"' || !string(k.s)) return fail("expected object key");
                ws();
                if (p >= end || *p != ':') return fail("expected ':'");
                p++;
                Json val;
                if (!value(val, depth + 1)) return false;
                v.o.emplace_back(k.s, std::move(val));
                ws();
                if (p < end && *p == ',') {
                    p++;
                    continue;
                }
                if (p < end && *p == '}') {
                    p++;
                    return true;
                }
                return fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = Json::Arr;
            p++;
            ws();
            if (p < end && *p == ']') {
                p++;
                return true;
            }
            while (true) {
                Json val;
                if (!value(val, depth + 1)) return false;
                v.a.push_back(std::move(val));
                ws();
                if (p < end && *p == ',') {
                    p++;
                    continue;
                }
                if (p < end && *p == ']') {
                    p++;
                    return true;
                }
                return fail("expected ',' or ']'");
            }
        }
        if (c == '"') {
            v.kind = Json::Str;
            return string(v.s);
        }
        if (c == 't' && end - p >= 4 && !std::strncmp(p, "true", 4)) {
            v.kind = Json::Bool;
            v.b = true;
            p += 4;
            return true;
        }
        if (c == 'f' && end - p >= 5 && !std::strncmp(p, "false", 5)) {
            v.kind = Json::Bool;
            v.b = false;
            p += 5;
            return true;
        }
        if (c == 'n' && end - p >= 4 && !std::strncmp(p, "null", 4)) {
            v.kind = Json::Null;
            p += 4;
            return true;
        }
        if (c == '-' || (c >= '0' && c <= '9')) {
            char* e = nullptr;
            std::string tmp(p, size_t(std::min<ptrdiff_t>(end - p, 64)));
            v.n = std::strtod(tmp.c_str(), &e);
            if (e == tmp.c_str()) return fail("bad number");
            p += (e - tmp.c_str());
            v.kind = Json::Num;
            return true;
        }
        return fail("unexpected character");
    }
    bool string(std::string& out) {
        p++;  // opening quote
        while (p < end && *p != '"') {
            if (*p == '\\') {
                p++;
                if (p >= end) return fail("bad escape");
                char e = *p++;
                switch (e) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'r': out += '\r'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'u': {
                        if (end - p < 4) return fail("bad unicode escape");
                        unsigned cp = unsigned(std::strtoul(std::string(p, 4).c_str(), nullptr, 16));
                        p += 4;
                        if (cp < 0x80) {
                            out += char(cp);
                        } else if (cp < 0x800) {
                            out += char(0xC0 | (cp >> 6));
                            out += char(0x80 | (cp & 0x3F));
                        } else {
                            out += char(0xE0 | (cp >> 12));
                            out += char(0x80 | ((cp >> 6) & 0x3F));
                            out += char(0x80 | (cp & 0x3F));
                        }
                        break;
                    }
                    default: out += e;
                }
            } else {
                out += *p++;
            }
        }
        if (p >= end) return fail("unterminated string");
        p++;
        return true;
    }
};

bool read_file(const std::string& path, std::string& out) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    std::stringstream ss;
    ss << f.rdbuf();
    out = ss.str();
    return true;
}

std::string join_path(const std::string& base, const std::string& rel) {
    if (rel.empty() || rel[0] == '/' || base.empty()) return rel;
    return base + "/" + rel;
}

std::string dir_of(const std::string& path) {
    size_t k = path.find_last_of('/');
    return k == std::string::npos ? std::string(".") : path.substr(0, k);
}

double num(const Json* j, double def) { return (j && j->kind == Json::Num) ? j->n : def; }
std::string str(const Json* j, const char* def) { return (j && j->kind == Json::Str) ? j->s : std::string(def); }
bool vec3(const Json* j, float out[3]) {
    if (!j) return false;
    if (j->kind == Json::Num) {
        out[0] = out[1] = out[2] = float(j->n);
        return true;
    }
    if (j->kind != Json::Arr || j->a.size() < 3) return false;
    for (int k = 0; k < 3; k++) out[k] = float(num(&j->a[size_t(k)], 0.0));
    return true;
}

void warn_unknown(const Json& obj, std::initializer_list<const char*> known, const char* where) {
    if (obj.kind != Json::Obj) return;
    for (auto& kv : obj.o) {
        bool ok = false;
        for (const char* k : known) ok = ok || kv.first == k;
        if (!ok) std::fprintf(stderr, "[optixrender_b200] scene JSON: ignoring unknown key '%s' in %s\n", kv.first.c_str(), where);
    }
}

// ------------------------------------------------------------------ OBJ
struct ObjData {
    std::vector<float> v, vt, vn;
    std::vector<float> pos, nrm, uv;  // de-indexed, 3 vertices per triangle
    std::vector<char> has_n, has_t;   // per triangle
};

bool parse_obj(const std::string& text, ObjData& d, std::string& err) {
    std::istringstream in(text);
    std::string line;
    int lineno = 0;
    while (std::getline(in, line)) {
        lineno++;
        const char* s = line.c_str();
        while (*s == ' ' || *s == '\t') s++;
        if (s[0] == 'v' && (s[1] == ' ' || s[1] == '\t')) {
            float x = 0, y = 0, z = 0;
            std::sscanf(s + 2, "%f %f %f", &x, &y, &z);
            d.v.insert(d.v.end(), {x, y, z});
        } else if (s[0] == 'v' && s[1] == 't') {
            float x = 0, y = 0;
            std::sscanf(s + 2, "%f %f", &x, &y);
            d.vt.insert(d.vt.end(), {x, y});
        } else if (s[0] == 'v' && s[1] == 'n') {
            float x = 0, y = 0, z = 0;
            std::sscanf(s + 2, "%f %f %f", &x, &y, &z);
            d.vn.insert(d.vn.end(), {x, y, z});
        } else if (s[0] == 'f' && (s[1] == ' ' || s[1] == '\t')) {
            std::istringstream fs(s + 2);
            std::string tok;
            std::vector<int> vi, ti, ni;
            while (fs >> tok) {
                int a = 0, b = 0, c = 0;
                int n = 0;
                const char* t = tok.c_str();
                a = std::atoi(t);
                const char* s1 = std::strchr(t, '/');
                if (s1) {
                    if (s1[1] != '/') b = std::atoi(s1 + 1);
                    const char* s2 = std::strchr(s1 + 1, '/');
                    if (s2) c = std::atoi(s2 + 1);
                }
                (void)n;
                auto fix = [](int i, size_t count) { return i < 0 ? int(count) + i : i - 1; };
                vi.push_back(fix(a, d.v.size() / 3));
                ti.push_back(b ? fix(b, d.vt.size() / 2) : -1);
                ni.push_back(c ? fix(c, d.vn.size() / 3) : -1);
            }
            if (vi.size() < 3) {
                err = "face with fewer than 3 vertices at line " + std::to_string(lineno);
                return false;
            }
            for (size_t k = 1; k + 1 < vi.size(); k++) {  // fan triangulation
                size_t ids[3] = {0, k, k + 1};
                bool hn = true, ht = true;
                for (size_t q : ids) {
                    if (vi[q] < 0 || size_t(vi[q]) * 3 >= d.v.size()) {
                        err = "vertex index out of range at line " + std::to_string(lineno);
                        return false;
                    }
                    hn = hn && ni[q] >= 0 && size_t(ni[q]) * 3 < d.vn.size();
                    ht = ht && ti[q] >= 0 && size_t(ti[q]) * 2 < d.vt.size();
                }
                for (size_t q : ids) {
                    for (int a = 0; a < 3; a++) d.pos.push_back(d.v[size_t(vi[q]) * 3 + a]);
                    for (int a = 0; a < 3; a++) d.nrm.push_back(hn ? d.vn[size_t(ni[q]) * 3 + a] : 0.0f);
                    for (int a = 0; a < 2; a++) d.uv.push_back(ht ? d.vt[size_t(ti[q]) * 2 + a] : 0.0f);
                }
                d.has_n.push_back(hn);
                d.has_t.push_back(ht);
            }
        }
    }
    if (d.pos.empty()) {
        err = "no faces";
        return false;
    }
    return true;
}

// Adds de-indexed OBJ triangles, filling missing normals / texcoords per face
// as Scene.cpp:150-165 does.
rt_status add_obj(rt_scene* s, const std::string& path, const rt_material* mat, int out_m, int in_m, const float* xform,
                  int32_t* out_id) {
    std::string text, err;
    if (!read_file(path, text)) return fail(RT_ERR_IO, "could not read OBJ model from " + path);
    ObjData d;
    if (!parse_obj(text, d, err)) return fail(RT_ERR_PARSE, "could not read OBJ model from " + path + " : " + err);
    size_t nt = d.has_n.size();
    if (xform) {
        for (size_t i = 0; i < d.pos.size() / 3; i++) {
            float* p = &d.pos[i * 3];
            float q[3];
            for (int r = 0; r < 3; r++) q[r] = xform[r * 4] * p[0] + xform[r * 4 + 1] * p[1] + xform[r * 4 + 2] * p[2] + xform[r * 4 + 3];
            p[0] = q[0];
            p[1] = q[1];
            p[2] = q[2];
            float* n = &d.nrm[i * 3];
            for (int r = 0; r < 3; r++) q[r] = xform[r * 4] * n[0] + xform[r * 4 + 1] * n[1] + xform[r * 4 + 2] * n[2];
            n[0] = q[0];
            n[1] = q[1];
            n[2] = q[2];
        }
    }
    bool all_n = true, all_t = true;
    for (size_t t = 0; t < nt; t++) {
        all_n = all_n && d.has_n[t];
        all_t = all_t && d.has_t[t];
    }
    if (!all_n) {
        for (size_t t = 0; t < nt; t++) {
            if (d.has_n[t]) continue;
            rtd::v3 v0 = rtd::ld3(&d.pos[t * 9]), v1 = rtd::ld3(&d.pos[t * 9 + 3]), v2 = rtd::ld3(&d.pos[t * 9 + 6]);
            rtd::v3 n = rtd::normalize(rtd::cross(rtd::normalize(v1 - v0), rtd::normalize(v2 - v0)));
            for (int k = 0; k < 3; k++) {
                d.nrm[t * 9 + k * 3 + 0] = n.x;
                d.nrm[t * 9 + k * 3 + 1] = n.y;
                d.nrm[t * 9 + k * 3 + 2] = n.z;
            }
        }
    }
    if (!all_t) {
        const float def[6] = {0.f, 0.f, 1.f, 0.f, 0.f, 1.f};
        for (size_t t = 0; t < nt; t++)
            if (!d.has_t[t])
                for (int k = 0; k < 6; k++) d.uv[t * 6 + k] = def[k];
    }
    rt_mesh_desc m;
    std::memset(&m, 0, sizeof(m));
    m.positions = d.pos.data();
    m.normals = d.nrm.data();
    m.texcoords = d.uv.data();
    m.num_vertices = int64_t(nt * 3);
    m.num_triangles = int64_t(nt);
    return rt_scene_add_mesh(s, &m, mat, out_m, in_m, out_id);
}

// ------------------------------------------------------------------ LDR images
// Texture files for Scene::AddTexture (core/src/Scene.cpp:66-69, 181-189:
// stbi_load forced to RGBA with a vertical flip, so row 0 is the bottom of
// the picture).  Read here without an image library: PNG (rt_png.cpp),
// baseline JPEG (rt_jpeg.cpp),
// uncompressed BMP (8-bit palette, 24-bit, 32-bit) and binary PGM/PPM (P5/P6,
// maxval <= 255).
uint32_t rd32(const std::string& d, size_t o) {
    return uint32_t(uint8_t(d[o])) | (uint32_t(uint8_t(d[o + 1])) << 8) | (uint32_t(uint8_t(d[o + 2])) << 16) |
           (uint32_t(uint8_t(d[o + 3])) << 24);
}
uint32_t rd16(const std::string& d, size_t o) { return uint32_t(uint8_t(d[o])) | (uint32_t(uint8_t(d[o + 1])) << 8); }

bool read_bmp(const std::string& d, std::vector<uint8_t>& rgba, int& w, int& h, std::string& err) {
    if (d.size() < 54) {
        err = "truncated BMP header";
        return false;
    }
    const uint32_t off = rd32(d, 10), hdr = rd32(d, 14);
    const int32_t bw = int32_t(rd32(d, 18)), bh = int32_t(rd32(d, 22));
    const uint32_t bpp = rd16(d, 28), comp = rd32(d, 30);
    if (hdr < 40 || bw <= 0 || bh == 0 || (bpp != 8 && bpp != 24 && bpp != 32) ||
        !(comp == 0 || (comp == 3 && bpp == 32))) {
        err = "unsupported BMP (only uncompressed 8/24/32-bit)";
        return false;
    }
    w = bw;
    h = bh < 0 ? -bh : bh;
    const size_t stride = (size_t(w) * bpp / 8 + 3) & ~size_t(3);
    if (size_t(off) + stride * size_t(h) > d.size()) {
        err = "truncated BMP pixel data";
        return false;
    }
    uint32_t masks[4] = {0x00FF0000u, 0x0000FF00u, 0x000000FFu, 0xFF000000u};
    if (comp == 3 && d.size() >= 14 + 52) {
        for (int c = 0; c < 3; c++) masks[c] = rd32(d, 54 + 4 * size_t(c));
        masks[3] = hdr >= 56 ? rd32(d, 66) : 0u;
    }
    const size_t ncol = bpp == 8 ? (rd32(d, 46) ? rd32(d, 46) : 256u) : 0u;
    if (bpp == 8 && 14 + hdr + ncol * 4 > d.size()) {
        err = "truncated BMP palette";
        return false;
    }
    auto channel = [](uint32_t px, uint32_t mask) -> uint8_t {
        if (!mask) return 255;
        int shift = __builtin_ctz(mask);
        uint32_t v = (px & mask) >> shift, mx = mask >> shift;
        return uint8_t((v * 255u + mx / 2) / mx);
    };
    rgba.assign(size_t(w) * h * 4, 0);
    bool any_alpha = false;
    for (int y = 0; y < h; y++) {
        // stored bottom-up when the height is positive: file row y is picture row y from the bottom
        const int out_row = bh > 0 ? y : h - 1 - y;
        const size_t row = size_t(off) + stride * size_t(y);
        for (int x = 0; x < w; x++) {
            uint8_t* o = &rgba[(size_t(out_row) * w + x) * 4];
            if (bpp == 8) {
                size_t idx = uint8_t(d[row + size_t(x)]);
                if (idx >= ncol) idx = 0;
                size_t pe = 14 + hdr + idx * 4;
                o[0] = uint8_t(d[pe + 2]), o[1] = uint8_t(d[pe + 1]), o[2] = uint8_t(d[pe]), o[3] = 255;
            } else if (bpp == 24) {
                size_t q = row + size_t(x) * 3;
                o[0] = uint8_t(d[q + 2]), o[1] = uint8_t(d[q + 1]), o[2] = uint8_t(d[q]), o[3] = 255;
            } else {
                uint32_t px = rd32(d, row + size_t(x) * 4);
                for (int c = 0; c < 3; c++) o[c] = channel(px, masks[c]);
                o[3] = masks[3] ? channel(px, masks[3]) : 255;
                any_alpha = any_alpha || o[3] != 0;
            }
        }
    }
    if (bpp == 32 && masks[3] && !any_alpha)  // an all-zero alpha channel is taken as opaque
        for (size_t i = 3; i < rgba.size(); i += 4) rgba[i] = 255;
    return true;
}

bool read_pnm(const std::string& d, std::vector<uint8_t>& rgba, int& w, int& h, std::string& err) {
    size_t pos = 2;
    auto token = [&]() -> long {
        while (pos < d.size()) {
            if (d[pos] == '#') {
                while (pos < d.size() && d[pos] != '\n') pos++;
            } else if (std::isspace(uint8_t(d[pos]))) {
                pos++;
            } else {
                break;
            }
        }
        long v = -1;
        while (pos < d.size() && std::isdigit(uint8_t(d[pos]))) v = (v < 0 ? 0 : v * 10) + (d[pos++] - '0');
        return v;
    };
    const bool color = d[1] == '6';
    long lw = token(), lh = token(), mx = token();
    if (lw <= 0 || lh <= 0 || mx <= 0 || mx > 255) {
        err = "unsupported PNM header (binary P5/P6 with maxval <= 255)";
        return false;
    }
    pos++;  // the single whitespace after maxval
    w = int(lw);
    h = int(lh);
    const size_t ch = color ? 3 : 1;
    if (pos + size_t(w) * h * ch > d.size()) {
        err = "truncated PNM pixel data";
        return false;
    }
    rgba.assign(size_t(w) * h * 4, 255);
    for (int y = 0; y < h; y++) {
        const int out_row = h - 1 - y;  // stored top-down
        for (int x = 0; x < w; x++) {
            const size_t q = pos + (size_t(y) * w + x) * ch;
            uint8_t* o = &rgba[(size_t(out_row) * w + x) * 4];
            for (int c = 0; c < 3; c++) {
                unsigned v = uint8_t(d[q + (color ? size_t(c) : 0)]);
                o[c] = uint8_t((v * 255u + unsigned(mx) / 2) / unsigned(mx));
            }
        }
    }
    return true;
}

bool read_image(const std::string& path, std::vector<uint8_t>& rgba, int& w, int& h, std::string& err) {
    std::string d;
    if (!read_file(path, d)) {
        err = "could not read " + path;
        return false;
    }
    bool ok;
    if (d.size() >= 2 && d[0] == 'B' && d[1] == 'M')
        ok = read_bmp(d, rgba, w, h, err);
    else if (d.size() >= 2 && d[0] == 'P' && (d[1] == '5' || d[1] == '6'))
        ok = read_pnm(d, rgba, w, h, err);
    else if (d.size() >= 8 && uint8_t(d[0]) == 137 && d[1] == 'P' && d[2] == 'N' && d[3] == 'G')
        ok = read_png(d, rgba, w, h, err);
    else if (d.size() >= 3 && uint8_t(d[0]) == 0xFF && uint8_t(d[1]) == 0xD8 && uint8_t(d[2]) == 0xFF)
        ok = read_jpeg(d, rgba, w, h, err);
    else {
        err = "unsupported image format (PNG, JPEG, BMP or binary PGM/PPM)";
        ok = false;
    }
    if (!ok) err = path + ": " + err;
    return ok;
}

// ------------------------------------------------------------------ RGBE
bool read_hdr(const std::string& path, std::vector<float>& rgba, int& w, int& h, std::string& err) {
    std::string data;
    if (!read_file(path, data)) {
        err = "could not read " + path;
        return false;
    }
    size_t pos = 0;
    auto line = [&]() {
        size_t e = data.find('\n', pos);
        if (e == std::string::npos) e = data.size();
        std::string l = data.substr(pos, e - pos);
        pos = e + 1;
        return l;
    };
    std::string first = line();
    if (first.rfind("#?", 0) != 0) {
        err = "not a Radiance HDR file";
        return false;
    }
    while (pos < data.size()) {
        std::string l = line();
        if (l.empty()) break;
        if (l.rfind("FORMAT=", 0) == 0 && l != "FORMAT=32-bit_rle_rgbe") {
            err = "unsupported HDR format " + l;
            return false;
        }
    }
    std::string res = line();
    char ya[3] = {0}, xa[3] = {0};
    if (std::sscanf(res.c_str(), "%2s %d %2s %d", ya, &h, xa, &w) != 4 || w <= 0 || h <= 0) {
        err = "bad HDR resolution line";
        return false;
    }
    bool flip_y = std::string(ya) == "-Y";  // top-to-bottom scanlines
    const unsigned char* p = reinterpret_cast<const unsigned char*>(data.data()) + pos;
    const unsigned char* end = reinterpret_cast<const unsigned char*>(data.data()) + data.size();
    std::vector<unsigned char> scan(size_t(w) * 4);
    rgba.assign(size_t(w) * h * 4, 0.0f);
    for (int y = 0; y < h; y++) {
        if (end - p >= 4 && p[0] == 2 && p[1] == 2 && ((p[2] << 8) | p[3]) == w && w >= 8 && w < 32768) {
            p += 4;
            for (int c = 0; c < 4; c++) {
                int x = 0;
                while (x < w) {
                    if (p >= end) {
                        err = "truncated HDR data";
                        return false;
                    }
                    int n = *p++;
                    if (n > 128) {
                        n -= 128;
                        if (p >= end || x + n > w) {
                            err = "bad HDR run";
                            return false;
                        }
                        unsigned char v = *p++;
                        for (int k = 0; k < n; k++) scan[size_t(x++) * 4 + c] = v;
                    } else {
                        if (n == 0 || end - p < n || x + n > w) {
                            err = "bad HDR literal";
                            return false;
                        }
                        for (int k = 0; k < n; k++) scan[size_t(x++) * 4 + c] = *p++;
                    }
                }
            }
        } else {
            if (end - p < ptrdiff_t(w) * 4) {
                err = "truncated HDR data";
                return false;
            }
            std::memcpy(scan.data(), p, size_t(w) * 4);
            p += size_t(w) * 4;
        }
        // stbi_set_flip_vertically_on_load(true) (Scene.cpp:198): row 0 = bottom
        int row = flip_y ? (h - 1 - y) : y;
        for (int x = 0; x < w; x++) {
            const unsigned char* q = &scan[size_t(x) * 4];
            float f = q[3] ? std::ldexp(1.0f, int(q[3]) - 136) : 0.0f;
            float* o = &rgba[(size_t(row) * w + x) * 4];
            o[0] = q[0] * f;
            o[1] = q[1] * f;
            o[2] = q[2] * f;
            o[3] = 1.0f;
        }
    }
    return true;
}

// ------------------------------------------------------------------ scene JSON
void rotation_matrix(const float deg[3], float m[9]) {
    float rx = deg[0] * 3.14159265358979f / 180.f, ry = deg[1] * 3.14159265358979f / 180.f,
          rz = deg[2] * 3.14159265358979f / 180.f;
    float cx = std::cos(rx), sx = std::sin(rx), cy = std::cos(ry), sy = std::sin(ry), cz = std::cos(rz), sz = std::sin(rz);
    // R = Rz * Ry * Rx
    m[0] = cz * cy;
    m[1] = cz * sy * sx - sz * cx;
    m[2] = cz * sy * cx + sz * sx;
    m[3] = sz * cy;
    m[4] = sz * sy * sx + cz * cx;
    m[5] = sz * sy * cx - cz * sx;
    m[6] = -sy;
    m[7] = cy * sx;
    m[8] = cy * cx;
}

bool material_from_json(const Json& j, rt_material& m, std::string& err, rt_scene* scene, const std::string& base) {
    rt_material_default(&m);
    std::string t = str(j.get("type"), "diffuse");
    float rough_default = m.roughness;
    if (t == "diffuse" || t == "smooth_diffuse" || t == "lambert") {
        m.type = RT_MAT_DIFFUSE;
        rough_default = t == "diffuse" ? 0.1f : 0.0f;
    } else if (t == "conductor" || t == "rough_conductor") {
        m.type = RT_MAT_CONDUCTOR;
    } else if (t == "dielectric" || t == "rough_dielectric") {
        m.type = RT_MAT_DIELECTRIC;
    } else if (t == "smooth_dielectric") {
        m.type = RT_MAT_DIELECTRIC;
        rough_default = 0.02f;  // roughness 0 is 0/0 in the GGX density; 0.02 is the defined minimum
    } else if (t == "plastic" || t == "rough_plastic") {
        m.type = RT_MAT_PLASTIC;
    } else if (t == "metal_workflow") {
        m.type = RT_MAT_METAL_WORKFLOW;
    } else if (t == "thin_dielectric") {
        m.type = RT_MAT_THIN_DIELECTRIC;
    } else if (t == "clearcoated_conductor") {
        m.type = RT_MAT_CLEARCOATED_CONDUCTOR;
    } else if (t == "diffuse_transmitter") {
        m.type = RT_MAT_DIFFUSE_TRANSMITTER;
    } else {
        err = "unknown material type '" + t + "'";
        return false;
    }
    m.roughness = float(num(j.get("roughness"), rough_default));
    vec3(j.get("albedo"), m.albedo);
    m.anisotropy = float(num(j.get("anisotropy"), m.anisotropy));
    vec3(j.get("eta"), m.eta);
    vec3(j.get("k"), m.k);
    m.int_ior = float(num(j.get("int_ior"), m.int_ior));
    m.ext_ior = float(num(j.get("ext_ior"), m.ext_ior));
    if (const Json* nl = j.get("nonlinear")) m.nonlinear = nl->kind == Json::Bool ? nl->b : int(num(nl, 1));
    vec3(j.get("specular"), m.specular);
    m.metallic = float(num(j.get("metallic"), m.metallic));
    m.coat_weight = float(num(j.get("coat_weight"), m.coat_weight));
    m.coat_roughness_u = float(num(j.get("coat_roughness_u"), m.coat_roughness_u));
    m.coat_roughness_v = float(num(j.get("coat_roughness_v"), m.coat_roughness_v));
    // "<name>_texture_type": "image" with "<name>_path" (models/test.json:67-74)
    static const char* kTexNames[8] = {"albedo",   "roughness",        "anisotropy",       "specular",
                                       "metallic", "coat_roughness_u", "coat_roughness_v", "normal"};
    for (int t = 0; t < 8; t++) {
        const std::string name = kTexNames[t];
        if (str(j.get((name + "_texture_type").c_str()), "constant") != "image") continue;
        const std::string path = str(j.get((name + "_path").c_str()), "");
        if (path.empty()) {
            err = name + "_texture_type is image but " + name + "_path is missing";
            return false;
        }
        std::vector<uint8_t> px;
        int w = 0, h = 0;
        if (!read_image(join_path(base, path), px, w, h, err)) return false;
        int32_t id = -1;
        if (rt_scene_add_texture(scene, px.data(), w, h, &id) != RT_OK) {
            err = g_error;
            return false;
        }
        m.texture_ids[t] = id;
    }
    return true;
}

rt_status load_json(rt_scene* s, const std::string& text, const std::string& base, rt_options* opts, rt_camera* cam) {
    JsonParser jp{text.data(), text.data() + text.size(), {}};
    Json root;
    if (!jp.value(root, 0) || root.kind != Json::Obj)
        return fail(RT_ERR_PARSE, "scene JSON: " + (jp.err.empty() ? std::string("top level is not an object") : jp.err));
    warn_unknown(root, {"width", "height", "depth", "spp", "seed", "filter", "camera", "light", "shape", "material",
                        "medium", "tonemap", "integrator"},
                 "the top level");
    if (opts) {
        opts->width = int(num(root.get("width"), 1024));   // SceneParser.cpp:12
        opts->height = int(num(root.get("height"), 1024)); // SceneParser.cpp:13
        opts->max_depth = int(num(root.get("depth"), opts->max_depth));
        opts->spp = int(num(root.get("spp"), opts->spp));
        opts->seed = uint64_t(num(root.get("seed"), double(opts->seed)));
        std::string ft = "gaussian";
        if (const Json* f = root.get("filter")) ft = str(f->get("type"), "gaussian");  // SceneParser.cpp:25-46
        opts->filter = ft == "box" ? RT_FILTER_BOX : ft == "tent" ? RT_FILTER_TENT : ft == "triangle" ? RT_FILTER_TRIANGLE
                                                                                                     : RT_FILTER_GAUSSIAN;
        if (const Json* tm = root.get("tonemap")) {
            std::string t = tm->kind == Json::Str ? tm->s : str(tm->get("type"), "reinhard");
            opts->tonemap = t == "aces" ? RT_TONEMAP_ACES_SRGB : t == "clamp" ? RT_TONEMAP_CLAMP : RT_TONEMAP_REINHARD;
            opts->exposure = float(num(tm->get("exposure"), opts->exposure));
        }
        if (const Json* in = root.get("integrator")) {
            std::string r = str(in->get("rng"), "lcg");
            opts->rng = r == "pcg32" ? RT_RNG_PCG32 : RT_RNG_LCG;
            opts->rr_depth = int(num(in->get("rr_depth"), opts->rr_depth));
            // learned proposal: {"guided": true, "guide_train_spp": 32, "guide_prob": 0.5, "guide_steps": 4}
            if (const Json* gd = in->get("guided")) opts->guided = gd->kind == Json::Bool ? gd->b : int(num(gd, 0)) != 0;
            opts->guide_train_spp = int(num(in->get("guide_train_spp"), opts->guide_train_spp));
            opts->guide_prob = float(num(in->get("guide_prob"), opts->guide_prob));
            opts->guide_steps = int(num(in->get("guide_steps"), opts->guide_steps));
            if (opts->guided) opts->rng = RT_RNG_PCG32;
        }
    }
    // media first, so shapes can refer to them by name
    std::map<std::string, int> medium_ids;
    int32_t nmed0 = int32_t(s->media.size());
    if (const Json* ms = root.get("medium")) {
        for (const Json& mj : ms->a) {
            rt_medium m;
            rt_medium_default(&m);
            std::string t = str(mj.get("type"), "homogeneous");
            std::vector<float> dens;
            if (t == "grid") {
                m.type = RT_MEDIUM_GRID;
                const Json* r = mj.get("resolution");
                float rf[3] = {0, 0, 0};
                if (!vec3(r, rf)) return fail(RT_ERR_PARSE, "grid medium needs 'resolution'");
                for (int a = 0; a < 3; a++) m.grid_res[a] = int(rf[a]);
                std::string dp = join_path(base, str(mj.get("density_path"), ""));
                std::string raw;
                if (!read_file(dp, raw)) return fail(RT_ERR_IO, "could not read density grid " + dp);
                size_t n = size_t(m.grid_res[0]) * m.grid_res[1] * m.grid_res[2];
                if (raw.size() != n * 4) return fail(RT_ERR_PARSE, "density grid size does not match resolution");
                dens.resize(n);
                std::memcpy(dens.data(), raw.data(), n * 4);
                m.density = dens.data();
                vec3(mj.get("bounds_min"), m.bounds_min);
                vec3(mj.get("bounds_max"), m.bounds_max);
                m.majorant_res = int(num(mj.get("majorant_resolution"), 8));
            } else if (t != "homogeneous") {
                return fail(RT_ERR_PARSE, "unknown medium type '" + t + "'");
            }
            std::string ph = str(mj.get("phase"), "isotropic");
            if (ph == "hg" || ph == "henyey_greenstein") {
                m.phase = RT_PHASE_HENYEY_GREENSTEIN;
                vec3(mj.get("g"), m.g);
            }
            vec3(mj.get("sigma_a"), m.sigma_a);
            vec3(mj.get("sigma_s"), m.sigma_s);
            m.scale = float(num(mj.get("scale"), m.scale));
            rt_status st = rt_scene_add_medium(s, &m);
            if (st) return st;
            medium_ids[str(mj.get("name"), "")] = nmed0++;
        }
    }
    std::map<std::string, rt_material> mats;
    if (const Json* ms = root.get("material")) {
        for (const Json& mj : ms->a) {
            rt_material m;
            std::string err;
            if (!material_from_json(mj, m, err, s, base)) return fail(RT_ERR_PARSE, "scene JSON: " + err);
            mats[str(mj.get("name"), "")] = m;
        }
    }
    auto medium_ref = [&](const Json* j) -> int {
        if (!j) return -1;
        if (j->kind == Json::Num) return int(j->n);
        auto it = medium_ids.find(str(j, ""));
        return it == medium_ids.end() ? -2 : it->second;
    };
    if (const Json* shapes = root.get("shape")) {
        for (const Json& sj : shapes->a) {
            std::string mname = str(sj.get("material"), "");
            rt_material m;
            if (mats.count(mname)) {
                m = mats[mname];
            } else {
                rt_material_default(&m);
                if (!mname.empty()) std::fprintf(stderr, "[optixrender_b200] scene JSON: unknown material '%s'\n", mname.c_str());
            }
            int in_m = medium_ref(sj.get("medium_int")), out_m = medium_ref(sj.get("medium_ext"));
            if (in_m == -2 || out_m == -2) return fail(RT_ERR_PARSE, "scene JSON: shape refers to an unknown medium");
            float t[3] = {0, 0, 0}, r[3] = {0, 0, 0}, sc[3] = {1, 1, 1};
            vec3(sj.get("translate"), t);
            vec3(sj.get("rotate"), r);
            vec3(sj.get("scale"), sc);
            float R[9];
            rotation_matrix(r, R);
            float X[12];
            for (int row = 0; row < 3; row++) {
                for (int c = 0; c < 3; c++) X[row * 4 + c] = R[row * 3 + c] * sc[c];
                X[row * 4 + 3] = t[row];
            }
            std::string type = str(sj.get("type"), "mesh");
            if (type != "mesh") return fail(RT_ERR_PARSE, "scene JSON: unknown shape type '" + type + "'");
            rt_status st = add_obj(s, join_path(base, str(sj.get("mesh_path"), "")), &m, out_m, in_m, X, nullptr);
            if (st) return st;
        }
    }
    if (const Json* lights = root.get("light")) {
        for (const Json& lj : lights->a) {
            std::string t = str(lj.get("type"), "");
            if (t == "infinite") {
                std::string path = join_path(base, str(lj.get("hdr_path"), ""));
                std::vector<float> img;
                int w = 0, h = 0;
                std::string err;
                if (!read_hdr(path, img, w, h, err)) return fail(RT_ERR_IO, "environment: " + err);
                rt_status st = rt_scene_set_env(s, img.data(), w, h, float(num(lj.get("scale"), 1.0)));
                if (st) return st;
                continue;
            }
            rt_light l;
            rt_light_default(&l);
            if (t == "quad" || t == "area") {
                l.type = RT_LIGHT_QUAD;
            } else if (t == "sphere") {
                l.type = RT_LIGHT_SPHERE;
            } else if (t == "point") {
                l.type = RT_LIGHT_POINT;
            } else {
                return fail(RT_ERR_PARSE, "scene JSON: unknown light type '" + t + "'");
            }
            vec3(lj.get("radiance"), l.radiance);
            if (!vec3(lj.get("position"), l.position)) vec3(lj.get("corner"), l.position);
            vec3(lj.get("u"), l.u);
            vec3(lj.get("v"), l.v);
            l.radius = float(num(lj.get("radius"), l.radius));
            if (const Json* ds = lj.get("double_side")) l.double_side = ds->kind == Json::Bool ? ds->b : int(num(ds, 0));
            l.medium = medium_ref(lj.get("medium"));
            if (l.medium == -2) return fail(RT_ERR_PARSE, "scene JSON: light refers to an unknown medium");
            rt_status st = rt_scene_add_light(s, &l);
            if (st) return st;
        }
    }
    if (cam) {
        rt_camera_default(cam);
        if (const Json* cj = root.get("camera")) {
            vec3(cj->get("look_from"), cam->from);
            vec3(cj->get("up"), cam->up);
            if (!vec3(cj->get("look_at"), cam->at)) {
                // main.cpp:221: the reference looks at the scene's bounds centre
                for (int a = 0; a < 3; a++) cam->at[a] = s->lo[a] <= s->hi[a] ? 0.5f * (s->lo[a] + s->hi[a]) : 0.0f;
            }
            cam->fov_y_deg = float(num(cj->get("fov"), 0.0));
            cam->medium = medium_ref(cj->get("medium"));
            if (cam->medium == -2) return fail(RT_ERR_PARSE, "scene JSON: camera refers to an unknown medium");
        }
    }
    return RT_OK;
}

}  // namespace

extern "C" {

rt_status rt_scene_add_mesh_obj(rt_scene* s, const char* path, const rt_material* mat, int32_t out_m, int32_t in_m,
                                int32_t* out_id) {
    if (!s || !path || !mat) return fail(RT_ERR_INVALID_ARG, "rt_scene_add_mesh_obj: NULL argument");
    return add_obj(s, path, mat, out_m, in_m, nullptr, out_id);
}

// Scene::AddTexture from pixels: RGBA8, row 0 at the bottom (v = 0).
RT_API rt_status rt_scene_add_texture(rt_scene* s, const uint8_t* rgba, int32_t width, int32_t height, int32_t* id) {
    if (!s || !rgba) return fail(RT_ERR_INVALID_ARG, "rt_scene_add_texture: NULL argument");
    if (width <= 0 || height <= 0 || int64_t(width) * height > (int64_t(1) << 28))
        return fail(RT_ERR_INVALID_ARG, "rt_scene_add_texture: bad size");
    const size_t n = size_t(width) * size_t(height);
    const int64_t off = int64_t(s->tex.size());
    if (off + int64_t(n) > int64_t(INT32_MAX))
        return fail(RT_ERR_OUT_OF_MEMORY, "rt_scene_add_texture: more than 2^31 texels in one scene");
    s->tex.resize(s->tex.size() + n);
    std::memcpy(s->tex.data() + off, rgba, n * 4);
    s->tex_info.push_back(int32_t(off));
    s->tex_info.push_back(width);
    s->tex_info.push_back(height);
    if (id) *id = int32_t(s->tex_info.size() / 3) - 1;
    return RT_OK;
}

RT_API rt_status rt_scene_get_texture(const rt_scene* s, int32_t id, int32_t* width, int32_t* height, uint8_t* rgba) {
    if (!s) return fail(RT_ERR_INVALID_ARG, "rt_scene_get_texture: NULL scene");
    if (id < 0 || size_t(id) * 3 >= s->tex_info.size()) return fail(RT_ERR_INVALID_ARG, "rt_scene_get_texture: bad id");
    const int32_t off = s->tex_info[3 * size_t(id)], w = s->tex_info[3 * size_t(id) + 1], h = s->tex_info[3 * size_t(id) + 2];
    if (width) *width = w;
    if (height) *height = h;
    if (rgba) std::memcpy(rgba, s->tex.data() + off, size_t(w) * size_t(h) * 4);
    return RT_OK;
}

// Scene::AddTexture(fileName): BMP or binary PGM/PPM.
RT_API rt_status rt_scene_add_texture_file(rt_scene* s, const char* path, int32_t* id) {
    if (!s || !path) return fail(RT_ERR_INVALID_ARG, "rt_scene_add_texture_file: NULL argument");
    std::vector<uint8_t> px;
    int w = 0, h = 0;
    std::string err;
    if (!read_image(path, px, w, h, err)) return fail(RT_ERR_IO, "rt_scene_add_texture_file: " + err);
    return rt_scene_add_texture(s, px.data(), w, h, id);
}

// Scene::AddEnv(fileName) + HdrTexture (core/src/Scene.cpp:79-81, 197-206):
// stbi_loadf with vertical flip.  Radiance .hdr files keep their floats; PNG,
// JPEG, BMP and PGM/PPM bytes become floats as stbi_loadf makes them
// ((v / 255)^2.2 for colour, v / 255 for alpha).
rt_status rt_scene_set_env_file(rt_scene* s, const char* path, float scale) {
    if (!s || !path) return fail(RT_ERR_INVALID_ARG, "rt_scene_set_env_file: NULL argument");
    std::string head;
    {
        std::FILE* f = std::fopen(path, "rb");
        if (!f) return fail(RT_ERR_IO, std::string("rt_scene_set_env_file: could not read ") + path);
        char b[2] = {0, 0};
        const size_t got = std::fread(b, 1, 2, f);
        std::fclose(f);
        head.assign(b, got);
    }
    std::vector<float> img;
    int w = 0, h = 0;
    std::string err;
    if (head == "#?") {
        if (!read_hdr(path, img, w, h, err)) return fail(RT_ERR_IO, "rt_scene_set_env_file: " + err);
    } else {
        std::vector<uint8_t> px;
        if (!read_image(path, px, w, h, err)) return fail(RT_ERR_IO, "rt_scene_set_env_file: " + err);
        float lut[256];
        for (int v = 0; v < 256; v++) lut[v] = float(std::pow(double(v) / 255.0, 2.2));
        img.resize(px.size());
        for (size_t i = 0; i < px.size(); i++) img[i] = (i & 3) == 3 ? float(px[i]) / 255.0f : lut[px[i]];
    }
    return rt_scene_set_env(s, img.data(), w, h, scale);
}

rt_status rt_scene_get_env(const rt_scene* s, float* rgba, int32_t* width, int32_t* height) {
    if (!s) return fail(RT_ERR_INVALID_ARG, "rt_scene_get_env: NULL scene");
    if (width) *width = s->env_w;
    if (height) *height = s->env_h;
    if (rgba && !s->env.empty()) std::memcpy(rgba, s->env.data(), s->env.size() * sizeof(float));
    return RT_OK;
}

rt_status rt_scene_load_json(rt_scene* s, const char* path, rt_options* opts, rt_camera* cam) {
    if (!s || !path) return fail(RT_ERR_INVALID_ARG, "rt_scene_load_json: NULL argument");
    std::string text;
    if (!read_file(path, text)) return fail(RT_ERR_IO, std::string("Open scene json failed: ") + path);
    return load_json(s, text, dir_of(path), opts, cam);
}

rt_status rt_scene_load_json_string(rt_scene* s, const char* json, const char* base_dir, rt_options* opts,
                                    rt_camera* cam) {
    if (!s || !json) return fail(RT_ERR_INVALID_ARG, "rt_scene_load_json_string: NULL argument");
    return load_json(s, json, base_dir ? base_dir : ".", opts, cam);
}

}  // extern "C"
