// accum_io.cpp — the reference's accumulation file formats (host, C++17).
//
// 1. Accumulation EXR (src/output/accum.rs): the radiance SUM of a sample
//    range and the per-pixel sample count, as an OpenEXR image with the f32
//    channels B, G, R and count (names sorted, as the reference writes them)
//    and the layer name "accum". `render merge` (accum.rs:88-119) adds the
//    files' sums and counts and divides. Written here as uncompressed
//    scanlines (any OpenEXR reader accepts them); read in the forms an
//    OpenEXR writer produces for a single-part flat image: scanline or
//    one-level tiled blocks, NONE / RLE / ZIPS / ZIP compression, FLOAT or
//    HALF channels.
// 2. Metal checkpoint (src/raytracer/metal/renderer.rs:219-254): "RCKP",
//    width, height, passes done (u32 LE), then the f32 RGBW accumulator.

#include <stdint.h>
#include <string.h>
#include <zlib.h>

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "rt_cuda.h"

namespace rt {

std::string& accum_error();  // defined in session.cu: the thread's last error

namespace {

int fail_io(int code, const std::string& msg) {
    accum_error() = msg;
    return code;
}

void put_u32(std::vector<uint8_t>& b, uint32_t v) {
    for (int k = 0; k < 4; k++) b.push_back((uint8_t)(v >> (8 * k)));
}
void put_u64(std::vector<uint8_t>& b, uint64_t v) {
    for (int k = 0; k < 8; k++) b.push_back((uint8_t)(v >> (8 * k)));
}
void put_f32(std::vector<uint8_t>& b, float f) {
    uint32_t v;
    memcpy(&v, &f, 4);
    put_u32(b, v);
}
void put_str(std::vector<uint8_t>& b, const char* s) { b.insert(b.end(), s, s + strlen(s) + 1); }
void put_attr(std::vector<uint8_t>& b, const char* name, const char* type, const std::vector<uint8_t>& v) {
    put_str(b, name);
    put_str(b, type);
    put_u32(b, (uint32_t)v.size());
    b.insert(b.end(), v.begin(), v.end());
}

uint32_t get_u32(const uint8_t* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24); }
uint64_t get_u64(const uint8_t* p) { return (uint64_t)get_u32(p) | ((uint64_t)get_u32(p + 4) << 32); }

float half_to_float(uint16_t h) {
    const uint32_t s = (uint32_t)(h >> 15) & 1u, e = (h >> 10) & 31u, m = h & 1023u;
    float v;
    if (e == 0) v = std::ldexp((float)m, -24);
    else if (e == 31) v = m ? NAN : INFINITY;
    else v = std::ldexp((float)(m | 1024u), (int)e - 25);
    return s ? -v : v;
}

const char* const CHANNELS[4] = {"B", "G", "R", "count"};

std::vector<uint8_t> exr_bytes(uint32_t w, uint32_t h, const double* rgbw) {
    std::vector<uint8_t> b;
    put_u32(b, 20000630u);  // magic 0x762f3101
    put_u32(b, 2u);         // version 2, single-part scanline
    std::vector<uint8_t> v;
    for (const char* c : CHANNELS) {
        put_str(v, c);
        put_u32(v, 2u);  // FLOAT
        put_u32(v, 0u);  // pLinear + reserved
        put_u32(v, 1u);  // x sampling
        put_u32(v, 1u);  // y sampling
    }
    v.push_back(0);
    put_attr(b, "channels", "chlist", v);
    put_attr(b, "compression", "compression", {0});
    v.clear();
    for (uint32_t x : {0u, 0u, w - 1, h - 1}) put_u32(v, x);
    put_attr(b, "dataWindow", "box2i", v);
    put_attr(b, "displayWindow", "box2i", v);
    put_attr(b, "lineOrder", "lineOrder", {0});
    v.clear();
    put_str(v, "accum");
    v.pop_back();  // string attributes carry no terminator
    put_attr(b, "name", "string", v);
    v.clear();
    put_f32(v, 1.0f);
    put_attr(b, "pixelAspectRatio", "float", v);
    v.clear();
    put_f32(v, 0.0f);
    put_f32(v, 0.0f);
    put_attr(b, "screenWindowCenter", "v2f", v);
    v.clear();
    put_f32(v, 1.0f);
    put_attr(b, "screenWindowWidth", "float", v);
    b.push_back(0);
    const uint64_t line_bytes = 8ull + 4ull * 4 * w;
    const uint64_t first = b.size() + 8ull * h;
    for (uint32_t y = 0; y < h; y++) put_u64(b, first + y * line_bytes);
    static const int src[4] = {2, 1, 0, 3};  // B, G, R, count from (r, g, b, w)
    for (uint32_t y = 0; y < h; y++) {
        put_u32(b, y);
        put_u32(b, 4u * 4u * w);
        for (int c = 0; c < 4; c++)
            for (uint32_t x = 0; x < w; x++) put_f32(b, (float)rgbw[4ull * ((uint64_t)y * w + x) + src[c]]);
    }
    return b;
}

// Undo the OpenEXR byte predictor and the even/odd split of RLE and ZIP blocks.
void exr_unpredict(std::vector<uint8_t>& t, std::vector<uint8_t>& out) {
    for (size_t i = 1; i < t.size(); i++) t[i] = (uint8_t)((int)t[i - 1] + (int)t[i] - 128);
    out.resize(t.size());
    const size_t half = (t.size() + 1) / 2;
    for (size_t i = 0; i < t.size(); i++) out[i] = (i & 1) ? t[half + i / 2] : t[i / 2];
}

bool exr_rle(const uint8_t* in, size_t n, size_t expect, std::vector<uint8_t>& t) {
    t.clear();
    size_t i = 0;
    while (i < n) {
        const int8_t c = (int8_t)in[i++];
        if (c < 0) {
            const size_t k = (size_t)(-(int)c);
            if (i + k > n || t.size() + k > expect) return false;
            t.insert(t.end(), in + i, in + i + k);
            i += k;
        } else {
            const size_t k = (size_t)c + 1;
            if (i >= n || t.size() + k > expect) return false;
            t.insert(t.end(), k, in[i++]);
        }
    }
    return t.size() == expect;
}

struct Exr {
    uint32_t w = 0, h = 0;
    std::vector<float> ch[4];  // B, G, R, count, row-major
};

int exr_read(const char* path, Exr* out, bool header_only) {
    FILE* f = fopen(path, "rb");
    if (!f) return fail_io(RT_ERR_IO, std::string("cannot open ") + path);
    std::vector<uint8_t> d;
    uint8_t buf[1 << 16];
    size_t k;
    while ((k = fread(buf, 1, sizeof(buf), f)) > 0) d.insert(d.end(), buf, buf + k);
    fclose(f);
    const std::string bad = std::string(path) + ": not an accumulation EXR: ";
    if (d.size() < 8 || get_u32(d.data()) != 20000630u) return fail_io(RT_ERR_IO, bad + "bad magic");
    const uint32_t ver = get_u32(d.data() + 4);
    if ((ver & 0xFFu) != 2u || (ver & 0x1800u)) return fail_io(RT_ERR_IO, bad + "multi-part or deep data");
    bool tiled = (ver & 0x200u) != 0;
    size_t p = 8;
    struct Chan {
        std::string name;
        uint32_t type;
    };
    std::vector<Chan> chans;
    int comp = -1;
    int32_t win[4] = {0, 0, -1, -1};
    uint32_t tx = 0, ty = 0, tmode = 0;
    for (;;) {
        if (p >= d.size()) return fail_io(RT_ERR_IO, bad + "truncated header");
        if (d[p] == 0) {
            p++;
            break;
        }
        std::string name((const char*)&d[p], strnlen((const char*)&d[p], d.size() - p));
        p += name.size() + 1;
        if (p >= d.size()) return fail_io(RT_ERR_IO, bad + "truncated header");
        std::string type((const char*)&d[p], strnlen((const char*)&d[p], d.size() - p));
        p += type.size() + 1;
        if (p + 4 > d.size()) return fail_io(RT_ERR_IO, bad + "truncated header");
        const uint32_t sz = get_u32(&d[p]);
        p += 4;
        if (p + sz > d.size()) return fail_io(RT_ERR_IO, bad + "truncated header");
        const uint8_t* v = &d[p];
        if (name == "channels") {
            size_t q = 0;
            while (q < sz && v[q]) {
                std::string cn((const char*)v + q, strnlen((const char*)v + q, sz - q));
                q += cn.size() + 1;
                if (q + 16 > sz) return fail_io(RT_ERR_IO, bad + "bad channel list");
                if (get_u32(v + q + 8) != 1u || get_u32(v + q + 12) != 1u)
                    return fail_io(RT_ERR_IO, bad + "subsampled channel");
                chans.push_back({cn, get_u32(v + q)});
                q += 16;
            }
        } else if (name == "compression") {
            comp = sz ? v[0] : -1;
        } else if (name == "dataWindow" && sz == 16) {
            for (int i = 0; i < 4; i++) win[i] = (int32_t)get_u32(v + 4 * i);
        } else if (name == "tiles" && sz == 9) {
            tx = get_u32(v);
            ty = get_u32(v + 4);
            tmode = v[8];
            tiled = true;
        }
        p += sz;
    }
    if (win[2] < win[0] || win[3] < win[1]) return fail_io(RT_ERR_IO, bad + "empty data window");
    const uint32_t w = (uint32_t)(win[2] - win[0] + 1), h = (uint32_t)(win[3] - win[1] + 1);
    out->w = w;
    out->h = h;
    int slot[4] = {-1, -1, -1, -1};
    for (int c = 0; c < 4; c++)
        for (size_t i = 0; i < chans.size(); i++)
            if (chans[i].name == CHANNELS[c]) slot[c] = (int)i;
    for (int c = 0; c < 4; c++)
        if (slot[c] < 0) return fail_io(RT_ERR_IO, bad + "missing channel " + CHANNELS[c]);
    for (const Chan& c : chans)
        if (c.type > 2u) return fail_io(RT_ERR_IO, bad + "unknown channel type");
    if (header_only) return RT_OK;
    if (comp != 0 && comp != 1 && comp != 2 && comp != 3)
        return fail_io(RT_ERR_IO, bad + "compression " + std::to_string(comp) + " not supported");
    if (tiled && (tx == 0 || ty == 0 || (tmode & 0xFu) != 0)) return fail_io(RT_ERR_IO, bad + "multi-level tiles");
    for (auto& v : out->ch) v.assign((size_t)w * h, 0.0f);
    // Blocks: a rectangle of pixels each (scanline groups or tiles).
    const uint32_t lines = comp == 3 ? 16u : 1u;
    const uint32_t bw = tiled ? tx : w, bh = tiled ? ty : lines;
    const uint32_t nbx = tiled ? (w + tx - 1) / tx : 1u, nby = (h + bh - 1) / bh;
    const uint64_t nblocks = (uint64_t)nbx * nby;
    if (p + 8 * nblocks > d.size()) return fail_io(RT_ERR_IO, bad + "truncated offset table");
    std::vector<uint8_t> raw, tmp;
    size_t pix_bytes = 0;
    for (const Chan& c : chans) pix_bytes += c.type == 1u ? 2 : 4;
    for (uint64_t bi = 0; bi < nblocks; bi++) {
        uint64_t off = get_u64(&d[p + 8 * bi]);
        uint32_t x0, y0, cw, chh;
        size_t q;
        if (tiled) {
            if (off + 20 > d.size()) return fail_io(RT_ERR_IO, bad + "truncated tile");
            const int32_t tix = (int32_t)get_u32(&d[off]), tiy = (int32_t)get_u32(&d[off + 4]);
            if (tix < 0 || tiy < 0 || (uint32_t)tix >= nbx || (uint32_t)tiy >= nby)
                return fail_io(RT_ERR_IO, bad + "tile out of range");
            x0 = (uint32_t)tix * tx;
            y0 = (uint32_t)tiy * ty;
            q = off + 16;
        } else {
            if (off + 8 > d.size()) return fail_io(RT_ERR_IO, bad + "truncated scanline block");
            const int32_t yy = (int32_t)get_u32(&d[off]) - win[1];
            if (yy < 0 || (uint32_t)yy >= h || (uint32_t)yy % bh) return fail_io(RT_ERR_IO, bad + "bad scanline block");
            x0 = 0;
            y0 = (uint32_t)yy;
            q = off + 4;
        }
        cw = std::min(bw, w - x0);
        chh = std::min(bh, h - y0);
        const uint32_t n = get_u32(&d[q]);
        q += 4;
        if (q + n > d.size()) return fail_io(RT_ERR_IO, bad + "truncated block");
        const size_t expect = pix_bytes * cw * chh;
        const uint8_t* blk = &d[q];
        if (n < expect && comp == 1) {
            if (!exr_rle(blk, n, expect, tmp)) return fail_io(RT_ERR_IO, bad + "corrupt RLE block");
            exr_unpredict(tmp, raw);
            blk = raw.data();
        } else if (n < expect && (comp == 2 || comp == 3)) {
            tmp.resize(expect);
            uLongf len = (uLongf)expect;
            if (uncompress(tmp.data(), &len, blk, n) != Z_OK || len != expect)
                return fail_io(RT_ERR_IO, bad + "corrupt ZIP block");
            exr_unpredict(tmp, raw);
            blk = raw.data();
        } else if (n != expect) {
            return fail_io(RT_ERR_IO, bad + "block size mismatch");
        }
        // Per scanline of the block: every channel's run of cw values.
        size_t o = 0;
        for (uint32_t yy = 0; yy < chh; yy++)
            for (size_t ci = 0; ci < chans.size(); ci++) {
                int dst = -1;
                for (int c = 0; c < 4; c++)
                    if (slot[c] == (int)ci) dst = c;
                const uint32_t t = chans[ci].type;
                for (uint32_t xx = 0; xx < cw; xx++) {
                    float val;
                    if (t == 1u) {
                        val = half_to_float((uint16_t)(blk[o] | (blk[o + 1] << 8)));
                        o += 2;
                    } else {
                        uint32_t u = get_u32(blk + o);
                        o += 4;
                        if (t == 2u) memcpy(&val, &u, 4);
                        else val = (float)u;
                    }
                    if (dst >= 0) out->ch[dst][(size_t)(y0 + yy) * w + x0 + xx] = val;
                }
            }
    }
    return RT_OK;
}

}  // namespace

}  // namespace rt

using namespace rt;

extern "C" {

int rt_accum_exr_write(const char* path, uint32_t width, uint32_t height, const double* rgbw) {
    if (!path || !rgbw || !width || !height) return fail_io(RT_ERR_INVALID, "NULL argument or empty image");
    std::vector<uint8_t> b = exr_bytes(width, height, rgbw);
    std::string tmp = std::string(path) + ".tmp";
    FILE* f = fopen(tmp.c_str(), "wb");
    if (!f) return fail_io(RT_ERR_IO, "cannot open " + tmp);
    bool ok = fwrite(b.data(), 1, b.size(), f) == b.size();
    ok = (fclose(f) == 0) && ok;
    if (!ok || rename(tmp.c_str(), path) != 0) {
        remove(tmp.c_str());
        return fail_io(RT_ERR_IO, std::string("cannot write ") + path);
    }
    return RT_OK;
}

int rt_accum_exr_info(const char* path, uint32_t* width, uint32_t* height) {
    if (!path || !width || !height) return fail_io(RT_ERR_INVALID, "NULL argument");
    Exr e;
    int rc = exr_read(path, &e, true);
    if (rc) return rc;
    *width = e.w;
    *height = e.h;
    return RT_OK;
}

int rt_accum_exr_read(const char* path, uint32_t width, uint32_t height, double* rgbw) {
    if (!path || !rgbw) return fail_io(RT_ERR_INVALID, "NULL argument");
    Exr e;
    int rc = exr_read(path, &e, false);
    if (rc) return rc;
    if (e.w != width || e.h != height) return fail_io(RT_ERR_MISMATCH, std::string(path) + ": resolution mismatch");
    const size_t n = (size_t)width * height;
    for (size_t i = 0; i < n; i++) {
        rgbw[4 * i + 0] = e.ch[2][i];
        rgbw[4 * i + 1] = e.ch[1][i];
        rgbw[4 * i + 2] = e.ch[0][i];
        rgbw[4 * i + 3] = e.ch[3][i];
    }
    return RT_OK;
}

int rt_accum_merge(const char* const* paths, uint32_t n_paths, uint32_t width, uint32_t height, float* rgb) {
    if (!paths || !n_paths || !rgb) return fail_io(RT_ERR_INVALID, "merge needs at least one accum file");
    const size_t n = (size_t)width * height;
    std::vector<double> sum(4 * n, 0.0), one(4 * n);
    for (uint32_t k = 0; k < n_paths; k++) {
        int rc = rt_accum_exr_read(paths[k], width, height, one.data());
        if (rc) return rc;
        for (size_t i = 0; i < 4 * n; i++) sum[i] += one[i];
    }
    for (size_t i = 0; i < n; i++) {
        const double c = sum[4 * i + 3];
        for (int a = 0; a < 3; a++) rgb[3 * i + a] = c > 0.0 ? (float)(sum[4 * i + a] / c) : 0.0f;
    }
    return RT_OK;
}

int rt_rckp_write(const char* path, uint32_t width, uint32_t height, uint32_t passes_done, const double* rgbw) {
    if (!path || !rgbw) return fail_io(RT_ERR_INVALID, "NULL argument");
    std::vector<uint8_t> b;
    b.insert(b.end(), {'R', 'C', 'K', 'P'});
    put_u32(b, width);
    put_u32(b, height);
    put_u32(b, passes_done);
    const size_t n = 4ull * width * height;
    b.reserve(16 + 4 * n);
    for (size_t i = 0; i < n; i++) put_f32(b, (float)rgbw[i]);
    std::string tmp = std::string(path) + ".tmp";
    FILE* f = fopen(tmp.c_str(), "wb");
    if (!f) return fail_io(RT_ERR_IO, "cannot open " + tmp);
    bool ok = fwrite(b.data(), 1, b.size(), f) == b.size();
    ok = (fclose(f) == 0) && ok;
    if (!ok || rename(tmp.c_str(), path) != 0) {
        remove(tmp.c_str());
        return fail_io(RT_ERR_IO, std::string("cannot write checkpoint ") + path);
    }
    return RT_OK;
}

int rt_film_exr_write(const char* path, uint32_t width, uint32_t height, const float* film, const char* manifest) {
    if (!path || !film || !width || !height) return fail_io(RT_ERR_INVALID, "NULL argument or empty image");
    // (name, film offset) in byte order of the names, as the reference sorts them.
    static const struct {
        const char* name;
        int off;
    } ch[RT_FILM_FLOATS] = {{"B", RT_FILM_BEAUTY + 2},        {"G", RT_FILM_BEAUTY + 1},
                            {"N.X", RT_FILM_NORMAL},          {"N.Y", RT_FILM_NORMAL + 1},
                            {"N.Z", RT_FILM_NORMAL + 2},      {"R", RT_FILM_BEAUTY},
                            {"albedo.B", RT_FILM_ALBEDO + 2}, {"albedo.G", RT_FILM_ALBEDO + 1},
                            {"albedo.R", RT_FILM_ALBEDO},     {"depth.Z", RT_FILM_DEPTH},
                            {"diffuse.B", RT_FILM_DIFFUSE + 2}, {"diffuse.G", RT_FILM_DIFFUSE + 1},
                            {"diffuse.R", RT_FILM_DIFFUSE},   {"id.coverage", RT_FILM_ID + 1},
                            {"id.x", RT_FILM_ID},             {"specular.B", RT_FILM_SPECULAR + 2},
                            {"specular.G", RT_FILM_SPECULAR + 1}, {"specular.R", RT_FILM_SPECULAR}};
    std::vector<uint8_t> b;
    put_u32(b, 20000630u);
    put_u32(b, 2u);
    std::vector<uint8_t> v;
    for (const auto& c : ch) {
        put_str(v, c.name);
        put_u32(v, 2u);
        put_u32(v, 0u);
        put_u32(v, 1u);
        put_u32(v, 1u);
    }
    v.push_back(0);
    put_attr(b, "channels", "chlist", v);
    put_attr(b, "compression", "compression", {0});
    v.clear();
    for (uint32_t x : {0u, 0u, width - 1, height - 1}) put_u32(v, x);
    put_attr(b, "dataWindow", "box2i", v);
    put_attr(b, "displayWindow", "box2i", v);
    put_attr(b, "lineOrder", "lineOrder", {0});
    v.assign({'r', 'g', 'b', 'a'});
    put_attr(b, "name", "string", v);
    v.clear();
    put_f32(v, 1.0f);
    put_attr(b, "pixelAspectRatio", "float", v);
    if (manifest && *manifest) {
        v.assign(manifest, manifest + strlen(manifest));
        put_attr(b, "render_rs/manifest", "string", v);
    }
    v.clear();
    put_f32(v, 0.0f);
    put_f32(v, 0.0f);
    put_attr(b, "screenWindowCenter", "v2f", v);
    v.clear();
    put_f32(v, 1.0f);
    put_attr(b, "screenWindowWidth", "float", v);
    b.push_back(0);
    const uint64_t line_bytes = 8ull + 4ull * RT_FILM_FLOATS * width;
    const uint64_t first = b.size() + 8ull * height;
    for (uint32_t y = 0; y < height; y++) put_u64(b, first + y * line_bytes);
    for (uint32_t y = 0; y < height; y++) {
        put_u32(b, y);
        put_u32(b, 4u * RT_FILM_FLOATS * width);
        for (const auto& c : ch)
            for (uint32_t x = 0; x < width; x++) put_f32(b, film[(size_t)RT_FILM_FLOATS * ((size_t)y * width + x) + c.off]);
    }
    std::string tmp = std::string(path) + ".tmp";
    FILE* f = fopen(tmp.c_str(), "wb");
    if (!f) return fail_io(RT_ERR_IO, "cannot open " + tmp);
    bool ok = fwrite(b.data(), 1, b.size(), f) == b.size();
    ok = (fclose(f) == 0) && ok;
    if (!ok || rename(tmp.c_str(), path) != 0) {
        remove(tmp.c_str());
        return fail_io(RT_ERR_IO, std::string("cannot write ") + path);
    }
    return RT_OK;
}

}  // extern "C"
