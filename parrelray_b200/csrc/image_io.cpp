// image_io.cpp - texture and frame files for the deck-driven host.
//
// The reference reads textures with stbi_loadf(path, ..., 3) under
// stbi_ldr_to_hdr_gamma(1) (cudamaths/image.cu:13-21), so a texel is
// byte/255, and writes frames with stbi_write_png after roundf(255*x)
// (cudamaths/image.cu:28-39).  Here: PNG (8/16-bit, grey, grey+alpha, RGB,
// RGBA, palette; Adam7 interlacing) and binary PNM (P6, P5) are decoded to
// RGBA8 with stb's channel rules (grey replicated; 16-bit samples keep their
// high byte; 1/2/4-bit grey scaled to 0..255; alpha dropped by the renderer);
// frames are written as 8-bit RGB PNG.  Inflate/deflate come from zlib.
// JPEG is not decoded (PRR_ERR_UNSUPPORTED): convert such textures to PNG.
#include <zlib.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "prr.h"

namespace {

void put_err(char *buf, size_t len, const std::string &msg)
{
    if (!buf || !len) return;
    size_t n = std::min(len - 1, msg.size());
    memcpy(buf, msg.data(), n);
    buf[n] = 0;
}

bool read_file(const char *path, std::vector<uint8_t> &out)
{
    FILE *f = fopen(path, "rb");
    if (!f) return false;
    uint8_t buf[1 << 16];
    size_t n;
    while ((n = fread(buf, 1, sizeof(buf), f)) > 0) out.insert(out.end(), buf, buf + n);
    fclose(f);
    return true;
}

uint32_t be32(const uint8_t *p) { return (uint32_t)p[0] << 24 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 8 | p[3]; }

// ------------------------------------------------------------------ PNM

bool pnm_token(const std::vector<uint8_t> &b, size_t &i, long &v)
{
    for (;;) {
        while (i < b.size() && (b[i] == ' ' || b[i] == '\t' || b[i] == '\n' || b[i] == '\r' || b[i] == '\v' || b[i] == '\f')) i++;
        if (i < b.size() && b[i] == '#') {
            while (i < b.size() && b[i] != '\n' && b[i] != '\r') i++;
            continue;
        }
        break;
    }
    if (i >= b.size() || b[i] < '0' || b[i] > '9') return false;
    v = 0;
    while (i < b.size() && b[i] >= '0' && b[i] <= '9') {
        v = v * 10 + (b[i] - '0');
        if (v > (1L << 30)) return false;
        i++;
    }
    return true;
}

prr_status load_pnm(const std::vector<uint8_t> &b, std::vector<uint8_t> &rgba, int &w, int &h, std::string &err)
{
    const int comp = b[1] == '6' ? 3 : 1;
    size_t i = 2;
    long W, H, maxv;
    if (!pnm_token(b, i, W) || !pnm_token(b, i, H) || !pnm_token(b, i, maxv)) { err = "malformed PNM header"; return PRR_ERR_IO; }
    if (maxv > 255) { err = "PNM with maxval > 255 is not supported"; return PRR_ERR_UNSUPPORTED; }
    if (W < 1 || H < 1 || W > 65536 || H > 65536) { err = "PNM size out of range"; return PRR_ERR_IO; }
    i++;  // the single whitespace byte after maxval
    size_t need = (size_t)W * H * comp;
    if (i > b.size() || b.size() - i < need) { err = "PNM pixel data truncated"; return PRR_ERR_IO; }
    w = (int)W; h = (int)H;
    rgba.resize((size_t)W * H * 4);
    for (size_t p = 0; p < (size_t)W * H; p++) {
        const uint8_t *s = &b[i + p * comp];
        rgba[4 * p] = s[0];
        rgba[4 * p + 1] = comp == 3 ? s[1] : s[0];
        rgba[4 * p + 2] = comp == 3 ? s[2] : s[0];
        rgba[4 * p + 3] = 255;
    }
    return PRR_OK;
}

// ------------------------------------------------------------------ PNG

int paeth(int a, int b, int c)
{
    int p = a + b - c, pa = abs(p - a), pb = abs(p - b), pc = abs(p - c);
    if (pa <= pb && pa <= pc) return a;
    return pb <= pc ? b : c;
}

// Reverses the per-row filters of one (sub-)image of `rows` rows of
// `rowbytes` bytes; `bpp` = bytes per complete pixel (at least 1).
bool unfilter(const uint8_t *src, size_t src_len, size_t rows, size_t rowbytes, int bpp, std::vector<uint8_t> &out)
{
    if (src_len < rows * (rowbytes + 1)) return false;
    out.assign(rows * rowbytes, 0);
    for (size_t y = 0; y < rows; y++) {
        const uint8_t ft = src[y * (rowbytes + 1)];
        const uint8_t *in = src + y * (rowbytes + 1) + 1;
        uint8_t *cur = &out[y * rowbytes];
        const uint8_t *prev = y ? &out[(y - 1) * rowbytes] : nullptr;
        for (size_t x = 0; x < rowbytes; x++) {
            int a = x >= (size_t)bpp ? cur[x - bpp] : 0;
            int up = prev ? prev[x] : 0;
            int c = (prev && x >= (size_t)bpp) ? prev[x - bpp] : 0;
            int v = in[x];
            switch (ft) {
            case 0: break;
            case 1: v += a; break;
            case 2: v += up; break;
            case 3: v += (a + up) >> 1; break;
            case 4: v += paeth(a, up, c); break;
            default: return false;
            }
            cur[x] = (uint8_t)v;
        }
    }
    return true;
}

struct PngInfo {
    uint32_t w = 0, h = 0;
    int depth = 0, ctype = 0, interlace = 0;
    int channels = 0;
    std::vector<uint8_t> palette;  // RGB triples
};

// Sample `k` (0..channels-1) of pixel x of an unfiltered row, as 8 bits.
uint8_t sample8(const PngInfo &I, const uint8_t *row, size_t x, int k)
{
    if (I.depth == 8) return row[x * I.channels + k];
    if (I.depth == 16) return row[2 * (x * I.channels + k)];  // high byte, as stb's 16 -> 8 conversion
    // 1, 2, 4 bits: grey or palette index, one channel
    size_t bit = x * I.depth;
    int v = (row[bit >> 3] >> (8 - I.depth - (int)(bit & 7))) & ((1 << I.depth) - 1);
    if (I.ctype == 3) return (uint8_t)v;
    static const int scale[5] = {0, 0xff, 0x55, 0, 0x11};
    return (uint8_t)(v * scale[I.depth]);
}

void put_pixel(const PngInfo &I, const uint8_t *row, size_t x, uint8_t *o)
{
    switch (I.ctype) {
    case 0: case 4: { uint8_t g = sample8(I, row, x, 0); o[0] = o[1] = o[2] = g; break; }
    case 2: case 6: o[0] = sample8(I, row, x, 0); o[1] = sample8(I, row, x, 1); o[2] = sample8(I, row, x, 2); break;
    case 3: {
        size_t idx = I.depth == 8 ? row[x] : sample8(I, row, x, 0);
        if (3 * idx + 2 < I.palette.size()) { o[0] = I.palette[3 * idx]; o[1] = I.palette[3 * idx + 1]; o[2] = I.palette[3 * idx + 2]; }
        else o[0] = o[1] = o[2] = 0;
        break;
    }
    }
    o[3] = 255;
}

prr_status load_png(const std::vector<uint8_t> &b, std::vector<uint8_t> &rgba, int &w, int &h, std::string &err)
{
    PngInfo I;
    std::vector<uint8_t> idat;
    size_t i = 8;
    bool have_ihdr = false, have_end = false;
    while (i + 8 <= b.size()) {
        uint32_t len = be32(&b[i]);
        const uint8_t *type = &b[i + 4];
        if (len > b.size() - i - 8 || b.size() - i - 8 - len < 4) { err = "PNG chunk truncated"; return PRR_ERR_IO; }
        const uint8_t *data = &b[i + 8];
        if (!memcmp(type, "IHDR", 4)) {
            if (len < 13) { err = "PNG IHDR too short"; return PRR_ERR_IO; }
            I.w = be32(data); I.h = be32(data + 4); I.depth = data[8]; I.ctype = data[9]; I.interlace = data[12];
            have_ihdr = true;
        } else if (!memcmp(type, "PLTE", 4)) {
            I.palette.assign(data, data + len);
        } else if (!memcmp(type, "IDAT", 4)) {
            idat.insert(idat.end(), data, data + len);
        } else if (!memcmp(type, "IEND", 4)) {
            have_end = true;
            break;
        }
        i += 12 + (size_t)len;
    }
    if (!have_ihdr || idat.empty()) { err = "PNG without IHDR or IDAT"; return PRR_ERR_IO; }
    (void)have_end;
    if (I.w < 1 || I.h < 1 || I.w > 65536 || I.h > 65536) { err = "PNG size out of range"; return PRR_ERR_IO; }
    switch (I.ctype) {
    case 0: I.channels = 1; break;
    case 2: I.channels = 3; break;
    case 3: I.channels = 1; break;
    case 4: I.channels = 2; break;
    case 6: I.channels = 4; break;
    default: err = "PNG colour type " + std::to_string(I.ctype) + " is invalid"; return PRR_ERR_IO;
    }
    bool depth_ok = I.depth == 8 || (I.depth == 16 && I.ctype != 3) ||
                    ((I.depth == 1 || I.depth == 2 || I.depth == 4) && (I.ctype == 0 || I.ctype == 3));
    if (!depth_ok) { err = "PNG bit depth " + std::to_string(I.depth) + " invalid for colour type " + std::to_string(I.ctype); return PRR_ERR_IO; }
    if (I.interlace > 1) { err = "PNG interlace method unknown"; return PRR_ERR_IO; }
    if (I.ctype == 3 && I.palette.empty()) { err = "palette PNG without PLTE"; return PRR_ERR_IO; }
    const int bits_px = I.depth * I.channels;
    const int bpp = std::max(1, bits_px / 8);
    auto rowbytes_of = [&](size_t width) { return (width * bits_px + 7) / 8; };
    // Adam7 passes: (x0, y0, dx, dy); a non-interlaced image is one pass
    static const int A7[7][4] = {{0, 0, 8, 8}, {4, 0, 8, 8}, {0, 4, 4, 8}, {2, 0, 4, 4}, {0, 2, 2, 4}, {1, 0, 2, 2}, {0, 1, 1, 2}};
    const int npass = I.interlace ? 7 : 1;
    size_t raw_len = 0;
    for (int p = 0; p < npass; p++) {
        size_t pw = I.interlace ? (I.w + A7[p][2] - 1 - A7[p][0]) / A7[p][2] : I.w;
        size_t ph = I.interlace ? (I.h + A7[p][3] - 1 - A7[p][1]) / A7[p][3] : I.h;
        if (I.interlace && (I.w <= (uint32_t)A7[p][0] || I.h <= (uint32_t)A7[p][1])) pw = ph = 0;
        if (pw && ph) raw_len += ph * (rowbytes_of(pw) + 1);
    }
    std::vector<uint8_t> raw(raw_len);
    z_stream zs;
    memset(&zs, 0, sizeof(zs));
    if (inflateInit(&zs) != Z_OK) { err = "zlib inflateInit failed"; return PRR_ERR_IO; }
    zs.next_in = idat.data();
    zs.avail_in = (uInt)idat.size();
    zs.next_out = raw.data();
    zs.avail_out = (uInt)raw.size();
    int zr = inflate(&zs, Z_FINISH);
    size_t got = raw.size() - zs.avail_out;
    inflateEnd(&zs);
    if ((zr != Z_STREAM_END && zr != Z_BUF_ERROR && zr != Z_OK) || got < raw_len) { err = "PNG image data is corrupt or truncated"; return PRR_ERR_IO; }
    w = (int)I.w; h = (int)I.h;
    rgba.assign((size_t)I.w * I.h * 4, 0);
    size_t off = 0;
    std::vector<uint8_t> rows;
    for (int p = 0; p < npass; p++) {
        const size_t x0 = I.interlace ? A7[p][0] : 0, y0 = I.interlace ? A7[p][1] : 0;
        const size_t dx = I.interlace ? A7[p][2] : 1, dy = I.interlace ? A7[p][3] : 1;
        if (I.w <= x0 || I.h <= y0) continue;
        size_t pw = (I.w - x0 + dx - 1) / dx, ph = (I.h - y0 + dy - 1) / dy;
        size_t rb = rowbytes_of(pw);
        if (!unfilter(raw.data() + off, raw.size() - off, ph, rb, bpp, rows)) { err = "PNG filter type invalid"; return PRR_ERR_IO; }
        off += ph * (rb + 1);
        for (size_t y = 0; y < ph; y++)
            for (size_t x = 0; x < pw; x++) put_pixel(I, &rows[y * rb], x, &rgba[4 * ((y0 + y * dy) * I.w + x0 + x * dx)]);
    }
    return PRR_OK;
}

void png_chunk(FILE *f, const char *type, const uint8_t *data, size_t len)
{
    uint8_t hdr[8] = {(uint8_t)(len >> 24), (uint8_t)(len >> 16), (uint8_t)(len >> 8), (uint8_t)len,
                      (uint8_t)type[0], (uint8_t)type[1], (uint8_t)type[2], (uint8_t)type[3]};
    fwrite(hdr, 1, 8, f);
    if (len) fwrite(data, 1, len, f);
    uLong crc = crc32(0L, Z_NULL, 0);
    crc = crc32(crc, (const Bytef *)type, 4);
    if (len) crc = crc32(crc, data, (uInt)len);
    uint8_t c[4] = {(uint8_t)(crc >> 24), (uint8_t)(crc >> 16), (uint8_t)(crc >> 8), (uint8_t)crc};
    fwrite(c, 1, 4, f);
}

}  // namespace

extern "C" {

prr_status prr_image_load(const char *path, uint8_t **rgba8, int *w, int *h, char *errbuf, size_t errlen)
{
    if (!path || !rgba8 || !w || !h) { put_err(errbuf, errlen, "prr_image_load: null argument"); return PRR_ERR_INVALID; }
    *rgba8 = nullptr;
    std::vector<uint8_t> b;
    if (!read_file(path, b)) { put_err(errbuf, errlen, std::string("cannot open image ") + path); return PRR_ERR_IO; }
    std::vector<uint8_t> px;
    std::string err;
    prr_status s;
    static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    if (b.size() >= 8 && !memcmp(b.data(), sig, 8)) s = load_png(b, px, *w, *h, err);
    else if (b.size() >= 2 && b[0] == 'P' && (b[1] == '6' || b[1] == '5')) s = load_pnm(b, px, *w, *h, err);
    else if (b.size() >= 2 && b[0] == 0xFF && b[1] == 0xD8) { err = "JPEG is not decoded: convert the texture to PNG or binary PPM"; s = PRR_ERR_UNSUPPORTED; }
    else { err = "unknown image format (PNG, binary PPM/PGM)"; s = PRR_ERR_UNSUPPORTED; }
    if (s != PRR_OK) { put_err(errbuf, errlen, std::string(path) + ": " + err); return s; }
    *rgba8 = (uint8_t *)malloc(px.size());
    if (!*rgba8) { put_err(errbuf, errlen, "out of host memory"); return PRR_ERR_NOMEM; }
    memcpy(*rgba8, px.data(), px.size());
    return PRR_OK;
}

void prr_image_free(uint8_t *rgba8) { free(rgba8); }

prr_status prr_png_write(const char *path, const uint8_t *rgb8, int w, int h)
{
    if (!path || !rgb8 || w < 1 || h < 1) return PRR_ERR_INVALID;
    const size_t rb = (size_t)w * 3;
    std::vector<uint8_t> raw((rb + 1) * h);
    for (int y = 0; y < h; y++) {
        raw[y * (rb + 1)] = 0;  // filter: none
        memcpy(&raw[y * (rb + 1) + 1], rgb8 + y * rb, rb);
    }
    uLongf zlen = compressBound((uLong)raw.size());
    std::vector<uint8_t> z(zlen);
    if (compress2(z.data(), &zlen, raw.data(), (uLong)raw.size(), 6) != Z_OK) return PRR_ERR_IO;
    FILE *f = fopen(path, "wb");
    if (!f) return PRR_ERR_IO;
    static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
    fwrite(sig, 1, 8, f);
    uint8_t ihdr[13] = {(uint8_t)(w >> 24), (uint8_t)(w >> 16), (uint8_t)(w >> 8), (uint8_t)w,
                        (uint8_t)(h >> 24), (uint8_t)(h >> 16), (uint8_t)(h >> 8), (uint8_t)h, 8, 2, 0, 0, 0};
    png_chunk(f, "IHDR", ihdr, 13);
    png_chunk(f, "IDAT", z.data(), zlen);
    png_chunk(f, "IEND", nullptr, 0);
    bool ok = !ferror(f);
    ok = (fclose(f) == 0) && ok;
    return ok ? PRR_OK : PRR_ERR_IO;
}

}  // extern "C"
