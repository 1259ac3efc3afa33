// Seeded procedural RGBA8 textures for the synthetic scenes: the reference
// ships none of its textures (ressources/moon8k.jpg and input/binback.ppm are
// absent), so every workload uses these.
//   kind 0 - sphere texture: 16x8 checkerboard modulated by two-octave value
//            noise and a per-seed tint (integer arithmetic only).
//   kind 1 - equirectangular starfield: dark vertical gradient plus point
//            stars placed by a per-pixel Bernoulli draw (a Poisson process at
//            this density), log-normal brightness, four star tints.
// Apart from one 1024-entry brightness table (double precision, built once),
// all arithmetic is integer, so the bytes are identical on every host.
#include <cmath>
#include <cstdint>
#include <cstring>

#include "prr.h"

namespace {

inline uint32_t mix32(uint32_t h)
{
    h ^= h >> 16; h *= 0x7feb352dU;
    h ^= h >> 15; h *= 0x846ca68bU;
    h ^= h >> 16;
    return h;
}

inline uint32_t hash3(uint32_t seed, uint32_t x, uint32_t y)
{
    return mix32(seed * 0x9E3779B1U ^ mix32(x * 0x85EBCA77U ^ mix32(y + 0xC2B2AE3DU)));
}

// Lattice value noise, period `w/cell` cells in x (wraps around the sphere's
// longitude), 8-bit result.
inline int value_noise(uint32_t seed, int x, int y, int w, int cell)
{
    int ncx = w / cell > 0 ? w / cell : 1;
    int gx = x / cell, gy = y / cell;
    int wx = ((x % cell) * 256) / cell, wy = ((y % cell) * 256) / cell;
    int x0 = gx % ncx, x1 = (gx + 1) % ncx;
    int v00 = hash3(seed, x0, gy) & 255, v10 = hash3(seed, x1, gy) & 255;
    int v01 = hash3(seed, x0, gy + 1) & 255, v11 = hash3(seed, x1, gy + 1) & 255;
    int top = v00 * (256 - wx) + v10 * wx;
    int bot = v01 * (256 - wx) + v11 * wx;
    return (top * (256 - wy) + bot * wy) >> 16;
}

// Acklam's rational approximation of the standard normal quantile function
// (P. J. Acklam, 2003; relative error < 1.2e-9).
double normal_quantile(double p)
{
    static const double a[] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                               1.383577518672690e+02, -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                               6.680131188771972e+01, -1.328068155288572e+01};
    static const double c[] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                               -2.549732539343734e+00, 4.374664141464968e+00, 2.938163982698783e+00};
    static const double d[] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                               3.754408661907416e+00};
    const double plow = 0.02425, phigh = 1 - plow;
    if (p < plow) {
        double q = std::sqrt(-2 * std::log(p));
        return (((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
               ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1);
    }
    if (p > phigh) {
        double q = std::sqrt(-2 * std::log(1 - p));
        return -(((((c[0] * q + c[1]) * q + c[2]) * q + c[3]) * q + c[4]) * q + c[5]) /
               ((((d[0] * q + d[1]) * q + d[2]) * q + d[3]) * q + 1);
    }
    double q = p - 0.5, r = q * q;
    return (((((a[0] * r + a[1]) * r + a[2]) * r + a[3]) * r + a[4]) * r + a[5]) * q /
           (((((b[0] * r + b[1]) * r + b[2]) * r + b[3]) * r + b[4]) * r + 1);
}

// Star brightness (0..255) at 1024 equiprobable log-normal quantiles,
// median 0.30, sigma 0.8 (natural-log units).
const uint8_t *star_levels()
{
    static uint8_t table[1024];
    static bool ready = false;
    if (!ready) {
        for (int i = 0; i < 1024; i++) {
            double L = std::exp(std::log(0.30) + 0.8 * normal_quantile((i + 0.5) / 1024.0));
            long v = std::lround(255.0 * L);
            table[i] = (uint8_t)(v < 24 ? 24 : (v > 255 ? 255 : v));
        }
        ready = true;
    }
    return table;
}

void make_sphere_texture(uint32_t seed, int w, int h, uint8_t *out)
{
    uint32_t th = hash3(seed, 7, 11);
    int tint[3] = {150 + (int)(th & 105), 150 + (int)((th >> 8) & 105), 150 + (int)((th >> 16) & 105)};
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            int chk = ((x * 16 / w) + (y * 8 / h)) & 1;
            int n = (3 * value_noise(seed, x, y, w, 32 > w ? w : 32) + value_noise(seed ^ 0x5bd1e995U, x, y, w, 8 > w ? w : 8)) / 4;
            int base = chk ? 210 : 60;
            uint8_t *p = out + 4 * ((size_t)y * w + x);
            for (int c = 0; c < 3; c++) {
                int v = base * tint[c] / 255;
                v = v * (90 + n * 166 / 255) / 256;
                p[c] = (uint8_t)(v < 0 ? 0 : (v > 255 ? 255 : v));
            }
            p[3] = 255;
        }
}

void make_starfield(uint32_t seed, int w, int h, uint8_t *out)
{
    static const int tints[4][3] = {{255, 214, 190}, {255, 255, 255}, {196, 214, 255}, {255, 236, 170}};
    const uint8_t *lv = star_levels();
    const uint32_t thresh = 12884902U;  // 0.003 stars per pixel
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            uint8_t *p = out + 4 * ((size_t)y * w + x);
            int r = 3 + 14 * y / h, g = 2 + 8 * y / h, b = 9 + 24 * (h - 1 - y) / h;
            uint32_t u = hash3(seed, x, y);
            if (u < thresh) {
                uint32_t v = hash3(seed ^ 0xA511E9B3U, x, y);
                int B = lv[v & 1023];
                const int *t = tints[(v >> 10) & 3];
                int sr = B * t[0] / 255, sg = B * t[1] / 255, sb = B * t[2] / 255;
                r = sr > r ? sr : r; g = sg > g ? sg : g; b = sb > b ? sb : b;
            }
            p[0] = (uint8_t)r; p[1] = (uint8_t)g; p[2] = (uint8_t)b; p[3] = 255;
        }
}

}  // namespace

extern "C" prr_status prr_make_texture(int kind, uint32_t seed, int w, int h, uint8_t *out_rgba8)
{
    if (!out_rgba8 || w < 2 || h < 2 || (long long)w * h > (1LL << 28)) return PRR_ERR_INVALID;
    if (kind == 0) make_sphere_texture(seed, w, h, out_rgba8);
    else if (kind == 1) make_starfield(seed, w, h, out_rgba8);
    else return PRR_ERR_INVALID;
    return PRR_OK;
}
