// post.cu - SSAA combine (kernels/ssaa.cuh:109-131), FXAA
// (kernels/ssaa.cuh:141-181) and quantisation (cudamaths/image.cu:31).
// Built with -fmad=false so the combine and the FXAA taps reproduce the
// reference's FP32 arithmetic.
#include "kernels.cuh"

namespace prr {

// combineSamples: S = 1 -> clamp(rgb, 0, 1); S > 1 -> sqrt(sum clamp(rgb^2, 0, 1) / S).
__global__ void k_combine(const float *__restrict__ rgb, int w, int h, int S, float *__restrict__ image)
{
    int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    size_t p = (size_t)y * w + x;
    float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f;
    if (S == 1) {
        c0 = fminf(fmaxf(rgb[3 * p], 0.0f), 1.0f);
        c1 = fminf(fmaxf(rgb[3 * p + 1], 0.0f), 1.0f);
        c2 = fminf(fmaxf(rgb[3 * p + 2], 0.0f), 1.0f);
    } else {
        for (int s = 0; s < S; s++) {
            const float *q = rgb + 3 * (p * S + s);
            c0 += fminf(fmaxf(q[0] * q[0], 0.0f), 1.0f);
            c1 += fminf(fmaxf(q[1] * q[1], 0.0f), 1.0f);
            c2 += fminf(fmaxf(q[2] * q[2], 0.0f), 1.0f);
        }
        c0 = sqrtf(c0 / (float)S); c1 = sqrtf(c1 / (float)S); c2 = sqrtf(c2 / (float)S);
    }
    image[3 * p] = c0; image[3 * p + 1] = c1; image[3 * p + 2] = c2;
}

// luma (ssaa.cuh:141-143): double-literal weights, so the sum is formed in
// FP64 and returned as FP32.
__device__ __forceinline__ float luma_ref(float r, float g, float b)
{
    return (float)(r * 0.299 * (double)(1.0f / 255.0f) + g * 0.587 * (double)(1.0f / 255.0f) + b * 0.114 * (double)(1.0f / 255.0f));
}

__device__ __forceinline__ uint8_t quant(float v)
{
    v = fminf(fmaxf(v, 0.0f), 1.0f);
    return (uint8_t)roundf(255.0f * v);
}

// FXAA + quantisation.  One CTA covers a TX x TY tile; the tile plus a halo
// of 5 pixels (the 3x3 neighbourhood and the four bilinear taps, which reach
// at most |dir|/2 <= 4 pixels plus one cell) is staged in shared memory, so
// each input pixel is read from HBM once per tile.
constexpr int TX = 32, TY = 8, HALO = 5;
constexpr int SW = TX + 2 * HALO, SH = TY + 2 * HALO;

__global__ void __launch_bounds__(TX *TY) k_finish(const float *__restrict__ in, int w, int h, int fxaa,
                                                   float *__restrict__ out_f, uint8_t *__restrict__ out_u8)
{
    __shared__ float tile[3][SH][SW];
    const int x0 = blockIdx.x * TX - HALO, y0 = blockIdx.y * TY - HALO;
    const int tid = threadIdx.y * TX + threadIdx.x;
    if (fxaa) {
        for (int i = tid; i < SW * SH; i += TX * TY) {
            int sx = i % SW, sy = i / SW;
            int gx = min(max(x0 + sx, 0), w - 1), gy = min(max(y0 + sy, 0), h - 1);
            const float *q = in + 3 * ((size_t)gy * w + gx);
            tile[0][sy][sx] = q[0]; tile[1][sy][sx] = q[1]; tile[2][sy][sx] = q[2];
        }
        __syncthreads();
    }
    const int x = blockIdx.x * TX + threadIdx.x, y = blockIdx.y * TY + threadIdx.y;
    if (x >= w || y >= h) return;
    size_t p = (size_t)y * w + x;
    float o[3];
    if (!fxaa || x < 1 || y < 1 || x > w - 2 || y > h - 2 || w < 3 || h < 3) {
        // pixels the reference kernel never writes keep the combined colour
        const float *q = in + 3 * p;
        o[0] = q[0]; o[1] = q[1]; o[2] = q[2];
    } else {
        auto at = [&](int gx, int gy, int c) -> float { return tile[c][gy - y0][gx - x0]; };
        auto lum = [&](int gx, int gy) -> float { return luma_ref(at(gx, gy, 0), at(gx, gy, 1), at(gx, gy, 2)); };
        float lNW = lum(x - 1, y - 1), lNE = lum(x + 1, y - 1), lSW = lum(x - 1, y + 1), lSE = lum(x + 1, y + 1);
        float lM = lum(x, y);
        float lMin = fminf(lM, fminf(fminf(lNW, lNE), fminf(lSW, lSE)));
        float lMax = fmaxf(lM, fmaxf(fmaxf(lNW, lNE), fmaxf(lSW, lSE)));
        float dx = -((lNW + lNE) - (lSW + lSE)), dy = ((lNW + lSW) - (lNE + lSE));
        float dirReduce = fmaxf((lNW + lNE + lSW + lSE) * (0.25f * (1.0f / 8.0f)), 1.0f / 128.0f);
        float rcp = 1.0f / (fminf(fabsf(dx), fabsf(dy)) + dirReduce);
        dx = fminf(fmaxf(dx * rcp, -8.0f), 8.0f);
        dy = fminf(fmaxf(dy * rcp, -8.0f), 8.0f);
        // tex2d::operator[](f2) at uv = (ij + dir*k)/res
        auto tap = [&](float k, float *c) {
            float ux = ((float)x + dx * k) / (float)w, uy = ((float)y + dy * k) / (float)h;
            ux = ux * (float)w; uy = uy * (float)h;
            int ix = (int)floorf(ux), iy = (int)floorf(uy);
            float px = ux - (float)ix, py = uy - (float)iy;
            ix = min(max(ix, 0), w - 2);
            iy = min(max(iy, 0), h - 2);
#pragma unroll
            for (int ch = 0; ch < 3; ch++)
                c[ch] = at(ix, iy, ch) * (1 - px) * (1 - py) + at(ix + 1, iy, ch) * px * (1 - py) +
                        at(ix, iy + 1, ch) * (1 - px) * py + at(ix + 1, iy + 1, ch) * px * py;
        };
        float t1[3], t2[3], t3[3], t4[3];
        tap(1.0f / 3.0f - 0.5f, t1);
        tap(2.0f / 3.0f - 0.5f, t2);
        tap(-0.5f, t3);
        tap(0.5f, t4);
        float A[3], B[3];
#pragma unroll
        for (int ch = 0; ch < 3; ch++) {
            A[ch] = t1[ch] * 0.5f + t2[ch] * 0.5f;
            B[ch] = 0.5f * A[ch] + (t3[ch] * 0.25f + t4[ch] * 0.25f);
        }
        float lB = luma_ref(B[0], B[1], B[2]);
        const float *src = (lB < lMin || lB > lMax) ? A : B;
        o[0] = src[0]; o[1] = src[1]; o[2] = src[2];
    }
    if (out_f) { out_f[3 * p] = o[0]; out_f[3 * p + 1] = o[1]; out_f[3 * p + 2] = o[2]; }
    if (out_u8) { out_u8[3 * p] = quant(o[0]); out_u8[3 * p + 1] = quant(o[1]); out_u8[3 * p + 2] = quant(o[2]); }
}

cudaError_t launch_combine(const float *rgb, int w, int h, int samples, float *image, cudaStream_t st)
{
    dim3 blk(32, 8), grd((w + 31) / 32, (h + 7) / 8);
    k_combine<<<grd, blk, 0, st>>>(rgb, w, h, samples, image);
    return cudaGetLastError();
}

cudaError_t launch_finish(const float *image, int w, int h, int fxaa, float *out_f, uint8_t *out_u8, cudaStream_t st)
{
    dim3 blk(TX, TY), grd((w + TX - 1) / TX, (h + TY - 1) / TY);
    k_finish<<<grd, blk, 0, st>>>(image, w, h, fxaa, out_f, out_u8);
    return cudaGetLastError();
}

}  // namespace prr
