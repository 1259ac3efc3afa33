#pragma once
// Kerr metric in Cartesian Kerr-Schild form, written as a ParRelRay metric
// plug-in header: it provides exactly the hooks the reference solver and frame
// loop call (kernels/solver.cuh:43,81,87,96,106,154,163-168,197,209 and
// prr.cpp:319) with the reference's signatures, and drops into
// main/metric.h in place of metrics/schwarzschild.cuh.  The reference's own
// metrics/kerr.cuh is a stub (getGeod returns zero, metrics/kerr.cuh:72-74;
// its hook signatures differ from the solver's call sites).
//
// Coordinates and index order follow metrics/schwarzschild.cuh:123-141:
// (x, y, z, t), signature (+,+,+,-), g = eta + f l (x) l with
//   r^4 - (R^2 - a^2) r^2 - a^2 z^2 = 0,     R^2 = x^2 + y^2 + z^2
//   f   = 2 M r^3 / (r^4 + a^2 z^2)
//   l   = ((r x + a y)/(r^2+a^2), (r y - a x)/(r^2+a^2), z/r, 1)
// At a = 0 this is exactly the reference's Schwarzschild metric
// (f = rs/r, l = (x/r, y/r, z/r, 1)).  The spin a = Spacetime::getBhSpin()
// is a length (J/M); a > 0 is angular momentum along +z.
//
// getGeod evaluates the geodesic acceleration the textbook way a plug-in
// author would: metric derivatives -> full Christoffel table
// Gamma^k_{mn} = 1/2 g^{kl}(d_m g_ln + d_n g_lm - d_l g_mn) -> contraction.
// This is the "plain" form; the B200 kernels use a restructured contraction
// (parrelray_b200/csrc/metric_ks.cuh) that never forms the table.
#include "../main/base.h"
#include "../main/Camera.h"
#include "../main/Spacetime.h"
#include "../cudamaths/mats.h"

__host__ void User_INIT(ray *rays, Camera *cam, Spacetime *space) {}
__host__ bool User_RAYINIT(ray *rays, Camera *cam, Spacetime *space) { return true; }
__host__ bool User_TRACING(ray *rays, Camera *cam, Spacetime *space) { return true; }
__host__ bool User_POST(ray *rays, Camera *cam, Spacetime *space) { return true; }
__host__ void User_END(ray *rays, Camera *cam, Spacetime *space) {}

// Kerr-Schild radius r(x, y, z).
__host__ __device__ inline float kerr_ks_r(float x, float y, float z, float a)
{
    float R2 = x * x + y * y + z * z;
    float b = R2 - a * a;
    float S = sqrtf(b * b + 4.0f * a * a * z * z);
    return sqrtf(0.5f * (b + S));
}

// Outer horizon r_+ = M + sqrt(M^2 - a^2) (clamped at extremality).
__host__ __device__ inline float kerr_r_plus(float M, float a)
{
    float d = M * M - a * a;
    return M + sqrtf(d > 0.0f ? d : 0.0f);
}

__device__ bool User_LOOP(ray *iray, Camera cam, Spacetime space) { return true; }

__device__ bool User_UPDATE(ray *iray, Camera cam, Spacetime space, float h)
{
    f3 c = space.IntersectsScene(iray->r.xyz(), iray->u.xyz(), h);
    if (c.x >= 0.0f) { iray->result = RESULT::INTERSECTION; return false; }
    return true;
}

__device__ bool User_ENDLOOP(ray *iray, Camera cam, Spacetime space, tracer trace)
{
    float a = space.getBhSpin();
    float r = kerr_ks_r(iray->r.x, iray->r.y, iray->r.z, a);
    if (r >= trace.sph1.rout || r <= kerr_r_plus(space.getBhMass(), a) + 0.001f) {
        iray->result = RESULT::SUCCESS;
        return false;
    }
    f3 c = space.IntersectsScene(iray->r.xyz(), iray->u.xyz(), trace.h);
    if (c.x >= 0.0f) { iray->u = f4(c, 0.0f); iray->result = RESULT::INTERSECTION; return false; }
    return true;
}

// f, l_mu and their spatial derivatives df[k], dl[mu][k] (k = x,y,z).
__host__ __device__ inline void kerr_ks_fields(float x, float y, float z, float M, float a,
                                               float &f, float l[4], float df[3], float dl[4][3])
{
    float R2 = x * x + y * y + z * z;
    float a2 = a * a;
    float b = R2 - a2;
    float S = sqrtf(b * b + 4.0f * a2 * z * z);
    float r2 = 0.5f * (b + S);
    float r = sqrtf(r2);
    float dr[3] = {x * r / S, y * r / S, z * (r2 + a2) / (r * S)};
    float q = r2 + a2;
    float Sig = r2 * r2 + a2 * z * z;
    f = 2.0f * M * r2 * r / Sig;
    for (int k = 0; k < 3; k++) {
        float dSig = 4.0f * r2 * r * dr[k] + (k == 2 ? 2.0f * a2 * z : 0.0f);
        df[k] = 2.0f * M * (3.0f * r2 * dr[k] * Sig - r2 * r * dSig) / (Sig * Sig);
    }
    float nx = r * x + a * y, ny = r * y - a * x;
    l[0] = nx / q; l[1] = ny / q; l[2] = z / r; l[3] = 1.0f;
    for (int k = 0; k < 3; k++) {
        float dq = 2.0f * r * dr[k];
        float dnx = dr[k] * x + (k == 0 ? r : 0.0f) + (k == 1 ? a : 0.0f);
        float dny = dr[k] * y + (k == 1 ? r : 0.0f) - (k == 0 ? a : 0.0f);
        dl[0][k] = (dnx * q - nx * dq) / (q * q);
        dl[1][k] = (dny * q - ny * dq) / (q * q);
        dl[2][k] = (k == 2 ? 1.0f / r : 0.0f) - z * dr[k] / r2;
        dl[3][k] = 0.0f;
    }
}

__device__ f4 getGeod(f4 p, f4 u, Spacetime space)
{
    float M = space.getBhMass(), a = space.getBhSpin();
    float f, l[4], df[3], dl[4][3];
    kerr_ks_fields(p.x, p.y, p.z, M, a, f, l, df, dl);
    const float eta[4] = {1.0f, 1.0f, 1.0f, -1.0f};
    // dg[m][n][k] = d_k g_mn (d_t g = 0)
    float dg[4][4][4];
    for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++) {
            for (int k = 0; k < 3; k++)
                dg[m][n][k] = df[k] * l[m] * l[n] + f * (dl[m][k] * l[n] + l[m] * dl[n][k]);
            dg[m][n][3] = 0.0f;
        }
    // inverse metric g^{mn} = eta^{mn} - f l^m l^n, l^m = eta^{mm} l_m
    float lu[4] = {l[0], l[1], l[2], -l[3]};
    float gi[4][4];
    for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++)
            gi[m][n] = (m == n ? eta[m] : 0.0f) - f * lu[m] * lu[n];
    // Christoffel symbols of the first kind, then raised.
    float G1[4][4][4];
    for (int l_ = 0; l_ < 4; l_++)
        for (int m = 0; m < 4; m++)
            for (int n = 0; n < 4; n++)
                G1[l_][m][n] = 0.5f * (dg[l_][n][m] + dg[l_][m][n] - dg[m][n][l_]);
    float uu[4] = {u.x, u.y, u.z, u.w};
    float acc[4];
    for (int k = 0; k < 4; k++) {
        float s = 0.0f;
        for (int m = 0; m < 4; m++)
            for (int n = 0; n < 4; n++) {
                float G = 0.0f;
                for (int l_ = 0; l_ < 4; l_++) G += gi[k][l_] * G1[l_][m][n];
                s += G * uu[m] * uu[n];
            }
        acc[k] = -s;
    }
    return f4(acc[0], acc[1], acc[2], acc[3]);
}

__device__ mat4 getMetric(ray *Ray, Spacetime space)
{
    mat4 g;
    float M = space.getBhMass(), a = space.getBhSpin();
    f4 p = Ray->r;
    float r = kerr_ks_r(p.x, p.y, p.z, a);
    float r2 = r * r, q = r2 + a * a;
    float f = 2.0f * M * r2 * r / (r2 * r2 + a * a * p.z * p.z);
    float l[4] = {(r * p.x + a * p.y) / q, (r * p.y - a * p.x) / q, p.z / r, 1.0f};
    const float eta[4] = {1.0f, 1.0f, 1.0f, -1.0f};
    for (int m = 0; m < 4; m++)
        for (int n = 0; n < 4; n++)
            g[m * 4 + n] = (m == n ? eta[m] : 0.0f) + f * l[m] * l[n];
    return g;
}

// Per-sample colour, same rules as metrics/schwarzschild.cuh:151-183 with the
// Kerr-Schild radius and the outer horizon in place of |x| and rs.
__global__ void rayToRGB(ray *rays, Camera cam, Spacetime space, tracer trace, int samples)
{
    i2 ij = i2(blockIdx.x * blockDim.x + threadIdx.x, blockIdx.y * blockDim.y + threadIdx.y);
    if ((ij.x >= cam.getRes().x * samples) || (ij.y >= cam.getRes().y)) return;
    int pid = ij.y * cam.getRes().x * samples + ij.x;
    ray R = rays[pid];
    float a = space.getBhSpin();
    float r = kerr_ks_r(R.r.x, R.r.y, R.r.z, a);
    if (R.result == RESULT::SUCCESS) {
        if (r <= kerr_r_plus(space.getBhMass(), a) * 1.01f) { rays[pid].u = f4(0.0f, 0.0f, 0.0f, 0.0f); return; }
        if (r >= trace.sph1.rout) { rays[pid].u = f4(trace.sph1.getColorDefault2(rays[pid].u), 0.0f); return; }
    } else if (R.result == RESULT::INTERSECTION) {
        return;
    } else {
        rays[pid].u = f4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}
