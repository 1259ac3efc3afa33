// k_adjoint.cu - discrete adjoint of the PHYSICAL-mode RKF45 render:
// d(loss)/d(spin a, mass M, camera inclination i, camera distance r, orbital
// phase of one sphere) given dL/d(image).
//
// Per ray, with the accepted step sizes and every discrete event
// (accept/reject, intersection mode, termination, which sphere is hit)
// frozen at the forward run.  The forward steps run in the frame's precision
// (TF = float: the FP32 PHYSICAL stepper with Kahan-compensated updates;
// TF = double: FP64); the adjoint and the gradient reduction are FP64:
//   1. forward: the PHYSICAL stepper runs the ray and saves its full state
//      every ADJ_K accepted steps (checkpoints in HBM, per thread);
//   2. colour adjoint: dL/dc of the ray's sample through the SSAA combine,
//      then lambda_N = dL/dc . dc/dy_N (+ the sphere-phase term) with c the
//      bilinear sky or the sphere texture at the hit point;
//   3. reverse: for each segment, last first, the steps are recomputed from
//      the checkpoint (bit-identical: same stepper) in two levels - a pass
//      that keeps a sub-checkpoint every ADJ_SUB steps, then, sub-segment by
//      sub-segment, a pass that keeps the ADJ_SUB states - so a thread holds
//      a few hundred bytes of states instead of a whole segment; lambda is
//      pulled back through each step of x' = u, u' = G(x, u) in the stepper's
//      form (only the velocity increments ku_i = h G(z_i) are kept: the
//      stage points z_i are rebuilt from them, and their adjoints carry the
//      position coupling); the products lambda^T dG/dz come from the
//      geodesic's hand-written reverse sweep (geod_vjp.cuh);
//   4. lambda_0 is pulled back through the initial data (camera position,
//      ray direction, null u^t), also by dual numbers.
// Gradients are accumulated per thread and reduced in FP64.
#include <cub/device/device_radix_sort.cuh>

#include "dual.cuh"
#include "geod_vjp.cuh"
#include "kernels.cuh"
#include "phys_stepper.cuh"

namespace prr {

using DC = Dual<13>;  // initial data / colour: 8 state components + 5 parameters
enum { P_SPIN = 0, P_MASS = 1, P_INCL = 2, P_CAMR = 3, P_PHASE = 4 };

// Sphere::getColor at p + v d for a T-valued centre (derivative-carrying
// version of sphere_colour; same arithmetic in FP64).
template <class T>
__device__ V3<T> sphere_colour_ad(const DevSphere &S, T cx, T cy, T cz, T px, T py, T pz, T vx, T vy, T vz, T d)
{
    T ix = (px + vx * d) - cx, iy = (py + vy * d) - cy, iz = (pz + vz * d) - cz, rad = (T)(double)S.r;
    T theta = acos(iz / rad);
    T phi = atan2(iy, ix) + (T)PI_SPHERE;
    T uu = phi / (T)(2.0 * PI_SPHERE), vv = theta / (T)PI_SPHERE;
    const T uvmax = (T)(double)0.999999999f;
    uu = fmin(fmax(uu, (T)0.0), uvmax);
    vv = fmin(fmax(vv, (T)0.0), uvmax);
    V3<T> col = {(T)0.5, (T)0.5, (T)0.5};
    if (S.tex.p) col = tex_bilinear<T>(S.tex, uu, vv);
    T shade = fmax((T)0.0, fmin((T)0.5 + (T)0.5 * iz / rad, (T)1.0));
    return {col.x * shade, col.y * shade, col.z * shade};
}

// Orbit camera and scene parameters of the frame, with the parameter
// derivatives seeded (tangent 8 + parameter index).
struct AdjParams {
    double spin, mass, incl, cam_r, phase, sph_R, sph_z;
    int sphere;  // index of the sphere whose phase is differentiated (-1: none)
};

__device__ void initial_state(const FrameParams &fp, const AdjParams &ap, float uvx, float uvy, double y[8], double dy[8][5])
{
    DC a = DC::var(ap.spin, 8 + P_SPIN), M = DC::var(ap.mass, 8 + P_MASS);
    DC inc = DC::var(ap.incl, 8 + P_INCL), r = DC::var(ap.cam_r, 8 + P_CAMR);
    if (fp.metric != PRR_METRIC_KERR) a = DC(0.0);
    if (fp.metric == PRR_METRIC_FLAT) M = DC(0.0);
    DC px = r * sin(inc), py = DC(0.0), pz = r * cos(inc);
    // Camera::rayDir_Spherical with a = pi, b = i - pi/2
    const double PI = 3.14159265358979323846;
    DC beta = inc - DC(0.5 * PI);
    double nu = (0.5 - (double)uvy) * (double)fp.vfov;
    double mu = (0.5 - (double)uvx) * (double)fp.width / (double)fp.height * (double)fp.vfov;
    DC cb = cos(beta + DC(nu));
    DC dx = cb * ::cos(PI + mu), dyv = cb * ::sin(PI + mu), dz = sin(beta + DC(nu));
    DC k = DC(1.0) / sqrt(dx * dx + dyv * dyv + dz * dz);
    dx = dx * k; dyv = dyv * k; dz = dz * k;
    DC g[16];
    metric_ks<DC>(px, py, pz, M, a, g);
    DC A = g[15];
    DC Bq = DC(2.0) * (g[12] * dx + g[13] * dyv + g[14] * dz);
    DC Cq = g[0] * dx * dx + g[5] * dyv * dyv + g[10] * dz * dz + DC(2.0) * (g[1] * dx * dyv + g[2] * dx * dz + g[6] * dyv * dz);
    DC rt = sqrt(Bq * Bq - DC(4.0) * A * Cq);
    DC u0 = fmax((-Bq + rt) / (DC(2.0) * A), (-Bq - rt) / (DC(2.0) * A));
    if (u0 < 0.0) u0 = DC(1.0);
    const DC s[8] = {px, py, pz, DC(0.0), dx, dyv, dz, u0};
    for (int c = 0; c < 8; c++) {
        y[c] = s[c].v;
        for (int p = 0; p < 5; p++) dy[c][p] = s[c].d[8 + p];
    }
}

// Fehlberg coefficients for runtime stage indices: A (stage weights), B = A*A
// (the position stages, phys_stepper.cuh) and c = A*1.
__constant__ double c_A[6][5] = {{0, 0, 0, 0, 0},
                                 {Fehlberg::A21, 0, 0, 0, 0},
                                 {Fehlberg::A31, Fehlberg::A32, 0, 0, 0},
                                 {Fehlberg::A41, Fehlberg::A42, Fehlberg::A43, 0, 0},
                                 {Fehlberg::A51, Fehlberg::A52, Fehlberg::A53, Fehlberg::A54, 0},
                                 {Fehlberg::A61, Fehlberg::A62, Fehlberg::A63, Fehlberg::A64, Fehlberg::A65}};
__constant__ double c_B[6][5] = {{0, 0, 0, 0, 0},
                                 {0, 0, 0, 0, 0},
                                 {Fehlberg::B31, 0, 0, 0, 0},
                                 {Fehlberg::B41, Fehlberg::B42, 0, 0, 0},
                                 {Fehlberg::B51, Fehlberg::B52, Fehlberg::B53, 0, 0},
                                 {Fehlberg::B61, Fehlberg::B62, Fehlberg::B63, Fehlberg::B64, 0}};
__constant__ double c_c[6] = {0.0, Fehlberg::c2, Fehlberg::c3, Fehlberg::c4, Fehlberg::c5, Fehlberg::c6};
__constant__ double c_K4[6] = {Fehlberg::K41, Fehlberg::K42, Fehlberg::K43, Fehlberg::K44, Fehlberg::K45, Fehlberg::K46};
__constant__ double c_beta[6] = {Fehlberg::b1, Fehlberg::b2, Fehlberg::b3, Fehlberg::b4, Fehlberg::b5, 0.0};

// Stage point i of the Fehlberg step from y = (x, u), h and the velocity
// increments ku_0..ku_{i-1} (x' = u is linear in the stages: phys_stepper.cuh):
//   z_i^u = u + sum_m A_im ku_m,  z_i^x = x + h (c_i u + sum_m B_im ku_m).
__device__ __forceinline__ void stage_point(const double y[8], double h, const double ku[6][4], int i, V4<double> &zx,
                                            V4<double> &zu)
{
    double sx[4], su[4];
#pragma unroll
    for (int c = 0; c < 4; c++) { su[c] = y[4 + c]; sx[c] = c_c[i] * y[4 + c]; }
    for (int m = 0; m < i; m++)
#pragma unroll
        for (int c = 0; c < 4; c++) { su[c] += c_A[i][m] * ku[m][c]; sx[c] += c_B[i][m] * ku[m][c]; }
    zx = {y[0] + h * sx[0], y[1] + h * sx[1], y[2] + h * sx[2], y[3] + h * sx[3]};
    zu = {su[0], su[1], su[2], su[3]};
}

// The geodesic's reverse sweep, one copy in the kernel (called at every stage).
__device__ __noinline__ void geod_vjp_call(const V4<double> &zx, const V4<double> &zu, double M, double a,
                                           const double w[4], double gx[4], double gu[4], double &gM, double &ga)
{
    geod_vjp(zx, zu, M, a, w, gx, gu, gM, ga);
}

// lambda <- lambda . dPhi/dy at (y, h), Phi the 4th-order Fehlberg step
//   u+ = u + sum_m K4_m ku_m,  x+ = x + h (u + sum_m beta_m ku_m);
// th[0..1] += lambda . dPhi/d(spin, mass).  Only the six velocity increments
// ku (24 doubles) and their adjoints (24 doubles) are kept; the stage points
// are rebuilt from them.
__device__ void step_vjp(const Hot<double> &q, const double y[8], double h, double lam[8], double th[2])
{
    if (q.metric == PRR_METRIC_FLAT) {  // G = 0: x+ = x + h u
#pragma unroll
        for (int c = 0; c < 4; c++) lam[4 + c] += h * lam[c];
        return;
    }
    double ku[6][4];
#pragma unroll 1
    for (int i = 0; i < 6; i++) {
        V4<double> zx, zu;
        stage_point(y, h, ku, i, zx, zu);
        const V4<double> g = geod_ks<double, true>(zx, zu, q.M, q.a);
        ku[i][0] = h * g.x; ku[i][1] = h * g.y; ku[i][2] = h * g.z; ku[i][3] = h * g.w;
    }
    // adjoints of the outputs: of ku_m, and of (x, u) through the direct terms
    double kb[6][4], ox[4], ou[4];
#pragma unroll
    for (int c = 0; c < 4; c++) {
        ox[c] = lam[c];
        ou[c] = lam[4 + c] + h * lam[c];
#pragma unroll
        for (int m = 0; m < 6; m++) kb[m][c] = c_K4[m] * lam[4 + c] + h * c_beta[m] * lam[c];
    }
#pragma unroll 1
    for (int i = 5; i >= 0; i--) {
        V4<double> zx, zu;
        stage_point(y, h, ku, i, zx, zu);
        double gx[4], gu[4], gM, ga;
        const double wv[4] = {kb[i][0], kb[i][1], kb[i][2], kb[i][3]};
        geod_vjp_call(zx, zu, q.M, q.a, wv, gx, gu, gM, ga);
        th[0] += h * ga;
        th[1] += h * gM;
        double zbx[4], zbu[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            zbx[c] = h * gx[c];
            zbu[c] = h * gu[c];
            ox[c] += zbx[c];
            ou[c] += zbu[c] + h * c_c[i] * zbx[c];
        }
        for (int m = 0; m < i; m++)
#pragma unroll
            for (int c = 0; c < 4; c++) kb[m][c] += c_A[i][m] * zbu[c] + h * c_B[i][m] * zbx[c];
    }
#pragma unroll
    for (int c = 0; c < 4; c++) { lam[c] = ox[c]; lam[4 + c] = ou[c]; }
}

struct AdjointArgs {
    const FrameParams *frame;  // device, one frame
    AdjParams ap;
    const float *dL_dimage;    // W*H*3 (device)
    const float *image;        // forward combined image W*H*3 (device)
    void *ckpt;                // per thread: max_ckpt checkpoints (PhysRay<TF>)
    int max_ckpt;
    double *grad;              // 5 doubles, accumulated
    unsigned long long *counters;
    long long nrays;
    const unsigned *order;     // ray visit order (null: 0, 1, 2, ...)
};

constexpr int ADJ_K = 64;    // accepted steps between checkpoints (HBM)
constexpr int ADJ_SUB = 16;  // accepted steps between sub-checkpoints of the reverse sweep (per thread)
static_assert(ADJ_K % ADJ_SUB == 0, "sub-segments tile a segment");

// At least PRR_ADJ_MINB resident CTAs of 128 threads per SM (caps registers).
#ifndef PRR_ADJ_MINB
#define PRR_ADJ_MINB 1
#endif

template <class TF> __device__ __forceinline__ void state8(const PhysRay<TF> &R, double y[8])
{
    y[0] = (double)R.x.x; y[1] = (double)R.x.y; y[2] = (double)R.x.z; y[3] = (double)R.x.w;
    y[4] = (double)R.u.x; y[5] = (double)R.u.y; y[6] = (double)R.u.z; y[7] = (double)R.u.w;
}

// One RKF45 attempt of the adjoint's own forward steps.  The forward pass and
// both recompute passes go through this one out-of-line copy, so a recomputed
// segment repeats the forward steps bit for bit: inlined copies of the same
// source may contract multiply-adds differently, and a recomputed step
// sequence that drifts from the forward one would pull lambda back through
// steps that were never taken.
template <class TF>
__device__ __noinline__ int adj_attempt(const FrameParams &fp, const Hot<TF> &q, PhysRay<TF> &R, int &result,
                                        V3<float> &col, int &hit)
{
    return phys_attempt<TF, 0>(fp, q, R, result, col, (TF)-1, &hit);
}

template <class TF> __global__ void __launch_bounds__(128, PRR_ADJ_MINB) k_adjoint(AdjointArgs A)
{
    const FrameParams &fp = *A.frame;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nth = (long long)gridDim.x * blockDim.x;
    PhysRay<TF> *ck = (PhysRay<TF> *)A.ckpt + tid * A.max_ckpt;
    Hot<TF> qf = make_hot<TF>(fp);
    qf.a = fp.metric == PRR_METRIC_KERR ? (TF)A.ap.spin : (TF)0;
    qf.M = fp.metric == PRR_METRIC_FLAT ? (TF)0 : (TF)A.ap.mass;
    Hot<double> q = make_hot<double>(fp);  // the adjoint's (FP64) copy
    q.a = fp.metric == PRR_METRIC_KERR ? A.ap.spin : 0.0;
    q.M = fp.metric == PRR_METRIC_FLAT ? 0.0 : A.ap.mass;
    double gacc[5] = {0, 0, 0, 0, 0};
    unsigned long long n_bad = 0, n_steps = 0;
    const int S = fp.samples;
    TF ystore[ADJ_SUB][8], hstore[ADJ_SUB];
    PhysRay<TF> sub[ADJ_K / ADJ_SUB];
    for (long long k = tid; k < A.nrays; k += nth) {
        const long long rid = A.order ? (long long)A.order[k] : k;
        long long pix = rid / S;
        int s = (int)(rid - pix * S);
        int px = (int)(pix % fp.width), py = (int)(pix / fp.width);
        // dL/dc through the SSAA combine (kernels/ssaa.cuh:116-130)
        float uvx, uvy;
        ray_uv(fp, px, py, s, uvx, uvy);
        double y0[8], dy0[8][5];
        initial_state(fp, A.ap, uvx, uvy, y0, dy0);
        PhysRay<TF> R;
        R.x = {(TF)y0[0], (TF)y0[1], (TF)y0[2], (TF)y0[3]};
        R.u = {(TF)y0[4], (TF)y0[5], (TF)y0[6], (TF)y0[7]};
        R.cx = {0, 0, 0, 0}; R.cu = {0, 0, 0, 0};
        R.h = (TF)fp.h; R.trace_h = (TF)fp.h; R.l = 0; R.i = 0; R.accepted = 0; R.intersect = 0;
        ck[0] = R;
        int result = 0, hit = -1;
        V3<float> col;
        bool ok = true;
        while (true) {
            int before = R.accepted;
            int st = adj_attempt<TF>(fp, qf, R, result, col, hit);
            if (st == STEP_CONTINUE && R.accepted > before && R.accepted % ADJ_K == 0) {
                int slot = R.accepted / ADJ_K;
                if (slot >= A.max_ckpt) { ok = false; break; }
                ck[slot] = R;
            }
            if (st != STEP_CONTINUE) break;
        }
        if (!ok) { n_bad++; continue; }
        const int N = R.accepted;
        n_steps += (unsigned long long)N;
        bool escaped = result == PRR_RESULT_SUCCESS && metric_radius<TF>(fp, R.x.x, R.x.y, R.x.z) >= (TF)fp.rout;
        if (!(escaped || result == PRR_RESULT_INTERSECTION)) continue;  // black: no gradient
        // dL/dc for this sample
        const float *gI = A.dL_dimage + 3 * pix;
        const float *I = A.image + 3 * pix;
        double gc[3];
        const float cc[3] = {col.x, col.y, col.z};
        bool any = false;
        for (int c = 0; c < 3; c++) {
            double d;
            if (S == 1) d = (cc[c] > 0.0f && cc[c] < 1.0f) ? 1.0 : 0.0;
            else d = (cc[c] * cc[c] > 0.0f && cc[c] * cc[c] < 1.0f && I[c] > 0.0f) ? (double)cc[c] / ((double)S * I[c]) : 0.0;
            gc[c] = (double)gI[c] * d;
            any |= gc[c] != 0.0;
        }
        if (!any) continue;
        // lambda_N = gc . dc/dy_N ; direct phase term
        double lam[8] = {0, 0, 0, 0, 0, 0, 0, 0}, th[2] = {0, 0}, phase_c = 0.0;
        {
            DC st[8];
            double yN[8];
            state8(R, yN);
            for (int c = 0; c < 8; c++) st[c] = DC::var(yN[c], c);
            V3<DC> cd;
            if (escaped) {
                cd = background_bilinear<DC>(fp.bg, st[4], st[5], st[6]);
                if (!fp.bg.p || fp.bg_filter != PRR_BG_BILINEAR) cd = {DC(0.0), DC(0.0), DC(0.0)};  // RMS2X2 is piecewise constant
            } else {
                const DevSphere &Sp = fp.sph[hit];
                DC cx = DC((double)Sp.cx), cy = DC((double)Sp.cy), cz = DC((double)Sp.cz);
                if (hit == A.ap.sphere) {
                    DC ph = DC::var(A.ap.phase, 8 + P_PHASE);
                    cx = DC(A.ap.sph_R) * cos(ph); cy = DC(A.ap.sph_R) * sin(ph); cz = DC(A.ap.sph_z);
                }
                DC k = DC(1.0) / sqrt(st[4] * st[4] + st[5] * st[5] + st[6] * st[6]);
                DC vx = st[4] * k, vy = st[5] * k, vz = st[6] * k;
                DC v2 = vx * vx + vy * vy + vz * vz;
                DC dx = st[0] - cx, dy = st[1] - cy, dz = st[2] - cz;
                DC dvp = vx * dx + vy * dy + vz * dz;
                DC disc = dvp * dvp - v2 * ((dx * dx + dy * dy + dz * dz) - DC((double)Sp.r * (double)Sp.r));
                DC d = (DC(-2.0) * dvp - sqrt(disc)) / v2;
                cd = sphere_colour_ad<DC>(Sp, cx, cy, cz, st[0], st[1], st[2], vx, vy, vz, d);
            }
            const DC *cc3 = &cd.x;
            for (int c = 0; c < 3; c++) {
                for (int j = 0; j < 8; j++) lam[j] += gc[c] * cc3[c].d[j];
                phase_c += gc[c] * cc3[c].d[8 + P_PHASE];
            }
        }
        // reverse sweep, segment by segment, each in two recompute passes.  A
        // recomputation that does not reach the steps the forward pass took
        // (it cannot, as both run the same code, but it is checked rather than
        // trusted) drops the ray: its states would be missing.
        int r2 = 0, h2 = -1;
        V3<float> c2;
        bool consistent = true;
        for (int seg = (N - 1) / ADJ_K; seg >= 0 && N > 0 && consistent; seg--) {
            const int lo = seg * ADJ_K, hi = min(N, lo + ADJ_K);
            const int nsub = (hi - lo + ADJ_SUB - 1) / ADJ_SUB;
            // pass 1: the segment's sub-checkpoints
            PhysRay<TF> Rs = ck[seg];
            sub[0] = Rs;
            while (Rs.accepted < lo + (nsub - 1) * ADJ_SUB) {
                int st = adj_attempt<TF>(fp, qf, Rs, r2, c2, h2);
                const int j = (Rs.accepted - lo) / ADJ_SUB;
                if ((Rs.accepted - lo) % ADJ_SUB == 0 && j < nsub) sub[j] = Rs;
                if (st != STEP_CONTINUE) break;
            }
            if (Rs.accepted < lo + (nsub - 1) * ADJ_SUB) { consistent = false; break; }
            // pass 2: each sub-segment, last first: keep its states, then pull lambda back
            for (int j = nsub - 1; j >= 0; j--) {
                Rs = sub[j];
                const int slo = lo + j * ADJ_SUB, shi = min(hi, slo + ADJ_SUB);
                while (Rs.accepted < shi) {
                    const int before = Rs.accepted;
                    TF yb[8] = {Rs.x.x, Rs.x.y, Rs.x.z, Rs.x.w, Rs.u.x, Rs.u.y, Rs.u.z, Rs.u.w};
                    const TF hb = Rs.h;
                    int st = adj_attempt<TF>(fp, qf, Rs, r2, c2, h2);
                    if (Rs.accepted > before) {
                        const int slot = before - slo;
                        for (int c = 0; c < 8; c++) ystore[slot][c] = yb[c];
                        hstore[slot] = hb;
                    }
                    if (st != STEP_CONTINUE) break;
                }
                if (Rs.accepted != shi) { consistent = false; break; }
                for (int n = shi - 1; n >= slo; n--) {
                    double y[8];
                    for (int c = 0; c < 8; c++) y[c] = (double)ystore[n - slo][c];
                    step_vjp(q, y, (double)hstore[n - slo], lam, th);
                }
            }
        }
        if (!consistent) { n_bad++; continue; }
        gacc[P_PHASE] += phase_c;
        gacc[P_SPIN] += th[0];
        gacc[P_MASS] += th[1];
        for (int c = 0; c < 8; c++)
            for (int p = 0; p < 5; p++) gacc[p] += lam[c] * dy0[c][p];
    }
    for (int p = 0; p < 5; p++) {
        double v = gacc[p];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&A.grad[p], v);
    }
    if (A.counters) {
        if (n_bad) atomicAdd(&A.counters[C_MATH_ERROR], n_bad);
        atomicAdd(&A.counters[C_ACCEPTED], n_steps);
    }
}

cudaError_t launch_adjoint(const FrameParams *d_fp, const AdjointParamsHost &p, const float *dL, const float *image,
                           void *ckpt, int max_ckpt, int threads_total, double *grad, unsigned long long *counters,
                           long long nrays, const unsigned *order, int precision, cudaStream_t st)
{
    AdjointArgs A;
    A.frame = d_fp;
    A.ap = {p.spin, p.mass, p.incl, p.cam_r, p.phase, p.sph_R, p.sph_z, p.sphere};
    A.dL_dimage = dL;
    A.image = image;
    A.ckpt = ckpt;
    A.max_ckpt = max_ckpt;
    A.grad = grad;
    A.counters = counters;
    A.nrays = nrays;
    A.order = order;
    if (precision == PRR_PREC_FP32) k_adjoint<float><<<threads_total / 128, 128, 0, st>>>(A);
    else k_adjoint<double><<<threads_total / 128, 128, 0, st>>>(A);
    return cudaGetLastError();
}

__global__ void k_iota(unsigned *v, long long n)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = (unsigned)i;
}

// scratch layout: [iota values | sorted keys | cub temporary storage]
size_t adjoint_order_bytes(long long nrays)
{
    size_t temp = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, temp, (const int *)nullptr, (int *)nullptr,
                                              (const unsigned *)nullptr, (unsigned *)nullptr, (int)nrays);
    const size_t n4 = ((size_t)nrays * 4 + 255) / 256 * 256;
    return 2 * n4 + temp + 256;
}

cudaError_t launch_adjoint_order(const int *steps, long long nrays, unsigned *order, void *scratch, cudaStream_t st)
{
    if (nrays <= 0) return cudaSuccess;
    const size_t n4 = ((size_t)nrays * 4 + 255) / 256 * 256;
    unsigned *iota = (unsigned *)scratch;
    int *keys_out = (int *)((char *)scratch + n4);
    void *temp = (char *)scratch + 2 * n4;
    k_iota<<<(unsigned)((nrays + 255) / 256), 256, 0, st>>>(iota, nrays);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    size_t temp_bytes = 0;
    e = cub::DeviceRadixSort::SortPairsDescending(nullptr, temp_bytes, steps, keys_out, iota, order, (int)nrays);
    if (e != cudaSuccess) return e;
    return cub::DeviceRadixSort::SortPairsDescending(temp, temp_bytes, steps, keys_out, iota, order, (int)nrays, 0,
                                                     32, st);
}

size_t adjoint_checkpoint_bytes(int precision)
{
    return precision == PRR_PREC_FP32 ? sizeof(PhysRay<float>) : sizeof(PhysRay<double>);
}

int adjoint_blocks_per_sm(int precision)
{
    int n = 0;
    cudaError_t e = precision == PRR_PREC_FP32 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_adjoint<float>, 128, 0)
                                               : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_adjoint<double>, 128, 0);
    if (e != cudaSuccess) { cudaGetLastError(); return 1; }
    return n > 0 ? n : 1;
}

}  // namespace prr
