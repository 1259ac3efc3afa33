// k_adjoint.cu - discrete adjoint of the PHYSICAL-mode RKF45 render:
// d(loss)/d(spin a, mass M, camera inclination i, camera distance r, orbital
// phase of one sphere) given dL/d(image).
//
// Per ray, FP64, with the accepted step sizes and every discrete event
// (accept/reject, intersection mode, termination, which sphere is hit)
// frozen at the forward run:
//   1. forward: the PHYSICAL stepper runs the ray and saves its full state
//      every ADJ_K accepted steps (checkpoints in HBM, per thread);
//   2. colour adjoint: dL/dc of the ray's sample through the SSAA combine,
//      then lambda_N = dL/dc . dc/dy_N (+ the sphere-phase term) with c the
//      bilinear sky or the sphere texture at the hit point;
//   3. reverse: for each segment, last first, the ADJ_K steps are recomputed
//      from the checkpoint (bit-identical: same stepper) and lambda is pulled
//      back through each step y_{n+1} = y_n + sum_i b_i k_i, k_i = h f(z_i),
//      z_i = y_n + sum_j a_ij k_j (Fehlberg, 4th order); the products
//      lambda^T dG/dz of the geodesic acceleration come from its hand-written
//      reverse sweep (geod_vjp.cuh);
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

// exact Fehlberg tableau and 4th-order weights
__constant__ double c_rkA[6][6] = {
    {0, 0, 0, 0, 0, 0},
    {1.0 / 4.0, 0, 0, 0, 0, 0},
    {3.0 / 32.0, 9.0 / 32.0, 0, 0, 0, 0},
    {1932.0 / 2197.0, -7200.0 / 2197.0, 7296.0 / 2197.0, 0, 0, 0},
    {439.0 / 216.0, -8.0, 3680.0 / 513.0, -845.0 / 4104.0, 0, 0},
    {-8.0 / 27.0, 2.0, -3544.0 / 2565.0, 1859.0 / 4104.0, -11.0 / 40.0, 0}};
__constant__ double c_rkB[6] = {25.0 / 216.0, 0.0, 1408.0 / 2565.0, 2197.0 / 4104.0, -1.0 / 5.0, 0.0};

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

__device__ void geod_val(const Hot<double> &q, const double z[8], double G[4])
{
    if (q.metric == PRR_METRIC_FLAT) { G[0] = G[1] = G[2] = G[3] = 0.0; return; }
    V4<double> g = geod_ks<double, true>({z[0], z[1], z[2], z[3]}, {z[4], z[5], z[6], z[7]}, q.M, q.a);
    G[0] = g.x; G[1] = g.y; G[2] = g.z; G[3] = g.w;
}

// lambda <- lambda . dPhi/dy at (y, h); th[0..1] += lambda . dPhi/d(spin, mass)
__device__ void step_vjp(const Hot<double> &q, const double y[8], double h, double lam[8], double th[2])
{
    double z[6][8], k[6][8];
    for (int i = 0; i < 6; i++) {
        for (int c = 0; c < 8; c++) {
            double s = y[c];
            for (int j = 0; j < i; j++) s += c_rkA[i][j] * k[j][c];
            z[i][c] = s;
        }
        double G[4];
        geod_val(q, z[i], G);
        for (int c = 0; c < 4; c++) { k[i][c] = h * z[i][4 + c]; k[i][4 + c] = h * G[c]; }
    }
    double kb[6][8], yb[8];
    for (int c = 0; c < 8; c++) yb[c] = lam[c];
    for (int i = 0; i < 6; i++)
        for (int c = 0; c < 8; c++) kb[i][c] = c_rkB[i] * lam[c];
    for (int i = 5; i >= 0; i--) {
        double zb[8];
        // k_i = h (z_u, G(z)):  zb = h (d f/dz)^T kb_i, by the reverse sweep of the geodesic
        if (q.metric == PRR_METRIC_FLAT) {
            for (int c = 0; c < 8; c++) zb[c] = 0.0;
        } else {
            double gx[4], gu[4], gM, ga;
            const double wv[4] = {kb[i][4], kb[i][5], kb[i][6], kb[i][7]};
            geod_vjp({z[i][0], z[i][1], z[i][2], z[i][3]}, {z[i][4], z[i][5], z[i][6], z[i][7]}, q.M, q.a, wv, gx, gu, gM, ga);
            for (int c = 0; c < 4; c++) { zb[c] = h * gx[c]; zb[4 + c] = h * gu[c]; }
            th[0] += h * ga;
            th[1] += h * gM;
        }
        for (int c = 0; c < 4; c++) zb[4 + c] += h * kb[i][c];
        for (int c = 0; c < 8; c++) yb[c] += zb[c];
        for (int j = 0; j < i; j++)
            for (int c = 0; c < 8; c++) kb[j][c] += c_rkA[i][j] * zb[c];
    }
    for (int c = 0; c < 8; c++) lam[c] = yb[c];
}

struct AdjointArgs {
    const FrameParams *frame;  // device, one frame
    AdjParams ap;
    const float *dL_dimage;    // W*H*3 (device)
    const float *image;        // forward combined image W*H*3 (device)
    PhysRay<double> *ckpt;     // per thread: max_ckpt checkpoints
    int max_ckpt;
    double *grad;              // 5 doubles, accumulated
    unsigned long long *counters;
    long long nrays;
    const unsigned *order;     // ray visit order (null: 0, 1, 2, ...)
};

constexpr int ADJ_K = 64;

// At least PRR_ADJ_MINB resident CTAs of 128 threads per SM (caps registers).
#ifndef PRR_ADJ_MINB
#define PRR_ADJ_MINB 1
#endif

__global__ void __launch_bounds__(128, PRR_ADJ_MINB) k_adjoint(AdjointArgs A)
{
    const FrameParams &fp = *A.frame;
    const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nth = (long long)gridDim.x * blockDim.x;
    PhysRay<double> *ck = A.ckpt + tid * A.max_ckpt;
    Hot<double> q = make_hot<double>(fp);
    q.a = fp.metric == PRR_METRIC_KERR ? A.ap.spin : 0.0;
    q.M = fp.metric == PRR_METRIC_FLAT ? 0.0 : A.ap.mass;
    double gacc[5] = {0, 0, 0, 0, 0};
    unsigned long long n_bad = 0, n_steps = 0;
    const int S = fp.samples;
    double ystore[ADJ_K][8], hstore[ADJ_K];
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
        PhysRay<double> R;
        R.x = {y0[0], y0[1], y0[2], y0[3]};
        R.u = {y0[4], y0[5], y0[6], y0[7]};
        R.cx = {0, 0, 0, 0}; R.cu = {0, 0, 0, 0};
        R.h = fp.h; R.trace_h = fp.h; R.l = 0; R.i = 0; R.accepted = 0; R.intersect = 0;
        ck[0] = R;
        int result = 0, hit = -1;
        V3<float> col;
        bool ok = true;
        while (true) {
            int before = R.accepted;
            int st = phys_attempt<double, 0>(fp, q, R, result, col, -1.0, &hit);
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
        bool escaped = result == PRR_RESULT_SUCCESS && metric_radius<double>(fp, R.x.x, R.x.y, R.x.z) >= (double)fp.rout;
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
        double lam[8] = {0, 0, 0, 0, 0, 0, 0, 0}, th[2] = {0, 0};
        {
            DC st[8];
            const double yN[8] = {R.x.x, R.x.y, R.x.z, R.x.w, R.u.x, R.u.y, R.u.z, R.u.w};
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
                gacc[P_PHASE] += gc[c] * cc3[c].d[8 + P_PHASE];
            }
        }
        // reverse sweep, segment by segment
        for (int seg = (N - 1) / ADJ_K; seg >= 0 && N > 0; seg--) {
            PhysRay<double> Rs = ck[seg];
            const int lo = seg * ADJ_K, hi = min(N, lo + ADJ_K);
            int r2 = 0, h2 = -1;
            V3<float> c2;
            while (Rs.accepted < hi) {
                int before = Rs.accepted;
                double yb[8] = {Rs.x.x, Rs.x.y, Rs.x.z, Rs.x.w, Rs.u.x, Rs.u.y, Rs.u.z, Rs.u.w};
                double hb = Rs.h;
                int st = phys_attempt<double, 0>(fp, q, Rs, r2, c2, -1.0, &h2);
                if (Rs.accepted > before) {
                    int slot = before - lo;
                    for (int c = 0; c < 8; c++) ystore[slot][c] = yb[c];
                    hstore[slot] = hb;
                }
                if (st != STEP_CONTINUE) break;
            }
            for (int n = hi - 1; n >= lo; n--) step_vjp(q, ystore[n - lo], hstore[n - lo], lam, th);
        }
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
                           long long nrays, const unsigned *order, cudaStream_t st)
{
    AdjointArgs A;
    A.frame = d_fp;
    A.ap = {p.spin, p.mass, p.incl, p.cam_r, p.phase, p.sph_R, p.sph_z, p.sphere};
    A.dL_dimage = dL;
    A.image = image;
    A.ckpt = (PhysRay<double> *)ckpt;
    A.max_ckpt = max_ckpt;
    A.grad = grad;
    A.counters = counters;
    A.nrays = nrays;
    A.order = order;
    k_adjoint<<<threads_total / 128, 128, 0, st>>>(A);
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

size_t adjoint_checkpoint_bytes() { return sizeof(PhysRay<double>); }

int adjoint_blocks_per_sm()
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_adjoint, 128, 0) != cudaSuccess) { cudaGetLastError(); return 1; }
    return n > 0 ? n : 1;
}

}  // namespace prr
