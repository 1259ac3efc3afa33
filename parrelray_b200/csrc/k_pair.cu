// k_pair.cu - the FP32 persistent renderer with RPT rays in flight per
// thread (RPT = 1 or 2).  Same scheduling as k_persistent.cu (persistent
// CTAs, warp-aggregated refill from one work counter over all frames, SSAA
// combine in registers), but each lane owns RPT pixel slots, and the RKF45
// stages of its slots are evaluated together (phys_pair.cuh: with RPT = 2 the
// two rays share paired FP32 instructions).  Accept/reject, the hooks and the
// colouring run per slot.  Both forms spell out the same operations; the
// paired instructions may round subnormal intermediates differently, so a
// ray's result can differ between RPT = 1 and 2 in the last bits (it never
// depends on the block shape or the refill interval).
//
// SPLIT (RPT = 1 only): the FP32 pass of a split-precision render.
// Per-sample colours go to sample_rgb (the per-pixel combine runs after the
// FP64 pass), and rays near a photon orbit (near_critical, tested before
// the first attempt) or that dip below fp64_rfac * r_+ are queued for
// k_fp64_requeue (k_persistent.cu).
//
// EMIS (RPT = 1, not SPLIT): plasma emission (emission.cuh) accumulated at
// every accepted step of frames that have it, composited into the colour.
#include <type_traits>

#include "kernels.cuh"
#include "phys_pair.cuh"

namespace prr {

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ int find_frame2(const long long *begin, int n, long long item)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(begin + mid) <= item) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void warp_sum_add(unsigned long long *p, unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(p, v);
}

__device__ __forceinline__ uint8_t q8(float v) { return (uint8_t)roundf(255.0f * fminf(fmaxf(v, 0.0f), 1.0f)); }

struct Slot {
    int frame, px, py, s, S;
    float acc0, acc1, acc2;
    bool busy, need;
    float flag_r;  // split precision: queue the ray for FP64 below this radius
    PhysRay<float> R;
    Hot<float> q;
    EmisRay<float> E;  // emission kernels only
};

struct Counts {
    unsigned long long att = 0, acc = 0, rays = 0, esc = 0, cap = 0, hit = 0, inf = 0, nan = 0, f64 = 0;
};

// Split precision: the next sample of slot `sl`, or true when its pixel is
// complete (the pixel itself is written by the combine after the FP64 pass).
__device__ __forceinline__ bool next_sample_split(const FrameParams &fp, Slot &sl)
{
    sl.s += 1;
    if (sl.s < sl.S) {
        phys_init<float>(fp, sl.px, sl.py, sl.s, sl.R);
        return false;
    }
    return true;
}

// Split precision: a ray queued for the FP64 pass.  Its colour slot is zeroed
// here and overwritten by k_fp64_requeue; it is counted as a ray there.
__device__ __forceinline__ bool flag_ray(const PersistentArgs &a, Slot &sl, Counts &c)
{
    const FrameParams &fp = a.frames[sl.frame];
    c.att += (unsigned)sl.R.i;
    c.acc += (unsigned)sl.R.accepted;
    c.f64++;
    const long long rid = ((long long)sl.py * fp.width + sl.px) * sl.S + sl.s;
    const unsigned long long slot = atomicAdd(&a.counters[C_FP64_QUEUED], 1ull);
    if ((long long)slot < a.fp64_capacity) a.fp64_queue[slot] = ((unsigned long long)sl.frame << 40) | (unsigned long long)rid;
    float *o = a.sample_rgb + 3 * (fp.ray_begin + rid);
    o[0] = o[1] = o[2] = 0.f;
    return next_sample_split(fp, sl);
}

// A finished ray of slot `sl`: counters, SSAA accumulation, next sample or
// pixel output.  Returns true when the slot's pixel is complete.
template <bool SPLIT, bool EMIS>
__device__ __forceinline__ bool finish_ray(const PersistentArgs &a, Slot &sl, int result, V3<float> col, Counts &c)
{
    const FrameParams &fp = a.frames[sl.frame];
    if constexpr (EMIS) col = emis_colour<float>(fp, sl.E, col);
    c.att += (unsigned)sl.R.i;
    c.acc += (unsigned)sl.R.accepted;
    c.rays++;
    if constexpr (SPLIT) {
        const long long rid = ((long long)sl.py * fp.width + sl.px) * sl.S + sl.s;
        float *o = a.sample_rgb + 3 * (fp.ray_begin + rid);
        o[0] = col.x; o[1] = col.y; o[2] = col.z;
        if (result == PRR_RESULT_SUCCESS) {
            if (col.x + col.y + col.z >= 0.f && metric_radius<float>(fp, sl.R.x.x, sl.R.x.y, sl.R.x.z) >= sl.q.rout) c.esc++;
            else c.cap++;
        } else if (result == PRR_RESULT_INTERSECTION) c.hit++;
        else if (result == PRR_RESULT_INFINITE_GEO) c.inf++;
        else c.nan++;
        return next_sample_split(fp, sl);
    }
    if (a.ray_state || a.sample_rgb) {  // per-ray outputs (single-frame parity runs)
        const long long rid = ((long long)sl.py * fp.width + sl.px) * sl.S + sl.s;
        if (a.ray_state) {
            float uvx, uvy;
            ray_uv(fp, sl.px, sl.py, sl.s, uvx, uvy);
            float *o = a.ray_state + 12 * rid;
            o[0] = uvx; o[1] = uvy; o[2] = (float)result;
            o[3] = sl.R.x.x; o[4] = sl.R.x.y; o[5] = sl.R.x.z; o[6] = sl.R.x.w;
            o[7] = sl.R.u.x; o[8] = sl.R.u.y; o[9] = sl.R.u.z; o[10] = sl.R.u.w;
            o[11] = (float)sl.R.accepted;
        }
        if (a.sample_rgb) {
            float *o = a.sample_rgb + 3 * (fp.ray_begin + rid);
            o[0] = col.x; o[1] = col.y; o[2] = col.z;
        }
    }
    if (result == PRR_RESULT_SUCCESS) {
        if (metric_radius<float>(fp, sl.R.x.x, sl.R.x.y, sl.R.x.z) >= sl.q.rout) c.esc++; else c.cap++;
    } else if (result == PRR_RESULT_INTERSECTION) c.hit++;
    else if (result == PRR_RESULT_INFINITE_GEO) c.inf++;
    else c.nan++;
    if (sl.S == 1) {
        sl.acc0 = fminf(fmaxf(col.x, 0.f), 1.f); sl.acc1 = fminf(fmaxf(col.y, 0.f), 1.f); sl.acc2 = fminf(fmaxf(col.z, 0.f), 1.f);
    } else {
        sl.acc0 += fminf(fmaxf(col.x * col.x, 0.f), 1.f);
        sl.acc1 += fminf(fmaxf(col.y * col.y, 0.f), 1.f);
        sl.acc2 += fminf(fmaxf(col.z * col.z, 0.f), 1.f);
    }
    sl.s += 1;
    if (sl.s < sl.S) {
        phys_init<float>(fp, sl.px, sl.py, sl.s, sl.R);
        if constexpr (EMIS) emis_init<float>(fp, sl.R.x, sl.R.u, sl.E);
        return false;
    }
    float o0 = sl.acc0, o1 = sl.acc1, o2 = sl.acc2;
    if (sl.S > 1) { o0 = sqrtf(o0 / (float)sl.S); o1 = sqrtf(o1 / (float)sl.S); o2 = sqrtf(o2 / (float)sl.S); }
    const long long op = fp.pix_begin + (long long)sl.py * fp.width + sl.px;
    if (a.image) { a.image[3 * op] = o0; a.image[3 * op + 1] = o1; a.image[3 * op + 2] = o2; }
    if (a.rgb8 && !fp.fxaa) { a.rgb8[3 * op] = q8(o0); a.rgb8[3 * op + 1] = q8(o1); a.rgb8[3 * op + 2] = q8(o2); }
    return true;
}

template <bool SPLIT, bool EMIS>
__device__ __forceinline__ void start_pixel(const PersistentArgs &a, Slot &sl, long long it)
{
    sl.frame = find_frame2(a.frame_pix_begin, a.nframes, it);
    const FrameParams &fp = a.frames[sl.frame];
    const long long p = it - __ldg(a.frame_pix_begin + sl.frame);
    sl.px = (int)(p % fp.width);
    sl.py = (int)(p / fp.width);
    sl.S = fp.samples;
    sl.s = 0;
    sl.acc0 = sl.acc1 = sl.acc2 = 0.f;
    sl.q = make_hot<float>(fp);
    sl.flag_r = SPLIT ? fp.fp64_rfac * kerr_r_plus<float>(sl.q.M, sl.q.a) : -1.f;
    phys_init<float>(fp, sl.px, sl.py, 0, sl.R);
    if constexpr (EMIS) emis_init<float>(fp, sl.R.x, sl.R.u, sl.E);
    sl.busy = true;
}

template <class V> __device__ __forceinline__ void load_in(pv::StageIn<V> &in, const Slot *sl);

template <> __device__ __forceinline__ void load_in<float>(pv::StageIn<float> &in, const Slot *sl)
{
    const Slot &A = sl[0];
    in.x = {A.R.x.x, A.R.x.y, A.R.x.z, A.R.x.w};
    in.u = {A.R.u.x, A.R.u.y, A.R.u.z, A.R.u.w};
    in.h = A.R.h; in.M = A.q.M; in.a = A.q.a; in.rtol = A.q.rtol; in.atol = A.q.atol; in.hmin = A.q.hmin; in.hmax = A.q.hmax;
}

template <> __device__ __forceinline__ void load_in<float2>(pv::StageIn<float2> &in, const Slot *sl)
{
    const Slot &A = sl[0], &B = sl[1];
    in.x = {make_float2(A.R.x.x, B.R.x.x), make_float2(A.R.x.y, B.R.x.y), make_float2(A.R.x.z, B.R.x.z), make_float2(A.R.x.w, B.R.x.w)};
    in.u = {make_float2(A.R.u.x, B.R.u.x), make_float2(A.R.u.y, B.R.u.y), make_float2(A.R.u.z, B.R.u.z), make_float2(A.R.u.w, B.R.u.w)};
    in.h = make_float2(A.R.h, B.R.h);
    in.M = make_float2(A.q.M, B.q.M);
    in.a = make_float2(A.q.a, B.q.a);
    in.rtol = make_float2(A.q.rtol, B.q.rtol);
    in.atol = make_float2(A.q.atol, B.q.atol);
    in.hmin = make_float2(A.q.hmin, B.q.hmin);
    in.hmax = make_float2(A.q.hmax, B.q.hmax);
}

}  // namespace

// One-slot threads pair the components of their ray's 4-vectors on the
// paired FP32 instructions (phys_pair.cuh: stages_xy) unless built with
// PRR_PAIR_XY=0.
#ifndef PRR_PAIR_XY
#define PRR_PAIR_XY 1
#endif

// Resident CTAs per SM the small-CTA instantiation is built for (its
// register cap: 65536 / (64 x MINB), rounded down to the allocation unit).
#ifndef PRR_PAIR_SMALL_MINB
#define PRR_PAIR_SMALL_MINB 8
#endif

// Launch bounds (MAXT threads per CTA at most, MINB resident CTAs per SM at
// least) cap the registers per thread.  One-slot threads in CTAs of up to 64
// threads use the instantiation capped at 127 registers (8 CTAs = 16 warps
// per SM, no spills; 4 % faster than 141 registers and 12 warps).
template <int RPT, int MAXT, int MINB, bool SPLIT, bool EMIS>
__global__ void __launch_bounds__(MAXT, MINB) k_pair(PersistentArgs a)
{
    static_assert(!SPLIT || RPT == 1, "split precision runs one ray per thread");
    static_assert(!EMIS || (RPT == 1 && !SPLIT), "emission runs one FP32 ray per thread");
    using V = typename std::conditional<RPT == 2, float2, float>::type;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    Slot sl[RPT];
    Counts cnt;
#pragma unroll
    for (int j = 0; j < RPT; j++) {
        sl[j].busy = false; sl[j].need = true; sl[j].flag_r = -1.f;
        sl[j].frame = 0; sl[j].px = sl[j].py = sl[j].s = 0; sl[j].S = 1;
        sl[j].acc0 = sl[j].acc1 = sl[j].acc2 = 0.f;
        sl[j].R.x = {30.f, 0.f, 0.f, 0.f}; sl[j].R.u = {-1.f, 0.f, 0.f, 1.f};
        sl[j].R.cx = {0.f, 0.f, 0.f, 0.f}; sl[j].R.cu = {0.f, 0.f, 0.f, 0.f};
        sl[j].R.h = sl[j].R.trace_h = 0.01f; sl[j].R.l = 0.f; sl[j].R.i = sl[j].R.accepted = sl[j].R.intersect = 0;
        sl[j].q = Hot<float>{1.f, 0.f, 1e-4f, 0.1f, 1e-6f, 1e-6f, 100.f, 2.f, PRR_METRIC_SCHWARZSCHILD, 1, 0};
    }
    const long long t0 = clock64();
    unsigned iter = 0;
    const unsigned ci = a.compaction_interval > 1 ? (unsigned)a.compaction_interval : 1u;
    unsigned since = ci;
    while (true) {
        // ---- warp-aggregated refill of the slots whose pixel is complete ----
        bool anybusy = false;
#pragma unroll
        for (int j = 0; j < RPT; j++) anybusy |= sl[j].busy;
        if (++since >= ci || __ballot_sync(FULL, anybusy) == 0) {
            since = 0;
            unsigned m[RPT];
            unsigned total = 0;
#pragma unroll
            for (int j = 0; j < RPT; j++) { m[j] = __ballot_sync(FULL, sl[j].need); total += __popc(m[j]); }
            if (total) {
                const int leader = __ffs(m[0] | (RPT == 2 ? m[RPT - 1] : 0u)) - 1;
                unsigned long long base = 0;
                if (lane == leader) base = atomicAdd(&a.counters[C_WORK], (unsigned long long)total);
                base = __shfl_sync(FULL, base, leader);
                unsigned off = 0;
#pragma unroll
                for (int j = 0; j < RPT; j++) {
                    if (sl[j].need) {
                        const long long it = (long long)base + off + __popc(m[j] & lt);
                        sl[j].need = false;
                        if (it < a.total_pixels) start_pixel<SPLIT, EMIS>(a, sl[j], it);
                        else sl[j].busy = false;
                    }
                    off += __popc(m[j]);
                }
            }
        }
        anybusy = false;
        bool anyneed = false;
#pragma unroll
        for (int j = 0; j < RPT; j++) { anybusy |= sl[j].busy; anyneed |= sl[j].need; }
        if (__ballot_sync(FULL, anybusy) == 0) {
            if (__ballot_sync(FULL, anyneed) == 0) break;  // the queue is exhausted for every slot
            since = ci;
            continue;
        }
        if (a.watchdog_cycles > 0 && ((++iter) & 255u) == 0) {
            unsigned stop = 0;
            if (lane == 0) {
                if (clock64() - t0 > a.watchdog_cycles) atomicExch((unsigned long long *)&a.counters[C_TIMEOUT], 1ull);
                stop = (unsigned)*(volatile unsigned long long *)&a.counters[C_TIMEOUT];
            }
            if (__shfl_sync(FULL, stop, 0)) break;
        }
        if (!anybusy) continue;

        // ---- caps before the attempt (per slot) ----
        bool go[RPT];
#pragma unroll
        for (int j = 0; j < RPT; j++) {
            go[j] = false;
            if (!sl[j].busy) continue;
            int result = 0;
            V3<float> col;
            if (SPLIT && sl[j].R.i == 0 && near_critical<float>(a.frames[sl[j].frame], sl[j].R)) {
                if (flag_ray(a, sl[j], cnt)) { sl[j].busy = false; sl[j].need = true; }
            } else if (phys_precheck<float>(sl[j].R, result, col) == STEP_DONE) {
                if (finish_ray<SPLIT, EMIS>(a, sl[j], result, col, cnt)) { sl[j].busy = false; sl[j].need = true; }
            } else {
                go[j] = true;
            }
        }
        bool anygo = false;
#pragma unroll
        for (int j = 0; j < RPT; j++) anygo |= go[j];
        if (!anygo) continue;

        // ---- stages of every slot at once ----
        pv::StageIn<V> in;
        load_in<V>(in, sl);
#if PRR_PAIR_XY
        pv::StageOut<V> out;
        if constexpr (RPT == 1) out = pv::stages_xy(in);
        else out = pv::stages<V>(in);
#else
        const pv::StageOut<V> out = pv::stages<V>(in);
#endif

        // ---- accept/reject, hooks, colour (per slot) ----
#pragma unroll
        for (int j = 0; j < RPT; j++) {
            if (!go[j]) continue;
            const FrameParams &fp = a.frames[sl[j].frame];
            float dxv[4] = {pv::get(out.dx[0], j), pv::get(out.dx[1], j), pv::get(out.dx[2], j), pv::get(out.dx[3], j)};
            float duv[4] = {pv::get(out.du[0], j), pv::get(out.du[1], j), pv::get(out.du[2], j), pv::get(out.du[3], j)};
            int result = 0;
            V3<float> col;
            const int st = phys_accept<float>(fp, sl[j].q, sl[j].R, dxv, duv, pv::get(out.err, j), pv::get(out.hn, j),
                                              result, col, SPLIT ? sl[j].flag_r : -1.0f, nullptr, EMIS ? &sl[j].E : nullptr);
            if (st == STEP_CONTINUE) continue;
            const bool done = (SPLIT && st == STEP_FLAG64) ? flag_ray(a, sl[j], cnt) : finish_ray<SPLIT, EMIS>(a, sl[j], result, col, cnt);
            if (done) { sl[j].busy = false; sl[j].need = true; }
        }
    }
    warp_sum_add(&a.counters[C_ATTEMPTS], cnt.att);
    warp_sum_add(&a.counters[C_ACCEPTED], cnt.acc);
    warp_sum_add(&a.counters[C_RAYS], cnt.rays);
    warp_sum_add(&a.counters[C_ESCAPED], cnt.esc);
    warp_sum_add(&a.counters[C_CAPTURED], cnt.cap);
    warp_sum_add(&a.counters[C_INTERSECTION], cnt.hit);
    warp_sum_add(&a.counters[C_INFINITE], cnt.inf);
    warp_sum_add(&a.counters[C_MATH_ERROR], cnt.nan);
    if (SPLIT) warp_sum_add(&a.counters[C_FP64], cnt.f64);
}

cudaError_t launch_pair(const PersistentArgs &a, int rpt, bool split, int block, int blocks_per_sm, int nsm, cudaStream_t st)
{
    if (block < 32 || block > 256 || block % 32) return cudaErrorInvalidValue;
    if (split && (rpt != 1 || !a.sample_rgb || !a.fp64_queue)) return cudaErrorInvalidValue;
    if (a.emission && split) return cudaErrorInvalidValue;
    int grid = nsm * blocks_per_sm;
    if (grid < 1) grid = 1;
    const bool small = block <= 64;
    if (a.emission) {
        if (small) k_pair<1, 64, PRR_PAIR_SMALL_MINB, false, true><<<grid, block, 0, st>>>(a);
        else k_pair<1, 256, 1, false, true><<<grid, block, 0, st>>>(a);
    } else if (split) {
        if (small) k_pair<1, 64, PRR_PAIR_SMALL_MINB, true, false><<<grid, block, 0, st>>>(a);
        else k_pair<1, 256, 1, true, false><<<grid, block, 0, st>>>(a);
    } else if (rpt == 2) {
        k_pair<2, 256, 1, false, false><<<grid, block, 0, st>>>(a);
    } else if (rpt == 1) {
        if (small) k_pair<1, 64, PRR_PAIR_SMALL_MINB, false, false><<<grid, block, 0, st>>>(a);
        else k_pair<1, 256, 1, false, false><<<grid, block, 0, st>>>(a);
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

int pair_occupancy(int rpt, bool split, int block, bool emission)
{
    int n = 0;
    const bool small = block <= 64;
    cudaError_t e;
    if (emission) e = small ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_pair<1, 64, PRR_PAIR_SMALL_MINB, false, true>, block, 0)
                            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_pair<1, 256, 1, false, true>, block, 0);
    else if (split) e = small ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_pair<1, 64, PRR_PAIR_SMALL_MINB, true, false>, block, 0)
                              : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_pair<1, 256, 1, true, false>, block, 0);
    else if (rpt == 2) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_pair<2, 256, 1, false, false>, block, 0);
    else e = small ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_pair<1, 64, PRR_PAIR_SMALL_MINB, false, false>, block, 0)
                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_pair<1, 256, 1, false, false>, block, 0);
    if (e != cudaSuccess) { cudaGetLastError(); return 0; }
    return n;
}

}  // namespace prr
