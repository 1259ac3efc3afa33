// k_persistent.cu - persistent, warp-compacted PHYSICAL-mode renderer.
//
// One CTA per SM slot, launched once for a whole batch of frames.  Each lane
// owns one pixel at a time and integrates its SSAA samples one after another
// (the per-pixel RMS combine of kernels/ssaa.cuh:109-131 is accumulated in
// registers, in sample order).  Every loop iteration a lane makes one RKF45
// attempt on its ray; lanes whose pixel is complete are refilled together:
// __ballot_sync finds them, one atomicAdd on the global work counter
// reserves __popc of them work items, and each lane takes base + its rank.
// So a warp never waits for its slowest ray, and work flows across frames
// of any size (the frame of a work item is found by binary search in the
// per-frame pixel prefix).  Nothing of a ray's state touches HBM.
//
// The FP64 and Christoffel-table renders run here; the FP32 pass of a
// split-precision render runs in k_pair.cu, and its FP64 pass (the rays
// queued near a photon orbit or below fp64_rfac*r_+) in k_fp64_requeue below.
#include "kernels.cuh"
#include "phys_stepper.cuh"

namespace prr {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ int find_frame(const long long *begin, int n, long long item)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(begin + mid) <= item) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ void warp_flush(unsigned long long *p, unsigned long long v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(p, v);
}

__device__ __forceinline__ uint8_t quant8(float v) { return (uint8_t)roundf(255.0f * fminf(fmaxf(v, 0.0f), 1.0f)); }

struct LaneCounts {
    unsigned long long att = 0, acc = 0, rays = 0, esc = 0, cap = 0, hit = 0, inf = 0, nan = 0, f64 = 0;
    __device__ void add(int result, bool escaped)
    {
        rays++;
        if (result == PRR_RESULT_SUCCESS) { if (escaped) esc++; else cap++; }
        else if (result == PRR_RESULT_INTERSECTION) hit++;
        else if (result == PRR_RESULT_INFINITE_GEO) inf++;
        else nan++;
    }
    __device__ void flush(unsigned long long *c)
    {
        warp_flush(&c[C_ATTEMPTS], att); warp_flush(&c[C_ACCEPTED], acc); warp_flush(&c[C_RAYS], rays);
        warp_flush(&c[C_ESCAPED], esc); warp_flush(&c[C_CAPTURED], cap); warp_flush(&c[C_INTERSECTION], hit);
        warp_flush(&c[C_INFINITE], inf); warp_flush(&c[C_MATH_ERROR], nan); warp_flush(&c[C_FP64], f64);
    }
};

template <class T, class O>
__device__ __forceinline__ void write_state(O *st, long long rid, const PhysRay<T> &R, int result, const float *uv)
{
    O *o = st + 12 * rid;
    o[0] = (O)uv[0]; o[1] = (O)uv[1]; o[2] = (O)result;
    o[3] = (O)R.x.x; o[4] = (O)R.x.y; o[5] = (O)R.x.z; o[6] = (O)R.x.w;
    o[7] = (O)R.u.x; o[8] = (O)R.u.y; o[9] = (O)R.u.z; o[10] = (O)R.u.w;
    o[11] = (O)R.accepted;
}

// Launch bounds: at most MAXT threads per CTA, at least MINB resident CTAs
// per SM (caps registers per thread).  CTAs of up to 64 threads use an
// instantiation built for several resident CTAs per SM.  The FP64 form is
// latency bound: on the 1080p frame 8 CTAs (128 registers, 16 warps, spills
// that hit L1) measured 1137 ms, 6 CTAs (168 registers) 1200 ms, 4 CTAs (215
// registers, no spills) 1369 ms.  The FP32 Christoffel-table form keeps 6
// (168 registers without spills).
#ifndef PRR_PERSISTENT_SMALL_MINB_F64
#define PRR_PERSISTENT_SMALL_MINB_F64 8
#endif
#ifndef PRR_PERSISTENT_SMALL_MINB_F32
#define PRR_PERSISTENT_SMALL_MINB_F32 6
#endif
template <class T> constexpr int small_minb() { return sizeof(T) == 8 ? PRR_PERSISTENT_SMALL_MINB_F64 : PRR_PERSISTENT_SMALL_MINB_F32; }

// EMIS: plasma emission (emission.cuh) accumulated at every accepted step of
// frames that have it, composited into the colour.
template <class T, int GEOD, bool EMIS, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) k_persistent(PersistentArgs a)
{
    const int lane = threadIdx.x & 31;
    long long item = -1;
    int frame = 0, px = 0, py = 0, s = 0, S = 1;
    float acc0 = 0.f, acc1 = 0.f, acc2 = 0.f, uv[2] = {0.f, 0.f};
    bool busy = false, need = true;
    PhysRay<T> R;
    Hot<T> q;
    EmisRay<T> E;
    LaneCounts cnt;
    const long long t0 = clock64();
    unsigned iter = 0;

    const unsigned ci = a.compaction_interval > 1 ? (unsigned)a.compaction_interval : 1u;
    unsigned since = ci;
    while (true) {
        // ---- refill lanes whose pixel is complete (warp-aggregated), at
        //      most every `ci` attempts unless the whole warp is idle ----
        unsigned needmask = 0;
        if (++since >= ci || __ballot_sync(FULL, busy) == 0) {
            needmask = __ballot_sync(FULL, need);
            since = 0;
        }
        if (needmask) {
            int leader = __ffs(needmask) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(&a.counters[C_WORK], (unsigned long long)__popc(needmask));
            base = __shfl_sync(FULL, base, leader);
            if (need) {
                long long it = (long long)base + __popc(needmask & ((1u << lane) - 1));
                need = false;
                if (it < a.total_pixels) {
                    item = it;
                    frame = find_frame(a.frame_pix_begin, a.nframes, it);
                    const FrameParams &fp = a.frames[frame];
                    long long p = it - __ldg(a.frame_pix_begin + frame);
                    px = (int)(p % fp.width); py = (int)(p / fp.width);
                    S = fp.samples; s = 0;
                    acc0 = acc1 = acc2 = 0.f;
                    q = make_hot<T>(fp);
                    phys_init<T>(fp, px, py, 0, R, uv);
                    if (EMIS) emis_init<T>(fp, R.x, R.u, E);
                    busy = true;
                } else {
                    busy = false;
                }
            }
        }
        if (__ballot_sync(FULL, busy) == 0) {
            if (__ballot_sync(FULL, need) == 0) break;  // queue exhausted for every lane
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
        if (!busy) continue;

        const FrameParams &fp = a.frames[frame];
        int result = 0;
        V3<float> col;
        const int st = phys_attempt<T, GEOD>(fp, q, R, result, col, (T)-1, nullptr, EMIS ? &E : nullptr);
        if (st == STEP_CONTINUE) continue;
        if (EMIS) col = emis_colour<T>(fp, E, col);

        cnt.att += (unsigned)R.i;
        cnt.acc += (unsigned)R.accepted;
        const long long rid = ((long long)py * fp.width + px) * S + s;
        cnt.add(result, result == PRR_RESULT_SUCCESS && metric_radius<T>(fp, R.x.x, R.x.y, R.x.z) >= q.rout);
        if (a.ray_steps) a.ray_steps[fp.ray_begin + rid] = R.accepted;
        if (a.ray_state) write_state<T, float>(a.ray_state, rid, R, result, uv);
        if (a.ray_state64) write_state<T, double>(a.ray_state64, rid, R, result, uv);
        if (a.sample_rgb) {
            float *o = a.sample_rgb + 3 * (fp.ray_begin + rid);
            o[0] = col.x; o[1] = col.y; o[2] = col.z;
        }
        if (S == 1) {
            acc0 = fminf(fmaxf(col.x, 0.f), 1.f); acc1 = fminf(fmaxf(col.y, 0.f), 1.f); acc2 = fminf(fmaxf(col.z, 0.f), 1.f);
        } else {
            acc0 += fminf(fmaxf(col.x * col.x, 0.f), 1.f);
            acc1 += fminf(fmaxf(col.y * col.y, 0.f), 1.f);
            acc2 += fminf(fmaxf(col.z * col.z, 0.f), 1.f);
        }
        s += 1;
        if (s < S) {
            phys_init<T>(fp, px, py, s, R, uv);
            if (EMIS) emis_init<T>(fp, R.x, R.u, E);
            continue;
        }
        if (S > 1) { acc0 = sqrtf(acc0 / (float)S); acc1 = sqrtf(acc1 / (float)S); acc2 = sqrtf(acc2 / (float)S); }
        const long long op = fp.pix_begin + (long long)py * fp.width + px;
        if (a.image) { a.image[3 * op] = acc0; a.image[3 * op + 1] = acc1; a.image[3 * op + 2] = acc2; }
        if (a.rgb8 && !fp.fxaa) { a.rgb8[3 * op] = quant8(acc0); a.rgb8[3 * op + 1] = quant8(acc1); a.rgb8[3 * op + 2] = quant8(acc2); }
        busy = false;
        need = true;
    }
    cnt.flush(a.counters);
}

// FP64 re-integration of the rays queued by a split-precision FP32 pass.
// 4 CTAs of 128 per SM (128 registers, 16 warps), as the FP64 persistent
// kernel's small-CTA form: the FP64 integration is latency bound.
__global__ void __launch_bounds__(128, 4) k_fp64_requeue(PersistentArgs a)
{
    const int lane = threadIdx.x & 31;
    bool busy = false, need = true;
    PhysRay<double> R;
    Hot<double> q;
    int frame = 0;
    long long rid = 0;
    LaneCounts cnt;
    long long nq = (long long)*(volatile unsigned long long *)&a.counters[C_FP64_QUEUED];
    if (nq > a.fp64_capacity) nq = a.fp64_capacity;
    while (true) {
        unsigned needmask = __ballot_sync(FULL, need);
        if (needmask) {
            int leader = __ffs(needmask) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(&a.counters[C_WORK_FP64], (unsigned long long)__popc(needmask));
            base = __shfl_sync(FULL, base, leader);
            if (need) {
                long long it = (long long)base + __popc(needmask & ((1u << lane) - 1));
                need = false;
                busy = false;
                if (it < nq) {
                    unsigned long long e = a.fp64_queue[it];
                    frame = (int)(e >> 40);
                    rid = (long long)(e & ((1ull << 40) - 1));
                    const FrameParams &fp = a.frames[frame];
                    long long pix = rid / fp.samples;
                    int s = (int)(rid - pix * fp.samples);
                    q = make_hot<double>(fp);
                    phys_init<double>(fp, (int)(pix % fp.width), (int)(pix / fp.width), s, R);
                    busy = true;
                }
            }
        }
        if (__ballot_sync(FULL, busy) == 0) break;
        if (!busy) continue;
        const FrameParams &fp = a.frames[frame];
        int result = 0;
        V3<float> col;
        int st = phys_attempt<double, 0>(fp, q, R, result, col, -1.0);
        if (st == STEP_CONTINUE) continue;
        cnt.att += (unsigned)R.i;
        cnt.acc += (unsigned)R.accepted;
        cnt.add(result, result == PRR_RESULT_SUCCESS && metric_radius<double>(fp, R.x.x, R.x.y, R.x.z) >= q.rout);
        float *o = a.sample_rgb + 3 * (fp.ray_begin + rid);
        o[0] = col.x; o[1] = col.y; o[2] = col.z;
        busy = false;
        need = true;
    }
    cnt.flush(a.counters);
}

template <class T, int GEOD, bool EMIS>
static cudaError_t launch_one(const PersistentArgs &a, int block, int blocks_per_sm, int nsm, cudaStream_t st)
{
    int grid = nsm * blocks_per_sm;
    if (grid < 1) grid = 1;
    if (block <= 64) k_persistent<T, GEOD, EMIS, 64, small_minb<T>()><<<grid, block, 0, st>>>(a);
    else k_persistent<T, GEOD, EMIS, 256, 1><<<grid, block, 0, st>>>(a);
    return cudaGetLastError();
}

template <class T, int GEOD, bool EMIS> static cudaError_t occupancy_one(int *n, int block)
{
    if (block <= 64) return cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, k_persistent<T, GEOD, EMIS, 64, small_minb<T>()>, block, 0);
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, k_persistent<T, GEOD, EMIS, 256, 1>, block, 0);
}

cudaError_t launch_persistent(const PersistentArgs &a, int precision, int block, int blocks_per_sm, int nsm, cudaStream_t st)
{
    if (block < 32 || block > 256 || block % 32) return cudaErrorInvalidValue;
    if (precision == PRR_PREC_FP64) {
        if (a.hamiltonian & PRR_HAM_FP64) return launch_ham(a, PRR_PREC_FP64, false, block, blocks_per_sm, nsm, st);
        if (a.emission) return launch_one<double, 0, true>(a, block, blocks_per_sm, nsm, st);
        return launch_one<double, 0, false>(a, block, blocks_per_sm, nsm, st);
    }
    if (precision == PRR_PREC_SPLIT) {
        if (a.hamiltonian & PRR_HAM_FP32) return launch_ham(a, PRR_PREC_FP32, true, block, blocks_per_sm, nsm, st);
        return launch_pair(a, 1, true, block, blocks_per_sm, nsm, st);
    }
    if (a.geod_table) {
        if (a.emission) return cudaErrorInvalidValue;  // emission runs with the register contraction
        return launch_one<float, 1, false>(a, block, blocks_per_sm, nsm, st);
    }
    if ((a.hamiltonian & PRR_HAM_FP32) && (a.rays_per_thread != 2 || a.emission))
        return launch_ham(a, PRR_PREC_FP32, false, block, blocks_per_sm, nsm, st);
    return launch_pair(a, a.rays_per_thread == 2 ? 2 : 1, false, block, blocks_per_sm, nsm, st);
}

int persistent_occupancy(int precision, int geod_table, int block, int rays_per_thread, int emission, int hamiltonian)
{
    int n = 0;
    cudaError_t e;
    if (precision == PRR_PREC_FP64 && (hamiltonian & PRR_HAM_FP64)) return ham_occupancy(PRR_PREC_FP64, block, false, emission != 0);
    if (precision == PRR_PREC_FP64) e = emission ? occupancy_one<double, 0, true>(&n, block) : occupancy_one<double, 0, false>(&n, block);
    else if (precision == PRR_PREC_SPLIT)
        return (hamiltonian & PRR_HAM_FP32) ? ham_occupancy(PRR_PREC_FP32, block, true) : pair_occupancy(1, true, block);
    else if (geod_table) e = occupancy_one<float, 1, false>(&n, block);
    else if ((hamiltonian & PRR_HAM_FP32) && (rays_per_thread != 2 || emission))
        return ham_occupancy(PRR_PREC_FP32, block, false, emission != 0);
    else return pair_occupancy(rays_per_thread == 2 ? 2 : 1, false, block, emission != 0);
    if (e != cudaSuccess) { cudaGetLastError(); return 0; }
    return n;
}

cudaError_t launch_fp64_requeue(const PersistentArgs &a, int block, int nsm, cudaStream_t st)
{
    if (a.hamiltonian & PRR_HAM_FP64) return launch_ham_requeue(a, nsm, st);
    int bpsm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bpsm, k_fp64_requeue, 128, 0);
    if (e != cudaSuccess) return e;
    k_fp64_requeue<<<nsm * (bpsm > 0 ? bpsm : 1), 128, 0, st>>>(a);
    (void)block;
    return cudaGetLastError();
}

}  // namespace prr
