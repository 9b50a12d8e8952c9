// Pieces shared by the persistent-warp walk kernels (FAST_FP32 / FAST_FP64
// walks in kernels_fast.cu, the Gaussian heat-source forward / adjoint walks
// in kernels_adjoint.cu).
#pragma once
#include <type_traits>

#include "common.cuh"

namespace wosb {

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ double dinf() { return __longlong_as_double(0x7ff0000000000000LL); }
__device__ __forceinline__ double dnan() { return __longlong_as_double(0x7ff8000000000000LL); }

// Walk stream of one (point, walk) pair: Philox4x32-10 keyed by the point's
// reference seed, counter (walk, step, draw); begin_step() opens a step's
// draws.  unit() is in (0, 1).
template <typename T>
struct FastRng {
    PhiloxStream s;
    __device__ FastRng(uint64_t pseed, uint32_t walk) : s(pseed, walk) {}
    __device__ FastRng(uint2 key, uint32_t walk) : s(key, walk) {}
    __device__ __forceinline__ void begin_step(int step) {
        s.begin_step(static_cast<uint32_t>(step));
    }
    __device__ __forceinline__ T unit();
    __device__ __forceinline__ T unit_open() { return unit(); }
    // (0, 1) with 53 random bits, for samplers that always work in double
    __device__ __forceinline__ double unit64() { return s.uniform_d(); }
    __device__ __forceinline__ double unit64_open() { return s.uniform_d(); }
};
template <>
__device__ __forceinline__ float FastRng<float>::unit() { return s.uniform_f(); }
template <>
__device__ __forceinline__ double FastRng<double>::unit() { return s.uniform_d(); }

// Chan et al. pairwise combination of (n, mean, M2).
__device__ __forceinline__ void chan_merge(double &n, double &mean, double &m2, double nb,
                                           double meanb, double m2b) {
    if (nb == 0.0) return;
    if (n == 0.0) {
        n = nb;
        mean = meanb;
        m2 = m2b;
        return;
    }
    const double tot = n + nb;
    const double delta = meanb - mean;
    mean += delta * (nb / tot);
    m2 += m2b + delta * delta * (n * nb / tot);
    n = tot;
}

template <int DIM>
__device__ __forceinline__ int bid_of(const SceneView &s, int slot) {
    return (DIM == 2 && slot >= 0) ? s.segid[slot].x : -1;
}

// Per-lane sums of walk values about a shift K (the lane's first value):
// S = sum (v - K), Q = sum (v - K)^2, so a finished walk costs two adds and
// a multiply; finish() turns them into Welford's (mean, M2) once per task.
struct ShiftedSums {
    int n = 0;
    double k = 0.0, s = 0.0, q = 0.0;
    __device__ __forceinline__ void add(double v) {
        if (n == 0) k = v;
        ++n;
        const double d = v - k;
        s += d;
        q += d * d;
    }
    __device__ __forceinline__ void finish(double &mean, double &m2) const {
        if (n == 0) {
            mean = 0.0;
            m2 = 0.0;
            return;
        }
        const double inv = 1.0 / static_cast<double>(n);
        mean = k + s * inv;
        m2 = fmax(q - s * s * inv, 0.0);
    }
};

// Squared FP64 distance from p to the primitive in binary-tree `slot` (the
// FP32 query's winner), its nearest point and (2D) boundary id.
template <int DIM>
__device__ __forceinline__ double reproject64_sq(const SceneView &s, int slot, double px,
                                                 double py, double pz, V3<double> &np, int &bid) {
    if (DIM == 2) {
        const double2 a = s.seg64[2 * slot], c = s.seg64[2 * slot + 1];
        double nx, ny;
        const double d2 = npq_seg64(a.x, a.y, c.x, c.y, px, py, nx, ny);
        np = V3<double>{nx, ny, 0.0};
        bid = s.segid[slot].x;
        return d2;
    }
    const double2 *r = s.tri64 + 7 * slot;
    const double2 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3], r4 = r[4], r5 = r[5], r6 = r[6];
    double nx, ny, nz;
    const double d2 = eberly<double>(px, py, pz, r0.x, r0.y, r1.x, r1.y, r2.x, r2.y, r3.x, r3.y,
                                     r4.x, r4.y, r5.x, r5.y, r6.x, r6.y, nx, ny, nz);
    np = V3<double>{nx, ny, nz};
    bid = -1;
    return d2;
}

// FP64 re-projection of p onto the primitive in binary-tree `slot` (the
// FP32 query's winner): exact distance, nearest point and (2D) boundary id.
template <int DIM>
__device__ __forceinline__ double reproject64(const SceneView &s, int slot, double px, double py,
                                              double pz, V3<double> &np, int &bid) {
    if (DIM == 2) {
        const double2 a = s.seg64[2 * slot], c = s.seg64[2 * slot + 1];
        double nx, ny;
        const double d2 = npq_seg64(a.x, a.y, c.x, c.y, px, py, nx, ny);
        np = V3<double>{nx, ny, 0.0};
        bid = s.segid[slot].x;
        return sqrt(d2);
    }
    const double2 *r = s.tri64 + 7 * slot;
    const double2 r0 = r[0], r1 = r[1], r2 = r[2], r3 = r[3], r4 = r[4], r5 = r[5], r6 = r[6];
    double nx, ny, nz;
    const double d2 = eberly<double>(px, py, pz, r0.x, r0.y, r1.x, r1.y, r2.x, r2.y, r3.x, r3.y,
                                     r4.x, r4.y, r5.x, r5.y, r6.x, r6.y, nx, ny, nz);
    np = V3<double>{nx, ny, nz};
    bid = -1;
    return sqrt(d2);
}

}  // namespace wosb
