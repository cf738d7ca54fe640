// Shared device helpers for the adock_b200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include "../../include/adock_b200.h"

namespace adock {

// thread-local error message (abi.cu)
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* where);
int sm_count();

#define ADOCK_CHECK_ARG(cond, ...)                 \
    do {                                           \
        if (!(cond)) {                             \
            ::adock::set_error(__VA_ARGS__);       \
            return ADOCK_E_ARG;                    \
        }                                          \
    } while (0)

#define ADOCK_CUDA(call)                                            \
    do {                                                            \
        cudaError_t _e = (call);                                    \
        if (_e != cudaSuccess) return ::adock::cuda_status(_e, #call); \
    } while (0)

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Counter-based uniform generator: SplitMix64 finaliser over (seed, chain, step, slot), 24-bit mantissa,
// identical on every lane. Same hash and bit layout as the reference's urand (mckernel.py:71-81) so that
// a chain's mutation sequence is reproducible across the two builds.
__host__ __device__ __forceinline__ unsigned long long splitmix(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
__host__ __device__ __forceinline__ float uniform01(unsigned long long seed, int chain, int step, int slot) {
    unsigned long long key = ((unsigned long long)chain << 32) ^ ((unsigned long long)step << 8) ^ (unsigned long long)slot;
    unsigned long long h = splitmix(seed ^ splitmix(key));
    return (float)(h >> 40) * (1.0f / 16777216.0f);
}
// rejection-sampled point in the unit ball (<= 32 tries, else 0), mckernel.py:82-90
__device__ __forceinline__ void unit_ball(unsigned long long seed, int chain, int step, int slot, float* v) {
    for (int k = 0; k < 32; ++k) {
        float a = 2.f * uniform01(seed, chain, step, slot + 3 * k) - 1.f;
        float b = 2.f * uniform01(seed, chain, step, slot + 3 * k + 1) - 1.f;
        float c = 2.f * uniform01(seed, chain, step, slot + 3 * k + 2) - 1.f;
        if (a * a + b * b + c * c < 1.f) { v[0] = a; v[1] = b; v[2] = c; return; }
    }
    v[0] = v[1] = v[2] = 0.f;
}

// q <- quat(rotation vector) * q, normalised (mckernel.py:93-105)
__device__ __forceinline__ void quat_apply_rotvec(float* q, float rx, float ry, float rz) {
    float ang = sqrtf(rx * rx + ry * ry + rz * rz);
    float hw, k;
    if (ang > 1e-6f) { float s, c; __sincosf(0.5f * ang, &s, &c); hw = c; k = s / ang; } else { hw = 1.f; k = 0.5f; }
    float aw = hw, ax = rx * k, ay = ry * k, az = rz * k;
    float bw = q[0], bx = q[1], by = q[2], bz = q[3];
    float w = aw * bw - ax * bx - ay * by - az * bz;
    float x = aw * bx + ax * bw + ay * bz - az * by;
    float y = aw * by - ax * bz + ay * bw + az * bx;
    float z = aw * bz + ax * by - ay * bx + az * bw;
    float nn = rsqrtf(w * w + x * x + y * y + z * z);
    q[0] = w * nn; q[1] = x * nn; q[2] = y * nn; q[3] = z * nn;
}

// Vina-family pair energy and dE/dr with the radius sum and the hydrophobic / H-bond pair flags precomputed.
// Same terms as mckernel.py:44-64 / scoring.pair_terms . weights.
struct PairPrm {
    float g1_off, g1_inv, g2_off, g2_inv, rep_off, hyd_good, hyd_bad, hyd_inv, hb_good, hb_bad, hb_inv, cutoff;
    float w_g1, w_g2, w_rep, w_hyd, w_hb;
};

__host__ inline PairPrm make_pair_prm(const float* prm) {
    PairPrm p;
    p.g1_off = prm[0]; p.g1_inv = 1.f / prm[1]; p.g2_off = prm[2]; p.g2_inv = 1.f / prm[3]; p.rep_off = prm[4];
    p.hyd_good = prm[5]; p.hyd_bad = prm[6]; p.hyd_inv = 1.f / (prm[6] - prm[5]);
    p.hb_good = prm[7]; p.hb_bad = prm[8]; p.hb_inv = 1.f / (prm[8] - prm[7]); p.cutoff = prm[9];
    p.w_g1 = prm[10]; p.w_g2 = prm[11]; p.w_rep = prm[12]; p.w_hyd = prm[13]; p.w_hb = prm[14];
    return p;
}

#define PF_HYD 1
#define PF_HB 2

// Branch-free: the repulsion acts below rep_off and the hydrophobic / H-bond terms are ramps from 1 (d <= good)
// to 0 (d >= bad); written as clamps and selects, which add exactly 0 where the piecewise form adds nothing.
__device__ __forceinline__ float pair_energy(float r, float rsum, int flags, const PairPrm& p, float& de) {
    const float d = r - rsum;
    const float u1 = (d - p.g1_off) * p.g1_inv, g1 = __expf(-u1 * u1);
    const float u2 = (d - p.g2_off) * p.g2_inv, g2 = __expf(-u2 * u2);
    float e = p.w_g1 * g1 + p.w_g2 * g2;
    de = p.w_g1 * (-2.f * u1 * p.g1_inv) * g1 + p.w_g2 * (-2.f * u2 * p.g2_inv) * g2;
    const float dr = fminf(d - p.rep_off, 0.f);
    e += p.w_rep * dr * dr;
    de += p.w_rep * 2.f * dr;
    const float wh = (flags & PF_HYD) ? p.w_hyd : 0.f, wb = (flags & PF_HB) ? p.w_hb : 0.f;
    const float vh = (p.hyd_bad - d) * p.hyd_inv, vb = (p.hb_bad - d) * p.hb_inv;
    e += wh * fminf(fmaxf(vh, 0.f), 1.f);
    e += wb * fminf(fmaxf(vb, 0.f), 1.f);
    de -= (vh > 0.f && vh < 1.f) ? wh * p.hyd_inv : 0.f;
    de -= (vb > 0.f && vb < 1.f) ? wb * p.hb_inv : 0.f;
    return e;
}

// float64 variant (final re-score)
__device__ __forceinline__ double pair_energy64(double r, double rsum, int flags, const float* prm) {
    double d = r - rsum;
    double u1 = (d - (double)prm[0]) / (double)prm[1], u2 = (d - (double)prm[2]) / (double)prm[3];
    double e = (double)prm[10] * exp(-u1 * u1) + (double)prm[11] * exp(-u2 * u2);
    double dr = d - (double)prm[4];
    if (dr < 0.0) e += (double)prm[12] * dr * dr;
    if (flags & PF_HYD) {
        double v = ((double)prm[6] - d) / ((double)prm[6] - (double)prm[5]);
        e += (double)prm[13] * fmin(fmax(v, 0.0), 1.0);
    }
    if (flags & PF_HB) {
        double v = ((double)prm[8] - d) / ((double)prm[8] - (double)prm[7]);
        e += (double)prm[14] * fmin(fmax(v, 0.0), 1.0);
    }
    return e;
}

template <typename GT> __device__ __forceinline__ float gload(const GT* p);
template <> __device__ __forceinline__ float gload<float>(const float* p) { return __ldg(p); }
template <> __device__ __forceinline__ float gload<__half>(const __half* p) { return __half2float(__ldg(p)); }
template <> __device__ __forceinline__ float gload<__nv_bfloat16>(const __nv_bfloat16* p) {
    return __bfloat162float(__ldg(p));
}

}  // namespace adock
