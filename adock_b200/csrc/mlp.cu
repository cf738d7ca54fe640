// Proposal network kernels (sm_100a): BF16 GEMM on the tensor cores with FP32 accumulation and fused epilogues,
// Gaussian negative log-likelihood + its gradient, SiLU backward, bias-gradient reduction, Adam.
//
// Network: x [320] -> SiLU(W1 x + b1) [256] -> SiLU(W2 h1 + b2) [256] -> W3 h2 + b3 [64]. Output columns 0..25 are
// the means and 32..57 the log standard deviations of the move (translation 3, rotation vector 3, torsions 20);
// with a translation mixture, columns 27..29 and 58..60 hold two more translation means and 26, 30, 61 the
// mixing logits.
//
// GEMM: C[M,N] = A[M,K] B[K,N] with A and B in BF16 at arbitrary (row, column) strides, so the same kernel serves
// the forward pass (X W), the input gradient (dY W^T) and the weight gradient (X^T dY). adock_gemm_bf16 runs it on
// the tcgen05 tensor cores with the accumulator in tensor memory (gemm_bf16_tc_kernel); gemm_bf16_kernel is an
// independent warp-level mma.sync version (64x64 CTA tile, 4 warps of 32x32, K step 32, m16n8k16 BF16 -> FP32)
// behind adock_gemm_bf16_mma, which the tests use as a cross-check.
#include "common.cuh"

namespace adock {

#define GM 64
#define GN 64
#define GK 32
#define APAD 8

struct GemmArgs {
    int M, N, K;
    const __nv_bfloat16* A;
    long long sAm, sAk;
    const __nv_bfloat16* B;
    long long sBk, sBn;
    // epilogue
    float* C;             // FP32 output [M, ldc] (optional)
    long long ldc;
    float beta;           // C = acc + beta * C
    const float* bias;    // [N] (optional)
    int act;              // 0 none, 1 SiLU
    float* pre;           // FP32 pre-activation copy [M, ldc] (optional)
    __nv_bfloat16* Cb;    // BF16 output [M, ldcb] (optional)
    long long ldcb;
};

__device__ __forceinline__ float silu(float x) { return x / (1.f + __expf(-x)); }

__device__ __forceinline__ void mma_bf16(float* d, const uint32_t* a, const uint32_t* b) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__global__ void __launch_bounds__(128) gemm_bf16_kernel(const __grid_constant__ GemmArgs g) {
    __shared__ __align__(16) __nv_bfloat16 As[GM][GK + APAD];   // [m][k]
    __shared__ __align__(16) __nv_bfloat16 Bs[GN][GK + APAD];   // [n][k] (transposed: k contiguous)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m0 = blockIdx.y * GM, n0 = blockIdx.x * GN;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int gid = lane >> 2, tig = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.f;
    const bool a_kfast = g.sAk == 1, b_kfast = g.sBk == 1;
    const __nv_bfloat16 zero = __float2bfloat16(0.f);
    for (int k0 = 0; k0 < g.K; k0 += GK) {
        // stage A[m0:m0+64, k0:k0+32] and B[k0:k0+32, n0:n0+64]; the contiguous dimension runs across threads
        for (int e = tid; e < GM * GK; e += 128) {
            const int mm = a_kfast ? e / GK : e % GM, kk = a_kfast ? e % GK : e / GM;
            const int m = m0 + mm, k = k0 + kk;
            As[mm][kk] = (m < g.M && k < g.K) ? g.A[(long long)m * g.sAm + (long long)k * g.sAk] : zero;
        }
        for (int e = tid; e < GN * GK; e += 128) {
            const int nn = b_kfast ? e / GK : e % GN, kk = b_kfast ? e % GK : e / GN;
            const int n = n0 + nn, k = k0 + kk;
            Bs[nn][kk] = (n < g.N && k < g.K) ? g.B[(long long)k * g.sBk + (long long)n * g.sBn] : zero;
        }
        __syncthreads();
#pragma unroll
        for (int ks = 0; ks < GK; ks += 16) {
            uint32_t af[2][4], bf[4][2];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const int r = wm + i * 16 + gid;
                af[i][0] = *(const uint32_t*)&As[r][ks + tig * 2];
                af[i][1] = *(const uint32_t*)&As[r + 8][ks + tig * 2];
                af[i][2] = *(const uint32_t*)&As[r][ks + tig * 2 + 8];
                af[i][3] = *(const uint32_t*)&As[r + 8][ks + tig * 2 + 8];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = wn + j * 8 + gid;
                bf[j][0] = *(const uint32_t*)&Bs[c][ks + tig * 2];
                bf[j][1] = *(const uint32_t*)&Bs[c][ks + tig * 2 + 8];
            }
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) mma_bf16(acc[i][j], af[i], bf[j]);
        }
        __syncthreads();
    }
    // epilogue: acc[i][j] = rows (gid, gid + 8), cols (tig * 2, tig * 2 + 1) of tile (i, j)
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int m = m0 + wm + i * 16 + gid + (r >> 1) * 8;
                const int n = n0 + wn + j * 8 + tig * 2 + (r & 1);
                if (m >= g.M || n >= g.N) continue;
                float v = acc[i][j][r];
                if (g.C && g.beta != 0.f) v += g.beta * g.C[(long long)m * g.ldc + n];
                if (g.bias) v += g.bias[n];
                if (g.pre) g.pre[(long long)m * g.ldc + n] = v;
                if (g.act == 1) v = silu(v);
                if (g.C) g.C[(long long)m * g.ldc + n] = v;
                if (g.Cb) g.Cb[(long long)m * g.ldcb + n] = __float2bfloat16(v);
            }
}

// ------------------------------------------------------------------------------------------------ tcgen05 GEMM
// Same product and epilogue on the 5th-generation tensor cores. One CTA of 128 threads computes a 128 x TN tile
// (TN = 64 or 128) of C with the FP32 accumulator in tensor memory (TMEM: 128 lanes = rows, TN columns):
//  - K is stepped by 64. The 128 threads stage A[128, 64] and B[64, TN] from global memory (any strides, zero
//    fill past M, N, K) into shared memory in the tensor core's canonical K-major layout without swizzle: 8-row x
//    16-byte core matrices, core matrix (row group g, K chunk c) at byte g * 1024 + c * 128, row r of it at + 16 r.
//    B is stored as its transpose (TN rows of K), so the MMA computes D[m, n] = sum_k A[m, k] B^T[n, k].
//  - After a proxy fence and a CTA barrier, one thread issues four tcgen05.mma (M 128, N TN, K 16; BF16 inputs,
//    FP32 accumulate; descriptor start address advanced by two core matrices per MMA, leading byte offset 128 =
//    the next K chunk, stride byte offset 1024 = the next row group) and tcgen05.commit, which arrives on an
//    mbarrier when they have completed; all threads wait on it before the tile buffers are refilled.
//  - Epilogue: warp w reads TMEM lanes 32w..32w+31 (its 32 rows) 16 columns at a time with tcgen05.ld and applies
//    C = acc + beta C + bias, pre-activation copy, SiLU, FP32 and BF16 stores, as gemm_bf16_kernel does.
// Every mbarrier wait is bounded; a wait that gives up sets g_tc_status (read by adock_gemm_status) and the CTA
// skips the rest of its tile, then frees its TMEM.
#define TC_BM 128
#define TC_BK 64
#define TC_WAIT_MAX (1 << 22)
#define TC_WAIT_NS 200000000ull   // 200 ms

__device__ int g_tc_status;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: start address, leading / stride byte offsets (all >> 4), version 1 at bit 46,
// base offset 0, layout type 0 (no swizzle) at bits 61..63.
__device__ __forceinline__ uint64_t tc_smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bit 4), A and B BF16 (bits 7 and 10), both K-major,
// N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for the mbarrier phase of the given parity; gives up after TC_WAIT_MAX polls or TC_WAIT_NS nanoseconds of
// the global timer, whichever comes first (a poll may suspend the thread for a system-dependent time).
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity) {
    const uint64_t t0 = global_ns();
    for (int i = 0; i < TC_WAIT_MAX; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        if (global_ns() - t0 > TC_WAIT_NS) return false;
    }
    return false;
}

template <int TN>
__global__ void __launch_bounds__(128) gemm_bf16_tc_kernel(const __grid_constant__ GemmArgs g) {
    extern __shared__ __align__(16) unsigned char tc_smem[];
    // tile buffers from the first 1024-byte boundary of the dynamic shared memory (the launch adds 1024 bytes)
    unsigned char* As = tc_smem + ((1024u - (smem_u32(tc_smem) & 1023u)) & 1023u);   // [16][8][8][16 B] = 16 KB
    unsigned char* Bs = As + TC_BM * TC_BK * 2;                                           // [TN / 8][8][8][16 B]
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base_sh;
    __shared__ int fail_sh;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * TC_BM, n0 = blockIdx.x * TN;
    const uint32_t mbar_a = smem_u32(&mbar);
    if (tid == 0) {
        fail_sh = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar_a), "r"(1) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_base_sh)), "r"(TN) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_sh;
    const bool a_kfast = g.sAk == 1, b_kfast = g.sBk == 1;
    const int nk = (g.K + TC_BK - 1) / TC_BK;
    bool ok = true;
    for (int kt = 0; kt < nk && ok; ++kt) {
        const int k0 = kt * TC_BK;
        // stage A[m0:m0+128, k0:k0+64] and B[k0:k0+64, n0:n0+TN]; the contiguous global dimension runs across threads
        for (int e = tid; e < TC_BM * TC_BK; e += 128) {
            const int mm = a_kfast ? e / TC_BK : e % TC_BM, kk = a_kfast ? e % TC_BK : e / TC_BM;
            const int m = m0 + mm, k = k0 + kk;
            const __nv_bfloat16 v = (m < g.M && k < g.K) ? g.A[(long long)m * g.sAm + (long long)k * g.sAk]
                                                         : __float2bfloat16(0.f);
            *(__nv_bfloat16*)(As + (mm >> 3) * 1024 + (kk >> 3) * 128 + (mm & 7) * 16 + (kk & 7) * 2) = v;
        }
        for (int e = tid; e < TN * TC_BK; e += 128) {
            const int nn = b_kfast ? e / TC_BK : e % TN, kk = b_kfast ? e % TC_BK : e / TN;
            const int n = n0 + nn, k = k0 + kk;
            const __nv_bfloat16 v = (n < g.N && k < g.K) ? g.B[(long long)k * g.sBk + (long long)n * g.sBn]
                                                         : __float2bfloat16(0.f);
            *(__nv_bfloat16*)(Bs + (nn >> 3) * 1024 + (kk >> 3) * 128 + (nn & 7) * 16 + (kk & 7) * 2) = v;
        }
        // make the generic-proxy stores visible to the tensor core (async proxy), then one thread issues the MMAs
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a0 = smem_u32(As), b0 = smem_u32(Bs);
#pragma unroll
            for (int s = 0; s < TC_BK / 16; ++s) {
                const uint64_t da = tc_smem_desc(a0 + s * 256, 128, 1024);
                const uint64_t db = tc_smem_desc(b0 + s * 256, 128, 1024);
                const uint32_t acc = (kt > 0 || s > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    ::"r"(tmem), "l"(da), "l"(db), "r"(tc_idesc(TC_BM, TN)), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         ::"r"(mbar_a) : "memory");
        }
        // the MMAs read the tile buffers: wait for their completion before the next stage overwrites them
        if (!tc_wait(mbar_a, (uint32_t)(kt & 1))) {
            atomicExch(&fail_sh, 1);
            atomicExch(&g_tc_status, 1);
        }
        __syncthreads();
        ok = fail_sh == 0;
        if (!ok) {
            // gave up waiting: before the tensor memory is released below, wait once more (bounded) for the MMAs
            // of this stage that may still be running; the tile is not written (its contents are undefined)
            tc_wait(mbar_a, (uint32_t)(kt & 1));
            __syncthreads();
        }
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok && nk > 0) {
        const int m = m0 + warp * 32 + lane;
#pragma unroll 1
        for (int c0 = 0; c0 < TN; c0 += 16) {
            uint32_t r[16];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15])
                : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (m < g.M) {
#pragma unroll
                for (int j = 0; j < 16; ++j) {
                    const int n = n0 + c0 + j;
                    if (n >= g.N) continue;
                    float v = __uint_as_float(r[j]);
                    if (g.C && g.beta != 0.f) v += g.beta * g.C[(long long)m * g.ldc + n];
                    if (g.bias) v += g.bias[n];
                    if (g.pre) g.pre[(long long)m * g.ldc + n] = v;
                    if (g.act == 1) v = silu(v);
                    if (g.C) g.C[(long long)m * g.ldc + n] = v;
                    if (g.Cb) g.Cb[(long long)m * g.ldcb + n] = __float2bfloat16(v);
                }
            }
        }
    } else if (nk == 0) {
        // K = 0: the product is zero; only the epilogue terms remain
        const int m = m0 + warp * 32 + lane;
        if (m < g.M)
            for (int j = 0; j < TN; ++j) {
                const int n = n0 + j;
                if (n >= g.N) break;
                float v = 0.f;
                if (g.C && g.beta != 0.f) v += g.beta * g.C[(long long)m * g.ldc + n];
                if (g.bias) v += g.bias[n];
                if (g.pre) g.pre[(long long)m * g.ldc + n] = v;
                if (g.act == 1) v = silu(v);
                if (g.C) g.C[(long long)m * g.ldc + n] = v;
                if (g.Cb) g.Cb[(long long)m * g.ldcb + n] = __float2bfloat16(v);
            }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN) : "memory");
    }
}

// Gaussian NLL over the move dimensions: out [B, 64] (mu = out[:, 0:26], log_sigma = out[:, 32:58] clamped to
// [-4, 2]); target [B, 32] (move in 0..25, torsion count in 26); rows of the batch weighted equally.
// n_comp = 3: the translation is a mixture of 3 Gaussians with the shared per-axis sigma (out[:, 32:35]), means at
// columns 0, 27, 58 (3 each) and mixing logits at columns 26, 30, 61; its term is
// -log sum_k softmax(logits)_k N(t | mu_k, sigma). Rotation and torsions stay single Gaussians.
// Writes dOut (BF16, [B, 64]) = d(mean loss)/d(out) and accumulates the loss sum into *loss.
__constant__ int MIX_MEAN[3] = {0, 27, 58};
__constant__ int MIX_LOGIT[3] = {26, 30, 61};

__global__ void nll_kernel(const float* __restrict__ out, const float* __restrict__ target, int B, int n_comp,
                           __nv_bfloat16* __restrict__ dout, float* __restrict__ loss) {
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (row >= B) return;
    const float* o = out + (long long)row * 64;
    const float* t = target + (long long)row * 32;
    const int nt = (int)t[26];
    const float inv = 1.f / (float)B;
    const bool mix = n_comp > 1;
    float l = 0.f, dmu = 0.f, dls = 0.f;
    const int d = lane;
    const bool active = d < 26 && (d < 6 || d - 6 < nt) && !(mix && d < 3);
    if (active) {
        const float mu = o[d], ls_raw = o[32 + d];
        const float ls = fminf(fmaxf(ls_raw, -4.f), 2.f);
        const float z = (t[d] - mu) * __expf(-ls);
        l = 0.5f * z * z + ls;
        dmu = -z * __expf(-ls) * inv;
        dls = (ls_raw > -4.f && ls_raw < 2.f) ? (1.f - z * z) * inv : 0.f;
    }
    dout[(long long)row * 64 + lane] = __float2bfloat16(dmu);
    dout[(long long)row * 64 + 32 + lane] = __float2bfloat16(dls);
    if (mix) {
        __syncwarp();
        if (lane == 0) {   // the translation mixture: overwrites its columns after the per-lane defaults (0)
            float ls[3], isd[3], lg[3], lp[3], z[3][3];
            for (int a = 0; a < 3; ++a) {
                ls[a] = fminf(fmaxf(o[32 + a], -4.f), 2.f);
                isd[a] = __expf(-ls[a]);
            }
            float mg = -3.4e38f, mp = -3.4e38f;
            for (int k = 0; k < 3; ++k) {
                lg[k] = o[MIX_LOGIT[k]];
                lp[k] = lg[k];
                for (int a = 0; a < 3; ++a) {
                    z[k][a] = (t[a] - o[MIX_MEAN[k] + a]) * isd[a];
                    lp[k] -= 0.5f * z[k][a] * z[k][a];
                }
                mg = fmaxf(mg, lg[k]);
                mp = fmaxf(mp, lp[k]);
            }
            float sg = 0.f, sp = 0.f;
            for (int k = 0; k < 3; ++k) {
                sg += __expf(lg[k] - mg);
                sp += __expf(lp[k] - mp);
            }
            const float lse_g = mg + __logf(sg), lse_p = mp + __logf(sp);
            l += lse_g - lse_p + ls[0] + ls[1] + ls[2];
            float dl[3] = {0.f, 0.f, 0.f};
            for (int k = 0; k < 3; ++k) {
                const float r = __expf(lp[k] - lse_p), p = __expf(lg[k] - lse_g);
                dout[(long long)row * 64 + MIX_LOGIT[k]] = __float2bfloat16((p - r) * inv);
                for (int a = 0; a < 3; ++a) {
                    dout[(long long)row * 64 + MIX_MEAN[k] + a] = __float2bfloat16(-r * z[k][a] * isd[a] * inv);
                    dl[a] += r * (1.f - z[k][a] * z[k][a]);
                }
            }
            for (int a = 0; a < 3; ++a) {
                const float raw = o[32 + a];
                dout[(long long)row * 64 + 32 + a] = __float2bfloat16((raw > -4.f && raw < 2.f) ? dl[a] * inv : 0.f);
            }
        }
    }
    l = warp_sum(l);
    if (lane == 0) atomicAdd(loss, l);
}

// dA = dH * SiLU'(A) (A = pre-activation FP32), BF16 output
__global__ void silu_backward_kernel(const float* __restrict__ dH, const float* __restrict__ A, long long n,
                                     __nv_bfloat16* __restrict__ dA) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float a = A[i];
        const float s = 1.f / (1.f + __expf(-a));
        dA[i] = __float2bfloat16(dH[i] * s * (1.f + a * (1.f - s)));
    }
}

// db[n] = sum_rows dA[row, n] (BF16 input, FP32 sums); one block per 32 columns
__global__ void bias_grad_kernel(const __nv_bfloat16* __restrict__ dA, int rows, int cols, float* __restrict__ db) {
    __shared__ float part[8][33];
    const int c = blockIdx.x * 32 + (threadIdx.x & 31), w = threadIdx.x >> 5;
    float s = 0.f;
    if (c < cols)
        for (int r = w; r < rows; r += 8) s += __bfloat162float(dA[(long long)r * cols + c]);
    part[w][threadIdx.x & 31] = s;
    __syncthreads();
    if (w == 0 && c < cols) {
        float t = 0.f;
        for (int i = 0; i < 8; ++i) t += part[i][threadIdx.x & 31];
        db[c] = t;
    }
}

// Adam on FP32 master parameters, refreshing their BF16 copies (bias_hat corrections from the step count)
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ grad, float* __restrict__ m,
                            float* __restrict__ v, __nv_bfloat16* __restrict__ pb, long long n, float lr, float b1,
                            float b2, float eps, float c1, float c2, float wd) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = grad[i] + wd * p[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = pi;
        if (pb) pb[i] = __float2bfloat16(pi);
    }
}

__global__ void f32_to_bf16_kernel(const float* __restrict__ x, __nv_bfloat16* __restrict__ y, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16(x[i]);
}

static unsigned grid1d(long long n) {
    long long b = (n + 255) / 256;
    const long long cap = 148LL * 32;
    return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

}  // namespace adock

using namespace adock;

static int gemm_args(GemmArgs& g, int M, int N, int K, const void* A, long long sAm, long long sAk, const void* B,
                     long long sBk, long long sBn, float* C, long long ldc, float beta, const float* bias, int act,
                     float* pre, void* Cb, long long ldcb) {
    ADOCK_CHECK_ARG(M >= 0 && N >= 0 && K >= 0, "negative GEMM size");
    ADOCK_CHECK_ARG(A && B && (C || Cb), "null GEMM operand");
    ADOCK_CHECK_ARG(act == 0 || act == 1, "act must be 0 (none) or 1 (SiLU)");
    ADOCK_CHECK_ARG(!pre || C, "pre-activation output needs C's leading dimension");
    g.M = M; g.N = N; g.K = K;
    g.A = (const __nv_bfloat16*)A; g.sAm = sAm; g.sAk = sAk;
    g.B = (const __nv_bfloat16*)B; g.sBk = sBk; g.sBn = sBn;
    g.C = C; g.ldc = ldc; g.beta = beta; g.bias = bias; g.act = act; g.pre = pre;
    g.Cb = (__nv_bfloat16*)Cb; g.ldcb = ldcb;
    return ADOCK_OK;
}

// Dynamic shared memory of the tcgen05 GEMM: tiles + 1024 bytes of alignment slack, rounded up so that at most
// 512 / TN CTAs are resident per SM (their TMEM allocations then always fit in the SM's 512 columns).
template <int TN>
static int launch_gemm_tc(const GemmArgs& g, cudaStream_t st) {
    const int per_sm = 512 / TN;
    const size_t smem = (size_t)(227 * 1024) / per_sm;
    static_assert(TC_BM * TC_BK * 2 + TN * TC_BK * 2 + 1024 <= 227 * 1024 / (512 / TN) - 256, "tile too large");
    ADOCK_CUDA(cudaFuncSetAttribute(gemm_bf16_tc_kernel<TN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((g.N + TN - 1) / TN, (g.M + TC_BM - 1) / TC_BM);
    ADOCK_CHECK_ARG(grid.y < 65536u, "M too large");
    gemm_bf16_tc_kernel<TN><<<grid, 128, smem, st>>>(g);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

extern "C" int adock_gemm_bf16(int M, int N, int K, const void* A, long long sAm, long long sAk, const void* B,
                               long long sBk, long long sBn, float* C, long long ldc, float beta, const float* bias,
                               int act, float* pre, void* Cb, long long ldcb, void* stream) {
    GemmArgs g;
    const int rc = gemm_args(g, M, N, K, A, sAm, sAk, B, sBk, sBn, C, ldc, beta, bias, act, pre, Cb, ldcb);
    if (rc != ADOCK_OK) return rc;
    if (M == 0 || N == 0) return ADOCK_OK;
    return N <= 64 ? launch_gemm_tc<64>(g, (cudaStream_t)stream) : launch_gemm_tc<128>(g, (cudaStream_t)stream);
}

extern "C" int adock_gemm_bf16_mma(int M, int N, int K, const void* A, long long sAm, long long sAk, const void* B,
                                   long long sBk, long long sBn, float* C, long long ldc, float beta,
                                   const float* bias, int act, float* pre, void* Cb, long long ldcb, void* stream) {
    GemmArgs g;
    const int rc = gemm_args(g, M, N, K, A, sAm, sAk, B, sBk, sBn, C, ldc, beta, bias, act, pre, Cb, ldcb);
    if (rc != ADOCK_OK) return rc;
    if (M == 0 || N == 0) return ADOCK_OK;
    dim3 grid((N + GN - 1) / GN, (M + GM - 1) / GM);
    ADOCK_CHECK_ARG(grid.y < 65536u, "M too large");
    gemm_bf16_kernel<<<grid, 128, 0, (cudaStream_t)stream>>>(g);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

extern "C" int adock_gemm_status(void) {
    int s = 0;
    ADOCK_CUDA(cudaMemcpyFromSymbol(&s, g_tc_status, sizeof(int)));
    if (s != 0) {
        const int zero = 0;
        ADOCK_CUDA(cudaMemcpyToSymbol(g_tc_status, &zero, sizeof(int)));
        set_error("a tcgen05 GEMM gave up waiting for its tensor-core work (mbarrier wait bound)");
        return ADOCK_E_DEVICE;
    }
    return ADOCK_OK;
}

extern "C" int adock_mlp_nll(const float* out, const float* target, int B, int n_comp, void* dout, float* loss,
                             void* stream) {
    ADOCK_CHECK_ARG(out && target && dout && loss && B >= 0, "bad argument");
    ADOCK_CHECK_ARG(n_comp == 1 || n_comp == 3, "n_comp must be 1 or 3 (got %d)", n_comp);
    if (B == 0) return ADOCK_OK;
    nll_kernel<<<(B + 3) / 4, 128, 0, (cudaStream_t)stream>>>(out, target, B, n_comp, (__nv_bfloat16*)dout, loss);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

extern "C" int adock_silu_backward(const float* dH, const float* A, long long n, void* dA, void* stream) {
    ADOCK_CHECK_ARG(dH && A && dA && n >= 0, "bad argument");
    if (n == 0) return ADOCK_OK;
    silu_backward_kernel<<<grid1d(n), 256, 0, (cudaStream_t)stream>>>(dH, A, n, (__nv_bfloat16*)dA);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

extern "C" int adock_bias_grad(const void* dA, int rows, int cols, float* db, void* stream) {
    ADOCK_CHECK_ARG(dA && db && rows >= 0 && cols >= 0, "bad argument");
    if (cols == 0) return ADOCK_OK;
    bias_grad_kernel<<<(cols + 31) / 32, 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)dA, rows, cols, db);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

extern "C" int adock_adam(float* p, const float* grad, float* m, float* v, void* pb, long long n, float lr, float b1,
                          float b2, float eps, int step, float wd, void* stream) {
    ADOCK_CHECK_ARG(p && grad && m && v && n >= 0 && step >= 1, "bad argument");
    if (n == 0) return ADOCK_OK;
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    adam_kernel<<<grid1d(n), 256, 0, (cudaStream_t)stream>>>(p, grad, m, v, (__nv_bfloat16*)pb, n, lr, b1, b2, eps, c1,
                                                             c2, wd);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

extern "C" int adock_f32_to_bf16(const float* x, void* y, long long n, void* stream) {
    ADOCK_CHECK_ARG(x && y && n >= 0, "bad argument");
    if (n == 0) return ADOCK_OK;
    f32_to_bf16_kernel<<<grid1d(n), 256, 0, (cudaStream_t)stream>>>(x, (__nv_bfloat16*)y, n);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}
