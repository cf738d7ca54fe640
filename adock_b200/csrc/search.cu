// Search entry points of the docking hot path (sm_100a): working-layout preparation (with the intra-pair round
// schedule), receptor neighbour lists, and the C-ABI of the energy/gradient, Monte-Carlo, Stage-A and float64
// re-score kernels. The grid-dtype-templated kernels live in search_impl.cuh and are instantiated in
// search_f32.cu / search_f16.cu / search_bf16.cu.
#include "search_impl.cuh"
#include <stdio.h>

namespace adock {

ADOCK_SEARCH_EXTERN(float)
ADOCK_SEARCH_EXTERN(__half)
ADOCK_SEARCH_EXTERN(__nv_bfloat16)

static inline int pad32(int x) { return ((x + 31) / 32) * 32; }

// ------------------------------------------------------------------------------------------ prepare
__global__ void prepare_kernel(adock_ligands_t lig, TypeTables tt, float4* atoms, uint32_t* masks, float4* tors,
                               int4* info, float* rg) {
    const int l = blockIdx.x;
    const int AM = lig.AM, KM = lig.KM;
    const int na = lig.na[l], nt = lig.nt[l], np = lig.np[l];
    for (int a = threadIdx.x; a < AM; a += blockDim.x) {
        const float* r = lig.ref + ((long long)l * AM + a) * 3;
        const int slot = lig.gslot[(long long)l * AM + a];
        const int typ = lig.typ[(long long)l * AM + a];
        const float4 v = make_float4(r[0], r[1], r[2], __int_as_float((slot & 0xffff) | (typ << 16)));
        uint32_t m = 0;
        if (a < na)
            for (int k = 0; k < nt && k < 32; ++k) m |= (lig.tm[((long long)l * KM + k) * AM + a] ? 1u : 0u) << k;
        atoms[(long long)l * AM + a] = v;
        masks[(long long)l * AM + a] = m;
    }
    for (int k = threadIdx.x; k < KM; k += blockDim.x) {
        const float* p = lig.axp + ((long long)l * KM + k) * 3;
        const float* u = lig.axu + ((long long)l * KM + k) * 3;
        const int* x = lig.ax + ((long long)l * KM + k) * 2;
        tors[((long long)l * KM + k) * 2] = make_float4(p[0], p[1], p[2], __int_as_float(x[0]));
        tors[((long long)l * KM + k) * 2 + 1] = make_float4(u[0], u[1], u[2], __int_as_float(x[1]));
    }
    if (threadIdx.x == 0) {
        info[l] = make_int4(na, nt, np, lig.rec_idx[l]);
        rg[l] = lig.rg[l];
    }
}

// Intra-pair schedule (one warp per ligand): the np pairs are placed into R = ceil(np / 32) rounds of 32 slots.
// eval_eg adds a pair's force to its first atom with one set of shared-memory atomics and to its second atom with
// another, so within a round only repeats of an atom on the same side collide (and serialise the atomic). The
// Vina pair term is symmetric, so each pair may also be stored either way round. Greedy in pair order: over the
// rounds with a free slot and both orientations, the choice where the larger of (the first atom's count as a first
// atom, the second atom's count as a second atom) is smallest, then their sum, then the lowest round, then the
// given orientation. Empty slots get x = -1. Counts live in dynamic shared memory, [R_cap][AM] per side; ligands
// with more than R_cap rounds keep the pair order.
__global__ void schedule_pairs_kernel(adock_ligands_t lig, TypeTables tt, int2* pairs, int P_pad, int R_cap) {
    extern __shared__ int sched_smem[];
    const int l = blockIdx.x, lane = threadIdx.x;
    const int np = lig.np[l], AM = lig.AM, P = lig.P;
    const int R = (np + 31) / 32;
    int* fill = sched_smem;                                            // [R_cap]
    unsigned char* c1 = (unsigned char*)(sched_smem + R_cap);          // [R_cap][AM] count as first atom
    unsigned char* c2 = c1 + (size_t)R_cap * AM;                       // [R_cap][AM] count as second atom
    int2* out = pairs + (long long)l * P_pad;
    auto record = [&](int q, int swap) {
        const int i = lig.pr[((long long)l * P + q) * 2], j = lig.pr[((long long)l * P + q) * 2 + 1];
        int ti = lig.typ[(long long)l * AM + i], tj = lig.typ[(long long)l * AM + j];
        ti = ti < 0 ? 0 : (ti & 63);
        tj = tj < 0 ? 0 : (tj & 63);
        const int fl = hyd_pair(tt.flags[ti], tt.flags[tj]) | hb_pair(tt.flags[ti], tt.flags[tj]);
        const int a = swap ? j : i, b = swap ? i : j;
        return make_int2((a & 0xff) | ((b & 0xff) << 8) | (fl << 16), __float_as_int(tt.radius[ti] + tt.radius[tj]));
    };
    if (R > R_cap) {  // very large ligands: keep the pair order
        for (int q = lane; q < P_pad; q += 32) out[q] = q < np ? record(q, 0) : make_int2(-1, 0);
        return;
    }
    for (int r = lane; r < R; r += 32) {
        fill[r] = 0;
        for (int a = 0; a < AM; ++a) {
            c1[(size_t)r * AM + a] = 0;
            c2[(size_t)r * AM + a] = 0;
        }
    }
    __syncwarp();
    for (int q = 0; q < np; ++q) {
        const int i = lig.pr[((long long)l * P + q) * 2] % AM, j = lig.pr[((long long)l * P + q) * 2 + 1] % AM;
        unsigned best = 0xffffffffu;
        for (int r = lane; r < R; r += 32) {
            if (fill[r] < 32) {
#pragma unroll
                for (int o = 0; o < 2; ++o) {
                    const unsigned x = c1[(size_t)r * AM + (o ? j : i)], y = c2[(size_t)r * AM + (o ? i : j)];
                    const unsigned key = (((x > y ? x : y) * 64u + x + y) << 17) | ((unsigned)r << 1) | (unsigned)o;
                    best = key < best ? key : best;
                }
            }
        }
        best = __reduce_min_sync(0xffffffffu, best);
        const int found = (int)((best >> 1) & 0xffffu), o = (int)(best & 1u);
        if (lane == 0) {
            const int slot = found * 32 + fill[found];
            fill[found] += 1;
            c1[(size_t)found * AM + (o ? j : i)] += 1;
            c2[(size_t)found * AM + (o ? i : j)] += 1;
            out[slot] = record(q, o);
        }
        __syncwarp();
    }
    for (int q = lane; q < P_pad; q += 32) {
        const int r = q >> 5;
        if (r >= R || (q & 31) >= fill[r]) out[q] = make_int2(-1, 0);
    }
}

// ------------------------------------------------------------------------------------------ pose coordinates
// World coordinates of the heavy atoms of one state (one warp), float32 path of eval_eg.
__device__ void pose_world(const SearchParams& P, int l, const float* s, float4* Xout, int lane) {
    const int4 inf = P.info[l];
    const int na = inf.x, nt = inf.y;
    float qw = s[3], qx = s[4], qy = s[5], qz = s[6];
    const float nq = rsqrtf(qw * qw + qx * qx + qy * qy + qz * qz);
    qw *= nq; qx *= nq; qy *= nq; qz *= nq;
    const float R00 = 1 - 2 * (qy * qy + qz * qz), R01 = 2 * (qx * qy - qz * qw), R02 = 2 * (qx * qz + qy * qw);
    const float R10 = 2 * (qx * qy + qz * qw), R11 = 1 - 2 * (qx * qx + qz * qz), R12 = 2 * (qy * qz - qx * qw);
    const float R20 = 2 * (qx * qz - qy * qw), R21 = 2 * (qy * qz + qx * qw), R22 = 1 - 2 * (qx * qx + qy * qy);
    const float4* tr = P.tors + (long long)l * P.KM * 2;
    for (int a = lane; a < na; a += 32) {
        const float4 v = P.atoms[(long long)l * P.AM + a];
        float px = v.x, py = v.y, pz = v.z;
        uint32_t m = P.masks[(long long)l * P.AM + a];
        while (m) {
            const int k = __ffs(m) - 1;
            m &= m - 1;
            if (k >= nt) break;
            const float4 A = tr[2 * k], U = tr[2 * k + 1];
            float sv, cv;
            __sincosf(s[7 + k], &sv, &cv);
            const float vx = px - A.x, vy = py - A.y, vz = pz - A.z;
            const float d = U.x * vx + U.y * vy + U.z * vz;
            const float cx = U.y * vz - U.z * vy, cy = U.z * vx - U.x * vz, cz = U.x * vy - U.y * vx;
            px = A.x + vx * cv + cx * sv + U.x * d * (1 - cv);
            py = A.y + vy * cv + cy * sv + U.y * d * (1 - cv);
            pz = A.z + vz * cv + cz * sv + U.z * d * (1 - cv);
        }
        Xout[a] = make_float4(R00 * px + R01 * py + R02 * pz + s[0], R10 * px + R11 * py + R12 * pz + s[1],
                              R20 * px + R21 * py + R22 * pz + s[2], v.w);
    }
    __syncwarp();
}

// ------------------------------------------------------------------------------------------ neighbour lists
// Block per chain: heavy-atom world coordinates in shared memory, threads over receptor atoms; pass 1 counts,
// pass 2 writes the indices in receptor order (ordered block compaction).
__global__ void __launch_bounds__(256) neighbours_kernel(const __grid_constant__ SearchParams P, const int* chain_lig,
                                                         int n, const float* state, float cut2, int* nbr, int* nbr_n,
                                                         int nb_max) {
    extern __shared__ float4 smem4[];
    float4* X = smem4;  // [AM]
    __shared__ float s[7 + 32];
    __shared__ int wsum[8];
    __shared__ int base_sh;
    const int ch = blockIdx.x;
    const int l = chain_lig[ch];
    const int SDM = 7 + P.KM;
    const int4 inf = P.info[l];
    const int na = inf.x, ri = inf.w;
    for (int i = threadIdx.x; i < 7 + min(P.KM, 32); i += blockDim.x) s[i] = state[(long long)ch * SDM + i];
    __syncthreads();
    if (threadIdx.x < 32) pose_world(P, l, s, X, threadIdx.x);
    __syncthreads();
    const float* rx = P.rxyz + (long long)ri * P.RN * 3;
    const int rn = P.rn[ri];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x == 0) base_sh = 0;
    __syncthreads();
    for (int r0 = 0; r0 < rn; r0 += blockDim.x) {
        const int r = r0 + threadIdx.x;
        bool near = false;
        if (r < rn) {
            const float x = rx[3 * r], y = rx[3 * r + 1], z = rx[3 * r + 2];
            for (int a = 0; a < na && !near; ++a) {
                const float4 v = X[a];
                const float dx = v.x - x, dy = v.y - y, dz = v.z - z;
                near = (dx * dx + dy * dy + dz * dz) < cut2;
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, near);
        if (lane == 0) wsum[wid] = __popc(bal);
        __syncthreads();
        int off = base_sh;
        for (int w = 0; w < wid; ++w) off += wsum[w];
        if (near && nbr) {
            const int pos = off + __popc(bal & ((1u << lane) - 1u));
            if (pos < nb_max) nbr[(long long)ch * nb_max + pos] = r;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < nw; ++w) t += wsum[w];
            base_sh += t;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) nbr_n[ch] = base_sh;
}

// ------------------------------------------------------------------------------------------ proposal sampling
// One thread per (chain c, slot kk): move d = mean[c, d] + max(exp(clamp(log_sd[c, d], -4, 2)), floor_d) * z with
// z ~ N(0, 1) by Box-Muller on the counter-based stream (seed, chain id, 64 * segment + kk, 2 d / 2 d + 1), applied
// to the chain's state: t + d[0:3], exp(d[3:6]) q, theta + d[6:26] below the torsion count (theta kept above it).
// The floors on the spread (0.5 A, 0.25 rad, 0.5 rad) keep the proposals exploring.
__global__ void prop_sample_kernel(const int4* info, const int* chain_lig, const int* chain_id, int n,
                                   const float* out, const float* state, int SD, int k, int n_comp,
                                   unsigned long long seed, int segment, float* targets) {
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)n * k) return;
    const int kk = (int)(idx % k);
    const int c = (int)(idx / k);
    const int nt = info[chain_lig[c]].y;
    const int cid = chain_id[c], step = (k > 64 ? k : 64) * segment + kk;
    const float* o = out + (long long)c * 64;
    const float* s = state + (long long)c * SD;
    float d[26];
#pragma unroll
    for (int j = 0; j < 26; ++j) {
        d[j] = 0.f;
        if (j < 6 || j - 6 < nt) {
            const float u1 = fmaxf(uniform01(seed, cid, step, 2 * j), 1e-7f);
            const float u2 = uniform01(seed, cid, step, 2 * j + 1);
            const float z = sqrtf(-2.f * __logf(u1)) * __cosf(6.28318531f * u2);
            const float ls = fminf(fmaxf(o[32 + j], -4.f), 2.f);
            const float floor_sd = j < 3 ? 0.5f : (j < 6 ? 0.25f : 0.5f);
            d[j] = o[j] + fmaxf(__expf(ls), floor_sd) * z;
        }
    }
    if (n_comp == 3) {
        // translation mixture: component by its softmax weight (mean columns 0, 27, 58; logits 26, 30, 61), the
        // same standard-normal draws and spread as the single Gaussian
        const float g0 = o[26], g1 = o[30], g2 = o[61];
        const float m = fmaxf(g0, fmaxf(g1, g2));
        const float w0 = __expf(g0 - m), w1 = __expf(g1 - m), w2 = __expf(g2 - m);
        const float u = uniform01(seed, cid, step, 52) * (w0 + w1 + w2);
        const int mc = u < w0 ? 0 : (u < w0 + w1 ? 27 : 58);
        for (int j = 0; j < 3; ++j) d[j] += o[mc + j] - o[j];
    }
    float* y = targets + idx * PROP_MOVE;
    y[0] = s[0] + d[0]; y[1] = s[1] + d[1]; y[2] = s[2] + d[2];
    float q[4] = {s[3], s[4], s[5], s[6]};
    quat_apply_rotvec(q, d[3], d[4], d[5]);
    y[3] = q[0]; y[4] = q[1]; y[5] = q[2]; y[6] = q[3];
#pragma unroll
    for (int t = 0; t < 20; ++t) y[7 + t] = (7 + t < SD) ? s[7 + t] + (t < nt ? d[6 + t] : 0.f) : 0.f;
#pragma unroll
    for (int t = 27; t < PROP_MOVE; ++t) y[t] = 0.f;
}

// ------------------------------------------------------------------------------------------ host side
TypeTables make_tables(const adock_sf_t* sf) {
    TypeTables t;
    for (int i = 0; i < 64; ++i) {
        t.radius[i] = i < sf->n_types ? sf->radius[i] : 0.f;
        t.flags[i] = i < sf->n_types ? ((sf->hyd[i] ? 1 : 0) | (sf->don[i] ? 2 : 0) | (sf->acc[i] ? 4 : 0)) : 0;
    }
    return t;
}

int make_params(SearchParams& P, const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
                       const adock_sf_t* sf, const adock_receptors_t* rec) {
    ADOCK_CHECK_ARG(lig && work && sf, "null ligand/work/sf argument");
    ADOCK_CHECK_ARG(lig->AM % 32 == 0 && lig->AM >= 32 && lig->AM <= 128, "AM must be 32, 64, 96 or 128 (got %d)", lig->AM);
    ADOCK_CHECK_ARG(lig->KM >= 1 && lig->KM <= 32, "KM must be in [1, 32] (got %d)", lig->KM);
    ADOCK_CHECK_ARG(lig->P >= 1, "P must be >= 1");
    ADOCK_CHECK_ARG(sf->n_types >= 1 && sf->n_types <= 64, "n_types must be in [1, 64]");
    P.atoms = (const float4*)work->atoms;
    P.masks = (const uint32_t*)work->masks;
    P.tors = (const float4*)work->tors;
    P.pairs = (const int2*)work->pairs;
    P.info = (const int4*)work->info;
    P.rg = (const float*)work->rg;
    P.AM = lig->AM; P.KM = lig->KM; P.P = lig->P; P.P_pad = pad32(lig->P);
    if (grids) {
        P.flat = grids->flat; P.offs = grids->offs; P.dims = grids->dims;
        P.origin = grids->origin; P.lo = grids->lo; P.hi = grids->hi;
        P.inv_s = 1.f / grids->spacing; P.pen = grids->penalty;
        P.nmaps = grids->nmaps;
    } else {
        P.flat = nullptr; P.offs = nullptr; P.dims = nullptr; P.origin = P.lo = P.hi = nullptr;
        P.inv_s = 1.f; P.pen = 0.f;
        P.nmaps = nullptr;
    }
    if (rec && rec->xyz) {
        P.rxyz = rec->xyz; P.rtyp = rec->typ; P.rn = rec->n; P.RN = rec->RN;
    } else {
        P.rxyz = nullptr; P.rtyp = nullptr; P.rn = nullptr; P.RN = 0;
    }
    P.pp = make_pair_prm(sf->prm);
    P.n_types = sf->n_types;
    return ADOCK_OK;
}

}  // namespace adock

using namespace adock;

extern "C" int adock_prepare(const adock_ligands_t* lig, const adock_sf_t* sf, adock_work_t* work, void* stream) {
    ADOCK_CHECK_ARG(lig && sf && work, "null argument");
    ADOCK_CHECK_ARG(lig->L >= 1, "L must be >= 1");
    ADOCK_CHECK_ARG(lig->AM % 32 == 0 && lig->AM >= 32 && lig->AM <= 128, "AM must be 32, 64, 96 or 128 (got %d)", lig->AM);
    ADOCK_CHECK_ARG(lig->KM >= 1 && lig->KM <= 32, "KM must be in [1, 32] (got %d)", lig->KM);
    ADOCK_CHECK_ARG(lig->P >= 1, "P must be >= 1");
    ADOCK_CHECK_ARG(sf->n_types >= 1 && sf->n_types <= 64, "n_types must be in [1, 64]");
    ADOCK_CHECK_ARG(work->atoms && work->masks && work->tors && work->pairs && work->info && work->rg, "null work buffer");
    const TypeTables tt = make_tables(sf);
    cudaStream_t st = (cudaStream_t)stream;
    prepare_kernel<<<lig->L, 128, 0, st>>>(*lig, tt, (float4*)work->atoms, (uint32_t*)work->masks, (float4*)work->tors,
                                           (int4*)work->info, (float*)work->rg);
    ADOCK_CUDA(cudaGetLastError());
    const int R_cap = min(pad32(lig->P) / 32, PAIR_ROUNDS_MAX);
    const size_t sched_smem = (size_t)R_cap * sizeof(int) + 2 * (size_t)R_cap * lig->AM;
    ADOCK_CUDA(cudaFuncSetAttribute(schedule_pairs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)sched_smem));
    schedule_pairs_kernel<<<lig->L, 32, sched_smem, st>>>(*lig, tt, (int2*)work->pairs, pad32(lig->P), R_cap);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

extern "C" int adock_eg(const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
                        const adock_sf_t* sf, const adock_receptors_t* rec, const int* chain_lig, int n,
                        const float* state, float* e_out, float* g_out, int exact, void* stream) {
    SearchParams P;
    int rc = make_params(P, lig, work, grids, sf, rec);
    if (rc) return rc;
    ADOCK_CHECK_ARG(grids && grids->flat, "grids are required");
    ADOCK_CHECK_ARG(!exact || P.rxyz, "exact mode needs receptor atoms");
    ADOCK_CHECK_ARG(n >= 0, "n must be >= 0");
    if (n == 0) return ADOCK_OK;
    ADOCK_CHECK_ARG(chain_lig && state && e_out && g_out, "null array argument");
    const TypeTables tt = make_tables(sf);
    cudaStream_t st = (cudaStream_t)stream;
    switch (grids->dtype) {
        case ADOCK_GRID_F32: return launch_eg<float>(P, chain_lig, n, state, e_out, g_out, exact, tt, st);
        case ADOCK_GRID_F16: return launch_eg<__half>(P, chain_lig, n, state, e_out, g_out, exact, tt, st);
        case ADOCK_GRID_BF16: return launch_eg<__nv_bfloat16>(P, chain_lig, n, state, e_out, g_out, exact, tt, st);
    }
    ADOCK_CHECK_ARG(false, "unknown grid dtype %d", grids->dtype);
}

extern "C" int adock_mc(const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
                        const adock_sf_t* sf, const adock_receptors_t* rec, const adock_mc_args_t* mc, void* stream) {
    SearchParams P;
    int rc = make_params(P, lig, work, grids, sf, rec);
    if (rc) return rc;
    ADOCK_CHECK_ARG(mc, "null mc argument");
    ADOCK_CHECK_ARG(grids && grids->flat, "grids are required");
    ADOCK_CHECK_ARG(!mc->exact || P.rxyz, "exact mode needs receptor atoms");
    ADOCK_CHECK_ARG(mc->n_chains >= 0 && mc->mc_steps >= 0, "negative size");
    if (mc->n_chains == 0) return ADOCK_OK;
    ADOCK_CHECK_ARG(mc->chain_lig && mc->chain_id && mc->cur && mc->cur_e && mc->best && mc->best_e && mc->queue,
                    "null array argument");
    ADOCK_CHECK_ARG(!mc->nbr || mc->nbr_n, "nbr without nbr_n");
    ADOCK_CHECK_ARG(mc->temp > 0.f, "temperature must be > 0");
    ADOCK_CHECK_ARG(mc->variant >= 0 && mc->variant < 4, "variant must be in [0, 3]");
    McParams M;
    M.chain_lig = mc->chain_lig; M.chain_id = mc->chain_id; M.n_chains = mc->n_chains;
    M.nbr = mc->nbr; M.nbr_n = mc->nbr_n; M.nb_max = mc->nb_max;
    M.cur = mc->cur; M.cur_e = mc->cur_e; M.best = mc->best; M.best_e = mc->best_e;
    M.init_opt = mc->init_opt; M.mc_steps = mc->mc_steps; M.bfgs_iters = mc->bfgs_iters;
    M.temp = mc->temp; M.amp_pos = mc->amp_pos; M.amp_rot = mc->amp_rot; M.seed = mc->seed;
    M.step_offset = mc->step_offset; M.exact = mc->exact; M.order = mc->order; M.queue = mc->queue; M.evals = mc->evals;
    ADOCK_CHECK_ARG(!mc->prop || mc->prop_k >= 1, "prop_k must be >= 1 with proposals");
    ADOCK_CHECK_ARG(!mc->log_x || (mc->log_y && mc->log_n && mc->log_cap >= 0), "incomplete training-data log");
    M.prop = mc->prop; M.prop_k = mc->prop_k; M.prop_stats = mc->prop_stats;
    M.prop_frac = (mc->prop_frac <= 0.f || mc->prop_frac >= 1.f) ? 1.f : mc->prop_frac;
    M.log_x = (__nv_bfloat16*)mc->log_x; M.log_y = mc->log_y; M.log_n = mc->log_n; M.log_cap = mc->log_cap;
    M.lig_active = mc->lig_active;
    M.hint = mc->hint;
    M.prop_tries = mc->prop_tries > 1 ? mc->prop_tries : 1;
    ADOCK_CHECK_ARG(!mc->prop || mc->prop_k % M.prop_tries == 0, "prop_k must be a multiple of prop_tries");
    const TypeTables tt = make_tables(sf);
    cudaStream_t st = (cudaStream_t)stream;
    switch (grids->dtype) {
        case ADOCK_GRID_F32: return launch_mc<float>(P, M, tt, st, mc->variant);
        case ADOCK_GRID_F16: return launch_mc<__half>(P, M, tt, st, mc->variant);
        case ADOCK_GRID_BF16: return launch_mc<__nv_bfloat16>(P, M, tt, st, mc->variant);
    }
    ADOCK_CHECK_ARG(false, "unknown grid dtype %d", grids->dtype);
}

static int stage_a_common(const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
                          const adock_sf_t* sf, const float* conf, int C, const float* quats, int Q, const float* trans,
                          const int* ntrans, int nt_max, const int* lig_box, float cap, float* best_e, int* best_i,
                          void* stream) {
    SearchParams P;
    int rc = make_params(P, lig, work, grids, sf, nullptr);
    if (rc) return rc;
    ADOCK_CHECK_ARG(grids && grids->flat, "grids are required");
    ADOCK_CHECK_ARG(C >= 1 && Q >= 1 && nt_max >= 1, "C, Q and nt_max must be >= 1");
    ADOCK_CHECK_ARG(conf && quats && trans && ntrans && best_e && best_i, "null array argument");
    const long long blocks = (long long)lig->L * C * Q;
    ADOCK_CHECK_ARG(blocks < (1LL << 31), "too many Stage-A blocks");
    cudaStream_t st = (cudaStream_t)stream;
    switch (grids->dtype) {
        case ADOCK_GRID_F32:
            return launch_stage_a<float>(P, blocks, conf, C, quats, Q, trans, ntrans, nt_max, lig_box, cap, best_e,
                                         best_i, st);
        case ADOCK_GRID_F16:
            return launch_stage_a<__half>(P, blocks, conf, C, quats, Q, trans, ntrans, nt_max, lig_box, cap, best_e,
                                          best_i, st);
        case ADOCK_GRID_BF16:
            return launch_stage_a<__nv_bfloat16>(P, blocks, conf, C, quats, Q, trans, ntrans, nt_max, lig_box, cap,
                                                 best_e, best_i, st);
    }
    ADOCK_CHECK_ARG(false, "unknown grid dtype %d", grids->dtype);
}

extern "C" int adock_stage_a(const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
                             const adock_sf_t* sf, const float* conf, int C, const float* quats, int Q,
                             const float* trans, const int* ntrans, int nt_max, float cap, float* best_e, int* best_i,
                             void* stream) {
    return stage_a_common(lig, work, grids, sf, conf, C, quats, Q, trans, ntrans, nt_max, nullptr, cap, best_e, best_i,
                          stream);
}

extern "C" int adock_stage_a_boxes(const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
                                   const adock_sf_t* sf, const float* conf, int C, const float* quats, int Q,
                                   const float* trans, const int* ntrans, int nt_max, const int* lig_box, float cap,
                                   float* best_e, int* best_i, void* stream) {
    ADOCK_CHECK_ARG(lig_box, "null lig_box");
    return stage_a_common(lig, work, grids, sf, conf, C, quats, Q, trans, ntrans, nt_max, lig_box, cap, best_e, best_i,
                          stream);
}

extern "C" int adock_neighbours(const adock_ligands_t* lig, const adock_work_t* work, const adock_sf_t* sf,
                                const adock_receptors_t* rec, const int* chain_lig, int n, const float* state,
                                float cut, int* nbr, int* nbr_n, int nb_max, void* stream) {
    SearchParams P;
    int rc = make_params(P, lig, work, nullptr, sf, rec);
    if (rc) return rc;
    ADOCK_CHECK_ARG(P.rxyz, "receptor atoms are required");
    ADOCK_CHECK_ARG(n >= 0, "n must be >= 0");
    if (n == 0) return ADOCK_OK;
    ADOCK_CHECK_ARG(chain_lig && state && nbr_n, "null array argument");
    ADOCK_CHECK_ARG(!nbr || nb_max >= 1, "nb_max must be >= 1");
    const size_t smem = (size_t)P.AM * sizeof(float4);
    neighbours_kernel<<<n, 256, smem, (cudaStream_t)stream>>>(P, chain_lig, n, state, cut * cut, nbr, nbr_n, nb_max);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

extern "C" int adock_rescore64(const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
                               const adock_sf_t* sf, const adock_receptors_t* rec, const int* chain_lig, int n,
                               const float* state, double* e_total, double* e_intra, float* X, void* stream) {
    SearchParams P;
    int rc = make_params(P, lig, work, grids, sf, rec);
    if (rc) return rc;
    ADOCK_CHECK_ARG(n >= 0, "n must be >= 0");
    if (n == 0) return ADOCK_OK;
    ADOCK_CHECK_ARG(chain_lig && state && e_total && e_intra && X, "null array argument");
    ADOCK_CHECK_ARG(P.rxyz || (grids && grids->flat), "grids or receptor atoms are required");
    const TypeTables tt = make_tables(sf);
    cudaStream_t st = (cudaStream_t)stream;
    const int dt = grids ? grids->dtype : ADOCK_GRID_F32;
    switch (dt) {
        case ADOCK_GRID_F32: return launch_rescore64<float>(P, chain_lig, n, state, e_total, e_intra, X, tt, *sf, st);
        case ADOCK_GRID_F16: return launch_rescore64<__half>(P, chain_lig, n, state, e_total, e_intra, X, tt, *sf, st);
        case ADOCK_GRID_BF16:
            return launch_rescore64<__nv_bfloat16>(P, chain_lig, n, state, e_total, e_intra, X, tt, *sf, st);
    }
    ADOCK_CHECK_ARG(false, "unknown grid dtype %d", dt);
}

// ------------------------------------------------------------------------------------------ no-allocation MC
// Some callers cannot allocate device memory: code that runs while a CUDA stream is being captured into a graph
// by a framework that forbids allocations during capture, embedders whose memory pool owns every device byte, or
// callers that only receive raw input/output pointers from a host application. adock_mc needs caller-allocated
// scratch (the B200 working layout of the ligand batch and a one-word work-queue counter); this variant keeps that
// scratch in one fixed-size device array instead, so the caller passes only inputs and outputs.
//
// The array lives for the whole process on every device that loads the library. In host code its name is only
// a host-side stand-in; the device address comes from cudaGetSymbolAddress, taken once per device on the first
// call with that device current (so the first call on a device should come before any stream capture). Every
// call reuses the same array: the work counter is cleared by each call, the working layout is rewritten by each
// call, and calls that overlap on the GPU (different streams, or other threads) race on it.
#define ADOCK_NOALLOC_SCRATCH_BYTES ADOCK_NOALLOC_SCRATCH_MAX

static __device__ __align__(256) unsigned char g_noalloc_scratch[ADOCK_NOALLOC_SCRATCH_BYTES];

namespace adock {
static void* g_noalloc_ptr[64];
static int g_noalloc_ready[64];

static size_t round256(size_t x) { return (x + 255) & ~(size_t)255; }

static int noalloc_scratch(void** out) {
    int dev = 0;
    ADOCK_CUDA(cudaGetDevice(&dev));
    ADOCK_CHECK_ARG(dev >= 0 && dev < 64, "device index %d out of range", dev);
    if (!__atomic_load_n(&g_noalloc_ready[dev], __ATOMIC_ACQUIRE)) {
        void* p = nullptr;
        ADOCK_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_ptr[dev] = p;
        __atomic_store_n(&g_noalloc_ready[dev], 1, __ATOMIC_RELEASE);
    }
    *out = g_noalloc_ptr[dev];
    return ADOCK_OK;
}
}  // namespace adock

extern "C" size_t adock_mc_noalloc_scratch_bytes(int L, int AM, int KM, int P) {
    using adock::round256;
    return round256(sizeof(int)) + round256((size_t)L * AM * 16) + round256((size_t)L * AM * 4) +
           round256((size_t)L * KM * 32) + round256((size_t)L * pad32(P) * 8) + round256((size_t)L * 16) +
           round256((size_t)L * 4);
}

extern "C" int adock_mc_noalloc(const adock_ligands_t* lig, const adock_grids_t* grids, const adock_sf_t* sf,
                                const adock_receptors_t* rec, const adock_mc_args_t* mc, void* stream) {
    ADOCK_CHECK_ARG(lig && grids && sf && mc, "null argument");
    ADOCK_CHECK_ARG(lig->L >= 1 && lig->AM >= 32 && lig->KM >= 1 && lig->P >= 1, "bad ligand batch dimensions");
    const size_t need = adock_mc_noalloc_scratch_bytes(lig->L, lig->AM, lig->KM, lig->P);
    ADOCK_CHECK_ARG(need <= ADOCK_NOALLOC_SCRATCH_BYTES,
                    "batch needs %zu bytes of scratch; adock_mc_noalloc holds at most %u (use adock_mc)", need,
                    (unsigned)ADOCK_NOALLOC_SCRATCH_BYTES);
    void* base = nullptr;
    int rc = noalloc_scratch(&base);
    if (rc) return rc;
    unsigned char* p = (unsigned char*)base;
    int* queue = (int*)p;
    p += round256(sizeof(int));
    adock_work_t work;
    work.atoms = p; p += round256((size_t)lig->L * lig->AM * 16);
    work.masks = p; p += round256((size_t)lig->L * lig->AM * 4);
    work.tors = p;  p += round256((size_t)lig->L * lig->KM * 32);
    work.pairs = p; p += round256((size_t)lig->L * pad32(lig->P) * 8);
    work.info = p;  p += round256((size_t)lig->L * 16);
    work.rg = p;
    rc = adock_prepare(lig, sf, &work, stream);
    if (rc) return rc;
    adock_mc_args_t m = *mc;
    m.queue = queue;   // adock_mc clears the counter on `stream` before its launch
    return adock_mc(lig, &work, grids, sf, rec, &m, stream);
}

// ------------------------------------------------------------------------------------------ proposal entry points
extern "C" int adock_prop_features(const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
                                   const adock_sf_t* sf, const int* chain_lig, int n, const float* state,
                                   const float* cur_e, const float* hint, void* feat, void* stream) {
    SearchParams P;
    int rc = make_params(P, lig, work, grids, sf, nullptr);
    if (rc) return rc;
    ADOCK_CHECK_ARG(grids && grids->flat, "grids are required");
    ADOCK_CHECK_ARG(n >= 0, "n must be >= 0");
    if (n == 0) return ADOCK_OK;
    ADOCK_CHECK_ARG(chain_lig && state && feat, "null array argument");
    cudaStream_t st = (cudaStream_t)stream;
    __nv_bfloat16* out = (__nv_bfloat16*)feat;
    switch (grids->dtype) {
        case ADOCK_GRID_F32: return launch_prop_features<float>(P, chain_lig, n, state, cur_e, hint, out, st);
        case ADOCK_GRID_F16: return launch_prop_features<__half>(P, chain_lig, n, state, cur_e, hint, out, st);
        case ADOCK_GRID_BF16:
            return launch_prop_features<__nv_bfloat16>(P, chain_lig, n, state, cur_e, hint, out, st);
    }
    ADOCK_CHECK_ARG(false, "unknown grid dtype %d", grids->dtype);
}

// Ligand-best rows of the proposal features. Pass 1 reduces, per ligand, the key (order-preserving bits of the
// chain's best energy << 32 | chain index) with atomicMin, so ties go to the lowest chain index and non-finite
// energies never win; pass 2 copies the winning chain's best state (t, q, torsions 0..19), its energy and a valid
// flag into hint[l].
namespace adock {
__device__ __forceinline__ unsigned long long energy_key(float e, int ch) {
    const unsigned u = __float_as_uint(e);
    const unsigned o = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return ((unsigned long long)o << 32) | (unsigned)ch;
}

__global__ void prop_hint_reduce_kernel(int n, const int* chain_lig, const float* best_e, int L,
                                        unsigned long long* keys) {
    const int ch = blockIdx.x * blockDim.x + threadIdx.x;
    if (ch >= n) return;
    const int l = chain_lig[ch];
    const float e = best_e[ch];
    if (l < 0 || l >= L || !isfinite(e)) return;
    atomicMin(keys + l, energy_key(e, ch));
}

__global__ void prop_hint_copy_kernel(int L, const unsigned long long* keys, const float* best, int SD,
                                      const float* best_e, float* hint) {
    const int l = blockIdx.x;
    const unsigned long long key = keys[l];
    const bool ok = key != ~0ull;
    const int ch = (int)(key & 0xffffffffull);
    float* h = hint + (long long)l * PROP_HINT;
    for (int i = threadIdx.x; i < PROP_HINT; i += blockDim.x) {
        float v = 0.f;
        if (ok) {
            if (i < 27 && i < SD) v = best[(long long)ch * SD + i];
            else if (i == 27) v = best_e[ch];
            else if (i == 28) v = 1.f;
        }
        h[i] = v;
    }
}
}  // namespace adock

extern "C" int adock_prop_hint(int L, int n, const int* chain_lig, const float* best, int SD, const float* best_e,
                               void* keys, float* hint, void* stream) {
    ADOCK_CHECK_ARG(L >= 0 && n >= 0, "negative size");
    ADOCK_CHECK_ARG(SD >= 7, "SD must be >= 7");
    if (L == 0) return ADOCK_OK;
    ADOCK_CHECK_ARG(keys && hint && (n == 0 || (chain_lig && best && best_e)), "null array argument");
    cudaStream_t st = (cudaStream_t)stream;
    ADOCK_CUDA(cudaMemsetAsync(keys, 0xff, (size_t)L * sizeof(unsigned long long), st));
    if (n > 0) {
        prop_hint_reduce_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, chain_lig, best_e, L,
                                                                            (unsigned long long*)keys);
        ADOCK_CUDA(cudaGetLastError());
    }
    prop_hint_copy_kernel<<<(unsigned)L, 32, 0, st>>>(L, (const unsigned long long*)keys, best, SD, best_e, hint);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

extern "C" int adock_prop_sample(const adock_ligands_t* lig, const adock_work_t* work, const int* chain_lig,
                                 const int* chain_id, int n, const float* net_out, const float* state, int SD, int k,
                                 int n_comp, unsigned long long seed, int segment, float* targets, void* stream) {
    ADOCK_CHECK_ARG(lig && work && work->info, "null argument");
    ADOCK_CHECK_ARG(n >= 0 && k >= 1 && k <= 512, "n must be >= 0 and k in [1, 512]");
    ADOCK_CHECK_ARG(n_comp == 1 || n_comp == 3, "n_comp must be 1 or 3 (got %d)", n_comp);
    ADOCK_CHECK_ARG(SD >= 7, "SD must be >= 7");
    if (n == 0) return ADOCK_OK;
    ADOCK_CHECK_ARG(chain_lig && chain_id && net_out && state && targets, "null array argument");
    const long long total = (long long)n * k;
    const unsigned blocks = (unsigned)((total + 127) / 128);
    prop_sample_kernel<<<blocks, 128, 0, (cudaStream_t)stream>>>((const int4*)work->info, chain_lig, chain_id, n,
                                                                 net_out, state, SD, k, n_comp, seed, segment,
                                                                 targets);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}
