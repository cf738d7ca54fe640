// Device-side search pipeline around the MC kernel (sm_100a): Stage-A conformers, the probe-filtered translation
// lattice, start-state selection, per-segment budget / early-stop bookkeeping, greedy pose clustering and all-atom
// output coordinates. With these the whole search (Stage A -> MC segments -> refine -> polish -> finalize) runs as
// a fixed sequence of launches on one stream, with no host round trip between the stages.
//
// Work decomposition: one CTA per ligand (conformers, start selection, clustering) or per box (lattice); one warp
// per pose (all-atom coordinates). All inputs are small next to the MC phase (< 0.5 % of a search); the kernels
// exist to take the host out of the loop, so they favour simple block-local sorts and scans over throughput.
#include "search_impl.cuh"

namespace adock {

__host__ __device__ inline int pad32i(int x) { return ((x + 31) / 32) * 32; }
static inline int pow2_at_least(int x) {
    int p = 1;
    while (p < x) p <<= 1;
    return p;
}

// ------------------------------------------------------------------------------------------ block primitives
// Ascending bitonic sort of (key, index) pairs in shared memory; n is a power of two; ties break on the index, so
// the order is the stable order of the keys.
template <typename K>
__device__ void block_sort_pairs(K* key, int* idx, int n) {
    for (int k = 2; k <= n; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < n; i += blockDim.x) {
                const int p = i ^ j;
                if (p > i) {
                    const bool up = (i & k) == 0;
                    const K a = key[i], b = key[p];
                    const int ia = idx[i], ib = idx[p];
                    const bool greater = (a > b) || (a == b && ia > ib);
                    if (greater == up) {
                        key[i] = b; key[p] = a;
                        idx[i] = ib; idx[p] = ia;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Exclusive prefix sum of one flag per thread over the block (blockDim.x <= 1024); returns the thread's offset and
// writes the block total into *total (shared).
__device__ int block_exclusive_scan(int flag, int* warp_tot, int* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    const unsigned bal = __ballot_sync(0xffffffffu, flag);
    const int in_warp = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) warp_tot[wid] = __popc(bal);
    __syncthreads();
    if (wid == 0) {
        int v = lane < nw ? warp_tot[lane] : 0;
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane < nw) warp_tot[lane] = incl - v;
        if (lane == 31) *total = incl;
    }
    __syncthreads();
    const int off = warp_tot[wid] + in_warp;
    __syncthreads();
    return off;
}

// ------------------------------------------------------------------------------------------ conformers
// Ligand-frame heavy-atom coordinates of torsion set `trial` of ligand l into X ([3][AM] in shared memory) and
// the set's torsion angles into th (shared, KM); returns the intra-ligand energy (all lanes). Set 0 is the input
// conformer (all angles 0); the others draw each torsion angle uniformly in [-pi, pi) from the counter-based
// stream (seed, ligand, set, torsion).
__device__ float conformer_set(const SearchParams& P, int l, int trial, unsigned long long seed, float* X, float* th,
                               float* cs, float* sn, int lane) {
    const int4 inf = P.info[l];
    const int na = inf.x, nt = inf.y, np = inf.z;
    const int AM = P.AM;
    for (int k = lane; k < P.KM; k += 32) {
        const float a = (trial == 0 || k >= nt) ? 0.f : (2.f * uniform01(seed, l, trial, k) - 1.f) * 3.14159265f;
        th[k] = a;
        float sv, cv;
        sincosf(a, &sv, &cv);
        cs[k] = cv;
        sn[k] = sv;
    }
    __syncwarp();
    const float4* tr = P.tors + (long long)l * P.KM * 2;
    for (int a = lane; a < AM; a += 32) {
        float px = 0.f, py = 0.f, pz = 0.f;
        if (a < na) {
            const float4 v = P.atoms[(long long)l * AM + a];
            px = v.x; py = v.y; pz = v.z;
            uint32_t m = P.masks[(long long)l * AM + a];
            while (m) {
                const int k = __ffs(m) - 1;
                m &= m - 1;
                const float4 A = tr[2 * k], U = tr[2 * k + 1];
                const float cv = cs[k], sv = sn[k];
                const float vx = px - A.x, vy = py - A.y, vz = pz - A.z;
                const float d = U.x * vx + U.y * vy + U.z * vz;
                const float cx = U.y * vz - U.z * vy, cy = U.z * vx - U.x * vz, cz = U.x * vy - U.y * vx;
                px = A.x + vx * cv + cx * sv + U.x * d * (1 - cv);
                py = A.y + vy * cv + cy * sv + U.y * d * (1 - cv);
                pz = A.z + vz * cv + cz * sv + U.z * d * (1 - cv);
            }
        }
        X[a] = px; X[AM + a] = py; X[2 * AM + a] = pz;
    }
    __syncwarp();
    float e = 0.f;
    const int2* pr = P.pairs + (long long)l * P.P_pad;
    const int nslot = pad32i(np);
    for (int q = lane; q < nslot; q += 32) {
        const int2 rec = pr[q];
        if (rec.x < 0) continue;
        const int i = rec.x & 0xff, j = (rec.x >> 8) & 0xff, fl = rec.x >> 16;
        const float rx = X[i] - X[j], ry = X[AM + i] - X[AM + j], rz = X[2 * AM + i] - X[2 * AM + j];
        const float r = sqrtf(rx * rx + ry * ry + rz * rz);
        if (r >= P.pp.cutoff) continue;
        float de;
        e += pair_energy(r, __int_as_float(rec.y), fl, P.pp, de);
    }
    e = warp_sum(e);
    __syncwarp();
    return e;
}

// One CTA per ligand: the intra energy of NT torsion sets, then the C lowest (ties: lower set index) in ascending
// energy order, written as angles theta [L, C, KM], heavy-atom coordinates conf [L, C, AM, 3] (0 past na) and
// energies e [L, C].
__global__ void __launch_bounds__(256) conformer_kernel(const __grid_constant__ SearchParams P, int NT, int C,
                                                        unsigned long long seed, float* theta_out, float* conf_out,
                                                        float* e_out) {
    extern __shared__ float csm[];
    const int l = blockIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int AM = P.AM, KM = P.KM;
    float* e_s = csm;                           // [NT]
    int* sel = (int*)(csm + NT);                // [C]
    float* ws = csm + NT + C + wid * (3 * AM + 3 * KM);
    float* X = ws;
    float* th = ws + 3 * AM;
    float* cs = th + KM;
    float* sn = cs + KM;
    for (int t = wid; t < NT; t += nw) {
        const float e = conformer_set(P, l, t, seed, X, th, cs, sn, lane);
        if (lane == 0) e_s[t] = (e == e) ? e : 3.4e38f;   // a NaN energy ranks last
    }
    __syncthreads();
    for (int t = threadIdx.x; t < NT; t += blockDim.x) {
        const float et = e_s[t];
        int rank = 0;
        for (int j = 0; j < NT; ++j) {
            const float ej = e_s[j];
            rank += (ej < et) || (ej == et && j < t);
        }
        if (rank < C) sel[rank] = t;
    }
    __syncthreads();
    for (int r = wid; r < C; r += nw) {
        const int t = sel[r];
        conformer_set(P, l, t, seed, X, th, cs, sn, lane);
        const long long o = (long long)l * C + r;
        for (int k = lane; k < KM; k += 32) theta_out[o * KM + k] = th[k];
        for (int a = lane; a < AM; a += 32) {
            float* dst = conf_out + (o * AM + a) * 3;
            dst[0] = X[a]; dst[1] = X[AM + a]; dst[2] = X[2 * AM + a];
        }
        if (lane == 0) e_out[o] = e_s[t];
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------------------ lattice
// One CTA per box: lattice points center - size/2 + 1 + i * step (i < box_n per axis, x slowest) whose nearest-grid
// energy of the probe map (+ out-of-box penalty) is <= probe_max, compacted in lattice order into trans
// [B, nt_max, 3]; the box centre alone when no point passes.
template <typename GT>
__global__ void __launch_bounds__(1024) lattice_kernel(const __grid_constant__ SearchParams P, const float* box,
                                                       const int* box_rec, const int* box_slot, const int* box_n,
                                                       float step, float probe_max, int nt_max, float* trans,
                                                       int* ntrans) {
    __shared__ int warp_tot[32];
    __shared__ int total;
    const int b = blockIdx.x;
    const float cx = box[6 * b], cy = box[6 * b + 1], cz = box[6 * b + 2];
    const float sx = box[6 * b + 3], sy = box[6 * b + 4], sz = box[6 * b + 5];
    const int ri = box_rec[b], slot = box_slot[b];
    const int mx = box_n[3 * b], my = box_n[3 * b + 1], mz = box_n[3 * b + 2];
    const long long npts = (long long)mx * my * mz;
    const int nx = (int)P.dims[3 * ri], ny = (int)P.dims[3 * ri + 1], nz = (int)P.dims[3 * ri + 2];
    const GT* G = (const GT*)P.flat + P.offs[ri] + (long long)slot * nx * ny * nz;
    const float ox = P.origin[3 * ri], oy = P.origin[3 * ri + 1], oz = P.origin[3 * ri + 2];
    const float lx = P.lo[3 * ri], ly = P.lo[3 * ri + 1], lz = P.lo[3 * ri + 2];
    const float hx = P.hi[3 * ri], hy = P.hi[3 * ri + 1], hz = P.hi[3 * ri + 2];
    const float x0 = -0.5f * sx + 1.f, y0 = -0.5f * sy + 1.f, z0 = -0.5f * sz + 1.f;
    float* out = trans + (long long)b * nt_max * 3;
    int base = 0;
    for (long long start = 0; start < npts; start += blockDim.x) {
        const long long p = start + threadIdx.x;
        int ok = 0;
        float px = 0.f, py = 0.f, pz = 0.f;
        if (p < npts) {
            const int i = (int)(p / ((long long)my * mz)), j = (int)((p / mz) % my), k = (int)(p % mz);
            px = (x0 + i * step) + cx;
            py = (y0 + j * step) + cy;
            pz = (z0 + k * step) + cz;
            const int gi = min(max(__float2int_rn((px - ox) * P.inv_s), 0), nx - 1);
            const int gj = min(max(__float2int_rn((py - oy) * P.inv_s), 0), ny - 1);
            const int gk = min(max(__float2int_rn((pz - oz) * P.inv_s), 0), nz - 1);
            float v = gload(G + ((long long)gi * ny + gj) * nz + gk);
            const float dx0 = fmaxf(lx - px, 0.f), dx1 = fmaxf(px - hx, 0.f);
            const float dy0 = fmaxf(ly - py, 0.f), dy1 = fmaxf(py - hy, 0.f);
            const float dz0 = fmaxf(lz - pz, 0.f), dz1 = fmaxf(pz - hz, 0.f);
            v += P.pen * (dx0 * dx0 + dx1 * dx1 + dy0 * dy0 + dy1 * dy1 + dz0 * dz0 + dz1 * dz1);
            ok = v <= probe_max;
        }
        const int off = block_exclusive_scan(ok, warp_tot, &total);
        if (ok && base + off < nt_max) {
            float* d = out + (long long)(base + off) * 3;
            d[0] = px; d[1] = py; d[2] = pz;
        }
        base += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (base == 0) {
            out[0] = cx; out[1] = cy; out[2] = cz;
            base = 1;
        }
        ntrans[b] = min(base, nt_max);
    }
}

// ------------------------------------------------------------------------------------------ start selection
// One CTA per ligand: total energy best_e[l, j] + e_conf[l, j / Q] of every (conformer, rotation) j < CQ, sorted
// ascending (ties: lower j); chain m of the ligand starts from the (m mod min(M, CQ))-th: translation = the best
// lattice point of j, rotation = quats[j % Q], torsions = theta[l, j / Q]. Writes state [L * M, 7 + KM] and
// e_start [L * M] (optional).
__global__ void __launch_bounds__(1024) select_starts_kernel(int CQ, int n2, int C, int Q, int KM, int M,
                                                             const float* best_e, const int* best_i,
                                                             const float* e_conf, const float* quats,
                                                             const float* theta, const float* trans,
                                                             const int* lig_box, int nt_max, float* state,
                                                             float* e_start) {
    extern __shared__ float ssm[];
    float* key = ssm;
    int* idx = (int*)(ssm + n2);
    const int l = blockIdx.x;
    for (int j = threadIdx.x; j < n2; j += blockDim.x) {
        float v = 3.4e38f;
        if (j < CQ) {
            v = best_e[(long long)l * CQ + j] + e_conf[(long long)l * C + j / Q];
            if (!(v == v)) v = 3.4e38f;
        }
        key[j] = v;
        idx[j] = j;
    }
    __syncthreads();
    block_sort_pairs(key, idx, n2);
    const int k = min(M, CQ);
    const int b = lig_box ? lig_box[l] : l;
    const int SD = 7 + KM;
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        const int j = idx[m % k];
        const int c = j / Q, q = j % Q;
        const int ti = best_i[(long long)l * CQ + j];
        float* s = state + ((long long)l * M + m) * SD;
        const float* t = trans + ((long long)b * nt_max + ti) * 3;
        s[0] = t[0]; s[1] = t[1]; s[2] = t[2];
        s[3] = quats[4 * q]; s[4] = quats[4 * q + 1]; s[5] = quats[4 * q + 2]; s[6] = quats[4 * q + 3];
        for (int kk = 0; kk < KM; ++kk) s[7 + kk] = theta[((long long)l * C + c) * KM + kk];
        if (e_start) e_start[(long long)l * M + m] = key[m % k];
    }
}

// ------------------------------------------------------------------------------------------ segment bookkeeping
// After MC segment `sg` (chains ligand-major, M per ligand): counts the chain-steps the segment ran, updates each
// ligand's best energy over its chains, its count of segments without an improvement of more than es_tol, and its
// active flag for segment sg + 1: still active, under its segment budget seg_lim, and (when es_rounds > 0) fewer
// than es_rounds segments without improvement.
__global__ void segment_update_kernel(int L, int M, int seg, int next_sg, int es_rounds, float es_tol,
                                      const float* best_e, const int* seg_lim, float* glob, int* stall, int* active,
                                      unsigned long long* chain_steps) {
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= L) return;
    const int was = active[l];
    if (was && chain_steps) atomicAdd(chain_steps, (unsigned long long)M * seg);
    float gb = 3.4e38f;
    for (int m = 0; m < M; ++m) gb = fminf(gb, best_e[(long long)l * M + m]);
    const float g = glob[l];
    const bool improved = gb < g - es_tol;
    glob[l] = fminf(g, gb);
    const int s = improved ? 0 : stall[l] + 1;
    stall[l] = s;
    active[l] = was && seg_lim[l] > next_sg && (es_rounds <= 0 || s < es_rounds);
}

// ------------------------------------------------------------------------------------------ clustering
// One CTA per ligand: its P final poses sorted by energy (ties: lower index), then greedy representatives: a pose
// joins when its heavy-atom RMSD (same atom order, no symmetry) to every earlier representative is >= cut, until
// n_out are found. reps [L, n_out] (pose index within the ligand, -1 past n_reps[l]).
__global__ void __launch_bounds__(256) cluster_kernel(const int4* info, int P, int n2, const double* e_total,
                                                      const float* X, int AM, float cut, int n_out, int* reps,
                                                      int* n_reps) {
    extern __shared__ double csm64[];
    double* key = csm64;
    int* idx = (int*)(csm64 + n2);
    __shared__ int rep_s[32];
    const int l = blockIdx.x;
    const int na = max(info[l].x, 1);
    for (int j = threadIdx.x; j < n2; j += blockDim.x) {
        double v = 1.7e308;
        if (j < P) {
            v = e_total[(long long)l * P + j];
            if (!(v == v)) v = 1.7e308;
        }
        key[j] = v;
        idx[j] = j;
    }
    __syncthreads();
    block_sort_pairs(key, idx, n2);
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        int nr = 0;
        const float* Xl = X + (long long)l * P * AM * 3;
        for (int c = 0; c < P && nr < n_out; ++c) {
            const int i = idx[c];
            bool ok = true;
            for (int r = 0; r < nr && ok; ++r) {
                const int j = rep_s[r];
                float s = 0.f;
                for (int a = lane; a < na; a += 32) {
                    const float* xi = Xl + ((long long)i * AM + a) * 3;
                    const float* xj = Xl + ((long long)j * AM + a) * 3;
                    const float dx = xi[0] - xj[0], dy = xi[1] - xj[1], dz = xi[2] - xj[2];
                    s += dx * dx + dy * dy + dz * dz;
                }
                s = warp_sum(s);
                ok = sqrtf(s / (float)na) >= cut;
            }
            if (ok) {
                if (lane == 0) rep_s[nr] = i;
                ++nr;
            }
            __syncwarp();
        }
        for (int r = lane; r < n_out; r += 32) reps[(long long)l * n_out + r] = r < nr ? rep_s[r] : -1;
        if (lane == 0) n_reps[l] = nr;
    }
}

// ------------------------------------------------------------------------------------------ all-atom coordinates
// One warp per state: world coordinates of all A atoms of the ligand (hydrogens included, in the caller's atom
// order), float32 forward kinematics with the batch's torsion axes: torsions applied to the reference coordinates
// leaf -> root (mask bit k = torsion k moves the atom), rotation by the normalised quaternion, translation.
// Atoms past a ligand's count sit at the translation (zero reference coordinates).
__global__ void __launch_bounds__(128) pose_atoms_kernel(const float4* tors, int KM, const float* ref_all,
                                                         const uint32_t* mask_all, int A, const int* chain_lig,
                                                         int n, const float* state, float* X) {
    __shared__ float trig[4][2][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int s_i = blockIdx.x * 4 + wid;
    if (s_i >= n) return;
    const int l = chain_lig[s_i];
    const int SD = 7 + KM;
    const float* s = state + (long long)s_i * SD;
    if (lane < KM) {
        float sv, cv;
        sincosf(s[7 + lane], &sv, &cv);
        trig[wid][0][lane] = cv;
        trig[wid][1][lane] = sv;
    }
    __syncwarp();
    float qw = s[3], qx = s[4], qy = s[5], qz = s[6];
    const float nq = rsqrtf(qw * qw + qx * qx + qy * qy + qz * qz);
    qw *= nq; qx *= nq; qy *= nq; qz *= nq;
    const float R00 = 1 - 2 * (qy * qy + qz * qz), R01 = 2 * (qx * qy - qz * qw), R02 = 2 * (qx * qz + qy * qw);
    const float R10 = 2 * (qx * qy + qz * qw), R11 = 1 - 2 * (qx * qx + qz * qz), R12 = 2 * (qy * qz - qx * qw);
    const float R20 = 2 * (qx * qz - qy * qw), R21 = 2 * (qy * qz + qx * qw), R22 = 1 - 2 * (qx * qx + qy * qy);
    const float4* tr = tors + (long long)l * KM * 2;
    for (int a = lane; a < A; a += 32) {
        const float* r = ref_all + ((long long)l * A + a) * 3;
        float px = r[0], py = r[1], pz = r[2];
        uint32_t m = mask_all[(long long)l * A + a];
        while (m) {
            const int k = __ffs(m) - 1;
            m &= m - 1;
            if (k >= KM) break;
            const float4 Ap = tr[2 * k], U = tr[2 * k + 1];
            const float cv = trig[wid][0][k], sv = trig[wid][1][k];
            const float vx = px - Ap.x, vy = py - Ap.y, vz = pz - Ap.z;
            const float d = U.x * vx + U.y * vy + U.z * vz;
            const float cx = U.y * vz - U.z * vy, cy = U.z * vx - U.x * vz, cz = U.x * vy - U.y * vx;
            px = Ap.x + vx * cv + cx * sv + U.x * d * (1 - cv);
            py = Ap.y + vy * cv + cy * sv + U.y * d * (1 - cv);
            pz = Ap.z + vz * cv + cz * sv + U.z * d * (1 - cv);
        }
        float* o = X + ((long long)s_i * A + a) * 3;
        o[0] = R00 * px + R01 * py + R02 * pz + s[0];
        o[1] = R10 * px + R11 * py + R12 * pz + s[1];
        o[2] = R20 * px + R21 * py + R22 * pz + s[2];
    }
}

}  // namespace adock

using namespace adock;

// ------------------------------------------------------------------------------------------ C-ABI
extern "C" int adock_conformers(const adock_ligands_t* lig, const adock_work_t* work, const adock_sf_t* sf, int NT,
                                int C, unsigned long long seed, float* theta, float* conf, float* e, void* stream) {
    SearchParams P;
    int rc = make_params(P, lig, work, nullptr, sf, nullptr);
    if (rc) return rc;
    ADOCK_CHECK_ARG(NT >= 1 && NT <= 4096, "NT must be in [1, 4096] (got %d)", NT);
    ADOCK_CHECK_ARG(C >= 1 && C <= NT, "C must be in [1, NT] (got %d)", C);
    ADOCK_CHECK_ARG(theta && conf && e, "null array argument");
    const int threads = 256;
    const size_t smem = ((size_t)NT + C + (threads / 32) * (3 * (size_t)P.AM + 3 * (size_t)P.KM)) * sizeof(float);
    ADOCK_CUDA(cudaFuncSetAttribute(conformer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    conformer_kernel<<<lig->L, threads, smem, (cudaStream_t)stream>>>(P, NT, C, splitmix(seed ^ 0xC0F0A11CE5ULL), theta,
                                                                      conf, e);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

extern "C" int adock_lattice(const adock_grids_t* grids, int B, const float* box, const int* box_rec,
                             const int* box_slot, const int* box_n, float step, float probe_max, int nt_max,
                             float* trans, int* ntrans, void* stream) {
    ADOCK_CHECK_ARG(grids && grids->flat && grids->dims && grids->offs, "grids are required");
    ADOCK_CHECK_ARG(B >= 1 && nt_max >= 1, "B and nt_max must be >= 1");
    ADOCK_CHECK_ARG(step > 0.f, "step must be > 0");
    ADOCK_CHECK_ARG(box && box_rec && box_slot && box_n && trans && ntrans, "null array argument");
    SearchParams P{};
    P.flat = grids->flat; P.offs = grids->offs; P.dims = grids->dims;
    P.origin = grids->origin; P.lo = grids->lo; P.hi = grids->hi;
    P.inv_s = 1.f / grids->spacing; P.pen = grids->penalty;
    cudaStream_t st = (cudaStream_t)stream;
    switch (grids->dtype) {
        case ADOCK_GRID_F32:
            lattice_kernel<float><<<B, 1024, 0, st>>>(P, box, box_rec, box_slot, box_n, step, probe_max, nt_max, trans, ntrans);
            break;
        case ADOCK_GRID_F16:
            lattice_kernel<__half><<<B, 1024, 0, st>>>(P, box, box_rec, box_slot, box_n, step, probe_max, nt_max, trans, ntrans);
            break;
        case ADOCK_GRID_BF16:
            lattice_kernel<__nv_bfloat16><<<B, 1024, 0, st>>>(P, box, box_rec, box_slot, box_n, step, probe_max, nt_max,
                                                              trans, ntrans);
            break;
        default:
            ADOCK_CHECK_ARG(false, "unknown grid dtype %d", grids->dtype);
    }
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

extern "C" int adock_select_starts(int L, int C, int Q, int KM, int M, const float* best_e, const int* best_i,
                                   const float* e_conf, const float* quats, const float* theta, const float* trans,
                                   const int* lig_box, int nt_max, float* state, float* e_start, void* stream) {
    ADOCK_CHECK_ARG(L >= 1 && C >= 1 && Q >= 1 && M >= 1 && KM >= 1 && nt_max >= 1, "sizes must be >= 1");
    const int CQ = C * Q;
    ADOCK_CHECK_ARG(CQ <= 16384, "C * Q must be <= 16384 (got %d)", CQ);
    ADOCK_CHECK_ARG(best_e && best_i && e_conf && quats && theta && trans && state, "null array argument");
    const int n2 = pow2_at_least(CQ);
    const size_t smem = (size_t)n2 * (sizeof(float) + sizeof(int));
    ADOCK_CUDA(cudaFuncSetAttribute(select_starts_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    select_starts_kernel<<<L, 1024, smem, (cudaStream_t)stream>>>(CQ, n2, C, Q, KM, M, best_e, best_i, e_conf, quats,
                                                                  theta, trans, lig_box, nt_max, state, e_start);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

extern "C" int adock_segment_update(int L, int M, int seg, int next_sg, int es_rounds, float es_tol,
                                    const float* best_e, const int* seg_lim, float* glob, int* stall, int* active,
                                    unsigned long long* chain_steps, void* stream) {
    ADOCK_CHECK_ARG(L >= 1 && M >= 1 && seg >= 0, "bad sizes");
    ADOCK_CHECK_ARG(best_e && seg_lim && glob && stall && active, "null array argument");
    segment_update_kernel<<<(L + 127) / 128, 128, 0, (cudaStream_t)stream>>>(L, M, seg, next_sg, es_rounds, es_tol,
                                                                              best_e, seg_lim, glob, stall, active,
                                                                              chain_steps);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

extern "C" int adock_cluster(const adock_work_t* work, int L, int P, const double* e_total, const float* X, int AM,
                             float cut, int n_out, int* reps, int* n_reps, void* stream) {
    ADOCK_CHECK_ARG(work && work->info, "null work argument");
    ADOCK_CHECK_ARG(L >= 1 && P >= 1 && AM >= 1, "sizes must be >= 1");
    ADOCK_CHECK_ARG(P <= 4096, "at most 4096 poses per ligand (got %d)", P);
    ADOCK_CHECK_ARG(n_out >= 1 && n_out <= 32, "n_out must be in [1, 32] (got %d)", n_out);
    ADOCK_CHECK_ARG(e_total && X && reps && n_reps, "null array argument");
    const int n2 = pow2_at_least(P);
    const size_t smem = (size_t)n2 * (sizeof(double) + sizeof(int));
    ADOCK_CUDA(cudaFuncSetAttribute(cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cluster_kernel<<<L, 256, smem, (cudaStream_t)stream>>>((const int4*)work->info, P, n2, e_total, X, AM, cut, n_out,
                                                            reps, n_reps);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

extern "C" int adock_pose_atoms(const adock_work_t* work, int KM, const float* ref_all, const unsigned* mask_all, int A,
                                const int* chain_lig, int n, const float* state, float* X, void* stream) {
    ADOCK_CHECK_ARG(work && work->tors, "null work argument");
    ADOCK_CHECK_ARG(KM >= 1 && KM <= 32 && A >= 1 && n >= 0, "bad sizes");
    if (n == 0) return ADOCK_OK;
    ADOCK_CHECK_ARG(ref_all && mask_all && chain_lig && state && X, "null array argument");
    pose_atoms_kernel<<<(n + 3) / 4, 128, 0, (cudaStream_t)stream>>>((const float4*)work->tors, KM, ref_all, mask_all, A,
                                                                     chain_lig, n, state, X);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}
