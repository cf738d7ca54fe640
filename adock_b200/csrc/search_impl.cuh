// Device code of the search kernels (sm_100a), included by the per-grid-dtype translation units
// (search_f32.cu, search_f16.cu, search_bf16.cu) that instantiate the launchers, and by search.cu.
//
// Execution model: one warp owns one chain (pose). Lanes own heavy atoms a = lane + 32*i (i < APL, AM = 32*APL)
// whose ligand-frame coordinates, grid slot and torsion bitmask stay in registers for the whole chain. Per-warp
// shared memory holds world coordinates, forces, torsion axes, the BFGS inverse Hessian and the state vectors.
// The Monte-Carlo kernel is persistent: warps pull chains from a device work counter (longest ligands first),
// so uneven ligands do not leave SMs idle at the tail.
#pragma once
#include "common.cuh"

namespace adock {

#define EPSF 1.1920929e-07f

// Code-size knobs of the MC kernel (instruction-cache footprint vs register allocation across calls).
#ifdef ADOCK_BFGS_INLINE
#define ADOCK_BFGS_ATTR __forceinline__
#else
#define ADOCK_BFGS_ATTR __noinline__
#endif
#ifdef ADOCK_COLD_NOINLINE
#define ADOCK_COLD_ATTR __noinline__
#else
#define ADOCK_COLD_ATTR __forceinline__
#endif
#define PAIR_ROUNDS_MAX 256   // pair schedule: at most 256 rounds of 32 (8,192 pairs) are reordered

struct SearchParams {
    // B200 working layout
    const float4* atoms;   // [L, AM]
    const uint32_t* masks; // [L, AM]
    const float4* tors;    // [L, KM, 2]
    const int2* pairs;     // [L, P_pad] scheduled in rounds of 32; empty slots have x = -1
    const int4* info;      // [L] na, nt, np, rec_idx
    const float* rg;       // [L]
    int AM, KM, P, P_pad;
    // grids
    const void* flat;
    const long long* offs;
    const long long* dims;
    const float* origin;
    const float* lo;
    const float* hi;
    const int* nmaps;      // [R] maps built per receptor (may be NULL)
    float inv_s, pen;
    // receptor atoms for exact mode
    const float* rxyz;
    const int* rtyp;
    const int* rn;
    int RN;
    PairPrm pp;
    int n_types;
};

// type tables for exact mode, staged in shared memory by every block that may need them
struct TypeTables {
    float radius[64];
    int flags[64];  // bit0 hydrophobic, bit1 donor, bit2 acceptor
};

struct McParams {
    const int* chain_lig;
    const int* chain_id;
    int n_chains;
    const int* nbr;
    const int* nbr_n;
    int nb_max;
    float* cur;
    float* cur_e;
    float* best;
    float* best_e;
    int init_opt, mc_steps, bfgs_iters;
    float temp, amp_pos, amp_rot;
    unsigned long long seed;
    int step_offset;
    int exact;
    const int* order;
    int* queue;
    unsigned long long* evals;
    // learned proposal: moves [N, prop_k, 32] for steps 0..prop_k-1 of this launch (NULL: plain MC only)
    const float* prop;
    int prop_k;
    float prop_frac;                 // fraction of steps that take the learned move (the rest: plain MC)
    unsigned long long* prop_stats;  // [4] proposals made, proposals accepted, plain steps, plain accepted
    // training-data log of accepted improving moves: features [cap, 320] BF16, moves [cap, 32]
    __nv_bfloat16* log_x;
    float* log_y;
    int* log_n;
    int log_cap;
    const int* lig_active;           // [L] or NULL: chains of a ligand with flag 0 are left unchanged
    int prop_tries;                  // learned steps: candidate targets per step (the lowest-energy one is optimised)
    const float* hint;               // [L, PROP_HINT] ligand-best rows for the logged features, or NULL
};

#define PROP_IN 320
#define PROP_HINT 32
#define PROP_MOVE 32
#define PROP_FAIL_MAX 8

__device__ __forceinline__ int hb_pair(int fa, int fb) {
    return (((fa & 2) && (fb & 4)) || ((fa & 4) && (fb & 2))) ? PF_HB : 0;
}
__device__ __forceinline__ int hyd_pair(int fa, int fb) { return ((fa & 1) && (fb & 1)) ? PF_HYD : 0; }

__device__ __forceinline__ void stage_tables(TypeTables& dst, const TypeTables& src) {
    for (int i = threadIdx.x; i < 64; i += blockDim.x) {
        dst.radius[i] = src.radius[i];
        dst.flags[i] = src.flags[i];
    }
    __syncthreads();
}

// ------------------------------------------------------------------------------------------ per-warp workspace
// Float offsets of the per-warp shared workspace for a given AM / KM (float4 arrays first).
struct WSLayout {
    int X, FF, ap, au, tp, tu, mk, ax, cs, sn, H, x, xn, xo, cur, best, g, gn, go, p, y, mhy, total;
    __host__ __device__ WSLayout(int AM, int KM) {
        const int DM = 6 + KM, SD = 7 + KM;
        int o = 0;
        X = o; o += 3 * AM;    // world coordinates, [3][AM] (x, y, z arrays)
        FF = o; o += 3 * AM;   // forces, [3][AM]
        ap = o; o += 4 * KM;
        au = o; o += 4 * KM;
        tp = o; o += 4 * KM;
        tu = o; o += 4 * KM;
        mk = o; o += AM;
        ax = o; o += KM;      // packed axis atom indices (a0 | a1 << 16)
        cs = o; o += KM;
        sn = o; o += KM;
        H = o; o += DM * DM;
        x = o; o += SD;
        xn = o; o += SD;
        xo = o; o += SD;
        cur = o; o += SD;
        best = o; o += SD;
        g = o; o += DM;
        gn = o; o += DM;
        go = o; o += DM;
        p = o; o += DM;
        y = o; o += DM;
        mhy = o; o += DM;
        total = (o + 3) & ~3;  // keep 16-byte alignment of the next warp
    }
};

// Per-chain context (registers).
template <int APL>
struct Chain {
    int na, nt, np, nrounds;
    float rg;
    const int2* pairs;
    const char* grid;
    long long n3;
    int ny, nz;
    float o[3], lo[3], hi[3], fmx[3];
    const float* rx;
    const int* rt;
    int rn;
    const int* nb;
    int nbn;
    int exact;
    float3 ref[APL];
    int slot[APL];
    int typ[APL];
    uint32_t mask[APL];
};

template <int APL, typename GT>
__device__ __forceinline__ void load_chain(Chain<APL>& c, const SearchParams& P, int l, float* ws, const WSLayout& L,
                                           int lane, int exact, const int* nb, int nbn) {
    const int4 inf = P.info[l];
    c.na = inf.x; c.nt = inf.y; c.np = inf.z;
    c.nrounds = (inf.z + 31) >> 5;
    const int ri = inf.w;
    c.rg = P.rg[l];
    c.pairs = P.pairs + (long long)l * P.P_pad;
    const long long nx = P.dims[3 * ri], ny = P.dims[3 * ri + 1], nz = P.dims[3 * ri + 2];
    c.n3 = nx * ny * nz;
    c.ny = (int)ny; c.nz = (int)nz;
    c.grid = (const char*)((const GT*)P.flat + P.offs[ri]);
    for (int d = 0; d < 3; ++d) {
        c.o[d] = P.origin[3 * ri + d]; c.lo[d] = P.lo[3 * ri + d]; c.hi[d] = P.hi[3 * ri + d];
    }
    c.fmx[0] = (float)(nx - 1) - 1e-4f; c.fmx[1] = (float)(ny - 1) - 1e-4f; c.fmx[2] = (float)(nz - 1) - 1e-4f;
    c.exact = exact;
    c.rx = P.rxyz ? P.rxyz + (long long)ri * P.RN * 3 : nullptr;
    c.rt = P.rtyp ? P.rtyp + (long long)ri * P.RN : nullptr;
    c.rn = P.rn ? P.rn[ri] : 0;
    c.nb = nb; c.nbn = nbn;
    const float4* at = P.atoms + (long long)l * P.AM;
    const uint32_t* mk = P.masks + (long long)l * P.AM;
    uint32_t* smk = (uint32_t*)(ws + L.mk);
#pragma unroll
    for (int i = 0; i < APL; ++i) {
        const int a = lane + 32 * i;
        const float4 v = at[a];
        c.ref[i] = make_float3(v.x, v.y, v.z);
        const int meta = __float_as_int(v.w);
        c.slot[i] = meta & 0xffff;
        c.typ[i] = meta >> 16;
        c.mask[i] = mk[a];
        smk[a] = c.mask[i];
    }
    const float4* tr = P.tors + (long long)l * P.KM * 2;
    float4* ap = (float4*)(ws + L.ap);
    float4* au = (float4*)(ws + L.au);
    int* axs = (int*)(ws + L.ax);
    for (int k = lane; k < P.KM; k += 32) {
        const float4 p = tr[2 * k], u = tr[2 * k + 1];
        ap[k] = p;
        au[k] = u;
        axs[k] = (__float_as_int(p.w) & 0xffff) | (__float_as_int(u.w) << 16);
    }
    __syncwarp();
}

// trilinear lookup + analytic gradient of one atom (mckernel.py:140-149, :176-195)
template <typename GT>
__device__ __forceinline__ float trilinear(const GT* G, int ny, int nz, const float* o, const float* fmx, float inv_s,
                                           float X0, float X1, float X2, float& gx, float& gy, float& gz) {
    const float xx[3] = {X0, X1, X2};
    float fw[3], inside[3];
    int i0[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float f = (xx[d] - o[d]) * inv_s;
        const float fc = fminf(fmaxf(f, 0.f), fmx[d]);
        inside[d] = (f > 0.f && f < fmx[d]) ? 1.f : 0.f;
        const int ii = (int)floorf(fc);
        i0[d] = ii;
        fw[d] = fc - ii;
    }
    const long long b000 = ((long long)i0[0] * ny + i0[1]) * nz + i0[2];
    const long long sx = (long long)ny * nz;
    const float v000 = gload(G + b000), v001 = gload(G + b000 + 1), v010 = gload(G + b000 + nz),
                v011 = gload(G + b000 + nz + 1);
    const float v100 = gload(G + b000 + sx), v101 = gload(G + b000 + sx + 1), v110 = gload(G + b000 + sx + nz),
                v111 = gload(G + b000 + sx + nz + 1);
    const float wx = fw[0], wy = fw[1], wz = fw[2];
    const float c00 = v000 * (1 - wz) + v001 * wz, c01 = v010 * (1 - wz) + v011 * wz;
    const float c10 = v100 * (1 - wz) + v101 * wz, c11 = v110 * (1 - wz) + v111 * wz;
    const float c0 = c00 * (1 - wy) + c01 * wy, c1 = c10 * (1 - wy) + c11 * wy;
    const float e = c0 * (1 - wx) + c1 * wx;
    gx = (c1 - c0) * inv_s * inside[0];
    gy = ((c01 - c00) * (1 - wx) + (c11 - c10) * wx) * inv_s * inside[1];
    gz = (((v001 - v000) * (1 - wy) + (v011 - v010) * wy) * (1 - wx) +
          ((v101 - v100) * (1 - wy) + (v111 - v110) * wy) * wx) * inv_s * inside[2];
    return e;
}

// Intra-ligand pair term of one scheduled slot: energy, and the force added into both atoms' entries. Positions X
// and forces F are three arrays of AM floats each (x, y, z), so that 32 lanes touching 32 different atoms hit 32
// different shared-memory banks (a float4 per atom would put the x components of 32 atoms on 8 banks).
template <int AM>
__device__ __forceinline__ float pair_slot(int2 pr, const float* X, float* F, const PairPrm& pp) {
    if (pr.x < 0) return 0.f;
    const int i = pr.x & 0xff, j = (pr.x >> 8) & 0xff, fl = pr.x >> 16;
    const float rx = X[i] - X[j], ry = X[AM + i] - X[AM + j], rz = X[2 * AM + i] - X[2 * AM + j];
    // r and 1/r from one reciprocal square root; clamping r^2 at 1e-12 is the reference's max(r, 1e-6)
    const float r2 = rx * rx + ry * ry + rz * rz;
    const float rinv = rsqrtf(fmaxf(r2, 1e-12f));
    const float r = r2 * rinv;
    if (r >= pp.cutoff) return 0.f;
    float de;
    const float e = pair_energy(r, __int_as_float(pr.y), fl, pp, de);
    const float sc = de * rinv;
    atomicAdd(F + i, sc * rx); atomicAdd(F + AM + i, sc * ry); atomicAdd(F + 2 * AM + i, sc * rz);
    atomicAdd(F + j, -sc * rx); atomicAdd(F + AM + j, -sc * ry); atomicAdd(F + 2 * AM + j, -sc * rz);
    return e;
}

// Energy + analytic pose gradient of state s (shared, SD floats) into g (shared, DM floats); E on all lanes.
// Same energy as mckernel.py:108-244: torsions applied leaf -> root on reference coordinates, rotation,
// translation; trilinear grid (or exact pairwise) inter energy with the quadratic out-of-box penalty; intra
// pairs. Gradient: dE/dt = sum F, torque = sum (X - t) x F, dE/dtheta_k = u_k . sum_{a moved by k} (X_a - p_k) x F_a,
// evaluated as u_k . (sum X' x F - p'_k x sum F) over the subtree of k (X' = X - t).
// EX selects the inter energy at compile time: exact pairwise over receptor atoms (or the chain's neighbour list),
// else the trilinear grid, so the grid-mode kernels carry no receptor loop.
template <int APL, typename GT, bool EX>
__device__ __forceinline__ float eval_eg(float* ws, const WSLayout& L, const float* s, float* g, const Chain<APL>& c,
                         const SearchParams& P, const TypeTables& tt, int lane) {
    constexpr int AM = 32 * APL;
    float* X = ws + L.X;     // [3][AM] world coordinates
    float* FF = ws + L.FF;   // [3][AM] forces dE/dX
    const float4* ap = (const float4*)(ws + L.ap);
    const float4* au = (const float4*)(ws + L.au);
    float4* tp = (float4*)(ws + L.tp);
    float4* tu = (float4*)(ws + L.tu);
    const uint32_t* smk = (const uint32_t*)(ws + L.mk);
    const int* axs = (const int*)(ws + L.ax);
    float* cs = ws + L.cs;
    float* sn = ws + L.sn;

    const float t0 = s[0], t1 = s[1], t2 = s[2];
    float qw = s[3], qx = s[4], qy = s[5], qz = s[6];
    const float nq = rsqrtf(qw * qw + qx * qx + qy * qy + qz * qz);
    qw *= nq; qx *= nq; qy *= nq; qz *= nq;
    const float R00 = 1 - 2 * (qy * qy + qz * qz), R01 = 2 * (qx * qy - qz * qw), R02 = 2 * (qx * qz + qy * qw);
    const float R10 = 2 * (qx * qy + qz * qw), R11 = 1 - 2 * (qx * qx + qz * qz), R12 = 2 * (qy * qz - qx * qw);
    const float R20 = 2 * (qx * qz - qy * qw), R21 = 2 * (qy * qz + qx * qw), R22 = 1 - 2 * (qx * qx + qy * qy);
    for (int k = lane; k < c.nt; k += 32) {
        float sv, cv;
        __sincosf(s[7 + k], &sv, &cv);
        cs[k] = cv;
        sn[k] = sv;
    }
    __syncwarp();
    float e = 0.f;
    const GT* grid = (const GT*)c.grid;
#pragma unroll
    for (int i = 0; i < APL; ++i) {
        const int a = lane + 32 * i;
        if (a < c.na) {
            float px = c.ref[i].x, py = c.ref[i].y, pz = c.ref[i].z;
            uint32_t m = c.mask[i];
            while (m) {
                const int k = __ffs(m) - 1;
                m &= m - 1;
                const float4 A = ap[k], U = au[k];
                const float cv = cs[k], sv = sn[k];
                const float vx = px - A.x, vy = py - A.y, vz = pz - A.z;
                const float d = U.x * vx + U.y * vy + U.z * vz;
                const float cx = U.y * vz - U.z * vy, cy = U.z * vx - U.x * vz, cz = U.x * vy - U.y * vx;
                px = A.x + vx * cv + cx * sv + U.x * d * (1 - cv);
                py = A.y + vy * cv + cy * sv + U.y * d * (1 - cv);
                pz = A.z + vz * cv + cz * sv + U.z * d * (1 - cv);
            }
            const float X0 = R00 * px + R01 * py + R02 * pz + t0;
            const float X1 = R10 * px + R11 * py + R12 * pz + t1;
            const float X2 = R20 * px + R21 * py + R22 * pz + t2;
            X[a] = X0;
            X[AM + a] = X1;
            X[2 * AM + a] = X2;
            float ea, gg[3];
            if constexpr (EX) {
                ea = 0.f;
                gg[0] = gg[1] = gg[2] = 0.f;
                const int ta = c.typ[i] & 63;
                const float ra = tt.radius[ta];
                const int fa = tt.flags[ta];
                const float cut2 = P.pp.cutoff * P.pp.cutoff;
                const int nloop = c.nb ? c.nbn : c.rn;
                for (int bb = 0; bb < nloop; ++bb) {
                    const int b = c.nb ? c.nb[bb] : bb;
                    const float rx = X0 - c.rx[3 * b], ry = X1 - c.rx[3 * b + 1], rz = X2 - c.rx[3 * b + 2];
                    const float r2 = rx * rx + ry * ry + rz * rz;
                    if (r2 >= cut2) continue;
                    const int tb = c.rt[b] & 63;   // index kept inside the 64-entry type tables
                    const int fb = tt.flags[tb];
                    const float rinv = rsqrtf(fmaxf(r2, 1e-12f));
                    const float r = r2 * rinv;
                    float de;
                    ea += pair_energy(r, ra + tt.radius[tb], hyd_pair(fa, fb) | hb_pair(fa, fb), P.pp, de);
                    const float sc = de * rinv;
                    gg[0] += sc * rx; gg[1] += sc * ry; gg[2] += sc * rz;
                }
            } else {
                ea = trilinear<GT>(grid + (long long)c.slot[i] * c.n3, c.ny, c.nz, c.o, c.fmx, P.inv_s, X0, X1, X2,
                                   gg[0], gg[1], gg[2]);
            }
            const float xx[3] = {X0, X1, X2};
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const float lo = fmaxf(c.lo[d] - xx[d], 0.f), hi = fmaxf(xx[d] - c.hi[d], 0.f);
                ea += P.pen * (lo * lo + hi * hi);
                gg[d] += P.pen * (-2.f * lo + 2.f * hi);
            }
            e += ea;
            FF[a] = gg[0];
            FF[AM + a] = gg[1];
            FF[2 * AM + a] = gg[2];
        }
    }
    __syncwarp();
    // intra-ligand pairs, scheduled in rounds of 32 in which an atom appears at most once (adock_prepare), so the
    // force atomics of one round do not collide; two rounds in flight per iteration
    // the next two rounds' records are loaded while the current two are evaluated
    {
        const int2 none = make_int2(-1, 0);
        int2 pa = c.nrounds > 0 ? c.pairs[lane] : none;
        int2 pb = c.nrounds > 1 ? c.pairs[32 + lane] : none;
        for (int r = 0; r < c.nrounds; r += 2) {
            const int2 qa = (r + 2 < c.nrounds) ? c.pairs[(r + 2) * 32 + lane] : none;
            const int2 qb = (r + 3 < c.nrounds) ? c.pairs[(r + 3) * 32 + lane] : none;
            e += pair_slot<AM>(pa, X, FF, P.pp);
            e += pair_slot<AM>(pb, X, FF, P.pp);
            pa = qa;
            pb = qb;
        }
    }
    // world torsion axes (axis atoms' current positions)
    for (int k = lane; k < c.nt; k += 32) {
        const int a0 = axs[k] & 0xffff, a1 = axs[k] >> 16;
        const float Ax = X[a0], Ay = X[AM + a0], Az = X[2 * AM + a0];
        const float ux = X[a1] - Ax, uy = X[AM + a1] - Ay, uz = X[2 * AM + a1] - Az;
        const float nn = rsqrtf(fmaxf(ux * ux + uy * uy + uz * uz, 1e-12f));
        tp[k] = make_float4(Ax - t0, Ay - t1, Az - t2, 0.f);
        tu[k] = make_float4(ux * nn, uy * nn, uz * nn, 0.f);
    }
    __syncwarp();
    // subtree sums of F and (X - t) x F: sum k < nt is torsion k's subtree, sum k == nt is the whole ligand.
    // The nt + 1 sums are spread over all 32 lanes: G lanes per atom chunk (G = next power of two >= nt + 1),
    // 32 / G chunks, combined by shuffles.
    if (c.nt < 32) {
        const int G = c.nt < 1 ? 1 : (c.nt < 3 ? 4 : (c.nt < 7 ? 8 : (c.nt < 15 ? 16 : 32)));
        const int k = lane & (G - 1), chunk = lane / G, C = 32 / G;
        float S0 = 0.f, S1 = 0.f, S2 = 0.f, T0 = 0.f, T1 = 0.f, T2 = 0.f;
        if (k <= c.nt) {
            const uint32_t bit = (k == c.nt) ? 0xffffffffu : (1u << k);
            const bool all = (k == c.nt);
            for (int a = chunk; a < c.na; a += C) {
                if (all || (smk[a] & bit)) {
                    const float Fx = FF[a], Fy = FF[AM + a], Fz = FF[2 * AM + a];
                    const float dx = X[a] - t0, dy = X[AM + a] - t1, dz = X[2 * AM + a] - t2;
                    S0 += Fx; S1 += Fy; S2 += Fz;
                    T0 += dy * Fz - dz * Fy; T1 += dz * Fx - dx * Fz; T2 += dx * Fy - dy * Fx;
                }
            }
        }
        for (int o = G; o < 32; o <<= 1) {
            S0 += __shfl_xor_sync(0xffffffffu, S0, o); S1 += __shfl_xor_sync(0xffffffffu, S1, o);
            S2 += __shfl_xor_sync(0xffffffffu, S2, o); T0 += __shfl_xor_sync(0xffffffffu, T0, o);
            T1 += __shfl_xor_sync(0xffffffffu, T1, o); T2 += __shfl_xor_sync(0xffffffffu, T2, o);
        }
        if (chunk == 0 && k <= c.nt) {
            if (k == c.nt) {
                g[0] = S0; g[1] = S1; g[2] = S2; g[3] = T0; g[4] = T1; g[5] = T2;
            } else {
                const float4 Pk = tp[k], Uk = tu[k];
                const float cx = T0 - (Pk.y * S2 - Pk.z * S1);
                const float cy = T1 - (Pk.z * S0 - Pk.x * S2);
                const float cz = T2 - (Pk.x * S1 - Pk.y * S0);
                g[6 + k] = cx * Uk.x + cy * Uk.y + cz * Uk.z;
            }
        }
    } else {
        for (int k = lane; k <= c.nt; k += 32) {
            float S0 = 0.f, S1 = 0.f, S2 = 0.f, T0 = 0.f, T1 = 0.f, T2 = 0.f;
            const bool all = (k == c.nt);
            const uint32_t bit = all ? 0u : (1u << k);
            for (int a = 0; a < c.na; ++a) {
                if (all || (smk[a] & bit)) {
                    const float Fx = FF[a], Fy = FF[AM + a], Fz = FF[2 * AM + a];
                    const float dx = X[a] - t0, dy = X[AM + a] - t1, dz = X[2 * AM + a] - t2;
                    S0 += Fx; S1 += Fy; S2 += Fz;
                    T0 += dy * Fz - dz * Fy; T1 += dz * Fx - dx * Fz; T2 += dx * Fy - dy * Fx;
                }
            }
            if (all) {
                g[0] = S0; g[1] = S1; g[2] = S2; g[3] = T0; g[4] = T1; g[5] = T2;
            } else {
                const float4 Pk = tp[k], Uk = tu[k];
                g[6 + k] = (T0 - (Pk.y * S2 - Pk.z * S1)) * Uk.x + (T1 - (Pk.z * S0 - Pk.x * S2)) * Uk.y +
                           (T2 - (Pk.x * S1 - Pk.y * S0)) * Uk.z;
            }
        }
    }
    e = warp_sum(e);
    __syncwarp();
    return e;
}

__device__ __forceinline__ float wdot(const float* a, const float* b, int D, int lane) {
    float s = 0.f;
    for (int i = lane; i < D; i += 32) s += a[i] * b[i];
    return warp_sum(s);
}
__device__ __forceinline__ double wdot64(const float* a, const float* b, int D, int lane) {
    double s = 0.0;
    for (int i = lane; i < D; i += 32) s += (double)a[i] * (double)b[i];
    return warp_sum_d(s);
}
__device__ __forceinline__ void wcopy(float* dst, const float* src, int D, int lane) {
    for (int i = lane; i < D; i += 32) dst[i] = src[i];
    __syncwarp();
}
// xn = x (+) alpha p: translation add, rotation-vector increment of the quaternion, torsion add (mckernel.py:256-265)
__device__ __forceinline__ void conf_step(float* xn, const float* x, const float* p, float alpha, int nt, int lane) {
    if (lane == 0) {
        xn[0] = x[0] + alpha * p[0]; xn[1] = x[1] + alpha * p[1]; xn[2] = x[2] + alpha * p[2];
        xn[3] = x[3]; xn[4] = x[4]; xn[5] = x[5]; xn[6] = x[6];
        quat_apply_rotvec(xn + 3, alpha * p[3], alpha * p[4], alpha * p[5]);
    }
    for (int k = lane; k < nt; k += 32) xn[7 + k] = x[7 + k] + alpha * p[6 + k];
    __syncwarp();
}
// out_i = -sum_j H_ij v_j; H symmetric, stored with lane i owning column i (conflict-free); two accumulators
__device__ __forceinline__ void neg_hv(const float* H, const float* v, float* out, int D, int lane) {
    for (int i = lane; i < D; i += 32) {
        float a0 = 0.f, a1 = 0.f;
        int j = 0;
        for (; j + 1 < D; j += 2) {
            a0 += H[j * D + i] * v[j];
            a1 += H[(j + 1) * D + i] * v[j + 1];
        }
        if (j < D) a0 += H[j * D + i] * v[j];
        out[i] = -(a0 + a1);
    }
    __syncwarp();
}

// Vina-1.2-style BFGS on state x (shared, in/out); returns the final energy (mckernel.py:267-326).
// The curvature scalar y.p and the update guard alpha * y.p >= eps are evaluated in float64.
// Not inlined: the MC kernel calls it from two sites (start optimisation and every step); one copy, with one
// inlined eval_eg, keeps the kernel small enough for the instruction cache (instruction-fetch stalls were the
// largest stall reason with four inlined copies of eval_eg).
template <int APL, typename GT, bool EX>
__device__ ADOCK_BFGS_ATTR float bfgs(float* ws, const WSLayout& L, float* x, int iters, const Chain<APL>& c_in,
                                   const SearchParams& P, const TypeTables& tt, int lane, unsigned& n_eval) {
    const Chain<APL> c = c_in;   // registers for the whole optimisation
    const int D = 6 + c.nt, S = 7 + c.nt;
    float* H = ws + L.H;
    float* g = ws + L.g;
    float* gn = ws + L.gn;
    float* go = ws + L.go;
    float* p = ws + L.p;
    float* y = ws + L.y;
    float* mhy = ws + L.mhy;
    float* xn = ws + L.xn;
    float* xo = ws + L.xo;
    // One evaluation per pass of this loop: the start point on the first pass, then the line-search trial points.
    // Keeping a single call site keeps a single inlined copy of eval_eg in the kernel.
    float f0 = 0.f, f_orig = 0.f, pg = 0.f, alpha = 1.f;
    int step = 0, trial = 0;
    bool first = true;
    while (true) {
        const float f = eval_eg<APL, GT, EX>(ws, L, first ? x : xn, first ? g : gn, c, P, tt, lane);
        ++n_eval;
        if (first) {
            first = false;
            f0 = f_orig = f;
            wcopy(xo, x, S, lane);
            wcopy(go, g, D, lane);
            for (int i = lane; i < D; i += 32)
                for (int j = 0; j < D; ++j) H[j * D + i] = (i == j) ? 1.f : 0.f;
            __syncwarp();
            if (iters <= 0) break;
            neg_hv(H, g, p, D, lane);
            pg = wdot(p, g, D, lane);
            alpha = 1.f;
            trial = 0;
            conf_step(xn, x, p, alpha, c.nt, lane);
            continue;
        }
        // Armijo test (c = 1e-4); up to 10 trials halving alpha. After a 10th failed trial the last point is taken
        // with alpha already halved, as in the reference's loop.
        if (!(f - f0 < 1e-4f * alpha * pg)) {
            alpha *= 0.5f;
            if (++trial < 10) {
                conf_step(xn, x, p, alpha, c.nt, lane);
                continue;
            }
        }
        for (int i = lane; i < D; i += 32) y[i] = gn[i] - g[i];
        __syncwarp();
        f0 = f;
        wcopy(x, xn, S, lane);
        const float gg = wdot(gn, gn, D, lane);
        wcopy(g, gn, D, lane);
        if (!(sqrtf(gg) >= 1e-5f)) break;
        const double yp = wdot64(y, p, D, lane);
        if (step == 0) {
            const float yy = wdot(y, y, D, lane);
            if (fabsf(yy) > EPSF) {
                const float dg = (float)((double)alpha * yp / (double)yy);
                for (int i = lane; i < D; i += 32)
                    for (int j = 0; j < D; ++j) H[j * D + i] = (i == j) ? dg : 0.f;
                __syncwarp();
            }
        }
        const double ayp = (double)alpha * yp;
        if (ayp >= (double)EPSF) {
            for (int i = lane; i < D; i += 32) mhy[i] = 0.f;
            neg_hv(H, y, mhy, D, lane);
            const float yhy = -wdot(y, mhy, D, lane);
            const float r = (float)(1.0 / ayp);
            const float c2 = alpha * alpha * (r * r * yhy + r);
            const float ar = alpha * r;
            for (int i = lane; i < D; i += 32) {
                const float mi = mhy[i], pi = p[i];
                for (int j = 0; j < D; ++j) H[j * D + i] += ar * (mi * p[j] + mhy[j] * pi) + c2 * pi * p[j];
            }
            __syncwarp();
        }
        if (++step >= iters) break;
        neg_hv(H, g, p, D, lane);
        pg = wdot(p, g, D, lane);
        alpha = 1.f;
        trial = 0;
        conf_step(xn, x, p, alpha, c.nt, lane);
    }
    if (!(f0 <= f_orig)) {
        f0 = f_orig;
        wcopy(x, xo, S, lane);
        wcopy(g, go, D, lane);
    }
    return f0;
}

// ------------------------------------------------------------------------------------------ proposal features
// sign(v) log(1 + |v|): energies and map values of any magnitude in a range the network handles
__device__ __forceinline__ float slog(float v) { return copysignf(log1pf(fabsf(v)), v); }

// Feature row (PROP_IN = 320 values, BF16) of state s (energy e) of ligand l, computed by one warp:
//   [0, 216)   27 samples x 8 maps: nearest-grid map values at the centroid + {-2, 0, 2} A per axis, as
//              sign(v) log(1 + |v|) (maps beyond the receptor's count are 0)
//   [216, 219) translation relative to the box centre / 10 A
//   [219, 223) orientation quaternion, sign chosen so that w >= 0
//   [223, 263) sin, cos of torsions 0..19 (0 beyond the ligand's torsion count)
//   [263, 275) heavy atoms / 64, torsions / 20, radius of gyration / 10, intra pairs / 2000, fraction of atoms
//              per map slot 0..7
//   ligand-best hint (hint: the lowest-energy state over the ligand's chains, PROP_HINT floats = t, q, torsions
//   0..19, energy at 27, valid flag at 28; all 0 when hint is NULL or not valid):
//   [275, 278) (t_hint - t) / 10 A
//   [278, 281) rotation vector of q_hint q^-1 (w >= 0) / pi
//   [281]      slog(e - e_hint)
//   [282]      slog(e) (0 when e is not finite)
//   [283]      1
//   [284, 288) 0
//   [288, 308) torsion differences theta_hint - theta wrapped to [-pi, pi), / pi (0 beyond the torsion count)
//   [308, 320) 0
template <typename GT>
__device__ ADOCK_COLD_ATTR void prop_features(const SearchParams& P, int l, const float* s, float e, const float* hint,
                                              __nv_bfloat16* out, int lane) {
    const int4 inf = P.info[l];
    const int na = inf.x, nt = inf.y, np = inf.z, ri = inf.w;
    const int nx = (int)P.dims[3 * ri], ny = (int)P.dims[3 * ri + 1], nz = (int)P.dims[3 * ri + 2];
    const long long n3 = (long long)nx * ny * nz;
    const int nm = P.nmaps ? min(P.nmaps[ri], 8) : 8;
    const GT* G = (const GT*)P.flat + P.offs[ri];
    if (lane < 27) {
        const float px = s[0] + 2.f * (float)(lane % 3 - 1), py = s[1] + 2.f * (float)((lane / 3) % 3 - 1),
                    pz = s[2] + 2.f * (float)(lane / 9 - 1);
        const int i = min(max(__float2int_rn((px - P.origin[3 * ri]) * P.inv_s), 0), nx - 1);
        const int j = min(max(__float2int_rn((py - P.origin[3 * ri + 1]) * P.inv_s), 0), ny - 1);
        const int k = min(max(__float2int_rn((pz - P.origin[3 * ri + 2]) * P.inv_s), 0), nz - 1);
        const long long idx = ((long long)i * ny + j) * nz + k;
        for (int q = 0; q < 8; ++q) {
            const float v = q < nm ? gload(G + q * n3 + idx) : 0.f;
            out[lane * 8 + q] = __float2bfloat16(slog(v));
        }
    }
    if (lane == 27) {
        for (int d = 0; d < 3; ++d)
            out[216 + d] = __float2bfloat16((s[d] - 0.5f * (P.lo[3 * ri + d] + P.hi[3 * ri + d])) * 0.1f);
        float qw = s[3], qx = s[4], qy = s[5], qz = s[6];
        const float nq = rsqrtf(qw * qw + qx * qx + qy * qy + qz * qz) * (qw < 0.f ? -1.f : 1.f);
        out[219] = __float2bfloat16(qw * nq); out[220] = __float2bfloat16(qx * nq);
        out[221] = __float2bfloat16(qy * nq); out[222] = __float2bfloat16(qz * nq);
        out[263] = __float2bfloat16(na / 64.f); out[264] = __float2bfloat16(nt / 20.f);
        out[265] = __float2bfloat16(P.rg[l] / 10.f); out[266] = __float2bfloat16(np / 2000.f);
    }
    if (lane < 20) {
        float sv = 0.f, cv = 0.f;
        if (lane < nt) __sincosf(s[7 + lane], &sv, &cv);
        out[223 + 2 * lane] = __float2bfloat16(sv);
        out[224 + 2 * lane] = __float2bfloat16(cv);
    }
    if (lane >= 24 && lane < 32) {   // fraction of atoms per map slot
        const int q = lane - 24;
        int cnt = 0;
        for (int a = 0; a < na; ++a) cnt += ((__float_as_int(P.atoms[(long long)l * P.AM + a].w) & 0xffff) == q);
        out[267 + q] = __float2bfloat16(na ? (float)cnt / na : 0.f);
    }
    // ligand-best hint
    const bool hv = hint != nullptr && hint[28] > 0.5f;
    if (lane == 0) {
        float f[9] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        if (hv) {
            for (int d = 0; d < 3; ++d) f[d] = (hint[d] - s[d]) * 0.1f;
            // r = q_hint * conj(q), both normalised; rotation vector 2 atan2(|v|, w) v / |v|
            const float na = rsqrtf(s[3] * s[3] + s[4] * s[4] + s[5] * s[5] + s[6] * s[6]);
            const float nb = rsqrtf(hint[3] * hint[3] + hint[4] * hint[4] + hint[5] * hint[5] + hint[6] * hint[6]);
            const float aw = s[3] * na, ax = -s[4] * na, ay = -s[5] * na, az = -s[6] * na;
            const float bw = hint[3] * nb, bx = hint[4] * nb, by = hint[5] * nb, bz = hint[6] * nb;
            float rw = bw * aw - bx * ax - by * ay - bz * az;
            float rx = bw * ax + bx * aw + by * az - bz * ay;
            float ry = bw * ay - bx * az + by * aw + bz * ax;
            float rz = bw * az + bx * ay - by * ax + bz * aw;
            if (rw < 0.f) { rw = -rw; rx = -rx; ry = -ry; rz = -rz; }
            const float sn = sqrtf(rx * rx + ry * ry + rz * rz);
            const float sc = sn > 1e-7f ? 2.f * atan2f(sn, rw) / sn : 2.f;
            f[3] = rx * sc * 0.31830988f; f[4] = ry * sc * 0.31830988f; f[5] = rz * sc * 0.31830988f;
            f[6] = isfinite(e) ? slog(e - hint[27]) : 0.f;
            f[8] = 1.f;
        }
        f[7] = (hv && isfinite(e)) ? slog(e) : 0.f;
        for (int i = 0; i < 9; ++i) out[275 + i] = __float2bfloat16(isfinite(f[i]) ? f[i] : 0.f);
        for (int i = 284; i < 288; ++i) out[i] = __float2bfloat16(0.f);
    }
    if (lane < 20) {
        float d = 0.f;
        if (hv && lane < nt) {
            d = hint[7 + lane] - s[7 + lane];
            d = d - 6.2831853f * floorf((d + 3.14159265f) * 0.15915494f);
            d = isfinite(d) ? d * 0.31830988f : 0.f;
        }
        out[288 + lane] = __float2bfloat16(d);
    }
    if (lane < 12) out[308 + lane] = __float2bfloat16(0.f);
    __syncwarp();
}

// True on all lanes when a learned target state (t, q and the ligand's first 20 torsions in x) is finite. A non-finite
// target is never optimised: clamped map lookups and ramps can give non-finite coordinates a finite energy.
__device__ __forceinline__ bool target_finite(const float* x, int nt, int lane) {
    bool ok = true;
    if (lane < 7) ok = isfinite(x[lane]);
    for (int k = lane; k < nt && k < 20; k += 32) ok = ok && isfinite(x[7 + k]);
    return __all_sync(0xffffffffu, ok);
}

// Training-log row of a state (lane 0 writes): t (3), q (4), theta 0..19 (0 past the torsion count), torsion
// count at 27, chain index at 28; the training target (the move to a later state of the same chain) is computed
// after the run.
static __device__ ADOCK_COLD_ATTR void log_state(const float* s, int nt, int ch, float* y) {
    for (int i = 0; i < 7; ++i) y[i] = s[i];
    for (int t = 0; t < 20; ++t) y[7 + t] = t < nt ? s[7 + t] : 0.f;
    y[27] = (float)nt;
    y[28] = (float)ch;
    for (int t = 29; t < 32; ++t) y[t] = 0.f;
}

template <int APL, typename GT, int MINB, bool EX>
__global__ void __launch_bounds__(128, MINB) mc_kernel(const __grid_constant__ SearchParams P,
                                                       const __grid_constant__ McParams M,
                                                       const __grid_constant__ TypeTables ttg) {
    extern __shared__ float4 smem4[];
    __shared__ TypeTables tt;
    stage_tables(tt, ttg);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const WSLayout L(P.AM, P.KM);
    float* ws = (float*)smem4 + (size_t)wid * L.total;
    const int SDM = 7 + P.KM;
    unsigned n_eval = 0;
    unsigned long long n_atom_eval = 0;
    while (true) {
        int idx = 0;
        if (lane == 0) idx = atomicAdd(M.queue, 1);
        idx = __shfl_sync(0xffffffffu, idx, 0);
        if (idx >= M.n_chains) break;
        const int ch = M.order ? M.order[idx] : idx;
        const int l = M.chain_lig[ch];
        if (M.lig_active && M.lig_active[l] == 0) continue;
        const int cid = M.chain_id[ch];
        const unsigned n_eval_start = n_eval;
        Chain<APL> c;
        const int* nb = M.nbr ? M.nbr + (long long)ch * M.nb_max : nullptr;
        const int nbn = M.nbr ? M.nbr_n[ch] : 0;
        load_chain<APL, GT>(c, P, l, ws, L, lane, M.exact, nb, nbn);
        const int S = 7 + c.nt;
        const int iters = M.bfgs_iters > 0 ? M.bfgs_iters : (25 + c.na) / 3;
        float* cur = ws + L.cur;
        float* best = ws + L.best;
        float* x = ws + L.x;
        float* gcur = M.cur + (long long)ch * SDM;
        float* gbest = M.best + (long long)ch * SDM;
        for (int i = lane; i < S; i += 32) {
            cur[i] = gcur[i];
            best[i] = gbest[i];
        }
        __syncwarp();
        float ec, eb = M.best_e[ch];
        if (M.init_opt) ec = bfgs<APL, GT, EX>(ws, L, cur, iters, c, P, tt, lane, n_eval);
        else ec = M.cur_e[ch];
        if (ec < eb) {
            eb = ec;
            wcopy(best, cur, S, lane);
        }
        int prop_fail = 0;
        unsigned long long n_prop = 0, n_prop_acc = 0, n_plain = 0, n_plain_acc = 0;
        for (int st = 0; st < M.mc_steps; ++st) {
            const int sg = M.step_offset + st;
            wcopy(x, cur, S, lane);
            // learned move while the proposal has not failed PROP_FAIL_MAX times in a row, else plain MC
            const bool use_prop = M.prop && prop_fail < PROP_FAIL_MAX &&
                                  (M.prop_frac >= 1.f || uniform01(M.seed, cid, sg, 3) < M.prop_frac);
            bool skip = false;   // a non-finite learned target: rejected without optimisation
            if (use_prop) {
                // the proposed target state (drawn around the state the network read at the segment start); with
                // several tries per step, each candidate is evaluated once and the lowest-energy one is kept
                const int T = M.prop_tries > 1 ? M.prop_tries : 1;
                const float* mv0 = M.prop + ((long long)ch * M.prop_k + (long long)(st % (M.prop_k / T)) * T) * PROP_MOVE;
                int pick = 0;
                if (T > 1) {
                    float e_min = 3.4e38f;
                    for (int tr = 0; tr < T; ++tr) {
                        const float* mv = mv0 + (long long)tr * PROP_MOVE;
                        for (int i = lane; i < S; i += 32) x[i] = cur[i];
                        __syncwarp();
                        if (lane < 7) x[lane] = mv[lane];
                        for (int k = lane; k < c.nt && k < 20; k += 32) x[7 + k] = mv[7 + k];
                        __syncwarp();
                        if (!target_finite(x, c.nt, lane)) continue;
                        const float et = bfgs<APL, GT, EX>(ws, L, x, 0, c, P, tt, lane, n_eval);   // one evaluation
                        if (et < e_min) { e_min = et; pick = tr; }
                    }
                    wcopy(x, cur, S, lane);
                }
                const float* mv = mv0 + (long long)pick * PROP_MOVE;
                if (lane < 7) x[lane] = mv[lane];
                for (int k = lane; k < c.nt && k < 20; k += 32) x[7 + k] = mv[7 + k];
                __syncwarp();
                skip = !target_finite(x, c.nt, lane);
            } else {
                const int nm = 2 + c.nt;
                const int which = min((int)(uniform01(M.seed, cid, sg, 0) * nm), nm - 1);
                if (lane == 0) {
                    float v[3];
                    if (which == 0) {
                        unit_ball(M.seed, cid, sg, 10, v);
                        x[0] += M.amp_pos * v[0]; x[1] += M.amp_pos * v[1]; x[2] += M.amp_pos * v[2];
                    } else if (which == 1) {
                        unit_ball(M.seed, cid, sg, 10, v);
                        const float sc = M.amp_rot / fmaxf(c.rg, 1.0f);
                        quat_apply_rotvec(x + 3, sc * v[0], sc * v[1], sc * v[2]);
                    } else {
                        x[7 + which - 2] = (2.f * uniform01(M.seed, cid, sg, 1) - 1.f) * 3.14159265f;
                    }
                }
            }
            __syncwarp();
            const float en = skip ? 3.4e38f : bfgs<APL, GT, EX>(ws, L, x, iters, c, P, tt, lane, n_eval);
            const bool accept =
                isfinite(en) && ((en < ec) || (uniform01(M.seed, cid, sg, 2) < __expf((ec - en) / M.temp)));
            if (use_prop) { ++n_prop; n_prop_acc += accept; } else { ++n_plain; n_plain_acc += accept; }
            prop_fail = accept ? 0 : (use_prop ? prop_fail + 1 : prop_fail);
            if (accept && en < ec && M.log_x) {   // training data: features of the pre-move state + the move
                int row = 0;
                if (lane == 0) row = atomicAdd(M.log_n, 1);
                row = __shfl_sync(0xffffffffu, row, 0);
                if (row < M.log_cap) {
                    prop_features<GT>(P, l, cur, ec, M.hint ? M.hint + (long long)l * PROP_HINT : nullptr,
                                      M.log_x + (long long)row * PROP_IN, lane);
                    if (lane == 0) log_state(cur, c.nt, ch, M.log_y + (long long)row * PROP_MOVE);
                }
                __syncwarp();
            }
            if (accept) {
                ec = en;
                wcopy(cur, x, S, lane);
                if (en < eb) {
                    eb = en;
                    wcopy(best, x, S, lane);
                }
            }
        }
        if (M.prop_stats && lane == 0 && M.mc_steps > 0) {
            atomicAdd(&M.prop_stats[0], n_prop); atomicAdd(&M.prop_stats[1], n_prop_acc);
            atomicAdd(&M.prop_stats[2], n_plain); atomicAdd(&M.prop_stats[3], n_plain_acc);
        }
        for (int i = lane; i < S; i += 32) {
            gcur[i] = cur[i];
            gbest[i] = best[i];
        }
        if (lane == 0) {
            M.cur_e[ch] = ec;
            M.best_e[ch] = eb;
        }
        n_atom_eval += (unsigned long long)(n_eval - n_eval_start) * c.na;
        __syncwarp();
    }
    if (M.evals && lane == 0 && n_eval) {
        atomicAdd(&M.evals[0], (unsigned long long)n_eval);
        atomicAdd(&M.evals[1], n_atom_eval);
    }
}

template <int APL, typename GT, bool EX>
__global__ void __launch_bounds__(128) eg_kernel(const __grid_constant__ SearchParams P, const int* chain_lig, int n,
                                                 const float* state, float* e_out, float* g_out, int exact,
                                                 const __grid_constant__ TypeTables ttg) {
    extern __shared__ float4 smem4[];
    __shared__ TypeTables tt;
    stage_tables(tt, ttg);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const WSLayout L(P.AM, P.KM);
    float* ws = (float*)smem4 + (size_t)wid * L.total;
    const int SDM = 7 + P.KM, DMM = 6 + P.KM;
    const int warps = (blockDim.x >> 5) * gridDim.x;
    for (int ch = blockIdx.x * (blockDim.x >> 5) + wid; ch < n; ch += warps) {
        const int l = chain_lig[ch];
        Chain<APL> c;
        load_chain<APL, GT>(c, P, l, ws, L, lane, exact, nullptr, 0);
        float* x = ws + L.x;
        float* g = ws + L.g;
        for (int i = lane; i < SDM; i += 32) x[i] = state[(long long)ch * SDM + i];
        __syncwarp();
        const float e = eval_eg<APL, GT, EX>(ws, L, x, g, c, P, tt, lane);
        for (int i = lane; i < 6 + c.nt; i += 32) g_out[(long long)ch * DMM + i] = g[i];
        if (lane == 0) e_out[ch] = e;
        __syncwarp();
    }
}

// ------------------------------------------------------------------------------------------ Stage A
// Block = (ligand l, conformer c, rotation q); threads over lattice translations; e(T) = sum_a min(cap,
// nearest-grid energy + out-of-box penalty); block min and argmin (ties -> lowest index), mckernel.py:451-521.
template <typename GT>
__global__ void __launch_bounds__(256) stage_a_kernel(const __grid_constant__ SearchParams P, const float* conf, int C,
                                                      const float* quats, int Q, const float* trans,
                                                      const int* ntrans, int NT_MAX, const int* lig_box,
                                                      float cap, float* best_e, int* best_i) {
    extern __shared__ float4 smem4[];
    float4* X = smem4;  // [AM] rotated conformer + slot bits
    __shared__ float red_e[256];
    __shared__ int red_i[256];
    const long long b = blockIdx.x;
    const int q = (int)(b % Q);
    const int cc = (int)((b / Q) % C);
    const int l = (int)(b / ((long long)Q * C));
    const int4 inf = P.info[l];
    const int n_at = inf.x, ri = inf.w;
    float qw = quats[4 * q], qx = quats[4 * q + 1], qy = quats[4 * q + 2], qz = quats[4 * q + 3];
    const float nq = rsqrtf(qw * qw + qx * qx + qy * qy + qz * qz);
    qw *= nq; qx *= nq; qy *= nq; qz *= nq;
    for (int a = threadIdx.x; a < n_at; a += blockDim.x) {
        const float* p = conf + (((long long)l * C + cc) * P.AM + a) * 3;
        const float px = p[0], py = p[1], pz = p[2];
        const int slot = __float_as_int(P.atoms[(long long)l * P.AM + a].w) & 0xffff;
        X[a] = make_float4((1 - 2 * (qy * qy + qz * qz)) * px + 2 * (qx * qy - qz * qw) * py + 2 * (qx * qz + qy * qw) * pz,
                           2 * (qx * qy + qz * qw) * px + (1 - 2 * (qx * qx + qz * qz)) * py + 2 * (qy * qz - qx * qw) * pz,
                           2 * (qx * qz - qy * qw) * px + 2 * (qy * qz + qx * qw) * py + (1 - 2 * (qx * qx + qy * qy)) * pz,
                           __int_as_float(slot));
    }
    __syncthreads();
    const GT* G = (const GT*)P.flat + P.offs[ri];
    const int nx = (int)P.dims[3 * ri], ny = (int)P.dims[3 * ri + 1], nz = (int)P.dims[3 * ri + 2];
    const long long n3 = (long long)nx * ny * nz;
    const float ox = P.origin[3 * ri], oy = P.origin[3 * ri + 1], oz = P.origin[3 * ri + 2];
    const float lx = P.lo[3 * ri], ly = P.lo[3 * ri + 1], lz = P.lo[3 * ri + 2];
    const float hx = P.hi[3 * ri], hy = P.hi[3 * ri + 1], hz = P.hi[3 * ri + 2];
    const float inv = P.inv_s, pen = P.pen;
    float be = 3.4e38f;
    int bi = 0;
    const int box = lig_box ? lig_box[l] : l;   // translations per ligand, or per box shared by ligands
    const int nT = ntrans[box];
    for (int ti = threadIdx.x; ti < nT; ti += blockDim.x) {
        const float* T = trans + ((long long)box * NT_MAX + ti) * 3;
        const float T0 = T[0], T1 = T[1], T2 = T[2];
        float e = 0.f;
        for (int a = 0; a < n_at; ++a) {
            const float4 v = X[a];
            const float x = v.x + T0, y = v.y + T1, z = v.z + T2;
            const int i = min(max(__float2int_rn((x - ox) * inv), 0), nx - 1);
            const int j = min(max(__float2int_rn((y - oy) * inv), 0), ny - 1);
            const int k = min(max(__float2int_rn((z - oz) * inv), 0), nz - 1);
            float ea = gload(G + (long long)__float_as_int(v.w) * n3 + ((long long)i * ny + j) * nz + k);
            const float dx0 = fmaxf(lx - x, 0.f), dx1 = fmaxf(x - hx, 0.f);
            const float dy0 = fmaxf(ly - y, 0.f), dy1 = fmaxf(y - hy, 0.f);
            const float dz0 = fmaxf(lz - z, 0.f), dz1 = fmaxf(z - hz, 0.f);
            ea += pen * (dx0 * dx0 + dx1 * dx1 + dy0 * dy0 + dy1 * dy1 + dz0 * dz0 + dz1 * dz1);
            e += fminf(ea, cap);
        }
        if (e < be) { be = e; bi = ti; }
    }
    red_e[threadIdx.x] = be;
    red_i[threadIdx.x] = bi;
    __syncthreads();
    for (int sft = blockDim.x / 2; sft > 0; sft >>= 1) {
        if (threadIdx.x < sft) {
            const float o = red_e[threadIdx.x + sft];
            const int oi = red_i[threadIdx.x + sft];
            if (o < red_e[threadIdx.x] || (o == red_e[threadIdx.x] && oi < red_i[threadIdx.x])) {
                red_e[threadIdx.x] = o;
                red_i[threadIdx.x] = oi;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        best_e[b] = red_e[0];
        best_i[b] = red_i[0];
    }
}

// ------------------------------------------------------------------------------------------ float64 re-score
// One warp per state: float64 forward kinematics, exact pairwise inter energy over all receptor atoms (or the
// grid interpolated in float64 when no receptor atoms are given), out-of-box penalty, intra pairs.
template <typename GT>
__global__ void __launch_bounds__(128) rescore64_kernel(const __grid_constant__ SearchParams P, const int* chain_lig, int n,
                                                        const float* state, double* e_total, double* e_intra,
                                                        float* Xout, const __grid_constant__ TypeTables ttg,
                                                        const __grid_constant__ adock_sf_t sf) {
    extern __shared__ double smemd[];
    __shared__ TypeTables tt;
    stage_tables(tt, ttg);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double* X = smemd + (size_t)wid * P.AM * 3;
    const int SDM = 7 + P.KM;
    const int ch = blockIdx.x * (blockDim.x >> 5) + wid;
    if (ch >= n) return;
    const int l = chain_lig[ch];
    const int4 inf = P.info[l];
    const int na = inf.x, nt = inf.y, np = inf.z, ri = inf.w;
    const float* s = state + (long long)ch * SDM;
    double qw = s[3], qx = s[4], qy = s[5], qz = s[6];
    const double nq = 1.0 / sqrt(qw * qw + qx * qx + qy * qy + qz * qz);
    qw *= nq; qx *= nq; qy *= nq; qz *= nq;
    const double R00 = 1 - 2 * (qy * qy + qz * qz), R01 = 2 * (qx * qy - qz * qw), R02 = 2 * (qx * qz + qy * qw);
    const double R10 = 2 * (qx * qy + qz * qw), R11 = 1 - 2 * (qx * qx + qz * qz), R12 = 2 * (qy * qz - qx * qw);
    const double R20 = 2 * (qx * qz - qy * qw), R21 = 2 * (qy * qz + qx * qw), R22 = 1 - 2 * (qx * qx + qy * qy);
    const float4* tr = P.tors + (long long)l * P.KM * 2;
    double einter = 0.0, eintra = 0.0;
    const double cut = P.pp.cutoff;
    for (int a = lane; a < na; a += 32) {
        const float4 v = P.atoms[(long long)l * P.AM + a];
        double px = v.x, py = v.y, pz = v.z;
        uint32_t m = P.masks[(long long)l * P.AM + a];
        while (m) {
            const int k = __ffs(m) - 1;
            m &= m - 1;
            if (k >= nt) break;
            const float4 A = tr[2 * k], U = tr[2 * k + 1];
            double sv, cv;
            sincos((double)s[7 + k], &sv, &cv);
            const double vx = px - A.x, vy = py - A.y, vz = pz - A.z;
            const double d = U.x * vx + U.y * vy + U.z * vz;
            const double cx = U.y * vz - U.z * vy, cy = U.z * vx - U.x * vz, cz = U.x * vy - U.y * vx;
            px = A.x + vx * cv + cx * sv + U.x * d * (1 - cv);
            py = A.y + vy * cv + cy * sv + U.y * d * (1 - cv);
            pz = A.z + vz * cv + cz * sv + U.z * d * (1 - cv);
        }
        const double X0 = R00 * px + R01 * py + R02 * pz + s[0];
        const double X1 = R10 * px + R11 * py + R12 * pz + s[1];
        const double X2 = R20 * px + R21 * py + R22 * pz + s[2];
        X[3 * a] = X0; X[3 * a + 1] = X1; X[3 * a + 2] = X2;
        Xout[((long long)ch * P.AM + a) * 3] = (float)X0;
        Xout[((long long)ch * P.AM + a) * 3 + 1] = (float)X1;
        Xout[((long long)ch * P.AM + a) * 3 + 2] = (float)X2;
        const int meta = __float_as_int(v.w);
        const int ta = (meta >> 16) & 63, slot = meta & 0xffff;
        double ea = 0.0;
        if (P.rxyz) {
            const float* rx = P.rxyz + (long long)ri * P.RN * 3;
            const int* rt = P.rtyp + (long long)ri * P.RN;
            const int rn = P.rn[ri];
            const int fa = tt.flags[ta];
            for (int b = 0; b < rn; ++b) {
                const double dx = X0 - rx[3 * b], dy = X1 - rx[3 * b + 1], dz = X2 - rx[3 * b + 2];
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 >= cut * cut) continue;
                const int tb = rt[b] & 63, fb = tt.flags[tb];
                ea += pair_energy64(sqrt(r2), (double)tt.radius[ta] + (double)tt.radius[tb],
                                    hyd_pair(fa, fb) | hb_pair(fa, fb), sf.prm);
            }
        } else {
            const GT* G = (const GT*)P.flat + P.offs[ri];
            const long long nx = P.dims[3 * ri], ny = P.dims[3 * ri + 1], nz = P.dims[3 * ri + 2];
            const double xx[3] = {X0, X1, X2};
            const double nn[3] = {(double)nx, (double)ny, (double)nz};
            double fw[3];
            long long i0[3];
            for (int d = 0; d < 3; ++d) {
                const double f = (xx[d] - P.origin[3 * ri + d]) / (double)(1.0f / P.inv_s);
                const double fc = fmin(fmax(f, 0.0), nn[d] - 1.0 - 1e-4);
                i0[d] = (long long)floor(fc);
                fw[d] = fc - (double)i0[d];
            }
            const GT* Gs = G + (long long)slot * nx * ny * nz;
            for (int dx = 0; dx < 2; ++dx)
                for (int dy = 0; dy < 2; ++dy)
                    for (int dz = 0; dz < 2; ++dz) {
                        const double w = (dx ? fw[0] : 1 - fw[0]) * (dy ? fw[1] : 1 - fw[1]) * (dz ? fw[2] : 1 - fw[2]);
                        ea += w * (double)gload(Gs + ((i0[0] + dx) * ny + (i0[1] + dy)) * nz + (i0[2] + dz));
                    }
        }
        const double xx[3] = {X0, X1, X2};
        for (int d = 0; d < 3; ++d) {
            const double lo = fmax((double)P.lo[3 * ri + d] - xx[d], 0.0), hi = fmax(xx[d] - (double)P.hi[3 * ri + d], 0.0);
            ea += (double)P.pen * (lo * lo + hi * hi);
        }
        einter += ea;
    }
    __syncwarp();
    const int2* pairs = P.pairs + (long long)l * P.P_pad;
    const int nslot = ((np + 31) >> 5) << 5;
    for (int q = lane; q < nslot; q += 32) {
        const int2 pr = pairs[q];
        if (pr.x < 0) continue;
        const int i = pr.x & 0xff, j = (pr.x >> 8) & 0xff, fl = pr.x >> 16;
        const double dx = X[3 * i] - X[3 * j], dy = X[3 * i + 1] - X[3 * j + 1], dz = X[3 * i + 2] - X[3 * j + 2];
        const double r = sqrt(dx * dx + dy * dy + dz * dz);
        if (r >= cut) continue;
        const int ti = (__float_as_int(P.atoms[(long long)l * P.AM + i].w) >> 16) & 63;
        const int tj = (__float_as_int(P.atoms[(long long)l * P.AM + j].w) >> 16) & 63;
        eintra += pair_energy64(r, (double)tt.radius[ti] + (double)tt.radius[tj], fl, sf.prm);
    }
    einter = warp_sum_d(einter);
    eintra = warp_sum_d(eintra);
    if (lane == 0) {
        e_total[ch] = einter + eintra;
        e_intra[ch] = eintra;
    }
}

// feature rows of n states (one warp per state); cur_e [n] and hint [L, PROP_HINT] may be NULL
template <typename GT>
__global__ void __launch_bounds__(128) prop_features_kernel(const __grid_constant__ SearchParams P, const int* chain_lig,
                                                            int n, const float* state, const float* cur_e,
                                                            const float* hint, __nv_bfloat16* out) {
    __shared__ float s[4][7 + 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int ch = blockIdx.x * 4 + wid;
    if (ch >= n) return;
    const int SDM = 7 + P.KM;
    for (int i = lane; i < SDM && i < 7 + 32; i += 32) s[wid][i] = state[(long long)ch * SDM + i];
    __syncwarp();
    const int l = chain_lig[ch];
    prop_features<GT>(P, l, s[wid], cur_e ? cur_e[ch] : 0.f, hint ? hint + (long long)l * PROP_HINT : nullptr,
                      out + (long long)ch * PROP_IN, lane);
}

// ------------------------------------------------------------------------------------------ launchers
// Launch variants of the persistent MC kernel (128 threads per block): minimum resident blocks per SM, which
// caps registers per thread (4 -> 128, 6 -> 80, 8 -> 64). Variant 0 is the default.
static const int MC_VARIANT_MINB[4] = {4, 4, 6, 8};

template <int APL, typename GT, int MINB>
static int launch_mc_v(const SearchParams& P, const McParams& M, const TypeTables& tt, cudaStream_t st) {
    const int wpb = 4;
    const WSLayout L(P.AM, P.KM);
    const size_t smem = (size_t)wpb * L.total * sizeof(float);
    auto kern = M.exact ? mc_kernel<APL, GT, MINB, true> : mc_kernel<APL, GT, MINB, false>;
    ADOCK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    ADOCK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 32 * wpb, smem));
    if (per_sm < 1) per_sm = 1;
    long long blocks = (long long)sm_count() * per_sm;
    const long long need = (M.n_chains + wpb - 1) / wpb;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    ADOCK_CUDA(cudaMemsetAsync(M.queue, 0, sizeof(int), st));
    kern<<<(unsigned)blocks, 32 * wpb, smem, st>>>(P, M, tt);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

template <int APL, typename GT>
static int launch_mc_apl(const SearchParams& P, const McParams& M, const TypeTables& tt, cudaStream_t st, int variant) {
    switch (MC_VARIANT_MINB[(variant >= 0 && variant < 4) ? variant : 0]) {
        case 6: return launch_mc_v<APL, GT, 6>(P, M, tt, st);
        case 8: return launch_mc_v<APL, GT, 8>(P, M, tt, st);
        default: return launch_mc_v<APL, GT, 4>(P, M, tt, st);
    }
}

template <typename GT>
int launch_mc(const SearchParams& P, const McParams& M, const TypeTables& tt, cudaStream_t st, int variant) {
    switch (P.AM / 32) {
        case 1: return launch_mc_apl<1, GT>(P, M, tt, st, variant);
        case 2: return launch_mc_apl<2, GT>(P, M, tt, st, variant);
        case 3: return launch_mc_apl<3, GT>(P, M, tt, st, variant);
        default: return launch_mc_apl<4, GT>(P, M, tt, st, variant);
    }
}

template <int APL, typename GT>
static int launch_eg_t(const SearchParams& P, const int* cl, int n, const float* state, float* e, float* g, int exact,
                       const TypeTables& tt, cudaStream_t st) {
    const int wpb = 4;
    const WSLayout L(P.AM, P.KM);
    const size_t smem = (size_t)wpb * L.total * sizeof(float);
    auto kern = exact ? eg_kernel<APL, GT, true> : eg_kernel<APL, GT, false>;
    ADOCK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    long long blocks = (n + wpb - 1) / wpb;
    const long long cap = (long long)sm_count() * 16;
    if (blocks > cap) blocks = cap;
    kern<<<(unsigned)blocks, 32 * wpb, smem, st>>>(P, cl, n, state, e, g, exact, tt);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

template <typename GT>
int launch_eg(const SearchParams& P, const int* cl, int n, const float* state, float* e, float* g, int exact,
              const TypeTables& tt, cudaStream_t st) {
    switch (P.AM / 32) {
        case 1: return launch_eg_t<1, GT>(P, cl, n, state, e, g, exact, tt, st);
        case 2: return launch_eg_t<2, GT>(P, cl, n, state, e, g, exact, tt, st);
        case 3: return launch_eg_t<3, GT>(P, cl, n, state, e, g, exact, tt, st);
        default: return launch_eg_t<4, GT>(P, cl, n, state, e, g, exact, tt, st);
    }
}

template <typename GT>
int launch_stage_a(const SearchParams& P, long long blocks, const float* conf, int C, const float* quats, int Q,
                   const float* trans, const int* ntrans, int nt_max, const int* lig_box, float cap, float* best_e,
                   int* best_i, cudaStream_t st) {
    const size_t smem = (size_t)P.AM * sizeof(float4);
    stage_a_kernel<GT><<<(unsigned)blocks, 256, smem, st>>>(P, conf, C, quats, Q, trans, ntrans, nt_max, lig_box, cap,
                                                            best_e, best_i);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

template <typename GT>
int launch_rescore64(const SearchParams& P, const int* cl, int n, const float* state, double* et, double* ei, float* X,
                     const TypeTables& tt, const adock_sf_t& sf, cudaStream_t st) {
    const int wpb = 4;
    const size_t smem = (size_t)wpb * P.AM * 3 * sizeof(double);
    const unsigned blocks = (unsigned)((n + wpb - 1) / wpb);
    rescore64_kernel<GT><<<blocks, 32 * wpb, smem, st>>>(P, cl, n, state, et, ei, X, tt, sf);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

template <typename GT>
int launch_prop_features(const SearchParams& P, const int* cl, int n, const float* state, const float* cur_e,
                         const float* hint, __nv_bfloat16* out, cudaStream_t st) {
    prop_features_kernel<GT><<<(unsigned)((n + 3) / 4), 128, 0, st>>>(P, cl, n, state, cur_e, hint, out);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

#define ADOCK_SEARCH_INSTANTIATE(GT)                                                                              \
    template int launch_prop_features<GT>(const SearchParams&, const int*, int, const float*, const float*,       \
                                          const float*, __nv_bfloat16*, cudaStream_t);                            \
    template int launch_mc<GT>(const SearchParams&, const McParams&, const TypeTables&, cudaStream_t, int);       \
    template int launch_eg<GT>(const SearchParams&, const int*, int, const float*, float*, float*, int,           \
                               const TypeTables&, cudaStream_t);                                                  \
    template int launch_stage_a<GT>(const SearchParams&, long long, const float*, int, const float*, int,         \
                                    const float*, const int*, int, const int*, float, float*, int*,              \
                                    cudaStream_t);                                                                \
    template int launch_rescore64<GT>(const SearchParams&, const int*, int, const float*, double*, double*,       \
                                      float*, const TypeTables&, const adock_sf_t&, cudaStream_t);

#define ADOCK_SEARCH_EXTERN(GT)                                                                                   \
    extern template int launch_prop_features<GT>(const SearchParams&, const int*, int, const float*, const float*, \
                                                 const float*, __nv_bfloat16*, cudaStream_t);                     \
    extern template int launch_mc<GT>(const SearchParams&, const McParams&, const TypeTables&, cudaStream_t, int); \
    extern template int launch_eg<GT>(const SearchParams&, const int*, int, const float*, float*, float*, int,    \
                                      const TypeTables&, cudaStream_t);                                           \
    extern template int launch_stage_a<GT>(const SearchParams&, long long, const float*, int, const float*, int,  \
                                           const float*, const int*, int, const int*, float, float*, int*,       \
                                           cudaStream_t);                                                         \
    extern template int launch_rescore64<GT>(const SearchParams&, const int*, int, const float*, double*,         \
                                             double*, float*, const TypeTables&, const adock_sf_t&, cudaStream_t);

// host helpers shared by the translation units of the search (defined in search.cu)
TypeTables make_tables(const adock_sf_t* sf);
int make_params(SearchParams& P, const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
                const adock_sf_t* sf, const adock_receptors_t* rec);

}  // namespace adock
