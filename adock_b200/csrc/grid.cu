// Receptor grid maps (sm_100a): Vina/Vinardo per-ligand-type maps and the fitted function's maps.
//
// The reference launches one thread per grid point that scans every receptor atom (grid.py:24-61,
// gridfit.py:21-57). Here a 128-thread CTA owns a 4 x 4 x 8 tile of points (z fastest, one warp per x-plane
// patch). The receptor comes as a cell list: atoms sorted by cell of a uniform grid, with the start of every cell.
// A CTA visits only the cells that overlap its tile's bounding box grown by the cutoff (columns of cells along z
// are contiguous in the sorted atoms), keeps the atoms inside the grown box in shared memory (ordered compaction)
// and each thread then evaluates its point against the staged atoms. Without a cell list (one cell holding every
// atom in receptor order) this is a scan of the whole receptor per CTA, and the summation order per point is the
// reference's receptor order; with one, it is the cell order.
//
// The distance-dependent parts of the terms depend on the ligand type only through its radius: the types of a
// launch are processed in order of radius (a permutation kept for the output), and the Gaussians, the repulsion
// and the two ramps are evaluated once per distinct radius and reused by the types that share it. Unweighted term
// sums are kept per type in registers (groups of 8 types) and weighted once at the end, the same order of
// operations as the reference kernel.
#include "common.cuh"

namespace adock {

#define TILE_X 4
#define TILE_Y 4
#define TILE_Z 8
#define TILE_THREADS 128
#define STAGE_CAP 2048
// The fitted kernel stages fewer atoms per pass: its per-block weight slice (receptor types x 8 ligand types x 6
// basis weights, 21 KB for the 108 receptor ext types) and 896 staged atoms (14 KB) fit 6 blocks per SM; at the
// 2,048 of the Vina kernel only 4 fit. A tile's cutoff region holds a few hundred atoms at protein density, so
// one pass still covers it.
#define FIT_STAGE_CAP 896
#define VINA_GROUP 8
#define FIT_GROUP 8
#define MAX_COLUMNS 64

struct VinaPrm {
    float cutoff, g1_off, g1_inv, g2_off, g2_inv, rep_off, hyd_good, hyd_bad, hyd_inv, hb_good, hb_bad, hb_inv;
    float w[5];
    int n_lt, n_xs, per_term;
    int lig_types[24];   // in order of radius
    int out_slot[24];    // output map of each (radius-ordered) type
    float radius[64];
    int flags[64];  // bit0 hydrophobic, bit1 donor, bit2 acceptor
};

struct FitPrm {
    float cutoff, g1_off, g1_inv, g2_off, g2_inv, rep_off, hyd_good, hyd_bad, hyd_inv, hb_good, hb_bad, hb_inv;
    float ion_rmin, rep_cap;
    int n_lt, n_rt;
    float rad_lig[64];   // in order of radius
    int out_slot[64];    // output map (and W column) of each (radius-ordered) type
};

// Uniform cell grid over the receptor: cell (cx, cy, cz) holds sorted atoms [start[c], start[c + 1]) with
// c = (cx * ny + cy) * nz + cz. start == NULL: one cell holding all n atoms in receptor order.
struct Cells {
    const int* start;
    int nx, ny, nz;
    float ox, oy, oz, size;
};

// The columns of cells (fixed cx, cy; the cz range of the box) that overlap [lo, hi]: begin and length of each
// column's atom range, prefix sums in off[0..ncol]. Called by all threads; returns the number of columns.
__device__ int tile_columns(const Cells& C, int n_rec, const float* lo, const float* hi, int* begin, int* off) {
    if (threadIdx.x == 0) {
        int nc = 0;
        if (!C.start) {
            begin[0] = 0;
            off[0] = 0;
            off[1] = n_rec;
            nc = 1;
        } else {
            auto cell = [&](float v, float o, int n) { return min(max((int)floorf((v - o) / C.size), 0), n - 1); };
            const int x0 = cell(lo[0], C.ox, C.nx), x1 = cell(hi[0], C.ox, C.nx);
            const int y0 = cell(lo[1], C.oy, C.ny), y1 = cell(hi[1], C.oy, C.ny);
            const int z0 = cell(lo[2], C.oz, C.nz), z1 = cell(hi[2], C.oz, C.nz);
            int acc = 0;
            off[0] = 0;
            for (int cx = x0; cx <= x1; ++cx)
                for (int cy = y0; cy <= y1 && nc < MAX_COLUMNS; ++cy) {
                    const int c = (cx * C.ny + cy) * C.nz;
                    const int b = C.start[c + z0], e = C.start[c + z1 + 1];
                    begin[nc] = b;
                    acc += e - b;
                    off[++nc] = acc;
                }
        }
        begin[MAX_COLUMNS] = nc;
    }
    __syncthreads();
    return begin[MAX_COLUMNS];
}

// Stage the atoms inside [lo, hi] (per axis) from position `start` of the concatenated columns, at most CAP
// (a multiple of TILE_THREADS); returns the position where staging stopped (the total when all atoms were seen).
// Staged order = column order.
template <int CAP>
__device__ __forceinline__ int stage_atoms(const float* __restrict__ rxyz, const int* __restrict__ rtype,
                                           const int* begin, const int* off, int ncol, int start, const float* lo,
                                           const float* hi, float4* S, int* count, int* wsum) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int total = off[ncol];
    int n = 0;
    int v0 = start;
    for (; v0 < total; v0 += TILE_THREADS) {
        if (n + TILE_THREADS > CAP) break;
        const int v = v0 + tid;
        bool in = false;
        float x = 0.f, y = 0.f, z = 0.f;
        int t = 0;
        if (v < total) {
            int c = 0;
            while (off[c + 1] <= v) ++c;            // <= 64 columns
            const int a = begin[c] + (v - off[c]);
            x = rxyz[3 * a]; y = rxyz[3 * a + 1]; z = rxyz[3 * a + 2];
            t = rtype[a];
            in = !(x < lo[0] || x > hi[0] || y < lo[1] || y > hi[1] || z < lo[2] || z > hi[2]);
        }
        const unsigned bal = __ballot_sync(0xffffffffu, in);
        if (lane == 0) wsum[wid] = __popc(bal);
        __syncthreads();
        int o = n;
        for (int w = 0; w < wid; ++w) o += wsum[w];
        if (in) S[o + __popc(bal & ((1u << lane) - 1u))] = make_float4(x, y, z, __int_as_float(t));
        int tot = 0;
        for (int w = 0; w < TILE_THREADS / 32; ++w) tot += wsum[w];
        n += tot;
        __syncthreads();
    }
    *count = n;
    return v0 < total ? v0 : total;
}

// Distance-dependent parts of the Vina terms at surface distance d.
struct VinaTerms {
    float g1, g2, rep, hyd, hb;
};
template <typename PRM>
__device__ __forceinline__ VinaTerms vina_terms(float d, const PRM& P) {
    VinaTerms t;
    float u = (d - P.g1_off) * P.g1_inv;
    t.g1 = __expf(-u * u);
    u = (d - P.g2_off) * P.g2_inv;
    t.g2 = __expf(-u * u);
    const float dr = fminf(d - P.rep_off, 0.f);
    t.rep = dr * dr;
    t.hyd = fminf(fmaxf((P.hyd_bad - d) * P.hyd_inv, 0.f), 1.f);
    t.hb = fminf(fmaxf((P.hb_bad - d) * P.hb_inv, 0.f), 1.f);
    return t;
}

#define TILE_SETUP(cutoff)                                                                                          \
    const int tx = blockIdx.x, ty = blockIdx.y, tz = blockIdx.z;                                                    \
    const int tid = threadIdx.x;                                                                                    \
    const int k = tz * TILE_Z + (tid % TILE_Z);                                                                     \
    const int j = ty * TILE_Y + (tid / TILE_Z) % TILE_Y;                                                            \
    const int i = tx * TILE_X + tid / (TILE_Z * TILE_Y);                                                            \
    const bool valid = i < nx && j < ny && k < nz;                                                                  \
    const float x = ox + i * spacing, y = oy + j * spacing, z = oz + k * spacing;                                   \
    const int i1 = min(tx * TILE_X + TILE_X, nx), j1 = min(ty * TILE_Y + TILE_Y, ny), k1 = min(tz * TILE_Z + TILE_Z, nz); \
    const float cut2 = (cutoff) * (cutoff);                                                                         \
    const float lo[3] = {ox + tx * TILE_X * spacing - (cutoff), oy + ty * TILE_Y * spacing - (cutoff),               \
                         oz + tz * TILE_Z * spacing - (cutoff)};                                                    \
    const float hi[3] = {ox + (i1 - 1) * spacing + (cutoff), oy + (j1 - 1) * spacing + (cutoff),                     \
                         oz + (k1 - 1) * spacing + (cutoff)};                                                       \
    const long long npts = (long long)nx * ny * nz;                                                                 \
    const long long p = ((long long)i * ny + j) * nz + k;                                                           \
    __shared__ int col_begin[MAX_COLUMNS + 1], col_off[MAX_COLUMNS + 1];                                           \
    const int ncol = tile_columns(C, n_rec, lo, hi, col_begin, col_off);

__global__ void __launch_bounds__(TILE_THREADS) grid_vina_kernel(const float* __restrict__ rxyz,
                                                                 const int* __restrict__ rtype, int n_rec,
                                                                 const __grid_constant__ Cells C, float ox, float oy,
                                                                 float oz, float spacing, int nx, int ny, int nz,
                                                                 const __grid_constant__ VinaPrm P,
                                                                 float* __restrict__ out) {
    __shared__ float4 S[STAGE_CAP];
    __shared__ int wsum[TILE_THREADS / 32];
    TILE_SETUP(P.cutoff)

    for (int q0 = 0; q0 < P.n_lt; q0 += VINA_GROUP) {
        float acc[VINA_GROUP][5];
#pragma unroll
        for (int q = 0; q < VINA_GROUP; ++q)
#pragma unroll
            for (int m = 0; m < 5; ++m) acc[q][m] = 0.f;
        float rl[VINA_GROUP];
        int fl[VINA_GROUP];
#pragma unroll
        for (int q = 0; q < VINA_GROUP; ++q) {
            const int tl = (q0 + q < P.n_lt) ? P.lig_types[q0 + q] : 0;
            rl[q] = P.radius[tl];
            fl[q] = P.flags[tl];
        }
        int start = 0;
        const int total = col_off[ncol];
        while (start < total) {
            int cnt;
            start = stage_atoms<STAGE_CAP>(rxyz, rtype, col_begin, col_off, ncol, start, lo, hi, S, &cnt, wsum);
            if (valid) {
                for (int s = 0; s < cnt; ++s) {
                    const float4 A = S[s];
                    const float dx = A.x - x, dy = A.y - y, dz = A.z - z;
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 >= cut2) continue;
                    const float r = sqrtf(r2);
                    const int ta = __float_as_int(A.w);
                    const float ra = P.radius[ta];
                    const int fa = P.flags[ta];
                    VinaTerms t = vina_terms(r - ra - rl[0], P);
#pragma unroll
                    for (int q = 0; q < VINA_GROUP; ++q) {
                        if (q0 + q < P.n_lt) {
                            if (q > 0 && rl[q] != rl[q - 1]) t = vina_terms(r - ra - rl[q], P);   // next radius
                            acc[q][0] += t.g1; acc[q][1] += t.g2; acc[q][2] += t.rep;
                            if ((fa & 1) && (fl[q] & 1)) acc[q][3] += t.hyd;
                            if (((fa & 2) && (fl[q] & 4)) || ((fa & 4) && (fl[q] & 2))) acc[q][4] += t.hb;
                        }
                    }
                }
            }
            __syncthreads();
        }
        if (valid) {
#pragma unroll
            for (int q = 0; q < VINA_GROUP; ++q) {
                const int qq = q0 + q;
                if (qq >= P.n_lt) break;
                const int o = P.out_slot[qq];
                if (P.per_term) {
#pragma unroll
                    for (int m = 0; m < 5; ++m) out[((long long)(m * P.n_lt + o)) * npts + p] = acc[q][m];
                } else {
                    float e = 0.f;
#pragma unroll
                    for (int m = 0; m < 5; ++m) e += P.w[m] * acc[q][m];
                    out[(long long)o * npts + p] = e;
                }
            }
        }
    }
}

__global__ void __launch_bounds__(TILE_THREADS) grid_fit_kernel(const float* __restrict__ rxyz,
                                                                const int* __restrict__ rext, int n_rec,
                                                                const __grid_constant__ Cells C, float ox, float oy,
                                                                float oz, float spacing, int nx, int ny, int nz,
                                                                const __grid_constant__ FitPrm P,
                                                                const float* __restrict__ W, const float* __restrict__ rad_rec,
                                                                float* __restrict__ out) {
    __shared__ float4 S[FIT_STAGE_CAP];
    __shared__ int wsum[TILE_THREADS / 32];
    extern __shared__ float Wsh[];   // [n_rt, FIT_GROUP, 6] slice of W (radius-ordered types), then rad_rec [n_rt]
    float* Rsh = Wsh + (size_t)P.n_rt * FIT_GROUP * 6;
    TILE_SETUP(P.cutoff)
    const float rc = P.cutoff;
    for (int t = tid; t < P.n_rt; t += TILE_THREADS) Rsh[t] = rad_rec[t];

    for (int q0 = 0; q0 < P.n_lt; q0 += FIT_GROUP) {
        const int gq = min(FIT_GROUP, P.n_lt - q0);
        __syncthreads();
        for (int e = tid; e < P.n_rt * FIT_GROUP * 6; e += TILE_THREADS) {
            const int t = e / (FIT_GROUP * 6), q = (e / 6) % FIT_GROUP, b = e % 6;
            Wsh[e] = q < gq ? W[((long long)t * P.n_lt + P.out_slot[q0 + q]) * 6 + b] : 0.f;
        }
        __syncthreads();
        float acc[FIT_GROUP];
        float rl[FIT_GROUP];
#pragma unroll
        for (int q = 0; q < FIT_GROUP; ++q) {
            acc[q] = 0.f;
            rl[q] = q < gq ? P.rad_lig[q0 + q] : 0.f;
        }
        int start = 0;
        const int total = col_off[ncol];
        while (start < total) {
            int cnt;
            start = stage_atoms<FIT_STAGE_CAP>(rxyz, rext, col_begin, col_off, ncol, start, lo, hi, S, &cnt, wsum);
            if (valid) {
                for (int s = 0; s < cnt; ++s) {
                    const float4 A = S[s];
                    const float dx = A.x - x, dy = A.y - y, dz = A.z - z;
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 >= cut2) continue;
                    const float r = sqrtf(r2);
                    const int ta = __float_as_int(A.w);
                    const float ra = Rsh[ta];
                    const float rr = fmaxf(r, P.ion_rmin);
                    const float ion = 1.f / (rr * rr) - 1.f / (rc * rc);
                    const float* Wa = Wsh + (size_t)ta * FIT_GROUP * 6;
                    VinaTerms t = vina_terms(r - ra - rl[0], P);
                    float rep = fminf(t.rep, P.rep_cap);
#pragma unroll
                    for (int q = 0; q < FIT_GROUP; ++q) {
                        if (q < gq) {
                            if (q > 0 && rl[q] != rl[q - 1]) {                                    // next radius
                                t = vina_terms(r - ra - rl[q], P);
                                rep = fminf(t.rep, P.rep_cap);
                            }
                            const float* w = Wa + q * 6;
                            float s_ = w[0] * t.g1;
                            s_ += w[1] * t.g2;
                            s_ += w[2] * rep;
                            s_ += w[3] * t.hyd;
                            s_ += w[4] * t.hb;
                            s_ += w[5] * ion;
                            acc[q] += s_;
                        }
                    }
                }
            }
            __syncthreads();
        }
        if (valid) {
#pragma unroll
            for (int q = 0; q < FIT_GROUP; ++q)
                if (q < gq) out[(long long)P.out_slot[q0 + q] * npts + p] = acc[q];
        }
    }
}

template <typename T>
__global__ void convert_kernel(const float* __restrict__ src, T* __restrict__ dst, long long n);
// FP16 saturates at +-65504 (map values inside receptor atoms can exceed the FP16 range; a clamped value keeps
// such points repulsive instead of turning the interpolation into inf/NaN)
template <>
__global__ void convert_kernel<__half>(const float* __restrict__ src, __half* __restrict__ dst, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = __float2half_rn(fminf(fmaxf(src[i], -65504.f), 65504.f));
}
template <>
__global__ void convert_kernel<__nv_bfloat16>(const float* __restrict__ src, __nv_bfloat16* __restrict__ dst, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = __float2bfloat16_rn(src[i]);
}

// Order of a launch's ligand types by radius (stable): positions order[0..n) into the caller's type list.
static void order_by_radius(const float* rad, int n, int* order) {
    for (int q = 0; q < n; ++q) order[q] = q;
    for (int a = 1; a < n; ++a) {   // insertion sort, n <= 64
        const int v = order[a];
        int b = a - 1;
        while (b >= 0 && rad[order[b]] > rad[v]) {
            order[b + 1] = order[b];
            --b;
        }
        order[b + 1] = v;
    }
}

static int check_cells(const Cells& C, int n_rec, float cutoff, float spacing) {
    if (!C.start) return ADOCK_OK;
    ADOCK_CHECK_ARG(C.nx >= 1 && C.ny >= 1 && C.nz >= 1 && C.size > 0.f, "bad cell grid");
    // columns a tile's grown box can touch: ceil(extent / size) + 1 per axis, at most 8 x 8
    const float ext = fmaxf(TILE_X, TILE_Y) * spacing + 2.f * cutoff;
    const int per = (int)ceilf(ext / C.size) + 1;
    ADOCK_CHECK_ARG(per * per <= MAX_COLUMNS, "cell size %.3f too small for the cutoff (at most %d columns per tile)",
                    C.size, MAX_COLUMNS);
    (void)n_rec;
    return ADOCK_OK;
}

static int grid_vina_launch(const float* rec_xyz, const int* rec_types, int n_rec, const Cells& C, const float* radius,
                            const int* hyd, const int* don, const int* acc, int n_xs, const int* lig_types, int n_lt,
                            float ox, float oy, float oz, float spacing, int nx, int ny, int nz, const float* prm,
                            int per_term, float* out, void* stream) {
    ADOCK_CHECK_ARG(n_rec >= 0 && (n_rec == 0 || (rec_xyz && rec_types)), "bad receptor arrays");
    ADOCK_CHECK_ARG(radius && hyd && don && acc && lig_types && prm && out, "null argument");
    ADOCK_CHECK_ARG(n_xs >= 1 && n_xs <= 64, "n_xs must be in [1, 64] (got %d)", n_xs);
    ADOCK_CHECK_ARG(n_lt >= 1 && n_lt <= 24, "n_lt must be in [1, 24] (got %d)", n_lt);
    ADOCK_CHECK_ARG(nx >= 1 && ny >= 1 && nz >= 1, "grid dimensions must be >= 1");
    ADOCK_CHECK_ARG(spacing > 0.f, "spacing must be > 0");
    int rc = check_cells(C, n_rec, prm[0], spacing);
    if (rc) return rc;
    VinaPrm P;
    P.cutoff = prm[0];
    P.g1_off = prm[1]; P.g1_inv = 1.f / prm[2]; P.g2_off = prm[3]; P.g2_inv = 1.f / prm[4]; P.rep_off = prm[5];
    P.hyd_good = prm[6]; P.hyd_bad = prm[7]; P.hyd_inv = 1.f / (prm[7] - prm[6]);
    P.hb_good = prm[8]; P.hb_bad = prm[9]; P.hb_inv = 1.f / (prm[9] - prm[8]);
    for (int m = 0; m < 5; ++m) P.w[m] = prm[10 + m];
    P.n_lt = n_lt; P.n_xs = n_xs; P.per_term = per_term ? 1 : 0;
    for (int q = 0; q < n_lt; ++q) ADOCK_CHECK_ARG(lig_types[q] >= 0 && lig_types[q] < n_xs, "ligand type out of range");
    float rl[24];
    int order[24];
    for (int q = 0; q < n_lt; ++q) rl[q] = radius[lig_types[q]];
    order_by_radius(rl, n_lt, order);
    for (int q = 0; q < 24; ++q) {
        P.lig_types[q] = q < n_lt ? lig_types[order[q]] : 0;
        P.out_slot[q] = q < n_lt ? order[q] : 0;
    }
    for (int t = 0; t < 64; ++t) {
        P.radius[t] = t < n_xs ? radius[t] : 0.f;
        P.flags[t] = t < n_xs ? ((hyd[t] ? 1 : 0) | (don[t] ? 2 : 0) | (acc[t] ? 4 : 0)) : 0;
    }
    dim3 grid((nx + TILE_X - 1) / TILE_X, (ny + TILE_Y - 1) / TILE_Y, (nz + TILE_Z - 1) / TILE_Z);
    ADOCK_CHECK_ARG(grid.y < 65536 && grid.z < 65536, "grid too large");
    grid_vina_kernel<<<grid, TILE_THREADS, 0, (cudaStream_t)stream>>>(rec_xyz, rec_types, n_rec, C, ox, oy, oz, spacing,
                                                                       nx, ny, nz, P, out);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

static int grid_fit_launch(const float* rec_xyz, const int* rec_ext, int n_rec, const Cells& C, const float* rad_rec,
                           int n_rt, const float* rad_lig, int n_lt, const float* W, float ox, float oy, float oz,
                           float spacing, int nx, int ny, int nz, const float* prm, float* out, void* stream) {
    ADOCK_CHECK_ARG(n_rec >= 0 && (n_rec == 0 || (rec_xyz && rec_ext)), "bad receptor arrays");
    ADOCK_CHECK_ARG(rad_rec && rad_lig && W && prm && out, "null argument");
    ADOCK_CHECK_ARG(n_lt >= 1 && n_lt <= 64, "n_lt must be in [1, 64] (got %d)", n_lt);
    ADOCK_CHECK_ARG(n_rt >= 1 && n_rt <= 1024, "n_rt must be in [1, 1024] (got %d)", n_rt);
    ADOCK_CHECK_ARG(nx >= 1 && ny >= 1 && nz >= 1, "grid dimensions must be >= 1");
    ADOCK_CHECK_ARG(spacing > 0.f, "spacing must be > 0");
    int rc = check_cells(C, n_rec, prm[0], spacing);
    if (rc) return rc;
    FitPrm P;
    P.cutoff = prm[0];
    P.g1_off = prm[1]; P.g1_inv = 1.f / prm[2]; P.g2_off = prm[3]; P.g2_inv = 1.f / prm[4]; P.rep_off = prm[5];
    P.hyd_good = prm[6]; P.hyd_bad = prm[7]; P.hyd_inv = 1.f / (prm[7] - prm[6]);
    P.hb_good = prm[8]; P.hb_bad = prm[9]; P.hb_inv = 1.f / (prm[9] - prm[8]);
    P.ion_rmin = prm[10]; P.rep_cap = prm[11];
    P.n_lt = n_lt; P.n_rt = n_rt;
    int order[64];
    order_by_radius(rad_lig, n_lt, order);
    for (int q = 0; q < 64; ++q) {
        P.rad_lig[q] = q < n_lt ? rad_lig[order[q]] : 0.f;
        P.out_slot[q] = q < n_lt ? order[q] : 0;
    }
    const size_t smem = ((size_t)n_rt * FIT_GROUP * 6 + n_rt) * sizeof(float);
    ADOCK_CUDA(cudaFuncSetAttribute(grid_fit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((nx + TILE_X - 1) / TILE_X, (ny + TILE_Y - 1) / TILE_Y, (nz + TILE_Z - 1) / TILE_Z);
    ADOCK_CHECK_ARG(grid.y < 65536 && grid.z < 65536, "grid too large");
    grid_fit_kernel<<<grid, TILE_THREADS, smem, (cudaStream_t)stream>>>(rec_xyz, rec_ext, n_rec, C, ox, oy, oz, spacing,
                                                                          nx, ny, nz, P, W, rad_rec, out);
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}

static Cells whole_receptor() {
    Cells C{};
    C.start = nullptr;
    return C;
}

static Cells make_cells(const int* cell_start, const int* cell_dims, const float* cell_origin, float cell_size) {
    Cells C;
    C.start = cell_start;
    C.nx = cell_dims[0]; C.ny = cell_dims[1]; C.nz = cell_dims[2];
    C.ox = cell_origin[0]; C.oy = cell_origin[1]; C.oz = cell_origin[2];
    C.size = cell_size;
    return C;
}

}  // namespace adock

using namespace adock;

extern "C" int adock_grid_vina(const float* rec_xyz, const int* rec_types, int n_rec, const float* radius,
                               const int* hyd, const int* don, const int* acc, int n_xs, const int* lig_types,
                               int n_lt, float ox, float oy, float oz, float spacing, int nx, int ny, int nz,
                               const float* prm, int per_term, float* out, void* stream) {
    return grid_vina_launch(rec_xyz, rec_types, n_rec, whole_receptor(), radius, hyd, don, acc, n_xs, lig_types, n_lt,
                            ox, oy, oz, spacing, nx, ny, nz, prm, per_term, out, stream);
}

extern "C" int adock_grid_vina_cells(const float* rec_xyz, const int* rec_types, int n_rec, const int* cell_start,
                                     const int* cell_dims, const float* cell_origin, float cell_size,
                                     const float* radius, const int* hyd, const int* don, const int* acc, int n_xs,
                                     const int* lig_types, int n_lt, float ox, float oy, float oz, float spacing,
                                     int nx, int ny, int nz, const float* prm, int per_term, float* out, void* stream) {
    ADOCK_CHECK_ARG(cell_start && cell_dims && cell_origin, "null cell-list argument");
    return grid_vina_launch(rec_xyz, rec_types, n_rec, make_cells(cell_start, cell_dims, cell_origin, cell_size),
                            radius, hyd, don, acc, n_xs, lig_types, n_lt, ox, oy, oz, spacing, nx, ny, nz, prm,
                            per_term, out, stream);
}

extern "C" int adock_grid_fit(const float* rec_xyz, const int* rec_ext, int n_rec, const float* rad_rec, int n_rt,
                              const float* rad_lig, int n_lt, const float* W, float ox, float oy, float oz,
                              float spacing, int nx, int ny, int nz, const float* prm, float* out, void* stream) {
    return grid_fit_launch(rec_xyz, rec_ext, n_rec, whole_receptor(), rad_rec, n_rt, rad_lig, n_lt, W, ox, oy, oz,
                           spacing, nx, ny, nz, prm, out, stream);
}

extern "C" int adock_grid_fit_cells(const float* rec_xyz, const int* rec_ext, int n_rec, const int* cell_start,
                                    const int* cell_dims, const float* cell_origin, float cell_size,
                                    const float* rad_rec, int n_rt, const float* rad_lig, int n_lt, const float* W,
                                    float ox, float oy, float oz, float spacing, int nx, int ny, int nz,
                                    const float* prm, float* out, void* stream) {
    ADOCK_CHECK_ARG(cell_start && cell_dims && cell_origin, "null cell-list argument");
    return grid_fit_launch(rec_xyz, rec_ext, n_rec, make_cells(cell_start, cell_dims, cell_origin, cell_size), rad_rec,
                           n_rt, rad_lig, n_lt, W, ox, oy, oz, spacing, nx, ny, nz, prm, out, stream);
}

extern "C" int adock_grid_convert(const float* src, void* dst, long long n, int dtype, void* stream) {
    ADOCK_CHECK_ARG(src && dst && n >= 0, "bad argument");
    if (n == 0) return ADOCK_OK;
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 32);
    if (dtype == ADOCK_GRID_F16)
        convert_kernel<__half><<<blocks, 256, 0, (cudaStream_t)stream>>>(src, (__half*)dst, n);
    else if (dtype == ADOCK_GRID_BF16)
        convert_kernel<__nv_bfloat16><<<blocks, 256, 0, (cudaStream_t)stream>>>(src, (__nv_bfloat16*)dst, n);
    else
        ADOCK_CHECK_ARG(false, "dtype must be ADOCK_GRID_F16 or ADOCK_GRID_BF16");
    ADOCK_CUDA(cudaGetLastError());
    return ADOCK_OK;
}
