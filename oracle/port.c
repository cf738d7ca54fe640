/*
 * CPU restatement of the reference's docking hot path, in plain C (C11 + OpenMP).
 *
 * TEST INFRASTRUCTURE ONLY (the oracle): built into oracle/liboracle_port.so and called by tests/, smoke()
 * and bench.py's CPU-baseline leg as the checker. The product (adock_b200) never links or calls it.
 *
 * Each function restates one piece of the reference, cited by file:line (paths inside the reference project):
 *   port_grid_vina   src/adock/grid.py:14-71            Vina/Vinardo maps (5 unweighted sums per type, weighted last)
 *   port_grid_fit    src/adock/fit/gridfit.py:13-58     fitted-function maps (6 basis functions x W table)
 *   eval_eg          src/adock/mckernel.py:108-244      pose energy + analytic gradient (grid or exact)
 *   bfgs             src/adock/mckernel.py:246-326      Vina-1.2 BFGS with Armijo backtracking
 *   port_mc          src/adock/mckernel.py:328-408      Monte-Carlo chains (mutation, BFGS, Metropolis)
 *   port_eg          src/adock/mckernel.py:411-447      batched energy + gradient
 *   port_stage_a     src/adock/mckernel.py:451-521      rigid enumeration (nearest grid point, capped)
 *   urand/rand_ball  src/adock/mckernel.py:71-90        counter-based SplitMix64 uniform numbers
 * Array layouts are those of pack_host (src/adock/mckernel.py:547-599). One chain = one sequential loop
 * (the reference's warp lanes collapse to a single thread); OpenMP runs chains / grid points in parallel.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define EPSF 1.1920929e-07f

typedef struct {
    const float* ref; const int* typ; const unsigned char* tm; const int* ax; const float* axp; const float* axu;
    const int* pr; const int* na; const int* nt; const int* np; const float* rg; const int* gslot; const int* rec_idx;
    int L, AM, KM, P;
} port_lig;

typedef struct {
    const float* flat; const long long* offs; const long long* dims; const float* origin; const float* lo;
    const float* hi; float spacing, penalty;
} port_grid;

typedef struct {
    float prm[15];  /* mckernel.py:594-596 order */
    const float* radius; const int* hyd; const int* don; const int* acc;
} port_sf;

typedef struct { const float* xyz; const int* typ; const int* n; int RN; } port_rec;

void port_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#endif
}

/* ------------------------------------------------------------------------------------------ grids */
void port_grid_vina(const float* rxyz, const int* rtype, int n_rec, const float* radius, const int* hyd,
                    const int* don, const int* acc, const int* lig_types, int n_lt, float ox, float oy, float oz,
                    float spacing, int nx, int ny, int nz, const float* prm, int per_term, float* out) {
    const long long npts = (long long)nx * ny * nz;
    const float cut2 = prm[0] * prm[0];
    #pragma omp parallel for schedule(dynamic, 64)
    for (long long p = 0; p < npts; ++p) {
        const int k = (int)(p % nz), j = (int)((p / nz) % ny), i = (int)(p / ((long long)ny * nz));
        const float x = ox + i * spacing, y = oy + j * spacing, z = oz + k * spacing;
        float acc_e[5 * 64];
        for (int q = 0; q < 5 * n_lt; ++q) acc_e[q] = 0.f;
        for (int a = 0; a < n_rec; ++a) {
            const float dx = rxyz[3 * a] - x, dy = rxyz[3 * a + 1] - y, dz = rxyz[3 * a + 2] - z;
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 >= cut2) continue;
            const float r = sqrtf(r2);
            const int ta = rtype[a];
            for (int q = 0; q < n_lt; ++q) {
                const int tl = lig_types[q];
                const float d = r - radius[ta] - radius[tl];
                float u = (d - prm[1]) / prm[2];
                const float g1 = expf(-u * u);
                u = (d - prm[3]) / prm[4];
                const float g2 = expf(-u * u);
                const float dr = d - prm[5];
                const float rep = dr < 0.f ? dr * dr : 0.f;
                float hy = 0.f, hb = 0.f;
                if (hyd[ta] && hyd[tl]) hy = fminf(fmaxf((prm[7] - d) / (prm[7] - prm[6]), 0.f), 1.f);
                if ((don[ta] && acc[tl]) || (acc[ta] && don[tl])) hb = fminf(fmaxf((prm[9] - d) / (prm[9] - prm[8]), 0.f), 1.f);
                acc_e[5 * q] += g1; acc_e[5 * q + 1] += g2; acc_e[5 * q + 2] += rep; acc_e[5 * q + 3] += hy;
                acc_e[5 * q + 4] += hb;
            }
        }
        for (int q = 0; q < n_lt; ++q) {
            if (per_term) {
                for (int m = 0; m < 5; ++m) out[(long long)(m * n_lt + q) * npts + p] = acc_e[5 * q + m];
            } else {
                float e = 0.f;
                for (int m = 0; m < 5; ++m) e += prm[10 + m] * acc_e[5 * q + m];
                out[(long long)q * npts + p] = e;
            }
        }
    }
}

void port_grid_fit(const float* rxyz, const int* rext, int n_rec, const float* rad_rec, const float* rad_lig, int n_lt,
                   const float* W, float ox, float oy, float oz, float spacing, int nx, int ny, int nz,
                   const float* prm, float* out) {
    const long long npts = (long long)nx * ny * nz;
    const float rc = prm[0], cut2 = rc * rc;
    #pragma omp parallel for schedule(dynamic, 64)
    for (long long p = 0; p < npts; ++p) {
        const int k = (int)(p % nz), j = (int)((p / nz) % ny), i = (int)(p / ((long long)ny * nz));
        const float x = ox + i * spacing, y = oy + j * spacing, z = oz + k * spacing;
        float e[64];
        for (int q = 0; q < n_lt; ++q) e[q] = 0.f;
        for (int a = 0; a < n_rec; ++a) {
            const float dx = rxyz[3 * a] - x, dy = rxyz[3 * a + 1] - y, dz = rxyz[3 * a + 2] - z;
            const float r2 = dx * dx + dy * dy + dz * dz;
            if (r2 >= cut2) continue;
            const float r = sqrtf(r2);
            const int ta = rext[a];
            const float rr = fmaxf(r, prm[10]);
            const float ion = 1.f / (rr * rr) - 1.f / cut2;
            for (int q = 0; q < n_lt; ++q) {
                const float* w = W + ((long long)ta * n_lt + q) * 6;
                const float d = r - rad_rec[ta] - rad_lig[q];
                float u = (d - prm[1]) / prm[2];
                float s = w[0] * expf(-u * u);
                u = (d - prm[3]) / prm[4];
                s += w[1] * expf(-u * u);
                const float dr = d - prm[5];
                if (dr < 0.f) s += w[2] * fminf(dr * dr, prm[11]);
                s += w[3] * fminf(fmaxf((prm[7] - d) / (prm[7] - prm[6]), 0.f), 1.f);
                s += w[4] * fminf(fmaxf((prm[9] - d) / (prm[9] - prm[8]), 0.f), 1.f);
                s += w[5] * ion;
                e[q] += s;
            }
        }
        for (int q = 0; q < n_lt; ++q) out[(long long)q * npts + p] = e[q];
    }
}

/* ------------------------------------------------------------------------------------------ search */
static float pair_e(float r, int ti, int tj, const port_sf* sf, float* de) {
    const float* prm = sf->prm;
    const float d = r - sf->radius[ti] - sf->radius[tj];
    const float u1 = (d - prm[0]) / prm[1], g1 = expf(-u1 * u1);
    const float u2 = (d - prm[2]) / prm[3], g2 = expf(-u2 * u2);
    float e = prm[10] * g1 + prm[11] * g2;
    float g = prm[10] * (-2.f * u1 / prm[1]) * g1 + prm[11] * (-2.f * u2 / prm[3]) * g2;
    const float dr = d - prm[4];
    if (dr < 0.f) { e += prm[12] * dr * dr; g += prm[12] * 2.f * dr; }
    if (sf->hyd[ti] && sf->hyd[tj]) {
        const float v = (prm[6] - d) / (prm[6] - prm[5]);
        if (v >= 1.f) e += prm[13];
        else if (v > 0.f) { e += prm[13] * v; g += prm[13] * (-1.f / (prm[6] - prm[5])); }
    }
    if ((sf->don[ti] && sf->acc[tj]) || (sf->acc[ti] && sf->don[tj])) {
        const float v = (prm[8] - d) / (prm[8] - prm[7]);
        if (v >= 1.f) e += prm[14];
        else if (v > 0.f) { e += prm[14] * v; g += prm[14] * (-1.f / (prm[8] - prm[7])); }
    }
    *de = g;
    return e;
}

static uint64_t smix(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
static float urand(uint64_t seed, int chain, int step, int slot) {
    const uint64_t h = smix(seed ^ smix(((uint64_t)chain << 32) ^ ((uint64_t)step << 8) ^ (uint64_t)slot));
    return (float)(h >> 40) * (1.0f / 16777216.0f);
}
static void rand_ball(uint64_t seed, int chain, int step, int slot, float* v) {
    for (int k = 0; k < 32; ++k) {
        const float a = 2.f * urand(seed, chain, step, slot + 3 * k) - 1.f;
        const float b = 2.f * urand(seed, chain, step, slot + 3 * k + 1) - 1.f;
        const float c = 2.f * urand(seed, chain, step, slot + 3 * k + 2) - 1.f;
        if (a * a + b * b + c * c < 1.f) { v[0] = a; v[1] = b; v[2] = c; return; }
    }
    v[0] = v[1] = v[2] = 0.f;
}
static void quat_inc(float* q, float rx, float ry, float rz) {
    const float ang = sqrtf(rx * rx + ry * ry + rz * rz);
    float hw, k;
    if (ang > 1e-6f) { hw = cosf(0.5f * ang); k = sinf(0.5f * ang) / ang; } else { hw = 1.f; k = 0.5f; }
    const float aw = hw, ax = rx * k, ay = ry * k, az = rz * k;
    const float bw = q[0], bx = q[1], by = q[2], bz = q[3];
    const float w = aw * bw - ax * bx - ay * by - az * bz, x = aw * bx + ax * bw + ay * bz - az * by;
    const float y = aw * by - ax * bz + ay * bw + az * bx, z = aw * bz + ax * by - ay * bx + az * bw;
    const float nn = 1.f / sqrtf(w * w + x * x + y * y + z * z);
    q[0] = w * nn; q[1] = x * nn; q[2] = y * nn; q[3] = z * nn;
}

/* per-chain context and scratch */
typedef struct {
    const float* ref; const int* typ; const unsigned char* tm; const int* ax; const float* axp; const float* axu;
    const int* pr; const int* gslot; int na, nt, np, AM; float rg;
    const float* grid; float o[3], lo[3], hi[3]; int nx, ny, nz; float inv_s, pen;
    const float* rx; const int* rt; int rn, exact; const int* nb; int nbn;
} ctx_t;

typedef struct {
    float *X, *F, *H, *x, *xn, *xo, *cur, *best, *g, *gn, *go, *p, *y, *mhy, *pw, *uw;
} ws_t;

static void ws_alloc(ws_t* w, int AM, int KM) {
    const int DM = 6 + KM, SD = 7 + KM;
    float* b = (float*)calloc((size_t)(6 * AM + DM * DM + 5 * SD + 6 * DM + 6 * KM), sizeof(float));
    w->X = b; b += 3 * AM; w->F = b; b += 3 * AM; w->H = b; b += DM * DM;
    w->x = b; b += SD; w->xn = b; b += SD; w->xo = b; b += SD; w->cur = b; b += SD; w->best = b; b += SD;
    w->g = b; b += DM; w->gn = b; b += DM; w->go = b; b += DM; w->p = b; b += DM; w->y = b; b += DM; w->mhy = b; b += DM;
    w->pw = b; b += 3 * KM; w->uw = b;
}
static void ws_free(ws_t* w) { free(w->X); }

static void ctx_init(ctx_t* c, const port_lig* L, const port_grid* G, const port_rec* R, int l, int exact,
                     const int* nb, int nbn) {
    const int AM = L->AM, KM = L->KM;
    c->ref = L->ref + (long long)l * AM * 3; c->typ = L->typ + (long long)l * AM; c->tm = L->tm + (long long)l * KM * AM;
    c->ax = L->ax + (long long)l * KM * 2; c->axp = L->axp + (long long)l * KM * 3; c->axu = L->axu + (long long)l * KM * 3;
    c->pr = L->pr + (long long)l * L->P * 2; c->gslot = L->gslot + (long long)l * AM;
    c->na = L->na[l]; c->nt = L->nt[l]; c->np = L->np[l]; c->rg = L->rg[l]; c->AM = AM;
    const int ri = L->rec_idx[l];
    c->grid = G->flat + G->offs[ri];
    c->nx = (int)G->dims[3 * ri]; c->ny = (int)G->dims[3 * ri + 1]; c->nz = (int)G->dims[3 * ri + 2];
    for (int d = 0; d < 3; ++d) { c->o[d] = G->origin[3 * ri + d]; c->lo[d] = G->lo[3 * ri + d]; c->hi[d] = G->hi[3 * ri + d]; }
    c->inv_s = 1.f / G->spacing; c->pen = G->penalty;
    c->rx = R && R->xyz ? R->xyz + (long long)ri * R->RN * 3 : NULL;
    c->rt = R && R->typ ? R->typ + (long long)ri * R->RN : NULL;
    c->rn = R && R->n ? R->n[ri] : 0;
    c->exact = exact; c->nb = nb; c->nbn = nbn;
}

static float eval_eg(ws_t* w, const float* s, float* g, const ctx_t* c, const port_sf* sf) {
    float qw = s[3], qx = s[4], qy = s[5], qz = s[6];
    const float nq = 1.f / sqrtf(qw * qw + qx * qx + qy * qy + qz * qz);
    qw *= nq; qx *= nq; qy *= nq; qz *= nq;
    const float R00 = 1 - 2 * (qy * qy + qz * qz), R01 = 2 * (qx * qy - qz * qw), R02 = 2 * (qx * qz + qy * qw);
    const float R10 = 2 * (qx * qy + qz * qw), R11 = 1 - 2 * (qx * qx + qz * qz), R12 = 2 * (qy * qz - qx * qw);
    const float R20 = 2 * (qx * qz - qy * qw), R21 = 2 * (qy * qz + qx * qw), R22 = 1 - 2 * (qx * qx + qy * qy);
    const long long n3 = (long long)c->nx * c->ny * c->nz;
    const float fmx[3] = {(float)(c->nx - 1) - 1e-4f, (float)(c->ny - 1) - 1e-4f, (float)(c->nz - 1) - 1e-4f};
    const float* prm = sf->prm;
    float e = 0.f;
    for (int a = 0; a < c->na; ++a) {
        float px = c->ref[3 * a], py = c->ref[3 * a + 1], pz = c->ref[3 * a + 2];
        for (int k = 0; k < c->nt; ++k) {
            if (!c->tm[k * c->AM + a]) continue;
            const float th = s[7 + k], cs = cosf(th), sn = sinf(th);
            const float ux = c->axu[3 * k], uy = c->axu[3 * k + 1], uz = c->axu[3 * k + 2];
            const float vx = px - c->axp[3 * k], vy = py - c->axp[3 * k + 1], vz = pz - c->axp[3 * k + 2];
            const float d = ux * vx + uy * vy + uz * vz;
            const float cx = uy * vz - uz * vy, cy = uz * vx - ux * vz, cz = ux * vy - uy * vx;
            px = c->axp[3 * k] + vx * cs + cx * sn + ux * d * (1 - cs);
            py = c->axp[3 * k + 1] + vy * cs + cy * sn + uy * d * (1 - cs);
            pz = c->axp[3 * k + 2] + vz * cs + cz * sn + uz * d * (1 - cs);
        }
        const float X[3] = {R00 * px + R01 * py + R02 * pz + s[0], R10 * px + R11 * py + R12 * pz + s[1],
                            R20 * px + R21 * py + R22 * pz + s[2]};
        w->X[3 * a] = X[0]; w->X[3 * a + 1] = X[1]; w->X[3 * a + 2] = X[2];
        float ea = 0.f, gg[3] = {0.f, 0.f, 0.f};
        if (c->exact) {
            const int ta = c->typ[a];
            const float cut2 = prm[9] * prm[9];
            const int nloop = c->nb ? c->nbn : c->rn;
            for (int bb = 0; bb < nloop; ++bb) {
                const int b = c->nb ? c->nb[bb] : bb;
                const float rx = X[0] - c->rx[3 * b], ry = X[1] - c->rx[3 * b + 1], rz = X[2] - c->rx[3 * b + 2];
                const float r2 = rx * rx + ry * ry + rz * rz;
                if (r2 >= cut2) continue;
                const float r = sqrtf(r2);
                float de;
                ea += pair_e(r, ta, c->rt[b], sf, &de);
                const float sc = de / fmaxf(r, 1e-6f);
                gg[0] += sc * rx; gg[1] += sc * ry; gg[2] += sc * rz;
            }
        } else {
            float fw[3], inside[3];
            int i0[3];
            for (int d = 0; d < 3; ++d) {
                const float f = (X[d] - c->o[d]) * c->inv_s;
                const float fc = fminf(fmaxf(f, 0.f), fmx[d]);
                inside[d] = (f > 0.f && f < fmx[d]) ? 1.f : 0.f;
                i0[d] = (int)floorf(fc);
                fw[d] = fc - i0[d];
            }
            const float* Gp = c->grid + (long long)c->gslot[a] * n3;
            const long long b000 = ((long long)i0[0] * c->ny + i0[1]) * c->nz + i0[2], bx = b000 + (long long)c->ny * c->nz;
            const float v000 = Gp[b000], v001 = Gp[b000 + 1], v010 = Gp[b000 + c->nz], v011 = Gp[b000 + c->nz + 1];
            const float v100 = Gp[bx], v101 = Gp[bx + 1], v110 = Gp[bx + c->nz], v111 = Gp[bx + c->nz + 1];
            const float wx = fw[0], wy = fw[1], wz = fw[2];
            const float c00 = v000 * (1 - wz) + v001 * wz, c01 = v010 * (1 - wz) + v011 * wz;
            const float c10 = v100 * (1 - wz) + v101 * wz, c11 = v110 * (1 - wz) + v111 * wz;
            const float c0 = c00 * (1 - wy) + c01 * wy, c1 = c10 * (1 - wy) + c11 * wy;
            ea = c0 * (1 - wx) + c1 * wx;
            gg[0] = (c1 - c0) * c->inv_s * inside[0];
            gg[1] = ((c01 - c00) * (1 - wx) + (c11 - c10) * wx) * c->inv_s * inside[1];
            gg[2] = (((v001 - v000) * (1 - wy) + (v011 - v010) * wy) * (1 - wx) +
                     ((v101 - v100) * (1 - wy) + (v111 - v110) * wy) * wx) * c->inv_s * inside[2];
        }
        for (int d = 0; d < 3; ++d) {
            const float lo = fmaxf(c->lo[d] - X[d], 0.f), hi = fmaxf(X[d] - c->hi[d], 0.f);
            ea += c->pen * (lo * lo + hi * hi);
            gg[d] += c->pen * (-2.f * lo + 2.f * hi);
        }
        e += ea;
        w->F[3 * a] = gg[0]; w->F[3 * a + 1] = gg[1]; w->F[3 * a + 2] = gg[2];
    }
    for (int q = 0; q < c->np; ++q) {
        const int i = c->pr[2 * q], j = c->pr[2 * q + 1];
        const float rx = w->X[3 * i] - w->X[3 * j], ry = w->X[3 * i + 1] - w->X[3 * j + 1], rz = w->X[3 * i + 2] - w->X[3 * j + 2];
        const float r = sqrtf(rx * rx + ry * ry + rz * rz);
        if (r >= prm[9]) continue;
        float de;
        e += pair_e(r, c->typ[i], c->typ[j], sf, &de);
        const float sc = de / fmaxf(r, 1e-6f);
        w->F[3 * i] += sc * rx; w->F[3 * i + 1] += sc * ry; w->F[3 * i + 2] += sc * rz;
        w->F[3 * j] -= sc * rx; w->F[3 * j + 1] -= sc * ry; w->F[3 * j + 2] -= sc * rz;
    }
    for (int k = 0; k < c->nt; ++k) {
        const int a = c->ax[2 * k], b = c->ax[2 * k + 1];
        const float ux = w->X[3 * b] - w->X[3 * a], uy = w->X[3 * b + 1] - w->X[3 * a + 1], uz = w->X[3 * b + 2] - w->X[3 * a + 2];
        const float nn = 1.f / sqrtf(fmaxf(ux * ux + uy * uy + uz * uz, 1e-12f));
        w->uw[3 * k] = ux * nn; w->uw[3 * k + 1] = uy * nn; w->uw[3 * k + 2] = uz * nn;
        w->pw[3 * k] = w->X[3 * a]; w->pw[3 * k + 1] = w->X[3 * a + 1]; w->pw[3 * k + 2] = w->X[3 * a + 2];
        g[6 + k] = 0.f;
    }
    float gt[3] = {0, 0, 0}, tq[3] = {0, 0, 0};
    for (int a = 0; a < c->na; ++a) {
        const float fx = w->F[3 * a], fy = w->F[3 * a + 1], fz = w->F[3 * a + 2];
        const float X0 = w->X[3 * a], X1 = w->X[3 * a + 1], X2 = w->X[3 * a + 2];
        gt[0] += fx; gt[1] += fy; gt[2] += fz;
        const float dx = X0 - s[0], dy = X1 - s[1], dz = X2 - s[2];
        tq[0] += dy * fz - dz * fy; tq[1] += dz * fx - dx * fz; tq[2] += dx * fy - dy * fx;
        for (int k = 0; k < c->nt; ++k) {
            if (!c->tm[k * c->AM + a]) continue;
            const float vx = X0 - w->pw[3 * k], vy = X1 - w->pw[3 * k + 1], vz = X2 - w->pw[3 * k + 2];
            const float cx = vy * fz - vz * fy, cy = vz * fx - vx * fz, cz = vx * fy - vy * fx;
            g[6 + k] += cx * w->uw[3 * k] + cy * w->uw[3 * k + 1] + cz * w->uw[3 * k + 2];
        }
    }
    g[0] = gt[0]; g[1] = gt[1]; g[2] = gt[2]; g[3] = tq[0]; g[4] = tq[1]; g[5] = tq[2];
    return e;
}

static float dot(const float* a, const float* b, int n) {
    float s = 0.f;
    for (int i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}
static void conf_inc(float* xn, const float* x, const float* p, float alpha, int nt) {
    xn[0] = x[0] + alpha * p[0]; xn[1] = x[1] + alpha * p[1]; xn[2] = x[2] + alpha * p[2];
    xn[3] = x[3]; xn[4] = x[4]; xn[5] = x[5]; xn[6] = x[6];
    quat_inc(xn + 3, alpha * p[3], alpha * p[4], alpha * p[5]);
    for (int k = 0; k < nt; ++k) xn[7 + k] = x[7 + k] + alpha * p[6 + k];
}

static float bfgs(ws_t* w, float* x, int iters, const ctx_t* c, const port_sf* sf, long long* n_eval) {
    const int D = 6 + c->nt, S = 7 + c->nt;
    float f0 = eval_eg(w, x, w->g, c, sf);
    ++*n_eval;
    const float f_orig = f0;
    memcpy(w->xo, x, S * sizeof(float));
    memcpy(w->go, w->g, D * sizeof(float));
    for (int i = 0; i < D * D; ++i) w->H[i] = (i / D == i % D) ? 1.f : 0.f;
    for (int step = 0; step < iters; ++step) {
        for (int i = 0; i < D; ++i) w->p[i] = -dot(w->H + i * D, w->g, D);
        const float pg = dot(w->p, w->g, D);
        float alpha = 1.f, f1 = 0.f;
        for (int trial = 0; trial < 10; ++trial) {
            conf_inc(w->xn, x, w->p, alpha, c->nt);
            f1 = eval_eg(w, w->xn, w->gn, c, sf);
            ++*n_eval;
            if (f1 - f0 < 1e-4f * alpha * pg) break;
            alpha *= 0.5f;
        }
        for (int i = 0; i < D; ++i) w->y[i] = w->gn[i] - w->g[i];
        f0 = f1;
        memcpy(x, w->xn, S * sizeof(float));
        const float gg = dot(w->gn, w->gn, D);
        memcpy(w->g, w->gn, D * sizeof(float));
        if (!(sqrtf(gg) >= 1e-5f)) break;
        const float yp = dot(w->y, w->p, D);
        if (step == 0) {
            const float yy = dot(w->y, w->y, D);
            if (fabsf(yy) > EPSF) {
                const float dg = alpha * yp / yy;
                for (int i = 0; i < D * D; ++i) w->H[i] = (i / D == i % D) ? dg : 0.f;
            }
        }
        if (alpha * yp < EPSF) continue;
        for (int i = 0; i < D; ++i) w->mhy[i] = -dot(w->H + i * D, w->y, D);
        const float yhy = -dot(w->y, w->mhy, D);
        const float r = 1.f / (alpha * yp);
        const float c2 = alpha * alpha * (r * r * yhy + r);
        for (int i = 0; i < D; ++i)
            for (int j = 0; j < D; ++j)
                w->H[i * D + j] += alpha * r * (w->mhy[i] * w->p[j] + w->mhy[j] * w->p[i]) + c2 * w->p[i] * w->p[j];
    }
    if (!(f0 <= f_orig)) {
        f0 = f_orig;
        memcpy(x, w->xo, S * sizeof(float));
        memcpy(w->g, w->go, D * sizeof(float));
    }
    return f0;
}

void port_eg(const port_lig* L, const port_grid* G, const port_sf* sf, const port_rec* R, int exact,
             const int* chain_lig, int n, const float* state, float* e_out, float* g_out) {
    const int SD = 7 + L->KM, DM = 6 + L->KM;
    #pragma omp parallel
    {
        ws_t w;
        ws_alloc(&w, L->AM, L->KM);
        #pragma omp for schedule(dynamic, 4)
        for (int ch = 0; ch < n; ++ch) {
            ctx_t c;
            ctx_init(&c, L, G, R, chain_lig[ch], exact, NULL, 0);
            memcpy(w.x, state + (long long)ch * SD, SD * sizeof(float));
            long long ne = 0;
            (void)ne;
            e_out[ch] = eval_eg(&w, w.x, w.g, &c, sf);
            for (int i = 0; i < 6 + c.nt; ++i) g_out[(long long)ch * DM + i] = w.g[i];
        }
        ws_free(&w);
    }
}

long long port_mc(const port_lig* L, const port_grid* G, const port_sf* sf, const port_rec* R, int exact,
                  const int* chain_lig, const int* chain_id, int n, const int* nbr, const int* nbr_n, int nb_max,
                  float* cur, float* cur_e, float* best, float* best_e, int init_opt, int mc_steps, int bfgs_iters,
                  float temp, float amp_pos, float amp_rot, unsigned long long seed, int step_offset) {
    const int SD = 7 + L->KM;
    long long total_eval = 0;
    #pragma omp parallel reduction(+ : total_eval)
    {
        ws_t w;
        ws_alloc(&w, L->AM, L->KM);
        #pragma omp for schedule(dynamic, 1)
        for (int ch = 0; ch < n; ++ch) {
            ctx_t c;
            ctx_init(&c, L, G, R, chain_lig[ch], exact, nbr ? nbr + (long long)ch * nb_max : NULL, nbr ? nbr_n[ch] : 0);
            const int cid = chain_id[ch], S = 7 + c.nt;
            const int iters = bfgs_iters > 0 ? bfgs_iters : (25 + c.na) / 3;
            long long ne = 0;
            memcpy(w.cur, cur + (long long)ch * SD, S * sizeof(float));
            memcpy(w.best, best + (long long)ch * SD, S * sizeof(float));
            float ec, eb = best_e[ch];
            ec = init_opt ? bfgs(&w, w.cur, iters, &c, sf, &ne) : cur_e[ch];
            if (ec < eb) { eb = ec; memcpy(w.best, w.cur, S * sizeof(float)); }
            for (int st = 0; st < mc_steps; ++st) {
                const int sg = step_offset + st;
                memcpy(w.x, w.cur, S * sizeof(float));
                const int nm = 2 + c.nt;
                int which = (int)(urand(seed, cid, sg, 0) * nm);
                if (which > nm - 1) which = nm - 1;
                float v[3];
                if (which == 0) {
                    rand_ball(seed, cid, sg, 10, v);
                    w.x[0] += amp_pos * v[0]; w.x[1] += amp_pos * v[1]; w.x[2] += amp_pos * v[2];
                } else if (which == 1) {
                    rand_ball(seed, cid, sg, 10, v);
                    const float sc = amp_rot / fmaxf(c.rg, 1.0f);
                    quat_inc(w.x + 3, sc * v[0], sc * v[1], sc * v[2]);
                } else {
                    w.x[7 + which - 2] = (2.f * urand(seed, cid, sg, 1) - 1.f) * 3.14159265f;
                }
                const float en = bfgs(&w, w.x, iters, &c, sf, &ne);
                const int accept = (en < ec) || (urand(seed, cid, sg, 2) < expf((ec - en) / temp));
                if (accept) {
                    ec = en;
                    memcpy(w.cur, w.x, S * sizeof(float));
                    if (en < eb) { eb = en; memcpy(w.best, w.x, S * sizeof(float)); }
                }
            }
            memcpy(cur + (long long)ch * SD, w.cur, S * sizeof(float));
            memcpy(best + (long long)ch * SD, w.best, S * sizeof(float));
            cur_e[ch] = ec;
            best_e[ch] = eb;
            total_eval += ne;
        }
        ws_free(&w);
    }
    return total_eval;
}

void port_stage_a(const port_lig* L, const port_grid* G, const float* conf, int C, const float* quats, int Q,
                  const float* trans, const int* ntrans, int NT_MAX, float cap, float* best_e, int* best_i) {
    const long long nb = (long long)L->L * C * Q;
    #pragma omp parallel
    {
        float* X = (float*)malloc((size_t)L->AM * 3 * sizeof(float));
        #pragma omp for schedule(dynamic, 4)
        for (long long b = 0; b < nb; ++b) {
            const int q = (int)(b % Q), cc = (int)((b / Q) % C), l = (int)(b / ((long long)Q * C));
            const int n_at = L->na[l];
            float qw = quats[4 * q], qx = quats[4 * q + 1], qy = quats[4 * q + 2], qz = quats[4 * q + 3];
            const float nq = 1.f / sqrtf(qw * qw + qx * qx + qy * qy + qz * qz);
            qw *= nq; qx *= nq; qy *= nq; qz *= nq;
            for (int a = 0; a < n_at; ++a) {
                const float* p = conf + (((long long)l * C + cc) * L->AM + a) * 3;
                X[3 * a] = (1 - 2 * (qy * qy + qz * qz)) * p[0] + 2 * (qx * qy - qz * qw) * p[1] + 2 * (qx * qz + qy * qw) * p[2];
                X[3 * a + 1] = 2 * (qx * qy + qz * qw) * p[0] + (1 - 2 * (qx * qx + qz * qz)) * p[1] + 2 * (qy * qz - qx * qw) * p[2];
                X[3 * a + 2] = 2 * (qx * qz - qy * qw) * p[0] + 2 * (qy * qz + qx * qw) * p[1] + (1 - 2 * (qx * qx + qy * qy)) * p[2];
            }
            const int ri = L->rec_idx[l];
            const float* Gp = G->flat + G->offs[ri];
            const int nx = (int)G->dims[3 * ri], ny = (int)G->dims[3 * ri + 1], nz = (int)G->dims[3 * ri + 2];
            const long long n3 = (long long)nx * ny * nz;
            const float inv = 1.f / G->spacing;
            float be = 3.4e38f;
            int bi = 0;
            for (int ti = 0; ti < ntrans[l]; ++ti) {
                const float* T = trans + ((long long)l * NT_MAX + ti) * 3;
                float e = 0.f;
                for (int a = 0; a < n_at; ++a) {
                    const float xx[3] = {X[3 * a] + T[0], X[3 * a + 1] + T[1], X[3 * a + 2] + T[2]};
                    const int dd[3] = {nx, ny, nz};
                    int id[3];
                    float ea = 0.f;
                    for (int d = 0; d < 3; ++d) {
                        int v = (int)nearbyintf((xx[d] - G->origin[3 * ri + d]) * inv);
                        id[d] = v < 0 ? 0 : (v > dd[d] - 1 ? dd[d] - 1 : v);
                        const float lo = fmaxf(G->lo[3 * ri + d] - xx[d], 0.f), hi = fmaxf(xx[d] - G->hi[3 * ri + d], 0.f);
                        ea += lo * lo + hi * hi;
                    }
                    ea = Gp[(long long)L->gslot[(long long)l * L->AM + a] * n3 + ((long long)id[0] * ny + id[1]) * nz + id[2]] +
                         G->penalty * ea;
                    e += fminf(ea, cap);
                }
                if (e < be) { be = e; bi = ti; }
            }
            best_e[b] = be;
            best_i[b] = bi;
        }
        free(X);
    }
}
