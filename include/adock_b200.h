/*
 * adock_b200 C-ABI: the docking hot path (receptor grid maps, batched pose energy/gradient, Monte-Carlo +
 * BFGS search, rigid Stage-A enumeration, receptor neighbour lists) as hand-written sm_100a CUDA.
 *
 * Conventions
 *  - Every entry point returns 0 on success or a negative ADOCK_E_* status; adock_last_error() returns a
 *    thread-local message for the last failure on the calling thread.
 *  - "dev" pointers are device memory of the current CUDA device; "host" pointers are small parameter tables
 *    read during the call. Nothing here allocates device memory unless the comment says so; scratch space is
 *    passed in by the caller (its size comes from the matching *_workspace query).
 *  - `stream` is a cudaStream_t (NULL = legacy default stream). Calls are asynchronous on that stream;
 *    device-side faults surface on the next synchronisation.
 *  - Array layouts follow the reference's packing so its Python layer can bind these symbols directly
 *    (state [N, 7+KM] = t(3), q(4, w x y z), theta(KM); gradient [N, 6+KM] = dE/dt(3), torque(3), dE/dtheta(KM)).
 */
#ifndef ADOCK_B200_H
#define ADOCK_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ADOCK_ABI_VERSION 1

#define ADOCK_OK 0
#define ADOCK_E_ARG (-1)     /* bad argument: null pointer, bad size, limit exceeded */
#define ADOCK_E_CUDA (-2)    /* CUDA runtime error (launch failure, bad device, ...) */
#define ADOCK_E_DEVICE (-3)  /* device-side status word reported an error (see adock_last_error) */

/* grid element storage */
#define ADOCK_GRID_F32 0
#define ADOCK_GRID_F16 1
#define ADOCK_GRID_BF16 2

/* ------------------------------------------------------------------------------------------------ tables */

/* Scoring-function tables shared by all search calls (host struct, copied at each call). */
typedef struct {
    float prm[15];      /* g1_off, g1_w, g2_off, g2_w, rep_off, hyd_good, hyd_bad, hb_good, hb_bad, cutoff,
                           w_g1, w_g2, w_rep, w_hyd, w_hb  (reference mckernel.py:594-596 order) */
    int n_types;        /* entries used in the tables below (<= 64) */
    float radius[64];
    int hyd[64], don[64], acc[64];
} adock_sf_t;

/* Packed ligand batch (dev), reference pack_host layout (mckernel.py:547-599). */
typedef struct {
    const float* ref;          /* [L, AM, 3] ligand-frame heavy-atom coordinates */
    const int* typ;            /* [L, AM] scoring type of each heavy atom */
    const unsigned char* tm;   /* [L, KM, AM] torsion k moves atom a */
    const int* ax;             /* [L, KM, 2] torsion axis atoms (parent side, child side) */
    const float* axp;          /* [L, KM, 3] reference axis point */
    const float* axu;          /* [L, KM, 3] reference axis unit vector */
    const int* pr;             /* [L, P, 2] intra-ligand pairs */
    const int* na;             /* [L] heavy atoms */
    const int* nt;             /* [L] torsions */
    const int* np;             /* [L] pairs */
    const float* rg;           /* [L] radius of gyration */
    const int* gslot;          /* [L, AM] grid slot of each atom */
    const int* rec_idx;        /* [L] receptor of each ligand */
    int L, AM, KM, P;
} adock_ligands_t;

/* Grid set (GridSet storage contract, grid.py:197-248), all dev. */
typedef struct {
    const void* flat;          /* concatenated per-receptor maps [T_r, nx, ny, nz], z fastest */
    const long long* offs;     /* [R] element offset of each receptor's maps in flat */
    const long long* dims;     /* [R, 3] */
    const float* origin;       /* [R, 3] */
    const float* lo;           /* [R, 3] box low corner (out-of-box penalty) */
    const float* hi;           /* [R, 3] box high corner */
    int R;
    int dtype;                 /* ADOCK_GRID_* of flat */
    float spacing, penalty;
    const int* nmaps;          /* [R] maps per receptor (dev, may be NULL: 8 assumed by the proposal features) */
} adock_grids_t;

/* Receptor atoms for the exact (grid-free) energy, dev; xyz == NULL when absent. */
typedef struct {
    const float* xyz;          /* [R, RN, 3] */
    const int* typ;            /* [R, RN] */
    const int* n;              /* [R] */
    int RN;
} adock_receptors_t;

/* B200 working layout of a ligand batch, filled by adock_prepare (dev, caller-allocated). */
typedef struct {
    void* atoms;               /* [L, AM] float4: ref xyz + (gslot | typ << 16) bits */
    void* masks;               /* [L, AM] uint32 torsion bitmask of each atom (KM <= 32) */
    void* tors;                /* [L, KM, 2] float4: axp + ax0 bits, axu + ax1 bits */
    void* pairs;               /* [L, ceil(P/32)*32] int2: (i | j << 8 | flags << 16, radius-sum bits), scheduled
                                  in rounds of 32 with no atom twice per round where possible; empty slots -1 */
    void* info;                /* [L] int4: na, nt, np, rec_idx */
    void* rg;                  /* [L] float */
} adock_work_t;

/* Monte-Carlo call arguments (reference run_mc, mckernel.py:706-726). */
typedef struct {
    const int* chain_lig;      /* dev [N] */
    const int* chain_id;       /* dev [N] RNG stream id */
    int n_chains;
    const int* nbr;            /* dev [N, NB] receptor neighbour lists or NULL */
    const int* nbr_n;          /* dev [N] */
    int nb_max;
    float* cur; float* cur_e; float* best; float* best_e;   /* dev, in place */
    int init_opt, mc_steps, bfgs_iters;
    float temp, amp_pos, amp_rot;
    unsigned long long seed;
    int step_offset;
    int exact;
    const int* order;          /* dev [N] processing order (longest first) or NULL */
    int* queue;                /* dev, 1 int work counter, zeroed by the call on `stream` */
    unsigned long long* evals; /* dev, 2 counters (accumulated): energy evaluations, atom evaluations; or NULL */
    int variant;               /* launch variant (0 = default; 1-3 = 4, 6, 8 resident blocks per SM), autotuned */
    /* learned proposal (no reference counterpart): target states [N, prop_k, 32] from adock_prop_sample for the
     * launch's steps (NULL = plain MC); a learned step proposes its target state (torsions past 20 unchanged);
     * after 8 consecutive rejections of proposed states a chain falls back to plain MC until a move is accepted */
    const float* prop;
    int prop_k;
    unsigned long long* prop_stats; /* dev [4] or NULL: proposed, proposed+accepted, plain, plain+accepted */
    /* training-data log (NULL = off): each accepted improving move appends features [320] (BF16) of the pre-move
     * state and that state [32] (t 3, q 4, torsions 20, torsion count at 27, chain index at 28) while
     * *log_n < cap; the training target (the move to the chain's final best state) is formed after the run */
    void* log_x;
    float* log_y;
    int* log_n;
    int log_cap;
    float prop_frac;           /* with proposals: fraction of steps that take the learned move (<= 0 or >= 1: all) */
    const int* lig_active;     /* dev [L] or NULL: chains of ligands whose flag is 0 are skipped (left unchanged);
                                  replaces the host-side compaction of active chains (search.py:614-627) */
    int prop_tries;            /* learned steps (no reference counterpart): candidate targets per step; each is
                                  evaluated once and BFGS runs from the lowest-energy one. prop then holds
                                  prop_k = steps x prop_tries targets per chain, the tries of a step consecutive.
                                  <= 1: one target per step */
    const float* hint;         /* dev [L, 32] or NULL: ligand-best rows (adock_prop_hint) for the logged features */
} adock_mc_args_t;

/* ------------------------------------------------------------------------------------------------ misc */
int adock_version(void);
const char* adock_last_error(void);

/* ------------------------------------------------------------------------------------------------ grids */

/* Vina/Vinardo maps: replaces the reference build_grid kernel (grid.py:14-71, launched at grid.py:132-166).
 * rec_xyz [n_rec,3], rec_types [n_rec] (dev); radius/hyd/don/acc [n_xs] and lig_types [n_lt] (host);
 * prm[15] (host, grid.py:84-87 order: cutoff, g1_off, g1_w, g2_off, g2_w, rep_off, hyd_good, hyd_bad,
 * hb_good, hb_bad, w_g1..w_hb). out (dev): [n_lt, nx, ny, nz], or [5, n_lt, nx, ny, nz] unweighted if per_term.
 * n_lt <= 24 (grid.py:74 MAX_TYPES), n_xs <= 64. */
int adock_grid_vina(const float* rec_xyz, const int* rec_types, int n_rec,
                    const float* radius, const int* hyd, const int* don, const int* acc, int n_xs,
                    const int* lig_types, int n_lt, float ox, float oy, float oz, float spacing,
                    int nx, int ny, int nz, const float* prm, int per_term, float* out, void* stream);

/* Fitted-function maps: replaces the reference build_grid_fit kernel (fit/gridfit.py:13-58, launched at
 * gridfit.py:71-93). rec_xyz [n_rec,3], rec_ext [n_rec], rad_rec [n_rt] and W [n_rt, n_lt, 6] (dev);
 * rad_lig [n_lt] and prm[12] (host, gridfit.py:80-81 order). out (dev) [n_lt, nx, ny, nz].
 * n_lt <= 64 (gridfit.py:61 MAX_LT). */
int adock_grid_fit(const float* rec_xyz, const int* rec_ext, int n_rec, const float* rad_rec, int n_rt,
                   const float* rad_lig, int n_lt, const float* W, float ox, float oy, float oz, float spacing,
                   int nx, int ny, int nz, const float* prm, float* out, void* stream);

/* The same two builders over a receptor cell list: rec_xyz / rec_types (or rec_ext) sorted by cell of a uniform
 * grid of cubic cells of edge cell_size from cell_origin [3] (host), cell_dims [3] cells per axis (host), and
 * cell_start [nx*ny*nz + 1] (dev): cell (cx, cy, cz) holds atoms [cell_start[c], cell_start[c+1]) with
 * c = (cx * ny + cy) * nz + cz. A tile of grid points reads only the cells within the cutoff of it (at most 8 x 8
 * columns of cells: cell_size >= (4 * spacing + 2 * cutoff) / 7); atoms outside the cell grid are not seen.
 * No reference counterpart (an input layout of the same kernels). */
int adock_grid_vina_cells(const float* rec_xyz, const int* rec_types, int n_rec, const int* cell_start,
                          const int* cell_dims, const float* cell_origin, float cell_size, const float* radius,
                          const int* hyd, const int* don, const int* acc, int n_xs, const int* lig_types, int n_lt,
                          float ox, float oy, float oz, float spacing, int nx, int ny, int nz, const float* prm,
                          int per_term, float* out, void* stream);
int adock_grid_fit_cells(const float* rec_xyz, const int* rec_ext, int n_rec, const int* cell_start,
                         const int* cell_dims, const float* cell_origin, float cell_size, const float* rad_rec, int n_rt,
                         const float* rad_lig, int n_lt, const float* W, float ox, float oy, float oz, float spacing,
                         int nx, int ny, int nz, const float* prm, float* out, void* stream);

/* Down-convert FP32 maps to FP16 (dtype ADOCK_GRID_F16, saturating at +-65504) or BF16 (ADOCK_GRID_BF16), round
 * to nearest. No reference counterpart (the reference stores FP32 maps only). */
int adock_grid_convert(const float* src, void* dst, long long n, int dtype, void* stream);

/* ------------------------------------------------------------------------------------------------ search */

/* Fill the B200 working layout from the reference layout (once per problem). Scalar KM <= 32, AM <= 128. */
int adock_prepare(const adock_ligands_t* lig, const adock_sf_t* sf, adock_work_t* work, void* stream);

/* Energy + analytic pose gradient of N states: replaces eg_kernel (mckernel.py:411-447) /
 * KernelProblem.energy_grad (mckernel.py:652-660). state [N, 7+KM], e [N], g [N, 6+KM] (dev). */
int adock_eg(const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
             const adock_sf_t* sf, const adock_receptors_t* rec, const int* chain_lig, int n, const float* state,
             float* e_out, float* g_out, int exact, void* stream);

/* Monte Carlo + BFGS chains in place: replaces mc_kernel (mckernel.py:328-408) / KernelProblem.run_mc
 * (mckernel.py:706-726). One persistent launch; chains are taken from a device work queue. */
int adock_mc(const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
             const adock_sf_t* sf, const adock_receptors_t* rec, const adock_mc_args_t* mc, void* stream);

/* Stage-A rigid enumeration: replaces stagea_kernel (mckernel.py:451-521) / KernelProblem.stage_a
 * (mckernel.py:690-704). conf [L, C, AM, 3], quats [Q, 4], trans [L, NT, 3], ntrans [L] (dev);
 * best_e, best_i [L, C*Q] (dev). */
int adock_stage_a(const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
                  const adock_sf_t* sf, const float* conf, int C, const float* quats, int Q, const float* trans,
                  const int* ntrans, int nt_max, float cap, float* best_e, int* best_i, void* stream);

/* adock_stage_a with the translation lattices per box instead of per ligand: trans [B, nt_max, 3], ntrans [B]
 * and lig_box [L] (dev), so ligands docked into one box share one lattice. Same kernel as adock_stage_a. */
int adock_stage_a_boxes(const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
                        const adock_sf_t* sf, const float* conf, int C, const float* quats, int Q, const float* trans,
                        const int* ntrans, int nt_max, const int* lig_box, float cap, float* best_e, int* best_i,
                        void* stream);

/* ---- device-side search pipeline: the host glue of the reference search (search.py:322-366, 506-537, 614-636)
 * as kernels, so that a whole search runs on one stream without host round trips. */

/* Stage-A conformers: replaces the torch conformer sampling of stage_a_kernel (search.py:329-337). Per ligand NT
 * torsion sets (set 0 = the input conformer; the others uniform in [-pi, pi) from a counter-based stream of
 * (seed, ligand, set, torsion)), their intra-ligand energy, and the C of lowest energy (ties: lower set index) in
 * ascending order: theta [L, C, KM], heavy-atom ligand-frame coordinates conf [L, C, AM, 3], energies e [L, C]
 * (dev). NT <= 4096, C <= NT. */
int adock_conformers(const adock_ligands_t* lig, const adock_work_t* work, const adock_sf_t* sf, int NT, int C,
                     unsigned long long seed, float* theta, float* conf, float* e, void* stream);

/* Stage-A translation lattice: replaces search.py:346-353. Per box b (box [B, 6] = centre xyz, size xyz;
 * receptor box_rec [B]; map slot of the probe type box_slot [B]; points per axis box_n [B, 3], all dev) the
 * points centre - size/2 + 1 + i * step whose nearest-grid probe energy plus out-of-box penalty is <= probe_max,
 * in lattice order (x slowest), into trans [B, nt_max, 3]; counts ntrans [B]; the box centre alone when no point
 * passes. */
int adock_lattice(const adock_grids_t* grids, int B, const float* box, const int* box_rec, const int* box_slot,
                  const int* box_n, float step, float probe_max, int nt_max, float* trans, int* ntrans, void* stream);

/* Start states: replaces search.py:356-366. Per ligand the M lowest of best_e[l, j] + e_conf[l, j / Q] over
 * j < C*Q (ties: lower j; cycled when C*Q < M); state [L*M, 7+KM] = (trans[lig_box[l], best_i[l, j]],
 * quats[j % Q], theta[l, j / Q]); e_start [L*M] the sorted totals (may be NULL). lig_box may be NULL (box = l).
 * C*Q <= 16384. */
int adock_select_starts(int L, int C, int Q, int KM, int M, const float* best_e, const int* best_i,
                        const float* e_conf, const float* quats, const float* theta, const float* trans,
                        const int* lig_box, int nt_max, float* state, float* e_start, void* stream);

/* Per-segment bookkeeping of the MC phase: replaces the host logic of search.py:615-636. After segment sg of
 * `seg` steps (chains ligand-major, M per ligand): *chain_steps += M * seg per active ligand (may be NULL); per
 * ligand glob = min(glob, best over its chains), stall = 0 if that improved glob by more than es_tol else +1,
 * active &= seg_lim > next_sg && (es_rounds <= 0 || stall < es_rounds). All arrays dev. */
int adock_segment_update(int L, int M, int seg, int next_sg, int es_rounds, float es_tol, const float* best_e,
                         const int* seg_lim, float* glob, int* stall, int* active, unsigned long long* chain_steps,
                         void* stream);

/* Greedy clustering of the final poses: replaces search.py:516-531. Per ligand its P poses (e_total [L*P],
 * heavy-atom coordinates X [L*P, AM, 3], dev) in ascending energy order (ties: lower index); a pose becomes a
 * representative when its heavy-atom RMSD to every earlier one is >= cut, until n_out are found:
 * reps [L, n_out] (pose index within the ligand, -1 past n_reps[l]). P <= 4096, n_out <= 32. */
int adock_cluster(const adock_work_t* work, int L, int P, const double* e_total, const float* X, int AM, float cut,
                  int n_out, int* reps, int* n_reps, void* stream);

/* All-atom world coordinates of n states: replaces ligand.pose_coords (ligand.py:216-237) for the returned poses.
 * ref_all [L, A, 3] ligand-frame coordinates of every atom (hydrogens included), mask_all [L, A] torsion bitmask
 * of each atom (bit k: torsion k moves it), torsion axes from `work`; X [n, A, 3] (all dev). */
int adock_pose_atoms(const adock_work_t* work, int KM, const float* ref_all, const unsigned* mask_all, int A,
                     const int* chain_lig, int n, const float* state, float* X, void* stream);

/* Receptor neighbour lists: replaces KernelProblem.receptor_neighbours (mckernel.py:662-688).
 * Pass 1 (nbr == NULL): counts [N] of receptor atoms within `cut` of any heavy atom of each chain's pose.
 * Pass 2: nbr [N, nb_max] filled in receptor index order (counts recomputed into nbr_n). */
int adock_neighbours(const adock_ligands_t* lig, const adock_work_t* work, const adock_sf_t* sf,
                     const adock_receptors_t* rec, const int* chain_lig, int n, const float* state, float cut,
                     int* nbr, int* nbr_n, int nb_max, void* stream);

/* Final re-score in float64 on the device: exact inter (pairwise over all receptor atoms when rec->xyz is
 * set, else the grid), out-of-box penalty and intra energy of N states; writes e_total, e_intra [N] (dev,
 * double) and world coordinates X [N, AM, 3] (dev, float). Replaces the rescoring half of finalize_kernel
 * (search.py:506-537). */
int adock_rescore64(const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
                    const adock_sf_t* sf, const adock_receptors_t* rec, const int* chain_lig, int n,
                    const float* state, double* e_total, double* e_intra, float* X, void* stream);

/* ------------------------------------------------------------------------------------------------ proposal net */
/* No reference counterpart: the learned MC proposal. Network 320 -> 256 (SiLU) -> 256 (SiLU) -> 64, BF16
 * weights, FP32 accumulation; output columns 0..25 = move means, 32..57 = log standard deviations. */

/* Feature rows (BF16 [n, 320], dev) of n states (layout in csrc/search_impl.cuh prop_features). cur_e [n] (the
 * states' energies) and hint [L, 32] (adock_prop_hint) may be NULL: the ligand-best columns are then 0. */
int adock_prop_features(const adock_ligands_t* lig, const adock_work_t* work, const adock_grids_t* grids,
                        const adock_sf_t* sf, const int* chain_lig, int n, const float* state, const float* cur_e,
                        const float* hint, void* feat, void* stream);
/* Ligand-best rows hint [L, 32] (dev): for each ligand, the best state (t 3, q 4, torsions 0..19) of its chain with
 * the lowest finite best_e (ties: the lowest chain index), that energy at 27 and 1 at 28; all 0 for a ligand
 * without such a chain. best [n, SD] and best_e [n] are the chains' best states and energies; keys is device
 * scratch of L x 8 bytes. */
int adock_prop_hint(int L, int n, const int* chain_lig, const float* best, int SD, const float* best_e, void* keys,
                    float* hint, void* stream);
/* Proposed target states [n, k, 32] (dev; t 3, q 4, torsions 20, rest 0) drawn from the network output [n, 64]
 * around the states state [n, SD] the network read: move = mean + max(exp(log_sd), floor) * z, z standard normal
 * from a counter-based stream of (seed, chain_id, segment, slot), applied to the state (translation added,
 * rotation vector composed on the left of q, torsion deltas added; torsions past a ligand's count keep their
 * value). k <= 512. n_comp = 3: the translation mean is one of the network's 3 mixture components (means at
 * columns 0, 27, 58, mixing logits at 26, 30, 61), drawn by its softmax weight; n_comp = 1: column 0 only. */
int adock_prop_sample(const adock_ligands_t* lig, const adock_work_t* work, const int* chain_lig, const int* chain_id,
                      int n, const float* net_out, const float* state, int SD, int k, int n_comp,
                      unsigned long long seed, int segment, float* targets, void* stream);
/* C[M,N] = A[M,K] B[K,N] on the 5th-generation tensor cores (tcgen05.mma, accumulator in tensor memory; BF16
 * operands at any strides, FP32 accumulation); epilogue C = acc + beta C + bias, optional pre-activation copy,
 * optional SiLU (act = 1), optional BF16 copy Cb. */
int adock_gemm_bf16(int M, int N, int K, const void* A, long long sAm, long long sAk, const void* B, long long sBk,
                    long long sBn, float* C, long long ldc, float beta, const float* bias, int act, float* pre,
                    void* Cb, long long ldcb, void* stream);
/* The same product on the warp-level mma.sync tensor-core path (an independent implementation, kept to
 * cross-check adock_gemm_bf16). */
int adock_gemm_bf16_mma(int M, int N, int K, const void* A, long long sAm, long long sAk, const void* B,
                        long long sBk, long long sBn, float* C, long long ldc, float beta, const float* bias, int act,
                        float* pre, void* Cb, long long ldcb, void* stream);
/* Device status of the tcgen05 GEMMs since the last call (synchronises): ADOCK_E_DEVICE if a CTA gave up waiting
 * for its tensor-core work (its tile is then not written), else 0. Clears the status. */
int adock_gemm_status(void);
/* Gaussian NLL of moves target [B, 32] under out [B, 64]; dout (BF16 [B, 64]) = gradient of the batch mean;
 * *loss += summed NLL. n_comp = 3: the translation term is a 3-component mixture (layout as adock_prop_sample). */
int adock_mlp_nll(const float* out, const float* target, int B, int n_comp, void* dout, float* loss, void* stream);
/* dA = dH * SiLU'(A), BF16 output. */
int adock_silu_backward(const float* dH, const float* A, long long n, void* dA, void* stream);
/* db = column sums of dA (BF16 [rows, cols]). */
int adock_bias_grad(const void* dA, int rows, int cols, float* db, void* stream);
/* Adam step on FP32 master parameters p (with BF16 copy pb, may be NULL). */
int adock_adam(float* p, const float* grad, float* m, float* v, void* pb, long long n, float lr, float b1, float b2,
               float eps, int step, float wd, void* stream);
int adock_f32_to_bf16(const float* x, void* y, long long n, void* stream);

/* ------------------------------------------------------------------------------------------------ no allocation */

/* No counterpart in the reference. adock_mc for callers that cannot allocate device memory (a stream being
 * captured into a graph by a framework that forbids allocation during capture, a memory pool that owns the
 * device, a host application that passes only raw input/output pointers). The ligand working layout and the
 * work-queue counter that adock_mc takes from the caller live instead in one library-owned device array of
 * ADOCK_NOALLOC_SCRATCH_MAX bytes, held on every device that loads the library until the process exits.
 * Inputs and outputs are as for adock_mc (mc->queue is ignored; mc->order and mc->evals are optional). Batches
 * whose scratch (adock_mc_noalloc_scratch_bytes) exceeds the limit are rejected with ADOCK_E_ARG. No call
 * allocates. The first call on a device looks up the array's device address and should come before any stream
 * capture on that device. All calls share the array: calls that overlap on the GPU race. */
#define ADOCK_NOALLOC_SCRATCH_MAX (16u << 20)
size_t adock_mc_noalloc_scratch_bytes(int L, int AM, int KM, int P);
int adock_mc_noalloc(const adock_ligands_t* lig, const adock_grids_t* grids, const adock_sf_t* sf,
                     const adock_receptors_t* rec, const adock_mc_args_t* mc, void* stream);

#ifdef __cplusplus
}
#endif
#endif
