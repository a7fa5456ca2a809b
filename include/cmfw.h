/* cmfw.h -- C ABI of the B200 pFq Conservative Matrix Field walk engine.
 *
 * Plain pointers and sizes only. Every walk entry point takes DEVICE
 * pointers and a CUDA stream (as `void *`, NULL = legacy default stream),
 * enqueues its kernels and returns without synchronising, except where a
 * comment says otherwise. The `_host` entry points take HOST buffers, copy
 * them to the device, run, copy the results back and synchronise.
 *
 * The reference (VesterlundCoder/RamanujanDreams-CUDA) exposes no library:
 * its boundary is three programs, each of which builds inputs, launches one
 * kernel `walk_kernel_<variant><<<grid, block>>>(inputs, results, desc, N, h,
 * n_traj[, n_primes])` and writes JSON. The entry points below replace those
 * launches (cited per function); the records keep the reference's byte
 * layout so that the reference's own input builders can feed them.
 *
 * Threading: calls are thread-safe; calls on different streams may overlap.
 * Errors: every entry point returns a cmfw_status; cmfw_last_error() gives
 * a message for the calling thread's most recent failure. Per-trajectory
 * failures are not call failures: they set `valid = 0` in the record, and
 * the optional status array says why (cmfw_traj_status).
 */
#ifndef CMFW_H
#define CMFW_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CMFW_MAX_DIM 8    /* cmf_pfq.cuh:36  MAX_DIM  */
#define CMFW_MAX_AXES 16  /* cmf_pfq.cuh:38  MAX_AXES */
#define CMFW_MAX_COMPAT_MODULI 64   /* cmf_walk_rns.cu:23 MAX_PRIMES */
#define CMFW_MAX_EXACT_PRIMES 4096

typedef enum {
    CMFW_OK = 0,
    CMFW_EINVAL = 1,      /* argument out of the supported range */
    CMFW_ECUDA = 2,       /* a CUDA runtime call failed */
    CMFW_ENOMEM = 3,      /* device or host allocation failed */
    CMFW_ETIMEOUT = 4,    /* a bounded device wait gave up */
    CMFW_EUNSUPPORTED = 5 /* built without the requested kernel */
} cmfw_status;

/* Why a trajectory is invalid (values of the optional status array). */
typedef enum {
    CMFW_TRAJ_OK = 0,
    CMFW_TRAJ_SINGULAR_LEAD = 1,   /* companion lead coefficient ~ 0 (cmf_pfq.cuh:173) */
    CMFW_TRAJ_SINGULAR_DENOM = 2,  /* axis denominator ~ 0 (cmf_pfq.cuh:193) */
    CMFW_TRAJ_SINGULAR_SOLVE = 3,  /* inverse-step scalar solve ~ 0 (cmf_pfq.cuh:225) */
    CMFW_TRAJ_NONFINITE = 4,       /* non-finite or all-zero walk matrix (cmf_pfq.cuh:109) */
    CMFW_TRAJ_BAD_DEPTH = 5,       /* N <= 0, h <= 0 or N - 2h <= 0 (cmf_pfq.cuh:352) */
    CMFW_TRAJ_STEP_CAP = 6,        /* |dir| beyond CMFW_MAX_DIR_COMPONENT */
    CMFW_TRAJ_MODULUS_ZERO = 7,    /* exact walk: a divisor vanished modulo this prime */
    CMFW_TRAJ_NOT_INTEGRAL = 8,    /* exact walk: a start coordinate is not an integer */
    CMFW_TRAJ_BAD_FAMILY = 9       /* mixed batch: descriptor index out of range */
} cmfw_traj_status;

/* Largest |dir[a]| a trajectory may use; larger components mark the
 * trajectory CMFW_TRAJ_STEP_CAP instead of walking (bounded device loops). */
#define CMFW_MAX_DIR_COMPONENT 4096
/* Largest depth N a walk call accepts (CMFW_EINVAL above it). */
#define CMFW_MAX_DEPTH (1 << 26)

/* CMFDesc (cmf_pfq.cuh:41-47), same field order and layout. */
typedef struct {
    int p;      /* numerator parameters (x axes), 1..8 */
    int q;      /* denominator parameters (y axes), 0..7 */
    int rank;   /* walk-matrix dimension, 2..8 */
    int naxes;  /* p + q */
    double z;
} cmfw_desc;

/* TrajectoryInput / DF64Input / RNSInput (cmf_walk_f64.cu:36-39): 192 bytes. */
typedef struct {
    int dir[CMFW_MAX_AXES];       /* lattice direction, x axes then y axes */
    double start[CMFW_MAX_AXES];  /* start position (x_1..x_p, y_1..y_q) */
} cmfw_traj_in;

/* DF64Result / RNSResult (cmf_walk_df64.cu:293-302): 56 bytes. The f64
 * program's TrajectoryResult (cmf_walk_f64.cu:41-51) is this record plus a
 * trailing, never-written `elapsed_ms`. */
typedef struct {
    double limit;      /* first Aitken limit, else first candidate */
    double delta;      /* irrationality-measure estimate */
    double p, q;       /* M[0][rank-1], M[1][rank-1] of the normalised matrix at depth N */
    double precision;  /* -log10 |p_N/q_N - p_{N-h}/q_{N-h}| */
    double log_scale;  /* log of the normalisation scale at depth N */
    int valid;         /* 1 = walked all N steps */
    int n_limits;      /* limit candidates found (capped at 256) */
} cmfw_traj_out;

/* Launch options; a zeroed struct (or NULL) selects the defaults. */
typedef struct {
    int block_size;        /* threads per block; 0 = tuned default */
    int flags;             /* CMFW_F_* below */
    uint8_t *d_status;     /* optional per-trajectory cmfw_traj_status */
    void *d_workspace;     /* optional caller-owned scratch (see *_workspace_bytes) */
    size_t workspace_bytes;
    int *d_limit_src;      /* optional per-trajectory source of `limit`:
                              (method << 12) | (i << 8) | (j << 4) | column for
                              the ratio M[i][column] / M[j][column]; method 1 =
                              Aitken, 0 = raw ratio; -1 = no candidate */
    void *ev_main_start;   /* optional cudaEvent_t pair recorded on the stream */
    void *ev_main_stop;    /* right before and after the walk's main kernel (the
                              chunk kernel of the chunked f64/df64 walk, the walk
                              kernel of the others): its own duration */
} cmfw_launch;

/* df64 arithmetic: reproduce the reference's float-reciprocal semantics
 * (cmf_walk_df64.cu:110-113, 138-153, 184, 194, 210). Default: accurate
 * float-float with refined reciprocals and power-of-two renormalisation. */
#define CMFW_F_DF64_COMPAT 0x1
/* RNS compat: evaluate the column polynomial with separately rounded
 * products and sums (the reference compiled for a CPU) instead of fused
 * multiply-adds (the reference compiled by nvcc). */
#define CMFW_F_UNFUSED_COLUMN 0x2
/* f64 / df64: walk each trajectory in one thread from step 1 to N instead of
 * the default chunked walk (a short one-thread prefix, then the remaining
 * steps split over one CTA per trajectory -- 256 threads up to rank 6, else
 * 128 -- and multiplied back in order).
 * block_size is the CTA size of the sequential kernels only. */
#define CMFW_F_SEQUENTIAL 0x4
/* f64 chunked walk: walk the runs and multiply them in plain FP64 instead of
 * double-double. Fewer instructions, but rounding inside a run can be
 * amplified when the runs are multiplied back together, so results may be
 * less accurate than the sequential walk's. */
#define CMFW_F_PLAIN_RUNS 0x8
/* f64 / df64 chunked walk: walk every trajectory that passes the filter in
 * one CTA, whatever the batch. By default a batch with fewer survivors than
 * SMs spreads each survivor over several CTAs, in numbers that depend on the
 * whole batch; that changes the association of the walk's product and so
 * its rounding (in f64 by about an ulp, in df64 visibly on ill-conditioned
 * walks). With this flag a trajectory's result is the same bits in every
 * batch (on a given GPU), at the cost of latency for small batches. */
#define CMFW_F_BATCH_INVARIANT 0x10

/* ---- descriptors and library state -------------------------------- */

const char *cmfw_version(void);
const char *cmfw_last_error(void);
/* make_cmf_desc (cmf_pfq.cuh:50-61). */
cmfw_desc cmfw_make_desc(int p, int q, double z);
/* CMFW_OK when desc is within the supported range (p <= 8, q <= 7,
 * 2 <= rank <= 8, naxes == p + q). */
cmfw_status cmfw_check_desc(const cmfw_desc *desc);

/* Scratch a walk call needs when the caller supplies d_workspace; when
 * d_workspace is NULL the library uses its own per-device buffer. */
size_t cmfw_walk_workspace_bytes(const cmfw_desc *desc, int n_traj);

/* ---- plain walks (device buffers) --------------------------------- */

/* Replaces walk_kernel_f64<<<...>>>(inputs, results, desc, N, h, n_traj)
 * (cmf_walk_f64.cu:94-96, 228). */
cmfw_status cmfw_walk_f64(const cmfw_desc *desc, const cmfw_traj_in *d_in, cmfw_traj_out *d_out,
                          int n_traj, int N, int h, const cmfw_launch *launch, void *stream);

/* ---- f64 walk without any allocation (no counterpart in the reference) --
 * For callers that cannot call cudaMalloc: code whose device memory all
 * comes from another allocator's pool (a framework's caching allocator that
 * must account for every byte), and code that may not synchronise the device
 * mid-run, which a first cudaMalloc/cudaFree can do. cmfw_walk_f64 without a
 * caller workspace allocates its scratch on first use; this entry point runs
 * the same walk (same kernels, same results) with its scratch in a fixed
 * array of CMFW_NOALLOC_SCRATCH_BYTES inside the library's device image,
 * which every GPU that loads the library holds until the process exits. The
 * caller passes device inputs and outputs as for cmfw_walk_f64.
 *  - Capacity: cmfw_walk_workspace_bytes(desc, n_traj) must not exceed
 *    CMFW_NOALLOC_SCRATCH_BYTES (about 50,000 trajectories at rank 5, 20,000
 *    at rank 8); a larger batch returns CMFW_EINVAL, and the caller splits it.
 *  - Set-up: the first call on a device looks up the array's device address
 *    (cudaGetSymbolAddress) with that device current; make that first call
 *    before capturing any stream.
 *  - Sharing: all calls on a device share the one array. Calls that overlap
 *    on the GPU (other streams, other host threads) race on it and give wrong
 *    results; serialise them on one stream. What must start at zero (the
 *    survivor counter) is cleared on the stream by each call. */
#define CMFW_NOALLOC_SCRATCH_BYTES (32u << 20)
cmfw_status cmfw_walk_f64_noalloc(const cmfw_desc *desc, const cmfw_traj_in *d_in, cmfw_traj_out *d_out,
                                  int n_traj, int N, int h, void *stream);

/* Replaces walk_kernel_df64<<<...>>>(inputs, results, desc, N, h, n_traj)
 * (cmf_walk_df64.cu:304-306, 410). */
cmfw_status cmfw_walk_df64(const cmfw_desc *desc, const cmfw_traj_in *d_in, cmfw_traj_out *d_out,
                           int n_traj, int N, int h, const cmfw_launch *launch, void *stream);

/* Replaces walk_kernel_rns<<<...>>>(inputs, results, desc, N, h, n_traj,
 * n_primes) (cmf_walk_rns.cu:260-262, 381). Residues are bit-identical to
 * the reference's: same 64-entry modulus table, same rounded column, same
 * 100-step two-modulus reconstruction. 1 <= n_primes <= 64. */
cmfw_status cmfw_walk_rns(const cmfw_desc *desc, const cmfw_traj_in *d_in, cmfw_traj_out *d_out,
                          int n_traj, int N, int h, int n_primes, const cmfw_launch *launch,
                          void *stream);

/* Residue matrices of the compat RNS walk after `steps` trajectory steps
 * (the state inside walk_kernel_rns, cmf_walk_rns.cu:281-298, which the
 * reference never exports). d_res: n_traj * n_primes * rank * rank uint32,
 * trajectory-major, then modulus, row, column. d_ok: n_traj ints. */
cmfw_status cmfw_rns_trace(const cmfw_desc *desc, const cmfw_traj_in *d_in, int n_traj, int N,
                           int h, int n_primes, int steps, int flags, uint32_t *d_res, int *d_ok,
                           void *stream);

/* ---- exact walk (no reference counterpart: the reference's RNS rounds) --
 * The walk product is kept exactly as rational residues modulo K primes
 * (one warp lane per prime, Montgomery arithmetic): each step multiplies by
 * I + C/a or its inverse with C's column -d/lead taken mod the prime. At
 * the snapshot depths N-2h, N-h, N two entries of one column are written,
 * M[i][c] and M[j][c] (by default i = 0, j = 1, c = rank-1: p and q), so
 * that their ratio (and each entry) can be recovered by CRT and rational
 * reconstruction on the host.
 * d_primes: K distinct odd primes below 2^31. d_pairs: optional n_traj
 * packed (i << 8) | (j << 4) | c selectors (the low 12 bits of
 * cmfw_launch.d_limit_src values are accepted as they are). d_res: n_traj
 * * 3 * 2 * K uint32 (trajectory, snapshot, {M[i][c], M[j][c]}, prime).
 * d_prime_ok: n_traj * K bytes, 1 where no divisor vanished modulo that
 * prime; 0 for every prime when the trajectory cannot be walked exactly
 * (bad depth, direction cap, non-integral start). */
cmfw_status cmfw_exact_residues(const cmfw_desc *desc, const cmfw_traj_in *d_in, int n_traj,
                                int N, int h, const uint32_t *d_primes, int K, const int *d_pairs,
                                uint32_t *d_res, uint8_t *d_prime_ok, void *stream);
/* The exact ratios of cmfw_exact_residues' output, reconstructed on the
 * device (no reference counterpart: the reference's CRT uses two primes and
 * rounds, cmf_walk_rns.cu:225-251). Per trajectory t and depth s (task
 * 3 t + s): the rational n / d whose residues modulo d_primes[0..K) are
 * res[t][s][0][k] / res[t][s][1][k], over the primes with prime_ok set and a
 * non-zero denominator residue; res and prime_ok are laid out with `stride`
 * primes per trajectory (K <= stride: a prefix of the walked primes may be
 * used). One warp per task: Garner's mixed-radix CRT with a lane per prime,
 * rational reconstruction by the half-extended Euclidean algorithm to
 * Wang's bound, and a check on the last 4 usable primes, which the fit
 * leaves out. Primes must be odd and in (2^30, 2^31). Outputs per task: the
 * magnitudes of n and d as little-endian 32-bit words in
 * d_num / d_den[task * cmfw_exact_recon_words(K) ...], their word counts, the
 * sign of n, and d_status: 0 = n / d, 1 = the denominator vanishes modulo
 * every usable prime (exactly zero), 2 = undetermined (too few primes for
 * its size, or the check failed: add primes), 3 = no usable prime (the
 * exact walk is singular). */
int cmfw_exact_recon_words(int K);
cmfw_status cmfw_exact_reconstruct(const uint32_t *d_res, const uint8_t *d_prime_ok, const uint32_t *d_primes,
                                   int n_traj, int stride, int K, uint32_t *d_num, uint32_t *d_den,
                                   int *d_num_words, int *d_den_words, int8_t *d_sign, uint8_t *d_status,
                                   void *stream);

/* ---- mixed batches (no reference counterpart: the reference walks one
 * family at one depth per program run, cmf_walk_f64.cu:156-305) ---------
 * Trajectories of up to 16 descriptors (family, z) with per-trajectory
 * depth N in one enqueue: a device counting sort by (descriptor, cost =
 * N * sum|dir| descending), then per descriptor a persistent kernel whose
 * warps take cost-sorted trajectories from a queue; the walk of one
 * trajectory is the sequential walk (f64, or df64 = float-float on the FP32
 * pipe with an FP64 snapshot reduction). Results land at each trajectory's
 * own index; a trajectory whose descriptor index is out of range gets
 * CMFW_TRAJ_BAD_FAMILY. The caller passes a workspace of
 * cmfw_mixed_workspace_bytes() in launch->d_workspace (the enqueue allocates
 * nothing, so it can be captured into a CUDA graph); launch->d_status and
 * d_limit_src work as for the plain walks, block_size is not used. */
#define CMFW_MAX_MIXED_DESCS 16
typedef struct {
    int desc; /* index into the descriptor array */
    int N;    /* depth; snapshots at N-2h, N-h, N */
} cmfw_mixed_item;
typedef struct {
    int block_size;  /* threads per CTA: 64, 128 or 256 */
    int grab;        /* trajectories a warp takes per queue access (multiple of
                        32); 0 = a plain grid, one sorted trajectory per thread */
    int ctas_per_sm; /* resident CTAs per SM, 0 = as many as fit */
} cmfw_mixed_tile;
typedef struct {
    int persistent; /* 1: cost-sorted queues (tiles below); 0: the baseline, one
                       thread per sorted trajectory in 256-thread CTAs */
    cmfw_mixed_tile tile[CMFW_MAX_MIXED_DESCS];
    int prescan;    /* with persistent: follow every trajectory through its N
                       steps with the position-only singularity tests first
                       and walk only the survivors */
} cmfw_mixed_tuning;
size_t cmfw_mixed_workspace_bytes(int n_traj, int n_descs);
/* tuning NULL = persistent, 128 threads, grab 32, full occupancy, no prescan.
 * After the sort (on `stream`), every descriptor's walk runs on a stream of
 * its own forked from `stream` and joined back into it, so the descriptors'
 * walks overlap (a walk ends with its longest trajectories on a few SMs). */
cmfw_status cmfw_walk_mixed(const cmfw_desc *descs, int n_descs, const cmfw_traj_in *d_in,
                            const cmfw_mixed_item *d_items, cmfw_traj_out *d_out, int n_traj, int h,
                            int variant, const cmfw_mixed_tuning *tuning, const cmfw_launch *launch,
                            void *stream);
/* Autotuner: per descriptor, times every (block 64/128/256) x (grab 0/32/64)
 * on a strided sample of up to `sample` (0 = 65536) of that descriptor's
 * cost-sorted trajectories; then, since the descriptors' walks run side by
 * side, times whole tunings on the joint sample (the plain grid everywhere,
 * the per-descriptor choices, each tile for every descriptor) and returns
 * the fastest. Synchronises the stream; writes scratch results into d_out. */
cmfw_status cmfw_mixed_autotune(const cmfw_desc *descs, int n_descs, const cmfw_traj_in *d_in,
                                const cmfw_mixed_item *d_items, cmfw_traj_out *d_out, int n_traj, int h,
                                int variant, const cmfw_launch *launch, int sample, cmfw_mixed_tuning *out,
                                void *stream);
/* The whole mixed walk (sort, queues reset, per-descriptor kernels) captured
 * once into a CUDA graph over fixed buffers and replayed with one launch.
 * Without launch->d_workspace the graph owns one. */
typedef struct cmfw_mixed_graph cmfw_mixed_graph;
cmfw_status cmfw_mixed_graph_create(const cmfw_desc *descs, int n_descs, const cmfw_traj_in *d_in,
                                    const cmfw_mixed_item *d_items, cmfw_traj_out *d_out, int n_traj, int h,
                                    int variant, const cmfw_mixed_tuning *tuning, const cmfw_launch *launch,
                                    cmfw_mixed_graph **out);
cmfw_status cmfw_mixed_graph_launch(cmfw_mixed_graph *graph, void *stream);
void cmfw_mixed_graph_destroy(cmfw_mixed_graph *graph);

/* ---- learned trajectory proposal (no reference counterpart) -----------
 * A 4-layer MLP (CMFW_MLP_IN -> 256 -> 256 -> 256 -> 1, ReLU) over a
 * trajectory's features -- direction components dir[0..14] / 4 and a
 * one-hot of the CMF family (0..4 = 3F2, 4F3, 5F4, 6F5, 8F7) -- that
 * regresses a walk outcome. Dense layers run as BF16 x BF16 -> FP32
 * tcgen05 tensor-core GEMMs with fused epilogues; parameters are FP32
 * masters (BF16 copies for the tensor cores) trained with Adam by the
 * library's own forward and backward kernels. Batches hold up to the
 * model's capacity (rounded up to 128). Parameters flatten in the order
 * W1 [256 x 64], b1, W2 [256 x 256], b2, W3 [256 x 256], b3, w4 [256], b4. */
#define CMFW_MLP_IN 64
#define CMFW_MLP_HIDDEN 256
typedef struct cmfw_mlp cmfw_mlp;
cmfw_status cmfw_mlp_create(int max_batch, uint64_t seed, cmfw_mlp **out);
void cmfw_mlp_destroy(cmfw_mlp *mlp);
size_t cmfw_mlp_param_count(void);
cmfw_status cmfw_mlp_get_params(cmfw_mlp *mlp, float *h_params);
cmfw_status cmfw_mlp_set_params(cmfw_mlp *mlp, const float *h_params);
/* d_score[i] = network(features(d_in[i], d_family[i])). */
cmfw_status cmfw_mlp_forward(cmfw_mlp *mlp, const cmfw_traj_in *d_in, const int *d_family, int n,
                             float *d_score, void *stream);
/* Gradients of loss = sum_i w_i (score_i - target_i)^2 / weight_sum (w = 1
 * when d_weight is NULL) into h_grads (cmfw_mlp_param_count floats) and the
 * loss into *h_loss; synchronises. Every sum over the batch is taken in a
 * fixed order: the same inputs give the same bits, and so does training. */
cmfw_status cmfw_mlp_gradients(cmfw_mlp *mlp, const cmfw_traj_in *d_in, const int *d_family,
                               const float *d_target, const float *d_weight, int n, float weight_sum,
                               float *h_grads, float *h_loss, void *stream);
/* One Adam step (beta 0.9 / 0.999) on that loss; *d_loss gets the loss. */
cmfw_status cmfw_mlp_train_step(cmfw_mlp *mlp, const cmfw_traj_in *d_in, const int *d_family,
                                const float *d_target, const float *d_weight, int n, float weight_sum,
                                float lr, float *d_loss, void *stream);
/* One epoch of Adam steps over trajectories d_perm[0..n) of the training
 * set in order, `batch` at a time (full batches only; batch <= the model's
 * capacity): each step weighs its rows by d_weight (NULL: 1) over their
 * sum, computed on the device, so the epoch needs no host round trip;
 * *d_loss gets the last step's loss (untouched when n < batch). */
cmfw_status cmfw_mlp_train_epoch(cmfw_mlp *mlp, const cmfw_traj_in *d_in, const int *d_family,
                                 const float *d_target, const float *d_weight, const long long *d_perm,
                                 long long n, int batch, float lr, float *d_loss, void *stream);
/* CMFW_ETIMEOUT if a bounded tensor-core wait of an earlier call gave up. */
cmfw_status cmfw_mlp_status(cmfw_mlp *mlp);
/* Candidates first .. first+n-1 of a seeded generator: direction component
 * a of candidate i is lo + (16-bit field of splitmix64 draws) mod
 * (hi - lo + 1) for the first naxes axes (naxes <= 15). Scores all of them
 * with the network (family one-hot `family`) into d_scores[0..n). */
cmfw_status cmfw_mlp_score_candidates(cmfw_mlp *mlp, uint64_t seed, long long first, long long n, int naxes,
                                      int lo, int hi, int family, float *d_scores, void *stream);
/* The same scores in one launch: clusters of two CTAs keep the three
 * hidden layers' weights resident in shared memory (each CTA half of every
 * layer), generate the candidates' features in place and exchange the
 * activation halves through distributed shared memory. */
cmfw_status cmfw_mlp_score_candidates_fused(cmfw_mlp *mlp, uint64_t seed, long long first, long long n,
                                            int naxes, int lo, int hi, int family, float *d_scores,
                                            void *stream);
/* The same network on candidates d_idx[0..n) of the generator (any subset,
 * e.g. the survivors of cmfw_filter_candidates), scores into d_scores[0..n).
 * No reference counterpart (the learned proposal is this project's). */
cmfw_status cmfw_mlp_score_indices(cmfw_mlp *mlp, uint64_t seed, const long long *d_idx, long long n, int naxes,
                                   int lo, int hi, int family, float *d_scores, void *stream);
/* The chunked walk's singularity filter on candidates first .. first+n-1
 * of the generator (start h_start[0..naxes), naxes <= 15): the position-only
 * tests of the first `steps` lattice steps (the walk itself uses 1), no
 * matrix work. The indices of the candidates that pass go to d_idx (at most
 * cap, in no particular order) and their number to *d_count (which may
 * exceed cap: then only cap were written); d_count is cleared on the
 * stream first. Every other candidate is an invalid walk (the reference's
 * tests of cmf_pfq.cuh:164-174, 193 and 225-232 on its first steps); with
 * N - 2h <= 0 none pass. No reference counterpart (the reference walks every
 * trajectory). */
cmfw_status cmfw_filter_candidates(const cmfw_desc *desc, uint64_t seed, long long first, long long n, int lo,
                                   int hi, const double *h_start, int N, int h, int steps, long long *d_idx,
                                   long long cap, unsigned long long *d_count, void *stream);
/* Records of the candidates d_idx[0..n) of the same generator, start d_start. */
cmfw_status cmfw_candidate_records(uint64_t seed, const long long *d_idx, int n, int naxes, int lo, int hi,
                                   const double *d_start, cmfw_traj_in *d_out, void *stream);
/* Indices of the k largest of d_scores[0..n) (n < 2^32; equal scores
 * ordered by lower index, so exactly min(k, n) are selected; at most cap
 * written, in no particular order) into d_idx, their number in *h_count;
 * synchronises. */
cmfw_status cmfw_select_top(const float *d_scores, long long n, long long k, long long *d_idx, int cap,
                            int *h_count, void *stream);

/* ---- input records -------------------------------------------------- */

/* The reference programs' input records for `mode` (0 = limit, 1 = delta)
 * and `use_zeta`, byte for byte as run_benchmark() builds them
 * (cmf_walk_f64.cu:166-199 with the generators of cmf_walk_f64.cu:61-91,
 * std::mt19937_64 seeded 42, including their write strides). */
cmfw_status cmfw_reference_inputs(int p, int q, int n_traj, int mode, int use_zeta, cmfw_traj_in *h_out);
/* n outputs of std::mt19937_64(seed), for seeded workload generators. */
void cmfw_mt64_fill(uint64_t seed, uint64_t *out, size_t n);
/* Outputs offset .. offset+n-1 of std::mt19937_64(seed): long seeded streams
 * drawn in pieces without regenerating their start. */
void cmfw_mt64_fill_at(uint64_t seed, uint64_t offset, uint64_t *out, size_t n);

/* ---- host-buffer convenience (what the drop-in programs call) ------- */

typedef enum { CMFW_VARIANT_F64 = 0, CMFW_VARIANT_DF64 = 1, CMFW_VARIANT_RNS = 2 } cmfw_variant;

/* Copies h_in to the device, runs the variant, copies results to h_out and
 * synchronises. *kernel_ms (optional) receives the event-timed duration of
 * the walk kernels alone; *total_ms (optional) the copies included. For the
 * chunked f64 and df64 walks the results start back to h_out on a side
 * stream once the filter kernel has written every early failure, and the
 * survivors' records, finished later by the chunk kernel, arrive through
 * mapped pinned memory and overwrite their stale copies before the call
 * returns. Device and pinned staging buffers are kept per calling thread
 * and device between calls. */
cmfw_status cmfw_walk_host(cmfw_variant variant, const cmfw_desc *desc, const cmfw_traj_in *h_in,
                           cmfw_traj_out *h_out, int n_traj, int N, int h, int n_primes,
                           const cmfw_launch *launch, float *kernel_ms, float *total_ms);

/* Device properties line for the programs' stderr banner. */
cmfw_status cmfw_device_banner(char *buf, size_t size);
/* Measured FMA throughput of one pipe on the current device, in tera-ops
 * per second (an FMA counts 2): pipe 0 = FP64, 1 = FP32, 2 = INT32 IMAD.
 * The roofline denominator for the walk kernels. Synchronises. */
cmfw_status cmfw_pipe_peak(int pipe, double *tera_ops_per_s);
/* cudaMemGetInfo of the current device (device-wide, all processes). */
cmfw_status cmfw_device_meminfo(size_t *free_bytes, size_t *total_bytes);

#ifdef __cplusplus
}
#endif
#endif /* CMFW_H */
