// C entry points over the reference's own kernel bodies, compiled for the
// host. Test infrastructure only (a checker for oracle/cmfw_oracle.c and a
// timed CPU baseline); never linked into the product.
//
// The `ref` target of oracle/Makefile compiles this file three times, once per reference variant,
// after copying cuda/cmf_walk_<variant>.cu with its `<<<grid, block>>>`
// launch brackets removed (the only construct a host compiler rejects).
// REF_SRC names that processed copy; REF_F64 / REF_DF64 / REF_RNS selects the
// variant. Each build is its own shared object, because the three reference
// programs define the same helper names.
//
// Every kernel body reads idx = blockIdx.x * blockDim.x + threadIdx.x, so the
// loops below set blockIdx.x = i, blockDim.x = 1, threadIdx.x = 0 on the
// calling thread and invoke the body once per trajectory (OpenMP, dynamic
// schedule, as the reference's CPU baseline plan describes).
#include "cuda_runtime.h"

thread_local ref_dim3 blockIdx = {0, 1, 1};
thread_local ref_dim3 blockDim = {1, 1, 1};
thread_local ref_dim3 threadIdx = {0, 0, 0};

#include REF_SRC

#include <omp.h>

#if defined(REF_F64)
typedef TrajectoryInput RefIn;
typedef TrajectoryResult RefOut;
#define REF_PREFIX(x) ref_f64_##x
#elif defined(REF_DF64)
typedef DF64Input RefIn;
typedef DF64Result RefOut;
#define REF_PREFIX(x) ref_df64_##x
#elif defined(REF_RNS)
typedef RNSInput RefIn;
typedef RNSResult RefOut;
#define REF_PREFIX(x) ref_rns_##x
#else
#error "define one of REF_F64, REF_DF64, REF_RNS"
#endif

static inline void ref_set_index(int i) {
    blockIdx.x = (unsigned)i;
    blockDim.x = 1;
    threadIdx.x = 0;
}

extern "C" {

int REF_PREFIX(sizeof_input)(void) { return (int)sizeof(RefIn); }
int REF_PREFIX(sizeof_result)(void) { return (int)sizeof(RefOut); }

// Builds the n_traj input records exactly as run_benchmark() does
// (cmf_walk_f64.cu:166-199, cmf_walk_df64.cu:375-395, cmf_walk_rns.cu:346-366),
// including the generators' 128-byte / 64-byte write strides over the
// 192-byte records. `buf` must hold n * sizeof_input() zeroed bytes.
void REF_PREFIX(make_inputs)(int p, int q, int n, int mode, int use_zeta, void *buf) {
    RefIn *in = (RefIn *)buf;
    if (mode == 0) {
        if (use_zeta) {
            Position zs = zeta_initial_point(p, q);
            // zeta_initial_point leaves v[p+q..] unset; pin those unused bytes.
            for (int a = p + q; a < MAX_AXES; ++a) zs.v[a] = 0.0;
            for (int i = 0; i < n; ++i) in[i].start = zs;
        } else {
            generate_initial_points(p, q, n, (Position *)buf, 42);
        }
        for (int i = 0; i < n; ++i) {
            memset(in[i].dir, 0, sizeof(in[i].dir));
            in[i].dir[0] = 1;
        }
    } else {
        Position fs;
        memset(&fs, 0, sizeof(fs));
        if (use_zeta) {
            fs = zeta_initial_point(p, q);
            for (int a = p + q; a < MAX_AXES; ++a) fs.v[a] = 0.0;
        } else {
            for (int a = 0; a < p + q; ++a) fs.v[a] = (a < p) ? 2.0 : 3.0;
        }
        for (int i = 0; i < n; ++i) in[i].start = fs;
        generate_trajectories(p, q, n, (int *)buf, 42);
    }
}

// Runs the variant's kernel body for every index in [0, n).
// threads <= 0 means "all OpenMP threads".
int REF_PREFIX(walk)(int p, int q, double z, int N, int h, const void *inputs,
                     void *results, int n, int n_primes, int threads) {
    CMFDesc desc = make_cmf_desc(p, q, z);
    const RefIn *in = (const RefIn *)inputs;
    RefOut *out = (RefOut *)results;
    if (threads > 0) omp_set_num_threads(threads);
    (void)n_primes;
#pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < n; ++i) {
        ref_set_index(i);
#if defined(REF_RNS)
        walk_kernel_rns(in, out, desc, N, h, n, n_primes);
#elif defined(REF_DF64)
        walk_kernel_df64(in, out, desc, N, h, n);
#else
        walk_kernel_f64(in, out, desc, N, h, n);
#endif
    }
    return 0;
}

#if defined(REF_F64)
// The three snapshot matrices of forward_walk (cmf_pfq.cuh:348-371),
// each as 64 doubles (MAX_DIM x MAX_DIM, row-major), and their log-scales.
int ref_f64_snapshots(int p, int q, double z, int N, int h, const int *dir,
                      const double *start, double *m123, double *ls123) {
    CMFDesc desc = make_cmf_desc(p, q, z);
    int d[MAX_AXES];
    Position s;
    for (int a = 0; a < MAX_AXES; ++a) { d[a] = dir[a]; s.v[a] = start[a]; }
    WalkSnapshots snaps;
    memset(&snaps, 0, sizeof(snaps));
    bool ok = forward_walk(d, s, desc, N, h, snaps);
    const WalkMatrix *ms[3] = {&snaps.m1, &snaps.m2, &snaps.m3};
    for (int k = 0; k < 3; ++k)
        for (int i = 0; i < MAX_DIM; ++i)
            for (int j = 0; j < MAX_DIM; ++j) m123[k * 64 + i * 8 + j] = ms[k]->a[i][j];
    ls123[0] = snaps.log_scale1;
    ls123[1] = snaps.log_scale2;
    ls123[2] = snaps.log_scale3;
    return ok ? 1 : 0;
}
#endif

#if defined(REF_RNS)
// Residue matrix after `steps` trajectory steps, following the loop of
// walk_kernel_rns (cmf_walk_rns.cu:267-298): identity start, one
// apply_trajectory_step_rns per step, and the CRT / normalise / re-reduce
// pass at every 100th step and at the snapshot steps N-2h, N-h, N.
// out: n_primes * rank * rank residues (prime-major, row-major).
int ref_rns_trace(int p, int q, double z, int N, int h, const int *dir,
                  const double *start, int n_primes, int steps,
                  uint32_t *out, double *log_scale_out) {
    CMFDesc desc = make_cmf_desc(p, q, z);
    static thread_local RNSMatrix walk;
    walk.dim = desc.rank;
    for (int k = 0; k < n_primes; ++k)
        for (int i = 0; i < walk.dim; ++i)
            for (int j = 0; j < walk.dim; ++j) walk.a[k][i][j] = (i == j) ? 1 : 0;
    int d[MAX_AXES];
    Position pos;
    for (int a = 0; a < MAX_AXES; ++a) { d[a] = dir[a]; pos.v[a] = start[a]; }
    int cp1 = N - 2 * h, cp2 = N - h;
    double log_scale = 0.0;
    int ok = 1;
    for (int step = 1; step <= steps; ++step) {
        if (!apply_trajectory_step_rns(walk, pos, d, desc, n_primes)) { ok = 0; break; }
        if (step % 100 == 0 || step == cp1 || step == cp2 || step == N) {
            WalkMatrix wm;
            rns_to_double(walk, wm, n_primes, log_scale);
            for (int k = 0; k < n_primes; ++k) {
                uint32_t pk = RNS_PRIMES[k];
                for (int i = 0; i < walk.dim; ++i)
                    for (int j = 0; j < walk.dim; ++j) walk.a[k][i][j] = to_mod(wm.a[i][j], pk);
            }
        }
    }
    for (int k = 0; k < n_primes; ++k)
        for (int i = 0; i < walk.dim; ++i)
            for (int j = 0; j < walk.dim; ++j)
                out[(k * walk.dim + i) * walk.dim + j] = walk.a[k][i][j];
    *log_scale_out = log_scale;
    return ok;
}

void ref_rns_primes(uint32_t *out, int n) {
    for (int k = 0; k < n && k < MAX_PRIMES; ++k) out[k] = RNS_PRIMES[k];
}
#endif

}  // extern "C"
