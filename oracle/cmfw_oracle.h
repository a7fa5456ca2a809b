/* CPU oracle for the pFq Conservative Matrix Field walk.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference
 * algorithm (VesterlundCoder/RamanujanDreams-CUDA, cuda/cmf_pfq.cuh and
 * cuda/cmf_walk_{f64,df64,rns}.cu), used by tests/, by the smoke check and by
 * the CPU-baseline leg of bench.py as the thing results are checked against.
 * The product library never links or calls it.
 *
 * Pinning: with the default (unfused) rounding mode every function here is
 * bitwise identical to the reference's own kernel bodies compiled for the
 * host (oracle/_ref, built by `make ref`), and the f64 rows agree with the
 * reference's published H100 results (tests/golden) within the tolerances the
 * tests state.
 *
 * Record layouts match the reference byte for byte:
 *   orc_in       == TrajectoryInput / DF64Input / RNSInput (192 bytes)
 *   orc_out_f64  == TrajectoryResult (64 bytes)
 *   orc_out      == DF64Result / RNSResult (56 bytes)
 */
#ifndef CMFW_ORACLE_H
#define CMFW_ORACLE_H
#include <stdint.h>

#define ORC_MAX_DIM 8
#define ORC_MAX_AXES 16
#define ORC_MAX_PRIMES 64

typedef struct { int p, q, rank, naxes; double z; } orc_desc;
typedef struct { int dir[ORC_MAX_AXES]; double start[ORC_MAX_AXES]; } orc_in;
typedef struct {
    double limit, delta, p, q, precision, log_scale;
    int valid, n_limits;
    double elapsed_ms;
} orc_out_f64;
typedef struct {
    double limit, delta, p, q, precision, log_scale;
    int valid, n_limits;
} orc_out;

orc_desc orc_make_desc(int p, int q, double z);

/* mode 0 = limit, 1 = delta; writes n records into buf (zeroed by caller). */
void orc_make_inputs(int p, int q, int n, int mode, int use_zeta, void *buf);
void orc_mt64_stream(uint64_t seed, uint64_t *out, int n);

/* Per-trajectory walks. `fused` = 1 evaluates the companion-polynomial
 * products with fused multiply-adds (the form an FMA-contracting compiler
 * emits); 0 rounds every product and sum separately. threads <= 0: all. */
int orc_walk_f64(int p, int q, double z, int N, int h, const orc_in *in,
                 orc_out_f64 *out, int n, int fused, int threads);
/* orc_walk_f64 plus each row's limit source in limit_src (n ints):
 * (method << 12) | (i << 8) | (j << 4) | c for the ratio M[i][c] / M[j][c]
 * the limit came from (method 1 = Aitken, 0 = raw), -1 when none. */
int orc_walk_f64_src(int p, int q, double z, int N, int h, const orc_in *in,
                     orc_out_f64 *out, int n, int fused, int threads, int *limit_src);
int orc_walk_df64(int p, int q, double z, int N, int h, const orc_in *in,
                  orc_out *out, int n, int fused, int threads);
int orc_walk_rns(int p, int q, double z, int N, int h, const orc_in *in,
                 orc_out *out, int n, int n_primes, int fused, int threads);

/* Snapshot matrices (3 x 8 x 8 doubles, row-major) and log-scales. */
int orc_f64_snapshots(int p, int q, double z, int N, int h, const int *dir,
                      const double *start, int fused, double *m123, double *ls123);
/* Residues after `steps` steps, n_primes * rank * rank (prime-major). */
int orc_rns_trace(int p, int q, double z, int N, int h, const int *dir,
                  const double *start, int n_primes, int steps, int fused,
                  uint32_t *out, double *log_scale_out);
void orc_rns_moduli(uint32_t *out, int n);

/* Exact walk modulo primes (odd, below 2^31), z = zn / zd: residues of the
 * entries (i, c) and (j, c) of the walk matrix at depths N-2h, N-h, N, with
 * (i, j, c) from pairs[t] = (i << 8) | (j << 4) | c (NULL or -1: 0, 1,
 * rank-1). res: n * 3 * 2 * K, index ((t * 3 + depth) * 2 + entry) * K + k;
 * ok: n * K, 0 where a divisor vanished modulo that prime. */
int orc_exact_residues(int p, int q, long long zn, long long zd, int N, int h,
                       const orc_in *in, int n, const uint32_t *primes, int K,
                       const int *pairs, uint32_t *res, uint8_t *ok, int threads);

/* Companion column at a position (for kernel-level checks). */
int orc_column(const double *pos, double z, int dim, int p, int q,
               double *col, int fused);

#endif
