// Learned trajectory proposal: a 4-layer MLP (64 -> 256 -> 256 -> 256 -> 1,
// ReLU) over a trajectory's direction and CMF family, trained on walk
// results by this file's kernels and used to rank candidate directions.
//
// The three dense layers run on the 5th-generation tensor cores:
// gemm_bf16_kernel computes C = epilogue(A * B^T) for BF16 K-major operands
// with tcgen05.mma (M = 128 rows per CTA, N = 64/128/256), the FP32
// accumulator in tensor memory, operands staged in shared memory through a
// four-stage cp.async ring in the interleaved canonical layout
// (tc_sm100.cuh), and the epilogue (bias + ReLU + BF16 rounding, or the
// ReLU-derivative mask of the backward pass, or FP32 out) fused after the
// tcgen05.ld of the accumulator. Forward:  Z = X W^T (A = activations,
// B = W stored [out x in]). Backward: dX = dZ W (B = W^T stored [in x out]),
// dW = dZ^T X (A = dZ^T, B = X^T, both transposed by transpose_bf16_kernel).
// The 256 -> 1 head, the loss, bias gradients and Adam are CUDA-core kernels.
//
// Inputs: features(t) = direction_features (candidates.cuh: counts of the
// x and y components by magnitude, signs, one-hot(family) over 5) padded
// with zeros to 64 BF16 values. Parameters are FP32 masters with BF16 copies for the
// tensor cores (W and W^T).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <cuda_bf16.h>
#include <map>
#include <vector>

#include "cmfw.h"
#include "candidates.cuh"
#include "cmfw_internal.cuh"
#include "tc_sm100.cuh"

#include <cooperative_groups.h>
namespace cg = cooperative_groups;

namespace cmfw {
cmfw_status record_error(cmfw_status s, const char *msg);

constexpr int kIn = CMFW_MLP_IN;       // 64
constexpr int kHid = CMFW_MLP_HIDDEN;  // 256
constexpr int kBK = 64;                // K per pipeline stage

enum { EPI_BIAS_RELU_BF16 = 0, EPI_F32 = 1, EPI_MASK_BF16 = 2 };

struct GemmArgs {
    const __nv_bfloat16 *A;  // M x K, row stride lda
    const __nv_bfloat16 *B;  // N x K, row stride ldb
    int M, N, K, lda, ldb;
    void *C;  // M x N, row stride ldc (bf16 or f32)
    int ldc;
    const float *bias;           // EPI_BIAS_RELU_BF16: N
    const __nv_bfloat16 *mask;   // EPI_MASK_BF16: M x N, row stride ldc; C = acc where mask > 0
    int *err;
    int ksplit;                  // CTAs along K (gridDim.z); EPI_F32 only, else 1
    float *part;                 // EPI_F32: the splits' partial sums, [ksplit][M][N]
};

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// One 64-wide K chunk of a ROWS x K operand into an interleaved tile.
template <int ROWS>
__device__ __forceinline__ void load_chunk(uint32_t tile, const __nv_bfloat16 *src, int ld, int row0, int k0) {
#pragma unroll
    for (int i = threadIdx.x; i < ROWS * 8; i += 128) {
        const int r = i >> 3, c = i & 7;
        cp_async16(tile + (uint32_t)((r >> 3) * 1024 + c * 128 + (r & 7) * 16),
                   src + (size_t)(row0 + r) * ld + k0 + c * 8);
    }
}

// Stages of the operand ring: the loads of up to kStages - 1 chunks are in
// flight while the MMAs of the current one run; the 128 x 256 tiles keep
// two stages (98 KB, two CTAs per SM).
template <int BN>
__host__ __device__ constexpr int gemm_stages() { return BN >= 256 ? 2 : 4; }

template <int BN, int EPI>
__global__ void __launch_bounds__(128) gemm_bf16_kernel(GemmArgs g) {
    constexpr int kStages = gemm_stages<BN>();
    constexpr int A_BYTES = 128 * kBK * 2;
    constexpr int B_BYTES = BN * kBK * 2;
    constexpr int STAGE = A_BYTES + B_BYTES;
    constexpr uint32_t TCOLS = BN < 32 ? 32 : BN;
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ uint64_t bar[kStages];
    __shared__ uint32_t tmem_base;
    __shared__ int s_bad;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m0 = blockIdx.y * 128, n0 = blockIdx.x * BN;
    // this CTA's K chunks: [kc0, kc0 + nk) of the K / kBK, split evenly over gridDim.z
    const int nchunks = g.K / kBK;
    const int kc0 = (int)((long long)blockIdx.z * nchunks / gridDim.z);
    const int nk = (int)((long long)(blockIdx.z + 1) * nchunks / gridDim.z) - kc0;
    const uint32_t sbase = tc::smem_u32(smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int i = 0; i < kStages; ++i) tc::mbar_init(&bar[i], 1);
        s_bad = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(&tmem_base, TCOLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, BN);
    bool ok = true;

    // prologue: chunks 0 .. kStages - 2, one commit group each (empty past nk)
#pragma unroll
    for (int i = 0; i < kStages - 1; ++i) {
        if (i < nk) {
            const uint32_t st = sbase + (uint32_t)(i * STAGE);
            load_chunk<128>(st, g.A, g.lda, m0, (kc0 + i) * kBK);
            load_chunk<BN>(st + A_BYTES, g.B, g.ldb, n0, (kc0 + i) * kBK);
        }
        cp_async_commit();
    }
    for (int kc = 0; kc < nk; ++kc) {
        const int s = kc % kStages;
        // chunk kc + kStages - 1 goes to the stage that the MMAs of chunk
        // kc - 1 read: wait for their commit first
        const int nxt = kc + kStages - 1;
        if (nxt < nk) {
            const int sn = nxt % kStages;
            if (kc >= 1 && !tc::mbar_wait(&bar[sn], ((kc - 1) / kStages) & 1)) ok = false;
            const uint32_t st = sbase + (uint32_t)(sn * STAGE);
            load_chunk<128>(st, g.A, g.lda, m0, (kc0 + nxt) * kBK);
            load_chunk<BN>(st + A_BYTES, g.B, g.ldb, n0, (kc0 + nxt) * kBK);
        }
        cp_async_commit();
        cp_async_wait<kStages - 1>();  // chunk kc's group is complete
        tc::fence_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            tc::fence_after_sync();
            const uint32_t a = sbase + (uint32_t)(s * STAGE), b = a + A_BYTES;
#pragma unroll
            for (int j = 0; j < kBK / 16; ++j)
                tc::mma_bf16(tmem, tc::smem_desc(a + j * 256, 128, 1024), tc::smem_desc(b + j * 256, 128, 1024),
                             idesc, kc > 0 || j > 0);
            tc::commit(&bar[s]);
        }
    }
    // the last commit covers every earlier MMA of this thread
    const int sl = (nk - 1) % kStages, pl = ((nk - 1) / kStages) & 1;
    if (!tc::mbar_wait(&bar[sl], pl)) {
        ok = false;
        tc::mbar_wait(&bar[sl], pl);  // one more bounded wait before freeing TMEM
    }
    if (!ok) s_bad = 1;
    __syncthreads();
    tc::fence_after_sync();
    if (s_bad) {
        if (threadIdx.x == 0) atomicExch(g.err, 1);
    } else {
        const int row = m0 + warp * 32 + lane;
        for (int c0 = 0; c0 < BN; c0 += 32) {
            float v[32];
            tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
            const int col = n0 + c0;
            if (EPI == EPI_F32) {
                // this split's partial sums; sum_parts_kernel adds the
                // splits in order into C (the same bits on every run)
                float *dst = g.part + ((size_t)blockIdx.z * g.M + row) * g.N + col;
#pragma unroll
                for (int i = 0; i < 32; i += 4) *(float4 *)(dst + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
            } else {
                __nv_bfloat16 *dst = (__nv_bfloat16 *)g.C + (size_t)row * g.ldc + col;
                if (EPI == EPI_BIAS_RELU_BF16) {
#pragma unroll
                    for (int i = 0; i < 32; ++i) v[i] = fmaxf(v[i] + g.bias[col + i], 0.0f);
                } else {
                    const __nv_bfloat16 *mk = g.mask + (size_t)row * g.ldc + col;
#pragma unroll
                    for (int i = 0; i < 32; ++i) v[i] = __bfloat162float(mk[i]) > 0.0f ? v[i] : 0.0f;
                }
#pragma unroll
                for (int i = 0; i < 32; i += 8) {
                    __nv_bfloat162 h[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) h[j] = __floats2bfloat162_rn(v[i + 2 * j], v[i + 2 * j + 1]);
                    *(uint4 *)(dst + i) = *(uint4 *)h;
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, TCOLS);
}

template <int BN, int EPI>
static cudaError_t gemm_launch(const GemmArgs &g, cudaStream_t s) {
    constexpr int smem = gemm_stages<BN>() * (128 * kBK * 2 + BN * kBK * 2) + 1024;
    cudaError_t e = cudaFuncSetAttribute((const void *)gemm_bf16_kernel<BN, EPI>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    dim3 grid(g.N / BN, g.M / 128, g.ksplit);
    gemm_bf16_kernel<BN, EPI><<<grid, 128, smem, s>>>(g);
    return cudaGetLastError();
}

// SMs of the current device (queried once per device).
static int gemm_sms() {
    static int sms_of[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return 148;
    }
    if (sms_of[dev] == 0) {
        int sms = 148;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
            cudaGetLastError();
            sms = 148;
        }
        sms_of[dev] = sms;
    }
    return sms_of[dev];
}

// Host-side shape rules: M % 128, K % 64, N % 64 == 0; 16-byte aligned rows.
// Tiles: 128 x 256 when that gives a full wave of CTAs (large M), else
// 128 x 64, so that the training batches' GEMMs (M of a few thousand
// rows, or 256 for dW) spread over more SMs. EPI_F32 (the weight
// gradients, K = the batch) also splits K over up to kMaxSplit CTAs, each
// writing its partial sums to g.part; *ksplit_out says how many, for the
// fixed-order sum that forms C.
constexpr int kMaxSplit = 16;
static cudaError_t gemm(GemmArgs g, int epi, cudaStream_t s, int *ksplit_out = nullptr) {
    if (g.M % 128 || g.K % kBK || g.N % 64 || g.M <= 0 || g.N <= 0 || g.K <= 0) return cudaErrorInvalidValue;
    if (epi == EPI_F32 && !g.part) return cudaErrorInvalidValue;
    const int sms = gemm_sms();
    const bool n256 = g.N % 256 == 0 && (long long)(g.M / 128) * (g.N / 256) >= sms;
    g.ksplit = 1;
    if (epi == EPI_F32) {
        const int tiles = (g.M / 128) * (g.N / (n256 ? 256 : 64));
        const int nchunks = g.K / kBK;
        while (g.ksplit < kMaxSplit && tiles * g.ksplit * 2 <= sms && 2 * g.ksplit * 2 <= nchunks) g.ksplit *= 2;
    }
    if (ksplit_out) *ksplit_out = g.ksplit;
    if (epi == EPI_BIAS_RELU_BF16) return n256 ? gemm_launch<256, EPI_BIAS_RELU_BF16>(g, s)
                                              : gemm_launch<64, EPI_BIAS_RELU_BF16>(g, s);
    if (epi == EPI_MASK_BF16) return n256 ? gemm_launch<256, EPI_MASK_BF16>(g, s) : gemm_launch<64, EPI_MASK_BF16>(g, s);
    return n256 ? gemm_launch<256, EPI_F32>(g, s) : gemm_launch<64, EPI_F32>(g, s);
}

// ---- CUDA-core kernels ------------------------------------------------------

// Features (direction_features) of n trajectories into X [n_pad x 64] bf16
// (rows >= n zero): trajectory idx[t] (t without idx) in row t. Its family
// is family[idx[t]]; its axes are the family's p + q.
__global__ void features_kernel(const cmfw_traj_in *in, const int *family, const long long *idx, int n, int n_pad,
                                __nv_bfloat16 *X) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pad * kIn) return;
    const int t = i / kIn, c = i % kIn;
    float v = 0.0f;
    if (t < n && c < 20) {
        const long long j = idx ? idx[t] : t;  // row t of the batch is trajectory j
        const int fam = family[j];
        const int p = family_p(fam);
        const cmfw_traj_in &r = in[j];
        float f[20];
        direction_features([&](int a) { return r.dir[a]; }, p + (p - 1), fam, f);
        v = f[c];
    }
    X[i] = __float2bfloat16_rn(v);
}

__global__ void candidate_features_kernel(uint64_t seed, long long first, int n, int n_pad, int naxes, int lo,
                                          int hi, int family, __nv_bfloat16 *X) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pad * kIn) return;
    const int t = i / kIn, c = i % kIn;
    float v = 0.0f;
    if (t < n && c < 20) {
        int comp[16];
        candidate_direction(seed, first + t, lo, SmallMod((uint32_t)(hi - lo + 1)), comp);
        float f[20];
        direction_features([&](int a) { return comp[a]; }, naxes, family, f);
        v = f[c];
    }
    X[i] = __float2bfloat16_rn(v);
}

__global__ void candidate_records_kernel(uint64_t seed, const long long *idx, int n, int naxes, int lo, int hi,
                                         const double *start, cmfw_traj_in *out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    int comp[16];
    candidate_direction(seed, idx[t], lo, SmallMod((uint32_t)(hi - lo + 1)), comp);
    cmfw_traj_in r;
    for (int a = 0; a < CMFW_MAX_AXES; ++a) {
        r.dir[a] = a < naxes ? comp[a] : 0;
        r.start[a] = a < naxes ? start[a] : 0.0;
    }
    out[t] = r;
}

// score[t] = H3[t] . w4 + b4, one warp per row.
__global__ void head_forward_kernel(const __nv_bfloat16 *H, const float *w4, const float *b4, int n, float *score) {
    const int row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    float s = 0.0f;
    for (int k = lane; k < kHid; k += 32) s = fmaf(__bfloat162float(H[(size_t)row * kHid + k]), w4[k], s);
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) score[row] = s + b4[0];
}

// Weighted squared error: loss = sum w (s - y)^2 / sum w, dscore = dloss/ds.
// Weighted MSE of row t against target y[j], weight w[j] (j = idx[t], or
// t), over the weight sum (*d_wsum when given, else wsum). Each block
// (256 threads, a grid of at most kMaxRowBlocks striding over the rows)
// writes its share of the loss to lpart[blockIdx.x], summed in a fixed
// order (warp shuffles, then the warps in order).
constexpr int kMaxRowBlocks = 512;
__global__ void loss_kernel(const float *score, const float *y, const float *w, const long long *idx, int n,
                            float wsum, const float *d_wsum, float *dscore, float *lpart) {
    __shared__ float wl[8];
    const float ws = d_wsum ? *d_wsum : wsum;
    float l = 0.0f;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const long long j = idx ? idx[t] : t;
        const float r = score[t] - y[j];
        const float wt = w ? w[j] : 1.0f;
        dscore[t] = 2.0f * wt * r / ws;
        l += wt * r * r / ws;
    }
    for (int o = 16; o; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) wl[threadIdx.x >> 5] = l;
    __syncthreads();
    if (threadIdx.x == 0) {
        float b = 0.0f;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) b += wl[i];
        lpart[blockIdx.x] = b;
    }
}

// dZ3 = (dscore w4^T) o [H3 > 0]; this row block's shares of gw4 = dscore^T
// H3 and gb4 = sum dscore into pw4[blockIdx.x][256] and pb4[blockIdx.x].
__global__ void head_backward_kernel(const __nv_bfloat16 *H, const float *w4, const float *dscore, int n,
                                     __nv_bfloat16 *dZ, float *pw4, float *pb4) {
    const int k = threadIdx.x;  // 256 threads: one hidden unit each
    const int rows = (n + gridDim.x - 1) / gridDim.x;
    const int r0 = blockIdx.x * rows, r1 = min(n, r0 + rows);
    float acc = 0.0f, bacc = 0.0f;
    for (int r = r0; r < r1; ++r) {
        const float h = __bfloat162float(H[(size_t)r * kHid + k]);
        const float d = dscore[r];
        acc = fmaf(d, h, acc);
        bacc += d;
        dZ[(size_t)r * kHid + k] = __float2bfloat16_rn(h > 0.0f ? d * w4[k] : 0.0f);
    }
    pw4[(size_t)blockIdx.x * kHid + k] = acc;
    if (k == 0) pb4[blockIdx.x] = bacc;
}

// Column sums of a [n x cols] bf16 matrix: row block blockIdx.y's sums into
// part[blockIdx.y][cols].
__global__ void colsum_kernel(const __nv_bfloat16 *Z, int n, int cols, float *part) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    const int rows = (n + gridDim.y - 1) / gridDim.y;
    const int r0 = blockIdx.y * rows, r1 = min(n, r0 + rows);
    float s = 0.0f;
    for (int r = r0; r < r1; ++r) s += __bfloat162float(Z[(size_t)r * cols + c]);
    part[(size_t)blockIdx.y * cols + c] = s;
}

// Fixed-order sums of partial results: task k writes dst[j] = sum over z
// in order of part[z * pstride + j], j < n. Every gradient and the loss go
// through here, so a batch trains to the same bits on every run.
struct SumTask {
    const float *part;
    float *dst;
    int n, nparts, pstride;
};
struct SumTable {
    SumTask t[9];
    int ntask;
    int start[10];  // prefix sums of the tasks' n
};
__global__ void sum_parts_kernel(SumTable T) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.start[T.ntask]) return;
    int k = 0;
    while (i >= T.start[k + 1]) ++k;
    const SumTask &t = T.t[k];
    const int j = i - T.start[k];
    float s = 0.0f;
    for (int z = 0; z < t.nparts; ++z) s += t.part[(size_t)z * t.pstride + j];
    t.dst[j] = s;
}

// out[c][r] = in[r][c] for a rows x cols bf16 matrix (32 x 32 tiles).
__global__ void transpose_bf16_kernel(const __nv_bfloat16 *in, int rows, int cols, __nv_bfloat16 *out) {
    __shared__ __nv_bfloat16 tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = by + j, c = bx + threadIdx.x;
        if (r < rows && c < cols) tile[j][threadIdx.x] = in[(size_t)r * cols + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int c = bx + j, r = by + threadIdx.x;
        if (r < rows && c < cols) out[(size_t)c * rows + r] = tile[threadIdx.x][j];
    }
}

// *out = sum of w[idx[t]] (t < n; w NULL: n), one block.
__global__ void weight_sum_kernel(const float *w, const long long *idx, int n, float *out) {
    __shared__ float part[32];
    float s = 0.0f;
    for (int t = threadIdx.x; t < n; t += blockDim.x) s += w ? w[idx[t]] : 1.0f;
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (int)(blockDim.x >> 5) ? part[threadIdx.x] : 0.0f;
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) *out = s;
    }
}

// Adam (beta1 0.9, beta2 0.999, eps 1e-8) on the FP32 masters of all eight
// parameter tensors in one launch; refreshes the BF16 copies W [rows x
// cols] and W^T [cols x rows] of the tensors that have them.
struct AdamTable {
    float *p[8], *m[8], *v[8];
    const float *g[8];
    __nv_bfloat16 *W[8], *WT[8];
    int rows[8], cols[8];
    int off[9];  // prefix sums of the tensors' sizes
};

__global__ void adam_all_kernel(AdamTable T, float lr, float bc1, float bc2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= T.off[8]) return;
    int s = 0;
#pragma unroll
    for (int k = 1; k < 8; ++k) s += (i >= T.off[k]) ? 1 : 0;
    const int e = i - T.off[s];
    const float gi = T.g[s][e];
    const float mi = 0.9f * T.m[s][e] + 0.1f * gi;
    const float vi = 0.999f * T.v[s][e] + 0.001f * gi * gi;
    T.m[s][e] = mi;
    T.v[s][e] = vi;
    const float pi = T.p[s][e] - lr * (mi / bc1) / (sqrtf(vi / bc2) + 1e-8f);
    T.p[s][e] = pi;
    if (T.W[s]) {
        const __nv_bfloat16 b = __float2bfloat16_rn(pi);
        T.W[s][e] = b;
        if (T.WT[s]) T.WT[s][(size_t)(e % T.cols[s]) * T.rows[s] + e / T.cols[s]] = b;
    }
}

__global__ void to_bf16_kernel(const float *p, int n, int rows, int cols, __nv_bfloat16 *W, __nv_bfloat16 *WT) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const __nv_bfloat16 b = __float2bfloat16_rn(p[i]);
    W[i] = b;
    if (WT) WT[(size_t)(i % cols) * rows + i / cols] = b;
}

// Order-preserving key of a float score (larger score -> larger key).
__device__ __forceinline__ uint32_t score_key(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Selection key of score i (n < 2^32): the score's key above the index's
// complement, so keys are distinct and order by score, then by lower index.
__device__ __forceinline__ uint64_t select_key(const float *score, long long i) {
    return ((uint64_t)score_key(score[i]) << 32) | (uint64_t)(0xFFFFFFFFu - (uint32_t)i);
}

// Histogram of the selection keys that match prefix under prefix_mask, by
// their `bits` bits above `shift` (bits <= 11).
__global__ void score_hist_kernel(const float *score, long long n, uint32_t shift, uint32_t bits, uint64_t prefix,
                                  uint64_t prefix_mask, unsigned long long *hist) {
    __shared__ unsigned int h[2048];
    for (int i = threadIdx.x; i < 2048; i += blockDim.x) h[i] = 0;
    __syncthreads();
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const uint64_t k = select_key(score, i);
        if ((k & prefix_mask) == prefix) atomicAdd(&h[(uint32_t)(k >> shift) & ((1u << bits) - 1u)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 2048; i += blockDim.x)
        if (h[i]) atomicAdd(&hist[i], (unsigned long long)h[i]);
}

__global__ void select_kernel(const float *score, long long n, uint64_t kmin, long long *out, int cap,
                              int *count) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (select_key(score, i) >= kmin) {
            const int pos = atomicAdd(count, 1);
            if (pos < cap) out[pos] = i;
        }
    }
}

// ---- fused scoring ----------------------------------------------------------
//
// Scoring a large candidate set in one launch: clusters of two CTAs stride
// over 128-candidate tiles. CTA r of a cluster owns hidden features
// [128 r, 128 r + 128) of every layer and keeps its halves of W1, W2, W3
// (16 + 64 + 64 KB, interleaved K-major) in shared memory for the whole
// launch, so weights are read from HBM once per CTA. Per tile: the
// candidates' features are generated in place (no records), then per layer
// one thread issues the M = 128, N = 128 tcgen05 MMAs into a 128-column TMEM
// accumulator; after the cluster barrier that ends both CTAs' MMAs, 256
// threads load the accumulator, add the bias, apply ReLU, round to BF16 and
// write their half of the activations into both CTAs' activation tiles
// (the peer's through distributed shared memory); a second barrier makes the
// tile complete on both sides. The head's 256-term dot product is split the
// same way and summed in CTA 0.

struct FusedArgs {
    const __nv_bfloat16 *W[3];  // [256 x 64], [256 x 256], [256 x 256] row-major
    const float *bias[3];       // 256 each
    const float *w4, *b4;
    uint64_t seed;
    long long first, n;
    const long long *idx;  // optional: score candidates idx[0..n) instead of first .. first+n-1
    int naxes, lo, hi, family;
    float *score;
    int *err;
};

constexpr int kFusedSmem = 16384 + 65536 + 65536 + 65536 + 4 * 128 * 4 + 4 * 128 * 4;

__device__ __forceinline__ void fence_async_cluster() {
    asm volatile("fence.proxy.async.shared::cluster;" ::: "memory");
}

// Rows [row0, row0 + rows) of a row-major [* x K] bf16 matrix into an
// interleaved K-major tile.
__device__ __forceinline__ void load_tile(unsigned char *dst, const __nv_bfloat16 *src, int row0, int rows, int K) {
    const int chunks = rows * (K / 8);
    for (int i = threadIdx.x; i < chunks; i += blockDim.x) {
        const int r = i / (K / 8), c = i % (K / 8);
        *(uint4 *)(dst + tc::tile_offset(r, c * 8, K)) = *(const uint4 *)(src + (size_t)(row0 + r) * K + c * 8);
    }
}

// Eight consecutive activations (columns k .. k+7 of one row) as a 16-byte chunk.
__device__ __forceinline__ uint4 pack8(const float *v) {
    __nv_bfloat162 h[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) h[j] = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
    return *(uint4 *)h;
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(256) mlp_score_fused_kernel(FusedArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *w1 = smem;                 // 128 x 64
    unsigned char *w2 = w1 + 16384;           // 128 x 256
    unsigned char *w3 = w2 + 65536;           // 128 x 256
    unsigned char *act = w3 + 65536;          // 128 x 256 (128 x 64 for the features)
    float *sbias = (float *)(act + 65536);    // 3 x 128 biases, then 128 of w4
    // head partial sums: [0, 256) per column half, [256, 384) this CTA's
    // half (CTA 0), [384, 512) CTA 1's half (written by CTA 1)
    float *spart = sbias + 4 * 128;
    __shared__ uint64_t bar;
    __shared__ uint32_t tmem_base;
    __shared__ int s_bad;
    cg::cluster_group cluster = cg::this_cluster();
    const int r = (int)cluster.block_rank();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char *peer_act = cluster.map_shared_rank(act, r ^ 1);
    float *peer_part0 = cluster.map_shared_rank(spart, 0);

    // resident weights and biases of this CTA's half
    load_tile(w1, a.W[0], 128 * r, 128, kIn);
    load_tile(w2, a.W[1], 128 * r, 128, kHid);
    load_tile(w3, a.W[2], 128 * r, 128, kHid);
    for (int i = threadIdx.x; i < 128; i += blockDim.x) {
        for (int l = 0; l < 3; ++l) sbias[l * 128 + i] = a.bias[l][128 * r + i];
        sbias[3 * 128 + i] = a.w4[128 * r + i];
    }
    if (threadIdx.x == 0) {
        tc::mbar_init(&bar, 1);
        s_bad = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(&tmem_base, 128);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    constexpr uint32_t idesc = tc::idesc_bf16_f32(128, 128);
    const uint32_t s_act = tc::smem_u32(act), s_w[3] = {tc::smem_u32(w1), tc::smem_u32(w2), tc::smem_u32(w3)};
    uint32_t uses = 0;
    bool ok = true;
    const long long ntiles = (a.n + 127) / 128;
    const int nclusters = gridDim.x / 2;
    const SmallMod mod((uint32_t)(a.hi - a.lo + 1));
    const int trow = (warp & 3) * 32 + lane;  // accumulator lane = tile row
    const int tcol = (warp >> 2) * 64;        // this thread's 64 accumulator columns

    for (long long tile = blockIdx.x / 2; tile < ntiles; tile += nclusters) {
        // features of the tile's candidates (K = 64 layout): thread `row` < 128
        // draws its candidate's 15 components (one 64-bit draw per four),
        // the other threads write the zero columns 24..63
        if (threadIdx.x < 128) {
            const int row = threadIdx.x;
            const long long cand = tile * 128 + row;
            float v[24];
#pragma unroll
            for (int f = 0; f < 24; ++f) v[f] = 0.0f;
            if (cand < a.n) {
                const long long idx = a.idx ? __ldg(a.idx + cand) : a.first + cand;
                int comp[16];
                candidate_direction(a.seed, idx, a.lo, mod, comp);
                direction_features([&](int k) { return comp[k]; }, a.naxes, a.family, v);
            }
#pragma unroll
            for (int c = 0; c < 3; ++c) *(uint4 *)(act + tc::tile_offset(row, 8 * c, kIn)) = pack8(v + 8 * c);
        } else {
            const int row = threadIdx.x - 128;
#pragma unroll
            for (int c = 3; c < 8; ++c) *(uint4 *)(act + tc::tile_offset(row, 8 * c, kIn)) = make_uint4(0, 0, 0, 0);
        }
        tc::fence_async_smem();
        __syncthreads();
        for (int l = 0; l < 3; ++l) {
            const int K = l == 0 ? kIn : kHid;
            if (threadIdx.x == 0) {
                tc::fence_after_sync();
                for (int j = 0; j < K / 16; ++j)
                    tc::mma_bf16(tmem, tc::smem_desc(s_act + j * 256, 128, K * 16),
                                 tc::smem_desc(s_w[l] + j * 256, 128, K * 16), idesc, j > 0);
                tc::commit(&bar);
            }
            if (!tc::mbar_wait(&bar, uses & 1)) ok = false;
            ++uses;
            tc::fence_after_sync();
            // both CTAs' MMAs have read their activation tiles
            tc::fence_before_sync();
            cluster.sync();
            tc::fence_after_sync();
            float v[64];
            tc::tmem_ld32(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)tcol, *(float(*)[32])v);
            tc::tmem_ld32(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(tcol + 32), *(float(*)[32])(v + 32));
            const float *b = sbias + l * 128 + tcol;
#pragma unroll
            for (int i = 0; i < 64; ++i) v[i] = fmaxf(v[i] + b[i], 0.0f);
            if (l < 2) {
                // this half of the next layer's input, into both CTAs
#pragma unroll
                for (int c = 0; c < 8; ++c) {
                    const uint4 q = pack8(v + 8 * c);
                    const uint32_t off = tc::tile_offset(trow, 128 * r + tcol + 8 * c, kHid);
                    *(uint4 *)(act + off) = q;
                    *(uint4 *)(peer_act + off) = q;
                }
                fence_async_cluster();
                tc::fence_before_sync();
                cluster.sync();
            } else {
                // head: this CTA's 128 of the 256 terms, on the BF16-rounded activations
                float sum = 0.0f;
#pragma unroll
                for (int i = 0; i < 64; ++i) sum = fmaf(__bfloat162float(__float2bfloat16_rn(v[i])), sbias[384 + tcol + i], sum);
                spart[(warp >> 2) * 128 + trow] = sum;
                __syncthreads();
                if (threadIdx.x < 128) {
                    const float half = spart[threadIdx.x] + spart[128 + threadIdx.x];
                    if (r == 1) peer_part0[384 + threadIdx.x] = half;
                    else spart[256 + threadIdx.x] = half;
                }
                tc::fence_before_sync();
                cluster.sync();
                if (r == 0 && threadIdx.x < 128) {
                    const long long cand = tile * 128 + threadIdx.x;
                    if (cand < a.n) a.score[cand] = spart[256 + threadIdx.x] + spart[384 + threadIdx.x] + a.b4[0];
                }
            }
        }
    }
    if (!ok) s_bad = 1;
    __syncthreads();
    if (s_bad && threadIdx.x == 0) atomicExch(a.err, 1);
    tc::fence_before_sync();
    cluster.sync();  // no peer writes into this CTA's shared memory after here
    if (warp == 0) tc::tmem_dealloc(tmem, 128);
}

}  // namespace cmfw

using namespace cmfw;

// ---- host object ------------------------------------------------------------

struct cmfw_mlp {
    int cap;  // batch capacity (multiple of 128)
    int dev;
    // parameters: FP32 masters, Adam state, gradients
    float *p[8], *m[8], *v[8], *g[8];
    int rows[8], cols[8];
    __nv_bfloat16 *W[3], *WT[3];  // bf16 copies of W1..W3 and their transposes
    // activations and gradients (cap x width, bf16)
    __nv_bfloat16 *X, *H1, *H2, *H3, *dZ, *dZ2, *T1, *T2;
    float *score, *dscore, *loss, *wsum;
    float *ws;  // partial sums of the gradients and the loss (ws_layout)
    int *err;
    long long step;
};

namespace {

// parameter index: 0 W1 [256 x 64], 1 b1, 2 W2 [256 x 256], 3 b2, 4 W3, 5 b3, 6 w4 [256], 7 b4 [1]
const int kRows[8] = {kHid, 1, kHid, 1, kHid, 1, 1, 1};
const int kCols[8] = {kIn, kHid, kHid, kHid, kHid, kHid, kHid, 1};

cmfw_status cuda_fail(cudaError_t e, const char *what) {
    char msg[256];
    snprintf(msg, sizeof(msg), "%s: %s", what, cudaGetErrorString(e));
    return record_error(CMFW_ECUDA, msg);
}

size_t psize(int i) { return (size_t)kRows[i] * kCols[i]; }

// Offsets (floats) in cmfw_mlp::ws of the partial sums of one backward
// pass: each weight gradient's K splits, each bias gradient's and the
// head's row blocks, the loss's blocks.
struct WsLayout {
    size_t gemm[3], bias[3], hw4, hb4, loss, total;
};
WsLayout ws_layout() {
    WsLayout L;
    size_t o = 0;
    for (int l = 0; l < 3; ++l) {
        L.gemm[l] = o;
        o += (size_t)kMaxSplit * psize(2 * l);
    }
    for (int l = 0; l < 3; ++l) {
        L.bias[l] = o;
        o += (size_t)kMaxRowBlocks * kHid;
    }
    L.hw4 = o;
    o += (size_t)kMaxRowBlocks * kHid;
    L.hb4 = o;
    o += kMaxRowBlocks;
    L.loss = o;
    o += kMaxRowBlocks;
    L.total = o;
    return L;
}

cudaError_t refresh_bf16(cmfw_mlp *M, cudaStream_t s) {
    for (int l = 0; l < 3; ++l) {
        const int n = (int)psize(2 * l);
        to_bf16_kernel<<<(n + 255) / 256, 256, 0, s>>>(M->p[2 * l], n, kRows[2 * l], kCols[2 * l], M->W[l], M->WT[l]);
    }
    return cudaGetLastError();
}

GemmArgs gemm_args(const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, int Mr, int N, int K, void *C,
                   int ldc, int *err) {
    GemmArgs g;
    memset(&g, 0, sizeof(g));
    g.A = A;
    g.B = B;
    g.M = Mr;
    g.N = N;
    g.K = K;
    g.lda = lda;
    g.ldb = ldb;
    g.C = C;
    g.ldc = ldc;
    g.err = err;
    return g;
}

// Forward pass over the first n_pad rows of M->X; H1..H3 and score filled.
cudaError_t forward(cmfw_mlp *M, int n, int n_pad, cudaStream_t s) {
    const __nv_bfloat16 *in = M->X;
    __nv_bfloat16 *outs[3] = {M->H1, M->H2, M->H3};
    int K = kIn;
    for (int l = 0; l < 3; ++l) {
        GemmArgs g = gemm_args(in, K, M->W[l], K, n_pad, kHid, K, outs[l], kHid, M->err);
        g.bias = M->p[2 * l + 1];
        cudaError_t e = gemm(g, EPI_BIAS_RELU_BF16, s);
        if (e != cudaSuccess) return e;
        in = outs[l];
        K = kHid;
    }
    head_forward_kernel<<<(n + 7) / 8, 256, 0, s>>>(M->H3, M->p[6], M->p[7], n, M->score);
    return cudaGetLastError();
}

cudaError_t transpose(const __nv_bfloat16 *in, int rows, int cols, __nv_bfloat16 *out, cudaStream_t s) {
    dim3 grid((cols + 31) / 32, (rows + 31) / 32), block(32, 8);
    transpose_bf16_kernel<<<grid, block, 0, s>>>(in, rows, cols, out);
    return cudaGetLastError();
}

// Gradients of the weighted MSE over the batch into M->g and the loss into
// M->loss (overwritten). Every sum over the batch is formed from partial
// sums in a fixed order (no atomics), so a batch gives the same bits on
// every run.
cudaError_t backward(cmfw_mlp *M, const float *y, const float *w, const long long *idx, const float *d_wsum, int n,
                     int n_pad, float wsum, cudaStream_t s) {
    const WsLayout L = ws_layout();
    SumTable T;
    memset(&T, 0, sizeof(T));
    int nt = 0;
    auto add = [&](const float *part, float *dst, int cnt, int nparts, int pstride) {
        T.t[nt++] = SumTask{part, dst, cnt, nparts, pstride};
    };
    cudaMemsetAsync(M->dscore, 0, sizeof(float) * n_pad, s);
    const int lblocks = std::max(1, std::min(kMaxRowBlocks, (n + 255) / 256));
    loss_kernel<<<lblocks, 256, 0, s>>>(M->score, y, w, idx, n, wsum, d_wsum, M->dscore, M->ws + L.loss);
    add(M->ws + L.loss, M->loss, 1, lblocks, 1);
    cudaMemsetAsync(M->dZ, 0, (size_t)n_pad * kHid * 2, s);
    // row blocks of about 8 rows: the batch's rows spread over the SMs
    const int rblocks = std::max(1, std::min(kMaxRowBlocks, n / 8));
    head_backward_kernel<<<rblocks, kHid, 0, s>>>(M->H3, M->p[6], M->dscore, n, M->dZ, M->ws + L.hw4,
                                                  M->ws + L.hb4);
    add(M->ws + L.hw4, M->g[6], kHid, rblocks, kHid);
    add(M->ws + L.hb4, M->g[7], 1, rblocks, 1);
    // layers 3, 2, 1: dZ holds dL/dZ_l (pre-activation) of layer l
    const __nv_bfloat16 *acts[3] = {M->X, M->H1, M->H2};  // inputs of layers 1..3
    const __nv_bfloat16 *masks[3] = {nullptr, M->H1, M->H2};
    __nv_bfloat16 *dz = M->dZ, *dz_next = M->dZ2;
    for (int l = 2; l >= 0; --l) {
        const int K_in = l == 0 ? kIn : kHid;
        // bias gradient
        const int cblocks = std::max(1, std::min(kMaxRowBlocks, n_pad / 8));
        colsum_kernel<<<dim3(1, cblocks), kHid, 0, s>>>(dz, n_pad, kHid, M->ws + L.bias[l]);
        add(M->ws + L.bias[l], M->g[2 * l + 1], kHid, cblocks, kHid);
        // dW_l = dZ^T [256 x n] . X^T [K_in x n]^T
        cudaError_t e = transpose(dz, n_pad, kHid, M->T1, s);
        if (e == cudaSuccess) e = transpose(acts[l], n_pad, K_in, M->T2, s);
        if (e != cudaSuccess) return e;
        GemmArgs gw = gemm_args(M->T1, n_pad, M->T2, n_pad, kHid, K_in, n_pad, M->g[2 * l], K_in, M->err);
        gw.part = M->ws + L.gemm[l];
        int ks = 1;
        e = gemm(gw, EPI_F32, s, &ks);
        if (e != cudaSuccess) return e;
        add(gw.part, M->g[2 * l], (int)psize(2 * l), ks, (int)psize(2 * l));
        if (l > 0) {
            // dZ_{l-1} = (dZ_l . W_l) o [H_{l-1} > 0]; W_l^T is [K_in x 256]
            GemmArgs gx = gemm_args(dz, kHid, M->WT[l], kHid, n_pad, K_in, kHid, dz_next, K_in, M->err);
            gx.mask = masks[l];
            e = gemm(gx, EPI_MASK_BF16, s);
            if (e != cudaSuccess) return e;
            __nv_bfloat16 *t = dz;
            dz = dz_next;
            dz_next = t;
        }
    }
    T.ntask = nt;
    for (int k = 0; k < nt; ++k) T.start[k + 1] = T.start[k] + T.t[k].n;
    sum_parts_kernel<<<(T.start[nt] + 255) / 256, 256, 0, s>>>(T);
    return cudaGetLastError();
}

cmfw_status check_batch(cmfw_mlp *M, int n) {
    if (!M) return record_error(CMFW_EINVAL, "NULL model");
    if (n < 0 || n > M->cap) return record_error(CMFW_EINVAL, "batch outside 0..capacity");
    return CMFW_OK;
}

// One Adam update of every parameter from M->g (bias corrections of the
// model's step count), one launch.
cudaError_t adam_step(cmfw_mlp *M, float lr, cudaStream_t s) {
    M->step += 1;
    const float bc1 = 1.0f - powf(0.9f, (float)M->step), bc2 = 1.0f - powf(0.999f, (float)M->step);
    AdamTable T;
    T.off[0] = 0;
    for (int i = 0; i < 8; ++i) {
        const bool w = (i % 2 == 0) && i < 6;
        T.p[i] = M->p[i];
        T.m[i] = M->m[i];
        T.v[i] = M->v[i];
        T.g[i] = M->g[i];
        T.W[i] = w ? M->W[i / 2] : nullptr;
        T.WT[i] = w ? M->WT[i / 2] : nullptr;
        T.rows[i] = kRows[i];
        T.cols[i] = kCols[i];
        T.off[i + 1] = T.off[i] + (int)psize(i);
    }
    adam_all_kernel<<<(T.off[8] + 255) / 256, 256, 0, s>>>(T, lr, bc1, bc2);
    return cudaGetLastError();
}

cmfw_status finish(cmfw_mlp *M, cudaError_t e, const char *what, cudaStream_t s) {
    if (e != cudaSuccess) return cuda_fail(e, what);
    (void)M;
    (void)s;
    return CMFW_OK;
}

}  // namespace

extern "C" {

cmfw_status cmfw_mlp_create(int max_batch, uint64_t seed, cmfw_mlp **out) {
    if (!out) return record_error(CMFW_EINVAL, "NULL output");
    *out = nullptr;
    if (max_batch <= 0 || max_batch > (1 << 24)) return record_error(CMFW_EINVAL, "max_batch outside 1..2^24");
    cmfw_mlp *M = new cmfw_mlp();
    memset(M, 0, sizeof(*M));
    M->cap = (max_batch + 127) / 128 * 128;
    cudaGetDevice(&M->dev);
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 8 && e == cudaSuccess; ++i) {
        const size_t b = psize(i) * sizeof(float);
        e = cudaMalloc(&M->p[i], b);
        if (e == cudaSuccess) e = cudaMalloc(&M->m[i], b);
        if (e == cudaSuccess) e = cudaMalloc(&M->v[i], b);
        if (e == cudaSuccess) e = cudaMalloc(&M->g[i], b);
        if (e == cudaSuccess) e = cudaMemset(M->m[i], 0, b);
        if (e == cudaSuccess) e = cudaMemset(M->v[i], 0, b);
    }
    for (int l = 0; l < 3 && e == cudaSuccess; ++l) {
        e = cudaMalloc(&M->W[l], psize(2 * l) * 2);
        if (e == cudaSuccess) e = cudaMalloc(&M->WT[l], psize(2 * l) * 2);
    }
    const size_t act = (size_t)M->cap * kHid * 2;
    __nv_bfloat16 **bufs[7] = {&M->H1, &M->H2, &M->H3, &M->dZ, &M->dZ2, &M->T1, &M->T2};
    for (int i = 0; i < 7 && e == cudaSuccess; ++i) e = cudaMalloc(bufs[i], act);
    if (e == cudaSuccess) e = cudaMalloc(&M->X, (size_t)M->cap * kIn * 2);
    if (e == cudaSuccess) e = cudaMalloc(&M->score, sizeof(float) * M->cap);
    if (e == cudaSuccess) e = cudaMalloc(&M->dscore, sizeof(float) * M->cap);
    if (e == cudaSuccess) e = cudaMalloc(&M->loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&M->wsum, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&M->ws, sizeof(float) * ws_layout().total);
    if (e == cudaSuccess) e = cudaMalloc(&M->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(M->err, 0, sizeof(int));
    if (e != cudaSuccess) {
        cmfw_mlp_destroy(M);
        return record_error(CMFW_ENOMEM, "model allocation failed");
    }
    // He-uniform initialisation from splitmix64(seed, index); biases zero
    std::vector<float> h;
    for (int i = 0; i < 8; ++i) {
        h.assign(psize(i), 0.0f);
        const bool weight = (i % 2 == 0) || i == 6;
        if (weight) {
            const float fan_in = (float)kCols[i];
            const float a = sqrtf(6.0f / fan_in);
            for (size_t j = 0; j < h.size(); ++j) {
                const uint64_t r = splitmix64(seed * 0x100000001B3ull + (uint64_t)i * 0x9E3779B9ull + j);
                h[j] = a * (2.0f * (float)((r >> 11) * (1.0 / 9007199254740992.0)) - 1.0f);
            }
        }
        e = cudaMemcpy(M->p[i], h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) break;
    }
    if (e == cudaSuccess) e = refresh_bf16(M, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cmfw_mlp_destroy(M);
        return cuda_fail(e, "model initialisation");
    }
    *out = M;
    return CMFW_OK;
}

void cmfw_mlp_destroy(cmfw_mlp *M) {
    if (!M) return;
    for (int i = 0; i < 8; ++i) {
        cudaFree(M->p[i]);
        cudaFree(M->m[i]);
        cudaFree(M->v[i]);
        cudaFree(M->g[i]);
    }
    for (int l = 0; l < 3; ++l) {
        cudaFree(M->W[l]);
        cudaFree(M->WT[l]);
    }
    __nv_bfloat16 *bufs[8] = {M->X, M->H1, M->H2, M->H3, M->dZ, M->dZ2, M->T1, M->T2};
    for (int i = 0; i < 8; ++i) cudaFree(bufs[i]);
    cudaFree(M->score);
    cudaFree(M->dscore);
    cudaFree(M->loss);
    cudaFree(M->wsum);
    cudaFree(M->ws);
    cudaFree(M->err);
    delete M;
}

size_t cmfw_mlp_param_count(void) {
    size_t n = 0;
    for (int i = 0; i < 8; ++i) n += psize(i);
    return n;
}

cmfw_status cmfw_mlp_get_params(cmfw_mlp *M, float *h_params) {
    if (!M || !h_params) return record_error(CMFW_EINVAL, "NULL argument");
    size_t off = 0;
    for (int i = 0; i < 8; ++i) {
        cudaError_t e = cudaMemcpy(h_params + off, M->p[i], psize(i) * sizeof(float), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "parameter copy");
        off += psize(i);
    }
    return CMFW_OK;
}

cmfw_status cmfw_mlp_set_params(cmfw_mlp *M, const float *h_params) {
    if (!M || !h_params) return record_error(CMFW_EINVAL, "NULL argument");
    size_t off = 0;
    for (int i = 0; i < 8; ++i) {
        cudaError_t e = cudaMemcpy(M->p[i], h_params + off, psize(i) * sizeof(float), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return cuda_fail(e, "parameter copy");
        off += psize(i);
    }
    cudaError_t e = refresh_bf16(M, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    return e == cudaSuccess ? CMFW_OK : cuda_fail(e, "parameter refresh");
}

cmfw_status cmfw_mlp_forward(cmfw_mlp *M, const cmfw_traj_in *d_in, const int *d_family, int n, float *d_score,
                             void *stream) {
    cmfw_status st = check_batch(M, n);
    if (st != CMFW_OK || n == 0) return st;
    cudaStream_t s = (cudaStream_t)stream;
    const int n_pad = (n + 127) / 128 * 128;
    features_kernel<<<(n_pad * kIn + 255) / 256, 256, 0, s>>>(d_in, d_family, nullptr, n, n_pad, M->X);
    cudaError_t e = forward(M, n, n_pad, s);
    if (e == cudaSuccess && d_score)
        e = cudaMemcpyAsync(d_score, M->score, sizeof(float) * n, cudaMemcpyDeviceToDevice, s);
    return finish(M, e, "mlp forward", s);
}

cmfw_status cmfw_mlp_gradients(cmfw_mlp *M, const cmfw_traj_in *d_in, const int *d_family, const float *d_target,
                               const float *d_weight, int n, float weight_sum, float *h_grads, float *h_loss,
                               void *stream) {
    cmfw_status st = check_batch(M, n);
    if (st != CMFW_OK) return st;
    if (n == 0 || !(weight_sum > 0.0f)) return record_error(CMFW_EINVAL, "empty batch or weight sum <= 0");
    cudaStream_t s = (cudaStream_t)stream;
    const int n_pad = (n + 127) / 128 * 128;
    features_kernel<<<(n_pad * kIn + 255) / 256, 256, 0, s>>>(d_in, d_family, nullptr, n, n_pad, M->X);
    cudaError_t e = forward(M, n, n_pad, s);
    if (e == cudaSuccess) e = backward(M, d_target, d_weight, nullptr, nullptr, n, n_pad, weight_sum, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(e, "mlp gradients");
    int bad = 0;
    cudaMemcpy(&bad, M->err, sizeof(int), cudaMemcpyDeviceToHost);
    if (bad) return record_error(CMFW_ETIMEOUT, "a tensor-core wait gave up");
    size_t off = 0;
    for (int i = 0; i < 8 && h_grads; ++i) {
        e = cudaMemcpy(h_grads + off, M->g[i], psize(i) * sizeof(float), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "gradient copy");
        off += psize(i);
    }
    if (h_loss) cudaMemcpy(h_loss, M->loss, sizeof(float), cudaMemcpyDeviceToHost);
    return CMFW_OK;
}

cmfw_status cmfw_mlp_train_step(cmfw_mlp *M, const cmfw_traj_in *d_in, const int *d_family, const float *d_target,
                                const float *d_weight, int n, float weight_sum, float lr, float *d_loss,
                                void *stream) {
    cmfw_status st = check_batch(M, n);
    if (st != CMFW_OK) return st;
    if (n == 0 || !(weight_sum > 0.0f)) return record_error(CMFW_EINVAL, "empty batch or weight sum <= 0");
    cudaStream_t s = (cudaStream_t)stream;
    const int n_pad = (n + 127) / 128 * 128;
    features_kernel<<<(n_pad * kIn + 255) / 256, 256, 0, s>>>(d_in, d_family, nullptr, n, n_pad, M->X);
    cudaError_t e = forward(M, n, n_pad, s);
    if (e == cudaSuccess) e = backward(M, d_target, d_weight, nullptr, nullptr, n, n_pad, weight_sum, s);
    if (e == cudaSuccess) e = adam_step(M, lr, s);
    if (e == cudaSuccess && d_loss) e = cudaMemcpyAsync(d_loss, M->loss, sizeof(float), cudaMemcpyDeviceToDevice, s);
    return finish(M, e, "mlp train step", s);
}

cmfw_status cmfw_mlp_train_epoch(cmfw_mlp *M, const cmfw_traj_in *d_in, const int *d_family, const float *d_target,
                                 const float *d_weight, const long long *d_perm, long long n, int batch, float lr,
                                 float *d_loss, void *stream) {
    cmfw_status st = check_batch(M, batch);
    if (st != CMFW_OK) return st;
    if (batch < 1 || n < 0 || (n >= batch && (!d_in || !d_family || !d_target || !d_perm)))
        return record_error(CMFW_EINVAL, "bad epoch arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const int n_pad = (batch + 127) / 128 * 128;
    cudaError_t e = cudaSuccess;
    if (n < batch) return CMFW_OK;  // no full batch: nothing to do, *d_loss untouched
    // full batches only: rows perm[b .. b + batch) for b = 0, batch, ...
    for (long long b = 0; b + batch <= n && e == cudaSuccess; b += batch) {
        const long long *idx = d_perm + b;
        weight_sum_kernel<<<1, 1024, 0, s>>>(d_weight, idx, batch, M->wsum);
        features_kernel<<<(n_pad * kIn + 255) / 256, 256, 0, s>>>(d_in, d_family, idx, batch, n_pad, M->X);
        e = forward(M, batch, n_pad, s);
        if (e == cudaSuccess) e = backward(M, d_target, d_weight, idx, M->wsum, batch, n_pad, 0.0f, s);
        if (e == cudaSuccess) e = adam_step(M, lr, s);
    }
    if (e == cudaSuccess && d_loss) e = cudaMemcpyAsync(d_loss, M->loss, sizeof(float), cudaMemcpyDeviceToDevice, s);
    return finish(M, e, "mlp train epoch", s);
}

cmfw_status cmfw_mlp_status(cmfw_mlp *M) {
    if (!M) return record_error(CMFW_EINVAL, "NULL model");
    int bad = 0;
    cudaError_t e = cudaMemcpy(&bad, M->err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "status copy");
    return bad ? record_error(CMFW_ETIMEOUT, "a tensor-core wait gave up") : CMFW_OK;
}

cmfw_status cmfw_mlp_score_candidates(cmfw_mlp *M, uint64_t seed, long long first, long long n, int naxes, int lo,
                                      int hi, int family, float *d_scores, void *stream) {
    if (!M || !d_scores) return record_error(CMFW_EINVAL, "NULL argument");
    if (n < 0 || naxes < 1 || naxes > 15 || hi < lo || family < 0 || family > 4)
        return record_error(CMFW_EINVAL, "candidate range out of bounds");
    cudaStream_t s = (cudaStream_t)stream;
    for (long long b = 0; b < n; b += M->cap) {
        const int nb = (int)((n - b) < M->cap ? (n - b) : M->cap);
        const int n_pad = (nb + 127) / 128 * 128;
        candidate_features_kernel<<<(n_pad * kIn + 255) / 256, 256, 0, s>>>(seed, first + b, nb, n_pad, naxes, lo,
                                                                            hi, family, M->X);
        cudaError_t e = forward(M, nb, n_pad, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_scores + b, M->score, sizeof(float) * nb, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return cuda_fail(e, "candidate scoring");
    }
    return CMFW_OK;
}

static cmfw_status score_fused(cmfw_mlp *M, uint64_t seed, long long first, const long long *d_idx, long long n,
                               int naxes, int lo, int hi, int family, float *d_scores, void *stream) {
    if (!M || !d_scores) return record_error(CMFW_EINVAL, "NULL argument");
    if (n < 0 || naxes < 1 || naxes > 15 || hi < lo || family < 0 || family > 4)
        return record_error(CMFW_EINVAL, "candidate range out of bounds");
    if (n == 0) return CMFW_OK;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaFuncSetAttribute((const void *)mlp_score_fused_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kFusedSmem);
    if (e != cudaSuccess) return cuda_fail(e, "fused scoring attributes");
    FusedArgs a;
    for (int l = 0; l < 3; ++l) {
        a.W[l] = M->W[l];
        a.bias[l] = M->p[2 * l + 1];
    }
    a.w4 = M->p[6];
    a.b4 = M->p[7];
    a.seed = seed;
    a.first = first;
    a.n = n;
    a.idx = d_idx;
    a.naxes = naxes;
    a.lo = lo;
    a.hi = hi;
    a.family = family;
    a.score = d_scores;
    a.err = M->err;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(sms / 2 * 2), 1, 1);
    cfg.blockDim = dim3(256, 1, 1);
    cfg.dynamicSmemBytes = kFusedSmem;
    cfg.stream = s;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, (const void *)mlp_score_fused_kernel, &cfg) != cudaSuccess ||
        clusters < 1) {
        cudaGetLastError();
        clusters = sms / 2;
    }
    const long long tiles = (n + 127) / 128;
    if ((long long)clusters > tiles) clusters = (int)tiles;
    cfg.gridDim = dim3((unsigned)(2 * clusters), 1, 1);
    e = cudaLaunchKernelEx(&cfg, mlp_score_fused_kernel, a);
    if (e == cudaSuccess) e = cudaGetLastError();
    return e == cudaSuccess ? CMFW_OK : cuda_fail(e, "fused scoring launch");
}

cmfw_status cmfw_mlp_score_candidates_fused(cmfw_mlp *M, uint64_t seed, long long first, long long n, int naxes,
                                            int lo, int hi, int family, float *d_scores, void *stream) {
    return score_fused(M, seed, first, nullptr, n, naxes, lo, hi, family, d_scores, stream);
}

cmfw_status cmfw_mlp_score_indices(cmfw_mlp *M, uint64_t seed, const long long *d_idx, long long n, int naxes,
                                   int lo, int hi, int family, float *d_scores, void *stream) {
    if (n > 0 && !d_idx) return record_error(CMFW_EINVAL, "NULL index list");
    return score_fused(M, seed, 0, d_idx, n, naxes, lo, hi, family, d_scores, stream);
}

cmfw_status cmfw_candidate_records(uint64_t seed, const long long *d_idx, int n, int naxes, int lo, int hi,
                                   const double *d_start, cmfw_traj_in *d_out, void *stream) {
    if (n < 0 || naxes < 1 || naxes > CMFW_MAX_AXES || hi < lo) return record_error(CMFW_EINVAL, "bad candidate range");
    if (n == 0) return CMFW_OK;
    candidate_records_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(seed, d_idx, n, naxes, lo, hi,
                                                                                  d_start, d_out);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? CMFW_OK : cuda_fail(e, "candidate records");
}

cmfw_status cmfw_select_top(const float *d_scores, long long n, long long k, long long *d_idx, int cap, int *h_count,
                            void *stream) {
    if (!d_scores || !d_idx || !h_count || k < 1 || cap < 1 || n < 0 || n > 0xFFFFFFFFll)
        return record_error(CMFW_EINVAL, "bad selection arguments");
    cudaStream_t s = (cudaStream_t)stream;
    // the histogram and the output counter: this thread's, on this device,
    // allocated by its first call and kept (a call synchronises before it
    // returns, so the next call on the thread may reuse them)
    struct SelectScratch {
        unsigned long long *hist = nullptr;
        int *count = nullptr;
    };
    thread_local std::map<int, SelectScratch> t_select;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "top-k selection");
    SelectScratch &S = t_select[dev];
    if (!S.hist && (e = cudaMalloc(&S.hist, 2048 * sizeof(unsigned long long))) != cudaSuccess) S.hist = nullptr;
    if (e == cudaSuccess && !S.count && (e = cudaMalloc(&S.count, sizeof(int))) != cudaSuccess) S.count = nullptr;
    unsigned long long *d_hist = S.hist;
    int *d_count = S.count;
    // radix select of the k-th largest selection key, 11 + 11 + 10 bits of
    // the score key then of the index part; it stops early once the
    // threshold's bin holds exactly the keys still needed (k >= n: all)
    uint64_t prefix = 0, mask = 0;
    long long need = k;
    const uint32_t shifts[6] = {53, 42, 32, 21, 10, 0};
    const uint32_t widths[6] = {11, 11, 10, 11, 11, 10};
    std::vector<unsigned long long> h(2048);
    for (int pass = 0; pass < 6 && e == cudaSuccess && k < n; ++pass) {
        e = cudaMemsetAsync(d_hist, 0, 2048 * sizeof(unsigned long long), s);
        if (e != cudaSuccess) break;
        score_hist_kernel<<<592, 256, 0, s>>>(d_scores, n, shifts[pass], widths[pass], prefix, mask, d_hist);
        e = cudaMemcpyAsync(h.data(), d_hist, 2048 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) break;
        const int nb = 1 << widths[pass];
        int b = nb - 1;
        for (; b > 0; --b) {
            if ((long long)h[b] >= need) break;
            need -= (long long)h[b];
        }
        prefix |= (uint64_t)b << shifts[pass];
        mask |= (uint64_t)(nb - 1) << shifts[pass];
        if ((long long)h[b] == need) break;  // every key of this bin is selected
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(d_count, 0, sizeof(int), s);
    if (e == cudaSuccess) {
        select_kernel<<<592, 256, 0, s>>>(d_scores, n, prefix, d_idx, cap, d_count);
        e = cudaMemcpyAsync(h_count, d_count, sizeof(int), cudaMemcpyDeviceToHost, s);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? CMFW_OK : cuda_fail(e, "top-k selection");
}

}  // extern "C"
