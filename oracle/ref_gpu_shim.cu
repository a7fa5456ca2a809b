// C entry points over the reference's own CUDA kernels, built unchanged for
// sm_100a -- a COMPARISON ARM for the benchmark (the "plain sm_100a kernel"
// the project's kernels are measured against), never part of the product.
//
// The `ref-gpu` target of oracle/Makefile compiles this file once per
// reference variant with REF_SRC naming a copy of cuda/cmf_walk_<variant>.cu
// whose main() is renamed (the only edit; the kernels, launch shapes and
// constant tables are the reference's). Each entry launches the reference
// kernel on caller-owned device buffers of the reference's record layouts
// (TrajectoryInput 192 B in; TrajectoryResult 64 B, DF64Result / RNSResult
// 56 B out) on the given stream, grid ceil(n / block) as run_benchmark()
// launches it (cmf_walk_f64.cu:212-228, cmf_walk_df64.cu:405-410,
// cmf_walk_rns.cu:376-381).
#include REF_SRC

extern "C" {

#if defined(REF_F64)
int ref_gpu_f64_launch(const void *d_in, void *d_out, int p, int q, double z, int N, int h, int n, int block,
                       void *stream) {
    if (n <= 0) return 0;
    CMFDesc desc = make_cmf_desc(p, q, z);
    walk_kernel_f64<<<(n + block - 1) / block, block, 0, (cudaStream_t)stream>>>(
        (const TrajectoryInput *)d_in, (TrajectoryResult *)d_out, desc, N, h, n);
    return (int)cudaGetLastError();
}
#elif defined(REF_DF64)
int ref_gpu_df64_launch(const void *d_in, void *d_out, int p, int q, double z, int N, int h, int n, int block,
                        void *stream) {
    if (n <= 0) return 0;
    CMFDesc desc = make_cmf_desc(p, q, z);
    walk_kernel_df64<<<(n + block - 1) / block, block, 0, (cudaStream_t)stream>>>(
        (const DF64Input *)d_in, (DF64Result *)d_out, desc, N, h, n);
    return (int)cudaGetLastError();
}
#elif defined(REF_RNS)
int ref_gpu_rns_launch(const void *d_in, void *d_out, int p, int q, double z, int N, int h, int n, int block,
                       int n_primes, void *stream) {
    if (n <= 0) return 0;
    CMFDesc desc = make_cmf_desc(p, q, z);
    walk_kernel_rns<<<(n + block - 1) / block, block, 0, (cudaStream_t)stream>>>(
        (const RNSInput *)d_in, (RNSResult *)d_out, desc, N, h, n, n_primes);
    return (int)cudaGetLastError();
}
#else
#error "define one of REF_F64, REF_DF64, REF_RNS"
#endif

}  // extern "C"
