// cmfw_walk_f64_noalloc: the f64 walk of cmfw_walk_f64 with its scratch in a
// fixed device array instead of memory the library allocates.
//
// Who needs it: callers that cannot call cudaMalloc -- code whose device
// memory all comes from another allocator's pool (a framework's caching
// allocator that accounts for every byte), and code that must not
// synchronise the device mid-run, which a first cudaMalloc or cudaFree may
// do. The walk's scratch (snapshot matrices, row exponents, survivor list
// and counter) lives in g_noalloc_scratch below; inputs and outputs remain
// the caller's.
//
// The array is a device symbol: in host code its name is a host-side
// stand-in, not a device address, so the address handed to the kernels is
// looked up once per device with cudaGetSymbolAddress (with that device
// current) and cached. Every call on a device shares the array: calls that
// overlap on the GPU race on it. Whatever must start at zero (the survivor
// counter) is cleared on the caller's stream by the walk itself.
#include <cstdio>
#include <mutex>

#include "cmfw.h"
#include "cmfw_internal.cuh"

namespace cmfw {
cmfw_status record_error(cmfw_status s, const char *msg);
}  // namespace cmfw

static __device__ __align__(256) unsigned char g_noalloc_scratch[CMFW_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
void *g_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (first call per
// device: cudaGetSymbolAddress).
cmfw_status scratch_address(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cmfw::record_error(CMFW_ECUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return cmfw::record_error(CMFW_EUNSUPPORTED, "device ordinal above 63");
    std::lock_guard<std::mutex> lk(g_addr_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            char msg[256];
            snprintf(msg, sizeof(msg), "cudaGetSymbolAddress of the fixed scratch array: %s",
                     cudaGetErrorString(e));
            return cmfw::record_error(CMFW_ECUDA, msg);
        }
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return CMFW_OK;
}

}  // namespace

extern "C" cmfw_status cmfw_walk_f64_noalloc(const cmfw_desc *desc, const cmfw_traj_in *d_in,
                                             cmfw_traj_out *d_out, int n_traj, int N, int h, void *stream) {
    cmfw_status st = cmfw_check_desc(desc);
    if (st != CMFW_OK) return st;
    if (n_traj < 0) return cmfw::record_error(CMFW_EINVAL, "n_traj is negative");
    const size_t need = cmfw_walk_workspace_bytes(desc, n_traj);
    if (need > CMFW_NOALLOC_SCRATCH_BYTES) {
        char msg[256];
        snprintf(msg, sizeof(msg),
                 "%d trajectories at rank %d need %zu scratch bytes; the fixed scratch array holds %u: "
                 "split the batch",
                 n_traj, desc->rank, need, (unsigned)CMFW_NOALLOC_SCRATCH_BYTES);
        return cmfw::record_error(CMFW_EINVAL, msg);
    }
    void *scratch = nullptr;
    st = scratch_address(&scratch);
    if (st != CMFW_OK) return st;
    cmfw_launch L = {};
    L.d_workspace = scratch;
    L.workspace_bytes = CMFW_NOALLOC_SCRATCH_BYTES;
    return cmfw_walk_f64(desc, d_in, d_out, n_traj, N, h, &L, stream);
}
