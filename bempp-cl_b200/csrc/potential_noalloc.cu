// Potential evaluation without any device allocation.
//
// bemppcuda_evaluate_potential needs a caller-provided workspace for the
// per-source table (points, normals, weighted coefficients).  Some callers
// cannot provide one: they receive only the input and output device buffers
// from a host application that owns all device memory (for example a plugin
// running inside a solver with its own memory pool, or an embedding runtime
// that has no CUDA allocation binding), and they cannot call cudaMalloc
// themselves -- it may fail inside a pool that has reserved the memory, and
// it synchronizes the whole device, stalling the host application's streams.
// This entry point serves them: the workspace is a fixed array that lives in
// the library image on every GPU that loads it.
//
// Limits and sharing:
//  * the array holds BEMPPCUDA_NOALLOC_SCRATCH_DOUBLES doubles (24 MiB); a
//    problem whose source table is larger is rejected with
//    BEMPPCUDA_ERR_WORKSPACE before anything is launched;
//  * every call on a device uses the same array, so calls whose kernels can
//    overlap on the GPU (different streams without ordering between them)
//    race on it; order them on one stream or with events;
//  * each call rewrites every workspace entry it reads, so nothing has to
//    start at zero and the contents left by the previous call do no harm;
//  * the array's device address comes from cudaGetSymbolAddress on the
//    current device.  It is looked up again on every call made outside a
//    stream capture, so a call after cudaDeviceReset (or anything else that
//    recreates the primary context and reloads the module) uses the array's
//    new address; a call made while its stream is capturing uses the address
//    of the last uncaptured call on that device, so make at least one call on
//    a device before any stream capture begins there, and none across a
//    context reset inside one capture.
#include <mutex>

#include "common.cuh"

int bc_potential_launch(const bemppcuda_potential_args *a, double *workspace, cudaStream_t st);
int64_t bc_potential_workspace_doubles(int64_t nsupport, int nq);

namespace {

static __device__ __align__(256) double g_noalloc_scratch[BEMPPCUDA_NOALLOC_SCRATCH_DOUBLES];

constexpr int kMaxDevices = 256;
std::mutex g_setup_mutex;
double *g_scratch_address[kMaxDevices] = {nullptr};

// Device address of the scratch array on the current device: looked up on every call outside a
// stream capture (the address changes when the context is recreated), cached for captured calls.
int scratch_address(cudaStream_t stream, double **out) {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        bc_set_error("evaluate_potential_noalloc: no usable current device (%s)", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    err = cudaStreamIsCapturing(stream, &capture);
    if (err != cudaSuccess) {
        bc_set_error("evaluate_potential_noalloc: cudaStreamIsCapturing failed: %s", cudaGetErrorString(err));
        return BEMPPCUDA_ERR_CUDA;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (capture == cudaStreamCaptureStatusNone) {
        void *addr = nullptr;
        err = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
        if (err != cudaSuccess || !addr) {
            bc_set_error("evaluate_potential_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                         cudaGetErrorString(err));
            return BEMPPCUDA_ERR_CUDA;
        }
        g_scratch_address[dev] = static_cast<double *>(addr);
    } else if (!g_scratch_address[dev]) {
        bc_set_error("evaluate_potential_noalloc: the first call on device %d is inside a stream capture; make "
                     "one call on the device before capturing", dev);
        return BEMPPCUDA_ERR_INVALID;
    }
    *out = g_scratch_address[dev];
    return BEMPPCUDA_OK;
}

}  // namespace

extern "C" int bemppcuda_evaluate_potential_noalloc(const bemppcuda_potential_args *a, void *stream) {
    if (!a) {
        bc_set_error("null argument struct");
        return BEMPPCUDA_ERR_INVALID;
    }
    if (a->space.nsupport < 0 || a->nq < 1 || a->nq > BEMPPCUDA_MAX_REGULAR_POINTS) {
        bc_set_error("evaluate_potential_noalloc: invalid support size or rule size");
        return BEMPPCUDA_ERR_INVALID;
    }
    const int64_t need = bc_potential_workspace_doubles(a->space.nsupport, a->nq);
    if (need < 0 || need > (int64_t)BEMPPCUDA_NOALLOC_SCRATCH_DOUBLES) {
        bc_set_error(
            "evaluate_potential_noalloc: %lld support elements x %d points need %lld workspace doubles, above the "
            "fixed maximum of %lld; use bemppcuda_evaluate_potential with a caller workspace",
            (long long)a->space.nsupport, a->nq, (long long)need, (long long)BEMPPCUDA_NOALLOC_SCRATCH_DOUBLES);
        return BEMPPCUDA_ERR_WORKSPACE;
    }
    // same argument checks as the allocating entry point, with the fixed array as workspace
    bemppcuda_potential_args local = *a;
    double *scratch = nullptr;
    int rc = scratch_address((cudaStream_t)stream, &scratch);
    if (rc) return rc;
    local.workspace = scratch;
    local.workspace_bytes = (int64_t)sizeof(double) * (int64_t)BEMPPCUDA_NOALLOC_SCRATCH_DOUBLES;
    return bemppcuda_evaluate_potential(&local, stream);
}
