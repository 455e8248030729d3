// Monitored-quantity reduction that allocates no device memory.
//
// mel_monitor_compute reduces kinetic energy, mass-weighted mean displacement and the number of
// active contact elements of a resident model into block partials held in memory the handle
// allocated with cudaMalloc.  Some callers cannot allocate device memory themselves: a framework or
// runtime that owns all device memory through its own allocator, or a deployment with a fixed device
// memory budget where no call may grow it, still needs these quantities from state arrays it already
// holds.  mel_monitor_reduce_static serves them: the caller passes its device input arrays and a
// device output array, and the block partials live in the file-scope array below instead of in
// memory allocated for the call.
//
// The array holds MEL_STATIC_MAX_BLOCKS partial records; each block of 256 threads covers up to
// MEL_STATIC_PER_BLOCK nodes (and as many contact elements), so one call handles at most
// MEL_STATIC_MAX_ELEMENTS nodes and contact elements; larger inputs are rejected with an error.
// Every GPU that loads the library keeps this array until the process exits.
#include <cstdio>
#include "mel_internal.h"

#define MEL_STATIC_MAX_BLOCKS 1024
#define MEL_STATIC_PER_BLOCK 2048
#define MEL_STATIC_MAX_ELEMENTS (MEL_STATIC_MAX_BLOCKS * MEL_STATIC_PER_BLOCK)

// five partial sums per block: kinetic energy, sum m*ux, sum m*uy, sum m, active contacts
static __device__ __align__(256) double mel_static_partials[5 * MEL_STATIC_MAX_BLOCKS];

namespace mel {

__global__ void static_partial_kernel(const double2* __restrict__ v, const double2* __restrict__ m,
                                      const double2* __restrict__ u, int n_nodes, const mel_contact* __restrict__ cont,
                                      int n_contacts, double* part, int nblk)
{
    __shared__ double s[5][256];
    double ke = 0., ux = 0., uy = 0., mt = 0., act = 0.;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += gridDim.x * blockDim.x) {
        double2 vv = v[i], mm = m[i], uu = u[i];
        ke += 0.5 * vv.x * vv.x * mm.x + 0.5 * vv.y * vv.y * mm.y;
        ux += uu.x * mm.x; uy += uu.y * mm.y; mt += mm.x;
    }
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n_contacts; c += gridDim.x * blockDim.x)
        if (cont[c].fx != 0. || cont[c].fy != 0.) act += 1.;
    s[0][threadIdx.x] = ke; s[1][threadIdx.x] = ux; s[2][threadIdx.x] = uy; s[3][threadIdx.x] = mt; s[4][threadIdx.x] = act;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int k = 0; k < 5; k++) s[k][threadIdx.x] += s[k][threadIdx.x + w];
        __syncthreads();
    }
    // every slot the final kernel reads is written here in the same call
    if (threadIdx.x < 5) part[threadIdx.x * nblk + blockIdx.x] = s[threadIdx.x][0];
}

__global__ void static_final_kernel(const double* part, int nblk, double* out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double t[5] = { 0., 0., 0., 0., 0. };
    for (int k = 0; k < 5; k++)
        for (int b = 0; b < nblk; b++) t[k] += part[k * nblk + b];
    out[0] = t[0];
    out[1] = t[3] > 0 ? t[1] / t[3] : 0.;
    out[2] = t[3] > 0 ? t[2] / t[3] : 0.;
    out[3] = t[4];
}

} // namespace mel

// Device address of mel_static_partials in the current device's context.  It is looked up on
// every call rather than cached: after a cudaDeviceReset (or any other teardown of the primary
// context) the module is loaded again and the array may sit at a new address, and the lookup costs
// little once the module is loaded.  The first call on a device loads the module, so that call
// should come before any stream capture.
static mel_status static_scratch(double** out)
{
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, mel_static_partials);
    if (e != cudaSuccess || !p) { mel_set_cuda_error(e, "cudaGetSymbolAddress(mel_static_partials)", __FILE__, __LINE__); return MEL_ERR_CUDA; }
    *out = static_cast<double*>(p);
    return MEL_OK;
}

extern "C" mel_status mel_monitor_reduce_static(const double* d_velocity, const double* d_mass, const double* d_displacement,
                                                int n_nodes, const mel_contact* d_contacts, int n_contacts, double* d_out,
                                                void* stream)
{
    if (n_nodes < 0 || n_contacts < 0) { mel_set_error("negative size"); return MEL_ERR_INVALID; }
    if (n_nodes > MEL_STATIC_MAX_ELEMENTS || n_contacts > MEL_STATIC_MAX_ELEMENTS) {
        mel_set_error("mel_monitor_reduce_static handles at most %d nodes and %d contact elements per call "
                      "(got %d and %d): its fixed scratch holds %d block partials",
                      MEL_STATIC_MAX_ELEMENTS, MEL_STATIC_MAX_ELEMENTS, n_nodes, n_contacts, MEL_STATIC_MAX_BLOCKS);
        return MEL_ERR_INVALID;
    }
    if (!d_out || (n_nodes > 0 && (!d_velocity || !d_mass || !d_displacement)) || (n_contacts > 0 && !d_contacts)) {
        mel_set_error("null device pointer");
        return MEL_ERR_INVALID;
    }
    // an error left by the caller's own launches is reported as such and left pending for the
    // caller (cudaPeekAtLastError does not clear it); nothing is launched on top of it
    cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        mel_set_error("a CUDA error from before this call is pending (%s: %s); nothing was launched",
                      cudaGetErrorName(pending), cudaGetErrorString(pending));
        return MEL_ERR_CUDA;
    }
    double* part = nullptr;
    mel_status rc = static_scratch(&part);
    if (rc) return rc;
    int n = n_nodes > n_contacts ? n_nodes : n_contacts;
    int nblk = (n + MEL_STATIC_PER_BLOCK - 1) / MEL_STATIC_PER_BLOCK;
    if (nblk < 1) nblk = 1;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    mel::static_partial_kernel<<<nblk, 256, 0, s>>>(reinterpret_cast<const double2*>(d_velocity),
                                                    reinterpret_cast<const double2*>(d_mass),
                                                    reinterpret_cast<const double2*>(d_displacement), n_nodes,
                                                    d_contacts, n_contacts, part, nblk);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { mel_set_cuda_error(e, "static_partial_kernel launch", __FILE__, __LINE__); return MEL_ERR_CUDA; }
    mel::static_final_kernel<<<1, 32, 0, s>>>(part, nblk, d_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) { mel_set_cuda_error(e, "static_final_kernel launch", __FILE__, __LINE__); return MEL_ERR_CUDA; }
    return MEL_OK;
}
