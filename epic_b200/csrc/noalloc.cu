// Allocation-free variant of the vorticity correction (apply_vortcor).
//
// Some callers cannot call cudaMalloc: a host program whose device memory is
// owned by another runtime's pool (for example a Fortran code that keeps its
// parcel arrays in OpenACC or CUDA Fortran device memory and runs under that
// runtime's memory budget), or a time loop that must not take the implicit
// device synchronisation of an allocation.  This entry point works on device
// arrays the caller already owns and keeps its only scratch -- the per-block
// partial sums of the reduction -- in a fixed file-scope __device__ array.
//
// The scratch holds NOALLOC_MAX_BLOCKS x 4 doubles (128 KiB) plus 8 doubles
// for the final correction; every GPU that loads the library keeps it until
// the process exits.  The number of blocks grows with the parcel count (one
// block per NOALLOC_CHUNK parcels), so the largest accepted parcel count is
// NOALLOC_MAX_BLOCKS * NOALLOC_CHUNK = 67,108,864.  All calls share the one
// array: two calls whose kernels overlap on the GPU (different streams, no
// ordering between them) race on it and give wrong results.
#include "../../include/epic_gpu.h"
#include "common.cuh"

#include <cuda_runtime.h>
#include <algorithm>
#include <mutex>

namespace {

constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_MAX_BLOCKS = 4096;
constexpr long long NOALLOC_CHUNK = 16384;   // parcels per block (64 per thread)

// Block partials (4 per block: sum V, sum V wx, sum V wy, sum V wz) followed
// by the final correction dvor[3].
__device__ __align__(256) double g_noalloc_scratch[NOALLOC_MAX_BLOCKS * 4 + 8];

// Device address of g_noalloc_scratch for each device (a host-side use of
// the symbol name is not a device address).  The address is looked up again,
// with the device current, on every call whose stream is not capturing, so a
// module that was loaded again (after cudaDeviceReset, or in a new primary
// context) is found at its new address; a call on a capturing stream uses the
// address found by the last call outside a capture on that device.
constexpr int MAX_DEVICES = 64;
double* g_scratch_addr[MAX_DEVICES] = {nullptr};
std::mutex g_scratch_mu;

int scratch_for_current_device(cudaStream_t st, double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return EPIC_ERR_CUDA;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return EPIC_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (cs == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return EPIC_ERR_CUDA;
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    if (!g_scratch_addr[dev]) return EPIC_ERR_CUDA;
    *out = g_scratch_addr[dev];
    return EPIC_OK;
}

// Pass 1: each block reduces its chunk in a fixed order and writes its slot.
__global__ void __launch_bounds__(NOALLOC_THREADS) k_na_partials(long long n, const double* vol, const double* vor,
                                                                double* scratch) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    long long b0 = (long long)blockIdx.x * NOALLOC_CHUNK;
    long long b1 = min(b0 + NOALLOC_CHUNK, n);
    for (long long i = b0 + threadIdx.x; i < b1; i += NOALLOC_THREADS) {
        double v = vol[i];
        acc[0] += v;
        acc[1] += vor[3 * i] * v;
        acc[2] += vor[3 * i + 1] * v;
        acc[3] += vor[3 * i + 2] * v;
    }
    __shared__ double red[NOALLOC_THREADS / 32][4];
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double v = acc[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffff, v, o);
        if (l == 0) red[w][k] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = 0.0;
        for (int q = 0; q < NOALLOC_THREADS / 32; ++q) v += red[q][threadIdx.x];
        scratch[blockIdx.x * 4 + threadIdx.x] = v;
    }
}

// Pass 2: fixed-order sum of the partials -> dvor = mean vorticity - vor_bar
// (parcel_correction.f90:117-124).
__global__ void k_na_final(int nb, double b0, double b1, double b2, double* scratch) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = 0; b < nb; ++b)
        for (int k = 0; k < 4; ++k) s[k] += scratch[b * 4 + k];
    double* dvor = scratch + NOALLOC_MAX_BLOCKS * 4;
    dvor[0] = s[1] / s[0] - b0;
    dvor[1] = s[2] / s[0] - b1;
    dvor[2] = s[3] / s[0] - b2;
}

// Pass 3: subtract the correction (parcel_correction.f90:126-133).
__global__ void k_na_apply(long long n, double* vor, const double* scratch) {
    const double* dvor = scratch + NOALLOC_MAX_BLOCKS * 4;
    double d0 = dvor[0], d1 = dvor[1], d2 = dvor[2];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        vor[3 * i] = vor[3 * i] - d0;
        vor[3 * i + 1] = vor[3 * i + 1] - d1;
        vor[3 * i + 2] = vor[3 * i + 2] - d2;
    }
}

}  // namespace

extern "C" int epic_gpu_apply_vortcor_noalloc(int64_t n, const double* vol, double* vor, const double vor_bar[3],
                                              double dvor_out[3], void* stream) {
    if (n <= 0 || !vol || !vor || !vor_bar) return EPIC_ERR_ARG;
    if (n > (int64_t)NOALLOC_MAX_BLOCKS * NOALLOC_CHUNK) return EPIC_ERR_CAPACITY;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* scratch = nullptr;
    int rc = scratch_for_current_device(st, &scratch);
    if (rc != EPIC_OK) return rc;
    int nb = (int)((n + NOALLOC_CHUNK - 1) / NOALLOC_CHUNK);
    k_na_partials<<<nb, NOALLOC_THREADS, 0, st>>>(n, vol, vor, scratch);
    k_na_final<<<1, 32, 0, st>>>(nb, vor_bar[0], vor_bar[1], vor_bar[2], scratch);
    int ab = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
    k_na_apply<<<ab, 256, 0, st>>>(n, vor, scratch);
    if (cudaGetLastError() != cudaSuccess) return EPIC_ERR_CUDA;
    if (dvor_out) {
        if (cudaMemcpyAsync(dvor_out, scratch + NOALLOC_MAX_BLOCKS * 4, 3 * sizeof(double), cudaMemcpyDeviceToHost,
                            st) != cudaSuccess)
            return EPIC_ERR_CUDA;
        if (cudaStreamSynchronize(st) != cudaSuccess) return EPIC_ERR_CUDA;
    }
    return EPIC_OK;
}
