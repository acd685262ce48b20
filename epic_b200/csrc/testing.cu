// Known-answer hooks (include/epic_gpu_testing.h).
#include "../../include/epic_gpu_testing.h"
#include "ctx.hpp"
#include "eigen.cuh"

using namespace epic;

template <class O>
__global__ void k_test_eigen(long long n, const double* A6, double* D, double* V, int values_only) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double* a = A6 + 6 * i;
        double A[9] = {a[0], a[1], a[2], a[1], a[3], a[4], a[2], a[4], a[5]};
        if (values_only) {
            sz_eigenvalues<O>(A, D + 3 * i);
        } else {
            sz_diagonalise<O>(A, D + 3 * i, V + 9 * i);
        }
    }
}

extern "C" int epic_gpu_test_eigen(int64_t n, const double* A6, double* D, double* V, int exact, int values_only) {
    if (n <= 0 || !A6 || !D || !V) return EPIC_ERR_ARG;
    double *dA = nullptr, *dD = nullptr, *dV = nullptr;
    int rc = EPIC_OK;
    if (cudaMalloc(&dA, sizeof(double) * 6 * n) != cudaSuccess || cudaMalloc(&dD, sizeof(double) * 3 * n) != cudaSuccess ||
        cudaMalloc(&dV, sizeof(double) * 9 * n) != cudaSuccess) {
        rc = EPIC_ERR_CUDA;
    } else {
        cudaMemcpy(dA, A6, sizeof(double) * 6 * n, cudaMemcpyHostToDevice);
        cudaMemset(dV, 0, sizeof(double) * 9 * n);
        int g = (int)((n + 255) / 256);
        if (exact) k_test_eigen<ExactOps><<<g, 256>>>(n, dA, dD, dV, values_only);
        else k_test_eigen<FastOps><<<g, 256>>>(n, dA, dD, dV, values_only);
        if (cudaDeviceSynchronize() != cudaSuccess) rc = EPIC_ERR_CUDA;
        cudaMemcpy(D, dD, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost);
        cudaMemcpy(V, dV, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost);
    }
    if (dA) cudaFree(dA);
    if (dD) cudaFree(dD);
    if (dV) cudaFree(dV);
    return rc;
}

struct epic_ctx {
    Ctx c;
};

extern "C" int epic_gpu_test_diverge(epic_ctx* ctx, const double* phi, double* grad) {
    if (!ctx || !phi || !grad) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    try {
        double* dphi = c.w(7);
        CK(cudaMemcpyAsync(dphi, phi, sizeof(double) * c.P.fsz, cudaMemcpyHostToDevice, c.stream));
        double* g[3] = {c.w(8), c.w(9), c.w(10)};
        diverge_laplace(c, dphi, g);
        for (int k = 0; k < 3; ++k)
            CK(cudaMemcpyAsync(grad + (size_t)k * c.P.fsz, g[k], sizeof(double) * c.P.fsz, cudaMemcpyDeviceToHost, c.stream));
        CK(cudaStreamSynchronize(c.stream));
    } catch (const CudaError& e) {
        c.err = e.what();
        return e.code;
    }
    return EPIC_OK;
}

extern "C" int epic_gpu_test_spectral(epic_ctx* ctx, int op, const double* f, double* out) {
    if (!ctx || !f || !out) return EPIC_ERR_ARG;
    if (op != 0) return EPIC_ERR_ARG;   // the step's vertical differences live inside fused column kernels
    Ctx& c = ctx->c;
    try {
        double* din = c.w(7);
        double* dout = c.w(8);
        CK(cudaMemcpyAsync(din, f, sizeof(double) * c.P.fsz, cudaMemcpyHostToDevice, c.stream));
        CK(cudaMemsetAsync(dout, 0, sizeof(double) * c.P.fsz, c.stream));
        lapinv_probe(c, din, dout);
        CK(cudaMemcpyAsync(out, dout, sizeof(double) * c.P.fsz, cudaMemcpyDeviceToHost, c.stream));
        CK(cudaStreamSynchronize(c.stream));
    } catch (const CudaError& e) {
        c.err = e.what();
        return e.code;
    }
    return EPIC_OK;
}

extern "C" int epic_gpu_test_delete(epic_ctx* ctx, int64_t n, const int32_t* idx) {
    if (!ctx || n < 0 || (n > 0 && !idx)) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    try {
        test_delete(c, idx, (int)n);
    } catch (const CudaError& e) {
        c.err = e.what();
        return e.code;
    }
    return EPIC_OK;
}

extern "C" int epic_gpu_test_reflective_bc(epic_ctx* ctx) {
    if (!ctx) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    try {
        reflective_all(c);
        CK(cudaStreamSynchronize(c.stream));
    } catch (const CudaError& e) {
        c.err = e.what();
        return e.code;
    }
    return EPIC_OK;
}

extern "C" int epic_gpu_test_set_fft_path(epic_ctx* ctx, int path) {
    if (!ctx) return EPIC_ERR_ARG;
    if (path < 0 || path > 3) return EPIC_ERR_ARG;
    ctx->c.fft_path = path;
    return EPIC_OK;
}

extern "C" int epic_gpu_test_set_scatter_groups(epic_ctx* ctx, int lg_vol2grid, int lg_par2grid, int lg_stage) {
    if (!ctx) return EPIC_ERR_ARG;
    int v[3] = {lg_vol2grid, lg_par2grid, lg_stage};
    for (int k = 0; k < 3; ++k)
        if (v[k] < 0 || v[k] > 5) return EPIC_ERR_ARG;
    for (int k = 0; k < 3; ++k) ctx->c.scatter_lg[k] = v[k];
    return EPIC_OK;
}

extern "C" int epic_gpu_test_set_vectors_kernel(epic_ctx* ctx, int on) {
    if (!ctx) return EPIC_ERR_ARG;
    ctx->c.vectors_kernel = on != 0;
    return EPIC_OK;
}

extern "C" int epic_gpu_test_set_spectral_fp64(epic_ctx* ctx, int on) {
    if (!ctx) return EPIC_ERR_ARG;
    ctx->c.spectral_fp64 = on != 0;
    return EPIC_OK;
}

extern "C" int epic_gpu_test_set_stage_window(epic_ctx* ctx, int on) {
    if (!ctx) return EPIC_ERR_ARG;
    ctx->c.stage_recwin = on != 0;
    return EPIC_OK;
}

extern "C" int epic_gpu_test_set_stage_vectors(epic_ctx* ctx, int on) {
    if (!ctx) return EPIC_ERR_ARG;
    ctx->c.stage_vectors = on != 0;
    return EPIC_OK;
}

extern "C" int epic_gpu_test_drop_sort_store(epic_ctx* ctx) {
    if (!ctx) return EPIC_ERR_ARG;
    Ctx& c = ctx->c;
    if (c.pv_alt) {
        if (cudaStreamSynchronize(c.stream) != cudaSuccess || cudaFree(c.pv_alt) != cudaSuccess) return EPIC_ERR_CUDA;
        c.pv_alt = nullptr;
    }
    return EPIC_OK;
}
