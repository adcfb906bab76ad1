// Test helper (not product): runs the device point-wise routines of
// dgsem_device.cuh -- the Newton-refined reciprocal and the logarithmic mean --
// over host arrays, beside CUDA's own IEEE division, so a test can sweep them.
// Built by tests/test_gpu_device_math.py with nvcc into a temporary folder.
#include <cuda_runtime.h>

#include "../../prandtl_b200/csrc/dgsem_device.cuh"

namespace {

template <typename T>
__global__ void rcp_kernel(const T *x, T *ours, T *div, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        ours[i] = prandtl::rcp(x[i]);
        div[i] = T(1) / x[i];   // IEEE round-to-nearest division
    }
}

template <typename T>
__global__ void log_mean_kernel(const T *x, const T *y, T *mean, T *inv_mean, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        T m, im, rs;
        prandtl::log_mean<T>(x[i], y[i], prandtl::rcp(x[i]), m, im, rs);
        mean[i] = m;
        inv_mean[i] = im;
    }
}

template <typename T>
int run_rcp(const T *x, T *ours, T *div, int n) {
    T *d = nullptr;
    if (n <= 0) return 1;
    if (cudaMalloc(&d, 3 * sizeof(T) * (size_t)n) != cudaSuccess) return 2;
    int rc = 0;
    if (cudaMemcpy(d, x, sizeof(T) * n, cudaMemcpyHostToDevice) != cudaSuccess) rc = 3;
    if (!rc) {
        rcp_kernel<T><<<(n + 255) / 256, 256>>>(d, d + n, d + 2 * (size_t)n, n);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) rc = 4;
    }
    if (!rc && (cudaMemcpy(ours, d + n, sizeof(T) * n, cudaMemcpyDeviceToHost) != cudaSuccess ||
                cudaMemcpy(div, d + 2 * (size_t)n, sizeof(T) * n, cudaMemcpyDeviceToHost) != cudaSuccess))
        rc = 5;
    cudaFree(d);
    return rc;
}

template <typename T>
int run_log_mean(const T *x, const T *y, T *mean, T *inv_mean, int n) {
    T *d = nullptr;
    if (n <= 0) return 1;
    if (cudaMalloc(&d, 4 * sizeof(T) * (size_t)n) != cudaSuccess) return 2;
    int rc = 0;
    if (cudaMemcpy(d, x, sizeof(T) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d + n, y, sizeof(T) * n, cudaMemcpyHostToDevice) != cudaSuccess)
        rc = 3;
    if (!rc) {
        log_mean_kernel<T><<<(n + 255) / 256, 256>>>(d, d + n, d + 2 * (size_t)n, d + 3 * (size_t)n, n);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) rc = 4;
    }
    if (!rc && (cudaMemcpy(mean, d + 2 * (size_t)n, sizeof(T) * n, cudaMemcpyDeviceToHost) != cudaSuccess ||
                cudaMemcpy(inv_mean, d + 3 * (size_t)n, sizeof(T) * n, cudaMemcpyDeviceToHost) != cudaSuccess))
        rc = 5;
    cudaFree(d);
    return rc;
}

}   // namespace

extern "C" {
int dm_rcp64(const double *x, double *ours, double *div, int n) { return run_rcp<double>(x, ours, div, n); }
int dm_rcp32(const float *x, float *ours, float *div, int n) { return run_rcp<float>(x, ours, div, n); }
int dm_log_mean64(const double *x, const double *y, double *m, double *im, int n) {
    return run_log_mean<double>(x, y, m, im, n);
}
int dm_log_mean32(const float *x, const float *y, float *m, float *im, int n) {
    return run_log_mean<float>(x, y, m, im, n);
}
}
