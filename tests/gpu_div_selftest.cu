// Self-test of the shared-reciprocal exact division of rp_device.cuh:
// compares rp_div_by(a, b, __drcp_rn(b)) with the IEEE quotient a / b.
#include <cstdint>
#include "rp_device.cuh"

__global__ void k_div(int64_t n, const double* a, const double* b, double* q, double* ref) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    q[i] = rp_div_by(a[i], b[i], rp_rcp(b[i]));
    ref[i] = a[i] / b[i];
}

extern "C" int div_selftest(int64_t n, const double* ha, const double* hb, double* hq, double* href) {
    double *a, *b, *q, *r;
    size_t bytes = (size_t)n * 8;
    if (cudaMalloc(&a, bytes) || cudaMalloc(&b, bytes) || cudaMalloc(&q, bytes) || cudaMalloc(&r, bytes)) return 1;
    cudaMemcpy(a, ha, bytes, cudaMemcpyHostToDevice);
    cudaMemcpy(b, hb, bytes, cudaMemcpyHostToDevice);
    k_div<<<(unsigned)((n + 255) / 256), 256>>>(n, a, b, q, r);
    cudaMemcpy(hq, q, bytes, cudaMemcpyDeviceToHost);
    cudaMemcpy(href, r, bytes, cudaMemcpyDeviceToHost);
    int err = cudaDeviceSynchronize() != cudaSuccess;
    cudaFree(a); cudaFree(b); cudaFree(q); cudaFree(r);
    return err;
}
