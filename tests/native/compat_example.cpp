// The reference's end-to-end call sequence (zmodel/main.cu:8-102: laplace -> forward ->
// inverse with scale 1/N^2) written against the compat header.  Built and run by
// tests/test_gpu_compat.py; reads the interleaved input from argv[1], writes the
// Laplacian, the spectrum and the round trip to argv[2..4].
#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "zmodel_compat.hpp"

int main(int argc, char **argv) {
    if (argc < 8) {
        std::fprintf(stderr, "usage: %s in lap spec back N B P\n", argv[0]);
        return 2;
    }
    const long long n = std::atoll(argv[5]), b = std::atoll(argv[6]), p = std::atoll(argv[7]);
    const size_t elems = (size_t)n * n, bytes = elems * sizeof(zmodel_b200::Complex);
    std::vector<zmodel_b200::Complex> host(elems);
    FILE *f = std::fopen(argv[1], "rb");
    if (!f || std::fread(host.data(), 1, bytes, f) != bytes) return 3;
    std::fclose(f);

    zmodel_b200::FftHostPlans plans;
    zmodel_b200::init_plans(plans, n, b, p);
    zmodel_b200::FftBuffers buffers;
    void *lap = nullptr;
    if (cudaMalloc(&buffers.device_buf0, bytes) || cudaMalloc(&buffers.device_buf1, bytes) ||
        cudaMalloc(&lap, bytes))
        return 4;
    cudaMemcpy(buffers.device_buf0, host.data(), bytes, cudaMemcpyHostToDevice);

    auto dump = [&](const void *dev, const char *path) {
        cudaMemcpy(host.data(), dev, bytes, cudaMemcpyDeviceToHost);
        FILE *o = std::fopen(path, "wb");
        std::fwrite(host.data(), 1, bytes, o);
        std::fclose(o);
    };
    // Laplace routine (main.cu:50-58): no pack / communicate step any more
    zmodel_b200::laplace(buffers.device_buf0, lap, plans);
    dump(lap, argv[2]);
    // main.cu:62: FFT input is buf0
    cudaMemcpy(buffers.device_buf0, lap, bytes, cudaMemcpyDeviceToDevice);
    zmodel_b200::forward_fft<true>(buffers, plans);
    dump(buffers.device_buf1, argv[3]);
    // main.cu:74-80: IFFT input is buf0, scale 1/N^2
    cudaMemcpy(buffers.device_buf0, buffers.device_buf1, bytes, cudaMemcpyDeviceToDevice);
    const double s = 1.0 / ((double)n * (double)n);
    zmodel_b200::inverse_fft<true>(buffers, zmodel_b200::Complex{s, 0.0}, plans);
    dump(buffers.device_buf1, argv[4]);
    int ky, kx;
    zmodel_b200::reciprocal_to_global(plans, 0, 0, 1, 2, ky, kx);
    std::printf("reciprocal_to_global(0,0,1,2) = (%d, %d)\n", ky, kx);
    zmodel_b200::destroy_plans(plans);
    cudaFree(buffers.device_buf0);
    cudaFree(buffers.device_buf1);
    cudaFree(lap);
    return 0;
}
