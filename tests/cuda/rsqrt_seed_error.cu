// Measures the maximum relative error of the double-precision approximate
// reciprocal square root instruction (PTX rsqrt.approx.ftz.f64) that seeds the
// FP64 force kernels' rsqrt (hermite_b200/csrc/hb_math.cuh), over 2^24
// log-spaced arguments in [1e-12, 1e12].  Used by tests/test_fp64_rsqrt.py.
#include <cmath>
#include <cstdio>

__global__ void seed_error(double lo, double hi, int n, unsigned long long *maxerr)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double x = exp(log(lo) + (log(hi) - log(lo)) * (i + 0.5) / n);
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    const double ref = 1.0 / sqrt(x);
    const double e = fabs(y - ref) / ref;   // non-negative: orders like its bits
    atomicMax(maxerr, (unsigned long long)__double_as_longlong(e));
}

int main()
{
    unsigned long long *d = nullptr;
    if (cudaMalloc(&d, sizeof(*d)) != cudaSuccess) return 1;
    cudaMemset(d, 0, sizeof(*d));
    const int n = 1 << 24;
    seed_error<<<n / 256, 256>>>(1e-12, 1e12, n, d);
    unsigned long long h = 0;
    cudaMemcpy(&h, d, sizeof(h), cudaMemcpyDeviceToHost);
    const double e = __builtin_bit_cast(double, h);
    std::printf("rsqrt.approx.ftz.f64 max relative error over [1e-12, 1e12], %d log-spaced x: "
                "%.3e (2^%.2f)\n", n, e, std::log2(e));
    cudaFree(d);
    return cudaDeviceSynchronize() != cudaSuccess;
}
