// Exhaustive error of __sincosf on this GPU: every FP32 x with |x| <= 8
// (both signs), sine and cosine against the FP64 library.  Prints the
// largest absolute errors for |x| <= 4 and for |x| <= 8, and "ok" when the
// latter is within kSincosfAbsErr (csrc/umc_math64.cuh), the bound the FP32
// XY decisions use.  One launch, a grid-stride loop over the 2^30 or so bit
// patterns of each sign; the only store is an atomicMax per warp.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>

#include <cuda_runtime.h>

#include "umc_math64.cuh"

__global__ void sincosf_error(unsigned int* out)
{
    const uint32_t last = __float_as_uint(umc::kSincosfDomain);
    float e4 = 0.f, e8 = 0.f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= last; i += gridDim.x * blockDim.x) {
#pragma unroll
        for (uint32_t sign = 0; sign < 2; ++sign) {
            const float x = __uint_as_float(i | (sign << 31));
            float s, c;
            __sincosf(x, &s, &c);
            const double es = fabs(double(s) - sin(double(x))), ec = fabs(double(c) - cos(double(x)));
            const float e = __double2float_ru(fmax(es, ec));
            if (i <= 0x40800000u) e4 = fmaxf(e4, e);  // |x| <= 4
            e8 = fmaxf(e8, e);
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        e4 = fmaxf(e4, __shfl_xor_sync(0xffffffffu, e4, o));
        e8 = fmaxf(e8, __shfl_xor_sync(0xffffffffu, e8, o));
    }
    if ((threadIdx.x & 31u) == 0) {
        atomicMax(out + 0, __float_as_uint(e4));
        atomicMax(out + 1, __float_as_uint(e8));
    }
}

int main()
{
    unsigned int* d = nullptr;
    if (cudaMalloc(&d, 2 * sizeof(unsigned int)) != cudaSuccess) return 2;
    cudaMemset(d, 0, 2 * sizeof(unsigned int));
    sincosf_error<<<148 * 8, 256>>>(d);
    unsigned int h[2] = {0, 0};
    if (cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return 3;
    cudaFree(d);
    float e4, e8;
    memcpy(&e4, h, 4);
    memcpy(&e8, h + 1, 4);
    printf("max |err| |x|<=4: %a (2^%.3f)  |x|<=8: %a (2^%.3f)\n", e4, log2(double(e4)), e8, log2(double(e8)));
    if (double(e8) <= umc::kSincosfAbsErr) printf("ok\n");
    return 0;
}
