// Arithmetic-pipe probe: independent FMA chains per thread, used to measure
// the FP32 and FP64 FMA throughput of the GPU that the assembly kernels are
// compared against (the roofline denominators).  No reference counterpart:
// it is a measurement utility of this library.
#include "common.cuh"

namespace bc {

template <typename T>
__global__ void __launch_bounds__(256) fma_chains(int64_t iters, T seed, T *sink) {
    T a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
    const T b = (T)0.999999, c = (T)1e-6;
    for (int64_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            a0 = a0 * b + c;
            a1 = a1 * b + c;
            a2 = a2 * b + c;
            a3 = a3 * b + c;
            a4 = a4 * b + c;
            a5 = a5 * b + c;
            a6 = a6 * b + c;
            a7 = a7 * b + c;
        }
    }
    const T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == (T)-12345.0) sink[blockIdx.x] = s;  // keeps the chains live
}

}  // namespace bc

extern "C" int bemppcuda_fma_probe(int32_t precision, int64_t iterations, int64_t blocks, void *sink, double *flops,
                                   void *stream) {
    if (iterations <= 0 || blocks <= 0 || blocks > (1 << 24) || !sink || !flops) {
        bc_set_error("fma_probe: bad arguments");
        return BEMPPCUDA_ERR_INVALID;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == BEMPPCUDA_FP64)
        bc::fma_chains<double><<<(unsigned)blocks, 256, 0, st>>>(iterations, 1.0, (double *)sink);
    else
        bc::fma_chains<float><<<(unsigned)blocks, 256, 0, st>>>(iterations, 1.0f, (float *)sink);
    *flops = 2.0 * 32.0 * (double)iterations * 256.0 * (double)blocks;
    return bc_check_launch("fma_probe");
}
