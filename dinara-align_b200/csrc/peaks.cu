// A measured int32 roofline for this device: the rate at which the SMs retire the integer instructions
// the sweeps are made of (DPX add-and-max, min/max, three-input add), from independent chains that keep
// every pipe busy. No published figure stands in for it.
#include "internal.cuh"

namespace dinara {
namespace {

constexpr int kChains = 8;

template <int KIND>
__global__ void __launch_bounds__(256) peak_kernel(int32_t seed, int32_t step, int iterations, int32_t *out) {
    int32_t x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = seed + int32_t(threadIdx.x) * (c + 1);
    const int32_t a = step, b = seed ^ 0x5a5a;
    for (int i = 0; i < iterations; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) {
            if (KIND == 0) x[c] = __viaddmax_s32(x[c], a, x[(c + 1) % kChains]);  // max(x + a, y)
            if (KIND == 1) x[c] = max(x[c], x[(c + 1) % kChains] - b);             // IMNMX (+ IADD)
            if (KIND == 2) x[c] = x[c] + x[(c + 1) % kChains] + a;                  // IADD3
            if (KIND == 3) x[c] = int32_t(__viaddmax_s16x2(uint32_t(x[c]), uint32_t(a), uint32_t(x[(c + 1) % kChains])));
            if (KIND == 4) x[c] = __vimax3_s32(x[c], x[(c + 1) % kChains], x[(c + 3) % kChains]);
            if (KIND == 5)
                x[c] = int32_t(__vimax3_s16x2(uint32_t(x[c]), uint32_t(x[(c + 1) % kChains]),
                                              uint32_t(x[(c + 3) % kChains])));
            if (KIND == 6) x[c] = int32_t(__byte_perm(uint32_t(x[c]), uint32_t(x[(c + 1) % kChains]), uint32_t(b)));
            if (KIND == 7) x[c] = max(x[c], x[(c + 1) % kChains]);                 // IMNMX alone
            if (KIND == 8) x[c] = int32_t(__vcmpgts2(uint32_t(x[c]), uint32_t(x[(c + 1) % kChains]))) + a;
            if (KIND == 9) {
                bool high = false, low = false;
                x[c] = int32_t(__vibmax_s16x2(uint32_t(x[c]), uint32_t(x[(c + 1) % kChains]), &high, &low));
                x[c] ^= int32_t(low);
            }
            if (KIND == 10)
                x[c] = int32_t(__viaddmax_s16x2_relu(uint32_t(x[c]), uint32_t(a), uint32_t(x[(c + 1) % kChains])));
            if (KIND == 11) x[c] = int32_t(__vsub2(uint32_t(x[c]), uint32_t(x[(c + 1) % kChains])));
        }
    }
    int32_t folded = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) folded ^= x[c];
    if (folded == 0x7fffffff) out[0] = folded;
}

}  // namespace
}  // namespace dinara

extern "C" int64_t dinara_gpu_int32_peak(dinara_gpu *gpu, int64_t kind, double *instructions_per_second) {
    using namespace dinara;
    if (!gpu || !instructions_per_second) return DINARA_INVALID_MODE;
    try {
        DINARA_CUDA(cudaSetDevice(gpu->device));
        int32_t *sink = gpu->counters.ensure<int32_t>(64);
        const int blocks = gpu->multiprocessors * 8, threads = 256, iterations = 4096;
        if (kind < 0 || kind > 11) return DINARA_INVALID_MODE;
        void (*const kernels[])(int32_t, int32_t, int, int32_t *) = {
            &peak_kernel<0>, &peak_kernel<1>, &peak_kernel<2>, &peak_kernel<3>,
            &peak_kernel<4>, &peak_kernel<5>, &peak_kernel<6>, &peak_kernel<7>,
            &peak_kernel<8>, &peak_kernel<9>, &peak_kernel<10>, &peak_kernel<11>};
        void (*fn)(int32_t, int32_t, int, int32_t *) = kernels[kind];
        fn<<<blocks, threads, 0, gpu->stream>>>(3, 1, 64, sink);  // warm-up
        DINARA_CUDA(cudaEventRecord(gpu->start, gpu->stream));
        fn<<<blocks, threads, 0, gpu->stream>>>(3, 1, iterations, sink);
        DINARA_CUDA(cudaEventRecord(gpu->stop, gpu->stream));
        DINARA_CUDA(cudaEventSynchronize(gpu->stop));
        float ms = 0.f;
        DINARA_CUDA(cudaEventElapsedTime(&ms, gpu->start, gpu->stop));
        // The counted instructions: one a chain step (kind 1: the subtraction is a second one). Kinds: 0
        // viaddmax, 1 max after a subtraction, 2 three-input add, 3 viaddmax on 16-bit pairs, 4 three-way
        // max, 5 three-way max on 16-bit pairs, 6 byte permute, 7 max alone, 8 16-bit pair compare to a
        // mask (and an add), 9 16-bit pair max with its predicates (one folded back), 10 kind 3 floored at
        // zero, 11 16-bit pair subtraction.
        const double per_step = kind == 1 ? 2.0 : 1.0;
        const double instructions = double(blocks) * threads * iterations * kChains * per_step;
        *instructions_per_second = instructions / (double(ms) * 1e-3);
        return 0;
    } catch (const Failure &failure) {
        gpu->error = failure.what();
        return failure.code;
    }
}
