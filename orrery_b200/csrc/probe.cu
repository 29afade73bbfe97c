// Throughput probes for the direct kernel's roofline: FP32 FFMA lane
// operations per second and SFU reciprocal-square-root lane operations per
// second, measured on the device this process runs on. The reference measures
// its ceilings the same way rather than quoting a data sheet
// (benchmarks/cuda_probes.cu:15-115).
#include <cuda_runtime.h>

#include "common.cuh"
#include "orrery_b200.h"
#include "runtime.hpp"

namespace ob {
namespace {

constexpr int kChains = 8;
constexpr int kProbeThreads = 256;

__global__ void __launch_bounds__(kProbeThreads) ffma_probe(float *out, int iterations, float a,
                                                            float b) {
    float v[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) {
        v[k] = threadIdx.x * 1e-3f + k;
    }
    for (int it = 0; it < iterations; ++it) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) {
            v[k] = fmaf(v[k], a, b);
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) {
        s += v[k];
    }
    if (s == 12345.678f) {
        out[threadIdx.x] = s;
    }
}

// Packed FP32x2 FMA (sm_100 FFMA2): each instruction does two FMAs.
__global__ void __launch_bounds__(kProbeThreads) ffma2_probe(float *out, int iterations, float a,
                                                             float b) {
    float2 v[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) {
        v[k] = make_float2(threadIdx.x * 1e-3f + k, threadIdx.x * 2e-3f + k);
    }
    const float2 a2 = make_float2(a, a);
    const float2 b2 = make_float2(b, b);
    for (int it = 0; it < iterations; ++it) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) {
            v[k] = __ffma2_rn(v[k], a2, b2);
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) {
        s += v[k].x + v[k].y;
    }
    if (s == 12345.678f) {
        out[threadIdx.x] = s;
    }
}

__global__ void __launch_bounds__(kProbeThreads) rsqrt_probe(float *out, int iterations) {
    float v[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) {
        v[k] = 1.0f + threadIdx.x * 1e-3f + k;
    }
    for (int it = 0; it < iterations; ++it) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) {
            v[k] = rsqrt_approx(v[k]);
        }
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kChains; ++k) {
        s += v[k];
    }
    if (s == 12345.678f) {
        out[threadIdx.x] = s;
    }
}

// FP64 FMA (DFMA) lane operations: the FP64 pipe's rate, the denominator of
// the parity-mode tree walk's roofline.
__global__ void __launch_bounds__(kProbeThreads) dfma_probe(double *out, int iterations,
                                                            double a, double b) {
    double v[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) {
        v[k] = threadIdx.x * 1e-3 + k;
    }
    for (int it = 0; it < iterations; ++it) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) {
            v[k] = fma(v[k], a, b);
        }
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) {
        s += v[k];
    }
    if (s == 12345.678) {
        out[threadIdx.x] = s;
    }
}

template <typename Launch> double lane_ops_per_second(Launch launch, double ops) {
    cudaEvent_t a, b;
    check(cudaEventCreate(&a), "probe event");
    check(cudaEventCreate(&b), "probe event");
    launch();
    check(cudaGetLastError(), "probe launch");
    check(cudaEventRecord(a), "probe event");
    launch();
    check(cudaEventRecord(b), "probe event");
    check(cudaEventSynchronize(b), "probe");
    float ms = 0.0f;
    check(cudaEventElapsedTime(&ms, a, b), "probe timing");
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ops / (ms * 1e-3);
}

} // namespace
} // namespace ob

extern "C" int ob_probe_fp32x2(double *ffma2_flop_lanes_per_s) {
    try {
        int device = 0, sms = 0;
        ob::check(cudaGetDevice(&device), "cudaGetDevice");
        ob::check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SMs");
        float *sink = nullptr;
        ob::check(cudaMalloc(&sink, ob::kProbeThreads * sizeof(float)), "probe buffer");
        const int blocks = sms * 8;
        const double threads = static_cast<double>(blocks) * ob::kProbeThreads;
        const int iterations = 1 << 15;
        *ffma2_flop_lanes_per_s = ob::lane_ops_per_second(
            [&] {
                ob::ffma2_probe<<<blocks, ob::kProbeThreads>>>(sink, iterations, 0.999f, 1e-3f);
            },
            threads * iterations * ob::kChains * 2.0);
        cudaFree(sink);
        return OB_OK;
    } catch (const ob::Error &e) {
        return ob::set_error(e.code(), e.what());
    }
}

extern "C" int ob_probe_fp32(double *ffma_lane_per_s, double *rsqrt_lane_per_s) {
    try {
        int device = 0, sms = 0;
        ob::check(cudaGetDevice(&device), "cudaGetDevice");
        ob::check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SMs");
        float *sink = nullptr;
        ob::check(cudaMalloc(&sink, ob::kProbeThreads * sizeof(float)), "probe buffer");
        const int blocks = sms * 8;
        const double threads = static_cast<double>(blocks) * ob::kProbeThreads;
        const int fma_iterations = 1 << 16;
        const int rsq_iterations = 1 << 13;
        if (ffma_lane_per_s != nullptr) {
            *ffma_lane_per_s = ob::lane_ops_per_second(
                [&] {
                    ob::ffma_probe<<<blocks, ob::kProbeThreads>>>(sink, fma_iterations, 0.999f,
                                                                  1e-3f);
                },
                threads * fma_iterations * ob::kChains);
        }
        if (rsqrt_lane_per_s != nullptr) {
            *rsqrt_lane_per_s = ob::lane_ops_per_second(
                [&] { ob::rsqrt_probe<<<blocks, ob::kProbeThreads>>>(sink, rsq_iterations); },
                threads * rsq_iterations * ob::kChains);
        }
        cudaFree(sink);
        return OB_OK;
    } catch (const ob::Error &e) {
        return ob::set_error(e.code(), e.what());
    }
}

extern "C" int ob_probe_fp64(double *dfma_lane_per_s) {
    try {
        int device = 0, sms = 0;
        ob::check(cudaGetDevice(&device), "cudaGetDevice");
        ob::check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SMs");
        double *sink = nullptr;
        ob::check(cudaMalloc(&sink, ob::kProbeThreads * sizeof(double)), "probe buffer");
        const int blocks = sms * 8;
        const double threads = static_cast<double>(blocks) * ob::kProbeThreads;
        const int iterations = 1 << 14;
        *dfma_lane_per_s = ob::lane_ops_per_second(
            [&] { ob::dfma_probe<<<blocks, ob::kProbeThreads>>>(sink, iterations, 0.999, 1e-3); },
            threads * iterations * ob::kChains);
        cudaFree(sink);
        return OB_OK;
    } catch (const ob::Error &e) {
        return ob::set_error(e.code(), e.what());
    }
}
