// Shared device/host definitions for the B200 growers.
//
// Everything here compiles with -fmad=false: the plain form promises results
// bit-identical to the reference's CPU grower, which is built with
// -ffp-contract=off, so no multiply-add may fuse anywhere in this library.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace bb
{

constexpr uint32_t k_leaf_flag = 0xFFFFFFFFu;

// The error the C ABI reports: "cuda: <what>: <cudaGetErrorString>", the
// reference's check() text (src/cuda/detail/device_buffer.cuh:96-103).
struct CudaError : std::runtime_error
{
    using std::runtime_error::runtime_error;
};

// A capacity or configuration refusal (the reference's ConfigError).
struct ConfigError : std::runtime_error
{
    using std::runtime_error::runtime_error;
};

inline void check(cudaError_t e, char const *what)
{
    if (e != cudaSuccess)
    {
        throw CudaError(std::string("cuda: ") + what + ": " + cudaGetErrorString(e));
    }
}

// Sets the calling thread's bb_last_error() text (defined with the C ABI).
void set_last_error(char const *msg);

#define BB_CHECK(call) ::bb::check((call), #call)
#define BB_LAUNCH(what) ::bb::check(cudaGetLastError(), what)

// Programmatic dependent launch. A kernel launched with the programmatic
// stream-serialization attribute may be scheduled while the kernel before it
// in the stream still runs; its first statement waits for that kernel's
// completion and memory (griddepcontrol.wait: a no-op for a kernel launched
// without the attribute), then lets the kernel after it be scheduled in turn.
// Nothing is read or written before the wait, so the order of effects is the
// plain stream order; what overlaps is the next grid's launch and the
// scheduling of its CTAs.
__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Launches kernel k like k<<<grid, block, smem, s>>>(args...), with the
// programmatic stream-serialization attribute when pdl is set (k must open
// with pdl_enter()).
template <typename... P, typename... A>
inline void launch_k(bool pdl, void (*k)(P...), dim3 grid, dim3 block, size_t smem,
                     cudaStream_t s, A &&...args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim          = grid;
    cfg.blockDim         = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream           = s;
    cudaLaunchAttribute at[1];
    at[0].id                                         = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs                                        = pdl ? at : nullptr;
    cfg.numAttrs                                     = pdl ? 1 : 0;
    check(cudaLaunchKernelEx(&cfg, k, static_cast<A &&>(args)...), "cudaLaunchKernelEx");
}

// ---- split math, restated from include/bonsai/split.hpp:112-158 ----------
// Double precision, IEEE round-to-nearest, no contraction (-fmad=false).

__host__ __device__ inline double l1_thresholded(double g, double l1)
{
    if (g > l1)
    {
        return g - l1;
    }
    if (g < -l1)
    {
        return g + l1;
    }
    return 0.0;
}

__host__ __device__ inline double split_score(double g, double h, double l1, double l2)
{
    double const t = l1_thresholded(g, l1);
    double const d = h + l2;
    return d > 0.0 ? (t * t) / d : 0.0;
}

__host__ __device__ inline double bounded_leaf_weight(double g, double h, double l1,
                                                      double l2, double lo, double hi)
{
    double const d = h + l2;
    double const w = d > 0.0 ? -l1_thresholded(g, l1) / d : 0.0;
    return w < lo ? lo : (hi < w ? hi : w);
}

// routes_left (include/bonsai/dataset.hpp:234-238): the last bin holds
// missing values and follows default_left; otherwise bin <= split_bin.
__host__ __device__ inline bool routes_left(uint32_t b, uint32_t last, uint32_t split,
                                            bool dl)
{
    return b == last ? dl : b <= split;
}

// Raw scores clamp to +-30 before the Poisson exp (k_poisson_max_log,
// include/bonsai/objective.hpp:47).
constexpr float k_poisson_max_log = 30.0F;

// The resident objectives' gradient pair at score s and label y
// (src/objective.cpp:44-58 squared error, 86-101 logistic loss, 267-278
// Poisson with a log link: g = exp(s) - y, h = exp(s), s clamped). Objective
// codes: 0 mse, 1 logloss, 3 poisson (2, softmax, has its own pass).
__device__ __forceinline__ float2 objective_gradient(int objective, float s, float y)
{
    if (objective == 0)
    {
        return make_float2(s - y, 1.0F);
    }
    if (objective == 3)
    {
        float const rate = expf(fminf(fmaxf(s, -k_poisson_max_log), k_poisson_max_log));
        return make_float2(rate - y, rate);
    }
    float const p = 1.0F / (1.0F + expf(-s));
    return make_float2(p - y, p * (1.0F - p));
}

// A weighted row scales both halves of its pair by its weight, one float
// multiply each (Booster::update_one_iter, include/bonsai/booster.hpp:546-555;
// the device form, src/cuda/detail/kernels.cuh:1001-1006); w == nullptr is
// the unweighted fit.
__device__ __forceinline__ float2 weighted(float2 g, float const *w, uint64_t r)
{
    if (w == nullptr)
    {
        return g;
    }
    float const x = w[r];
    return make_float2(g.x * x, g.y * x);
}

// Tree-level knobs the device reads (TreeConfig, include/bonsai/config/
// tree_config.hpp:9-29). Floats stay float: the reference widens them to
// double at each use, and so does every kernel here.
struct TreeParams
{
    float    min_child_hess;
    float    min_gain_to_split;
    float    lambda_l2;
    float    lambda_l1;
    uint32_t max_depth;
    uint32_t min_data_in_leaf;
    uint32_t max_leaves;
};

inline uint32_t ceil_div(uint64_t a, uint64_t b)
{
    return static_cast<uint32_t>((a + b - 1) / b);
}

} // namespace bb
