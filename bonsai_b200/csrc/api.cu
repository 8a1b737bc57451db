// The C ABI (include/bonsai_b200.h): planes, the device-resident booster,
// single-tree growth and ensemble predict.
#include "bonsai_b200.h"
#include "shard.cuh"
#include "grow.cuh"
#include "ingest.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <future>
#include <iterator>
#include <memory>
#include <mutex>
#include <numeric>
#include <random>
#include <string>
#include <vector>

struct bb_plane
{
    bb::Plane p;
};

namespace bb
{
namespace
{

thread_local std::string g_err;

} // namespace

void set_last_error(char const *msg)
{
    g_err = msg;
}

namespace
{

template <typename F> int guarded(F &&f)
{
    try
    {
        f();
        g_err.clear();
        return BB_OK;
    }
    catch (CudaError const &e)
    {
        g_err = e.what();
        return BB_ERR_CUDA;
    }
    catch (ConfigError const &e)
    {
        g_err = e.what();
        return BB_ERR_CONFIG;
    }
    catch (std::invalid_argument const &e)
    {
        g_err = e.what();
        return BB_ERR_ARG;
    }
    catch (std::exception const &e)
    {
        g_err = e.what();
        return BB_ERR_CUDA;
    }
}

void need(bool ok, char const *what)
{
    if (!ok)
    {
        throw std::invalid_argument(what);
    }
}

// ---- objectives (the resident gradient kernel) ----------------------------
// mse: g = s - y, h = 1 (src/objective.cpp:44-58); logloss: p = 1/(1+e^-s),
// g = p - y, h = p(1-p) (src/objective.cpp:86-101).
__global__ void gradient_kernel(int objective, float const *__restrict__ scores,
                                float const *__restrict__ labels, float2 *__restrict__ gh,
                                uint64_t n, float const *__restrict__ weights)
{
    uint64_t const i = (static_cast<uint64_t>(blockIdx.x) * blockDim.x) + threadIdx.x;
    if (i >= n)
    {
        return;
    }
    gh[i] = weighted(objective_gradient(objective, scores[i], labels[i]), weights, i);
}

// Softmax gradients for K classes (MulticlassBooster::update_one_iter,
// include/bonsai/multiclass_booster.hpp:105-140, row_softmax_exp :525-541):
// per row the double max of its class scores, e_k = exp(s_k - max) in
// double, summed in class order; p_k = float(e_k) / float(sum); g = p - 1[y
// == k], h = max(p (1 - p), 1e-6). Scores and pairs are class-major (k * n + i).
constexpr uint32_t k_max_classes = 16;

__global__ void softmax_gradient_kernel(float const *__restrict__ scores,
                                        float const *__restrict__ labels,
                                        float2 *__restrict__ gh, uint64_t n, uint32_t K,
                                        float const *__restrict__ weights)
{
    uint64_t const i = (static_cast<uint64_t>(blockIdx.x) * blockDim.x) + threadIdx.x;
    if (i >= n)
    {
        return;
    }
    double maxv = scores[i];
    for (uint32_t k = 1; k < K; ++k)
    {
        maxv = fmax(maxv, static_cast<double>(scores[(k * n) + i]));
    }
    double e[k_max_classes];
    double sum = 0.0;
    for (uint32_t k = 0; k < K; ++k)
    {
        e[k] = exp(static_cast<double>(scores[(k * n) + i]) - maxv);
        sum += e[k];
    }
    long const    lab = lround(labels[i]);
    uint32_t const c  = lab >= 0 && static_cast<uint64_t>(lab) < K ? static_cast<uint32_t>(lab) : 0;
    float const   fs  = static_cast<float>(sum);
    for (uint32_t k = 0; k < K; ++k)
    {
        float const p = static_cast<float>(e[k]) / fs;
        float const y = c == k ? 1.0F : 0.0F;
        gh[(k * n) + i] = weighted(make_float2(p - y, fmaxf(p * (1.0F - p), 1e-6F)), weights, i);
    }
}

// ---- the validation plane ------------------------------------------------
// CudaDeviceContext::eval_begin / eval_accumulate (src/cuda/detail/
// device_context.cu:1666-1760): each round walks its new tree(s) over the
// validation rows, adds lr x leaf to their scores (scores[i] += lr * value,
// accumulate_last_round, include/bonsai/booster.hpp:995-1006) and records the
// round's loss -- without leaving the device, so it runs inside the round's
// CUDA graph. The loss terms are the reference's device forms
// (eval_loss_pass1_kernel, src/cuda/detail/kernels.cuh:1062-1103: squared
// error in FP64, logloss in float), and softmax cross-entropy from the
// double max and exp of logloss_from_scores (include/bonsai/
// multiclass_booster.hpp:545-559); per-row terms summed in FP64 in a fixed
// order (grid-stride per thread, a fixed tree per block, blocks in order).

constexpr uint32_t k_eval_threads = 256;
constexpr uint32_t k_eval_blocks  = 1024;

template <typename BinT>
__global__ void __launch_bounds__(k_eval_threads)
    eval_walk_kernel(BinT const *__restrict__ bins, uint64_t n_pad, uint64_t n,
                     uint32_t const *__restrict__ n_bins, TreeOut slots, uint32_t cap,
                     uint32_t const *round, uint32_t K, float lr, int objective,
                     float const *__restrict__ labels, float *__restrict__ vs,
                     double *__restrict__ partial)
{
    __shared__ double red[k_eval_threads];
    uint32_t const    t_end = *round; // this round's trees are [t_end - K, t_end)
    double            acc   = 0.0;
    for (uint64_t r = (static_cast<uint64_t>(blockIdx.x) * blockDim.x) + threadIdx.x; r < n;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    {
        for (uint32_t k = 0; k < K; ++k)
        {
            uint64_t const off = static_cast<uint64_t>(t_end - K + k) * cap;
            uint32_t       idx = 0;
            for (uint32_t step = 0; step < cap && slots.feature[off + idx] != k_leaf_flag; ++step)
            {
                uint32_t const f = slots.feature[off + idx];
                uint32_t const b = bins[(static_cast<uint64_t>(f) * n_pad) + r];
                idx = routes_left(b, n_bins[f] - 1, slots.split_bin[off + idx],
                                  slots.default_left[off + idx] != 0)
                          ? slots.left[off + idx]
                          : slots.right[off + idx];
            }
            float *sk = vs + (static_cast<uint64_t>(k) * n) + r;
            *sk       = *sk + (lr * slots.value[off + idx]);
        }
        float const y = labels[r];
        if (objective == 0)
        {
            double const d = static_cast<double>(vs[r]) - static_cast<double>(y);
            acc += d * d;
        }
        else if (objective == 1)
        {
            float const s  = vs[r];
            float const ax = fabsf(s);
            acc += fmaxf(0.0F, s) + log1pf(expf(-ax)) - (y * s);
        }
        else if (objective == 3)
        {
            // Poisson NLL up to a label-only constant, the raw score clamped
            float const f = fminf(fmaxf(vs[r], -k_poisson_max_log), k_poisson_max_log);
            acc += static_cast<double>(expf(f)) - (static_cast<double>(y) * static_cast<double>(f));
        }
        else
        {
            double maxv = vs[r];
            for (uint32_t k = 1; k < K; ++k)
            {
                maxv = fmax(maxv, static_cast<double>(vs[(static_cast<uint64_t>(k) * n) + r]));
            }
            double sum = 0.0;
            for (uint32_t k = 0; k < K; ++k)
            {
                sum += exp(static_cast<double>(vs[(static_cast<uint64_t>(k) * n) + r]) - maxv);
            }
            long const     lab = lround(y);
            uint32_t const c =
                lab >= 0 && static_cast<uint64_t>(lab) < K ? static_cast<uint32_t>(lab) : 0;
            acc -= (static_cast<double>(vs[(static_cast<uint64_t>(c) * n) + r]) - maxv) - log(sum);
        }
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (uint32_t w = k_eval_threads / 2; w > 0; w >>= 1)
    {
        if (threadIdx.x < w)
        {
            red[threadIdx.x] += red[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        partial[blockIdx.x] = red[0];
    }
}

// The round's loss: the block partials in block order, / n, as float, into
// losses[*count] (count advances; rounds past cap are not recorded).
__global__ void eval_finish_kernel(double const *partial, uint32_t n_blocks, uint64_t n,
                                   float *losses, uint32_t *count, uint32_t cap)
{
    if (threadIdx.x != 0 || blockIdx.x != 0)
    {
        return;
    }
    double total = 0.0;
    for (uint32_t b = 0; b < n_blocks; ++b)
    {
        total += partial[b];
    }
    uint32_t const c = *count;
    if (c < cap)
    {
        losses[c] = static_cast<float>(total / static_cast<double>(n));
    }
    *count = c + 1;
}

__global__ void iota_kernel(uint32_t *rows, uint64_t n)
{
    uint64_t const i = (static_cast<uint64_t>(blockIdx.x) * blockDim.x) + threadIdx.x;
    if (i < n)
    {
        rows[i] = static_cast<uint32_t>(i);
    }
}

__global__ void fill_kernel(float *x, float v, uint64_t n)
{
    uint64_t const i = (static_cast<uint64_t>(blockIdx.x) * blockDim.x) + threadIdx.x;
    if (i < n)
    {
        x[i] = v;
    }
}

// Copies the scratch tree into slot *round and advances the round counter,
// so a captured boosting round needs no per-round pointer.
__global__ void commit_tree_kernel(TreeOut scratch, TreeOut slots, uint32_t cap,
                                   uint32_t *round)
{
    uint32_t const r   = *round;
    uint64_t const off = static_cast<uint64_t>(r) * cap;
    for (uint32_t i = threadIdx.x; i < cap; i += blockDim.x)
    {
        slots.feature[off + i]      = scratch.feature[i];
        slots.value[off + i]        = scratch.value[i];
        slots.left[off + i]         = scratch.left[i];
        slots.right[off + i]        = scratch.right[i];
        slots.default_left[off + i] = scratch.default_left[i];
        slots.gain[off + i]         = scratch.gain[i];
        slots.cover[off + i]        = scratch.cover[i];
        slots.split_bin[off + i]    = scratch.split_bin[i];
    }
    if (threadIdx.x < 3)
    {
        slots.meta[(3 * static_cast<uint64_t>(r)) + threadIdx.x] = scratch.meta[threadIdx.x];
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        *round = r + 1;
    }
}

template <typename T> T *dmalloc(size_t n)
{
    void *p = nullptr;
    BB_CHECK(cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(T)));
    return static_cast<T *>(p);
}

struct TreeStore
{
    uint32_t cap  = 0;
    uint32_t n    = 0;
    TreeOut  t{};
    void     alloc(uint32_t capacity, uint32_t slots)
    {
        cap                = capacity;
        n                  = slots;
        size_t const total = static_cast<size_t>(capacity) * slots;
        t.feature          = dmalloc<uint32_t>(total);
        t.value            = dmalloc<float>(total);
        t.left             = dmalloc<uint32_t>(total);
        t.right            = dmalloc<uint32_t>(total);
        t.default_left     = dmalloc<uint8_t>(total);
        t.gain             = dmalloc<float>(total);
        t.cover            = dmalloc<float>(total);
        t.split_bin        = dmalloc<uint32_t>(total);
        t.meta             = dmalloc<uint32_t>(3 * static_cast<size_t>(slots));
    }
    void release()
    {
        void *ps[] = {t.feature, t.value,     t.left, t.right, t.default_left,
                      t.gain,    t.cover,     t.split_bin, t.meta};
        for (void *p : ps)
        {
            if (p != nullptr)
            {
                cudaFree(p);
            }
        }
        t = {};
    }
    // slots [slot, slot + count), each array's entries back to back
    void download(uint32_t slot, uint32_t *feature, float *value, uint32_t *left,
                  uint32_t *right, uint8_t *dl, float *gain, float *cover,
                  uint32_t *split_bin, uint32_t *meta, uint32_t count = 1) const
    {
        size_t const o = static_cast<size_t>(slot) * cap;
        size_t const m = static_cast<size_t>(count) * cap;
        BB_CHECK(cudaMemcpy(feature, t.feature + o, m * 4, cudaMemcpyDeviceToHost));
        BB_CHECK(cudaMemcpy(value, t.value + o, m * 4, cudaMemcpyDeviceToHost));
        BB_CHECK(cudaMemcpy(left, t.left + o, m * 4, cudaMemcpyDeviceToHost));
        BB_CHECK(cudaMemcpy(right, t.right + o, m * 4, cudaMemcpyDeviceToHost));
        BB_CHECK(cudaMemcpy(dl, t.default_left + o, m, cudaMemcpyDeviceToHost));
        BB_CHECK(cudaMemcpy(gain, t.gain + o, m * 4, cudaMemcpyDeviceToHost));
        BB_CHECK(cudaMemcpy(cover, t.cover + o, m * 4, cudaMemcpyDeviceToHost));
        BB_CHECK(cudaMemcpy(split_bin, t.split_bin + o, m * 4, cudaMemcpyDeviceToHost));
        BB_CHECK(cudaMemcpy(meta, t.meta + (3 * static_cast<size_t>(slot)), 12 * count,
                            cudaMemcpyDeviceToHost));
    }
};

GrowConfig grow_config(bb_train_cfg const &c)
{
    need(c.grower >= 0 && c.grower <= 2,
         "grower must be 0 (depthwise), 1 (levelwise) or 2 (leafwise)");
    need(c.grower == 2 ? c.max_depth <= 255 : c.max_depth <= 8,
         "max_depth must be <= 8 on the device level plane (leafwise: <= 255)");
    need(c.hist_mode >= 0 && c.hist_mode <= 2, "hist_mode must be 0, 1 or 2");
    if (c.grower == 1)
    {
        for (uint32_t f = 0; c.monotone != nullptr && f < c.n_monotone; ++f)
        {
            if (c.monotone[f] != 0)
            {
                // ObliviousGrower's constructor (src/grower_impl.hpp:582-590)
                throw ConfigError("monotone_constraints are not supported by the levelwise "
                                  "grower");
            }
        }
    }
    GrowConfig g;
    g.level                = c.grower == 1;
    g.leaf                 = c.grower == 2;
    g.tp.min_child_hess    = c.min_child_hess;
    g.tp.min_gain_to_split = c.min_gain_to_split;
    g.tp.lambda_l2         = c.lambda_l2;
    g.tp.lambda_l1         = c.lambda_l1;
    g.tp.max_depth         = c.max_depth;
    g.tp.min_data_in_leaf  = c.min_data_in_leaf;
    g.tp.max_leaves        = c.grower == 2 ? c.max_leaves : 0;
    g.mode                 = static_cast<HistMode>(c.hist_mode);
    g.hist_ctas            = c.hist_ctas;
    return g;
}

std::vector<uint32_t> selection(bb_train_cfg const &c, uint32_t F)
{
    std::vector<uint32_t> sel;
    if (c.selected == nullptr)
    {
        sel.resize(F);
        std::iota(sel.begin(), sel.end(), 0U);
        return sel;
    }
    sel.assign(c.selected, c.selected + c.n_selected);
    for (size_t i = 0; i < sel.size(); ++i)
    {
        need(sel[i] < F, "selected feature out of range");
        need(i == 0 || sel[i] > sel[i - 1], "selected features must be ascending");
    }
    return sel;
}

std::vector<int8_t> monotone(bb_train_cfg const &c)
{
    if (c.monotone == nullptr)
    {
        return {};
    }
    return {c.monotone, c.monotone + c.n_monotone};
}

// Interaction constraints (TreeConfig::interaction_constraints, parsed by
// parse_interaction_groups, src/grower_impl.hpp:83-109): group g holds
// features[offsets[g] .. offsets[g + 1]); per feature, the bit mask of the
// groups containing it. Empty groups are dropped, as the reference drops them.
std::vector<uint64_t> interaction(bb_train_cfg const &c, uint32_t n_feats)
{
    if (c.n_interaction_groups == 0)
    {
        return {};
    }
    need(c.interaction_offsets != nullptr, "interaction constraints: null offset array");
    need(c.interaction_offsets[c.n_interaction_groups] == c.interaction_offsets[0] ||
             c.interaction_features != nullptr,
         "interaction constraints: null feature array");
    std::vector<uint64_t> masks(n_feats, 0);
    uint32_t              g = 0;
    for (uint32_t k = 0; k < c.n_interaction_groups; ++k)
    {
        uint32_t const b = c.interaction_offsets[k];
        uint32_t const e = c.interaction_offsets[k + 1];
        need(b <= e, "interaction constraints: offsets must not decrease");
        if (b == e)
        {
            continue;
        }
        if (g >= 64)
        {
            throw ConfigError("interaction constraints: at most 64 non-empty groups");
        }
        for (uint32_t x = b; x < e; ++x)
        {
            need(c.interaction_features[x] < n_feats,
                 "interaction constraints: feature id out of range");
            masks[c.interaction_features[x]] |= uint64_t{1} << g;
        }
        ++g;
    }
    if (g == 0)
    {
        return {};
    }
    return masks;
}

uint32_t blocks(uint64_t n, uint32_t t = 256)
{
    return ceil_div(std::max<uint64_t>(n, 1), t);
}

// ---- the row sample ---------------------------------------------------------
// BernoulliSampler::sample (src/sampler.cpp:36-55) keeps row i when
// std::bernoulli_distribution(p) says so, drawing row by row from the
// booster's std::mt19937 (seeded with booster_config.random_seed,
// include/bonsai/booster.hpp:496), one draw per tree (per class tree in a
// softmax round, include/bonsai/multiclass_booster.hpp:138). The draw stays on
// the host in exactly those library calls -- one sequential generator stream
// -- and runs a round ahead on a worker thread; the device receives one bit
// per row and compacts the bits into the ascending row list the grower's root
// takes.

constexpr uint32_t k_smp_threads = 256;
constexpr uint32_t k_smp_words   = 4;                              // mask words per thread
constexpr uint32_t k_smp_block   = k_smp_threads * k_smp_words;     // mask words per block
constexpr uint32_t k_scan_threads = 1024;

// Exclusive prefix sum of v over the block; total receives the block's sum.
template <uint32_t T> __device__ __forceinline__ uint32_t block_scan(uint32_t v, uint32_t &total)
{
    __shared__ uint32_t warp_s[T / 32];
    uint32_t const      lane = threadIdx.x & 31;
    uint32_t const      wid  = threadIdx.x >> 5;
    uint32_t            x    = v;
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1)
    {
        uint32_t const y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        x += lane >= o ? y : 0u;
    }
    if (lane == 31)
    {
        warp_s[wid] = x;
    }
    __syncthreads();
    uint32_t base = 0;
    total         = 0;
    for (uint32_t w = 0; w < T / 32; ++w)
    {
        uint32_t const c = warp_s[w];
        base += w < wid ? c : 0u;
        total += c;
    }
    __syncthreads();
    return base + x - v;
}

__device__ __forceinline__ uint32_t thread_words(uint32_t const *bits, uint64_t n_words,
                                                 uint64_t w0, uint32_t w[k_smp_words])
{
    uint32_t c = 0;
#pragma unroll
    for (uint32_t j = 0; j < k_smp_words; ++j)
    {
        w[j] = w0 + j < n_words ? bits[w0 + j] : 0u;
        c += __popc(w[j]);
    }
    return c;
}

// Pass 1: each block's kept rows.
__global__ void __launch_bounds__(k_smp_threads)
    sample_count_kernel(uint32_t const *__restrict__ bits, uint64_t n_words,
                        uint32_t *__restrict__ bsum)
{
    uint32_t       w[k_smp_words];
    uint64_t const w0 = (static_cast<uint64_t>(blockIdx.x) * k_smp_block) +
                        (static_cast<uint64_t>(threadIdx.x) * k_smp_words);
    uint32_t       total = 0;
    block_scan<k_smp_threads>(thread_words(bits, n_words, w0, w), total);
    if (threadIdx.x == 0)
    {
        bsum[blockIdx.x] = total;
    }
}

// Pass 2 (one block): the blocks' offsets in place, and the sample's size.
__global__ void __launch_bounds__(k_scan_threads)
    sample_scan_kernel(uint32_t *bsum, uint32_t n_blocks, uint32_t *count)
{
    uint32_t carry = 0;
    for (uint32_t b0 = 0; b0 < n_blocks; b0 += k_scan_threads)
    {
        uint32_t const i     = b0 + threadIdx.x;
        uint32_t const v     = i < n_blocks ? bsum[i] : 0u;
        uint32_t       total = 0;
        uint32_t const ex    = block_scan<k_scan_threads>(v, total);
        if (i < n_blocks)
        {
            bsum[i] = carry + ex;
        }
        carry += total;
    }
    if (threadIdx.x == 0)
    {
        *count = carry;
    }
}

// Pass 3: every kept row's id at its rank, so the list is ascending.
__global__ void __launch_bounds__(k_smp_threads)
    sample_list_kernel(uint32_t const *__restrict__ bits, uint64_t n_words,
                       uint32_t const *__restrict__ boff, uint32_t *__restrict__ rows)
{
    uint32_t       w[k_smp_words];
    uint64_t const w0 = (static_cast<uint64_t>(blockIdx.x) * k_smp_block) +
                        (static_cast<uint64_t>(threadIdx.x) * k_smp_words);
    uint32_t       total = 0;
    uint32_t       pos   = boff[blockIdx.x] +
                   block_scan<k_smp_threads>(thread_words(bits, n_words, w0, w), total);
#pragma unroll
    for (uint32_t j = 0; j < k_smp_words; ++j)
    {
        uint32_t x = w[j];
        while (x != 0u)
        {
            uint32_t const b = __ffs(static_cast<int>(x)) - 1;
            rows[pos++]      = static_cast<uint32_t>(((w0 + j) << 5) + b);
            x &= x - 1u;
        }
    }
}

// The leafwise plane stamps the sampled rows from its leaves' segments; the
// rest walk the finished tree (route_unsampled, src/grower_impl.hpp:438-461:
// routes_left on the split bin, the last bin following default_left) over the
// feature-major codes and take the same update, scores[r] + lr x value.
template <typename BinT>
__global__ void __launch_bounds__(256)
    route_unsampled_kernel(BinT const *__restrict__ bins, uint64_t n_pad, uint64_t n,
                           uint32_t const *__restrict__ n_bins, TreeOut t, uint32_t cap,
                           uint32_t const *__restrict__ sbits, float *__restrict__ scores,
                           uint32_t *__restrict__ leaf_id, float lr)
{
    for (uint64_t r = (static_cast<uint64_t>(blockIdx.x) * blockDim.x) + threadIdx.x; r < n;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    {
        if (((sbits[r >> 5] >> (r & 31)) & 1u) != 0)
        {
            continue;
        }
        uint32_t idx = 0;
        for (uint32_t step = 0; step < cap && t.feature[idx] != k_leaf_flag; ++step)
        {
            uint32_t const f = t.feature[idx];
            uint32_t const b = bins[(static_cast<uint64_t>(f) * n_pad) + r];
            idx = routes_left(b, n_bins[f] - 1, t.split_bin[idx], t.default_left[idx] != 0)
                      ? t.left[idx]
                      : t.right[idx];
        }
        scores[r] = scores[r] + (lr * t.value[idx]);
        if (leaf_id != nullptr)
        {
            leaf_id[r] = idx;
        }
    }
}

// sample_features (src/grower_impl.hpp:163-180): a sorted draw of
// max(1, ceil(fraction x n)) distinct feature ids by std::sample over the
// grower's std::mt19937, the same library calls, so the same features.
std::vector<uint32_t> sample_features(uint32_t n_features, float fraction, std::mt19937 &rng)
{
    std::vector<uint32_t> all(n_features);
    std::iota(all.begin(), all.end(), 0U);
    if (fraction >= 1.0F || n_features <= 1)
    {
        return all;
    }
    auto const k = std::max<size_t>(
        1, static_cast<size_t>(std::ceil(fraction * static_cast<float>(n_features))));
    std::vector<uint32_t> selected;
    selected.reserve(k);
    std::sample(all.begin(), all.end(), std::back_inserter(selected), k, rng);
    return selected;
}

// The host side of the sample: two pinned slots of one round's masks (K trees
// x words, tree-major). upload() sends the next round's masks and starts
// drawing the round after into the other slot, once that slot's previous
// copy has left it.
class RowSampler
{
  public:
    // external: the caller supplies each round's rows (set_rows) instead of
    // the Bernoulli draws
    RowSampler(float p, uint32_t seed, uint64_t n, uint32_t trees, int device,
               bool external = false)
        : p_(p), rng_(seed), n_(n), trees_(trees), words_((n + 31) / 32), device_(device),
          external_(external)
    {
        for (int j = 0; j < 2; ++j)
        {
            BB_CHECK(cudaMallocHost(&slot_[j], bytes()));
            BB_CHECK(cudaEventCreateWithFlags(&copied_[j], cudaEventDisableTiming));
            counts_[j].assign(trees_, 0);
        }
    }
    ~RowSampler()
    {
        if (pending_.valid())
        {
            pending_.wait();
        }
        for (int j = 0; j < 2; ++j)
        {
            cudaFreeHost(slot_[j]);
            cudaEventDestroy(copied_[j]);
        }
    }
    RowSampler(RowSampler const &)            = delete;
    RowSampler &operator=(RowSampler const &) = delete;

    uint64_t words() const
    {
        return words_;
    }
    size_t bytes() const
    {
        return static_cast<size_t>(words_) * trees_ * 4;
    }

    // The caller's rows for the next round (external mode): ascending ids
    // below n into the current slot's mask, once its last copy has left.
    void set_rows(uint32_t const *rows, uint64_t m)
    {
        need(external_, "bb_booster_set_rows: the booster draws its own rows "
                        "(create it with external_sample)");
        need(m <= n_, "bb_booster_set_rows: more rows than the plane holds");
        BB_CHECK(cudaEventSynchronize(copied_[cur_]));
        uint32_t *w = slot_[cur_];
        std::memset(w, 0, bytes());
        for (uint64_t i = 0; i < m; ++i)
        {
            need(rows[i] < n_ && (i == 0 || rows[i - 1] < rows[i]),
                 "bb_booster_set_rows: row ids must be ascending and below the row count");
            w[rows[i] >> 5] |= 1u << (rows[i] & 31);
        }
        counts_[cur_][0] = static_cast<uint32_t>(m);
        ready_           = true;
    }

    // The next round's masks into dev (on s); returns each tree's row count.
    std::vector<uint32_t> const &upload(uint32_t *dev, cudaStream_t s)
    {
        if (external_)
        {
            need(ready_, "bb_booster_update: no rows for this round (bb_booster_set_rows "
                         "before every round of an external_sample booster)");
            int const done = cur_;
            BB_CHECK(cudaMemcpyAsync(dev, slot_[done], bytes(), cudaMemcpyHostToDevice, s));
            BB_CHECK(cudaEventRecord(copied_[done], s));
            cur_   = done ^ 1;
            ready_ = false;
            return counts_[done];
        }
        if (pending_.valid())
        {
            pending_.get();
        }
        else
        {
            draw(cur_);
        }
        int const done = cur_;
        BB_CHECK(cudaMemcpyAsync(dev, slot_[done], bytes(), cudaMemcpyHostToDevice, s));
        BB_CHECK(cudaEventRecord(copied_[done], s));
        int const next = done ^ 1;
        cur_           = next;
        pending_       = std::async(std::launch::async,
                                    [this, next]
                                    {
                                  BB_CHECK(cudaSetDevice(device_));
                                  BB_CHECK(cudaEventSynchronize(copied_[next]));
                                  draw(next);
                              });
        return counts_[done];
    }

  private:
    void draw(int j)
    {
        uint32_t *m = slot_[j];
        std::memset(m, 0, bytes());
        std::bernoulli_distribution keep(p_);
        for (uint32_t k = 0; k < trees_; ++k)
        {
            uint32_t *w = m + (static_cast<size_t>(k) * words_);
            uint32_t  c = 0;
            for (uint64_t i = 0; i < n_; ++i)
            {
                if (keep(rng_))
                {
                    w[i >> 5] |= 1u << (i & 31);
                    ++c;
                }
            }
            counts_[j][k] = c;
        }
    }

    float                 p_;
    std::mt19937          rng_;
    uint64_t              n_;
    uint32_t              trees_;
    uint64_t              words_;
    int                   device_;
    uint32_t             *slot_[2]{};
    cudaEvent_t           copied_[2]{};
    std::vector<uint32_t> counts_[2];
    int                   cur_ = 0;
    std::future<void>     pending_;
    bool                  external_ = false;
    bool                  ready_    = false;
};

} // namespace
} // namespace bb

using namespace bb;

struct bb_booster
{
    bb::Plane const            *plane = nullptr;
    cudaStream_t                stream{};
    int                         objective = 0;
    float                       lr        = 0.1F;
    float                       init      = 0.0F;
    float                      *labels    = nullptr;
    float                      *weights   = nullptr; // per row, or nullptr (unweighted)
    float                      *scores    = nullptr;
    float2                     *gh        = nullptr;
    uint32_t                   *rows      = nullptr;
    uint32_t                   *leaf_id   = nullptr;
    uint32_t                   *round     = nullptr;
    std::unique_ptr<bb::Grower> grower;
    bb::TreeStore               scratch;
    bb::TreeStore               trees;
    uint32_t                    n_trees = 0;
    bool                        use_graph = false;
    bool                        record_leaf_ids = false;
    uint32_t                    n_classes = 1;  // softmax: K score and gradient columns
    std::vector<float>          init_k;         // softmax: per-class log priors
    cudaGraphExec_t             graph     = nullptr;
    cudaEvent_t                 ev0{}, ev1{};
    float                       last_ms = 0.0F;
    bool                        truncated = false;
    bool                        sharded   = false;
    // the validation plane (armed by bb_booster_eval_arm)
    bb::Plane const            *vplane   = nullptr;
    float                      *vlabels  = nullptr;
    float                      *vscores  = nullptr; // K columns, class-major
    float                      *vlosses  = nullptr; // one per round since arming
    uint32_t                   *vcount   = nullptr;
    double                     *vpartial = nullptr;
    uint32_t                    vcap     = 0;
    // the row sample (subsample < 1): a round's masks, one tree's rows
    std::unique_ptr<RowSampler> sampler;
    uint32_t                   *sbits  = nullptr; // K x words, tree-major
    uint32_t                   *srows  = nullptr; // the tree's kept rows, ascending
    uint32_t                   *scount = nullptr; // their number
    uint32_t                   *sbsum  = nullptr; // per mask block: counts, then offsets
    std::vector<uint32_t>       host_counts;      // this round's, per tree
    // the feature sample (feature_fraction < 1): the grower's std::mt19937
    std::mt19937                feat_rng;
    float                       feat_frac = 1.0F;
    uint32_t                    feat_k    = 0; // features per tree; 0: every feature

    // Sends the next round's masks and feature samples (before its graph or
    // its eager body).
    void upload_sample()
    {
        if (sampler)
        {
            host_counts = sampler->upload(sbits, stream);
        }
        for (uint32_t k = 0; feat_k > 0 && k < n_classes; ++k)
        {
            grower->set_selection(k, sample_features(plane->n_feats, feat_frac, feat_rng));
        }
    }

    // Class k's tree reads table set k (the one set of a single-output fit).
    void use_features(uint32_t k)
    {
        if (feat_k > 0)
        {
            grower->use_set(k);
        }
    }

    // Tree k's kept rows into srows / scount.
    RootSample sample_tree(uint32_t k)
    {
        uint64_t const  words = sampler->words();
        uint32_t const *bits  = sbits + (static_cast<uint64_t>(k) * words);
        uint32_t const  nb    = static_cast<uint32_t>(ceil_div(words, k_smp_block));
        sample_count_kernel<<<nb, k_smp_threads, 0, stream>>>(bits, words, sbsum);
        BB_LAUNCH("sample_count_kernel");
        sample_scan_kernel<<<1, k_scan_threads, 0, stream>>>(sbsum, nb, scount);
        BB_LAUNCH("sample_scan_kernel");
        sample_list_kernel<<<nb, k_smp_threads, 0, stream>>>(bits, words, sbsum, srows);
        BB_LAUNCH("sample_list_kernel");
        round_launches += 3;
        return RootSample{scount, bits};
    }

    // One tree over tree k's sample: the depthwise and levelwise planes walk
    // every row; the leafwise plane stamps its rows and routes the rest.
    void grow_sampled(uint32_t k, float2 const *g, float *sc, NextRound const *next)
    {
        RootSample const rs = sample_tree(k);
        uint64_t const   n  = plane->n_rows;
        uint32_t *const  li = record_leaf_ids ? leaf_id : nullptr;
        if (grower->fuses_next())
        {
            grower->grow(g, srows, static_cast<uint32_t>(n), scratch.t, li, sc, lr, false, next,
                         &rs);
            return;
        }
        grower->grow(g, srows, host_counts[k], scratch.t, li, sc, lr, false, nullptr);
        uint32_t const grid = std::min<uint32_t>(blocks(n), 148u * 16u);
        if (plane->u8)
        {
            route_unsampled_kernel<uint8_t><<<grid, 256, 0, stream>>>(
                static_cast<uint8_t const *>(plane->bins), plane->n_pad, n, plane->n_bins,
                scratch.t, scratch.cap, rs.bits, sc, li, lr);
        }
        else
        {
            route_unsampled_kernel<uint16_t><<<grid, 256, 0, stream>>>(
                static_cast<uint16_t const *>(plane->bins), plane->n_pad, n, plane->n_bins,
                scratch.t, scratch.cap, rs.bits, sc, li, lr);
        }
        BB_LAUNCH("route_unsampled_kernel");
        round_launches += 1;
    }

    uint32_t round_launches = 0; // kernels the last round_body enqueued

    void round_body()
    {
        round_launches = 0;
        grow_round();
        if (vplane != nullptr)
        {
            eval_round();
            round_launches += 2;
        }
    }

    // one grow's kernels and the commit after it
    void count_tree()
    {
        round_launches += grower->launches_per_tree() + 1;
    }

    void eval_round()
    {
        uint64_t const n    = vplane->n_rows;
        uint32_t const grid = static_cast<uint32_t>(
            std::min<uint64_t>(k_eval_blocks, std::max<uint64_t>(1, (n + 255) / 256)));
        if (vplane->u8)
        {
            eval_walk_kernel<uint8_t><<<grid, k_eval_threads, 0, stream>>>(
                static_cast<uint8_t const *>(vplane->bins), vplane->n_pad, n, vplane->n_bins,
                trees.t, trees.cap, round, n_classes, lr, objective, vlabels, vscores,
                vpartial);
        }
        else
        {
            eval_walk_kernel<uint16_t><<<grid, k_eval_threads, 0, stream>>>(
                static_cast<uint16_t const *>(vplane->bins), vplane->n_pad, n, vplane->n_bins,
                trees.t, trees.cap, round, n_classes, lr, objective, vlabels, vscores,
                vpartial);
        }
        BB_LAUNCH("eval_walk_kernel");
        eval_finish_kernel<<<1, 32, 0, stream>>>(vpartial, grid, n, vlosses, vcount, vcap);
        BB_LAUNCH("eval_finish_kernel");
    }

    void release_eval()
    {
        void *ps[] = {vlabels, vscores, vlosses, vcount, vpartial};
        for (void *q : ps)
        {
            cudaFree(q);
        }
        vlabels  = nullptr;
        vscores  = nullptr;
        vlosses  = nullptr;
        vcount   = nullptr;
        vpartial = nullptr;
        vplane   = nullptr;
    }

    // gh always holds the gradients of the current scores: computed once at
    // creation, then by each round's final walk for the next round
    void grow_round()
    {
        uint64_t const n = plane->n_rows;
        if (objective == 2)
        {
            // one round: the softmax pairs of the round's scores, then one
            // tree per class, each adding lr x leaf to its class's scores
            softmax_gradient_kernel<<<blocks(n), 256, 0, stream>>>(scores, labels, gh, n,
                                                                    n_classes, weights);
            BB_LAUNCH("softmax_gradient_kernel");
            round_launches += 1;
            for (uint32_t k = 0; k < n_classes; ++k)
            {
                use_features(k);
                if (sampler)
                {
                    grow_sampled(k, gh + (k * n), scores + (k * n), nullptr);
                }
                else
                {
                    grower->grow(gh + (k * n), rows, static_cast<uint32_t>(n), scratch.t,
                                 record_leaf_ids ? leaf_id : nullptr, scores + (k * n), lr,
                                 true, nullptr);
                }
                commit_tree_kernel<<<1, 256, 0, stream>>>(scratch.t, trees.t, trees.cap, round);
                BB_LAUNCH("commit_tree_kernel");
                count_tree();
            }
            return;
        }
        use_features(0);
        if (!grower->fuses_next())
        {
            // the leafwise plane stamps from its leaves' segments: gradients
            // of the current scores come from their own pass
            gradient_kernel<<<blocks(n), 256, 0, stream>>>(objective, scores, labels, gh, n,
                                                           weights);
            BB_LAUNCH("gradient_kernel");
            if (sampler)
            {
                grow_sampled(0, gh, scores, nullptr);
            }
            else
            {
                grower->grow(gh, rows, static_cast<uint32_t>(n), scratch.t,
                             record_leaf_ids ? leaf_id : nullptr, scores, lr, true, nullptr);
            }
            commit_tree_kernel<<<1, 256, 0, stream>>>(scratch.t, trees.t, trees.cap, round);
            BB_LAUNCH("commit_tree_kernel");
            count_tree();
            round_launches += 1; // the gradient pass
            return;
        }
        bb::NextRound const next{objective, labels, gh, weights};
        if (sampler)
        {
            grow_sampled(0, gh, scores, &next);
        }
        else
        {
            grower->grow(gh, rows, static_cast<uint32_t>(n), scratch.t,
                         record_leaf_ids ? leaf_id : nullptr, scores, lr, true, &next);
        }
        commit_tree_kernel<<<1, 256, 0, stream>>>(scratch.t, trees.t, trees.cap, round);
        BB_LAUNCH("commit_tree_kernel");
        count_tree();
    }
};

namespace
{

// bb_booster_create's body; a sharded fit also passes its reducer, the
// shard's first row in the fit, the fit's row count and the fit's init score
// (the mean over every shard's labels, which no shard can form alone).
bb_booster *create_booster(bb_plane const *plane, float const *labels, float const *init_scores,
                           bb_train_cfg const *cfg, uint32_t max_trees, bb::Reducer *red,
                           uint64_t row_offset, uint64_t total_rows, float const *init_score)
{
    need(plane != nullptr && labels != nullptr && cfg != nullptr,
         "bb_booster_create: null argument");
    need(cfg->objective >= 0 && cfg->objective <= 3,
         "objective must be 0 (mse), 1 (logloss), 2 (softmax) or 3 (poisson)");
    need(cfg->objective != 2 || (cfg->n_classes >= 2 && cfg->n_classes <= k_max_classes),
         "softmax needs 2 <= n_classes <= 16");
    need(cfg->objective != 2 || red == nullptr, "softmax fits do not shard");
    need(max_trees > 0, "max_trees must be positive");
    // sampler.subsample (src/sampler.cpp:27-34): 0 (a zeroed config) and
    // values >= 1 keep every row
    need(!(cfg->subsample < 0.0F) && !std::isnan(cfg->subsample),
         "sampler.subsample must be > 0");
    bool const external = cfg->external_sample != 0;
    bool const sampled  = external || (cfg->subsample > 0.0F && cfg->subsample < 1.0F);
    need(!sampled || red == nullptr, "a sharded fit keeps every row (subsample 1)");
    need(!external || cfg->objective != 2,
         "external_sample: single-output objectives only (a softmax round draws per class)");
    need(!(cfg->feature_fraction < 0.0F) && !std::isnan(cfg->feature_fraction),
         "tree_config.feature_fraction must be > 0");
    uint32_t const F_all = plane->p.n_feats;
    uint32_t const feat_k =
        cfg->feature_fraction > 0.0F && cfg->feature_fraction < 1.0F && F_all > 1
            ? static_cast<uint32_t>(std::max<size_t>(
                  1, static_cast<size_t>(
                         std::ceil(cfg->feature_fraction * static_cast<float>(F_all)))))
            : 0;
    need(feat_k == 0 || cfg->selected == nullptr,
         "feature_fraction < 1 draws each tree's features: pass no `selected`");
    auto           b = std::make_unique<bb_booster>();
    Plane const   &p = plane->p;
    uint64_t const n = p.n_rows;
    b->plane         = &p;
    b->objective     = cfg->objective;
    b->lr            = cfg->learning_rate;
    BB_CHECK(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    uint32_t const K = cfg->objective == 2 ? cfg->n_classes : 1;
    b->n_classes     = K;
    if (cfg->objective == 2)
    {
        // log class priors (multiclass_booster.hpp:60-77)
        std::vector<double> counts(K, 0.0);
        for (uint64_t i = 0; i < n; ++i)
        {
            long const c = std::lround(labels[i]);
            counts[c >= 0 && static_cast<uint64_t>(c) < K ? c : 0] += 1.0;
        }
        for (uint32_t k = 0; k < K; ++k)
        {
            b->init_k.push_back(static_cast<float>(
                std::log(std::max(counts[k], 1.0) / static_cast<double>(n))));
        }
        b->init = b->init_k[0];
    }
    else if (init_score != nullptr)
    {
        b->init = *init_score;
    }
    else if (cfg->objective == 3)
    {
        // PoissonObjective::init_score (src/objective.cpp:293-308): the log of
        // the mean label (an FP64 sum), floored at 1e-9
        double sum = 0.0;
        for (uint64_t i = 0; i < n; ++i)
        {
            need(labels[i] >= 0.0F && !std::isnan(labels[i]),
                 "poisson objective requires non-negative labels");
            sum += labels[i];
        }
        double const mean = sum / static_cast<double>(std::max<uint64_t>(n, 1));
        b->init           = static_cast<float>(std::log(std::max(mean, 1e-9)));
    }
    else
    {
        // init_score: a float serial sum, as std::accumulate does
        float sum = 0.0F;
        for (uint64_t i = 0; i < n; ++i)
        {
            sum += labels[i];
        }
        float const nn = static_cast<float>(n);
        b->init = cfg->objective == 0 ? sum / nn : std::log((sum / nn) / (1.0F - (sum / nn)));
    }
    b->labels  = dmalloc<float>(n);
    b->scores  = dmalloc<float>(n * K);
    b->gh      = dmalloc<float2>(n * K);
    b->rows    = dmalloc<uint32_t>(n);
    b->leaf_id = dmalloc<uint32_t>(n);
    b->round   = dmalloc<uint32_t>(1);
    BB_CHECK(cudaMemcpyAsync(b->labels, labels, n * 4, cudaMemcpyHostToDevice, b->stream));
    if (init_scores != nullptr)
    {
        BB_CHECK(cudaMemcpyAsync(b->scores, init_scores, n * 4, cudaMemcpyHostToDevice,
                                 b->stream));
    }
    else
    {
        for (uint32_t k = 0; k < K; ++k)
        {
            fill_kernel<<<blocks(n), 256, 0, b->stream>>>(b->scores + (k * n),
                                                          K > 1 ? b->init_k[k] : b->init, n);
            BB_LAUNCH("fill_kernel");
        }
    }
    iota_kernel<<<blocks(n), 256, 0, b->stream>>>(b->rows, n);
    BB_LAUNCH("iota_kernel");
    BB_CHECK(cudaMemsetAsync(b->round, 0, 4, b->stream));
    GrowConfig gc = grow_config(*cfg);
    gc.fit_rows   = red != nullptr ? total_rows : n; // a shard's cells hold the fit's sums
    if (feat_k > 0 && feat_k < p.n_feats)
    {
        // every tree draws its own features into table set k (class k)
        gc.sample_k   = feat_k;
        gc.sel_sets   = K;
        b->feat_k     = feat_k;
        b->feat_frac  = cfg->feature_fraction;
        b->feat_rng.seed(cfg->feature_seed);
    }
    b->grower = std::make_unique<Grower>(p, gc, selection(*cfg, p.n_feats),
                                         static_cast<uint32_t>(n), b->stream);
    b->grower->set_monotone(monotone(*cfg));
    b->grower->set_interaction(interaction(*cfg, p.n_feats));
    b->grower->set_seed(cfg->seed);
    if (red != nullptr)
    {
        b->grower->set_shard(red, row_offset, total_rows);
        b->sharded = true;
    }
    if (sampled)
    {
        int dev = 0;
        BB_CHECK(cudaGetDevice(&dev));
        b->sampler = std::make_unique<RowSampler>(cfg->subsample, cfg->random_seed, n, K, dev,
                                                  external);
        uint64_t const words = b->sampler->words();
        b->sbits  = dmalloc<uint32_t>(words * K);
        b->srows  = dmalloc<uint32_t>(n);
        b->scount = dmalloc<uint32_t>(1);
        b->sbsum  = dmalloc<uint32_t>(ceil_div(words, k_smp_block));
    }
    b->scratch.alloc(b->grower->max_nodes(), 1);
    b->trees.alloc(b->grower->max_nodes(), max_trees * K); // round-major: r * K + k
    // a leafwise round reads every pop back to the host: it runs eagerly
    b->use_graph       = cfg->use_graph != 0 && b->grower->fuses_next();
    b->record_leaf_ids = cfg->record_leaf_ids != 0;
    if (K == 1)
    {
        gradient_kernel<<<blocks(n), 256, 0, b->stream>>>(b->objective, b->scores, b->labels,
                                                          b->gh, n, nullptr);
        BB_LAUNCH("gradient_kernel");
        b->grower->seed_absmax(b->gh);
    }
    BB_CHECK(cudaEventCreate(&b->ev0));
    BB_CHECK(cudaEventCreate(&b->ev1));
    BB_CHECK(cudaStreamSynchronize(b->stream));
    return b.release();
}

} // namespace

extern "C"
{

    char const *bb_last_error(void)
    {
        return g_err.c_str();
    }

    uint32_t bb_tree_capacity(bb_train_cfg const *cfg)
    {
        if (cfg == nullptr)
        {
            return 0;
        }
        if (cfg->grower == 2)
        {
            uint32_t const l = cfg->max_leaves == 0 && cfg->max_depth <= 9
                                   ? 1u << cfg->max_depth
                                   : cfg->max_leaves;
            return 4 * std::max<uint32_t>(l, 1);
        }
        return cfg->max_depth <= 8 ? (2u << cfg->max_depth) - 1 : 0;
    }

    int bb_available(void)
    {
        int n = 0;
        return cudaGetDeviceCount(&n) == cudaSuccess && n > 0 ? 1 : 0;
    }

    int bb_select_device(uint32_t device_id)
    {
        return guarded(
            [&]
            {
                int n = 0;
                BB_CHECK(cudaGetDeviceCount(&n));
                if (device_id >= static_cast<uint32_t>(n))
                {
                    throw ConfigError("parallel.device_id " + std::to_string(device_id) +
                                      " is out of range for " + std::to_string(n) +
                                      " visible CUDA devices");
                }
                BB_CHECK(cudaSetDevice(static_cast<int>(device_id)));
            });
    }

    int bb_ingest(float const *X, uint64_t n_rows, uint32_t n_feats, int x_on_device,
                  float const *cuts, uint32_t const *cut_off, bb_plane **out)
    {
        return guarded(
            [&]
            {
                need(out != nullptr && X != nullptr && cuts != nullptr && cut_off != nullptr,
                     "bb_ingest: null argument");
                need(n_rows > 0 && n_feats > 0, "bb_ingest: empty matrix");
                need(n_rows < (1ull << 32), "bb_ingest: more than 2^32 - 1 rows");
                auto pl = std::make_unique<bb_plane>();
                Plane &p = pl->p;
                p.n_rows  = n_rows;
                p.n_pad   = ((n_rows + 63) / 64) * 64;
                p.n_feats = n_feats;
                BB_CHECK(cudaGetDevice(&p.device));
                uint32_t const n_cuts = cut_off[n_feats];
                uint32_t       max_nb = 0;
                for (uint32_t f = 0; f < n_feats; ++f)
                {
                    need(cut_off[f + 1] > cut_off[f] + 1, "bb_ingest: a feature needs >= 2 bins");
                    max_nb = std::max(max_nb, cut_off[f + 1] - cut_off[f]);
                }
                need(max_nb <= 65535, "bb_ingest: more than 65535 bins");
                p.u8        = max_nb <= 256;
                p.h_cuts    = new float[n_cuts];
                p.h_cut_off = new uint32_t[n_feats + 1];
                std::memcpy(p.h_cuts, cuts, n_cuts * sizeof(float));
                std::memcpy(p.h_cut_off, cut_off, (n_feats + 1) * sizeof(uint32_t));
                std::vector<uint32_t> nb(n_feats);
                for (uint32_t f = 0; f < n_feats; ++f)
                {
                    nb[f] = cut_off[f + 1] - cut_off[f];
                }
                p.cuts    = dmalloc<float>(n_cuts);
                p.cut_off = dmalloc<uint32_t>(n_feats + 1);
                p.n_bins  = dmalloc<uint32_t>(n_feats);
                BB_CHECK(cudaMemcpy(p.cuts, cuts, n_cuts * 4, cudaMemcpyHostToDevice));
                BB_CHECK(cudaMemcpy(p.cut_off, cut_off, (n_feats + 1) * 4,
                                    cudaMemcpyHostToDevice));
                BB_CHECK(cudaMemcpy(p.n_bins, nb.data(), n_feats * 4, cudaMemcpyHostToDevice));
                size_t const bytes = static_cast<size_t>(n_feats) * p.n_pad * (p.u8 ? 1 : 2);
                BB_CHECK(cudaMalloc(&p.bins, bytes));
                BB_CHECK(cudaMemset(p.bins, 0, bytes));
                cudaStream_t s;
                BB_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
                try
                {
                    ingest(p, X, x_on_device != 0, s);
                    build_mirror(p, s);
                    BB_CHECK(cudaStreamSynchronize(s));
                }
                catch (...)
                {
                    cudaStreamDestroy(s);
                    throw;
                }
                BB_CHECK(cudaStreamDestroy(s));
                *out = pl.release();
            });
    }

    int bb_plane_from_bins(void const *bins, int is_u8, uint64_t n_rows, uint32_t n_feats,
                           float const *cuts, uint32_t const *cut_off, bb_plane **out)
    {
        return guarded(
            [&]
            {
                need(out != nullptr && bins != nullptr && cuts != nullptr && cut_off != nullptr,
                     "bb_plane_from_bins: null argument");
                need(n_rows > 0 && n_feats > 0, "bb_plane_from_bins: empty matrix");
                need(n_rows < (1ull << 32), "bb_plane_from_bins: more than 2^32 - 1 rows");
                uint32_t max_nb = 0;
                for (uint32_t f = 0; f < n_feats; ++f)
                {
                    need(cut_off[f + 1] > cut_off[f] + 1,
                         "bb_plane_from_bins: a feature needs >= 2 bins");
                    max_nb = std::max(max_nb, cut_off[f + 1] - cut_off[f]);
                }
                need(is_u8 == 0 || max_nb <= 256, "bb_plane_from_bins: u8 codes need <= 256 bins");
                need(max_nb <= 65535, "bb_plane_from_bins: more than 65535 bins");
                // every code indexes a histogram cell: check them all
                for (uint32_t f = 0; f < n_feats; ++f)
                {
                    uint32_t const nb = cut_off[f + 1] - cut_off[f];
                    for (uint64_t r = 0; r < n_rows; ++r)
                    {
                        uint32_t const b =
                            is_u8 != 0 ? static_cast<uint8_t const *>(bins)[(f * n_rows) + r]
                                       : static_cast<uint16_t const *>(bins)[(f * n_rows) + r];
                        need(b < nb, "bb_plane_from_bins: a code is not below its bin count");
                    }
                }
                auto   pl = std::make_unique<bb_plane>();
                Plane &p  = pl->p;
                p.n_rows  = n_rows;
                p.n_pad   = ((n_rows + 63) / 64) * 64;
                p.n_feats = n_feats;
                p.u8      = is_u8 != 0;
                BB_CHECK(cudaGetDevice(&p.device));
                uint32_t const n_cuts = cut_off[n_feats];
                p.h_cuts              = new float[n_cuts];
                p.h_cut_off           = new uint32_t[n_feats + 1];
                std::memcpy(p.h_cuts, cuts, n_cuts * sizeof(float));
                std::memcpy(p.h_cut_off, cut_off, (n_feats + 1) * sizeof(uint32_t));
                std::vector<uint32_t> nb(n_feats);
                for (uint32_t f = 0; f < n_feats; ++f)
                {
                    nb[f] = cut_off[f + 1] - cut_off[f];
                }
                p.cuts    = dmalloc<float>(n_cuts);
                p.cut_off = dmalloc<uint32_t>(n_feats + 1);
                p.n_bins  = dmalloc<uint32_t>(n_feats);
                BB_CHECK(cudaMemcpy(p.cuts, cuts, n_cuts * 4, cudaMemcpyHostToDevice));
                BB_CHECK(cudaMemcpy(p.cut_off, cut_off, (n_feats + 1) * 4,
                                    cudaMemcpyHostToDevice));
                BB_CHECK(cudaMemcpy(p.n_bins, nb.data(), n_feats * 4, cudaMemcpyHostToDevice));
                size_t const el    = p.u8 ? 1 : 2;
                size_t const bytes = static_cast<size_t>(n_feats) * p.n_pad * el;
                BB_CHECK(cudaMalloc(&p.bins, bytes));
                BB_CHECK(cudaMemset(p.bins, 0, bytes));
                BB_CHECK(cudaMemcpy2D(p.bins, p.n_pad * el, bins, n_rows * el, n_rows * el,
                                      n_feats, cudaMemcpyHostToDevice));
                cudaStream_t s;
                BB_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
                try
                {
                    build_mirror(p, s);
                    BB_CHECK(cudaStreamSynchronize(s));
                }
                catch (...)
                {
                    cudaStreamDestroy(s);
                    throw;
                }
                BB_CHECK(cudaStreamDestroy(s));
                *out = pl.release();
            });
    }

    int bb_plane_is_u8(bb_plane const *plane)
    {
        return plane->p.u8 ? 1 : 0;
    }

    int bb_plane_download(bb_plane const *plane, uint16_t *out)
    {
        return guarded(
            [&]
            {
                Plane const &p = plane->p;
                if (p.u8)
                {
                    std::vector<uint8_t> tmp(p.n_rows);
                    for (uint32_t f = 0; f < p.n_feats; ++f)
                    {
                        BB_CHECK(cudaMemcpy(tmp.data(),
                                            static_cast<uint8_t const *>(p.bins) + (f * p.n_pad),
                                            p.n_rows, cudaMemcpyDeviceToHost));
                        for (uint64_t r = 0; r < p.n_rows; ++r)
                        {
                            out[(f * p.n_rows) + r] = tmp[r];
                        }
                    }
                }
                else
                {
                    for (uint32_t f = 0; f < p.n_feats; ++f)
                    {
                        BB_CHECK(cudaMemcpy(out + (f * p.n_rows),
                                            static_cast<uint16_t const *>(p.bins) + (f * p.n_pad),
                                            p.n_rows * 2, cudaMemcpyDeviceToHost));
                    }
                }
            });
    }

    int bb_plane_create_like(bb_plane const *like, uint64_t max_rows, bb_plane **out)
    {
        return guarded(
            [&]
            {
                need(like != nullptr && out != nullptr, "bb_plane_create_like: null argument");
                need(max_rows > 0 && max_rows < (1ull << 32),
                     "bb_plane_create_like: max_rows must be in [1, 2^32 - 1]");
                Plane const &q  = like->p;
                auto         pl = std::make_unique<bb_plane>();
                Plane       &p  = pl->p;
                // an empty plane until the first refill; sized for max_rows
                p.n_rows   = 0;
                p.n_pad    = 0;
                p.n_feats  = q.n_feats;
                p.u8       = q.u8;
                p.cap_rows = max_rows;
                BB_CHECK(cudaGetDevice(&p.device));
                uint32_t const F      = q.n_feats;
                uint32_t const n_cuts = q.h_cut_off[F];
                p.h_cuts              = new float[n_cuts];
                p.h_cut_off           = new uint32_t[F + 1];
                std::memcpy(p.h_cuts, q.h_cuts, n_cuts * sizeof(float));
                std::memcpy(p.h_cut_off, q.h_cut_off, (F + 1) * sizeof(uint32_t));
                p.cuts    = dmalloc<float>(n_cuts);
                p.cut_off = dmalloc<uint32_t>(F + 1);
                p.n_bins  = dmalloc<uint32_t>(F);
                BB_CHECK(cudaMemcpy(p.cuts, q.cuts, n_cuts * 4, cudaMemcpyDeviceToDevice));
                BB_CHECK(cudaMemcpy(p.cut_off, q.cut_off, (F + 1) * 4, cudaMemcpyDeviceToDevice));
                BB_CHECK(cudaMemcpy(p.n_bins, q.n_bins, F * 4, cudaMemcpyDeviceToDevice));
                uint64_t const cap_pad = ((max_rows + 63) / 64) * 64;
                size_t const   el      = p.u8 ? 1 : 2;
                BB_CHECK(cudaMalloc(&p.bins, static_cast<size_t>(F) * cap_pad * el));
                BB_CHECK(cudaMemset(p.bins, 0, static_cast<size_t>(F) * cap_pad * el));
                uint32_t const per = k_mirror_bytes / (p.u8 ? 1 : 2);
                p.n_tiles          = (F + per - 1) / per;
                BB_CHECK(cudaMalloc(&p.mirror,
                                    static_cast<size_t>(p.n_tiles) * max_rows * k_mirror_bytes));
                // host rows go up through a staging buffer of at most 64 MB
                uint64_t const row_bytes = static_cast<uint64_t>(F) * sizeof(float);
                p.stage_rows             = stage_rows_for(F, max_rows);
                BB_CHECK(cudaMalloc(&p.stage, p.stage_rows * row_bytes));
                BB_CHECK(cudaStreamCreateWithFlags(&p.stream, cudaStreamNonBlocking));
                *out = pl.release();
            });
    }

    int bb_plane_refill(bb_plane *plane, float const *X, uint64_t n_rows, int x_on_device)
    {
        return guarded(
            [&]
            {
                need(plane != nullptr && X != nullptr, "bb_plane_refill: null argument");
                Plane &p = plane->p;
                need(p.cap_rows > 0, "bb_plane_refill: not a request plane "
                                     "(make one with bb_plane_create_like)");
                if (n_rows == 0 || n_rows > p.cap_rows)
                {
                    throw ConfigError("bb_plane_refill: " + std::to_string(n_rows) +
                                      " rows; the plane holds 1 to " +
                                      std::to_string(p.cap_rows));
                }
                p.n_rows = n_rows;
                p.n_pad  = ((n_rows + 63) / 64) * 64;
                ingest(p, X, x_on_device != 0, p.stream, p.stage, p.stage_rows);
                fill_mirror(p, p.stream);
                BB_CHECK(cudaStreamSynchronize(p.stream));
            });
    }

    void bb_plane_destroy(bb_plane *plane)
    {
        if (plane == nullptr)
        {
            return;
        }
        Plane &p = plane->p;
        if (p.stream != nullptr)
        {
            cudaStreamSynchronize(p.stream);
            cudaStreamDestroy(p.stream);
        }
        cudaFree(p.stage);
        cudaFree(p.bins);
        cudaFree(p.mirror);
        cudaFree(p.cuts);
        cudaFree(p.cut_off);
        cudaFree(p.n_bins);
        delete[] p.h_cuts;
        delete[] p.h_cut_off;
        delete plane;
    }

    int bb_booster_create(bb_plane const *plane, float const *labels,
                          float const *init_scores, bb_train_cfg const *cfg,
                          uint32_t max_trees, bb_booster **out)
    {
        return guarded([&] { *out = create_booster(plane, labels, init_scores, cfg, max_trees,
                                                   nullptr, 0, 0, nullptr); });
    }

    int bb_booster_create_sharded(bb_plane const *plane, float const *labels,
                                  float const *init_scores, bb_train_cfg const *cfg,
                                  uint32_t max_trees, bb_comm *comm, uint64_t row_offset,
                                  uint64_t total_rows, float init_score, bb_booster **out)
    {
        return guarded(
            [&]
            {
                need(comm != nullptr, "bb_booster_create_sharded: null comm");
                need(plane != nullptr && row_offset + plane->p.n_rows <= total_rows,
                     "bb_booster_create_sharded: the shard lies outside the fit's rows");
                if (comm->member && cfg != nullptr && cfg->use_graph != 0)
                {
                    throw ConfigError("bb_booster_create_sharded: an in-process shard group "
                                      "orders its shards by host threads; use_graph needs a "
                                      "process per shard");
                }
                *out = create_booster(plane, labels, init_scores, cfg, max_trees,
                                      comm->reducer(), row_offset, total_rows, &init_score);
            });
    }

    int bb_booster_set_rows(bb_booster *b, uint32_t const *rows, uint64_t n_rows)
    {
        return guarded(
            [&]
            {
                need(b != nullptr && (rows != nullptr || n_rows == 0),
                     "bb_booster_set_rows: null argument");
                need(b->sampler != nullptr, "bb_booster_set_rows: the booster keeps every row "
                                            "(create it with external_sample)");
                b->sampler->set_rows(rows, n_rows);
            });
    }

    int bb_booster_update(bb_booster *b, uint32_t n_iters)
    {
        return guarded(
            [&]
            {
                need(b->n_trees + (n_iters * b->n_classes) <= b->trees.n,
                     "bb_booster_update: tree capacity");
                need(!b->truncated, "bb_booster_update: the booster was truncated");
                if (b->use_graph && b->graph == nullptr)
                {
                    cudaGraph_t g;
                    // the capture records the round; the first round's masks
                    // (if sampled) go up before it runs
                    BB_CHECK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
                    try
                    {
                        b->round_body();
                    }
                    catch (...)
                    {
                        cudaStreamEndCapture(b->stream, &g);
                        throw;
                    }
                    BB_CHECK(cudaStreamEndCapture(b->stream, &g));
                    BB_CHECK(cudaGraphInstantiate(&b->graph, g, 0));
                    BB_CHECK(cudaGraphDestroy(g));
                }
                BB_CHECK(cudaEventRecord(b->ev0, b->stream));
                for (uint32_t i = 0; i < n_iters; ++i)
                {
                    b->upload_sample();
                    if (b->graph != nullptr)
                    {
                        BB_CHECK(cudaGraphLaunch(b->graph, b->stream));
                    }
                    else
                    {
                        b->round_body();
                    }
                }
                BB_CHECK(cudaEventRecord(b->ev1, b->stream));
                b->n_trees += n_iters * b->n_classes;
            });
    }

    // ---- many boosters, one graph launch per round -----------------------
    // Every booster's round graph becomes a child node of one parent graph
    // with no edges between them, so a round of the whole batch is one
    // cudaGraphLaunch and the boosters' kernels run concurrently.
    struct bb_batch_impl
    {
        std::vector<bb_booster *> boosters;
        cudaGraphExec_t           exec = nullptr;
        cudaStream_t              stream{};
        cudaEvent_t               ev0{}, ev1{};
        std::vector<cudaEvent_t>  ready;
    };

    int bb_batch_create(bb_booster *const *boosters, uint32_t n, bb_batch **out)
    {
        return guarded(
            [&]
            {
                need(boosters != nullptr && out != nullptr && n > 0,
                     "bb_batch_create: null argument");
                auto        bt = std::make_unique<bb_batch_impl>();
                cudaGraph_t parent{};
                BB_CHECK(cudaGraphCreate(&parent, 0));
                try
                {
                    for (uint32_t i = 0; i < n; ++i)
                    {
                        bb_booster *b = boosters[i];
                        need(b != nullptr, "bb_batch_create: null booster");
                        if (!b->use_graph || b->sampler != nullptr || b->feat_k > 0 ||
                            b->sharded || b->truncated)
                        {
                            throw ConfigError(
                                "bb_batch_create: a batch takes graph-captured boosters without "
                                "row or feature sampling, unsharded and not truncated (a "
                                "leafwise round is not captured)");
                        }
                        cudaGraph_t g{};
                        BB_CHECK(cudaStreamBeginCapture(b->stream,
                                                        cudaStreamCaptureModeThreadLocal));
                        try
                        {
                            b->round_body();
                        }
                        catch (...)
                        {
                            cudaStreamEndCapture(b->stream, &g);
                            throw;
                        }
                        BB_CHECK(cudaStreamEndCapture(b->stream, &g));
                        cudaGraphNode_t node{};
                        cudaError_t const e = cudaGraphAddChildGraphNode(&node, parent, nullptr,
                                                                         0, g);
                        cudaGraphDestroy(g);
                        check(e, "cudaGraphAddChildGraphNode");
                        bt->boosters.push_back(b);
                        cudaEvent_t ev{};
                        BB_CHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
                        bt->ready.push_back(ev);
                    }
                    BB_CHECK(cudaGraphInstantiate(&bt->exec, parent, 0));
                }
                catch (...)
                {
                    cudaGraphDestroy(parent);
                    for (cudaEvent_t ev : bt->ready)
                    {
                        cudaEventDestroy(ev);
                    }
                    throw;
                }
                BB_CHECK(cudaGraphDestroy(parent));
                BB_CHECK(cudaStreamCreateWithFlags(&bt->stream, cudaStreamNonBlocking));
                BB_CHECK(cudaEventCreate(&bt->ev0));
                BB_CHECK(cudaEventCreate(&bt->ev1));
                *out = reinterpret_cast<bb_batch *>(bt.release());
            });
    }

    int bb_batch_update(bb_batch *batch, uint32_t n_rounds)
    {
        return guarded(
            [&]
            {
                need(batch != nullptr, "bb_batch_update: null batch");
                auto *bt = reinterpret_cast<bb_batch_impl *>(batch);
                for (bb_booster *b : bt->boosters)
                {
                    need(b->n_trees + (n_rounds * b->n_classes) <= b->trees.n,
                         "bb_batch_update: a booster's tree capacity");
                    need(!b->truncated, "bb_batch_update: a booster was truncated");
                }
                // the batch runs after every booster's queued work ...
                for (size_t i = 0; i < bt->boosters.size(); ++i)
                {
                    BB_CHECK(cudaEventRecord(bt->ready[i], bt->boosters[i]->stream));
                    BB_CHECK(cudaStreamWaitEvent(bt->stream, bt->ready[i], 0));
                }
                BB_CHECK(cudaEventRecord(bt->ev0, bt->stream));
                for (uint32_t r = 0; r < n_rounds; ++r)
                {
                    BB_CHECK(cudaGraphLaunch(bt->exec, bt->stream));
                }
                BB_CHECK(cudaEventRecord(bt->ev1, bt->stream));
                // ... and before anything later on each booster's stream
                for (bb_booster *b : bt->boosters)
                {
                    BB_CHECK(cudaStreamWaitEvent(b->stream, bt->ev1, 0));
                    b->n_trees += n_rounds * b->n_classes;
                }
            });
    }

    int bb_batch_sync(bb_batch *batch)
    {
        return guarded(
            [&]
            {
                need(batch != nullptr, "bb_batch_sync: null batch");
                BB_CHECK(cudaStreamSynchronize(reinterpret_cast<bb_batch_impl *>(batch)->stream));
            });
    }

    int bb_batch_last_ms(bb_batch const *batch, float *ms)
    {
        return guarded(
            [&]
            {
                need(batch != nullptr && ms != nullptr, "bb_batch_last_ms: null argument");
                auto const *bt = reinterpret_cast<bb_batch_impl const *>(batch);
                BB_CHECK(cudaEventSynchronize(bt->ev1));
                BB_CHECK(cudaEventElapsedTime(ms, bt->ev0, bt->ev1));
            });
    }

    void bb_batch_destroy(bb_batch *batch)
    {
        if (batch == nullptr)
        {
            return;
        }
        auto *bt = reinterpret_cast<bb_batch_impl *>(batch);
        cudaStreamSynchronize(bt->stream);
        cudaGraphExecDestroy(bt->exec);
        for (cudaEvent_t ev : bt->ready)
        {
            cudaEventDestroy(ev);
        }
        cudaEventDestroy(bt->ev0);
        cudaEventDestroy(bt->ev1);
        cudaStreamDestroy(bt->stream);
        delete bt;
    }

    int bb_booster_set_weights(bb_booster *b, float const *weights)
    {
        return guarded(
            [&]
            {
                need(b != nullptr, "bb_booster_set_weights: null booster");
                need(b->n_trees == 0, "bb_booster_set_weights: set weights before the first round");
                uint64_t const n = b->plane->n_rows;
                BB_CHECK(cudaStreamSynchronize(b->stream));
                if (weights == nullptr)
                {
                    cudaFree(b->weights);
                    b->weights = nullptr;
                }
                else
                {
                    if (b->weights == nullptr)
                    {
                        b->weights = dmalloc<float>(n);
                    }
                    BB_CHECK(cudaMemcpyAsync(b->weights, weights, n * 4, cudaMemcpyHostToDevice,
                                             b->stream));
                }
                if (b->n_classes == 1)
                {
                    // the first round's pairs (a softmax round forms its own)
                    gradient_kernel<<<blocks(n), 256, 0, b->stream>>>(
                        b->objective, b->scores, b->labels, b->gh, n, b->weights);
                    BB_LAUNCH("gradient_kernel");
                    b->grower->seed_absmax(b->gh);
                }
                BB_CHECK(cudaStreamSynchronize(b->stream));
            });
    }

    int bb_booster_sync(bb_booster *b)
    {
        return guarded(
            [&]
            {
                BB_CHECK(cudaStreamSynchronize(b->stream));
                BB_CHECK(cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1));
            });
    }

    int bb_booster_last_ms(bb_booster const *b, float *ms)
    {
        *ms = b->last_ms;
        return BB_OK;
    }

    int bb_booster_n_trees(bb_booster const *b, uint32_t *n)
    {
        *n = b->n_trees;
        return BB_OK;
    }

    float bb_booster_init_score(bb_booster const *b)
    {
        return b->init;
    }

    uint32_t bb_booster_tree_capacity(bb_booster const *b)
    {
        return b->trees.cap;
    }

    int bb_booster_tree(bb_booster const *b, uint32_t t, uint32_t *feature, float *value,
                        uint32_t *left, uint32_t *right, uint8_t *default_left, float *gain,
                        float *cover, uint32_t *split_bin, uint32_t *meta)
    {
        return guarded(
            [&]
            {
                need(t < b->n_trees, "bb_booster_tree: tree index out of range");
                BB_CHECK(cudaStreamSynchronize(b->stream));
                b->trees.download(t, feature, value, left, right, default_left, gain, cover,
                                  split_bin, meta);
            });
    }

    int bb_booster_trees(bb_booster const *b, uint32_t first, uint32_t count,
                         uint32_t *feature, float *value, uint32_t *left, uint32_t *right,
                         uint8_t *default_left, float *gain, float *cover, uint32_t *split_bin,
                         uint32_t *meta)
    {
        return guarded(
            [&]
            {
                need(first <= b->n_trees && count <= b->n_trees - first,
                     "bb_booster_trees: tree range out of range");
                if (count == 0)
                {
                    return;
                }
                BB_CHECK(cudaStreamSynchronize(b->stream));
                b->trees.download(first, feature, value, left, right, default_left, gain, cover,
                                  split_bin, meta, count);
            });
    }

    int bb_booster_scores(bb_booster const *b, float *out)
    {
        return guarded(
            [&]
            {
                BB_CHECK(cudaStreamSynchronize(b->stream));
                uint64_t const n = b->plane->n_rows;
                uint32_t const K = b->n_classes;
                if (K == 1)
                {
                    BB_CHECK(cudaMemcpy(out, b->scores, n * 4, cudaMemcpyDeviceToHost));
                    return;
                }
                // class-major on the device, row-major (n x K) for the caller
                std::vector<float> cm(n * K);
                BB_CHECK(cudaMemcpy(cm.data(), b->scores, n * K * 4, cudaMemcpyDeviceToHost));
                for (uint64_t i = 0; i < n; ++i)
                {
                    for (uint32_t k = 0; k < K; ++k)
                    {
                        out[(i * K) + k] = cm[(k * n) + i];
                    }
                }
            });
    }

    uint32_t bb_booster_n_classes(bb_booster const *b)
    {
        return b->n_classes;
    }

    int bb_booster_init_scores(bb_booster const *b, float *out)
    {
        return guarded(
            [&]
            {
                need(out != nullptr, "bb_booster_init_scores: null argument");
                if (b->n_classes == 1)
                {
                    out[0] = b->init;
                    return;
                }
                std::copy(b->init_k.begin(), b->init_k.end(), out);
            });
    }

    int bb_booster_leaf_ids(bb_booster const *b, uint32_t *out)
    {
        return guarded(
            [&]
            {
                need(b->record_leaf_ids, "bb_booster_leaf_ids: create with record_leaf_ids");
                BB_CHECK(cudaStreamSynchronize(b->stream));
                BB_CHECK(cudaMemcpy(out, b->leaf_id, b->plane->n_rows * 4, cudaMemcpyDeviceToHost));
            });
    }

    int bb_booster_profile_round(bb_booster *b, bb_profile *out)
    {
        return guarded(
            [&]
            {
                need(b->n_trees + b->n_classes <= b->trees.n,
                     "bb_booster_profile_round: tree capacity");
                BB_CHECK(cudaStreamSynchronize(b->stream));
                Profile p;
                b->grower->set_profile(&p);
                b->upload_sample();
                BB_CHECK(cudaEventRecord(b->ev0, b->stream));
                try
                {
                    b->round_body();
                }
                catch (...)
                {
                    b->grower->set_profile(nullptr);
                    throw;
                }
                b->grower->set_profile(nullptr);
                BB_CHECK(cudaEventRecord(b->ev1, b->stream));
                BB_CHECK(cudaEventSynchronize(b->ev1));
                float ms = 0.0F;
                BB_CHECK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
                b->n_trees += b->n_classes;
                out->hist_ms      = p.hist_ms;
                out->partition_ms = p.partition_ms;
                out->find_ms      = p.find_ms;
                out->other_ms     = p.other_ms;
                out->total_ms     = ms;
                out->hist_bytes   = p.hist_bytes;
                out->hist_rows    = p.hist_rows;
                out->hist_builds  = p.hist_builds;
                out->launches     = b->round_launches;
                for (uint32_t k = 0; k < 16; ++k)
                {
                    out->build_ms[k]   = p.build_ms[k];
                    out->build_rows[k] = p.build_rows[k];
                }
            });
    }

    int bb_booster_eval_arm(bb_booster *b, bb_plane const *valid, float const *labels,
                            float const *init_scores)
    {
        return guarded(
            [&]
            {
                need(b != nullptr && valid != nullptr && labels != nullptr,
                     "bb_booster_eval_arm: null argument");
                if (b->sharded)
                {
                    throw ConfigError("bb_booster_eval_arm: a row-sharded fit has no "
                                      "validation plane; score the model with a predict plan");
                }
                Plane const &v = valid->p;
                Plane const &t = *b->plane;
                need(v.n_feats == t.n_feats && v.u8 == t.u8 &&
                         std::equal(t.h_cut_off, t.h_cut_off + t.n_feats + 1, v.h_cut_off) &&
                         std::equal(t.h_cuts, t.h_cuts + t.h_cut_off[t.n_feats], v.h_cuts),
                     "bb_booster_eval_arm: the validation plane was not binned with the "
                     "training plane's cuts");
                BB_CHECK(cudaStreamSynchronize(b->stream));
                b->release_eval();
                uint64_t const n = v.n_rows;
                uint32_t const K = b->n_classes;
                b->vcap          = b->trees.n / K;
                b->vlabels       = dmalloc<float>(n);
                b->vscores       = dmalloc<float>(n * K);
                b->vlosses       = dmalloc<float>(b->vcap);
                b->vcount        = dmalloc<uint32_t>(1);
                b->vpartial      = dmalloc<double>(k_eval_blocks);
                BB_CHECK(cudaMemcpyAsync(b->vlabels, labels, n * 4, cudaMemcpyHostToDevice,
                                         b->stream));
                if (init_scores != nullptr)
                {
                    BB_CHECK(cudaMemcpyAsync(b->vscores, init_scores, n * K * 4,
                                             cudaMemcpyHostToDevice, b->stream));
                }
                else
                {
                    for (uint32_t k = 0; k < K; ++k)
                    {
                        fill_kernel<<<blocks(n), 256, 0, b->stream>>>(
                            b->vscores + (k * n), K > 1 ? b->init_k[k] : b->init, n);
                        BB_LAUNCH("fill_kernel");
                    }
                }
                BB_CHECK(cudaMemsetAsync(b->vcount, 0, 4, b->stream));
                b->vplane = &v;
                // a captured round without the eval step is stale
                if (b->graph != nullptr)
                {
                    BB_CHECK(cudaGraphExecDestroy(b->graph));
                    b->graph = nullptr;
                }
                BB_CHECK(cudaStreamSynchronize(b->stream));
            });
    }

    int bb_booster_eval_losses(bb_booster const *b, float *out, uint32_t cap, uint32_t *n)
    {
        return guarded(
            [&]
            {
                need(b != nullptr && n != nullptr && (out != nullptr || cap == 0),
                     "bb_booster_eval_losses: null argument");
                need(b->vplane != nullptr, "bb_booster_eval_losses: no validation plane armed");
                BB_CHECK(cudaStreamSynchronize(b->stream));
                uint32_t c = 0;
                BB_CHECK(cudaMemcpy(&c, b->vcount, 4, cudaMemcpyDeviceToHost));
                c  = std::min(c, b->vcap);
                *n = c;
                uint32_t const m = std::min(c, cap);
                if (m > 0)
                {
                    BB_CHECK(cudaMemcpy(out, b->vlosses, m * 4ull, cudaMemcpyDeviceToHost));
                }
            });
    }

    int bb_booster_eval_scores(bb_booster const *b, float *out)
    {
        return guarded(
            [&]
            {
                need(b != nullptr && out != nullptr, "bb_booster_eval_scores: null argument");
                need(b->vplane != nullptr, "bb_booster_eval_scores: no validation plane armed");
                BB_CHECK(cudaStreamSynchronize(b->stream));
                uint64_t const n = b->vplane->n_rows;
                uint32_t const K = b->n_classes;
                std::vector<float> cm(n * K);
                BB_CHECK(cudaMemcpy(cm.data(), b->vscores, n * K * 4, cudaMemcpyDeviceToHost));
                for (uint64_t i = 0; i < n; ++i)
                {
                    for (uint32_t k = 0; k < K; ++k)
                    {
                        out[(i * K) + k] = cm[(k * n) + i];
                    }
                }
            });
    }

    int bb_booster_truncate(bb_booster *b, uint32_t n_rounds)
    {
        return guarded(
            [&]
            {
                need(b != nullptr, "bb_booster_truncate: null argument");
                need(n_rounds * b->n_classes <= b->n_trees,
                     "bb_booster_truncate: more rounds than the booster ran");
                BB_CHECK(cudaStreamSynchronize(b->stream));
                b->n_trees   = n_rounds * b->n_classes;
                b->truncated = true;
            });
    }

    void bb_booster_destroy(bb_booster *b)
    {
        if (b == nullptr)
        {
            return;
        }
        cudaStreamSynchronize(b->stream);
        if (b->graph != nullptr)
        {
            cudaGraphExecDestroy(b->graph);
        }
        b->release_eval();
        b->sampler.reset();
        b->grower.reset();
        b->scratch.release();
        b->trees.release();
        void *ps[] = {b->labels, b->scores, b->gh,     b->rows,   b->leaf_id, b->round,
                      b->sbits,  b->srows,  b->scount, b->sbsum, b->weights};
        for (void *p : ps)
        {
            cudaFree(p);
        }
        cudaEventDestroy(b->ev0);
        cudaEventDestroy(b->ev1);
        cudaStreamDestroy(b->stream);
        delete b;
    }

    int bb_grow_tree(bb_plane const *plane, bb_train_cfg const *cfg, float const *grad,
                     float const *hess, uint32_t const *rows, uint64_t n_sel_rows,
                     uint32_t *feature, float *value, uint32_t *left, uint32_t *right,
                     uint8_t *default_left, float *gain, float *cover, uint32_t *split_bin,
                     uint32_t *meta, float *values, uint32_t *leaf_ids)
    {
        return guarded(
            [&]
            {
                need(plane != nullptr && cfg != nullptr && grad != nullptr && hess != nullptr,
                     "bb_grow_tree: null argument");
                Plane const   &p = plane->p;
                uint64_t const n = p.n_rows;
                uint64_t const m = rows == nullptr ? n : n_sel_rows;
                need(m <= n, "bb_grow_tree: more sampled rows than rows");
                for (uint64_t k = 0; rows != nullptr && k < m; ++k)
                {
                    need(rows[k] < n && (k == 0 || rows[k] > rows[k - 1]),
                         "bb_grow_tree: rows must be ascending row ids below n_rows");
                }
                cudaStream_t   s;
                BB_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
                std::vector<float2> gh(n);
                for (uint64_t i = 0; i < n; ++i)
                {
                    gh[i] = make_float2(grad[i], hess[i]);
                }
                float2   *d_gh  = dmalloc<float2>(n);
                uint32_t *d_rows = dmalloc<uint32_t>(std::max<uint64_t>(m, 1));
                uint32_t *d_leaf = dmalloc<uint32_t>(n);
                float    *d_val  = dmalloc<float>(n);
                TreeStore ts;
                try
                {
                    BB_CHECK(cudaMemcpyAsync(d_gh, gh.data(), n * 8, cudaMemcpyHostToDevice, s));
                    if (rows == nullptr)
                    {
                        iota_kernel<<<blocks(n), 256, 0, s>>>(d_rows, n);
                        BB_LAUNCH("iota_kernel");
                    }
                    else if (m > 0)
                    {
                        BB_CHECK(cudaMemcpyAsync(d_rows, rows, m * 4, cudaMemcpyHostToDevice, s));
                    }
                    // values via the fused score update on a zeroed buffer, lr = 1
                    BB_CHECK(cudaMemsetAsync(d_val, 0, n * 4, s));
                    Grower g(p, grow_config(*cfg), selection(*cfg, p.n_feats),
                             static_cast<uint32_t>(std::max<uint64_t>(m, 1)), s);
                    g.set_monotone(monotone(*cfg));
                    g.set_interaction(interaction(*cfg, p.n_feats));
                    g.set_seed(cfg->seed);
                    ts.alloc(g.max_nodes(), 1);
                    g.grow(d_gh, d_rows, static_cast<uint32_t>(m), ts.t, d_leaf, d_val, 1.0F);
                    BB_CHECK(cudaStreamSynchronize(s));
                    ts.download(0, feature, value, left, right, default_left, gain, cover,
                                split_bin, meta);
                    std::vector<uint32_t> ids(n);
                    BB_CHECK(cudaMemcpy(ids.data(), d_leaf, n * 4, cudaMemcpyDeviceToHost));
                    // each row takes its leaf's value itself (a stamped 0 + v
                    // would turn a -0.0 leaf into +0.0)
                    for (uint64_t k = 0; k < m; ++k)
                    {
                        uint64_t const r = rows == nullptr ? k : rows[k];
                        values[r]        = value[ids[r]];
                        leaf_ids[r]      = ids[r];
                    }
                }
                catch (...)
                {
                    ts.release();
                    cudaFree(d_gh);
                    cudaFree(d_rows);
                    cudaFree(d_leaf);
                    cudaFree(d_val);
                    cudaStreamDestroy(s);
                    throw;
                }
                ts.release();
                cudaFree(d_gh);
                cudaFree(d_rows);
                cudaFree(d_leaf);
                cudaFree(d_val);
                BB_CHECK(cudaStreamDestroy(s));
            });
    }

    int bb_populate(bb_plane const *plane, bb_train_cfg const *cfg, float const *grad,
                    float const *hess, uint32_t const *rows, uint64_t n_sel_rows, double *out)
    {
        return guarded(
            [&]
            {
                need(plane != nullptr && cfg != nullptr && grad != nullptr && hess != nullptr &&
                         out != nullptr,
                     "bb_populate: null argument");
                Plane const   &p = plane->p;
                uint64_t const n = p.n_rows;
                uint64_t const m = rows == nullptr ? n : n_sel_rows;
                need(m <= n, "bb_populate: more rows than the plane holds");
                for (uint64_t k = 0; rows != nullptr && k < m; ++k)
                {
                    need(rows[k] < n && (k == 0 || rows[k] > rows[k - 1]),
                         "bb_populate: rows must be ascending row ids below n_rows");
                }
                cudaStream_t s;
                BB_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
                std::vector<float2> gh(n);
                for (uint64_t i = 0; i < n; ++i)
                {
                    gh[i] = make_float2(grad[i], hess[i]);
                }
                float2   *d_gh   = dmalloc<float2>(n);
                uint32_t *d_rows = dmalloc<uint32_t>(std::max<uint64_t>(m, 1));
                try
                {
                    BB_CHECK(cudaMemcpyAsync(d_gh, gh.data(), n * 8, cudaMemcpyHostToDevice, s));
                    if (rows == nullptr)
                    {
                        iota_kernel<<<blocks(n), 256, 0, s>>>(d_rows, n);
                        BB_LAUNCH("iota_kernel");
                    }
                    else if (m > 0)
                    {
                        BB_CHECK(cudaMemcpyAsync(d_rows, rows, m * 4, cudaMemcpyHostToDevice, s));
                    }
                    GrowConfig gc = grow_config(*cfg);
                    gc.tp.max_depth = 1;
                    Grower g(p, gc, selection(*cfg, p.n_feats),
                             static_cast<uint32_t>(std::max<uint64_t>(m, 1)), s);
                    g.set_seed(cfg->seed);
                    g.populate(d_gh, d_rows, static_cast<uint32_t>(m),
                               reinterpret_cast<double2 *>(out));
                }
                catch (...)
                {
                    cudaFree(d_gh);
                    cudaFree(d_rows);
                    cudaStreamDestroy(s);
                    throw;
                }
                cudaFree(d_gh);
                cudaFree(d_rows);
                BB_CHECK(cudaStreamDestroy(s));
            });
    }
}

// ---------------------------------------------------------------------------
// bb_predict_static: ensemble predict that allocates no device memory.
//
// Who needs this: a caller that may not call cudaMalloc / cudaFree on its
// serving path. Two kinds are common. A host whose device memory belongs to
// another allocator under a fixed budget (a framework's caching allocator,
// or a serving process that reserves all device memory up front) cannot let
// a library take more. And a latency-bound caller cannot afford the
// device-wide synchronisation that cudaMalloc and cudaFree imply. bb_predict
// copies the packed ensemble into freshly allocated device buffers on every
// call; this variant copies it into one fixed array that the library holds
// for the life of the process instead.
//
// The array: k_static_bytes (11,534,336 bytes, 11 MiB) of file-scope device
// memory, present on every GPU that loads the library until the process
// exits. It holds at most k_max_static_nodes (524,288) tree nodes,
// k_max_static_trees (65,536) trees and k_max_static_feats (65,536)
// features; larger ensembles are refused with BB_ERR_CONFIG and nothing runs.
//
// Set-up: the first call on each device resolves the array's device address
// (cudaGetSymbolAddress, with that device current) and caches it; make that
// first call before any stream capture. Every call shares the one array and
// leaves the last ensemble in it: calls whose work overlaps on the GPU (from
// several host threads, or before the previous call's kernel has run) race
// on it. The kernel runs on the legacy default stream and the call returns
// once it is enqueued; synchronise that stream before reading out. The
// plane's device must be the calling thread's current device (refused with
// BB_ERR_CONFIG otherwise), and a plane with no rows (a request plane before
// its first refill) returns success without touching the array.

namespace bb
{
namespace
{

constexpr uint32_t k_max_static_nodes = 524288;
constexpr uint32_t k_max_static_trees = 65536;
constexpr uint32_t k_max_static_feats = 65536;

// layout (4-byte words, then the u8 default directions)
constexpr size_t k_off_roots   = 0;
constexpr size_t k_off_last    = k_off_roots + k_max_static_trees;
constexpr size_t k_off_feature = k_off_last + k_max_static_feats;
constexpr size_t k_off_split   = k_off_feature + k_max_static_nodes;
constexpr size_t k_off_left    = k_off_split + k_max_static_nodes;
constexpr size_t k_off_right   = k_off_left + k_max_static_nodes;
constexpr size_t k_off_value   = k_off_right + k_max_static_nodes;
constexpr size_t k_words       = k_off_value + k_max_static_nodes;
constexpr size_t k_static_bytes = (k_words * 4) + k_max_static_nodes;

static __device__ __align__(256) unsigned char g_predict_scratch[k_static_bytes];

constexpr int k_max_devices = 64;
std::mutex    g_mu;
void         *g_addr[k_max_devices] = {};

// The array's device address on the current device, resolved once.
unsigned char *scratch_address()
{
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= k_max_devices)
    {
        throw ConfigError("bb_predict_static: device ordinal above 63");
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_addr[dev] == nullptr)
    {
        void *p = nullptr;
        check(cudaGetSymbolAddress(&p, g_predict_scratch), "cudaGetSymbolAddress");
        g_addr[dev] = p;
    }
    return static_cast<unsigned char *>(g_addr[dev]);
}

// The predict walk of bb_predict (one thread per row, trees in order, leaves
// summed in float, out = init + sum * lr), reading the ensemble from the
// fixed array.
template <typename BinT>
__global__ void predict_static_kernel(BinT const *__restrict__ bins, uint64_t n_pad,
                                      uint64_t n, uint32_t n_trees,
                                      unsigned char const *__restrict__ scratch, float lr,
                                      float init, float *__restrict__ out)
{
    uint64_t const r = (static_cast<uint64_t>(blockIdx.x) * blockDim.x) + threadIdx.x;
    if (r >= n)
    {
        return;
    }
    auto const *w       = reinterpret_cast<uint32_t const *>(scratch);
    auto const *roots   = w + k_off_roots;
    auto const *last    = w + k_off_last;
    auto const *feature = w + k_off_feature;
    auto const *split   = w + k_off_split;
    auto const *left    = w + k_off_left;
    auto const *right   = w + k_off_right;
    auto const *value   = reinterpret_cast<float const *>(w + k_off_value);
    auto const *dl      = scratch + (k_words * 4);
    float       acc     = 0.0F;
    for (uint32_t t = 0; t < n_trees; ++t)
    {
        uint32_t const base = roots[t];
        uint32_t       idx  = base;
        while (feature[idx] != k_leaf_flag)
        {
            uint32_t const f = feature[idx];
            uint32_t const b = bins[(static_cast<uint64_t>(f) * n_pad) + r];
            idx = base + (routes_left(b, last[f], split[idx], dl[idx] != 0) ? left[idx]
                                                                           : right[idx]);
        }
        acc = acc + value[idx];
    }
    out[r] = init + (acc * lr);
}

} // namespace
} // namespace bb

extern "C" int bb_predict_static(bb_plane const *plane, uint32_t n_trees,
                                 uint32_t const *roots, uint32_t n_nodes,
                                 uint32_t const *feature, uint32_t const *split_bin,
                                 uint32_t const *left, uint32_t const *right,
                                 uint8_t const *default_left, float const *value, float lr,
                                 float init, float *out_device)
{
    return guarded([&] {
        need(plane != nullptr && roots != nullptr && feature != nullptr &&
                        split_bin != nullptr && left != nullptr && right != nullptr &&
                        default_left != nullptr && value != nullptr && out_device != nullptr,
                    "bb_predict_static: null argument");
        Plane const &p = plane->p;
        if (n_nodes > k_max_static_nodes || n_trees > k_max_static_trees ||
            p.n_feats > k_max_static_feats)
        {
            throw ConfigError(
                "bb_predict_static: the ensemble exceeds the fixed device array (at most "
                "524,288 nodes, 65,536 trees, 65,536 features); use bb_predict");
        }
        need(n_trees > 0 && n_nodes > 0, "bb_predict_static: empty ensemble");
        // every walk must end: children lie after their parent inside the tree
        for (uint32_t t = 0; t < n_trees; ++t)
        {
            uint32_t const b = roots[t];
            uint32_t const e = t + 1 < n_trees ? roots[t + 1] : n_nodes;
            need(b < e && e <= n_nodes, "bb_predict_static: bad tree roots");
            for (uint32_t i = b; i < e; ++i)
            {
                if (feature[i] == k_leaf_flag)
                {
                    continue;
                }
                need(feature[i] < p.n_feats,
                            "bb_predict_static: node feature out of range");
                need(left[i] > i - b && right[i] > i - b && b + left[i] < e &&
                                b + right[i] < e,
                            "bb_predict_static: a child id must follow its parent in its tree");
            }
        }
        int cur = 0;
        check(cudaGetDevice(&cur), "cudaGetDevice");
        if (cur != p.device)
        {
            throw ConfigError("bb_predict_static: the plane's device must be the current "
                              "device (cudaSetDevice / bb_select_device first)");
        }
        if (p.n_rows == 0)
        {
            return; // a request plane before its first refill: nothing to score
        }
        unsigned char *scr = scratch_address();
        auto          *w   = reinterpret_cast<uint32_t *>(scr);
        uint32_t       last_bins[256];
        // last bins go up in slices through a small host buffer
        for (uint32_t f0 = 0; f0 < p.n_feats; f0 += 256)
        {
            uint32_t const m = p.n_feats - f0 < 256 ? p.n_feats - f0 : 256;
            for (uint32_t k = 0; k < m; ++k)
            {
                last_bins[k] = p.h_cut_off[f0 + k + 1] - p.h_cut_off[f0 + k] - 1;
            }
            check(cudaMemcpy(w + k_off_last + f0, last_bins, m * 4, cudaMemcpyHostToDevice),
                  "cudaMemcpy");
        }
        check(cudaMemcpy(w + k_off_roots, roots, n_trees * 4ULL, cudaMemcpyHostToDevice),
              "cudaMemcpy");
        check(cudaMemcpy(w + k_off_feature, feature, n_nodes * 4ULL, cudaMemcpyHostToDevice),
              "cudaMemcpy");
        check(cudaMemcpy(w + k_off_split, split_bin, n_nodes * 4ULL, cudaMemcpyHostToDevice),
              "cudaMemcpy");
        check(cudaMemcpy(w + k_off_left, left, n_nodes * 4ULL, cudaMemcpyHostToDevice),
              "cudaMemcpy");
        check(cudaMemcpy(w + k_off_right, right, n_nodes * 4ULL, cudaMemcpyHostToDevice),
              "cudaMemcpy");
        check(cudaMemcpy(w + k_off_value, value, n_nodes * 4ULL, cudaMemcpyHostToDevice),
              "cudaMemcpy");
        check(cudaMemcpy(scr + (k_words * 4), default_left, n_nodes, cudaMemcpyHostToDevice),
              "cudaMemcpy");
        uint64_t const n      = p.n_rows;
        uint32_t const blocks = static_cast<uint32_t>((n + 255) / 256);
        if (p.u8)
        {
            predict_static_kernel<uint8_t><<<blocks, 256>>>(
                static_cast<uint8_t const *>(p.bins), p.n_pad, n, n_trees, scr, lr, init,
                out_device);
        }
        else
        {
            predict_static_kernel<uint16_t><<<blocks, 256>>>(
                static_cast<uint16_t const *>(p.bins), p.n_pad, n, n_trees, scr, lr, init,
                out_device);
        }
        check(cudaGetLastError(), "predict_static_kernel");
    });
}
