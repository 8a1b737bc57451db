// Cut fitting on the device (bb_fit_cuts): BinMapper::from_sample per column
// (src/bin_mapper.cpp:240-252 over create_cuts, :159-232), the same cuts as
// the host restatement in bonsai_b200/binning.py for the same working set.
//
// Per column of the sample: the NaN-free values as order-preserving 32-bit
// keys (the reference's radix key: flip every bit of a negative, the sign bit
// of a non-negative, so -0.0 sorts before +0.0 as in its sort_floats,
// :115-157); an LSD radix sort by one CTA (four 8-bit passes, each a digit
// histogram, a scan and a stable scatter ranked per warp with match_any);
// then the runs of equal values (run-length encoding under operator<, so the
// two zeros are one run whose representative is the first, -0.0 when
// present), and the lightest exact rule: every distinct value when they fit
// the cut budget, else the count-weighted greedy walk when some value is at
// least a mean bin (greedy_weighted_cuts, :38-96; one thread walks the
// runs), else the quantile stride over the sorted values; then the FLT_MAX
// closer and the +inf missing sentinel.
#include "bonsai_b200.h"
#include "common.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace bb
{
namespace
{

constexpr uint32_t k_cut_threads  = 1024;
constexpr uint32_t k_tile_rows_c  = 256;
constexpr uint32_t k_tile_feats_c = 32;
constexpr size_t   k_cut_mem      = size_t{1} << 30; // device scratch per column group

__device__ __forceinline__ uint32_t key_of(float v)
{
    uint32_t const b = __float_as_uint(v);
    return b ^ ((b >> 31) != 0 ? 0xFFFFFFFFu : 0x80000000u);
}

__device__ __forceinline__ float value_of(uint32_t k)
{
    return __uint_as_float((k >> 31) != 0 ? k ^ 0x80000000u : ~k);
}

// std::midpoint for float, the greedy rule's cut (src/bin_mapper.cpp:95): the
// correctly rounded half-sum that never overflows. With both magnitudes at
// most FLT_MAX / 2 the sum cannot overflow; above that each operand is halved
// before the add, except one below twice the smallest normal (halving it
// would round), which is added whole -- the cases of the C++ standard's
// midpoint proposal (P0811). Division by 2 is exact or correctly rounded, and
// the build keeps denormals (no flush to zero).
__device__ __forceinline__ float midpoint_f(float a, float b)
{
    float const hi = FLT_MAX / 2.0F;
    float const lo = FLT_MIN * 2.0F;
    float const aa = fabsf(a);
    float const ab = fabsf(b);
    if (aa <= hi && ab <= hi)
    {
        return (a + b) / 2.0F;
    }
    if (aa < lo)
    {
        return a + b / 2.0F;
    }
    if (ab < lo)
    {
        return a / 2.0F + b;
    }
    return a / 2.0F + b / 2.0F;
}

// The NaN-free values of columns [f0, f0 + nf) of row-major S (n x F) as
// keys, column c's at keys[c * n + ...] (order within a column is free: the
// sort makes it canonical); counts[c] ends as the column's count.
__global__ void __launch_bounds__(k_tile_rows_c)
    gather_keys_kernel(float const *__restrict__ S, uint64_t n, uint32_t F, uint32_t f0,
                       uint32_t nf, uint32_t *__restrict__ keys, uint32_t *counts)
{
    __shared__ float    tile[k_tile_rows_c][k_tile_feats_c + 1];
    __shared__ uint32_t wcnt[k_tile_feats_c][k_tile_rows_c / 32];
    __shared__ uint32_t base[k_tile_feats_c];
    uint64_t const      r0   = static_cast<uint64_t>(blockIdx.x) * k_tile_rows_c;
    uint32_t const      c0   = blockIdx.y * k_tile_feats_c; // within the group
    uint32_t const      ncol = min(k_tile_feats_c, nf - c0);
    uint32_t const      t    = threadIdx.x;
    uint32_t const      lane = t & 31u;
    uint32_t const      w    = t >> 5;
    for (uint32_t i = t; i < k_tile_rows_c * k_tile_feats_c; i += k_tile_rows_c)
    {
        uint32_t const rr = i / k_tile_feats_c;
        uint32_t const cc = i % k_tile_feats_c;
        uint64_t const r  = r0 + rr;
        tile[rr][cc] = (r < n && cc < ncol) ? S[(r * F) + f0 + c0 + cc] : __int_as_float(0x7FC00000);
    }
    __syncthreads();
    bool     valid[k_tile_feats_c];
    uint32_t rank[k_tile_feats_c];
#pragma unroll
    for (uint32_t cc = 0; cc < k_tile_feats_c; ++cc)
    {
        valid[cc]           = !isnan(tile[t][cc]);
        uint32_t const mask = __ballot_sync(0xFFFFFFFFu, valid[cc]);
        rank[cc]            = __popc(mask & ((1u << lane) - 1u));
        if (lane == 0)
        {
            wcnt[cc][w] = __popc(mask);
        }
    }
    __syncthreads();
    if (t < ncol)
    {
        uint32_t run = 0;
        for (uint32_t x = 0; x < k_tile_rows_c / 32; ++x)
        {
            uint32_t const c = wcnt[t][x];
            wcnt[t][x]       = run;
            run += c;
        }
        base[t] = run > 0 ? atomicAdd(&counts[c0 + t], run) : 0u;
    }
    __syncthreads();
    for (uint32_t cc = 0; cc < ncol; ++cc)
    {
        if (valid[cc])
        {
            keys[(static_cast<uint64_t>(c0 + cc) * n) + base[cc] + wcnt[cc][w] + rank[cc]] =
                key_of(tile[t][cc]);
        }
    }
}

// Column blockIdx.x's keys sorted ascending: four stable 8-bit LSD passes
// between a and b (the result back in a).
__global__ void __launch_bounds__(k_cut_threads)
    sort_keys_kernel(uint32_t *__restrict__ a, uint32_t *__restrict__ b, uint64_t n,
                     uint32_t const *counts)
{
    __shared__ uint32_t hist[256];
    __shared__ uint32_t base[256];
    __shared__ uint32_t tot[256];
    __shared__ uint16_t wc[k_cut_threads / 32][256];
    uint32_t const      col  = blockIdx.x;
    uint32_t const      m    = counts[col];
    uint32_t const      t    = threadIdx.x;
    uint32_t const      lane = t & 31u;
    uint32_t const      w    = t >> 5;
    uint32_t           *src  = a + (static_cast<uint64_t>(col) * n);
    uint32_t           *dst  = b + (static_cast<uint64_t>(col) * n);
    for (uint32_t shift = 0; shift < 32; shift += 8)
    {
        if (t < 256)
        {
            hist[t] = 0;
        }
        __syncthreads();
        for (uint32_t i = t; i < m; i += k_cut_threads)
        {
            atomicAdd(&hist[(src[i] >> shift) & 0xFFu], 1u);
        }
        __syncthreads();
        if (t == 0)
        {
            uint32_t run = 0;
            for (uint32_t d = 0; d < 256; ++d)
            {
                base[d] = run;
                run += hist[d];
            }
        }
        __syncthreads();
        for (uint32_t t0 = 0; t0 < m; t0 += k_cut_threads)
        {
            for (uint32_t x = t; x < (k_cut_threads / 32) * 256; x += k_cut_threads)
            {
                wc[x / 256][x % 256] = 0;
            }
            __syncthreads();
            uint32_t const i     = t0 + t;
            bool const     ok    = i < m;
            uint32_t const key   = ok ? src[i] : 0u;
            uint32_t const d     = (key >> shift) & 0xFFu;
            // lanes with the same digit, in lane order (an idle lane only
            // matches itself)
            uint32_t const peers = __match_any_sync(0xFFFFFFFFu, ok ? d : 256u + lane);
            uint32_t const r     = __popc(peers & ((1u << lane) - 1u));
            if (ok && r == 0)
            {
                wc[w][d] = static_cast<uint16_t>(__popc(peers));
            }
            __syncthreads();
            if (t < 256)
            {
                uint32_t run = 0;
                for (uint32_t x = 0; x < k_cut_threads / 32; ++x)
                {
                    uint32_t const c = wc[x][t];
                    wc[x][t]         = static_cast<uint16_t>(run);
                    run += c;
                }
                tot[t] = run;
            }
            __syncthreads();
            if (ok)
            {
                dst[base[d] + wc[w][d] + r] = key;
            }
            __syncthreads();
            if (t < 256)
            {
                base[t] += tot[t];
            }
            __syncthreads();
        }
        uint32_t *x = src;
        src         = dst;
        dst         = x;
    }
}

// Column blockIdx.x's cuts from its sorted keys into cuts[col * max_bin ...],
// their number into n_cuts[col]. starts: scratch for the run starts.
__global__ void __launch_bounds__(k_cut_threads)
    column_cuts_kernel(uint32_t const *__restrict__ keys, uint64_t n,
                       uint32_t const *counts, uint32_t *__restrict__ starts,
                       uint32_t max_bin, float *__restrict__ cuts, uint32_t *n_cuts)
{
    __shared__ uint32_t wsum[k_cut_threads / 32];
    __shared__ uint32_t s_maxrun;
    uint32_t const      col    = blockIdx.x;
    uint32_t const      m      = counts[col];
    uint32_t const      t      = threadIdx.x;
    uint32_t const      lane   = t & 31u;
    uint32_t const      w      = t >> 5;
    uint32_t const     *k      = keys + (static_cast<uint64_t>(col) * n);
    uint32_t           *st     = starts + (static_cast<uint64_t>(col) * n);
    float              *out    = cuts + (static_cast<uint64_t>(col) * max_bin);
    uint32_t const      budget = max_bin - 2;
    // the runs of equal values: starts in order (value(i - 1) < value(i))
    uint32_t done = 0;
    for (uint32_t t0 = 0; t0 < m; t0 += k_cut_threads)
    {
        uint32_t const i    = t0 + t;
        bool const     head = i < m && (i == 0 || value_of(k[i - 1]) < value_of(k[i]));
        uint32_t const mask = __ballot_sync(0xFFFFFFFFu, head);
        if (lane == 0)
        {
            wsum[w] = __popc(mask);
        }
        __syncthreads();
        uint32_t before = 0;
        uint32_t total  = 0;
        for (uint32_t x = 0; x < k_cut_threads / 32; ++x)
        {
            before += x < w ? wsum[x] : 0u;
            total += wsum[x];
        }
        if (head)
        {
            st[done + before + __popc(mask & ((1u << lane) - 1u))] = i;
        }
        done += total;
        __syncthreads();
    }
    uint32_t const nd = done;
    // the longest run
    uint32_t longest = 0;
    for (uint32_t j = t; j < nd; j += k_cut_threads)
    {
        uint32_t const e = j + 1 < nd ? st[j + 1] : m;
        longest          = max(longest, e - st[j]);
    }
    for (uint32_t o = 16; o > 0; o >>= 1)
    {
        longest = max(longest, __shfl_xor_sync(0xFFFFFFFFu, longest, o));
    }
    if (t == 0)
    {
        s_maxrun = 0;
    }
    __syncthreads();
    if (lane == 0)
    {
        atomicMax(&s_maxrun, longest);
    }
    __syncthreads();
    double const mean_bin = static_cast<double>(m) / static_cast<double>(budget + 1);
    if (nd <= budget)
    {
        // every distinct value, its run's first element
        for (uint32_t j = t; j < nd; j += k_cut_threads)
        {
            out[j] = value_of(k[st[j]]);
        }
        __syncthreads();
        if (t == 0)
        {
            uint32_t c = nd;
            if (c == 0 || out[c - 1] < FLT_MAX)
            {
                out[c++] = FLT_MAX;
            }
            out[c++]    = __int_as_float(0x7F800000); // +inf
            n_cuts[col] = c;
        }
        return;
    }
    if (t != 0)
    {
        return;
    }
    uint32_t c = 0;
    if (static_cast<double>(s_maxrun) >= mean_bin)
    {
        // greedy_weighted_cuts over the runs
        uint64_t n_big   = 0;
        uint64_t big_sum = 0;
        for (uint32_t j = 0; j < nd; ++j)
        {
            uint32_t const cnt = (j + 1 < nd ? st[j + 1] : m) - st[j];
            if (static_cast<double>(cnt) >= mean_bin)
            {
                ++n_big;
                big_sum += cnt;
            }
        }
        uint64_t const n_groups    = static_cast<uint64_t>(budget) + 1;
        int64_t        rest_sum    = static_cast<int64_t>(m) - static_cast<int64_t>(big_sum);
        uint64_t       rest_groups = n_groups - n_big;
        double bin_size = rest_groups != 0 ? static_cast<double>(rest_sum) /
                                                 static_cast<double>(rest_groups)
                                           : mean_bin;
        uint64_t in_bin = 0;
        for (uint32_t j = 0; j + 1 < nd && c < budget; ++j)
        {
            uint32_t const cnt  = st[j + 1] - st[j];
            uint32_t const cnt1 = (j + 2 < nd ? st[j + 2] : m) - st[j + 1];
            bool const     big  = static_cast<double>(cnt) >= mean_bin;
            bool const     big1 = static_cast<double>(cnt1) >= mean_bin;
            if (!big)
            {
                rest_sum -= cnt;
            }
            in_bin += cnt;
            if (big || static_cast<double>(in_bin) >= bin_size ||
                (big1 && static_cast<double>(in_bin) >= bin_size / 2.0))
            {
                float const a   = value_of(k[st[j]]);
                float const b   = value_of(k[st[j + 1]]);
                float const mid = midpoint_f(a, b);
                if (c == 0 || out[c - 1] < mid)
                {
                    out[c++] = mid;
                }
                in_bin = 0;
                if (!big && rest_groups > 1)
                {
                    --rest_groups;
                    bin_size = static_cast<double>(rest_sum) / static_cast<double>(rest_groups);
                }
            }
        }
    }
    else
    {
        // the quantile stride over the sorted values
        uint64_t const q    = (static_cast<uint64_t>(m) + budget) / (budget + 1);
        uint64_t const step = q > 0 ? q : 1;
        for (uint64_t x = step; x < m; x += step)
        {
            float const v = value_of(k[x]);
            if (c == 0 || out[c - 1] < v)
            {
                out[c++] = v;
            }
        }
    }
    if (c == 0 || out[c - 1] < FLT_MAX)
    {
        out[c++] = FLT_MAX;
    }
    out[c++]    = __int_as_float(0x7F800000);
    n_cuts[col] = c;
}

struct Scratch
{
    void *p[7] = {};
    ~Scratch()
    {
        for (void *q : p)
        {
            if (q != nullptr)
            {
                cudaFree(q);
            }
        }
    }
};

} // namespace
} // namespace bb

using namespace bb;

extern "C" int bb_fit_cuts(float const *S, uint64_t n_rows, uint32_t n_feats, int s_on_device,
                           uint32_t max_bin, float *cuts, uint32_t cuts_cap, uint32_t *cut_off)
{
    try
    {
        if (S == nullptr || cuts == nullptr || cut_off == nullptr || n_feats == 0)
        {
            throw std::invalid_argument("bb_fit_cuts: null argument or no features");
        }
        if (max_bin < 3 || max_bin > 65535)
        {
            throw std::invalid_argument("bb_fit_cuts: max_bin must be in [3, 65535]");
        }
        if (n_rows >= (1ull << 32))
        {
            throw ConfigError("bb_fit_cuts: a sample of 2^32 or more rows; sample the rows first");
        }
        uint64_t const n = std::max<uint64_t>(n_rows, 1);
        // columns per group: keys twice and the run starts, 12 bytes per value
        uint32_t const group = static_cast<uint32_t>(std::max<uint64_t>(
            1, std::min<uint64_t>(n_feats, k_cut_mem / (12 * n))));
        Scratch        sc;
        size_t const   s_bytes = static_cast<size_t>(n_rows) * n_feats * sizeof(float);
        float const   *Sd      = S;
        if (s_on_device == 0 && n_rows > 0)
        {
            check(cudaMalloc(&sc.p[0], s_bytes), "cudaMalloc");
            check(cudaMemcpy(sc.p[0], S, s_bytes, cudaMemcpyHostToDevice), "cudaMemcpy");
            Sd = static_cast<float const *>(sc.p[0]);
        }
        check(cudaMalloc(&sc.p[1], static_cast<size_t>(group) * n * 4), "cudaMalloc");
        check(cudaMalloc(&sc.p[2], static_cast<size_t>(group) * n * 4), "cudaMalloc");
        check(cudaMalloc(&sc.p[3], static_cast<size_t>(group) * n * 4), "cudaMalloc");
        check(cudaMalloc(&sc.p[4], static_cast<size_t>(group) * max_bin * 4), "cudaMalloc");
        check(cudaMalloc(&sc.p[5], static_cast<size_t>(group) * 4), "cudaMalloc");
        check(cudaMalloc(&sc.p[6], static_cast<size_t>(group) * 4), "cudaMalloc");
        auto *ka    = static_cast<uint32_t *>(sc.p[1]);
        auto *kb    = static_cast<uint32_t *>(sc.p[2]);
        auto *st    = static_cast<uint32_t *>(sc.p[3]);
        auto *cd    = static_cast<float *>(sc.p[4]);
        auto *cn    = static_cast<uint32_t *>(sc.p[5]); // values per column
        auto *nc    = static_cast<uint32_t *>(sc.p[6]); // cuts per column
        std::vector<float>    hc(static_cast<size_t>(group) * max_bin);
        std::vector<uint32_t> hn(group);
        uint32_t              at = 0;
        cut_off[0]               = 0;
        for (uint32_t f0 = 0; f0 < n_feats; f0 += group)
        {
            uint32_t const nf = std::min(group, n_feats - f0);
            check(cudaMemset(cn, 0, nf * 4ull), "cudaMemset");
            if (n_rows > 0)
            {
                dim3 const grid(ceil_div(n_rows, k_tile_rows_c), ceil_div(nf, k_tile_feats_c));
                gather_keys_kernel<<<grid, k_tile_rows_c>>>(Sd, n_rows, n_feats, f0, nf, ka, cn);
                check(cudaGetLastError(), "gather_keys_kernel");
                sort_keys_kernel<<<nf, k_cut_threads>>>(ka, kb, n, cn);
                check(cudaGetLastError(), "sort_keys_kernel");
            }
            column_cuts_kernel<<<nf, k_cut_threads>>>(ka, n, cn, st, max_bin, cd, nc);
            check(cudaGetLastError(), "column_cuts_kernel");
            check(cudaMemcpy(hn.data(), nc, nf * 4ull, cudaMemcpyDeviceToHost), "cudaMemcpy");
            check(cudaMemcpy(hc.data(), cd, static_cast<size_t>(nf) * max_bin * 4,
                             cudaMemcpyDeviceToHost),
                  "cudaMemcpy");
            for (uint32_t c = 0; c < nf; ++c)
            {
                if (static_cast<uint64_t>(at) + hn[c] > cuts_cap)
                {
                    throw ConfigError("bb_fit_cuts: cuts_cap is too small (n_feats x max_bin "
                                      "always suffices)");
                }
                std::memcpy(cuts + at, hc.data() + (static_cast<size_t>(c) * max_bin),
                            hn[c] * sizeof(float));
                at += hn[c];
                cut_off[f0 + c + 1] = at;
            }
        }
        return BB_OK;
    }
    catch (ConfigError const &e)
    {
        set_last_error(e.what());
        return BB_ERR_CONFIG;
    }
    catch (std::invalid_argument const &e)
    {
        set_last_error(e.what());
        return BB_ERR_ARG;
    }
    catch (std::exception const &e)
    {
        set_last_error(e.what());
        return BB_ERR_CUDA;
    }
}
