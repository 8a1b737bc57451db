#include "ingest.cuh"

#include <algorithm>
#include <vector>

namespace bb
{
namespace
{

constexpr uint32_t k_tile_rows  = 256; // rows per CTA tile
constexpr uint32_t k_tile_feats = 32;  // features per CTA tile
constexpr uint32_t k_threads    = 256;

// lower_bound over cuts[0, nb): first index whose cut is not below x.
__device__ __forceinline__ uint32_t lower_bound_cut(float const *c, uint32_t nb, float x)
{
    uint32_t lo = 0;
    uint32_t n  = nb;
    while (n > 0)
    {
        uint32_t const half = n >> 1;
        if (c[lo + half] < x)
        {
            lo += half + 1;
            n -= half + 1;
        }
        else
        {
            n = half;
        }
    }
    return lo;
}

__device__ __forceinline__ uint32_t bin_of(float x, float const *c, uint32_t nb)
{
    return isnan(x) ? nb - 1 : lower_bound_cut(c, nb, x);
}

// grid: (ceil(rows / 256), ceil(F / 32)); block 256.
// Shared: the tile of X (256 x 32 floats) and the tile's features' cuts.
template <typename BinT>
__global__ void __launch_bounds__(k_threads)
    bin_apply_kernel(float const *__restrict__ X, uint64_t n_rows, uint32_t F,
                     uint64_t row0, float const *__restrict__ cuts,
                     uint32_t const *__restrict__ cut_off, BinT *__restrict__ bins,
                     uint64_t n_pad, uint32_t max_tile_cuts, bool vec4)
{
    extern __shared__ float smem[];
    float    *tile   = smem;                                // [k_tile_rows][33]
    float    *c_s    = smem + (k_tile_rows * (k_tile_feats + 1));
    uint32_t *coff_s = reinterpret_cast<uint32_t *>(c_s + max_tile_cuts);

    uint64_t const r0 = static_cast<uint64_t>(blockIdx.x) * k_tile_rows;
    uint32_t const f0 = blockIdx.y * k_tile_feats;
    uint32_t const nf = min(k_tile_feats, F - f0);
    uint32_t const nr = static_cast<uint32_t>(n_rows - r0 < k_tile_rows ? n_rows - r0 : k_tile_rows);

    // the tile's cuts
    if (threadIdx.x <= nf)
    {
        coff_s[threadIdx.x] = cut_off[f0 + threadIdx.x] - cut_off[f0];
    }
    uint32_t const c_begin = cut_off[f0];
    uint32_t const c_count = cut_off[f0 + nf] - c_begin;
    for (uint32_t i = threadIdx.x; i < c_count; i += k_threads)
    {
        c_s[i] = cuts[c_begin + i];
    }
    // the tile of X: rows r0.., features f0..f0+nf
    if (vec4)
    {
        uint32_t const q = nf / 4; // float4 per row
        for (uint32_t i = threadIdx.x; i < nr * q; i += k_threads)
        {
            uint32_t const rr = i / q;
            uint32_t const qq = i % q;
            float4 const   v  = *reinterpret_cast<float4 const *>(
                X + ((r0 + rr) * F) + f0 + (qq * 4));
            float *dst = tile + (rr * (k_tile_feats + 1)) + (qq * 4);
            dst[0]     = v.x;
            dst[1]     = v.y;
            dst[2]     = v.z;
            dst[3]     = v.w;
        }
    }
    else
    {
        for (uint32_t i = threadIdx.x; i < nr * nf; i += k_threads)
        {
            uint32_t const rr = i / nf;
            uint32_t const ff = i % nf;
            tile[(rr * (k_tile_feats + 1)) + ff] = X[((r0 + rr) * F) + f0 + ff];
        }
    }
    __syncthreads();

    // one 16-byte store per (feature, run of rows)
    constexpr uint32_t per = 16 / sizeof(BinT);
    uint32_t const     runs = k_tile_rows / per;
    for (uint32_t i = threadIdx.x; i < nf * runs; i += k_threads)
    {
        uint32_t const ff  = i / runs;
        uint32_t const run = i % runs;
        uint32_t const rb  = run * per;
        if (rb >= nr)
        {
            continue;
        }
        float const   *c  = c_s + coff_s[ff];
        uint32_t const nb = coff_s[ff + 1] - coff_s[ff];
        alignas(16) BinT out[per];
#pragma unroll
        for (uint32_t k = 0; k < per; ++k)
        {
            uint32_t const rr = rb + k;
            out[k]            = rr < nr ? static_cast<BinT>(bin_of(
                                   tile[(rr * (k_tile_feats + 1)) + ff], c, nb))
                                        : BinT{0};
        }
        BinT *dst = bins + (static_cast<uint64_t>(f0 + ff) * n_pad) + row0 + r0 + rb;
        *reinterpret_cast<uint4 *>(dst) = *reinterpret_cast<uint4 const *>(out);
    }
}

// One thread per (row, tile): gathers the tile's codes from the
// feature-major columns (coalesced across the warp's consecutive rows) and
// writes the row's 32-byte tile as two 16-byte stores.
template <typename BinT>
__global__ void __launch_bounds__(k_threads)
    mirror_kernel(BinT const *__restrict__ bins, uint64_t n_rows, uint64_t n_pad,
                  uint32_t F, uint4 *__restrict__ mirror)
{
    constexpr uint32_t per = k_mirror_bytes / sizeof(BinT);
    uint64_t const     r   = (static_cast<uint64_t>(blockIdx.x) * k_threads) + threadIdx.x;
    uint32_t const     t   = blockIdx.y;
    if (r >= n_rows)
    {
        return;
    }
    alignas(16) BinT v[per];
#pragma unroll
    for (uint32_t k = 0; k < per; ++k)
    {
        uint32_t const f = (t * per) + k;
        v[k]             = f < F ? bins[(static_cast<uint64_t>(f) * n_pad) + r] : BinT{0};
    }
    uint4 const   *src = reinterpret_cast<uint4 const *>(v);
    uint64_t const o   = ((static_cast<uint64_t>(t) * n_rows) + r) * 2;
    mirror[o]          = src[0];
    mirror[o + 1]      = src[1];
}

} // namespace

void build_mirror(Plane &p, cudaStream_t stream)
{
    uint32_t const per = k_mirror_bytes / (p.u8 ? 1 : 2);
    p.n_tiles          = (p.n_feats + per - 1) / per;
    size_t const bytes = static_cast<size_t>(p.n_tiles) * p.n_rows * k_mirror_bytes;
    BB_CHECK(cudaMalloc(&p.mirror, bytes));
    fill_mirror(p, stream);
}

void fill_mirror(Plane &p, cudaStream_t stream)
{
    dim3 const grid(ceil_div(p.n_rows, k_threads), p.n_tiles);
    if (p.u8)
    {
        mirror_kernel<uint8_t><<<grid, k_threads, 0, stream>>>(
            static_cast<uint8_t const *>(p.bins), p.n_rows, p.n_pad, p.n_feats,
            static_cast<uint4 *>(p.mirror));
    }
    else
    {
        mirror_kernel<uint16_t><<<grid, k_threads, 0, stream>>>(
            static_cast<uint16_t const *>(p.bins), p.n_rows, p.n_pad, p.n_feats,
            static_cast<uint4 *>(p.mirror));
    }
    BB_LAUNCH("mirror_kernel");
}

uint64_t stage_rows_for(uint32_t n_feats, uint64_t max_rows)
{
    // at most 64 MB; when a batch can take more than one chunk, every chunk
    // starts on a tile boundary (the kernel's 16-byte code stores need the
    // chunk's first row aligned)
    uint64_t const row_bytes = static_cast<uint64_t>(n_feats) * sizeof(float);
    uint64_t       rows      = std::min<uint64_t>(max_rows, (64ull << 20) / row_bytes);
    if (rows < max_rows)
    {
        rows = std::max<uint64_t>(k_tile_rows, rows - (rows % k_tile_rows));
    }
    return std::max<uint64_t>(rows, 1);
}

void ingest(Plane &p, float const *X, bool x_on_device, cudaStream_t stream, float *owned_stage,
            uint64_t owned_rows)
{
    uint32_t const F = p.n_feats;
    // the largest per-tile cut table
    uint32_t max_tile_cuts = 0;
    for (uint32_t f0 = 0; f0 < F; f0 += k_tile_feats)
    {
        uint32_t const f1 = std::min(F, f0 + k_tile_feats);
        max_tile_cuts     = std::max(max_tile_cuts, p.h_cut_off[f1] - p.h_cut_off[f0]);
    }
    size_t const smem = (k_tile_rows * (k_tile_feats + 1) * sizeof(float)) +
                        (max_tile_cuts * sizeof(float)) +
                        ((k_tile_feats + 1) * sizeof(uint32_t));
    if (smem > 227 * 1024)
    {
        throw ConfigError("ingest: a 32-feature tile's cuts exceed shared memory");
    }
    auto kern = p.u8 ? reinterpret_cast<void const *>(&bin_apply_kernel<uint8_t>)
                     : reinterpret_cast<void const *>(&bin_apply_kernel<uint16_t>);
    BB_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)));
    bool const vec4 = (F % 4) == 0 &&
                      (!x_on_device || (reinterpret_cast<uintptr_t>(X) % 16) == 0);

    auto launch = [&](float const *Xd, uint64_t rows, uint64_t row0)
    {
        dim3 const grid(ceil_div(rows, k_tile_rows), ceil_div(F, k_tile_feats));
        if (p.u8)
        {
            bin_apply_kernel<uint8_t><<<grid, k_threads, smem, stream>>>(
                Xd, rows, F, row0, p.cuts, p.cut_off, static_cast<uint8_t *>(p.bins),
                p.n_pad, max_tile_cuts, vec4);
        }
        else
        {
            bin_apply_kernel<uint16_t><<<grid, k_threads, smem, stream>>>(
                Xd, rows, F, row0, p.cuts, p.cut_off, static_cast<uint16_t *>(p.bins),
                p.n_pad, max_tile_cuts, vec4);
        }
        BB_LAUNCH("bin_apply_kernel");
    };

    if (x_on_device)
    {
        launch(X, p.n_rows, 0);
        return;
    }
    if (owned_stage != nullptr)
    {
        if (owned_rows < p.n_rows && owned_rows % k_tile_rows != 0)
        {
            throw std::logic_error("ingest: a staging buffer that chunks must hold whole tiles");
        }
        // a request plane: one staging buffer the plane owns, copy then bin
        // chunk by chunk on the one stream (no allocation)
        uint64_t const row_bytes = static_cast<uint64_t>(F) * sizeof(float);
        for (uint64_t r0 = 0; r0 < p.n_rows; r0 += owned_rows)
        {
            uint64_t const rows = std::min(owned_rows, p.n_rows - r0);
            BB_CHECK(cudaMemcpyAsync(owned_stage, X + (r0 * F), rows * row_bytes,
                                     cudaMemcpyHostToDevice, stream));
            launch(owned_stage, rows, r0);
        }
        return;
    }
    // Host input: stream it through two device staging buffers of <= 64 MB
    // (a multiple of the tile rows), copy of chunk k+1 overlapping the bin
    // kernel of chunk k.
    uint64_t const row_bytes  = static_cast<uint64_t>(F) * sizeof(float);
    uint64_t       chunk_rows = std::max<uint64_t>(k_tile_rows, (64ull << 20) / row_bytes);
    chunk_rows -= chunk_rows % k_tile_rows;
    chunk_rows = std::min<uint64_t>(chunk_rows, ((p.n_rows + k_tile_rows - 1) / k_tile_rows) *
                                                    k_tile_rows);
    float      *stage[2] = {nullptr, nullptr};
    cudaEvent_t done[2];
    cudaStream_t copy_s;
    BB_CHECK(cudaStreamCreateWithFlags(&copy_s, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i)
    {
        BB_CHECK(cudaMallocAsync(&stage[i], chunk_rows * row_bytes, stream));
        BB_CHECK(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming));
        BB_CHECK(cudaEventRecord(done[i], stream));
    }
    cudaEvent_t copied;
    BB_CHECK(cudaEventCreateWithFlags(&copied, cudaEventDisableTiming));
    int k = 0;
    for (uint64_t r0 = 0; r0 < p.n_rows; r0 += chunk_rows, k ^= 1)
    {
        uint64_t const rows = std::min(chunk_rows, p.n_rows - r0);
        BB_CHECK(cudaStreamWaitEvent(copy_s, done[k], 0));
        BB_CHECK(cudaMemcpyAsync(stage[k], X + (r0 * F), rows * row_bytes,
                                 cudaMemcpyHostToDevice, copy_s));
        BB_CHECK(cudaEventRecord(copied, copy_s));
        BB_CHECK(cudaStreamWaitEvent(stream, copied, 0));
        launch(stage[k], rows, r0);
        BB_CHECK(cudaEventRecord(done[k], stream));
    }
    for (int i = 0; i < 2; ++i)
    {
        BB_CHECK(cudaFreeAsync(stage[i], stream));
        BB_CHECK(cudaEventDestroy(done[i]));
    }
    BB_CHECK(cudaEventDestroy(copied));
    BB_CHECK(cudaStreamSynchronize(stream));
    BB_CHECK(cudaStreamDestroy(copy_s));
}

} // namespace bb
