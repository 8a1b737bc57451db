// Level kernels and the device-resident tree loop. See grow.cuh.
//
// Reference behaviour each kernel restates (paths within the project):
//   find_kernel + plan_kernel    HistogramNodeSplitFinder::find
//                                (src/split.cpp:101-162,271-297) and
//                                plan_level (src/grower_impl.hpp:212-255)
//   pcount/plan2/pscatter        host_partition (src/step/primitives.hpp:
//                                262-374), demote_empty_splits
//                                (src/grower_impl.hpp:262-298),
//                                commit_children (:303-326)
//   count/offsets/scatter/chain  the column fill's serial cell order
//                                (src/fill/columns.hpp:31-89)
//   subtract_totals_kernel       finish_split (src/step/primitives.hpp:
//                                156-173), Histogram::totals
//                                (include/bonsai/histogram.hpp:84-95),
//                                propagate_monotone_bounds
//                                (src/grower_impl.hpp:52-80)
//   stamp/final kernels          finalize_as_leaf / write_leaf
//                                (src/step/primitives.hpp:42-69)
#include "grow.cuh"

#include <algorithm>
#include <cmath>
#include <functional>
#include <limits>
#include <numeric>
#include <type_traits>

namespace bb
{
namespace
{

constexpr uint32_t k_threads    = 256;
constexpr uint32_t k_part_rows  = 4096; // rows per partition chunk
constexpr uint32_t k_build_rows = 4096; // rows per histogram-build chunk (exact)
constexpr uint32_t k_qbuild_rows = 2048;  // rows per histogram-build chunk (quantised)
constexpr uint32_t k_qctas = 148;        // persistent quantised-histogram CTAs per tile (one per SM)
constexpr uint32_t k_qthreads    = 512;   // threads per quantised-histogram CTA
constexpr uint32_t k_tthreads    = 1024;  // threads per conflict-free (u8) histogram CTA
constexpr uint32_t k_warps_feat = 8;    // features per count/scatter CTA
constexpr uint32_t k_find_thr   = 128;  // threads per (node, feature) find CTA
constexpr uint32_t k_chain_stg  = 32;   // elements per lane per cp.async stage
constexpr uint32_t k_chain_nst  = 4;    // cp.async stages per lane
constexpr uint32_t k_max_bins   = 4096; // per feature, this engine's ceiling
constexpr uint32_t k_plan_thr   = 512;  // plan kernels: one thread per node

// The walked tree's decision heap (depthwise trees, depth <= 8): slot h's
// children are 2h + 1 and 2h + 2; an entry is x = tile << 8 | position,
// y = split bin | (the missing bin if missing rows go left, else 0xFFFF)
// << 16. The plan kernels fill it as the tree grows (a node carries its
// slot): a split node's entry, and for a leaf above the last level the leaf
// map entry of its leftmost last-level descendant; every other slot keeps
// the always-left entry the tree starts from (split bin 0xFFFF takes every
// code, no tile).
constexpr uint32_t k_no_tile    = 0xFFFFFFu;
constexpr uint32_t k_heap_slots = 255;         // decision slots of a depth-8 heap
constexpr uint32_t k_heap_pass  = 0xFFFFFFFFu; // an always-left entry's y

struct HeapOut
{
    uint2    *heap;    // k_heap_slots entries, or null: no heap for this tree
    uint16_t *leafmap; // 2^depth last-level slots -> leaf node id
    uint32_t  depth;
    uint32_t  per;     // codes per 32-byte mirror tile
};

// y = split bin | (the missing bin when missing rows go left, else 0xFFFF,
// which no code equals) << 16: routes_left is then code <= split bin or code
// == y >> 16, since the split bin is below the missing bin
__device__ __forceinline__ uint2 heap_entry(uint32_t f, uint32_t per, uint32_t split,
                                            uint32_t last, bool dl)
{
    return make_uint2(((f / per) << 8) | (f % per), split | ((dl ? last : 0xFFFFu) << 16));
}

// Slot h holds a leaf: its leftmost last-level descendant names it.
__device__ __forceinline__ void heap_leaf(HeapOut const &ho, uint32_t h, uint32_t id)
{
    uint32_t const lvl = 31 - __clz(h + 1);
    if (ho.heap == nullptr || lvl > ho.depth)
    {
        return;
    }
    if (h < k_heap_slots)
    {
        ho.heap[h] = make_uint2(k_no_tile << 8, k_heap_pass);
    }
    ho.leafmap[((h + 1) << (ho.depth - lvl)) - (1u << ho.depth)] = static_cast<uint16_t>(id);
}

// L2 eviction hints (createpolicy): the mirror's tiles, which a pass reads
// once, are evict-first, so that the arrays every pass of a tree reads again
// (gradient codes, row lists, gradients) stay in L2.
__device__ __forceinline__ uint64_t l2_policy_first()
{
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ uint64_t l2_policy_last()
{
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// A read-only 16-byte load that skips L1 and carries an L2 policy.
__device__ __forceinline__ uint4 ld_nc_v4(uint4 const *src, uint64_t pol)
{
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(src), "l"(pol));
    return v;
}

// A 4-byte load with an L2 policy, through the coherent path.
__device__ __forceinline__ uint32_t ld_hint_b32(void const *src, uint64_t pol)
{
    uint32_t v;
    asm volatile("ld.global.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(src), "l"(pol));
    return v;
}

__device__ __forceinline__ uint32_t ld_nc_u16(uint16_t const *src, uint64_t pol)
{
    uint16_t v;
    asm volatile("ld.global.nc.L2::cache_hint.u16 %0, [%1], %2;" : "=h"(v) : "l"(src), "l"(pol));
    return v;
}

__device__ __forceinline__ uint32_t ld_nc_code(uint8_t const *src, uint64_t pol)
{
    uint16_t v;
    asm volatile("ld.global.nc.L2::cache_hint.u8 %0, [%1], %2;" : "=h"(v) : "l"(src), "l"(pol));
    return v;
}

__device__ __forceinline__ uint32_t ld_nc_code(uint16_t const *src, uint64_t pol)
{
    return ld_nc_u16(src, pol);
}

__device__ __forceinline__ uint32_t lanemask_lt()
{
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

template <typename BinT>
__device__ __forceinline__ uint32_t bin_at(void const *bins, uint64_t n_pad, uint32_t f,
                                           uint32_t r)
{
    return static_cast<BinT const *>(bins)[(static_cast<uint64_t>(f) * n_pad) + r];
}

// Block-wide exclusive scan of one value per thread (blockDim <= 1024).
template <uint32_t NT>
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *total)
{
    __shared__ uint32_t warp_sums[NT / 32];
    uint32_t const      lane = threadIdx.x & 31;
    uint32_t const      w    = threadIdx.x >> 5;
    uint32_t            x    = v;
#pragma unroll
    for (uint32_t o = 1; o < 32; o <<= 1)
    {
        uint32_t const y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o)
        {
            x += y;
        }
    }
    if (lane == 31)
    {
        warp_sums[w] = x;
    }
    __syncthreads();
    if (w == 0)
    {
        uint32_t s = lane < NT / 32 ? warp_sums[lane] : 0;
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1)
        {
            uint32_t const y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o)
            {
                s += y;
            }
        }
        if (lane < NT / 32)
        {
            warp_sums[lane] = s;
        }
    }
    __syncthreads();
    uint32_t const before = w > 0 ? warp_sums[w - 1] : 0;
    if (total != nullptr)
    {
        *total = warp_sums[NT / 32 - 1];
    }
    __syncthreads();
    return before + x - v;
}

__device__ __forceinline__ void write_leaf_node(TreeOut const &t, uint32_t id, float v)
{
    t.feature[id]      = k_leaf_flag;
    t.value[id]        = v;
    t.left[id]         = 0;
    t.right[id]        = 0;
    t.default_left[id] = 0;
    t.split_bin[id]    = 0;
}

__device__ __forceinline__ float leaf_value(Node const &nd, TreeParams const &tp)
{
    return static_cast<float>(bounded_leaf_weight(nd.sum_g, nd.sum_h, tp.lambda_l1,
                                                  tp.lambda_l2, nd.lo, nd.hi));
}

// ---------------------------------------------------------------- root ----

// n_root_dev (nullable): the root's row count lives on the device (a row
// sample drawn for this tree); an unsharded root's global count is then the
// same number.
__global__ void root_setup_kernel(Ctl *ctl, Node *nodes, uint32_t n_root, Chunk *bchunks,
                                  uint32_t *brange, uint32_t *build, TreeOut t,
                                  uint32_t crows, uint32_t g_root, uint32_t const *n_root_dev,
                                  uint2 *heap)
{
    pdl_enter();
    for (uint32_t i = threadIdx.x; heap != nullptr && i < k_heap_slots; i += blockDim.x)
    {
        heap[i] = make_uint2(k_no_tile << 8, k_heap_pass);
    }
    if (n_root_dev != nullptr)
    {
        n_root = *n_root_dev;
        g_root = n_root;
    }
    uint32_t const nch = (n_root + crows - 1) / crows;
    if (threadIdx.x == 0)
    {
        Ctl c{};
        c.n_cur      = 1;
        c.n_nodes    = 1;
        c.n_build    = 1;
        c.n_bchunks  = nch;
        c.built_rows = n_root;
        *ctl         = c;
        Node nd{};
        nd.start  = 0;
        nd.count  = n_root;
        nd.gcount = g_root;
        nd.id     = 0;
        nd.lo     = -INFINITY;
        nd.hi     = INFINITY;
        nodes[0]  = nd;
        build[0]  = 0;
        brange[0] = 0;
        brange[1] = nch;
        write_leaf_node(t, 0, 0.0F);
        t.gain[0]  = 0.0F;
        t.cover[0] = static_cast<float>(g_root);
    }
    for (uint32_t c = threadIdx.x; c < nch; c += blockDim.x)
    {
        uint32_t const b = c * crows;
        bchunks[c]       = {0, b, min(crows, n_root - b), 0};
    }
}

// Node totals from the first selected feature's cells: double sums over
// every cell in bin order, rounded to float once (Histogram::totals), with
// one warp: lanes load 32 cells at a time and every lane adds them in bin
// order from the shuffles, so each lane holds the serial FP64 sums (one
// dependent add per bin, no dependent global load).
__device__ __forceinline__ void warp_totals(float2 const *cells, uint32_t nb, float &g,
                                            float &h)
{
    uint32_t const lane = threadIdx.x & 31;
    double         sg   = 0.0;
    double         sh   = 0.0;
    for (uint32_t b0 = 0; b0 < nb; b0 += 32)
    {
        float2 const   c = b0 + lane < nb ? cells[b0 + lane] : make_float2(0.0F, 0.0F);
        uint32_t const m = min(32u, nb - b0);
        for (uint32_t i = 0; i < m; ++i)
        {
            sg += __shfl_sync(0xFFFFFFFFu, c.x, i);
            sh += __shfl_sync(0xFFFFFFFFu, c.y, i);
        }
    }
    g = static_cast<float>(sg);
    h = static_cast<float>(sh);
}

__global__ void root_totals_kernel(Node *nodes, float2 const *hist, uint32_t const *sel_nb)
{
    pdl_enter();
    float g, h;
    warp_totals(hist, sel_nb[0], g, h);
    if (threadIdx.x == 0)
    {
        nodes[0].sum_g = g;
        nodes[0].sum_h = h;
    }
}

// ------------------------------------------------------- histogram build ----
// The plain form's cells must equal the CPU fill's serial float chains, so
// each built node's rows are stably counting-sorted by bin per feature
// (count -> offsets -> scatter), after which every cell's (g, h) values sit
// contiguous in the node's row order and one lane folds each cell.

template <typename BinT>
__global__ void __launch_bounds__(k_threads)
    count_kernel(Ctl const *ctl, Chunk const *bchunks, uint32_t const *rows,
                 void const *bins, uint64_t n_pad, uint32_t const *sel,
                 uint32_t const *sel_nb, uint32_t nfb, uint32_t *ccount, uint32_t cs)
{
    pdl_enter();
    extern __shared__ uint32_t cnt_s[]; // [k_warps_feat][cs]
    uint32_t const             c = blockIdx.x;
    if (c >= ctl->n_bchunks)
    {
        return;
    }
    Chunk const    ch   = bchunks[c];
    uint32_t const lane = threadIdx.x & 31;
    uint32_t const w    = threadIdx.x >> 5;
    uint32_t const j    = (blockIdx.y * k_warps_feat) + w;
    if (j >= nfb)
    {
        return;
    }
    uint32_t const f   = sel[j];
    uint32_t const nb  = sel_nb[j];
    uint32_t      *cnt = cnt_s + (w * cs);
    for (uint32_t b = lane; b < nb; b += 32)
    {
        cnt[b] = 0;
    }
    __syncwarp();
    for (uint32_t k = lane; k < ch.count; k += 32)
    {
        uint32_t const r = rows[ch.begin + k];
        atomicAdd(&cnt[bin_at<BinT>(bins, n_pad, f, r)], 1U);
    }
    __syncwarp();
    uint32_t *out = ccount + ((static_cast<uint64_t>(c) * nfb + j) * cs);
    for (uint32_t b = lane; b < nb; b += 32)
    {
        out[b] = cnt[b];
    }
}

// Per (built node, feature): bin totals over the node's chunks, their
// exclusive scan (the bin segments of the node's sorted payload), and each
// chunk's per-bin write base, in place of its counts.
__global__ void __launch_bounds__(k_threads)
    offsets_kernel(Ctl const *ctl, uint32_t const *brange, uint32_t *ccount,
                   uint32_t *seg, uint32_t const *sel_nb, uint32_t nfb, uint32_t cs,
                   Chunk const *bchunks)
{
    pdl_enter();
    __shared__ uint32_t tot_s[k_max_bins];
    __shared__ uint32_t carry_s;
    uint32_t const      i = blockIdx.x;
    if (i >= ctl->n_build)
    {
        return;
    }
    uint32_t const j  = blockIdx.y;
    uint32_t const nb = sel_nb[j];
    uint32_t const c0 = brange[i];
    uint32_t const c1 = brange[i + 1];
    for (uint32_t b = threadIdx.x; b < nb; b += k_threads)
    {
        uint32_t s = 0;
        for (uint32_t c = c0; c < c1; ++c)
        {
            s += ccount[((static_cast<uint64_t>(c) * nfb + j) * cs) + b];
        }
        tot_s[b] = s;
    }
    if (threadIdx.x == 0)
    {
        carry_s = 0;
    }
    __syncthreads();
    // exclusive scan over bins, 256 at a time
    for (uint32_t b0 = 0; b0 < nb; b0 += k_threads)
    {
        uint32_t const b     = b0 + threadIdx.x;
        uint32_t const v     = b < nb ? tot_s[b] : 0;
        uint32_t       total = 0;
        uint32_t const ex    = block_excl_scan<k_threads>(v, &total);
        uint32_t const carry = carry_s;
        if (b < nb)
        {
            tot_s[b] = carry + ex;
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            carry_s = carry + total;
        }
        __syncthreads();
    }
    uint32_t *sg = seg + ((static_cast<uint64_t>(i) * nfb + j) * cs);
    for (uint32_t b = threadIdx.x; b < nb; b += k_threads)
    {
        uint32_t run = tot_s[b];
        sg[b]        = run;
        for (uint32_t c = c0; c < c1; ++c)
        {
            uint32_t *p = ccount + ((static_cast<uint64_t>(c) * nfb + j) * cs) + b;
            uint32_t  v = *p;
            *p          = run;
            run += v;
        }
    }
    if (threadIdx.x == 0)
    {
        sg[nb] = carry_s;
    }
    (void)bchunks;
}

template <typename BinT>
__global__ void __launch_bounds__(k_threads)
    scatter_kernel(Ctl const *ctl, Chunk const *bchunks, uint32_t const *rows,
                   void const *bins, uint64_t n_pad, float2 const *gh,
                   uint32_t const *sel, uint32_t const *sel_nb, uint32_t nfb,
                   uint32_t const *ccount, uint32_t cs, float2 *payload,
                   uint64_t p_stride)
{
    pdl_enter();
    extern __shared__ unsigned char smem_raw[];
    uint32_t const c = blockIdx.x;
    if (c >= ctl->n_bchunks)
    {
        return;
    }
    Chunk const ch     = bchunks[c];
    auto       *rows_s = reinterpret_cast<uint32_t *>(smem_raw);
    auto       *gh_s   = reinterpret_cast<float2 *>(rows_s + k_build_rows);
    auto       *base_s = reinterpret_cast<uint32_t *>(gh_s + k_build_rows);
    auto       *bins_s = reinterpret_cast<BinT *>(base_s + (k_warps_feat * cs));
    for (uint32_t k = threadIdx.x; k < ch.count; k += k_threads)
    {
        uint32_t const r = rows[ch.begin + k];
        rows_s[k]        = r;
        gh_s[k]          = gh[r];
    }
    __syncthreads();
    uint32_t const lane = threadIdx.x & 31;
    uint32_t const w    = threadIdx.x >> 5;
    uint32_t const j    = (blockIdx.y * k_warps_feat) + w;
    if (j >= nfb)
    {
        return;
    }
    uint32_t const  f    = sel[j];
    uint32_t const  nb   = sel_nb[j];
    uint32_t       *base = base_s + (w * cs);
    BinT           *bw   = bins_s + (w * k_build_rows);
    uint32_t const *off  = ccount + ((static_cast<uint64_t>(c) * nfb + j) * cs);
    for (uint32_t b = lane; b < nb; b += 32)
    {
        base[b] = off[b];
    }
    for (uint32_t k = lane; k < ch.count; k += 32)
    {
        bw[k] = static_cast<BinT>(bin_at<BinT>(bins, n_pad, f, rows_s[k]));
    }
    __syncwarp();
    float2 *out = payload + (static_cast<uint64_t>(j) * p_stride) + ch.aux;
    for (uint32_t k0 = 0; k0 < ch.count; k0 += 32)
    {
        uint32_t const k     = k0 + lane;
        bool const     valid = k < ch.count;
        uint32_t const b     = valid ? static_cast<uint32_t>(bw[k]) : 0xFFFFFFFFu;
        uint32_t const peers = __match_any_sync(0xFFFFFFFFu, b);
        uint32_t       pos   = 0;
        if (valid)
        {
            pos      = base[b] + __popc(peers & lanemask_lt());
            out[pos] = gh_s[k];
        }
        __syncwarp();
        if (valid && (peers & lanemask_lt()) == 0)
        {
            base[b] += __popc(peers);
        }
        __syncwarp();
    }
}

__device__ __forceinline__ void cp_async8(void *smem_dst, void const *gsrc)
{
    uint32_t const s = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gsrc));
}
__device__ __forceinline__ void cp_async_commit()
{
    asm volatile("cp.async.commit_group;\n" ::);
}
template <int N> __device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// One lane per cell: the serial float chain over the cell's contiguous
// (g, h) run, streamed through a per-lane cp.async ring in shared memory so
// that many bytes are in flight even when few cells exist (the root).
// grid (build nodes, features, ceil(max_bins / 32)), one warp per CTA.
__global__ void __launch_bounds__(32)
    chain_kernel(Ctl const *ctl, uint32_t const *build, Chunk const *bchunks,
                 uint32_t const *brange, uint32_t const *seg, float2 const *payload,
                 uint64_t p_stride, uint32_t const *sel_nb, uint32_t const *cell_off,
                 uint32_t nfb, uint32_t cs, float2 *hist, uint32_t total_cells)
{
    pdl_enter();
    extern __shared__ float2 ring_s[];
    uint32_t const i = blockIdx.x;
    if (i >= ctl->n_build)
    {
        return;
    }
    uint32_t const j    = blockIdx.y;
    uint32_t const nb   = sel_nb[j];
    uint32_t const lane = threadIdx.x;
    uint32_t const b    = (blockIdx.z * 32) + lane;
    if (blockIdx.z * 32 >= nb)
    {
        return;
    }
    uint32_t const  slot  = build[i];
    uint32_t const  nbase = bchunks[brange[i]].aux;
    uint32_t const *sg    = seg + ((static_cast<uint64_t>(i) * nfb + j) * cs);
    uint32_t        s0    = 0;
    uint32_t        s1    = 0;
    if (b < nb)
    {
        s0 = sg[b];
        s1 = sg[b + 1];
    }
    float2 const *src  = payload + (static_cast<uint64_t>(j) * p_stride) + nbase;
    float2       *ring = ring_s + (lane * k_chain_stg * k_chain_nst);
    uint32_t      next = s0;
    auto          issue = [&](uint32_t st)
    {
        float2 *dst = ring + (st * k_chain_stg);
#pragma unroll 8
        for (uint32_t e = 0; e < k_chain_stg; ++e)
        {
            if (next + e < s1)
            {
                cp_async8(dst + e, src + next + e);
            }
        }
        next = min(s1, next + k_chain_stg);
        cp_async_commit();
    };
#pragma unroll
    for (uint32_t st = 0; st < k_chain_nst - 1; ++st)
    {
        issue(st);
    }
    float    g  = 0.0F;
    float    h  = 0.0F;
    uint32_t st = 0;
    for (uint32_t s = s0; s < s1;)
    {
        issue((st + k_chain_nst - 1) % k_chain_nst);
        cp_async_wait<k_chain_nst - 1>();
        float2 const  *v = ring + (st * k_chain_stg);
        uint32_t const n = min(k_chain_stg, s1 - s);
        for (uint32_t e = 0; e < n; ++e)
        {
            float2 const x = v[e];
            g += x.x;
            h += x.y;
        }
        s += n;
        st = (st + 1) % k_chain_nst;
    }
    cp_async_wait<0>();
    if (b < nb)
    {
        hist[(static_cast<uint64_t>(slot) * total_cells) + cell_off[j] + b] =
            make_float2(g, h);
    }
}

// A quantised cell: with cw == 1 (int8 codes) one packed word -- the int32
// gradient sum in the high half (two's complement), the uint32 hessian sum in
// the low half; with cw == 2 (int16 codes, whose sums outgrow 32 bits) two
// words, the int64 gradient sum then the uint64 hessian sum. x counts cells.
__device__ __forceinline__ void qcell(unsigned long long const *h, uint64_t x, uint32_t cw,
                                      int64_t &g, int64_t &hs)
{
    if (cw == 2)
    {
        g  = static_cast<int64_t>(h[2 * x]);
        hs = static_cast<int64_t>(h[(2 * x) + 1]);
    }
    else
    {
        unsigned long long const c = h[x];
        g  = static_cast<int32_t>(static_cast<uint32_t>(c >> 32));
        hs = static_cast<uint32_t>(c);
    }
}

// ------------------------------------------------------------ split find ----

// The per-candidate core of update_best_for_feature_for_node
// (src/split.cpp:55-82,101-162) for one (bin, default_left).
template <typename M>
__device__ __forceinline__ bool candidate_gain(double lg, double lh, M mg, M mh,
                                               double real_g, double real_h, bool dl,
                                               double node_score, TreeParams const &tp,
                                               int mc, double lo, double hi,
                                               double &gain)
{
    double const rg = real_g - lg;
    double const rh = real_h - lh;
    double const gL = lg + (dl ? static_cast<double>(mg) : 0.0);
    double const hL = lh + (dl ? static_cast<double>(mh) : 0.0);
    double const gR = rg + (!dl ? static_cast<double>(mg) : 0.0);
    double const hR = rh + (!dl ? static_cast<double>(mh) : 0.0);
    double const mch = tp.min_child_hess;
    if (hL < mch || hR < mch)
    {
        return false;
    }
    double const l1       = tp.lambda_l1;
    double const l2       = tp.lambda_l2;
    double const children = split_score(gL, hL, l1, l2) + split_score(gR, hR, l1, l2);
    if (mc != 0)
    {
        double const wl = bounded_leaf_weight(gL, hL, l1, l2, lo, hi);
        double const wr = bounded_leaf_weight(gR, hR, l1, l2, lo, hi);
        if (static_cast<double>(mc) * (wr - wl) < 0.0)
        {
            return false;
        }
    }
    gain = children - node_score;
    return true;
}

// Warp reduce of (gain, order): the larger gain, the earlier scan order on a
// tie, so the winner is the serial scan's strict-> first maximum.
__device__ __forceinline__ void warp_best(double &gain, uint32_t &order)
{
#pragma unroll
    for (uint32_t o = 16; o > 0; o >>= 1)
    {
        double const   g2 = __shfl_xor_sync(0xFFFFFFFFu, gain, o);
        uint32_t const o2 = __shfl_xor_sync(0xFFFFFFFFu, order, o);
        if (g2 > gain || (g2 == gain && o2 < order))
        {
            gain  = g2;
            order = o2;
        }
    }
}

// grid (frontier, n_sel): one CTA of k_find_thr threads per (node,
// feature), each thread a few candidates. The exact form's prefix is one
// serial FP64 chain (the reference's summation order); the quantised form's
// is an exact integer block scan.
// Interaction constraints (allowed_features / propagate_interaction_state,
// src/grower_impl.hpp:114-160). fgroups[f]: the groups containing feature f
// as a bit mask (at most 64 groups). A node may split on f when its path is
// empty, when a group containing its whole path contains f, or when f is the
// path's only feature.
__device__ __forceinline__ bool interaction_allows(Node const &nd, uint64_t const *fgroups,
                                                   uint32_t f)
{
    uint32_t const plen = nd.ipath & 3u;
    return fgroups == nullptr || plen == 0 || (fgroups[f] & nd.icover) != 0 ||
           (plen == 1 && (nd.ipath >> 2) == f);
}

// Both children's path state after the parent splits on f.
__device__ __forceinline__ void interaction_children(Node const &par, uint64_t const *fgroups,
                                                     uint32_t f, Node &L, Node &R)
{
    if (fgroups == nullptr)
    {
        return;
    }
    uint32_t const plen = par.ipath & 3u;
    uint64_t       cover;
    uint32_t       path;
    if (plen == 0)
    {
        cover = fgroups[f];
        path  = 1u | (f << 2);
    }
    else
    {
        cover = par.icover & fgroups[f];
        path  = (plen == 1 && (par.ipath >> 2) == f) ? par.ipath : 2u;
    }
    L.icover = cover;
    R.icover = cover;
    L.ipath  = path;
    R.ipath  = path;
}

template <bool Q>
__global__ void __launch_bounds__(k_find_thr)
    find_kernel(Ctl const *ctl, Node const *nodes, void const *hist_v,
                uint32_t total_cells, uint32_t const *cell_off, uint32_t const *sel_nb,
                uint32_t const *sel, uint32_t n_sel, int8_t const *mono, uint32_t n_mono,
                TreeParams tp, Best *cand, uint32_t max_nb, double2 const *qscale,
                uint32_t const *slot_of, uint32_t cw, uint64_t const *fgroups)
{
    pdl_enter();
    extern __shared__ unsigned char smem_raw[];
    __shared__ double   bg_s[k_find_thr / 32];
    __shared__ uint32_t bo_s[k_find_thr / 32];
    __shared__ int64_t  wg_s[k_find_thr / 32];
    __shared__ int64_t  wh_s[k_find_thr / 32];
    uint32_t const      i = blockIdx.x;
    if (i >= ctl->n_cur)
    {
        return;
    }
    uint32_t const tid  = threadIdx.x;
    uint32_t const lane = tid & 31;
    uint32_t const w    = tid >> 5;
    uint32_t const j    = blockIdx.y;
    auto          *pref = reinterpret_cast<double2 *>(smem_raw);                  // [max_nb]
    auto          *raw  = reinterpret_cast<unsigned long long *>(pref + max_nb); // [max_nb]
    Node const     nd   = nodes[i];
    uint32_t const nb   = sel_nb[j];
    Best           out  = {0.0, j, 0, 1, 0};
    if (nd.gcount < 2 * tp.min_data_in_leaf || nb < 2 ||
        !interaction_allows(nd, fgroups, sel[j]))
    {
        if (tid == 0)
        {
            cand[(i * n_sel) + j] = out;
        }
        return;
    }
    uint32_t const n_cut = nb - 2;
    // the cells, 8 bytes each (packed integers or a float2); a node's slot
    // is its frontier index unless slot_of names it (the leafwise pool)
    uint32_t const slot = slot_of != nullptr ? slot_of[i] : i;
    auto const *src = static_cast<unsigned long long const *>(hist_v) +
                      (((static_cast<uint64_t>(slot) * total_cells) + cell_off[j]) * cw);
    for (uint32_t b = tid; b < nb * cw; b += k_find_thr)
    {
        raw[b] = src[b];
    }
    __syncthreads();
    using MissT = typename std::conditional<Q, double, float>::type;
    MissT        mg;
    MissT        mh;
    double       node_sc;
    double       real_g;
    double       real_h;
    bool         miss_empty;
    double const l1 = tp.lambda_l1;
    double const l2 = tp.lambda_l2;
    if constexpr (Q)
    {
        double2 const  sc  = *qscale;
        uint32_t const run = (n_cut + k_find_thr - 1) / k_find_thr;
        uint32_t const b0  = min(n_cut, tid * run);
        uint32_t const b1  = min(n_cut, b0 + run);
        int64_t        tg  = 0;
        int64_t        th  = 0;
        for (uint32_t b = b0; b < b1; ++b)
        {
            int64_t cg, ch;
            qcell(raw, b, cw, cg, ch);
            tg += cg;
            th += ch;
        }
        int64_t eg = tg;
        int64_t eh = th;
#pragma unroll
        for (uint32_t o = 1; o < 32; o <<= 1)
        {
            int64_t const ug = __shfl_up_sync(0xFFFFFFFFu, eg, o);
            int64_t const uh = __shfl_up_sync(0xFFFFFFFFu, eh, o);
            if (lane >= o)
            {
                eg += ug;
                eh += uh;
            }
        }
        if (lane == 31)
        {
            wg_s[w] = eg;
            wh_s[w] = eh;
        }
        __syncthreads();
        int64_t pg = eg - tg;
        int64_t ph = eh - th;
        for (uint32_t x = 0; x < w; ++x)
        {
            pg += wg_s[x];
            ph += wh_s[x];
        }
        for (uint32_t b = b0; b < b1; ++b)
        {
            int64_t cg, ch;
            qcell(raw, b, cw, cg, ch);
            pg += cg;
            ph += ch;
            pref[b] = make_double2(static_cast<double>(pg) * sc.x,
                                   static_cast<double>(ph) * sc.y);
        }
        int64_t mqg, mqh;
        qcell(raw, nb - 1, cw, mqg, mqh);
        mg         = static_cast<double>(mqg) * sc.x;
        mh         = static_cast<double>(mqh) * sc.y;
        node_sc    = split_score(static_cast<double>(nd.qg) * sc.x,
                                 static_cast<double>(nd.qh) * sc.y, l1, l2);
        real_g     = static_cast<double>(nd.qg - mqg) * sc.x;
        real_h     = static_cast<double>(nd.qh - mqh) * sc.y;
        miss_empty = mqg == 0 && mqh == 0;
    }
    else
    {
        auto const *cell = reinterpret_cast<float2 const *>(raw);
        if (tid == 0)
        {
            double lg = 0.0;
            double lh = 0.0;
            for (uint32_t b = 0; b < n_cut; ++b)
            {
                lg += cell[b].x;
                lh += cell[b].y;
                pref[b] = make_double2(lg, lh);
            }
        }
        mg      = cell[nb - 1].x;
        mh      = cell[nb - 1].y;
        node_sc = split_score(nd.sum_g, nd.sum_h, l1, l2);
        // float fields subtract in float, then widen (src/split.cpp:117-118)
        real_g     = static_cast<double>(nd.sum_g - mg);
        real_h     = static_cast<double>(nd.sum_h - mh);
        miss_empty = mg == 0.0F && mh == 0.0F;
    }
    __syncthreads();
    uint32_t const f        = sel[j];
    int const      mc       = (mono != nullptr && f < n_mono) ? mono[f] : 0;
    uint32_t const n_dir    = miss_empty ? 1 : 2;
    double         best     = 0.0;
    uint32_t       order    = 0xFFFFFFFFu;
    double const   min_gain = tp.min_gain_to_split;
    for (uint32_t b = tid; b < n_cut; b += k_find_thr)
    {
        double2 const p = pref[b];
        for (uint32_t d = 0; d < n_dir; ++d)
        {
            double gain = 0.0;
            if (candidate_gain<MissT>(p.x, p.y, mg, mh, real_g, real_h, d == 0, node_sc, tp,
                                      mc, nd.lo, nd.hi, gain) &&
                gain > best && gain >= min_gain)
            {
                best  = gain;
                order = (b * 2) + d;
            }
        }
    }
    warp_best(best, order);
    if (lane == 0)
    {
        bg_s[w] = best;
        bo_s[w] = order;
    }
    __syncthreads();
    if (tid == 0)
    {
        for (uint32_t x = 1; x < k_find_thr / 32; ++x)
        {
            if (bg_s[x] > best || (bg_s[x] == best && bo_s[x] < order))
            {
                best  = bg_s[x];
                order = bo_s[x];
            }
        }
        if (order != 0xFFFFFFFFu)
        {
            out.gain  = best;
            out.bin   = order >> 1;
            out.dl    = (order & 1) == 0 ? 1 : 0;
            out.valid = 1;
        }
        cand[(i * n_sel) + j] = out;
    }
}


// The quantised form's find with a warp per (node, feature): grid (frontier,
// ceil(n_sel / k_qfind_warps)), k_qfind_warps warps per CTA, no block
// barrier. The cut bins go by in 32-bin chunks (lane l holds bin c + l), a
// group of chunks loaded at once; the exact integer prefix (order-free) is
// each chunk's warp scan plus the carry, each bin's candidates are scored
// by its lane, and (largest gain, lowest bin x 2 + direction) over the warp
// is the choice of the per-(node, feature) CTA above, which one
// barrier-free warp replaces.
constexpr uint32_t k_qfind_warps = 8;
constexpr uint32_t k_qfind_group = 4; // 32-bin chunks in flight per lane

__global__ void __launch_bounds__(k_qfind_warps * 32)
    qfind_warp_kernel(Ctl const *ctl, Node const *nodes, void const *hist_v,
                      uint32_t total_cells, uint32_t const *cell_off, uint32_t const *sel_nb,
                      uint32_t const *sel, uint32_t n_sel, int8_t const *mono, uint32_t n_mono,
                      TreeParams tp, Best *cand, double2 const *qscale, uint32_t const *slot_of,
                      uint32_t cw, uint64_t const *fgroups)
{
    pdl_enter();
    uint32_t const i = blockIdx.x;
    if (i >= ctl->n_cur)
    {
        return;
    }
    uint32_t const lane = threadIdx.x & 31;
    uint32_t const j    = (blockIdx.y * k_qfind_warps) + (threadIdx.x >> 5);
    if (j >= n_sel)
    {
        return;
    }
    Node const     nd  = nodes[i];
    uint32_t const nb  = sel_nb[j];
    Best           out = {0.0, j, 0, 1, 0};
    if (nd.gcount < 2 * tp.min_data_in_leaf || nb < 2 ||
        !interaction_allows(nd, fgroups, sel[j]))
    {
        if (lane == 0)
        {
            cand[(i * n_sel) + j] = out;
        }
        return;
    }
    uint32_t const n_cut = nb - 2;
    uint32_t const slot  = slot_of != nullptr ? slot_of[i] : i;
    auto const    *src   = static_cast<unsigned long long const *>(hist_v) +
                      (((static_cast<uint64_t>(slot) * total_cells) + cell_off[j]) * cw);
    double2 const sc = *qscale;
    int64_t       mqg, mqh;
    qcell(src, nb - 1, cw, mqg, mqh);
    double const   l1       = tp.lambda_l1;
    double const   l2       = tp.lambda_l2;
    double const   mg       = static_cast<double>(mqg) * sc.x;
    double const   mh       = static_cast<double>(mqh) * sc.y;
    double const   node_sc  = split_score(static_cast<double>(nd.qg) * sc.x,
                                          static_cast<double>(nd.qh) * sc.y, l1, l2);
    double const   real_g   = static_cast<double>(nd.qg - mqg) * sc.x;
    double const   real_h   = static_cast<double>(nd.qh - mqh) * sc.y;
    uint32_t const n_dir    = (mqg == 0 && mqh == 0) ? 1 : 2;
    uint32_t const f        = sel[j];
    int const      mc       = (mono != nullptr && f < n_mono) ? mono[f] : 0;
    double const   min_gain = tp.min_gain_to_split;
    double         best     = 0.0;
    uint32_t       order    = 0xFFFFFFFFu;
    int64_t        carry_g  = 0;
    int64_t        carry_h  = 0;
    // 32-bin chunks, a group of them loaded (coalesced, all in flight)
    // before the group's scans; lane l holds bin c + l of chunk c
    for (uint32_t c0 = 0; c0 < n_cut; c0 += 32 * k_qfind_group)
    {
        int64_t vg[k_qfind_group];
        int64_t vh[k_qfind_group];
#pragma unroll
        for (uint32_t q = 0; q < k_qfind_group; ++q)
        {
            uint32_t const b = c0 + (q * 32) + lane;
            vg[q]            = 0;
            vh[q]            = 0;
            if (b < n_cut)
            {
                qcell(src, b, cw, vg[q], vh[q]);
            }
        }
#pragma unroll
        for (uint32_t q = 0; q < k_qfind_group; ++q)
        {
            int64_t sg = vg[q];
            int64_t sh = vh[q];
#pragma unroll
            for (uint32_t o = 1; o < 32; o <<= 1)
            {
                int64_t const ug = __shfl_up_sync(0xFFFFFFFFu, sg, o);
                int64_t const uh = __shfl_up_sync(0xFFFFFFFFu, sh, o);
                if (lane >= o)
                {
                    sg += ug;
                    sh += uh;
                }
            }
            uint32_t const b = c0 + (q * 32) + lane;
            if (b < n_cut)
            {
                double const lg = static_cast<double>(carry_g + sg) * sc.x;
                double const lh = static_cast<double>(carry_h + sh) * sc.y;
                for (uint32_t d = 0; d < n_dir; ++d)
                {
                    double gain = 0.0;
                    if (candidate_gain<double>(lg, lh, mg, mh, real_g, real_h, d == 0, node_sc,
                                               tp, mc, nd.lo, nd.hi, gain) &&
                        gain > best && gain >= min_gain)
                    {
                        best  = gain;
                        order = (b * 2) + d;
                    }
                }
            }
            carry_g += __shfl_sync(0xFFFFFFFFu, sg, 31);
            carry_h += __shfl_sync(0xFFFFFFFFu, sh, 31);
        }
    }
    warp_best(best, order);
    if (lane == 0)
    {
        if (order != 0xFFFFFFFFu)
        {
            out.gain  = best;
            out.bin   = order >> 1;
            out.dl    = (order & 1) == 0 ? 1 : 0;
            out.valid = 1;
        }
        cand[(i * n_sel) + j] = out;
    }
}


// ------------------------------------------------------- level split find ----
//
// update_best_for_feature_for_level (src/split.cpp:164-235): one split for
// the whole frontier. Per feature and candidate (bin, default_left), the sum
// over the frontier's nodes, in frontier order, of each node's children
// score when both children clear min_child_hess and of its own score
// otherwise (issue #60: an infeasible node no longer vetoes the cut), minus
// the sum of the nodes' scores. grid (n_sel), k_lfind_thr threads: warps
// take the nodes of a group in parallel (prefix over the cut bins: the
// exact form's serial FP64 chain, the quantised form's exact integer scan),
// then every thread adds the group's nodes for its bins in frontier order,
// so the FP64 sums follow the reference's order bit for bit.
constexpr uint32_t k_lfind_thr = 1024;

struct LevelNode
{
    double score; // the node's own split score
    double real_g;
    double real_h;
    double mg;    // its missing cell
    double mh;
};

template <typename M>
__device__ __forceinline__ double level_term(double lg, double lh, M mg, M mh, double real_g,
                                             double real_h, bool dl, double node_score,
                                             TreeParams const &tp)
{
    double const rg = real_g - lg;
    double const rh = real_h - lh;
    double const gL = lg + (dl ? static_cast<double>(mg) : 0.0);
    double const hL = lh + (dl ? static_cast<double>(mh) : 0.0);
    double const gR = rg + (!dl ? static_cast<double>(mg) : 0.0);
    double const hR = rh + (!dl ? static_cast<double>(mh) : 0.0);
    double const mch = tp.min_child_hess;
    if (hL < mch || hR < mch)
    {
        return node_score;
    }
    double const l1 = tp.lambda_l1;
    double const l2 = tp.lambda_l2;
    return split_score(gL, hL, l1, l2) + split_score(gR, hR, l1, l2);
}

template <bool Q>
__global__ void __launch_bounds__(k_lfind_thr)
    level_find_kernel(Ctl const *ctl, Node const *nodes, void const *hist_v,
                      uint32_t total_cells, uint32_t const *cell_off, uint32_t const *sel_nb,
                      uint32_t n_sel, TreeParams tp, Best *cand, uint32_t max_nb,
                      uint32_t group, double2 const *qscale, uint32_t cw)
{
    pdl_enter();
    extern __shared__ unsigned char smem_raw[];
    __shared__ LevelNode ln_s[k_lfind_thr / 32];
    __shared__ double    bg_s[k_lfind_thr / 32];
    __shared__ uint32_t  bo_s[k_lfind_thr / 32];
    constexpr uint32_t   k_bins_per_thr = k_max_bins / k_lfind_thr;
    uint32_t const       j     = blockIdx.x;
    uint32_t const       tid   = threadIdx.x;
    uint32_t const       lane  = tid & 31;
    uint32_t const       w     = tid >> 5;
    uint32_t const       n_cur = ctl->n_cur;
    uint32_t const       nb    = sel_nb[j];
    Best                 out   = {0.0, j, 0, 1, 0};
    if (nb < 3 || n_cur == 0)
    {
        if (tid == 0)
        {
            cand[j] = out;
        }
        return;
    }
    uint32_t const n_cut = nb - 2;
    auto          *pref  = reinterpret_cast<double2 *>(smem_raw); // [group][max_nb]
    double         acc[2 * k_bins_per_thr];
#pragma unroll
    for (uint32_t x = 0; x < 2 * k_bins_per_thr; ++x)
    {
        acc[x] = 0.0;
    }
    double         parent_sum = 0.0;
    double2 const  sc         = Q ? *qscale : make_double2(1.0, 1.0);
    for (uint32_t g0 = 0; g0 < n_cur; g0 += group)
    {
        // warp w prefixes node g0 + w of the group
        if (w < group && g0 + w < n_cur)
        {
            uint32_t const p   = g0 + w;
            Node const     nd  = nodes[p];
            double2       *pr  = pref + (static_cast<uint64_t>(w) * max_nb);
            auto const    *src = static_cast<unsigned long long const *>(hist_v) +
                              (((static_cast<uint64_t>(p) * total_cells) + cell_off[j]) * cw);
            if constexpr (Q)
            {
                uint32_t const run = (n_cut + 31) / 32;
                uint32_t const b0  = min(n_cut, lane * run);
                uint32_t const b1  = min(n_cut, b0 + run);
                int64_t        tg  = 0;
                int64_t        th  = 0;
                for (uint32_t b = b0; b < b1; ++b)
                {
                    int64_t cg, ch;
                    qcell(src, b, cw, cg, ch);
                    tg += cg;
                    th += ch;
                }
                int64_t eg = tg;
                int64_t eh = th;
#pragma unroll
                for (uint32_t o = 1; o < 32; o <<= 1)
                {
                    int64_t const ug = __shfl_up_sync(0xFFFFFFFFu, eg, o);
                    int64_t const uh = __shfl_up_sync(0xFFFFFFFFu, eh, o);
                    if (lane >= o)
                    {
                        eg += ug;
                        eh += uh;
                    }
                }
                int64_t pg = eg - tg;
                int64_t ph = eh - th;
                for (uint32_t b = b0; b < b1; ++b)
                {
                    int64_t cg, ch;
                    qcell(src, b, cw, cg, ch);
                    pg += cg;
                    ph += ch;
                    pr[b] = make_double2(static_cast<double>(pg) * sc.x,
                                         static_cast<double>(ph) * sc.y);
                }
                if (lane == 0)
                {
                    int64_t mqg, mqh;
                    qcell(src, nb - 1, cw, mqg, mqh);
                    LevelNode     l;
                    l.score  = split_score(static_cast<double>(nd.qg) * sc.x,
                                           static_cast<double>(nd.qh) * sc.y, tp.lambda_l1,
                                           tp.lambda_l2);
                    l.real_g = static_cast<double>(nd.qg - mqg) * sc.x;
                    l.real_h = static_cast<double>(nd.qh - mqh) * sc.y;
                    l.mg     = static_cast<double>(mqg) * sc.x;
                    l.mh     = static_cast<double>(mqh) * sc.y;
                    ln_s[w]  = l;
                }
            }
            else
            {
                auto const *cell = reinterpret_cast<float2 const *>(src);
                if (lane == 0)
                {
                    // Histogram::fill_prefix (include/bonsai/histogram.hpp:139-160):
                    // double running sums, each entry stored as a float cell
                    double lg = 0.0;
                    double lh = 0.0;
                    for (uint32_t b = 0; b < n_cut; ++b)
                    {
                        float2 const c = cell[b];
                        lg += c.x;
                        lh += c.y;
                        pr[b] = make_double2(static_cast<float>(lg), static_cast<float>(lh));
                    }
                    float2 const m = cell[nb - 1];
                    LevelNode    l;
                    l.score  = split_score(nd.sum_g, nd.sum_h, tp.lambda_l1, tp.lambda_l2);
                    // float fields subtract in float, then widen
                    l.real_g = static_cast<double>(nd.sum_g - m.x);
                    l.real_h = static_cast<double>(nd.sum_h - m.y);
                    l.mg     = m.x;
                    l.mh     = m.y;
                    ln_s[w]  = l;
                }
            }
        }
        __syncthreads();
        uint32_t const gn = min(group, n_cur - g0);
        // every (node, bin) pair's two terms, all threads at once (the FP64
        // divisions are independent), in place of the pair's prefix
        for (uint32_t x = tid; x < gn * n_cut; x += k_lfind_thr)
        {
            uint32_t const  q    = x / n_cut;
            uint32_t const  b    = x - (q * n_cut);
            LevelNode const l    = ln_s[q];
            double2        *cell = pref + ((static_cast<uint64_t>(q) * max_nb) + b);
            double2 const   p2   = *cell;
            double          t0;
            double          t1;
            if constexpr (Q)
            {
                t0 = level_term<double>(p2.x, p2.y, l.mg, l.mh, l.real_g, l.real_h, true,
                                        l.score, tp);
                t1 = level_term<double>(p2.x, p2.y, l.mg, l.mh, l.real_g, l.real_h, false,
                                        l.score, tp);
            }
            else
            {
                float const mg = static_cast<float>(l.mg);
                float const mh = static_cast<float>(l.mh);
                t0 = level_term<float>(p2.x, p2.y, mg, mh, l.real_g, l.real_h, true, l.score,
                                       tp);
                t1 = level_term<float>(p2.x, p2.y, mg, mh, l.real_g, l.real_h, false, l.score,
                                       tp);
            }
            *cell = make_double2(t0, t1);
        }
        __syncthreads();
        // then each bin adds the group's terms in frontier order
        for (uint32_t q = 0; q < gn; ++q)
        {
            double2 const *pr = pref + (static_cast<uint64_t>(q) * max_nb);
#pragma unroll
            for (uint32_t x = 0; x < k_bins_per_thr; ++x)
            {
                uint32_t const b = tid + (x * k_lfind_thr);
                if (b < n_cut)
                {
                    double2 const t2 = pr[b];
                    acc[2 * x] += t2.x;
                    acc[(2 * x) + 1] += t2.y;
                }
            }
            parent_sum += ln_s[q].score;
        }
        __syncthreads();
    }
    // every node's missing cell empty: both routings sum the same, and the
    // first (default left) wins the strict > below, as the serial scan does
    double         best     = 0.0;
    uint32_t       order    = 0xFFFFFFFFu;
    double const   min_gain = tp.min_gain_to_split;
#pragma unroll
    for (uint32_t x = 0; x < k_bins_per_thr; ++x)
    {
        uint32_t const b = tid + (x * k_lfind_thr);
        if (b < n_cut)
        {
            for (uint32_t d = 0; d < 2; ++d)
            {
                double const gain = acc[(2 * x) + d] - parent_sum;
                if (gain > best && gain >= min_gain)
                {
                    best  = gain;
                    order = (b * 2) + d;
                }
            }
        }
    }
    warp_best(best, order);
    if (lane == 0)
    {
        bg_s[w] = best;
        bo_s[w] = order;
    }
    __syncthreads();
    if (tid == 0)
    {
        for (uint32_t x = 1; x < k_lfind_thr / 32; ++x)
        {
            if (bg_s[x] > best || (bg_s[x] == best && bo_s[x] < order))
            {
                best  = bg_s[x];
                order = bo_s[x];
            }
        }
        if (order != 0xFFFFFFFFu)
        {
            out.gain  = best;
            out.bin   = order >> 1;
            out.dl    = (order & 1) == 0 ? 1 : 0;
            out.valid = 1;
        }
        cand[j] = out;
    }
}

// Cuts n row segments (n <= k_plan_thr) into chunks of `rows` rows with the
// whole block: segment i owns chunks [range[i], range[i + 1]), and
// seg(i, start, count, aux) describes it. One thread per segment stages its
// chunk origin and description in shared memory first (range and what seg
// reads are in global memory, written before a barrier), so a chunk's binary
// search and lookup read no global memory.
template <typename Seg>
__device__ __forceinline__ void fill_chunk_table(uint32_t n, uint32_t const *range,
                                                 uint32_t total, uint32_t rows, Seg seg,
                                                 Chunk *out)
{
    __shared__ uint32_t range_s[k_plan_thr];
    __shared__ uint32_t start_s[k_plan_thr];
    __shared__ uint32_t count_s[k_plan_thr];
    __shared__ uint32_t aux_s[k_plan_thr];
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
    {
        uint32_t st  = 0;
        uint32_t cnt = 0;
        uint32_t aux = 0;
        seg(i, st, cnt, aux);
        range_s[i] = range[i];
        start_s[i] = st;
        count_s[i] = cnt;
        aux_s[i]   = aux;
    }
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < total; c += blockDim.x)
    {
        uint32_t lo = 0;
        uint32_t hi = n;
        while (hi - lo > 1)
        {
            uint32_t const mid = (lo + hi) >> 1;
            if (range_s[mid] <= c)
            {
                lo = mid;
            }
            else
            {
                hi = mid;
            }
        }
        uint32_t const b = (c - range_s[lo]) * rows;
        out[c]           = {lo, start_s[lo] + b, min(rows, count_s[lo] - b), aux_s[lo]};
    }
}

// ------------------------------------------------------------- planning ----

__global__ void __launch_bounds__(k_plan_thr)
    plan_kernel(Ctl *ctl, Node *nodes, Best const *cand, Best *best, uint32_t n_sel,
                uint32_t const *sel, float const *cuts, uint32_t const *cut_off,
                TreeParams tp, TreeOut t, Chunk *pchunks, uint32_t *pcr, double2 *nbound,
                bool level, HeapOut ho, uint32_t *nleft, uint32_t *nright)
{
    pdl_enter();
    __shared__ Best    level_s;
    uint32_t const n_cur = ctl->n_cur;
    uint32_t const lane  = threadIdx.x & 31;
    uint32_t const w     = threadIdx.x >> 5;
    if (level)
    {
        // one split for the level (reduce_in_feature_order, src/split.cpp:239-250),
        // broadcast to every frontier node
        if (w == 0)
        {
            double   g = 0.0;
            uint32_t o = 0xFFFFFFFFu;
            for (uint32_t j = lane; j < n_sel; j += 32)
            {
                Best const c = cand[j];
                if (c.valid != 0 && (c.gain > g || (c.gain == g && j < o)))
                {
                    g = c.gain;
                    o = j;
                }
            }
            warp_best(g, o);
            if (lane == 0)
            {
                level_s = o == 0xFFFFFFFFu ? Best{0.0, 0, 0, 1, 0} : cand[o];
            }
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n_cur; i += k_plan_thr)
        {
            best[i] = level_s;
        }
    }
    // per node: the first feature (ascending) holding the largest gain
    for (uint32_t i = w; !level && i < n_cur; i += k_plan_thr / 32)
    {
        double   g = 0.0;
        uint32_t o = 0xFFFFFFFFu;
        for (uint32_t j = lane; j < n_sel; j += 32)
        {
            Best const c = cand[(i * n_sel) + j];
            if (c.valid != 0 && (c.gain > g || (c.gain == g && j < o)))
            {
                g = c.gain;
                o = j;
            }
        }
        warp_best(g, o);
        if (lane == 0)
        {
            best[i] = o == 0xFFFFFFFFu ? Best{0.0, 0, 0, 1, 0} : cand[(i * n_sel) + o];
        }
    }
    __syncthreads();
    uint32_t const i     = threadIdx.x;
    bool const     live  = i < n_cur;
    Best const     bs    = live ? best[i] : Best{};
    bool const     split = live && bs.valid != 0;
    uint32_t       n_split_total = 0;
    uint32_t const rank  = block_excl_scan<k_plan_thr>(split ? 1 : 0, &n_split_total);
    uint32_t const n_nodes0 = ctl->n_nodes;
    Node           nd       = live ? nodes[i] : Node{};
    if (live)
    {
        nleft[i]      = 0; // the one-pass partition's per-node counters
        nright[i]     = 0;
        nbound[nd.id] = make_double2(nd.lo, nd.hi); // for a later leaf renewal
        if (split)
        {
            uint32_t const f     = sel[bs.feature];
            uint32_t const left  = n_nodes0 + (2 * rank);
            uint32_t const right = left + 1;
            t.feature[nd.id]      = f;
            t.value[nd.id]        = cuts[cut_off[f] + bs.bin];
            t.left[nd.id]         = left;
            t.right[nd.id]        = right;
            t.default_left[nd.id] = static_cast<uint8_t>(bs.dl);
            t.gain[nd.id]         = static_cast<float>(bs.gain);
            t.split_bin[nd.id]    = bs.bin;
            write_leaf_node(t, left, 0.0F);
            write_leaf_node(t, right, 0.0F);
            t.gain[left]   = 0.0F;
            t.gain[right]  = 0.0F;
            t.cover[left]  = 0.0F;
            t.cover[right] = 0.0F;
            nd.flags       = 1;
            if (ho.heap != nullptr && nd.heap < k_heap_slots)
            {
                ho.heap[nd.heap] = heap_entry(f, ho.per, bs.bin,
                                              cut_off[f + 1] - cut_off[f] - 1, bs.dl != 0);
            }
        }
        else
        {
            heap_leaf(ho, nd.heap, nd.id);
            write_leaf_node(t, nd.id, leaf_value(nd, tp));
            nd.flags = 0;
        }
        nodes[i] = nd;
    }
    // partition chunk table over every frontier node
    uint32_t const nch    = live ? (nd.count + k_part_rows - 1) / k_part_rows : 0;
    uint32_t       total  = 0;
    uint32_t const c0     = block_excl_scan<k_plan_thr>(nch, &total);
    if (live)
    {
        pcr[i] = c0;
    }
    if (i == 0)
    {
        pcr[n_cur]      = total;
        ctl->n_pchunks  = total;
        ctl->n_psplit   = n_split_total;
        ctl->n_nodes    = n_nodes0 + (2 * n_split_total);
        ctl->n_leaves  += n_cur - n_split_total;
    }
    __syncthreads();
    fill_chunk_table(
        n_cur, pcr, total, k_part_rows,
        [&](uint32_t x, uint32_t &st, uint32_t &cnt, uint32_t &aux)
        {
            Node const nx = nodes[x];
            st            = nx.start;
            cnt           = nx.count;
            aux           = 0;
        },
        pchunks);
}

// Partition pass 1: each warp routes a contiguous run of the chunk's rows
// (lanes = consecutive rows, coalesced), keeps the directions as a bitmask
// (one word per 32 rows) so pass 2 never re-reads the bins, and the block
// sums the left counts.
constexpr uint32_t k_warp_rows = k_part_rows / (k_threads / 32); // 512

template <typename BinT>
__global__ void __launch_bounds__(k_threads)
    pcount_kernel(Ctl const *ctl, Chunk const *pchunks, Node const *nodes,
                  Best const *best, uint32_t const *__restrict__ rows,
                  void const *__restrict__ bins, uint64_t n_pad, uint32_t const *sel,
                  uint32_t const *sel_nb, uint32_t *__restrict__ pleft,
                  uint32_t *__restrict__ dirs)
{
    pdl_enter();
    __shared__ uint32_t wsum[k_threads / 32];
    uint32_t const      c = blockIdx.x;
    if (c >= ctl->n_pchunks)
    {
        return;
    }
    Chunk const ch = pchunks[c];
    if ((nodes[ch.node].flags & 1) == 0)
    {
        if (threadIdx.x == 0)
        {
            pleft[c] = 0; // a leaf's chunk routes nothing
        }
        return;
    }
    Best const     bs   = best[ch.node];
    uint32_t const f    = sel[bs.feature];
    uint32_t const last = sel_nb[bs.feature] - 1;
    BinT const    *col  = static_cast<BinT const *>(bins) + (static_cast<uint64_t>(f) * n_pad);
    uint32_t const lane = threadIdx.x & 31;
    uint32_t const w    = threadIdx.x >> 5;
    uint32_t      *dw   = dirs + (static_cast<uint64_t>(c) * (k_part_rows / 32));
    uint32_t const k0   = (w * k_warp_rows) + lane;
    // every row id of the warp's run, then every code, then the ballots:
    // all loads in flight together
    constexpr uint32_t steps = k_warp_rows / 32;
    uint32_t           r[steps];
#pragma unroll
    for (uint32_t i = 0; i < steps; ++i)
    {
        uint32_t const k = k0 + (32 * i);
        r[i]             = k < ch.count ? rows[ch.begin + k] : k_leaf_flag;
    }
    // (plain loads: nodes splitting on the same feature share the column's
    // sectors, which an evict-first hint would give up early)
    uint32_t b[steps];
#pragma unroll
    for (uint32_t i = 0; i < steps; ++i)
    {
        b[i] = r[i] != k_leaf_flag ? static_cast<uint32_t>(col[r[i]]) : 0u;
    }
    uint32_t n = 0;
#pragma unroll
    for (uint32_t i = 0; i < steps; ++i)
    {
        bool const     lf = r[i] != k_leaf_flag && routes_left(b[i], last, bs.bin, bs.dl != 0);
        uint32_t const m  = __ballot_sync(0xFFFFFFFFu, lf);
        if (lane == i)
        {
            dw[(w * steps) + i] = m;
        }
        n += __popc(m);
    }
    if (lane == 0)
    {
        wsum[w] = n;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        uint32_t t = 0;
        for (uint32_t x = 0; x < k_threads / 32; ++x)
        {
            t += wsum[x];
        }
        pleft[c] = t;
    }
}

// A sharded level's per-node left counts before they are combined across
// shards: the sum of the node's chunks' counts from partition pass 1.
__global__ void __launch_bounds__(k_plan_thr)
    node_left_kernel(Ctl const *ctl, uint32_t const *pcr, uint32_t const *pleft,
                     uint64_t *gleft, uint32_t n_slots)
{
    pdl_enter();
    uint32_t const n_cur = ctl->n_cur;
    for (uint32_t i = threadIdx.x; i < n_slots; i += k_plan_thr)
    {
        uint64_t nl = 0;
        if (i < n_cur)
        {
            for (uint32_t c = pcr[i]; c < pcr[i + 1]; ++c)
            {
                nl += pleft[c];
            }
        }
        gleft[i] = nl;
    }
}

__global__ void __launch_bounds__(k_plan_thr)
    plan2_kernel(Ctl *ctl, Node *nodes, Node *next, Best const *best,
                 Chunk const *pchunks, uint32_t const *pcr, uint32_t *pleft,
                 uint32_t *prbase, uint32_t *nleft, uint32_t *dst, uint32_t *bpair,
                 uint32_t *build, uint32_t *brange, Chunk *bchunks, TreeParams tp,
                 TreeOut t, uint32_t crows, uint32_t *bbase, bool level,
                 uint64_t const *gleft, uint64_t const *fgroups, HeapOut ho, bool fused)
{
    pdl_enter();
    __shared__ uint32_t grand_s;
    __shared__ uint32_t flags_s[k_plan_thr]; // per node: flags, start, prefix origin
    __shared__ uint32_t start_s[k_plan_thr];
    __shared__ uint32_t p0_s[k_plan_thr];
    uint32_t const      n_cur = ctl->n_cur;
    uint32_t const      n_ch  = ctl->n_pchunks;
    // A. exclusive prefix of the chunks' left counts over the whole level
    //    (leaf chunks count zero), each thread a contiguous run of chunks
    //    (the one-pass partition placed its rows already: no chunk runs)
    uint32_t const per = fused ? 0 : (n_ch + k_plan_thr - 1) / k_plan_thr;
    uint32_t const c_a = min(n_ch, threadIdx.x * per);
    uint32_t const c_b = min(n_ch, c_a + per);
    uint32_t       sum = 0;
    for (uint32_t c = c_a; c < c_b; ++c)
    {
        sum += pleft[c];
    }
    uint32_t       grand = 0;
    uint32_t const base  = block_excl_scan<k_plan_thr>(sum, &grand);
    for (uint32_t c = c_a, run = base; c < c_b; ++c)
    {
        uint32_t const v = pleft[c];
        pleft[c]         = run;
        run += v;
    }
    if (threadIdx.x == 0)
    {
        grand_s = grand;
    }
    __syncthreads();
    // B. per split node: its left count, or demotion when a side is empty
    uint32_t const i    = threadIdx.x;
    bool const     live = i < n_cur;
    Node           nd   = live ? nodes[i] : Node{};
    bool           surv = false;
    uint32_t       nl   = 0;
    uint32_t       gnl  = 0; // rows routed left over every shard
    uint32_t       p0   = 0;
    if (live && (nd.flags & 1) != 0)
    {
        if (fused)
        {
            nl = nleft[i]; // the one-pass partition's left counter
        }
        else
        {
            uint32_t const c0 = pcr[i];
            uint32_t const c1 = pcr[i + 1];
            // a node without chunks (a level split of an empty node) past
            // the last chunk: its prefix origin is the grand total
            p0       = c0 < n_ch ? pleft[c0] : grand_s;
            nl       = (c1 < n_ch ? pleft[c1] : grand_s) - p0;
            nleft[i] = nl;
        }
        gnl               = gleft != nullptr ? static_cast<uint32_t>(gleft[i]) : nl;
        if (!level && (gnl == 0 || gnl == nd.gcount))
        {
            // demote_empty_splits: the parent is a leaf after all (a level
            // split applies to every node, empty children included)
            nd.flags |= 2;
            write_leaf_node(t, nd.id, leaf_value(nd, tp));
            t.gain[nd.id] = 0.0F;
            nodes[i]      = nd;
            heap_leaf(ho, nd.heap, nd.id);
        }
        else
        {
            surv = true;
        }
    }
    if (live)
    {
        flags_s[i] = nd.flags;
        start_s[i] = nd.start;
        p0_s[i]    = p0; // the node's prefix origin, consumed by C below
    }
    __syncthreads();
    // C. per chunk of a split node: its left and right write bases
    for (uint32_t c = threadIdx.x; !fused && c < n_ch; c += k_plan_thr)
    {
        Chunk const    ch = pchunks[c];
        uint32_t const fl = flags_s[ch.node];
        if ((fl & 1) != 0 && (fl & 2) == 0)
        {
            uint32_t const lb = pleft[c] - p0_s[ch.node];
            pleft[c]          = lb;
            prbase[c]         = (ch.begin - start_s[ch.node]) - lb;
        }
    }
    __syncthreads();
    // D. survivors: their children in the next frontier, and the chunk table
    //    of the smaller children whose histograms are built
    uint32_t       n_surv     = 0;
    uint32_t const k          = block_excl_scan<k_plan_thr>(surv ? 1 : 0, &n_surv);
    uint32_t       rows_total = 0;
    uint32_t const start = block_excl_scan<k_plan_thr>(surv ? nd.count : 0, &rows_total);
    uint32_t small_count = 0;
    if (surv)
    {
        // the children's rows: compacted by pscatter, or where the one-pass
        // partition left them (the parent's segment, lefts first)
        uint32_t const s0   = fused ? nd.start : start;
        dst[i]              = s0;
        uint32_t const nr   = nd.count - nl;
        uint32_t const gnr  = nd.gcount - gnl;
        uint32_t const lid  = t.left[nd.id];
        uint32_t const rid  = t.right[nd.id];
        Node           L{s0, nl, lid, 0, 0.0F, 0.0F, nd.lo, nd.hi, 0, 0, gnl, 0, 0};
        Node           R{s0 + nl, nr, rid, 0, 0.0F, 0.0F, nd.lo, nd.hi, 0, 0, gnr, 0, 0};
        L.heap              = (2 * nd.heap) + 1;
        R.heap              = (2 * nd.heap) + 2;
        interaction_children(nd, fgroups, t.feature[nd.id], L, R);
        next[2 * k]         = L;
        next[(2 * k) + 1]   = R;
        t.cover[lid]        = static_cast<float>(gnl);
        t.cover[rid]        = static_cast<float>(gnr);
        // the smaller child over the whole fit: every shard builds the same one
        bool const left_sm  = gnl <= gnr;
        bpair[(3 * k) + 0]  = i;
        bpair[(3 * k) + 1]  = (2 * k) + (left_sm ? 0 : 1);
        bpair[(3 * k) + 2]  = (2 * k) + (left_sm ? 1 : 0);
        build[k]            = (2 * k) + (left_sm ? 0 : 1);
        small_count         = left_sm ? nl : nr;
    }
    uint32_t const nch   = surv ? (small_count + crows - 1) / crows : 0;
    uint32_t       nch_t = 0;
    uint32_t const c0    = block_excl_scan<k_plan_thr>(nch, &nch_t);
    uint32_t       built = 0;
    uint32_t const pbase = block_excl_scan<k_plan_thr>(small_count, &built);
    if (surv)
    {
        brange[k] = c0;
        bbase[k]  = pbase; // the built node's payload base
    }
    uint32_t n_dem = 0;
    block_excl_scan<k_plan_thr>((live && (nd.flags & 2) != 0) ? 1 : 0, &n_dem);
    if (i == 0)
    {
        brange[n_surv]  = nch_t;
        ctl->n_leaves  += n_dem;
        ctl->n_next     = 2 * n_surv;
        ctl->n_splits   = n_surv;
        ctl->n_build    = n_surv;
        ctl->n_bchunks  = nch_t;
        ctl->built_rows = built;
        if (n_surv > 0)
        {
            ctl->depth += 1;
        }
    }
    __syncthreads();
    fill_chunk_table(
        n_surv, brange, nch_t, crows,
        [&](uint32_t x, uint32_t &st, uint32_t &cnt, uint32_t &aux)
        {
            Node const sm = next[build[x]];
            st            = sm.start;
            cnt           = sm.count;
            aux           = bbase[x];
        },
        bchunks);
}

// Rows of this level's leaves (never split, or demoted): their leaf id and
// the fused score update scores[r] += lr * value.
__global__ void __launch_bounds__(k_threads)
    stamp_kernel(Ctl const *ctl, Chunk const *pchunks, Node const *nodes,
                 uint32_t const *rows, TreeOut t, uint32_t *leaf_id, float *scores,
                 float lr)
{
    pdl_enter();
    uint32_t const c = blockIdx.x;
    if (c >= ctl->n_pchunks)
    {
        return;
    }
    Chunk const ch = pchunks[c];
    Node const  nd = nodes[ch.node];
    if ((nd.flags & 1) != 0 && (nd.flags & 2) == 0)
    {
        return;
    }
    float const v = t.value[nd.id];
    for (uint32_t k = threadIdx.x; k < ch.count; k += k_threads)
    {
        uint32_t const r = rows[ch.begin + k];
        if (leaf_id != nullptr)
        {
            leaf_id[r] = nd.id;
        }
        if (scores != nullptr)
        {
            scores[r] = scores[r] + (lr * v);
        }
    }
}

// The final walk, for trees grown over every row: each row (one thread,
// rows in order) walks the finished tree through its 32-byte mirror tiles
// with the partition's own rule (routes_left on the split bin, the last bin
// following default_left), so it reaches the leaf whose segment held it --
// and rows read in order are coalesced, where the partitioned rows are a
// gather. The walk takes a fixed number of steps through the tree's
// decision heap (a leaf above the last level repeats down its left spine, and
// the last level's slot names the leaf). One pass (exact form) updates
// scores[r] = scores[r] + lr * value -- the stamp's arithmetic -- and the
// leaf ids and, for a resident booster, writes the next round's gradient
// pairs and their maxima. The quantised form renews its leaves from
// full-precision gradients first: pass A walks and sums each leaf's
// (g, h) as exact fixed-point integers (u / max |g| and u / max h per unit,
// u = 2^38 up to 2^24 rows and halved per doubling above, so no sum passes
// 2^62; integer sums are order-free, hence deterministic), a one-CTA kernel
// turns them into FP64 Newton values, and
// pass B applies them from the leaf id pass A recorded.
constexpr uint32_t k_no_sel_tile = 0xFFFFFFFFu; // an unused tile slot of a selection
constexpr uint32_t k_walk_nodes = 512;     // a depth-8 tree has at most 511

struct WalkArgs
{
    float        *scores;
    uint32_t     *leaf_id;
    float         lr;
    int           objective;
    float const  *labels;
    float2       *gh;
    uint32_t     *absmax;
    float const  *weights;
};

__device__ __forceinline__ uint32_t pick_word(uint32_t const w[8], uint32_t i)
{
    uint32_t const a = (i & 1) != 0 ? w[1] : w[0];
    uint32_t const b = (i & 1) != 0 ? w[3] : w[2];
    uint32_t const c = (i & 1) != 0 ? w[5] : w[4];
    uint32_t const d = (i & 1) != 0 ? w[7] : w[6];
    uint32_t const e = (i & 2) != 0 ? b : a;
    uint32_t const f = (i & 2) != 0 ? d : c;
    return (i & 4) != 0 ? f : e;
}

template <bool U8>
__device__ __forceinline__ uint32_t tile_code(uint32_t const w[8], uint32_t pos)
{
    if constexpr (U8)
    {
        return __byte_perm(pick_word(w, pos >> 2), 0u, 0x4440u | (pos & 3u));
    }
    else
    {
        return __byte_perm(pick_word(w, pos >> 1), 0u, 0x4410u | ((pos & 1u) * 0x22u));
    }
}

// The walk steps through the tree's decision heap (filled by the plan
// kernels): slot h's children are 2h + 1 and 2h + 2, so a step reads one
// 8-byte entry and no child ids. A leaf above the last level repeats down
// its left spine, and the slot a row ends in after `depth` steps names its
// leaf through leafmap.

__device__ __forceinline__ uint32_t heap_step(uint2 const e, uint32_t code, uint32_t h)
{
    bool const left = code <= (e.y & 0xFFFFu) || code == (e.y >> 16);
    return (2 * h) + (left ? 1u : 2u);
}

// The heap's entries and leaf map, staged in shared memory by the block.
__device__ __forceinline__ void load_heap(uint2 *heap_s, uint16_t *leaf_s, uint2 const *heap,
                                          uint16_t const *leafmap, uint32_t depth)
{
    uint32_t const n_int = (1u << depth) - 1;
    for (uint32_t i = threadIdx.x; i < n_int; i += blockDim.x)
    {
        heap_s[i] = heap[i];
    }
    for (uint32_t i = threadIdx.x; i <= n_int; i += blockDim.x)
    {
        leaf_s[i] = leafmap[i];
    }
    __syncthreads();
}

// Row r's last-level slot (leaf_s names its leaf): its tile of the root's
// feature is passed in; with MULTI the walk fetches another tile when a
// slot's feature lives there.
template <bool U8, bool MULTI>
__device__ __forceinline__ uint32_t walk_heap(uint2 const *heap_s,
                                              uint4 const *__restrict__ mirror, uint64_t n_rows,
                                              uint64_t r, uint32_t depth, uint4 ta, uint4 tb,
                                              uint32_t held)
{
    uint32_t w[8] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w};
    uint32_t h    = 0;
#pragma unroll
    for (uint32_t d = 0; d < 8; ++d)
    {
        if (d < depth)
        {
            uint2 const e = heap_s[h];
            if constexpr (MULTI)
            {
                uint32_t const tile = e.x >> 8;
                if (tile != held && tile != k_no_tile)
                {
                    uint4 const *src = mirror + (((static_cast<uint64_t>(tile) * n_rows) + r) * 2);
                    uint4 const  xa  = src[0];
                    uint4 const  xb  = src[1];
                    w[0] = xa.x; w[1] = xa.y; w[2] = xa.z; w[3] = xa.w;
                    w[4] = xb.x; w[5] = xb.y; w[6] = xb.z; w[7] = xb.w;
                    held = tile;
                }
            }
            h = heap_step(e, tile_code<U8>(w, e.x & 0xFFu), h);
        }
    }
    return h - ((1u << depth) - 1); // the row's slot among the last level's 2^depth
}

// The tile that holds the root's feature (0 when the root is a leaf).
__device__ __forceinline__ uint32_t heap_root_tile(uint2 const *heap_s, uint32_t depth)
{
    uint32_t const t = depth > 0 ? heap_s[0].x >> 8 : k_no_tile;
    return t == k_no_tile ? 0u : t;
}

// Block maxima of |g| and h into the quantiser's two words.
__device__ __forceinline__ void block_absmax(float mg, float mh, uint32_t *absmax)
{
    __shared__ float mg_s[k_threads / 32];
    __shared__ float mh_s[k_threads / 32];
#pragma unroll
    for (uint32_t o = 16; o > 0; o >>= 1)
    {
        mg = fmaxf(mg, __shfl_xor_sync(0xFFFFFFFFu, mg, o));
        mh = fmaxf(mh, __shfl_xor_sync(0xFFFFFFFFu, mh, o));
    }
    if ((threadIdx.x & 31) == 0)
    {
        mg_s[threadIdx.x >> 5] = mg;
        mh_s[threadIdx.x >> 5] = mh;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        for (uint32_t w = 1; w < k_threads / 32; ++w)
        {
            mg = fmaxf(mg, mg_s[w]);
            mh = fmaxf(mh, mh_s[w]);
        }
        atomicMax(&absmax[0], __float_as_uint(mg));
        atomicMax(&absmax[1], __float_as_uint(mh));
    }
}

// A row's score update and, for a resident booster, its next gradient pair.
__device__ __forceinline__ void apply_leaf(WalkArgs const &a, uint64_t r, uint32_t leaf,
                                           float s_old, float y, float v, float &mg, float &mh)
{
    if (a.leaf_id != nullptr)
    {
        a.leaf_id[r] = leaf;
    }
    if (a.scores == nullptr)
    {
        return;
    }
    float const s = s_old + (a.lr * v);
    a.scores[r]   = s;
    if (a.gh != nullptr)
    {
        float2 const g = weighted(objective_gradient(a.objective, s, y), a.weights, r);
        a.gh[r]        = g;
        mg             = fmaxf(mg, fabsf(g.x));
        mh             = fmaxf(mh, fmaxf(g.y, 0.0F));
    }
}

// One pass: walk and apply (exact form), two rows per thread so their
// chains interleave.
template <bool U8, bool MULTI>
__global__ void __launch_bounds__(k_threads)
    walk_kernel(Ctl const *ctl, TreeOut t, uint4 const *__restrict__ mirror, uint64_t n_rows,
                uint2 const *heap, uint16_t const *leafmap, uint32_t depth, WalkArgs a)
{
    pdl_enter();
    __shared__ uint2    heap_s[k_heap_slots];
    __shared__ uint16_t leaf_s[k_heap_slots + 1];
    __shared__ float    val_s[k_walk_nodes];
    uint32_t const      n_nodes = min(ctl->n_nodes, k_walk_nodes);
    for (uint32_t i = threadIdx.x; i < n_nodes; i += k_threads)
    {
        val_s[i] = t.value[i];
    }
    load_heap(heap_s, leaf_s, heap, leafmap, depth);
    uint32_t const root_tile = heap_root_tile(heap_s, depth);
    uint4 const   *mt        = mirror + (static_cast<uint64_t>(root_tile) * n_rows * 2);
    float          mg        = 0.0F;
    float          mh        = 0.0F;
    uint64_t const stride    = static_cast<uint64_t>(gridDim.x) * k_threads;
    uint64_t const pol       = l2_policy_first();
    for (uint64_t r0 = (static_cast<uint64_t>(blockIdx.x) * k_threads) + threadIdx.x;
         r0 < n_rows; r0 += 2 * stride)
    {
        uint64_t const r1  = r0 + stride;
        bool const     two = r1 < n_rows;
        uint64_t const rb  = two ? r1 : r0;
        uint4 const    a0  = ld_nc_v4(mt + (r0 * 2), pol);
        uint4 const    b0  = ld_nc_v4(mt + (r0 * 2) + 1, pol);
        uint4 const    a1  = ld_nc_v4(mt + (rb * 2), pol);
        uint4 const    b1  = ld_nc_v4(mt + (rb * 2) + 1, pol);
        float const    s0  = a.scores != nullptr ? a.scores[r0] : 0.0F;
        float const    s1  = a.scores != nullptr ? a.scores[rb] : 0.0F;
        float const    y0  = a.gh != nullptr ? a.labels[r0] : 0.0F;
        float const    y1  = a.gh != nullptr ? a.labels[rb] : 0.0F;
        uint32_t const n0 =
            leaf_s[walk_heap<U8, MULTI>(heap_s, mirror, n_rows, r0, depth, a0, b0, root_tile)];
        uint32_t const n1 =
            leaf_s[walk_heap<U8, MULTI>(heap_s, mirror, n_rows, rb, depth, a1, b1, root_tile)];
        apply_leaf(a, r0, n0, s0, y0, val_s[n0], mg, mh);
        if (two)
        {
            apply_leaf(a, r1, n1, s1, y1, val_s[n1], mg, mh);
        }
    }
    if (a.absmax != nullptr)
    {
        block_absmax(mg, mh, a.absmax);
    }
}

__device__ __forceinline__ bool in_sample(uint32_t const *bits, uint64_t r)
{
    return bits == nullptr || ((bits[r >> 5] >> (r & 31)) & 1u) != 0;
}

// Pass A of the quantised form: each row's leaf (as 16 bits) and every
// leaf's exact fixed-point (g, h) sums -- shared-memory 64-bit integer adds,
// then one global add per touched leaf and CTA. The shared sums are kept in
// k_wsum_copies lane-interleaved copies per last-level slot, laid out
// [slot][g, h][copy], so a warp's 64-bit adds -- copy = lane & 15 -- touch
// 16 distinct 8-byte words per half warp whatever slots its rows reach: two
// conflict-free wavefronts per add instead of one pass per row sharing a
// leaf. (Dynamic shared memory: 2^depth x 2 x 16 x 8 B.)
constexpr uint32_t k_wsum_thr    = 512;
constexpr uint32_t k_wsum_copies = 16;

template <bool U8, bool MULTI>
__global__ void __launch_bounds__(k_wsum_thr)
    walk_sum_kernel(Ctl const *ctl, uint4 const *__restrict__ mirror, uint64_t n_rows,
                    uint2 const *heap, uint16_t const *leafmap, uint32_t depth,
                    float2 const *__restrict__ gh, uint32_t const *absmax,
                    uint16_t *__restrict__ leaf16, unsigned long long *acc,
                    uint32_t const *__restrict__ bits, double fix_unit)
{
    pdl_enter();
    extern __shared__ unsigned long long acc_s[];
    __shared__ uint2    heap_s[k_heap_slots];
    __shared__ uint16_t leaf_s[k_heap_slots + 1];
    uint32_t const      n_slot = 1u << depth;
    for (uint32_t i = threadIdx.x; i < n_slot * 2 * k_wsum_copies; i += k_wsum_thr)
    {
        acc_s[i] = 0ULL;
    }
    load_heap(heap_s, leaf_s, heap, leafmap, depth);
    uint32_t const root_tile = heap_root_tile(heap_s, depth);
    uint4 const   *mt        = mirror + (static_cast<uint64_t>(root_tile) * n_rows * 2);
    float const    mgx       = __uint_as_float(absmax[0]);
    float const    mhx       = __uint_as_float(absmax[1]);
    double const   fg        = mgx > 0.0F ? fix_unit / static_cast<double>(mgx) : 1.0;
    double const   fh        = mhx > 0.0F ? fix_unit / static_cast<double>(mhx) : 1.0;
    uint64_t const stride    = static_cast<uint64_t>(gridDim.x) * k_wsum_thr;
    uint64_t const pol       = l2_policy_first();
    uint32_t const cp        = threadIdx.x & (k_wsum_copies - 1);
    auto           add       = [&](uint32_t o, float2 g)
    {
        uint32_t const x = (o * 2 * k_wsum_copies) + cp;
        atomicAdd(&acc_s[x],
                  static_cast<unsigned long long>(llrint(static_cast<double>(g.x) * fg)));
        atomicAdd(&acc_s[x + k_wsum_copies],
                  static_cast<unsigned long long>(
                      llrint(static_cast<double>(fmaxf(g.y, 0.0F)) * fh)));
    };
    for (uint64_t r0 = (static_cast<uint64_t>(blockIdx.x) * k_wsum_thr) + threadIdx.x;
         r0 < n_rows; r0 += 2 * stride)
    {
        uint64_t const r1  = r0 + stride;
        bool const     two = r1 < n_rows;
        uint64_t const rb  = two ? r1 : r0;
        uint4 const    a0  = ld_nc_v4(mt + (r0 * 2), pol);
        uint4 const    b0  = ld_nc_v4(mt + (r0 * 2) + 1, pol);
        uint4 const    a1  = ld_nc_v4(mt + (rb * 2), pol);
        uint4 const    b1  = ld_nc_v4(mt + (rb * 2) + 1, pol);
        // a row outside this tree's sample takes its leaf but adds nothing
        float2 const   g0  = in_sample(bits, r0) ? gh[r0] : make_float2(0.0F, 0.0F);
        float2 const   g1  = in_sample(bits, rb) ? gh[rb] : make_float2(0.0F, 0.0F);
        uint32_t const o0 =
            walk_heap<U8, MULTI>(heap_s, mirror, n_rows, r0, depth, a0, b0, root_tile);
        uint32_t const o1 =
            walk_heap<U8, MULTI>(heap_s, mirror, n_rows, rb, depth, a1, b1, root_tile);
        leaf16[r0] = leaf_s[o0];
        add(o0, g0);
        if (two)
        {
            leaf16[r1] = leaf_s[o1];
            add(o1, g1);
        }
    }
    __syncthreads();
    // slot o's (g, h) over the copies, into its leaf's global sums (slots
    // that no row reaches hold zeros)
    for (uint32_t x = threadIdx.x; x < 2 * n_slot; x += k_wsum_thr)
    {
        unsigned long long v = 0ULL;
#pragma unroll
        for (uint32_t k = 0; k < k_wsum_copies; ++k)
        {
            v += acc_s[(x * k_wsum_copies) + k];
        }
        if (v != 0ULL)
        {
            atomicAdd(&acc[(2 * leaf_s[x >> 1]) + (x & 1)], v);
        }
    }
}

// The quantised form's leaf values from pass A's sums: FP64 Newton values
// under each leaf's monotone bounds.
__global__ void __launch_bounds__(k_threads)
    leaf_fix_kernel(Ctl const *ctl, TreeOut t, unsigned long long const *acc,
                    double2 const *nbound, uint32_t const *absmax, TreeParams tp,
                    double fix_unit)
{
    pdl_enter();
    float const  mgx = __uint_as_float(absmax[0]);
    float const  mhx = __uint_as_float(absmax[1]);
    double const fg  = mgx > 0.0F ? fix_unit / static_cast<double>(mgx) : 1.0;
    double const fh  = mhx > 0.0F ? fix_unit / static_cast<double>(mhx) : 1.0;
    uint32_t const n_nodes = min(ctl->n_nodes, k_walk_nodes);
    for (uint32_t i = threadIdx.x; i < n_nodes; i += k_threads)
    {
        if (t.feature[i] != k_leaf_flag)
        {
            continue;
        }
        double const g = static_cast<double>(static_cast<int64_t>(acc[2 * i])) / fg;
        double const h = static_cast<double>(static_cast<int64_t>(acc[(2 * i) + 1])) / fh;
        double2 const b = nbound[i];
        t.value[i] = static_cast<float>(
            bounded_leaf_weight(g, h, tp.lambda_l1, tp.lambda_l2, b.x, b.y));
    }
}

// Pass B of the quantised form: apply the renewed values by pass A's leaf ids.
__global__ void __launch_bounds__(k_threads)
    walk_apply_kernel(Ctl const *ctl, TreeOut t, uint64_t n_rows,
                      uint16_t const *__restrict__ leaf16, WalkArgs a)
{
    pdl_enter();
    __shared__ float val_s[k_walk_nodes];
    uint32_t const   n_nodes = min(ctl->n_nodes, k_walk_nodes);
    for (uint32_t i = threadIdx.x; i < n_nodes; i += k_threads)
    {
        val_s[i] = t.value[i];
    }
    __syncthreads();
    float          mg     = 0.0F;
    float          mh     = 0.0F;
    uint64_t const stride = static_cast<uint64_t>(gridDim.x) * k_threads;
    uint64_t const pol    = l2_policy_first(); // leaf ids, scores, labels: once a round
    for (uint64_t r = (static_cast<uint64_t>(blockIdx.x) * k_threads) + threadIdx.x; r < n_rows;
         r += stride)
    {
        uint32_t const n = ld_nc_u16(leaf16 + r, pol);
        float const    s = a.scores != nullptr ? __uint_as_float(ld_hint_b32(a.scores + r, pol))
                                               : 0.0F;
        float const    y = a.gh != nullptr ? __uint_as_float(ld_hint_b32(a.labels + r, pol))
                                           : 0.0F;
        apply_leaf(a, r, n, s, y, val_s[n], mg, mh);
    }
    if (a.absmax != nullptr)
    {
        block_absmax(mg, mh, a.absmax);
    }
}

// Partition pass 2, the stable scatter: lefts keep their order at
// dst + left base, rights at dst + n_left + right base. Each warp takes the
// same run of rows as pass 1, its base from the bitmask's popcounts (one
// block barrier), its in-warp ranks from the bitmask words.
__global__ void __launch_bounds__(k_threads)
    pscatter_kernel(Ctl const *ctl, Chunk const *pchunks, Node const *nodes,
                    Best const *best, uint32_t const *pleft, uint32_t const *prbase,
                    uint32_t const *nleft, uint32_t const *dst,
                    uint32_t const *__restrict__ rows, uint32_t *__restrict__ rows_out,
                    uint32_t const *__restrict__ dirs, unsigned long long *zhist,
                    uint32_t const *build, uint32_t total_cells, uint32_t n_zcells)
{
    pdl_enter();
    __shared__ uint32_t wsum[k_threads / 32];
    uint32_t const      c = blockIdx.x;
    // the quantised build that follows adds into zeroed cells: every CTA
    // clears a share of the built slots' first n_zcells cells
    uint64_t const nz = static_cast<uint64_t>(ctl->n_build) * n_zcells;
    for (uint64_t x = (static_cast<uint64_t>(c) * k_threads) + threadIdx.x; x < nz;
         x += static_cast<uint64_t>(gridDim.x) * k_threads)
    {
        uint64_t const i = x / n_zcells;
        zhist[(static_cast<uint64_t>(build[i]) * total_cells) + (x - (i * n_zcells))] = 0ULL;
    }
    if (c >= ctl->n_pchunks)
    {
        return;
    }
    Chunk const ch = pchunks[c];
    Node const  nd = nodes[ch.node];
    if ((nd.flags & 1) == 0 || (nd.flags & 2) != 0)
    {
        return;
    }
    constexpr uint32_t steps = k_warp_rows / 32;
    uint32_t const     lane  = threadIdx.x & 31;
    uint32_t const     w     = threadIdx.x >> 5;
    uint32_t const     w0    = w * k_warp_rows;
    // the warp's direction words (lane i holds step i's) and row ids
    uint32_t const mword = lane < steps ? dirs[(static_cast<uint64_t>(c) * (k_part_rows / 32)) +
                                               (w * steps) + lane]
                                        : 0u;
    uint32_t r[steps];
#pragma unroll
    for (uint32_t i = 0; i < steps; ++i)
    {
        uint32_t const k = w0 + (32 * i) + lane;
        r[i]             = k < ch.count ? rows[ch.begin + k] : 0u;
    }
    // this warp's left count
    uint32_t mine = __popc(mword);
#pragma unroll
    for (uint32_t o = 16; o > 0; o >>= 1)
    {
        mine += __shfl_xor_sync(0xFFFFFFFFu, mine, o);
    }
    if (lane == 0)
    {
        wsum[w] = mine;
    }
    __syncthreads();
    uint32_t lb = 0;
    for (uint32_t x = 0; x < w; ++x)
    {
        lb += wsum[x];
    }
    uint32_t const d0  = dst[ch.node];
    uint32_t       lo  = d0 + pleft[c] + lb;                                   // next left
    uint32_t       ro  = d0 + nleft[ch.node] + prbase[c] + (min(w0, ch.count) - lb); // next right
    uint32_t const ltm = (1u << lane) - 1u;
#pragma unroll
    for (uint32_t i = 0; i < steps; ++i)
    {
        uint32_t const base = w0 + (32 * i);
        if (base >= ch.count)
        {
            break;
        }
        uint32_t const m      = __shfl_sync(0xFFFFFFFFu, mword, i);
        uint32_t const nvalid = min(32u, ch.count - base);
        uint32_t const vm     = nvalid == 32 ? 0xFFFFFFFFu : ((1u << nvalid) - 1u);
        uint32_t const lm     = m & vm;
        if (lane < nvalid)
        {
            if ((m >> lane) & 1u)
            {
                rows_out[lo + __popc(lm & ltm)] = r[i];
            }
            else
            {
                rows_out[ro + __popc(~lm & vm & ltm)] = r[i];
            }
        }
        lo += __popc(lm);
        ro += nvalid - __popc(lm);
    }
}

constexpr uint32_t k_psteps = k_warp_rows / 32; // 32-row steps of a partition warp

// One warp's 512 rows of a one-pass partition chunk: their ids (the level's
// list and the split column's codes are read once here, evict-first: the
// gradient codes and the next lists are what the level reads again), their
// codes of the split feature, their directions (lane i keeps step i's bits).
template <bool FULL, typename BinT>
__device__ __forceinline__ void psplit_route(Chunk const &ch, uint32_t const *__restrict__ rows,
                                             BinT const *col, uint32_t last, Best const &bs,
                                             uint32_t w0, uint32_t lane, uint32_t (&r)[k_psteps],
                                             uint32_t &mword, uint32_t &n)
{
    uint64_t const pol = l2_policy_first();
#pragma unroll
    for (uint32_t i = 0; i < k_psteps; ++i)
    {
        uint32_t const k = w0 + (32 * i) + lane;
        r[i]             = FULL || k < ch.count ? ld_hint_b32(rows + ch.begin + k, pol)
                                                : k_leaf_flag;
    }
    uint32_t b[k_psteps];
#pragma unroll
    for (uint32_t i = 0; i < k_psteps; ++i)
    {
        b[i] = FULL || r[i] != k_leaf_flag ? ld_nc_code(col + r[i], pol) : 0u;
    }
#pragma unroll
    for (uint32_t i = 0; i < k_psteps; ++i)
    {
        bool const lf =
            (FULL || r[i] != k_leaf_flag) && routes_left(b[i], last, bs.bin, bs.dl != 0);
        uint32_t const m = __ballot_sync(0xFFFFFFFFu, lf);
        mword            = lane == i ? m : mword;
        n += __popc(m);
    }
}

// ... and their places: lefts from lo up, rights from top down (rank rk on).
template <bool FULL>
__device__ __forceinline__ void psplit_place(Chunk const &ch, uint32_t w0, uint32_t lane,
                                             uint32_t const (&r)[k_psteps], uint32_t mword,
                                             uint32_t lo, uint32_t rk, uint32_t top,
                                             uint32_t *__restrict__ rows_out)
{
    uint32_t const ltm = (1u << lane) - 1u;
#pragma unroll
    for (uint32_t i = 0; i < k_psteps; ++i)
    {
        uint32_t const base = w0 + (32 * i);
        if (!FULL && base >= ch.count)
        {
            break;
        }
        uint32_t const m      = __shfl_sync(0xFFFFFFFFu, mword, i);
        uint32_t const nvalid = FULL ? 32u : min(32u, ch.count - base);
        uint32_t const vm     = FULL || nvalid == 32 ? 0xFFFFFFFFu : ((1u << nvalid) - 1u);
        uint32_t const lm     = m & vm;
        if (FULL || lane < nvalid)
        {
            if ((m >> lane) & 1u)
            {
                rows_out[lo + __popc(lm & ltm)] = r[i];
            }
            else
            {
                rows_out[top - (rk + __popc(~lm & vm & ltm))] = r[i];
            }
        }
        lo += __popc(lm);
        rk += __popc(~lm & vm);
    }
}

// The partition in one pass, for trees the final walk stamps in the
// quantised form, whose every consumer of the row lists is order-free (the
// histogram build adds exact integers; the next partition routes row by
// row). Each chunk routes its rows as pcount_kernel does, then reserves its
// lefts' and rights' places in the node's own segment with one atomic add per
// side on per-node counters (zeroed by plan_kernel): lefts fill the segment
// from its start, rights from its end backwards, so pass 2, its re-read of the
// row ids and the chunk prefix sums in plan2_kernel fall away. Which chunk's
// rows come first inside a child depends on the order chunks finish; the
// histograms, splits and leaves do not. With SCATTER false (the last level,
// whose rows are never listed) only the left counts are taken. Also zeroes
// the next level's histogram slots [0, 2 x splits) for the build's adds.
template <typename BinT, bool SCATTER>
__global__ void __launch_bounds__(k_threads)
    psplit_kernel(Ctl const *ctl, Chunk const *pchunks, Node const *nodes, Best const *best,
                  uint32_t const *__restrict__ rows, uint32_t *__restrict__ rows_out,
                  void const *__restrict__ bins, uint64_t n_pad, uint32_t const *sel,
                  uint32_t const *sel_nb, uint32_t *nleft, uint32_t *nright,
                  unsigned long long *zhist, uint32_t total_cells, uint32_t n_zcells)
{
    pdl_enter();
    __shared__ uint32_t wsum[k_threads / 32];
    __shared__ uint32_t base_s[2];
    uint32_t const      c = blockIdx.x;
    if constexpr (SCATTER)
    {
        uint64_t const nz = 2ULL * ctl->n_psplit * n_zcells;
        for (uint64_t x = (static_cast<uint64_t>(c) * k_threads) + threadIdx.x; x < nz;
             x += static_cast<uint64_t>(gridDim.x) * k_threads)
        {
            uint64_t const i = x / n_zcells;
            zhist[(i * total_cells) + (x - (i * n_zcells))] = 0ULL;
        }
    }
    if (c >= ctl->n_pchunks)
    {
        return;
    }
    Chunk const ch = pchunks[c];
    Node const  nd = nodes[ch.node];
    if ((nd.flags & 1) == 0)
    {
        return; // a leaf's chunk routes nothing
    }
    Best const     bs   = best[ch.node];
    uint32_t const f    = sel[bs.feature];
    uint32_t const last = sel_nb[bs.feature] - 1;
    BinT const    *col  = static_cast<BinT const *>(bins) + (static_cast<uint64_t>(f) * n_pad);
    uint32_t const lane = threadIdx.x & 31;
    uint32_t const w    = threadIdx.x >> 5;
    uint32_t const w0   = w * k_warp_rows;
    // a warp whose 512 rows all lie in the chunk (the common case) skips the
    // per-row range checks
    bool const     full = w0 + k_warp_rows <= ch.count;
    uint32_t       r[k_psteps];
    uint32_t       mword = 0; // lane i: step i's direction bits
    uint32_t       n     = 0;
    if (full)
    {
        psplit_route<true>(ch, rows, col, last, bs, w0, lane, r, mword, n);
    }
    else
    {
        psplit_route<false>(ch, rows, col, last, bs, w0, lane, r, mword, n);
    }
    if (lane == 0)
    {
        wsum[w] = n;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        uint32_t lc = 0;
        for (uint32_t x = 0; x < k_threads / 32; ++x)
        {
            lc += wsum[x];
        }
        uint32_t const rc = ch.count - lc;
        base_s[0]         = lc != 0 ? atomicAdd(&nleft[ch.node], lc) : 0u;
        base_s[1]         = SCATTER && rc != 0 ? atomicAdd(&nright[ch.node], rc) : 0u;
    }
    if constexpr (!SCATTER)
    {
        return;
    }
    __syncthreads();
    uint32_t lb = 0;
    for (uint32_t x = 0; x < w; ++x)
    {
        lb += wsum[x];
    }
    uint32_t const lo  = nd.start + base_s[0] + lb;                       // next left
    uint32_t const rk  = base_s[1] + (min(w0, ch.count) - lb);            // next right's rank
    uint32_t const top = nd.start + nd.count - 1;                          // rights count down
    if (full)
    {
        psplit_place<true>(ch, w0, lane, r, mword, lo, rk, top, rows_out);
    }
    else
    {
        psplit_place<false>(ch, w0, lane, r, mword, lo, rk, top, rows_out);
    }
}

// Larger child = parent - smaller child, cell by cell in float
// (finish_split); then both children's totals and monotone bounds.
__global__ void __launch_bounds__(k_threads)
    subtract_totals_kernel(Ctl *ctl, uint32_t const *bpair, float2 const *hist_cur,
                           float2 *hist_nxt, uint32_t total_cells, uint32_t n_cells,
                           Node const *cur, Node *next, Best const *best,
                           uint32_t const *sel, uint32_t const *sel_nb,
                           int8_t const *mono, uint32_t n_mono, TreeParams tp)
{
    pdl_enter();
    uint32_t const k = blockIdx.x;
    if (k == 0 && threadIdx.x == 0)
    {
        ctl->n_cur = ctl->n_next; // the level's last kernel advances the frontier
    }
    if (k >= ctl->n_splits)
    {
        return;
    }
    uint32_t const p  = bpair[3 * k];
    uint32_t const s  = bpair[(3 * k) + 1];
    uint32_t const l  = bpair[(3 * k) + 2];
    float2 const  *hp = hist_cur + (static_cast<uint64_t>(p) * total_cells);
    float2 const  *hs = hist_nxt + (static_cast<uint64_t>(s) * total_cells);
    float2        *hl = hist_nxt + (static_cast<uint64_t>(l) * total_cells);
    for (uint32_t x = threadIdx.x; x < n_cells; x += k_threads)
    {
        float2 const a = hp[x];
        float2 const b = hs[x];
        hl[x]          = make_float2(a.x - b.x, a.y - b.y);
    }
    __syncthreads();
    // the children's totals: warp c sums child c's first feature
    __shared__ float tot_s[4];
    uint32_t const   wc = threadIdx.x >> 5;
    if (wc < 2)
    {
        float g, h;
        warp_totals(hist_nxt + (static_cast<uint64_t>((2 * k) + wc) * total_cells), sel_nb[0],
                    g, h);
        if ((threadIdx.x & 31) == 0)
        {
            tot_s[2 * wc]       = g;
            tot_s[(2 * wc) + 1] = h;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        Node L  = next[2 * k];
        Node R  = next[(2 * k) + 1];
        L.sum_g = tot_s[0];
        L.sum_h = tot_s[1];
        R.sum_g = tot_s[2];
        R.sum_h = tot_s[3];
        Node const     par = cur[p];
        uint32_t const f   = sel[best[p].feature];
        int const      mc  = (mono != nullptr && f < n_mono) ? mono[f] : 0;
        if (mc != 0)
        {
            double const l1  = tp.lambda_l1;
            double const l2  = tp.lambda_l2;
            double const wl  = bounded_leaf_weight(L.sum_g, L.sum_h, l1, l2, par.lo, par.hi);
            double const wr  = bounded_leaf_weight(R.sum_g, R.sum_h, l1, l2, par.lo, par.hi);
            double const mid = 0.5 * (wl + wr);
            if (mc > 0)
            {
                L.hi = fmin(L.hi, mid);
                R.lo = fmax(R.lo, mid);
            }
            else
            {
                L.lo = fmax(L.lo, mid);
                R.hi = fmin(R.hi, mid);
            }
        }
        next[2 * k]       = L;
        next[(2 * k) + 1] = R;
    }
}

// The surviving frontier after the last level: leaves (end_tree). Marks
// every node a leaf and lays out its partition-chunk table, so the stamp
// (and, quantised, the leaf renewal) run chunk by chunk as on any level.
__global__ void __launch_bounds__(k_plan_thr)
    final_kernel(Ctl *ctl, Node *nodes, TreeParams tp, TreeOut t, Chunk *pchunks,
                 uint32_t *pcr, double2 *nbound, HeapOut ho)
{
    pdl_enter();
    uint32_t const n    = ctl->n_cur;
    uint32_t const i    = threadIdx.x;
    bool const     live = i < n;
    Node           nd   = live ? nodes[i] : Node{};
    if (live)
    {
        nbound[nd.id] = make_double2(nd.lo, nd.hi);
        write_leaf_node(t, nd.id, leaf_value(nd, tp));
        nd.flags = 0;
        nodes[i] = nd;
        heap_leaf(ho, nd.heap, nd.id);
    }
    uint32_t const nch   = live ? (nd.count + k_part_rows - 1) / k_part_rows : 0;
    uint32_t       total = 0;
    uint32_t const c0    = block_excl_scan<k_plan_thr>(nch, &total);
    if (live)
    {
        pcr[i] = c0;
    }
    if (i == 0)
    {
        pcr[n]          = total;
        ctl->n_pchunks  = total;
        ctl->n_leaves  += n;
        t.meta[0]       = ctl->n_nodes;
        t.meta[1]       = ctl->depth;
        t.meta[2]       = ctl->n_leaves;
    }
    __syncthreads();
    fill_chunk_table(
        n, pcr, total, k_part_rows,
        [&](uint32_t x, uint32_t &st, uint32_t &cnt, uint32_t &aux)
        {
            Node const nx = nodes[x];
            st            = nx.start;
            cnt           = nx.count;
            aux           = 0;
        },
        pchunks);
}



// ------------------------------------------------------ quantised form ----
// Per tree: (g, h) scaled by FP64 scales max|g| / 127 and max h / 127 and
// stochastically rounded to int8 with a counter-based generator, so the
// histograms are exact integer sums (order-independent, deterministic). The
// split gain is evaluated in FP64 from the integer sums; leaf values are
// renewed in FP64 from the full-precision gradients of each leaf's rows
// (the scheme of Shi et al., "Quantized Training of Gradient Boosting
// Decision Trees", NeurIPS 2022).

// Philox4x32-10 (Salmon, Moraes, Dror and Shaw, "Parallel random numbers:
// as easy as 1, 2, 3", SC 2011): ten rounds of the Philox S-box with the
// published multipliers and Weyl key increments.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k)
{
    constexpr uint32_t m0 = 0xD2511F53u;
    constexpr uint32_t m1 = 0xCD9E8D57u;
    constexpr uint32_t w0 = 0x9E3779B9u;
    constexpr uint32_t w1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r)
    {
        uint32_t const hi0 = __umulhi(m0, c.x);
        uint32_t const lo0 = m0 * c.x;
        uint32_t const hi1 = __umulhi(m1, c.z);
        uint32_t const lo1 = m1 * c.z;
        c                  = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += w0;
        k.y += w1;
    }
    return c;
}

__global__ void __launch_bounds__(k_threads)
    absmax_kernel(float2 const *__restrict__ gh, uint32_t n, uint32_t *absmax)
{
    pdl_enter();
    __shared__ float sg[k_threads / 32];
    __shared__ float sh[k_threads / 32];
    float            mg = 0.0F;
    float            mh = 0.0F;
    for (uint32_t i = (blockIdx.x * k_threads) + threadIdx.x; i < n;
         i += gridDim.x * k_threads)
    {
        float2 const v = gh[i];
        mg             = fmaxf(mg, fabsf(v.x));
        mh             = fmaxf(mh, fmaxf(v.y, 0.0F));
    }
#pragma unroll
    for (uint32_t o = 16; o > 0; o >>= 1)
    {
        mg = fmaxf(mg, __shfl_xor_sync(0xFFFFFFFFu, mg, o));
        mh = fmaxf(mh, __shfl_xor_sync(0xFFFFFFFFu, mh, o));
    }
    if ((threadIdx.x & 31) == 0)
    {
        sg[threadIdx.x >> 5] = mg;
        sh[threadIdx.x >> 5] = mh;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        for (uint32_t w = 1; w < k_threads / 32; ++w)
        {
            mg = fmaxf(mg, sg[w]);
            mh = fmaxf(mh, sh[w]);
        }
        // non-negative floats order as their bit patterns
        atomicMax(&absmax[0], __float_as_uint(mg));
        atomicMax(&absmax[1], __float_as_uint(mh));
    }
}

// W16: int16 codes (scales max / 32767, g in the low half of a 32-bit word,
// h in the high half) instead of int8 (max / 127, a 16-bit word).
template <bool W16>
__global__ void __launch_bounds__(k_threads)
    quantise_kernel(float2 const *__restrict__ gh, uint32_t n,
                    uint32_t const *__restrict__ absmax, uint2 key,
                    uint32_t const *__restrict__ tree_no, void *__restrict__ qout,
                    double2 *__restrict__ scale, uint64_t row_off)
{
    pdl_enter();
    constexpr double qmax = W16 ? 32767.0 : 127.0;
    constexpr int    imax = W16 ? 32767 : 127;
    double const mg = __uint_as_float(absmax[0]);
    double const mh = __uint_as_float(absmax[1]);
    double const sg = mg > 0.0 ? mg / qmax : 1.0;
    double const sh = mh > 0.0 ? mh / qmax : 1.0;
    double const ig = 1.0 / sg; // one division per thread, a multiply per row
    double const ih = 1.0 / sh;
    uint32_t const t = *tree_no;
    if (blockIdx.x == 0 && threadIdx.x == 0)
    {
        *scale = make_double2(sg, sh);
    }
    for (uint32_t i = (blockIdx.x * k_threads) + threadIdx.x; i < n;
         i += gridDim.x * k_threads)
    {
        float2 const v  = gh[i];
        // counter: the row's index in the whole fit, so shards round alike
        uint64_t const gi = row_off + i;
        uint4 const  r  = philox4x32_10(make_uint4(static_cast<uint32_t>(gi), t, 0x5157u,
                                                   static_cast<uint32_t>(gi >> 32)),
                                        key);
        double const ug = static_cast<double>(r.x >> 8) * (1.0 / 16777216.0);
        double const uh = static_cast<double>(r.y >> 8) * (1.0 / 16777216.0);
        double const xg = static_cast<double>(v.x) * ig;
        double const xh = static_cast<double>(fmaxf(v.y, 0.0F)) * ih;
        int          qg = isnan(xg) ? 0 : static_cast<int>(floor(xg + ug));
        int          qh = isnan(xh) ? 0 : static_cast<int>(floor(xh + uh));
        qg              = max(-imax, min(imax, qg));
        qh              = max(0, min(imax, qh));
        if constexpr (W16)
        {
            static_cast<uint32_t *>(qout)[i] =
                static_cast<uint32_t>(static_cast<uint16_t>(static_cast<int16_t>(qg))) |
                (static_cast<uint32_t>(qh) << 16);
        }
        else
        {
            static_cast<uint16_t *>(qout)[i] = static_cast<uint16_t>(
                static_cast<uint8_t>(static_cast<int8_t>(qg)) | (static_cast<uint32_t>(qh) << 8));
        }
    }
}

// Zeroes the cells of the nodes about to be built.
__global__ void __launch_bounds__(k_threads)
    zero_build_kernel(Ctl const *ctl, uint32_t const *build, unsigned long long *hist,
                      uint32_t total_cells, uint32_t n_cells)
{
    pdl_enter();
    uint32_t const i = blockIdx.x;
    if (i >= ctl->n_build)
    {
        return;
    }
    unsigned long long *h = hist + (static_cast<uint64_t>(build[i]) * total_cells);
    for (uint32_t x = threadIdx.x; x < n_cells; x += k_threads)
    {
        h[x] = 0ULL;
    }
}

// Exact integer histogram of a chunk of a built node's rows over one mirror
// tile: one gathered 32-byte sector per row, two native 32-bit
// shared-memory adds per (row, feature) -- the gradient word signed, the
// hessian word unsigned; a chunk's sums stay below 2^31 since a chunk holds
// at most 32,768 rows of |q| <= 127 -- then one packed 64-bit global add per
// touched cell (gradient in the high word, two's complement; hessian in the
// low word). grid (chunks, tiles), 256 threads.
// W16: int16 codes (a 32-bit word per row) into two-word cells (int64
// gradient, uint64 hessian sums); a 2,048-row chunk's sums of |q| <= 32767
// still fit the 32-bit shared words.
template <typename BinT, bool W16 = false, bool CW2 = W16>
__global__ void __launch_bounds__(k_qthreads, 3)
    qhist_kernel(Ctl const *ctl, Chunk const *bchunks, uint32_t const *build,
                 uint32_t const *rows, uint4 const *__restrict__ mirror, uint64_t n_rows,
                 void const *__restrict__ qgh, uint32_t const *tile_ids,
                 int32_t const *tile_j, uint32_t const *sel_nb, uint32_t const *cell_off,
                 uint32_t max_nb, unsigned long long *hist, uint32_t total_cells)
{
    pdl_enter();
    constexpr uint32_t per = k_mirror_bytes / sizeof(BinT);
    constexpr uint32_t U   = 2; // rows in flight per thread
    extern __shared__ int32_t hq_s[]; // [per][max_nb] gradient words, then hessian words
    __shared__ int32_t        j_s[per];
    uint32_t const            c = blockIdx.x;
    if (c >= ctl->n_bchunks)
    {
        return;
    }
    uint32_t const tile  = tile_ids[blockIdx.y];
    if (tile == k_no_sel_tile)
    {
        return; // a tile slot this selection leaves unused
    }
    uint32_t const cells = per * max_nb;
    int32_t       *hg_s  = hq_s;
    uint32_t      *hh_s  = reinterpret_cast<uint32_t *>(hq_s + cells);
    if (threadIdx.x < per)
    {
        j_s[threadIdx.x] = tile_j[(blockIdx.y * per) + threadIdx.x];
    }
    for (uint32_t x = threadIdx.x; x < 2 * cells; x += k_qthreads)
    {
        hq_s[x] = 0;
    }
    __syncthreads();
    Chunk const  ch = bchunks[c];
    uint4 const *mt = mirror + (static_cast<uint64_t>(tile) * n_rows * 2);
    for (uint32_t k0 = threadIdx.x; k0 < ch.count; k0 += k_qthreads * U)
    {
        uint32_t r[U];
        bool     ok[U];
#pragma unroll
        for (uint32_t u = 0; u < U; ++u)
        {
            uint32_t const k = k0 + (u * k_qthreads);
            ok[u]            = k < ch.count;
            r[u]             = ok[u] ? (rows != nullptr ? rows[ch.begin + k] : ch.begin + k) : 0;
        }
        uint4    va[U];
        uint4    vb[U];
        uint32_t q[U];
#pragma unroll
        for (uint32_t u = 0; u < U; ++u)
        {
            if (ok[u])
            {
                q[u]  = W16 ? static_cast<uint32_t const *>(qgh)[r[u]]
                            : static_cast<uint32_t>(static_cast<uint16_t const *>(qgh)[r[u]]);
                va[u] = mt[static_cast<uint64_t>(r[u]) * 2];
                vb[u] = mt[(static_cast<uint64_t>(r[u]) * 2) + 1];
            }
        }
#pragma unroll
        for (uint32_t u = 0; u < U; ++u)
        {
            if (!ok[u])
            {
                continue;
            }
            int32_t const  qg   = W16 ? static_cast<int16_t>(q[u] & 0xFFFFu)
                                      : static_cast<int8_t>(q[u] & 0xFFu);
            uint32_t const qh   = W16 ? q[u] >> 16 : q[u] >> 8;
            uint32_t const w[8] = {va[u].x, va[u].y, va[u].z, va[u].w,
                                   vb[u].x, vb[u].y, vb[u].z, vb[u].w};
#pragma unroll
            for (uint32_t i = 0; i < per; ++i)
            {
                if (j_s[i] >= 0)
                {
                    uint32_t const bin =
                        sizeof(BinT) == 1 ? (w[i >> 2] >> ((i & 3) * 8)) & 0xFFu
                                          : (w[i >> 1] >> ((i & 1) * 16)) & 0xFFFFu;
                    uint32_t const x = (i * max_nb) + bin;
                    atomicAdd(&hg_s[x], qg);
                    atomicAdd(&hh_s[x], qh);
                }
            }
        }
    }
    __syncthreads();
    constexpr uint32_t  cw  = CW2 ? 2 : 1;
    unsigned long long *dst = hist + (static_cast<uint64_t>(build[ch.node]) * total_cells * cw);
    for (uint32_t x = threadIdx.x; x < cells; x += k_qthreads)
    {
        uint32_t const i  = x / max_nb;
        uint32_t const bb = x % max_nb;
        int32_t const  jj = j_s[i];
        if (jj >= 0 && bb < sel_nb[jj] && (hg_s[x] != 0 || hh_s[x] != 0))
        {
            uint64_t const cell = cell_off[jj] + bb;
            if constexpr (CW2)
            {
                atomicAdd(&dst[2 * cell],
                          static_cast<unsigned long long>(static_cast<int64_t>(hg_s[x])));
                atomicAdd(&dst[(2 * cell) + 1], static_cast<unsigned long long>(hh_s[x]));
            }
            else
            {
                atomicAdd(&dst[cell],
                          (static_cast<unsigned long long>(static_cast<uint32_t>(hg_s[x])) << 32) +
                              static_cast<unsigned long long>(hh_s[x]));
            }
        }
    }
}


// The u8 form of the quantised histogram, bank-conflict free without any
// staging: lane = row. At (unrolled) step i every lane handles feature
// i ^ lane of its row, so the 32 lanes touch 32 different features at every
// step. The shared table is [bin][g: 32 features][h: 32 features], 256 bytes
// per bin, so cell (b, f) sits in bank f whatever the bins, and its address
// is (b << 8) | (f << 2): one byte permute puts the row's code of feature
// i ^ lane at bits 8..15, one three-input logic op ORs in ((4 i) ^ (4 lane)),
// and two 32-bit shared reductions (gradient word signed, hessian word
// unsigned, at +0 and +128) complete the (row, feature). The 32-byte tile is
// brought into that order once per row by a word permutation (j -> j ^ lane/4,
// three select stages); the byte within a word is chosen by the permute's
// per-lane selector. Slots of unselected features accumulate into columns
// that are never flushed.
//
// Persistent: a grid of up to k_qctas CTAs per tile (one per SM; fewer for a
// small dataset, so several fits share the GPU), each walking a
// contiguous range of the level's chunks (node-ordered), so no wave tail.
// The gathers are software-pipelined through registers: while a chunk's rows
// are added, the thread's loads of the next chunk's row ids, gradient codes
// and 32-byte tiles (two 16-byte non-coherent loads per row) are in flight,
// the loop unrolled by two so the prefetched registers are never moved (a
// move would wait for its load); with no shared staging the load/store path
// carries only the reductions. The shared
// histogram flushes -- one packed 64-bit global add per touched cell,
// gradient in the high word (two's complement), hessian in the low word --
// only when the node changes. The 32-bit shared words cannot overflow in
// between: a CTA adds at most k_tshare_chunks chunks of 2,048 rows (the
// launch raises its CTA count to keep every share within that), so a word
// sums at most 16,908,288 codes of magnitude at most 127, below 2^31.
// Global cells are packed 64-bit words while 127 x the fit's rows stays
// below 2^31, and two words (int64 gradient, uint64 hessian sums, CW2)
// beyond that.
//
// The loads carry L2 eviction hints: the tiles are read once per build
// (evict-first), the 2-byte gradient codes by every build of the tree
// (evict-last), so below the root the codes are L2 hits instead of one
// random DRAM sector per built row.
constexpr uint32_t k_ttable_bytes = 256 * 256; // 256 bins x (32 g + 32 h) x 4 B
constexpr uint32_t k_tshare_chunks = 0x7FFFFFFFu / (127u * 2048u);


__device__ __forceinline__ void red_shared_u32(uint32_t addr, uint32_t v)
{
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

__device__ __forceinline__ void red_shared_u32_hi(uint32_t addr, uint32_t v)
{
    asm volatile("red.shared.add.u32 [%0+128], %1;" ::"r"(addr), "r"(v) : "memory");
}

template <bool CW2>
__device__ __forceinline__ void qflush_t(uint32_t *tbl, uint32_t max_nb, int32_t const *j_s,
                                         uint32_t const *sel_nb, uint32_t const *cell_off,
                                         unsigned long long *dst)
{
    __syncthreads();
    for (uint32_t x = threadIdx.x; x < 256 * 32; x += k_tthreads)
    {
        uint32_t const f  = x & 31;
        uint32_t const bb = x >> 5;
        uint32_t const gi = (bb * 64) + f;
        uint32_t const g  = tbl[gi];
        uint32_t const h  = tbl[gi + 32];
        int32_t const  j2 = j_s[f];
        if (bb < max_nb && j2 >= 0 && bb < sel_nb[j2] && (g != 0 || h != 0))
        {
            uint64_t const cell = cell_off[j2] + bb;
            if constexpr (CW2)
            {
                // two-word cells: the int64 gradient sum, the uint64 hessian sum
                atomicAdd(&dst[2 * cell], static_cast<unsigned long long>(
                                              static_cast<int64_t>(static_cast<int32_t>(g))));
                atomicAdd(&dst[(2 * cell) + 1], static_cast<unsigned long long>(h));
            }
            else
            {
                atomicAdd(&dst[cell], (static_cast<unsigned long long>(g) << 32) +
                                          static_cast<unsigned long long>(h));
            }
        }
        tbl[gi]      = 0;
        tbl[gi + 32] = 0;
    }
    __syncthreads();
}

// One row's 32 (feature, bin) cells: va, vb are the row's 32-byte tile.
__device__ __forceinline__ void qrow_t(uint32_t base, uint32_t lane4, uint32_t wsel,
                                       uint32_t const sel[4], uint4 va, uint4 vb, uint32_t q)
{
    uint32_t const qg = static_cast<uint32_t>(static_cast<int32_t>(static_cast<int8_t>(q & 0xFFu)));
    uint32_t const qh = q >> 8;
    uint32_t       w[8] = {va.x, va.y, va.z, va.w, vb.x, vb.y, vb.z, vb.w};
#pragma unroll
    for (uint32_t st = 1; st < 8; st <<= 1)
    {
        bool const take = (wsel & st) != 0;
        uint32_t   t[8];
#pragma unroll
        for (uint32_t i = 0; i < 8; ++i)
        {
            t[i] = take ? w[i ^ st] : w[i];
        }
#pragma unroll
        for (uint32_t i = 0; i < 8; ++i)
        {
            w[i] = t[i];
        }
    }
#pragma unroll
    for (uint32_t i = 0; i < 32; ++i)
    {
        uint32_t const off  = __byte_perm(w[i >> 2], 0u, sel[i & 3]) | ((4u * i) ^ lane4);
        uint32_t const addr = base + off;
        red_shared_u32(addr, qg);
        red_shared_u32_hi(addr, qh);
    }
}

constexpr uint32_t k_tper   = k_qbuild_rows / k_tthreads; // rows per thread per chunk
constexpr uint32_t k_tsmem  = k_ttable_bytes;               // the table
constexpr uint32_t k_no_row = 0xFFFFFFFFu;
static_assert(k_tper == 2, "the prefetch holds two rows per thread");

template <bool CW2>
__global__ void __launch_bounds__(k_tthreads, 1)
    qhist_t_kernel(Ctl const *ctl, Chunk const *bchunks, uint32_t const *build,
                   uint32_t const *__restrict__ rows, uint4 const *__restrict__ mirror,
                   uint64_t n_rows, uint16_t const *__restrict__ qgh, uint32_t const *tile_ids,
                   int32_t const *tile_j, uint32_t const *sel_nb, uint32_t const *cell_off,
                   uint32_t max_nb, unsigned long long *hist, uint32_t total_cells)
{
    pdl_enter();
    extern __shared__ uint4 t_smem[];
    __shared__ int32_t      j_s[32];
    uint32_t const          total = ctl->n_bchunks;
    uint32_t const          c_a   = static_cast<uint32_t>((static_cast<uint64_t>(blockIdx.x) * total) / gridDim.x);
    uint32_t const          c_b   = static_cast<uint32_t>((static_cast<uint64_t>(blockIdx.x + 1) * total) / gridDim.x);
    if (c_a >= c_b)
    {
        return;
    }
    uint32_t const tile = tile_ids[blockIdx.y];
    if (tile == k_no_sel_tile)
    {
        return; // a tile slot this selection leaves unused
    }
    uint32_t const tid  = threadIdx.x;
    uint32_t const lane = tid & 31;
    auto          *tbl  = reinterpret_cast<uint32_t *>(t_smem);
    uint32_t const base = static_cast<uint32_t>(__cvta_generic_to_shared(tbl));
    if (tid < 32)
    {
        j_s[tid] = tile_j[(blockIdx.y * 32) + tid];
    }
    for (uint32_t x = tid; x < k_ttable_bytes / 4; x += k_tthreads)
    {
        tbl[x] = 0;
    }
    __syncthreads();
    uint32_t sel[4];
#pragma unroll
    for (uint32_t k = 0; k < 4; ++k)
    {
        sel[k] = 0x4404u | (((k ^ lane) & 3u) << 4);
    }
    uint32_t const lane4 = lane * 4;
    uint32_t const wsel  = lane >> 2;
    uint4 const   *mt    = mirror + (static_cast<uint64_t>(tile) * n_rows * 2);
    uint64_t const pol_t = l2_policy_first();
    uint64_t const pol_q = l2_policy_last();
    // one chunk's share of this thread: two rows, their codes and tiles
    struct Stage
    {
        uint32_t id[k_tper];
        uint32_t q[k_tper];
        uint4    a[k_tper];
        uint4    b[k_tper];
        uint32_t node;
    };
    auto load = [&](uint32_t c, Stage &S)
    {
        Chunk const ch = c < c_b ? bchunks[c] : Chunk{0, 0, 0, 0};
        S.node         = ch.node;
#pragma unroll
        for (uint32_t m = 0; m < k_tper; ++m)
        {
            uint32_t const k = (m * k_tthreads) + tid;
            S.id[m] = k < ch.count ? (rows != nullptr ? rows[ch.begin + k] : ch.begin + k)
                                   : k_no_row;
        }
#pragma unroll
        for (uint32_t m = 0; m < k_tper; ++m)
        {
            if (S.id[m] != k_no_row)
            {
                uint4 const *src = mt + (static_cast<uint64_t>(S.id[m]) * 2);
                S.q[m]           = ld_nc_u16(qgh + S.id[m], pol_q);
                S.a[m]           = ld_nc_v4(src, pol_t);
                S.b[m]           = ld_nc_v4(src + 1, pol_t);
            }
            else
            {
                S.q[m] = 0;
                S.a[m] = make_uint4(0, 0, 0, 0);
                S.b[m] = make_uint4(0, 0, 0, 0);
            }
        }
    };
    uint32_t node = bchunks[c_a].node;
    auto     run  = [&](Stage const &S)
    {
        if (S.node != node)
        {
            qflush_t<CW2>(tbl, max_nb, j_s, sel_nb, cell_off,
                          hist + (static_cast<uint64_t>(build[node]) * total_cells * (CW2 ? 2 : 1)));
            node = S.node;
        }
#pragma unroll
        for (uint32_t m = 0; m < k_tper; ++m)
        {
            if (S.id[m] != k_no_row)
            {
                qrow_t(base, lane4, wsel, sel, S.a[m], S.b[m], S.q[m]);
            }
        }
    };
    Stage s0;
    Stage s1;
    load(c_a, s0);
    for (uint32_t c = c_a; c < c_b; c += 2)
    {
        load(c + 1, s1);
        run(s0);
        if (c + 1 >= c_b)
        {
            break;
        }
        load(c + 2, s0);
        run(s1);
    }
    qflush_t<CW2>(tbl, max_nb, j_s, sel_nb, cell_off,
                  hist + (static_cast<uint64_t>(build[node]) * total_cells * (CW2 ? 2 : 1)));
}

// The quantised form's node totals: exact integer sums of the first selected
// feature's cells with one warp (order-free), every lane holding them.
__device__ __forceinline__ void warp_qtotals(unsigned long long const *cells, uint32_t nb,
                                             uint32_t cw, int64_t &g, int64_t &h)
{
    int64_t sg = 0;
    int64_t sh = 0;
    for (uint32_t b = threadIdx.x & 31; b < nb; b += 32)
    {
        int64_t cg, ch;
        qcell(cells, b, cw, cg, ch);
        sg += cg;
        sh += ch;
    }
#pragma unroll
    for (uint32_t o = 16; o > 0; o >>= 1)
    {
        sg += __shfl_xor_sync(0xFFFFFFFFu, sg, o);
        sh += __shfl_xor_sync(0xFFFFFFFFu, sh, o);
    }
    g = sg;
    h = sh;
}

__global__ void qroot_totals_kernel(Node *nodes, unsigned long long const *hist,
                                    uint32_t const *sel_nb, uint32_t cw)
{
    pdl_enter();
    int64_t g, h;
    warp_qtotals(hist, sel_nb[0], cw, g, h);
    if (threadIdx.x == 0)
    {
        nodes[0].qg = g;
        nodes[0].qh = h;
    }
}

constexpr uint32_t k_sub_cells = 1024; // cells per subtraction CTA

// Larger child = parent - smaller child in exact integers (both packed
// words subtract without borrow: a child's hessian sum never exceeds its
// parent's); children's totals and monotone bounds from the integer sums.
__global__ void __launch_bounds__(k_threads)
    qsubtract_totals_kernel(Ctl *ctl, uint32_t const *bpair,
                            unsigned long long const *hist_cur, unsigned long long *hist_nxt,
                            uint32_t total_cells, uint32_t n_cells, Node const *cur,
                            Node *next, Best const *best, uint32_t const *sel,
                            uint32_t const *sel_nb, int8_t const *mono, uint32_t n_mono,
                            TreeParams tp, double2 const *qscale, int64_t const *btot,
                            uint32_t cw)
{
    pdl_enter();
    uint32_t const k = blockIdx.x;
    if (k == 0 && blockIdx.y == 0 && threadIdx.x == 0)
    {
        ctl->n_cur = ctl->n_next; // the level's last kernel advances the frontier
    }
    if (k >= ctl->n_splits)
    {
        return;
    }
    uint32_t const p  = bpair[3 * k];
    uint32_t const s  = bpair[(3 * k) + 1];
    uint32_t const l  = bpair[(3 * k) + 2];
    // words: cw per cell (two for int16 codes); the subtraction is word-wise
    auto const    *hp = hist_cur + (static_cast<uint64_t>(p) * total_cells * cw);
    auto const    *hs = hist_nxt + (static_cast<uint64_t>(s) * total_cells * cw);
    auto          *hl = hist_nxt + (static_cast<uint64_t>(l) * total_cells * cw);
    // blockIdx.y takes words [y * k_sub_cells, (y + 1) * k_sub_cells)
    uint32_t const x0 = blockIdx.y * k_sub_cells;
    uint32_t const x1 = min(n_cells * cw, x0 + k_sub_cells);
#pragma unroll 4
    for (uint32_t x = x0 + threadIdx.x; x < x1; x += k_threads)
    {
        hl[x] = hp[x] - hs[x];
    }
    if (blockIdx.y != 0 || threadIdx.x >= 32)
    {
        return;
    }
    // the smaller child's exact totals: its first feature's cells (every row
    // lands in one of them), or the per-build sums when no cells were built;
    // the larger child's are the parent's minus them
    int64_t sg = 0;
    int64_t sh = 0;
    if (btot != nullptr)
    {
        if (threadIdx.x == 0)
        {
            sg = btot[2 * k];
            sh = btot[(2 * k) + 1];
        }
    }
    else
    {
        for (uint32_t b = threadIdx.x; b < sel_nb[0]; b += 32)
        {
            int64_t cg, ch;
            qcell(hs, b, cw, cg, ch);
            sg += cg;
            sh += ch;
        }
    }
#pragma unroll
    for (uint32_t o = 16; o > 0; o >>= 1)
    {
        sg += __shfl_xor_sync(0xFFFFFFFFu, sg, o);
        sh += __shfl_xor_sync(0xFFFFFFFFu, sh, o);
    }
    if (threadIdx.x == 0)
    {
        Node const par = cur[p];
        Node       S   = next[s];
        Node       G   = next[l];
        S.qg           = sg;
        S.qh           = sh;
        G.qg           = par.qg - sg;
        G.qh           = par.qh - sh;
        Node          &L  = s == 2 * k ? S : G;
        Node          &R  = s == 2 * k ? G : S;
        uint32_t const f  = sel[best[p].feature];
        int const      mc = (mono != nullptr && f < n_mono) ? mono[f] : 0;
        if (mc != 0)
        {
            double2 const sc  = *qscale;
            double const  l1  = tp.lambda_l1;
            double const  l2  = tp.lambda_l2;
            double const  wl  = bounded_leaf_weight(static_cast<double>(L.qg) * sc.x,
                                                    static_cast<double>(L.qh) * sc.y, l1, l2,
                                                    par.lo, par.hi);
            double const  wr  = bounded_leaf_weight(static_cast<double>(R.qg) * sc.x,
                                                    static_cast<double>(R.qh) * sc.y, l1, l2,
                                                    par.lo, par.hi);
            double const  mid = 0.5 * (wl + wr);
            if (mc > 0)
            {
                L.hi = fmin(L.hi, mid);
                R.lo = fmax(R.lo, mid);
            }
            else
            {
                L.lo = fmax(L.lo, mid);
                R.hi = fmin(R.hi, mid);
            }
        }
        next[2 * k]       = L;
        next[(2 * k) + 1] = R;
    }
}

// Exact integer totals of the smaller children when no histogram is built
// for them (the last level): per build chunk, the sums of its rows' codes,
// added into the chunk's build slot.
// The last level of a walked quantised tree: each built (smaller) child's
// exact integer totals straight from its parent's cells of the split
// feature -- the bins routes_left sends left (b <= split bin, and the missing
// bin when it defaults left), or the parent's totals minus them -- so the
// level needs neither the row scatter nor a gather of the children's codes.
// The parent's cells are the fit's (a sharded fit reduced them already).
// A warp per built child.
__global__ void qsplit_totals_kernel(Ctl const *ctl, uint32_t const *bpair, Node const *cur,
                                     Best const *best, unsigned long long const *hist_cur,
                                     uint32_t total_cells, uint32_t const *cell_off,
                                     uint32_t const *sel_nb, uint32_t cw, int64_t *btot)
{
    pdl_enter();
    uint32_t const k = (blockIdx.x * (blockDim.x / 32)) + (threadIdx.x >> 5);
    if (k >= ctl->n_splits)
    {
        return;
    }
    uint32_t const i       = bpair[3 * k];
    bool const     left_sm = (bpair[(3 * k) + 1] & 1u) == 0;
    Best const     b       = best[i];
    uint32_t const nb      = sel_nb[b.feature];
    uint32_t const last    = nb - 1;
    auto const    *cells   = hist_cur + (static_cast<uint64_t>(i) * total_cells * cw) +
                      (static_cast<uint64_t>(cell_off[b.feature]) * cw);
    int64_t lg = 0;
    int64_t lh = 0;
    for (uint32_t x = threadIdx.x & 31; x < nb; x += 32)
    {
        if (x == last ? b.dl != 0 : x <= b.bin)
        {
            int64_t cg, ch;
            qcell(cells, x, cw, cg, ch);
            lg += cg;
            lh += ch;
        }
    }
#pragma unroll
    for (uint32_t o = 16; o > 0; o >>= 1)
    {
        lg += __shfl_xor_sync(0xFFFFFFFFu, lg, o);
        lh += __shfl_xor_sync(0xFFFFFFFFu, lh, o);
    }
    if ((threadIdx.x & 31) == 0)
    {
        Node const nd  = cur[i];
        btot[2 * k]     = left_sm ? lg : nd.qg - lg;
        btot[(2 * k) + 1] = left_sm ? lh : nd.qh - lh;
    }
}

__global__ void __launch_bounds__(k_threads)
    qbuilt_totals_kernel(Ctl const *ctl, Chunk const *bchunks, uint32_t const *rows,
                         uint16_t const *__restrict__ qgh, uint32_t const *__restrict__ qgh16,
                         int64_t *btot)
{
    pdl_enter();
    uint32_t const c = blockIdx.x;
    if (c >= ctl->n_bchunks)
    {
        return;
    }
    Chunk const ch = bchunks[c];
    int64_t     g  = 0;
    int64_t     h  = 0;
    for (uint32_t k = threadIdx.x; k < ch.count; k += k_threads)
    {
        uint32_t const r = rows[ch.begin + k];
        if (qgh16 != nullptr)
        {
            uint32_t const q = qgh16[r];
            g += static_cast<int16_t>(q & 0xFFFFu);
            h += q >> 16;
        }
        else
        {
            uint32_t const q = qgh[r];
            g += static_cast<int8_t>(q & 0xFFu);
            h += q >> 8;
        }
    }
#pragma unroll
    for (uint32_t o = 16; o > 0; o >>= 1)
    {
        g += __shfl_xor_sync(0xFFFFFFFFu, g, o);
        h += __shfl_xor_sync(0xFFFFFFFFu, h, o);
    }
    if ((threadIdx.x & 31) == 0)
    {
        atomicAdd(reinterpret_cast<unsigned long long *>(&btot[2 * ch.node]),
                  static_cast<unsigned long long>(g));
        atomicAdd(reinterpret_cast<unsigned long long *>(&btot[(2 * ch.node) + 1]),
                  static_cast<unsigned long long>(h));
    }
}

// Leaf renewal: per partition chunk of a leaf node, the FP64 sums of the
// full-precision (g, h) of its rows in a fixed reduction order; the last CTA
// to finish (a ticket after a fence) then sums each leaf's chunks in chunk
// order and writes the FP64 Newton value under the node's bounds.
__global__ void __launch_bounds__(k_threads)
    leafsum_kernel(Ctl const *ctl, Chunk const *pchunks, Node const *nodes,
                   uint32_t const *__restrict__ rows, float2 const *__restrict__ gh,
                   double2 *partial, uint32_t const *pcr, TreeParams tp, TreeOut t,
                   uint32_t *done)
{
    pdl_enter();
    __shared__ double sg_s[k_threads / 32];
    __shared__ double sh_s[k_threads / 32];
    __shared__ bool   last_s;
    uint32_t const    c    = blockIdx.x;
    bool              work = c < ctl->n_pchunks;
    Chunk             ch{};
    if (work)
    {
        ch               = pchunks[c];
        Node const nd    = nodes[ch.node];
        work             = (nd.flags & 1) == 0 || (nd.flags & 2) != 0;
    }
    if (work)
    {
        double g = 0.0;
        double h = 0.0;
#pragma unroll 8
        for (uint32_t k = threadIdx.x; k < ch.count; k += k_threads)
        {
            float2 const v = gh[rows[ch.begin + k]];
            g += v.x;
            h += v.y;
        }
#pragma unroll
        for (uint32_t o = 16; o > 0; o >>= 1)
        {
            g += __shfl_xor_sync(0xFFFFFFFFu, g, o);
            h += __shfl_xor_sync(0xFFFFFFFFu, h, o);
        }
        if ((threadIdx.x & 31) == 0)
        {
            sg_s[threadIdx.x >> 5] = g;
            sh_s[threadIdx.x >> 5] = h;
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            double tg = 0.0;
            double th = 0.0;
            for (uint32_t w = 0; w < k_threads / 32; ++w)
            {
                tg += sg_s[w];
                th += sh_s[w];
            }
            partial[c] = make_double2(tg, th);
        }
    }
    if (threadIdx.x == 0)
    {
        __threadfence();
        last_s = atomicAdd(done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last_s)
    {
        return;
    }
    __threadfence();
    for (uint32_t i = threadIdx.x; i < ctl->n_cur; i += k_threads)
    {
        Node const nd = nodes[i];
        if ((nd.flags & 1) != 0 && (nd.flags & 2) == 0)
        {
            continue;
        }
        double g = 0.0;
        double h = 0.0;
        for (uint32_t x = pcr[i]; x < pcr[i + 1]; ++x)
        {
            double2 const v = __ldcg(&partial[x]);
            g += v.x;
            h += v.y;
        }
        t.value[nd.id] = static_cast<float>(
            bounded_leaf_weight(g, h, tp.lambda_l1, tp.lambda_l2, nd.lo, nd.hi));
    }
    if (threadIdx.x == 0)
    {
        *done = 0; // ready for the next launch
    }
}

// ----------------------------------------------------------------- leafwise ----
//
// One heap pop of the leafwise grower (LeafwiseGrower::grow,
// src/grower_impl.hpp:744-850; split_node, src/step/primitives.hpp:381-430) on
// the device data plane. The host keeps the gain heap and the tree (pop order,
// child ids, demotions, the leaf budget); the device partitions the popped
// node's segment of the row buffer with the two partition passes (stable),
// builds its smaller child's histograms into a free slot of a histogram pool,
// subtracts the larger child in place in the parent's slot (finish_split),
// and finds both children's best splits with the node finder.

struct LeafPop
{
    Node     node; // the popped node: its segment of the row buffer, totals, bounds
    Best     best; // its split
    uint32_t left_id;
    uint32_t right_id;
    uint32_t parent_slot;
    uint32_t small_slot;
};

// What the host reads back after a pop (or after the root).
struct LeafOut
{
    Node     child[2];
    Best     best[2];
    uint32_t split; // 0: the partition emptied a side (the split is demoted)
    uint32_t small_left;
    uint32_t pad[2];
};

// After partition pass 1: the chunks' left bases, the node's left count, and
// either the demotion (a side came out empty) or the two children, the
// smaller child's build chunks (in the scatter's output, which starts at 0)
// and the pool slots each child's histograms will sit in.
__global__ void __launch_bounds__(k_plan_thr)
    leaf_plan_kernel(Ctl *ctl, Chunk const *pchunks, uint32_t *pleft, uint32_t *prbase,
                     uint32_t *nleft, uint32_t *dst, uint32_t *build, uint32_t *brange,
                     uint32_t *bbase, Chunk *bchunks, uint32_t *bpair, Node *nodes, Node *next,
                     uint32_t *slot_of, LeafOut *out, uint32_t crows, LeafPop const *pp)
{
    pdl_enter();
    LeafPop const  p    = *pp;
    uint32_t const n_ch = ctl->n_pchunks;
    uint32_t const per  = (n_ch + k_plan_thr - 1) / k_plan_thr;
    uint32_t const c_a  = min(n_ch, threadIdx.x * per);
    uint32_t const c_b  = min(n_ch, c_a + per);
    uint32_t       sum  = 0;
    for (uint32_t c = c_a; c < c_b; ++c)
    {
        sum += pleft[c];
    }
    uint32_t       nl   = 0;
    uint32_t const base = block_excl_scan<k_plan_thr>(sum, &nl);
    for (uint32_t c = c_a, run = base; c < c_b; ++c)
    {
        uint32_t const v = pleft[c];
        pleft[c]         = run;
        prbase[c]        = (pchunks[c].begin - p.node.start) - run;
        run += v;
    }
    uint32_t const count = p.node.count;
    uint32_t const nr    = count - nl;
    bool const     split = nl != 0 && nl != count;
    bool const     sl    = nl <= nr; // the left child wins a size tie
    uint32_t const sc    = sl ? nl : nr;
    uint32_t const sb    = sl ? 0 : nl;
    uint32_t const nchb  = split ? (sc + crows - 1) / crows : 0;
    if (threadIdx.x == 0)
    {
        nleft[0]        = nl;
        dst[0]          = 0;
        out->split      = split ? 1 : 0;
        out->small_left = sl ? 1 : 0;
        ctl->n_build    = split ? 1 : 0;
        ctl->n_bchunks  = nchb;
        ctl->n_splits   = split ? 1 : 0;
        ctl->built_rows = split ? sc : 0;
        if (!split)
        {
            nodes[0].flags |= 2; // the scatter leaves a demoted node's rows alone
        }
        else
        {
            Node L    = p.node;
            L.count   = nl;
            L.gcount  = nl;
            L.id      = p.left_id;
            L.flags   = 0;
            Node R    = p.node;
            R.start   = p.node.start + nl;
            R.count   = nr;
            R.gcount  = nr;
            R.id      = p.right_id;
            R.flags   = 0;
            next[0]   = L;
            next[1]   = R;
            build[0]  = p.small_slot;
            brange[0] = 0;
            brange[1] = nchb;
            bbase[0]  = 0;
            slot_of[0] = sl ? p.small_slot : p.parent_slot;
            slot_of[1] = sl ? p.parent_slot : p.small_slot;
            bpair[0]   = p.parent_slot;
            bpair[1]   = p.small_slot;
            bpair[2]   = p.parent_slot;
        }
    }
    for (uint32_t c = threadIdx.x; c < nchb; c += k_plan_thr)
    {
        uint32_t const b = c * crows;
        bchunks[c]       = {0, sb + b, min(crows, sc - b), 0};
    }
}

// The partitioned segment back into the row buffer.
__global__ void leaf_copyback_kernel(LeafOut const *out, uint32_t const *__restrict__ tmp,
                                     uint32_t *__restrict__ rows, LeafPop const *pp)
{
    pdl_enter();
    if (out->split == 0)
    {
        return;
    }
    uint32_t const start = pp->node.start;
    uint32_t const count = pp->node.count;
    for (uint32_t k = (blockIdx.x * blockDim.x) + threadIdx.x; k < count;
         k += gridDim.x * blockDim.x)
    {
        rows[start + k] = tmp[k];
    }
}

// Larger child = parent - smaller, in place in the parent's slot (float
// cells in float, finish_split; packed integers without borrow).
template <bool Q>
__global__ void leaf_sub_kernel(LeafOut const *out, uint32_t const *bpair, void *pool,
                                uint32_t total_cells, uint32_t n_cells)
{
    pdl_enter();
    // quantised: total_cells and n_cells count words (cw per cell)
    if (out->split == 0)
    {
        return;
    }
    uint64_t const hp = static_cast<uint64_t>(bpair[0]) * total_cells;
    uint64_t const hs = static_cast<uint64_t>(bpair[1]) * total_cells;
    for (uint32_t x = (blockIdx.x * blockDim.x) + threadIdx.x; x < n_cells;
         x += gridDim.x * blockDim.x)
    {
        if constexpr (Q)
        {
            auto *h = static_cast<unsigned long long *>(pool);
            h[hp + x] -= h[hs + x];
        }
        else
        {
            auto        *h = static_cast<float2 *>(pool);
            float2 const a = h[hp + x];
            float2 const b = h[hs + x];
            h[hp + x]      = make_float2(a.x - b.x, a.y - b.y);
        }
    }
}

// The children's totals from their cells (Histogram::totals) and their
// monotone bounds (propagate_monotone_bounds, src/grower_impl.hpp:52-80).
template <bool Q>
__global__ void leaf_totals_kernel(Ctl *ctl, LeafOut const *out, Node *next,
                                   uint32_t const *slot_of, void const *pool,
                                   uint32_t total_cells, uint32_t const *sel,
                                   uint32_t const *sel_nb, int8_t const *mono, uint32_t n_mono,
                                   TreeParams tp, double2 const *qscale, LeafPop const *pp,
                                   uint32_t cw, uint64_t const *fgroups)
{
    pdl_enter();
    __shared__ int64_t qtot_s[4];
    __shared__ float   tot_s[4];
    if (out->split == 0)
    {
        if (threadIdx.x == 0)
        {
            ctl->n_cur = 0;
        }
        return;
    }
    // warp c sums child c's first feature
    uint32_t const wc = threadIdx.x >> 5;
    if (wc < 2)
    {
        if constexpr (Q)
        {
            int64_t g, h;
            warp_qtotals(static_cast<unsigned long long const *>(pool) +
                             (static_cast<uint64_t>(slot_of[wc]) * total_cells * cw),
                         sel_nb[0], cw, g, h);
            if ((threadIdx.x & 31) == 0)
            {
                qtot_s[2 * wc]       = g;
                qtot_s[(2 * wc) + 1] = h;
            }
        }
        else
        {
            float g, h;
            warp_totals(static_cast<float2 const *>(pool) +
                            (static_cast<uint64_t>(slot_of[wc]) * total_cells),
                        sel_nb[0], g, h);
            if ((threadIdx.x & 31) == 0)
            {
                tot_s[2 * wc]       = g;
                tot_s[(2 * wc) + 1] = h;
            }
        }
    }
    __syncthreads();
    if (threadIdx.x != 0)
    {
        return;
    }
    LeafPop const p = *pp;
    Node          L = next[0];
    Node          R = next[1];
    double gl, hl, gr, hr;
    if constexpr (Q)
    {
        L.qg             = qtot_s[0];
        L.qh             = qtot_s[1];
        R.qg             = qtot_s[2];
        R.qh             = qtot_s[3];
        double2 const sc = *qscale;
        gl = static_cast<double>(L.qg) * sc.x;
        hl = static_cast<double>(L.qh) * sc.y;
        gr = static_cast<double>(R.qg) * sc.x;
        hr = static_cast<double>(R.qh) * sc.y;
    }
    else
    {
        L.sum_g = tot_s[0];
        L.sum_h = tot_s[1];
        R.sum_g = tot_s[2];
        R.sum_h = tot_s[3];
        gl = L.sum_g;
        hl = L.sum_h;
        gr = R.sum_g;
        hr = R.sum_h;
    }
    uint32_t const f  = sel[p.best.feature];
    int const      mc = (mono != nullptr && f < n_mono) ? mono[f] : 0;
    interaction_children(p.node, fgroups, f, L, R);
    if (mc != 0)
    {
        double const wl  = bounded_leaf_weight(gl, hl, tp.lambda_l1, tp.lambda_l2, p.node.lo,
                                               p.node.hi);
        double const wr  = bounded_leaf_weight(gr, hr, tp.lambda_l1, tp.lambda_l2, p.node.lo,
                                               p.node.hi);
        double const mid = 0.5 * (wl + wr);
        if (mc > 0)
        {
            L.hi = fmin(L.hi, mid);
            R.lo = fmax(R.lo, mid);
        }
        else
        {
            L.lo = fmax(L.lo, mid);
            R.hi = fmin(R.hi, mid);
        }
    }
    next[0]    = L;
    next[1]    = R;
    ctl->n_cur = 2;
}

// Each node's best split over the features (the lowest feature wins a gain
// tie), no split past the depth cap; the nodes and splits go to the host.
// grid 2 (a CTA per node) x k_best_thr: each thread scans a stride of the
// features, then (largest gain, lowest feature) over the block -- the serial
// scan's choice, whatever the order.
constexpr uint32_t k_best_thr = 256;

__global__ void __launch_bounds__(k_best_thr)
    leaf_best_kernel(Ctl const *ctl, Best const *cand, uint32_t n_sel, Node const *nodes,
                     LeafOut *out, uint32_t const *may_split_p)
{
    pdl_enter();
    uint32_t const      may_split = *may_split_p;
    __shared__ double   g_s[k_best_thr / 32];
    __shared__ uint32_t o_s[k_best_thr / 32];
    uint32_t const      w    = blockIdx.x;
    uint32_t const      lane = threadIdx.x & 31;
    bool const          live = w < ctl->n_cur;
    double              g    = 0.0;
    uint32_t            o    = 0xFFFFFFFFu;
    for (uint32_t j = threadIdx.x; live && may_split != 0 && j < n_sel; j += k_best_thr)
    {
        Best const c = cand[(w * n_sel) + j];
        if (c.valid != 0 && (c.gain > g || (c.gain == g && j < o)))
        {
            g = c.gain;
            o = j;
        }
    }
    warp_best(g, o);
    if (lane == 0)
    {
        g_s[threadIdx.x >> 5] = g;
        o_s[threadIdx.x >> 5] = o;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        for (uint32_t x = 1; x < k_best_thr / 32; ++x)
        {
            if (g_s[x] > g || (g_s[x] == g && o_s[x] < o))
            {
                g = g_s[x];
                o = o_s[x];
            }
        }
        out->best[w] = o == 0xFFFFFFFFu ? Best{0.0, 0, 0, 1, 0} : cand[(w * n_sel) + o];
        if (live)
        {
            out->child[w] = nodes[w];
        }
    }
}

// ---- the leafwise pop loop on the device -----------------------------------
// LeafwiseGrower::grow's heap loop (src/grower_impl.hpp:744-850): the gain
// max-heap (ties to the lower node id, so growth is deterministic), the
// histogram pool's free slots, the node table and the leaf list all live on
// the device, and one pop is a fixed sequence of launches that a CUDA graph's
// conditional WHILE node repeats until the heap is empty or the leaf budget
// is spent -- no host round trip per pop.

struct LeafCand
{
    Node     node;
    Best     best;
    uint32_t depth;
    uint32_t slot;
};

struct LeafLoop
{
    LeafPop  pop;        // the current pop
    uint32_t pop_depth;
    uint32_t may_split;  // the pop's children may split (depth cap)
    uint32_t root_may;   // the root may split
    uint32_t noop;       // this iteration has nothing to pop
    uint32_t n_cand;
    uint32_t n_leaves;
    uint32_t n_nodes;
    uint32_t live;
    uint32_t depth;
    uint32_t n_free;
    uint32_t error;      // 1: the node table is full, 2: the histogram pool is
    uint32_t pops;       // pops taken this tree
};

// After the root's find: the root a candidate (or a leaf), the node table's
// first entry, every pool slot but the root's free.
__global__ void __launch_bounds__(k_plan_thr)
    leaf_loop_init_kernel(LeafLoop *st, LeafCand *cand, Node *leaves, uint32_t *free_slots,
                          LeafOut const *out, TreeOut const *tp_, uint32_t n_root,
                          uint32_t max_front, uint32_t max_depth)
{
    pdl_enter();
    for (uint32_t k = threadIdx.x; k + 1 < max_front; k += k_plan_thr)
    {
        free_slots[k] = max_front - 1 - k; // popped from the top: slot 1 first
    }
    if (threadIdx.x != 0)
    {
        return;
    }
    TreeOut const t   = *tp_;
    t.feature[0]      = k_leaf_flag;
    t.left[0]         = 0;
    t.right[0]        = 0;
    t.split_bin[0]    = 0;
    t.value[0]        = 0.0F;
    t.gain[0]         = 0.0F;
    t.cover[0]        = static_cast<float>(n_root);
    t.default_left[0] = 0;
    LeafCand const root{out->child[0], out->best[0], 0, 0};
    bool const     ok = root.best.valid != 0 && max_depth > 0;
    st->n_cand        = ok ? 1 : 0;
    if (ok)
    {
        cand[0] = root;
    }
    else
    {
        leaves[0] = root.node;
    }
    st->n_leaves = ok ? 0 : 1;
    st->n_nodes  = 1;
    st->live     = 1;
    st->depth    = 0;
    st->n_free   = max_front - 1;
    st->error    = 0;
    st->pops     = 0;
    st->noop     = 0;
}

// One pop: the best candidate off the heap, commit_split_node
// (src/grower_impl.hpp:189-206) into the node table, a pool slot for the
// smaller child, and the popped node's partition chunks (the setup of one
// pop). With nothing to pop it sets the iteration's no-op flag and leaves
// no chunks, so the rest of the iteration does nothing.
constexpr uint32_t k_pop_thr = 256;

__global__ void __launch_bounds__(k_pop_thr)
    leaf_pop_kernel(LeafLoop *st, LeafCand *cand, uint32_t *free_slots, TreeOut const *tp_,
                    float const *cuts, uint32_t const *cut_off, uint32_t const *sel,
                    uint32_t max_leaves, uint32_t max_nodes, uint32_t max_depth, Ctl *ctl,
                    Node *nodes, Best *best, Chunk *pchunks, uint32_t *pcr)
{
    pdl_enter();
    __shared__ double   g_s[k_pop_thr / 32];
    __shared__ uint32_t id_s[k_pop_thr / 32];
    __shared__ uint32_t ix_s[k_pop_thr / 32];
    __shared__ uint32_t go_s;
    uint32_t const      n    = st->n_cand;
    uint32_t const      lane = threadIdx.x & 31;
    if (threadIdx.x == 0)
    {
        bool const go = st->error == 0 && n > 0 && (max_leaves == 0 || st->live < max_leaves);
        go_s          = go ? 1 : 0;
        st->noop      = go ? 0 : 1;
        if (!go)
        {
            ctl->n_cur     = 0;
            ctl->n_pchunks = 0;
            ctl->n_build   = 0;
            ctl->n_bchunks = 0;
            pcr[0]         = 0;
            pcr[1]         = 0;
            st->pop.node.count = 0;
        }
    }
    __syncthreads();
    if (go_s == 0)
    {
        return;
    }
    // the heap's top: the largest gain, then the lowest node id
    double   g  = -1.0;
    uint32_t id = 0xFFFFFFFFu;
    uint32_t ix = 0;
    for (uint32_t i = threadIdx.x; i < n; i += k_pop_thr)
    {
        double const   cg  = cand[i].best.gain;
        uint32_t const cid = cand[i].node.id;
        if (cg > g || (cg == g && cid < id))
        {
            g  = cg;
            id = cid;
            ix = i;
        }
    }
#pragma unroll
    for (uint32_t o = 16; o > 0; o >>= 1)
    {
        double const   og  = __shfl_xor_sync(0xFFFFFFFFu, g, o);
        uint32_t const oid = __shfl_xor_sync(0xFFFFFFFFu, id, o);
        uint32_t const oix = __shfl_xor_sync(0xFFFFFFFFu, ix, o);
        if (og > g || (og == g && oid < id))
        {
            g  = og;
            id = oid;
            ix = oix;
        }
    }
    if (lane == 0)
    {
        g_s[threadIdx.x >> 5]  = g;
        id_s[threadIdx.x >> 5] = id;
        ix_s[threadIdx.x >> 5] = ix;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        for (uint32_t w = 1; w < k_pop_thr / 32; ++w)
        {
            if (g_s[w] > g || (g_s[w] == g && id_s[w] < id))
            {
                g  = g_s[w];
                id = id_s[w];
                ix = ix_s[w];
            }
        }
        LeafCand const c = cand[ix];
        cand[ix]         = cand[n - 1];
        st->n_cand       = n - 1;
        uint32_t const lid = st->n_nodes;
        uint32_t const rid = lid + 1;
        if (rid >= max_nodes || st->n_free == 0)
        {
            st->error          = rid >= max_nodes ? 1 : 2;
            st->noop           = 1;
            ctl->n_cur         = 0;
            ctl->n_pchunks     = 0;
            ctl->n_build       = 0;
            ctl->n_bchunks     = 0;
            pcr[0]             = 0;
            pcr[1]             = 0;
            st->pop.node.count = 0;
            go_s               = 0;
        }
        else
        {
            TreeOut const t = *tp_;
            for (uint32_t k = lid; k <= rid; ++k)
            {
                t.feature[k]      = k_leaf_flag;
                t.left[k]         = 0;
                t.right[k]        = 0;
                t.split_bin[k]    = 0;
                t.value[k]        = 0.0F;
                t.gain[k]         = 0.0F;
                t.cover[k]        = 0.0F;
                t.default_left[k] = 0;
            }
            uint32_t const f     = sel[c.best.feature];
            uint32_t const nid   = c.node.id;
            t.feature[nid]       = f;
            t.value[nid]         = cuts[cut_off[f] + c.best.bin];
            t.left[nid]          = lid;
            t.right[nid]         = rid;
            t.default_left[nid]  = static_cast<uint8_t>(c.best.dl);
            t.gain[nid]          = static_cast<float>(c.best.gain);
            t.split_bin[nid]     = c.best.bin;
            st->n_nodes          = rid + 1;
            uint32_t const small = free_slots[--st->n_free];
            st->pop       = LeafPop{c.node, c.best, lid, rid, c.slot, small};
            st->pop_depth = c.depth;
            st->may_split = c.depth + 1 < max_depth ? 1 : 0;
            st->pops += 1;
            // the pop's setup: the node's partition chunks
            uint32_t const nch = (c.node.count + k_part_rows - 1) / k_part_rows;
            ctl->n_cur         = 1;
            ctl->n_pchunks     = nch;
            Node nd            = c.node;
            nd.flags           = 1;
            nodes[0]           = nd;
            best[0]            = c.best;
            pcr[0]             = 0;
            pcr[1]             = nch;
        }
    }
    __syncthreads();
    if (go_s == 0)
    {
        return;
    }
    LeafPop const &p   = st->pop;
    uint32_t const cnt = p.node.count;
    uint32_t const nch = (cnt + k_part_rows - 1) / k_part_rows;
    for (uint32_t c = threadIdx.x; c < nch; c += k_pop_thr)
    {
        uint32_t const b = c * k_part_rows;
        pchunks[c]       = {0, p.node.start + b, min(k_part_rows, cnt - b), 0};
    }
}

// The pop's outcome into the loop's state (commit_pop's demotion, or the two
// children queued: queue_children, src/grower_impl.hpp:405-425), then whether
// the loop goes on.
__global__ void leaf_commit_kernel(LeafLoop *st, LeafCand *cand, Node *leaves,
                                   uint32_t *free_slots, LeafOut const *out,
                                   TreeOut const *tp_, uint32_t max_leaves, uint32_t max_pops,
                                   cudaGraphConditionalHandle handle)
{
    pdl_enter();
    if (st->noop == 0)
    {
        LeafPop const &p = st->pop;
        TreeOut const  t = *tp_;
        if (out->split == 0)
        {
            // the survivor holds the parent's rows and takes its id and
            // bounds; the two children stay placeholders
            t.gain[p.node.id]           = 0.0F;
            leaves[st->n_leaves++]      = p.node;
            free_slots[st->n_free++]    = p.small_slot;
            free_slots[st->n_free++]    = p.parent_slot;
        }
        else
        {
            Node const     L  = out->child[0];
            Node const     R  = out->child[1];
            bool const     sl = out->small_left != 0;
            uint32_t const d  = st->pop_depth + 1;
            t.cover[p.left_id]  = static_cast<float>(L.gcount);
            t.cover[p.right_id] = static_cast<float>(R.gcount);
            st->live += 1;
            st->depth = max(st->depth, d);
            LeafCand const kids[2] = {{L, out->best[0], d, sl ? p.small_slot : p.parent_slot},
                                      {R, out->best[1], d, sl ? p.parent_slot : p.small_slot}};
            for (LeafCand const &k : kids)
            {
                if (k.best.valid != 0)
                {
                    cand[st->n_cand++] = k;
                }
                else
                {
                    leaves[st->n_leaves++]   = k.node;
                    free_slots[st->n_free++] = k.slot;
                }
            }
        }
    }
    // every pop either adds a leaf or retires a candidate, so at most
    // 2 x max_leaves pops ever run; past max_pops the loop stops with an error
    // rather than spin
    if (st->pops >= max_pops && st->noop == 0)
    {
        st->error = 3;
    }
    bool const more = st->noop == 0 && st->error == 0 && st->n_cand > 0 &&
                      (max_leaves == 0 || st->live < max_leaves);
    cudaGraphSetConditional(handle, more ? 1u : 0u);
}

// The tree's epilogue: every remaining candidate is a leaf; the leaf list,
// node count and depth go to the level plane's control block.
__global__ void leaf_loop_end_kernel(LeafLoop *st, LeafCand const *cand, Node *leaves,
                                     Node *nodes, Ctl *ctl)
{
    pdl_enter();
    uint32_t const nl = st->n_leaves;
    uint32_t const nc = st->n_cand;
    for (uint32_t i = threadIdx.x; i < nl + nc; i += blockDim.x)
    {
        nodes[i] = i < nl ? leaves[i] : cand[i - nl].node;
    }
    if (threadIdx.x == 0)
    {
        ctl->n_cur    = nl + nc;
        ctl->n_nodes  = st->n_nodes;
        ctl->depth    = st->depth;
        ctl->n_leaves = 0;
    }
}

__global__ void leaf_set_tree_kernel(TreeOut *dst, TreeOut t, LeafLoop *st, uint32_t root_may)
{
    pdl_enter();
    *dst          = t;
    st->root_may  = root_may;
}

__global__ void tree_counter_kernel(uint32_t *tree_no)
{
    pdl_enter();
    *tree_no += 1;
}

template <typename T> T *dalloc(size_t n, cudaStream_t s)
{
    void *p = nullptr;
    BB_CHECK(cudaMallocAsync(&p, std::max<size_t>(1, n) * sizeof(T), s));
    return static_cast<T *>(p);
}

} // namespace

Grower::Grower(Plane const &plane, GrowConfig const &cfg, std::vector<uint32_t> selected,
               uint32_t max_root_rows, cudaStream_t stream)
    : plane_(plane), cfg_(cfg), sel_h_(std::move(selected)), stream_(stream)
{
    pdl_ = plane_.n_rows >= (uint64_t{1} << 19);
    if (cfg_.sample_k > 0)
    {
        // per-tree samples: the first sample_k features until set_selection
        if (cfg_.sample_k > plane_.n_feats || cfg_.sel_sets == 0)
        {
            throw ConfigError("grower: a feature sample larger than the plane");
        }
        sel_h_.resize(cfg_.sample_k);
        std::iota(sel_h_.begin(), sel_h_.end(), 0U);
    }
    n_sel_ = static_cast<uint32_t>(sel_h_.size());
    quant_ = cfg_.mode != HistMode::exact;
    if (n_sel_ == 0)
    {
        throw ConfigError("grower: the feature selection is empty");
    }
    if (cfg_.leaf)
    {
        if (cfg_.tp.max_leaves == 0 && cfg_.tp.max_depth <= 9)
        {
            cfg_.tp.max_leaves = 1u << cfg_.tp.max_depth; // unbounded: the depth's cap
        }
        if (cfg_.tp.max_leaves < 1 || cfg_.tp.max_leaves > 512 || cfg_.tp.max_depth > 255)
        {
            throw ConfigError("grower: leafwise needs 1 <= max_leaves <= 512 and "
                              "max_depth <= 255");
        }
    }
    else if (cfg_.tp.max_depth > 8)
    {
        throw ConfigError("grower: max_depth above 8 exceeds the level plane's "
                          "512-node frontier; use a host grower");
    }
    {
        uint64_t const fit_rows = std::max<uint64_t>(cfg_.fit_rows, max_root_rows);
        wide_codes_ = cfg_.mode == HistMode::quant16;
        // int16 sums always outgrow a packed 32-bit half; int8 sums do once
        // 127 x rows reaches 2^31 (16,909,320 rows)
        cw_ = wide_codes_ || (cfg_.mode == HistMode::quant8 && fit_rows * 127ULL >= (1ULL << 31))
                  ? 2
                  : 1;
        // the leaf sums add at most one unit per row: 2^38 up to 2^24 rows,
        // then one bit less per doubling, so no sum leaves the int64 range
        uint32_t lg = 24;
        while (lg < 62 && (uint64_t{1} << lg) < fit_rows)
        {
            ++lg;
        }
        fix_unit_ = std::ldexp(1.0, 62 - static_cast<int>(lg));
    }
    std::vector<uint32_t> off(n_sel_ + 1, 0);
    std::vector<uint32_t> nb(n_sel_, 0);
    for (uint32_t j = 0; j < n_sel_; ++j)
    {
        uint32_t const f = sel_h_[j];
        nb[j]            = plane_.h_cut_off[f + 1] - plane_.h_cut_off[f];
        off[j + 1]       = off[j] + nb[j];
        max_nb_          = std::max(max_nb_, nb[j]);
    }
    if (max_nb_ > k_max_bins)
    {
        throw ConfigError("grower: a feature has more than 4096 bins; lower "
                          "bin_mapper.max_bin or use a host grower");
    }
    total_cells_ = off[n_sel_];
    off_h_       = off;
    if (cfg_.sample_k > 0)
    {
        // bounds over every sample: the largest feature's bins, and per node
        // the cells of the sample_k largest features (off_h_ is read at the
        // whole sample and at its first feature only)
        std::vector<uint32_t> all(plane_.n_feats);
        for (uint32_t f = 0; f < plane_.n_feats; ++f)
        {
            all[f]  = plane_.h_cut_off[f + 1] - plane_.h_cut_off[f];
            max_nb_ = std::max(max_nb_, all[f]);
        }
        std::sort(all.begin(), all.end(), std::greater<>());
        total_cells_ = std::accumulate(all.begin(), all.begin() + n_sel_, 0U);
        off_h_.assign(n_sel_ + 1, 0);
        off_h_[1]      = max_nb_;
        off_h_[n_sel_] = total_cells_;
        if (max_nb_ > k_max_bins)
        {
            throw ConfigError("grower: a feature has more than 4096 bins; lower "
                              "bin_mapper.max_bin or use a host grower");
        }
    }
    cell_stride_ = ((max_nb_ + 1 + 3) / 4) * 4;
    // leafwise: a pool slot per live leaf plus the one being built; a pop
    // consumes a heap entry (at most 2 per split + the root), two nodes each
    max_front_   = cfg_.leaf ? cfg_.tp.max_leaves + 1 : 1u << cfg_.tp.max_depth;
    max_nodes_   = cfg_.leaf ? 4 * cfg_.tp.max_leaves : (2u << cfg_.tp.max_depth) - 1;
    max_rows_    = std::max<uint32_t>(max_root_rows, 1);
    crows_       = quant_ ? k_qbuild_rows : k_build_rows;
    // the histogram grid: one CTA per SM for a large fit, about one per four
    // 2,048-row chunks of the root for a small one
    qctas_       = cfg_.hist_ctas > 0
                       ? std::min(cfg_.hist_ctas, 64u * k_qctas)
                       : std::max(1u, std::min(k_qctas, ceil_div(max_rows_, 4 * k_qbuild_rows)));
    max_pchunks_ = ceil_div(max_rows_, k_part_rows) + max_front_;
    max_bchunks_ = ceil_div(max_rows_, crows_) + max_front_;

    cudaStream_t   s     = stream_;
    uint32_t const nsets = std::max(1u, cfg_.sel_sets);
    sel_base_      = dalloc<uint32_t>(static_cast<size_t>(nsets) * n_sel_, s);
    cell_off_base_ = dalloc<uint32_t>(static_cast<size_t>(nsets) * (n_sel_ + 1), s);
    sel_nb_base_   = dalloc<uint32_t>(static_cast<size_t>(nsets) * n_sel_, s);
    if (quant_)
    {
        // the mirror tiles a selection can touch: all selected features (v
        // 0), and the first one alone (v 1: the last level builds only its
        // totals); a sampled grower sizes them for any sample
        uint32_t const per     = k_mirror_bytes / (plane_.u8 ? 1 : 2);
        uint32_t const n_tiles = ceil_div(plane_.n_feats, per);
        for (int v = 0; v < 2; ++v)
        {
            uint32_t cap = 1;
            if (v == 0)
            {
                cap = 0;
                for (uint32_t j = 0; j < n_sel_; ++j)
                {
                    cap += (j == 0 || sel_h_[j] / per != sel_h_[j - 1] / per) ? 1 : 0;
                }
                if (cfg_.sample_k > 0)
                {
                    cap = std::min(n_sel_, n_tiles);
                }
            }
            n_tiles_[v]       = cap;
            tile_ids_base_[v] = dalloc<uint32_t>(static_cast<size_t>(nsets) * cap, s);
            tile_j_base_[v]   = dalloc<int32_t>(static_cast<size_t>(nsets) * cap * per, s);
        }
    }
    sets_h_.assign(nsets, sel_h_);
    for (uint32_t k = 0; k < nsets; ++k)
    {
        write_tables(k, sel_h_);
    }
    use_set(0);
    ctl_      = dalloc<Ctl>(1, s);
    nodes_[0] = dalloc<Node>(max_front_, s);
    nodes_[1] = dalloc<Node>(max_front_, s);
    hist_[0]  = dalloc<float2>(static_cast<size_t>(max_front_) * total_cells_ * cw_, s);
    // (leafwise uses the first buffer as its slot pool)
    hist_[1]  = dalloc<float2>(static_cast<size_t>(cfg_.leaf ? 1 : max_front_) * total_cells_ * cw_,
                               s);
    cand_     = dalloc<Best>(static_cast<size_t>(max_front_) * n_sel_, s);
    best_     = dalloc<Best>(max_front_, s);
    pchunks_  = dalloc<Chunk>(max_pchunks_, s);
    pleft_    = dalloc<uint32_t>(max_pchunks_, s);
    dirs_     = dalloc<uint32_t>(static_cast<size_t>(max_pchunks_) * (k_part_rows / 32), s);
    prbase_   = dalloc<uint32_t>(max_pchunks_, s);
    dst_      = dalloc<uint32_t>(max_front_ + 1, s);
    build_    = dalloc<uint32_t>(max_front_ * 2 + 2, s);
    bpair_    = dalloc<uint32_t>(3 * max_front_, s);
    bbase_    = dalloc<uint32_t>(max_front_ + 1, s);
    brange_   = dalloc<uint32_t>(max_front_ + 2, s);
    bchunks_  = dalloc<Chunk>(max_bchunks_, s);
    rows_[0]  = dalloc<uint32_t>(max_rows_, s);
    rows_[1]  = dalloc<uint32_t>(max_rows_, s);
    pcr_      = dalloc<uint32_t>(max_front_ + 2, s);
    nbound_   = dalloc<double2>(std::max<uint32_t>(max_nodes_, k_walk_nodes), s);
    heap_     = dalloc<uint2>(k_heap_slots, s);
    leafmap_  = dalloc<uint16_t>(k_heap_slots + 1, s);
    if (cfg_.leaf)
    {
        lout_      = dalloc<LeafOut>(1, s);
        slot_of_   = dalloc<uint32_t>(2, s);
        loop_      = dalloc<LeafLoop>(1, s);
        cand_heap_ = dalloc<LeafCand>(max_front_ + 2, s);
        leaves_    = dalloc<Node>(max_front_ + 2, s);
        free_      = dalloc<uint32_t>(max_front_ + 2, s);
        tree_dev_  = dalloc<TreeOut>(1, s);
        BB_CHECK(cudaMallocHost(&lout_h_, sizeof(LeafLoop)));
    }
    nleft_    = dalloc<uint32_t>(max_front_ + 1, s);
    nright_   = dalloc<uint32_t>(max_front_ + 1, s);
    dtree_    = dalloc<uint32_t>(1, s);
    BB_CHECK(cudaMemsetAsync(dtree_, 0, 4, s));
    if (quant_)
    {
        absmax_  = dalloc<uint32_t>(2, s);
        qscale_  = dalloc<double2>(1, s);
        // +2: the histogram copies whole 4-byte words of codes
        qgh8_    = dalloc<uint16_t>((max_rows_ > plane_.n_rows ? max_rows_ : plane_.n_rows) + 2, s);
        if (wide_codes_)
        {
            qgh16_ = dalloc<uint32_t>((max_rows_ > plane_.n_rows ? max_rows_ : plane_.n_rows) + 1,
                                      s);
        }
        partial_ = dalloc<double2>(max_pchunks_, s);
        btot_    = dalloc<int64_t>(2 * static_cast<size_t>(max_front_), s);
        done_    = dalloc<uint32_t>(1, s);
        wacc_    = dalloc<unsigned long long>(2 * k_walk_nodes, s);
        leaf16_  = dalloc<uint16_t>(plane_.n_rows, s);
        BB_CHECK(cudaMemsetAsync(done_, 0, 4, s));
        uint32_t const per = k_mirror_bytes / (plane_.u8 ? 1 : 2);
        size_t const qsmem = static_cast<size_t>(per) * max_nb_ * 8;
        if (qsmem > 200 * 1024)
        {
            throw ConfigError("grower: quantised histograms of this many bins exceed "
                              "shared memory; lower bin_mapper.max_bin");
        }
        BB_CHECK(cudaFuncSetAttribute(qhist_kernel<uint16_t>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(qsmem)));
        BB_CHECK(cudaFuncSetAttribute(qhist_kernel<uint16_t, true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(qsmem)));
        BB_CHECK(cudaFuncSetAttribute(qhist_kernel<uint16_t, false, true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(qsmem)));
        BB_CHECK(cudaFuncSetAttribute(qhist_kernel<uint8_t, true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(static_cast<size_t>(32) * max_nb_ * 8)));
        size_t const tsmem = k_tsmem;
        BB_CHECK(cudaFuncSetAttribute(qhist_t_kernel<false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(tsmem)));
        BB_CHECK(cudaFuncSetAttribute(qhist_t_kernel<true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(tsmem)));
        // the summing walk's accumulator copies at depth 8
        int const wsmem = static_cast<int>((size_t{2} << 8) * k_wsum_copies * 8);
        BB_CHECK(cudaFuncSetAttribute(walk_sum_kernel<true, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, wsmem));
        BB_CHECK(cudaFuncSetAttribute(walk_sum_kernel<true, true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, wsmem));
        BB_CHECK(cudaFuncSetAttribute(walk_sum_kernel<false, false>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, wsmem));
        BB_CHECK(cudaFuncSetAttribute(walk_sum_kernel<false, true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, wsmem));
    }
    else
    {
        ccount_  = dalloc<uint32_t>(static_cast<size_t>(max_bchunks_) * n_sel_ * cell_stride_, s);
        seg_     = dalloc<uint32_t>(static_cast<size_t>(max_front_) * n_sel_ * cell_stride_, s);
        payload_ = dalloc<float2>(static_cast<size_t>(n_sel_) * max_rows_, s);
    }
    scale_ = dalloc<float2>(1, s);
    BB_CHECK(cudaMemsetAsync(scale_, 0, sizeof(float2), s));
    BB_CHECK(cudaStreamSynchronize(s));

    // dynamic shared memory ceilings
    size_t const find_smem = max_nb_ * (sizeof(double2) + (sizeof(unsigned long long) * cw_));
    if (find_smem > 227 * 1024)
    {
        throw ConfigError("grower: bins per feature exceed the shared-memory budget");
    }
    BB_CHECK(cudaFuncSetAttribute(find_kernel<false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(find_smem)));
    BB_CHECK(cudaFuncSetAttribute(find_kernel<true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(find_smem)));
    // the level finder prefixes up to 16 nodes at a time in shared memory
    lgroup_ = static_cast<uint32_t>(std::min<size_t>(
        k_lfind_thr / 32, std::max<size_t>(1, (192 * 1024) / (max_nb_ * sizeof(double2)))));
    size_t const lsmem = static_cast<size_t>(lgroup_) * max_nb_ * sizeof(double2);
    BB_CHECK(cudaFuncSetAttribute(level_find_kernel<false>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(lsmem)));
    BB_CHECK(cudaFuncSetAttribute(level_find_kernel<true>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(lsmem)));
    if (!quant_)
    {
        size_t const cnt_smem   = k_warps_feat * cell_stride_ * sizeof(uint32_t);
        size_t const bin_bytes  = plane_.u8 ? 1 : 2;
        size_t const sc_smem    = (k_build_rows * (4 + 8)) + cnt_smem +
                               (k_warps_feat * k_build_rows * bin_bytes);
        size_t const chain_smem = 32 * k_chain_stg * k_chain_nst * sizeof(float2);
        if (sc_smem > 227 * 1024)
        {
            throw ConfigError("grower: bins per feature exceed the shared-memory budget");
        }
        auto ck = plane_.u8 ? reinterpret_cast<void const *>(&count_kernel<uint8_t>)
                            : reinterpret_cast<void const *>(&count_kernel<uint16_t>);
        auto sk = plane_.u8 ? reinterpret_cast<void const *>(&scatter_kernel<uint8_t>)
                            : reinterpret_cast<void const *>(&scatter_kernel<uint16_t>);
        BB_CHECK(cudaFuncSetAttribute(ck, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(cnt_smem)));
        BB_CHECK(cudaFuncSetAttribute(sk, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(sc_smem)));
        BB_CHECK(cudaFuncSetAttribute(chain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(chain_smem)));
    }
    BB_CHECK(cudaEventCreate(&pev_[0]));
    BB_CHECK(cudaEventCreate(&pev_[1]));
}

// Set k's tables for the ascending feature ids sel: the ids, each one's
// first cell and bin count, and (quantised) the mirror tiles holding them
// with each tile slot's selection index, unused slots marked. The host
// vectors are pageable, so each copy has left them when it returns.
void Grower::write_tables(uint32_t set, std::vector<uint32_t> const &sel)
{
    cudaStream_t          s = stream_;
    std::vector<uint32_t> off(n_sel_ + 1, 0);
    std::vector<uint32_t> nb(n_sel_, 0);
    for (uint32_t j = 0; j < n_sel_; ++j)
    {
        uint32_t const f = sel[j];
        nb[j]            = plane_.h_cut_off[f + 1] - plane_.h_cut_off[f];
        off[j + 1]       = off[j] + nb[j];
    }
    BB_CHECK(cudaMemcpyAsync(sel_base_ + (static_cast<size_t>(set) * n_sel_), sel.data(),
                             n_sel_ * 4, cudaMemcpyHostToDevice, s));
    BB_CHECK(cudaMemcpyAsync(cell_off_base_ + (static_cast<size_t>(set) * (n_sel_ + 1)),
                             off.data(), (n_sel_ + 1) * 4, cudaMemcpyHostToDevice, s));
    BB_CHECK(cudaMemcpyAsync(sel_nb_base_ + (static_cast<size_t>(set) * n_sel_), nb.data(),
                             n_sel_ * 4, cudaMemcpyHostToDevice, s));
    if (!quant_)
    {
        return;
    }
    uint32_t const per = k_mirror_bytes / (plane_.u8 ? 1 : 2);
    for (int v = 0; v < 2; ++v)
    {
        uint32_t const        cap = n_tiles_[v];
        std::vector<uint32_t> ids;
        std::vector<int32_t>  js(static_cast<size_t>(cap) * per, -1);
        uint32_t const        nfb = v == 0 ? n_sel_ : 1;
        for (uint32_t j = 0; j < nfb; ++j)
        {
            uint32_t const t = sel[j] / per;
            if (ids.empty() || ids.back() != t)
            {
                ids.push_back(t);
            }
            js[((ids.size() - 1) * per) + (sel[j] % per)] = static_cast<int32_t>(j);
        }
        if (ids.size() > cap)
        {
            throw std::logic_error("grower: a selection touches more tiles than its tables hold");
        }
        ids.resize(cap, k_no_sel_tile);
        BB_CHECK(cudaMemcpyAsync(tile_ids_base_[v] + (static_cast<size_t>(set) * cap), ids.data(),
                                 cap * 4, cudaMemcpyHostToDevice, s));
        BB_CHECK(cudaMemcpyAsync(tile_j_base_[v] + (static_cast<size_t>(set) * cap * per),
                                 js.data(), js.size() * 4, cudaMemcpyHostToDevice, s));
    }
}

void Grower::set_selection(uint32_t set, std::vector<uint32_t> const &sel)
{
    if (cfg_.sample_k == 0 || set >= sets_h_.size() || sel.size() != n_sel_)
    {
        throw std::logic_error("grower: set_selection outside a sampled grower's sets");
    }
    for (size_t j = 0; j < sel.size(); ++j)
    {
        if (sel[j] >= plane_.n_feats || (j > 0 && sel[j] <= sel[j - 1]))
        {
            throw std::logic_error("grower: a feature sample must be ascending plane features");
        }
    }
    write_tables(set, sel);
    sets_h_[set] = sel;
}

void Grower::use_set(uint32_t set)
{
    if (set >= sets_h_.size())
    {
        throw std::logic_error("grower: no such selection set");
    }
    uint32_t const per = k_mirror_bytes / (plane_.u8 ? 1 : 2);
    sel_      = sel_base_ + (static_cast<size_t>(set) * n_sel_);
    cell_off_ = cell_off_base_ + (static_cast<size_t>(set) * (n_sel_ + 1));
    sel_nb_   = sel_nb_base_ + (static_cast<size_t>(set) * n_sel_);
    for (int v = 0; v < 2; ++v)
    {
        if (tile_ids_base_[v] != nullptr)
        {
            tile_ids_[v] = tile_ids_base_[v] + (static_cast<size_t>(set) * n_tiles_[v]);
            tile_j_[v]   = tile_j_base_[v] + (static_cast<size_t>(set) * n_tiles_[v] * per);
        }
    }
    sel_h_ = sets_h_[set];
}

Grower::~Grower()
{
    void *ptrs[] = {sel_base_, cell_off_base_, sel_nb_base_, ctl_, nodes_[0], nodes_[1],
                    hist_[0], hist_[1],  cand_,    best_,     pchunks_,    pleft_,
                    prbase_,  dst_,      build_,   bpair_,    brange_,     bchunks_,
                    ccount_,  seg_,      payload_, rows_[0],  rows_[1],    scale_,
                    absmax_,  qgh_,      pcr_,     nleft_,    mono_,       qscale_,
                    qgh8_,    partial_,  dtree_,   tile_ids_base_[0], tile_ids_base_[1],
                    tile_j_base_[0], tile_j_base_[1], bbase_, dirs_, btot_, done_, wacc_,
                    leaf16_,  nbound_,  gleft_,   qgh16_,   fgroups_, heap_, leafmap_, nright_};
    for (void *p : ptrs)
    {
        if (p != nullptr)
        {
            cudaFreeAsync(p, stream_);
        }
    }
    if (lout_ != nullptr)
    {
        cudaFreeAsync(lout_, stream_);
        cudaFreeAsync(slot_of_, stream_);
        cudaFreeAsync(loop_, stream_);
        cudaFreeAsync(cand_heap_, stream_);
        cudaFreeAsync(leaves_, stream_);
        cudaFreeAsync(free_, stream_);
        cudaFreeAsync(tree_dev_, stream_);
    }
    if (loop_x_ != nullptr)
    {
        cudaGraphExecDestroy(loop_x_);
    }
    if (loop_g_ != nullptr)
    {
        cudaGraphDestroy(loop_g_);
    }
    cudaStreamSynchronize(stream_);
    if (lout_h_ != nullptr)
    {
        cudaFreeHost(lout_h_);
    }
    cudaEventDestroy(pev_[0]);
    cudaEventDestroy(pev_[1]);
}

void Grower::phase_begin()
{
    if (prof_ != nullptr)
    {
        BB_CHECK(cudaEventRecord(pev_[0], stream_));
    }
}

void Grower::phase_end(double &acc)
{
    if (prof_ != nullptr)
    {
        float ms = 0.0F;
        BB_CHECK(cudaEventRecord(pev_[1], stream_));
        BB_CHECK(cudaEventSynchronize(pev_[1]));
        BB_CHECK(cudaEventElapsedTime(&ms, pev_[0], pev_[1]));
        acc += ms;
    }
}

void Grower::set_shard(Reducer *r, uint64_t row_offset, uint64_t total_rows)
{
    if (r != nullptr && !quant_)
    {
        throw ConfigError("grower: a sharded fit needs the quantised form (integer "
                          "histograms combine exactly; float cells would not)");
    }
    if (r != nullptr && total_rows > std::max<uint64_t>(cfg_.fit_rows, max_rows_))
    {
        throw ConfigError("grower: a shard's grower must be sized for the whole fit's rows "
                          "(GrowConfig::fit_rows)");
    }
    red_        = r;
    row_off_    = row_offset;
    total_rows_ = total_rows;
    if (r != nullptr)
    {
        // a shard's rounds put NCCL's kernels between this grower's: plain
        // stream order there
        pdl_ = false;
    }
    if (gleft_ == nullptr)
    {
        gleft_ = dalloc<uint64_t>(max_front_, stream_);
        BB_CHECK(cudaStreamSynchronize(stream_));
    }
}

void Grower::seed_absmax(float2 const *gh)
{
    if (!quant_)
    {
        return;
    }
    cudaStream_t   s    = stream_;
    uint32_t const n    = static_cast<uint32_t>(plane_.n_rows);
    uint32_t const grid = std::min<uint32_t>(ceil_div(std::max<uint32_t>(n, 1), k_threads),
                                             148u * 8u);
    BB_CHECK(cudaMemsetAsync(absmax_, 0, 8, s));
    launch_k(pdl_, absmax_kernel, grid, k_threads, 0, s, gh, n, absmax_);
    BB_LAUNCH("absmax_kernel");
}

void Grower::quantise(float2 const *gh, uint32_t n, bool have_absmax)
{
    cudaStream_t s = stream_;
    uint32_t const grid = std::min<uint32_t>(ceil_div(std::max<uint32_t>(n, 1), k_threads),
                                             148u * 8u);
    if (!have_absmax)
    {
        BB_CHECK(cudaMemsetAsync(absmax_, 0, 8, s));
        launch_k(pdl_, absmax_kernel, grid, k_threads, 0, s, gh, n, absmax_);
        BB_LAUNCH("absmax_kernel");
        n_launch_ += 1;
    }
    if (red_ != nullptr)
    {
        red_->max_u32(absmax_, 2, s); // the fit's maxima: one scale for every shard
    }
    uint2 const key = make_uint2(static_cast<uint32_t>(seed_),
                                 static_cast<uint32_t>(seed_ >> 32));
    if (wide_codes_)
    {
        launch_k(pdl_, quantise_kernel<true>, grid, k_threads, 0, s, gh, n, absmax_, key, dtree_,
                 qgh16_, qscale_, row_off_);
    }
    else
    {
        launch_k(pdl_, quantise_kernel<false>, grid, k_threads, 0, s, gh, n, absmax_, key, dtree_,
                 qgh8_, qscale_, row_off_);
    }
    BB_LAUNCH("quantise_kernel");
    n_launch_ += 1;
}

void Grower::build(uint32_t const *rows, uint32_t nfb, int dst, bool zeroed)
{
    cudaStream_t s = stream_;
    phase_begin();
    if (quant_)
    {
        int const v = nfb == n_sel_ ? 0 : 1;
        if (!zeroed)
        {
            launch_k(pdl_, zero_build_kernel, max_front_, k_threads, 0, s, ctl_, build_,
                     static_cast<unsigned long long *>(hist_[dst]), total_cells_ * cw_,
                     off_h_[nfb] * cw_);
            BB_LAUNCH("zero_build_kernel");
            n_launch_ += 1;
        }
        uint32_t const per   = k_mirror_bytes / (plane_.u8 ? 1 : 2);
        size_t const   qsmem = static_cast<size_t>(per) * max_nb_ * 8;
        dim3 const     grid(max_bchunks_, n_tiles_[v]);
        if (wide_codes_)
        {
            // int16 codes: the per-chunk kernel with two-word cells
            if (plane_.u8)
            {
                launch_k(pdl_, qhist_kernel<uint8_t, true>, grid, k_qthreads, qsmem, s, ctl_,
                         bchunks_, build_, rows, static_cast<uint4 const *>(plane_.mirror),
                         plane_.n_rows, qgh16_, tile_ids_[v], tile_j_[v], sel_nb_, cell_off_,
                         max_nb_, static_cast<unsigned long long *>(hist_[dst]), total_cells_);
            }
            else
            {
                launch_k(pdl_, qhist_kernel<uint16_t, true>, grid, k_qthreads, qsmem, s, ctl_,
                         bchunks_, build_, rows, static_cast<uint4 const *>(plane_.mirror),
                         plane_.n_rows, qgh16_, tile_ids_[v], tile_j_[v], sel_nb_, cell_off_,
                         max_nb_, static_cast<unsigned long long *>(hist_[dst]), total_cells_);
            }
        }
        else if (plane_.u8)
        {
            size_t const tsmem = k_tsmem;
            // CTAs per tile: the caller's count, else one per SM for a plane of
            // one tile, and about two waves over all tiles for a wide plane (a
            // CTA zeroes and flushes a 64 KB table per node, so many tiles
            // want fewer, longer CTAs each)
            // (at least enough CTAs that no CTA's share of the chunks can
            // overflow its 32-bit shared words)
            uint32_t const ctas = std::max(
                ceil_div(max_bchunks_, k_tshare_chunks),
                cfg_.hist_ctas > 0
                    ? qctas_
                    : std::max(1u, std::min(qctas_, ceil_div(2 * k_qctas, n_tiles_[v]))));
            auto const kern = cw_ == 2 ? qhist_t_kernel<true> : qhist_t_kernel<false>;
            launch_k(pdl_, kern, dim3(ctas, n_tiles_[v]), k_tthreads, tsmem, s, ctl_, bchunks_,
                     build_, rows, static_cast<uint4 const *>(plane_.mirror), plane_.n_rows, qgh8_,
                     tile_ids_[v], tile_j_[v], sel_nb_, cell_off_, max_nb_,
                     static_cast<unsigned long long *>(hist_[dst]), total_cells_);
        }
        else
        {
            auto const kern =
                cw_ == 2 ? qhist_kernel<uint16_t, false, true> : qhist_kernel<uint16_t>;
            launch_k(pdl_, kern, grid, k_qthreads, qsmem, s, ctl_, bchunks_, build_, rows,
                     static_cast<uint4 const *>(plane_.mirror), plane_.n_rows, qgh8_, tile_ids_[v],
                     tile_j_[v], sel_nb_, cell_off_, max_nb_,
                     static_cast<unsigned long long *>(hist_[dst]), total_cells_);
        }
        BB_LAUNCH("qhist_kernel");
        n_launch_ += 1;
    }
    else
    {
        size_t const bin_bytes = plane_.u8 ? 1 : 2;
        size_t const cnt_smem  = k_warps_feat * cell_stride_ * sizeof(uint32_t);
        size_t const sc_smem   = (k_build_rows * (4 + 8)) + cnt_smem +
                               (k_warps_feat * k_build_rows * bin_bytes);
        dim3 const   gcs(max_bchunks_, ceil_div(nfb, k_warps_feat));
        uint32_t const *crow = rows != nullptr ? rows : root_rows_;
        if (plane_.u8)
        {
            launch_k(pdl_, count_kernel<uint8_t>, gcs, k_threads, cnt_smem, s, ctl_, bchunks_, crow,
                     plane_.bins, plane_.n_pad, sel_, sel_nb_, nfb, ccount_, cell_stride_);
        }
        else
        {
            launch_k(pdl_, count_kernel<uint16_t>, gcs, k_threads, cnt_smem, s, ctl_, bchunks_,
                     crow, plane_.bins, plane_.n_pad, sel_, sel_nb_, nfb, ccount_, cell_stride_);
        }
        BB_LAUNCH("count_kernel");
        launch_k(pdl_, offsets_kernel, dim3(max_front_, nfb), k_threads, 0, s, ctl_, brange_,
                 ccount_, seg_, sel_nb_, nfb, cell_stride_, bchunks_);
        BB_LAUNCH("offsets_kernel");
        if (plane_.u8)
        {
            launch_k(pdl_, scatter_kernel<uint8_t>, gcs, k_threads, sc_smem, s, ctl_, bchunks_,
                     crow, plane_.bins, plane_.n_pad, gh_cur_, sel_, sel_nb_, nfb, ccount_,
                     cell_stride_, payload_, max_rows_);
        }
        else
        {
            launch_k(pdl_, scatter_kernel<uint16_t>, gcs, k_threads, sc_smem, s, ctl_, bchunks_,
                     crow, plane_.bins, plane_.n_pad, gh_cur_, sel_, sel_nb_, nfb, ccount_,
                     cell_stride_, payload_, max_rows_);
        }
        BB_LAUNCH("scatter_kernel");
        size_t const chain_smem = 32 * k_chain_stg * k_chain_nst * sizeof(float2);
        launch_k(pdl_, chain_kernel, dim3(max_front_, nfb, ceil_div(max_nb_, 32)), 32, chain_smem,
                 s, ctl_, build_, bchunks_, brange_, seg_, payload_, max_rows_, sel_nb_, cell_off_,
                 nfb, cell_stride_, static_cast<float2 *>(hist_[dst]), total_cells_);
        BB_LAUNCH("chain_kernel");
        n_launch_ += 4;
    }
    if (prof_ != nullptr)
    {
        double const before = prof_->hist_ms;
        phase_end(prof_->hist_ms);
        Ctl c{};
        BB_CHECK(cudaMemcpy(&c, ctl_, sizeof(Ctl), cudaMemcpyDeviceToHost));
        double const bin_bytes = plane_.u8 ? 1.0 : 2.0;
        // per built row: the codes read, the gradient pair, the row id
        double const per_row = quant_ ? ((nfb * bin_bytes) + 2.0 + 4.0)
                                      : ((nfb * bin_bytes) + 8.0 + 4.0);
        prof_->hist_rows += c.built_rows;
        prof_->hist_bytes += (static_cast<double>(c.built_rows) * per_row) +
                             (static_cast<double>(c.n_build) * off_h_[nfb] * 8.0);
        if (prof_->hist_builds < Profile::k_prof_builds)
        {
            prof_->build_ms[prof_->hist_builds]   = prof_->hist_ms - before;
            prof_->build_rows[prof_->hist_builds] = c.built_rows;
        }
        prof_->hist_builds += 1;
    }
}

void Grower::leaf_values(TreeOut const &t, bool)
{
    if (!quant_)
    {
        return;
    }
    cudaStream_t s = stream_;
    launch_k(pdl_, leafsum_kernel, max_pchunks_, k_threads, 0, s, ctl_, pchunks_, nodes_cur_,
             rows_cur_, gh_cur_, partial_, pcr_, cfg_.tp, t, done_);
    BB_LAUNCH("leafsum_kernel");
    n_launch_ += 1;
}

void Grower::level(uint32_t L, uint32_t const *rows_in, uint32_t *rows_out,
                   TreeOut const &t, uint32_t *leaf_id, float *scores, float lr)
{
    cudaStream_t s   = stream_;
    int const    cur = static_cast<int>(L & 1);
    int const    nxt = cur ^ 1;
    // grids sized for this level: at most 2^L frontier nodes, and at most one
    // partial partition chunk per node beyond the rows' whole chunks
    uint32_t const front = std::min(max_front_, 1u << std::min(L, 30u));
    uint32_t const pch   = std::min(max_pchunks_, ceil_div(max_rows_, k_part_rows) + front);
    size_t const find_smem = max_nb_ * (sizeof(double2) + (sizeof(unsigned long long) * cw_));
    phase_begin();
    dim3 const fgrid(front, n_sel_);
    if (cfg_.level)
    {
        size_t const lsmem = static_cast<size_t>(lgroup_) * max_nb_ * sizeof(double2);
        if (quant_)
        {
            launch_k(pdl_, level_find_kernel<true>, n_sel_, k_lfind_thr, lsmem, s, ctl_,
                     nodes_[cur], hist_[cur], total_cells_, cell_off_, sel_nb_, n_sel_, cfg_.tp,
                     cand_, max_nb_, lgroup_, qscale_, cw_);
        }
        else
        {
            launch_k(pdl_, level_find_kernel<false>, n_sel_, k_lfind_thr, lsmem, s, ctl_,
                     nodes_[cur], hist_[cur], total_cells_, cell_off_, sel_nb_, n_sel_, cfg_.tp,
                     cand_, max_nb_, lgroup_, qscale_, cw_);
        }
    }
    else if (quant_)
    {
        launch_k(pdl_, qfind_warp_kernel, dim3(front, ceil_div(n_sel_, k_qfind_warps)),
                 k_qfind_warps * 32, 0, s, ctl_, nodes_[cur], hist_[cur], total_cells_, cell_off_,
                 sel_nb_, sel_, n_sel_, mono_, n_mono_, cfg_.tp, cand_, qscale_, nullptr, cw_,
                 fgroups_);
    }
    else
    {
        launch_k(pdl_, find_kernel<false>, fgrid, k_find_thr, find_smem, s, ctl_, nodes_[cur],
                 hist_[cur], total_cells_, cell_off_, sel_nb_, sel_, n_sel_, mono_, n_mono_,
                 cfg_.tp, cand_, max_nb_, qscale_, nullptr, cw_, fgroups_);
    }
    BB_LAUNCH("find_kernel");
    launch_k(pdl_, plan_kernel, 1, k_plan_thr, 0, s, ctl_, nodes_[cur], cand_, best_, n_sel_, sel_,
             plane_.cuts, plane_.cut_off, cfg_.tp, t, pchunks_, pcr_, nbound_, cfg_.level,
             HeapOut{heap_, leafmap_, cfg_.tp.max_depth, k_mirror_bytes / (plane_.u8 ? 1u : 2u)}, nleft_, nright_);
    BB_LAUNCH("plan_kernel");
    if (prof_ != nullptr)
    {
        phase_end(prof_->find_ms);
    }
    phase_begin();
    bool const     last     = (L + 1) == cfg_.tp.max_depth;
    uint32_t const nfb      = last ? 1 : n_sel_;
    uint32_t const n_zcells = quant_ && !last ? off_h_[nfb] * cw_ : 0;
    // a walked quantised tree (unsharded) partitions in one pass: nothing
    // downstream of its row lists depends on the rows' order inside a node
    bool const     fused    = quant_ && walk_ && red_ == nullptr;
    if (fused)
    {
        auto const kern = plane_.u8 ? (last ? psplit_kernel<uint8_t, false>
                                            : psplit_kernel<uint8_t, true>)
                                    : (last ? psplit_kernel<uint16_t, false>
                                            : psplit_kernel<uint16_t, true>);
        launch_k(pdl_, kern, pch, k_threads, 0, s, ctl_, pchunks_, nodes_[cur], best_,
                 rows_in, rows_out, plane_.bins, plane_.n_pad, sel_, sel_nb_, nleft_, nright_,
                 static_cast<unsigned long long *>(hist_[nxt]), total_cells_ * cw_, n_zcells);
        BB_LAUNCH("psplit_kernel");
    }
    else if (plane_.u8)
    {
        launch_k(pdl_, pcount_kernel<uint8_t>, pch, k_threads, 0, s, ctl_, pchunks_,
                 nodes_[cur], best_, rows_in, plane_.bins, plane_.n_pad, sel_, sel_nb_, pleft_,
                 dirs_);
    }
    else
    {
        launch_k(pdl_, pcount_kernel<uint16_t>, pch, k_threads, 0, s, ctl_, pchunks_,
                 nodes_[cur], best_, rows_in, plane_.bins, plane_.n_pad, sel_, sel_nb_, pleft_,
                 dirs_);
    }
    if (!fused)
    {
        BB_LAUNCH("pcount_kernel");
    }
    if (red_ != nullptr)
    {
        launch_k(pdl_, node_left_kernel, 1, k_plan_thr, 0, s, ctl_, pcr_, pleft_, gleft_,
                 max_front_);
        BB_LAUNCH("node_left_kernel");
        red_->sum_u64(gleft_, max_front_, s);
        n_launch_ += 1;
    }
    launch_k(pdl_, plan2_kernel, 1, k_plan_thr, 0, s, ctl_, nodes_[cur], nodes_[nxt], best_,
             pchunks_, pcr_, pleft_, prbase_, nleft_, dst_, bpair_, build_, brange_, bchunks_,
             cfg_.tp, t, crows_, bbase_, cfg_.level, red_ != nullptr ? gleft_ : nullptr, fgroups_,
             HeapOut{heap_, leafmap_, cfg_.tp.max_depth, k_mirror_bytes / (plane_.u8 ? 1u : 2u)}, fused);
    BB_LAUNCH("plan2_kernel");
    nodes_cur_ = nodes_[cur];
    rows_cur_  = rows_in;
    if (!(walk_ && quant_))
    {
        leaf_values(t, false);
    }
    if (!walk_)
    {
        launch_k(pdl_, stamp_kernel, pch, k_threads, 0, s, ctl_, pchunks_, nodes_[cur],
                 rows_in, t, leaf_id, scores, lr);
        BB_LAUNCH("stamp_kernel");
        n_launch_ += 1;
    }
    if (quant_ && last && walk_)
    {
        // a walked tree's last level: the leaves' rows are never listed (the
        // walk routes every row) and their exact totals come from the
        // parents' split cells
        if (prof_ != nullptr)
        {
            phase_end(prof_->partition_ms);
        }
        phase_begin();
        launch_k(pdl_, qsplit_totals_kernel, ceil_div(std::min(max_front_, 2 * front), 8u), 256, 0, s, ctl_, bpair_,
                 nodes_[cur], best_, static_cast<unsigned long long const *>(hist_[cur]),
                 total_cells_, cell_off_, sel_nb_, cw_, btot_);
        BB_LAUNCH("qsplit_totals_kernel");
        launch_k(pdl_, qsubtract_totals_kernel, front, k_threads, 0, s, ctl_, bpair_,
                 static_cast<unsigned long long const *>(hist_[cur]),
                 static_cast<unsigned long long *>(hist_[nxt]), total_cells_, 0, nodes_[cur],
                 nodes_[nxt], best_, sel_, sel_nb_, mono_, n_mono_, cfg_.tp, qscale_, btot_, cw_);
        BB_LAUNCH("qsubtract_totals_kernel");
        n_launch_ += 6; // count, plan2, the two totals kernels (+ find, plan)
        if (prof_ != nullptr)
        {
            phase_end(prof_->other_ms);
        }
        return;
    }
    if (!fused)
    {
        launch_k(pdl_, pscatter_kernel, pch, k_threads, 0, s, ctl_, pchunks_,
                 nodes_[cur], best_, pleft_, prbase_, nleft_, dst_, rows_in, rows_out, dirs_,
                 static_cast<unsigned long long *>(hist_[nxt]), build_, total_cells_ * cw_,
                 n_zcells);
        BB_LAUNCH("pscatter_kernel");
    }
    if (prof_ != nullptr)
    {
        phase_end(prof_->partition_ms);
    }
    n_launch_ += fused ? 4 : 5;
    if (quant_ && last)
    {
        // the last level's nodes are leaves: the quantised form needs their
        // exact totals only (monotone bounds), not their histograms
        phase_begin();
        BB_CHECK(cudaMemsetAsync(btot_, 0, sizeof(int64_t) * 2 * max_front_, s));
        launch_k(pdl_, qbuilt_totals_kernel, max_bchunks_, k_threads, 0, s, ctl_, bchunks_,
                 rows_out, qgh8_, qgh16_, btot_);
        BB_LAUNCH("qbuilt_totals_kernel");
        if (red_ != nullptr)
        {
            red_->sum_u64(btot_, 2 * static_cast<size_t>(max_front_), s);
        }
        launch_k(pdl_, qsubtract_totals_kernel, front, k_threads, 0, s, ctl_, bpair_,
                 static_cast<unsigned long long const *>(hist_[cur]),
                 static_cast<unsigned long long *>(hist_[nxt]), total_cells_, 0, nodes_[cur],
                 nodes_[nxt], best_, sel_, sel_nb_, mono_, n_mono_, cfg_.tp, qscale_, btot_, cw_);
        BB_LAUNCH("qsubtract_totals_kernel");
        n_launch_ += 2;
        if (prof_ != nullptr)
        {
            phase_end(prof_->other_ms);
        }
        return;
    }
    build(rows_out, nfb, nxt, true);
    uint32_t const n_cells = off_h_[nfb]; // the built features: a selection prefix
    if (red_ != nullptr)
    {
        // the next frontier's slots (at most 2^(L+1)): the built ones carry
        // this shard's partial cells, the rest are rewritten by the subtraction
        size_t const slots = std::min<size_t>(size_t{2} << L, max_front_);
        red_->sum_u64(hist_[nxt], slots * total_cells_ * cw_, s);
    }
    phase_begin();
    if (quant_)
    {
        launch_k(pdl_, qsubtract_totals_kernel,
                 dim3(front, std::max(1u, ceil_div(n_cells * cw_, k_sub_cells))), k_threads, 0,
                 s, ctl_, bpair_, static_cast<unsigned long long const *>(hist_[cur]),
                 static_cast<unsigned long long *>(hist_[nxt]), total_cells_, n_cells, nodes_[cur],
                 nodes_[nxt], best_, sel_, sel_nb_, mono_, n_mono_, cfg_.tp, qscale_, nullptr, cw_);
        BB_LAUNCH("qsubtract_totals_kernel");
    }
    else
    {
        launch_k(pdl_, subtract_totals_kernel, front, k_threads, 0, s, ctl_, bpair_,
                 static_cast<float2 const *>(hist_[cur]), static_cast<float2 *>(hist_[nxt]),
                 total_cells_, n_cells, nodes_[cur], nodes_[nxt], best_, sel_, sel_nb_, mono_,
                 n_mono_, cfg_.tp);
        BB_LAUNCH("subtract_totals_kernel");
    }
    n_launch_ += 1;
    if (prof_ != nullptr)
    {
        phase_end(prof_->other_ms);
    }
}

void Grower::grow(float2 const *gh, uint32_t const *root_rows, uint32_t n_root,
                  TreeOut const &t, uint32_t *leaf_id, float *scores, float lr,
                  bool identity_root, NextRound const *next, RootSample const *sample)
{
    if (n_root > max_rows_)
    {
        throw ConfigError("grower: more sampled rows than the grower was sized for");
    }
    cudaStream_t s = stream_;
    gh_cur_        = gh;
    root_rows_     = root_rows;
    n_launch_      = 0;
    if (cfg_.leaf)
    {
        if (next != nullptr || red_ != nullptr || sample != nullptr)
        {
            throw ConfigError("grower: the leafwise plane takes neither a fused next round "
                              "nor row shards");
        }
        walk_ = false;
        if (quant_)
        {
            quantise(gh, static_cast<uint32_t>(plane_.n_rows), false);
        }
        grow_leafwise(root_rows, n_root, t, leaf_id, scores, lr);
        return;
    }
    if (sample != nullptr && (identity_root || red_ != nullptr))
    {
        throw ConfigError("grower: a device row sample is neither the identity root nor a "
                          "row shard");
    }
    walk_ = (sample != nullptr || (identity_root && n_root == plane_.n_rows)) &&
            (leaf_id != nullptr || scores != nullptr || next != nullptr);
    if (next != nullptr && !walk_)
    {
        throw ConfigError("grower: a fused next round needs every row as the root");
    }
    if (red_ != nullptr && (!quant_ || !walk_))
    {
        throw ConfigError("grower: a sharded fit needs the quantised form and every row as "
                          "the root");
    }
    if (quant_)
    {
        phase_begin();
        quantise(gh, static_cast<uint32_t>(plane_.n_rows), next != nullptr);
        if (prof_ != nullptr)
        {
            phase_end(prof_->other_ms);
        }
    }
    uint32_t const g_root = red_ != nullptr ? static_cast<uint32_t>(total_rows_) : n_root;
    launch_k(pdl_, root_setup_kernel, 1, k_threads, 0, s, ctl_, nodes_[0], n_root, bchunks_,
             brange_, build_, t, crows_, g_root, sample != nullptr ? sample->count : nullptr,
             heap_);
    BB_LAUNCH("root_setup_kernel");
    n_launch_ += 1;
    // the root's rows: the quantised build reads an identity list implicitly
    build(quant_ && identity_root ? nullptr : root_rows,
          cfg_.tp.max_depth == 0 ? 1 : n_sel_, 0);
    if (red_ != nullptr)
    {
        red_->sum_u64(hist_[0], total_cells_ * cw_, s);
    }
    phase_begin();
    if (quant_)
    {
        launch_k(pdl_, qroot_totals_kernel, 1, 32, 0, s, nodes_[0],
                 static_cast<unsigned long long const *>(hist_[0]), sel_nb_, cw_);
        BB_LAUNCH("qroot_totals_kernel");
    }
    else
    {
        launch_k(pdl_, root_totals_kernel, 1, 32, 0, s, nodes_[0],
                 static_cast<float2 const *>(hist_[0]), sel_nb_);
        BB_LAUNCH("root_totals_kernel");
    }
    n_launch_ += 1;
    if (prof_ != nullptr)
    {
        phase_end(prof_->other_ms);
    }
    uint32_t const *rows_in = root_rows;
    for (uint32_t L = 0; L < cfg_.tp.max_depth; ++L)
    {
        uint32_t *rows_out = rows_[L & 1];
        level(L, rows_in, rows_out, t, leaf_id, scores, lr);
        rows_in = rows_out;
    }
    phase_begin();
    int const fin = static_cast<int>(cfg_.tp.max_depth & 1);
    launch_k(pdl_, final_kernel, 1, k_plan_thr, 0, s, ctl_, nodes_[fin], cfg_.tp, t, pchunks_, pcr_,
             nbound_, HeapOut{heap_, leafmap_, cfg_.tp.max_depth, k_mirror_bytes / (plane_.u8 ? 1u : 2u)});
    BB_LAUNCH("final_kernel");
    nodes_cur_ = nodes_[fin];
    rows_cur_  = rows_in;
    if (walk_)
    {
        uint32_t const n    = static_cast<uint32_t>(plane_.n_rows);
        uint32_t const grid = std::min<uint32_t>(ceil_div(std::max<uint32_t>(n, 1), k_threads),
                                                 148u * 8u);
        uint32_t const per   = k_mirror_bytes / (plane_.u8 ? 1u : 2u);
        bool const     multi = plane_.n_feats > per;
        auto const    *mir   = static_cast<uint4 const *>(plane_.mirror);
        uint32_t const depth = cfg_.tp.max_depth;
        WalkArgs a{};
        a.scores    = scores;
        a.leaf_id   = leaf_id;
        a.lr        = lr;
        a.objective = next != nullptr ? next->objective : 0;
        a.weights   = next != nullptr ? next->weights : nullptr;
        a.labels    = next != nullptr ? next->labels : nullptr;
        a.gh        = next != nullptr ? next->gh : nullptr;
        a.absmax    = next != nullptr && quant_ ? absmax_ : nullptr;
        if (quant_)
        {
            BB_CHECK(cudaMemsetAsync(wacc_, 0, sizeof(unsigned long long) * 2 * k_walk_nodes, s));
            auto sum = [&](auto kern)
            {
                uint32_t const wgrid =
                    std::min<uint32_t>(ceil_div(std::max<uint32_t>(n, 1), k_wsum_thr), 148u * 2u);
                launch_k(pdl_, kern, wgrid, k_wsum_thr,
                         (size_t{2} << depth) * k_wsum_copies * sizeof(unsigned long long), s,
                         ctl_, mir, plane_.n_rows, heap_, leafmap_, depth, gh_cur_, absmax_,
                         leaf16_, wacc_, sample != nullptr ? sample->bits : nullptr, fix_unit_);
            };
            if (plane_.u8)
            {
                multi ? sum(walk_sum_kernel<true, true>) : sum(walk_sum_kernel<true, false>);
            }
            else
            {
                multi ? sum(walk_sum_kernel<false, true>) : sum(walk_sum_kernel<false, false>);
            }
            BB_LAUNCH("walk_sum_kernel");
            if (red_ != nullptr)
            {
                red_->sum_u64(wacc_, 2 * static_cast<size_t>(k_walk_nodes), s);
            }
            launch_k(pdl_, leaf_fix_kernel, 1, k_threads, 0, s, ctl_, t, wacc_, nbound_, absmax_,
                     cfg_.tp, fix_unit_);
            BB_LAUNCH("leaf_fix_kernel");
            if (next != nullptr)
            {
                BB_CHECK(cudaMemsetAsync(absmax_, 0, 8, s));
            }
            launch_k(pdl_, walk_apply_kernel, grid, k_threads, 0, s, ctl_, t, plane_.n_rows,
                     leaf16_, a);
            BB_LAUNCH("walk_apply_kernel");
            n_launch_ += 3;
        }
        else
        {
            auto walk = [&](auto kern)
            {
                launch_k(pdl_, kern, grid, k_threads, 0, s, ctl_, t, mir, plane_.n_rows, heap_,
                         leafmap_, depth, a);
            };
            if (plane_.u8)
            {
                multi ? walk(walk_kernel<true, true>) : walk(walk_kernel<true, false>);
            }
            else
            {
                multi ? walk(walk_kernel<false, true>) : walk(walk_kernel<false, false>);
            }
            BB_LAUNCH("walk_kernel");
            n_launch_ += 1;
        }
    }
    else
    {
        leaf_values(t, true);
        launch_k(pdl_, stamp_kernel, max_pchunks_, k_threads, 0, s, ctl_, pchunks_, nodes_[fin],
                 rows_in, t, leaf_id, scores, lr);
        BB_LAUNCH("stamp_kernel");
        n_launch_ += 1;
    }
    launch_k(pdl_, tree_counter_kernel, 1, 1, 0, s, dtree_);
    BB_LAUNCH("tree_counter_kernel");
    n_launch_ += 2;
    if (prof_ != nullptr)
    {
        phase_end(prof_->other_ms);
    }
    launches_ = n_launch_;
    ++tree_no_;
}

namespace
{

// A leaf awaiting expansion (Candidate, src/step/primitives.hpp:440-450): its
// node, its best split, its depth and the pool slot holding its histograms.

} // namespace

// LeafwiseGrower::grow with the host as the control plane: the same gain
// heap (max gain, the lower node id on a tie), child ids allocated at the
// pop, demotion when the partition empties a side (its two children stay as
// zero leaf placeholders), no children's split at the depth cap, the leaf
// budget; every pop's data plane on the device, one read-back per pop.
void Grower::grow_leafwise(uint32_t const *root_rows, uint32_t n_root, TreeOut const &t,
                           uint32_t *leaf_id, float *scores, float lr)
{
    cudaStream_t      s         = stream_;
    TreeParams const &tp        = cfg_.tp;
    size_t const      find_smem = max_nb_ * (sizeof(double2) + (sizeof(unsigned long long) * cw_));
    auto             *lout      = static_cast<LeafOut *>(lout_);
    auto             *st        = static_cast<LeafLoop *>(loop_);
    auto             *cand      = static_cast<LeafCand *>(cand_heap_);
    auto             *tdev      = static_cast<TreeOut *>(tree_dev_);
    LeafPop const    *pp        = &st->pop;
    void             *pool      = hist_[0];
    uint32_t          launches  = 0;
    BB_CHECK(cudaMemcpyAsync(rows_[0], root_rows, size_t{n_root} * 4, cudaMemcpyDeviceToDevice,
                             s));
    launch_k(pdl_, leaf_set_tree_kernel, 1, 1, 0, s, tdev, t, st, tp.max_depth > 0 ? 1u : 0u);
    BB_LAUNCH("leaf_set_tree_kernel");
    launch_k(pdl_, root_setup_kernel, 1, k_threads, 0, s, ctl_, nodes_[0], n_root, bchunks_,
             brange_, build_, t, crows_, n_root, nullptr, static_cast<uint2 *>(nullptr));
    BB_LAUNCH("root_setup_kernel");
    launches += 2;
    build(rows_[0], n_sel_, 0);
    if (quant_)
    {
        launch_k(pdl_, qroot_totals_kernel, 1, 32, 0, s, nodes_[0],
                 static_cast<unsigned long long const *>(pool), sel_nb_, cw_);
    }
    else
    {
        launch_k(pdl_, root_totals_kernel, 1, 32, 0, s, nodes_[0],
                 static_cast<float2 const *>(pool), sel_nb_);
    }
    BB_LAUNCH("root_totals_kernel");
    launches += 1;
    // each node's best split, then the pair's outcome (the children and their
    // bests) into lout; may_split: the depth cap's verdict, on the device
    auto find = [&](Node const *nodes, uint32_t const *slot_of, uint32_t const *may_split)
    {
        dim3 const fgrid(2, n_sel_);
        if (quant_)
        {
            launch_k(pdl_, qfind_warp_kernel, dim3(2, ceil_div(n_sel_, k_qfind_warps)),
                     k_qfind_warps * 32, 0, s, ctl_, nodes, pool, total_cells_, cell_off_, sel_nb_,
                     sel_, n_sel_, mono_, n_mono_, tp, cand_, qscale_, slot_of, cw_, fgroups_);
        }
        else
        {
            launch_k(pdl_, find_kernel<false>, fgrid, k_find_thr, find_smem, s, ctl_, nodes, pool,
                     total_cells_, cell_off_, sel_nb_, sel_, n_sel_, mono_, n_mono_, tp, cand_,
                     max_nb_, qscale_, slot_of, cw_, fgroups_);
        }
        BB_LAUNCH("find_kernel");
        launch_k(pdl_, leaf_best_kernel, 2, k_best_thr, 0, s, ctl_, cand_, n_sel_, nodes, lout,
                 may_split);
        BB_LAUNCH("leaf_best_kernel");
    };
    find(nodes_[0], nullptr, &st->root_may);
    launch_k(pdl_, leaf_loop_init_kernel, 1, k_plan_thr, 0, s, st, cand, leaves_, free_, lout, tdev,
             n_root, max_front_, tp.max_depth);
    BB_LAUNCH("leaf_loop_init_kernel");
    launches += 3;

    // one pop as a fixed sequence of launches, repeated by the loop graph's
    // WHILE node until leaf_commit_kernel says the heap is done; captured
    // once (the loop's buffers and the tree's device record do not move)
    if (loop_x_ == nullptr)
    {
        Profile *const saved = prof_;
        prof_                = nullptr; // no per-phase events inside the loop graph
        BB_CHECK(cudaGraphCreate(&loop_g_, 0));
        cudaGraphConditionalHandle handle{};
        BB_CHECK(cudaGraphConditionalHandleCreate(&handle, loop_g_, 1,
                                                  cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp{};
        cp.type               = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type   = cudaGraphCondTypeWhile;
        cp.conditional.size   = 1;
        cudaGraphNode_t cnode{};
        BB_CHECK(cudaGraphAddNode(&cnode, loop_g_, nullptr, 0, &cp));
        cudaGraph_t const body = cp.conditional.phGraph_out[0];
        BB_CHECK(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal));
        uint32_t const n0 = n_launch_;
        try
        {
            launch_k(pdl_, leaf_pop_kernel, 1, k_pop_thr, 0, s, st, cand, free_, tdev, plane_.cuts,
                     plane_.cut_off, sel_, tp.max_leaves, max_nodes_, tp.max_depth, ctl_, nodes_[0],
                     best_, pchunks_, pcr_);
            BB_LAUNCH("leaf_pop_kernel");
            if (plane_.u8)
            {
                launch_k(pdl_, pcount_kernel<uint8_t>, max_pchunks_, k_threads, 0, s, ctl_,
                         pchunks_, nodes_[0], best_, rows_[0], plane_.bins, plane_.n_pad, sel_,
                         sel_nb_, pleft_, dirs_);
            }
            else
            {
                launch_k(pdl_, pcount_kernel<uint16_t>, max_pchunks_, k_threads, 0, s, ctl_,
                         pchunks_, nodes_[0], best_, rows_[0], plane_.bins, plane_.n_pad, sel_,
                         sel_nb_, pleft_, dirs_);
            }
            BB_LAUNCH("pcount_kernel");
            launch_k(pdl_, leaf_plan_kernel, 1, k_plan_thr, 0, s, ctl_, pchunks_, pleft_, prbase_,
                     nleft_, dst_, build_, brange_, bbase_, bchunks_, bpair_, nodes_[0], nodes_[1],
                     slot_of_, lout, crows_, pp);
            BB_LAUNCH("leaf_plan_kernel");
            launch_k(pdl_, pscatter_kernel, max_pchunks_, k_threads, 0, s, ctl_, pchunks_,
                     nodes_[0], best_, pleft_, prbase_, nleft_, dst_, rows_[0], rows_[1], dirs_,
                     static_cast<unsigned long long *>(pool), build_, total_cells_ * cw_,
                     quant_ ? total_cells_ * cw_ : 0);
            BB_LAUNCH("pscatter_kernel");
            n_launch_ = 0;
            build(rows_[1], n_sel_, 0, true);
            uint32_t const nb = n_launch_;
            launch_k(pdl_, leaf_copyback_kernel, 148u * 8u, 256, 0, s, lout, rows_[1], rows_[0], pp);
            BB_LAUNCH("leaf_copyback_kernel");
            uint32_t const sgrid =
                std::max(1u, std::min(ceil_div(total_cells_ * cw_, 256), 148u * 8u));
            if (quant_)
            {
                launch_k(pdl_, leaf_sub_kernel<true>, sgrid, 256, 0, s, lout, bpair_, pool,
                         total_cells_ * cw_, total_cells_ * cw_);
                launch_k(pdl_, leaf_totals_kernel<true>, 1, 64, 0, s, ctl_, lout, nodes_[1],
                         slot_of_, pool, total_cells_, sel_, sel_nb_, mono_, n_mono_, tp, qscale_,
                         pp, cw_, fgroups_);
            }
            else
            {
                launch_k(pdl_, leaf_sub_kernel<false>, sgrid, 256, 0, s, lout, bpair_, pool,
                         total_cells_, total_cells_);
                launch_k(pdl_, leaf_totals_kernel<false>, 1, 64, 0, s, ctl_, lout, nodes_[1],
                         slot_of_, pool, total_cells_, sel_, sel_nb_, mono_, n_mono_, tp, qscale_,
                         pp, 1, fgroups_);
            }
            BB_LAUNCH("leaf_totals_kernel");
            find(nodes_[1], slot_of_, &st->may_split);
            launch_k(pdl_, leaf_commit_kernel, 1, 1, 0, s, st, cand, leaves_, free_, lout, tdev,
                     tp.max_leaves, 4 * max_front_ + 8, handle);
            BB_LAUNCH("leaf_commit_kernel");
            // pop, count, plan, scatter, the build, copy-back, subtraction,
            // totals, find, best, commit
            body_launches_ = 4 + nb + 3 + 2 + 1;
        }
        catch (...)
        {
            cudaGraph_t dummy{};
            cudaStreamEndCapture(s, &dummy);
            prof_     = saved;
            n_launch_ = n0;
            throw;
        }
        cudaGraph_t captured{};
        BB_CHECK(cudaStreamEndCapture(s, &captured));
        BB_CHECK(cudaGraphInstantiate(&loop_x_, loop_g_, 0));
        prof_     = saved;
        n_launch_ = n0;
    }
    if (prof_ != nullptr)
    {
        phase_begin();
    }
    BB_CHECK(cudaGraphLaunch(loop_x_, s));
    if (prof_ != nullptr)
    {
        phase_end(prof_->other_ms);
    }
    launch_k(pdl_, leaf_loop_end_kernel, 1, k_plan_thr, 0, s, st, cand, leaves_, nodes_[0], ctl_);
    BB_LAUNCH("leaf_loop_end_kernel");
    launches += 1;
    // write_leaf for every leaf, then (quantised) the FP64 renewal, then the
    // rows' leaf ids and score updates from the leaves' segments
    launch_k(pdl_, final_kernel, 1, k_plan_thr, 0, s, ctl_, nodes_[0], tp, t, pchunks_, pcr_,
             nbound_, HeapOut{nullptr, nullptr, 0, 1});
    BB_LAUNCH("final_kernel");
    launches += 1;
    nodes_cur_ = nodes_[0];
    rows_cur_  = rows_[0];
    uint32_t const before = n_launch_;
    leaf_values(t, true);
    launches += n_launch_ - before;
    launch_k(pdl_, stamp_kernel, max_pchunks_, k_threads, 0, s, ctl_, pchunks_, nodes_[0], rows_[0],
             t, leaf_id, scores, lr);
    BB_LAUNCH("stamp_kernel");
    launch_k(pdl_, tree_counter_kernel, 1, 1, 0, s, dtree_);
    BB_LAUNCH("tree_counter_kernel");
    launches += 2;
    // the loop's verdict: a full node table or pool is the reference's
    // capacity refusal
    auto *lh = static_cast<LeafLoop *>(lout_h_);
    BB_CHECK(cudaMemcpyAsync(lh, st, sizeof(LeafLoop), cudaMemcpyDeviceToHost, s));
    BB_CHECK(cudaStreamSynchronize(s));
    if (lh->error == 1)
    {
        throw ConfigError("grower: leafwise tree outgrew its node table");
    }
    if (lh->error == 2)
    {
        throw ConfigError("grower: leafwise histogram pool exhausted");
    }
    if (lh->error == 3)
    {
        throw std::runtime_error("grower: leafwise pop loop exceeded its pop bound");
    }
    // every pop ran the body, and the last iteration found nothing to pop
    // (or stopped at the budget) -- one graph launch on the host's side
    n_launch_ += launches + (lh->pops + (lh->noop != 0 ? 1 : 0)) * body_launches_;
    launches_ = n_launch_;
    ++tree_no_;
}

void Grower::populate(float2 const *gh, uint32_t const *rows, uint32_t n, double2 *out)
{
    cudaStream_t s = stream_;
    gh_cur_        = gh;
    root_rows_     = rows;
    TreeOut t{};
    std::vector<uint32_t> meta_dummy(3);
    // a tree output the setup kernel may write node 0 into
    uint32_t *scratch = dalloc<uint32_t>(64, s);
    t.feature = t.left = t.right = t.split_bin = t.meta = scratch;
    t.value = t.gain = t.cover = reinterpret_cast<float *>(scratch + 16);
    t.default_left = reinterpret_cast<uint8_t *>(scratch + 32);
    if (quant_)
    {
        quantise(gh, static_cast<uint32_t>(plane_.n_rows), false);
    }
    walk_ = false;
    launch_k(pdl_, root_setup_kernel, 1, k_threads, 0, s, ctl_, nodes_[0], n, bchunks_, brange_,
             build_, t, crows_, n, nullptr, heap_);
    BB_LAUNCH("root_setup_kernel");
    build(rows, n_sel_, 0);
    std::vector<double2> cells(total_cells_);
    if (quant_)
    {
        std::vector<unsigned long long> q(static_cast<size_t>(total_cells_) * cw_);
        double2                         sc{};
        BB_CHECK(cudaMemcpyAsync(q.data(), hist_[0], q.size() * 8ULL, cudaMemcpyDeviceToHost, s));
        BB_CHECK(cudaMemcpyAsync(&sc, qscale_, sizeof(double2), cudaMemcpyDeviceToHost, s));
        BB_CHECK(cudaStreamSynchronize(s));
        for (uint32_t x = 0; x < total_cells_; ++x)
        {
            int64_t const g = cw_ == 2 ? static_cast<int64_t>(q[2 * x])
                                       : static_cast<int32_t>(static_cast<uint32_t>(q[x] >> 32));
            int64_t const h = cw_ == 2 ? static_cast<int64_t>(q[(2 * x) + 1])
                                       : static_cast<int64_t>(static_cast<uint32_t>(q[x]));
            out[x] = make_double2(static_cast<double>(g) * sc.x, static_cast<double>(h) * sc.y);
        }
    }
    else
    {
        std::vector<float2> f(total_cells_);
        BB_CHECK(cudaMemcpyAsync(f.data(), hist_[0], total_cells_ * 8ULL, cudaMemcpyDeviceToHost, s));
        BB_CHECK(cudaStreamSynchronize(s));
        for (uint32_t x = 0; x < total_cells_; ++x)
        {
            out[x] = make_double2(f[x].x, f[x].y);
        }
    }
    BB_CHECK(cudaFreeAsync(scratch, s));
    BB_CHECK(cudaStreamSynchronize(s));
}

void Grower::set_interaction(std::vector<uint64_t> const &fgroups)
{
    if (fgroups_ != nullptr)
    {
        BB_CHECK(cudaFreeAsync(fgroups_, stream_));
        fgroups_ = nullptr;
    }
    if (fgroups.empty())
    {
        return;
    }
    if (cfg_.level)
    {
        // ObliviousGrower refuses them (src/grower_impl.hpp:591-595)
        throw ConfigError("interaction_constraints are not supported by the levelwise grower");
    }
    if (fgroups.size() != plane_.n_feats)
    {
        throw std::invalid_argument("grower: one interaction mask per feature");
    }
    BB_CHECK(cudaMallocAsync(reinterpret_cast<void **>(&fgroups_), fgroups.size() * 8, stream_));
    BB_CHECK(cudaMemcpyAsync(fgroups_, fgroups.data(), fgroups.size() * 8, cudaMemcpyHostToDevice,
                             stream_));
    BB_CHECK(cudaStreamSynchronize(stream_));
}

void Grower::set_monotone(std::vector<int8_t> const &m)
{
    if (mono_ != nullptr)
    {
        BB_CHECK(cudaFreeAsync(mono_, stream_));
        mono_ = nullptr;
    }
    n_mono_ = static_cast<uint32_t>(m.size());
    if (m.empty())
    {
        return;
    }
    BB_CHECK(cudaMallocAsync(reinterpret_cast<void **>(&mono_), m.size(), stream_));
    BB_CHECK(cudaMemcpyAsync(mono_, m.data(), m.size(), cudaMemcpyHostToDevice, stream_));
    BB_CHECK(cudaStreamSynchronize(stream_));
}

} // namespace bb
