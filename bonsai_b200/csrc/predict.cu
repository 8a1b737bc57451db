// Ensemble predict: bb_predict_plan_* (pack once, run many) and bb_predict
// (pack, run, release in one call).
//
// The reference packs the ensemble into SoA node tables once
// (cuda_predict_plan, src/cuda/predict.cu:147-196) and walks it with one
// thread per row over every tree, the nodes read from global memory
// (predict_walk_kernel, src/cuda/predict.cu:51-85). Its contract is bit
// equality with the host walk predict_at_binned (include/bonsai/booster.hpp:
// 831-845): each row's leaves summed in float in tree order, then
// init + lr * sum, nothing fused.
//
// Here the ensemble is re-laid for the device as complete binary heaps
// ("heap form"): every tree padded to the ensemble's depth D, a leaf above
// depth D standing in for its whole subtree (its node routes every row left,
// its left descendants repeat it). The root is slot 1 and slot n's children
// are 2n and 2n + 1, so a walk is D unrolled steps with no child tables and
// no exit test, ending on a leaf slot in [2^D, 2^(D+1)). A node is one
// 4-byte word: the byte offset of its feature's code in the row's staged
// codes, and a threshold; the row goes right iff code >= threshold. The
// missing-bin rule of routes_left (include/bonsai/dataset.hpp:234-238)
// becomes the choice of which of two staged variants of the code the node
// reads (the heap node comment below).
//
// Kernel: a CTA stages 1,024 rows' codes (both variants) from the plane's
// row-major mirror into shared memory, word-interleaved by lane so that
// every lane's code load hits its own bank whatever feature it reads, then
// streams the heaps through shared memory in 16 KB chunks; each of 512
// threads walks 2 rows per tree, addressing the heap by shared-window byte
// address (from p = base + 4n the child is 2p - base (+4)). A grid of one
// resident wave splits the rows evenly, so no SM idles in a tail. Small
// batches, which cannot fill the GPU with rows, split the trees across CTAs
// too: each (row, tree) leaf value goes to a workspace and a second kernel
// sums every row's values in tree order, so the scores stay bit-identical.
// Ensembles deeper than 10 or planes wider than 8 mirror tiles (256 u8 / 128
// u16 features) use the node form: the reference's layout and walk, nodes in
// global memory.
#include "bonsai_b200.h"
#include "ingest.cuh"

#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
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

constexpr uint32_t k_max_heap_depth = 10;
constexpr uint32_t k_max_heap_tiles = 8;
constexpr uint32_t k_chunk_bytes    = 16384;
constexpr uint32_t k_sms            = 148;
constexpr size_t   k_max_vals_bytes = size_t{256} << 20;

void need(bool ok, char const *what)
{
    if (!ok)
    {
        throw std::invalid_argument(what);
    }
}

template <typename F> int guarded(F &&f)
{
    try
    {
        f();
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

// ---- heap form ---------------------------------------------------------------

// A heap node: off << 16 | thr. The row's code for the node's feature, in
// the variant its default direction needs, sits at byte off of the row's
// staged codes; the row goes right iff code >= thr. A leaf slot holds the
// leaf value's bits.
//
// Two variants of every code are staged. v1 is the code itself: the missing
// (last) bin is the largest code, so with default_left false "code > split
// or missing" is code >= split + 1. v0 maps the missing bin to 0 and every
// other code c to c + 1: with default_left true "code > split and not
// missing" is v0 >= split + 2. No code reaches the threshold 256 (u8) or
// 65535 (u16), which routes a node left: an always-left pad, or a split that
// sends nothing right.

// The v0 word of a staged v1 word: per code lane, 0 where the code is its
// feature's last bin, else code + 1 (no lane overflows: a non-missing code is
// at most 254, or 65533 for u16).
__device__ __forceinline__ uint32_t missing_low(uint32_t c, uint32_t last, bool u8)
{
    uint32_t const keep = ~(u8 ? __vcmpeq4(c, last) : __vcmpeq2(c, last));
    return (c & keep) + ((u8 ? 0x01010101u : 0x00010001u) & keep);
}

__device__ __forceinline__ uint32_t lds_u32(uint32_t a)
{
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
}

template <typename CodeT> __device__ __forceinline__ uint32_t lds_code(uint32_t a)
{
    uint32_t v;
    if constexpr (sizeof(CodeT) == 1)
    {
        asm volatile("ld.shared.u8 %0, [%1];" : "=r"(v) : "r"(a));
    }
    else
    {
        asm volatile("ld.shared.u16 %0, [%1];" : "=r"(v) : "r"(a));
    }
    return v;
}

// Scores of rows [blockIdx.x * rows_per_cta, + rows_per_cta) over trees
// [blockIdx.y * trees_per_split, + trees_per_split), taken T x R rows at a
// time. vals == nullptr: out[r] = init + lr * sum (blockIdx.y is 0 and the
// split holds every tree); else every (tree, row) leaf value into
// vals[t * n_rows + r].
template <typename CodeT, uint32_t D, uint32_t T, uint32_t R>
__global__ void __launch_bounds__(T)
    heap_predict_kernel(uint4 const *__restrict__ mirror, uint64_t n_rows, uint32_t n_tiles,
                        uint32_t const *__restrict__ last_words,
                        uint32_t const *__restrict__ heaps, uint32_t n_trees,
                        uint32_t trees_per_split, uint32_t chunk_trees, uint32_t rows_per_cta,
                        float lr, float init, float *__restrict__ out,
                        float *__restrict__ vals)
{
    constexpr uint32_t slots = 2u << D; // per tree: root at 1, leaves at [2^D, 2^(D+1))
    constexpr uint32_t warps = T / 32;
    constexpr bool     u8    = sizeof(CodeT) == 1;
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t const words  = n_tiles * 8;     // v1 words per row; v0 follows
    uint32_t const lane   = threadIdx.x & 31u;
    uint32_t const warp   = threadIdx.x >> 5;
    auto *const    codes  = smem;
    auto *const    heap_s = reinterpret_cast<uint32_t *>(
        smem + (static_cast<size_t>(T) * R * words * 8));
    uint32_t const codes_a =
        static_cast<uint32_t>(__cvta_generic_to_shared(codes));
    uint32_t const heap_a = static_cast<uint32_t>(__cvta_generic_to_shared(heap_s));
    uint64_t const begin = static_cast<uint64_t>(blockIdx.x) * rows_per_cta;
    uint64_t const end   = min(n_rows, begin + rows_per_cta);
    uint32_t const t0    = blockIdx.y * trees_per_split;
    uint32_t const t1    = min(n_trees, t0 + trees_per_split);

    for (uint64_t row0 = begin; row0 < end; row0 += T * R)
    {
        // this thread's rows: slot s = warp + 8k holds 32 consecutive rows;
        // word j of a row in lane l sits at word (s * 2 words + j) * 32 + l
        uint64_t row[R];
        uint32_t base[R];
        __syncthreads(); // the previous pass's walks are done with the codes
#pragma unroll
        for (uint32_t k = 0; k < R; ++k)
        {
            uint32_t const s = warp + (warps * k);
            row[k]           = row0 + (s * 32u) + lane;
            base[k]          = codes_a + (((s * words * 64u) + lane) * 4u);
            auto *cw = reinterpret_cast<uint32_t *>(codes) + (s * words * 64u) + lane;
            for (uint32_t t = 0; t < n_tiles; ++t)
            {
                uint4 x = make_uint4(0, 0, 0, 0);
                uint4 y = make_uint4(0, 0, 0, 0);
                if (row[k] < end)
                {
                    uint4 const *src =
                        mirror + (((static_cast<uint64_t>(t) * n_rows) + row[k]) * 2);
                    x = src[0];
                    y = src[1];
                }
                uint32_t const w[8] = {x.x, x.y, x.z, x.w, y.x, y.y, y.z, y.w};
#pragma unroll
                for (uint32_t j = 0; j < 8; ++j)
                {
                    uint32_t const wd = (t * 8u) + j;
                    cw[wd * 32u]           = w[j];
                    cw[(words + wd) * 32u] = missing_low(w[j], last_words[wd], u8);
                }
            }
        }
        float acc[R];
#pragma unroll
        for (uint32_t k = 0; k < R; ++k)
        {
            acc[k] = 0.0F;
        }
        for (uint32_t c0 = t0; c0 < t1; c0 += chunk_trees)
        {
            uint32_t const nc = min(chunk_trees, t1 - c0);
            __syncthreads(); // codes staged; the previous chunk's walks done
            {
                auto const *src =
                    reinterpret_cast<uint4 const *>(heaps + (static_cast<size_t>(c0) * slots));
                auto          *dst = reinterpret_cast<uint4 *>(heap_s);
                uint32_t const n16 = nc * slots / 4u;
                for (uint32_t i = threadIdx.x; i < n16; i += T)
                {
                    dst[i] = src[i];
                }
            }
            __syncthreads();
            for (uint32_t j = 0; j < nc; ++j)
            {
                // byte addresses in the shared window: slot i of this tree
                // at tb + 4i; from p = tb + 4n the child 2n (+1) is
                // 2p - tb (+4)
                uint32_t const tb = heap_a + (j * slots * 4u);
                uint32_t const cl = 0u - tb;
                uint32_t const cr = 4u - tb;
                uint32_t p[R];
#pragma unroll
                for (uint32_t k = 0; k < R; ++k)
                {
                    p[k] = tb + 4u;
                }
#pragma unroll
                for (uint32_t d = 0; d < D; ++d)
                {
#pragma unroll
                    for (uint32_t k = 0; k < R; ++k)
                    {
                        uint32_t const e    = lds_u32(p[k]);
                        uint32_t const code = lds_code<CodeT>(base[k] + (e >> 16));
                        p[k] = (2u * p[k]) + (code >= (e & 0xFFFFu) ? cr : cl);
                    }
                }
#pragma unroll
                for (uint32_t k = 0; k < R; ++k)
                {
                    float const v = __uint_as_float(lds_u32(p[k]));
                    if (vals == nullptr)
                    {
                        acc[k] = acc[k] + v;
                    }
                    else if (row[k] < end)
                    {
                        vals[(static_cast<uint64_t>(c0 + j) * n_rows) + row[k]] = v;
                    }
                }
            }
        }
        if (vals == nullptr)
        {
#pragma unroll
            for (uint32_t k = 0; k < R; ++k)
            {
                if (row[k] < end)
                {
                    out[row[k]] = __fadd_rn(init, __fmul_rn(acc[k], lr));
                }
            }
        }
    }
}

// Every row's leaf values summed in tree order: one thread per row.
__global__ void sum_rows_kernel(float const *__restrict__ vals, uint64_t n_rows, uint32_t n_trees,
                                float lr, float init, float *__restrict__ out)
{
    uint64_t const r = (static_cast<uint64_t>(blockIdx.x) * blockDim.x) + threadIdx.x;
    if (r >= n_rows)
    {
        return;
    }
    float acc = 0.0F;
#pragma unroll 8
    for (uint32_t t = 0; t < n_trees; ++t)
    {
        acc = acc + vals[(static_cast<uint64_t>(t) * n_rows) + r];
    }
    out[r] = __fadd_rn(init, __fmul_rn(acc, lr));
}

// The same sum with one warp per row, for batches too small to fill the GPU
// with rows: lanes load 32 trees' values at once, every lane adds them in
// order from the shuffles.
__global__ void sum_warp_kernel(float const *__restrict__ vals, uint64_t n_rows, uint32_t n_trees,
                                float lr, float init, float *__restrict__ out)
{
    uint64_t const r    = ((static_cast<uint64_t>(blockIdx.x) * blockDim.x) + threadIdx.x) >> 5;
    uint32_t const lane = threadIdx.x & 31u;
    if (r >= n_rows)
    {
        return;
    }
    float acc = 0.0F;
    for (uint32_t t0 = 0; t0 < n_trees; t0 += 32)
    {
        uint32_t const m = min(32u, n_trees - t0);
        float const    v = lane < m ? vals[(static_cast<uint64_t>(t0 + lane) * n_rows) + r] : 0.0F;
        for (uint32_t j = 0; j < m; ++j)
        {
            acc = acc + __shfl_sync(0xFFFFFFFFu, v, static_cast<int>(j));
        }
    }
    if (lane == 0)
    {
        out[r] = __fadd_rn(init, __fmul_rn(acc, lr));
    }
}

// ---- node form (deep trees, wide planes) ---------------------------------------

// One thread per row, every tree in order: the bin-space walk of
// routes_left over tree-local child ids, nodes in global memory.
template <typename BinT>
__global__ void node_predict_kernel(BinT const *__restrict__ bins, uint64_t n_pad, uint64_t n,
                                    uint32_t const *__restrict__ last_bin, uint32_t n_trees,
                                    uint32_t const *__restrict__ roots,
                                    uint32_t const *__restrict__ feature,
                                    uint32_t const *__restrict__ split_bin,
                                    uint32_t const *__restrict__ left,
                                    uint32_t const *__restrict__ right,
                                    uint8_t const *__restrict__ dl,
                                    float const *__restrict__ value, float lr, float init,
                                    float *__restrict__ out)
{
    uint64_t const r = (static_cast<uint64_t>(blockIdx.x) * blockDim.x) + threadIdx.x;
    if (r >= n)
    {
        return;
    }
    float acc = 0.0F;
    for (uint32_t t = 0; t < n_trees; ++t)
    {
        uint32_t const base = roots[t];
        uint32_t       idx  = base;
        while (feature[idx] != k_leaf_flag)
        {
            uint32_t const f = feature[idx];
            uint32_t const b = bins[(static_cast<uint64_t>(f) * n_pad) + r];
            idx = base + (routes_left(b, last_bin[f], split_bin[idx], dl[idx] != 0) ? left[idx]
                                                                                   : right[idx]);
        }
        acc = acc + value[idx];
    }
    out[r] = __fadd_rn(init, __fmul_rn(acc, lr));
}

// ---- host packing ---------------------------------------------------------------

} // namespace

// A device buffer released with its owner.
struct DeviceBuf
{
    void *p = nullptr;
    DeviceBuf() = default;
    DeviceBuf(DeviceBuf const &) = delete;
    DeviceBuf &operator=(DeviceBuf const &) = delete;
    ~DeviceBuf()
    {
        if (p != nullptr)
        {
            cudaFree(p);
        }
    }
    void upload(void const *src, size_t bytes)
    {
        check(cudaMalloc(&p, std::max<size_t>(bytes, 16)), "cudaMalloc");
        check(cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy");
    }
    template <typename T> T *as() const
    {
        return static_cast<T *>(p);
    }
};

} // namespace bb

struct bb_predict_plan
{
    // the plane shape the ensemble was packed for
    uint32_t              n_feats = 0;
    bool                  u8      = true;
    std::vector<uint32_t> cut_off;
    uint32_t              n_trees = 0;
    float                 lr      = 0.0F;
    float                 init    = 0.0F;
    // heap form (depth > 0) or node form (depth == 0)
    uint32_t    depth   = 0;
    uint32_t    n_tiles = 0;
    bb::DeviceBuf heaps;
    bb::DeviceBuf last_words; // per staged code word, its features' last bins
    bb::DeviceBuf last, roots, feature, split, left, right, dl, value;
    // per-run workspace, grown on demand; runs through one plan serialise
    std::mutex   mu;
    float       *vals     = nullptr;
    size_t       vals_cap = 0;
    float       *out      = nullptr;
    size_t       out_cap  = 0;
    cudaStream_t stream   = nullptr;
    ~bb_predict_plan()
    {
        if (vals != nullptr)
        {
            cudaFree(vals);
        }
        if (out != nullptr)
        {
            cudaFree(out);
        }
        if (stream != nullptr)
        {
            cudaStreamDestroy(stream);
        }
    }
};

namespace bb
{
namespace
{

void validate_trees(Plane const &p, uint32_t n_trees, uint32_t const *roots, uint32_t n_nodes,
                    uint32_t const *feature, uint32_t const *left, uint32_t const *right)
{
    // every walk must end: children lie after their parent inside the tree,
    // and split features exist
    for (uint32_t t = 0; t < n_trees; ++t)
    {
        uint32_t const b = roots[t];
        uint32_t const e = t + 1 < n_trees ? roots[t + 1] : n_nodes;
        need(b < e && e <= n_nodes, "bb_predict: bad tree roots");
        for (uint32_t i = b; i < e; ++i)
        {
            if (feature[i] == k_leaf_flag)
            {
                continue;
            }
            need(feature[i] < p.n_feats, "bb_predict: node feature out of range");
            need(left[i] > i - b && right[i] > i - b && b + left[i] < e && b + right[i] < e,
                 "bb_predict: a child id must follow its parent in its tree");
        }
    }
}

// Longest root-to-leaf path of tree [b, e) (children follow parents, so one
// pass in id order settles every node's depth).
uint32_t tree_depth(uint32_t b, uint32_t e, uint32_t const *feature, uint32_t const *left,
                    uint32_t const *right)
{
    std::vector<uint32_t> d(e - b, 0);
    uint32_t              deepest = 0;
    for (uint32_t i = 0; i < e - b; ++i)
    {
        deepest = std::max(deepest, d[i]);
        if (feature[b + i] != k_leaf_flag)
        {
            d[left[b + i]]  = std::max(d[left[b + i]], d[i] + 1);
            d[right[b + i]] = std::max(d[right[b + i]], d[i] + 1);
        }
    }
    return deepest;
}

// One tree into its heap: node thresholds and code offsets for a plane of
// u8 (or u16) codes with `words` staged v1 words per row.
struct HeapPacker
{
    uint32_t        D;
    bool            u8;
    uint32_t        words;
    uint32_t const *cut_off;
    uint32_t const *feature;
    uint32_t const *split;
    uint32_t const *left;
    uint32_t const *right;
    uint8_t const  *dl;
    float const    *value;

    uint32_t never() const
    {
        return u8 ? 256u : 65535u;
    }
    // Byte offset of feature f's code in the staged row, variant v1 or v0.
    uint32_t code_offset(uint32_t f, bool v0) const
    {
        uint32_t const wd = u8 ? f >> 2 : f >> 1;
        uint32_t const b  = u8 ? f & 3u : (f & 1u) * 2u;
        return (((v0 ? words : 0u) + wd) * 128u) + b;
    }
    // routes_left(code, last, split, dl) == !(variant code >= thr).
    uint32_t route(uint32_t f, uint32_t split_bin, bool default_left, uint32_t last) const
    {
        if (split_bin >= last)
        {
            // only the missing bin can go right, and only with default_left false
            return default_left ? never() : (code_offset(f, false) << 16) | last;
        }
        if (default_left)
        {
            return (code_offset(f, true) << 16) | (split_bin + 2);
        }
        return (code_offset(f, false) << 16) | (split_bin + 1);
    }
    static uint32_t leaf_slot(float v)
    {
        uint32_t u = 0;
        std::memcpy(&u, &v, 4);
        return u;
    }
    // Node i (global id; b its tree's first) into heap slot h at depth d.
    void fill(uint32_t *heap, uint32_t b, uint32_t i, uint32_t h, uint32_t d) const
    {
        if (d == D)
        {
            heap[h] = leaf_slot(value[i]);
            return;
        }
        if (feature[i] == k_leaf_flag)
        {
            // a leaf above depth D: route everything left, repeat it below
            heap[h] = never();
            fill(heap, b, i, 2 * h, d + 1);
            fill(heap, b, i, (2 * h) + 1, d + 1);
            return;
        }
        uint32_t const f = feature[i];
        heap[h] = route(f, split[i], dl[i] != 0, cut_off[f + 1] - cut_off[f] - 1);
        fill(heap, b, b + left[i], 2 * h, d + 1);
        fill(heap, b, b + right[i], (2 * h) + 1, d + 1);
    }
};

void plan_check_plane(bb_predict_plan const &pl, Plane const &p)
{
    need(p.n_feats == pl.n_feats && p.u8 == pl.u8,
         "bb_predict_plan: the plane's shape differs from the plan's");
    need(std::equal(pl.cut_off.begin(), pl.cut_off.end(), p.h_cut_off),
         "bb_predict_plan: the plane's bin counts differ from the plan's");
}

template <typename F> void set_smem(F *kern, size_t smem)
{
    check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem)),
          "cudaFuncSetAttribute");
}

using HeapFn = void (*)(uint4 const *, uint64_t, uint32_t, uint32_t const *, uint32_t const *,
                        uint32_t, uint32_t, uint32_t, uint32_t, float, float, float *, float *);

// The kernel shapes: 256 threads x 1 row per pass (small batches, trees
// split across CTAs) and 512 threads x 2 rows (1,024 rows per pass).
template <typename CodeT, uint32_t D> HeapFn heap_fn_r(uint32_t T, uint32_t R)
{
    if (T == 512 && R == 2)
    {
        return heap_predict_kernel<CodeT, D, 512, 2>;
    }
    return heap_predict_kernel<CodeT, D, 256, 1>;
}

template <typename CodeT> HeapFn heap_fn_d(uint32_t D, uint32_t T, uint32_t R)
{
    switch (D)
    {
    case 1: return heap_fn_r<CodeT, 1>(T, R);
    case 2: return heap_fn_r<CodeT, 2>(T, R);
    case 3: return heap_fn_r<CodeT, 3>(T, R);
    case 4: return heap_fn_r<CodeT, 4>(T, R);
    case 5: return heap_fn_r<CodeT, 5>(T, R);
    case 6: return heap_fn_r<CodeT, 6>(T, R);
    case 7: return heap_fn_r<CodeT, 7>(T, R);
    case 8: return heap_fn_r<CodeT, 8>(T, R);
    case 9: return heap_fn_r<CodeT, 9>(T, R);
    case 10: return heap_fn_r<CodeT, 10>(T, R);
    default: throw std::logic_error("bb_predict_plan: heap depth out of range");
    }
}

uint32_t sm_count()
{
    int dev = 0;
    int n   = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    check(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
    return static_cast<uint32_t>(std::max(n, 1));
}

// Enqueues the scores of the plan's first n_trees trees over plane p into
// out (device, n_rows floats) on stream s. Returns the kernel launches made.
uint32_t plan_launch(bb_predict_plan &pl, Plane const &p, uint32_t n_trees, float *out,
                     cudaStream_t s)
{
    uint64_t const n = p.n_rows;
    if (n == 0)
    {
        return 0; // an empty request plane: nothing to score
    }
    if (pl.depth == 0)
    {
        if (p.u8)
        {
            node_predict_kernel<uint8_t><<<ceil_div(n, 256), 256, 0, s>>>(
                static_cast<uint8_t const *>(p.bins), p.n_pad, n, pl.last.as<uint32_t>(),
                n_trees, pl.roots.as<uint32_t>(), pl.feature.as<uint32_t>(),
                pl.split.as<uint32_t>(), pl.left.as<uint32_t>(), pl.right.as<uint32_t>(),
                pl.dl.as<uint8_t>(), pl.value.as<float>(), pl.lr, pl.init, out);
        }
        else
        {
            node_predict_kernel<uint16_t><<<ceil_div(n, 256), 256, 0, s>>>(
                static_cast<uint16_t const *>(p.bins), p.n_pad, n, pl.last.as<uint32_t>(),
                n_trees, pl.roots.as<uint32_t>(), pl.feature.as<uint32_t>(),
                pl.split.as<uint32_t>(), pl.left.as<uint32_t>(), pl.right.as<uint32_t>(),
                pl.dl.as<uint8_t>(), pl.value.as<float>(), pl.lr, pl.init, out);
        }
        BB_LAUNCH("node_predict_kernel");
        return 1;
    }
    uint32_t const tree_bytes = (2u << pl.depth) * 4u;
    uint32_t const chunk      = std::max(1u, k_chunk_bytes / tree_bytes);
    uint32_t const sms        = sm_count();
    size_t const   vals_bytes = n * static_cast<size_t>(n_trees) * 4;
    // both code variants of a row: 64 bytes per mirror tile
    size_t const   row_bytes  = static_cast<size_t>(pl.n_tiles) * 64;
    bool const     split_mode = ceil_div(n, 256) < sms && vals_bytes <= k_max_vals_bytes;
    uint32_t       T          = 256;
    uint32_t       R          = 1;
    if (!split_mode)
    {
        T = 512;
        R = 2;
    }
    size_t const smem = (static_cast<size_t>(T) * R * row_bytes) +
                        (static_cast<size_t>(chunk) * tree_bytes);
    HeapFn const fn   = pl.u8 ? heap_fn_d<uint8_t>(pl.depth, T, R)
                              : heap_fn_d<uint16_t>(pl.depth, T, R);
    set_smem(fn, smem);
    uint32_t rows_per_cta = T * R;
    uint32_t splits       = 1;
    uint32_t tps          = n_trees;
    dim3     grid;
    if (split_mode)
    {
        // few rows: the trees split across CTAs too, every leaf value kept
        uint32_t const row_blks = ceil_div(n, rows_per_cta);
        uint32_t const n_chunks = ceil_div(n_trees, chunk);
        splits = std::min(ceil_div(2 * sms, row_blks), n_chunks);
        tps    = ceil_div(ceil_div(n_trees, splits), chunk) * chunk;
        splits = ceil_div(n_trees, tps);
        grid   = dim3(row_blks, splits);
    }
    else
    {
        // one wave of resident CTAs, each over an equal run of rows
        int occ = 0;
        check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, static_cast<int>(T), smem),
              "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        uint64_t const ctas = static_cast<uint64_t>(std::max(occ, 1)) * sms;
        uint64_t const per  = std::max<uint64_t>(32, ((((n + ctas - 1) / ctas) + 31) / 32) * 32);
        rows_per_cta        = static_cast<uint32_t>(per);
        grid                = dim3(ceil_div(n, per), 1);
    }
    float *vals = nullptr;
    if (splits > 1)
    {
        if (pl.vals_cap < vals_bytes)
        {
            if (pl.vals != nullptr)
            {
                check(cudaFree(pl.vals), "cudaFree");
                pl.vals     = nullptr;
                pl.vals_cap = 0;
            }
            check(cudaMalloc(&pl.vals, vals_bytes), "cudaMalloc");
            pl.vals_cap = vals_bytes;
        }
        vals = pl.vals;
    }
    fn<<<grid, T, smem, s>>>(static_cast<uint4 const *>(p.mirror), n, pl.n_tiles,
                                          pl.last_words.as<uint32_t>(), pl.heaps.as<uint32_t>(),
                                          n_trees, tps, chunk, rows_per_cta, pl.lr, pl.init, out,
                                          vals);
    BB_LAUNCH("heap_predict_kernel");
    if (splits == 1)
    {
        return 1;
    }
    if (n < 4096)
    {
        sum_warp_kernel<<<ceil_div(n * 32, 256), 256, 0, s>>>(vals, n, n_trees, pl.lr, pl.init,
                                                              out);
    }
    else
    {
        sum_rows_kernel<<<ceil_div(n, 256), 256, 0, s>>>(vals, n, n_trees, pl.lr, pl.init, out);
    }
    BB_LAUNCH("predict sum kernel");
    return 2;
}

std::unique_ptr<bb_predict_plan> make_plan(Plane const &p, uint32_t n_trees,
                                           uint32_t const *roots, uint32_t n_nodes,
                                           uint32_t const *feature, uint32_t const *split_bin,
                                           uint32_t const *left, uint32_t const *right,
                                           uint8_t const *default_left, float const *value,
                                           float lr, float init)
{
    need(roots != nullptr && feature != nullptr && split_bin != nullptr && left != nullptr &&
             right != nullptr && default_left != nullptr && value != nullptr,
         "bb_predict_plan_create: null argument");
    need(n_trees > 0 && n_nodes > 0, "bb_predict_plan_create: empty ensemble");
    validate_trees(p, n_trees, roots, n_nodes, feature, left, right);
    auto pl     = std::make_unique<bb_predict_plan>();
    pl->n_feats = p.n_feats;
    pl->u8      = p.u8;
    pl->cut_off.assign(p.h_cut_off, p.h_cut_off + p.n_feats + 1);
    pl->n_trees = n_trees;
    pl->lr      = lr;
    pl->init    = init;
    uint32_t D  = 1;
    for (uint32_t t = 0; t < n_trees; ++t)
    {
        uint32_t const e = t + 1 < n_trees ? roots[t + 1] : n_nodes;
        D = std::max(D, tree_depth(roots[t], e, feature, left, right));
    }
    uint32_t const per     = k_mirror_bytes / (p.u8 ? 1u : 2u);
    uint32_t const n_tiles = (p.n_feats + per - 1) / per;
    if (D <= k_max_heap_depth && n_tiles <= k_max_heap_tiles && p.mirror != nullptr)
    {
        pl->depth          = D;
        pl->n_tiles        = n_tiles;
        size_t const   slots = static_cast<size_t>(2u << D);
        uint32_t const words = n_tiles * 8;
        std::vector<uint32_t> h(slots * n_trees, 0u);
        HeapPacker const      pk{D,     p.u8,      words, pl->cut_off.data(), feature, split_bin,
                            left,  right,     default_left, value};
        for (uint32_t t = 0; t < n_trees; ++t)
        {
            pk.fill(h.data() + (t * slots), roots[t], roots[t], 1, 0);
        }
        pl->heaps.upload(h.data(), h.size() * 4);
        // the last bin of every code lane of every staged word (padding
        // lanes: a value no code has)
        std::vector<uint32_t> lw(words, 0u);
        uint32_t const        lanes = p.u8 ? 4u : 2u;
        for (uint32_t wd = 0; wd < words; ++wd)
        {
            uint32_t v = 0;
            for (uint32_t k = 0; k < lanes; ++k)
            {
                uint32_t const f    = (wd * lanes) + k;
                uint32_t const last = f < p.n_feats ? p.h_cut_off[f + 1] - p.h_cut_off[f] - 1
                                                    : (p.u8 ? 0xFFu : 0xFFFFu);
                v |= last << (k * (32u / lanes));
            }
            lw[wd] = v;
        }
        pl->last_words.upload(lw.data(), lw.size() * 4);
    }
    else
    {
        std::vector<uint32_t> last(p.n_feats);
        for (uint32_t f = 0; f < p.n_feats; ++f)
        {
            last[f] = p.h_cut_off[f + 1] - p.h_cut_off[f] - 1;
        }
        pl->last.upload(last.data(), p.n_feats * 4ull);
        pl->roots.upload(roots, n_trees * 4ull);
        pl->feature.upload(feature, n_nodes * 4ull);
        pl->split.upload(split_bin, n_nodes * 4ull);
        pl->left.upload(left, n_nodes * 4ull);
        pl->right.upload(right, n_nodes * 4ull);
        pl->dl.upload(default_left, n_nodes);
        pl->value.upload(value, n_nodes * 4ull);
    }
    check(cudaStreamCreateWithFlags(&pl->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    return pl;
}

void plan_run_host(bb_predict_plan &pl, Plane const &p, uint32_t n_trees, float *out)
{
    std::lock_guard<std::mutex> lock(pl.mu);
    size_t const bytes = p.n_rows * sizeof(float);
    if (bytes == 0)
    {
        return;
    }
    if (pl.out_cap < bytes)
    {
        if (pl.out != nullptr)
        {
            check(cudaFree(pl.out), "cudaFree");
            pl.out     = nullptr;
            pl.out_cap = 0;
        }
        check(cudaMalloc(&pl.out, bytes), "cudaMalloc");
        pl.out_cap = bytes;
    }
    plan_launch(pl, p, n_trees, pl.out, pl.stream);
    check(cudaMemcpyAsync(out, pl.out, bytes, cudaMemcpyDeviceToHost, pl.stream),
          "cudaMemcpyAsync");
    check(cudaStreamSynchronize(pl.stream), "cudaStreamSynchronize");
}

uint32_t trees_to_run(bb_predict_plan const &pl, uint32_t n_trees)
{
    need(n_trees <= pl.n_trees, "bb_predict_plan: more trees asked than the plan holds");
    return n_trees == 0 ? pl.n_trees : n_trees;
}

} // namespace
} // namespace bb

using namespace bb;

extern "C"
{
    int bb_predict_plan_create(bb_plane const *plane, uint32_t n_trees, uint32_t const *roots,
                               uint32_t n_nodes, uint32_t const *feature,
                               uint32_t const *split_bin, uint32_t const *left,
                               uint32_t const *right, uint8_t const *default_left,
                               float const *value, float lr, float init, bb_predict_plan **out)
    {
        return guarded(
            [&]
            {
                need(plane != nullptr && out != nullptr, "bb_predict_plan_create: null argument");
                *out = make_plan(plane->p, n_trees, roots, n_nodes, feature, split_bin, left,
                                 right, default_left, value, lr, init)
                           .release();
            });
    }

    int bb_predict_plan_run(bb_predict_plan *plan, bb_plane const *plane, uint32_t n_trees,
                            float *out)
    {
        return guarded(
            [&]
            {
                need(plan != nullptr && plane != nullptr && out != nullptr,
                     "bb_predict_plan_run: null argument");
                plan_check_plane(*plan, plane->p);
                plan_run_host(*plan, plane->p, trees_to_run(*plan, n_trees), out);
            });
    }

    int bb_predict_plan_launch(bb_predict_plan *plan, bb_plane const *plane, uint32_t n_trees,
                               float *out_device, void *stream, uint32_t *launches)
    {
        return guarded(
            [&]
            {
                need(plan != nullptr && plane != nullptr && out_device != nullptr,
                     "bb_predict_plan_launch: null argument");
                plan_check_plane(*plan, plane->p);
                std::lock_guard<std::mutex> lock(plan->mu);
                uint32_t const k = plan_launch(*plan, plane->p, trees_to_run(*plan, n_trees),
                                               out_device, static_cast<cudaStream_t>(stream));
                if (launches != nullptr)
                {
                    *launches = k;
                }
            });
    }

    int bb_predict_plan_depth(bb_predict_plan const *plan, uint32_t *depth)
    {
        return guarded(
            [&]
            {
                need(plan != nullptr && depth != nullptr, "bb_predict_plan_depth: null argument");
                *depth = plan->depth;
            });
    }

    void bb_predict_plan_destroy(bb_predict_plan *plan)
    {
        delete plan;
    }

    int bb_predict(bb_plane const *plane, uint32_t n_trees, uint32_t const *roots,
                   uint32_t n_nodes, uint32_t const *feature, uint32_t const *split_bin,
                   uint32_t const *left, uint32_t const *right, uint8_t const *default_left,
                   float const *value, float lr, float init, float *out)
    {
        return guarded(
            [&]
            {
                need(plane != nullptr && out != nullptr, "bb_predict: null argument");
                auto pl = make_plan(plane->p, n_trees, roots, n_nodes, feature, split_bin, left,
                                    right, default_left, value, lr, init);
                plan_run_host(*pl, plane->p, n_trees, out);
            });
    }
}
