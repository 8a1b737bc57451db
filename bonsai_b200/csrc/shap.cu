// Device TreeSHAP (bb_pred_contribs): per-row SHAP contributions of an
// ensemble in bin space, in FP64.
//
// The reference computes them host-side with Lundberg et al.'s Algorithm 2
// (extend/unwind over a "unique path", src/shap.cpp:20-213) and device-side
// in FP32 over packed leaf paths (src/cuda/shap.cu:63-169, packer
// src/shap_paths.cpp). This kernel uses the path form of the same quantity:
// every root-to-leaf path, with the conditions on one feature merged into a
// single element i carrying its cover fraction z_i (the product of
// cover(child) / cover(parent) over that feature's splits) and the row's
// indicator o_i (1 when the row satisfies all of them), contributes
//
//     phi[f_i] += v * (o_i - z_i) * integral_0^1 prod_{j != i} (z_j + (o_j - z_j) t) dt
//
// because the Shapley weights |S|!(n-1-|S|)!/n! are the Beta integrals
// integral t^|S| (1-t)^(n-1-|S|) dt. The integrand is a polynomial of degree
// n - 1, so an m-point Gauss-Legendre rule with 2m - 1 >= n - 1 is exact; the
// products over j != i come from prefix and suffix products, with no
// division. The bias column is the reference's expected value per tree
// (tree_expected_value, src/shap.cpp:250-290), then the booster's
// composition: phi *= lr, phi[F] += init (include/bonsai/booster.hpp:903-924).
//
// The ensemble's paths are packed once (bb_shap_plan_create; the reference's
// cuda_shap_plan, include/bonsai/cuda/shap.hpp:31-35) into fixed-stride
// records of K elements (K = 8, 16 or 32 by the longest path) and streamed
// through shared memory in chunks. A CTA covers a tile of rows crossed with
// PL path lanes: thread (row, lane) takes every PL-th path of the chunk
// against its row's codes (staged in shared memory) and accumulates into its
// own FP64 slice; with PL = 1 every thread of a warp reads the same path
// (broadcast loads, no divergence). Small batches raise PL and split the
// paths across CTAs, each split writing its partial sums; slices and splits
// are summed in a fixed order, so results are bit-identical run to run.
#include "bonsai_b200.h"
#include "ingest.cuh"

#include <algorithm>
#include <cmath>
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

constexpr uint32_t k_max_path       = 32; // merged elements per path
constexpr uint32_t k_max_gauss      = 16;
constexpr uint32_t k_max_shap_feats = 128;
constexpr uint32_t k_sms            = 148;
constexpr size_t   k_chunk_budget   = 16384;
constexpr size_t   k_max_ws_bytes   = size_t{256} << 20;

// One merged path element: the feature and whether the missing (last) bin
// passes, the non-missing bins [lo, hi] its conditions leave (lo > hi:
// none), and the product of its cover fractions.
struct PathElem
{
    uint32_t fm;   // feature | miss_ok << 31
    uint32_t lohi; // lo | hi << 16
    double   zero;
};

struct PathHead
{
    double   value;
    uint32_t count;
    uint32_t pad;
};

struct Gauss
{
    double   x[k_max_gauss];
    double   w[k_max_gauss];
    uint32_t m;
};

// Contributions of the paths [blockIdx.y * paths_per_split, + paths_per_split)
// for rows [blockIdx.x * rpb, + rpb), rpb = blockDim.x >> lane_shift. Thread
// t is row t >> lane_shift, lane t & (PL - 1). out != nullptr: the composed
// row (x lr, bias column + bias and init); else the split's raw sums into
// ws[(blockIdx.y * n_rows + r) * (F + 1) + f].
template <uint32_t K>
__global__ void __launch_bounds__(128)
    shap_tile_kernel(uint8_t const *__restrict__ bins8, uint16_t const *__restrict__ bins16,
                     uint64_t n_pad, uint64_t n_rows, uint32_t const *__restrict__ last_bin,
                     uint32_t F, PathHead const *__restrict__ heads,
                     PathElem const *__restrict__ elems, uint32_t n_paths,
                     uint32_t paths_per_split, uint32_t chunk, uint32_t lane_shift, Gauss g,
                     double lr, double bias, double init, double *__restrict__ out,
                     double *__restrict__ ws)
{
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t const T    = blockDim.x;
    uint32_t const t    = threadIdx.x;
    uint32_t const PL   = 1u << lane_shift;
    uint32_t const rpb  = T >> lane_shift;
    uint32_t const rl   = t >> lane_shift;
    uint32_t const lane = t & (PL - 1u);
    auto *const    phi_s   = reinterpret_cast<double *>(smem);             // [F + 1][T]
    auto *const    heads_s = reinterpret_cast<PathHead *>(phi_s + ((F + 1) * T));
    // path j's elements at elems_s[j * (K + 1)]: the odd stride puts the
    // paths of different lanes on different banks
    auto *const    elems_s = reinterpret_cast<PathElem *>(heads_s + chunk);
    // row rl's code of feature f at codes_s[f * (rpb + 1) + rl]: lanes of one
    // row reading different features land on different banks
    auto *const    codes_s = reinterpret_cast<uint16_t *>(elems_s + (chunk * (K + 1)));
    auto *const    last_s  = reinterpret_cast<uint32_t *>(codes_s + (((F * (rpb + 1)) + 1) & ~1u));
    uint64_t const row0 = static_cast<uint64_t>(blockIdx.x) * rpb;
    uint64_t const row  = row0 + rl;

    for (uint32_t i = t; i < F * rpb; i += T)
    {
        uint32_t const f  = i / rpb;
        uint32_t const rr = i - (f * rpb);
        uint64_t const r  = row0 + rr;
        uint32_t       c = 0;
        if (r < n_rows)
        {
            c = bins8 != nullptr ? bins8[(static_cast<uint64_t>(f) * n_pad) + r]
                                 : bins16[(static_cast<uint64_t>(f) * n_pad) + r];
        }
        codes_s[(f * (rpb + 1)) + rr] = static_cast<uint16_t>(c);
    }
    __shared__ double gx_s[k_max_gauss];
    __shared__ double gw_s[k_max_gauss];
    for (uint32_t f = t; f < F; f += T)
    {
        last_s[f] = last_bin[f];
    }
    if (t < g.m)
    {
        gx_s[t] = g.x[t];
        gw_s[t] = g.w[t];
    }
    for (uint32_t f = 0; f <= F; ++f)
    {
        phi_s[(f * T) + t] = 0.0;
    }
    uint32_t const p0 = blockIdx.y * paths_per_split;
    uint32_t const p1 = min(n_paths, p0 + paths_per_split);
    for (uint32_t c0 = p0; c0 < p1; c0 += chunk)
    {
        uint32_t const nc = min(chunk, p1 - c0);
        __syncthreads(); // the previous chunk's paths are done (and codes staged)
        {
            auto const *hs = reinterpret_cast<uint4 const *>(heads + c0);
            auto       *hd = reinterpret_cast<uint4 *>(heads_s);
            for (uint32_t i = t; i < nc; i += T)
            {
                hd[i] = hs[i];
            }
            auto const    *es = reinterpret_cast<uint4 const *>(elems + (static_cast<size_t>(c0) * K));
            auto          *ed = reinterpret_cast<uint4 *>(elems_s);
            uint32_t const ne = nc * K;
            for (uint32_t i = t; i < ne; i += T)
            {
                uint32_t const j = i / K;
                ed[i + j]        = es[i];
            }
        }
        __syncthreads();
        if (row >= n_rows)
        {
            continue;
        }
        for (uint32_t j = lane; j < nc; j += PL)
        {
            PathHead const  h = heads_s[j];
            PathElem const *e = elems_s + (j * (K + 1));
            uint32_t const  n = h.count;
            double          z[K];
            double          d[K];
            double          S[K];
            uint32_t        fe[K];
#pragma unroll
            for (uint32_t i = 0; i < K; ++i)
            {
                z[i]  = 1.0;
                d[i]  = 0.0;
                S[i]  = 0.0;
                fe[i] = 0;
                if (i < n)
                {
                    PathElem const x  = e[i];
                    uint32_t const f  = x.fm & 0x7FFFFFFFu;
                    uint32_t const bn = codes_s[(f * (rpb + 1)) + rl];
                    bool const     on = bn == last_s[f] ? (x.fm >> 31) != 0
                                                        : (bn >= (x.lohi & 0xFFFFu) &&
                                                           bn <= (x.lohi >> 16));
                    z[i]  = x.zero;
                    d[i]  = (on ? 1.0 : 0.0) - x.zero;
                    fe[i] = f;
                }
            }
            // the Gauss-Legendre points are independent chains: unrolled, a
            // thread keeps several in flight. Padded elements have factor
            // exactly 1 (z = 1, d = 0), so the products need no predicate.
            constexpr uint32_t KU = K <= 16 ? K / 2 : 1; // points per unrolled step
            for (uint32_t k0 = 0; k0 < g.m; k0 += KU)
            {
#pragma unroll
                for (uint32_t kk = 0; kk < KU; ++kk)
                {
                    uint32_t const k = k0 + kk;
                    if (k >= g.m)
                    {
                        break;
                    }
                    double const x = gx_s[k];
                    double const w = gw_s[k];
                    double       fk[K];
                    double       pre[K];
#pragma unroll
                    for (uint32_t i = 0; i < K; ++i)
                    {
                        fk[i] = __fma_rn(d[i], x, z[i]);
                    }
                    pre[0] = 1.0;
#pragma unroll
                    for (uint32_t i = 1; i < K; ++i)
                    {
                        pre[i] = pre[i - 1] * fk[i - 1];
                    }
                    double suf = 1.0;
#pragma unroll
                    for (uint32_t ii = K; ii-- > 0;)
                    {
                        S[ii] = __fma_rn(w, pre[ii] * suf, S[ii]);
                        suf *= fk[ii];
                    }
                }
            }
#pragma unroll
            for (uint32_t i = 0; i < K; ++i)
            {
                if (i < n)
                {
                    phi_s[(fe[i] * T) + t] += h.value * d[i] * S[i];
                }
            }
        }
    }
    __syncthreads();
    // a row's lanes in a fixed order, then composed or kept as the split's sum
    for (uint32_t i = t; i < rpb * (F + 1); i += T)
    {
        uint32_t const r_l = i / (F + 1);
        uint32_t const f   = i - (r_l * (F + 1));
        uint64_t const r   = row0 + r_l;
        if (r >= n_rows)
        {
            continue;
        }
        double s = 0.0;
        for (uint32_t l = 0; l < PL; ++l)
        {
            s += phi_s[(f * T) + (r_l << lane_shift) + l];
        }
        if (out != nullptr)
        {
            out[(r * (F + 1)) + f] = f == F ? ((s + bias) * lr) + init : s * lr;
        }
        else
        {
            ws[((static_cast<uint64_t>(blockIdx.y) * n_rows + r) * (F + 1)) + f] = s;
        }
    }
}

// The splits' sums in split order, composed.
__global__ void shap_reduce_kernel(double const *__restrict__ ws, uint64_t n_rows, uint32_t F,
                                   uint32_t splits, double lr, double bias, double init,
                                   double *__restrict__ out)
{
    uint64_t const i = (static_cast<uint64_t>(blockIdx.x) * blockDim.x) + threadIdx.x;
    uint64_t const n = n_rows * (F + 1);
    if (i >= n)
    {
        return;
    }
    uint32_t const f = static_cast<uint32_t>(i % (F + 1));
    double         s = 0.0;
    for (uint32_t k = 0; k < splits; ++k)
    {
        s += ws[(static_cast<uint64_t>(k) * n) + i];
    }
    out[i] = f == F ? ((s + bias) * lr) + init : s * lr;
}

// Gauss-Legendre nodes and weights on [0, 1]: the roots of the degree-m
// Legendre polynomial by Newton's method on the three-term recurrence,
// weights 2 / ((1 - x^2) P'(x)^2), mapped from [-1, 1].
void gauss_legendre(uint32_t m, std::vector<double> &x01, std::vector<double> &w01)
{
    x01.assign(m, 0.0);
    w01.assign(m, 0.0);
    double const pi = 3.14159265358979323846;
    for (uint32_t i = 0; i < m; ++i)
    {
        double x = std::cos(pi * (i + 0.75) / (m + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; ++it)
        {
            double p0 = 1.0;
            double p1 = x;
            for (uint32_t k = 2; k <= m; ++k)
            {
                double const p2 = (((2.0 * k) - 1.0) * x * p1 - ((k - 1.0) * p0)) / k;
                p0              = p1;
                p1              = p2;
            }
            double const pm = m == 0 ? 1.0 : (m == 1 ? x : p1);
            double const pmm1 = m == 1 ? 1.0 : p0;
            dp                = m * (x * pm - pmm1) / ((x * x) - 1.0);
            double const dx   = pm / dp;
            x -= dx;
            if (std::fabs(dx) < 1e-16)
            {
                break;
            }
        }
        x01[i] = 0.5 * (x + 1.0);
        w01[i] = 1.0 / ((1.0 - (x * x)) * dp * dp); // 2 / (...) on [-1,1], halved
    }
}

struct Packed
{
    std::vector<PathHead> paths;
    std::vector<uint32_t> first; // each path's first element in elems
    std::vector<PathElem> elems;
    uint32_t              max_len = 0;
    double                bias    = 0.0; // sum over trees of the expected values
};

struct TreeView
{
    uint32_t const *feature;
    uint32_t const *split_bin;
    uint32_t const *left;
    uint32_t const *right;
    uint8_t const  *dl;
    float const    *value;
    float const    *cover;
    uint32_t        n;
};

// tree_expected_value (src/shap.cpp:250-290): cover-weighted leaf mean.
double expected_value(TreeView const &t, uint32_t id)
{
    if (t.feature[id] == k_leaf_flag)
    {
        return t.value[id];
    }
    double const cover = t.cover[id];
    if (cover <= 0.0)
    {
        return 0.0;
    }
    return ((static_cast<double>(t.cover[t.left[id]]) * expected_value(t, t.left[id])) +
            (static_cast<double>(t.cover[t.right[id]]) * expected_value(t, t.right[id]))) /
           cover;
}

struct Cond
{
    uint32_t feature;
    uint32_t lo, hi; // passing non-missing bins [lo, hi]
    bool     miss_ok;
    double   zero;
};

// Every root-to-leaf path of one tree, conditions on one feature merged:
// left at split s keeps bins <= s (and missing when default_left), right
// keeps bins > s (and missing otherwise), cover fractions multiply.
void collect(TreeView const &t, uint32_t const *last, uint32_t id, std::vector<Cond> &path,
             Packed &out)
{
    if (t.feature[id] == k_leaf_flag)
    {
        PathHead const h{static_cast<double>(t.value[id]), static_cast<uint32_t>(path.size()),
                         0u};
        out.first.push_back(static_cast<uint32_t>(out.elems.size()));
        for (Cond const &c : path)
        {
            out.elems.push_back({c.feature | (c.miss_ok ? 0x80000000u : 0u),
                                 (c.lo & 0xFFFFu) | ((c.hi & 0xFFFFu) << 16), c.zero});
        }
        out.max_len = std::max<uint32_t>(out.max_len, h.count);
        out.paths.push_back(h);
        return;
    }
    uint32_t const f     = t.feature[id];
    double const   cover = t.cover[id];
    for (int side = 0; side < 2; ++side)
    {
        uint32_t const child = side == 0 ? t.left[id] : t.right[id];
        double const   frac  = cover > 0.0 ? static_cast<double>(t.cover[child]) / cover : 0.0;
        size_t         k     = 0;
        while (k < path.size() && path[k].feature != f)
        {
            ++k;
        }
        bool const fresh = k == path.size();
        Cond const saved = fresh ? Cond{} : path[k];
        if (fresh)
        {
            path.push_back({f, 0, last[f] - 1, true, 1.0});
        }
        Cond &c = path[k];
        if (side == 0)
        {
            c.hi      = std::min(c.hi, t.split_bin[id]);
            c.miss_ok = c.miss_ok && t.dl[id] != 0;
        }
        else
        {
            c.lo      = std::max(c.lo, t.split_bin[id] + 1);
            c.miss_ok = c.miss_ok && t.dl[id] == 0;
        }
        c.zero *= frac;
        collect(t, last, child, path, out);
        if (fresh)
        {
            path.pop_back();
        }
        else
        {
            path[k] = saved;
        }
    }
}

} // namespace

// A device buffer released with its owner.
struct ShapBuf
{
    void *p = nullptr;
    ShapBuf() = default;
    ShapBuf(ShapBuf const &) = delete;
    ShapBuf &operator=(ShapBuf const &) = delete;
    ~ShapBuf()
    {
        if (p != nullptr)
        {
            cudaFree(p);
        }
    }
    void upload(void const *src, size_t bytes)
    {
        check(cudaMalloc(&p, std::max<size_t>(bytes, 16)), "cudaMalloc");
        if (bytes > 0)
        {
            check(cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy");
        }
    }
    void grow(size_t bytes, size_t &cap)
    {
        if (cap >= bytes)
        {
            return;
        }
        if (p != nullptr)
        {
            check(cudaFree(p), "cudaFree");
            p   = nullptr;
            cap = 0;
        }
        check(cudaMalloc(&p, bytes), "cudaMalloc");
        cap = bytes;
    }
    template <typename T> T *as() const
    {
        return static_cast<T *>(p);
    }
};

} // namespace bb

struct bb_shap_plan
{
    uint32_t              n_feats = 0;
    bool                  u8      = true;
    std::vector<uint32_t> cut_off;
    uint32_t              K       = 8;
    uint32_t              n_paths = 0;
    double                bias    = 0.0;
    double                lr      = 0.0;
    double                init    = 0.0;
    bb::Gauss             gauss{};
    bb::ShapBuf           heads, elems, last;
    std::mutex            mu;
    bb::ShapBuf           ws, out;
    size_t                ws_cap = 0, out_cap = 0;
    cudaStream_t          stream = nullptr;
    ~bb_shap_plan()
    {
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

std::unique_ptr<bb_shap_plan> make_shap_plan(Plane const &p, uint32_t n_trees,
                                             uint32_t const *roots, uint32_t n_nodes,
                                             uint32_t const *feature, uint32_t const *split_bin,
                                             uint32_t const *left, uint32_t const *right,
                                             uint8_t const *default_left, float const *value,
                                             float const *cover, float lr, float init)
{
    if (roots == nullptr || feature == nullptr || split_bin == nullptr || left == nullptr ||
        right == nullptr || default_left == nullptr || value == nullptr || cover == nullptr ||
        n_trees == 0)
    {
        throw std::invalid_argument("bb_shap_plan_create: null argument or empty ensemble");
    }
    uint32_t const F = p.n_feats;
    if (F > k_max_shap_feats)
    {
        throw ConfigError("bb_shap_plan_create: more than 128 features; use the host "
                          "TreeSHAP walk");
    }
    std::vector<uint32_t> last(F);
    for (uint32_t f = 0; f < F; ++f)
    {
        last[f] = p.h_cut_off[f + 1] - p.h_cut_off[f] - 1;
    }
    Packed pk;
    for (uint32_t t = 0; t < n_trees; ++t)
    {
        uint32_t const b = roots[t];
        uint32_t const e = t + 1 < n_trees ? roots[t + 1] : n_nodes;
        if (!(b < e && e <= n_nodes))
        {
            throw std::invalid_argument("bb_shap_plan_create: bad tree roots");
        }
        for (uint32_t i = b; i < e; ++i)
        {
            if (feature[i] == k_leaf_flag)
            {
                continue;
            }
            if (feature[i] >= F || !(left[i] > i - b && right[i] > i - b &&
                                     b + left[i] < e && b + right[i] < e) ||
                split_bin[i] + 1 > last[feature[i]])
            {
                throw std::invalid_argument("bb_shap_plan_create: malformed tree");
            }
        }
        TreeView const tv{feature + b, split_bin + b, left + b, right + b,
                          default_left + b, value + b, cover + b, e - b};
        std::vector<Cond> path;
        collect(tv, last.data(), 0, path, pk);
        pk.bias += expected_value(tv, 0);
    }
    if (pk.max_len > k_max_path)
    {
        throw ConfigError("bb_shap_plan_create: a path holds more than 32 distinct features");
    }
    auto pl     = std::make_unique<bb_shap_plan>();
    pl->n_feats = F;
    pl->u8      = p.u8;
    pl->cut_off.assign(p.h_cut_off, p.h_cut_off + F + 1);
    pl->K       = pk.max_len <= 8 ? 8u : (pk.max_len <= 16 ? 16u : 32u);
    pl->n_paths = static_cast<uint32_t>(pk.paths.size());
    pl->bias    = pk.bias;
    pl->lr      = static_cast<double>(lr);
    pl->init    = static_cast<double>(init);
    uint32_t const      m = std::max<uint32_t>(1, (pk.max_len + 1) / 2);
    std::vector<double> gx;
    std::vector<double> gw;
    gauss_legendre(m, gx, gw);
    pl->gauss.m = m;
    for (uint32_t k = 0; k < m; ++k)
    {
        pl->gauss.x[k] = gx[k];
        pl->gauss.w[k] = gw[k];
    }
    // fixed-stride element records: path j's elements at [j * K, j * K + count)
    std::vector<PathElem> el(static_cast<size_t>(pl->n_paths) * pl->K, PathElem{0, 0, 1.0});
    for (uint32_t j = 0; j < pl->n_paths; ++j)
    {
        std::copy_n(pk.elems.begin() + pk.first[j], pk.paths[j].count,
                    el.begin() + (static_cast<size_t>(j) * pl->K));
    }
    pl->heads.upload(pk.paths.data(), pk.paths.size() * sizeof(PathHead));
    pl->elems.upload(el.data(), el.size() * sizeof(PathElem));
    pl->last.upload(last.data(), F * 4ull);
    check(cudaStreamCreateWithFlags(&pl->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    return pl;
}

void shap_check_plane(bb_shap_plan const &pl, Plane const &p)
{
    if (p.n_feats != pl.n_feats || p.u8 != pl.u8 ||
        !std::equal(pl.cut_off.begin(), pl.cut_off.end(), p.h_cut_off))
    {
        throw std::invalid_argument(
            "bb_shap_plan: the plane's features or bin counts differ from the plan's");
    }
    if (p.n_rows > 0x7FFFFFFFull)
    {
        throw ConfigError("bb_shap_plan: more than 2^31 - 1 rows in one call");
    }
}

using TileFn = void (*)(uint8_t const *, uint16_t const *, uint64_t, uint64_t, uint32_t const *,
                        uint32_t, PathHead const *, PathElem const *, uint32_t, uint32_t,
                        uint32_t, uint32_t, Gauss, double, double, double, double *, double *);

TileFn tile_fn(uint32_t K)
{
    return K == 8 ? shap_tile_kernel<8> : (K == 16 ? shap_tile_kernel<16> : shap_tile_kernel<32>);
}

// Enqueues the contributions of every row of p into out (device,
// n_rows x (F + 1)); returns the kernels launched.
uint32_t shap_launch(bb_shap_plan &pl, Plane const &p, double *out, cudaStream_t s)
{
    uint64_t const n  = p.n_rows;
    if (n == 0)
    {
        return 0; // an empty request plane: nothing to explain
    }
    uint32_t const F  = pl.n_feats;
    TileFn const   fn = tile_fn(pl.K);
    // 128 threads while their FP64 slices fit 100 KB, else 64
    uint32_t const T   = (static_cast<size_t>(F) + 1) * 128 * 8 <= 102400 ? 128u : 64u;
    size_t const   rec = sizeof(PathHead) + ((pl.K + 1ull) * sizeof(PathElem));
    auto const chunk_of = [&](uint32_t PL)
    { return PL * std::max<uint32_t>(1, static_cast<uint32_t>(k_chunk_budget / (rec * PL))); };
    auto const smem_of = [&](uint32_t PL)
    {
        return ((static_cast<size_t>(F) + 1) * T * sizeof(double)) + (chunk_of(PL) * rec) +
               ((((static_cast<size_t>(F) * ((T / PL) + 1)) + 1) & ~size_t{1}) * 2) + (F * 4ull);
    };
    // one wave of resident CTAs is the target
    int occ = 0;
    check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem_of(1))),
          "cudaFuncSetAttribute");
    check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, static_cast<int>(T), smem_of(1)),
          "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    uint32_t const target = static_cast<uint32_t>(std::max(occ, 1)) * k_sms;
    // path lanes per row: raised until the row tiles fill the wave, or one row
    uint32_t lane_shift = 0;
    while ((1u << lane_shift) < T && ceil_div(n, T >> lane_shift) < target)
    {
        ++lane_shift;
    }
    uint32_t const PL       = 1u << lane_shift;
    uint32_t const rpb      = T >> lane_shift;
    uint32_t const row_blks = ceil_div(n, rpb);
    uint32_t const chunk    = chunk_of(PL);
    // split the paths when the row tiles still leave the wave short, each
    // lane keeping at least eight paths per split
    uint32_t splits = 1;
    if (row_blks < target)
    {
        uint32_t const most = std::max<uint32_t>(1, pl.n_paths / (8 * PL));
        splits              = std::min(ceil_div(target, row_blks), most);
        size_t const per    = n * (static_cast<size_t>(F) + 1) * sizeof(double);
        splits = static_cast<uint32_t>(
            std::min<size_t>(splits, std::max<size_t>(1, k_max_ws_bytes / per)));
    }
    uint32_t const pps = ceil_div(ceil_div(pl.n_paths, splits), chunk) * chunk;
    splits             = ceil_div(pl.n_paths, pps);
    size_t const smem  = smem_of(PL);
    double      *ws    = nullptr;
    if (splits > 1)
    {
        pl.ws.grow(static_cast<size_t>(splits) * n * (F + 1) * sizeof(double), pl.ws_cap);
        ws = pl.ws.as<double>();
    }
    check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem)),
          "cudaFuncSetAttribute");
    dim3 const grid(row_blks, splits);
    fn<<<grid, T, smem, s>>>(p.u8 ? static_cast<uint8_t const *>(p.bins) : nullptr,
                             p.u8 ? nullptr : static_cast<uint16_t const *>(p.bins), p.n_pad,
                             n, pl.last.as<uint32_t>(), F, pl.heads.as<PathHead>(),
                             pl.elems.as<PathElem>(), pl.n_paths, pps, chunk, lane_shift,
                             pl.gauss, pl.lr, pl.bias, pl.init, splits > 1 ? nullptr : out, ws);
    check(cudaGetLastError(), "shap_tile_kernel");
    if (splits == 1)
    {
        return 1;
    }
    uint64_t const cells = n * (F + 1);
    shap_reduce_kernel<<<ceil_div(cells, 256), 256, 0, s>>>(ws, n, F, splits, pl.lr, pl.bias,
                                                           pl.init, out);
    check(cudaGetLastError(), "shap_reduce_kernel");
    return 2;
}

void shap_run_host(bb_shap_plan &pl, Plane const &p, double *out)
{
    std::lock_guard<std::mutex> lock(pl.mu);
    size_t const bytes = p.n_rows * (pl.n_feats + 1ull) * sizeof(double);
    if (bytes == 0)
    {
        return;
    }
    pl.out.grow(bytes, pl.out_cap);
    shap_launch(pl, p, pl.out.as<double>(), pl.stream);
    check(cudaMemcpyAsync(out, pl.out.p, bytes, cudaMemcpyDeviceToHost, pl.stream),
          "cudaMemcpyAsync");
    check(cudaStreamSynchronize(pl.stream), "cudaStreamSynchronize");
}

template <typename F> int shap_guard(F &&f)
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

} // namespace
} // namespace bb

using namespace bb;

extern "C"
{
    int bb_shap_plan_create(bb_plane const *plane, uint32_t n_trees, uint32_t const *roots,
                            uint32_t n_nodes, uint32_t const *feature, uint32_t const *split_bin,
                            uint32_t const *left, uint32_t const *right,
                            uint8_t const *default_left, float const *value, float const *cover,
                            float lr, float init, bb_shap_plan **out)
    {
        return shap_guard(
            [&]
            {
                if (plane == nullptr || out == nullptr)
                {
                    throw std::invalid_argument("bb_shap_plan_create: null argument");
                }
                *out = make_shap_plan(plane->p, n_trees, roots, n_nodes, feature, split_bin,
                                      left, right, default_left, value, cover, lr, init)
                           .release();
            });
    }

    int bb_shap_plan_run(bb_shap_plan *plan, bb_plane const *plane, double *out)
    {
        return shap_guard(
            [&]
            {
                if (plan == nullptr || plane == nullptr || out == nullptr)
                {
                    throw std::invalid_argument("bb_shap_plan_run: null argument");
                }
                shap_check_plane(*plan, plane->p);
                shap_run_host(*plan, plane->p, out);
            });
    }

    int bb_shap_plan_launch(bb_shap_plan *plan, bb_plane const *plane, double *out_device,
                            void *stream, uint32_t *launches)
    {
        return shap_guard(
            [&]
            {
                if (plan == nullptr || plane == nullptr || out_device == nullptr)
                {
                    throw std::invalid_argument("bb_shap_plan_launch: null argument");
                }
                shap_check_plane(*plan, plane->p);
                std::lock_guard<std::mutex> lock(plan->mu);
                uint32_t const k = shap_launch(*plan, plane->p, out_device,
                                               static_cast<cudaStream_t>(stream));
                if (launches != nullptr)
                {
                    *launches = k;
                }
            });
    }

    void bb_shap_plan_destroy(bb_shap_plan *plan)
    {
        delete plan;
    }

    int bb_pred_contribs(bb_plane const *plane, uint32_t n_trees, uint32_t const *roots,
                         uint32_t n_nodes, uint32_t const *feature, uint32_t const *split_bin,
                         uint32_t const *left, uint32_t const *right,
                         uint8_t const *default_left, float const *value, float const *cover,
                         float lr, float init, double *out)
    {
        return shap_guard(
            [&]
            {
                if (plane == nullptr || out == nullptr)
                {
                    throw std::invalid_argument("bb_pred_contribs: null argument");
                }
                auto pl = make_shap_plan(plane->p, n_trees, roots, n_nodes, feature, split_bin,
                                         left, right, default_left, value, cover, lr, init);
                shap_check_plane(*pl, plane->p);
                shap_run_host(*pl, plane->p, out);
            });
    }
}
