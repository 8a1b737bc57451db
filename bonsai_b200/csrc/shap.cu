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
// One CTA per row: each thread takes every 64th leaf path, accumulates into its own
// FP64 slice of shared memory, and the CTA sums the slices in a fixed order,
// so results are bit-identical run to run.
#include "bonsai_b200.h"
#include "ingest.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
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

constexpr uint32_t k_shap_threads = 64;
constexpr uint32_t k_max_path     = 32; // merged elements per path
constexpr uint32_t k_max_gauss    = 16;
constexpr uint32_t k_max_shap_feats = 128;

// One merged path element: the feature, the non-missing bins [lo, hi] its
// conditions leave, whether the missing bin passes, and the product of its
// cover fractions.
struct PathElem
{
    uint32_t feature;
    uint16_t lo;      // first passing non-missing bin
    uint16_t hi;      // last passing non-missing bin (lo > hi: none)
    uint32_t miss_ok; // the missing (last) bin passes
    double   zero;
};

struct PathHead
{
    uint32_t first; // index of the first element
    uint32_t count;
    double   value;
};

template <uint32_t K>
__global__ void __launch_bounds__(k_shap_threads)
    shap_kernel(uint8_t const *bins8, uint16_t const *bins16, uint64_t n_pad,
                uint32_t const *last_bin, uint32_t F, uint32_t n_paths,
                PathHead const *paths, PathElem const *elems,
                double const *gx, double const *gw, uint32_t m, double lr, double bias,
                double init, double *out)
{
    extern __shared__ double phi_s[]; // [k_shap_threads][F + 1]
    __shared__ uint32_t      rowbin_s[k_max_shap_feats];
    __shared__ uint32_t      last_s[k_max_shap_feats];
    uint64_t const           row = blockIdx.x;
    uint32_t const           t   = threadIdx.x;
    for (uint32_t f = t; f < F; f += k_shap_threads)
    {
        rowbin_s[f] = bins8 != nullptr ? bins8[(static_cast<uint64_t>(f) * n_pad) + row]
                                       : bins16[(static_cast<uint64_t>(f) * n_pad) + row];
        last_s[f]   = last_bin[f];
    }
    double *phi = phi_s + (t * (F + 1));
    for (uint32_t f = 0; f <= F; ++f)
    {
        phi[f] = 0.0;
    }
    __syncthreads();
    {
        for (uint32_t p = t; p < n_paths; p += k_shap_threads)
        {
            PathHead const  h = paths[p];
            PathElem const *e = elems + h.first;
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
                    PathElem const  x  = e[i];
                    uint32_t const  bn = rowbin_s[x.feature];
                    bool const      on = bn == last_s[x.feature] ? x.miss_ok != 0
                                                                 : (bn >= x.lo && bn <= x.hi);
                    z[i]               = x.zero;
                    d[i]               = (on ? 1.0 : 0.0) - x.zero;
                    fe[i]              = x.feature;
                }
            }
            for (uint32_t k = 0; k < m; ++k)
            {
                double const x = gx[k];
                double       pre[K + 1];
                pre[0] = 1.0;
#pragma unroll
                for (uint32_t i = 0; i < K; ++i)
                {
                    pre[i + 1] = i < n ? pre[i] * (z[i] + (d[i] * x)) : pre[i];
                }
                double suf = 1.0;
#pragma unroll
                for (uint32_t ii = K; ii-- > 0;)
                {
                    if (ii < n)
                    {
                        S[ii] += gw[k] * (pre[ii] * suf);
                        suf *= z[ii] + (d[ii] * x);
                    }
                }
            }
#pragma unroll
            for (uint32_t i = 0; i < K; ++i)
            {
                if (i < n)
                {
                    phi[fe[i]] += h.value * d[i] * S[i];
                }
            }
        }
    }
    __syncthreads();
    // fixed-order sum of the thread slices, one column per thread, then the
    // booster's composition: bias column + expected values, x lr, + init
    for (uint32_t f = t; f <= F; f += k_shap_threads)
    {
        double s = 0.0;
        for (uint32_t u = 0; u < k_shap_threads; ++u)
        {
            s += phi_s[(u * (F + 1)) + f];
        }
        out[(row * (F + 1)) + f] = f == F ? ((s + bias) * lr) + init : s * lr;
    }
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
    std::vector<PathHead>  paths;
    std::vector<PathElem>  elems;
    uint32_t               max_len = 0;
    double                 bias    = 0.0; // sum over trees of the expected values
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
        PathHead h{static_cast<uint32_t>(out.elems.size()),
                   static_cast<uint32_t>(path.size()), static_cast<double>(t.value[id])};
        for (Cond const &c : path)
        {
            out.elems.push_back({c.feature, static_cast<uint16_t>(c.lo),
                                 static_cast<uint16_t>(c.hi), c.miss_ok ? 1u : 0u, c.zero});
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
} // namespace bb

using namespace bb;

extern "C" int bb_pred_contribs(bb_plane const *plane, uint32_t n_trees, uint32_t const *roots,
                                uint32_t n_nodes, uint32_t const *feature,
                                uint32_t const *split_bin, uint32_t const *left,
                                uint32_t const *right, uint8_t const *default_left,
                                float const *value, float const *cover, float lr, float init,
                                double *out)
{
    try
    {
        if (plane == nullptr || roots == nullptr || feature == nullptr || split_bin == nullptr ||
            left == nullptr || right == nullptr || default_left == nullptr || value == nullptr ||
            cover == nullptr || out == nullptr || n_trees == 0)
        {
            throw std::invalid_argument("bb_pred_contribs: null argument or empty ensemble");
        }
        Plane const   &p = plane->p;
        uint32_t const F = p.n_feats;
        if (p.n_rows > 0x7FFFFFFFull)
        {
            throw ConfigError("bb_pred_contribs: more than 2^31 - 1 rows in one call");
        }
        if (F > k_max_shap_feats)
        {
            throw ConfigError("bb_pred_contribs: more than 128 features; use the host "
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
                throw std::invalid_argument("bb_pred_contribs: bad tree roots");
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
                    throw std::invalid_argument("bb_pred_contribs: malformed tree");
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
            throw ConfigError("bb_pred_contribs: a path holds more than 32 distinct features");
        }
        uint32_t const      m = std::max<uint32_t>(1, (pk.max_len + 1) / 2);
        std::vector<double> gx;
        std::vector<double> gw;
        gauss_legendre(m, gx, gw);
        // device copies, released on every exit
        std::vector<void *> held;
        struct Release
        {
            std::vector<void *> &h;
            ~Release()
            {
                for (void *q : h)
                {
                    cudaFree(q);
                }
            }
        } release{held};
        auto up = [&](void const *src, size_t bytes) -> void *
        {
            void *d = nullptr;
            check(cudaMalloc(&d, std::max<size_t>(bytes, 16)), "cudaMalloc");
            held.push_back(d);
            if (bytes > 0)
            {
                check(cudaMemcpy(d, src, bytes, cudaMemcpyHostToDevice), "cudaMemcpy");
            }
            return d;
        };
        void *d_last  = up(last.data(), F * 4);
        void *d_paths = up(pk.paths.data(), pk.paths.size() * sizeof(PathHead));
        void *d_elems = up(pk.elems.data(), pk.elems.size() * sizeof(PathElem));
        void *d_gx    = up(gx.data(), m * 8);
        void *d_gw    = up(gw.data(), m * 8);
        uint64_t const n     = p.n_rows;
        if (n == 0)
        {
            return BB_OK;
        }
        size_t const   bytes = n * (F + 1) * sizeof(double);
        double        *d_out = nullptr;
        check(cudaMalloc(&d_out, bytes), "cudaMalloc");
        held.push_back(d_out);
        size_t const smem = k_shap_threads * (F + 1) * sizeof(double);
        uint8_t const  *b8  = p.u8 ? static_cast<uint8_t const *>(p.bins) : nullptr;
        uint16_t const *b16 = p.u8 ? nullptr : static_cast<uint16_t const *>(p.bins);
        auto launch = [&](auto kern)
        {
            check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(smem)),
                  "cudaFuncSetAttribute");
            kern<<<static_cast<uint32_t>(n), k_shap_threads, smem>>>(
                b8, b16, p.n_pad, static_cast<uint32_t const *>(d_last), F,
                static_cast<uint32_t>(pk.paths.size()), static_cast<PathHead const *>(d_paths),
                static_cast<PathElem const *>(d_elems), static_cast<double const *>(d_gx),
                static_cast<double const *>(d_gw), m, static_cast<double>(lr), pk.bias,
                static_cast<double>(init), d_out);
        };
        if (pk.max_len <= 8)
        {
            launch(shap_kernel<8>);
        }
        else if (pk.max_len <= 16)
        {
            launch(shap_kernel<16>);
        }
        else
        {
            launch(shap_kernel<32>);
        }
        check(cudaGetLastError(), "shap_kernel");
        check(cudaMemcpy(out, d_out, bytes, cudaMemcpyDeviceToHost), "cudaMemcpy");
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
