// TEST INFRASTRUCTURE — the oracle harness. Not part of the product.
//
// A C-ABI driver over the reference's own CPU implementation of the
// CUDA-grower hot path, compiled from the reference's sources by
// oracle/Makefile into oracle/_ref/libbonsai_ref.so. Only tests/, the smoke
// check and bench.py's CPU-baseline leg load it, always as the checker.
//
// What it drives (reference files, by path within the project):
//   BinMapper::fit / transform        src/bin_mapper.cpp:232-291
//   Dataset::bin (host bin fill)      src/dataset.cpp:45-160
//   Booster<Obj, Grower, Sampler>     include/bonsai/booster.hpp:484-592
//   DepthwiseGrower / ObliviousGrower / LeafwiseGrower<CpuHistogramEngine>
//                                     src/grower.cpp:155-157, src/grower_impl.hpp
//   HistogramNodeSplitFinder          src/split.cpp:271-297
//   DenseTree walk, tree_shap_binned  src/tree.cpp, src/shap.cpp
//
// libstdc++ 13 cannot compile src/bin_mappers.cpp (ranges::sample over an
// iota_view), so the three BinMappers accessors the other sources call are
// defined here, and per-column mappers are assembled with from_mappers.
// For <= n_samples rows that equals BinMappers::fit exactly.

#include "bonsai/bin_mapper.hpp"
#include "bonsai/bin_mappers.hpp"
#include "bonsai/booster.hpp"
#include "bonsai/config/config.hpp"
#include "bonsai/dataset.hpp"
#include "bonsai/grower.hpp"
#include "bonsai/multiclass_booster.hpp"
#include "bonsai/objective.hpp"
#include "bonsai/parallel.hpp"
#include "bonsai/sampler.hpp"
#include "bonsai/shap.hpp"
#include "bonsai/split.hpp"
#include "bonsai/tree.hpp"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

namespace bonsai
{
BinMapper const &BinMappers::operator[](size_t fid) const
{
    return mappers_[fid];
}
size_t BinMappers::size() const
{
    return mappers_.size();
}
std::span<std::string const> BinMappers::feature_names() const
{
    return feature_names_;
}
} // namespace bonsai

using namespace bonsai;

namespace
{

thread_local std::string g_err;

template <typename F> int guarded(F &&f)
{
    try
    {
        f();
        return 0;
    }
    catch (std::exception const &e)
    {
        g_err = e.what();
        return 1;
    }
    catch (...)
    {
        g_err = "unknown exception";
        return 1;
    }
}

BinMappers mappers_from_cuts(float const *cuts, uint32_t const *cut_off, size_t F)
{
    std::vector<BinMapper>   ms;
    std::vector<std::string> names;
    for (size_t f = 0; f < F; ++f)
    {
        ms.push_back(BinMapper::from_cuts(
            std::vector<float>(cuts + cut_off[f], cuts + cut_off[f + 1])));
        names.push_back("f" + std::to_string(f));
    }
    return BinMappers::from_mappers(std::move(ms), std::move(names));
}

// One flattened tree: DenseTree nodes plus their gains and covers. Oblivious
// trees are reported through their dense equivalent and their own tables.
struct FlatTree
{
    std::vector<uint32_t> feature;
    std::vector<float>    value; // threshold (internal) or leaf value
    std::vector<uint32_t> left, right;
    std::vector<uint8_t>  default_left;
    std::vector<float>    gains, covers;
    uint32_t              depth = 0, n_leaves = 0;
};

FlatTree flatten(DenseTree const &t)
{
    FlatTree ft;
    for (auto const &n : t.nodes())
    {
        ft.feature.push_back(n.feature_id);
        ft.value.push_back(n.threshold_or_value);
        ft.left.push_back(n.left);
        ft.right.push_back(n.right);
        ft.default_left.push_back(n.default_left ? 1 : 0);
    }
    ft.gains  = t.split_gains();
    ft.covers = t.covers();
    ft.gains.resize(ft.feature.size(), 0.0F);
    ft.covers.resize(ft.feature.size(), 0.0F);
    ft.depth    = static_cast<uint32_t>(t.params().depth);
    ft.n_leaves = static_cast<uint32_t>(t.params().n_leaves);
    return ft;
}

} // namespace

struct ref_cfg
    {
        int32_t  grower;    // 0 depthwise, 1 levelwise (oblivious), 2 leafwise
        int32_t  objective; // 0 mse, 1 logloss, 2 softmax, 3 poisson, 4 mae, 5 huber, 6 quantile
        uint32_t n_iters;
        float    learning_rate;
        float    min_child_hess;
        float    min_gain_to_split;
        float    lambda_l2;
        float    lambda_l1;
        float    feature_fraction;
        uint32_t max_depth;
        uint32_t min_data_in_leaf;
        uint32_t max_leaves;
        uint32_t feature_seed;
        float    subsample; // < 1 selects the Bernoulli sampler
        uint32_t random_seed;
        uint32_t n_threads;
        uint32_t n_classes;
        int32_t const *monotone;
        uint32_t       n_monotone;
        char const    *interaction; // groups as the TOML strings, ';'-separated, or null
        float          quantile_alpha;
        float          huber_delta;
        float          dart_drop_rate;
        float          goss_top_rate;   // > 0 selects the GOSS sampler
        float          goss_other_rate;
        int32_t        hist_mode; // the drop-in grower's form: 0 plain, 1 int8, 2 int16
    };

    struct RefModel
    {
        std::unique_ptr<IBooster> booster;
        std::vector<FlatTree>     trees;
        std::vector<float>        init_scores;
        int32_t                   grower = 0;
        // oblivious tables, per tree
        std::vector<std::vector<ObliviousTree::LevelSplit>> level_splits;
        std::vector<std::vector<float>>                     leaf_tables;
    };

namespace
{
    Config make_config(ref_cfg const &c)
    {
        Config cfg;
        cfg.tree_config.min_child_hess    = c.min_child_hess;
        cfg.tree_config.min_gain_to_split = c.min_gain_to_split;
        cfg.tree_config.lambda_l2         = c.lambda_l2;
        cfg.tree_config.lambda_l1         = c.lambda_l1;
        cfg.tree_config.feature_fraction  = c.feature_fraction;
        cfg.tree_config.max_depth         = static_cast<uint8_t>(c.max_depth);
        cfg.tree_config.min_data_in_leaf  = static_cast<uint8_t>(c.min_data_in_leaf);
        cfg.tree_config.max_leaves        = c.max_leaves;
        cfg.tree_config.feature_seed      = c.feature_seed;
        if (c.monotone != nullptr)
        {
            cfg.tree_config.monotone_constraints.assign(c.monotone,
                                                        c.monotone + c.n_monotone);
        }
        if (c.interaction != nullptr)
        {
            std::string const all(c.interaction);
            size_t            at = 0;
            while (at <= all.size())
            {
                size_t const e = std::min(all.find(';', at), all.size());
                if (e > at)
                {
                    cfg.tree_config.interaction_constraints.push_back(all.substr(at, e - at));
                }
                at = e + 1;
            }
        }
        cfg.booster_config.n_iters       = c.n_iters;
        cfg.booster_config.learning_rate = c.learning_rate;
        cfg.booster_config.random_seed   = c.random_seed;
        cfg.sampler.subsample            = c.subsample;
        cfg.objective.n_classes          = c.n_classes;
        cfg.objective.quantile_alpha     = c.quantile_alpha;
        cfg.objective.huber_delta        = c.huber_delta;
        cfg.booster_config.dart_drop_rate = c.dart_drop_rate;
        if (c.goss_top_rate > 0.0F)
        {
            cfg.sampler.top_rate   = c.goss_top_rate;
            cfg.sampler.other_rate = c.goss_other_rate;
        }
        return cfg;
    }

    template <typename Gr, typename Sa>
    std::unique_ptr<IBooster> make_for_objective(ref_cfg const &c, Config const &cfg)
    {
        switch (c.objective)
        {
        case 0:
            return std::make_unique<Booster<MSEObjective, Gr, Sa>>(cfg);
        case 1:
            return std::make_unique<Booster<LogLossObjective, Gr, Sa>>(cfg);
        case 2:
            return std::make_unique<MulticlassBooster<Gr, Sa>>(cfg);
        case 3:
            return std::make_unique<Booster<PoissonObjective, Gr, Sa>>(cfg);
        case 4:
            return std::make_unique<Booster<MAEObjective, Gr, Sa>>(cfg);
        case 5:
            return std::make_unique<Booster<HuberObjective, Gr, Sa>>(cfg);
        case 6:
            return std::make_unique<Booster<QuantileObjective, Gr, Sa>>(cfg);
        default:
            throw std::runtime_error("unknown objective");
        }
    }

    template <typename Gr>
    std::unique_ptr<IBooster> make_for_sampler(ref_cfg const &c, Config const &cfg)
    {
        if (c.goss_top_rate > 0.0F)
        {
            return make_for_objective<Gr, GossSampler>(c, cfg);
        }
        if (c.subsample < 1.0F)
        {
            return make_for_objective<Gr, BernoulliSampler>(c, cfg);
        }
        return make_for_objective<Gr, AllRowsSampler>(c, cfg);
    }

    template <typename B> void harvest_dense(RefModel &m, B const &b)
    {
        for (auto const &t : b.trees())
        {
            m.trees.push_back(flatten(t));
        }
    }

    template <typename B> void harvest_oblivious(RefModel &m, B const &b)
    {
        for (auto const &t : b.trees())
        {
            m.level_splits.push_back(t.splits());
            m.leaf_tables.push_back(t.leaf_table());
            m.trees.push_back(flatten(dense_equivalent(t)));
        }
    }

    template <typename Gr> void harvest(RefModel &m, ref_cfg const &c)
    {
        auto *raw = m.booster.get();
        auto  go  = [&](auto *b)
        {
            if (b == nullptr)
            {
                return false;
            }
            if constexpr (std::same_as<typename Gr::Tree, DenseTree>)
            {
                harvest_dense(m, *b);
            }
            else
            {
                harvest_oblivious(m, *b);
            }
            return true;
        };
        bool ok = false;
        if (c.goss_top_rate > 0.0F)
        {
            ok = go(dynamic_cast<Booster<MSEObjective, Gr, GossSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<LogLossObjective, Gr, GossSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<PoissonObjective, Gr, GossSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<MAEObjective, Gr, GossSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<HuberObjective, Gr, GossSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<QuantileObjective, Gr, GossSampler> *>(raw)) ||
                 go(dynamic_cast<MulticlassBooster<Gr, GossSampler> *>(raw));
        }
        else if (c.subsample < 1.0F)
        {
            ok = go(dynamic_cast<Booster<MSEObjective, Gr, BernoulliSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<LogLossObjective, Gr, BernoulliSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<PoissonObjective, Gr, BernoulliSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<MAEObjective, Gr, BernoulliSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<HuberObjective, Gr, BernoulliSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<QuantileObjective, Gr, BernoulliSampler> *>(raw)) ||
                 go(dynamic_cast<MulticlassBooster<Gr, BernoulliSampler> *>(raw));
        }
        else
        {
            ok = go(dynamic_cast<Booster<MSEObjective, Gr, AllRowsSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<LogLossObjective, Gr, AllRowsSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<PoissonObjective, Gr, AllRowsSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<MAEObjective, Gr, AllRowsSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<HuberObjective, Gr, AllRowsSampler> *>(raw)) ||
                 go(dynamic_cast<Booster<QuantileObjective, Gr, AllRowsSampler> *>(raw)) ||
                 go(dynamic_cast<MulticlassBooster<Gr, AllRowsSampler> *>(raw));
        }
        if (!ok)
        {
            throw std::runtime_error("booster type not recognised");
        }
    }

    template <typename B> void read_init(RefModel &m, B const *b)
    {
        if (b != nullptr)
        {
            m.init_scores = {b->init_score()};
        }
    }

    // MulticlassBooster keeps one log-prior per class.
    template <typename G> void read_init_multi(RefModel &m, void const *raw)
    {
        if (auto const *b = dynamic_cast<MulticlassBooster<G, AllRowsSampler> const *>(
                static_cast<IBooster const *>(raw)))
        {
            m.init_scores = b->init_scores();
        }
    }
} // namespace


extern "C"
{



    char const *ref_last_error()
    {
        return g_err.c_str();
    }

    // BinMapper::fit per column (row-major X), cuts written flattened.
    // cut_off must hold F + 1 entries; cuts_cap bounds the cut buffer.
    int ref_fit_cuts(float const *X, size_t n, size_t F, int32_t max_bin,
                     size_t n_samples, uint64_t seed, float *cuts, size_t cuts_cap,
                     uint32_t *cut_off)
    {
        return guarded(
            [&]
            {
                BinMapperConfig cfg;
                cfg.max_bin   = max_bin;
                cfg.n_samples = n_samples;
                cfg.seed      = seed;
                size_t             pos = 0;
                std::vector<float> col(n);
                for (size_t f = 0; f < F; ++f)
                {
                    for (size_t r = 0; r < n; ++r)
                    {
                        col[r] = X[(r * F) + f];
                    }
                    BinMapper const m = BinMapper::fit(col, cfg);
                    auto const      c = m.cuts();
                    if (pos + c.size() > cuts_cap)
                    {
                        throw std::runtime_error("ref_fit_cuts: cut buffer too small");
                    }
                    cut_off[f] = static_cast<uint32_t>(pos);
                    std::memcpy(cuts + pos, c.data(), c.size() * sizeof(float));
                    pos += c.size();
                }
                cut_off[F] = static_cast<uint32_t>(pos);
            });
    }

    // Cuts from an explicit NaN-free sample per column (the shared row sample
    // for tall data), via BinMapper::from_sample.
    int ref_cuts_from_sample(float const *sample_rowmajor, size_t n, size_t F,
                             int32_t max_bin, float *cuts, size_t cuts_cap,
                             uint32_t *cut_off)
    {
        return guarded(
            [&]
            {
                BinMapperConfig cfg;
                cfg.max_bin = max_bin;
                size_t pos  = 0;
                for (size_t f = 0; f < F; ++f)
                {
                    std::vector<float> col;
                    for (size_t r = 0; r < n; ++r)
                    {
                        float const v = sample_rowmajor[(r * F) + f];
                        if (!std::isnan(v))
                        {
                            col.push_back(v);
                        }
                    }
                    BinMapper const m = BinMapper::from_sample(std::move(col), cfg);
                    auto const      c = m.cuts();
                    if (pos + c.size() > cuts_cap)
                    {
                        throw std::runtime_error("ref_cuts_from_sample: buffer");
                    }
                    cut_off[f] = static_cast<uint32_t>(pos);
                    std::memcpy(cuts + pos, c.data(), c.size() * sizeof(float));
                    pos += c.size();
                }
                cut_off[F] = static_cast<uint32_t>(pos);
            });
    }

    // A binned Dataset over row-major X under the given cuts.
    void *ref_dataset_create(float const *X, float const *y, size_t n, size_t F,
                             float const *cuts, uint32_t const *cut_off)
    {
        Dataset *out = nullptr;
        int const rc = guarded(
            [&]
            {
                BinMappers const mappers = mappers_from_cuts(cuts, cut_off, F);
                features_view    Xv(X, n, F);
                std::vector<float> labels(y, y + n);
                out = new Dataset(Dataset::bin(Xv, labels, mappers, DataConfig{}));
            });
        return rc == 0 ? out : nullptr;
    }

    // The same with per-row sample weights (Dataset::bin's weights argument).
    void *ref_dataset_create_weighted(float const *X, float const *y, float const *w, size_t n,
                                      size_t F, float const *cuts, uint32_t const *cut_off)
    {
        Dataset *out = nullptr;
        int const rc = guarded(
            [&]
            {
                BinMappers const   mappers = mappers_from_cuts(cuts, cut_off, F);
                features_view      Xv(X, n, F);
                std::vector<float> labels(y, y + n);
                std::vector<float> weights(w, w + n);
                out = new Dataset(
                    Dataset::bin(Xv, labels, mappers, DataConfig{}, nullptr, weights));
            });
        return rc == 0 ? out : nullptr;
    }

    void ref_dataset_destroy(void *ds)
    {
        delete static_cast<Dataset *>(ds);
    }

    int ref_dataset_u8(void const *ds)
    {
        return static_cast<Dataset const *>(ds)->bins_are_u8() ? 1 : 0;
    }

    // Feature-major bin codes, widened to u16.
    int ref_dataset_bins(void const *dsp, uint16_t *out)
    {
        return guarded(
            [&]
            {
                auto const  &ds = *static_cast<Dataset const *>(dsp);
                size_t const n  = ds.n_rows();
                for (size_t f = 0; f < ds.n_features(); ++f)
                {
                    for (size_t r = 0; r < n; ++r)
                    {
                        out[(f * n) + r] = ds.bin_at(f, r);
                    }
                }
            });
    }

    // Trains a Booster on ds for cfg.n_iters rounds. Returns a model handle.
    void *ref_train(void const *dsp, ref_cfg const *c)
    {
        RefModel *m  = nullptr;
        int const rc = guarded(
            [&]
            {
                auto const &ds  = *static_cast<Dataset const *>(dsp);
                Config      cfg = make_config(*c);
                parallel::set_n_threads(c->n_threads);
                auto mm    = std::make_unique<RefModel>();
                mm->grower = c->grower;
                switch (c->grower)
                {
                case 0:
                    mm->booster = make_for_sampler<DepthwiseGrower<>>(*c, cfg);
                    break;
                case 1:
                    mm->booster = make_for_sampler<ObliviousGrower<>>(*c, cfg);
                    break;
                case 2:
                    mm->booster = make_for_sampler<LeafwiseGrower<>>(*c, cfg);
                    break;
                default:
                    throw std::runtime_error("unknown grower");
                }
                for (uint32_t i = 0; i < c->n_iters; ++i)
                {
                    mm->booster->update_one_iter(ds);
                }
                switch (c->grower)
                {
                case 0:
                    harvest<DepthwiseGrower<>>(*mm, *c);
                    break;
                case 1:
                    harvest<ObliviousGrower<>>(*mm, *c);
                    break;
                default:
                    harvest<LeafwiseGrower<>>(*mm, *c);
                    break;
                }
                auto *raw = mm->booster.get();
                read_init(*mm, dynamic_cast<Booster<MSEObjective, DepthwiseGrower<>,
                                                    AllRowsSampler> const *>(raw));
                read_init(*mm, dynamic_cast<Booster<PoissonObjective, DepthwiseGrower<>,
                                                    AllRowsSampler> const *>(raw));
                read_init(*mm, dynamic_cast<Booster<PoissonObjective, LeafwiseGrower<>,
                                                    AllRowsSampler> const *>(raw));
                read_init(*mm, dynamic_cast<Booster<PoissonObjective, ObliviousGrower<>,
                                                    AllRowsSampler> const *>(raw));
                read_init(*mm, dynamic_cast<Booster<LogLossObjective, DepthwiseGrower<>,
                                                    AllRowsSampler> const *>(raw));
                read_init(*mm, dynamic_cast<Booster<MSEObjective, ObliviousGrower<>,
                                                    AllRowsSampler> const *>(raw));
                read_init(*mm, dynamic_cast<Booster<LogLossObjective, ObliviousGrower<>,
                                                    AllRowsSampler> const *>(raw));
                read_init(*mm, dynamic_cast<Booster<MSEObjective, LeafwiseGrower<>,
                                                    AllRowsSampler> const *>(raw));
                read_init(*mm, dynamic_cast<Booster<LogLossObjective, LeafwiseGrower<>,
                                                    AllRowsSampler> const *>(raw));
                read_init(*mm, dynamic_cast<Booster<MSEObjective, DepthwiseGrower<>,
                                                    BernoulliSampler> const *>(raw));
                read_init(*mm, dynamic_cast<Booster<MSEObjective, LeafwiseGrower<>,
                                                    BernoulliSampler> const *>(raw));
                read_init_multi<DepthwiseGrower<>>(*mm, raw);
                read_init_multi<ObliviousGrower<>>(*mm, raw);
                read_init_multi<LeafwiseGrower<>>(*mm, raw);
                m = mm.release();
            });
        return rc == 0 ? m : nullptr;
    }

    void ref_model_destroy(void *mp)
    {
        delete static_cast<RefModel *>(mp);
    }

    size_t ref_model_n_trees(void const *mp)
    {
        return static_cast<RefModel const *>(mp)->trees.size();
    }

    float ref_model_init_score(void const *mp)
    {
        auto const *m = static_cast<RefModel const *>(mp);
        return m->init_scores.empty() ? 0.0F : m->init_scores[0];
    }

    // Every init score (one per class for softmax); returns how many.
    size_t ref_model_init_scores(void const *mp, float *out, size_t cap)
    {
        auto const  *m = static_cast<RefModel const *>(mp);
        size_t const n = std::min(cap, m->init_scores.size());
        std::memcpy(out, m->init_scores.data(), n * 4);
        return m->init_scores.size();
    }

    size_t ref_model_tree_size(void const *mp, size_t t)
    {
        return static_cast<RefModel const *>(mp)->trees[t].feature.size();
    }

    // Copies tree t's node table (n = ref_model_tree_size entries each).
    void ref_model_tree(void const *mp, size_t t, uint32_t *feature, float *value,
                        uint32_t *left, uint32_t *right, uint8_t *default_left,
                        float *gains, float *covers)
    {
        auto const &ft = static_cast<RefModel const *>(mp)->trees[t];
        size_t const n = ft.feature.size();
        std::memcpy(feature, ft.feature.data(), n * 4);
        std::memcpy(value, ft.value.data(), n * 4);
        std::memcpy(left, ft.left.data(), n * 4);
        std::memcpy(right, ft.right.data(), n * 4);
        std::memcpy(default_left, ft.default_left.data(), n);
        std::memcpy(gains, ft.gains.data(), n * 4);
        std::memcpy(covers, ft.covers.data(), n * 4);
    }

    // Oblivious tree t: depth level splits and 2^depth leaf values.
    size_t ref_model_oblivious_depth(void const *mp, size_t t)
    {
        auto const *m = static_cast<RefModel const *>(mp);
        return t < m->level_splits.size() ? m->level_splits[t].size() : 0;
    }

    void ref_model_oblivious(void const *mp, size_t t, uint32_t *feature,
                             float *threshold, uint8_t *default_left, float *leaves)
    {
        auto const *m  = static_cast<RefModel const *>(mp);
        auto const &ls = m->level_splits[t];
        for (size_t i = 0; i < ls.size(); ++i)
        {
            feature[i]      = ls[i].feature_id;
            threshold[i]    = ls[i].threshold;
            default_left[i] = ls[i].default_left ? 1 : 0;
        }
        auto const &lt = m->leaf_tables[t];
        std::memcpy(leaves, lt.data(), lt.size() * 4);
    }

    // Binned predict over ds: init + lr * sum of leaves (predict_at_binned).
    int ref_model_predict_binned(void const *mp, void const *dsp, float *out)
    {
        return guarded(
            [&]
            {
                auto const *m  = static_cast<RefModel const *>(mp);
                auto const &ds = *static_cast<Dataset const *>(dsp);
                m->booster->predict_at_binned(ds, {out, ds.n_rows()}, 0);
            });
    }

    // Raw-feature predict over row-major X (predict_at).
    int ref_model_predict(void const *mp, float const *X, size_t n, size_t F, float *out)
    {
        return guarded(
            [&]
            {
                auto const *m = static_cast<RefModel const *>(mp);
                m->booster->predict(features_view(X, n, F), {out, n});
            });
    }

    // TreeSHAP over ds in bin space: n_rows x (F + 1) doubles, bias last.
    int ref_model_contribs_binned(void const *mp, void const *dsp, double *out)
    {
        return guarded(
            [&]
            {
                auto const  *m  = static_cast<RefModel const *>(mp);
                auto const  &ds = *static_cast<Dataset const *>(dsp);
                size_t const F  = ds.n_features();
                m->booster->pred_contribs_binned(ds, {out, ds.n_rows() * (F + 1)}, F);
            });
    }

    // Warm start (include/bonsai/booster.hpp:512-524, load_state :1065-1069):
    // the reference's depthwise booster loaded with n_trees given DenseTrees
    // (node arrays concatenated, tree t's nodes at [off[t], off[t + 1])) and
    // init_score, then trained c.n_iters more rounds; the model holds every
    // tree, the loaded ones first. MSE and logloss, every row.
    void *ref_warm_train(void const *dsp, ref_cfg const *c, uint32_t n_trees,
                         uint32_t const *off, uint32_t const *feature, float const *value,
                         uint32_t const *left, uint32_t const *right,
                         uint8_t const *default_left, float const *gains,
                         float const *covers, uint32_t const *depth,
                         uint32_t const *n_leaves, float init_score)
    {
        RefModel *m  = nullptr;
        int const rc = guarded(
            [&]
            {
                auto const &ds  = *static_cast<Dataset const *>(dsp);
                Config      cfg = make_config(*c);
                parallel::set_n_threads(c->n_threads);
                std::vector<DenseTree> trees;
                for (uint32_t t = 0; t < n_trees; ++t)
                {
                    DenseTree::Nodes nodes;
                    for (uint32_t i = off[t]; i < off[t + 1]; ++i)
                    {
                        nodes.push_back(feature[i] == DenseTree::k_leaf_flag
                                            ? DenseTree::leaf(value[i])
                                            : DenseTree::internal(feature[i], value[i],
                                                                  left[i], right[i],
                                                                  default_left[i] != 0));
                    }
                    trees.emplace_back(std::move(nodes),
                                       DenseTree::Params{.depth = depth[t], .n_leaves = n_leaves[t]},
                                       std::vector<float>(gains + off[t], gains + off[t + 1]),
                                       std::vector<float>(covers + off[t], covers + off[t + 1]));
                }
                auto mm    = std::make_unique<RefModel>();
                mm->grower = 0;
                auto go    = [&](auto b)
                {
                    b->load_state(trees, init_score);
                    for (uint32_t i = 0; i < c->n_iters; ++i)
                    {
                        b->update_one_iter(ds);
                    }
                    harvest_dense(*mm, *b);
                    mm->init_scores = {b->init_score()};
                    mm->booster     = std::move(b);
                };
                if (c->objective == 0)
                {
                    go(std::make_unique<Booster<MSEObjective, DepthwiseGrower<>, AllRowsSampler>>(cfg));
                }
                else if (c->objective == 1)
                {
                    go(std::make_unique<
                        Booster<LogLossObjective, DepthwiseGrower<>, AllRowsSampler>>(cfg));
                }
                else
                {
                    throw std::runtime_error("ref_warm_train: mse or logloss");
                }
                m = mm.release();
            });
        return rc == 0 ? m : nullptr;
    }

    // The same for a model of n_classes outputs: out holds n x n_classes x (F + 1)
    // (MulticlassBooster's layout, include/bonsai/multiclass_booster.hpp:411-436).
    int ref_model_contribs_binned_k(void const *mp, void const *dsp, double *out,
                                    size_t n_classes)
    {
        return guarded(
            [&]
            {
                auto const  *m  = static_cast<RefModel const *>(mp);
                auto const  &ds = *static_cast<Dataset const *>(dsp);
                size_t const F  = ds.n_features();
                m->booster->pred_contribs_binned(ds, {out, ds.n_rows() * n_classes * (F + 1)},
                                                 F);
            });
    }

    // Grows ONE depthwise/levelwise/leafwise tree on given grad/hess over the
    // given ascending rows, through the reference's CPU grower. Outputs the
    // per-row leaf values and leaf ids over all ds rows (unsampled rows are
    // routed, as grow does) and keeps the tree for the getters below.
    void *ref_grow_tree(void const *dsp, ref_cfg const *c, float const *grad,
                        float const *hess, uint32_t const *rows, size_t n_sel,
                        float *values, uint32_t *leaf_ids)
    {
        RefModel *m  = nullptr;
        int const rc = guarded(
            [&]
            {
                auto const &ds  = *static_cast<Dataset const *>(dsp);
                Config      cfg = make_config(*c);
                parallel::set_n_threads(c->n_threads);
                size_t const       n = ds.n_rows();
                floats_view const  g{grad, n};
                floats_view const  h{hess, n};
                row_index_view const ri{rows, n_sel};
                auto mm    = std::make_unique<RefModel>();
                mm->grower = c->grower;
                auto take  = [&](auto &&res)
                {
                    std::memcpy(values, res.values.data(), n * 4);
                    std::memcpy(leaf_ids, res.leaf_ids.data(), n * 4);
                    return std::move(res.tree);
                };
                switch (c->grower)
                {
                case 0:
                {
                    DepthwiseGrower<> gr(cfg.tree_config);
                    mm->trees.push_back(flatten(take(gr.grow(ds, g, h, ri))));
                    break;
                }
                case 1:
                {
                    ObliviousGrower<> gr(cfg.tree_config);
                    ObliviousTree     t = take(gr.grow(ds, g, h, ri));
                    mm->level_splits.push_back(t.splits());
                    mm->leaf_tables.push_back(t.leaf_table());
                    mm->trees.push_back(flatten(dense_equivalent(t)));
                    break;
                }
                default:
                {
                    LeafwiseGrower<> gr(cfg.tree_config);
                    mm->trees.push_back(flatten(take(gr.grow(ds, g, h, ri))));
                    break;
                }
                }
                m = mm.release();
            });
        return rc == 0 ? m : nullptr;
    }

    // The reference's node split finder on one hand-built histogram set:
    // hist is [F][n_bins] cells of (g, h) floats, F features sharing n_bins.
    // Writes (gain, feature, bin, default_left, valid).
    int ref_find_split(float const *hist, size_t F, size_t n_bins, size_t n_rows,
                       ref_cfg const *c, double *gain, uint32_t *feature,
                       uint32_t *bin, uint8_t *default_left, uint8_t *valid)
    {
        return guarded(
            [&]
            {
                Config     cfg = make_config(*c);
                SplitInput in;
                for (size_t f = 0; f < F; ++f)
                {
                    Histogram hh(n_bins);
                    for (size_t b = 0; b < n_bins; ++b)
                    {
                        float const *cell = hist + (((f * n_bins) + b) * 2);
                        hh.add(static_cast<bin_id_t>(b), cell[0], cell[1]);
                    }
                    in.hists.push_back(std::move(hh));
                }
                in.rows.assign(n_rows, 0);
                SplitOutput const s = HistogramNodeSplitFinder::find(in, cfg.tree_config);
                *gain               = s.gain;
                *feature            = s.feature_id;
                *bin                = s.bin_id;
                *default_left       = s.default_left ? 1 : 0;
                *valid              = s.valid ? 1 : 0;
            });
    }
}

#ifdef BONSAI_B200_DROPIN
// The drop-in check: the reference's own Booster and boosting loop
// (include/bonsai/booster.hpp:484-592) with bonsai_b200's grower shim in
// place of DepthwiseGrower<CudaHistogramEngine>. Trains cfg.n_iters rounds
// on ds; the model handle reads back like ref_train's.
#include "bonsai_b200_grower.hpp"

namespace
{
// The reference's booster over one of the shims (Gr), trained and harvested.
template <typename Gr> RefModel *b200_train_with(Dataset const &ds, ref_cfg const &c)
{
    Config cfg = make_config(c);
    parallel::set_n_threads(c.n_threads);
    auto mm     = std::make_unique<RefModel>();
    mm->grower  = c.grower;
    mm->booster = make_for_sampler<Gr>(c, cfg);
    for (uint32_t i = 0; i < c.n_iters; ++i)
    {
        mm->booster->update_one_iter(ds);
    }
    harvest<Gr>(*mm, c);
    auto *raw = mm->booster.get();
    read_init(*mm, dynamic_cast<Booster<MSEObjective, Gr, AllRowsSampler> const *>(raw));
    read_init(*mm, dynamic_cast<Booster<LogLossObjective, Gr, AllRowsSampler> const *>(raw));
    read_init(*mm, dynamic_cast<Booster<MSEObjective, Gr, BernoulliSampler> const *>(raw));
    read_init(*mm, dynamic_cast<Booster<LogLossObjective, Gr, BernoulliSampler> const *>(raw));
    return mm.release();
}
} // namespace

namespace
{
// The shim of grower kind K in the form c.hist_mode.
template <int K, typename F> void with_form(ref_cfg const &c, F &&f)
{
    switch (c.hist_mode)
    {
    case 1:
        f(static_cast<B200Grower<K, 1> *>(nullptr));
        break;
    case 2:
        f(static_cast<B200Grower<K, 2> *>(nullptr));
        break;
    default:
        f(static_cast<B200Grower<K, 0> *>(nullptr));
        break;
    }
}

template <typename F> void with_shim(ref_cfg const &c, F &&f)
{
    switch (c.grower)
    {
    case 1:
        with_form<1>(c, f);
        break;
    case 2:
        with_form<2>(c, f);
        break;
    default:
        with_form<0>(c, f);
        break;
    }
}

// The validation route the reference's fit loop takes with a device grower
// (src/cli/pipeline.cpp:380-450): after round 0 the booster arms its
// resident validation plane with the initial scores; every round then asks
// it to add the round's tree and report the loss, falling back to the host
// bin-space walk and host loss when it declines.
template <typename Gr>
RefModel *b200_train_valid_with(Dataset const &ds, Dataset const &valid, ref_cfg const &c,
                                float *losses, int32_t *on_device)
{
    Config cfg = make_config(c);
    parallel::set_n_threads(c.n_threads);
    auto mm     = std::make_unique<RefModel>();
    mm->grower  = c.grower;
    mm->booster = make_for_sampler<Gr>(c, cfg);
    IBooster          &b = *mm->booster;
    std::vector<float> es;
    bool               device_eval = false;
    for (uint32_t i = 0; i < c.n_iters; ++i)
    {
        b.update_one_iter(ds);
        if (i == 0)
        {
            auto *raw = mm->booster.get();
            read_init(*mm, dynamic_cast<Booster<MSEObjective, Gr, AllRowsSampler> const *>(raw));
            read_init(*mm,
                      dynamic_cast<Booster<LogLossObjective, Gr, AllRowsSampler> const *>(raw));
            es.assign(valid.n_rows(), mm->init_scores.at(0));
            device_eval = b.begin_resident_validation(valid, std::span<float const>{es});
        }
        std::optional<float> loss;
        if (device_eval)
        {
            device_eval = b.accumulate_last_round_resident(valid, es, loss);
        }
        if (!device_eval)
        {
            b.accumulate_last_round_binned(valid, es);
        }
        losses[i]    = loss.has_value() ? *loss : b.validation_loss(es, valid.labels());
        on_device[i] = loss.has_value() ? 1 : 0;
    }
    harvest<Gr>(*mm, c);
    return mm.release();
}
} // namespace

extern "C" void *ref_b200_train(void const *dsp, ref_cfg const *c)
{
    RefModel *m  = nullptr;
    int const rc = guarded(
        [&]
        {
            auto const &ds = *static_cast<Dataset const *>(dsp);
            with_shim(*c, [&](auto *tag)
                      { m = b200_train_with<std::remove_pointer_t<decltype(tag)>>(ds, *c); });
        });
    return rc == 0 ? m : nullptr;
}

// ref_b200_train with a validation set: per-round losses, and whether each
// came from the device plane.
extern "C" void *ref_b200_train_valid(void const *dsp, void const *vdsp, ref_cfg const *c,
                                      float *losses, int32_t *on_device)
{
    RefModel *m  = nullptr;
    int const rc = guarded(
        [&]
        {
            auto const &ds = *static_cast<Dataset const *>(dsp);
            auto const &vs = *static_cast<Dataset const *>(vdsp);
            with_shim(*c,
                      [&](auto *tag)
                      {
                          m = b200_train_valid_with<std::remove_pointer_t<decltype(tag)>>(
                              ds, vs, *c, losses, on_device);
                      });
        });
    return rc == 0 ? m : nullptr;
}
#endif
