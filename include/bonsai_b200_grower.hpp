// B200DepthwiseGrower, B200ObliviousGrower, B200LeafwiseGrower: the
// reference-side binding of the B200 growers.
//
// C++ growers satisfying bonsai's TreeGrower concept
// (include/bonsai/grower.hpp:54-62) and the booster's grower seams
// (recycle, resident_begin/end, eval_begin/accumulate; booster.hpp:562-676,
// 1008-1021), implemented entirely through the C ABI in bonsai_b200.h. They
// compile against bonsai's own headers, so a maintainer drops this file into
// include/bonsai/cuda/ and registers each beside its Cuda* twin
// (include/bonsai/registry/typelists.hpp:19-22). One grow() call is one
// grow of the reference's grower -- DepthwiseGrower (src/grower_impl.hpp:
// 465-577), ObliviousGrower (:579-720) or LeafwiseGrower (:744-850): the same
// feature draw (std::sample over the ids with a mt19937 seeded by
// feature_seed, as sample_features does, grower_impl.hpp:165-180), the same
// tree (a DenseTree node table, or the ObliviousTree's level splits, leaf
// table, level gains and leaf covers), the same per-row values and leaf ids
// (DenseTree node ids, or leaf-table indices), rows outside the sample
// routed through the finished tree in bin space (route_unsampled,
// grower_impl.hpp:438-461; the level walk, :705-725).
//
// Status codes rethrow as the reference does: BB_ERR_CONFIG as
// bonsai::ConfigError, everything else as std::runtime_error.
#pragma once

#include "bonsai/config/errors.hpp"
#include "bonsai/dataset.hpp"
#include "bonsai/grower.hpp"
#include "bonsai/tree.hpp"
#include "bonsai_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <iterator>
#include <numeric>
#include <optional>
#include <random>
#include <span>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

namespace bonsai
{

inline void b200_rethrow(int rc)
{
    if (rc == BB_OK)
    {
        return;
    }
    std::string const msg = bb_last_error();
    if (rc == BB_ERR_CONFIG)
    {
        throw ConfigError(msg);
    }
    throw std::runtime_error(msg);
}

// Kind: bb_train_cfg.grower -- 0 depthwise, 1 levelwise (oblivious), 2 leafwise.
// Hist: bb_train_cfg.hist_mode -- 0 the plain form (float cells in the CPU
// grower's order: trees bit-identical to it), 1 int8 and 2 int16 quantised
// gradients with exact integer histograms.
template <int Kind, int Hist = 0> class B200Grower
{
  public:
    using Tree = std::conditional_t<Kind == 1, ObliviousTree, DenseTree>;

    // Trees one device booster holds before the resident seam starts a fresh
    // one from the current scores.
    static constexpr uint32_t k_resident_trees = 4096;

    explicit B200Grower(TreeConfig const &cfg) : config_(cfg), feature_rng_(cfg.feature_seed)
    {
    }
    B200Grower(B200Grower const &)            = delete;
    B200Grower &operator=(B200Grower const &) = delete;
    ~B200Grower()
    {
        drop_booster();
        if (vplane_ != nullptr)
        {
            bb_plane_destroy(vplane_);
        }
        if (plane_ != nullptr)
        {
            bb_plane_destroy(plane_);
        }
    }

    GrowResult<Tree> grow(Dataset const &ds, floats_view grad, floats_view hess,
                          row_index_view rows)
    {
        if (res_armed_)
        {
            return resident_grow(ds, rows);
        }
        bind(ds);
        ++host_grows_;
        std::vector<uint32_t> const selected = sample_features(ds.n_features());
        std::vector<int8_t>         mono(config_.monotone_constraints.begin(),
                                         config_.monotone_constraints.end());
        bb_train_cfg c{};
        c.grower            = Kind;
        c.max_leaves        = Kind == 2 ? config_.max_leaves : 0;
        c.objective         = 0;
        c.learning_rate     = 1.0F;
        c.min_child_hess    = config_.min_child_hess;
        c.min_gain_to_split = config_.min_gain_to_split;
        c.lambda_l2         = config_.lambda_l2;
        c.lambda_l1         = config_.lambda_l1;
        c.max_depth         = config_.max_depth;
        c.min_data_in_leaf  = config_.min_data_in_leaf;
        c.hist_mode         = Hist;
        c.monotone          = mono.empty() ? nullptr : mono.data();
        c.n_monotone        = static_cast<uint32_t>(mono.size());
        c.selected          = selected.data();
        c.n_selected        = static_cast<uint32_t>(selected.size());
        std::vector<uint32_t> ifeat;
        std::vector<uint32_t> ioff{0};
        interaction_groups(ifeat, ioff);
        c.interaction_features = ifeat.empty() ? nullptr : ifeat.data();
        c.interaction_offsets  = ioff.data();
        c.n_interaction_groups = static_cast<uint32_t>(ioff.size() - 1);
        size_t const cap    = std::max<uint32_t>(bb_tree_capacity(&c), 1);
        std::vector<uint32_t> feat(cap), left(cap), right(cap), split_bin(cap), meta(3);
        std::vector<float>    value(cap), gain(cap), cover(cap);
        std::vector<uint8_t>  dl(cap);
        size_t const          n = ds.n_rows();
        train_leaf_values     values(n, 0.0F);
        std::vector<node_id_t> leaf_ids(n, 0);
        bool const all = rows.size() == n;
        b200_rethrow(bb_grow_tree(plane_, &c, grad.data(), hess.data(),
                                  all ? nullptr : rows.data(), rows.size(), feat.data(),
                                  value.data(), left.data(), right.data(), dl.data(),
                                  gain.data(), cover.data(), split_bin.data(), meta.data(),
                                  values.data(), leaf_ids.data()));
        size_t const n_nodes = meta[0];
        if constexpr (Kind == 1)
        {
            return oblivious(ds, rows, all, feat, value, left, dl, gain, cover, split_bin,
                             std::move(values), std::move(leaf_ids), true);
        }
        else
        {
            return dense(ds, rows, all, n_nodes, meta, feat, value, left, right, dl, gain,
                         cover, split_bin, std::move(values), std::move(leaf_ids));
        }
    }

    // The booster's seams. The per-row buffers are rebuilt every grow, so
    // recycling is a no-op.
    void recycle(train_leaf_values, std::vector<node_id_t>) {}

    // The resident round (Booster::try_resident_round / resident_round,
    // include/bonsai/booster.hpp:630-676; the engine's resident_begin /
    // resident_finalize / resident_end, include/bonsai/cuda/
    // histogram_engine.hpp:255-268): labels and scores move to the device
    // once, and every later grow() is one round of a device booster
    // (bb_booster_*) -- gradients from the resident objective, the tree, and
    // scores += lr x leaf fused into the round's CUDA graph -- over the rows
    // the booster's sampler passes (handed over with bb_booster_set_rows
    // when they are a sample). grow() then returns the tree with no per-row
    // output, as the reference's resident grow does. Arms for the squared
    // error, logloss and Poisson kinds; declines (the booster keeps its host
    // objective) for any other kind, and for a feature-sampled fit whose
    // feature draws already started on the host.
    bool resident_begin(Dataset const &ds, DeviceObjectiveKind kind,
                        std::span<float const> scores, float learning_rate)
    {
        resident_reset();
        int const obj = kind == DeviceObjectiveKind::mse       ? 0
                        : kind == DeviceObjectiveKind::logloss ? 1
                        : kind == DeviceObjectiveKind::poisson ? 3
                                                               : -1;
        if (obj < 0 || scores.size() != ds.n_rows() || ds.labels().size() != ds.n_rows() ||
            (config_.feature_fraction < 1.0F && host_grows_ > 0))
        {
            return false;
        }
        bind(ds);
        res_ds_        = &ds;
        res_objective_ = obj;
        res_lr_        = learning_rate;
        res_scores_.assign(scores.begin(), scores.end());
        res_armed_ = true;
        return true;
    }
    void resident_end(std::span<float> scores)
    {
        if (res_armed_)
        {
            pull_scores();
            std::copy_n(res_scores_.begin(), std::min(scores.size(), res_scores_.size()),
                        scores.begin());
        }
        resident_reset();
    }
    bool resident() const
    {
        return res_armed_;
    }

    // The device validation plane (Booster::begin_resident_validation /
    // accumulate_last_round_resident, booster.hpp:1008-1021; the engine's
    // eval_begin / eval_accumulate, src/cuda/detail/device_context.cu:
    // 1666-1760). Armed after the resident round that precedes it: that
    // round's tree is added to the given scores here (a bin-space predict of
    // the one tree, lr x leaf added in float as the device walk adds it) and
    // its loss is left to the host; from the next round on, every round walks
    // its tree over the validation plane and records its loss on the device.
    bool eval_begin(Dataset const &valid, DeviceObjectiveKind kind,
                    std::span<float const> scores)
    {
        eval_armed_ = false;
        if (!res_armed_ || booster_ == nullptr || res_trees_ == 0 ||
            valid.labels().size() != valid.n_rows() || scores.size() != valid.n_rows() ||
            kind == DeviceObjectiveKind::none)
        {
            return false;
        }
        bind_valid(valid);
        uint32_t const        t   = res_trees_ - 1;
        uint32_t const        cap = bb_booster_tree_capacity(booster_);
        std::vector<uint32_t> feat(cap), left(cap), right(cap), split_bin(cap), meta(3);
        std::vector<float>    value(cap), gain(cap), cover(cap);
        std::vector<uint8_t>  dl(cap);
        b200_rethrow(bb_booster_tree(booster_, t, feat.data(), value.data(), left.data(),
                                     right.data(), dl.data(), gain.data(), cover.data(),
                                     split_bin.data(), meta.data()));
        uint32_t const     root = 0;
        std::vector<float> add(valid.n_rows());
        b200_rethrow(bb_predict(vplane_, 1, &root, meta[0], feat.data(), split_bin.data(),
                                left.data(), right.data(), dl.data(), value.data(), res_lr_,
                                0.0F, add.data()));
        eval_first_.resize(valid.n_rows());
        for (size_t i = 0; i < eval_first_.size(); ++i)
        {
            eval_first_[i] = scores[i] + add[i];
        }
        b200_rethrow(bb_booster_eval_arm(booster_, vplane_, valid.labels().data(),
                                         eval_first_.data()));
        eval_armed_   = true;
        eval_pending_ = true;
        return true;
    }
    bool eval_accumulate(Tree const &, Dataset const &valid, float, std::span<float> scores_out,
                         std::optional<float> &loss)
    {
        if (!eval_armed_)
        {
            if (!eval_handoff_.empty() && eval_handoff_.size() == scores_out.size())
            {
                // the device booster was replaced: its validation scores up to
                // the last round go back to the host, which adds this round's
                std::copy(eval_handoff_.begin(), eval_handoff_.end(), scores_out.begin());
                eval_handoff_.clear();
            }
            return false;
        }
        if (eval_pending_)
        {
            std::copy_n(eval_first_.begin(), std::min(scores_out.size(), eval_first_.size()),
                        scores_out.begin());
            eval_pending_ = false;
            loss.reset();
            return true;
        }
        (void)valid;
        uint32_t n = 0;
        b200_rethrow(bb_booster_eval_losses(booster_, nullptr, 0, &n));
        if (n == 0)
        {
            return false;
        }
        std::vector<float> losses(n);
        b200_rethrow(bb_booster_eval_losses(booster_, losses.data(), n, &n));
        loss = losses[n - 1];
        return true;
    }

  private:
    // One resident round over `rows` (every row, or the sampler's rows).
    GrowResult<Tree> resident_grow(Dataset const &ds, row_index_view rows)
    {
        bool const all = rows.size() == ds.n_rows();
        if (booster_ != nullptr && (external_ == all || res_trees_ == k_resident_trees))
        {
            // another row mode, or a full tree store: a fresh device booster
            // continues from the current scores
            pull_scores();
            drop_booster();
        }
        if (booster_ == nullptr)
        {
            make_booster(ds, !all);
        }
        if (!all)
        {
            b200_rethrow(bb_booster_set_rows(booster_, rows.data(), rows.size()));
        }
        b200_rethrow(bb_booster_update(booster_, 1));
        b200_rethrow(bb_booster_sync(booster_));
        uint32_t const        t   = res_trees_++;
        uint32_t const        cap = bb_booster_tree_capacity(booster_);
        std::vector<uint32_t> feat(cap), left(cap), right(cap), split_bin(cap), meta(3);
        std::vector<float>    value(cap), gain(cap), cover(cap);
        std::vector<uint8_t>  dl(cap);
        b200_rethrow(bb_booster_tree(booster_, t, feat.data(), value.data(), left.data(),
                                     right.data(), dl.data(), gain.data(), cover.data(),
                                     split_bin.data(), meta.data()));
        if constexpr (Kind == 1)
        {
            return oblivious(ds, rows, true, feat, value, left, dl, gain, cover, split_bin, {},
                             {}, false);
        }
        else
        {
            return dense(ds, rows, true, meta[0], meta, feat, value, left, right, dl, gain,
                         cover, split_bin, {}, {});
        }
    }

    void make_booster(Dataset const &ds, bool external)
    {
        std::vector<int8_t> mono(config_.monotone_constraints.begin(),
                                 config_.monotone_constraints.end());
        bb_train_cfg c{};
        c.objective         = res_objective_;
        c.learning_rate     = res_lr_;
        c.min_child_hess    = config_.min_child_hess;
        c.min_gain_to_split = config_.min_gain_to_split;
        c.lambda_l2         = config_.lambda_l2;
        c.lambda_l1         = config_.lambda_l1;
        c.max_depth         = config_.max_depth;
        c.min_data_in_leaf  = config_.min_data_in_leaf;
        c.hist_mode         = Hist;
        c.seed              = 0;
        c.monotone          = mono.empty() ? nullptr : mono.data();
        c.n_monotone        = static_cast<uint32_t>(mono.size());
        c.use_graph         = 1;
        c.grower            = Kind;
        c.max_leaves        = Kind == 2 ? config_.max_leaves : 0;
        c.feature_fraction  = config_.feature_fraction;
        c.feature_seed      = config_.feature_seed;
        c.external_sample   = external ? 1 : 0;
        std::vector<uint32_t> ifeat;
        std::vector<uint32_t> ioff{0};
        interaction_groups(ifeat, ioff);
        c.interaction_features = ifeat.empty() ? nullptr : ifeat.data();
        c.interaction_offsets  = ioff.data();
        c.n_interaction_groups = static_cast<uint32_t>(ioff.size() - 1);
        b200_rethrow(bb_booster_create(plane_, ds.labels().data(), res_scores_.data(), &c,
                                       k_resident_trees, &booster_));
        if (!ds.weights().empty())
        {
            b200_rethrow(bb_booster_set_weights(booster_, ds.weights().data()));
        }
        external_  = external;
        res_trees_ = 0;
    }

    // The device booster's scores into res_scores_ (and, with a validation
    // plane armed, its validation scores for the host to continue from).
    void pull_scores()
    {
        if (booster_ == nullptr)
        {
            return;
        }
        b200_rethrow(bb_booster_scores(booster_, res_scores_.data()));
        if (eval_armed_)
        {
            eval_handoff_.resize(eval_first_.size());
            b200_rethrow(bb_booster_eval_scores(booster_, eval_handoff_.data()));
            eval_armed_ = false;
        }
    }

    void drop_booster()
    {
        if (booster_ != nullptr)
        {
            bb_booster_destroy(booster_);
            booster_ = nullptr;
        }
    }

    void resident_reset()
    {
        drop_booster();
        res_armed_    = false;
        res_trees_    = 0;
        eval_armed_   = false;
        eval_pending_ = false;
        eval_handoff_.clear();
    }

    void interaction_groups(std::vector<uint32_t> &ifeat, std::vector<uint32_t> &ioff) const
    {
        // interaction_constraints as the reference parses them ("0,1" or
        // "0+1" per group): features in groups, group g's at [off[g], off[g+1])
        for (auto const &entry : config_.interaction_constraints)
        {
            size_t start = 0;
            while (start < entry.size())
            {
                size_t const sep = std::min(entry.find(',', start), entry.find('+', start));
                size_t const end = sep == std::string::npos ? entry.size() : sep;
                if (end > start)
                {
                    ifeat.push_back(
                        static_cast<uint32_t>(std::stoul(entry.substr(start, end - start))));
                }
                start = end + 1;
            }
            ioff.push_back(static_cast<uint32_t>(ifeat.size()));
        }
    }

    GrowResult<DenseTree> dense(Dataset const &ds, row_index_view rows, bool all, size_t n_nodes,
                                std::vector<uint32_t> const &meta,
                                std::vector<uint32_t> const &feat, std::vector<float> const &value,
                                std::vector<uint32_t> const &left,
                                std::vector<uint32_t> const &right,
                                std::vector<uint8_t> const &dl, std::vector<float> const &gain,
                                std::vector<float> const     &cover,
                                std::vector<uint32_t> const  &split_bin,
                                train_leaf_values values, std::vector<node_id_t> leaf_ids)
    {
        DenseTree::Nodes nodes(n_nodes);
        for (size_t i = 0; i < n_nodes; ++i)
        {
            nodes[i] = feat[i] == DenseTree::k_leaf_flag
                           ? DenseTree::leaf(value[i])
                           : DenseTree::internal(feat[i], value[i], left[i], right[i],
                                                 dl[i] != 0);
        }
        if (!all)
        {
            route_unsampled(ds, nodes, split_bin, rows, values, leaf_ids);
        }
        return {.tree     = DenseTree(std::move(nodes), {.depth = meta[1], .n_leaves = meta[2]},
                                      std::vector<float>(gain.begin(), gain.begin() + n_nodes),
                                      std::vector<float>(cover.begin(), cover.begin() + n_nodes)),
                .values   = std::move(values),
                .leaf_ids = std::move(leaf_ids)};
    }

    // The levelwise tree comes back perfect and in level order (level L
    // starts at node 2^L - 1, leaves in the reference's path order): each
    // level's split, gain and bin from its first node, the leaf table and
    // leaf covers from the last level; a leaf id becomes its table index.
    GrowResult<ObliviousTree> oblivious(Dataset const &ds, row_index_view rows, bool all,
                                        std::vector<uint32_t> const &feat,
                                        std::vector<float> const    &value,
                                        std::vector<uint32_t> const &left,
                                        std::vector<uint8_t> const  &dl,
                                        std::vector<float> const    &gain,
                                        std::vector<float> const    &cover,
                                        std::vector<uint32_t> const &split_bin,
                                        train_leaf_values values, std::vector<node_id_t> leaf_ids,
                                        bool per_row)
    {
        ObliviousTree::LevelSplits splits;
        std::vector<float>         level_gains;
        std::vector<bin_id_t>      level_bins;
        size_t                     idx = 0;
        while (feat[idx] != DenseTree::k_leaf_flag)
        {
            splits.push_back({.feature_id   = static_cast<feature_id_t>(feat[idx]),
                              .threshold    = value[idx],
                              .default_left = dl[idx] != 0});
            level_gains.push_back(gain[idx]);
            level_bins.push_back(static_cast<bin_id_t>(split_bin[idx]));
            idx = left[idx];
        }
        size_t const       first = (size_t{1} << splits.size()) - 1;
        size_t const       n_lf  = size_t{1} << splits.size();
        std::vector<float> table(value.begin() + first, value.begin() + first + n_lf);
        std::vector<float> covers(cover.begin() + first, cover.begin() + first + n_lf);
        size_t             j = 0;
        for (size_t r = 0; per_row && r < ds.n_rows(); ++r)
        {
            if (all || (j < rows.size() && rows[j] == r))
            {
                ++j;
                leaf_ids[r] = static_cast<node_id_t>(leaf_ids[r] - first);
                continue;
            }
            size_t index = 0;
            for (size_t lvl = 0; lvl < splits.size(); ++lvl)
            {
                auto const    &sp   = splits[lvl];
                auto const     last = static_cast<bin_id_t>(ds.n_bins(sp.feature_id) - 1);
                bin_id_t const b    = ds.bin_at(sp.feature_id, static_cast<row_id_t>(r));
                index = (index << 1U) |
                        (routes_left(b, last, level_bins[lvl], sp.default_left) ? 0U : 1U);
            }
            values[r]   = table[index];
            leaf_ids[r] = static_cast<node_id_t>(index);
        }
        return {.tree     = ObliviousTree(std::move(splits), std::move(table),
                                          std::move(level_gains), std::move(covers)),
                .values   = std::move(values),
                .leaf_ids = std::move(leaf_ids)};
    }

    // The device plane for ds, built once per Dataset from its host columns.
    void bind(Dataset const &ds)
    {
        if (plane_ != nullptr && bound_ == &ds && bound_rows_ == ds.n_rows())
        {
            return;
        }
        if (plane_ != nullptr)
        {
            drop_booster(); // a device booster reads the plane
            bb_plane_destroy(plane_);
            plane_ = nullptr;
        }
        plane_      = make_plane(ds);
        bound_      = &ds;
        bound_rows_ = ds.n_rows();
    }

    // The validation plane, built once per validation Dataset.
    void bind_valid(Dataset const &ds)
    {
        if (vplane_ != nullptr && vbound_ == &ds && vbound_rows_ == ds.n_rows())
        {
            return;
        }
        if (vplane_ != nullptr)
        {
            bb_plane_destroy(vplane_);
            vplane_ = nullptr;
        }
        vplane_      = make_plane(ds);
        vbound_      = &ds;
        vbound_rows_ = ds.n_rows();
    }

    static bb_plane *make_plane(Dataset const &ds)
    {
        size_t const          n = ds.n_rows();
        size_t const          F = ds.n_features();
        std::vector<float>    cuts;
        std::vector<uint32_t> off(F + 1, 0);
        for (size_t f = 0; f < F; ++f)
        {
            auto const c = ds.cuts(static_cast<feature_id_t>(f));
            cuts.insert(cuts.end(), c.begin(), c.end());
            off[f + 1] = static_cast<uint32_t>(cuts.size());
        }
        bool const            u8 = ds.bins_are_u8();
        std::vector<uint8_t>  b8;
        std::vector<uint16_t> b16;
        if (u8)
        {
            b8.resize(n * F);
        }
        else
        {
            b16.resize(n * F);
        }
        for (size_t f = 0; f < F; ++f)
        {
            ds.visit_bins(f,
                          [&](auto bins)
                          {
                              for (size_t r = 0; r < n; ++r)
                              {
                                  if (u8)
                                  {
                                      b8[(f * n) + r] = static_cast<uint8_t>(bins[r]);
                                  }
                                  else
                                  {
                                      b16[(f * n) + r] = static_cast<uint16_t>(bins[r]);
                                  }
                              }
                          });
        }
        bb_plane *out = nullptr;
        b200_rethrow(bb_plane_from_bins(u8 ? static_cast<void const *>(b8.data())
                                           : static_cast<void const *>(b16.data()),
                                        u8 ? 1 : 0, n, static_cast<uint32_t>(F), cuts.data(),
                                        off.data(), &out));
        return out;
    }

    std::vector<uint32_t> sample_features(size_t n_features)
    {
        std::vector<uint32_t> all(n_features);
        std::iota(all.begin(), all.end(), uint32_t{0});
        float const fraction = config_.feature_fraction;
        if (fraction >= 1.0F || n_features <= 1)
        {
            return all;
        }
        auto const k = std::max<size_t>(
            1, static_cast<size_t>(std::ceil(fraction * static_cast<float>(n_features))));
        std::vector<uint32_t> selected;
        selected.reserve(k);
        std::sample(all.begin(), all.end(), std::back_inserter(selected), k, feature_rng_);
        return selected;
    }

    static void route_unsampled(Dataset const &ds, DenseTree::Nodes const &nodes,
                                std::vector<uint32_t> const &split_bin, row_index_view rows,
                                train_leaf_values &values, std::vector<node_id_t> &leaf_ids)
    {
        size_t j = 0;
        for (size_t r = 0; r < ds.n_rows(); ++r)
        {
            if (j < rows.size() && rows[j] == r)
            {
                ++j;
                continue;
            }
            node_id_t idx = 0;
            while (!DenseTree::is_leaf(nodes[idx]))
            {
                auto const &nd   = nodes[idx];
                auto const  last = static_cast<bin_id_t>(ds.n_bins(nd.feature_id) - 1);
                bin_id_t const b = ds.bin_at(nd.feature_id, r);
                idx = routes_left(b, last, static_cast<bin_id_t>(split_bin[idx]),
                                  nd.default_left)
                          ? nd.left
                          : nd.right;
            }
            values[r]   = nodes[idx].threshold_or_value;
            leaf_ids[r] = idx;
        }
    }

    TreeConfig     config_;
    std::mt19937   feature_rng_;
    bb_plane      *plane_       = nullptr;
    Dataset const *bound_       = nullptr;
    size_t         bound_rows_  = 0;
    bb_plane      *vplane_      = nullptr;
    Dataset const *vbound_      = nullptr;
    size_t         vbound_rows_ = 0;
    size_t         host_grows_  = 0; // grows with host gradients so far
    // the resident round
    bool               res_armed_     = false;
    Dataset const     *res_ds_        = nullptr;
    int                res_objective_ = 0;
    float              res_lr_        = 0.1F;
    std::vector<float> res_scores_;   // scores at arming, or when the booster was last replaced
    bb_booster        *booster_       = nullptr;
    bool               external_      = false;
    uint32_t           res_trees_     = 0; // trees in the current device booster
    // the validation plane
    bool               eval_armed_   = false;
    bool               eval_pending_ = false; // the arming round's scores not yet handed back
    std::vector<float> eval_first_;
    std::vector<float> eval_handoff_;
};

// The plain form: trees bit-identical to the CPU growers'.
using B200DepthwiseGrower = B200Grower<0>;
using B200ObliviousGrower = B200Grower<1>;
using B200LeafwiseGrower  = B200Grower<2>;
// The quantised forms (int8, int16 gradients; exact integer histograms).
using B200DepthwiseGrowerInt8  = B200Grower<0, 1>;
using B200ObliviousGrowerInt8  = B200Grower<1, 1>;
using B200LeafwiseGrowerInt8   = B200Grower<2, 1>;
using B200DepthwiseGrowerInt16 = B200Grower<0, 2>;
using B200ObliviousGrowerInt16 = B200Grower<1, 2>;
using B200LeafwiseGrowerInt16  = B200Grower<2, 2>;

static_assert(TreeGrower<B200DepthwiseGrower>);
static_assert(TreeGrower<B200ObliviousGrower>);
static_assert(TreeGrower<B200LeafwiseGrower>);
static_assert(TreeGrower<B200DepthwiseGrowerInt8>);

} // namespace bonsai
