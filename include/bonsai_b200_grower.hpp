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
template <int Kind> class B200Grower
{
  public:
    using Tree = std::conditional_t<Kind == 1, ObliviousTree, DenseTree>;

    explicit B200Grower(TreeConfig const &cfg) : config_(cfg), feature_rng_(cfg.feature_seed)
    {
    }
    B200Grower(B200Grower const &)            = delete;
    B200Grower &operator=(B200Grower const &) = delete;
    ~B200Grower()
    {
        if (plane_ != nullptr)
        {
            bb_plane_destroy(plane_);
        }
    }

    GrowResult<Tree> grow(Dataset const &ds, floats_view grad, floats_view hess,
                          row_index_view rows)
    {
        bind(ds);
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
        c.hist_mode         = 0;
        c.monotone          = mono.empty() ? nullptr : mono.data();
        c.n_monotone        = static_cast<uint32_t>(mono.size());
        c.selected          = selected.data();
        c.n_selected        = static_cast<uint32_t>(selected.size());
        // interaction_constraints as the reference parses them ("0,1" or
        // "0+1" per group): features in groups, group g's at [off[g], off[g+1])
        std::vector<uint32_t> ifeat;
        std::vector<uint32_t> ioff{0};
        for (auto const &entry : config_.interaction_constraints)
        {
            size_t start = 0;
            while (start < entry.size())
            {
                size_t const sep = std::min(entry.find(',', start), entry.find('+', start));
                size_t const end = sep == std::string::npos ? entry.size() : sep;
                if (end > start)
                {
                    ifeat.push_back(static_cast<uint32_t>(std::stoul(entry.substr(start, end - start))));
                }
                start = end + 1;
            }
            ioff.push_back(static_cast<uint32_t>(ifeat.size()));
        }
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
                             std::move(values), std::move(leaf_ids));
        }
        else
        {
            return dense(ds, rows, all, n_nodes, meta, feat, value, left, right, dl, gain,
                         cover, split_bin, std::move(values), std::move(leaf_ids));
        }
    }

    // The booster's seams. The per-row buffers are rebuilt every grow, so
    // recycling is a no-op; the resident and device-validation seams decline,
    // so the booster keeps its host objective and host eval walk.
    void recycle(train_leaf_values, std::vector<node_id_t>) {}
    bool resident_begin(Dataset const &, DeviceObjectiveKind, std::span<float const>, float)
    {
        return false;
    }
    void resident_end(std::span<float>) {}
    bool resident() const
    {
        return false;
    }
    bool eval_begin(Dataset const &, DeviceObjectiveKind, std::span<float const>)
    {
        return false;
    }
    bool eval_accumulate(Tree const &, Dataset const &, float, std::span<float>,
                         std::optional<float> &)
    {
        return false;
    }

  private:
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
                                        train_leaf_values values, std::vector<node_id_t> leaf_ids)
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
        for (size_t r = 0; r < ds.n_rows(); ++r)
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
            bb_plane_destroy(plane_);
            plane_ = nullptr;
        }
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
        b200_rethrow(bb_plane_from_bins(u8 ? static_cast<void const *>(b8.data())
                                           : static_cast<void const *>(b16.data()),
                                        u8 ? 1 : 0, n, static_cast<uint32_t>(F), cuts.data(),
                                        off.data(), &plane_));
        bound_      = &ds;
        bound_rows_ = n;
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
    bb_plane      *plane_      = nullptr;
    Dataset const *bound_      = nullptr;
    size_t         bound_rows_ = 0;
};

using B200DepthwiseGrower = B200Grower<0>;
using B200ObliviousGrower = B200Grower<1>;
using B200LeafwiseGrower  = B200Grower<2>;

static_assert(TreeGrower<B200DepthwiseGrower>);
static_assert(TreeGrower<B200ObliviousGrower>);
static_assert(TreeGrower<B200LeafwiseGrower>);

} // namespace bonsai
