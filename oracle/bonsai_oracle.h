/* TEST INFRASTRUCTURE — the oracle. Not part of the product.
 *
 * A plain-C restatement of the reference's CPU algorithm for the CUDA-grower
 * hot path, used only by tests/, the smoke check and bench.py's CPU-baseline
 * leg as the checker. Every function cites the reference file:line it follows
 * (paths within the daniel-m-campos/bonsai project). It is pinned against the
 * reference itself: tests compare it with oracle/_ref/libbonsai_ref.so (the
 * reference's own sources, compiled by oracle/Makefile) and with the golden
 * fixtures under tests/golden/ that the same library produced.
 *
 * Bins are feature-major u16 codes (bins[f * n + r]); u8 datasets are widened.
 * All float/double arithmetic is plain IEEE round-to-nearest with no
 * contraction (built with -ffp-contract=off, as the reference is).
 */
#ifndef BONSAI_ORACLE_H
#define BONSAI_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct
{
    float          min_child_hess;
    float          min_gain_to_split;
    float          lambda_l2;
    float          lambda_l1;
    uint32_t       max_depth;
    uint32_t       min_data_in_leaf;
    uint32_t       max_leaves; /* leafwise only */
    int32_t const *monotone;   /* per-feature +1/-1/0; may be NULL */
    uint32_t       n_monotone;
    int32_t        grower;     /* 0 depthwise, 1 levelwise (oblivious) */
} orc_tree_cfg;

/* One grown tree in the reference's DenseTree layout (tree.hpp:38-45):
 * feature == 0xFFFFFFFF marks a leaf whose value is in value[]. */
typedef struct
{
    uint32_t  cap; /* capacity of every array below */
    uint32_t *feature;
    float    *value;
    uint32_t *left;
    uint32_t *right;
    uint8_t  *default_left;
    float    *gains;
    float    *covers;
    uint32_t *split_bin; /* bin-space split (the grower's bin_id), 0 for leaves */
    uint32_t  n_nodes;
    uint32_t  depth;
    uint32_t  n_leaves;
} orc_tree;

/* BinMapper::transform (src/bin_mapper.cpp:284-291) over row-major X. */
void orc_transform(float const *X, size_t n, size_t F, float const *cuts,
                   uint32_t const *cut_off, uint16_t *bins);

/* Serial-order histogram of one node (src/fill/columns.hpp:31-89 at one
 * thread): hist[2 * (off[j] + b) + {0,1}] for selected feature j. */
void orc_fill(uint16_t const *bins, size_t n, uint32_t const *selected, size_t n_sel,
              uint32_t const *n_bins, float const *grad, float const *hess,
              uint32_t const *rows, size_t n_rows, float *hist);

/* HistogramNodeSplitFinder::find (src/split.cpp:101-162,271-297) on a node's
 * full per-feature histogram set: hist[f] has n_bins[f] cells, f in [0, F);
 * present[f] == 0 marks an unselected (empty) histogram. */
typedef struct
{
    double   gain;
    uint32_t feature;
    uint32_t bin;
    uint8_t  default_left;
    uint8_t  valid;
} orc_split;

orc_split orc_find_split(float const *const *hist, uint32_t const *n_bins,
                         uint8_t const *present, size_t F, size_t n_rows,
                         float tot_g, float tot_h, double lo, double hi,
                         orc_tree_cfg const *cfg);

/* DepthwiseGrower<CpuHistogramEngine>::grow (src/grower_impl.hpp:465-577 with
 * src/step/level.hpp:30-153 and src/step/primitives.hpp:42-374). rows are the
 * sampled rows (ascending); selected the tree's features (ascending).
 * values/leaf_ids receive every row's leaf value and node id. Returns 0, or
 * -1 when the tree outgrows t->cap. */
int orc_grow_depthwise(uint16_t const *bins, size_t n, size_t F, uint32_t const *n_bins,
                       float const *cuts, uint32_t const *cut_off, float const *grad,
                       float const *hess, uint32_t const *rows, size_t n_rows,
                       uint32_t const *selected, size_t n_sel, orc_tree_cfg const *cfg,
                       orc_tree *t, float *values, uint32_t *leaf_ids);

/* Booster::update_one_iter rounds (include/bonsai/booster.hpp:500-592) with
 * the depthwise grower over all rows: objective 0 = mse
 * (src/objective.cpp:44-58,76-83), 1 = logloss (:86-101,124-131).
 * trees[i] receives round i's tree; scores (n) the final training scores. */
int orc_train_depthwise(uint16_t const *bins, size_t n, size_t F,
                        uint32_t const *n_bins, float const *cuts,
                        uint32_t const *cut_off, float const *labels, int objective,
                        uint32_t n_iters, float learning_rate, orc_tree_cfg const *cfg,
                        orc_tree *trees, float *init_score, float *scores);

/* Objective gradients (src/objective.cpp:44-58 mse, :86-101 logloss). */
void orc_gradients(int objective, float const *scores, float const *labels, size_t n,
                   float *grad, float *hess);

/* init_score (src/objective.cpp:76-83 mse, :124-131 logloss). */
float orc_init_score(int objective, float const *labels, size_t n);

/* Bin-space ensemble predict (booster.hpp:831-845 with detail/bin_walk.hpp):
 * out[r] = init + (sum over trees of leaf(r)) * lr, summed in tree order. */
void orc_predict_binned(uint16_t const *bins, size_t n, uint32_t const *n_bins,
                        orc_tree const *trees, size_t n_trees, float init, float lr,
                        float *out);

#ifdef __cplusplus
}
#endif

#endif
