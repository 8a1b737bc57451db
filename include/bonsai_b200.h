/* bonsai_b200 — C ABI of the B200-native CUDA growers.
 *
 * The drop-in boundary for the reference's CUDA grower surface
 * (daniel-m-campos/bonsai). Plain pointers and sizes only. Every call returns
 * 0 on success or a nonzero status; bb_last_error() then holds the message,
 * "cuda: <what>: <detail>" for CUDA failures (the reference's check() text,
 * src/cuda/detail/device_buffer.cuh:96-103) and the remedy text for capacity
 * refusals (the reference's ConfigError, src/cuda/detail/device_context.cu:
 * 60-87). Status BB_DECLINED means "not handled on the device": the caller
 * falls back to its host path, as the reference's nullptr/false declines do
 * (src/cuda/histogram_engine.cu:336-340, src/cuda/predict.cu:151-170).
 *
 * Each entry point names the reference interface it replaces.
 */
#ifndef BONSAI_B200_H
#define BONSAI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

enum
{
    BB_OK          = 0,
    BB_ERR_CUDA    = 1, /* a CUDA runtime failure */
    BB_ERR_CONFIG  = 2, /* a capacity / configuration refusal */
    BB_ERR_ARG     = 3, /* an invalid argument */
    BB_DECLINED    = 4  /* not handled here; use the host path */
};

typedef struct bb_plane   bb_plane;   /* a device-resident binned dataset */
typedef struct bb_booster bb_booster; /* a device-resident boosting fit */

/* Last error message of the calling thread ("" when none). */
char const *bb_last_error(void);

/* 1 when a usable CUDA device is present.
 * Replaces bonsai::cuda_available (include/bonsai/cuda/histogram_engine.hpp:22). */
int bb_available(void);

/* Select the device for the calling thread's later calls.
 * Replaces bonsai::cuda_select_device (histogram_engine.hpp:31). */
int bb_select_device(uint32_t device_id);

/* ---- ingest: bin application -------------------------------------------
 * Bins a row-major float32 matrix (n_rows x n_feats) against per-feature
 * cuts (cuts[cut_off[f] .. cut_off[f+1]), strictly increasing, the last two
 * FLT_MAX and +inf) into a device plane of feature-major u8 codes (u16 when
 * any feature has more than 256 bins). x_on_device selects whether X is a
 * device pointer (read, not retained) or host memory (streamed up in 64 MB
 * chunks). Bin codes are bit-identical to BinMapper::transform.
 * Replaces bonsai::cuda_ingest(features_view, BinMappers) and
 * cuda_ingest_device(DeviceMatrix, BinMappers) (histogram_engine.hpp:41-68). */
int bb_ingest(float const *X, uint64_t n_rows, uint32_t n_feats, int x_on_device,
              float const *cuts, uint32_t const *cut_off, bb_plane **out);

/* Per-feature cuts fitted on the device from a working set S (n_rows x n_feats
 * row-major float32, NaN allowed; host memory, or device memory when
 * s_on_device): each column's NaN-free values sorted, run-length encoded,
 * and cut by the reference's rules for max_bin (every distinct value within
 * the budget of max_bin - 2 cuts, the count-weighted greedy walk when a
 * value is at least a mean bin, else the quantile stride), closed by FLT_MAX
 * and +inf -- the cuts BinMapper::from_sample gives the same working set
 * (src/bin_mapper.cpp:159-252). Outputs to host: cuts (cuts_cap >=
 * n_feats x max_bin suffices) and cut_off (n_feats + 1). The row sample for
 * tall data is the caller's (the reference draws one shared sample,
 * src/bin_mappers.cpp:31-44). Replaces the host fit behind cuda_ingest's
 * mappers (the reference's ingest_fit phase). */
int bb_fit_cuts(float const *S, uint64_t n_rows, uint32_t n_feats, int s_on_device,
                uint32_t max_bin, float *cuts, uint32_t cuts_cap, uint32_t *cut_off);

/* A plane from codes already binned on the host: feature-major codes
 * (bins[f * n_rows + r], u8 when is_u8 else u16), each below its feature's bin
 * count (checked), and the cuts they were binned with. Replaces the engine
 * adopting a host Dataset's columns (CudaDeviceContext's ensure_dataset,
 * src/cuda/detail/device_context.cuh:55-62, device_context.cu:499-520). */
int bb_plane_from_bins(void const *bins, int is_u8, uint64_t n_rows, uint32_t n_feats,
                       float const *cuts, uint32_t const *cut_off, bb_plane **out);

/* 1 when the plane stores u8 codes, 0 for u16. */
int bb_plane_is_u8(bb_plane const *plane);

/* Copies the plane's codes to host, feature-major, widened to u16
 * (out[f * n_rows + r]). Replaces IngestPlane::materialize
 * (include/bonsai/dataset.hpp:44-45). */
int bb_plane_download(bb_plane const *plane, uint16_t *out);

void bb_plane_destroy(bb_plane *plane);

/* A request plane for serving: the mappers of `like` (its cuts, bin counts
 * and code width) and device room for up to max_rows rows, allocated once.
 * It holds no rows until bb_plane_refill. No counterpart in the reference,
 * whose serving path ingests a fresh device plane per request (cuda_ingest,
 * include/bonsai/cuda/histogram_engine.hpp:41-68). */
int bb_plane_create_like(bb_plane const *like, uint64_t max_rows, bb_plane **out);

/* Bins a new batch of n_rows (1..max_rows) row-major float32 rows into a
 * request plane, replacing its rows, with no device allocation: host X goes
 * up through the plane's own staging buffer. Returns when the plane is
 * ready. Predict and SHAP plans made against `like` score it directly.
 * More rows than the plane was made for: BB_ERR_CONFIG. */
int bb_plane_refill(bb_plane *plane, float const *X, uint64_t n_rows, int x_on_device);

/* ---- training ------------------------------------------------------------ */

/* The TreeConfig / BoosterConfig keys the device path reads
 * (include/bonsai/config/tree_config.hpp:9-29, booster_config.hpp:8-24). */
typedef struct
{
    int32_t        objective;  /* 0 mse, 1 logloss, 2 softmax (MulticlassBooster:
                                  n_classes trees per round, round-major), 3 poisson
                                  (log link, raw scores clamped to +-30) */
    float          learning_rate;
    float          min_child_hess;
    float          min_gain_to_split;
    float          lambda_l2;
    float          lambda_l1;
    uint32_t       max_depth;  /* <= 8 */
    uint32_t       min_data_in_leaf;
    int32_t        hist_mode;  /* 0 exact (plain), 1 int8 quantised, 2 int16 quantised
                                  (two-word cells; finer, slower) */
    uint64_t       seed;       /* quantised stochastic-rounding seed */
    int8_t const  *monotone;   /* per-feature +1/-1/0, or NULL */
    uint32_t       n_monotone;
    uint32_t const *selected;  /* ascending feature ids, or NULL for all */
    uint32_t       n_selected;
    int32_t        use_graph;  /* capture one boosting round as a CUDA graph */
    int32_t        record_leaf_ids; /* keep each row's leaf id of the last tree */
    int32_t        grower;     /* 0 depthwise (DepthwiseGrower), 1 levelwise
                                  (ObliviousGrower: one split per level over the
                                  whole frontier, src/grower_impl.hpp:579-720),
                                  2 leafwise (LeafwiseGrower: best-first, one
                                  node per heap pop, :744-850; the host keeps the
                                  heap, so its rounds are not graph-captured) */
    uint32_t       max_leaves; /* leafwise: 1..512 (0: 2^max_depth, depth <= 9);
                                  max_depth <= 255 caps its depth */
    uint32_t       n_classes;  /* objective 2 (softmax): 2..16 */
    /* interaction constraints (TreeConfig::interaction_constraints): group g
     * holds interaction_features[interaction_offsets[g] ..
     * interaction_offsets[g + 1]); a node splits only on features of a group
     * containing every feature on its path, or on its path's only feature
     * (src/grower_impl.hpp:114-160). At most 64 non-empty groups;
     * n_interaction_groups 0: unconstrained. Depthwise and leafwise only. */
    uint32_t const *interaction_features;
    uint32_t const *interaction_offsets; /* n_interaction_groups + 1 */
    uint32_t       n_interaction_groups;
    /* sampler.subsample (BernoulliSampler, src/sampler.cpp:27-55) and
     * booster_config.random_seed (booster_config.hpp:12, the reference's
     * default is 42): a resident booster with 0 < subsample < 1 grows each
     * tree over the rows std::bernoulli_distribution(subsample) keeps,
     * drawn from std::mt19937(random_seed) row by row and tree by tree as
     * the reference's booster draws them; every row's score still takes the
     * tree. 0 (a zeroed config) or >= 1 keeps every row; negative values are
     * refused. bb_grow_tree ignores both: its caller passes the rows. */
    float          subsample;
    uint32_t       random_seed;
    /* tree_config.feature_fraction and .feature_seed (tree_config.hpp:15,19;
     * the reference's default seed is 2): a resident booster with
     * 0 < feature_fraction < 1 grows each tree over max(1, ceil(fraction x
     * n_feats)) features drawn by std::sample from std::mt19937(feature_seed)
     * as sample_features does (src/grower_impl.hpp:163-180), tree by tree
     * (class tree by class tree in a softmax round). 0 (a zeroed config) or
     * >= 1 keeps every feature; negative values and a feature_fraction < 1
     * with `selected` are refused. bb_grow_tree ignores both: its caller
     * passes the selection. */
    float          feature_fraction;
    uint32_t       feature_seed;
    /* 1: the caller draws each round's rows on the host and hands them over
     * with bb_booster_set_rows before the round (the rows the reference's
     * Booster passes to grow() in its resident round, booster.hpp:664-676,
     * from its own sampler); subsample and random_seed are then unused.
     * Single-output objectives, unsharded fits. */
    int32_t        external_sample;
    /* The quantised histogram build's CTAs per mirror tile (a persistent
     * grid over the level's row chunks): 0 picks the default (one per SM,
     * fewer for a small dataset); bonsai_b200.autotune times candidates and
     * caches the fastest per shape. Results do not depend on it (the
     * quantised cells are order-free integer sums). No reference key: the
     * reference's launch shapes are fixed. */
    uint32_t       hist_ctas;
} bb_train_cfg;

/* A device-resident boosting fit over the plane: labels (host, n_rows) and
 * the scores stay on the device; every round derives (g, h) on the device,
 * grows a depthwise tree and fuses scores += lr * leaf into the grow.
 * init_scores (host, n_rows) may be NULL: the objective's init_score
 * (src/objective.cpp:76-83, :124-131, :293-308) is then used.
 * Replaces Booster<Obj, DepthwiseGrower<CudaHistogramEngine>, AllRows> with
 * the resident round armed (include/bonsai/booster.hpp:630-676) and the
 * engine's resident_begin (histogram_engine.hpp:251-253). */
int bb_booster_create(bb_plane const *plane, float const *labels,
                      float const *init_scores, bb_train_cfg const *cfg,
                      uint32_t max_trees, bb_booster **out);

/* Per-row sample weights for the fit (Dataset::weights, include/bonsai/
 * dataset.hpp:73,86): weights (host, n_rows) scale every round's gradient
 * and hessian, each by one float multiply, as Booster::update_one_iter
 * (include/bonsai/booster.hpp:546-555) and the reference's device gradient
 * kernel (src/cuda/detail/kernels.cuh:1001-1006) do; the initial scores stay
 * unweighted, as the reference's are. NULL returns to the unweighted fit.
 * Before the first round only (BB_ERR_ARG after). A sharded fit sets each
 * shard's weights on its own rank. */
int bb_booster_set_weights(bb_booster *b, float const *weights);

/* The rows the next round grows over, for a booster created with
 * external_sample: n_rows ascending row ids (host), every row's score still
 * taking the tree. Called once before each round (each bb_booster_update of
 * one round); a round without rows is refused. Replaces the row list the
 * reference's resident round passes to its grower (Booster::resident_round,
 * include/bonsai/booster.hpp:664-676). */
int bb_booster_set_rows(bb_booster *b, uint32_t const *rows, uint64_t n_rows);

/* Many boosters, one launch per round: the boosters' round graphs become
 * the child graphs of one parent graph with no edges between them, so one
 * cudaGraphLaunch runs a round of every booster, concurrently. Each booster
 * must run its rounds as a CUDA graph (use_graph; a leafwise round is not
 * captured) with no row or feature sampling, unsharded and not truncated;
 * others are refused (BB_ERR_CONFIG). The boosters must outlive the batch.
 * bb_batch_update runs n_rounds rounds of every booster after any work
 * already queued on their streams, and orders their later calls after it;
 * their trees and scores are read with bb_booster_tree / bb_booster_scores
 * as usual, and equal the same rounds run booster by booster. No
 * counterpart in the reference, which fits one booster per device
 * (include/bonsai/config/sections/parallel.hpp:10-12). */
typedef struct bb_batch bb_batch;
int  bb_batch_create(bb_booster *const *boosters, uint32_t n, bb_batch **out);
int  bb_batch_update(bb_batch *batch, uint32_t n_rounds);
int  bb_batch_sync(bb_batch *batch);
/* Device time of the last bb_batch_update, in milliseconds. */
int  bb_batch_last_ms(bb_batch const *batch, float *ms);
void bb_batch_destroy(bb_batch *batch);

/* Runs n_iters more rounds (asynchronous; bb_booster_sync waits). */
int bb_booster_update(bb_booster *b, uint32_t n_iters);
int bb_booster_sync(bb_booster *b);

int   bb_booster_n_trees(bb_booster const *b, uint32_t *n);
float bb_booster_init_score(bb_booster const *b);
/* Nodes per tree slot (2^(max_depth+1) - 1). */
uint32_t bb_booster_tree_capacity(bb_booster const *b);

/* Copies tree t in the reference's DenseTree layout (tree.hpp:38-45):
 * feature == 0xFFFFFFFF marks a leaf holding value; internal nodes hold
 * the threshold cuts[feature][split_bin]. Arrays hold capacity entries;
 * meta = (n_nodes, depth, n_leaves). */
int bb_booster_tree(bb_booster const *b, uint32_t t, uint32_t *feature, float *value,
                    uint32_t *left, uint32_t *right, uint8_t *default_left,
                    float *gain, float *cover, uint32_t *split_bin, uint32_t *meta);

/* Trees first .. first + count - 1 at once (one copy per array): tree
 * first + i in entries [i * capacity, (i + 1) * capacity) of each array and
 * its meta in [3 i, 3 i + 3). The model download of a whole fit (the
 * reference's save after training, src/io/model.cpp:158-387) in nine copies
 * instead of nine per tree. */
int bb_booster_trees(bb_booster const *b, uint32_t first, uint32_t count, uint32_t *feature,
                     float *value, uint32_t *left, uint32_t *right, uint8_t *default_left,
                     float *gain, float *cover, uint32_t *split_bin, uint32_t *meta);

/* The training scores (host, n_rows). Replaces resident_end
 * (histogram_engine.hpp:262). */
int bb_booster_scores(bb_booster const *b, float *out);

/* Per-row leaf node id of the last tree (host, n_rows); needs
 * record_leaf_ids set at creation. */
int bb_booster_leaf_ids(bb_booster const *b, uint32_t *out);

/* Device time of the last bb_booster_update, in milliseconds. */
int bb_booster_last_ms(bb_booster const *b, float *ms);

/* Arms the booster's validation plane: valid is a plane binned with the
 * training plane's cuts (it must outlive the booster), labels its host labels
 * (class ids for softmax), init_scores its starting raw scores (host,
 * n_valid x K row-major) or NULL for the booster's initial scores. From the
 * next round on, every round walks its new tree(s) over the plane, adds
 * lr x leaf to the validation scores and records the round's loss on the
 * device -- mean squared error, logloss, or softmax cross-entropy, by the
 * booster's objective -- inside the round's CUDA graph, with no host round
 * trip. Re-arming starts a new loss record. A row-sharded booster refuses
 * (BB_ERR_CONFIG). Replaces the eval plane (CudaDeviceContext::eval_begin /
 * eval_accumulate, src/cuda/detail/device_context.cu:1666-1760) behind
 * Booster::begin_resident_validation / accumulate_last_round_resident
 * (include/bonsai/booster.hpp:1008-1021). */
int bb_booster_eval_arm(bb_booster *b, bb_plane const *valid, float const *labels,
                        float const *init_scores);

/* The validation losses recorded since arming, one per round, into host out
 * (the first min(cap, *n)); *n receives how many rounds were recorded. */
int bb_booster_eval_losses(bb_booster const *b, float *out, uint32_t cap, uint32_t *n);

/* The current validation raw scores (host, n_valid x K row-major). */
int bb_booster_eval_scores(bb_booster const *b, float *out);

/* Keeps the first n_rounds rounds' trees (early stopping's truncate,
 * src/cli/pipeline.cpp:458-461); a truncated booster runs no more rounds. */
int bb_booster_truncate(bb_booster *b, uint32_t n_rounds);

/* Per-phase device time of one profiled boosting round (the reference's
 * BONSAI_CUDA_PROFILE counters, src/cuda/detail/profile.cuh:20-122): the
 * round runs like any other (its tree is kept) but synchronises between
 * phases to time them with CUDA events. hist_bytes are the histogram
 * build's algorithmic bytes: per built node rows x (features x bin bytes +
 * 8 B gradient pair + 4 B row id) plus the cells written. */
typedef struct
{
    double   hist_ms;
    double   partition_ms;
    double   find_ms;
    double   other_ms;
    double   total_ms;
    double   hist_bytes;
    uint64_t hist_rows;
    uint32_t hist_builds;
    uint32_t launches; /* this library's kernel launches per round */
    /* per histogram build of the round in launch order (root first; the
     * first 16 builds): device time and built rows */
    double   build_ms[16];
    uint64_t build_rows[16];
} bb_profile;

int bb_booster_profile_round(bb_booster *b, bb_profile *out);

/* Softmax: the class count (1 otherwise) and the per-class log-prior init
 * scores (out holds n_classes floats; the one init score otherwise).
 * bb_booster_scores then writes n_rows x n_classes, row-major, and tree t of
 * bb_booster_tree is round t / n_classes, class t % n_classes
 * (include/bonsai/multiclass_booster.hpp:28-33). */
uint32_t bb_booster_n_classes(bb_booster const *b);
int      bb_booster_init_scores(bb_booster const *b, float *out);

void bb_booster_destroy(bb_booster *b);

/* Node-table entries one tree of this configuration may need: 2^(max_depth+1)
 * - 1 for the depthwise and levelwise growers, 4 x max_leaves for leafwise
 * (each heap pop allocates two nodes, demoted ones included). */
uint32_t bb_tree_capacity(bb_train_cfg const *cfg);

/* One tree from caller-provided gradients: grad/hess (host, n_rows), the
 * sampled rows (host, ascending, n_sel_rows of them; NULL = all). Returns
 * the tree (node arrays of bb_tree_capacity(cfg) entries) and every sampled
 * row's leaf value and node id (values/leaf_ids host, n_rows; entries of
 * unsampled rows are left untouched).
 * Replaces one DepthwiseGrower<CudaHistogramEngine>::grow call
 * (src/grower_impl.hpp:465-577) over the engine's level plane
 * (begin_tree .. finalize_tree, histogram_engine.hpp:94-170), or with
 * cfg->grower an ObliviousGrower / LeafwiseGrower one (the latter over the
 * leaf plane, LeafStep<GPULeafEngine>, src/step/leaf.hpp:124-269). */
int bb_grow_tree(bb_plane const *plane, bb_train_cfg const *cfg, float const *grad,
                 float const *hess, uint32_t const *rows, uint64_t n_sel_rows,
                 uint32_t *feature, float *value, uint32_t *left, uint32_t *right,
                 uint8_t *default_left, float *gain, float *cover,
                 uint32_t *split_bin, uint32_t *meta, float *values,
                 uint32_t *leaf_ids);

/* One node's histograms: every selected feature's cells over the given rows
 * (host, ascending; NULL = all rows) from grad/hess (host, n_rows), written
 * to out as (sum_g, sum_h) doubles per cell, features in selection order,
 * n_bins(f) cells each (out holds the selection's total bins x 2). The
 * plain form's cells are the serial-order float sums; the quantised form's
 * are its exact integer sums times the round's FP64 scales.
 * Replaces HistogramEngine::populate (include/bonsai/grower.hpp:78-84,
 * CudaHistogramEngine::populate, histogram_engine.hpp:92-93). */
int bb_populate(bb_plane const *plane, bb_train_cfg const *cfg, float const *grad,
                float const *hess, uint32_t const *rows, uint64_t n_sel_rows,
                double *out);

/* ---- row shards: one fit over several GPUs ----------------------------------
 * No counterpart in the reference's code: its multi-GPU plan is parked
 * (docs/architecture/19-multi-gpu.md, "The algorithm maps onto bonsai's
 * control flow"). Each shard holds a contiguous range of the fit's rows in its
 * own plane; per level the shards combine their integer partial histograms,
 * per-node row counts, the quantisation maxima and the leaves' fixed-point
 * sums (in place, every shard the same calls), so every shard takes the same
 * decisions and the trees equal a one-GPU fit's bit for bit. Rows never move.
 * The quantised form only (float cells would not combine exactly). */
typedef struct bb_comm bb_comm;

#define BB_COMM_ID_BYTES 128

/* A fresh NCCL unique id (rank 0 makes it and shares it with the others). */
int bb_comm_unique_id(uint8_t *out /* BB_COMM_ID_BYTES */);

/* One process's member of an NCCL communicator over n_ranks processes (one
 * GPU each, the calling thread's current device); collectives run in place
 * on the booster's stream and are captured into its CUDA graph. NCCL is
 * resolved at the first bb_comm call: the libnccl.so.2 the process already
 * loaded if any (load the framework's NCCL first), else the system's. */
int bb_comm_create(uint8_t const *id, uint32_t n_ranks, uint32_t rank, bb_comm **out);

/* n_shards (<= 16) members of an in-process group: shards of one fit driven
 * from one host thread each (boosters created without use_graph, updated
 * concurrently); they order through CUDA events on the boosters' streams. */
int bb_comm_group(uint32_t n_shards, bb_comm **members);

void bb_comm_destroy(bb_comm *comm);

/* bb_booster_create for one shard: plane and labels hold the fit's rows
 * [row_offset, row_offset + plane rows) of total_rows; init_score is the
 * fit's (the objective's initial score over every shard's labels). hist_mode
 * must be quantised. */
int bb_booster_create_sharded(bb_plane const *plane, float const *labels,
                              float const *init_scores, bb_train_cfg const *cfg,
                              uint32_t max_trees, bb_comm *comm, uint64_t row_offset,
                              uint64_t total_rows, float init_score, bb_booster **out);

/* ---- inference ------------------------------------------------------------
 * Ensemble predict over a plane: out[r] = init + lr * sum_t leaf_t(r), the
 * leaves summed in tree order (bit-identical to predict_at_binned,
 * include/bonsai/booster.hpp:831-845). Trees are concatenated node tables
 * (n_nodes total), tree t starting at roots[t]; child ids are tree-local.
 * out is host memory (n_rows).
 * Replaces cuda_predict_plan + cuda_predict (include/bonsai/cuda/predict.hpp:
 * 29-38). */
int bb_predict(bb_plane const *plane, uint32_t n_trees, uint32_t const *roots,
               uint32_t n_nodes, uint32_t const *feature, uint32_t const *split_bin,
               uint32_t const *left, uint32_t const *right,
               uint8_t const *default_left, float const *value, float lr, float init,
               float *out);

/* The ensemble packed for the device once, walked over any plane with the
 * same features and bin counts: bb_predict split into its two halves.
 * Arguments as bb_predict; the plan copies what it needs (the caller's
 * arrays may be freed after the call). Runs through one plan serialise.
 * Replaces cuda_predict_plan (include/bonsai/cuda/predict.hpp:29-31). */
typedef struct bb_predict_plan bb_predict_plan;
int bb_predict_plan_create(bb_plane const *plane, uint32_t n_trees, uint32_t const *roots,
                           uint32_t n_nodes, uint32_t const *feature,
                           uint32_t const *split_bin, uint32_t const *left,
                           uint32_t const *right, uint8_t const *default_left,
                           float const *value, float lr, float init, bb_predict_plan **out);

/* Scores of the plan's first n_trees trees (every tree when 0) for every row
 * of plane into host out (n_rows floats), bit-identical to bb_predict over
 * those trees. A plane whose features or bin counts differ from the plan's
 * is refused with BB_ERR_ARG. Replaces cuda_predict (include/bonsai/cuda/
 * predict.hpp:33-38). */
int bb_predict_plan_run(bb_predict_plan *plan, bb_plane const *plane, uint32_t n_trees,
                        float *out);

/* bb_predict_plan_run enqueued on a caller's stream (a cudaStream_t; NULL is
 * the legacy default stream) into device out_device, without waiting.
 * *launches (if not NULL) receives the kernels enqueued. Small batches use a
 * workspace the plan owns: one launch per plan in flight at a time, and the
 * first launch of a new largest small batch allocates it (not inside a
 * stream capture). */
int bb_predict_plan_launch(bb_predict_plan *plan, bb_plane const *plane, uint32_t n_trees,
                           float *out_device, void *stream, uint32_t *launches);

/* The depth the plan padded its trees to (1..10), or 0 when it kept the
 * reference's node tables (deeper ensembles, planes over 256 u8 or 128 u16
 * features). */
int bb_predict_plan_depth(bb_predict_plan const *plan, uint32_t *depth);

void bb_predict_plan_destroy(bb_predict_plan *plan);

/* TreeSHAP contributions over a plane, FP64: out is host memory, n_rows x
 * (n_feats + 1) row-major, the last column the bias. Same tree layout as
 * bb_predict plus per-node covers (the hessian sums the booster recorded).
 * The values are the reference's: per tree, Lundberg's path-dependent
 * TreeSHAP with a repeated feature's conditions merged, zero-cover branches
 * carrying nothing, the bias its cover-weighted expected value; then every
 * column x lr and init added to the bias (contribs_impl,
 * include/bonsai/booster.hpp:901-924). At most 128 features and 32 distinct
 * features on one root-to-leaf path (BB_ERR_CONFIG otherwise).
 * Replaces cuda_shap_plan + cuda_pred_contribs
 * (include/bonsai/cuda/shap.hpp:31-43) and the host pred_contribs_binned
 * (include/bonsai/booster.hpp:887-899). */
int bb_pred_contribs(bb_plane const *plane, uint32_t n_trees, uint32_t const *roots,
                     uint32_t n_nodes, uint32_t const *feature, uint32_t const *split_bin,
                     uint32_t const *left, uint32_t const *right,
                     uint8_t const *default_left, float const *value, float const *cover,
                     float lr, float init, double *out);

/* The TreeSHAP paths of an ensemble packed for the device once, evaluated
 * over any plane with the same features and bin counts: bb_pred_contribs
 * split into its two halves. Arguments and limits as bb_pred_contribs; the
 * plan copies what it needs. Results are bit-identical run to run; runs
 * through one plan serialise. Replaces cuda_shap_plan + cuda_pred_contribs
 * (include/bonsai/cuda/shap.hpp:31-43). */
typedef struct bb_shap_plan bb_shap_plan;
int bb_shap_plan_create(bb_plane const *plane, uint32_t n_trees, uint32_t const *roots,
                        uint32_t n_nodes, uint32_t const *feature, uint32_t const *split_bin,
                        uint32_t const *left, uint32_t const *right,
                        uint8_t const *default_left, float const *value, float const *cover,
                        float lr, float init, bb_shap_plan **out);

/* Contributions for every row of plane into host out (n_rows x (n_feats + 1)
 * doubles, bias last). A plane whose features or bin counts differ from the
 * plan's is refused with BB_ERR_ARG. */
int bb_shap_plan_run(bb_shap_plan *plan, bb_plane const *plane, double *out);

/* bb_shap_plan_run enqueued on a caller's stream (a cudaStream_t; NULL is
 * the legacy default stream) into device out_device, without waiting.
 * *launches (if not NULL) receives the kernels enqueued. Small batches use a
 * workspace the plan owns: one launch per plan in flight at a time, and the
 * first launch of a new largest small batch allocates it (not inside a
 * stream capture). */
int bb_shap_plan_launch(bb_shap_plan *plan, bb_plane const *plane, double *out_device,
                        void *stream, uint32_t *launches);

void bb_shap_plan_destroy(bb_shap_plan *plan);

/* Ensemble predict that allocates no device memory. No counterpart in the
 * reference: it exists for callers that may not call cudaMalloc / cudaFree on
 * their serving path -- a host whose device memory belongs to another
 * allocator under a fixed budget, or a latency-bound caller that cannot
 * absorb the device-wide synchronisation cudaMalloc and cudaFree imply.
 * Same arguments and arithmetic as bb_predict (bit-identical scores), but
 * the ensemble is copied into one fixed 11 MiB device array that the library
 * holds on every GPU that loads it until the process exits, and out_device
 * is the caller's device buffer (n_rows floats). Limits: at most 524,288
 * nodes, 65,536 trees and 65,536 features; larger ensembles are refused
 * with BB_ERR_CONFIG before anything runs. The first call on a device
 * resolves the array's address there (make it before any stream capture).
 * All calls share the array: calls whose work overlaps on the GPU race on
 * it. The kernel runs on the legacy default stream; the call returns once it
 * is enqueued, so synchronise before reading out_device. The plane's device
 * must be the current device (BB_ERR_CONFIG otherwise); a plane with no rows
 * (a request plane before its first refill) returns 0 and runs nothing. */
int bb_predict_static(bb_plane const *plane, uint32_t n_trees, uint32_t const *roots,
                      uint32_t n_nodes, uint32_t const *feature, uint32_t const *split_bin,
                      uint32_t const *left, uint32_t const *right,
                      uint8_t const *default_left, float const *value, float lr,
                      float init, float *out_device);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif
