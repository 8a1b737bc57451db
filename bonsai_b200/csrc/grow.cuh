// Device-resident tree growth: the level plane of the reference's
// CudaHistogramEngine (include/bonsai/cuda/histogram_engine.hpp:75-284,
// driven by LevelStep<GPULevelEngine>, src/step/level.hpp:159-366), with the
// control decisions of DepthwiseGrower::grow (src/grower_impl.hpp:465-577)
// also taken on the device, so a whole tree is one stream of launches with
// static shapes (capturable as a CUDA graph) and no host round trip.
#pragma once

#include "common.cuh"
#include "ingest.cuh"

#include <vector>

namespace bb
{

// A frontier node: its row segment in the level's row buffer, its tree node
// id, the reference's node totals (float, SplitInput::sums) and monotone
// leaf-value bounds.
struct Node
{
    uint32_t start;
    uint32_t count;
    uint32_t id;
    uint32_t flags; // bit0 split, bit1 demoted
    float    sum_g;
    float    sum_h;
    double   lo;
    double   hi;
    int64_t  qg; // quantised form: exact integer totals
    int64_t  qh;
    uint32_t gcount; // rows over every shard of the fit (count when unsharded)
    // interaction constraints (the node's path state): the number of
    // distinct features on its path (0, 1 or 2 for two or more) | the one
    // feature when it is 1, << 2; and the groups that contain the whole path
    uint32_t ipath;
    uint64_t icover;
    uint32_t heap; // depthwise: the node's slot in the walked tree's decision heap
};

// SplitOutput (include/bonsai/split.hpp:62-69), one per (node, feature)
// candidate and one per node after the feature reduce.
struct Best
{
    double   gain;
    uint32_t feature; // index into the selection (j), not the feature id
    uint32_t bin;
    uint32_t dl;
    uint32_t valid;
};

// A node-aligned run of rows, the unit of partition and histogram work.
struct Chunk
{
    uint32_t node;  // frontier slot (partition) or build index (histogram)
    uint32_t begin; // first row position in the row buffer
    uint32_t count;
    uint32_t aux;
};

// Per-tree device control block.
struct Ctl
{
    uint32_t n_cur;      // frontier size at the current level
    uint32_t n_next;     // frontier size the level produced
    uint32_t n_nodes;    // tree node count
    uint32_t n_leaves;
    uint32_t depth;
    uint32_t n_pchunks;  // partition chunks at the current level
    uint32_t n_bchunks;  // histogram-build chunks
    uint32_t n_build;    // nodes whose histograms are built this level
    uint32_t n_splits;   // surviving splits this level
    uint32_t built_rows; // rows across the built nodes
    uint32_t n_psplit;   // splits plan_kernel committed at the current level
    uint32_t pad[5];
};

// A row sample on the device: its size and one bit per dataset row (bit r of
// word r / 32).
struct RootSample
{
    uint32_t const *count;
    uint32_t const *bits;
};

struct TreeOut
{
    uint32_t *feature;
    float    *value;
    uint32_t *left;
    uint32_t *right;
    uint8_t  *default_left;
    float    *gain;
    float    *cover;
    uint32_t *split_bin;
    uint32_t *meta; // n_nodes, depth, n_leaves
};

enum class HistMode : int32_t
{
    exact = 0,  // serial-order float cells, bit-identical to the CPU grower
    quant8 = 1, // int8 gradients, exact integer histograms
    quant16 = 2 // int16 gradients
};

// Per-phase device time of profiled trees (CUDA events on the grower's
// stream) and the histogram build's algorithmic bytes: per built node,
// rows x (features x bin bytes + 8 B gradient pair + 4 B row id) read plus
// its cells written.
struct Profile
{
    double   hist_ms      = 0.0;
    double   partition_ms = 0.0;
    double   find_ms      = 0.0;
    double   other_ms     = 0.0;
    double   hist_bytes   = 0.0;
    uint64_t hist_rows    = 0;
    uint32_t hist_builds  = 0;
    // per histogram build of the round, in order (root first): its time and
    // built rows (the first k_prof_builds builds)
    static constexpr uint32_t k_prof_builds = 16;
    double   build_ms[k_prof_builds]   = {};
    uint64_t build_rows[k_prof_builds] = {};
};

// Combines a device buffer across the row shards of one fit, in stream
// order and in place: sums of 64-bit two's-complement integers, or maxima of
// 32-bit unsigned words. Every shard makes the same calls in the same order.
// The shard-parallel design of the reference's parked multi-GPU plan
// (docs/architecture/19-multi-gpu.md:20-35): rows stay where they are, only
// integer histograms and a few counts cross between shards.
class Reducer
{
  public:
    virtual ~Reducer()                                            = default;
    virtual void sum_u64(void *buf, size_t n, cudaStream_t s) = 0;
    virtual void max_u32(void *buf, size_t n, cudaStream_t s) = 0;
};

// A resident booster's next round, computed by the final walk over every
// row once the tree is complete: gh[r] from the updated score and the label,
// and (quantised form) the maxima the next quantisation scales come from.
struct NextRound
{
    int          objective = 0;
    float const *labels    = nullptr;
    float2      *gh        = nullptr;
    float const *weights   = nullptr; // per row, or nullptr (unweighted)
};

struct GrowConfig
{
    TreeParams tp;
    HistMode   mode  = HistMode::exact;
    // levelwise (ObliviousGrower, src/grower_impl.hpp:579-720): one split per
    // level over the whole frontier, broadcast to every node; trees are
    // perfect to their depth, empty children included
    bool       level = false;
    // leafwise (LeafwiseGrower, src/grower_impl.hpp:744-850): best-first, one
    // node per heap pop, at most tp.max_leaves leaves (<= 512), tp.max_depth
    // caps the depth (<= 255)
    bool       leaf  = false;
    // > 0: every tree draws its own sample of this many features
    // (feature_fraction, sample_features, src/grower_impl.hpp:163-180) into one
    // of sel_sets table sets (set_selection / use_set); the grower is sized
    // for any such sample, so its launches do not depend on which
    uint32_t   sample_k = 0;
    uint32_t   sel_sets = 1;
    // rows of the whole fit (every shard's, for a row-sharded fit; 0: the
    // grower's own rows): sizes the quantised cells and fixed-point sums
    uint64_t   fit_rows = 0;
    // the quantised build's CTAs per mirror tile (0: one per SM, fewer for a
    // small dataset); a launch shape only -- the cells are order-free sums
    uint32_t   hist_ctas = 0;
};

// All device buffers one tree's growth needs, sized once for a dataset and
// a selection, reused for every tree.
class Grower
{
  public:
    Grower(Plane const &plane, GrowConfig const &cfg, std::vector<uint32_t> selected,
           uint32_t max_root_rows, cudaStream_t stream);
    ~Grower();
    Grower(Grower const &)            = delete;
    Grower &operator=(Grower const &) = delete;

    // Enqueues one tree on the stream. gh: float2 (g, h) per dataset row;
    // root_rows: the sampled rows (ascending), n_root of them. out receives
    // the tree; leaf_id (nullable) each sampled row's leaf; scores (nullable)
    // gets scores[r] += lr * leaf value for every sampled row.
    //
    // With identity_root (every dataset row, in order) the rows take their
    // leaf ids and score updates from one walk of the finished tree in row
    // order, and next (nullable) also has the walk write the next round's
    // gradient pairs; the quantised form then reads their maxima from that
    // walk, so the first such round must follow seed_absmax.
    //
    // With sample (depthwise and levelwise) the root is a row sample built on
    // the device: root_rows holds sample->count[0] ascending rows (n_root is
    // only their bound), and every dataset row still takes the walk -- the
    // unsampled ones routed through the finished tree as the sampled ones
    // are -- while the quantised form renews its leaves from the sampled
    // rows alone (sample->bits, one bit per row).
    void grow(float2 const *gh, uint32_t const *root_rows, uint32_t n_root,
              TreeOut const &out, uint32_t *leaf_id, float *scores, float lr,
              bool identity_root = false, NextRound const *next = nullptr,
              RootSample const *sample = nullptr);
    // The quantised form's gradient maxima of gh (every dataset row), for a
    // first grow() whose next round is fused.
    void seed_absmax(float2 const *gh);
    // Makes this grower one row shard of a fit: its plane holds the fit's
    // rows [row_offset, row_offset + n_rows) of total_rows, and r combines the
    // shards' integer partial sums so every shard takes the same decisions.
    // Quantised form with every row as the root only; the trees equal an
    // unsharded fit's bit for bit.
    void set_shard(Reducer *r, uint64_t row_offset, uint64_t total_rows);

    // One node's histograms (HistogramEngine::populate): quantises (when
    // quantised) and builds every selected feature over the given rows;
    // out receives total_cells (g, h) pairs as FP64 cell sums, scaled back
    // from integers in the quantised form.
    void populate(float2 const *gh, uint32_t const *rows, uint32_t n, double2 *out_host);

    uint32_t total_cells() const
    {
        return total_cells_;
    }

    // Per-tree feature samples (GrowConfig::sample_k): writes the tables of
    // table set `set` for the ascending feature ids sel (sample_k of them),
    // enqueued on the grower's stream; use_set picks the set the next
    // grow() reads (a captured grow keeps the set it was captured with).
    void set_selection(uint32_t set, std::vector<uint32_t> const &sel);
    void use_set(uint32_t set);

    uint32_t max_nodes() const
    {
        return max_nodes_;
    }
    uint32_t n_sel() const
    {
        return n_sel_;
    }

    // the quantisation scales of the last tree (g, h); 0 for the exact form
    float2 const *quant_scale() const
    {
        return scale_;
    }

  private:
    void level(uint32_t L, uint32_t const *rows_in, uint32_t *rows_out,
               TreeOut const &out, uint32_t *leaf_id, float *scores, float lr);
    void grow_leafwise(uint32_t const *root_rows, uint32_t n_root, TreeOut const &out,
                       uint32_t *leaf_id, float *scores, float lr);
    void find_nodes(void const *hist, uint32_t n_nodes, uint32_t const *slot_of);
    // zeroed: the quantised slots were already cleared (by the partition)
    void build(uint32_t const *rows, uint32_t n_feat_build, int dst, bool zeroed = false);

    Plane const          &plane_;
    GrowConfig            cfg_;
    std::vector<uint32_t> sel_h_;
    cudaStream_t          stream_;
    uint32_t              n_sel_       = 0;
    uint32_t              total_cells_ = 0;
    uint32_t              max_nb_      = 0;
    uint32_t              max_front_   = 0;
    uint32_t              max_nodes_   = 0;
    uint32_t              max_rows_    = 0;
    uint32_t              max_pchunks_ = 0;
    uint32_t              max_bchunks_ = 0;
    uint32_t              cell_stride_ = 0; // per-(chunk, feature) count stride
    uint32_t              lgroup_      = 1; // nodes per level-finder group
    uint32_t              qctas_       = 1; // u8 quantised histogram CTAs per tile
    // words per quantised cell: 2 (an int64 gradient and a uint64 hessian
    // sum) for int16 codes, and for int8 codes once the fit's rows could carry
    // a packed 32-bit half past its range (127 x rows >= 2^31)
    uint32_t              cw_          = 1;
    bool                  wide_codes_  = false;          // int16 codes (one u32 per row)
    double                fix_unit_    = 274877906944.0; // fixed-point leaf-sum unit (2^38 at
                                                         // up to 2^24 rows, halved per doubling)

    // device
    uint32_t *sel_      = nullptr; // selected feature ids
    uint32_t *cell_off_ = nullptr; // per selected feature, its first cell
    uint32_t *sel_nb_   = nullptr; // per selected feature, its bin count
    Ctl      *ctl_      = nullptr;
    Node     *nodes_[2] = {nullptr, nullptr};
    void     *hist_[2]  = {nullptr, nullptr}; // [front][total_cells] cells
    Best     *cand_     = nullptr;             // [front][n_sel]
    Best     *best_     = nullptr;             // [front]
    Chunk    *pchunks_  = nullptr;
    uint32_t *pleft_    = nullptr; // per partition chunk: left count, then base
    uint32_t *prbase_   = nullptr;
    uint32_t *dirs_     = nullptr; // per partition chunk: one direction bit per row
    uint32_t *dst_      = nullptr; // per frontier slot: child segment start
    uint32_t *build_    = nullptr; // per build index: frontier slot in next
    uint32_t *bpair_    = nullptr; // per split: (parent, small, large) slots
    uint32_t *bbase_    = nullptr; // per build index: its payload base
    uint32_t *brange_   = nullptr; // per build index: chunk range [c0, c1)
    Chunk    *bchunks_  = nullptr;
    uint32_t *ccount_   = nullptr; // [bchunk][n_sel][cell_stride] counts/offsets
    uint32_t *seg_      = nullptr; // [build][n_sel][cell_stride] bin segment starts
    float2   *payload_  = nullptr; // [n_sel][max_rows] bin-sorted (g, h)
    uint32_t *rows_[2]  = {nullptr, nullptr};
    uint32_t *pcr_      = nullptr; // per frontier slot: partition chunk range
    uint32_t *nleft_    = nullptr; // per frontier slot: rows routed left
    int8_t   *mono_     = nullptr; // per feature monotone direction, or null
    uint64_t *fgroups_  = nullptr; // per feature interaction-group mask, or null
    uint32_t  n_mono_   = 0;
    float2 const *gh_cur_ = nullptr;
    std::vector<uint32_t> off_h_;
    // quantised form
    int32_t  *qgh_      = nullptr; // per row, packed (g, h) integers
    float2   *scale_    = nullptr;
    uint32_t *absmax_   = nullptr; // max |g| and max h, as float bits
    double2  *qscale_   = nullptr; // (scale_g, scale_h) in FP64
    uint16_t *qgh8_     = nullptr; // per row: int8 g | uint8 h << 8
    uint32_t *qgh16_    = nullptr; // per row (int16 codes): int16 g | uint16 h << 16
    double2  *partial_  = nullptr; // per partition chunk: leaf (G, H) in FP64
    int64_t  *btot_     = nullptr; // per build index: exact (G, H) of the last level
    uint32_t *done_     = nullptr; // leaf-renewal CTA ticket (zero between launches)
    unsigned long long *wacc_ = nullptr; // per tree node: fixed-point (G, H) of the walk
    uint16_t *leaf16_   = nullptr; // per row: its leaf, from the walk
    double2  *nbound_   = nullptr; // per tree node: monotone bounds (lo, hi)
    uint32_t *nright_   = nullptr; // per frontier node: rights placed (one-pass partition)
    uint2    *heap_     = nullptr; // the walked tree's decision heap (plan kernels)
    uint16_t *leafmap_  = nullptr; // its last heap level's leaf node ids
    // leafwise
    void     *lout_     = nullptr; // the pop's results (device)
    void     *lout_h_   = nullptr; // the loop's state read back after a tree (pinned host)
    uint32_t *slot_of_  = nullptr; // the children's pool slots
    // the device-side pop loop: its state (the candidate heap, free pool
    // slots, the leaves, the node count), the tree being grown, and the
    // loop's graph (a conditional WHILE node over one pop's launches)
    void            *loop_      = nullptr;
    void            *cand_heap_ = nullptr;
    Node            *leaves_    = nullptr;
    uint32_t        *free_      = nullptr;
    void            *tree_dev_  = nullptr;
    cudaGraph_t      loop_g_    = nullptr;
    cudaGraphExec_t  loop_x_    = nullptr;
    uint32_t         body_launches_ = 0;
    uint32_t  crows_    = 0;       // rows per histogram-build chunk
    bool      quant_    = false;
    uint32_t *dtree_    = nullptr; // device tree counter (the rounding stream)
    uint32_t *tile_ids_[2] = {nullptr, nullptr};
    int32_t  *tile_j_[2]   = {nullptr, nullptr};
    uint32_t  n_tiles_[2]  = {0, 0};
    // the selection tables of every set (sel_, cell_off_, sel_nb_ and the
    // tile tables point into set k's part); unused tile slots hold
    // k_no_sel_tile, so their CTAs exit
    std::vector<std::vector<uint32_t>> sets_h_;
    uint32_t *sel_base_      = nullptr;
    uint32_t *cell_off_base_ = nullptr;
    uint32_t *sel_nb_base_   = nullptr;
    uint32_t *tile_ids_base_[2] = {nullptr, nullptr};
    int32_t  *tile_j_base_[2]   = {nullptr, nullptr};
    void      write_tables(uint32_t set, std::vector<uint32_t> const &sel);
    Node const     *nodes_cur_ = nullptr;
    uint32_t const *rows_cur_  = nullptr;
    uint32_t const *root_rows_ = nullptr;
    void      quantise(float2 const *gh, uint32_t n, bool have_absmax);
    bool      walk_ = false; // this tree's rows are stamped by the final walk
    Reducer  *red_        = nullptr; // shard reducer, or none
    uint64_t  row_off_    = 0;       // the shard's first row in the fit
    uint64_t  total_rows_ = 0;       // rows of the whole fit
    uint64_t *gleft_      = nullptr; // per frontier node: rows routed left, all shards
    void      leaf_values(TreeOut const &t, bool final_level);
    uint64_t  seed_     = 0;
    uint32_t  tree_no_  = 0;

  public:
    void set_seed(uint64_t s)
    {
        seed_ = s;
    }
    // per-feature monotone directions (+1 / -1 / 0), copied to the device
    void set_monotone(std::vector<int8_t> const &m);
    // Interaction constraints: per feature, the groups containing it as a
    // bit mask (empty: unconstrained).
    void set_interaction(std::vector<uint64_t> const &fgroups);
    // non-null: the next grow() calls time their phases into *p (synchronous)
    void set_profile(Profile *p)
    {
        prof_ = p;
    }
    // whether grow() can take a fused next round (and be graph-captured):
    // not on the leafwise plane, whose host reads each pop back
    bool fuses_next() const
    {
        return !cfg_.leaf;
    }
    // kernel launches one grow() enqueues
    uint32_t launches_per_tree() const
    {
        return launches_;
    }

  private:
    Profile    *prof_     = nullptr;
    uint32_t    launches_ = 0;
    uint32_t    n_launch_ = 0;
    // every kernel opens with pdl_enter(): launched with programmatic
    // stream serialization, a kernel's CTAs are scheduled while its
    // predecessor drains. Set for planes of 2^19 rows or more, whose kernels
    // each fill the GPU; small planes are the ones several boosters fit at
    // once, where CTAs waiting for their predecessor would hold SM resources
    // the other boosters' kernels could use.
    bool        pdl_      = false;
    cudaEvent_t pev_[2]   = {nullptr, nullptr};
    void        phase_begin();
    void        phase_end(double &acc);
};

} // namespace bb
