/* TEST INFRASTRUCTURE — the oracle. Not part of the product; see
 * bonsai_oracle.h for what it is pinned against. Citations are
 * file:line within the daniel-m-campos/bonsai project. */
#include "bonsai_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define LEAF_FLAG 0xFFFFFFFFu

/* ---- bin application --------------------------------------------------- */

/* lower_bound over the feature's cuts; NaN -> last bin
 * (src/bin_mapper.cpp:284-291). */
static uint16_t transform_one(float x, float const *c, uint32_t nb)
{
    if (isnan(x))
    {
        return (uint16_t)(nb - 1);
    }
    uint32_t lo = 0, hi = nb;
    while (lo < hi)
    {
        uint32_t const mid = lo + ((hi - lo) >> 1);
        if (c[mid] < x)
        {
            lo = mid + 1;
        }
        else
        {
            hi = mid;
        }
    }
    return (uint16_t)lo;
}

void orc_transform(float const *X, size_t n, size_t F, float const *cuts,
                   uint32_t const *cut_off, uint16_t *bins)
{
    for (size_t f = 0; f < F; ++f)
    {
        float const   *c  = cuts + cut_off[f];
        uint32_t const nb = cut_off[f + 1] - cut_off[f];
        for (size_t r = 0; r < n; ++r)
        {
            bins[(f * n) + r] = transform_one(X[(r * F) + f], c, nb);
        }
    }
}

/* ---- split math (include/bonsai/split.hpp:112-158) ---------------------- */

static double l1_thresholded(double g, double l1)
{
    if (g > l1)
    {
        return g - l1;
    }
    if (g < -l1)
    {
        return g + l1;
    }
    return 0.0;
}

static double score(double g, double h, double l1, double l2)
{
    double const t = l1_thresholded(g, l1);
    double const d = h + l2;
    return d > 0.0 ? (t * t) / d : 0.0;
}

static double bounded_leaf_weight(double g, double h, double l1, double l2, double lo,
                                  double hi)
{
    double const d = h + l2;
    double const w = d > 0.0 ? -l1_thresholded(g, l1) / d : 0.0;
    /* std::clamp(w, lo, hi) */
    return w < lo ? lo : (hi < w ? hi : w);
}

static int monotone_of(orc_tree_cfg const *cfg, uint32_t f)
{
    return (cfg->monotone != NULL && f < cfg->n_monotone) ? cfg->monotone[f] : 0;
}

/* ---- histograms ---------------------------------------------------------- */

/* Histogram::totals (include/bonsai/histogram.hpp:84-95): double sums over
 * every cell, missing included, rounded to float once. */
static void totals(float const *cells, uint32_t nb, float *g, float *h)
{
    double sg = 0.0, sh = 0.0;
    for (uint32_t b = 0; b < nb; ++b)
    {
        sg += cells[2 * b];
        sh += cells[(2 * b) + 1];
    }
    *g = (float)sg;
    *h = (float)sh;
}

void orc_fill(uint16_t const *bins, size_t n, uint32_t const *selected, size_t n_sel,
              uint32_t const *n_bins, float const *grad, float const *hess,
              uint32_t const *rows, size_t n_rows, float *hist)
{
    size_t off = 0;
    for (size_t j = 0; j < n_sel; ++j)
    {
        uint32_t const f  = selected[j];
        uint32_t const nb = n_bins[f];
        float *const   c  = hist + (2 * off);
        memset(c, 0, sizeof(float) * 2 * nb);
        uint16_t const *col = bins + ((size_t)f * n);
        /* one serial float chain per cell, in the node's row order */
        for (size_t k = 0; k < n_rows; ++k)
        {
            uint32_t const r = rows[k];
            uint16_t const b = col[r];
            c[2 * b] += grad[r];
            c[(2 * b) + 1] += hess[r];
        }
        off += nb;
    }
}

/* ---- split finder -------------------------------------------------------- */

/* update_best_for_feature_for_node (src/split.cpp:101-162). */
static void best_for_feature(float const *cells, uint32_t nb, uint32_t fid, float tot_g,
                             float tot_h, double lo, double hi, orc_tree_cfg const *cfg,
                             orc_split *best)
{
    double const l1        = cfg->lambda_l1;
    double const l2        = cfg->lambda_l2;
    float const  miss_g    = cells[2 * (nb - 1)];
    float const  miss_h    = cells[(2 * (nb - 1)) + 1];
    double const node_sc   = score(tot_g, tot_h, l1, l2);
    /* HistCell fields are float: the reference subtracts in float, then
     * widens (src/split.cpp:117-118) */
    double const real_grad = (double)(float)(tot_g - miss_g);
    double const real_hess = (double)(float)(tot_h - miss_h);
    int const    mc        = monotone_of(cfg, fid);
    int const    n_dirs    = (miss_g == 0.0F && miss_h == 0.0F) ? 1 : 2;
    double       lg = 0.0, lh = 0.0;
    uint32_t const n_cut = nb >= 2 ? nb - 2 : 0;
    for (uint32_t b = 0; b < n_cut; ++b)
    {
        lg += cells[2 * b];
        lh += cells[(2 * b) + 1];
        for (int d = 0; d < n_dirs; ++d)
        {
            int const    dl = d == 0;
            double const rg = real_grad - lg;
            double const rh = real_hess - lh;
            /* split_sums_at (src/split.cpp:33-45) */
            double const gL = lg + (dl ? (double)miss_g : 0.0);
            double const hL = lh + (dl ? (double)miss_h : 0.0);
            double const gR = rg + (!dl ? (double)miss_g : 0.0);
            double const hR = rh + (!dl ? (double)miss_h : 0.0);
            if (hL < (double)cfg->min_child_hess || hR < (double)cfg->min_child_hess)
            {
                continue;
            }
            double const children = score(gL, hL, l1, l2) + score(gR, hR, l1, l2);
            if (mc != 0)
            {
                double const wl = bounded_leaf_weight(gL, hL, l1, l2, lo, hi);
                double const wr = bounded_leaf_weight(gR, hR, l1, l2, lo, hi);
                if ((double)mc * (wr - wl) < 0.0)
                {
                    continue;
                }
            }
            double const gain = children - node_sc;
            /* update_best (src/split.cpp:84-95): strict > and the gain gate */
            if (gain > best->gain && gain >= (double)cfg->min_gain_to_split)
            {
                best->gain         = gain;
                best->feature      = fid;
                best->bin          = b;
                best->default_left = (uint8_t)dl;
                best->valid        = 1;
            }
        }
    }
}

orc_split orc_find_split(float const *const *hist, uint32_t const *n_bins,
                         uint8_t const *present, size_t F, size_t n_rows,
                         float tot_g, float tot_h, double lo, double hi,
                         orc_tree_cfg const *cfg)
{
    orc_split best = {0.0, 0, 0, 1, 0};
    /* cannot_split (src/split.cpp:254-258) */
    if (n_rows < 2 * (size_t)cfg->min_data_in_leaf)
    {
        return best;
    }
    for (size_t f = 0; f < F; ++f)
    {
        if (!present[f])
        {
            continue;
        }
        orc_split cand = {0.0, 0, 0, 1, 0};
        best_for_feature(hist[f], n_bins[f], (uint32_t)f, tot_g, tot_h, lo, hi, cfg,
                         &cand);
        if (cand.valid && cand.gain > best.gain)
        {
            best = cand;
        }
    }
    return best;
}

/* ---- depthwise grower ------------------------------------------------------ */

typedef struct
{
    size_t   start, count; /* segment of the grower's row order */
    uint32_t id;
    float   *hist; /* total_cells cells of (g, h) over the selected features */
    float    sum_g, sum_h;
    double   lo, hi;
} onode;

typedef struct
{
    uint16_t const *bins;
    size_t          n;
    size_t          F;
    uint32_t const *n_bins;
    float const    *cuts;
    uint32_t const *cut_off;
    float const    *grad;
    float const    *hess;
    uint32_t const *selected;
    size_t          n_sel;
    size_t         *off;         /* per selected feature, its cell offset */
    size_t          total_cells; /* over the selected features */
    orc_tree_cfg const *cfg;
    orc_tree           *t;
} gctx;

static int push_node(orc_tree *t, uint32_t feature, float value)
{
    if (t->n_nodes >= t->cap)
    {
        return -1;
    }
    uint32_t const i = t->n_nodes++;
    t->feature[i]      = feature;
    t->value[i]        = value;
    t->left[i]         = 0;
    t->right[i]        = 0;
    t->default_left[i] = 0;
    t->gains[i]        = 0.0F;
    t->covers[i]       = 0.0F;
    t->split_bin[i]    = 0;
    return (int)i;
}

/* The node's totals: the first selected feature's histogram
 * (SplitInput::totals, include/bonsai/split.hpp:36-52). */
static void node_totals(gctx const *c, onode *nd)
{
    uint32_t const f0 = c->selected[0];
    totals(nd->hist, c->n_bins[f0], &nd->sum_g, &nd->sum_h);
}

static orc_split find_node(gctx const *c, onode const *nd)
{
    float const **h       = (float const **)calloc(c->F, sizeof(float *));
    uint8_t      *present = (uint8_t *)calloc(c->F, 1);
    for (size_t j = 0; j < c->n_sel; ++j)
    {
        h[c->selected[j]]       = nd->hist + (2 * c->off[j]);
        present[c->selected[j]] = 1;
    }
    orc_split const s = orc_find_split(h, c->n_bins, present, c->F, nd->count,
                                       nd->sum_g, nd->sum_h, nd->lo, nd->hi, c->cfg);
    free(h);
    free(present);
    return s;
}

/* The levelwise grower's split finder: update_best_for_feature_for_level
 * (src/split.cpp:164-235) per selected feature, then reduce_in_feature_order
 * (:239-250). Per candidate (bin, default_left) the frontier's nodes are
 * summed in frontier order: a node's children score when both children clear
 * min_child_hess, else its own score (issue #60); the gain is that sum minus
 * the sum of the nodes' scores. No min_data_in_leaf gate, no monotone
 * bounds (the levelwise grower rejects them). */
static orc_split find_level(gctx const *c, onode const *cur, size_t n_cur)
{
    orc_tree_cfg const *cfg  = c->cfg;
    double const        l1   = cfg->lambda_l1;
    double const        l2   = cfg->lambda_l2;
    orc_split           best = {0.0, 0, 0, 1, 0};
    if (n_cur == 0)
    {
        return best;
    }
    double *pscore = (double *)malloc(sizeof(double) * n_cur);
    double *rg     = (double *)malloc(sizeof(double) * n_cur);
    double *rh     = (double *)malloc(sizeof(double) * n_cur);
    float  *mg     = (float *)malloc(sizeof(float) * n_cur);
    float  *mh     = (float *)malloc(sizeof(float) * n_cur);
    for (size_t j = 0; j < c->n_sel; ++j)
    {
        uint32_t const f     = c->selected[j];
        uint32_t const nb    = c->n_bins[f];
        uint32_t const n_cut = nb >= 2 ? nb - 2 : 0;
        if (n_cut == 0)
        {
            continue;
        }
        double *pref       = (double *)malloc(sizeof(double) * 2 * n_cur * n_cut);
        double  sum_parent = 0.0;
        int     all_empty  = 1;
        for (size_t p = 0; p < n_cur; ++p)
        {
            float const *cells = cur[p].hist + (2 * c->off[j]);
            mg[p]              = cells[2 * (nb - 1)];
            mh[p]              = cells[(2 * (nb - 1)) + 1];
            /* Histogram::fill_prefix (include/bonsai/histogram.hpp:139-160):
               double running sums, each entry stored as a float cell */
            double lg = 0.0, lh = 0.0;
            for (uint32_t b = 0; b < n_cut; ++b)
            {
                lg += cells[2 * b];
                lh += cells[(2 * b) + 1];
                pref[2 * ((p * n_cut) + b)]       = (double)(float)lg;
                pref[(2 * ((p * n_cut) + b)) + 1] = (double)(float)lh;
            }
            pscore[p] = score(cur[p].sum_g, cur[p].sum_h, l1, l2);
            sum_parent += pscore[p];
            rg[p]     = (double)(float)(cur[p].sum_g - mg[p]);
            rh[p]     = (double)(float)(cur[p].sum_h - mh[p]);
            all_empty = all_empty && mg[p] == 0.0F && mh[p] == 0.0F;
        }
        int const n_dirs = all_empty ? 1 : 2;
        orc_split cand   = {0.0, 0, 0, 1, 0};
        for (uint32_t b = 0; b < n_cut; ++b)
        {
            for (int d = 0; d < n_dirs; ++d)
            {
                int const dl       = d == 0;
                double    children = 0.0;
                for (size_t p = 0; p < n_cur; ++p)
                {
                    double const lg = pref[2 * ((p * n_cut) + b)];
                    double const lh = pref[(2 * ((p * n_cut) + b)) + 1];
                    double const gL = lg + (dl ? (double)mg[p] : 0.0);
                    double const hL = lh + (dl ? (double)mh[p] : 0.0);
                    double const gR = (rg[p] - lg) + (!dl ? (double)mg[p] : 0.0);
                    double const hR = (rh[p] - lh) + (!dl ? (double)mh[p] : 0.0);
                    int const    ok = !(hL < (double)cfg->min_child_hess ||
                                     hR < (double)cfg->min_child_hess);
                    children += ok ? score(gL, hL, l1, l2) + score(gR, hR, l1, l2)
                                   : pscore[p];
                }
                double const gain = children - sum_parent;
                if (gain > cand.gain && gain >= (double)cfg->min_gain_to_split)
                {
                    cand.gain         = gain;
                    cand.feature      = f;
                    cand.bin          = b;
                    cand.default_left = (uint8_t)dl;
                    cand.valid        = 1;
                }
            }
        }
        free(pref);
        if (cand.valid && cand.gain > best.gain)
        {
            best = cand;
        }
    }
    free(pscore);
    free(rg);
    free(rh);
    free(mg);
    free(mh);
    return best;
}

/* write_leaf + stamping (src/step/primitives.hpp:42-69). */
static void finalize_leaf(gctx *c, onode const *nd, uint32_t const *order,
                          float *values, uint32_t *leaf_ids)
{
    orc_tree_cfg const *cfg = c->cfg;
    float const v = (float)bounded_leaf_weight(nd->sum_g, nd->sum_h, cfg->lambda_l1,
                                               cfg->lambda_l2, nd->lo, nd->hi);
    c->t->feature[nd->id]      = LEAF_FLAG;
    c->t->value[nd->id]        = v;
    c->t->left[nd->id]         = 0;
    c->t->right[nd->id]        = 0;
    c->t->default_left[nd->id] = 0;
    c->t->split_bin[nd->id]    = 0;
    c->t->n_leaves++;
    for (size_t k = 0; k < nd->count; ++k)
    {
        values[order[nd->start + k]]   = v;
        leaf_ids[order[nd->start + k]] = nd->id;
    }
}

static int routes_left(uint32_t b, uint32_t last, uint32_t split, int dl)
{
    return b == last ? dl : b <= split;
}

int orc_grow_depthwise(uint16_t const *bins, size_t n, size_t F, uint32_t const *n_bins,
                       float const *cuts, uint32_t const *cut_off, float const *grad,
                       float const *hess, uint32_t const *rows, size_t n_rows,
                       uint32_t const *selected, size_t n_sel, orc_tree_cfg const *cfg,
                       orc_tree *t, float *values, uint32_t *leaf_ids)
{
    gctx c = {bins, n, F, n_bins, cuts, cut_off, grad, hess, selected, n_sel,
              NULL, 0, cfg, t};
    c.off  = (size_t *)malloc(sizeof(size_t) * (n_sel + 1));
    for (size_t j = 0; j < n_sel; ++j)
    {
        c.off[j] = c.total_cells;
        c.total_cells += n_bins[selected[j]];
    }
    t->n_nodes  = 0;
    t->n_leaves = 0;
    t->depth    = 0;
    int rc      = 0;

    uint32_t *order = (uint32_t *)malloc(sizeof(uint32_t) * (n_rows + 1));
    uint32_t *tmp   = (uint32_t *)malloc(sizeof(uint32_t) * (n_rows + 1));
    memcpy(order, rows, sizeof(uint32_t) * n_rows);

    size_t  cap_nodes = 1;
    onode  *cur       = (onode *)calloc(1, sizeof(onode));
    size_t  n_cur     = 1;
    cur[0].start = 0;
    cur[0].count = n_rows;
    cur[0].id    = 0;
    cur[0].lo    = -INFINITY;
    cur[0].hi    = INFINITY;
    cur[0].hist  = (float *)malloc(sizeof(float) * 2 * (c.total_cells + 1));
    orc_fill(bins, n, selected, n_sel, n_bins, grad, hess, order, n_rows, cur[0].hist);
    node_totals(&c, &cur[0]);
    push_node(t, LEAF_FLAG, 0.0F);
    t->covers[0] = (float)n_rows;
    (void)cap_nodes;

    uint32_t depth = 0;
    while (depth < cfg->max_depth)
    {
        /* open_level: one split per frontier node (src/step/level.hpp:55-80) */
        orc_split *sp = (orc_split *)malloc(sizeof(orc_split) * (n_cur + 1));
        if (cfg->grower == 1)
        {
            /* ObliviousGrower::grow (src/grower_impl.hpp:599-720): one split
             * broadcast to every frontier node, or none and the tree ends */
            orc_split const lv = find_level(&c, cur, n_cur);
            for (size_t i = 0; i < n_cur; ++i)
            {
                sp[i] = lv;
            }
        }
        else
        {
            for (size_t i = 0; i < n_cur; ++i)
            {
                sp[i] = find_node(&c, &cur[i]);
            }
        }
        /* plan_level (src/grower_impl.hpp:212-255) + host_partition
         * (src/step/primitives.hpp:262-374) + demote_empty_splits (:262-298)
         * + build_children/finish_split (level.hpp:96-112, primitives.hpp:
         * 156-173) + commit_children (grower_impl.hpp:303-326). */
        onode  *next   = (onode *)calloc(2 * n_cur + 1, sizeof(onode));
        size_t  n_next = 0;
        for (size_t i = 0; i < n_cur; ++i)
        {
            onode *nd = &cur[i];
            if (!sp[i].valid)
            {
                finalize_leaf(&c, nd, order, values, leaf_ids);
                free(nd->hist);
                nd->hist = NULL;
                continue;
            }
            int const li = push_node(t, LEAF_FLAG, 0.0F);
            int const ri = push_node(t, LEAF_FLAG, 0.0F);
            if (li < 0 || ri < 0)
            {
                rc = -1;
                break;
            }
            uint32_t const f = sp[i].feature;
            t->feature[nd->id]      = f;
            t->value[nd->id]        = cuts[cut_off[f] + sp[i].bin];
            t->left[nd->id]         = (uint32_t)li;
            t->right[nd->id]        = (uint32_t)ri;
            t->default_left[nd->id] = sp[i].default_left;
            t->gains[nd->id]        = (float)sp[i].gain;
            t->split_bin[nd->id]    = sp[i].bin;
        }
        if (rc != 0)
        {
            free(sp);
            free(next);
            break;
        }
        /* partition, smaller-child fill, subtraction, child stats */
        for (size_t i = 0; i < n_cur; ++i)
        {
            onode *nd = &cur[i];
            if (!sp[i].valid)
            {
                continue;
            }
            uint32_t const  f    = sp[i].feature;
            uint32_t const  last = n_bins[f] - 1;
            uint16_t const *col  = bins + ((size_t)f * n);
            size_t          nl = 0, nr = 0;
            for (size_t k = 0; k < nd->count; ++k)
            {
                uint32_t const r = order[nd->start + k];
                if (routes_left(col[r], last, sp[i].bin, sp[i].default_left))
                {
                    ++nl;
                }
            }
            {
                size_t li2 = 0, ri2 = 0;
                for (size_t k = 0; k < nd->count; ++k)
                {
                    uint32_t const r = order[nd->start + k];
                    if (routes_left(col[r], last, sp[i].bin, sp[i].default_left))
                    {
                        tmp[nd->start + li2++] = r;
                    }
                    else
                    {
                        tmp[nd->start + nl + ri2++] = r;
                    }
                }
                nr = ri2;
                memcpy(order + nd->start, tmp + nd->start, sizeof(uint32_t) * nd->count);
            }
            uint32_t const lid = t->left[nd->id];
            uint32_t const rid = t->right[nd->id];
            if (cfg->grower != 1 && (nl == 0 || nr == 0))
            {
                /* demote_empty_splits: the survivor's rows return to the
                 * parent, which becomes a leaf with its own sums */
                t->gains[nd->id] = 0.0F;
                finalize_leaf(&c, nd, order, values, leaf_ids);
                free(nd->hist);
                nd->hist = NULL;
                continue;
            }
            onode *L = &next[n_next++];
            onode *R = &next[n_next++];
            L->start = nd->start;
            L->count = nl;
            L->id    = lid;
            R->start = nd->start + nl;
            R->count = nr;
            R->id    = rid;
            /* smaller child: the left wins a size tie (primitives.hpp:94-99) */
            onode *small = nl <= nr ? L : R;
            onode *large = nl <= nr ? R : L;
            small->hist  = (float *)malloc(sizeof(float) * 2 * (c.total_cells + 1));
            orc_fill(bins, n, selected, n_sel, n_bins, grad, hess, order + small->start,
                     small->count, small->hist);
            large->hist = nd->hist;
            nd->hist    = NULL;
            for (size_t k = 0; k < 2 * c.total_cells; ++k)
            {
                large->hist[k] -= small->hist[k];
            }
            node_totals(&c, small);
            node_totals(&c, large);
            t->covers[lid] = (float)nl;
            t->covers[rid] = (float)nr;
            /* propagate_monotone_bounds (src/grower_impl.hpp:52-80) */
            L->lo = R->lo = nd->lo;
            L->hi = R->hi = nd->hi;
            int const mc  = monotone_of(cfg, f);
            if (mc != 0)
            {
                double const wl  = bounded_leaf_weight(L->sum_g, L->sum_h, cfg->lambda_l1,
                                                       cfg->lambda_l2, nd->lo, nd->hi);
                double const wr  = bounded_leaf_weight(R->sum_g, R->sum_h, cfg->lambda_l1,
                                                       cfg->lambda_l2, nd->lo, nd->hi);
                double const mid = 0.5 * (wl + wr);
                if (mc > 0)
                {
                    L->hi = L->hi < mid ? L->hi : mid;
                    R->lo = R->lo > mid ? R->lo : mid;
                }
                else
                {
                    L->lo = L->lo > mid ? L->lo : mid;
                    R->hi = R->hi < mid ? R->hi : mid;
                }
            }
        }
        free(sp);
        for (size_t i = 0; i < n_cur; ++i)
        {
            free(cur[i].hist);
        }
        free(cur);
        cur   = next;
        n_cur = n_next;
        if (n_cur == 0)
        {
            break;
        }
        ++depth;
    }
    if (rc == 0)
    {
        /* end_tree: the surviving frontier becomes leaves (level.hpp:116-126) */
        for (size_t i = 0; i < n_cur; ++i)
        {
            finalize_leaf(&c, &cur[i], order, values, leaf_ids);
        }
        t->depth = depth;
        /* route_unsampled (src/grower_impl.hpp:438-461) */
        if (n_rows < n)
        {
            uint8_t *in = (uint8_t *)calloc(n, 1);
            for (size_t k = 0; k < n_rows; ++k)
            {
                in[rows[k]] = 1;
            }
            for (size_t r = 0; r < n; ++r)
            {
                if (in[r])
                {
                    continue;
                }
                uint32_t idx = 0;
                while (t->feature[idx] != LEAF_FLAG)
                {
                    uint32_t const f = t->feature[idx];
                    uint32_t const b = bins[((size_t)f * n) + r];
                    idx = routes_left(b, n_bins[f] - 1, t->split_bin[idx],
                                      t->default_left[idx])
                              ? t->left[idx]
                              : t->right[idx];
                }
                values[r]   = t->value[idx];
                leaf_ids[r] = idx;
            }
            free(in);
        }
    }
    for (size_t i = 0; i < n_cur; ++i)
    {
        free(cur[i].hist);
    }
    free(cur);
    free(order);
    free(tmp);
    free(c.off);
    return rc;
}

/* ---- objectives and the boosting loop ------------------------------------- */

void orc_gradients(int objective, float const *scores, float const *labels, size_t n,
                   float *grad, float *hess)
{
    for (size_t i = 0; i < n; ++i)
    {
        if (objective == 0)
        {
            grad[i] = scores[i] - labels[i];
            hess[i] = 1.0F;
        }
        else
        {
            float const p = 1.0F / (1.0F + expf(-scores[i]));
            grad[i]       = p - labels[i];
            hess[i]       = p * (1.0F - p);
        }
    }
}

float orc_init_score(int objective, float const *labels, size_t n)
{
    float sum = 0.0F;
    for (size_t i = 0; i < n; ++i)
    {
        sum += labels[i];
    }
    float const nn = (float)n;
    if (objective == 0)
    {
        return sum / nn;
    }
    float const p = sum / nn;
    return logf(p / (1.0F - p));
}

int orc_train_depthwise(uint16_t const *bins, size_t n, size_t F,
                        uint32_t const *n_bins, float const *cuts,
                        uint32_t const *cut_off, float const *labels, int objective,
                        uint32_t n_iters, float learning_rate, orc_tree_cfg const *cfg,
                        orc_tree *trees, float *init_score, float *scores)
{
    float    *grad   = (float *)malloc(sizeof(float) * n);
    float    *hess   = (float *)malloc(sizeof(float) * n);
    float    *vals   = (float *)malloc(sizeof(float) * n);
    uint32_t *ids    = (uint32_t *)malloc(sizeof(uint32_t) * n);
    uint32_t *rows   = (uint32_t *)malloc(sizeof(uint32_t) * n);
    uint32_t *sel    = (uint32_t *)malloc(sizeof(uint32_t) * F);
    float const init = orc_init_score(objective, labels, n);
    int         rc   = 0;
    *init_score      = init;
    for (size_t i = 0; i < n; ++i)
    {
        scores[i] = init;
        rows[i]   = (uint32_t)i;
    }
    for (size_t f = 0; f < F; ++f)
    {
        sel[f] = (uint32_t)f;
    }
    for (uint32_t it = 0; it < n_iters && rc == 0; ++it)
    {
        orc_gradients(objective, scores, labels, n, grad, hess);
        rc = orc_grow_depthwise(bins, n, F, n_bins, cuts, cut_off, grad, hess, rows, n,
                                sel, F, cfg, &trees[it], vals, ids);
        for (size_t i = 0; i < n; ++i)
        {
            scores[i] += learning_rate * vals[i];
        }
    }
    free(grad);
    free(hess);
    free(vals);
    free(ids);
    free(rows);
    free(sel);
    return rc;
}

void orc_predict_binned(uint16_t const *bins, size_t n, uint32_t const *n_bins,
                        orc_tree const *trees, size_t n_trees, float init, float lr,
                        float *out)
{
    for (size_t r = 0; r < n; ++r)
    {
        out[r] = 0.0F;
    }
    for (size_t t = 0; t < n_trees; ++t)
    {
        orc_tree const *tr = &trees[t];
        for (size_t r = 0; r < n; ++r)
        {
            uint32_t idx = 0;
            while (tr->feature[idx] != LEAF_FLAG)
            {
                uint32_t const f = tr->feature[idx];
                uint32_t const b = bins[((size_t)f * n) + r];
                idx = routes_left(b, n_bins[f] - 1, tr->split_bin[idx],
                                  tr->default_left[idx])
                          ? tr->left[idx]
                          : tr->right[idx];
            }
            out[r] += tr->value[idx];
        }
    }
    for (size_t r = 0; r < n; ++r)
    {
        out[r] = init + (out[r] * lr);
    }
}
