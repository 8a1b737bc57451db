"""Interaction constraints (TreeConfig::interaction_constraints; the allowed-
feature state of src/grower_impl.hpp:83-160 and the mask check of
update_best_for_feature_for_node, src/split.cpp:111-114) on the device
growers, against the reference's own CPU growers: the whole node table and
every row's leaf bit for bit, for depthwise and leafwise trees and boosters,
under overlapping groups, a feature in no group, one-feature groups and the
TOML string forms; the quantised form's trees obey the constraints; the
levelwise grower and more than 64 groups are refused."""

from __future__ import annotations

import numpy as np
import pytest
from conftest import TREE_FIELDS

from oracle import TreeCfg

pytestmark = pytest.mark.gpu

LEAF = 0xFFFFFFFF
CONSTRAINTS = [["0,1", "2+5"], ["0,1,2", "2,3,4"], ["7"], ["0,1", "0,2", "1,2,3"],
               ["0+1+2+3+4+5+6+7"]]


def _data(seed, n=6_000, F=8):
    rng = np.random.Generator(np.random.PCG64(seed))
    X = rng.standard_normal((n, F)).astype(np.float32)
    X[rng.random((n, F)) < 0.05] = np.nan
    Z = np.nan_to_num(X)
    g = (Z[:, 0] * Z[:, 1] + Z[:, 2] * Z[:, 5] + 0.5 * np.sin(2 * Z[:, 3]) + 0.3 * Z[:, 7]
         + rng.normal(0, 0.1, n)).astype(np.float32)
    h = rng.uniform(0.5, 1.5, n).astype(np.float32)
    return X, g, h


def _same(a, b, where):
    n = len(b.feature)
    for k in TREE_FIELDS:
        x, y = np.asarray(getattr(a, k)), np.asarray(getattr(b, k))
        assert len(x) == n, (where, k)
        assert np.array_equal(x.view(np.uint8), y.view(np.uint8)), (where, k)


def _paths_ok(tree, groups):
    """Every root-to-leaf path's feature set lies inside one group, or is a
    single feature."""
    sets = [set(int(x) for x in g.replace("+", ",").split(",")) for g in groups]

    def walk(i, path):
        if tree.feature[i] == LEAF:
            return len(path) <= 1 or any(path <= s for s in sets)
        p = path | {int(tree.feature[i])}
        return walk(int(tree.left[i]), p) and walk(int(tree.right[i]), p)
    return walk(0, frozenset())


@pytest.mark.parametrize("groups", CONSTRAINTS)
@pytest.mark.parametrize("grower,cfg", [("depthwise", dict(max_depth=6)),
                                        ("leafwise", dict(max_leaves=40, max_depth=10))])
def test_tree_matches_reference(bb, ref, groups, grower, cfg):
    X, g, h = _data(len(groups) + len(grower))
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, np.zeros(len(X), np.float32), cuts, off)
    rt, rvals, rids, _ = ref.grow_tree(
        ds, TreeCfg(grower=grower, interaction_constraints=groups, **cfg), g, h)
    plane = bb.Plane(X, cuts, off)
    t, vals, ids = bb.grow_tree(
        plane, bb.TrainParams(grower=grower, interaction_constraints=groups, **cfg), g, h)
    _same(t, rt, (grower, groups))
    assert np.array_equal(vals.view(np.uint32), rvals.view(np.uint32))
    assert np.array_equal(ids, rids)
    assert _paths_ok(t, groups)


@pytest.mark.parametrize("grower", ["depthwise", "leafwise"])
def test_booster_matches_reference(bb, ref, grower):
    X, g, _ = _data(21, n=8_000)
    y = g
    groups = ["0,1", "2+5", "3,7"]
    cuts, off = ref.fit_cuts(X)
    ds = ref.dataset(X, y, cuts, off)
    m = ref.train(ds, TreeCfg(grower=grower, max_depth=6, max_leaves=31, n_iters=6,
                              interaction_constraints=groups))
    plane = bb.Plane(X, cuts, off)
    b = bb.Booster(plane, y, bb.TrainParams(grower=grower, max_depth=6, max_leaves=31,
                                            interaction_constraints=[[0, 1], [2, 5], [3, 7]],
                                            use_graph=True), max_trees=6)
    b.update(6)
    for i, rt in enumerate(m.trees()):
        _same(b.tree(i), rt, f"tree {i}")


def test_quantised_trees_obey_constraints(bb):
    X, g, h = _data(5, n=20_000)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    for groups in CONSTRAINTS:
        b = bb.Booster(plane, g, bb.TrainParams(max_depth=6, hist_mode="int8",
                                                interaction_constraints=groups), max_trees=4)
        b.update(4)
        assert all(_paths_ok(t, groups) for t in b.trees()), groups


def test_refusals(bb):
    X, g, h = _data(7, n=2_000)
    cuts, off = bb.fit_cuts(X)
    plane = bb.Plane(X, cuts, off)
    with pytest.raises(bb.ConfigError):
        bb.Booster(plane, g, bb.TrainParams(grower="levelwise", interaction_constraints=["0,1"]))
    with pytest.raises(bb.ConfigError):
        bb.Booster(plane, g, bb.TrainParams(interaction_constraints=[[k % 8] for k in range(65)]))
    with pytest.raises(bb.BonsaiError):
        bb.Booster(plane, g, bb.TrainParams(interaction_constraints=[[0, 9]]))
