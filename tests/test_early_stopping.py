"""The early-stopping rule bonsai_b200.early_stop_round applies to a device
loss record, against a direct restatement of the reference's per-round loop
(src/cli/pipeline.cpp:452-462: the first round is the best; a strictly lower
loss becomes the best; the fit stops, keeping best + 1 rounds, once a round
is `patience` rounds past the best). CPU only."""

from __future__ import annotations

import numpy as np
import pytest


def _loop(losses, patience):
    best_loss, best_iter = 0.0, 0
    for i, loss in enumerate(losses):
        if i == 0 or loss < best_loss:
            best_loss, best_iter = loss, i
        elif i - best_iter >= patience:
            return best_iter + 1, True
    return len(losses), False


@pytest.mark.parametrize("patience", [1, 2, 5, 20])
def test_rule_matches_the_loop(patience):
    from bonsai_b200 import early_stop_round
    rng = np.random.Generator(np.random.PCG64(patience))
    for trial in range(200):
        n = int(rng.integers(1, 60))
        # a falling curve that turns up, with noise and exact ties
        t = np.arange(n)
        losses = (1.0 / (1 + t) + 0.002 * t + rng.normal(0, 0.01, n)).astype(np.float32)
        if trial % 3 == 0:
            losses = np.round(losses, 2)
        assert early_stop_round(losses, patience) == _loop(list(losses), patience)


def test_rule_edge_cases():
    from bonsai_b200 import early_stop_round
    assert early_stop_round([], 3) == (0, False)
    assert early_stop_round([1.0], 1) == (1, False)
    assert early_stop_round([1.0, 1.0], 1) == (1, True)       # a tie is no improvement
    assert early_stop_round([2.0, 1.0, 1.5, 1.4, 1.3], 3) == (2, True)
    assert early_stop_round([3.0, 2.0, 1.0], 1) == (3, False)
