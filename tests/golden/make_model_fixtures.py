"""Copies the reference's two committed format-v7 model files (its
tests/data/fixture_v7_regressor.bonsai and fixture_v7_softmax.bonsai, the
vectors of its "committed v7 fixtures re-save byte-identically" test,
tests/unit/test_model_io.cpp:269-296) into tests/golden/ as
model_v7_regressor.bonsai and model_v7_softmax.bonsai.

    python tests/golden/make_model_fixtures.py /path/to/reference
"""

import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_model_fixtures.py <reference source tree>")
    ref = sys.argv[1]
    for kind in ("regressor", "softmax"):
        shutil.copyfile(os.path.join(ref, "tests", "data", f"fixture_v7_{kind}.bonsai"),
                        os.path.join(HERE, f"model_v7_{kind}.bonsai"))
