"""CPU checks of the C ABI boundary: the library loads without a GPU and
exports every entry point include/*.h declares; host-side logic (cut
fitting) matches the reference."""

from __future__ import annotations

import ctypes as C
import glob
import os
import re

import numpy as np
import pytest
from conftest import ROOT, load_golden


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(bb_[a-z0-9_]+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    from bonsai_b200.build import LIB, build_library
    build_library()
    lib = C.CDLL(LIB)
    declared = _declared()
    assert len(declared) >= 15
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing


def test_library_reports_no_device_without_raising():
    import bonsai_b200 as bb
    assert bb.available() in (True, False)


def test_error_text_of_a_refused_call():
    """A device call with a null plane fails with a status, not a crash,
    and sets the thread's error text."""
    import bonsai_b200 as bb
    from bonsai_b200._lib import lib
    rc = lib().bb_ingest(None, 0, 0, 0, None, None, C.byref(C.c_void_p()))
    assert rc != 0
    assert lib().bb_last_error().decode()


def test_fit_cuts_matches_golden():
    import bonsai_b200 as bb
    from bonsai_b200 import synth
    d = load_golden("small_regression.npz")
    X, _ = synth.regression_small()
    cuts, off = bb.fit_cuts(X)
    assert np.array_equal(off, d["cut_off"])
    assert np.array_equal(cuts.view(np.uint32), d["cuts"].view(np.uint32))
    m = load_golden("missing_values.npz")
    cuts, off = bb.fit_cuts(m["X"])
    assert np.array_equal(off, m["cut_off"])
    assert np.array_equal(cuts.view(np.uint32), m["cuts"].view(np.uint32))


@pytest.mark.parametrize("seed", range(4))
def test_fit_cuts_matches_reference_live(ref, seed):
    import bonsai_b200 as bb
    rng = np.random.Generator(np.random.PCG64(seed))
    n = 5000
    X = np.stack([
        rng.standard_normal(n),                                   # quantile stride
        rng.integers(0, 12, n),                                   # distinct values
        np.where(rng.random(n) < 0.8, 0.0, rng.standard_normal(n)),  # heavy value: greedy
        np.round(rng.lognormal(0, 1, n), 1),                      # duplicates
    ], 1).astype(np.float32)
    X[rng.random((n, 4)) < 0.1] = np.nan
    for max_bin in (16, 63, 255):
        rc, ro = ref.fit_cuts(X, max_bin=max_bin)
        cuts, off = bb.fit_cuts(X, max_bin=max_bin)
        assert np.array_equal(off, ro), max_bin
        assert np.array_equal(cuts.view(np.uint32), rc.view(np.uint32)), max_bin


def test_fit_cuts_signed_zeros_match_reference(ref):
    """Runs of zeros of both signs: the reference sorts samples of 2,048 or
    more values by radix key, so the run's representative is -0.0 whenever
    one is present; the restatement sorts the same way."""
    import bonsai_b200 as bb
    rng = np.random.Generator(np.random.PCG64(3))
    n = 3000
    X = np.stack([np.array([0.0, -0.0, 1.0] * 1000),
                  rng.choice([-0.0, 0.0, 2.5], n),
                  np.where(rng.random(n) < 0.5, -0.0, rng.standard_normal(n))], 1)
    X = X.astype(np.float32)
    rc, ro = ref.fit_cuts(X)
    cuts, off = bb.fit_cuts(X)
    assert np.array_equal(off, ro)
    assert np.array_equal(cuts.view(np.uint32), rc.view(np.uint32))


@pytest.mark.parametrize("py_name,c_name", [("TrainCfg", "bb_train_cfg"),
                                             ("Profile", "bb_profile")])
def test_struct_layout_matches_the_header(tmp_path, py_name, c_name):
    """The Python binding's structs (bonsai_b200._lib) have the C header's
    layout: every field at the header's offset, the same size (fields are
    appended over time; a mismatch would pass wrong values silently)."""
    import shutil
    import subprocess
    from bonsai_b200 import _lib
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    T = getattr(_lib, py_name)
    fields = [f[0] for f in T._fields_]
    src = tmp_path / "layout.c"
    src.write_text("#include <stddef.h>\n#include <stdio.h>\n#include \"bonsai_b200.h\"\n"
                   "int main(void) {\n"
                   + "".join(f'  printf("{f} %zu\\n", offsetof({c_name}, {f}));\n'
                             for f in fields)
                   + f'  printf("sizeof %zu\\n", sizeof({c_name}));\n  return 0;\n}}\n')
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True)
    got = dict(line.split() for line in subprocess.run(
        [str(exe)], check=True, capture_output=True, text=True).stdout.splitlines())
    for f in fields:
        assert int(got[f]) == getattr(T, f).offset, f
    assert int(got["sizeof"]) == C.sizeof(T)


def _extreme_columns(rng, n=5000):
    """Greedy-rule columns (a value heavier than a mean bin) at magnitudes
    where the cut's midpoint matters: above FLT_MAX / 2, where a plain
    (a + b) / 2 overflows; mixed huge and subnormal neighbours (one operand
    added whole); subnormal and near-subnormal runs; the float extremes."""
    big = rng.uniform(2e38, 3.4e38, n)
    heavy = rng.random(n) < 0.4
    tiny = rng.uniform(-1.2e-38, 1.2e-38, n)
    cols = [
        np.where(heavy, 2.5e38, big),                                   # huge, one sign
        np.where(heavy, -2.5e38, -big),                                 # its mirror
        np.where(heavy, 0.0, rng.choice([-1.0, 1.0], n) * big),         # huge either side of 0
        np.where(heavy, 1e-42, rng.choice([-1.0, 1.0], n) * big),       # huge next to subnormal
        np.where(heavy, 1e-39, tiny),                                   # subnormal runs
        np.where(heavy, -3e-38, rng.uniform(-4e-38, 4e-38, n)),         # near the normal edge
        np.where(heavy, 1.0, rng.choice([-3.4028235e38, 3.4028235e38, 1.7e38, -1.7e38], n)),
        np.where(heavy, 3e38, rng.choice([np.inf, -np.inf, 1e38], n)),  # infinities
    ]
    return np.stack(cols, 1).astype(np.float32)


def test_midpoint_follows_std_midpoint():
    """The greedy cut's midpoint never overflows and equals the half-sum in
    float where that is exact."""
    from bonsai_b200.binning import midpoint
    f = np.float32
    fmax = np.finfo(np.float32).max
    assert midpoint(f(3e38), f(3.2e38)) == f(3.1e38)
    assert midpoint(fmax, fmax) == fmax
    assert midpoint(-fmax, fmax) == 0.0
    assert midpoint(f(1.0), f(2.0)) == f(1.5)
    d = np.float32(1e-45)                      # the smallest subnormal
    assert midpoint(d, d) == d
    assert midpoint(f(-3e38), d) == f(-1.5e38)


@pytest.mark.parametrize("max_bin", [16, 255])
def test_fit_cuts_extreme_magnitudes_match_reference(ref, max_bin):
    import bonsai_b200 as bb
    X = _extreme_columns(np.random.Generator(np.random.PCG64(41)))
    rc, ro = ref.fit_cuts(X, max_bin=max_bin)
    cuts, off = bb.fit_cuts(X, max_bin=max_bin)
    assert np.array_equal(off, ro)
    assert np.array_equal(cuts.view(np.uint32), rc.view(np.uint32))
