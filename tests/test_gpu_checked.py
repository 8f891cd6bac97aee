"""The bounds-checked build (lib/libcgb_checked.so, compiled with
-DCGB_CHECKED): every stream index, gathered column and output row of the
single-system SpMVs is tested against its buffer, a failure recorded in a
check word and the access skipped (no trap).  Run over the row plan, a CSR
with an odd entry count (its last pair), the allocation-free entry on
unpadded caller buffers, both sliced instances with an L2 keep, and the
FP64, mixed and learned modes: no index may leave its buffer, and the
outputs must equal the normal build's bit for bit (the checks change no
arithmetic)."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "npb-gpu_b200", "lib")


def _run(lib, out):
    subprocess.run([sys.executable, os.path.join(ROOT, "tests", "checked_case.py"), lib, out],
                   check=True, timeout=900)
    return np.load(out)


def test_checked_build_no_index_leaves_its_buffer(tmp_path):
    checked = os.path.join(LIBDIR, "libcgb_checked.so")
    if not os.path.exists(checked):
        pytest.fail("lib/libcgb_checked.so is missing: run npb-gpu_b200/build.py --checked")
    c = _run(checked, str(tmp_path / "checked.npz"))
    n = _run(os.path.join(LIBDIR, "libcgb.so"), str(tmp_path / "normal.npz"))
    words = dict(zip(c["word_names"], c["words"]))
    assert all(v == 0 for v in words.values()), words
    assert all(v == -1 for v in n["words"])  # the normal build has no check word
    for key in n.files:
        if key in ("words", "word_names"):
            continue
        assert np.array_equal(c[key], n[key]), key
