"""The bounds-checked build (HYALITE_CUDA_BUILD=bounds, libhyalite_cuda_bounds.so): every scan
kernel verifies, before it uses an item, each index the item's metadata and residue codes can
produce (residue columns, boundary region, db indices, profile letters) and reports DeviceCheck
instead of reading outside an array. Run on the small parity cases, it must find nothing and give
the oracle's results. It runs in a child process because the library is chosen at import."""
import os
import subprocess
import sys

import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu


def test_small_parity_cases_under_the_bounds_checked_build():
    lib = os.path.join(ROOT, "hyalite_b200", "libhyalite_cuda_bounds.so")
    if not os.path.exists(lib):
        pytest.fail("the bounds-checked build is missing: make -C hyalite_b200/csrc bounds")
    env = dict(os.environ, HYALITE_CUDA_BUILD="bounds")
    files = ["tests/test_scan_gpu.py", "tests/test_layout_gpu.py", "tests/test_batch_gpu.py",
             "tests/test_zz_no_alloc.py"]
    r = subprocess.run([sys.executable, "-m", "pytest", "-q", "-m", "gpu", "-p", "no:cacheprovider"] + files,
                       cwd=ROOT, env=env, capture_output=True, text=True, timeout=1800)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-2000:]
    assert " passed" in r.stdout and "failed" not in r.stdout
