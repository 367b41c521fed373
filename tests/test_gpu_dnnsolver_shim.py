"""The C++ dnnsolver classes (include/drwc_dnnsolver.hpp) on the device give
the Python mirror's results bit for bit: Poisson and first-hop samples (same
Philox seed and stream sequence), ParallelSampler results in submission
order (batching does not change a query's draw), the reference's exceptions,
and structureConstruction's maxima."""
import subprocess

import numpy as np
import pytest

from deeprwcap_b200 import engine
from deeprwcap_b200 import workloads as W
from test_dnnsolver_shim import build_shim

pytestmark = pytest.mark.gpu


def test_cpp_classes_match_python_mirror(ctx, tmp_path):
    n = 37
    L, Cb = W.query_batch(n, seed=5)
    ax = np.random.default_rng(5).integers(0, 3, n).astype(np.int32)
    q = tmp_path / "q.bin"
    with open(q, "wb") as f:
        np.array([n], dtype=np.int32).tofile(f)
        L.tofile(f)
        Cb.tofile(f)
        ax.tofile(f)
    exe = build_shim(tmp_path / "shim")
    r = subprocess.run([str(exe), str(q), str(tmp_path / "o.bin")], capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, (r.returncode, r.stderr)
    assert "will be ignored" in r.stderr
    got = np.fromfile(tmp_path / "o.bin", dtype=np.float32)
    assert got.size == 3 * n + 3 * n + 5 * n + 3 * n + 5 * n + n
    p = engine.DNNSolverPoisson(0)
    first = np.array(p.sample(L, Cb), dtype=np.float32)
    second = np.array(p.sample(L, Cb), dtype=np.float32)
    grad = np.array(engine.DNNSolverGrad(0).sample(L, Cb, ax), dtype=np.float32)
    _, mx = p.structureConstruction(L, Cb)
    o = 0
    for want in (first, second, grad, first, grad, mx):
        np.testing.assert_array_equal(got[o:o + want.size], want)
        o += want.size
