"""The Jacobi cluster-size autotuner (wqc_cuda_autotune): a first call
measures and writes the fingerprinted cache, a second call on the same
machine loads it without measuring, a cache with another fingerprint is
measured again, and the tuned sizes leave results within the parity
tolerances of the oracle."""
import os
import time

import numpy as np
import pytest

import oracle as O
import wqc_cuda as W
from wqc_cuda import circuits as C

pytestmark = pytest.mark.gpu


def test_autotune_writes_then_reuses_its_cache(cuda_ctx, tmp_path):
    path = str(tmp_path / "jacobi-clusters")
    t0 = time.perf_counter()
    n1 = cuda_ctx.autotune(path)
    t1 = time.perf_counter()
    assert n1 == 16  # 4 chi values x 2 forms x 2 kinds of wave
    lines = open(path).read().splitlines()
    assert lines[0].startswith("wqc-jacobi-clusters v1|") and "|sm=" in lines[0]
    rows = [tuple(int(x) for x in ln.split()) for ln in lines[1:]]
    assert len(rows) == 16 and all(r[5] >= 1 for r in rows)
    n2 = cuda_ctx.autotune(path)
    t2 = time.perf_counter()
    assert n2 == n1 and (t2 - t1) < 0.25 * (t1 - t0)  # loaded, not measured
    with open(path, "w") as f:  # another machine's cache is not used
        f.write("wqc-jacobi-clusters v1|another device|sm=1\n32 32 32 16 0 1\n")
    assert cuda_ctx.autotune(path) == 16
    assert open(path).read().splitlines()[0] == lines[0]


def test_tuned_sizes_keep_parity(cuda_ctx, tmp_path):
    cuda_ctx.autotune(str(tmp_path / "jacobi-clusters"))
    w = C.config0()
    m = W.CudaMps(w.n, w.chi, ctx=cuda_ctx)
    m.apply_gates(w.gates)
    o = O.run(w.n, w.chi, w.gates)
    a, b = m.amplitude_zero(), o.amplitude_zero()
    assert abs(a - b) <= 1e-10 * abs(b)
    rec, ref = m.split_records(), o.records()
    assert np.array_equal(rec["chi"], ref["chi"]) and np.array_equal(rec["path"], ref["path"])
    assert os.path.exists(str(tmp_path / "jacobi-clusters"))
