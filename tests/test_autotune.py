"""The launch-shape autotuner: cache keys and persistence on the host, and on
the GPU that every candidate it times computes the same correlation."""

import math

import numpy as np
import pytest

from tbplas_b200 import autotune
from tbplas_b200.fortran import f2py

from conftest import bessel_series, rel_err


def test_cache_roundtrip_and_lookup(tmp_path):
    path = str(tmp_path / "tune.json")
    assert autotune.load_cache(path) == {}
    key = autotune._key("fp32", 16, 1 << 20, 3 << 20)
    assert key == "fp32/ld16/2^20rows/3.0nnz"
    autotune.save({"key": key, "best": {"threads_per_block": 256, "vector_width": 2,
                                        "ms_per_step": 1.0}}, path)
    autotune.save({"key": "fp64/ld8/2^19rows/3.0nnz",
                   "best": {"threads_per_block": 128, "vector_width": 0, "ms_per_step": 2.0}},
                  path)
    got = autotune.lookup("fp32", 16, 1 << 20, 3 << 20, path)
    assert got == {"threads_per_block": 256, "vector_width": 2, "ms_per_step": 1.0}
    assert autotune.lookup("fp32", 8, 1 << 20, 3 << 20, path) is None
    saved = f2py.get_backend()
    try:
        autotune.apply(got)
        b = f2py.get_backend()
        assert b["threads_per_block"] == 256 and b["vector_width"] == 2
    finally:
        f2py.set_backend(threads_per_block=saved["threads_per_block"],
                         vector_width=saved["vector_width"])


def test_corrupt_cache_reads_as_empty(tmp_path):
    p = tmp_path / "tune.json"
    p.write_text("{not json")
    assert autotune.load_cache(str(p)) == {}


@pytest.mark.gpu
def test_tuned_shapes_compute_the_same_correlation():
    import tbplas_b200 as tb
    s = tb.make_graphene_sample(40, 36, disorder=1.0, rescale=9.0, seed=3)
    h = s.build_ham_csr()
    bes = bessel_series(2 * math.pi / 18.0 * 9.0)
    r = autotune.tune_dos(h.indptr, h.indices, h.data, 4, "fp32", threads=(64, 256), steps=2,
                          bessel=bes)
    assert len(r["timings"]) == 6 and r["best"] in r["timings"]  # widths 0, 1, 2 x 2 shapes
    assert all(t["ms_per_step"] > 0 for t in r["timings"])
    saved = f2py.get_backend()
    ref = None
    try:
        for t in r["timings"]:
            f2py.set_backend(precision="fp32", threads_per_block=t["threads_per_block"],
                             vector_width=t["vector_width"])
            c = f2py.tbpm_dos(bes, h.indptr, h.indices, h.data, 7, 24, 4, "", 0, 128, 1e-9)
            if ref is None:
                ref = c
            assert rel_err(c, ref) < 1e-6
    finally:
        f2py.set_backend(precision="fp64", threads_per_block=saved["threads_per_block"],
                         vector_width=saved["vector_width"])
