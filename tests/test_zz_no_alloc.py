"""tbpm_cheb_timestep_noalloc: the time step for callers that cannot allocate.

Some callers cannot call cudaMalloc, nor let a library call it: a framework
whose caching allocator already holds nearly all of HBM, or a loop where
allocation after start-up is forbidden.  They pass their own device buffers
(here: tensors from torch's allocator), and the entry point takes its
Chebyshev work vectors from a fixed 16 MiB array inside the library.

The tests compare two consecutive calls of the entry point with two calls of
the allocating entry point tbpm_cheb_timestep, and with the oracle's time step
at exactly the largest size the work array holds (several sweeps of the
persistent grid), to the 1e-12 relative tolerance of the time-step tests.
They check that one value more, invalid CSR input, a misaligned view and a
host pointer are rejected before any launch.  The file is collected last, so
that a run that stops at the first failure has run every other test first;
it also passes alone in a fresh process.
"""

import math

import numpy as np
import pytest

import tbplas_b200 as tb
from tbplas_b200 import _native as nat

from conftest import bessel_series, rel_err, unit_states
from oracle import oracle

pytestmark = pytest.mark.gpu

MAX_VALUES = ((16 << 20) - 256) // 32  # n_rows * n_states the work array holds
assert MAX_VALUES == 524280


def _device_csr(torch, h):
    dev = torch.device("cuda", 0)
    ip = torch.from_numpy(h.indptr.astype(np.int32)).to(dev)
    ix = torch.from_numpy(h.indices.astype(np.int32)).to(dev)
    hv = torch.from_numpy(np.ascontiguousarray(h.data).view(np.float64)).to(dev)
    return ip, ix, hv


def _noalloc_step(ctx, bes, ip, ix, hv, n, nnz, wf_dev, n_states, forward):
    ctx.call("tbpm_cheb_timestep_noalloc", nat.ptr(bes), bes.size, ip.data_ptr(),
             ix.data_ptr(), hv.data_ptr(), n, nnz, wf_dev.data_ptr(), n_states,
             1 if forward else 0)


@pytest.mark.parametrize("forward", [True, False])
def test_noalloc_matches_allocating_entry_point_twice(forward):
    import torch
    s = tb.make_graphene_sample(24, 20, disorder=1.0, rescale=9.0, seed=17)
    h = s.build_ham_csr()
    n, nnz, ns = h.shape[0], h.nnz, 4
    bes = np.asarray(bessel_series(math.pi))
    wf0 = unit_states(ns, n, seed=23)  # (n_states, n)

    # reference: the allocating entry point, twice
    ctx_ref = nat.Context(0)
    ip32, ix32 = h.indptr.astype(np.int32), h.indices.astype(np.int32)
    hv = np.ascontiguousarray(h.data)
    ctx_ref.call("tbpm_ham_upload", nat.ptr(ip32), nat.ptr(ix32), nat.ptr(hv), n, nnz, None,
                 None, s.rescale)
    ref = np.ascontiguousarray(wf0.copy())
    ctx_ref.call("tbpm_cheb_timestep", nat.ptr(bes), bes.size, nat.ptr(ref), ns,
                 1 if forward else 0)
    ref1 = ref.copy()
    ctx_ref.call("tbpm_cheb_timestep", nat.ptr(bes), bes.size, nat.ptr(ref), ns,
                 1 if forward else 0)
    ref2 = ref.copy()
    ctx_ref.close()

    # the no-alloc entry point on caller-owned device buffers, twice
    ctx = nat.Context(0)
    ip, ix, hvd = _device_csr(torch, h)
    inter = np.ascontiguousarray(wf0.T)  # row-interleaved [n][n_states]
    wf_dev = torch.from_numpy(inter.view(np.float64)).to(torch.device("cuda", 0))
    _noalloc_step(ctx, bes, ip, ix, hvd, n, nnz, wf_dev, ns, forward)
    got1 = wf_dev.cpu().numpy().view(np.complex128).reshape(n, ns).T
    _noalloc_step(ctx, bes, ip, ix, hvd, n, nnz, wf_dev, ns, forward)
    got2 = wf_dev.cpu().numpy().view(np.complex128).reshape(n, ns).T
    ctx.close()
    assert rel_err(got1, ref1) < 1e-12
    assert rel_err(got2, ref2) < 1e-12
    assert np.allclose(np.linalg.norm(got2, axis=1), 1.0, atol=1e-12)


def test_noalloc_rejects_oversized_and_invalid_input():
    import torch
    ctx = nat.Context(0)
    bes = np.asarray(bessel_series(math.pi))
    s = tb.make_graphene_sample(8, 8, rescale=9.0)
    h = s.build_ham_csr()
    ip, ix, hvd = _device_csr(torch, h)
    wf = torch.zeros(2 * h.shape[0] * 2, dtype=torch.float64, device="cuda")
    # n_rows * n_states beyond the fixed work array: rejected before any launch
    big_rows = MAX_VALUES // 2 + 1
    with pytest.raises(ValueError, match="16 MiB"):
        ctx.call("tbpm_cheb_timestep_noalloc", nat.ptr(bes), bes.size, ip.data_ptr(),
                 ix.data_ptr(), hvd.data_ptr(), big_rows, h.nnz, wf.data_ptr(), 2, 1)
    # a column index out of range: found by the device-side check
    bad = h.indices.astype(np.int32).copy()
    bad[5] = h.shape[0] + 3
    ix_bad = torch.from_numpy(bad).to("cuda")
    with pytest.raises(ValueError, match="column index"):
        ctx.call("tbpm_cheb_timestep_noalloc", nat.ptr(bes), bes.size, ip.data_ptr(),
                 ix_bad.data_ptr(), hvd.data_ptr(), h.shape[0], h.nnz, wf.data_ptr(), 2, 1)
    ctx.close()


@pytest.mark.parametrize("forward", [True, False])
def test_noalloc_at_the_size_limit_matches_oracle(forward):
    """255 x 257 graphene cells = 131,070 rows x 4 states = 524,280 values, the
    largest request the work array holds.  With 32 rows per 128-thread block
    that is 4,096 row tiles, more than the 148 x 16 blocks a B200 can hold at
    once, so every block sweeps the rows more than once."""
    import torch
    s = tb.make_graphene_sample(255, 257, disorder=1.0, rescale=9.0, seed=29)
    h = s.build_ham_csr()
    n, nnz, ns = h.shape[0], h.nnz, 4
    assert n * ns == MAX_VALUES
    bes = np.asarray(bessel_series(math.pi))
    wf0 = unit_states(ns, n, seed=37)
    ctx = nat.Context(0)
    ip, ix, hvd = _device_csr(torch, h)
    wf_dev = torch.from_numpy(np.ascontiguousarray(wf0.T).view(np.float64)).to("cuda")
    ref = wf0.copy()
    for _ in range(2):
        _noalloc_step(ctx, bes, ip, ix, hvd, n, nnz, wf_dev, ns, forward)
        got = wf_dev.cpu().numpy().view(np.complex128).reshape(n, ns).T
        ref = np.stack([oracle.cheb_timestep(bes, h.indptr, h.indices, h.data, ref[b],
                                             forward=forward) for b in range(ns)])
        assert rel_err(got, ref) < 1e-12
    ctx.close()


def test_noalloc_rejects_one_value_over_the_limit_misaligned_and_host_buffers():
    import torch
    ctx = nat.Context(0)
    bes = np.asarray(bessel_series(math.pi))
    s = tb.make_graphene_sample(8, 8, rescale=9.0)
    h = s.build_ham_csr()
    n, nnz = h.shape[0], h.nnz
    ip, ix, hvd = _device_csr(torch, h)
    wf = torch.zeros(2 * n * 2 + 2, dtype=torch.float64, device="cuda")
    # 131,071 rows x 4 states = MAX_VALUES + 4 (the size is checked first)
    with pytest.raises(ValueError, match="16 MiB"):
        ctx.call("tbpm_cheb_timestep_noalloc", nat.ptr(bes), bes.size, ip.data_ptr(),
                 ix.data_ptr(), hvd.data_ptr(), MAX_VALUES // 4 + 1, nnz, wf.data_ptr(), 4, 1)
    # a view of wf offset by one double: 8-byte aligned only
    with pytest.raises(ValueError, match="aligned"):
        ctx.call("tbpm_cheb_timestep_noalloc", nat.ptr(bes), bes.size, ip.data_ptr(),
                 ix.data_ptr(), hvd.data_ptr(), n, nnz, wf[1:].data_ptr(), 2, 1)
    # hop offset by one double
    hv_off = torch.zeros(hvd.numel() + 1, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError, match="hop must be 16-byte aligned"):
        ctx.call("tbpm_cheb_timestep_noalloc", nat.ptr(bes), bes.size, ip.data_ptr(),
                 ix.data_ptr(), hv_off[1:].data_ptr(), n, nnz, wf.data_ptr(), 2, 1)
    # a host buffer in place of wf
    host = np.zeros(2 * n * 2, dtype=np.float64)
    with pytest.raises(ValueError, match="device"):
        ctx.call("tbpm_cheb_timestep_noalloc", nat.ptr(bes), bes.size, ip.data_ptr(),
                 ix.data_ptr(), hvd.data_ptr(), n, nnz, nat.ptr(host), 2, 1)
    # nothing above was launched: the context still runs a valid call
    ctx.call("tbpm_cheb_timestep_noalloc", nat.ptr(bes), bes.size, ip.data_ptr(),
             ix.data_ptr(), hvd.data_ptr(), n, nnz, wf.data_ptr(), 2, 1)
    ctx.close()
