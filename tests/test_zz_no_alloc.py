"""The allocation-free FP64 direct type-1 sum (nnb_direct_type1_f64_noalloc).

It serves callers that cannot call cudaMalloc (for example code running inside a memory pool
that owns the whole device, or code that must not allocate after start-up): its scratch is a
fixed array in the library's own device memory. This test calls it through the C ABI twice in
a row and checks both results against the allocating entry point nnb_direct_type1_f64 on the
same inputs, within the tolerance of the other FP64 direct-sum checks (1e-12 relative), and that
the two calls agree bit for bit (the partial sums are added in a fixed order). The rejection of a
request beyond the fixed scratch is tested without a GPU (tests/test_capi_cpu.py), so that a
regressed size check fails there with an error instead of reading past buffers here. The file is
named so that pytest collects it last; it also passes when run alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _call(lib, fn, dim, sign, loc, c, kidx, out):
    from neonufft_b200 import _lib as L
    ptrs = L.ptr_array([t.data_ptr() for t in loc])
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    return getattr(lib, fn)(dim, sign, int(loc[0].numel()), ptrs, c.data_ptr(),
                            int(kidx.shape[0]), kidx.data_ptr(), out.data_ptr(), stream)


def test_noalloc_direct_type1_matches_allocating_entry_point(cuda, engine):
    import torch
    from neonufft_b200 import _lib as L
    lib = L.load()
    rng = np.random.default_rng(31)
    dim, M, S = 3, 20000, 257
    loc = [torch.from_numpy(rng.uniform(-np.pi, np.pi, M)).cuda() for _ in range(dim)]
    c = torch.from_numpy(rng.standard_normal(M) + 1j * rng.standard_normal(M)).cuda()
    kidx = torch.from_numpy(rng.integers(-40, 40, size=(S, dim)).astype(np.int64)).cuda()
    ref = torch.zeros(2 * S, dtype=torch.float64, device="cuda")
    assert _call(lib, "nnb_direct_type1_f64", dim, -1, loc, c, kidx, ref) == 0
    first = None
    for _ in range(2):
        out = torch.full((2 * S,), float("nan"), dtype=torch.float64, device="cuda")
        assert _call(lib, "nnb_direct_type1_f64_noalloc", dim, -1, loc, c, kidx, out) == 0
        torch.cuda.synchronize()
        r = ref.cpu().numpy()
        o = out.cpu().numpy()
        assert np.all(np.isfinite(o))
        assert np.linalg.norm(o - r) <= 1e-12 * np.linalg.norm(r)
        if first is None:
            first = o
        else:
            assert np.array_equal(o, first)  # fixed-order reduction: bit-reproducible

