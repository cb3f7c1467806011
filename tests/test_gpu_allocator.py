"""Plans whose device buffers come from the caller's allocator (the reference's
neonufft::Allocator, through the C ABI's allocate / deallocate callbacks).

The allocator here returns addresses 16 bytes past a 256-byte boundary: every buffer is 16-byte
aligned (what the kernels' vector accesses need) but none is 32-byte aligned, so the binning
scatter takes its two-16-byte-store form instead of the single 256-bit store. Results must match
a plan on the engine's own allocator and the FP64 direct sums, for type 1, type 2 and several
type-1 transforms of one point set (whose extra fine grids come from the same allocator).
"""
import numpy as np
import pytest

from gpu_helpers import col_strides, tdtypes
from test_gpu_methods import direct

pytestmark = pytest.mark.gpu


class OffsetAllocator:
    """Device memory from torch, handed out 16 bytes past the tensor's (256-byte aligned)
    start; counts the allocations it served."""

    def __init__(self, torch):
        self.torch = torch
        self.live = {}
        self.count = 0

    def allocate(self, size):
        t = self.torch.empty(int(size) + 64, dtype=self.torch.uint8, device="cuda")
        p = t.data_ptr() + 16
        assert p % 32 == 16
        self.live[p] = t
        self.count += 1
        return p

    def deallocate(self, ptr):
        self.live.pop(int(ptr), None)


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_plan_on_a_16_byte_aligned_allocator(dtype, cuda, engine, oracle):
    torch = cuda
    rdt, cdt, npc = tdtypes(torch, dtype)
    rng = np.random.default_rng(61)
    M, modes, count = 20_000, [24, 20, 16], 3
    nm = int(np.prod(modes))
    pts = [rng.uniform(-np.pi, np.pi, M) for _ in range(3)]
    loc = [torch.from_numpy(p.astype(np.dtype(dtype))).cuda() for p in pts]
    vecs = [rng.standard_normal(M) + 1j * rng.standard_normal(M) for _ in range(count)]
    inp = torch.from_numpy(np.concatenate(vecs).astype(npc)).cuda()
    f = rng.standard_normal(nm) + 1j * rng.standard_normal(nm)
    fin = torch.from_numpy(f.astype(npc)).cuda()
    tol = 1e-6 if dtype == "float32" else 1e-9
    results = {}
    for name in ("offset", "default"):
        alloc = OffsetAllocator(torch) if name == "offset" else None
        plan = engine.Plan(engine.Options(tol=tol, n_spread=8 if dtype == "float32" else 0,
                                          tile=(4, 4, 1) if dtype == "float32" else (0, 0, 0)),
                           -1, M, loc, modes, device_alloc=alloc)
        one = torch.empty(nm, dtype=cdt, device="cuda")
        plan.transform_type_1(inp[:M], one, col_strides(modes))
        many = torch.empty(count * nm, dtype=cdt, device="cuda")
        plan.transform_type_1_many(inp, many, count, col_strides(modes))
        two = torch.empty(M, dtype=cdt, device="cuda")
        plan.transform_type_2(fin, col_strides(modes), two)
        torch.cuda.synchronize()
        results[name] = (one.cpu().numpy(), many.cpu().numpy().reshape(count, nm),
                         two.cpu().numpy())
        plan.close()
        if alloc is not None:
            assert alloc.count > 0 and not alloc.live  # every buffer returned
    same = 1e-6 if dtype == "float32" else 1e-12
    for a, b in zip(results["offset"], results["default"]):
        assert np.all(np.isfinite(a))
        assert oracle.rel_l2(a, b) < same
    one, many, two = results["offset"]
    ref1 = direct(oracle, 1, -1, pts, vecs[0], modes, dtype)
    bound = 2e-6 if dtype == "float32" else 1e-8
    assert oracle.rel_l2(one, ref1) < bound
    for v in range(count):
        assert oracle.rel_l2(many[v], direct(oracle, 1, -1, pts, vecs[v], modes, dtype)) < bound
    sample = rng.integers(0, M, 400)
    ref2 = direct(oracle, 2, -1, [p[sample] for p in pts], f, modes, dtype)
    assert oracle.rel_l2(two[sample], ref2) < bound
