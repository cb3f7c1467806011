"""Several type-1 transforms of one point set (nnb_plan_transform_type_1_many) and the
two-vector z-window spreading behind it and behind type-3 batches.

Single-precision plans on the z-window kernels (default and 4-row tiles) spread two strength
vectors per pass (each staged point and its kernel values serve both); other plans run the
transforms one at a time. Either way every output must equal the single transform's (same
kernels: to 1e-6 relative in single precision, where only the atomic summation order
differs) and meet the tolerance against the FP64 direct sums, with odd counts (a lone last
vector), clustered points (work items split over CTAs) and type-3 batches of odd size. The FFTs
and deconvolutions of each pair run on an internal stream while the next pair spreads, on two
alternating sets of grids: counts of 5 and more reuse a set, and work enqueued on the plan's
stream after the call must see every output.
"""
import numpy as np
import pytest

from gpu_helpers import col_strides, tdtypes
from test_gpu_methods import direct

pytestmark = pytest.mark.gpu


def _run(engine, torch, dtype, pts, vecs, modes, **opt):
    rdt, cdt, npc = tdtypes(torch, dtype)
    loc = [torch.from_numpy(np.ascontiguousarray(p, dtype=np.dtype(dtype))).cuda() for p in pts]
    M, nm, count = len(pts[0]), int(np.prod(modes)), len(vecs)
    plan = engine.Plan(engine.Options(tol=opt.pop("tol", 1e-6), **opt), -1, M, loc, modes)
    inp = torch.from_numpy(np.concatenate(vecs).astype(npc)).cuda()
    many = torch.full((count * nm,), float("nan"), dtype=cdt, device="cuda")
    plan.transform_type_1_many(inp, many, count, col_strides(modes))
    singles = torch.zeros((count, nm), dtype=cdt, device="cuda")
    for v in range(count):
        plan.transform_type_1(inp[v * M:(v + 1) * M], singles[v], col_strides(modes))
    torch.cuda.synchronize()
    info = plan.info()
    plan.close()
    return many.cpu().numpy().reshape(count, nm), singles.cpu().numpy(), info


@pytest.mark.parametrize("tile", [(0, 0, 0), (4, 4, 1)])
@pytest.mark.parametrize("count", [2, 3, 4, 5, 8])
@pytest.mark.parametrize("case", ["uniform", "clustered"])
def test_many_single_precision_pairs(tile, count, case, cuda, engine, oracle):
    rng = np.random.default_rng(100 + count)
    modes = [20, 18, 16]
    if case == "clustered":  # ~9000 points in one column chunk: several work items
        pts = [np.concatenate([0.5 + rng.uniform(0, 0.02, 9000), rng.uniform(-np.pi, np.pi, 500)])
               for _ in range(3)]
    else:
        pts = [rng.uniform(-np.pi, np.pi, 6000) for _ in range(3)]
    M = len(pts[0])
    vecs = [rng.standard_normal(M) + 1j * rng.standard_normal(M) for _ in range(count)]
    many, singles, info = _run(engine, cuda, "float32", pts, vecs, modes, n_spread=8, tile=tile)
    assert info["spread_method"] == 3
    # ~9000 clustered points land on the same cells and their column splits into several work
    # items whose partial grids meet in float atomics: the single-precision sums of two runs
    # differ by about 2e-6, so the bound against the FP64 direct sums is 4e-6 there.
    bound = 2e-6 if case == "uniform" else 4e-6
    for v in range(count):
        assert np.all(np.isfinite(many[v]))
        assert oracle.rel_l2(many[v], singles[v]) < 1e-6
        ref = direct(oracle, 1, -1, pts, vecs[v], modes, "float32")
        assert oracle.rel_l2(many[v], ref) < bound


def test_many_outputs_ordered_on_the_plan_stream(cuda, engine, oracle):
    """The FFTs and deconvolutions of each pair run on the plan's internal stream; work that the
    caller enqueues on the plan's stream right after the call (no host synchronisation) must see
    every output."""
    torch = cuda
    rng = np.random.default_rng(77)
    M, modes, count = 400_000, [48, 40, 44], 7
    nm = int(np.prod(modes))
    pts = [rng.uniform(-np.pi, np.pi, M) for _ in range(3)]
    vecs = np.concatenate([rng.standard_normal(M) + 1j * rng.standard_normal(M)
                           for _ in range(count)]).astype(np.complex64)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        loc = [torch.from_numpy(p.astype(np.float32)).cuda() for p in pts]
        inp = torch.from_numpy(vecs).cuda()
        plan = engine.Plan(engine.Options(tol=1e-6, n_spread=8, tile=(4, 4, 1)), -1, M, loc,
                           modes, stream=s)
        out = torch.full((count * nm,), float("nan"), dtype=torch.complex64, device="cuda")
        plan.transform_type_1_many(inp, out, count, col_strides(modes))
        copy = out.clone()  # enqueued on s behind the call
        singles = torch.zeros((count, nm), dtype=torch.complex64, device="cuda")
        for v in range(count):
            plan.transform_type_1(inp[v * M:(v + 1) * M], singles[v], col_strides(modes))
    s.synchronize()
    plan.close()
    got = copy.cpu().numpy().reshape(count, nm)
    ref = singles.cpu().numpy()
    for v in range(count):
        assert np.all(np.isfinite(got[v]))
        assert oracle.rel_l2(got[v], ref[v]) < 1e-6


@pytest.mark.parametrize("dtype,dim", [("float64", 3), ("float32", 2), ("float64", 2)])
def test_many_falls_back_to_single_transforms(dtype, dim, cuda, engine, oracle):
    rng = np.random.default_rng(7 + dim)
    modes = [24, 20, 16][:dim]
    pts = [rng.uniform(-np.pi, np.pi, 3000) for _ in range(dim)]
    vecs = [rng.standard_normal(3000) + 1j * rng.standard_normal(3000) for _ in range(3)]
    tol = 1e-9 if dtype == "float64" else 1e-6
    many, singles, _ = _run(engine, cuda, dtype, pts, vecs, modes, tol=tol)
    bound = 1e-12 if dtype == "float64" else 1e-6
    for v in range(3):
        assert oracle.rel_l2(many[v], singles[v]) < bound


def test_many_rejects_bad_arguments(cuda, engine):
    torch = cuda
    loc = [torch.zeros(8, device="cuda") for _ in range(3)]
    plan = engine.Plan(engine.Options(tol=1e-6), -1, 8, loc, [8, 8, 8])
    buf = torch.zeros(8 * 4, dtype=torch.complex64, device="cuda")
    out = torch.zeros(512 * 4, dtype=torch.complex64, device="cuda")
    with pytest.raises(engine.InputError):
        plan.transform_type_1_many(buf, out, -1, [1, 8, 64])
    with pytest.raises(engine.InputError):  # outputs would overlap
        plan.transform_type_1_many(buf, out, 2, [1, 8, 64], out_bdist=100)
    plan.transform_type_1_many(buf, out, 0, [1, 8, 64])  # nothing to do
    plan.close()


def test_type3_odd_batch_on_two_vector_spreading(cuda, engine, oracle):
    """A single-precision type-3 plan with 3 inputs per batch: the z-window spreading takes
    inputs 0 and 1 in one pass and input 2 alone."""
    torch = cuda
    rng = np.random.default_rng(21)
    M, K, B = 900, 400, 3
    xin = [rng.uniform(-3, 5, M) for _ in range(3)]
    xout = [rng.uniform(-20, 12, K) for _ in range(3)]
    c = rng.standard_normal(M * B) + 1j * rng.standard_normal(M * B)
    a = [torch.from_numpy(p.astype(np.float32)).cuda() for p in xin]
    b = [torch.from_numpy(p.astype(np.float32)).cuda() for p in xout]
    plan = engine.PlanT3(engine.Options(tol=1e-5, spread_method=3), 1, M, a, K, b, batch_size=B)
    out = torch.zeros(K * B, dtype=torch.complex64, device="cuda")
    plan.add_input(torch.from_numpy(c.astype(np.complex64)).cuda(), M)
    plan.transform(out, K)
    torch.cuda.synchronize()
    res = out.cpu().numpy()
    plan.close()
    p_in = [p.astype(np.float32).astype(np.float64) for p in xin]
    p_out = [p.astype(np.float32).astype(np.float64) for p in xout]
    for k in range(B):
        ref = oracle.direct_type3(1, p_in, c[k * M:(k + 1) * M], p_out)
        assert oracle.rel_l2(res[k * K:(k + 1) * K], ref) < 5e-5
