"""Edge cases of the plans on the GPU, beyond the reference's test matrix.

- Non-finite coordinates: set_points raises InputError (the reference reads out of bounds on
  them) and the plan stays usable with a finite point set afterwards.
- Empty point sets: type 2 with M = 0 writes nothing; type 3 with no inputs gives zeros, with no
  targets writes nothing.
- One point, and one mode per dimension (N = 1: the k = 0 mode is the plain sum of strengths).
"""
import numpy as np
import pytest

from gpu_helpers import col_strides, tdtypes

pytestmark = pytest.mark.gpu

DTYPES = ["float32", "float64"]


def _tol(dtype):
    return 1e-5 if dtype == "float32" else 1e-10


def _bound(dtype):
    return 1e-4 if dtype == "float32" else 1e-8


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("bad", [float("nan"), float("inf"), -float("inf")])
@pytest.mark.parametrize("dim", [1, 3])
def test_non_finite_points_rejected(dtype, bad, dim, cuda, engine, oracle):
    torch = cuda
    rdt, cdt, npc = tdtypes(torch, dtype)
    rng = np.random.default_rng(3)
    M = 50
    pts = [rng.uniform(-np.pi, np.pi, M).astype(dtype) for _ in range(dim)]
    modes = [6] * dim
    good = [torch.from_numpy(p).cuda() for p in pts]
    bad_pts = [p.copy() for p in pts]
    bad_pts[dim - 1][17] = bad
    with pytest.raises(engine.InputError):
        engine.Plan(engine.Options(tol=_tol(dtype)), -1, M, [torch.from_numpy(p).cuda() for p in bad_pts],
                    modes)
    plan = engine.Plan(engine.Options(tol=_tol(dtype)), -1, M, good, modes)
    with pytest.raises(engine.InputError):
        plan.set_points(M, [torch.from_numpy(p).cuda() for p in bad_pts])
    # the plan takes a finite point set again and transforms it
    plan.set_points(M, good)
    c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    out = torch.zeros(int(np.prod(modes)), dtype=cdt, device="cuda")
    plan.transform_type_1(torch.from_numpy(c.astype(npc)).cuda(), out, col_strides(modes))
    torch.cuda.synchronize()
    ref = oracle.direct_type1(-1, [p.astype(np.float64) for p in pts], c, modes).reshape(-1)
    assert oracle.rel_l2(out.cpu().numpy(), ref) < _bound(dtype)
    plan.close()


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_type2_without_points_writes_nothing(dtype, dim, cuda, engine):
    torch = cuda
    rdt, cdt, npc = tdtypes(torch, dtype)
    modes = [8] * dim
    empty = [torch.empty(0, dtype=rdt, device="cuda") for _ in range(dim)]
    plan = engine.Plan(engine.Options(tol=_tol(dtype)), 1, 0, empty, modes)
    f = torch.ones(int(np.prod(modes)), dtype=cdt, device="cuda")
    sentinel = torch.full((4,), 5.0 + 0j, dtype=cdt, device="cuda")
    plan.transform_type_2(f, col_strides(modes), sentinel)
    torch.cuda.synchronize()
    assert torch.all(sentinel == 5.0).item()
    plan.close()


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("type_", [1, 2])
def test_single_point(dtype, dim, type_, cuda, engine, oracle):
    torch = cuda
    rdt, cdt, npc = tdtypes(torch, dtype)
    rng = np.random.default_rng(dim + 10 * type_)
    pts = [np.array([rng.uniform(-np.pi, np.pi)], dtype=dtype) for _ in range(dim)]
    modes = [int(m) for m in rng.integers(3, 12, dim)]
    loc = [torch.from_numpy(p).cuda() for p in pts]
    plan = engine.Plan(engine.Options(tol=_tol(dtype)), -1, 1, loc, modes)
    x64 = [p.astype(np.float64) for p in pts]
    if type_ == 1:
        c = np.array([0.7 - 1.3j])
        out = torch.zeros(int(np.prod(modes)), dtype=cdt, device="cuda")
        plan.transform_type_1(torch.from_numpy(c.astype(npc)).cuda(), out, col_strides(modes))
        ref = oracle.direct_type1(-1, x64, c, modes).reshape(-1)
    else:
        f = rng.standard_normal(int(np.prod(modes))) + 1j * rng.standard_normal(int(np.prod(modes)))
        out = torch.zeros(1, dtype=cdt, device="cuda")
        plan.transform_type_2(torch.from_numpy(f.astype(npc)).cuda(), col_strides(modes), out)
        ref = oracle.direct_type2(-1, modes, f, x64)
    torch.cuda.synchronize()
    assert oracle.rel_l2(out.cpu().numpy(), ref) < _bound(dtype)
    plan.close()


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_one_mode_is_the_sum(dtype, dim, cuda, engine):
    torch = cuda
    rdt, cdt, npc = tdtypes(torch, dtype)
    rng = np.random.default_rng(dim)
    M = 300
    pts = [rng.uniform(-np.pi, np.pi, M).astype(dtype) for _ in range(dim)]
    c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    modes = [1] * dim
    plan = engine.Plan(engine.Options(tol=_tol(dtype)), -1, M,
                       [torch.from_numpy(p).cuda() for p in pts], modes)
    out = torch.zeros(1, dtype=cdt, device="cuda")
    plan.transform_type_1(torch.from_numpy(c.astype(npc)).cuda(), out, [1] * dim)
    torch.cuda.synchronize()
    got = complex(out.cpu().numpy()[0])
    assert abs(got - c.sum()) / abs(c.sum()) < _bound(dtype)
    plan.close()


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_type3_empty_point_sets(dtype, dim, cuda, engine):
    torch = cuda
    rdt, cdt, npc = tdtypes(torch, dtype)
    rng = np.random.default_rng(5)
    K = 40
    empty = [torch.empty(0, dtype=rdt, device="cuda") for _ in range(dim)]
    targets = [torch.from_numpy(rng.uniform(-20, 20, K).astype(dtype)).cuda() for _ in range(dim)]
    # no input points: the transform of nothing is zero
    plan = engine.PlanT3(engine.Options(tol=_tol(dtype)), -1, 0, empty, K, targets)
    plan.add_input(torch.zeros(1, dtype=cdt, device="cuda"))
    out = torch.full((K,), 9.0 + 0j, dtype=cdt, device="cuda")
    plan.transform(out)
    torch.cuda.synchronize()
    assert torch.count_nonzero(out).item() == 0
    plan.close()
    # no targets: nothing is written
    M = 30
    sources = [torch.from_numpy(rng.uniform(-2, 2, M).astype(dtype)).cuda() for _ in range(dim)]
    plan = engine.PlanT3(engine.Options(tol=_tol(dtype)), -1, M, sources, 0, empty)
    c = torch.ones(M, dtype=cdt, device="cuda")
    plan.add_input(c)
    sentinel = torch.full((3,), 4.0 + 0j, dtype=cdt, device="cuda")
    plan.transform(sentinel)
    torch.cuda.synchronize()
    assert torch.all(sentinel == 4.0).item()
    plan.close()
