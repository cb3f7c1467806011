"""Type-3 parity on the GPU: the reference's type-3 test matrix (tests/test_type_3.cpp:387-429)
with its exact inputs, its edge cases (:278-315) and its batched cases (:317-340), through the
engine's C ABI. Acceptance rule of the reference (test_type_3.cpp:206-233): every per-element
squared relative error < 300 tol, and more than 94 % (85 % for <= 20 outputs) <= tol."""
import numpy as np
import pytest

import refcases
from gpu_helpers import engine_t3, ref_gpu_or_none

pytestmark = pytest.mark.gpu

CASES = refcases.t3_suites()


def check(oracle, out, ref, tol, n_out):
    frac = 0.94 if n_out > 20 else 0.85
    ok, mx, fr = oracle.reference_compare(ref, out, tol, 300.0, frac)
    assert ok, f"reference acceptance failed: max e {mx:.3e}, fraction <= tol {fr:.3f}"


@pytest.mark.parametrize("case", CASES, ids=[refcases.case_id(c) for c in CASES])
def test_reference_matrix(case, cuda, engine, oracle):
    name, dtype, dim, n_in, n_out, up, tol, sign = case
    xin, xout, inp = refcases.t3_inputs(dtype, dim, n_in, n_out)
    out = engine_t3(engine, cuda, dtype, sign, xin, xout, inp, tol, up)
    ref = oracle.direct_type3(sign, [a.astype(np.float64) for a in xin], inp.astype(np.complex128),
                              [a.astype(np.float64) for a in xout])
    check(oracle, out, ref, tol, n_out)
    # FP64 phase and rescale steps: single-precision plans reach the float accuracy of the
    # spread/FFT path, not the (much larger) error of float phases at |x s| ~ 10^3.
    bound = max(20 * tol, 1e-12) if dtype == "float64" else max(20 * tol, 1e-4)
    assert oracle.rel_l2(out, ref) <= bound


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_edges(dim, cuda, engine, oracle):
    """Type3TestEdges (test_type_3.cpp:278-315): points at -pi, 0, pi, tol 1e-15, double."""
    vals = [-np.pi, np.pi] if dim == 1 else [-np.pi, 0.0, np.pi]
    grids = np.meshgrid(*([vals] * dim), indexing="ij")
    pts = [g.reshape(-1).astype(np.float64) for g in grids]
    (inp,) = refcases.draw("float64", [(len(pts[0]), -4, 4, True)])
    out = engine_t3(engine, cuda, "float64", -1, pts, pts, inp, 1e-15)
    ref = oracle.direct_type3(-1, pts, inp, pts)
    check(oracle, out, ref, 1e-15, len(pts[0]))


@pytest.mark.parametrize("dim,n_in", [(1, 200), (2, 80), (3, 80)])
def test_batched(dim, n_in, cuda, engine, oracle):
    """Type3TestBatched (test_type_3.cpp:317-357; the reference disables 3D): batch 3, double,
    tol 1e-6. Batches are compared at their own offsets."""
    n_out, batch = 55, 3
    xin, xout, inp = refcases.t3_inputs("float64", dim, n_in, n_out, batch=batch)
    out = engine_t3(engine, cuda, "float64", -1, xin, xout, inp, 1e-6, batch=batch)
    for b in range(batch):
        ref = oracle.direct_type3(-1, xin, inp[b * n_in:(b + 1) * n_in], xout)
        check(oracle, out[b * n_out:(b + 1) * n_out], ref, 1e-6, n_out)


def test_accumulate_and_reset(cuda, engine, oracle):
    """add_input accumulates until reset (reference plan_t3_impl.hpp:240-252)."""
    import torch
    rng = np.random.default_rng(11)
    M, K = 400, 300
    x = [rng.uniform(-5, 7, M) for _ in range(2)]
    s = [rng.uniform(-30, 10, K) for _ in range(2)]
    c1 = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    c2 = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    a = [torch.from_numpy(v).cuda() for v in x]
    b = [torch.from_numpy(v).cuda() for v in s]
    plan = engine.PlanT3(engine.Options(tol=1e-9), 1, M, a, K, b)
    out = torch.zeros(K, dtype=torch.complex128, device="cuda")
    plan.add_input(torch.from_numpy(c1).cuda())
    plan.add_input(torch.from_numpy(c2).cuda())
    plan.transform(out)
    torch.cuda.synchronize()
    ref = oracle.direct_type3(1, x, c1 + c2, s)
    assert oracle.rel_l2(out.cpu().numpy(), ref) < 1e-8
    plan.reset()
    plan.add_input(torch.from_numpy(c2).cuda())
    plan.transform(out)
    torch.cuda.synchronize()
    assert oracle.rel_l2(out.cpu().numpy(), oracle.direct_type3(1, x, c2, s)) < 1e-8


def test_bounds_constructor(cuda, engine, oracle):
    """PlanT3 from bounds, points set later (reference plan.hpp:63-66)."""
    import torch
    rng = np.random.default_rng(3)
    M, K = 500, 256
    x = [rng.uniform(-2, 3, M) for _ in range(3)]
    s = [rng.uniform(-8, 8, K) for _ in range(3)]
    c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    plan = engine.PlanT3.from_bounds(engine.Options(tol=1e-7), -1, [-2, -2, -2], [3, 3, 3],
                                     [-8, -8, -8], [8, 8, 8], dtype="float64")
    plan.set_input_points(M, [torch.from_numpy(v).cuda() for v in x])
    plan.set_output_points(K, [torch.from_numpy(v).cuda() for v in s])
    plan.add_input(torch.from_numpy(c).cuda())
    out = torch.zeros(K, dtype=torch.complex128, device="cuda")
    plan.transform(out)
    torch.cuda.synchronize()
    assert oracle.rel_l2(out.cpu().numpy(), oracle.direct_type3(-1, x, c, s)) < 1e-6


REF_CASES = [c for c in CASES if c[3] in (10, 200) and c[4] in (10, 200)]


@pytest.mark.parametrize("case", REF_CASES, ids=[refcases.case_id(c) for c in REF_CASES])
def test_against_reference_gpu_build(case, cuda, engine, oracle):
    rg = ref_gpu_or_none()
    if rg is None:
        pytest.skip("reference GPU build (oracle/_ref) not present")
    name, dtype, dim, n_in, n_out, up, tol, sign = case
    xin, xout, inp = refcases.t3_inputs(dtype, dim, n_in, n_out)
    out = engine_t3(engine, cuda, dtype, sign, xin, xout, inp, tol, up)
    ref_out = rg.t3(cuda, dtype, sign, xin, xout, inp, tol, up)
    exact = oracle.direct_type3(sign, [a.astype(np.float64) for a in xin], inp.astype(np.complex128),
                                [a.astype(np.float64) for a in xout])
    e_ref = oracle.rel_l2(ref_out, exact)
    e_eng = oracle.rel_l2(out, exact)
    assert oracle.rel_l2(out, ref_out) <= e_ref + e_eng + 1e-12
    assert e_eng <= 2.0 * e_ref + (1e-12 if dtype == "float64" else 1e-6)
