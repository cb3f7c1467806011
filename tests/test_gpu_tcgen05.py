"""Spreading on the tcgen05 tensor cores (spread method 5, csrc/spread_tc.cu) on the GPU.

The 3D single-precision spreading of method 5 keeps the column region's accumulator in tensor
memory and adds each group of 8 points as TF32 matrix products with split operands (value and
remainder). It must give the transform of method 3 (the z-window kernels, same 4 x 4 x 1 tiles)
and of the FP64 direct NUDFT (oracle) on the same inputs: every kernel width 2..8, grids smaller
than the region (periodic wraps), points clustered into one column (work items split over
CTAs), sparse columns whose points jump over many planes (the tensor-memory window moves by more
than its three blocks), type 2 (interpolation by method 3) and type 3 with a batch. Every run
ends with the device status check: no bounded wait in the kernel gave up.
"""
import numpy as np
import pytest

from test_gpu_methods import direct, run_t12, width_bound

pytestmark = pytest.mark.gpu


def _case(rng, case):
    if case == "tiny":
        modes = [3, 2, 4]  # fine grid 2w: the region wraps around the grid
        pts = [rng.uniform(-4, 4, 300) for _ in range(3)]
    elif case == "clustered":  # one column chunk of ~9000 points: split over CTAs
        modes = [20, 18, 16]
        pts = [np.concatenate([0.5 + rng.uniform(0, 0.02, 9000), rng.uniform(-np.pi, np.pi, 300)])
               for _ in range(3)]
    elif case == "sparse":  # few points per column, far apart in z
        modes = [24, 20, 64]
        pts = [rng.uniform(-np.pi, np.pi, 600) for _ in range(3)]
    else:
        modes = [20, 17, 12]
        pts = [rng.uniform(-np.pi, np.pi, 4000) for _ in range(3)]
    return modes, pts


@pytest.mark.parametrize("w", [2, 3, 4, 5, 6, 7, 8])
@pytest.mark.parametrize("case", ["uniform", "tiny", "clustered", "sparse"])
def test_tcgen05_spreading_matches_zwin_and_direct(w, case, cuda, engine, oracle):
    rng = np.random.default_rng(80 + w)
    modes, pts = _case(rng, case)
    M = len(pts[0])
    c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    out5, info5 = run_t12(engine, cuda, "float32", -1, pts, c, modes, 1, n_spread=w,
                          spread_method=5)
    engine.check_device_status()
    out3, _ = run_t12(engine, cuda, "float32", -1, pts, c, modes, 1, n_spread=w, spread_method=3,
                      tile=(4, 4, 1))
    assert info5["spread_method"] == 5 and list(info5["tile"]) == [4, 4, 1]
    ref = direct(oracle, 1, -1, pts, c, modes, "float32")
    assert oracle.rel_l2(out5, ref) < width_bound("float32", w)
    # Both methods add in single precision in a run-dependent order (float atomics; the tensor
    # core's partial sums): with ~9000 points on the same cells (clustered) the two sums differ
    # by about 2e-6 relative from run to run, elsewhere by a few 1e-7.
    assert oracle.rel_l2(out5, out3) < (4e-6 if case == "clustered" else 2e-6)


@pytest.mark.parametrize("sign", [-1, 1])
def test_tcgen05_plan_type2_and_type1_round_pair(sign, cuda, engine, oracle):
    """A method-5 plan runs type 2 through the z-window interpolation and type 1 on the tensor
    cores, both at the width-8 accuracy."""
    rng = np.random.default_rng(91)
    modes = [24, 20, 18]
    pts = [rng.uniform(-np.pi, np.pi, 5000) for _ in range(3)]
    nm = int(np.prod(modes))
    f = rng.standard_normal(nm) + 1j * rng.standard_normal(nm)
    c = rng.standard_normal(5000) + 1j * rng.standard_normal(5000)
    o2, info = run_t12(engine, cuda, "float32", sign, pts, f, modes, 2, n_spread=8,
                       spread_method=5)
    o1, _ = run_t12(engine, cuda, "float32", sign, pts, c, modes, 1, n_spread=8, spread_method=5)
    engine.check_device_status()
    assert info["spread_method"] == 5
    assert oracle.rel_l2(o2, direct(oracle, 2, sign, pts, f, modes, "float32")) < 2e-6
    assert oracle.rel_l2(o1, direct(oracle, 1, sign, pts, c, modes, "float32")) < 2e-6


def test_tcgen05_type3_batched(cuda, engine, oracle):
    import torch
    rng = np.random.default_rng(92)
    M, K, B = 900, 400, 2
    xin = [rng.uniform(-3, 5, M).astype(np.float32) for _ in range(3)]
    xout = [rng.uniform(-20, 12, K).astype(np.float32) for _ in range(3)]
    c = rng.standard_normal(M * B) + 1j * rng.standard_normal(M * B)
    plan = engine.PlanT3(engine.Options(tol=1e-5, spread_method=5), 1, M,
                         [torch.from_numpy(p).cuda() for p in xin], K,
                         [torch.from_numpy(p).cuda() for p in xout], batch_size=B)
    assert plan.info()["spread_method"] == 5
    out = torch.zeros(K * B, dtype=torch.complex64, device="cuda")
    plan.add_input(torch.from_numpy(c.astype(np.complex64)).cuda(), M)
    plan.transform(out, K)
    torch.cuda.synchronize()
    engine.check_device_status()
    res = out.cpu().numpy()
    plan.close()
    for k in range(B):
        ref = oracle.direct_type3(1, [p.astype(np.float64) for p in xin], c[k * M:(k + 1) * M],
                                  [p.astype(np.float64) for p in xout])
        assert oracle.rel_l2(res[k * K:(k + 1) * K], ref) < 5e-5


def test_tcgen05_large_uniform_set(cuda, engine):
    """2e6 uniform points on a 128^3 fine grid (about one point per cell, as at the north-star
    density): against method 3 on the same points."""
    import math
    import torch
    g = torch.Generator(device="cuda")
    g.manual_seed(93)
    M, N = 2_000_000, 64
    loc = [(torch.rand(M, generator=g, device="cuda") * 2 - 1) * math.pi for _ in range(3)]
    c = torch.complex(torch.randn(M, generator=g, device="cuda"),
                      torch.randn(M, generator=g, device="cuda"))
    outs = {}
    for method, tile in ((5, (4, 4, 1)), (3, (4, 4, 1))):
        plan = engine.Plan(engine.Options(tol=1e-6, n_spread=8, spread_method=method, tile=tile),
                           -1, M, loc, [N] * 3)
        out = torch.empty(N ** 3, dtype=torch.complex64, device="cuda")
        plan.transform_type_1(c, out, [1, N, N * N])
        torch.cuda.synchronize()
        outs[method] = out
        plan.close()
    engine.check_device_status()
    d = float(torch.linalg.norm(outs[5] - outs[3]) / torch.linalg.norm(outs[3]))
    assert d < 2e-6, d


def test_method5_rejected_outside_its_domain(cuda, engine):
    import torch
    loc2 = [torch.zeros(4, device="cuda") for _ in range(2)]
    with pytest.raises(engine.InputError):
        engine.Plan(engine.Options(tol=1e-6, spread_method=5), -1, 4, loc2, [8, 8])
    loc3 = [torch.zeros(4, device="cuda") for _ in range(3)]
    with pytest.raises(engine.InputError):
        engine.Plan(engine.Options(tol=1e-6, spread_method=5, n_spread=9), -1, 4, loc3, [8, 8, 8])
    with pytest.raises(engine.InputError):
        engine.Plan(engine.Options(tol=1e-6, spread_method=5, tile=(8, 8, 1)), -1, 4, loc3,
                    [8, 8, 8])
    loc64 = [torch.zeros(4, device="cuda", dtype=torch.float64) for _ in range(3)]
    with pytest.raises(engine.InputError):
        engine.Plan(engine.Options(tol=1e-6, spread_method=5), -1, 4, loc64, [8, 8, 8])
