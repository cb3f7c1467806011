"""Parity of the engine's spreading / interpolation methods on the GPU.

Method 3 (z-window, the 3D default for kernel widths <= 8), method 1 (shared-memory slabs) and
method 2 (thread per point) must give the same transform: each is checked against the FP64
direct NUDFT (oracle) and against method 1 on the same inputs. Inputs cover every kernel width
2..8, grids whose size is not a multiple of the tile (partial last tiles), grids smaller than a
tile's halo region (several periodic wraps), points clustered into one tile (several batches
per plane), and the type-3 plan with a batch of inputs.
"""
import numpy as np
import pytest

from gpu_helpers import col_strides, tdtypes

pytestmark = pytest.mark.gpu


def run_t12(nnb, torch, dtype, sign, pts, inp, modes, type_, **opt):
    rdt, cdt, npc = tdtypes(torch, dtype)
    loc = [torch.from_numpy(np.ascontiguousarray(p, dtype=np.dtype(dtype))).cuda() for p in pts]
    plan = nnb.Plan(nnb.Options(tol=opt.pop("tol", 1e-6), **opt), sign, len(pts[0]), loc, modes)
    info = plan.info()
    x = torch.from_numpy(np.ascontiguousarray(inp, dtype=npc)).cuda()
    if type_ == 1:
        out = torch.zeros(int(np.prod(modes)), dtype=cdt, device="cuda")
        plan.transform_type_1(x, out, col_strides(modes))
    else:
        out = torch.zeros(len(pts[0]), dtype=cdt, device="cuda")
        plan.transform_type_2(x, col_strides(modes), out)
    torch.cuda.synchronize()
    res = out.cpu().numpy()
    plan.close()
    return res, info


def width_bound(dtype, w):
    # ES kernel of width w at upsampling 2 reaches about 10^(1 - w) (the reference heuristic
    # w = ceil(-log10(tol / 10))); single precision stops near 1e-6.
    b = 10.0 * 10.0 ** (1 - w)
    return max(b, 2e-5) if dtype == "float32" else max(b, 1e-12)


def direct(oracle, type_, sign, pts, inp, modes, dtype):
    # the points as the plan sees them (rounded to the plan precision)
    p64 = [p.astype(dtype).astype(np.float64) for p in pts]
    if type_ == 1:
        return oracle.direct_type1(sign, p64, inp, modes).reshape(-1)
    return oracle.direct_type2(sign, modes, inp, p64)


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("w", [2, 3, 4, 5, 6, 7, 8])
@pytest.mark.parametrize("type_", [1, 2])
def test_zwin_matches_slabs_and_direct(dtype, w, type_, cuda, engine, oracle):
    rng = np.random.default_rng(100 + w + 10 * type_)
    modes = [20, 17, 12]  # fine grid 40 x 34 x 24 (w <= 8): partial tiles in y
    M = 3000
    pts = [rng.uniform(-np.pi, np.pi, M) for _ in range(3)]
    n_in = M if type_ == 1 else int(np.prod(modes))
    inp = rng.standard_normal(n_in) + 1j * rng.standard_normal(n_in)
    sign = -1 if type_ == 1 else 1
    out3, info3 = run_t12(engine, cuda, dtype, sign, pts, inp, modes, type_, n_spread=w,
                          spread_method=3)
    out1, info1 = run_t12(engine, cuda, dtype, sign, pts, inp, modes, type_, n_spread=w,
                          spread_method=1)
    assert info3["spread_method"] == 3 and info1["spread_method"] == 1
    assert info3["n_spread"] == w
    ref = direct(oracle, type_, sign, pts, inp, modes, dtype)
    assert oracle.rel_l2(out3, ref) < width_bound(dtype, w)
    same = 2e-6 if dtype == "float32" else 1e-13
    assert oracle.rel_l2(out3, out1) < same


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("type_", [1, 2])
@pytest.mark.parametrize("method,tile", [(1, (0, 0, 0)), (2, (0, 0, 0)), (3, (0, 0, 0)),
                                         (3, (4, 16, 1)), (3, (4, 4, 1))])
def test_clustered_points(dtype, type_, method, tile, cuda, engine, oracle):
    """500 points inside one tile and plane (several batches of one plane) plus scattered ones."""
    if tile[1] in (4, 16) and dtype == "float64":
        pytest.skip("4- and 16-row tiles are single precision")
    rng = np.random.default_rng(7 + type_)
    modes = [24, 24, 24]
    M0, M1 = 500, 300
    pts = []
    for d in range(3):
        cl = 0.3 + rng.uniform(0, 0.01, M0)
        pts.append(np.concatenate([cl, rng.uniform(-np.pi, np.pi, M1)]))
    M = M0 + M1
    n_in = M if type_ == 1 else int(np.prod(modes))
    inp = rng.standard_normal(n_in) + 1j * rng.standard_normal(n_in)
    tol = 1e-5 if dtype == "float32" else 1e-7  # kernel widths 6 and 8
    out, info = run_t12(engine, cuda, dtype, 1, pts, inp, modes, type_, tol=tol,
                        spread_method=method, tile=tile)
    assert info["spread_method"] == method
    ref = direct(oracle, type_, 1, pts, inp, modes, dtype)
    bound = 3e-5 if dtype == "float32" else 1e-6
    assert oracle.rel_l2(out, ref) < bound


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("w", [2, 8])
@pytest.mark.parametrize("type_", [1, 2])
@pytest.mark.parametrize("tx,ty", [(2, 8), (4, 8), (8, 8), (4, 16), (4, 4)])
def test_zwin_tiny_grid(dtype, w, type_, tx, ty, cuda, engine, oracle):
    """Fine grids of 2w cells per dimension: the tile's halo region wraps around the grid."""
    if ty != 8 and dtype == "float64":
        pytest.skip("4- and 16-row tiles are single precision")
    rng = np.random.default_rng(3 * w + type_)
    modes = [3, 2, 4]
    M = 200
    pts = [rng.uniform(-4, 4, M) for _ in range(3)]
    n_in = M if type_ == 1 else int(np.prod(modes))
    inp = rng.standard_normal(n_in) + 1j * rng.standard_normal(n_in)
    out3, _ = run_t12(engine, cuda, dtype, -1, pts, inp, modes, type_, n_spread=w,
                      spread_method=3, tile=(tx, ty, 1))
    out1, _ = run_t12(engine, cuda, dtype, -1, pts, inp, modes, type_, n_spread=w,
                      spread_method=1)
    ref = direct(oracle, type_, -1, pts, inp, modes, dtype)
    assert oracle.rel_l2(out3, ref) < width_bound(dtype, w)
    assert oracle.rel_l2(out3, out1) < (2e-6 if dtype == "float32" else 1e-13)


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("tx,ty", [(2, 8), (4, 8), (8, 8), (2, 16), (4, 16), (8, 16), (4, 4)])
def test_zwin_tile_widths(dtype, tx, ty, cuda, engine, oracle):
    if ty != 8 and dtype == "float64":
        pytest.skip("4- and 16-row tiles are single precision")
    rng = np.random.default_rng(tx)
    modes = [33, 20, 18]
    M = 4000
    pts = [rng.uniform(-np.pi, np.pi, M) for _ in range(3)]
    c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    f = rng.standard_normal(int(np.prod(modes))) + 1j * rng.standard_normal(int(np.prod(modes)))
    tol = 1e-6 if dtype == "float32" else 1e-7
    o1, info = run_t12(engine, cuda, dtype, -1, pts, c, modes, 1, tol=tol, spread_method=3,
                       tile=(tx, ty, 1))
    o2, _ = run_t12(engine, cuda, dtype, 1, pts, f, modes, 2, tol=tol, spread_method=3,
                    tile=(tx, ty, 1))
    assert list(info["tile"]) == [tx, ty, 1]
    bound = 2e-5 if dtype == "float32" else 1e-6
    assert oracle.rel_l2(o1, direct(oracle, 1, -1, pts, c, modes, dtype)) < bound
    assert oracle.rel_l2(o2, direct(oracle, 2, 1, pts, f, modes, dtype)) < bound


def test_method3_rejected_outside_its_domain(cuda, engine):
    import torch
    loc2 = [torch.zeros(4, device="cuda") for _ in range(2)]
    with pytest.raises(engine.InputError):
        engine.Plan(engine.Options(tol=1e-6, spread_method=3), -1, 4, loc2, [8, 8])
    loc3 = [torch.zeros(4, device="cuda", dtype=torch.float64) for _ in range(3)]
    with pytest.raises(engine.InputError):
        engine.Plan(engine.Options(tol=1e-6, spread_method=3, n_spread=9), -1, 4, loc3,
                    [8, 8, 8])
    with pytest.raises(engine.InputError):
        engine.Plan(engine.Options(tol=1e-6, spread_method=3, tile=(16, 8, 1)), -1, 4, loc3,
                    [8, 8, 8])


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("method", [1, 3])
def test_type3_methods_batched(dtype, method, cuda, engine, oracle):
    import torch
    rng = np.random.default_rng(11 + method)
    M, K, B = 700, 500, 2
    xin = [rng.uniform(-3, 5, M) for _ in range(3)]
    xout = [rng.uniform(-20, 12, K) for _ in range(3)]
    c = rng.standard_normal(M * B) + 1j * rng.standard_normal(M * B)
    rdt, cdt, npc = tdtypes(torch, dtype)
    a = [torch.from_numpy(p.astype(dtype)).cuda() for p in xin]
    b = [torch.from_numpy(p.astype(dtype)).cuda() for p in xout]
    tol = 1e-5 if dtype == "float32" else 1e-7
    plan = engine.PlanT3(engine.Options(tol=tol, spread_method=method), 1, M, a, K, b,
                         batch_size=B)
    assert plan.info()["spread_method"] == method
    out = torch.zeros(K * B, dtype=cdt, device="cuda")
    plan.add_input(torch.from_numpy(c.astype(npc)).cuda(), M)
    plan.transform(out, K)
    torch.cuda.synchronize()
    res = out.cpu().numpy()
    plan.close()
    p_in = [p.astype(dtype).astype(np.float64) for p in xin]
    p_out = [p.astype(dtype).astype(np.float64) for p in xout]
    bound = 5e-5 if dtype == "float32" else 1e-6
    for k in range(B):
        ref = oracle.direct_type3(1, p_in, c[k * M:(k + 1) * M], p_out)
        assert oracle.rel_l2(res[k * K:(k + 1) * K], ref) < bound


@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("dim,method", [(2, 1), (2, 2), (3, 1), (3, 2), (3, 3)])
@pytest.mark.parametrize("type_", [1, 2])
def test_heavy_tile_split_over_ctas(dtype, dim, method, type_, cuda, engine, oracle):
    """12000 points inside one tile: the tile's points are split into several work items of at
    most 4096 points, each on its own CTA (partial grids added with atomics for spreading)."""
    rng = np.random.default_rng(17 + dim + type_)
    modes = [20, 18, 16][:dim]
    M0, M1 = 12000, 200
    pts = [np.concatenate([-1.0 + rng.uniform(0, 0.02, M0), rng.uniform(-np.pi, np.pi, M1)])
           for _ in range(dim)]
    M = M0 + M1
    n_in = M if type_ == 1 else int(np.prod(modes))
    inp = rng.standard_normal(n_in) + 1j * rng.standard_normal(n_in)
    tol = 1e-5 if dtype == "float32" else 1e-7
    out, info = run_t12(engine, cuda, dtype, -1, pts, inp, modes, type_, tol=tol,
                        spread_method=method)
    assert info["spread_method"] == method
    ref = direct(oracle, type_, -1, pts, inp, modes, dtype)
    # the bound of the reference matrix tests: max(10 tol, 2e-5) in single precision
    assert oracle.rel_l2(out, ref) < (1e-4 if dtype == "float32" else 1e-6)


@pytest.mark.parametrize("w", [5, 6, 7, 8])
@pytest.mark.parametrize("case", ["uniform", "tiny", "clustered"])
def test_tensor_core_spreading_matches_zwin_and_direct(w, case, cuda, engine, oracle):
    """Method 4 (z-window with TF32 tensor-core spreading, operands split into value and
    remainder) against method 3 and the FP64 direct sum, FP32 type 1."""
    rng = np.random.default_rng(60 + w)
    if case == "tiny":
        modes = [3, 2, 4]  # fine grid 2w: the region wraps around the grid
        pts = [rng.uniform(-4, 4, 300) for _ in range(3)]
    elif case == "clustered":  # one column chunk of ~9000 points: split over CTAs
        modes = [20, 18, 16]
        pts = [np.concatenate([0.5 + rng.uniform(0, 0.02, 9000), rng.uniform(-np.pi, np.pi, 300)])
               for _ in range(3)]
    else:
        modes = [20, 17, 12]
        pts = [rng.uniform(-np.pi, np.pi, 4000) for _ in range(3)]
    M = len(pts[0])
    c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    out4, info4 = run_t12(engine, cuda, "float32", -1, pts, c, modes, 1, n_spread=w,
                          spread_method=4)
    out3, _ = run_t12(engine, cuda, "float32", -1, pts, c, modes, 1, n_spread=w, spread_method=3)
    assert info4["spread_method"] == 4
    ref = direct(oracle, 1, -1, pts, c, modes, "float32")
    assert oracle.rel_l2(out4, ref) < width_bound("float32", w)
    assert oracle.rel_l2(out4, out3) < 2e-6


def test_tensor_core_spreading_type3_batched(cuda, engine, oracle):
    import torch
    rng = np.random.default_rng(70)
    M, K, B = 900, 400, 2
    xin = [rng.uniform(-3, 5, M).astype(np.float32) for _ in range(3)]
    xout = [rng.uniform(-20, 12, K).astype(np.float32) for _ in range(3)]
    c = rng.standard_normal(M * B) + 1j * rng.standard_normal(M * B)
    plan = engine.PlanT3(engine.Options(tol=1e-5, spread_method=4), 1, M,
                         [torch.from_numpy(p).cuda() for p in xin], K,
                         [torch.from_numpy(p).cuda() for p in xout], batch_size=B)
    out = torch.zeros(K * B, dtype=torch.complex64, device="cuda")
    plan.add_input(torch.from_numpy(c.astype(np.complex64)).cuda(), M)
    plan.transform(out, K)
    torch.cuda.synchronize()
    res = out.cpu().numpy()
    plan.close()
    for k in range(B):
        ref = oracle.direct_type3(1, [p.astype(np.float64) for p in xin], c[k * M:(k + 1) * M],
                                  [p.astype(np.float64) for p in xout])
        assert oracle.rel_l2(res[k * K:(k + 1) * K], ref) < 5e-5


def test_method4_rejected_outside_its_domain(cuda, engine):
    import torch
    loc3 = [torch.zeros(4, device="cuda") for _ in range(3)]
    with pytest.raises(engine.InputError):
        engine.Plan(engine.Options(tol=1e-3, spread_method=4), -1, 4, loc3, [8, 8, 8])  # w = 4
    loc64 = [torch.zeros(4, device="cuda", dtype=torch.float64) for _ in range(3)]
    with pytest.raises(engine.InputError):
        engine.Plan(engine.Options(tol=1e-6, spread_method=4), -1, 4, loc64, [8, 8, 8])
