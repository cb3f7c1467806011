"""Binning of large point sets on the GPU.

The binning scatter writes each point's 32-byte record to a random slot (bin_start of its tile +
its rank); with 4.5e6 points the records (144 MB) outgrow the L2, so every record reaches the
memory on its own, as one whole sector (one 256-bit store); the sets of 2^24 + 4099 points hold
537 MB of records. The checks are the transforms' own: type 1 against FP64 direct sums on
sampled modes, type 2 against FP64 direct sums at sampled points, type 3 against FP64 direct
sums at sampled targets; for uniform and clustered points, in 1D, 2D and 3D, single and double
precision, with slab and z-window tiles. A non-finite coordinate in a large set is rejected and
leaves the plan usable.
"""
import numpy as np
import pytest

from gpu_helpers import col_strides, tdtypes

pytestmark = pytest.mark.gpu

LARGE = 4_500_001  # records larger than the L2 (126 MB)
HUGE = (1 << 24) + 4099  # 537 MB of records
MODES = {1: [2000], 2: [96, 80], 3: [40, 36, 32]}
SAMPLES = 256


def _tol(dtype):
    return (1e-5, 1e-4) if dtype == "float32" else (1e-10, 1e-8)


def _points(torch, rng, M, dim, dist):
    """Points in [-pi, pi)^dim as float64 tensors; `clustered`: 90 % in a small ball, so that
    a few tiles hold most of the records."""
    if dist == "uniform":
        pts = rng.uniform(-np.pi, np.pi, (dim, M))
    else:
        pts = rng.uniform(-np.pi, np.pi, (dim, M))
        k = int(0.9 * M)
        pts[:, :k] = np.mod(0.7 + 0.05 * rng.standard_normal((dim, k)) + np.pi,
                            2 * np.pi) - np.pi
    return [torch.from_numpy(p).cuda() for p in pts]


def _sample_modes(torch, rng, modes):
    flat = rng.integers(0, int(np.prod(modes)), SAMPLES)
    kk, rem = [], flat.copy()
    for n in modes:
        kk.append(rem % n - n // 2)
        rem //= n
    return (torch.from_numpy(flat).cuda(),
            torch.from_numpy(np.stack(kk, axis=1).astype(np.int64)).cuda())


def _rel(torch, got, ref):
    got = got.to(torch.complex128)
    return float(torch.linalg.norm(got - ref) / torch.linalg.norm(ref))


@pytest.mark.parametrize("M", [LARGE, HUGE])
@pytest.mark.parametrize("dist", ["uniform", "clustered"])
@pytest.mark.parametrize("dtype", ["float32", "float64"])
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_type1_type2_large_point_sets(dim, dtype, dist, M, cuda, engine):
    torch = cuda
    rdt, cdt, npc = tdtypes(torch, dtype)
    tol, bound = _tol(dtype)
    rng = np.random.default_rng(10 * dim + (dist == "clustered"))
    modes = MODES[dim]
    x64 = _points(torch, rng, M, dim, dist)
    x = [a.to(rdt) for a in x64]
    x64 = [a.double() for a in x]  # the plan's positions, exactly
    plan = engine.Plan(engine.Options(tol=tol), -1, M, x, modes)

    # type 1
    c64 = torch.complex(torch.from_numpy(rng.standard_normal(M)).cuda(),
                        torch.from_numpy(rng.standard_normal(M)).cuda())
    out = torch.empty(int(np.prod(modes)), dtype=cdt, device="cuda")
    plan.transform_type_1(c64.to(cdt), out, col_strides(modes))
    flat, kk = _sample_modes(torch, rng, modes)
    ref = torch.empty(SAMPLES, dtype=torch.complex128, device="cuda")
    engine.direct_type1_f64(-1, x64, c64.to(cdt).to(torch.complex128), kk, ref)
    torch.cuda.synchronize()
    assert _rel(torch, out[flat], ref) < bound

    # type 2 on the same sorted points
    nm = int(np.prod(modes))
    f64 = torch.complex(torch.from_numpy(rng.standard_normal(nm)).cuda(),
                        torch.from_numpy(rng.standard_normal(nm)).cuda()).to(cdt)
    vals = torch.empty(M, dtype=cdt, device="cuda")
    plan.transform_type_2(f64, col_strides(modes), vals)
    pidx = torch.from_numpy(rng.integers(0, M, SAMPLES).astype(np.int64)).cuda()
    ref2 = torch.empty(SAMPLES, dtype=torch.complex128, device="cuda")
    engine.direct_type2_f64(-1, modes, f64.to(torch.complex128), x64, pidx, ref2)
    torch.cuda.synchronize()
    assert _rel(torch, vals[pidx], ref2) < bound
    plan.close()


@pytest.mark.parametrize("method", [1, 3])
def test_spread_methods_large_set(method, cuda, engine):
    """Slab tiles (method 1, x-fastest tile order) and z-window tiles (method 3, plane-fastest
    tile order) on a large set."""
    torch = cuda
    M = LARGE
    rng = np.random.default_rng(7 + method)
    modes = [48, 40, 44]
    x = [a.float() for a in _points(torch, rng, M, 3, "uniform")]
    c = torch.complex(torch.from_numpy(rng.standard_normal(M)).cuda(),
                      torch.from_numpy(rng.standard_normal(M)).cuda()).to(torch.complex64)
    plan = engine.Plan(engine.Options(tol=1e-5, spread_method=method), -1, M, x, modes)
    out = torch.empty(int(np.prod(modes)), dtype=torch.complex64, device="cuda")
    plan.transform_type_1(c, out, col_strides(modes))
    flat, kk = _sample_modes(torch, rng, modes)
    ref = torch.empty(SAMPLES, dtype=torch.complex128, device="cuda")
    engine.direct_type1_f64(-1, [a.double() for a in x], c.to(torch.complex128), kk, ref)
    torch.cuda.synchronize()
    assert _rel(torch, out[flat], ref) < 1e-4
    plan.close()


@pytest.mark.parametrize("M", [LARGE, HUGE])
def test_type3_large_input_set(M, cuda, engine):
    torch = cuda
    K = 2000
    rng = np.random.default_rng(21)
    a = [torch.from_numpy(rng.uniform(-2.0, 3.0, M)).cuda().float() for _ in range(3)]
    b = [torch.from_numpy(rng.uniform(-9.0, 7.0, K)).cuda().float() for _ in range(3)]
    c = torch.complex(torch.from_numpy(rng.standard_normal(M)).cuda(),
                      torch.from_numpy(rng.standard_normal(M)).cuda()).to(torch.complex64)
    plan = engine.PlanT3(engine.Options(tol=1e-5), 1, M, a, K, b)
    plan.add_input(c)
    out = torch.empty(K, dtype=torch.complex64, device="cuda")
    plan.transform(out)
    tidx = torch.from_numpy(rng.integers(0, K, SAMPLES).astype(np.int64)).cuda()
    ref = torch.empty(SAMPLES, dtype=torch.complex128, device="cuda")
    engine.direct_type3_f64(1, [v.double() for v in a], c.to(torch.complex128),
                            [v.double() for v in b], tidx, ref)
    torch.cuda.synchronize()
    assert _rel(torch, out[tidx], ref) < 1e-4
    plan.close()


@pytest.mark.parametrize("M", [LARGE, HUGE])
@pytest.mark.parametrize("bad", [float("nan"), float("inf")])
def test_non_finite_point_in_large_set(bad, M, cuda, engine):
    torch = cuda
    rng = np.random.default_rng(5)
    modes = [32, 32, 32]
    x = [a.float() for a in _points(torch, rng, M, 3, "uniform")]
    plan = engine.Plan(engine.Options(tol=1e-5), -1, M, x, modes)
    bad_x = [a.clone() for a in x]
    bad_x[1][1234567] = bad
    with pytest.raises(engine.InputError):
        plan.set_points(M, bad_x)
    plan.set_points(M, x)
    c = torch.complex(torch.from_numpy(rng.standard_normal(M)).cuda(),
                      torch.from_numpy(rng.standard_normal(M)).cuda()).to(torch.complex64)
    out = torch.empty(32 ** 3, dtype=torch.complex64, device="cuda")
    plan.transform_type_1(c, out, col_strides(modes))
    flat, kk = _sample_modes(torch, rng, modes)
    ref = torch.empty(SAMPLES, dtype=torch.complex128, device="cuda")
    engine.direct_type1_f64(-1, [a.double() for a in x], c.to(torch.complex128), kk, ref)
    torch.cuda.synchronize()
    assert _rel(torch, out[flat], ref) < 1e-4
    plan.close()
