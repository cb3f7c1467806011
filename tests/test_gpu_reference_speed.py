"""Speed and accuracy against the reference's own GPU plan on the same B200.

oracle/_ref/libneonufft_ref.so is the reference's GPU path (src/neonufft/gpu/**) compiled from its
own sources for sm_100a; its plans run here on device pointers through oracle/ref_shim.cu. One
step is set_points + transform_type_1 (3D, uniform points in [-pi, pi)^3, tol 1e-6), timed with
CUDA events on the legacy default stream, where both libraries launch:
  - reference FP64 and FP32 plans (its heuristic width for tol 1e-6, upsampfac 2);
  - the engine's plain FP64 plan (the same heuristic) and its tuned FP32 plan (w = 8).
Accuracy: relative l2 against FP64 direct sums on 512 sampled modes.

Sizes: NNB_SPEED_M points (default 2e6) and NNB_SPEED_N modes per dimension (default 64), so
that the 3D type-1 case M = 1e8, N = 256^3 runs with NNB_SPEED_M=100000000 NNB_SPEED_N=256.
"""
import ctypes as C
import math
import os

import pytest

from gpu_helpers import ref_gpu_or_none

M = int(float(os.environ.get("NNB_SPEED_M", "2e6")))
N = int(os.environ.get("NNB_SPEED_N", "64"))
TOL = 1e-6


def _events(torch, fn, warmup=1, reps=3):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return sorted(times)[len(times) // 2]


@pytest.mark.gpu
def test_engine_against_reference_gpu_plan(cuda, engine):
    torch = cuda
    rg = ref_gpu_or_none()
    if rg is None:
        pytest.skip("reference GPU build (oracle/_ref) not present")
    L = rg.ref.L
    assert torch.cuda.current_stream().cuda_stream == 0  # the legacy default stream
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    # single-precision points, so that every plan and the direct sums see the same positions
    x64 = [((torch.rand(M, generator=g, device="cuda", dtype=torch.float64) * 2 - 1) * math.pi)
           .float().double() for _ in range(3)]
    c64 = torch.complex(torch.randn(M, generator=g, device="cuda", dtype=torch.float64),
                        torch.randn(M, generator=g, device="cuda", dtype=torch.float64))
    modes = [N, N, N]
    strides = [1, N, N * N]
    S = 512
    idx = torch.randint(0, N ** 3, (S,), generator=g, device="cuda")
    kk, rem = [], idx.clone()
    for _ in range(3):
        kk.append(rem % N - N // 2)
        rem = rem // N
    ref = torch.empty(S, dtype=torch.complex128, device="cuda")
    engine.direct_type1_f64(-1, x64, c64, torch.stack(kk, dim=1).contiguous(), ref)

    def err(out):
        got = out[idx].to(torch.complex128)
        return float(torch.linalg.norm(got - ref) / torch.linalg.norm(ref))

    results = {}
    for prec in ("f64", "f32"):
        rdt = torch.float64 if prec == "f64" else torch.float32
        cdt = torch.complex128 if prec == "f64" else torch.complex64
        x = [a.to(rdt) for a in x64]
        c = c64.to(cdt)
        out = torch.empty(N ** 3, dtype=cdt, device="cuda")
        lp = (C.c_void_p * 3)(*[a.data_ptr() for a in x])
        md = (C.c_int64 * 3)(*modes)
        st = (C.c_int64 * 3)(*strides)

        # reference plan (its heuristic width)
        h = C.c_void_p()
        assert L.ref_plan12_create(C.byref(h), int(prec == "f32"), 3, TOL, 2.0, -1, M, lp, md) == 0

        def ref_step():
            assert L.ref_plan12_set_points(h, M, lp) == 0
            assert L.ref_plan12_t1(h, c.data_ptr(), out.data_ptr(), st) == 0

        ms = _events(torch, ref_step)
        results[f"reference {prec}"] = (ms, err(out))
        L.ref_plan12_destroy(h)
        torch.cuda.synchronize()

        # engine plan: plain heuristic for FP64, tuned width w = 8 for FP32
        opt = engine.Options(tol=TOL, n_spread=8 if prec == "f32" else 0)
        plan = engine.Plan(opt, -1, M, x, modes)

        def eng_step():
            plan.set_points(M, x)
            plan.transform_type_1(c, out, strides)

        ms = _events(torch, eng_step)
        results[f"engine {prec}"] = (ms, err(out))
        plan.close()
        del x, c, out
        torch.cuda.empty_cache()

    line = ", ".join(f"{k}: {v[0]:.2f} ms ({M / (v[0] * 1e-3):.3g} pts/s, rel-l2 {v[1]:.2e})"
                     for k, v in results.items())
    print(f"\n3D type 1, M={M}, N={N}^3, tol {TOL}: {line}")
    # the tuned FP32 engine meets the target accuracy and beats both reference plans
    assert results["engine f32"][1] <= 1e-6
    assert results["engine f32"][0] < results["reference f64"][0]
    assert results["engine f32"][0] < results["reference f32"][0]
    # the engine's FP64 plan is at least as accurate as the reference's FP64 plan (same width)
    assert results["engine f64"][1] <= 1.5 * results["reference f64"][1] + 1e-12


@pytest.mark.gpu
def test_engine_type2_against_reference_gpu_plan(cuda, engine):
    """Type 2 on the reference's interpolation path (src/neonufft/gpu/kernels/
    interpolation_kernel.cu:84-319): 3D, M = 2e6 points, N = 64^3 modes, tol 1e-6. Both
    libraries' FP64 plans and the engine's tuned FP32 plan against FP64 direct sums on 512
    sampled points; the two FP64 plans also against each other."""
    torch = cuda
    rg = ref_gpu_or_none()
    if rg is None:
        pytest.skip("reference GPU build (oracle/_ref) not present")
    L = rg.ref.L
    assert torch.cuda.current_stream().cuda_stream == 0
    M2, N2 = 2_000_000, 64
    g = torch.Generator(device="cuda")
    g.manual_seed(12)
    x64 = [((torch.rand(M2, generator=g, device="cuda", dtype=torch.float64) * 2 - 1) * math.pi)
           .float().double() for _ in range(3)]
    nm = N2 ** 3
    f64 = torch.complex(torch.randn(nm, generator=g, device="cuda", dtype=torch.float64),
                        torch.randn(nm, generator=g, device="cuda", dtype=torch.float64))
    modes = [N2] * 3
    strides = [1, N2, N2 * N2]
    S = 512
    pidx = torch.randint(0, M2, (S,), generator=g, device="cuda")
    ref = torch.empty(S, dtype=torch.complex128, device="cuda")
    engine.direct_type2_f64(-1, modes, f64, x64, pidx, ref)

    def err(out):
        got = out[pidx].to(torch.complex128)
        return float(torch.linalg.norm(got - ref) / torch.linalg.norm(ref))

    results, outs = {}, {}
    for prec in ("f64", "f32"):
        rdt = torch.float64 if prec == "f64" else torch.float32
        cdt = torch.complex128 if prec == "f64" else torch.complex64
        x = [a.to(rdt) for a in x64]
        f = f64.to(cdt)
        lp = (C.c_void_p * 3)(*[a.data_ptr() for a in x])
        md = (C.c_int64 * 3)(*modes)
        st = (C.c_int64 * 3)(*strides)
        out = torch.empty(M2, dtype=cdt, device="cuda")
        h = C.c_void_p()
        assert L.ref_plan12_create(C.byref(h), int(prec == "f32"), 3, TOL, 2.0, -1, M2, lp,
                                   md) == 0

        def ref_step():
            assert L.ref_plan12_set_points(h, M2, lp) == 0
            assert L.ref_plan12_t2(h, f.data_ptr(), st, out.data_ptr()) == 0

        ms = _events(torch, ref_step)
        results[f"reference {prec}"] = (ms, err(out))
        outs[f"reference {prec}"] = out.clone()
        L.ref_plan12_destroy(h)
        torch.cuda.synchronize()

        opt = engine.Options(tol=TOL, n_spread=8 if prec == "f32" else 0)
        plan = engine.Plan(opt, -1, M2, x, modes)

        def eng_step():
            plan.set_points(M2, x)
            plan.transform_type_2(f, strides, out)

        ms = _events(torch, eng_step)
        results[f"engine {prec}"] = (ms, err(out))
        outs[f"engine {prec}"] = out.clone()
        plan.close()
        del x, f, out
        torch.cuda.empty_cache()

    line = ", ".join(f"{k}: {v[0]:.2f} ms (rel-l2 {v[1]:.2e})" for k, v in results.items())
    print(f"\n3D type 2, M={M2}, N={N2}^3, tol {TOL}: {line}")
    a, b = outs["engine f64"], outs["reference f64"]
    diff = float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
    # same heuristic width: the two FP64 plans agree to within their truncation error
    assert diff <= 2.0 * max(results["engine f64"][1], results["reference f64"][1])
    assert results["engine f64"][1] <= 1.5 * results["reference f64"][1] + 1e-12
    assert results["engine f32"][1] <= 1e-6
    assert results["engine f32"][0] < results["reference f64"][0]
