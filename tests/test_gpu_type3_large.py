"""Single-precision type 3 at large space-bandwidth (sources in a box of half-width 50, targets
in half-width 200, the C3 extents; reference path src/neonufft/gpu/plan_t3_impl.hpp:216-252).

At these extents |x s| reaches 1e4, so any relative error delta in the target frequencies costs
about delta * |x s| of relative error. The reference computes the spread-grid spacing
h = T(2) T(pi) / T(nf1) in T; in single precision delta = h_float nf1 / (2 pi) - 1 is 1.4e-8 at
w = 7 (nf1 = 12740) and 2.5e-8 at w = 8, which alone gives 6.6e-5 / 1.1e-4 relative l2 in 2D,
above tol 1e-5, however accurately the spread, the FFT and the interpolation run. The engine
maps the targets with the exact spacing 2 pi / nf1 (in FP64, with the other type-3 rescaling and
phase steps), so its single-precision spread and FFT meet tol.

Each case checks (a) the amplification: FP64 direct sums at the targets scaled by 1 + delta
differ from the exact ones by more than tol, and (b) the engine's single-precision plan meets
tol against FP64 direct sums on sampled targets.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _float_h_delta(w, X, S, up=2.0):
    """delta of the T-precision spacing, from the reference's nf1 formula (util.hpp:64-105)."""
    pi_f = np.float32(math.pi)
    nf1 = int(2.0 * float(np.float32(up)) * float(np.float32(S)) * float(np.float32(X))
              / float(pi_f) + (w + 1))
    nf1 += nf1 % 2
    h_f = np.float32(2) * pi_f / np.float32(nf1)
    return float(h_f) / (2 * math.pi / nf1) - 1.0, nf1


@pytest.mark.parametrize("dim,M,w", [(1, 400_000, 7), (1, 400_000, 8), (2, 1_000_000, 7)])
def test_single_precision_type3_at_c3_extents(dim, M, w, cuda, engine):
    torch = cuda
    X, S, tol = 50.0, 200.0, 1e-5
    g = torch.Generator(device="cuda")
    g.manual_seed(40 + dim + w)
    xin = [((torch.rand(M, generator=g, device="cuda") * 2 - 1) * X) for _ in range(dim)]
    xout = [((torch.rand(M, generator=g, device="cuda") * 2 - 1) * S) for _ in range(dim)]
    c = torch.complex(torch.randn(M, generator=g, device="cuda"),
                      torch.randn(M, generator=g, device="cuda"))
    Ns = 1000
    tidx = torch.randint(0, M, (Ns,), generator=g, device="cuda")
    x64 = [a.double() for a in xin]
    s64 = [a.double() for a in xout]
    c128 = c.to(torch.complex128)
    exact = torch.empty(Ns, dtype=torch.complex128, device="cuda")
    engine.direct_type3_f64(-1, x64, c128, s64, tidx, exact)

    # (a) the amplification of a float spacing: targets scaled by 1 + delta
    delta, nf1 = _float_h_delta(w, X, S)
    assert abs(delta) > 5e-9
    scaled = torch.empty(Ns, dtype=torch.complex128, device="cuda")
    engine.direct_type3_f64(-1, x64, c128, [a * (1.0 + delta) for a in s64], tidx, scaled)
    amplified = float(torch.linalg.norm(scaled - exact) / torch.linalg.norm(exact))
    assert amplified > tol, amplified

    # (b) the engine: FP32 spread, FFT and interpolation, FP64 rescaling and phases
    plan = engine.PlanT3(engine.Options(tol=tol, n_spread=w), -1, M, xin, M, xout)
    info = plan.info()
    assert info["spread_grid"][0] == nf1
    out = torch.empty(M, dtype=torch.complex64, device="cuda")
    plan.add_input(c)
    plan.transform(out)
    got = out[tidx].to(torch.complex128)
    err = float(torch.linalg.norm(got - exact) / torch.linalg.norm(exact))
    plan.close()
    print(f"\n{dim}D type 3, X={X}, S={S}, w={w}, nf1={nf1}: float-h error {amplified:.2e}, "
          f"engine FP32 {err:.2e}")
    assert err <= tol, err
    assert err < amplified / 5
