"""The oracle, checked on the CPU before it is trusted as the checker:

* its FP64 direct sums reproduce the committed golden outputs (tests/golden/direct_small.npz,
  made on the reference tests' exact inputs) and agree with numpy definitions;
* its restated reference CPU plans (types 1, 2, 3) pass the reference's own acceptance rule on
  the reference tests' inputs (tests/test_type_1_2.cpp:191-198, tests/test_type_3.cpp:206-233);
* the input generator reproduces the reference's std::minstd_rand / uniform_real_distribution
  stream;
* the acceptance rule itself rejects a planted error (planted in the oracle's output, on the CPU).
"""
from pathlib import Path

import numpy as np
import pytest

import refcases

ROOT = Path(__file__).resolve().parent.parent
GOLD = np.load(ROOT / "tests" / "golden" / "direct_small.npz")


def test_generator_matches_libstdcxx_minstd():
    # minstd_rand: x_{n+1} = 48271 x_n mod (2^31 - 1), x_0 = 42. For double the libstdc++
    # generate_canonical draws two values: (u1 - 1 + (u2 - 1) R) / R^2, R = 2^31 - 2.
    m = 2**31 - 1
    x = 42
    us = []
    for _ in range(4):
        x = (48271 * x) % m
        us.append(x)
    R = float(2**31 - 2)
    v0 = ((us[0] - 1) + (us[1] - 1) * R) / (R * R)
    v1 = ((us[2] - 1) + (us[3] - 1) * R) / (R * R)
    (d,) = refcases.draw("float64", [(2, 20, 30, False)])
    assert np.allclose(d, [20 + 10 * v0, 20 + 10 * v1], rtol=0, atol=1e-13)


@pytest.mark.parametrize("key", sorted(GOLD.files))
def test_direct_sums_reproduce_golden(key, oracle):
    parts = key.split("_")
    if parts[0] == "t3":
        dtype, dim = parts[1], int(parts[2])
        xin, xout, inp = refcases.t3_inputs(dtype, dim, 50, 40)
        out = oracle.direct_type3(1, [a.astype(np.float64) for a in xin], inp.astype(np.complex128),
                                  [a.astype(np.float64) for a in xout])
    else:
        type_, dtype, modes = int(parts[0][1]), parts[1], [int(v) for v in parts[2].split("x")]
        pts, inp = refcases.t12_inputs(dtype, len(modes), 100, modes, type_)
        p64 = [p.astype(np.float64) for p in pts]
        if type_ == 1:
            out = oracle.direct_type1(-1, p64, inp.astype(np.complex128), modes).reshape(-1)
        else:
            out = oracle.direct_type2(-1, modes, inp.astype(np.complex128), p64)
    assert np.allclose(out, GOLD[key], rtol=1e-12, atol=1e-10)


def test_direct_sums_match_numpy_definition(oracle):
    rng = np.random.default_rng(0)
    M = 37
    x = [rng.uniform(-7, 7, M) for _ in range(2)]
    c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    modes = [6, 5]
    k0 = np.arange(6) - 3
    k1 = np.arange(5) - 2
    f = np.array([[np.sum(c * np.exp(-1j * (a * x[0] + b * x[1]))) for a in k0] for b in k1])
    assert np.allclose(oracle.direct_type1(-1, x, c, modes), f, atol=1e-11)
    g = oracle.direct_type2(1, modes, f, x)
    g_np = np.array([np.sum(f * np.exp(1j * (k0[None, :] * x[0][j] + k1[:, None] * x[1][j])))
                     for j in range(M)])
    assert np.allclose(g, g_np, atol=1e-10)
    s = [rng.uniform(-3, 3, 11) for _ in range(2)]
    t3 = oracle.direct_type3(-1, x, c, s)
    t3_np = np.array([np.sum(c * np.exp(-1j * (x[0] * s[0][k] + x[1] * s[1][k])))
                      for k in range(11)])
    assert np.allclose(t3, t3_np, atol=1e-11)


T12 = [c for c in refcases.t12_suites()
       if c[0] in ("Sign", "UpF", "UpD", "Tol") or (c[0] == "Modes" and max(c[3]) <= 23)]


@pytest.mark.parametrize("case", T12, ids=[refcases.case_id(c) for c in T12])
def test_restated_cpu_plan_passes_reference_rule(case, oracle):
    name, dtype, M, modes, up, tol, sign, type_ = case
    pts, inp = refcases.t12_inputs(dtype, len(modes), M, modes, type_)
    plan = oracle.RefPlan(dtype, sign, pts, modes, tol=tol, upsampfac=up, workers=2)
    p64 = [p.astype(np.float64) for p in pts]
    if type_ == 1:
        out = plan.transform_type_1(inp).reshape(-1)
        ref = oracle.direct_type1(sign, p64, inp.astype(np.complex128), modes).reshape(-1)
    else:
        out = plan.transform_type_2(inp)
        ref = oracle.direct_type2(sign, modes, inp.astype(np.complex128), p64)
    elem = 200000.0 if (type_ == 1 and dtype == "float32") else 400.0
    ok, mx, frac = oracle.reference_compare(ref, out, tol, elem, 0.85)
    assert ok, (mx, frac)


T3 = [c for c in refcases.t3_suites() if c[3] <= 200 and c[4] <= 200]


@pytest.mark.parametrize("case", T3[::3], ids=[refcases.case_id(c) for c in T3[::3]])
def test_restated_cpu_t3_passes_reference_rule(case, oracle):
    name, dtype, dim, n_in, n_out, up, tol, sign = case
    xin, xout, inp = refcases.t3_inputs(dtype, dim, n_in, n_out)
    plan = oracle.RefPlanT3(dtype, sign, xin, xout, tol=tol, upsampfac=up, workers=2)
    plan.add_input(inp)
    out = plan.transform()[0]
    ref = oracle.direct_type3(sign, [a.astype(np.float64) for a in xin], inp.astype(np.complex128),
                              [a.astype(np.float64) for a in xout])
    ok, mx, frac = oracle.reference_compare(ref, out, tol, 300.0, 0.94 if n_out > 20 else 0.85)
    assert ok, (mx, frac)


def test_acceptance_rule_rejects_planted_error(oracle):
    """Plant a wrong value into an oracle result (on the CPU) and check the rule catches it."""
    pts, inp = refcases.t12_inputs("float64", 1, 20, [45], 1)
    plan = oracle.RefPlan("float64", -1, pts, [45], tol=1e-8)
    out = plan.transform_type_1(inp).reshape(-1)
    ref = oracle.direct_type1(-1, pts, inp, [45]).reshape(-1)
    assert oracle.reference_compare(ref, out, 1e-8, 400, 0.85)[0]
    bad = out.copy()
    bad[7] *= 1.01  # squared relative error 1e-4 > 400 * tol
    assert not oracle.reference_compare(ref, bad, 1e-8, 400, 0.85)[0]
    assert oracle.rel_l2(bad, ref) > 10 * oracle.rel_l2(out, ref)


def test_mlp_oracle_gradient_matches_finite_differences():
    """The cost-model oracle's analytic gradient against central differences (float64)."""
    from oracle import mlp_oracle as MO
    rng = np.random.default_rng(3)
    widths = [5, 7, 6, 1]
    p = rng.standard_normal(MO.param_count(widths)) * 0.5
    x = rng.standard_normal((11, 5))
    t = rng.standard_normal(11)

    def loss(params):
        return MO.mse(MO.forward(widths, params, x)[-1], t)[0]

    acts = MO.forward(widths, p, x)
    _, dy = MO.mse(acts[-1], t)
    g = MO.backward(widths, p, x, acts, dy.reshape(-1, 1))
    h = 1e-6
    fd = np.array([(loss(p + h * e) - loss(p - h * e)) / (2 * h) for e in np.eye(p.size)])
    assert np.max(np.abs(fd - g)) < 1e-7 * max(1.0, np.max(np.abs(g)))
