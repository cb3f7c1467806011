"""The reference's test matrix and inputs, restated for this engine's tests.

Parametrisations follow tests/test_type_1_2.cpp:339-392 and tests/test_type_3.cpp:387-429 of
the reference; inputs are drawn exactly as there (std::minstd_rand(42) +
std::uniform_real_distribution<T>) through tests/golden/libgen_inputs.so.
"""
from __future__ import annotations

import ctypes as C
import itertools
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE / "golden"))
import build_gen  # noqa: E402

_gen = None


def _lib():
    global _gen
    if _gen is None:
        _gen = C.CDLL(str(build_gen.build()))
        for suf in ("f32", "f64"):
            getattr(_gen, f"gen_segments_{suf}").argtypes = [
                C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return _gen


def draw(dtype, segments):
    """One minstd_rand(42) stream over segments [(n, a, b, is_complex)] -> list of arrays."""
    dt = np.float32 if np.dtype(dtype) == np.float32 else np.float64
    n = np.array([s[0] for s in segments], dtype=np.int64)
    a = np.array([s[1] for s in segments], dtype=np.float64)
    b = np.array([s[2] for s in segments], dtype=np.float64)
    cp = np.array([1 if s[3] else 0 for s in segments], dtype=np.int32)
    total = int(sum((2 if s[3] else 1) * s[0] for s in segments))
    out = np.zeros(max(1, total), dtype=dt)
    fn = getattr(_lib(), "gen_segments_f32" if dt == np.float32 else "gen_segments_f64")
    fn(len(segments), n.ctypes.data, a.ctypes.data, b.ctypes.data, cp.ctypes.data, out.ctypes.data)
    res, off = [], 0
    for s in segments:
        m = (2 if s[3] else 1) * s[0]
        v = out[off:off + m]
        off += m
        if s[3]:
            v = v[0::2] + 1j * v[1::2]
        res.append(v.copy())
    return res


def t12_inputs(dtype, dim, num_nu, modes, type_):
    """Points and input of PlanTest::test_random / test_transform (test_type_1_2.cpp:110-229)."""
    segs = [(num_nu, 20, 30, False)]
    if dim >= 2:
        segs.append((num_nu, -20, 20, False))
    if dim == 3:
        segs.append((num_nu, -20, -15, False))
    pts = draw(dtype, segs)
    n_in = int(np.prod(modes)) if type_ == 2 else num_nu
    (inp,) = draw(dtype, [(n_in, -4, 4, True)])
    return pts, inp


def t3_inputs(dtype, dim, num_in, num_out, batch=1):
    """Points and input of Type3Test::test_random / compare_t3 (test_type_3.cpp:76-265)."""
    segs = [(num_in, 20, 30, False), (num_out, 20, 30, False)]
    if dim >= 2:
        segs += [(num_in, -20, 20, False), (num_out, -20, 20, False)]
    if dim == 3:
        segs += [(num_in, -20, -15, False), (num_out, -20, -15, False)]
    v = draw(dtype, segs)
    xin = [v[0]] + ([v[2]] if dim >= 2 else []) + ([v[4]] if dim == 3 else [])
    xout = [v[1]] + ([v[3]] if dim >= 2 else []) + ([v[5]] if dim == 3 else [])
    (inp,) = draw(dtype, [(num_in * batch, -4, 4, True)])
    return xin, xout, inp


def generate_modes(sizes):
    """generate_modes of test_type_1_2.cpp:306-331 as lists of length dim."""
    out = [[s] for s in sizes]
    out += [[a, b] for a in sizes for b in sizes]
    out += [[a, b, c] for a in sizes for b in sizes for c in sizes]
    return out


def t12_suites():
    """(name, dtype, num_nu, modes, upsampfac, tol, sign, type) for every reference case."""
    cases = []
    for m in generate_modes([1, 2, 23, 256]):
        for t in (1, 2):
            cases.append(("Modes", "float32", 100, m, 2.0, 1e-4, -1, t))
    for m in generate_modes([16]):
        for s in (1, -1):
            for t in (1, 2):
                cases.append(("Sign", "float32", 10, m, 2.0, 1e-5, s, t))
    for m in generate_modes([16]):
        for up in (1.25, 1.6, 2.0):
            for t in (1, 2):
                cases.append(("UpF", "float32", 10, m, up, 1e-5, -1, t))
    for m in generate_modes([32]):
        for up in (1.25, 1.6, 2.0):
            for t in (1, 2):
                cases.append(("UpD", "float64", 10, m, up, 1e-5, -1, t))
    for m in generate_modes([45]):
        for tol in (1e-3, 1e-8, 1e-14):
            for t in (1, 2):
                cases.append(("Tol", "float64", 20, m, 2.0, tol, -1, t))
    return cases


def t3_suites():
    """(name, dtype, dim, num_in, num_out, upsampfac, tol, sign) of test_type_3.cpp:387-429."""
    cases = []
    for dt in ("float32", "float64"):
        for dim, n_in, n_out, tol, sign in itertools.product(
                (1, 2), (1, 10, 200, 503), (1, 10, 200, 503), (1e-4, 1e-7), (1, -1)):
            cases.append(("Type3", dt, dim, n_in, n_out, 2.0, tol, sign))
        for n_in, n_out, tol in itertools.product((1, 10, 99), (1, 10, 99), (1e-4, 1e-7)):
            cases.append(("Type3D3", dt, 3, n_in, n_out, 2.0, tol, 1))
    return cases


def case_id(c):
    return "-".join(str(v) if not isinstance(v, list) else "x".join(map(str, v)) for v in c)
