"""C-ABI checks that need no GPU: the library loads, exports every entry point declared in
include/neonufft_gpu.h, the host-only parameter functions agree with the reference's own code
(pinned in tests/golden/pins.json), and invalid arguments return the reference's error codes
before any device work."""
import ctypes as C
import json
import math
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
PINS = json.loads((ROOT / "tests" / "golden" / "pins.json").read_text())


def declared_symbols():
    text = (ROOT / "include" / "neonufft_gpu.h").read_text()
    return sorted(set(re.findall(r"NNB_API[^;(]*?\b(nnb_\w+)\s*\(", text, flags=re.S)))


def test_exports_every_declared_symbol(engine):
    from neonufft_b200 import _lib
    lib = _lib.load()
    names = declared_symbols()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), f"missing export {n}"
    bound = {s[0] for s in _lib.SIGNATURES}
    assert set(names) == bound, f"binding mismatch: {set(names) ^ bound}"


def test_version_and_defaults(engine):
    from neonufft_b200 import _lib
    lib = _lib.load()
    assert b"sm_100a" in lib.nnb_version()
    o = _lib.NnbOptions()
    lib.nnb_options_default(C.byref(o))
    # reference defaults (include/neonufft/plan.hpp:19-29)
    assert (o.tol, o.upsampfac, o.recenter_threshold, o.order) == (0.001, 2.0, 0.1, 1)


@pytest.mark.parametrize("entry", PINS["kernel_params"], ids=lambda e: f"{e['single']}-{e['tol']}-{e['upsampfac']}")
def test_kernel_params_match_reference(entry, engine, oracle):
    from neonufft_b200 import _lib
    lib = _lib.load()
    w = C.c_int()
    beta = C.c_double()
    c = C.c_double()
    prec = _lib.NNB_FLOAT if entry["single"] else _lib.NNB_DOUBLE
    assert lib.nnb_es_kernel_params(entry["tol"], entry["upsampfac"], prec, C.byref(w),
                                    C.byref(beta), C.byref(c)) == 0
    assert w.value == entry["w"]
    assert beta.value == entry["beta"]  # bit-exact: same formula, same rounding to T
    assert c.value == entry["c"]
    # the oracle's restatement agrees too
    ow, ob, oc = oracle.kernel_params(entry["tol"], entry["upsampfac"], entry["single"])
    assert (ow, ob, oc) == (entry["w"], entry["beta"], entry["c"])


@pytest.mark.parametrize("entry", PINS["t3_geometry"], ids=lambda e: f"{e['single']}-{e['bounds']}-{e['tol']}-{e['upsampfac']}")
def test_t3_geometry_matches_reference(entry, engine, oracle):
    from neonufft_b200 import _lib
    lib = _lib.load()
    from neonufft_b200.plan import Options
    o = Options(tol=entry["tol"], upsampfac=entry["upsampfac"]).to_c()
    a, b, c, d = entry["bounds"]
    nf1 = (C.c_int64 * 1)()
    nfft = (C.c_int64 * 1)()
    vals = [(C.c_double * 1)() for _ in range(4)]
    prec = _lib.NNB_FLOAT if entry["single"] else _lib.NNB_DOUBLE
    rc = lib.nnb_plan_t3_geometry(prec, 1, C.byref(o), _lib.f64_array([a]), _lib.f64_array([b]),
                                  _lib.f64_array([c]), _lib.f64_array([d]), nf1, nfft, *vals)
    assert rc == 0
    assert (nf1[0], nfft[0]) == (entry["nf1"], entry["nfft"])
    assert vals[0][0] == entry["C"] and vals[1][0] == entry["D"]
    assert vals[2][0] == entry["gamma"] and vals[3][0] == entry["h"]
    dt = np.float32 if entry["single"] else np.float64
    g = oracle.t3_geometry(entry["w"], entry["upsampfac"], 0.1, a, b, c, d, dt)
    assert (g["nf1"], g["nfft"]) == (entry["nf1"], entry["nfft"])
    assert float(g["gamma"]) == entry["gamma"] and float(g["h"]) == entry["h"]
    # grid_memory_size follows the reference GPU accounting (plan_t3_impl.hpp:69-71)
    size = C.c_uint64()
    assert lib.nnb_plan_t3_grid_memory_size(prec, 1, C.byref(o), _lib.f64_array([a]),
                                            _lib.f64_array([b]), _lib.f64_array([c]),
                                            _lib.f64_array([d]), C.byref(size)) == 0
    cb = 8 if entry["single"] else 16
    assert size.value == cb * (entry["nf1"] + 2 * entry["nfft"])


def test_next235even_matches_reference(oracle):
    ref = PINS["next235even"]
    assert [oracle.next235even(n) for n in range(len(ref))] == ref


def test_deconv_factors(engine, oracle):
    """Host FP64 deconvolution factors (engine) vs the restated reference fseries (oracle, FP64)
    and vs a brute-force integral of the ES kernel's Fourier transform."""
    from neonufft_b200 import _lib
    lib = _lib.load()
    for tol, up, nf in ((1e-6, 2.0, 512), (1e-4, 1.25, 80), (1e-12, 2.0, 90), (1e-3, 2.0, 14)):
        out = np.zeros(nf // 2 + 1)
        assert lib.nnb_deconv_factors(tol, up, _lib.NNB_DOUBLE, nf,
                                      out.ctypes.data_as(C.POINTER(C.c_double))) == 0
        w, beta, c = oracle.kernel_params(tol, up, False)
        ref = oracle.fseries_inverse(w, beta, c, nf, np.float64)
        assert np.allclose(out, ref, rtol=1e-12, atol=0)
        # independent quadrature: phi_hat(xi) = int phi(z) cos(xi z) dz after z = (w/2) sin(t),
        # which removes the square-root endpoint of the kernel (smooth integrand in t)
        u, wu = np.polynomial.legendre.leggauss(64)
        t = (u + 1) * np.pi / 4
        z = (w / 2) * np.sin(t)
        jac = wu * (np.pi / 4) * (w / 2) * np.cos(t)
        phi = oracle.es_kernel(z, beta, c, np.float64)
        k = np.array([0, 1, nf // 4, nf // 2])
        ph = np.array([2 * np.sum(jac * phi * np.cos(2 * math.pi * kk / nf * z)) for kk in k])
        # The q = w + w%2 + 10 node rule in z (the reference CPU path's count) is limited by that
        # endpoint (a step of exp(-beta) at |z| = w/2): a few 1e-7 relative at upsampfac 1.25.
        assert np.allclose(np.abs(1 / out[k]), ph, rtol=5e-7)
        assert np.all(np.sign(out[k]) == np.where(k % 2 == 1, -1, 1))


def test_legendre_pins(oracle):
    """The reference's Gauss-Legendre nodes (legendre_compute_glr) vs numpy's; the engine's own
    rule is checked through the deconvolution factors above."""
    for e in PINS["legendre"]:
        x, w = np.polynomial.legendre.leggauss(e["n"])
        assert np.allclose(np.sort(e["x"]), x, atol=2e-15)
        assert np.allclose(np.asarray(e["w"])[np.argsort(e["x"])], w, atol=2e-14)


@pytest.mark.parametrize("kw,code_name", [
    (dict(dim=4), "INPUT_ERROR"), (dict(dim=0), "INPUT_ERROR"), (dict(precision=7), "INPUT_ERROR"),
    (dict(tol=-1.0), "INPUT_ERROR"), (dict(tol=float("nan")), "INPUT_ERROR"),
    (dict(upsampfac=1.0), "INPUT_ERROR"), (dict(order=5), "INPUT_ERROR"),
])
def test_invalid_arguments_fail_before_device_work(kw, code_name, engine):
    from neonufft_b200 import _lib
    lib = _lib.load()
    o = _lib.NnbOptions()
    lib.nnb_options_default(C.byref(o))
    for k in ("tol", "upsampfac", "order"):
        if k in kw:
            setattr(o, k, kw[k])
    h = C.c_void_p()
    rc = lib.nnb_plan_create(C.byref(h), kw.get("precision", 0), kw.get("dim", 1), C.byref(o), -1,
                             0, None, _lib.i64_array([8]), None, None)
    assert rc == getattr(_lib, code_name)
    assert not h.value
    assert lib.nnb_last_error_message()


def test_t3_invalid_bounds(engine):
    from neonufft_b200 import _lib
    lib = _lib.load()
    size = C.c_uint64()
    assert lib.nnb_plan_t3_grid_memory_size(0, 1, None, None, None, None, None,
                                            C.byref(size)) == _lib.INPUT_ERROR


def test_noalloc_rejects_requests_beyond_its_scratch():
    """The allocation-free direct sum rejects sizes beyond its fixed scratch before any device
    work. Run in a child process that sees no GPU (CUDA_VISIBLE_DEVICES empty), so that a
    regressed size check ends in a CUDA error there rather than in a launch over these
    placeholder buffers."""
    import os
    import subprocess
    import sys
    code = r'''
import ctypes as C
from neonufft_b200 import _lib as L
lib = L.load()
M, S = 4096 * 20000, 60  # 60 samples x 20000 chunks > 2^20 partial sums
buf = (C.c_double * 256)()
ptrs = L.ptr_array([C.addressof(buf)])
kidx = (C.c_int64 * (S + 1))()
rc = lib.nnb_direct_type1_f64_noalloc(1, -1, M, ptrs, C.addressof(buf), S, C.addressof(kidx),
                                      C.addressof(buf), None)
msg = lib.nnb_last_error_message()
assert rc == L.INPUT_ERROR, (rc, msg)
assert b"scratch" in msg, msg
# the largest request that fits is accepted by the size check (it then needs a device)
M = 4096 * (1048576 // S)
rc = lib.nnb_direct_type1_f64_noalloc(1, -1, M, ptrs, C.addressof(buf), S, C.addressof(kidx),
                                      C.addressof(buf), None)
assert rc != L.INPUT_ERROR or b"scratch" not in lib.nnb_last_error_message()
print("ok")
'''
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    res = subprocess.run([sys.executable, "-c", code], cwd=str(ROOT), env=env,
                         capture_output=True, text=True, timeout=120)
    assert res.returncode == 0 and "ok" in res.stdout, res.stdout + res.stderr


def test_tuner_rows_round_trip_through_a_file(tmp_path):
    """The tuner's measured rows (problem, configuration, time, error) survive save / load with
    their features recomputed identically; a wrong format or version is refused."""
    from neonufft_b200 import tuner as T
    t = T.Tuner()
    probs = [T.Problem(dim=3, type=1, M=10 ** 6, N=64, tol=1e-6, seed=1),
             T.Problem(dim=2, type=2, M=20000, N=256, tol=1e-3, precision="f32", blob=True, seed=2),
             T.Problem(dim=3, type=2, M=5 * 10 ** 5, N=48, tol=1e-9, precision="f64", seed=3)]
    for i, p in enumerate(probs):
        for j, c in enumerate(T.candidates(p)[:4]):
            t.rows.append((T.features(p, c), 0.1 * i + 0.01 * j, 1e-7 * (j + 1), p, c))
    path = tmp_path / "tuner.json"
    t.save(path)
    u = T.Tuner.load(path, with_model=False)
    assert len(u.rows) == len(t.rows)
    for a, b in zip(t.rows, u.rows):
        assert np.array_equal(a[0], b[0]) and a[1:] == b[1:]
    assert u.autotune(probs[0]) == t.autotune(probs[0])
    doc = json.loads(path.read_text())
    doc["version"] = 99
    bad = tmp_path / "bad.json"
    bad.write_text(json.dumps(doc))
    with pytest.raises(ValueError):
        T.Tuner.load(bad)
