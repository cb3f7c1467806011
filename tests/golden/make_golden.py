"""Generates the committed golden fixtures of tests/golden/ from the reference's own code.

Run where the reference's sources are present (after `make -C oracle ref REF=<checkout>`):
    NEONUFFT_REFERENCE_DIR=<checkout> python tests/golden/make_golden.py

Writes
  pins.json  -- values computed by the reference's own host code compiled from its sources
                (oracle/_ref/libneonufft_ref.so): KernelParameters for a grid of
                (tol, upsampfac, precision), GridInfoT3 + set_nhg_type3 for a set of bounds,
                next235even for n = 0..3000, Gauss-Legendre rules (legendre_compute_glr) for
                n = 2..64.
  direct_small.npz -- FP64 direct NUDFT outputs (oracle) for small cases on the reference tests'
                exact inputs, pinning the oracle's direct sums against regressions.
"""
from __future__ import annotations

import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE.parent))

from oracle import oracle as O  # noqa: E402
import refcases  # noqa: E402

TOLS = [1e-1, 1e-2, 1e-3, 1e-4, 1e-5, 1e-6, 1e-7, 1e-8, 1e-9, 1e-10, 1e-12, 1e-14, 1e-15, 3e-6]
UPS = [1.25, 1.5, 1.6, 2.0, 2.5]
T3_BOUNDS = [
    (20, 30, 20, 30), (-20, 20, -20, 20), (-20, -15, -20, -15), (-50, 50, -200, 200),
    (-9, 9, -36, 36), (0, 0, 0, 0), (0, 0, -3, 3), (-np.pi, np.pi, -np.pi, np.pi),
    (1.0, 1.0, 5.0, 7.0), (-1e3, -999, 0.5, 0.75), (3.3, 9.1, -0.01, 40.0),
]


def main() -> None:
    ref = O.Ref()
    pins = {"kernel_params": [], "t3_geometry": [], "next235even": [], "legendre": []}
    for single in (True, False):
        for tol in TOLS:
            for up in UPS:
                w, beta, c = ref.kernel_param(tol, up, single)
                pins["kernel_params"].append(dict(single=single, tol=tol, upsampfac=up, w=w,
                                                  beta=beta, c=c))
    for single in (True, False):
        for (a, b, c, d) in T3_BOUNDS:
            for tol, up in ((1e-4, 2.0), (1e-7, 2.0), (1e-5, 1.25), (1e-12, 2.0)):
                w = ref.kernel_param(tol, up, single)[0]
                g = ref.t3_geometry(single, w, up, 0.1, a, b, c, d)
                pins["t3_geometry"].append(dict(single=single, tol=tol, upsampfac=up, w=w,
                                                bounds=[a, b, c, d], **g))
    pins["next235even"] = [ref.next235even(n) for n in range(0, 3001)]
    for n in range(2, 65):
        x, wt = ref.legendre(n)
        pins["legendre"].append(dict(n=n, x=x.tolist(), w=wt.tolist()))
    (HERE / "pins.json").write_text(json.dumps(pins))

    # Small FP64 direct sums on the reference tests' exact inputs.
    arrays = {}
    for dtype in ("float32", "float64"):
        for modes in ([23], [16, 9], [5, 4, 3]):
            for type_ in (1, 2):
                pts, inp = refcases.t12_inputs(dtype, len(modes), 100, modes, type_)
                p64 = [p.astype(np.float64) for p in pts]
                if type_ == 1:
                    out = O.direct_type1(-1, p64, inp.astype(np.complex128), modes).reshape(-1)
                else:
                    out = O.direct_type2(-1, modes, inp.astype(np.complex128), p64)
                key = f"t{type_}_{dtype}_{'x'.join(map(str, modes))}"
                arrays[key] = out
        for dim in (1, 2, 3):
            xin, xout, inp = refcases.t3_inputs(dtype, dim, 50, 40)
            out = O.direct_type3(1, [a.astype(np.float64) for a in xin], inp.astype(np.complex128),
                                 [a.astype(np.float64) for a in xout])
            arrays[f"t3_{dtype}_{dim}"] = out
    np.savez_compressed(HERE / "direct_small.npz", **arrays)
    print("wrote", HERE / "pins.json", HERE / "direct_small.npz")


if __name__ == "__main__":
    main()
