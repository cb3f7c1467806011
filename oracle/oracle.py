"""ORACLE -- test infrastructure only.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg (and its ``--impl reference``
arm) may import this module, and only as the checker. The engine never calls it.

Contents
--------
* FP64 direct NUDFT sums (C++/OpenMP, libnufft_oracle.so): the definition of the transforms,
  restated from the reference's test oracle (tests/nuft_direct_kernels.cpp:73-293).
* ``RefPlan`` / ``RefPlanT3``: a CPU restatement of the reference's CPU plans
  (src/neonufft/plan_impl.hpp:37-134, src/neonufft/plan_t3_impl.hpp:66-380) in precision T:
  parameter heuristics, rescaling, padded spreading + fold, FFT, deconvolution, interpolation,
  type-3 pre/post phase. Heavy loops run in libnufft_oracle.so; the FFT is scipy's (the
  reference uses FFTW, absent here), with every host thread.
* ``Ref`` -- thin ctypes wrapper of oracle/_ref/libneonufft_ref.so when it has been built: the
  reference's own parameter code and its own GPU plans compiled from its sources.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from pathlib import Path

import numpy as np

try:
    import scipy.fft as _sfft
except Exception:  # pragma: no cover
    _sfft = None

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libnufft_oracle.so"
REF_LIB_PATH = HERE / "_ref" / "libneonufft_ref.so"

_lib = None


def build() -> None:
    """Builds libnufft_oracle.so, and the reference pin library when NEONUFFT_REFERENCE_DIR names
    a NeoNUFFT source checkout."""
    import os
    import subprocess
    subprocess.run(["make", "-C", str(HERE), "all"], check=True, capture_output=True)
    ref = os.environ.get("NEONUFFT_REFERENCE_DIR", "")
    if ref and Path(ref).is_dir():
        subprocess.run(["make", "-C", str(HERE), "ref", f"REF={ref}", "-j8"], check=True,
                       capture_output=True)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = C.CDLL(str(LIB_PATH))
        i64 = C.c_int64
        dp = C.POINTER(C.c_double)
        for name in ("oracle_direct_type1",):
            getattr(_lib, name).argtypes = [C.c_int, C.c_int, i64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.oracle_direct_type2.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, i64, C.c_void_p, C.c_void_p]
        _lib.oracle_direct_type3.argtypes = [C.c_int, C.c_int, i64, C.c_void_p, C.c_void_p, i64, C.c_void_p, C.c_void_p]
        for suf, ct in (("f32", C.c_float), ("f64", C.c_double)):
            getattr(_lib, f"oracle_rescale_{suf}").argtypes = [i64, C.c_void_p, ct, ct, C.c_int, C.c_void_p]
            for nm in ("spread", "spread_slabs"):
                getattr(_lib, f"oracle_{nm}_{suf}").argtypes = [C.c_int, C.c_int, ct, ct, i64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
            getattr(_lib, f"oracle_interp_{suf}").argtypes = [C.c_int, C.c_int, ct, ct, C.c_void_p, C.c_void_p, i64, C.c_void_p, C.c_void_p]
        _lib.oracle_num_threads.restype = C.c_int
        _lib.oracle_set_threads.argtypes = [C.c_int]
        del dp
    return _lib


def set_threads(n: int) -> None:
    lib().oracle_set_threads(int(n))


def num_threads() -> int:
    return int(lib().oracle_num_threads())


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def _ptrs(arrs):
    keep = [np.ascontiguousarray(a) for a in arrs]
    arr = (C.c_void_p * 3)()
    for i, a in enumerate(keep):
        arr[i] = a.ctypes.data
    return arr, keep


# ---------------------------------------------------------------------------------------------
# FP64 direct sums
# ---------------------------------------------------------------------------------------------
def direct_type1(sign: int, x, c, modes) -> np.ndarray:
    """f[k] = sum_j c_j exp(i sign k.x_j) on the full CMCL mode box; returns complex128 array
    shaped like modes reversed (C-order [z, y, x])."""
    dim = len(modes)
    xs = [np.asarray(a, dtype=np.float64) for a in x]
    cc = np.ascontiguousarray(np.asarray(c, dtype=np.complex128))
    out = np.zeros(int(np.prod(modes)), dtype=np.complex128)
    ptrs, keep = _ptrs(xs)
    m = (C.c_int64 * 3)(*[int(v) for v in modes] + [1] * (3 - dim))
    lib().oracle_direct_type1(dim, int(sign), len(cc), ptrs, _p(cc), m, _p(out))
    return out.reshape(tuple(reversed([int(v) for v in modes])))


def direct_type2(sign: int, modes, f, x) -> np.ndarray:
    """c_j = sum_k f[k] exp(i sign k.x_j), f in CMCL order, column-major (C-order [z, y, x])."""
    dim = len(modes)
    ff = np.ascontiguousarray(np.asarray(f, dtype=np.complex128)).reshape(-1)
    xs = [np.asarray(a, dtype=np.float64) for a in x]
    M = len(xs[0])
    out = np.zeros(M, dtype=np.complex128)
    ptrs, keep = _ptrs(xs)
    m = (C.c_int64 * 3)(*[int(v) for v in modes] + [1] * (3 - dim))
    lib().oracle_direct_type2(dim, int(sign), m, _p(ff), M, ptrs, _p(out))
    return out


def direct_type3(sign: int, x, c, s) -> np.ndarray:
    dim = len(x)
    xs = [np.asarray(a, dtype=np.float64) for a in x]
    ss = [np.asarray(a, dtype=np.float64) for a in s]
    cc = np.ascontiguousarray(np.asarray(c, dtype=np.complex128))
    K = len(ss[0])
    out = np.zeros(K, dtype=np.complex128)
    px, k1 = _ptrs(xs)
    ps, k2 = _ptrs(ss)
    lib().oracle_direct_type3(dim, int(sign), len(cc), px, _p(cc), K, ps, _p(out))
    return out


# ---------------------------------------------------------------------------------------------
# Restated reference parameter code (host, double / T precision)
# ---------------------------------------------------------------------------------------------
def kernel_params(tol: float, upsampfac: float, single: bool):
    """KernelParameters<T> (reference src/neonufft/es_kernel_param.hpp:24-56) -> (w, beta, c)."""
    if upsampfac == 2.0:
        w = math.ceil(-math.log10(tol / 10.0))
    else:
        w = math.ceil(-math.log(tol) / (math.pi * math.sqrt(1.0 - 1.0 / upsampfac)))
    w = min(16, max(2, w))
    beta_fac = {2: 2.20, 3: 2.26, 4: 2.38}.get(w, 2.30)
    if upsampfac != 2.0:
        beta_fac = 0.97 * math.pi * (1.0 - 1.0 / (2 * upsampfac))
    beta = beta_fac * w
    c = 4.0 / (w * w)
    if single:
        beta = float(np.float32(beta))
        c = float(np.float32(c))
    return w, beta, c


def fine_grid_size(modes: int, upsampfac: float, w: int) -> int:
    """src/neonufft/plan_impl.hpp:45-48: max(2w, size_t(modes * upsampfac))."""
    return max(2 * w, int(modes * upsampfac))


def next235even(n: int) -> int:
    """src/contrib/es_kernel/util.hpp:39-61."""
    if n <= 2:
        return 2
    if n % 2:
        n += 1
    while True:
        r = n
        for f in (2, 3, 5):
            while r % f == 0:
                r //= f
        if r == 1:
            return n
        n += 2


def t3_geometry(w: int, upsampfac: float, recenter: float, in_min, in_max, out_min, out_max,
                dt):
    """GridInfoT3 + t3_grid_size + set_nhg_type3 for one dimension, in precision dt
    (reference src/neonufft/util/grid_info_t3.hpp:18-52, src/contrib/es_kernel/util.hpp:64-105).
    Returns dict(C, D, X, S, nf1, nfft, h, gamma) with T-rounded floats."""
    T = dt
    a, b, c, d = T(in_min), T(in_max), T(out_min), T(out_max)
    C_ = T((b + a) / T(2))
    D_ = T((d + c) / T(2))
    X = max(abs(T(b - C_)), abs(T(a - C_)))
    S = max(abs(T(d - D_)), abs(T(c - D_)))
    rec = T(recenter)
    if abs(C_) < T(rec * X):
        C_ = T(0)
        X = max(abs(b), abs(a))
    if abs(D_) < T(rec * S):
        D_ = T(0)
        S = max(abs(d), abs(c))
    up = T(upsampfac)
    pi = T(math.pi)
    Xs, Ss = X, S
    if X == 0:
        if S == 0:
            Xs, Ss = T(1), T(1)
        else:
            Xs = max(Xs, T(T(1) / S))
    else:
        Ss = max(Ss, T(T(1) / X))
    nf1 = int(2.0 * float(up) * float(Ss) * float(Xs) / float(pi) + float(w + 1))
    nf1 = max(nf1, 2 * w)
    nf1 += nf1 % 2
    nfft = next235even(max(2 * w, int(nf1 * upsampfac)))
    h = T(T(2) * pi / T(nf1))
    Sg = S
    if X == 0 and S == 0:
        Sg = T(1)
    elif S == 0:
        Sg = max(Sg, T(T(1) / X))
    gamma = T(float(T(nf1)) / (2.0 * float(up) * float(Sg)))
    return dict(C=C_, D=D_, X=X, S=S, nf1=nf1, nfft=nfft, h=h, gamma=gamma)


def _gl_half(q: int):
    """Positive half of a 2q-node Gauss-Legendre rule (numpy, double)."""
    x, wt = np.polynomial.legendre.leggauss(2 * q)
    return x[q:], wt[q:]


def es_kernel(x, beta, c, dt):
    x = np.asarray(x, dtype=dt)
    arg = dt(1) - dt(c) * x * x
    out = np.exp(dt(beta) * (np.sqrt(np.maximum(arg, 0)).astype(dt) - dt(1))).astype(dt)
    return np.where(arg > 0, out, dt(0)).astype(dt)


def fseries_inverse(w, beta, c, nf, dt):
    """src/neonufft/kernels/fseries_kernel.cpp:33-77, N_QUAD = w + w%2 + 10, in precision dt."""
    q = w + (w % 2) + 10
    z, wt = _gl_half(q)
    half = dt(w) / dt(2)
    kv = (dt(w) * wt.astype(dt) * es_kernel(z.astype(dt) * half, beta, c, dt)).astype(dt)
    alpha = dt(math.pi) * dt(w) / dt(nf)
    ph = (alpha * z.astype(dt)).astype(dt)
    k = np.arange(nf // 2 + 1)
    s = (kv[None, :] * np.cos(k[:, None].astype(dt) * ph[None, :])).astype(dt).sum(axis=1, dtype=dt)
    sign = np.where(k % 2 == 1, -1, 1).astype(dt)
    return (sign / s).astype(dt)


def phi_hat(w, beta, c, xi, dt):
    """Kernel Fourier transform at xi (radians per cell), N_QUAD = w + w%2 nodes
    (reference src/neonufft/kernels/nuft_real_kernel.cpp:31-105), in precision dt."""
    q = w + (w % 2)
    z, wt = _gl_half(q)
    half = dt(w) / dt(2)
    nodes = (z.astype(dt) * half).astype(dt)
    kv = (dt(2) * half * wt.astype(dt) * es_kernel(nodes, beta, c, dt)).astype(dt)
    xi = np.asarray(xi, dtype=dt)
    return (kv[None, :] * np.cos(xi[:, None] * nodes[None, :])).astype(dt).sum(axis=1, dtype=dt)


# ---------------------------------------------------------------------------------------------
# Mode reordering + deconvolution (reference downsample/upsample, CPU and GPU agree)
# ---------------------------------------------------------------------------------------------
def _mode_numbers(n: int, order_cmcl: bool) -> np.ndarray:
    i = np.arange(n)
    n_neg = n // 2
    if order_cmcl:
        return i - n_neg
    return np.where(i < n - n_neg, i, i - n)


def downsample(grid: np.ndarray, modes, corr, order_cmcl=True) -> np.ndarray:
    """grid: C-order [z, y, x] fine grid; returns modes array C-order [z, y, x]."""
    dim = len(modes)
    idx = []
    fac = None
    for d in range(dim):
        k = _mode_numbers(int(modes[d]), order_cmcl)
        nf = grid.shape[dim - 1 - d]
        idx.append(np.where(k >= 0, k, nf + k))
        cd = corr[d][np.abs(k)]
        fac = cd if fac is None else np.multiply.outer(cd, fac)
    sub = grid[np.ix_(*reversed(idx))]
    return (sub * fac.astype(sub.real.dtype)).astype(grid.dtype)


def upsample(f: np.ndarray, modes, nf, corr, order_cmcl=True) -> np.ndarray:
    dim = len(modes)
    grid = np.zeros(tuple(reversed([int(v) for v in nf])), dtype=f.dtype)
    idx = []
    fac = None
    for d in range(dim):
        k = _mode_numbers(int(modes[d]), order_cmcl)
        idx.append(np.where(k >= 0, k, int(nf[d]) + k))
        cd = corr[d][np.abs(k)]
        fac = cd if fac is None else np.multiply.outer(cd, fac)
    grid[np.ix_(*reversed(idx))] = (f.reshape(tuple(reversed([int(v) for v in modes]))) *
                                    fac.astype(f.real.dtype)).astype(f.dtype)
    return grid


def _fft(grid: np.ndarray, sign: int, workers: int) -> np.ndarray:
    """Unnormalised FFT with exponent sign `sign` (FFTW_FORWARD = -1), in the grid's precision."""
    if _sfft is not None:
        if sign < 0:
            return _sfft.fftn(grid, norm="backward", workers=workers)
        return _sfft.ifftn(grid, norm="forward", workers=workers)
    if sign < 0:
        return np.fft.fftn(grid).astype(grid.dtype)
    return (np.fft.ifftn(grid) * grid.size).astype(grid.dtype)


# ---------------------------------------------------------------------------------------------
# Restated reference CPU plans
# ---------------------------------------------------------------------------------------------
class RefPlan:
    """CPU restatement of neonufft::Plan<T, DIM> (reference src/neonufft/plan_impl.hpp:37-134)."""

    def __init__(self, dtype, sign, loc, modes, tol=1e-3, upsampfac=2.0, order_cmcl=True,
                 workers=None):
        self.dt = np.float32 if np.dtype(dtype) == np.float32 else np.float64
        self.cdt = np.complex64 if self.dt == np.float32 else np.complex128
        self.sfx = "f32" if self.dt == np.float32 else "f64"
        self.sign = -1 if sign < 0 else 1
        self.dim = len(modes)
        self.modes = [int(m) for m in modes]
        self.order_cmcl = order_cmcl
        self.workers = workers or os.cpu_count() or 1
        self.w, self.beta, self.c = kernel_params(tol, upsampfac, self.dt == np.float32)
        self.nf = [fine_grid_size(m, upsampfac, self.w) for m in self.modes]
        self.corr = [fseries_inverse(self.w, self.beta, self.c, n, self.dt) for n in self.nf]
        self.set_points(loc)

    def set_points(self, loc):
        """rescale_loc (src/neonufft/kernels/rescale_loc_kernel.cpp:33-74), in T."""
        self.p = []
        for a in loc:
            a = np.ascontiguousarray(np.asarray(a, dtype=self.dt))
            out = np.empty_like(a)
            getattr(lib(), f"oracle_rescale_{self.sfx}")(len(a), _p(a), 0.0, 1.0, 0, _p(out))
            self.p.append(out)
        self.M = len(self.p[0]) if self.p else 0

    def _nf3(self):
        return (C.c_int64 * 3)(*self.nf + [1] * (3 - self.dim))

    def spread(self, c, pre=None, slabs=False) -> np.ndarray:
        cc = np.ascontiguousarray(np.asarray(c, dtype=self.cdt))
        grid = np.zeros(tuple(reversed(self.nf)), dtype=self.cdt)
        ptrs, keep = _ptrs(self.p)
        pp = None if pre is None else np.ascontiguousarray(pre, dtype=self.cdt)
        fn = getattr(lib(), f"oracle_{'spread_slabs' if slabs else 'spread'}_{self.sfx}")
        fn(self.dim, self.w, self.beta, self.c, self.M, ptrs, _p(cc),
           None if pp is None else _p(pp), self._nf3(), _p(grid))
        return grid

    def interp(self, grid: np.ndarray) -> np.ndarray:
        g = np.ascontiguousarray(grid, dtype=self.cdt)
        out = np.zeros(self.M, dtype=self.cdt)
        ptrs, keep = _ptrs(self.p)
        getattr(lib(), f"oracle_interp_{self.sfx}")(self.dim, self.w, self.beta, self.c, _p(g),
                                                     self._nf3(), self.M, ptrs, _p(out))
        return out

    def transform_type_1(self, c) -> np.ndarray:
        """plan_impl.hpp:77-97: spread (serial), fold, FFT, downsample. Returns modes C-order."""
        grid = self.spread(c)
        grid = _fft(grid, self.sign, self.workers).astype(self.cdt)
        return downsample(grid, self.modes, self.corr, self.order_cmcl)

    def transform_type_2(self, f) -> np.ndarray:
        """plan_impl.hpp:99-126: upsample, FFT, interpolate (threaded)."""
        grid = upsample(np.asarray(f, dtype=self.cdt), self.modes, self.nf, self.corr,
                        self.order_cmcl)
        grid = _fft(grid, self.sign, self.workers).astype(self.cdt)
        return self.interp(grid)


class RefPlanT3:
    """CPU restatement of neonufft::PlanT3<T, DIM> (reference src/neonufft/plan_t3_impl.hpp:66-380)."""

    def __init__(self, dtype, sign, x, s, tol=1e-3, upsampfac=2.0, recenter=0.1, batch=1,
                 workers=None):
        self.dt = np.float32 if np.dtype(dtype) == np.float32 else np.float64
        self.cdt = np.complex64 if self.dt == np.float32 else np.complex128
        self.sfx = "f32" if self.dt == np.float32 else "f64"
        self.sign = -1 if sign < 0 else 1
        self.dim = len(x)
        self.batch = batch
        self.workers = workers or os.cpu_count() or 1
        self.w, self.beta, self.c = kernel_params(tol, upsampfac, self.dt == np.float32)
        x = [np.ascontiguousarray(np.asarray(a, dtype=self.dt)) for a in x]
        s = [np.ascontiguousarray(np.asarray(a, dtype=self.dt)) for a in s]
        self.geo = []
        for d in range(self.dim):
            g = t3_geometry(self.w, upsampfac, recenter, x[d].min() if len(x[d]) else 0,
                            x[d].max() if len(x[d]) else 0, s[d].min() if len(s[d]) else 0,
                            s[d].max() if len(s[d]) else 0, self.dt)
            self.geo.append(g)
        self.nf1 = [g["nf1"] for g in self.geo]
        self.nfft = [g["nfft"] for g in self.geo]
        self.corr = [fseries_inverse(self.w, self.beta, self.c, n, self.dt) for n in self.nfft]
        self.grid = np.zeros((batch,) + tuple(reversed(self.nf1)), dtype=self.cdt)
        self._set_input(x)
        self._set_output(s)

    def _rescale(self, a, off, scale):
        out = np.empty_like(a)
        getattr(lib(), f"oracle_rescale_{self.sfx}")(len(a), _p(a), off, scale, 1, _p(out))
        return out

    def _set_input(self, x):
        """Prephase exp(i sign x.D) in T (compute_prephase_kernel.cpp) and rescale by 1/gamma."""
        dt = self.dt
        self.M = len(x[0])
        if any(g["D"] != 0 for g in self.geo):
            ph = np.zeros(self.M, dtype=dt)
            for d in range(self.dim):
                ph = (ph + x[d] * self.geo[d]["D"]).astype(dt)
            self.pre = (np.cos(ph) + 1j * self.sign * np.sin(ph)).astype(self.cdt)
        else:
            self.pre = None
        self.px = [self._rescale(x[d], self.geo[d]["C"], dt(dt(1) / self.geo[d]["gamma"]))
                   for d in range(self.dim)]

    def _set_output(self, s):
        """Rescale by gamma*h, phi_hat (nuft_real_kernel.cpp) and postphase
        (compute_postphase_kernel.cpp), in T."""
        dt = self.dt
        self.K = len(s[0])
        self.ps = []
        prod = np.ones(self.K, dtype=dt)
        phase = np.zeros(self.K, dtype=dt)
        for d in range(self.dim):
            g = self.geo[d]
            sc = dt(g["gamma"] * g["h"])
            self.ps.append(self._rescale(s[d], g["D"], sc))
            xi = ((s[d] - g["D"]) * sc).astype(dt)
            prod = (prod * phi_hat(self.w, self.beta, self.c, xi, dt)).astype(dt)
            phase = (phase + (s[d] - g["D"]).astype(dt) * g["C"]).astype(dt)
        self.post = ((np.cos(phase) + 1j * self.sign * np.sin(phase)) / prod).astype(self.cdt)

    def add_input(self, c):
        c = np.asarray(c, dtype=self.cdt).reshape(self.batch, -1)
        nf3 = (C.c_int64 * 3)(*self.nf1 + [1] * (3 - self.dim))
        ptrs, keep = _ptrs(self.px)
        pp = None if self.pre is None else np.ascontiguousarray(self.pre)
        for b in range(self.batch):
            cb = np.ascontiguousarray(c[b])
            g = np.zeros(tuple(reversed(self.nf1)), dtype=self.cdt)
            getattr(lib(), f"oracle_spread_slabs_{self.sfx}")(
                self.dim, self.w, self.beta, self.c, self.M, ptrs, _p(cb),
                None if pp is None else _p(pp), nf3, _p(g))
            self.grid[b] += g

    def transform(self) -> np.ndarray:
        out = np.zeros((self.batch, self.K), dtype=self.cdt)
        nf3 = (C.c_int64 * 3)(*self.nfft + [1] * (3 - self.dim))
        ptrs, keep = _ptrs(self.ps)
        for b in range(self.batch):
            fine = upsample(self.grid[b], self.nf1, self.nfft, self.corr, True)
            fine = np.ascontiguousarray(_fft(fine, self.sign, self.workers).astype(self.cdt))
            o = np.zeros(self.K, dtype=self.cdt)
            getattr(lib(), f"oracle_interp_{self.sfx}")(self.dim, self.w, self.beta, self.c,
                                                         _p(fine), nf3, self.K, ptrs, _p(o))
            out[b] = (o * self.post).astype(self.cdt)
        return out


# ---------------------------------------------------------------------------------------------
# Error metrics
# ---------------------------------------------------------------------------------------------
def rel_l2(out, ref) -> float:
    out = np.asarray(out, dtype=np.complex128).reshape(-1)
    ref = np.asarray(ref, dtype=np.complex128).reshape(-1)
    den = np.linalg.norm(ref)
    return float(np.linalg.norm(out - ref) / (den if den > 0 else 1.0))


def reference_compare(ref, out, tol: float, element_factor: float, fraction: float):
    """Acceptance rule of the reference tests (tests/test_type_1_2.cpp:84-108,
    tests/test_type_3.cpp:206-233): per element e = |out - ref|^2 / |ref|^2 (squared norms,
    as written there); every e < element_factor * tol and more than `fraction` of the
    elements with e <= tol. Returns (ok, max_e, frac_below)."""
    out = np.asarray(out, dtype=np.complex128).reshape(-1)
    ref = np.asarray(ref, dtype=np.complex128).reshape(-1)
    with np.errstate(divide="ignore", invalid="ignore"):
        e = np.abs(out - ref) ** 2 / np.abs(ref) ** 2
    e = np.where(np.isnan(e), 0.0, e)
    frac = float(np.mean(e <= tol)) if len(e) else 1.0
    mx = float(e.max()) if len(e) else 0.0
    return (mx < element_factor * tol and frac > fraction), mx, frac


# ---------------------------------------------------------------------------------------------
# Reference pin library (oracle/_ref), when built
# ---------------------------------------------------------------------------------------------
class Ref:
    """The reference's own code compiled from its sources (see oracle/Makefile `ref`)."""

    def __init__(self, path: Path = REF_LIB_PATH):
        if not path.exists():
            raise FileNotFoundError(path)
        L = C.CDLL(str(path))
        L.ref_kernel_param.argtypes = [C.c_double, C.c_double, C.c_int, C.POINTER(C.c_int),
                                       C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.ref_t3_geometry.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                      C.c_double, C.c_double, C.c_double,
                                      C.POINTER(C.c_double), C.POINTER(C.c_int64)]
        L.ref_next235even.argtypes = [C.c_int64]
        L.ref_next235even.restype = C.c_int64
        L.ref_legendre.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
        L.ref_gpu_type12.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                     C.c_int, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p]
        L.ref_gpu_type12.restype = C.c_int
        L.ref_gpu_type3.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int64,
                                    C.c_void_p, C.c_int64, C.c_void_p, C.c_int, C.c_void_p,
                                    C.c_void_p]
        L.ref_gpu_type3.restype = C.c_int
        L.ref_plan12_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_double,
                                        C.c_double, C.c_int, C.c_int64, C.c_void_p, C.c_void_p]
        L.ref_plan12_create.restype = C.c_int
        L.ref_plan12_set_points.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
        L.ref_plan12_set_points.restype = C.c_int
        L.ref_plan12_t1.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_plan12_t1.restype = C.c_int
        L.ref_plan12_t2.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_plan12_t2.restype = C.c_int
        L.ref_plan12_destroy.argtypes = [C.c_void_p]
        L.ref_plan12_destroy.restype = None
        self.L = L

    def kernel_param(self, tol, upsampfac, single):
        w = C.c_int()
        b = C.c_double()
        c = C.c_double()
        self.L.ref_kernel_param(tol, upsampfac, int(single), C.byref(w), C.byref(b), C.byref(c))
        return w.value, b.value, c.value

    def t3_geometry(self, single, w, upsampfac, recenter, in_min, in_max, out_min, out_max):
        out = (C.c_double * 6)()
        grids = (C.c_int64 * 2)()
        self.L.ref_t3_geometry(int(single), w, upsampfac, recenter, in_min, in_max, out_min,
                               out_max, out, grids)
        return dict(C=out[0], D=out[1], X=out[2], S=out[3], h=out[4], gamma=out[5],
                    nf1=grids[0], nfft=grids[1])

    def next235even(self, n):
        return int(self.L.ref_next235even(int(n)))

    def legendre(self, n):
        x = np.zeros(n)
        w = np.zeros(n)
        self.L.ref_legendre(n, _p(x), _p(w))
        return x, w
