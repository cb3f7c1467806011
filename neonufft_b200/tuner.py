"""Configuration tuning for the engine's plans: the plain heuristic, a measuring autotuner, and a
learned picker.

A configuration is (upsampling factor, kernel width, spreading method, tile). The plain
heuristic is the reference's parameter choice (upsampfac 2, w from the tolerance,
es_kernel_param.hpp:24-56) with the plan's default method and tile. The autotuner runs every
candidate configuration of a problem on the GPU, measures its time and its error against the
engine's FP64 direct sums on sampled outputs, and keeps the fastest one that meets the
tolerance. The learned picker ranks the candidates with a cost model (costmodel.CostModel, an
MLP trained on the autotuner's timings) and accepts the best-ranked candidate only once its
measured error meets the tolerance, falling back to the heuristic otherwise. No counterpart in
the reference.
"""
from __future__ import annotations

import ctypes as C
import json
import math
from dataclasses import asdict, dataclass

import numpy as np

from . import _lib as L
from .plan import Options, Plan, check, direct_type1_f64, direct_type2_f64


@dataclass(frozen=True)
class Problem:
    dim: int
    type: int          # 1 or 2
    M: int
    N: int             # modes per dimension
    tol: float
    precision: str = "f32"
    blob: bool = False  # points in a Gaussian blob (sigma 0.1) instead of uniform
    seed: int = 0


@dataclass(frozen=True)
class Config:
    upsampfac: float = 2.0
    n_spread: int = 0        # 0: the reference heuristic for (tol, upsampfac)
    method: int = 0          # 0: the plan's default
    tile: tuple = (0, 0, 0)  # (0, 0, 0): the plan's default

    def options(self, tol: float) -> Options:
        return Options(tol=tol, upsampfac=self.upsampfac, n_spread=self.n_spread,
                       spread_method=self.method, tile=self.tile)


HEURISTIC = Config()


def heuristic_width(tol: float, upsampfac: float, precision: str) -> int:
    w, beta, c = C.c_int(0), C.c_double(0), C.c_double(0)
    prec = L.NNB_DOUBLE if precision == "f64" else L.NNB_FLOAT
    check(L.load().nnb_es_kernel_params(tol, upsampfac, prec, C.byref(w), C.byref(beta),
                                        C.byref(c)))
    return w.value


def resolved(p: Problem, c: Config):
    """(kernel width, method, x tile, y tile) that a plan with configuration c uses."""
    w = c.n_spread or heuristic_width(p.tol, c.upsampfac, p.precision)
    method = c.method or (3 if p.dim == 3 and w <= 8 else 1)
    tile0 = c.tile[0] or (4 if method == 3 else 0)
    tile1 = c.tile[1] or (8 if method == 3 else 0)
    return w, method, tile0, tile1


def candidates(p: Problem):
    """The heuristic first, then every (upsampfac, width, method, tile) the tuner considers."""
    out = [HEURISTIC]
    for sigma in (2.0, 1.5):
        w0 = heuristic_width(p.tol, sigma, p.precision)
        for w in (w0, w0 + 1):
            if w > 16:
                continue
            if p.dim == 3:
                methods = [(1, (0, 0, 0))]
                if w <= 8:
                    methods = [(3, (8, 8, 1)), (3, (4, 8, 1))] + methods
                    if p.precision == "f32" and w >= 5:
                        methods.insert(2, (3, (4, 4, 1)))  # 4-row tiles: single precision
            elif p.dim == 2:
                methods = [(1, (0, 0, 0)), (2, (0, 0, 0))]
            else:
                methods = [(1, (0, 0, 0))]
            for m, tile in methods:
                c = Config(sigma, w, m, tile)
                if c not in out:
                    out.append(c)
    return out


def features(p: Problem, c: Config) -> np.ndarray:
    w, method, tile0, tile1 = resolved(p, c)
    nf = max(2 * w, int(p.N * c.upsampfac))
    lcells = p.dim * math.log10(nf)
    return np.array([
        float(p.dim == 3), float(p.type == 2), math.log10(p.M), p.dim * math.log10(p.N), lcells,
        -math.log10(p.tol), float(p.precision == "f64"), float(p.blob), c.upsampfac, float(w),
        float(method == 1), float(method == 2), float(method == 3), float(tile0),
        math.log10(p.M) - lcells, float(w) ** p.dim / 100.0, float(tile1),
    ], dtype=np.float64)


N_FEATURES = 17


class ProblemData:
    """Seeded device inputs of a problem (points, strengths or modes, output buffer)."""

    def __init__(self, p: Problem):
        import torch
        self.p = p
        rdt = torch.float64 if p.precision == "f64" else torch.float32
        cdt = torch.complex128 if p.precision == "f64" else torch.complex64
        g = torch.Generator(device="cuda")
        g.manual_seed(1000 + p.seed)
        if p.blob:
            centre = (torch.rand(p.dim, generator=g, device="cuda", dtype=torch.float64) * 2 - 1) * math.pi
            self.loc = [torch.remainder(centre[d] + 0.1 * torch.randn(p.M, generator=g, device="cuda",
                                                                        dtype=torch.float64) + math.pi,
                                        2 * math.pi).sub(math.pi).to(rdt) for d in range(p.dim)]
        else:
            self.loc = [((torch.rand(p.M, generator=g, device="cuda", dtype=torch.float64) * 2 - 1)
                         * math.pi).to(rdt) for _ in range(p.dim)]
        n_in = p.M if p.type == 1 else p.N ** p.dim
        self.inp = torch.complex(torch.randn(n_in, generator=g, device="cuda", dtype=torch.float64),
                                 torch.randn(n_in, generator=g, device="cuda", dtype=torch.float64)).to(cdt)
        n_out = p.N ** p.dim if p.type == 1 else p.M
        self.out = torch.empty(n_out, dtype=cdt, device="cuda")
        self.strides = [p.N ** d for d in range(p.dim)]
        self._ref = None

    def reference(self, samples: int = 256):
        """(indices, FP64 direct sums) on sampled outputs, computed once."""
        import torch
        if self._ref is None:
            p = self.p
            g = torch.Generator(device="cuda")
            g.manual_seed(7)
            loc64 = [a.double() for a in self.loc]
            ref = torch.empty(samples, dtype=torch.complex128, device="cuda")
            if p.type == 1:
                idx = torch.randint(0, p.N ** p.dim, (samples,), generator=g, device="cuda")
                kk, rem = [], idx.clone()
                for _ in range(p.dim):
                    kk.append(rem % p.N - p.N // 2)
                    rem = rem // p.N
                direct_type1_f64(-1, loc64, self.inp.to(torch.complex128),
                                 torch.stack(kk, dim=1).contiguous(), ref)
            else:
                idx = torch.randint(0, p.M, (samples,), generator=g, device="cuda")
                direct_type2_f64(-1, [p.N] * p.dim, self.inp.to(torch.complex128), loc64, idx, ref)
            self._ref = (idx, ref)
        return self._ref


def measure(p: Problem, c: Config, data: ProblemData = None, reps: int = 3):
    """(milliseconds per set_points + transform, relative l2 error on sampled outputs)."""
    import torch
    data = data or ProblemData(p)
    plan = Plan(c.options(p.tol), -1, p.M, data.loc, [p.N] * p.dim)

    def run():
        plan.set_points(p.M, data.loc)
        if p.type == 1:
            plan.transform_type_1(data.inp, data.out, data.strides)
        else:
            plan.transform_type_2(data.inp, data.strides, data.out)

    run()
    torch.cuda.synchronize()
    times = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    idx, ref = data.reference()
    got = data.out[idx].to(torch.complex128)
    err = float(torch.linalg.norm(got - ref) / torch.linalg.norm(ref))
    plan.close()
    return float(np.median(times)), err


def measure_or_none(p: Problem, c: Config, data: ProblemData = None):
    """measure(), or None when the configuration does not fit in device memory or is refused
    (an InputError for a shape the methods do not support)."""
    from .plan import InputError, MemoryAllocError
    try:
        return measure(p, c, data)
    except (InputError, MemoryAllocError):
        import torch
        torch.cuda.empty_cache()
        return None


class Tuner:
    """Heuristic, autotuner and learned picker over the candidates of a problem."""

    def __init__(self, model=None):
        self.model = model
        self.rows = []  # (features, log10 ms, error, problem, config)

    def sweep(self, problems):
        """Measures every candidate of every problem (the autotuner's data and the model's)."""
        for p in problems:
            data = ProblemData(p)
            for c in candidates(p):
                r = measure_or_none(p, c, data)
                if r is not None:
                    self.rows.append((features(p, c), math.log10(r[0]), r[1], p, c))
        return self.rows

    def autotune(self, p: Problem):
        """Fastest measured candidate of p meeting its tolerance (from the sweep rows)."""
        best = None
        for f, lms, err, q, c in self.rows:
            if q == p and err <= p.tol and (best is None or lms < best[0]):
                best = (lms, c)
        return best[1] if best else HEURISTIC

    def train(self, rows=None, epochs: int = 3000, seed: int = 0) -> float:
        from .costmodel import CostModel
        rows = rows if rows is not None else self.rows
        feats = np.stack([r[0] for r in rows])
        y = np.array([r[1] for r in rows])
        self.model = CostModel(feats.shape[1], seed=seed)
        return self.model.fit(feats, y, epochs=epochs)

    # ---- persistence: the measured rows and the trained network, versioned -----------------
    FORMAT = "neonufft_b200.tuner"
    VERSION = 1

    def save(self, path) -> None:
        """Writes the sweep's rows (problem, configuration, log10 ms, error) and, when trained,
        the cost model to a JSON file, so that a tuning run can be reproduced or reused."""
        doc = {"format": self.FORMAT, "version": self.VERSION, "n_features": N_FEATURES,
               "rows": [{"problem": asdict(p), "config": {**asdict(c), "tile": list(c.tile)},
                         "log10_ms": float(lms), "error": float(err)}
                        for f, lms, err, p, c in self.rows],
               "model": self.model.state() if self.model is not None else None}
        with open(path, "w") as fh:
            json.dump(doc, fh)

    @classmethod
    def load(cls, path, with_model: bool = True) -> "Tuner":
        """Reads a file written by save(); the features are recomputed from each row's problem
        and configuration (host-only). The model needs a GPU; with_model=False skips it."""
        with open(path) as fh:
            doc = json.load(fh)
        if doc.get("format") != cls.FORMAT or int(doc.get("version", 0)) != cls.VERSION:
            raise ValueError(f"not a version-{cls.VERSION} tuner file: {path}")
        if int(doc.get("n_features", -1)) != N_FEATURES:
            raise ValueError("the file's feature set differs from this version's")
        t = cls()
        for r in doc["rows"]:
            p = Problem(**r["problem"])
            cd = dict(r["config"])
            cd["tile"] = tuple(int(v) for v in cd["tile"])
            c = Config(**cd)
            t.rows.append((features(p, c), float(r["log10_ms"]), float(r["error"]), p, c))
        if with_model and doc.get("model") is not None:
            from .costmodel import CostModel
            t.model = CostModel.from_state(doc["model"])
        return t

    def pick(self, p: Problem, data: ProblemData = None):
        """(configuration, measured (ms, error), candidates tried): the best-ranked candidate
        whose measured error meets tol; the heuristic when none does."""
        cands = candidates(p)
        if self.model is None:
            return HEURISTIC, None, 0
        pred = self.model.predict(np.stack([features(p, c) for c in cands]))
        data = data or ProblemData(p)
        for tried, i in enumerate(np.argsort(pred), start=1):
            r = measure_or_none(p, cands[int(i)], data)
            if r is not None and r[1] <= p.tol:
                return cands[int(i)], r, tried
        return HEURISTIC, measure(p, HEURISTIC, data), len(cands)


def rule_plus_one(p: Problem) -> Config:
    """The simplest fix of the heuristic's tolerance misses: its width plus one, upsampfac 2,
    the plan's default method and tile."""
    return Config(2.0, min(16, heuristic_width(p.tol, 2.0, p.precision) + 1), 0, (0, 0, 0))


def evaluate(tuner: Tuner, held, exhaustive: bool = True) -> dict:
    """Scores the learned picks on held-out problems against the reference heuristic, the
    width-plus-one rule and (optionally) exhaustive autotuning over every candidate.

    Time ratios are geometric means of (other configuration's time / pick's time), each over
    the problems where that configuration meets tol; `measurements_*` count the candidate
    configurations measured (plan built, run, error checked) per problem."""
    def geo(v):
        return float(np.exp(np.mean(np.log(v)))) if v else None

    r_heur, r_rule, r_best, tried, n_cands = [], [], [], [], []
    heur_miss = rule_miss = pick_miss = 0
    for p in held:
        data = ProblemData(p)
        cfg, (ms, err), k = tuner.pick(p, data)
        tried.append(k)
        pick_miss += int(err > p.tol)
        h_ms, h_err = measure(p, HEURISTIC, data)
        if h_err <= p.tol:
            r_heur.append(h_ms / ms)
        else:
            heur_miss += 1
        rr = measure_or_none(p, rule_plus_one(p), data)
        if rr is not None and rr[1] <= p.tol:
            r_rule.append(rr[0] / ms)
        else:
            rule_miss += 1
        cands = candidates(p)
        n_cands.append(len(cands))
        if exhaustive:
            best = None
            for c in cands:
                r = measure_or_none(p, c, data)
                if r is not None and r[1] <= p.tol and (best is None or r[0] < best):
                    best = r[0]
            if best is not None:
                r_best.append(best / ms)
        del data
    return {
        "problems": len(held), "picks_missing_tol": pick_miss,
        "heuristic_missed_tol": heur_miss, "rule_plus_one_missed_tol": rule_miss,
        "speedup_vs_heuristic_geomean": geo(r_heur),
        "speedup_vs_rule_plus_one_geomean": geo(r_rule),
        "pick_time_over_exhaustive_best_geomean": (1.0 / geo(r_best)) if r_best else None,
        "measurements_per_pick": float(np.mean(tried)) if tried else None,
        "measurements_exhaustive": float(np.mean(n_cands)) if n_cands else None,
    }
