"""Batched execution of uneven transforms (nnb_batch_*) on the GPU.

A batch of 2D and 3D, type-1 and type-2 transforms with uneven point counts, grid sizes and
point distributions (uniform and Gaussian blobs) must give, in each of its modes (serial,
concurrent streams, captured CUDA graph, and the fused modes, whose 3D z-window steps run as
persistent launches over one work queue per kernel shape, direct or captured), the results of the
same transforms run one at a time through single plans, and meet the tolerance against the FP64
direct sum. A replayed graph must pick up new data written into the same input buffers.
"""
import numpy as np
import pytest

from gpu_helpers import col_strides, tdtypes

pytestmark = pytest.mark.gpu


def make_problems(rng, dtype, n):
    probs = []
    for i in range(n):
        dim = 2 if i % 2 == 0 else 3
        type_ = 1 if i % 3 != 2 else 2
        M = int(rng.integers(50, 3000))
        modes = [int(rng.choice([8, 12, 16, 24, 33])) for _ in range(dim)]
        if i % 4 == 1:  # Gaussian blob, wrapped into [-pi, pi)
            centre = rng.uniform(-np.pi, np.pi, dim)
            pts = [np.mod(centre[d] + 0.1 * rng.standard_normal(M) + np.pi, 2 * np.pi) - np.pi
                   for d in range(dim)]
        else:
            pts = [rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]
        n_in = M if type_ == 1 else int(np.prod(modes))
        inp = rng.standard_normal(n_in) + 1j * rng.standard_normal(n_in)
        probs.append(dict(dim=dim, type=type_, M=M, modes=modes,
                          pts=[p.astype(dtype) for p in pts], inp=inp,
                          sign=-1 if i % 2 else 1))
    return probs


def device_buffers(torch, dtype, p):
    rdt, cdt, npc = tdtypes(torch, dtype)
    loc = [torch.from_numpy(x).cuda() for x in p["pts"]]
    inp = torch.from_numpy(p["inp"].astype(npc)).cuda()
    n_out = int(np.prod(p["modes"])) if p["type"] == 1 else p["M"]
    out = torch.zeros(n_out, dtype=cdt, device="cuda")
    return loc, inp, out


def single(nnb, torch, dtype, p, tol):
    loc, inp, out = device_buffers(torch, dtype, p)
    plan = nnb.Plan(nnb.Options(tol=tol), p["sign"], p["M"], loc, p["modes"])
    if p["type"] == 1:
        plan.transform_type_1(inp, out, col_strides(p["modes"]))
    else:
        plan.transform_type_2(inp, col_strides(p["modes"]), out)
    torch.cuda.synchronize()
    plan.close()
    return out.cpu().numpy()


def direct(oracle, p):
    x = [a.astype(np.float64) for a in p["pts"]]
    if p["type"] == 1:
        return oracle.direct_type1(p["sign"], x, p["inp"], p["modes"]).reshape(-1)
    return oracle.direct_type2(p["sign"], p["modes"], p["inp"], x)


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_batch_modes_match_single_plans(dtype, cuda, engine, oracle):
    torch = cuda
    rng = np.random.default_rng(41)
    tol = 1e-5 if dtype == "float32" else 1e-9
    probs = make_problems(rng, dtype, 12)
    refs = [single(engine, torch, dtype, p, tol) for p in probs]
    batch = engine.Batch(engine.Options(tol=tol), getattr(torch, dtype), num_streams=3)
    outs = []
    for p in probs:
        loc, inp, out = device_buffers(torch, dtype, p)
        batch.add(p["type"], p["sign"], loc, p["modes"], inp, out, col_strides(p["modes"]))
        outs.append(out)
    assert len(batch) == len(probs)
    same = 2e-6 if dtype == "float32" else 1e-12
    bound = 1e-4 if dtype == "float32" else 1e-7
    for mode in (engine.Batch.SERIAL, engine.Batch.STREAMS, engine.Batch.GRAPH, engine.Batch.GRAPH,
                 engine.Batch.FUSED, engine.Batch.FUSED_GRAPH, engine.Batch.FUSED_GRAPH):
        for o in outs:
            o.fill_(float("nan"))
        batch.execute(mode)
        torch.cuda.synchronize()
        for p, o, r in zip(probs, outs, refs):
            got = o.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert oracle.rel_l2(got, r) < same
    for p, o in zip(probs, outs):
        assert oracle.rel_l2(o.cpu().numpy(), direct(oracle, p)) < bound
    batch.close()


@pytest.mark.parametrize("mode", ["GRAPH", "FUSED_GRAPH"])
def test_batch_graph_replays_new_inputs(mode, cuda, engine, oracle):
    torch = cuda
    rng = np.random.default_rng(5)
    probs = make_problems(rng, "float32", 6)
    batch = engine.Batch(engine.Options(tol=1e-6), torch.float32, num_streams=2)
    bufs = []
    for p in probs:
        loc, inp, out = device_buffers(torch, "float32", p)
        batch.add(p["type"], p["sign"], loc, p["modes"], inp, out, col_strides(p["modes"]))
        bufs.append((inp, out))
    batch.execute(getattr(engine.Batch, mode))
    for p, (inp, out) in zip(probs, bufs):
        p["inp"] = rng.standard_normal(inp.numel()) + 1j * rng.standard_normal(inp.numel())
        inp.copy_(torch.from_numpy(p["inp"].astype(np.complex64)))
    batch.execute(getattr(engine.Batch, mode))
    torch.cuda.synchronize()
    for p, (inp, out) in zip(probs, bufs):
        assert oracle.rel_l2(out.cpu().numpy(), direct(oracle, p)) < 2e-5
    batch.close()


def make_3d_problems(rng, dtype, n, big=False):
    """3D transforms only (all on the z-window kernels), both types, uniform and blob points."""
    probs = []
    for i in range(n):
        type_ = 1 if i % 3 != 1 else 2
        M = int(rng.integers(20000, 60000)) if big and i < 2 else int(rng.integers(100, 4000))
        modes = [int(rng.choice([10, 16, 20, 24])) for _ in range(3)]
        if i % 2 == 1:  # Gaussian blob, wrapped into [-pi, pi)
            centre = rng.uniform(-np.pi, np.pi, 3)
            pts = [np.mod(centre[d] + 0.1 * rng.standard_normal(M) + np.pi, 2 * np.pi) - np.pi
                   for d in range(3)]
        else:
            pts = [rng.uniform(-np.pi, np.pi, M) for _ in range(3)]
        n_in = M if type_ == 1 else int(np.prod(modes))
        inp = rng.standard_normal(n_in) + 1j * rng.standard_normal(n_in)
        probs.append(dict(dim=3, type=type_, M=M, modes=modes,
                          pts=[p.astype(dtype) for p in pts], inp=inp,
                          sign=-1 if i % 2 else 1))
    return probs


@pytest.mark.parametrize("dtype", ["float32", "float64"])
def test_fused_groups_share_persistent_launches(dtype, cuda, engine, oracle):
    """Transforms with two kernel widths (per-transform option overrides) form four groups
    (two types x two widths); each group's step is one persistent launch. Checked against single
    plans with the same options, and through the launch count: the fused modes launch one kernel
    per group where the stream mode launches one per transform."""
    torch = cuda
    rng = np.random.default_rng(77)
    tol = 1e-5 if dtype == "float32" else 1e-7
    probs = make_3d_problems(rng, dtype, 12, big=True)
    widths = [6 if i % 2 else 8 for i in range(len(probs))]
    batch = engine.Batch(engine.Options(tol=tol), getattr(torch, dtype), num_streams=4)
    outs, refs = [], []
    for p, w in zip(probs, widths):
        opt = engine.Options(tol=tol, n_spread=w)
        loc, inp, out = device_buffers(torch, dtype, p)
        batch.add(p["type"], p["sign"], loc, p["modes"], inp, out, col_strides(p["modes"]), opt=opt)
        outs.append(out)
        loc2, inp2, out2 = device_buffers(torch, dtype, p)
        plan = engine.Plan(opt, p["sign"], p["M"], loc2, p["modes"])
        assert plan.info()["spread_method"] == 3
        if p["type"] == 1:
            plan.transform_type_1(inp2, out2, col_strides(p["modes"]))
        else:
            plan.transform_type_2(inp2, col_strides(p["modes"]), out2)
        torch.cuda.synchronize()
        refs.append(out2.cpu().numpy())
        plan.close()
    groups = len({(p["type"], w) for p, w in zip(probs, widths)})
    assert groups == 4
    same = 2e-6 if dtype == "float32" else 1e-12
    launches = {}
    for mode in ("STREAMS", "FUSED", "FUSED", "FUSED_GRAPH", "FUSED_GRAPH"):
        for o in outs:
            o.fill_(float("nan"))
        torch.cuda.synchronize()
        l0 = engine.kernel_launches()
        batch.execute(getattr(engine.Batch, mode))
        torch.cuda.synchronize()
        launches[mode] = engine.kernel_launches() - l0
        for o, r in zip(outs, refs):
            got = o.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert oracle.rel_l2(got, r) < same
    assert launches["STREAMS"] - launches["FUSED"] == len(probs) - groups
    for p, o, w in zip(probs, outs, widths):
        # w = 6 leaves ~1e-5 of kernel truncation error in either precision
        bound = 2e-4 if w == 6 else (1e-4 if dtype == "float32" else 1e-6)
        assert oracle.rel_l2(o.cpu().numpy(), direct(oracle, p)) < bound
    batch.close()


def test_batch_rejects_bad_requests(cuda, engine):
    torch = cuda
    batch = engine.Batch(engine.Options(tol=1e-6), torch.float32, num_streams=1)
    loc = [torch.zeros(4, device="cuda") for _ in range(2)]
    c = torch.zeros(4, dtype=torch.complex64, device="cuda")
    out = torch.zeros(64, dtype=torch.complex64, device="cuda")
    with pytest.raises(engine.InputError):
        batch.add(3, 1, loc, [8, 8], c, out, [1, 8])
    with pytest.raises(engine.InputError):
        batch.execute(7)
    batch.execute(engine.Batch.FUSED)  # empty batch: nothing to do
    with pytest.raises(engine.InputError):
        engine.Batch(engine.Options(tol=1e-6), torch.float32, num_streams=0)
    batch.execute(engine.Batch.GRAPH)  # empty batch: nothing to do
    batch.close()


@pytest.mark.parametrize("world", [2, 3])
def test_batch_split_over_ranks(world, cuda, engine, oracle):
    """One batch split over `world` ranks (neonufft_b200.replicas.ShardedBatch), the ranks
    emulated one after another on this GPU (they never wait on one another): every transform
    is held by exactly one rank, and the union of the ranks' outputs matches the FP64 direct
    sums and the whole batch run by one process."""
    from neonufft_b200 import replicas
    torch = cuda
    dtype, tol = "float32", 1e-5
    rng = np.random.default_rng(43)
    probs = make_problems(rng, dtype, 11)
    costs = [replicas.transform_cost(p["dim"], p["M"], p["modes"], tol) for p in probs]
    owners = replicas.shard_owners(costs, world)
    outs = [None] * len(probs)
    held = []
    for rank in range(world):
        sb = replicas.ShardedBatch(engine.Options(tol=tol), torch.float32, owners, rank,
                                   num_streams=2)
        for i, p in enumerate(probs):
            if not sb.owns(i):
                continue
            loc, inp, out = device_buffers(torch, dtype, p)
            sb.add(i, p["type"], p["sign"], loc, p["modes"], inp, out, col_strides(p["modes"]))
            outs[i] = out
        with pytest.raises(ValueError):
            sb.add(next(i for i in range(len(probs)) if not sb.owns(i)), 1, -1, [], [8], None,
                   None, [1])
        sb.execute()
        torch.cuda.synchronize()
        held += sb.local
        sb.close()
    assert sorted(held) == list(range(len(probs)))
    whole = engine.Batch(engine.Options(tol=tol), torch.float32, num_streams=2)
    wouts = []
    for p in probs:
        loc, inp, out = device_buffers(torch, dtype, p)
        whole.add(p["type"], p["sign"], loc, p["modes"], inp, out, col_strides(p["modes"]))
        wouts.append(out)
    whole.execute()
    torch.cuda.synchronize()
    for i, p in enumerate(probs):
        got = outs[i].cpu().numpy()
        ref = direct(oracle, p)
        assert oracle.rel_l2(got, ref) <= 10 * tol
        w = wouts[i].cpu().numpy()
        assert np.linalg.norm(got - w) <= 1e-5 * np.linalg.norm(w)
    whole.close()
