"""Batched execution of uneven transforms (nnb_batch_*) on the GPU.

A batch of 2D and 3D, type-1 and type-2 transforms with uneven point counts, grid sizes and
point distributions (uniform and Gaussian blobs) must give, in each of its three modes (serial,
concurrent streams, captured CUDA graph), the results of the same transforms run one at a time
through single plans, and meet the tolerance against the FP64 direct sum. A replayed graph must
pick up new data written into the same input buffers.
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
    for mode in (engine.Batch.SERIAL, engine.Batch.STREAMS, engine.Batch.GRAPH, engine.Batch.GRAPH):
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


def test_batch_graph_replays_new_inputs(cuda, engine, oracle):
    torch = cuda
    rng = np.random.default_rng(5)
    probs = make_problems(rng, "float32", 6)
    batch = engine.Batch(engine.Options(tol=1e-6), torch.float32, num_streams=2)
    bufs = []
    for p in probs:
        loc, inp, out = device_buffers(torch, "float32", p)
        batch.add(p["type"], p["sign"], loc, p["modes"], inp, out, col_strides(p["modes"]))
        bufs.append((inp, out))
    batch.execute(engine.Batch.GRAPH)
    for p, (inp, out) in zip(probs, bufs):
        p["inp"] = rng.standard_normal(inp.numel()) + 1j * rng.standard_normal(inp.numel())
        inp.copy_(torch.from_numpy(p["inp"].astype(np.complex64)))
    batch.execute(engine.Batch.GRAPH)
    torch.cuda.synchronize()
    for p, (inp, out) in zip(probs, bufs):
        assert oracle.rel_l2(out.cpu().numpy(), direct(oracle, p)) < 2e-5
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
    with pytest.raises(engine.InputError):
        engine.Batch(engine.Options(tol=1e-6), torch.float32, num_streams=0)
    batch.execute(engine.Batch.GRAPH)  # empty batch: nothing to do
    batch.close()
