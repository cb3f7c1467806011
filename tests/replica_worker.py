"""One rank of the multi-process replica tests (tests/test_replicas_cpu.py), launched by
torch.distributed.run exactly as bench.py is for N > 1, but on CPU with the gloo backend.

    replica_worker.py ok <out_dir>       host-side replica logic; writes rank<r>.json
    replica_worker.py raise <out_dir>    rank 1 raises before the barrier that rank 0 waits in
    replica_worker.py shard <out_dir>    one batch of transforms split over the ranks
                                         (ShardedBatch's owner rule); each rank runs its share
                                         on the CPU oracle as a stand-in for its GPU, and rank 0
                                         gathers every result; writes rank<r>.json
"""
import datetime
import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def main():
    mode, out_dir = sys.argv[1], Path(sys.argv[2])
    import numpy as np
    import torch
    import torch.distributed as dist
    from neonufft_b200 import replicas

    env = replicas.rank_env()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=20))
    assert dist.get_world_size() == env.world and dist.get_rank() == env.rank

    if mode == "shard":
        return shard(env, out_dir)

    if mode == "raise":
        if env.rank == 1:
            raise RuntimeError("rank 1 fails between steps")
        replicas.barrier()
        return 0

    # every rank draws its own point set from its own seed
    seed = replicas.rank_seed(1234, env.rank)
    x = np.random.default_rng(seed).uniform(-np.pi, np.pi, 1000)
    seeds = [None] * env.world
    dist.all_gather_object(seeds, seed)
    first = [None] * env.world
    dist.all_gather_object(first, float(x[0]))

    # ranks time different durations; the job's step time is the slowest rank's
    local_ms = 10.0 + 5.0 * env.rank
    replicas.barrier()
    job_ms = replicas.max_over_ranks(local_ms)
    value = replicas.job_throughput(env.world, 1000, job_ms)
    rec = {"rank": env.rank, "world": env.world, "seeds": seeds, "first": first,
           "local_ms": local_ms, "job_ms": job_ms, "value": value}
    (out_dir / f"rank{env.rank}.json").write_text(json.dumps(rec))
    replicas.barrier()
    dist.destroy_process_group()
    return 0


def batch_specs(n=14, seed=5):
    """The same list of small independent type-1 transforms on every rank."""
    import numpy as np
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n):
        dim = 2 if i % 2 == 0 else 3
        M = int(rng.integers(50, 400))
        modes = [int(rng.choice([6, 8, 10]))] * dim
        x = [rng.uniform(-np.pi, np.pi, M) for _ in range(dim)]
        c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
        specs.append(dict(dim=dim, M=M, modes=modes, x=x, c=c))
    return specs


def run_transform(spec):
    from oracle import oracle as O
    return O.direct_type1(-1, spec["x"], spec["c"], spec["modes"]).reshape(-1)


def shard(env, out_dir):
    import json
    import numpy as np
    import torch.distributed as dist
    from neonufft_b200 import replicas

    specs = batch_specs()
    costs = [replicas.transform_cost(s["dim"], s["M"], s["modes"]) for s in specs]
    owners = replicas.shard_owners(costs, env.world)
    mine = [i for i, r in enumerate(owners) if r == env.rank]
    results = {i: run_transform(specs[i]) for i in mine}  # this rank's share only
    gathered = [None] * env.world
    dist.all_gather_object(gathered, {"rank": env.rank, "owners": owners,
                                      "ran": sorted(results),
                                      "res": {i: (v.real.tolist(), v.imag.tolist())
                                              for i, v in results.items()}})
    rec = {"rank": env.rank, "world": env.world, "owners": owners, "ran": sorted(results),
           "loads": replicas.shard_loads(costs, owners, env.world), "costs": costs}
    if env.rank == 0:
        counts = [0] * len(specs)
        union = {}
        for g in gathered:
            assert g["owners"] == owners  # the same assignment on every rank
            for i in g["ran"]:
                counts[i] += 1
            for i, (re, im) in g["res"].items():
                union[int(i)] = np.array(re) + 1j * np.array(im)
        serial = [run_transform(s) for s in specs]  # one process runs the whole batch
        rec["counts"] = counts
        rec["max_abs_diff"] = max(float(np.max(np.abs(union[i] - serial[i])))
                                  for i in range(len(specs)))
    (out_dir / f"rank{env.rank}.json").write_text(json.dumps(rec))
    replicas.barrier()
    dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
