"""One rank of the multi-process replica tests (tests/test_replicas_cpu.py), launched by
torch.distributed.run exactly as bench.py is for N > 1, but on CPU with the gloo backend.

    replica_worker.py ok <out_dir>       host-side replica logic; writes rank<r>.json
    replica_worker.py raise <out_dir>    rank 1 raises before the barrier that rank 0 waits in
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


if __name__ == "__main__":
    sys.exit(main())
