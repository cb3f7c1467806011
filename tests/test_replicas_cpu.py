"""Multi-GPU replica path, host side, as world_size-2 gloo ranks on CPU. bench.py --gpus N runs N
independent replicas (each rank its own point set; no data-path collective), times each rank
between barriers and reports the whole job's throughput over the slowest rank's time. These
tests launch tests/replica_worker.py through torch.distributed.run on 127.0.0.1, as bench.py is
launched, and check the helpers of neonufft_b200.replicas and a rank failing between steps.
"""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
WORKER = ROOT / "tests" / "replica_worker.py"


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _launch(mode, out_dir, nproc=2, timeout=180):
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={nproc}", "--master-addr", "127.0.0.1",
           "--master-port", str(_free_port()), str(WORKER), mode, str(out_dir)]
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="1")
    return subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env)


def test_replica_helpers_single_process():
    from neonufft_b200 import replicas
    assert replicas.max_over_ranks(3.5) == 3.5
    replicas.barrier()  # no group: nothing to wait for
    assert replicas.rank_seed(7, 0) == 7 and replicas.rank_seed(7, 1) != 7
    assert replicas.job_throughput(4, 1e6, 2.0) == pytest.approx(2e9)
    with pytest.raises(ValueError):
        replicas.job_throughput(1, 1e6, 0.0)


def test_two_ranks_gloo(tmp_path):
    r = _launch("ok", tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    recs = [json.loads((tmp_path / f"rank{i}.json").read_text()) for i in range(2)]
    for i, rec in enumerate(recs):
        assert rec["rank"] == i and rec["world"] == 2
        # distinct point sets per rank
        assert len(set(rec["seeds"])) == 2 and rec["first"][0] != rec["first"][1]
        # the job's step time is the slowest rank's, the same on every rank
        assert rec["job_ms"] == pytest.approx(15.0)
        # whole-job throughput: 2 ranks x 1000 points in 15 ms
        assert rec["value"] == pytest.approx(2 * 1000 / 15e-3)


def test_rank_failure_ends_the_job(tmp_path):
    """A rank that raises between steps ends the whole job with an error, within the launch's
    bound, instead of leaving the other rank waiting in its barrier."""
    r = _launch("raise", tmp_path, timeout=150)
    assert r.returncode != 0
    assert "rank 1 fails between steps" in (r.stdout + r.stderr)


def test_shard_owners_balanced_and_deterministic():
    from neonufft_b200 import replicas
    costs = [5.0, 1.0, 4.0, 4.0, 3.0, 3.0, 2.0, 2.0, 9.0]
    for world in (1, 2, 3, 4):
        owners = replicas.shard_owners(costs, world)
        assert owners == replicas.shard_owners(list(costs), world)
        assert sorted(set(owners)) == list(range(min(world, len(costs))))
        loads = replicas.shard_loads(costs, owners, world)
        assert sum(loads) == pytest.approx(sum(costs))
        # longest-processing-time bound: the largest load is at most 4/3 of the optimum,
        # which is at least max(mean load, largest transform)
        assert max(loads) <= 4.0 / 3.0 * max(sum(costs) / world, max(costs)) + 1e-9
    with pytest.raises(ValueError):
        replicas.shard_owners(costs, 0)


def test_transform_cost_follows_work_and_grid():
    from neonufft_b200 import replicas
    a = replicas.transform_cost(3, 10 ** 6, [64] * 3)
    assert replicas.transform_cost(3, 2 * 10 ** 6, [64] * 3) > a
    assert replicas.transform_cost(3, 10 ** 6, [128] * 3) > a
    # FP32 tol 1e-6: w = 7, fine grid 128^3
    cells = 128.0 ** 3
    import math
    assert a == pytest.approx(1e6 * 7 ** 3 + 5 * cells * math.log2(cells))


def test_one_batch_split_over_two_ranks(tmp_path):
    """Each transform of the batch runs on exactly one rank, both ranks compute the same
    assignment, and the union of the ranks' results equals one process running the whole
    batch."""
    r = _launch("shard", tmp_path)
    assert r.returncode == 0, r.stdout + r.stderr
    recs = [json.loads((tmp_path / f"rank{i}.json").read_text()) for i in range(2)]
    assert recs[0]["owners"] == recs[1]["owners"]
    ran0, ran1 = set(recs[0]["ran"]), set(recs[1]["ran"])
    assert not ran0 & ran1 and ran0 | ran1 == set(range(len(recs[0]["owners"])))
    assert recs[0]["counts"] == [1] * len(recs[0]["owners"])
    assert recs[0]["max_abs_diff"] == 0.0
    loads = recs[0]["loads"]
    assert max(loads) <= 4.0 / 3.0 * max(sum(loads) / 2, max(recs[0]["costs"]))
