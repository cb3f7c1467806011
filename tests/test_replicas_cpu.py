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
