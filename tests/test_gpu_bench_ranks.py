"""bench.py under torchrun: the rank exchange (NCCL process group, barriers,
max-over-ranks timing, the rank-order sum of the accumulators in the
end-to-end step) runs even with one rank, so this one-GPU test walks the code
path that several GPUs take.  Small job: the single-axon workload at 65536
walkers x 1000 steps."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("workload", ["single", "batch"])
def test_bench_one_rank_under_torchrun(workload):
    extra = ["--walkers", "65536", "--tn", "1000"] if workload == "single" else ["--walkers", "200000", "--tn", "400",
                                                                                  "--timepoints", "20"]
    cmd = ["timeout", "-k", "30", "600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           "--nproc-per-node", "1", "--master-addr", "127.0.0.1", "--master-port", "29517", "bench.py",
           "--gpus", "1", "--workload", workload, "--steps", "1", "--warmup", "1", "--no-cpu-baseline",
           "--no-error", "--no-reference-cuda", "--plain-steps", "0"] + extra
    env = dict(os.environ, NCCL_NVLS_ENABLE="0")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert lines, r.stdout[-2000:]
    d = json.loads(lines[-1])
    assert d["n_gpus"] == 1 and d["value"] > 0 and d["e2e"]["value"] > 0
    assert d["e2e"]["d2h_bytes_per_step"] > 0
