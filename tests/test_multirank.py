"""The multi-rank path of bench.py on the host: two ranks over gloo (world size 2), as
torchrun launches them.  The GPU arm runs replicas (each rank the whole grid on its own
GPU, no data-path collective); what it shares with the ranks is the start barrier and the
max-over-ranks timing, checked here, and the reference arm, which rank 0 alone runs."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _env():
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", MASTER_ADDR="127.0.0.1", OMP_NUM_THREADS="2")
    env["PYTHONPATH"] = str(ROOT) + os.pathsep + env.get("PYTHONPATH", "")
    return env


def _worker(rank, port, out):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import bench
    world, r, _ = bench.dist_setup()
    bench.barrier(world)
    m = bench.allreduce_max(10.0 + r, world)  # rank 1 is the slow one
    bench.barrier(world)
    import torch.distributed as dist
    backend = dist.get_backend()
    dist.destroy_process_group()
    Path(out, f"rank{r}.json").write_text(json.dumps({"world": world, "max": m, "backend": backend}))


def test_max_over_ranks_gloo(tmp_path):
    import torch.multiprocessing as mp
    os.environ["CUDA_VISIBLE_DEVICES"] = ""
    mp.start_processes(_worker, args=(_port(), str(tmp_path)), nprocs=2, start_method="spawn", join=True)
    for r in (0, 1):
        d = json.loads((tmp_path / f"rank{r}.json").read_text())
        assert d == {"world": 2, "max": 11.0, "backend": "gloo"}


@pytest.mark.timeout(600)
def test_reference_arm_two_ranks(built):
    """`bench.py --impl reference` under torchrun with 2 ranks: rank 0 prints one JSON line,
    rank 1 does no work, both exit 0."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(_port()), "bench.py", "--impl", "reference",
           "--gpus", "2", "--steps", "1", "--warmup", "0", "--glevel", "3", "--kall", "6", "--ref-kall", "4",
           "--ntr", "1"]
    r = subprocess.run(cmd, cwd=ROOT, env=_env(), capture_output=True, text=True, timeout=540)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0


@pytest.mark.timeout(600)
def test_reference_arm_loads_no_library_code(built):
    """The reference arm (and bench.py's cpu_baseline leg) builds its grid from the oracle's own
    topology and halo plan: the process never maps the library under test."""
    code = ("import bench; bench.cpu_reference(3, 6, 2, 1, 0, 2); "
            "print('MAPPED', any('libicoadv' in ln for ln in open('/proc/self/maps')))")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=_env(), capture_output=True, text=True,
                       timeout=540)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "MAPPED False" in r.stdout, r.stdout
