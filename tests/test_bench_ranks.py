"""The multi-replica path of bench.py on CPU: two gloo ranks aggregate like
the NCCL ranks of a multi-GPU run (max of the times, sum of the edges and
launches), and the reference arm's non-zero ranks exit without work."""
import os
import socket
import subprocess
import sys
import tempfile

import pytest

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    dist.barrier()
    res = bench.aggregate_ranks(dist, 10.0 + rank, 1.0 + 2 * rank, 1000 * (rank + 1), 5 + rank, device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
        f.write(repr(res))


def test_two_rank_aggregation():
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank, args=(2, _free_port(), d), nprocs=2, start_method="spawn", join=True)
        for r in range(2):
            dev_ms, wall_s, edges, launches = eval(open(os.path.join(d, f"r{r}.txt")).read())
            assert (dev_ms, wall_s, edges, launches) == (11.0, 3.0, 3000.0, 11)


def test_single_process_aggregation_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate_ranks(None, 2.5, 3.5, 7, 4) == (2.5, 3.5, 7.0, 4)


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=300)
    assert p.returncode == 0 and p.stdout.strip() == ""


def test_reference_arm_loads_only_the_oracle():
    """The reference arm builds its graph with the oracle's generator and times
    the reference's own build: the process maps no library of the product, and
    its line carries the GPU arm's config block."""
    import oracle
    if not all(oracle.ref_available(a) for a in ("BFS", "PR", "SPMV")):
        pytest.skip("reference binaries not built here")
    code = ("import json, sys; sys.argv = ['bench.py', '--impl', 'reference', '--scale', '10', '--partitions', '4', "
            "'--steps', '1', '--warmup', '1', '--no-one-thread']; sys.path.insert(0, %r); import bench; bench.main(); "
            "maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'module': 'graphgrind_b200' in sys.modules, 'libgg': 'libgg.so' in maps}))" % ROOT)
    env = dict(os.environ, OMP_NUM_THREADS="2")
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    import json
    line, probe = [json.loads(x) for x in p.stdout.strip().splitlines()[-2:]]
    assert probe == {"module": False, "libgg": False}
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"]["n"] == 1024 and line["config"]["partitions"] == 4
    assert line["reference_detail"]["edges"]["SPMV"] == line["config"]["m"]
