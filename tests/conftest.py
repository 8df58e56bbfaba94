import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")

# FP32 device results against the FP64 oracle: relative L1 and max-abs bounds
# (PageRank: relative L1 <= 1e-5 and max abs <= 1e-6).
PR_REL_L1 = 1e-5
PR_MAX_ABS = 1e-6


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")


def golden_names():
    """Golden graphs with app outputs (partition sizes and VEBO orders have their own fixtures)."""
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz") and f not in ("partitions.npz", "partitions_src.npz", "vebo.npz", "adjoint_fd_rmat22.npz"))


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return {k: z[k] for k in z.files}


def host_graph_from_golden(gd):
    import graphgrind_b200 as gg
    return gg.HostGraph.from_csr(gd["offsets"], gd["indices"], gd.get("weights"), symmetric=bool(gd["symmetric"]))


def golden_flags(gd):
    return str(gd["flags"]).split()


def golden_partitions(gd):
    fl = golden_flags(gd)
    return int(fl[fl.index("-c") + 1]) if "-c" in fl else 384


def ok_partitions(hg, preferred):
    """Largest P <= preferred that the reference partitioner accepts for hg
    (partitionByDegree asserts for some (graph, P) pairs)."""
    import graphgrind_b200 as gg
    outd = hg.degrees()
    ind = hg.transpose().degrees() if not hg.symmetric else outd
    for P in range(preferred, 0, -1):
        try:
            gg.partition_sizes(ind, outd, hg.m, P)
            return P
        except gg.GGError:
            continue
    raise AssertionError("no partition count accepted")


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).sum() / max(np.abs(b).sum(), 1e-300))


@pytest.fixture(scope="session")
def gg():
    import graphgrind_b200
    return graphgrind_b200


@pytest.fixture(scope="session")
def orc():
    import oracle
    return oracle
