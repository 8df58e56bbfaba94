"""gg_run, the parallel_main replacement: flags, output format and errors."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GG_RUN = os.path.join(ROOT, "graphgrind_b200", "gg_run")


def run(*args):
    return subprocess.run([GG_RUN, *args], capture_output=True, text=True, timeout=300)


def test_cli_rejects_bad_flags_like_the_reference(tmp_path):
    assert os.path.exists(GG_RUN), "build with make -C graphgrind_b200"
    r = run("BFS")
    assert r.returncode == 1 and "usage" in r.stderr
    r = run("BFS", "-P", "sideways", str(tmp_path / "g.adj"))
    assert r.returncode == 1 and 'Illegal value for -P: "sideways"' in r.stderr
    r = run("BFS", "-v", "both", str(tmp_path / "g.adj"))
    assert r.returncode == 1 and 'Illegal value for -v: "both"' in r.stderr
    r = run("BFS", str(tmp_path / "missing.adj"))
    assert r.returncode == 1


@pytest.mark.gpu
@pytest.mark.parametrize("app", ["BFS", "BC", "Components", "PageRank", "PageRankBit", "PageRankDelta",
                                 "PageRankConverage", "SPMV", "BellmanFord", "BP"])
def test_cli_runs_every_app(gg, tmp_path, app):
    hg = gg.HostGraph.rmat(10, 8, seed=3, symmetric=True)
    weighted = app in ("BellmanFord", "SPMV")
    if weighted:
        hg.add_weights(gg.W_INT32, seed=1, lo=1, hi=100)
    path = str(tmp_path / "g.gr")
    hg.write_gr(path)
    r = run(app, "-s", "-b", "-rounds", "2", "-c", "8", "-r", "5", path)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    assert [ln.split(" : ")[0] for ln in lines] == ["Running", "Running", "Average"]
    assert all(float(ln.split(" : ")[1]) >= 0 for ln in lines)
