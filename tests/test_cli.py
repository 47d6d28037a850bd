"""The `output` command line (drop-in for the reference's ./output <args>)."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
from vcgpu import workloads as W

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(REPO, "parallel-vertex-cover-algorithms-on-gpus_b200", "output")
needs_cli = pytest.mark.skipif(not os.path.exists(CLI), reason="output not built")


def run(args, cwd):
    return subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True, timeout=120)


@needs_cli
def test_help_and_bad_options(tmp_path):
    r = run(["-h"], tmp_path)
    assert r.returncode == 0 and "-v <Version>" in r.stderr
    r = run(["-x"], tmp_path)
    assert r.returncode == 0 and "Unrecognized option" in r.stderr
    r = run(["-v", "fast"], tmp_path)
    assert r.returncode == 0 and "Unrecognized -v option" in r.stderr
    r = run(["-i", "mis"], tmp_path)
    assert r.returncode == 0 and "Unrecognized -i option" in r.stderr


@needs_cli
def test_sequential_refused(tmp_path):
    r = run(["-v", "sequential", "-f", "x.txt"], tmp_path)
    assert r.returncode == 1 and "not part of this build" in r.stderr


@needs_cli
@pytest.mark.parametrize("body,msg", [("3 1\n1 1\n", "self-loop"), ("3 2\n1 2\n2 1\n", "duplicate"),
                                      ("3 1\n0 2\n", "out of range"), ("3 2\n1 2\n", "fewer edges"),
                                      ("", "header")])
def test_malformed_files(tmp_path, body, msg):
    p = tmp_path / "g.txt"
    p.write_text(body)
    r = run(["-f", str(p)], tmp_path)
    assert r.returncode == 1 and msg in r.stderr


@needs_cli
@pytest.mark.parametrize("body", ["3 1\n0 3\n", "3 2\n0 1\n1 1\n"])
def test_zero_based_mode_checks(tmp_path, body):
    """-z reads 0-based ids (the formated_* inputs); id n is out of range there,
    and the other checks still apply."""
    p = tmp_path / "g0.txt"
    p.write_text(body)
    r = run(["-z", "-f", str(p)], tmp_path)
    assert r.returncode == 1 and ("out of range" in r.stderr or "self-loop" in r.stderr)


@needs_cli
@pytest.mark.gpu
def test_cli_solves_and_writes_results_row(tmp_path):
    g = W.config1_graph()
    p = tmp_path / "g60.txt"
    W.write_reference_file(g, str(p))
    opt = O.mvc(g)[1]
    r = run(["-f", str(p), "-o", "run7"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert f"Size of minimum vertex cover: {opt}" in r.stdout
    r = run(["-f", str(p), "-o", "run8", "-i", "pvc", "-k", str(opt - 1)], tmp_path)
    assert r.returncode == 0 and f"Minimum is greater than K: {opt - 1}" in r.stdout
    r = run(["-f", str(p), "-o", "run9", "-i", "pvc", "-k", str(opt)], tmp_path)
    assert f"Minimum is less than or equal to K: {opt}" in r.stdout
    rows = (tmp_path / "Results" / "Results.csv").read_text().strip().splitlines()
    assert len(rows) == 3
    f = rows[0].split(",")
    assert len(f) == 22
    assert f[0] == "run7" and f[2] == "60" and f[3] == str(g.m) and f[4] == "mvc" and f[5] == "hybrid"
    assert f[6] == str(1 << 19) and f[18] == str(opt)
    assert rows[1].split(",")[20] == "0" and rows[2].split(",")[20] == "1"


@pytest.mark.gpu
def test_cli_counters_files(tmp_path):
    """VC_COUNTERS=1 writes the reference's NODES_PER_SM file (SM_1..SM_n header,
    tree nodes per SM) and a per-search-unit Counters file."""
    g = W.config1_graph()
    p = tmp_path / "g60.txt"
    W.write_reference_file(g, str(p))
    env = dict(os.environ, VC_COUNTERS="1")
    r = subprocess.run([CLI, "-f", str(p), "-o", "c1"], cwd=tmp_path, capture_output=True, text=True, env=env,
                       timeout=120)
    assert r.returncode == 0, r.stderr
    nodes = (tmp_path / "NODES_PER_SM" / "NODES_PER_SM_c1_g60.txt").read_text().splitlines()
    hdr, vals = nodes[0].split(","), [int(x) for x in nodes[1].split(",")]
    assert hdr[0] == "SM_1" and len(hdr) == len(vals) and len(hdr) >= 100
    cnt = (tmp_path / "Counters" / "Counters_c1_g60.txt").read_text().splitlines()
    assert cnt[0].startswith("SU_NO,NODES,")
    su_nodes = sum(int(l.split(",")[1]) for l in cnt[1:])
    assert su_nodes == sum(vals) > 0


@needs_cli
@pytest.mark.gpu
def test_cli_zero_based_file_same_answer(tmp_path):
    """A graph written with 0-based ids and read with -z gives the same cover
    size as the 1-based file."""
    g = W.config1_graph()
    p1 = tmp_path / "g1.txt"
    W.write_reference_file(g, str(p1))
    lines = p1.read_text().strip().splitlines()
    p0 = tmp_path / "g0.txt"
    p0.write_text("\n".join([lines[0]] + [" ".join(str(int(x) - 1) for x in l.split()) for l in lines[1:]]) + "\n")
    opt = O.mvc(g)[1]
    r = run(["-z", "-f", str(p0)], tmp_path)
    assert r.returncode == 0, r.stderr
    assert f"Size of minimum vertex cover: {opt}" in r.stdout


@needs_cli
@pytest.mark.gpu
def test_cli_upper_bounds(tmp_path):
    """-u runs both of the reference's upper-bound heuristics on the GPU, prints
    their lines and fills the Results.csv fields the fork leaves at zero."""
    g = W.config1_graph()
    p = tmp_path / "g60.txt"
    W.write_reference_file(g, str(p))
    r = run(["-u", "-f", str(p), "-o", "u1"], tmp_path)
    assert r.returncode == 0, r.stderr
    want = O.remove_max_ub(g)[0]
    assert f"Approximate Remove Max Minimum is: {want}" in r.stdout
    edge = int(r.stdout.split("Approximate Remove Edge Minimum is: ")[1].split()[0])
    assert edge >= O.mvc(g)[1]
    f = (tmp_path / "Results" / "Results.csv").read_text().strip().splitlines()[-1].split(",")
    assert f[14] == str(want) and f[16] == str(edge)


@needs_cli
@pytest.mark.gpu
def test_cli_stack_only_version(tmp_path):
    """-v stackonly (the reference's LocalStacks kernels, main.cu:306-308,340-342)
    runs the same exact search: the same MVC size and PVC verdicts, with the
    version field of the Results.csv row reading stackonly."""
    g = W.config1_graph()
    p = tmp_path / "g60.txt"
    W.write_reference_file(g, str(p))
    opt = O.mvc(g)[1]
    r = run(["-v", "stackonly", "-d", "4", "-f", str(p), "-o", "s1"], tmp_path)
    assert r.returncode == 0, r.stderr
    assert f"Size of minimum vertex cover: {opt}" in r.stdout
    r = run(["-v", "stackonly", "-i", "pvc", "-k", str(opt - 1), "-f", str(p), "-o", "s2"], tmp_path)
    assert r.returncode == 0 and f"Minimum is greater than K: {opt - 1}" in r.stdout
    r = run(["-v", "stackonly", "-i", "pvc", "-k", str(opt), "-f", str(p), "-o", "s3"], tmp_path)
    assert r.returncode == 0 and f"Minimum is less than or equal to K: {opt}" in r.stdout
    rows = (tmp_path / "Results" / "Results.csv").read_text().strip().splitlines()
    assert [row.split(",")[5] for row in rows] == ["stackonly"] * 3
    assert rows[0].split(",")[18] == str(opt)
