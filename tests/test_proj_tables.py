"""Host-side invariants of the projector tables the H kernels index by (tile
segments, plane-local accumulators, point order inside each tile, per-tile point
index, atom-major chunks), for the 24^3, 32^3, 40^3 and 64^3 diamond cells.  Runs
on the CPU: the tables are built by the library's host code."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "proj_tables_check.cpp")
LIBDIR = os.path.join(ROOT, "inq-wannier-fork_b200", "lib")


def test_projector_table_invariants(pb, tmp_path):
    exe = os.path.join(str(tmp_path), "proj_tables_check")
    cmd = ["g++", "-std=c++17", "-O1", SRC, "-I/usr/local/cuda/include", "-L" + LIBDIR, "-linqb200",
           "-L/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 4 and all(line.endswith("bad=0") for line in lines), r.stdout
