"""The persistent batch launch's work list and queue protocol, on the CPU: counter
targets, backward-only waits, and simulated execution by 1-64 CTAs with random
interleavings (no deadlock, every item after its inputs), plus the stall that one
unreachable wait causes.  Links libinqb200 for build_batch_items."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "batch_plan_check.cpp")
LIBDIR = os.path.join(ROOT, "inq-wannier-fork_b200", "lib")


def test_batch_plan_protocol(pb, tmp_path):
    exe = os.path.join(str(tmp_path), "batch_plan_check")
    cmd = ["g++", "-std=c++17", "-O2", SRC, "-I/usr/local/cuda/include", "-L" + LIBDIR, "-linqb200",
           "-L/usr/local/cuda/lib64", "-lcudart", "-Wl,-rpath," + LIBDIR, "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("bad=0"), r.stdout
