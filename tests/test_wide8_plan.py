"""The surface-area plan that chooses the 8-wide nodes (Wide8PlanNode and
Wide8Gather, bulbit_b200/csrc/wide8_build.cuh, run by the host and the device
collapse alike) against brute force on the CPU: tests/cpp/wide8_plan_test.cpp,
compiled here against the built library (for bbg_bvh_build, the reference's
SAH build), checks on 240 trees of 1 to 40 random boxes that the plan's cost
is the least summed surface area of wide nodes over every valid collapse,
that the collapse it gathers has that cost, and that every leaf is reached
exactly once."""
import os
import shutil
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "bulbit_b200")
SRC = os.path.join(ROOT, "tests", "cpp", "wide8_plan_test.cpp")


def test_wide8_plan_is_the_least_surface_area_collapse(tmp_path):
    assert os.path.exists(os.path.join(LIBDIR, "libbulbit_b200.so")), "build the library first"
    cuda_include = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    exe = str(tmp_path / "wide8_plan_test")
    cmd = [shutil.which("g++") or "g++", "-std=c++20", "-O2", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(LIBDIR, "csrc"), "-I", cuda_include, "-o", exe, SRC,
           "-L", LIBDIR, "-lbulbit_b200", "-Wl,-rpath," + LIBDIR]
    built = subprocess.run(cmd, capture_output=True, text=True)
    assert built.returncode == 0, built.stderr[-2000:]
    p = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(p.stdout[-600:])
    assert p.returncode == 0 and " 0 failures" in p.stdout, p.stdout[-2000:]
