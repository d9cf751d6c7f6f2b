"""The C++ drop-in (include/bulbit_gpu.hpp): a program built on the
reference library swaps BVH -> GpuBVH and PathIntegrator ->
GpuPathIntegrator and keeps its Intersect / IntersectAny / Render / Film
calls. tests/cpp/dropin_test.cpp builds two scenes with the reference's
Scene API (the README sphere with spot and sky light; two meshes with
Lambertian, gold conductor, glass and a ceiling area light) and compares:
the same primitive and intersection record from GpuBVH::Intersect as from
BVH::Intersect, the same IntersectAny answers, IntersectBatch hits, and the
Film left by GpuPathIntegrator::Render against PathIntegrator::Render
(image means within 1e-3 relative, 99.5 % of pixels within 1e-3)."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BINARY = os.path.join(ROOT, "oracle", "_ref", "dropin_test")


@pytest.mark.gpu
def test_dropin_matches_reference_classes():
    if not os.path.exists(BINARY):
        pytest.fail(f"{BINARY} not built (make -C oracle)")
    p = subprocess.run([BINARY], capture_output=True, text=True, timeout=600)
    line = p.stdout.strip().splitlines()[-1] if p.stdout.strip() else "{}"
    print(line)
    res = json.loads(line)
    assert "error" not in res, res
    for key, v in res.items():
        if key.endswith("_ok"):
            assert v == 1, (key, res)
    assert p.returncode == 0 and res.get("ok") == 1


def test_dropin_program_is_built():
    """The drop-in compiles against the reference headers (oracle/Makefile)."""
    assert os.path.exists(BINARY)
