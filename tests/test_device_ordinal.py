"""Handles run on the device that was current when they were created: the
library sets no fixed device and queries no fixed device ordinal. Checked on
the sources (this runs without a GPU; more than one GPU is not available to
the tests): every cudaSetDevice goes through the scope guard that restores
the caller's device, and device attributes are asked of the current device."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SOURCES = [os.path.join(ROOT, "bulbit_b200", "csrc", f) for f in os.listdir(os.path.join(ROOT, "bulbit_b200", "csrc"))
           if f.endswith((".cu", ".cuh", ".cpp", ".h"))] + \
          [os.path.join(ROOT, "bulbit_b200", "cpp", f) for f in os.listdir(os.path.join(ROOT, "bulbit_b200", "cpp"))
           if f.endswith((".cpp", ".h", ".hpp"))]


def code_of(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return re.sub(r"//[^\n]*", "", text)


def test_no_fixed_device_ordinal():
    offenders = []
    for p in SOURCES:
        code = code_of(p)
        for pat in (r"cudaSetDevice\s*\(\s*\d+\s*\)", r"cudaGetDeviceProperties\s*\([^,]*,\s*\d+\s*\)",
                    r"cudaDeviceGetAttribute\s*\([^;]*,\s*\d+\s*\)\s*;"):
            for m in re.finditer(pat, code):
                offenders.append((os.path.basename(p), m.group(0)))
    assert not offenders, offenders


def test_set_device_only_in_the_scope_guard():
    where = []
    for p in SOURCES:
        if re.search(r"\bcudaSetDevice\s*\(", code_of(p)):
            where.append(os.path.basename(p))
    assert where == ["cuda_util.cuh"], where


def test_handles_record_their_device():
    csrc = os.path.join(ROOT, "bulbit_b200", "csrc")
    accel = code_of(os.path.join(csrc, "accel.cu"))
    assert "cudaGetDevice(&a->device)" in accel
    assert len(re.findall(r"DeviceScope ds\(a->device\)", accel)) >= 3
    render = code_of(os.path.join(csrc, "render.cu"))
    assert "I->device = accel->device" in render
    assert len(re.findall(r"DeviceScope ds\((I|B)->device\)", render)) >= 6
    guide = code_of(os.path.join(csrc, "guide.cu"))
    assert "cudaGetDevice(&G->device)" in guide
    assert len(re.findall(r"DeviceScope ds\(G->device\)", guide)) >= 5
    assert "DeviceScope ds(accel->device)" in code_of(os.path.join(csrc, "noalloc.cu"))
