"""The CLI route to the GPU integrator: the reference CLI's scene -> BVH ->
Integrator::Create -> Render -> image sequence (cli/main.cpp:191-297) with
GpuBVH and CreateGpuIntegrator (IntegratorType::path -> GpuPathIntegrator,
src/integrator/integrator.cpp:16-31), over the CLI's own built-in sample
scenes (Sample::Get, cli/samples.h). bulbit_b200/cpp/bbcli_gpu.cpp is that
program; oracle/harness/cli_ref.cpp renders the same sample through the
reference's BVH and PathIntegrator.

Bar, cornell-box (stratified sampler, Gaussian filter, 64 bounces): the same
sampler streams, so pixels agree to within 1e-3 relative except where a path
diverged (at least 97 % of pixels), image means within 0.5 %, and every 10x10
block of the difference image within 5 standard errors of zero. A tree other
than the reference's (linear BVH built on the device) changes only which of
two equal-t hits is taken: the same statistical bar."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BBCLI = os.path.join(ROOT, "oracle", "_ref", "bbcli_gpu")
CLIREF = os.path.join(ROOT, "oracle", "_ref", "cli_ref")


def read_pfm(path):
    with open(path, "rb") as f:
        data = f.read()
    magic, dims, scale, body = data.split(b"\n", 3)
    assert magic == b"PF" and float(scale) < 0
    w, h = map(int, dims.split())
    img = np.frombuffer(body, dtype="<f4", count=w * h * 3).reshape(h, w, 3)
    return img[::-1].astype(np.float64)  # top row first


def run(args, timeout=600):
    return subprocess.run(args, capture_output=True, text=True, timeout=timeout)


def need(binary):
    if not os.path.exists(binary):
        pytest.fail(f"{binary} not built (make -C oracle)")


def block_z(diff, block=10):
    h, w, _ = diff.shape
    zs = []
    for y in range(0, h - block + 1, block):
        for x in range(0, w - block + 1, block):
            d = diff[y:y + block, x:x + block].reshape(-1)
            sd = d.std(ddof=1)
            if sd > 0:
                zs.append(abs(d.mean()) / (sd / np.sqrt(d.size)))
    return np.array(zs)


def test_cli_lists_samples_and_reports_xml():
    need(BBCLI)
    p = run([BBCLI, "--list-samples"])
    assert p.returncode == 0 and "cornell-box" in p.stdout.split()
    p = run([BBCLI, "--help"])
    assert p.returncode == 0 and "-s <samples_per_pixel>" in p.stdout
    p = run([BBCLI, "scene.xml"])
    assert p.returncode == 1 and "XML scenes need the CLI's scene loader" in p.stderr
    p = run([BBCLI, "no-such-sample"])
    assert p.returncode == 1 and "Failed to load scene or sample" in p.stderr
    p = run([BBCLI, "-s"])
    assert p.returncode == 1 and "needs a value" in p.stderr


@pytest.fixture(scope="module")
def cornell_ref(tmp_path_factory):
    need(CLIREF)
    out = str(tmp_path_factory.mktemp("cli") / "ref.pfm")
    p = run([CLIREF, "-r", "0.2", "-s", "16", "-o", out, "cornell-box"])
    assert p.returncode == 0, p.stderr
    return read_pfm(out)


@pytest.mark.gpu
@pytest.mark.parametrize("tree", ["reference", "device"])
def test_cli_cornell_box_matches_reference(tmp_path, cornell_ref, tree):
    need(BBCLI)
    out = str(tmp_path / "gpu.pfm")
    p = run([BBCLI, "-r", "0.2", "-s", "16", "--tree", tree, "-o", out, "cornell-box"])
    print(p.stdout[-600:])
    assert p.returncode == 0, p.stderr
    gpu, ref = read_pfm(out), cornell_ref
    assert gpu.shape == ref.shape == (100, 100, 3)
    assert np.isfinite(gpu).all()
    rel_mean = np.abs(gpu.mean(axis=(0, 1)) - ref.mean(axis=(0, 1))) / ref.mean(axis=(0, 1))
    assert (rel_mean < 5e-3).all(), rel_mean
    z = block_z(gpu - ref)
    assert z.size > 50 and z.max() < 5.0, z.max()
    if tree == "reference":
        rel = np.abs(gpu - ref).max(axis=2) / np.maximum(np.abs(ref).max(axis=2), 1e-3)
        assert (rel < 1e-3).mean() >= 0.97, (rel < 1e-3).mean()


@pytest.mark.gpu
def test_cli_rejects_integrators_without_gpu_implementation(tmp_path):
    need(BBCLI)
    p = run([BBCLI, "-r", "0.1", "-s", "1", "-i", "1", "-o", str(tmp_path / "x.pfm"), "cornell-box"])
    assert p.returncode == 1 and "has no GPU implementation" in p.stderr
    assert not (tmp_path / "x.pfm").exists()


@pytest.mark.gpu
def test_cli_writes_radiance_hdr(tmp_path):
    need(BBCLI)
    out = tmp_path / "img.png"
    p = run([BBCLI, "-r", "0.1", "-s", "4", "-o", str(out), "cornell-box"])
    assert p.returncode == 0, p.stderr
    hdr = tmp_path / "img.hdr"
    assert "saving as .hdr" in p.stdout and hdr.exists()
    data = hdr.read_bytes()
    head, body = data.split(b"\n\n", 1)
    assert head.startswith(b"#?RADIANCE")
    res, pixels = body.split(b"\n", 1)
    assert res == b"-Y 50 +X 50" and len(pixels) == 50 * 50 * 4
