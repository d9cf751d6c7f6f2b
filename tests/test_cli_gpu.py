"""The CLI route to the GPU integrator: the reference CLI's scene -> BVH ->
Integrator::Create -> Render -> image sequence (cli/main.cpp:191-297) with
GpuBVH and CreateGpuIntegrator (IntegratorType::path -> GpuPathIntegrator,
src/integrator/integrator.cpp:16-31), over the CLI's own built-in sample
scenes (Sample::Get, cli/samples.h) and XML scene files read by the CLI's
scene and model loaders (LoadScene, cli/scene_loader.cpp:2147; LoadModel,
cli/model_loader.cpp:1045) on this project's XML / OBJ / glTF readers
(bulbit_b200/cpp/scene_io). bulbit_b200/cpp/bbcli_gpu.cpp is that program;
oracle/harness/cli_ref.cpp renders the same scene through the reference's
BVH and PathIntegrator.

Bar, for the cornell-box sample (stratified sampler, Gaussian filter, 64
bounces) and the XML scenes under tests/scenes (rectangles, cubes, spheres,
OBJ with MTL materials, .gltf and .glb models; area, point, spot and uniform
environment lights; diffuse, conductor, dielectric and metallic-roughness
materials): the same sampler streams, so pixels agree to within 1e-3
relative except where a path diverged (at least 97 % of pixels), image means
within 0.5 %, and every 10x10 block of the difference image within 5
standard errors of zero. A tree other than the reference's (linear BVH built
on the device) changes only which of two equal-t hits is taken: the same
statistical bar."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BBCLI = os.path.join(ROOT, "oracle", "_ref", "bbcli_gpu")
CLIREF = os.path.join(ROOT, "oracle", "_ref", "cli_ref")
SIO_TEST = os.path.join(ROOT, "oracle", "_ref", "scene_io_test")
SCENES = os.path.join(ROOT, "tests", "scenes")
XML_SCENES = ["cornell.xml", "lights.xml"]


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


def block_z(diff, ref, block=10, rel_floor=1e-3):
    """z of each block's mean difference. The two images draw the same
    sampler streams, so most per-pixel differences are float rounding and a
    block's spread can be far below its size; the spread is therefore taken
    as at least rel_floor of the block's RMS reference value (the per-pixel
    tolerance), so that rounding-level offsets do not read as bias."""
    h, w, _ = diff.shape
    zs = []
    for y in range(0, h - block + 1, block):
        for x in range(0, w - block + 1, block):
            d = diff[y:y + block, x:x + block].reshape(-1)
            r = ref[y:y + block, x:x + block].reshape(-1)
            sd = max(d.std(ddof=1), rel_floor * float(np.sqrt(np.mean(r * r))))
            if sd > 0:
                zs.append(abs(d.mean()) / (sd / np.sqrt(d.size)))
    return np.array(zs)


def test_cli_lists_samples_and_reports_xml():
    need(BBCLI)
    p = run([BBCLI, "--list-samples"])
    assert p.returncode == 0 and "cornell-box" in p.stdout.split()
    p = run([BBCLI, "--help"])
    assert p.returncode == 0 and "-s <samples_per_pixel>" in p.stdout
    p = run([BBCLI, "no-such-scene.xml"])
    assert p.returncode == 1 and "Failed to load scene or sample: no-such-scene.xml" in p.stderr
    assert "File was not found" in p.stderr  # the scene loader's report
    p = run([BBCLI, "no-such-sample"])
    assert p.returncode == 1 and "Failed to load scene or sample" in p.stderr
    p = run([BBCLI, "-s"])
    assert p.returncode == 1 and "needs a value" in p.stderr


def test_scene_file_readers(tmp_path):
    """The XML, OBJ / MTL and glTF / GLB readers on their own
    (tests/cpp/scene_io_test.cpp: DOM, entities, every error status, face
    triangulation and indices, MTL statements, data URIs, .glb chunks,
    reference checks)."""
    need(SIO_TEST)
    p = run([SIO_TEST, str(tmp_path)])
    print(p.stdout[-400:])
    assert p.returncode == 0, p.stdout


def test_model_fixtures_match_their_generator(tmp_path):
    """tests/scenes/models holds exactly what make_models.py writes."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_models", os.path.join(SCENES, "make_models.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.OUT = str(tmp_path)
    mod.main()
    for name in ("pyramid.obj", "pyramid.mtl", "prism.gltf", "prism.glb"):
        with open(os.path.join(SCENES, "models", name), "rb") as f, open(tmp_path / name, "rb") as g:
            assert f.read() == g.read(), name


# Primitives and lights each XML scene makes: cornell.xml has 5 wall and 1
# light rectangles (2 triangles each), a cube (12), a sphere, the OBJ pyramid
# (4 sides + a quad base = 6 triangles; its MTL materials carry an emission
# term, zero here, so each triangle is also an area light) and the glTF prism
# (8); lights.xml a floor rectangle, 3 spheres and the .glb prism, and a
# point, a spot and a constant emitter.
XML_COUNTS = {"cornell.xml": (39, 8), "lights.xml": (13, 3)}


@pytest.mark.parametrize("scene", XML_SCENES)
def test_reference_cli_loads_xml_scene(tmp_path, scene):
    """The reference route renders the XML scenes on the host: every shape,
    model and light of the file loaded (primitive and light counts), a lit
    image of the file's resolution."""
    need(CLIREF)
    out = str(tmp_path / "ref.pfm")
    p = run([CLIREF, "-s", "4", "-o", out, os.path.join(SCENES, scene)])
    assert p.returncode == 0, p.stderr
    assert f"primitives {XML_COUNTS[scene][0]} lights {XML_COUNTS[scene][1]}" in p.stdout, p.stdout
    img = read_pfm(out)
    assert img.shape == (96, 96, 3) and np.isfinite(img).all()
    assert img.mean() > 0.05
    assert "not supported" not in p.stderr and "Failed" not in p.stderr and "error" not in p.stderr.lower()


def test_reference_cli_reports_broken_xml(tmp_path):
    bad = tmp_path / "bad.xml"
    bad.write_text('<scene version="3.0.0"><shape type="sphere"></scene>')
    p = run([CLIREF, "-s", "1", "-o", str(tmp_path / "x.pfm"), str(bad)])
    assert p.returncode == 1
    assert "Start and end tags do not match" in p.stderr


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
    z = block_z(gpu - ref, ref)
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


@pytest.mark.gpu
@pytest.mark.parametrize("tree", ["reference", "device"])
@pytest.mark.parametrize("scene", XML_SCENES)
def test_cli_xml_scene_matches_reference(tmp_path, scene, tree):
    need(BBCLI)
    need(CLIREF)
    path = os.path.join(SCENES, scene)
    ref_out, gpu_out = str(tmp_path / "ref.pfm"), str(tmp_path / "gpu.pfm")
    p = run([CLIREF, "-s", "16", "-o", ref_out, path])
    assert p.returncode == 0, p.stderr
    p = run([BBCLI, "-s", "16", "--tree", tree, "-o", gpu_out, path])
    print(p.stdout[-600:])
    assert p.returncode == 0, p.stderr
    gpu, ref = read_pfm(gpu_out), read_pfm(ref_out)
    assert gpu.shape == ref.shape == (96, 96, 3)
    assert np.isfinite(gpu).all()
    rel_mean = np.abs(gpu.mean(axis=(0, 1)) - ref.mean(axis=(0, 1))) / ref.mean(axis=(0, 1))
    z = block_z(gpu - ref, ref)
    rel = np.abs(gpu - ref).max(axis=2) / np.maximum(np.abs(ref).max(axis=2), 1e-3)
    print(f"{scene} [{tree}]: channel mean rel diff {rel_mean}, max block z {z.max():.2f}, "
          f"pixels within 1e-3 {(rel < 1e-3).mean():.4f}")
    assert (rel_mean < 5e-3).all(), rel_mean
    assert z.size > 50 and z.max() < 5.0, z.max()
    if tree == "reference":
        assert (rel < 1e-3).mean() >= 0.97, (rel < 1e-3).mean()
