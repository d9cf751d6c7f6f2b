"""BxDF parity: for every supported material, Material::GetBSDF then
BSDF::f, PDF and Sample_f on random directions and random numbers, the
device (bbg_bsdf_probe) against the reference (the oracle's probe of the
reference's own material and BSDF classes).

Bar: f and pdf within 1e-5 relative (the reference's glibc float pow and the
device's differ by an ulp at most); samples: the same success, direction
within 1e-5, f and pdf within 1e-4 relative (the VNDF sampler's sin/cos),
except for at most 0.2 % of queries whose random number falls within an ulp
of a lobe-selection threshold."""
import numpy as np
import pytest

from bulbit_b200 import abi, lib, scenes

pytestmark = pytest.mark.gpu

MATERIALS = {
    "diffuse": lambda: scenes.diffuse((0.7, 0.4, 0.2)),
    "conductor_smooth": lambda: scenes.conductor(scenes.GOLD_ETA, scenes.GOLD_K, 0.0),
    "conductor_rough": lambda: scenes.conductor(scenes.GOLD_ETA, scenes.GOLD_K, 0.3),
    "conductor_anisotropic": lambda: scenes.conductor(scenes.GOLD_ETA, scenes.GOLD_K, 0.2),
    "conductor_energy_compensated": lambda: scenes.conductor(scenes.GOLD_ETA, scenes.GOLD_K, 0.4,
                                                             energy_compensation=True),
    "dielectric_smooth": lambda: scenes.dielectric(1.5, 0.0),
    "dielectric_rough": lambda: scenes.dielectric(1.5, 0.3),
    "dielectric_energy_compensated": lambda: scenes.dielectric(1.5, 0.4, (0.9, 0.8, 0.7), energy_compensation=True),
    "metallic_roughness": lambda: scenes.metallic_roughness((0.8, 0.5, 0.3), 0.4, 0.35),
}


def rel(a, b):
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-6)


def queries(n, seed):
    rng = np.random.default_rng(seed)
    wo = rng.normal(size=(n, 3))
    wo /= np.linalg.norm(wo, axis=1, keepdims=True)
    wi = rng.normal(size=(n, 3))
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    u = rng.random((n, 3))
    return wo.astype(np.float32), wi.astype(np.float32), u.astype(np.float32)


# Every material from the front; the dielectric (the only BxDF whose relative
# eta depends on the side) from the back too.
CASES = [(name, True) for name in MATERIALS] + [(name, False) for name in MATERIALS if name.startswith("dielectric")]


@pytest.mark.parametrize("name,front_face", CASES, ids=[f"{n}-{'front' if f else 'back'}" for n, f in CASES])
def test_bsdf_matches_reference(oracle, name, front_face):
    m = MATERIALS[name]()
    if name == "conductor_anisotropic":
        m.roughness[:] = [0.15, 0.45]
    wo, wi, u = queries(20_000, seed=sum(map(ord, name)))
    g = lib.bsdf_probe(m, wo, wi, u, front_face=front_face)
    r = oracle.bsdf_probe(m, wo, wi, u, front_face=front_face)
    # f and pdf at given directions
    f_bad = (rel(g[:, 0:3], r[:, 0:3]) > 1e-5).any(axis=1) | (rel(g[:, 3], r[:, 3]) > 1e-5)
    # samples
    ok_same = (g[:, 11] >= 0) == (r[:, 11] >= 0)
    both = (g[:, 11] >= 0) & (r[:, 11] >= 0)
    s_bad = ~ok_same.copy()
    s_bad[both] = ((np.abs(g[both, 7:10] - r[both, 7:10]) > 1e-5).any(axis=1)
                   | (rel(g[both, 4:7], r[both, 4:7]) > 1e-4).any(axis=1)
                   | (rel(g[both, 10], r[both, 10]) > 1e-4)
                   | (g[both, 11] != r[both, 11]))
    print(f"{name} ({'front' if front_face else 'back'}): f/pdf mismatches {f_bad.mean():.5f}, "
          f"sample mismatches {s_bad.mean():.5f}, samples taken {both.mean():.3f}, "
          f"nonzero f {(np.abs(r[:, 0:3]).max(1) > 0).mean():.3f}")
    assert f_bad.mean() <= 0.002
    assert s_bad.mean() <= 0.002
    assert both.mean() > 0.2
