"""Host-side set-up that the kernels depend on bit for bit: the camera basis
(PerspectiveCamera ctor, src/camera/perspective_camera.cpp:8-38)."""
import numpy as np
import pytest

from bulbit_b200 import lib, scenes


def cam_fields(c):
    return np.array([c.origin[:], c.lower_left[:], c.horizontal[:], c.vertical[:], c.u[:], c.v[:]],
                    np.float32), np.float32(c.lens_radius)


@pytest.mark.parametrize("spec", [
    scenes.readme_sphere().camera,
    scenes.cornell_icosphere(levels=1, width=64, height=48).camera,
    scenes.camera_spec((0.5, 0.5, 2.05), (0.5, 0.5, 0.0), (0, 1, 0), 28, 0, 2.05, 500, 500),
    scenes.camera_spec((-3, -2, 1), (0.2, 0.1, -0.3), (0, 0, 1), 50, 0.2, 3.0, 77, 33),
], ids=["readme", "cornell", "cli_cornell", "tilted"])
def test_camera_matches_reference(oracle, spec):
    mine, mr = cam_fields(lib.camera(spec))
    ref, rr = cam_fields(oracle.camera(spec))
    assert np.array_equal(mine.view(np.uint32), ref.view(np.uint32))
    assert mr == rr
