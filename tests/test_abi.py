"""The C ABI library (no GPU needed): it loads and exports every entry point
include/pm_api.h declares; host-only entry points behave."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pm_api.h")


def declared():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(pm_\w+)\s*\(", txt, re.M)))


@pytest.fixture(scope="module")
def lib():
    from photonmap import core
    if not os.path.exists(core.LIB_PATH):
        import subprocess
        subprocess.run(["make", "-C", os.path.join(ROOT, "cuda-photon-mapping_b200", "csrc")], check=True,
                       stdout=subprocess.DEVNULL)
    return core.library()


def test_exports_every_declared_symbol(lib):
    names = declared()
    assert len(names) >= 19
    for n in names:
        assert hasattr(lib, n), n


def test_camera_setup_matches_oracle(lib, orc):
    import photonmap
    from photonmap import scenes
    for cs in [scenes.default_camera(320, 240), scenes.CameraSpec((0.3, 0.2, 3.0), (-0.1, -0.05, -1.0), (0, 1, 0), 60.0, 64, 48)]:
        cam = photonmap.camera_setup(cs.position, cs.direction, cs.up, cs.fov_deg, cs.width, cs.height)
        assert np.array_equal(cam.as_vector(), orc.camera(cs))


def test_invalid_arguments_are_errors_not_crashes(lib):
    import photonmap
    with pytest.raises(photonmap.PMError):
        photonmap.camera_setup((0, 0, 0), (0, 0, -1), (0, 1, 0), 45.0, 0, 10)
    assert lib.pm_create(None, None) == -1
    assert lib.pm_sync(None) == -1
    assert lib.pm_status(None, None) == -1
