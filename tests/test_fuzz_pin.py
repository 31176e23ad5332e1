"""The oracle's photon tracer against the reference's own tracer (compiled as
host code, oracle/ref_host/ref_trace.cu) on seeded random rooms: random
light offsets, sphere sizes and tessellations, and blobs of random triangles
(degenerate ones included) with diffuse, mirror, glossy, glass and
translucent materials of random IOR.  Every field of every path (photon
counts, uniforms consumed, positions, directions, bounces, the global /
caustic split) must agree bit for bit.  No GPU."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(HERE, "golden"))
import fuzz_scenes  # noqa: E402
import ref_cases  # noqa: E402

from oracle import REF_TRACE_SO  # noqa: E402

PATHS = 3000


@pytest.mark.skipif(not os.path.exists(REF_TRACE_SO), reason="reference tracer harness not built (make -C oracle ref)")
@pytest.mark.parametrize("seed", range(8))
def test_random_room_tracer_matches_reference(orc, seed):
    from oracle import RefTrace
    sc = fuzz_scenes.random_scene(seed)
    ref = RefTrace().scene(sc)
    s = orc.scene(sc)
    assert sorted(map(tuple, s.critical_angles())) == sorted(map(tuple, ref.critical_angles()))
    cap = 20_000
    r = ref.trace_paths(seed, cap, 0, PATHS)
    o = s.trace_paths(seed, ref_cases.MAX_BOUNCES, cap, 0, PATHS)
    for f in ref_cases.FIELDS:
        assert np.array_equal(o[f], r[f]), f"seed {seed}: {f} differs from the reference's tracer"
    # the rooms exercise the rules: multi-bounce paths, caustic photons, paths without a photon
    assert o["counts"].sum() > PATHS // 2 and (o["counts"].sum(1) == 0).any()


def test_random_rooms_reach_every_material():
    kinds = set()
    for seed in range(8):
        sc = fuzz_scenes.random_scene(seed)
        m = sc.materials[8:]
        for row in m:
            spec, opaque = row[3:6].max(), row[10]
            kinds.add("glass" if opaque == 0 else "translucent" if opaque < 1 else
                      "mirror" if spec == 1 and row[0:3].max() == 0 else "glossy" if spec > 0 else "diffuse")
    assert kinds == {"diffuse", "mirror", "glossy", "glass", "translucent"}
