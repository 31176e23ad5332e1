"""The oracle's photon tracer pinned to the reference's own tracer (no GPU).

The reference's CudaPhotonMapping/PhotonTracing.cu (emission, trace, destiny,
Fresnel, the medium stack, the critical-angle table, the store and caustic
rules) and the functions it calls (Model light sampling and intersection,
Ray::reflect / refract / reflect_spherical, PathOperator, PhotonArray) are
compiled from the reference sources as host code into
oracle/_ref/libref_trace.so and driven one path at a time with the injected
per-path streams (oracle/ref_host/ref_trace.cu).  The GPU tracer is checked
against the same oracle bit for bit in tests/test_gpu_parity.py, so these pins
carry over to it.

Two forms:
  * golden: tests/golden/tracer_ref.npz holds the reference's results
    (checksums of whole path ranges, full records of their first paths),
    written by tests/golden/make_golden.py; this runs everywhere;
  * live: where the harness library is built (make -C oracle ref), the
    reference's tracer runs here and every record is compared.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import ref_cases  # noqa: E402

from oracle import REF_TRACE_SO  # noqa: E402

CASES = list(ref_cases.CASES)


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(HERE, "golden", "tracer_ref.npz"))


def _oracle_paths(orc, name, p1=None):
    build, seed, cap, p0, end, _ = ref_cases.CASES[name]
    s = orc.scene(build())
    return s.trace_paths(seed, ref_cases.MAX_BOUNCES, cap, p0, end if p1 is None else p1)


@pytest.mark.parametrize("name", CASES)
def test_tracer_matches_reference_golden(orc, golden, name):
    build, seed, cap, p0, end, sub = ref_cases.CASES[name]
    part = _oracle_paths(orc, name, sub)
    for f in ref_cases.FIELDS:
        assert np.array_equal(part[f], golden[f"{name}__{f}"]), f"{name}: {f} differs from the reference"
    full = _oracle_paths(orc, name)
    assert ref_cases.checksum(full) == int(golden[f"{name}__checksum"])
    assert [full["g_pos"].shape[0], full["c_pos"].shape[0]] == list(golden[f"{name}__n"])
    # photon power: intensity / capacity for every photon (CudaPhotonMapping/PhotonTracing.cu:369)
    assert np.float32(1.0) / np.float32(cap) == golden[f"{name}__power"][0, 0]


def test_golden_cases_exercise_the_rules(golden):
    # the cases reach what the pin is about: caustic photons (specular / refractive
    # paths before any diffuse bounce), multi-bounce paths, paths that end without
    # a photon, paths of every length up to the bounce limit
    for name in CASES:
        cnt = golden[f"{name}__counts"]
        assert cnt[:, 0].max() >= 3 and (cnt.sum(1) == 0).any()
        assert golden[f"{name}__g_bounce"].max() >= 5
    assert golden["stress_glass__c_pos"].shape[0] > 100
    assert golden["cornell_small__c_pos"].shape[0] > 10


@pytest.mark.skipif(not os.path.exists(REF_TRACE_SO), reason="reference tracer harness not built (make -C oracle ref)")
@pytest.mark.parametrize("name", CASES)
def test_tracer_matches_reference_live(orc, name):
    from oracle import RefTrace
    build, seed, cap, p0, end, _ = ref_cases.CASES[name]
    sc = build()
    ref = RefTrace().scene(sc)
    s = orc.scene(sc)
    # the critical-angle table: the same (n1, n2) -> cos pairs
    a = sorted(map(tuple, s.critical_angles()))
    b = sorted(map(tuple, ref.critical_angles()))
    assert a == b
    r = ref.trace_paths(seed, cap, p0, end)
    o = s.trace_paths(seed, ref_cases.MAX_BOUNCES, cap, p0, end)
    for f in ref_cases.FIELDS:
        assert np.array_equal(o[f], r[f]), f"{name}: {f} differs from the reference's tracer"
    pw = np.float32(1.0) / np.float32(cap)
    assert (r["g_pow"] == pw).all() and (r["c_pow"] == pw).all()
