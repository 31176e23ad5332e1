"""The photon-map file (pm_save_photons / pm_load_photons) in the reference's
layout: a little-endian u64 count, then per photon pos[3], power[3], inc_dir[3]
as float32, the layout CudaPhotonMapping/Initializer.cu:102-141 reads.

The reference ships one such file, CudaPhotonMapping/global_map_test.txt (100
photons, 3,608 bytes).  tests/golden/fixture100.npz holds its fields, read as
the reference's reader reads them (tests/golden/make_golden.py); rebuilding the
file from those fields gives the reference's bytes (its SHA-256 below), so the
GPU tests load and save exactly the reference's file.
"""
import hashlib
import os
import struct

import numpy as np
import pytest

# SHA-256 of CudaPhotonMapping/global_map_test.txt
REF_DUMP_SHA256 = "195903773ce029255367509e9c000ccbdaee26eaefcee5afa83a17a9983392ba"


def _file_bytes(pos, power, direction):
    rec = np.concatenate([pos, power, direction], 1).astype("<f4")
    return struct.pack("<Q", rec.shape[0]) + rec.tobytes()


@pytest.fixture(scope="module")
def fixture100(golden_dir):
    return np.load(os.path.join(golden_dir, "fixture100.npz"))


def test_fixture_rebuilds_the_reference_file(fixture100):
    b = _file_bytes(fixture100["pos"], fixture100["power"], fixture100["dir"])
    assert len(b) == 8 + 36 * 100 == 3608
    assert hashlib.sha256(b).hexdigest() == REF_DUMP_SHA256


# ------------------------------------------------------------------ GPU ----
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def ctx():
    import photonmap
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return photonmap.Context(0)


@pytest.mark.gpu
def test_load_and_save_the_reference_file(ctx, fixture100, tmp_path):
    ref = tmp_path / "global_map_test.txt"
    ref.write_bytes(_file_bytes(fixture100["pos"], fixture100["power"], fixture100["dir"]))
    ctx.load_photons(0, ref)
    ph = ctx.photons(0, sorted_=False)
    assert ph["count"] == 100
    assert np.array_equal(ph["list_pos"].cpu().numpy(), fixture100["pos"])
    assert np.array_equal(ph["list_power"].cpu().numpy(), fixture100["power"])
    assert np.array_equal(ph["list_dir"].cpu().numpy(), fixture100["dir"])
    out = tmp_path / "saved.bin"
    ctx.save_photons(0, out)
    assert hashlib.sha256(out.read_bytes()).hexdigest() == REF_DUMP_SHA256   # the reference's bytes


@pytest.mark.gpu
def test_traced_map_round_trip(ctx, tmp_path):
    from photonmap import scenes
    sc, _, w = scenes.workload("cornell_small")
    ctx.set_scene(sc)
    ctx.trace_photons(11, w["max_bounces"], 50_000, 5_000)
    a = tmp_path / "g.bin"
    c = tmp_path / "c.bin"
    ctx.save_photons(0, a)
    ctx.save_photons(1, c)
    g0 = {k: v.cpu().numpy().copy() for k, v in ctx.photons(0, sorted_=False).items() if k.startswith("list_")}
    assert a.stat().st_size == 8 + 36 * 50_000 and c.stat().st_size == 8 + 36 * 5_000
    # load the caustic file into the global map and back: every field bit for bit
    ctx.load_photons(0, c)
    assert ctx.photons(0, sorted_=False)["count"] == 5_000
    ctx.load_photons(0, a)
    g1 = ctx.photons(0, sorted_=False)
    for k, v in g0.items():
        assert np.array_equal(g1[k].cpu().numpy(), v), k
    b = tmp_path / "g2.bin"
    ctx.save_photons(0, b)
    assert a.read_bytes() == b.read_bytes()
    ctx.build_grid(0)   # a loaded map builds like a traced one
    assert ctx.status() == 0


@pytest.mark.gpu
def test_bad_files_are_errors_not_crashes(ctx, fixture100, tmp_path):
    import photonmap
    good = _file_bytes(fixture100["pos"], fixture100["power"], fixture100["dir"])
    ctx.set_photons(0, fixture100["pos"], fixture100["power"], fixture100["dir"])
    cases = {
        "missing": None,
        "empty": b"",
        "short_header": good[:5],
        "truncated": good[:8 + 36 * 60 + 7],
        # a header that claims 2^31 photons in a 3,608-byte file: refused before
        # anything is allocated (the reference's reader would try 2^31 photons)
        "oversized_count": struct.pack("<Q", 1 << 31) + good[8:],
        "absurd_count": struct.pack("<Q", (1 << 64) - 1) + good[8:],
    }
    for name, data in cases.items():
        p = tmp_path / f"{name}.bin"
        if data is not None:
            p.write_bytes(data)
        with pytest.raises(photonmap.PMError) as e:
            ctx.load_photons(0, p)
        assert e.value.code == -6, name   # PM_ERR_IO
    # the context still works: the reference's file loads, builds and gathers
    p = tmp_path / "ok.bin"
    p.write_bytes(good)
    ctx.load_photons(0, p)
    ctx.build_grid(0, desired=int(fixture100["desired"]), aabb=fixture100["aabb"])
    rad, _, _ = ctx.gather(torch.from_numpy(fixture100["q"]), torch.from_numpy(fixture100["qn"]), int(fixture100["k"]),
                           float(fixture100["r"]))
    np.testing.assert_allclose(rad.cpu().numpy(), fixture100["ref_rad"], rtol=1e-4, atol=1e-9)
    assert ctx.status() == 0
