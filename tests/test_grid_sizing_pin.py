"""The grid sizing of the oracle pinned to the reference's own code (no GPU).

The reference sizes its photon grid in PhotonGrid::compute_grid_and_cell_size
(CudaPhotonMapping/PhotonGrid.cu:41-56: ceil(n / desired) cells of the scene
box's volume, a cubic cell, ceil(extent / cell) cells per axis) and re-sizes it
with desired / 5 when a cell of the first grid holds more than 5 x desired
photons (analyze_density, :92-141).  oracle/_ref/libref_host.so runs that code
on the host (oracle/ref_host/ref_driver.cu ref_grid_sizing); its results on the
seeded photon sets of tests/golden/ref_cases.py are in
tests/golden/grid_sizing_ref.npz.  The CUDA grid build is checked against the
oracle's grid (dims, cell size, cell arrays) in tests/test_gpu_parity.py.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import ref_cases  # noqa: E402

from oracle import REF_SO  # noqa: E402

CASES = list(ref_cases.GRID_CASES)


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(HERE, "golden", "grid_sizing_ref.npz"))


@pytest.fixture(scope="module")
def photon_sets():
    return {name: build() for name, (build, _) in ref_cases.GRID_CASES.items()}


@pytest.mark.parametrize("name", CASES)
def test_oracle_grid_sizing_matches_reference(orc, golden, photon_sets, name):
    pos, aabb = photon_sets[name]
    desired = ref_cases.GRID_CASES[name][1]
    z = np.zeros_like(pos)
    g = orc.grid_build(pos, z, z, aabb, desired=desired)
    assert np.array_equal(g.dims, golden[f"{name}__dims"])
    assert np.float32(g.cell) == golden[f"{name}__cell"]
    # the oracle's cell counts add up to n, and the largest cell of the final
    # grid stays below the reference's first-grid maximum when it re-gridded
    assert int(g.sizes.sum()) == pos.shape[0]
    if int(golden[f"{name}__regrid"]):
        assert int(g.sizes.max()) < int(golden[f"{name}__max"])


def test_cases_cover_both_branches(golden):
    flags = [int(golden[f"{n}__regrid"]) for n in CASES]
    assert 0 in flags and 1 in flags


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference host harness not built (make -C oracle ref)")
@pytest.mark.parametrize("name", CASES)
def test_reference_grid_sizing_live(golden, photon_sets, name):
    from oracle import RefHost
    pos, aabb = photon_sets[name]
    dims, cell, regrid, mx = RefHost().grid_sizing(pos, aabb, ref_cases.GRID_CASES[name][1])
    assert np.array_equal(dims, golden[f"{name}__dims"]) and np.float32(cell) == golden[f"{name}__cell"]
    assert int(regrid) == int(golden[f"{name}__regrid"]) and mx == int(golden[f"{name}__max"])


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference host harness not built (make -C oracle ref)")
def test_fixture100_grid_is_the_reference_grid(golden_dir):
    # the reference's 100-photon dump, desired 10 per cell: the dims and cell size
    # stored with the fixture (built by the oracle) are the reference's own
    from oracle import RefHost
    f = np.load(os.path.join(golden_dir, "fixture100.npz"))
    dims, cell, regrid, _ = RefHost().grid_sizing(f["pos"], f["aabb"], int(f["desired"]))
    assert np.array_equal(dims, f["dims"]) and np.float32(cell) == f["cell"]
