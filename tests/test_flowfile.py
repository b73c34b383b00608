"""Flow files in the reference's structured-block format
(src/eilmer/sfluidblock.d:1778-1956, fvcell.d:2374-2560,
globalconfig.d:791-836): variable list, header, exact round trips in both
formats, and cell volumes equal to the CPU oracle's geometry."""
import gzip

import numpy as np
import pytest

from eilmer4_b200 import flowfile as F
from eilmer4_b200 import workloads as W


def test_variable_lists():
    assert F.variable_names(["air"]) == [
        "pos.x", "pos.y", "pos.z", "volume", "rho", "vel.x", "vel.y", "vel.z", "p", "a", "mu",
        "k", "mu_t", "k_t", "S", "tke", "omega", "massf[0]-air", "u", "T"]
    names = F.variable_names(["N2", "O2", "NO", "N", "O"])
    assert names[17:24] == ["massf[0]-N2", "massf[1]-O2", "massf[2]-NO", "massf[3]-N",
                            "massf[4]-O", "dt_chem", "u"]
    assert names[-1] == "T"


@pytest.mark.parametrize("fmt", ["gziptext", "rawbinary"])
def test_round_trip_is_exact(tmp_path, fmt):
    wl = W.reacting_channel(ni=12, nj=6)
    b = wl.blocks[0]
    rng = np.random.default_rng(2)
    prim = b.prim * (1.0 + 1e-3 * rng.standard_normal(b.prim.shape))
    dt_chem = rng.random(b.ncell) * 1e-8
    pos, vol = F.cell_geometry(b.vtx, b.ni, b.nj, b.nk, 2)
    path = str(tmp_path / ("b.flow" + (".gz" if fmt == "gziptext" else "")))
    F.write_flow(path, prim=prim, pos=pos, volume=vol, dimensions=2, ni=b.ni, nj=b.nj, nk=1,
                 species=wl.thermochem.species, sim_time=1.25e-4, label="ramp", dt_chem=dt_chem,
                 fmt=fmt)
    fl = F.read_flow(path, fmt)
    assert fl["sim_time"] == 1.25e-4 and fl["label"] == "ramp"
    assert (fl["dimensions"], fl["nicell"], fl["njcell"], fl["nkcell"]) == (2, 12, 6, 1)
    p2, d2 = F.prim_from_flow(fl, 5)
    assert np.array_equal(p2, prim) and np.array_equal(d2, dt_chem)
    assert np.array_equal(fl["data"][3], vol)


def test_text_layout(tmp_path):
    wl = W.sod_2d(4, 2)
    b = wl.blocks[0]
    pos, vol = F.cell_geometry(b.vtx, b.ni, b.nj, b.nk, 2)
    path = str(tmp_path / "s.flow.gz")
    F.write_flow(path, prim=b.prim, pos=pos, volume=vol, dimensions=2, ni=4, nj=2, nk=1,
                 species=["air"], sim_time=0.0)
    lines = gzip.open(path, "rt").read().splitlines()
    assert lines[0] == "structured_grid_flow 1.0"
    assert lines[1] == "label: " and lines[2] == "sim_time: 0.000000000000000000e+00"
    assert lines[3] == "variables: 20"
    assert lines[4].startswith(' "pos.x" "pos.y"') and lines[5] == "dimensions: 2"
    assert lines[6:9] == ["nicell: 4", "njcell: 2", "nkcell: 1"]
    assert len(lines) == 9 + 8
    vals = lines[9].split()
    assert len(vals) == 20 and vals[14] == "0" and lines[9].startswith(" ")


@pytest.mark.parametrize("case", ["box3d", "ramp2d"])
def test_volumes_match_the_oracle_geometry(oracle, case):
    if case == "box3d":
        wl = W.inflow_3d(n=6)
        cfg = oracle.default_config(dimensions=3)
    else:
        wl = W.reacting_channel(ni=10, nj=5)
        cfg = oracle.default_config(dimensions=2)
    b = wl.blocks[0]
    sim = oracle.OracleSim(cfg)
    sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
    cells, _ = sim.geometry(0)
    _, vol = F.cell_geometry(b.vtx, b.ni, b.nj, b.nk, wl.dimensions)
    assert np.allclose(vol, cells[0], rtol=1e-14, atol=0.0)
