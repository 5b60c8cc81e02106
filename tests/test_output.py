"""Chunked snapshot output and restart (suetes_b200/output.py) on the CPU:
the NetCDF classic files the writer appends, read back with scipy; the
RESUME seed; the synchronous path of the asynchronous writer."""

import os

import numpy as np
import pytest
import scipy.io
import torch

from suetes_b200 import RegionalGrid3D
from suetes_b200.output import AsyncSnapshotWriter, NetcdfSnapshots, SimulationOutputWriter, restart_seed

C = {"p0": 1e5, "Rd": 287.0, "cvd": 717.0}


def _grid():
    return RegionalGrid3D(6, 5, 4, 1000.0, 1000.0, 500.0, 45.0, 10.0, device="cpu")


def _snap(rng):
    return {"u": rng.random((7, 5, 4)), "v": rng.random((6, 6, 4)), "w": rng.random((6, 5, 5)),
            "th_v": 300.0 + rng.random((6, 5, 4)), "pi": 0.9 + 0.01 * rng.random((6, 5, 4)),
            "sfc": rng.random((6, 5))}


def test_writer_round_trip_dims_attrs_and_fill(tmp_path):
    rng = np.random.default_rng(0)
    path = str(tmp_path / "run_prog.nc")
    keys = ["u", "v", "w", "th_v", "pi", "sfc"]
    w = SimulationOutputWriter(path, _grid(), keys, attrs={"experiment": "unit"}, ref_date="2024-01-01")
    snaps = [_snap(rng) for _ in range(3)]
    del snaps[2]["sfc"]
    sizes = []
    for s in snaps:
        w.write_snapshot(s)
        sizes.append(os.path.getsize(path))
    w.close()
    assert sizes[2] - sizes[1] == sizes[1] - sizes[0] > 0  # one record appended per snapshot
    f = scipy.io.netcdf_file(path, "r", mmap=False)
    try:
        v = f.variables
        assert v["u"].dimensions == ("time", "z", "y", "xc")
        assert v["v"].dimensions == ("time", "z", "yc", "x")
        assert v["w"].dimensions == ("time", "zc", "y", "x")
        assert v["sfc"].dimensions == ("time", "y", "x")
        assert list(v["time"][:]) == [0.0, 3600.0, 7200.0]
        assert v["time"].units == b"seconds since 2024-01-01 00:00:00"
        assert f.Conventions == b"CF-1.7" and f.experiment == b"unit"
        assert v["crs"].grid_mapping_name == b"stereographic"
        assert v["th_v"].coordinates == b"lat lon" and v["th_v"].grid_mapping == b"crs"
        np.testing.assert_allclose(v["x"][:], _grid().x_m.numpy())
        assert abs(float(v["lat"][:].mean()) - 45.0) < 0.1
        assert float(v["sfc"][2].min()) > 9e36  # missing key: fill value
    finally:
        f.close()
    rd = NetcdfSnapshots(path)
    try:
        assert len(rd) == 3
        for i in range(2):
            for k in keys:
                np.testing.assert_array_equal(rd[i][k], snaps[i][k].astype(np.float32))
    finally:
        rd.close()


def test_writer_rejects_shapes_off_the_grid(tmp_path):
    w = SimulationOutputWriter(str(tmp_path / "x.nc"), _grid(), ["bad"])
    with pytest.raises(ValueError):
        w.write_snapshot({"bad": np.zeros((9, 5, 4))})


def test_restart_seed_from_last_snapshot(tmp_path):
    rng = np.random.default_rng(1)
    path = str(tmp_path / "r.nc")
    w = SimulationOutputWriter(path, _grid(), ["u", "v", "w", "th_v", "pi"])
    snaps = [_snap(rng) for _ in range(2)]
    for s in snaps:
        w.write_snapshot(s)
    w.close()
    seed, kt = restart_seed(path, ["u", "v", "w", "th_v", "pi"], C)
    assert kt == 1
    th = torch.as_tensor(snaps[1]["th_v"].astype(np.float32), dtype=torch.float64)
    pi = torch.as_tensor(snaps[1]["pi"].astype(np.float32), dtype=torch.float64)
    assert torch.allclose(seed["rho"], C["p0"] / (C["Rd"] * th) * pi ** (C["cvd"] / C["Rd"]), rtol=1e-14)
    assert seed["eta_dot"].shape == (6, 5, 5) and float(seed["eta_dot"].abs().max()) == 0.0
    seed0, k0 = restart_seed(path, ["u"] + ["th_v", "pi"], C, index=0)
    assert k0 == 0 and torch.equal(seed0["u"], torch.as_tensor(snaps[0]["u"].astype(np.float32), dtype=torch.float64))


def test_async_writer_cpu_tensors_write_in_order(tmp_path):
    rng = np.random.default_rng(2)
    path = str(tmp_path / "a.nc")
    aw = AsyncSnapshotWriter(SimulationOutputWriter(path, _grid(), ["u", "th_v"]))
    snaps = [{k: torch.as_tensor(v) for k, v in _snap(rng).items()} for _ in range(4)]
    for n, s in enumerate(snaps):
        aw.submit(s, t_seconds=10.0 * n)
    aw.close()
    rd = NetcdfSnapshots(path)
    try:
        assert list(rd.times) == [0.0, 10.0, 20.0, 30.0]
        for n in range(4):
            np.testing.assert_array_equal(rd[n]["u"], snaps[n]["u"].numpy().astype(np.float32))
    finally:
        rd.close()


def test_file_without_snapshots_is_valid(tmp_path):
    path = str(tmp_path / "empty.nc")
    SimulationOutputWriter(path, _grid(), ["u"]).close()
    f = scipy.io.netcdf_file(path, "r", mmap=False)
    try:
        assert f.variables["time"].shape == (0,) and "u" not in f.variables
        assert f.variables["x"].shape == (6,)
    finally:
        f.close()
