"""Chunked snapshot output and restart for long device-resident runs.

Mirrors ``suetes/shared/output.py:34-141`` (``SimulationOutputWriter``: one
time slice per chunk on an unlimited ``time`` dimension, staggered fields on
their native ``x``/``xc``, ``y``/``yc``, ``z``/``zc`` dimensions stored
``(time, z, y, x)``, 1-D projection axes, 2-D lat/lon, the stereographic
``crs`` and CF-1.7) and the RESUME seed of ``runs/run_simulation.py:170-194``.
The reference writes NetCDF4/HDF5 through the ``netCDF4`` package, which is
not installed here; these files are NetCDF classic with 64-bit offsets
(CDF-2), the same variables, dimensions and attributes, readable by xarray,
ncview and ``scipy.io.netcdf_file``, uncompressed.  ``ClassicFile`` writes
the format directly: the header once (at the first snapshot, when the
fields' shapes are known), then each snapshot appended as one record and
the record count updated in place, so memory and the work per snapshot
stay constant over a run.

``AsyncSnapshotWriter`` is the device side of a long run: a snapshot of
device tensors is copied into a device staging slot on the producing stream
(a device-to-device copy), then to page-locked host memory on a side stream,
and a host thread writes it to disk while the next steps run.  The producing
stream only waits when every staging slot still has its host copy in flight;
the host only waits when every pinned slot is still being written.
"""

import queue
import struct
import threading

import numpy as np
import scipy.io
import torch

_NC_TYPES = {"i4": (4, ">i4"), "f4": (5, ">f4"), "f8": (6, ">f8")}  # nc_type, big-endian dtype
_NC_CHAR, _NC_INT, _NC_DOUBLE = 2, 4, 6
_NC_DIMENSION, _NC_VARIABLE, _NC_ATTRIBUTE = 10, 11, 12


def _pad4(b):
    return b + b"\0" * (-len(b) % 4)


def _name(s):
    b = s.encode()
    return struct.pack(">i", len(b)) + _pad4(b)


def _attrs(attrs):
    if not attrs:
        return struct.pack(">ii", 0, 0)
    out = struct.pack(">ii", _NC_ATTRIBUTE, len(attrs))
    for k, v in attrs.items():
        out += _name(k)
        if isinstance(v, str):
            b = v.encode()
            out += struct.pack(">ii", _NC_CHAR, len(b)) + _pad4(b)
        elif isinstance(v, (int, np.integer)) and not isinstance(v, bool):
            out += struct.pack(">iii", _NC_INT, 1, int(v))
        else:
            out += struct.pack(">ii", _NC_DOUBLE, 1) + struct.pack(">d", float(v))
    return out


class ClassicFile:
    """Minimal NetCDF classic (CDF-2, 64-bit offsets) writer with one
    unlimited record dimension: declare dimensions, global attributes and
    variables, then ``begin()`` writes the header and the fixed variables,
    and ``append(record)`` adds one record."""

    def __init__(self, path):
        self.path = path
        self.dims = {}     # name -> length (None: the record dimension)
        self.gattrs = {}
        self.vars = {}     # name -> dict(dims, type, attrs, data)
        self._f = None
        self.numrecs = 0

    def add_var(self, name, nctype, dims, attrs=None, data=None):
        self.vars[name] = {"dims": tuple(dims), "type": nctype, "attrs": dict(attrs or {}), "data": data}

    def _is_rec(self, v):
        return bool(v["dims"]) and self.dims[v["dims"][0]] is None

    def _vsize(self, v):
        n = 1
        for d in v["dims"]:
            if self.dims[d] is not None:
                n *= self.dims[d]
        size = n * int(_NC_TYPES[v["type"]][1][-1])
        return size + (-size % 4)

    def _header(self, begins):
        dimids = {d: i for i, d in enumerate(self.dims)}
        h = b"CDF\x02" + struct.pack(">i", self.numrecs)
        h += struct.pack(">ii", _NC_DIMENSION, len(self.dims)) if self.dims else struct.pack(">ii", 0, 0)
        for d, n in self.dims.items():
            h += _name(d) + struct.pack(">i", 0 if n is None else n)
        h += _attrs(self.gattrs)
        h += struct.pack(">ii", _NC_VARIABLE, len(self.vars)) if self.vars else struct.pack(">ii", 0, 0)
        for name, v in self.vars.items():
            h += _name(name) + struct.pack(">i", len(v["dims"]))
            h += b"".join(struct.pack(">i", dimids[d]) for d in v["dims"])
            h += _attrs(v["attrs"])
            h += struct.pack(">iiq", _NC_TYPES[v["type"]][0], self._vsize(v), begins.get(name, 0))
        return h

    def begin(self):
        fixed = [n for n, v in self.vars.items() if not self._is_rec(v)]
        rec = [n for n, v in self.vars.items() if self._is_rec(v)]
        off = len(self._header({}))
        begins = {}
        for n in fixed:
            begins[n] = off
            off += self._vsize(self.vars[n])
        self._rec_off, self._recsize = off, 0
        for n in rec:
            begins[n] = off + self._recsize
            self._recsize += self._vsize(self.vars[n])
        self._begins, self._rec = begins, rec
        self._f = open(self.path, "wb")
        self._f.write(self._header(begins))
        for n in fixed:
            v = self.vars[n]
            b = np.ascontiguousarray(np.asarray(v["data"]), dtype=_NC_TYPES[v["type"]][1]).tobytes()
            self._f.write(_pad4(b) if len(b) % 4 else b)
        self._f.flush()

    def append(self, record):
        """record: name -> array in the declared (non-record) dimension order."""
        base = self._rec_off + self.numrecs * self._recsize
        for n in self._rec:
            v = self.vars[n]
            a = np.ascontiguousarray(np.asarray(record[n]), dtype=_NC_TYPES[v["type"]][1])
            self._f.seek(self._begins[n] - self._rec_off + base)
            self._f.write(_pad4(a.tobytes()))
        self.numrecs += 1
        self._f.seek(4)
        self._f.write(struct.pack(">i", self.numrecs))
        self._f.flush()

    def close(self):
        if self._f is None:
            self.begin()
        self._f.close()


def _host(a):
    if torch.is_tensor(a):
        return a.detach().cpu().numpy()
    return np.asarray(a)


_FILL_F4 = np.float32(9.9692099683868690e36)  # NetCDF's default float fill value


class SimulationOutputWriter:
    """Append-per-chunk NetCDF writer (constant memory in run length)."""

    def __init__(self, path, grid, keys, attrs=None, dt_hours=1.0, ref_date=None):
        self.path = path
        self.keys = list(keys)
        self._t = 0
        self._dt_seconds = float(dt_hours) * 3600.0
        nx, ny, nz = grid.nx, grid.ny, grid.nz
        self._sizes = (nx, ny, nz)
        f = ClassicFile(path)
        f.dims = {"time": None, "x": nx, "xc": nx + 1, "y": ny, "yc": ny + 1, "z": nz, "zc": nz + 1}

        def coord(name, data, units, long_name, std=None, axis=None, positive=None):
            at = {"units": units, "long_name": long_name}
            if std:
                at["standard_name"] = std
            if axis:
                at["axis"] = axis
            if positive:
                at["positive"] = positive
            f.add_var(name, "f8", (name,), at, _host(data).astype(np.float64))

        coord("x", grid.x_m, "m", "projection x (mass)", "projection_x_coordinate", "X")
        coord("y", grid.y_m, "m", "projection y (mass)", "projection_y_coordinate", "Y")
        coord("xc", grid.x_c, "m", "projection x (u faces)", "projection_x_coordinate", "X")
        coord("yc", grid.y_c, "m", "projection y (v faces)", "projection_y_coordinate", "Y")
        coord("z", np.arange(nz), "1", "model level (mass)", axis="Z", positive="up")
        coord("zc", np.arange(nz + 1), "1", "model level (w)", axis="Z", positive="up")
        proj = grid.proj
        xm = torch.as_tensor(grid.x_m, dtype=torch.float64).cpu()
        ym = torch.as_tensor(grid.y_m, dtype=torch.float64).cpu()
        lat, lon = proj.get_lat_lon(*torch.meshgrid(xm, ym, indexing="ij"))
        for name, val, units, std in (("lat", lat, "degrees_north", "latitude"),
                                      ("lon", lon, "degrees_east", "longitude")):
            f.add_var(name, "f4", ("y", "x"), {"units": units, "standard_name": std, "long_name": std},
                      _host(val).T.astype(np.float32))
        f.add_var("crs", "i4", (), {"grid_mapping_name": "stereographic",
                                    "latitude_of_projection_origin": float(np.degrees(proj.phi_c)),
                                    "longitude_of_projection_origin": float(np.degrees(proj.lam_c)),
                                    "scale_factor_at_projection_origin": 1.0, "false_easting": 0.0,
                                    "false_northing": 0.0, "earth_radius": float(proj.R)}, np.zeros((), np.int32))
        f.add_var("time", "f8", ("time",), {"units": f"seconds since {ref_date} 00:00:00" if ref_date else "seconds",
                                            "long_name": "time"})
        f.gattrs = {"Conventions": "CF-1.7", **dict(attrs or {})}
        self._file = f
        self._shapes = {}

    def _dims_for_shape(self, shape):
        nx, ny, nz = self._sizes
        maps = [{nx: "x", nx + 1: "xc"}, {ny: "y", ny + 1: "yc"}, {nz: "z", nz + 1: "zc"}]
        dims = []
        for ax, n in enumerate(shape):
            if n not in maps[ax]:
                raise ValueError(f"output field axis {ax} size {n} matches no grid dimension {set(maps[ax])}")
            dims.append(maps[ax][n])
        return tuple(reversed(dims))

    def write_snapshot(self, state, t_seconds=None):
        """Write one time slice; ``state`` maps keys to (x, y[, z]) arrays
        (numpy, or tensors on any device).  The fields' variables are
        declared at the first snapshot; a key missing later is written as
        the fill value."""
        f = self._file
        arrays = {k: _host(state[k]) for k in self.keys if k in state}
        if f.numrecs == 0 and f._f is None:
            for k in self.keys:
                if k not in arrays:
                    continue
                spatial = self._dims_for_shape(arrays[k].shape)
                at = {}
                if len(spatial) >= 2 and spatial[-2:] == ("y", "x"):
                    at["coordinates"] = "lat lon"
                if len(spatial) >= 2:
                    at["grid_mapping"] = "crs"
                f.add_var(k, "f4", ("time",) + spatial, at)
                self._shapes[k] = tuple(f.dims[d] for d in spatial)
            f.begin()
        rec = {"time": np.float64(self._t * self._dt_seconds if t_seconds is None else float(t_seconds))}
        for k, shape in self._shapes.items():
            if k in arrays:
                a = arrays[k]
                rec[k] = np.transpose(a, tuple(reversed(range(a.ndim)))).astype(np.float32)
            else:
                rec[k] = np.full(shape, _FILL_F4, np.float32)
        f.append(rec)
        self._t += 1

    def close(self):
        self._file.close()


class NetcdfSnapshots:
    """Read a writer's file back as a list of per-time dicts of native
    (x, y[, z]) arrays (the stored (z, y, x) transposed back)."""

    def __init__(self, path, keys=None):
        self._ds = scipy.io.netcdf_file(path, "r", mmap=True)  # records are read on access
        avail = [k for k, v in self._ds.variables.items()
                 if v.dimensions and v.dimensions[0] == "time" and k != "time"]
        self.keys = [k for k in (keys or avail) if k in avail]
        self.n = self._ds.variables["time"].shape[0]
        self.times = np.array(self._ds.variables["time"][:], dtype=np.float64)

    def __len__(self):
        return self.n

    def __getitem__(self, i):
        i = range(self.n)[i]
        out = {}
        for k in self.keys:
            a = self._ds.variables[k][i]
            a = a.astype(a.dtype.newbyteorder("="))  # a native-order copy of the big-endian record
            out[k] = np.transpose(a, tuple(reversed(range(a.ndim))))
        return out

    def close(self):
        self._ds.close()


def restart_seed(path, keys, constants, index=-1):
    """The RESUME seed (runs/run_simulation.py:172-194): the saved fields of
    snapshot ``index`` as float64 (x, y, z) tensors, density from the
    equation of state and eta_dot zero.  Returns (seed, snapshot index)."""
    snaps = NetcdfSnapshots(path, keys)
    try:
        kt = range(len(snaps))[index]
        seed = {k: torch.as_tensor(v, dtype=torch.float64) for k, v in snaps[kt].items()}
    finally:
        snaps.close()
    c = constants
    seed["rho"] = c["p0"] / (c["Rd"] * seed["th_v"]) * seed["pi"] ** (c["cvd"] / c["Rd"])
    nx, ny, nz = seed["th_v"].shape
    seed["eta_dot"] = torch.zeros(nx, ny, nz + 1, dtype=torch.float64)
    return seed, kt


class AsyncSnapshotWriter:
    """Overlap snapshot output with the run (see the module docstring).

    ``submit(state, t_seconds)`` returns as soon as the copies are enqueued;
    ``close()`` drains the queue, joins the writer thread and closes the
    file.  Tensors on the CPU are written synchronously."""

    def __init__(self, writer, depth=2):
        self.writer = writer
        self.depth = int(depth)
        self._slots = [None] * self.depth  # per slot: {key: (staging, pinned)}, copy-done event
        self._free = queue.Queue()
        for s in range(self.depth):
            self._free.put(s)
        self._jobs = queue.Queue()
        self._error = None
        self._next = 0
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()

    def _run(self):
        while True:
            job = self._jobs.get()
            if job is None:
                return
            slot, event, arrays, t = job
            try:
                if event is not None:
                    event.synchronize()
                self.writer.write_snapshot(arrays, t_seconds=t)
            except Exception as e:  # reported on the next submit or close
                self._error = e
            finally:
                self._free.put(slot)

    def _check(self):
        if self._error is not None:
            err, self._error = self._error, None
            raise RuntimeError("snapshot write failed") from err

    def submit(self, state, t_seconds=None):
        self._check()
        keys = [k for k in self.writer.keys if k in state]
        tensors = {k: state[k] for k in keys}
        on_gpu = any(torch.is_tensor(v) and v.is_cuda for v in tensors.values())
        if not on_gpu:
            self.writer.write_snapshot({k: _host(v) for k, v in tensors.items()}, t_seconds=t_seconds)
            return
        slot = self._free.get()  # waits only while every pinned slot is being written
        bufs, done = self._slots[slot] or ({}, None)
        main = torch.cuda.current_stream()
        if done is not None:
            main.wait_event(done)  # the staging slot's previous host copy has finished
        side = getattr(self, "_side", None)
        if side is None:
            side = self._side = torch.cuda.Stream(device=main.device)
        for k, v in tensors.items():
            b = bufs.get(k)
            if b is None or b[0].shape != v.shape or b[0].dtype != v.dtype:
                staging = torch.empty_strided(tuple(v.shape), tuple(v.stride()), dtype=v.dtype, device=v.device)
                pinned = torch.empty_strided(tuple(v.shape), tuple(v.stride()), dtype=v.dtype, pin_memory=True)
                b = bufs[k] = (staging, pinned)
            b[0].copy_(v)  # device to device on the producing stream
        staged = torch.cuda.Event()
        staged.record(main)
        side.wait_event(staged)
        with torch.cuda.stream(side):
            for k in tensors:
                bufs[k][1].copy_(bufs[k][0], non_blocking=True)
            done = torch.cuda.Event()
            done.record(side)
        self._slots[slot] = (bufs, done)
        self._jobs.put((slot, done, {k: bufs[k][1].numpy() for k in tensors}, t_seconds))

    def close(self):
        self._jobs.put(None)
        self._thread.join()
        self.writer.close()
        self._check()
