"""Checkpoints with the content and layout of the reference's restart files
(escru.F90:9-251 escribezy + writeheader escru.F90:950-995, read back by
getstartzy-bg.F90 h5load + readheader :490-581).

The reference writes one HDF5 file per variable, <chfile>.<ifile:03d>.<var>
.h5 for var in u, v, w, p, each holding the dataset "value" as big-endian
REAL4 (H5T_IEEE_F32BE) of Fortran shape (nz1, ny(+1), nx), which is the C
array [nx][ny(+1)][nz1] of the plane layout, and the header datasets
Variable (string), tiempo, cfl, Re, lx, ly, lz (float64), nx, ny, nz2, xout,
procs (int32), timeinit, dt (float64), y (ny+2) and um (ny+1). The right-hand
side history is not written: a restart starts it from zero.

No HDF5 library is available to this package, so the same datasets go into
a self-describing container, <chfile>.<ifile:03d>.<var>.otc: the magic
b"OTBLCKP1", a little-endian u64 header length, a JSON list of
{name, dtype (numpy str), shape, offset, nbytes}, then the raw arrays, each
with its declared byte order. `to_hdf5` writes the reference's .h5 files
from a checkpoint when h5py is importable.
"""
from __future__ import annotations

import json
import math
import os
import struct

import numpy as np


MAGIC = b"OTBLCKP1"
VARS = ("u", "v", "w", "p")


def write_container(path: str, datasets: list) -> None:
    """datasets: (name, numpy array) pairs, written with their own dtype."""
    arrs = [(n, np.ascontiguousarray(a)) for n, a in datasets]
    meta, off = [], 0
    for n, a in arrs:
        meta.append({"name": n, "dtype": a.dtype.str, "shape": list(a.shape), "offset": off,
                     "nbytes": int(a.nbytes)})
        off += int(a.nbytes)
    head = json.dumps(meta).encode()
    tmp = path + ".tmp"
    with open(tmp, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<Q", len(head)))
        f.write(head)
        for _, a in arrs:
            f.write(a.tobytes())
    os.replace(tmp, path)


def read_container(path: str) -> dict:
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise ValueError(f"{path}: not a checkpoint container")
        (hl,) = struct.unpack("<Q", f.read(8))
        meta = json.loads(f.read(hl).decode())
        base = f.tell()
        out = {}
        for m in meta:
            f.seek(base + m["offset"])
            buf = f.read(m["nbytes"])
            out[m["name"]] = np.frombuffer(buf, dtype=np.dtype(m["dtype"])).reshape(m["shape"]).copy()
    return out


def file_name(chfile: str, ifile: int, var: str) -> str:
    """escru.F90:39-42: chfile.NNN.var (plus the container extension)."""
    return f"{chfile}.{ifile:03d}.{var}.otc"


def header(box, var: str, procs: int = 1) -> list:
    """writeheader (escru.F90:950-995) of a box: lx = ax*pi, ly, lz = 2*pi*az."""
    cfg = box.cfg
    um, st = box.inflow()
    f64 = lambda x: np.array([x], dtype="<f8")
    i32 = lambda x: np.array([x], dtype="<i4")
    return [("Variable", np.frombuffer(var.encode(), dtype="S1").copy()),
            ("tiempo", f64(st["tiempo"])), ("cfl", f64(cfg.cfl)), ("Re", f64(box.re)),
            ("lx", f64(cfg.ax * math.pi)), ("ly", f64(cfg.ly)), ("lz", f64(cfg.az * 2 * math.pi)),
            ("nx", i32(cfg.nx)), ("ny", i32(cfg.ny)), ("nz2", i32(cfg.nz2)),
            ("xout", i32(box.xout)), ("procs", i32(procs)),
            ("timeinit", f64(st["timeinit"])), ("dt", f64(st["dt"])),
            ("y", np.asarray(box.y, dtype="<f8")), ("um", np.asarray(um, dtype="<f8"))]


def write(box, chfile: str, ifile: int) -> list:
    """escribezy (escru.F90:9): u, v, w, p of a Box as REAL4 with the header;
    returns the file names."""
    box.sync()
    names = []
    for var in VARS:
        value = box.field(var).astype(">f4")   # real(u, kind=4), H5T_IEEE_F32BE
        path = file_name(chfile, ifile, var)
        write_container(path, [("value", value)] + header(box, var))
        names.append(path)
    return names


def read(chfile: str, ifile: int) -> dict:
    """The restart state in the form Box/make_initial use: u, v, w, p as
    float64 (from REAL4), a zero right-hand-side history, y, re, xout, the
    inlet profiles u0 = u(k=0, :, 1) and v0 (getstartzy-bg.F90:273-276),
    um, tiempo, timeinit and dt (readheader)."""
    d = {var: read_container(file_name(chfile, ifile, var)) for var in VARS}
    h = d["u"]
    for var in VARS:
        if bytes(d[var]["Variable"].tobytes()).decode() != var:
            raise ValueError(f"checkpoint {chfile}.{ifile:03d}.{var}: Variable mismatch")
    nx, ny, nz2 = int(h["nx"][0]), int(h["ny"][0]), int(h["nz2"][0])
    nz1 = 2 * (nz2 + 1)
    st = {var: d[var]["value"].astype(np.float64) for var in VARS}
    if st["u"].shape != (nx, ny + 1, nz1) or st["v"].shape != (nx, ny, nz1):
        raise ValueError("checkpoint dimensions do not match its header")
    return dict(
        u=st["u"], v=st["v"], w=st["w"], p=st["p"],
        rhsupa=np.zeros((nx, ny + 1, nz1)), rhsvpa=np.zeros((nx, ny, nz1)),
        rhswpa=np.zeros((nx, ny + 1, nz1)),
        y=h["y"].astype(np.float64), re=float(h["Re"][0]), xout=int(h["xout"][0]),
        u0=st["u"][0, :, 0].copy(), v0=st["v"][0, :, 0].copy(), um=h["um"].astype(np.float64),
        tiempo=float(h["tiempo"][0]), timeinit=float(h["timeinit"][0]), dt=float(h["dt"][0]),
        cfl=float(h["cfl"][0]), lx=float(h["lx"][0]), ly=float(h["ly"][0]), lz=float(h["lz"][0]))


def to_hdf5(chfile: str, ifile: int) -> list:
    """The reference's own files (<chfile>.NNN.var.h5, datasets as written by
    escribezy/writeheader) from a checkpoint; needs h5py."""
    import h5py  # not part of this image; the export runs where it is installed
    out = []
    for var in VARS:
        d = read_container(file_name(chfile, ifile, var))
        path = f"{chfile}.{ifile:03d}.{var}.h5"
        with h5py.File(path, "w") as f:
            for name, a in d.items():
                if name == "Variable":
                    f.create_dataset(name, data=np.bytes_(a.tobytes()))
                else:
                    f.create_dataset(name, data=a)
        out.append(path)
    return out
