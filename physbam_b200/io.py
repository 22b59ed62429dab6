"""PhysBAM's on-disk formats for MPM output and restart (host side).

The reference writes, per frame, into its viewer directory
(`MPM_EXAMPLE::Write_Output_Files`, Hybrid_Methods/Examples_And_Drivers/MPM_EXAMPLE.cpp:53-92;
`VIEWER_DIR`):

    <dir>/common/grid.gz                  GRID: counts, domain (per axis min, max), MAC offset
    <dir>/common/last_frame               the last frame written, as text
    <dir>/<frame>/deformable_object_particles.gz   the particle attributes
    <dir>/<frame>/mpm_particles.gz        a link to the file above
    <dir>/<frame>/restart_data.gz         the time
    <dir>/<frame>/frame_title             empty

and restarts from `mpm_particles` and `restart_data` (`Read_Output_Files`,
l.97-102).  Every file is a gzip stream whose first byte is the stream type
(1: doubles, 0: floats), then `Write_Binary` data in little-endian order.
The particle stream (`PARTICLES::Write`, Tools/Particles/PARTICLES.cpp:364-373)
is version 2: the particle count, the attribute count, and per attribute a
coded type id, its name (int length + bytes) and its array (int count + raw
elements).  The coded id packs the registered element type
(`ATTRIBUTE_INFO::Encode`, PARTICLES.cpp:15-26): id << 20 | scalar << 16 |
m << 12 | n << 8 | element bytes, with the element kinds used for MPM
particles: 1 (scalar), 2 (VECTOR<T,n>), 3 (MATRIX<T,m,n>); bool is id 1 with
scalar code 3.  Matrices are stored column-major (MATRIX::x[i + m j]).
"""
from __future__ import annotations

import gzip
import os
import struct
from typing import Dict, Optional

import numpy as np

# element kinds of the attribute registry
_SCALAR, _VECTOR, _MATRIX = 1, 2, 3
_BOOL_SCALAR_CODE = 3

# the reference's names for the per-particle arrays the library keeps
PARTICLE_ATTRIBUTES = ("X", "V", "F", "B", "mass", "volume", "mu", "lambda", "valid",
                       "Fp", "mu0", "lambda0", "plastic_deformation", "dp_rho_f", "dp_cohesion", "vcp", "color")
# plastic-state keys of the driver (get_plastic_state) -> attribute names
PLASTIC_NAMES = {"Fp": "Fp", "mu0": "mu0", "lam0": "lambda0", "pdef": "plastic_deformation",
                 "rho_F": "dp_rho_f", "cohesion": "dp_cohesion", "vc": "vcp"}


def _coded_id(kind: int, m: int, n: int, use_doubles: bool, bool_elem: bool = False) -> int:
    if bool_elem:
        return (_SCALAR << 20) | (_BOOL_SCALAR_CODE << 16) | 1
    es = 8 if use_doubles else 4
    count = {_SCALAR: 1, _VECTOR: n, _MATRIX: m * n}[kind]
    return (kind << 20) | ((1 if use_doubles else 0) << 16) | (m << 12) | (n << 8) | (es * count)


def write_particles(path: str, arrays: Dict[str, np.ndarray], use_doubles: bool = True):
    """Write a particle collection as `PARTICLES::Write` does.  `arrays` maps attribute
    names to numpy arrays: (n,) scalars, (n, d) vectors, (n, d, d) matrices (row/column as
    numpy indexes them), or (n,) bool; written in name order, as the reference's
    collection keeps them."""
    n = None
    body = []
    ftype = np.float64 if use_doubles else np.float32
    for name in sorted(arrays):
        a = np.asarray(arrays[name])
        if n is None:
            n = a.shape[0]
        if a.shape[0] != n:
            raise ValueError("attribute %s has %d entries, expected %d" % (name, a.shape[0], n))
        if a.dtype == np.bool_ or name == "valid":
            cid, data = _coded_id(_SCALAR, 0, 0, use_doubles, bool_elem=True), np.ascontiguousarray(a, np.uint8)
        elif a.ndim == 1:
            cid, data = _coded_id(_SCALAR, 0, 0, use_doubles), np.ascontiguousarray(a, ftype)
        elif a.ndim == 2:
            cid, data = _coded_id(_VECTOR, 0, a.shape[1], use_doubles), np.ascontiguousarray(a, ftype)
        elif a.ndim == 3:
            # MATRIX<T,m,n>: x[i + m j], i.e. the transpose of numpy's row-major order
            cid = _coded_id(_MATRIX, a.shape[1], a.shape[2], use_doubles)
            data = np.ascontiguousarray(np.swapaxes(a, 1, 2), ftype)
        else:
            raise ValueError("attribute %s: unsupported shape %s" % (name, a.shape))
        nm = name.encode()
        body.append(struct.pack("<ii", cid, len(nm)) + nm + struct.pack("<i", n) + data.tobytes())
    head = struct.pack("<B", 1 if use_doubles else 0) + struct.pack("<iii", 2, n or 0, len(body))
    with gzip.open(path, "wb") as f:
        f.write(head + b"".join(body))


def read_particles(path: str) -> Dict[str, np.ndarray]:
    """Read a version-2 particle stream (`PARTICLES::Read`, PARTICLES.cpp:322-362) into
    numpy arrays shaped as write_particles takes them."""
    with gzip.open(path, "rb") as f:
        b = f.read()
    use_doubles = b[0] == 1
    off = 1
    version, n, na = struct.unpack_from("<iii", b, off)
    off += 12
    if version != 2:
        raise ValueError("particle stream version %d (only version 2 is read)" % version)
    out = {}
    for _ in range(na):
        cid, ln = struct.unpack_from("<ii", b, off)
        off += 8
        name = b[off:off + ln].decode()
        off += ln
        (count,) = struct.unpack_from("<i", b, off)
        off += 4
        kind, sc, m, nn, es = cid >> 20, (cid >> 16) & 0xF, (cid >> 12) & 0xF, (cid >> 8) & 0xF, cid & 0xFF
        nbytes = es * count
        raw = b[off:off + nbytes]
        off += nbytes
        if sc == _BOOL_SCALAR_CODE:
            out[name] = np.frombuffer(raw, np.uint8).astype(bool)
            continue
        dt = np.float64 if (sc == 1 or (sc >= 2 and use_doubles)) else np.float32
        a = np.frombuffer(raw, dt)
        if kind == _SCALAR:
            out[name] = a.copy()
        elif kind == _VECTOR:
            out[name] = a.reshape(count, nn).copy()
        elif kind == _MATRIX:
            out[name] = np.swapaxes(a.reshape(count, nn, m), 1, 2).copy()
        else:
            raise ValueError("attribute %s: element kind %d is not read" % (name, kind))
    return out


def _write_scalar_file(path: str, fmt: str, values, use_doubles: bool = True):
    with gzip.open(path, "wb") as f:
        f.write(struct.pack("<B", 1 if use_doubles else 0) + struct.pack("<" + fmt, *values))


def write_frame(directory: str, frame: int, time: float, particles: Dict[str, np.ndarray],
                counts=None, domain_min=None, domain_max=None, use_doubles: bool = True):
    """One output frame in the reference's viewer layout (see the module docstring);
    `counts` / `domain_*` also write common/grid.gz."""
    fdir = os.path.join(directory, str(frame))
    cdir = os.path.join(directory, "common")
    os.makedirs(fdir, exist_ok=True)
    os.makedirs(cdir, exist_ok=True)
    write_particles(os.path.join(fdir, "deformable_object_particles.gz"), particles, use_doubles)
    link = os.path.join(fdir, "mpm_particles.gz")
    if os.path.lexists(link):
        os.remove(link)
    os.symlink("./deformable_object_particles.gz", link)
    _write_scalar_file(os.path.join(fdir, "restart_data.gz"), "d" if use_doubles else "f", [time], use_doubles)
    open(os.path.join(fdir, "frame_title"), "w").close()
    if counts is not None:
        d = len(counts)
        fmt = "%di%d%s" % (d, 2 * d + 1, "d" if use_doubles else "f")
        rng = [x for k in range(d) for x in (domain_min[k], domain_max[k])]   # RANGE: per axis min, max
        _write_scalar_file(os.path.join(cdir, "grid.gz"), fmt, list(counts) + rng + [0.5], use_doubles)
    with open(os.path.join(cdir, "last_frame"), "w") as f:
        f.write("%d\n" % frame)


def read_restart_time(directory: str, frame: int) -> float:
    with gzip.open(os.path.join(directory, str(frame), "restart_data.gz"), "rb") as f:
        b = f.read()
    return struct.unpack_from("<d" if b[0] == 1 else "<f", b, 1)[0]


def read_grid(directory: str, dim: int):
    """common/grid.gz -> (counts, domain_min, domain_max, MAC offset)."""
    with gzip.open(os.path.join(directory, "common", "grid.gz"), "rb") as f:
        b = f.read()
    ft = "d" if b[0] == 1 else "f"
    counts = struct.unpack_from("<%di" % dim, b, 1)
    vals = struct.unpack_from("<%d%s" % (2 * dim + 1, ft), b, 1 + 4 * dim)
    return list(counts), list(vals[0:2 * dim:2]), list(vals[1:2 * dim:2]), vals[-1]


def read_frame(directory: str, frame: int) -> Dict[str, np.ndarray]:
    """The particle attributes of a frame (through mpm_particles, as the reference
    restarts) and its time under the key "time"."""
    p = os.path.join(directory, str(frame), "mpm_particles.gz")
    if not os.path.exists(p):
        p = os.path.join(directory, str(frame), "deformable_object_particles.gz")
    out = read_particles(p)
    out["time"] = read_restart_time(directory, frame)
    return out
