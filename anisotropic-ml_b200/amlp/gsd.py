"""GSD file format (version 2.0) reader and writer with the HOOMD schema.

Written from the public GSD specification, not from the ``gsd`` package, which
the reference imports (``nep_simulator/GsdHandler.py:2``, ``nep_simulator/Sim.py:5``)
but which is not a dependency of this library.

File layout (all little endian):

* header, 256 bytes: magic ``0x65DF65DF65DF65DF`` (u64), index_location (u64),
  index_allocated_entries (u64), namelist_location (u64),
  namelist_allocated_entries (u64), schema_version (u32), gsd_version (u32),
  application (char[64]), schema (char[64]), reserved (char[80]);
* index: ``index_allocated_entries`` records of 32 bytes: frame (u64), N (u64),
  location (i64), M (u32), id (u16), type (u8), flags (u8); unused records are zero;
* namelist: ``namelist_allocated_entries * 64`` bytes of NUL-terminated chunk
  names, one after the other; a chunk's ``id`` is the position of its name;
* data chunks: ``N * M`` elements of ``type`` each, C order.

HOOMD schema semantics used here (same as the reference relies on in
``GsdHandler.read_system`` ``GsdHandler.py:9-69``): a chunk missing from frame
``k > 0`` takes its value from frame 0; a chunk missing from frame 0 takes the
schema default (mass 1, typeid 0, orientation (1,0,0,0), zeros elsewhere).
"""
from __future__ import annotations

import os
import struct
from dataclasses import dataclass, field

import numpy as np

GSD_MAGIC = 0x65DF65DF65DF65DF
GSD_VERSION_2_0 = (2 << 16) | 0
HOOMD_SCHEMA_VERSION = (1 << 16) | 4
NAME_SIZE = 64
HEADER_SIZE = 256
INDEX_ENTRY_SIZE = 32

_TYPES = {
    1: np.uint8, 2: np.uint16, 3: np.uint32, 4: np.uint64,
    5: np.int8, 6: np.int16, 7: np.int32, 8: np.int64,
    9: np.float32, 10: np.float64, 11: np.uint8,  # 11 = character
}
_TYPE_IDS = {np.dtype(v).str: k for k, v in _TYPES.items() if k != 11}


class GsdError(RuntimeError):
    """Malformed or unsupported GSD file."""


@dataclass
class _Entry:
    frame: int
    N: int
    location: int
    M: int
    id: int
    type: int
    flags: int = 0


# HOOMD schema: per-particle chunk -> (columns, dtype, default value)
_PARTICLE_CHUNKS = {
    "position": (3, np.float32, 0.0),
    "orientation": (4, np.float32, None),  # default (1,0,0,0)
    "typeid": (1, np.uint32, 0),
    "mass": (1, np.float32, 1.0),
    "charge": (1, np.float32, 0.0),
    "diameter": (1, np.float32, 1.0),
    "body": (1, np.int32, -1),
    "moment_inertia": (3, np.float32, 0.0),
    "velocity": (3, np.float32, 0.0),
    "angmom": (4, np.float32, 0.0),
    "image": (3, np.int32, 0),
}


@dataclass
class Frame:
    """One HOOMD-schema frame: configuration plus particle arrays."""

    step: int = 0
    dimensions: int = 3
    box: np.ndarray = field(default_factory=lambda: np.array([1, 1, 1, 0, 0, 0], np.float32))
    N: int = 0
    types: list = field(default_factory=lambda: ["A"])
    particles: dict = field(default_factory=dict)
    log: dict = field(default_factory=dict)

    def get(self, name: str) -> np.ndarray:
        """Particle array ``name`` with the schema default filled in."""
        if name in self.particles:
            return self.particles[name]
        cols, dt, default = _PARTICLE_CHUNKS[name]
        shape = (self.N,) if cols == 1 else (self.N, cols)
        if name == "orientation":
            a = np.zeros(shape, dt)
            a[:, 0] = 1
            return a
        return np.full(shape, default, dtype=dt)


class GsdFile:
    """Random-access reader / appending writer of one GSD 2.0 file."""

    def __init__(self, path: str, mode: str = "r", application: str = "anisotropic-ml-b200",
                 schema: str = "hoomd"):
        if mode not in ("r", "w", "r+", "a"):
            raise ValueError(f"unsupported mode {mode!r}")
        self.path = path
        self.mode = mode
        if mode == "w" or (mode == "a" and not os.path.exists(path)):
            self._create(application, schema)
        self._fh = open(path, "rb" if mode == "r" else "r+b")
        self._load_header()

    # ------------------------------------------------------------------ io
    def _create(self, application: str, schema: str, index_entries: int = 128,
                name_entries: int = 32) -> None:
        hdr = struct.pack("<QQQQQII", GSD_MAGIC, HEADER_SIZE, index_entries,
                          HEADER_SIZE + index_entries * INDEX_ENTRY_SIZE, name_entries,
                          HOOMD_SCHEMA_VERSION, GSD_VERSION_2_0)
        hdr += application.encode()[:63].ljust(64, b"\0") + schema.encode()[:63].ljust(64, b"\0")
        hdr = hdr.ljust(HEADER_SIZE, b"\0")
        with open(self.path, "wb") as fh:
            fh.write(hdr)
            fh.write(b"\0" * (index_entries * INDEX_ENTRY_SIZE))
            fh.write(b"\0" * (name_entries * NAME_SIZE))

    def _load_header(self) -> None:
        fh = self._fh
        fh.seek(0)
        raw = fh.read(HEADER_SIZE)
        if len(raw) < HEADER_SIZE:
            raise GsdError(f"{self.path}: file shorter than the GSD header")
        (magic, self._index_loc, self._index_alloc, self._names_loc, self._names_alloc,
         self.schema_version, self.gsd_version) = struct.unpack("<QQQQQII", raw[:48])
        if magic != GSD_MAGIC:
            raise GsdError(f"{self.path}: not a GSD file (bad magic)")
        if self.gsd_version >> 16 != 2:
            raise GsdError(f"{self.path}: GSD version {self.gsd_version >> 16}.{self.gsd_version & 0xffff}"
                           " is not supported (only 2.x)")
        self.application = raw[48:112].split(b"\0")[0].decode()
        self.schema = raw[112:176].split(b"\0")[0].decode()
        fh.seek(self._names_loc)
        blob = fh.read(self._names_alloc * NAME_SIZE)
        self._names = [n.decode() for n in blob.rstrip(b"\0").split(b"\0")] if blob.strip(b"\0") else []
        fh.seek(self._index_loc)
        blob = fh.read(self._index_alloc * INDEX_ENTRY_SIZE)
        self._entries: list[_Entry] = []
        for k in range(self._index_alloc):
            rec = blob[k * INDEX_ENTRY_SIZE:(k + 1) * INDEX_ENTRY_SIZE]
            if len(rec) < INDEX_ENTRY_SIZE:
                raise GsdError(f"{self.path}: truncated index")
            e = _Entry(*struct.unpack("<QQqIHBB", rec))
            if e.location == 0:
                break
            if e.type not in _TYPES or e.id >= len(self._names):
                raise GsdError(f"{self.path}: corrupt index entry {k}")
            self._entries.append(e)
        self._nframes = (self._entries[-1].frame + 1) if self._entries else 0

    def close(self) -> None:
        if self._fh is not None:
            self._fh.close()
            self._fh = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __len__(self) -> int:
        return self._nframes

    # ------------------------------------------------------------------ read
    def chunk_names(self, frame: int) -> list[str]:
        return [self._names[e.id] for e in self._entries if e.frame == frame]

    def read_chunk(self, frame: int, name: str):
        """Array stored under ``name`` in ``frame`` or None."""
        if name not in self._names:
            return None
        cid = self._names.index(name)
        for e in self._entries:
            if e.frame == frame and e.id == cid:
                dt = _TYPES[e.type]
                self._fh.seek(e.location)
                nbytes = e.N * e.M * np.dtype(dt).itemsize
                buf = self._fh.read(nbytes)
                if len(buf) != nbytes:
                    raise GsdError(f"{self.path}: chunk {name} of frame {frame} is truncated")
                a = np.frombuffer(buf, dtype=dt).copy()
                if e.type == 11:
                    return a.tobytes()
                return a.reshape(e.N, e.M) if e.M > 1 else a
        return None

    def _chunk(self, frame: int, name: str):
        v = self.read_chunk(frame, name)
        if v is None and frame != 0:
            v = self.read_chunk(0, name)
        return v

    def read_frame(self, frame: int) -> Frame:
        if frame < 0:
            frame += self._nframes
        if not 0 <= frame < self._nframes:
            raise IndexError(f"frame {frame} out of range (file has {self._nframes})")
        f = Frame()
        step = self._chunk(frame, "configuration/step")
        f.step = int(step[0]) if step is not None else 0
        dim = self._chunk(frame, "configuration/dimensions")
        f.dimensions = int(dim[0]) if dim is not None else 3
        box = self._chunk(frame, "configuration/box")
        f.box = box.astype(np.float32).reshape(6) if box is not None else np.array([1, 1, 1, 0, 0, 0], np.float32)
        n = self._chunk(frame, "particles/N")
        f.N = int(n[0]) if n is not None else 0
        types = self._chunk(frame, "particles/types")
        if types is not None:
            arr = np.atleast_2d(types)
            f.types = [bytes(r).split(b"\0")[0].decode() for r in arr]
        for name, (cols, dt, _) in _PARTICLE_CHUNKS.items():
            v = self._chunk(frame, "particles/" + name)
            if v is not None:
                v = v.astype(dt)
                f.particles[name] = v.reshape(f.N) if cols == 1 else v.reshape(f.N, cols)
        for nm in self._names:
            if nm.startswith("log/"):
                v = self.read_chunk(frame, nm)
                if v is not None:
                    f.log[nm[4:]] = v
        return f

    def __getitem__(self, k: int) -> Frame:
        return self.read_frame(k)

    # ------------------------------------------------------------------ write
    def _name_id(self, name: str) -> int:
        if name in self._names:
            return self._names.index(name)
        used = sum(len(n) + 1 for n in self._names)
        if used + len(name) + 1 > self._names_alloc * NAME_SIZE:
            # relocate the namelist to the end of the file with twice the room
            self._names_alloc *= 2
            self._fh.seek(0, os.SEEK_END)
            self._names_loc = self._fh.tell()
            self._fh.write(b"\0" * (self._names_alloc * NAME_SIZE))
        self._names.append(name)
        blob = b"".join(n.encode() + b"\0" for n in self._names)
        self._fh.seek(self._names_loc)
        self._fh.write(blob.ljust(self._names_alloc * NAME_SIZE, b"\0"))
        self._write_header()
        return len(self._names) - 1

    def _write_header(self) -> None:
        self._fh.seek(8)
        self._fh.write(struct.pack("<QQQQ", self._index_loc, self._index_alloc,
                                   self._names_loc, self._names_alloc))

    def _write_index(self) -> None:
        if len(self._entries) > self._index_alloc:
            while len(self._entries) > self._index_alloc:
                self._index_alloc *= 2
            self._fh.seek(0, os.SEEK_END)
            self._index_loc = self._fh.tell()
            self._fh.write(b"\0" * (self._index_alloc * INDEX_ENTRY_SIZE))
            self._write_header()
        blob = b"".join(struct.pack("<QQqIHBB", e.frame, e.N, e.location, e.M, e.id, e.type, e.flags)
                        for e in self._entries)
        self._fh.seek(self._index_loc)
        self._fh.write(blob)

    def write_chunk(self, name: str, data, frame: int | None = None) -> None:
        if self.mode == "r":
            raise GsdError("file opened read-only")
        frame = self._nframes if frame is None else frame
        if isinstance(data, (bytes, bytearray)):
            arr, tid = np.frombuffer(bytes(data), np.uint8), 11
        else:
            arr = np.ascontiguousarray(data)
            if arr.ndim == 0:
                arr = arr.reshape(1)
            tid = _TYPE_IDS.get(arr.dtype.str)
            if tid is None:
                raise GsdError(f"dtype {arr.dtype} cannot be stored in GSD")
        N = arr.shape[0]
        M = int(np.prod(arr.shape[1:])) if arr.ndim > 1 else 1
        cid = self._name_id(name)
        self._fh.seek(0, os.SEEK_END)
        loc = self._fh.tell()
        self._fh.write(arr.tobytes())
        self._entries.append(_Entry(frame, N, loc, M, cid, tid, 0))
        self._pending_frame = frame

    def end_frame(self) -> None:
        self._entries.sort(key=lambda e: (e.frame, e.id))
        self._write_index()
        self._fh.flush()
        self._nframes = (self._entries[-1].frame + 1) if self._entries else 0

    def append(self, f: Frame) -> None:
        """Write ``f`` as the next frame (HOOMD schema)."""
        k = self._nframes
        self.write_chunk("configuration/step", np.array([f.step], np.uint64), k)
        self.write_chunk("configuration/dimensions", np.array([f.dimensions], np.uint8), k)
        self.write_chunk("configuration/box", np.asarray(f.box, np.float32).reshape(6), k)
        self.write_chunk("particles/N", np.array([f.N], np.uint32), k)
        width = max(len(t) for t in f.types) + 1
        tarr = np.zeros((len(f.types), width), np.uint8)
        for r, t in enumerate(f.types):
            tarr[r, :len(t)] = np.frombuffer(t.encode(), np.uint8)
        self.write_chunk("particles/types", tarr, k)
        for name, (cols, dt, _) in _PARTICLE_CHUNKS.items():
            if name in f.particles:
                v = np.asarray(f.particles[name]).astype(dt)
                self.write_chunk("particles/" + name, v.reshape(f.N, cols) if cols > 1 else v.reshape(f.N), k)
        for name, v in f.log.items():
            self.write_chunk("log/" + name, np.asarray(v), k)
        self.end_frame()


def read_last_frame(path: str) -> Frame:
    with GsdFile(path, "r") as g:
        if len(g) == 0:
            raise GsdError(f"{path}: file has no frames")
        return g.read_frame(len(g) - 1)
