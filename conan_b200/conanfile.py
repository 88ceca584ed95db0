"""Reader and writer of the reference's `.conan` container format.

Layout (src/base/misc.hh:27-78, src/base/header.cc:30-74,
src/base/history.cc:20-75, src/base/array.hh:75-105):

  block   := uint64 nbytes, nbytes of payload, uint64 nbytes   (native endian)
  file    := header-block history-block (record-header-block data-block)*
  header  := "key=value\\n" lines in std::map (byte-wise sorted) key order
  history := "seconds-since-epoch:command line\\n" lines in time order
  record  := header with keys dtype, name; data block of raw values

dtype names follow src/base/mtypeid.cc:49-64 (float64, 3f8, ...).
"""
from __future__ import annotations

import struct
import time
from typing import Dict, List, Tuple

import numpy as np

DTYPES = {
    "int32": (np.int32, 1), "uint32": (np.uint32, 1), "float32": (np.float32, 1),
    "float64": (np.float64, 1), "complex64": (np.complex64, 1), "complex128": (np.complex128, 1),
    "3i4": (np.int32, 3), "2i4": (np.int32, 2), "3f4": (np.float32, 3), "2f4": (np.float32, 2),
    "3f8": (np.float64, 3), "2f8": (np.float64, 2),
}


def write_block(f, payload: bytes):
    n = struct.pack("<Q", len(payload))
    f.write(n)
    f.write(payload)
    f.write(n)


def read_block(f) -> bytes:
    s = f.read(8)
    if len(s) < 8:
        raise IOError("Could not read from file")
    (n,) = struct.unpack("<Q", s)
    data = f.read(n)
    t = f.read(8)
    if len(data) != n or len(t) < 8 or struct.unpack("<Q", t)[0] != n:
        raise IOError("The block seems to be corrupted")
    return data


def skip_block(f):
    s = f.read(8)
    if len(s) < 8:
        raise IOError("Could not read from file")
    (n,) = struct.unpack("<Q", s)
    f.seek(n, 1)
    t = f.read(8)
    if len(t) < 8 or struct.unpack("<Q", t)[0] != n:
        raise IOError("The block seems to be corrupted")


def _strip(v: str) -> str:
    return str(v).split("\n", 1)[0]


def header_bytes(h: Dict[str, str]) -> bytes:
    keys = sorted(h.keys(), key=lambda k: k.encode())
    return "".join(f"{k}={_strip(h[k])}\n" for k in keys).encode()


def parse_header(raw: bytes) -> Dict[str, str]:
    out: Dict[str, str] = {}
    s = raw.decode()
    pos = 0
    while pos < len(s):
        p1 = s.find("=", pos)
        p2 = s.find("\n", pos)
        out.setdefault(s[pos:p1], s[p1 + 1:p2])  # std::map::insert keeps the first
        pos = p2 + 1
    return out


def history_bytes(hist: List[Tuple[int, str]]) -> bytes:
    return "".join(f"{t}:{_strip(c)}\n" for t, c in sorted(hist, key=lambda x: x[0])).encode()


def parse_history(raw: bytes) -> List[Tuple[int, str]]:
    out = []
    s = raw.decode()
    pos = 0
    while pos < len(s):
        p1 = s.find(":", pos)
        p2 = s.find("\n", pos)
        out.append((int(s[pos:p1]), s[p1 + 1:p2]))
        pos = p2 + 1
    return sorted(out, key=lambda x: x[0])


def dtype_name(a: np.ndarray) -> str:
    comp = 1 if a.ndim == 1 else a.shape[-1]
    for name, (dt, c) in DTYPES.items():
        if np.dtype(dt) == a.dtype and c == comp:
            return name
    raise ValueError(f"no .conan dtype for {a.dtype} x {comp}")


class ConanFile:
    """In-memory .conan file: header dict, history list, named records."""

    def __init__(self, header=None, history=None):
        self.header: Dict[str, str] = dict(header or {})
        self.history: List[Tuple[int, str]] = list(history or [])
        self.records: Dict[str, np.ndarray] = {}
        self.order: List[str] = []

    def add(self, name: str, data: np.ndarray):
        if name not in self.records:
            self.order.append(name)
        self.records[name] = np.ascontiguousarray(data)

    def update_history(self, command: str, t: int = None):
        self.history.append((int(time.time()) if t is None else int(t), command))

    def write(self, path: str):
        with open(path, "wb") as f:
            write_block(f, header_bytes(self.header))
            write_block(f, history_bytes(self.history))
            for name in self.order:
                a = self.records[name]
                write_block(f, header_bytes({"name": name, "dtype": dtype_name(a)}))
                write_block(f, a.tobytes())

    @classmethod
    def read(cls, path: str) -> "ConanFile":
        c = cls()
        with open(path, "rb") as f:
            c.header = parse_header(read_block(f))
            c.history = parse_history(read_block(f))
            while True:
                try:
                    sub = parse_header(read_block(f))
                except IOError:
                    break
                data = read_block(f)
                dt, comp = DTYPES.get(sub.get("dtype", "float64"), (np.uint8, 1))
                a = np.frombuffer(data, dtype=dt).copy()
                if comp > 1:
                    a = a.reshape(-1, comp)
                c.add(sub.get("name", f"record{len(c.order)}"), a)
        return c
