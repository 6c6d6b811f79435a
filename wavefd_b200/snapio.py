"""Snapshot files: saved forward wavefields on disk with an offsets/lengths index.

The role of `Compressor` / `compressedwrite` / `compressedread!` (src/compressedio.jl:1-137): the
forward run writes field i of the file once, the adjoint run reads the fields back in any order.
The work is done by the library's `WFD_Snap_*` entry points (wavefd_b200/csrc/wfd_snapio.cu):
device arrays move through device and pinned staging and a worker thread's pwrite/pread, ordered
on the caller's CUDA stream; host arrays (numpy) go straight through pwrite/pread.

File layout (little-endian): a header of a multiple of 4096 bytes ("WFDSNAP1", u32 version, u32
flags, i64 nfields, i64 slot, i64 data offset, then per field i64 offset and i64 length, -1 =
never written), then field i's payload at data offset + i * slot.
"""
from __future__ import annotations

import struct

import numpy as np

from . import _lib

READ, HOST, DIRECT, CODEC = 1, 2, 4, 8
MAGIC = b"WFDSNAP1"


def _addr(a):
    """(pointer, bytes, is_host) of a contiguous torch tensor or numpy array."""
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("snapshot arrays must be C-contiguous")
        return a.ctypes.data, a.nbytes, True
    if not a.is_contiguous():
        raise ValueError("snapshot arrays must be contiguous")
    return a.data_ptr(), a.numel() * a.element_size(), not a.is_cuda


class SnapshotFile:
    """Open a snapshot file. mode "w": create (or truncate) with `nfields` slots of up to
    `max_bytes` each; mode "r": open an existing file. host=True: the arrays are numpy arrays
    (no CUDA use); otherwise CUDA tensors, with the transfers ordered on `stream` (a
    torch.cuda.Stream, default the current one). direct=True asks for O_DIRECT."""

    def __init__(self, path, mode="w", nfields=0, max_bytes=0, host=False, direct=False, codec=False):
        self.lib = _lib.library()
        flags = (READ if mode == "r" else 0) | (HOST if host else 0) | (DIRECT if direct else 0) | (CODEC if codec else 0)
        self.host = host
        self.path = str(path)
        self.f = self.lib.WFD_Snap_Open(self.path.encode(), int(nfields), int(max_bytes), flags)
        if not self.f:
            raise _lib.WaveFDError(f"WFD_Snap_Open({self.path}): {self.lib.WFD_LastErrorMessage().decode()}")

    def _stream(self, stream):
        if self.host:
            return None
        import torch
        s = stream if stream is not None else torch.cuda.current_stream()
        return s.cuda_stream

    @property
    def nfields(self):
        return self.lib.WFD_Snap_NumFields(self.f)

    @property
    def flags(self):
        return self.lib.WFD_Snap_Flags(self.f)

    def length(self, i):
        return self.lib.WFD_Snap_Length(self.f, int(i))

    def write(self, i, array, stream=None):
        p, n, _ = _addr(array)
        _lib.check(self.lib.WFD_Snap_Write(self.f, int(i), p, n, self._stream(stream)), f"WFD_Snap_Write({i})")

    def prefetch(self, i):
        _lib.check(self.lib.WFD_Snap_Prefetch(self.f, int(i)), f"WFD_Snap_Prefetch({i})")

    def read(self, i, out, stream=None):
        p, n, _ = _addr(out)
        _lib.check(self.lib.WFD_Snap_Read(self.f, int(i), p, n, self._stream(stream)), f"WFD_Snap_Read({i})")
        return out

    def sync(self):
        _lib.check(self.lib.WFD_Snap_Sync(self.f), "WFD_Snap_Sync")

    def close(self):
        if self.f:
            f, self.f = self.f, None
            _lib.check(self.lib.WFD_Snap_Close(f), "WFD_Snap_Close")

    def __enter__(self):
        return self

    def __exit__(self, etype, *exc):
        if etype is None:
            self.close()
        elif self.f:  # already failing: close without raising a second error
            f, self.f = self.f, None
            self.lib.WFD_Snap_Close(f)

    def __del__(self):
        if getattr(self, "f", None):
            self.lib.WFD_Snap_Close(self.f)
            self.f = None


def read_index(path):
    """(flags, nfields, slot, data offset, [(offset, length)] per field) from a file's header."""
    with open(path, "rb") as fh:
        head = fh.read(48)
        if head[:8] != MAGIC:
            raise ValueError(f"{path}: not a snapshot file")
        version, flags = struct.unpack_from("<II", head, 8)
        nfields, slot, data = struct.unpack_from("<qqq", head, 16)
        if version != 1:
            raise ValueError(f"{path}: unsupported version {version}")
        idx = struct.unpack(f"<{2 * nfields}q", fh.read(16 * nfields))
    return flags, nfields, slot, data, [(idx[2 * i], idx[2 * i + 1]) for i in range(nfields)]
