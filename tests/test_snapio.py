"""Snapshot files on the host path (no GPU): the on-disk layout (header, offsets/lengths index,
4096-aligned slots) read back by an independent parser, random-order writes and reads, rewriting a
field, and the error behaviour of compressedio.jl:35-40 / :62-66 (a short write names the bytes
written and the file; the file's later calls report it), plus the argument errors."""
import os
import struct

import numpy as np
import pytest

snapio = pytest.importorskip("wavefd_b200.snapio")
from wavefd_b200 import _lib  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("library not built")


def _fields(n, seed=0):
    rng = np.random.default_rng(seed)
    return [rng.standard_normal(500 + 97 * i).astype(np.float32) for i in range(n)]


def test_layout_and_round_trip(tmp_path):
    p = tmp_path / "a.snap"
    arrs = _fields(6)
    order = [4, 1, 5, 0, 2]  # field 3 never written
    with snapio.SnapshotFile(p, "w", 6, 4 * 2000, host=True) as f:
        for i in order:
            f.write(i, arrs[i])
    flags, nf, slot, data, idx = snapio.read_index(p)
    assert (flags, nf) == (0, 6)
    assert slot == 8192 and data == 4096 and data % 4096 == 0
    raw = p.read_bytes()
    assert raw[:8] == b"WFDSNAP1" and struct.unpack_from("<I", raw, 8)[0] == 1
    for i in range(6):
        off, ln = idx[i]
        assert off == data + i * slot
        if i == 3:
            assert ln == -1
        else:
            assert ln == arrs[i].nbytes
            assert np.array_equal(np.frombuffer(raw[off:off + ln], dtype=np.float32), arrs[i])
    with snapio.SnapshotFile(p, "r", host=True) as f:
        assert f.nfields == 6 and f.flags == 0
        assert [f.length(i) for i in range(6)] == [a.nbytes if i != 3 else -1 for i, a in enumerate(arrs)]
        for i in [5, 2, 0, 4, 1]:
            out = np.zeros(arrs[i].size + 3, dtype=np.float32)  # a larger buffer is fine
            f.read(i, out)
            assert np.array_equal(out[:arrs[i].size], arrs[i])


def test_rewrite_and_codec_flag(tmp_path):
    p = tmp_path / "b.snap"
    a, b = np.arange(100, dtype=np.uint8), np.arange(60, dtype=np.uint8)[::-1].copy()
    with snapio.SnapshotFile(p, "w", 2, 100, host=True, codec=True) as f:
        f.write(1, a)
        f.write(1, b)  # the second write of a field wins, with its own length
    flags, nf, slot, data, idx = snapio.read_index(p)
    assert flags == snapio.CODEC and idx[1][1] == 60 and idx[0][1] == -1
    with snapio.SnapshotFile(p, "r", host=True) as f:
        out = np.zeros(60, dtype=np.uint8)
        f.read(1, out)
        assert np.array_equal(out, b)


def test_argument_errors_do_not_poison_the_file(tmp_path):
    p = tmp_path / "c.snap"
    x = np.ones(10, dtype=np.float32)
    with snapio.SnapshotFile(p, "w", 2, 40, host=True) as f:
        with pytest.raises(_lib.WaveFDError, match="bad arguments"):
            f.write(2, x)  # field out of range
        with pytest.raises(_lib.WaveFDError, match="bad arguments"):
            f.write(0, np.ones(1025, dtype=np.float32))  # larger than the slot (max_bytes rounded up to 4096)
        with pytest.raises(_lib.WaveFDError, match="never written"):
            f.read(1, x.copy())
        f.write(0, x)
    with snapio.SnapshotFile(p, "r", host=True) as f:
        with pytest.raises(_lib.WaveFDError, match="larger than the buffer"):
            f.read(0, np.zeros(5, dtype=np.float32))
        with pytest.raises(_lib.WaveFDError, match="bad arguments"):
            f.write(0, x)  # read-only


def test_open_errors(tmp_path):
    with pytest.raises(_lib.WaveFDError, match="cannot open"):
        snapio.SnapshotFile(tmp_path / "missing.snap", "r", host=True)
    bad = tmp_path / "bad.snap"
    bad.write_bytes(b"NOTASNAP" + bytes(100))
    with pytest.raises(_lib.WaveFDError, match="not a snapshot file"):
        snapio.SnapshotFile(bad, "r", host=True)
    with pytest.raises(_lib.WaveFDError, match="must be positive"):
        snapio.SnapshotFile(tmp_path / "z.snap", "w", 0, 10, host=True)


@pytest.mark.skipif(not os.path.exists("/dev/full"), reason="no /dev/full")
def test_short_write_is_an_io_error_naming_the_bytes():
    f = snapio.SnapshotFile("/dev/full", "w", 2, 4096, host=True)
    with pytest.raises(_lib.WaveFDError, match=r"status 6.*wrote 0 of 400 bytes of field 1 in /dev/full"):
        f.write(1, np.zeros(100, dtype=np.float32))
    # the I/O error stays with the file
    with pytest.raises(_lib.WaveFDError, match="status 6"):
        f.write(0, np.zeros(100, dtype=np.float32))
    with pytest.raises(_lib.WaveFDError, match="status 6"):
        f.close()
