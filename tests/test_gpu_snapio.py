"""Snapshot files with device arrays: writes are ordered on the caller's stream (the source may be
overwritten by the next work on that stream), reads in any order with prefetch, the index on disk,
O_DIRECT, codec codes as payloads, and a Born image whose forward fields went through a snapshot
file, which must equal the image with the fields kept in device memory bit for bit (plain FP32
storage is exact)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


@pytest.mark.parametrize("direct", [False, True])
def test_device_round_trip(torch, tmp_path, direct):
    from wavefd_b200.snapio import SnapshotFile, read_index
    p = tmp_path / "d.snap"
    g = torch.Generator(device="cuda").manual_seed(3)
    sizes = [1 << 20, (1 << 20) + 37, 123457, 1 << 18, 999, 1 << 20]
    ref = [torch.randn(n, device="cuda", generator=g) for n in sizes]
    s = torch.cuda.Stream()
    src = torch.empty(max(sizes), device="cuda")
    with SnapshotFile(p, "w", len(sizes), 4 * max(sizes), direct=direct) as f:
        with torch.cuda.stream(s):
            for i, r in enumerate(ref):
                src[:r.numel()].copy_(r)
                f.write(i, src[:r.numel()], s)
                src.fill_(-7.0)  # the next work on the stream may overwrite the source
        # reads before the writes have landed wait for them; reverse order with prefetch
        outs = [torch.full_like(r, 5.0) for r in ref]
        with torch.cuda.stream(s):
            for i in reversed(range(len(sizes))):
                f.read(i, outs[i], s)
                if i > 0:
                    f.prefetch(i - 1)
        s.synchronize()
        for r, o in zip(ref, outs):
            assert torch.equal(r, o)
    flags, nf, slot, data, idx = read_index(p)
    assert nf == len(sizes) and [ln for _, ln in idx] == [4 * n for n in sizes]
    # reopen for reading, random order
    with SnapshotFile(p, "r", direct=direct) as f:
        for i in [2, 5, 0, 4, 1, 3]:
            o = torch.zeros_like(ref[i])
            f.read(i, o)
            torch.cuda.synchronize()
            assert torch.equal(o, ref[i])


def test_codec_codes_as_payload(torch, tmp_path):
    from wavefd_b200.codec import WavefieldCodec
    from wavefd_b200.snapio import CODEC, SnapshotFile
    shape = (40, 48, 56)
    codec = WavefieldCodec(seed=2)
    x = torch.linspace(0, 6.0, int(np.prod(shape)), device="cuda").reshape(shape)
    field = torch.sin(x) * torch.cos(0.5 * x)
    code = codec.empty_code(shape)
    codec.encode(field, shape, code)
    p = tmp_path / "c.snap"
    with SnapshotFile(p, "w", 4, code.numel(), codec=True) as f:
        f.write(2, code)
        back = torch.zeros_like(code)
        f.read(2, back)
        torch.cuda.synchronize()
        assert f.flags == CODEC
    assert torch.equal(back, code)
    a, b = torch.empty(shape, device="cuda"), torch.empty(shape, device="cuda")
    codec.decode(code, shape, a)
    codec.decode(back, shape, b)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_born_image_through_a_snapshot_file_is_exact(torch, tmp_path):
    from wavefd_b200 import imaging
    shot = imaging.make_shot("tti", (64, 64, 64), seed=7, nsponge=12, nt=240, nrec=(12, 12))
    data = imaging.born_data(shot)
    nsnap, nf = 240 // 4, 2
    img_dev, _ = imaging.born_image(shot, data, imaging.DeviceStore(shot["shape"], nsnap, nf), every=4)
    store = imaging.DiskStore(shot["shape"], nsnap, nf, tmp_path / "born.snap")
    img_disk, _ = imaging.born_image(shot, data, store, every=4)
    store.close()
    assert not os.path.exists(tmp_path / "born.snap")
    assert float(img_dev.abs().max()) > 0
    assert torch.equal(img_dev, img_disk)
