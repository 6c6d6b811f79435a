"""Born imaging with exact forward fields held by recomputation from checkpoints
(imaging.born_image_checkpointed) against storing every snapshot in device memory
(imaging.born_image with a DeviceStore): the recomputed snapshots come from the same kernels on the
same restored state, so the images are bitwise equal. With a second store passed along (here exact
snapshots in device memory, so that nothing but the imaging path differs), its image, accumulated
through the same adjoint wavefield by the drop-in imaging call, matches the fused imaging step's to
FP32 rounding."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("physics", ["tti", "iso"])
def test_checkpointed_image_equals_device_store(physics):
    import torch

    from wavefd_b200 import imaging
    shape, nt, every = (64, 56, 72), 400, 4
    shot = imaging.make_shot(physics, shape, seed=3, nsponge=12, nt=nt, nrec=(8, 8), horizons=(0.1, 0.6))
    data = imaging.born_data(shot)
    exact, _ = imaging.born_image(shot, data, imaging.DeviceStore(shape, nt // every, 1 + (physics != "iso")),
                                  every=every)
    # segments of 96 steps: the last one is shorter (400 = 4 x 96 + 16)
    ck, secs, none = imaging.born_image_checkpointed(shot, data, every=every, seg=96)
    assert none is None and secs > 0
    assert float(exact.abs().max()) > 0
    assert torch.equal(ck, exact)

    nf = 1 + (physics != "iso")
    ck2, _, ck_l = imaging.born_image_checkpointed(shot, data, every=every, seg=100,
                                                   learned=imaging.DeviceStore(shape, nt // every, nf))
    assert torch.equal(ck2, exact)
    rel = float(torch.linalg.norm(ck_l.double() - exact.double()) / torch.linalg.norm(exact.double()))
    assert rel <= 1e-5, rel
