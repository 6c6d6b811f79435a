"""Host-side logic restated from src/spacetime.jl and src/wavelet.jl, checked the way the
reference's own tests check it (test/spacetime.jl:199-414), on the CPU."""
import numpy as np
import pytest

from wavefd_b200 import spacetime as st


def _rand_points(n, nz, nx, seed, three=False, ny=None):
    rng = np.random.default_rng(seed)
    dz = dx = 10.0
    z = 5 * dz + (dz * (nz - 6) - 5 * dz) * rng.random(n)
    x = 5 * dx + (dx * (nx - 6) - 5 * dx) * rng.random(n)
    if three:
        y = 5 * dx + (dx * (ny - 6) - 5 * dx) * rng.random(n)
        return z, y, x
    return z, x


@pytest.mark.parametrize("fn", ["hicks", "linear"])
def test_ongrid_points_collapse_to_one_with_unit_weight(fn):
    # test/spacetime.jl:306-339
    nz, nx = 50, 60
    z = np.array([10.0 * 7, 10.0 * 20])
    x = np.array([10.0 * 9, 10.0 * 33])
    f = st.hickscoeffs if fn == "hicks" else st.linearcoeffs
    pts = f(10.0, 10.0, 0.0, 0.0, nz, nx, z, x)
    assert len(pts) == 2
    assert np.allclose(pts["c"], 1.0, atol=1e-6)
    assert list(pts["iu"]) == [8 + 9 * nz, 21 + 33 * nz]


@pytest.mark.parametrize("fn", ["hicks", "linear"])
@pytest.mark.parametrize("nthreads", [1, 4])
def test_partitions_share_no_grid_point(fn, nthreads):
    # test/spacetime.jl:199-305
    nz, nx = 100, 100
    z, x = _rand_points(40, nz, nx, 0)
    f = st.hickscoeffs if fn == "hicks" else st.linearcoeffs
    pts = f(10.0, 10.0, 0.0, 0.0, nz, nx, z, x)
    blocks = st.source_blocking(pts, nthreads)
    assert sum(len(b) for b in blocks) == len(pts)
    sets = [set(b["iu"]) for b in blocks]
    for i in range(len(sets)):
        for j in range(len(sets)):
            if i != j:
                assert not (sets[i] & sets[j])
    rblocks = st.receiver_blocking(pts, nthreads)
    rs = [set(b["ir"]) for b in rblocks]
    for i in range(len(rs)):
        for j in range(len(rs)):
            if i != j:
                assert not (rs[i] & rs[j])


@pytest.mark.parametrize("fn", ["hicks", "linear"])
def test_inject_extract_dot_product(oracle, fn):
    # test/spacetime.jl:390-414, on the C restatement
    nz, nx, nr = 100, 100, 10
    z, x = _rand_points(nr, nz, nx, 3)
    f = st.hickscoeffs if fn == "hicks" else st.linearcoeffs
    pts = f(10.0, 10.0, 0.0, 0.0, nz, nx, z, x)
    rng = np.random.default_rng(0)
    f1 = rng.random(nr).astype(np.float32)  # data (nt=1, nr)
    g1 = rng.random(nz * nx).astype(np.float32)
    g2 = np.zeros(nz * nx, np.float32)
    f2 = np.zeros(nr, np.float32)
    oracle.inject(g2, f1, 1, 1, pts["iu"], pts["ir"], pts["c"])
    oracle.extract(f2, g1, 1, 1, pts["iu"], pts["ir"], pts["c"])
    lhs = float(np.dot(f1.astype(np.float64), f2))
    rhs = float(np.dot(g1.astype(np.float64), g2))
    assert abs(lhs - rhs) / abs(lhs + rhs) < 1e-6


def test_hicks_3d_weights_sum_and_free_surface_fold():
    nz, ny, nx = 40, 40, 40
    pts = st.hickscoeffs(10.0, 10.0, 0.0, 0.0, nz, nx, [123.4], [201.7], dy=10.0, y0=0.0, ny=ny, y=[187.2])
    assert len(pts) <= 512 and len(pts) > 300
    assert abs(float(pts["c"].astype(np.float64).sum()) - 1.0) < 0.02
    # near the surface the weights above kz=1 are folded back with a sign flip
    near = st.hickscoeffs(10.0, 10.0, 0.0, 0.0, nz, nx, [5.0], [200.0], dy=10.0, y0=0.0, ny=ny, y=[200.0])
    assert np.all((near["iu"] - 1) % nz < 5 + 4)


def test_blocking_rejects_empty():
    with pytest.raises(ValueError):
        st.source_blocking(np.zeros(0, st.SOURCEPOINT32), 4)


def test_causal_ricker_starts_at_threshold():
    t = 0.001 * np.arange(500)
    w = st.causal_ricker(t, f=15.0)
    assert abs(w[0]) > 1e-4 and abs(w[0]) < 1e-2
    assert 0.99 < np.abs(w).max() <= 1.0
