"""The class-row shortcut of the server's stem (csrc/stem.cuh: conv1_uaxis,
conv2_uaxis, conv2_pair), checked on the CPU with the convolutions written out
in numpy: for a cube whose values vary along one axis alone, a conv1 output
row is fixed by its index along that axis and, along each other axis, by
which of its three taps leave the grid (class 0: the first, 1: none, 2: the
last); a conv2 output row likewise by its index along the axis and the
classes of the conv1 rows its taps read (0 at the first index, 2 at the last
one when N is odd, else 1). Rows of one class are equal, so computing one row
per class and copying it gives the full convolution's values."""
import numpy as np
import pytest


def conv3d_s2(x, w, b):
    """3^3 convolution, stride 2, zero padding 1, channels last, then ReLU.
    x: [D, D, D, Ci], w: [Co, 27, Ci] (tap = dz * 9 + dy * 3 + dx)."""
    D = x.shape[0]
    Do = (D - 1) // 2 + 1
    xp = np.zeros((D + 2, D + 2, D + 2, x.shape[3]))
    xp[1:D + 1, 1:D + 1, 1:D + 1] = x
    out = np.zeros((Do, Do, Do, w.shape[0]))
    for z in range(Do):
        for y in range(Do):
            for xx in range(Do):
                patch = xp[2 * z:2 * z + 3, 2 * y:2 * y + 3, 2 * xx:2 * xx + 3].reshape(27, -1)
                out[z, y, xx] = np.einsum("tc,otc->o", patch, w) + b
    return np.maximum(out, 0.0)


def c1_class(p, N):
    return 0 if p == 0 else (2 if 2 * p + 1 >= N else 1)


def c2_class(q, N):
    D3 = ((N - 1) // 2) // 2 + 1
    return 0 if q == 0 else (2 if (q == D3 - 1 and N % 2 == 1) else 1)


def split(idx, uaxis):
    """(index along uaxis, first other index, second other index), z-y-x order."""
    z, y, x = idx
    if uaxis == 2:
        return z, y, x
    if uaxis == 1:
        return y, z, x
    return x, z, y


@pytest.mark.parametrize("N", [16, 21, 23])
@pytest.mark.parametrize("uaxis", [0, 1, 2])
def test_rows_of_a_class_are_equal(N, uaxis):
    rng = np.random.default_rng(N * 10 + uaxis)
    vals = rng.uniform(0.2, 1.0, N)
    zz, yy, xx = np.meshgrid(np.arange(N), np.arange(N), np.arange(N), indexing="ij")
    u = (zz, yy, xx)[2 - uaxis]  # the index along uaxis (0 = x, 1 = y, 2 = z)
    cube = vals[u][..., None]
    a1 = conv3d_s2(cube, rng.normal(size=(16, 27, 1)), rng.normal(size=16) * 0.1)
    a2 = conv3d_s2(a1, rng.normal(size=(32, 27, 16)) * 0.3, rng.normal(size=32) * 0.1)
    D2, D3 = a1.shape[0], a2.shape[0]
    # conv1: one class row per (index along uaxis, class, class)
    rows1 = {}
    for idx in np.ndindex(D2, D2, D2):
        pu, pa, pb = split(idx, uaxis)
        key = (pu, c1_class(pa, N), c1_class(pb, N))
        if key in rows1:
            np.testing.assert_array_equal(a1[idx], rows1[key])
        else:
            rows1[key] = a1[idx]
    assert len(rows1) <= 9 * D2
    # conv2: the same with the conv2 classes
    rows2 = {}
    for idx in np.ndindex(D3, D3, D3):
        qu, qa, qb = split(idx, uaxis)
        key = (qu, c2_class(qa, N), c2_class(qb, N))
        if key in rows2:
            np.testing.assert_array_equal(a2[idx], rows2[key])
        else:
            rows2[key] = a2[idx]
    assert len(rows2) <= 9 * D3
    # and the classes are not coarser than the rows: distinct classes differ
    if N % 2 == 1:
        assert len(rows2) == 9 * D3
