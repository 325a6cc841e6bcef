"""The image-preparation oracle (oracle/image.cpp) against independent numpy restatements of
frontend/src/app/vision/image/gray-image.ts and mvs/depth-maps.ts:9-42."""
import numpy as np
import pytest

import oracle


def _js_round(x):
    f = np.floor(x)
    return np.where(x - f >= 0.5, f + 1, f)


def _rgba(h, w, seed=0):
    return np.random.default_rng(seed).integers(0, 256, size=(h, w, 4), dtype=np.uint8)


@pytest.mark.parametrize("shape,target", [((48, 64), (16, 12)), ((30, 40), (40, 30)), ((24, 24), (24, 24))])
def test_gray_integer_ratio_is_the_block_mean(shape, target):
    h, w = shape
    tw, th = target
    if w % tw or h % th:
        pytest.skip("not an integer ratio")
    a = _rgba(h, w)
    c = a.astype(np.int64)
    luma = 77 * c[..., 0] + 150 * c[..., 1] + 29 * c[..., 2]
    blocks = luma.reshape(th, h // th, tw, w // tw).sum((1, 3)).astype(np.float64)
    want = _js_round(blocks / (256 * (h // th) * (w // tw))).astype(np.uint8)
    np.testing.assert_array_equal(oracle.rgba_to_gray(a, tw, th), want)


def _coverage(source, target):
    scale = source / target
    out = []
    for t in range(target):
        start, end = t * scale, min(source, (t + 1) * scale)
        first = int(np.floor(start))
        w, i = [], first
        while i < end:
            w.append((min(end, i + 1) - max(start, i)) / scale)
            i += 1
        out.append((first, w))
    return out


def _area(src, tw, th):
    h, w = src.shape
    cols, rows = _coverage(w, tw), _coverage(h, th)
    temp = np.zeros((h, tw), np.float32)
    for x, (f, ws) in enumerate(cols):
        acc = np.zeros(h)
        for k, wt in enumerate(ws):
            acc = acc + wt * src[:, f + k].astype(np.float64)
        temp[:, x] = acc
    out = np.zeros((th, tw), np.uint8)
    for y, (f, ws) in enumerate(rows):
        acc = np.zeros(tw)
        for k, wt in enumerate(ws):
            acc = acc + wt * temp[f + k].astype(np.float64)
        out[y] = np.minimum(255, _js_round(acc))
    return out


def test_gray_other_ratio_is_the_exact_box_filter():
    a = _rgba(37, 53, 1)
    c = a.astype(np.float64)
    luma = ((77 * c[..., 0] + 150 * c[..., 1] + 29 * c[..., 2]) / 256).astype(np.float32)
    np.testing.assert_array_equal(oracle.rgba_to_gray(a, 20, 15), _area(luma, 20, 15))


def test_downsample_gray_and_rgb():
    g = np.random.default_rng(2).integers(0, 256, size=(45, 70), dtype=np.uint8)
    np.testing.assert_array_equal(oracle.downsample_gray(g, 33, 20), _area(g, 33, 20))
    blocks = g.reshape(15, 3, 14, 5).astype(np.float64).mean((1, 3))
    np.testing.assert_array_equal(oracle.downsample_gray(g, 14, 15), _js_round(blocks).astype(np.uint8))
    a = _rgba(40, 60, 3)
    means = a[..., :3].reshape(10, 4, 20, 3, 3).astype(np.float64).mean((1, 3))
    np.testing.assert_array_equal(oracle.downsample_rgb(a, 20, 10), np.trunc(means).astype(np.uint8))


def test_upsample_depth_ignores_empty_cells():
    grid = np.array([[1.0, 2.0], [0.0, 4.0]], np.float32)
    out = oracle.upsample_depth(grid, 4, 4)
    assert out[0, 0] == 1.0 and out[0, 3] == 2.0 and out[3, 3] == 4.0
    assert out[3, 0] == 0.0                      # only the empty cell covers this corner
    # a constant grid stays constant; an empty grid stays empty
    np.testing.assert_array_equal(oracle.upsample_depth(np.full((3, 5), 2.5, np.float32), 17, 9), 2.5)
    np.testing.assert_array_equal(oracle.upsample_depth(np.zeros((3, 5), np.float32), 17, 9), 0.0)


def _ramp_rgba(width=1280, height=8):
    """The horizontal ramp of image.spec.ts:4-14: value round(20 + 0.15 x) in R, G and B."""
    x = np.arange(width)
    v = _js_round(20 + x * 0.15).astype(np.uint8)
    rgba = np.zeros((height, width, 4), np.uint8)
    rgba[..., :3] = v[None, :, None]
    return rgba


def ramp_worst_error(gray, width=1280, target=960):
    """image.spec.ts:15-22: worst distance of row 2 from the ramp at the output pixel centres."""
    scale = width / target
    x = np.arange(2, target - 2)
    expected = 20 + ((x + 0.5) * scale - 0.5) * 0.15
    return float(np.abs(gray[2, x].astype(np.float64) - expected).max())


def test_reference_ramp_keeps_pixel_centres_aligned():
    """image.spec.ts:9-24: rgbaToGray 1280x8 -> 960x6 of a ramp is off by at most one level."""
    gray = oracle.rgba_to_gray(_ramp_rgba(), 960, 6)
    assert ramp_worst_error(gray) <= 1.0


def test_reference_integer_ratio_blocks():
    """image.spec.ts:26-30: downsampleGray of an 8x4 ramp to 4x2 averages exact blocks."""
    data = ((np.arange(32) % 8) * 10).astype(np.uint8).reshape(4, 8)
    half = oracle.downsample_gray(data, 4, 2)
    assert half[0].tolist() == [5, 25, 45, 65]
