"""Image preparation on the GPU (csrc/image.cu) against the oracle, bit for bit."""
import numpy as np
import pytest

import oracle

torch = pytest.importorskip("torch")

from luvas3d import image as I  # noqa: E402

pytestmark = pytest.mark.gpu


def _rgba(h, w, seed=0):
    return np.random.default_rng(seed).integers(0, 256, size=(h, w, 4), dtype=np.uint8)


@pytest.mark.parametrize("src,dst", [((1440, 1920), (480, 640)), ((1440, 1920), (525, 700)),
                                     ((97, 131), (40, 52)), ((64, 64), (64, 64))])
def test_rgba_to_gray(src, dst):
    a = _rgba(*src)
    got = I.rgba_to_gray(torch.from_numpy(a).cuda(), dst[1], dst[0]).cpu().numpy()
    np.testing.assert_array_equal(got, oracle.rgba_to_gray(a, dst[1], dst[0]))


@pytest.mark.parametrize("src,dst", [((1440, 1920), (90, 120)), ((97, 131), (30, 41))])
def test_downsample_rgb(src, dst):
    a = _rgba(*src, seed=1)
    got = I.downsample_rgb(torch.from_numpy(a).cuda(), dst[1], dst[0]).cpu().numpy()
    np.testing.assert_array_equal(got, oracle.downsample_rgb(a, dst[1], dst[0]))


@pytest.mark.parametrize("dst", [(240, 320), (180, 250)])
def test_downsample_gray(dst):
    g = np.random.default_rng(2).integers(0, 256, size=(480, 640), dtype=np.uint8)
    got = I.downsample_gray(torch.from_numpy(g).cuda(), dst[1], dst[0]).cpu().numpy()
    np.testing.assert_array_equal(got, oracle.downsample_gray(g, dst[1], dst[0]))


def test_upsample_depth():
    rng = np.random.default_rng(3)
    grid = rng.uniform(0.3, 4.0, size=(192, 256)).astype(np.float32)
    grid[rng.random(grid.shape) < 0.2] = 0
    got = I.upsample_depth(torch.from_numpy(grid).cuda(), 640, 480).cpu().numpy()
    want = oracle.upsample_depth(grid, 640, 480)
    np.testing.assert_array_equal(got.view(np.uint32), want.view(np.uint32))


def test_reference_image_spec_cases():
    """The two cases of image.spec.ts on the device: the 1280x8 ramp to 960x6 stays within one
    level of the ramp at the pixel centres, and 2x2 blocks of an 8x4 ramp average exactly."""
    from test_image_oracle import _ramp_rgba, ramp_worst_error
    gray = I.rgba_to_gray(torch.from_numpy(_ramp_rgba()).cuda(), 960, 6).cpu().numpy()
    assert ramp_worst_error(gray) <= 1.0
    data = torch.from_numpy(((np.arange(32) % 8) * 10).astype(np.uint8).reshape(4, 8)).cuda()
    assert I.downsample_gray(data, 4, 2).cpu().numpy()[0].tolist() == [5, 25, 45, 65]
