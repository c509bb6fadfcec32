"""The optional PNG outputs (common/file_io.cpp:7-135): kl_write_png against
the reference's own stb-based writers on the same float data, compared by the
decoded pixels (the compressed bytes come from different deflate encoders)."""
import numpy as np
import pytest

import klitho as K
from oracle import oracle as O
from pngread import read_png


def _cases():
    rng = np.random.default_rng(0)
    a = rng.standard_normal((37, 53)).astype(np.float32)
    b = (rng.random((64, 48)) * 0.4).astype(np.float32)
    c = np.zeros((9, 11), dtype=np.float32)  # uniform: min == max
    return [("noise", a, float(a.min()), float(a.max())),
            ("intensity", b, 0.0, 0.225),
            ("clipped", b, 0.05, 0.3),
            ("uniform", c, 0.0, 0.0)]


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("case", range(4))
def test_png_pixels_match_reference(ref_built, tmp_path, mode, case):
    name, data, mn, mx = _cases()[case]
    if mode == 0 and mn == mx:
        pytest.skip("the reference's grey map divides by zero for a uniform image")
    ours, theirs = tmp_path / "ours.png", tmp_path / "ref.png"
    K.check(K.lib().kl_write_png(str(ours).encode(), K._fp(np.ascontiguousarray(data)), data.shape[1],
                                 data.shape[0], mn, mx, mode), "kl_write_png")
    O.ref_write_png(theirs, data, mn, mx, mode)
    a, b = read_png(ours), read_png(theirs)
    assert a.shape == b.shape
    assert np.array_equal(a, b), (name, mode, int(np.sum(a != b)))


def test_png_rejects_bad_colormap(tmp_path):
    d = np.zeros((2, 2), dtype=np.float32)
    assert K.lib().kl_write_png(str(tmp_path / "x.png").encode(), K._fp(d), 2, 2, 0.0, 1.0, 7) == K.KL_ERR_INVALID
