"""FFT engine parity (tc_fft_c2c) against numpy's FP64 FFT."""
import numpy as np
import pytest

from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu

# smooth sizes run as mixed radix, the others through Bluestein
SIZES = [1, 2, 3, 4, 5, 7, 8, 16, 30, 64, 96, 181, 256, 362, 727, 768, 1000, 1024, 1454,
         1536, 2048, 2908, 3072, 4096, 5832, 8192]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("direction", [-1, 1])
def test_fft_matches_numpy(n, direction):
    import torch
    from tomocam_b200.plan import fft_c2c
    rng = np.random.default_rng(n)
    nb = 3
    x = (rng.standard_normal((nb, n)) + 1j * rng.standard_normal((nb, n))).astype(np.complex64)
    y = fft_c2c(torch.from_numpy(x).cuda(), direction).cpu().numpy()
    ref = np.fft.fft(x.astype(np.complex128), axis=-1) if direction < 0 else \
        np.fft.ifft(x.astype(np.complex128), axis=-1) * n
    assert rel_l2(y, ref) < 2e-6


def test_fft_in_place_and_roundtrip():
    import torch
    from tomocam_b200.plan import fft_c2c
    rng = np.random.default_rng(1)
    x = (rng.standard_normal((5, 1536)) + 1j * rng.standard_normal((5, 1536))).astype(np.complex64)
    t = torch.from_numpy(x).cuda()
    fft_c2c(t, -1, out=t)
    fft_c2c(t, +1, out=t)
    assert rel_l2(t.cpu().numpy() / 1536, x) < 2e-6


def test_fft_rejects_bad_direction():
    import torch
    from tomocam_b200 import _lib
    from tomocam_b200.plan import fft_c2c
    t = torch.zeros((1, 8), dtype=torch.complex64, device="cuda")
    with pytest.raises(_lib.TomocamError):
        fft_c2c(t, 0)
