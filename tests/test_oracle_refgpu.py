"""The oracle pinned to outputs of the reference's own GPU build (CPU only).

tests/golden/make_golden_refgpu.py ran the reference's sources -- compiled
for sm_100a by `make -C oracle ref`, cuFINUFFT replaced by the exact
non-uniform DFT that cuFINUFFT approximates -- on a B200 and committed
inputs and outputs:

* preproc (src/preproc.cpp:74-102), postproc (src/postproc.cpp:70-97), the
  host pad2d (src/padding.cpp) and gpu::roll (src/gpu/fftshift.cu:30-40):
  the oracle must reproduce them bit for bit (they only move data);
* the reference module's radon, backproject (preproc + back-projection +
  postproc) and mbir (mbir2 end to end, 8 iterations): the FP64 oracle must
  agree to the operators' 1e-5 and the reconstructions' 1e-4 (the reference
  computes in FP32).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import load
from tests.helpers import rel_l2


@pytest.fixture(scope="module")
def prep():
    return load("refgpu_prep")


@pytest.fixture(scope="module")
def module():
    return load("refgpu_module")


def _count(d, prefix):
    return len([k for k in d if k.startswith(prefix) and k.endswith("_out")])


def test_preproc_bit_exact(prep):
    n = _count(prep, "pre")
    assert n >= 9
    for k in range(n):
        got = O.preproc(prep[f"pre{k}_in"].astype(np.float64), float(prep[f"pre{k}_center"]))
        want = prep[f"pre{k}_out"]
        assert got.shape == want.shape, k
        assert np.array_equal(got.astype(np.float32), want), k


def test_postproc_and_pad2d_bit_exact(prep):
    for k in range(_count(prep, "post")):
        got = O.postproc(prep[f"post{k}_in"].astype(np.float64), int(prep[f"post{k}_npix"]))
        assert np.array_equal(got.astype(np.float32), prep[f"post{k}_out"]), k
    for k in range(_count(prep, "pad")):
        got = O.pad2d_symmetric(prep[f"pad{k}_in"].astype(np.float64), int(prep[f"pad{k}_npad"]))
        assert np.array_equal(got.astype(np.float32), prep[f"pad{k}_out"]), k


def test_roll_is_numpy_roll(prep):
    for k in range(_count(prep, "roll")):
        x, d = prep[f"roll{k}_in"], int(prep[f"roll{k}_delta"])
        assert np.array_equal(np.roll(x, -d, axis=-1), prep[f"roll{k}_out"]), k


def test_radon_and_backproject_match_reference(module):
    a = module["radon_angles"].astype(np.float64)
    assert rel_l2(module["radon_out"], O.project(module["radon_in"].astype(np.float64), a)) < 1e-5
    a2 = module["bp_angles"].astype(np.float64)
    D = module["bp_in"].shape[-1]
    want = O.postproc(O.backproject(O.preproc(module["bp_in"].astype(np.float64),
                                              float(module["bp_center"])), a2), D)
    assert rel_l2(module["bp_out"], want) < 1e-5


def test_mbir2_matches_reference(module):
    out = O.mbir2(module["mbir_in"], module["mbir_angles"].astype(np.float64),
                  float(module["mbir_center"]), int(module["mbir_iters"]),
                  float(module["mbir_sigma"]))
    assert out.shape == module["mbir_out"].shape
    assert rel_l2(module["mbir_out"], out) < 1e-4
