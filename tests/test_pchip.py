"""Drive preparation (PCHIP): the oracle's restatement against the reference's own values
(pchip.npz, made by running emu_base/math/pchip_torch.py), and the package's validation
(CPU); the GPU kernel (emusv_pchip_eval) against the same fixtures, bit for bit."""

import numpy as np
import pytest
import torch

from conftest import cases, golden


def test_oracle_pchip_matches_reference(oracle):
    for c in cases(golden("pchip")):
        got = oracle.pchip(c["x"], c["y"], c["xq"])
        np.testing.assert_array_equal(got, c["yq"])


@pytest.mark.parametrize("x,y,err,match", [
    (torch.tensor([0, 1, 2]), torch.tensor([0.0, 1.0, 2.0]), TypeError, "floating point"),
    (torch.tensor([0.0, 1.0]), torch.tensor([0.0, 1.0, 2.0]), ValueError, "same length"),
    (torch.tensor([0.0, 1.0, 1.0]), torch.tensor([0.0, 1.0, 2.0]), ValueError, "strictly increasing"),
    (torch.tensor([0.0]), torch.tensor([0.0]), ValueError, "at least 2"),
])
def test_pchip_validation(x, y, err, match):
    """pchip_torch.py:235-256 messages (test/emu_base/math/test_pchip.py cases)."""
    from emulators_b200.pchip import PCHIP1D

    with pytest.raises(err, match=match):
        PCHIP1D._validate_xy(x, y)


@pytest.mark.gpu
def test_gpu_pchip_matches_reference_bitwise():
    from emulators_b200.pchip import PCHIP1D

    for c in cases(golden("pchip")):
        f = PCHIP1D(torch.as_tensor(c["x"]), torch.as_tensor(c["y"]))
        got = f(torch.as_tensor(c["xq"])).numpy()
        np.testing.assert_array_equal(got, c["yq"])


@pytest.mark.gpu
def test_gpu_midpoint_samples_batched(oracle):
    """Many signals in one launch: every (qubit, parameter) signal equals its own
    interpolation, and the last amplitude sample is clamped at zero from below
    (pulser_adapter.py:188-231)."""
    from emulators_b200.pchip import midpoint_samples

    rng = np.random.default_rng(3)
    Q, T = 12, 500
    t = np.arange(T, dtype=np.float64)
    amp = np.abs(rng.normal(size=(Q, 1))) * np.sin(np.pi * t / T)[None, :] ** 2
    amp[:, -40:] = -1e-3  # a negative tail: the last midpoint must be clamped
    det = rng.uniform(-10, 10, (Q, 1)) + 0.01 * t[None, :]
    ph = np.zeros((Q, T))
    target = list(np.arange(0, T + 1, 7.0)) + [float(T)]
    target = sorted(set(target))
    om, de, phi = midpoint_samples(torch.as_tensor(amp), torch.as_tensor(det), torch.as_tensor(ph),
                                   target)
    tm = 0.5 * (np.array(target[:-1]) + np.array(target[1:]))
    for q in range(Q):
        ref_a = oracle.pchip(t, amp[q], tm)
        ref_a[-1] = max(ref_a[-1], 0.0)
        np.testing.assert_array_equal(om[:, q].real.cpu().numpy(), ref_a)
        np.testing.assert_array_equal(de[:, q].real.cpu().numpy(), oracle.pchip(t, det[q], tm))
    assert om.dtype == torch.complex128 and om.shape == (len(target) - 1, Q)
    assert float(om[-1].real.min()) >= 0.0
