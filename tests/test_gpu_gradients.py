"""GPU parity of the batched, checkpointed pulse gradients (emulators_b200.gradients,
C ABI emusv_batch_launch_steps / emusv_batch_adjoint_*) against the reference's autograd
gradients, central finite differences and the per-set autograd chain."""

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def _batch(gw, sets, nseg, precision="c128", ck=16, **kw):
    from emulators_b200.gradients import PulseGradientBatch

    return PulseGradientBatch(gw.U, gw.dt, gw.omega_seg[sets, :nseg], gw.delta_seg[sets, :nseg],
                              gw.steps_per_segment, gw.target, precision=precision,
                              checkpoint_every=ck, tolerance=gw.tolerance, **kw)


def test_batched_gradients_match_reference_autograd():
    """First 2 segments (20 steps, checkpoints every 16) of 2 parameter sets of the N=16
    ring vs the reference's autograd through its per-step Function."""
    from emulators_b200 import workloads as wl

    g = golden("ring_n16_grad")
    gw = wl.ring_n16_grad()
    nseg, sets = int(g["nseg"]), int(g["sets"])
    b = _batch(gw, list(range(sets)), nseg)
    loss, go, gd, _ = b.loss_and_grad()
    for p in range(sets):
        assert abs(loss[p] - float(g[f"p{p}_loss"])) < 1e-11
        np.testing.assert_allclose(go[p], g[f"p{p}_g_omega"], rtol=1e-7, atol=1e-11)
        np.testing.assert_allclose(gd[p], g[f"p{p}_g_delta"], rtol=1e-7, atol=1e-11)


def test_batched_gradients_checkpoint_independent_and_c64():
    """The checkpoint interval does not change the result (bit for bit); complex64 vectors
    stay within 1e-5 relative of complex128."""
    from emulators_b200 import workloads as wl

    gw = wl.ring_n16_grad()
    sets = [0, 5, 9, 33]
    ref = _batch(gw, sets, 3, ck=16).loss_and_grad()
    alt = _batch(gw, sets, 3, ck=7).loss_and_grad()
    for a, b in zip(ref[:3], alt[:3]):
        np.testing.assert_array_equal(a, b)
    c64 = _batch(gw, sets, 3, precision="c64", tile_bits=10).loss_and_grad()
    for a, b in zip(ref[1:3], c64[1:3]):
        err = np.abs(a - b).max() / np.abs(a).max()
        assert err < 1e-5, err


def test_batched_gradients_central_differences():
    """dL/dOmega_seg, dL/ddelta_seg vs central differences with h = 1e-4."""
    from emulators_b200 import workloads as wl

    gw = wl.ring_n16_grad()
    s, nseg, h = 12, 3, 1e-4
    b = _batch(gw, [s], nseg)
    _, go, gd, _ = b.loss_and_grad()
    for which, grad in (("omega", go[0]), ("delta", gd[0])):
        for k in range(nseg):
            vals = []
            for sign in (1, -1):
                om = gw.omega_seg[[s], :nseg].copy()
                de = gw.delta_seg[[s], :nseg].copy()
                (om if which == "omega" else de)[0, k] += sign * h
                from emulators_b200.gradients import PulseGradientBatch

                bb = PulseGradientBatch(gw.U, gw.dt, om, de, gw.steps_per_segment, gw.target,
                                        tolerance=gw.tolerance)
                bb.forward()
                occ = bb.occupations()
                vals.append(float(((occ - bb.target.to(occ.device)) ** 2).mean()))
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(fd - grad[k]) <= 1e-5 * max(abs(grad[k]), 1e-3), (which, k, fd, grad[k])


def test_plain_torch_gradient_arm_matches_reference_autograd():
    """The bench's plain complex128 torch gradient path (the baseline the batched gradients
    are compared with) reproduces the reference's autograd gradients for the first 20 steps
    of parameter set 0."""
    import bench
    from emulators_b200 import workloads as wl

    g = golden("ring_n16_grad")
    gw = wl.ring_n16_grad()
    r = bench.plain_torch_grads_c128(gw, torch.device("cuda", 0), p=0,
                                     steps=int(g["nseg"]) * gw.steps_per_segment)
    nseg = int(g["nseg"])
    assert abs(r["loss"] - float(g["p0_loss"])) < 1e-11
    np.testing.assert_allclose(r["g_omega"][:nseg], g["p0_g_omega"], rtol=1e-7, atol=1e-11)
    np.testing.assert_allclose(r["g_delta"][:nseg], g["p0_g_delta"], rtol=1e-7, atol=1e-11)
    assert not np.any(r["g_omega"][nseg:]) and not np.any(r["g_delta"][nseg:])
