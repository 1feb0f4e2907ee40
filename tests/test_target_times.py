"""The target-time grid and the observables' evaluation-time test of the backend time
loop against the reference's own outputs (emu_base/pulser_adapter.py:80-151, fixtures made
by tests/golden/make_golden.py from the reference's _get_target_times)."""

import numpy as np
import pytest

from conftest import golden


def test_target_times_match_reference():
    from emulators_b200.sv_backend import TIME_TOLERANCE, get_target_times

    g = golden("target_times")
    assert float(g["tolerance"]) == TIME_TOLERANCE
    for k in range(int(g["count"])):
        got = get_target_times(float(g[f"c{k}_duration"]), float(g[f"c{k}_dt"]),
                               list(g[f"c{k}_obs"]))
        np.testing.assert_array_equal(np.array(got), g[f"c{k}_expected"], err_msg=f"case {k}")


def test_target_times_known_answers():
    """test/emu_base/test_adapter.py:905-966: duration 20, dt 5.5."""
    from emulators_b200.sv_backend import get_target_times

    eval_abs = [0, 0.9, 11.9, 18.1]
    got = get_target_times(20, 5.5, [t / 20 for t in eval_abs])
    np.testing.assert_allclose(got, sorted(set([0, 5.5, 11, 16.5, 20] + eval_abs)))
    np.testing.assert_allclose(get_target_times(20, 5.5, [0.5]), [0, 5.5, 10, 11, 16.5, 20])


def test_fuzzy_union_keeps_base_and_drops_near_duplicates():
    from emulators_b200.sv_backend import fuzzy_union

    assert fuzzy_union([0.0, 0.5, 1.0], [0.5 + 5e-7, 0.25, 0.25 + 1e-7, 1.0 - 2e-6]) == \
        [0.0, 0.25, 0.5, 1.0 - 2e-6, 1.0]
    assert fuzzy_union([], [0.3, 0.1]) == [0.1, 0.3]  # inserted in order


def test_observable_due_to_time_tolerance():
    from emulators_b200.sv_backend import Occupation

    o = Occupation([0.5, 1.0])
    assert o.due(0.5) and o.due(0.5 + 9e-7) and o.due(1.0 - 1e-7)
    assert not o.due(0.5 + 2e-6) and not o.due(0.45)
    assert Occupation().due(0.123)


def test_config_default_evaluation_times():
    """Observables without their own times take the config's default times."""
    from emulators_b200.sv_backend import Energy, Occupation, SVConfig

    cfg = SVConfig(observables=[Occupation(), Energy([0.5])], default_evaluation_times=[1.0])
    occ, en = cfg.observables
    d = cfg.default_evaluation_times
    assert d == (1.0,)
    assert not occ.due(0.5, d) and occ.due(1.0, d) and en.due(0.5, d) and not en.due(1.0, d)
    assert SVConfig(default_evaluation_times="Full").default_evaluation_times is None


@pytest.mark.gpu
def test_sequence_data_from_samples():
    """The adapter path on the GPU: grid with an off-grid observation time, then the PCHIP
    midpoints of every signal at that grid's midpoints."""
    import torch

    from emulators_b200.pchip import midpoint_samples
    from emulators_b200.sv_backend import SequenceData, get_target_times

    rng = np.random.default_rng(5)
    Q, T = 4, 300
    t = np.arange(T, dtype=np.float64)
    amp = np.abs(rng.normal(size=(Q, 1))) * np.sin(np.pi * t / T)[None, :] ** 2
    det = rng.uniform(-10, 10, (Q, 1)) + 0.02 * t[None, :]
    ph = np.zeros((Q, T))
    U = np.eye(Q)
    d = SequenceData.from_samples(torch.as_tensor(amp), torch.as_tensor(det),
                                  torch.as_tensor(ph), T, 7.0, U, observable_times=[0.4321])
    times = get_target_times(T, 7.0, [0.4321])
    assert d.target_times == times and any(abs(x - 0.4321 * T) < 1e-9 for x in times)
    om, de, phi = midpoint_samples(torch.as_tensor(amp), torch.as_tensor(det),
                                   torch.as_tensor(ph), times)
    assert torch.equal(d.omega, om.cpu()) and torch.equal(d.delta, de.cpu())
    assert d.omega.shape == (len(times) - 1, Q) and d.omega.device.type == "cpu"
