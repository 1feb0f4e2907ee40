"""The time loop's drop-in behaviour beyond the stepper (reference
emu_sv/sv_backend_impl.py): dark qubits under a state-preparation error (162-184) and the
per-step statistics (32-71, 244-255)."""

import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def _data(g, **kw):
    from emulators_b200.sv_backend import SequenceData

    steps = g["omega"].shape[0]
    dt_ns = float(g["dt"]) * 1000.0
    times = [k * dt_ns for k in range(steps + 1)]
    return SequenceData(torch.as_tensor(g["omega"]), torch.as_tensor(g["delta"]),
                        torch.as_tensor(g["phi"]), times, torch.as_tensor(g["U"]),
                        tuple(f"q{i}" for i in range(g["U"].shape[0])), **kw)


def test_dark_qubits_match_reference():
    """The reference's masks and its stepper chain on the masked data (dark_qubits.npz):
    same final state; the caller's samples are left as they were."""
    from emulators_b200.sv_backend import SVBackendImpl, SVConfig

    g = golden("dark_qubits")
    data = _data(g, bad_atoms=tuple(bool(b) for b in g["bad_atoms"]), state_prep_error=0.1)
    impl = SVBackendImpl(SVConfig(dt=float(g["dt"]) * 1000.0), data)
    impl._run()
    np.testing.assert_allclose(impl.state.data.cpu().numpy(), g["final"], atol=1e-10, rtol=0)
    np.testing.assert_array_equal(data.omega.numpy(), g["omega"])
    np.testing.assert_array_equal(impl.omega.numpy(), g["omega_masked"])
    np.testing.assert_array_equal(impl._U(0.0).numpy(), g["U_masked"])
    # no state-preparation error: the bad-atom list is ignored
    impl2 = SVBackendImpl(SVConfig(dt=float(g["dt"]) * 1000.0),
                          _data(g, bad_atoms=tuple(bool(b) for b in g["bad_atoms"])))
    assert impl2.dark_qubits is None


def test_initial_state_with_state_prep_error_is_rejected():
    from emulators_b200 import StateVector
    from emulators_b200.sv_backend import SVBackendImpl, SVConfig

    g = golden("dark_qubits")
    n = g["U"].shape[0]
    with pytest.raises(NotImplementedError):
        SVBackendImpl(SVConfig(initial_state=StateVector.make(n)),
                      _data(g, bad_atoms=(True,) + (False,) * (n - 1), state_prep_error=0.1))


def test_statistics_every_step():
    """One 'statistics' entry per step (RSS in MB, the step's wall time), at every step's
    normalised time, whatever the observables' evaluation times."""
    from emulators_b200.sv_backend import Energy, SVBackendImpl, SVConfig

    g = golden("dark_qubits")
    steps = g["omega"].shape[0]
    res = SVBackendImpl(SVConfig(dt=float(g["dt"]) * 1000.0, observables=[Energy([1.0])]),
                        _data(g))._run()
    st = res.get("statistics")
    assert len(st) == steps and res.statistics is not None
    assert all(set(e) == {"RSS", "duration"} and e["RSS"] > 0 and e["duration"] >= 0 for e in st)
    np.testing.assert_allclose(res.times("statistics"), [(k + 1) / steps for k in range(steps)])
    assert len(res.get("energy")) == 1
