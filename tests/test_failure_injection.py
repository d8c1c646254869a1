"""Failure detection without a GPU fault: a poisoned state written from the
host must end the step with FX_ERR_NONFINITE and leave the state as it was.

The reference has no such check: a NaN in P reaches the Poisson right-hand
side, MLMG never meets its tolerance and ComputePhi_Rho's Newton loop
(ElectrostaticSolver.cpp:703-744) has no iteration cap.  Here every solve loop
stops at the first non-finite residual norm, the step's TDGL update and
steady-state check are skipped, the status names the failure, and phi and
the charge density return to their values at the end of the last completed
step, so the same context can step again once the input is fixed.  The
poison is planted from the host (fx_set_field) between steps, in the step
graph and in the host-driven loop, on a dielectric stack (one Poisson solve)
and on a semiconductor stack (the Newton loop)."""
import numpy as np
import pytest

from ferrox_b200 import api, decks

pytestmark = pytest.mark.gpu

NONFINITE = -6


def _deck(kind):
    if kind == "mfim":
        return decks.mfim(16, 16, 24, Phi_Bc_hi=0.3)
    return decks.mfism(16, 16, 48, extra={"Phi_Bc_hi": 0.4})


@pytest.mark.parametrize("graph", [1, 0], ids=["step_graph", "host_loop"])
@pytest.mark.parametrize("kind", ["mfim", "mfism"])
@pytest.mark.parametrize("where", ["Pz", "Phi"])
def test_nan_in_state_is_reported_and_state_kept(kind, graph, where):
    f = api.FerroX(_deck(kind))
    f.set_param("fx.step_graph", graph)
    f.step(2)
    phi_before, rho_before = f.field("Phi"), f.field("charge")
    poisoned = f.field(where)
    fe = np.argwhere(f.field("mask") == 0)
    k, j, i = fe[len(fe) // 2]
    poisoned[k, j, i] = np.nan
    f.set_field(where, poisoned)
    P0 = f.field("Pz")
    step0 = f.stats()["step"]
    with pytest.raises(api.FxError) as e:
        f.step(1)
    assert e.value.code == NONFINITE, str(e.value)
    # the failed step changed neither P nor the step count
    assert np.array_equal(f.field("Pz"), P0, equal_nan=True)
    assert f.stats()["step"] == step0
    # phi and the charge are those of the end of the last completed step
    assert np.array_equal(f.field("Phi"), phi_before)
    assert np.array_equal(f.field("charge"), rho_before)
    # with the poison removed the same context steps again
    clean = f.field(where)
    clean[k, j, i] = 0.0
    f.set_field(where, clean)
    f.step(1)
    assert np.isfinite(f.field("Pz")).all() and np.isfinite(f.field("Phi")).all()
    f.close()


def test_failure_stops_at_the_first_nonfinite_cycle():
    """The multigrid does not spin to its cycle cap on a NaN residual."""
    f = api.FerroX(_deck("mfim"))
    f.step(1)
    Pz = f.field("Pz")
    Pz[Pz.shape[0] - 2, 3, 3] = np.inf
    f.set_field("Pz", Pz)
    before = f.stats()["mg_cycles_total"]
    with pytest.raises(api.FxError) as e:
        f.step(1)
    assert e.value.code == NONFINITE
    assert f.stats()["mg_cycles_total"] - before <= 1
    f.close()
