"""GPU: Monte Carlo on the device (pdgpu_mc_run: MonteCarlo::run_core and
MonteCarlo::accept, protocols/montecarlo.cpp:24-159) against the same
protocol driven from the host through the plain calls (perturb, list
rebuild, forces, the Metropolis decision in numpy).

The device draws its acceptance uniforms from Philox, the host cannot
replay them, so the exact comparisons use the two temperature limits where
the decision needs no draw: near 0 K only lower energies are accepted
(d < -50 otherwise), at an enormous temperature every finite energy is.
The kernels are the same, so positions and energies must agree bit for bit.
"""
import numpy as np
import pytest

from conftest import build_workspace, load_library

pytestmark = pytest.mark.gpu

SIGMA = np.deg2rad(15.0)
STEPS = 24


def _batch(gpu_ctx, count=4, keys=(31, 32, 33, 34)):
    import pdgpu
    wss = []
    for a, m in load_library("lib16_amber_s3")[:count]:
        ws, ff = build_workspace(a, m, gpu_ctx)
        ws.setTorsionMoves()
        wss.append(ws)
    b = pdgpu.Batch(wss)
    b.setPairPath(0)
    b.setSeeds(np.asarray(keys[:count], dtype=np.uint64))
    b.calcNewList()
    return b, wss


def _host_mc(b, steps, accept):
    """The protocol with the plain calls; `accept(e_new, e_old, t)` decides
    per member.  Returns (acceptances, last accepted positions, their epot)."""
    from pdgpu import _abi as A
    base = b.positions()
    e_old = np.full(b.nSystems, np.nan)
    acc = np.zeros(b.nSystems, dtype=np.int32)
    for t in range(steps):
        b.setPositions(base)
        b.saveBasePositions()
        if t:
            b.perturbTorsions(sigma=SIGMA, trial=t)
        b.calcNewList()
        b.calcForces()
        e = b.energies()[:, A.ENE_EPOT]
        pos = b.positions()
        for s in range(b.nSystems):
            if np.isfinite(e[s]) and (t == 0 or accept(e[s], e_old[s])):
                lo, hi = b.offsets[s], b.offsets[s + 1]
                base[lo:hi] = pos[lo:hi]
                e_old[s] = e[s]
                acc[s] += 1
    return acc, base, e_old


@pytest.mark.parametrize("limit", ["cold", "hot"])
def test_mc_matches_host_driven_protocol(gpu_ctx, limit):
    from pdgpu import _abi as A
    temp = 1e-30 if limit == "cold" else 1e30
    rule = (lambda new, old: new < old) if limit == "cold" else (lambda new, old: True)
    b, wss = _batch(gpu_ctx)
    start = b.positions()
    acc_h, base_h, e_h = _host_mc(b, STEPS, rule)
    b.setPositions(start)
    acc_d, low_d = b.runMC(STEPS, temperature=temp, sigma=SIGMA, final_state=A.MC_LAST_ACC)
    assert np.array_equal(acc_d, acc_h)
    if limit == "hot":  # every finite energy accepted (a clashing trial can be non-finite)
        assert acc_d.max() == STEPS
    else:
        assert np.all(acc_d >= 1) and np.all(acc_d < STEPS)
    # ends in the last accepted state, evaluated there
    assert np.array_equal(b.positions(), base_h)
    assert np.array_equal(b.energies()[:, A.ENE_EPOT], e_h)
    b.close()


def test_mc_lowest_state_and_room_temperature(gpu_ctx):
    from pdgpu import _abi as A
    b, wss = _batch(gpu_ctx)
    start = b.positions()
    acc, low = b.runMC(STEPS, temperature=300.0, sigma=SIGMA, final_state=A.MC_LOWEST_EPOT)
    assert np.all((acc >= 1) & (acc <= STEPS))
    # the handle ends in the lowest accepted state, re-evaluated: its epot
    assert np.array_equal(b.energies()[:, A.ENE_EPOT], low)
    # the same run again gives the same bits (keys and step counters only)
    b.setPositions(start)
    acc2, low2 = b.runMC(STEPS, temperature=300.0, sigma=SIGMA, final_state=A.MC_LOWEST_EPOT)
    assert np.array_equal(acc, acc2) and np.array_equal(low, low2)
    b.close()


def test_mc_protocol_surface(gpu_ctx):
    """pdgpu.MonteCarlo on one WorkSpace: ends in its lowest accepted state,
    re-evaluated, and at 1e-30 K that state is never above the start."""
    import pdgpu
    a, m = load_library("lib16_amber_s3")[0]
    ws, ff = build_workspace(a, m, gpu_ctx)
    ff.calcForces()
    e0 = ws.ene.epot
    mc = pdgpu.MonteCarlo(ff)
    mc.Steps = 12
    mc.Temperature = 1e-30
    mc.FinalState = pdgpu.MonteCarlo.LowestEpot
    mc.run()
    assert 1 <= mc.acceptances <= 12
    assert ws.ene.epot == mc.lowest and mc.lowest <= e0
    assert ws.Step == 11
