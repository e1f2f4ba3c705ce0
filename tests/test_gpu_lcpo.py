"""GPU: the LCPO surface-area term (FF_SASA_LCPO, forcefields/lcpo.cpp)
through the C ABI against the oracle (pinned bit for bit to the reference,
tests/test_oracle_golden.py) and the reference's own outputs.

Tolerances:
  per-atom SASA, SASAderiv     bit-exact against the oracle (FP64 in the
                               reference's operation order, no FMA)
  LCPO forces                  relative RMS 1e-8 (added to the forces in
                               64-bit fixed point: 2^-32 kcal/mol/A steps on
                               forces of ~0.1 kcal/mol/A)
  epot_surf                    relative 1e-12 (per-atom terms summed in a
                               fixed tree order, not the reference's loop)
  whole-forcefield forces      relative RMS 1e-5 (FP32 GB pair arithmetic)
"""
import ctypes

import numpy as np
import pytest

from conftest import load_fixture, rel_rms

import oracle as O

pytestmark = pytest.mark.gpu

NAME = "lcpo_pep24_s5"
J2K = (1.0 / 4184.0) * 6.0221418e23


def _ws(gpu_ctx, with_gb=True, update=None):
    import pdgpu
    a, meta = load_fixture(NAME)
    ws = pdgpu.WorkSpace(pdgpu.SystemSpec(a, meta), gpu_ctx)
    ff = pdgpu.Forcefield(ws)
    if with_gb:
        ff.add(pdgpu.FF_Bonded(ws))
        gb = pdgpu.FF_GeneralizedBorn_Still(ws)
        gb.Cutoff, gb.InnerCutoff = float(meta["cutoff"]), float(meta["inner"])
        gb.VdwCutoff, gb.VdwInnerCutoff = float(meta["vdwcut"]), float(meta["vdwinner"])
        ff.add(gb)
    sasa = pdgpu.FF_SASA_LCPO(ws)
    sasa.GlobalASP = float(a["lcpo_cfg"][0])
    sasa.UpdateSasa = int(a["lcpo_cfg"][1]) if update is None else update
    ff.add(sasa)
    ff.ensuresetup()
    return ws, ff, sasa, a


def _oracle(a, pos, ptr, data, energy_only=False, p=None):
    asp = float(a["lcpo_cfg"][0])  # kcal/mol/A^2: the device's sigma unit
    return O.lcpo(pos, ptr, data, a["lcpo_radius"], a["lcpo_p"] if p is None else p, asp, a["lcpo_use"],
                  energy_only=energy_only)


@pytest.mark.parametrize("dense", [False, True])
@pytest.mark.parametrize("path", [0, 1])
def test_lcpo_alone_bit_exact(gpu_ctx, dense, path):
    """path 0: overlap candidates from the list rows; 1: from the tiles of a
    tile search (the rows are then built only for the export below)."""
    ws, ff, sasa, a = _ws(gpu_ctx, with_gb=False)
    pre = "lcpo_dense_" if dense else "lcpo_"
    pos = a["lcpo_dense_pos"] if dense else a["pos"]
    ws.cur.p[:] = pos
    ws._pos_dirty = True
    ws.nlist().calcNewList()
    ws.setPairPath(path)
    ws.nlist().calcNewList()  # on the tile layout: a tile search, no rows
    ref_ptr, ref_data = (a["lcpo_dense_nl_ptr"], a["lcpo_dense_nl_data"]) if dense else (a["nl_ptr"], a["nl_data"])
    ws.Step = 0
    ff.calcForces()
    area, deriv = sasa.sasa()
    ptr, data = ws.nlist().getData(shadow=True)
    o_area, o_deriv, o_e, lost = _oracle(a, pos, ptr, data)
    assert (lost > 0) == dense  # the dense packing overflows 80-partner lists
    assert np.array_equal(area, o_area)
    assert np.array_equal(deriv, o_deriv)
    # the reference's list gives the same result (same pair set)
    r_area, _, _, _ = _oracle(a, pos, ref_ptr, ref_data)
    assert np.array_equal(area, r_area)
    assert rel_rms(ws.cur.f, a[pre + "f"]) <= 1e-8
    assert ws.ene.epot_surf == pytest.approx(a[pre + "ene"][10], rel=1e-12)
    assert ws.ene.epot == pytest.approx(a[pre + "ene"][0], rel=1e-12)
    # the energies path (calcEnergies): its own overlap formula, no forces
    if path == 1:
        ws.nlist().calcNewList()  # tiles again
    ff.calcEnergies()
    e_area, _ = sasa.sasa()
    o2, _, _, _ = _oracle(a, pos, ptr, data, energy_only=True)
    assert np.array_equal(e_area, o2)
    assert ws.ene.epot_surf == pytest.approx(a[pre + "ene_energypath"][10], rel=1e-12)
    assert np.all(ws.cur.f == 0)


def test_lcpo_negative_areas_are_clamped(gpu_ctx):
    """P1 planted at a tenth of its value: buried atoms get a negative LCPO
    area, which the reference sets to 0 together with its derivative."""
    import pdgpu
    a, meta = load_fixture(NAME)
    p = a["lcpo_p"].copy()
    p[:, 0] *= 0.1
    a2 = dict(a)
    a2["lcpo_p"] = p
    ws = pdgpu.WorkSpace(pdgpu.SystemSpec(a2, meta), gpu_ctx)
    ff = pdgpu.Forcefield(ws)
    sasa = pdgpu.FF_SASA_LCPO(ws)
    sasa.GlobalASP = 0.005
    ff.add(sasa)
    ff.calcForces()
    area, deriv = sasa.sasa()
    ptr, data = ws.nlist().getData(shadow=True)
    o_area, o_deriv, _, _ = _oracle(a, a["pos"], ptr, data, p=p)
    clamped = (o_area == 0) & (a["lcpo_use"] == 1)
    assert clamped.sum() > 10
    assert np.all(o_deriv[clamped] == 0)
    assert np.array_equal(area, o_area)
    assert np.array_equal(deriv, o_deriv)


def test_lcpo_with_gb_single_point(gpu_ctx):
    ws, ff, sasa, a = _ws(gpu_ctx)
    ws.nlist().calcNewList()
    ff.calcForces()
    assert rel_rms(ws.cur.f, a["lcpo_f_total"]) <= 1e-5
    assert ws.ene.epot_surf == pytest.approx(a["lcpo_ene_total"][10], rel=1e-12)
    assert abs(ws.ene.epot - a["lcpo_ene_total"][0]) * J2K <= max(1e-5 * abs(a["lcpo_ene_total"][0]) * J2K, 1e-3)
    # the one-call path (pdgpu_calc_forces) gives the same forces and record
    from pdgpu import _abi as A
    f1, e1 = ws._pull_forces(), ws._pull_energies()
    A.check(A.lib().pdgpu_zero_forces(ws.ctx.ptr, ws._sys))
    A.check(A.lib().pdgpu_calc_forces(ws.ctx.ptr, ws._sys))
    assert rel_rms(ws._pull_forces(), f1) <= 1e-12
    assert ws._pull_energies()[A.ENE_SURF] == pytest.approx(e1[A.ENE_SURF], rel=1e-14)


def test_lcpo_update_cadence_per_step(gpu_ctx):
    """Each velocity-Verlet step from the reference's own state at
    WorkSpace.Step = s: the surface term is recomputed when s % 5 == 0 and
    its held forces are added otherwise, as the reference did."""
    from pdgpu import _abi as A
    ws, ff, sasa, a = _ws(gpu_ctx)
    K = a["lcpo_mdvv_x"].shape[0]
    p = A.md_params_default()
    p.Integrator, p.Timestep = A.INTEGRATOR_VELOCITY_VERLET, 1e-15
    x, v = a["lcpo_mdvv_x0"], a["lcpo_mdvv_v0"]
    zeros = np.zeros(6 * ws.nAtoms())
    for s in range(K):
        ws.cur.p[:] = x
        ws._push_positions()
        ws.cur.v[:] = v
        ws._push_velocities()
        ws.nlist().calcNewList()
        ws.Step = s
        ff.calcForces()
        assert rel_rms(ws.cur.f, a["lcpo_mdvv_f"][s]) <= 1e-5, s
        if s % 5 == 0:
            ptr, data = ws.nlist().getData(shadow=True)
            area, deriv = sasa.sasa()
            o_area, o_deriv, _, _ = _oracle(a, x, ptr, data)
            assert np.array_equal(area, o_area) and np.array_equal(deriv, o_deriv), s
        A.check(A.lib().pdgpu_md_step_with_normals(ws.ctx.ptr, ws._sys, ctypes.byref(p), s, K, A.dptr(zeros)))
        ws._pull_positions()
        ws._pull_velocities()
        assert rel_rms(ws.cur.p - x, a["lcpo_mdvv_x"][s] - x) <= 1e-5, s
        x, v = a["lcpo_mdvv_x"][s], a["lcpo_mdvv_v"][s]


@pytest.mark.parametrize("use_graph", [True, False])
def test_lcpo_md_run_follows_the_reference(gpu_ctx, use_graph):
    """The whole protocol on the device (list every 10 steps, the step
    counter driving the surface term's cadence) against the reference's
    12 velocity-Verlet steps."""
    import pdgpu
    ws, ff, sasa, a = _ws(gpu_ctx)
    ws.setPairPath(1)  # tiles requested: the term makes every rebuild build the list rows too
    ws.cur.p[:] = a["lcpo_mdvv_x0"]
    ws._pos_dirty = True
    ws.cur.v[:] = a["lcpo_mdvv_v0"]
    md = pdgpu.MolecularDynamics(ff)
    md.Integrator = pdgpu.MolecularDynamics.VelocityVerlet
    md.Timestep = 1e-15
    md.RandVel = False
    md.Steps = a["lcpo_mdvv_x"].shape[0]
    md.UpdateNList = 10
    md.UseGraph = use_graph
    ws.nlist().calcNewList()
    md.run()
    x0 = a["lcpo_mdvv_x0"]
    assert rel_rms(ws.cur.p - x0, a["lcpo_mdvv_x"][-1] - x0) <= 1e-4
    assert ws.Step == md.Steps - 1
    # the record of each step carries epot with the surface term
    ep = md.history[:, 0]
    assert np.all(np.abs(ep - a["lcpo_mdvv_epot"]) * J2K <= np.maximum(1e-5 * np.abs(a["lcpo_mdvv_epot"]) * J2K, 1e-3))


def test_lcpo_minimiser_and_served_job(gpu_ctx):
    import pdgpu
    ws, ff, sasa, a = _ws(gpu_ctx)
    r = a["lcpo_minsd_result"]
    ws.cur.p[:] = a["lcpo_minsd_x0"]
    ws._pos_dirty = True
    m = pdgpu.Minimisation(ff)
    m.Algorithm = pdgpu.Minimisation.SteepestDescent
    m.Steps = int(r[0])
    assert m.run() == int(r[0])
    assert np.max(np.abs(ws.cur.p - a["lcpo_minsd_x"])) <= 1e-4
    assert abs(ws.ene.epot - r[1]) * J2K <= max(1e-5 * abs(r[1]) * J2K, 1e-3)
    assert ws.ene.epot_surf > 0
    plain_x, plain_e = ws.cur.p.copy(), ws._pull_energies()
    # the same job through the request loop: the same numbers
    srv = pdgpu.Server(gpu_ctx, max_active=4, tiles=False)
    job = pdgpu.Server.job(pdgpu.Server.MINIMISE, int(r[0]))
    job.min.Algorithm = pdgpu.Minimisation.SteepestDescent
    jid = srv.submit(ws, job, positions=a["lcpo_minsd_x0"])
    assert srv.wait(jid, 120.0) == 0
    res = srv.result(jid)
    srv.release(jid)
    srv.close()
    assert np.max(np.abs(res["positions"] - a["lcpo_minsd_x"])) <= 1e-4
    assert res["energies"][15] == pytest.approx(plain_e[15], rel=1e-6)


def test_lcpo_batch_members_equal_alone(gpu_ctx):
    """Two members (the fixture and a shifted copy) evaluated together give
    each member's own areas and derivatives bit for bit."""
    import pdgpu
    wss = []
    for shift in (0.0, 0.3):
        ws, ff, sasa, a = _ws(gpu_ctx)
        ws.cur.p[:] = a["pos"] + shift * np.sin(np.arange(a["pos"].size)).reshape(-1, 3)
        ws._pos_dirty = True
        ws.nlist().calcNewList()
        ff.calcForces()
        wss.append((ws, sasa.sasa(), ws._pull_forces(), ws._pull_energies()))
    b = pdgpu.Batch([w[0] for w in wss])
    b.setPairPath(0)
    f, e = b.evaluate()
    area = np.zeros(b.nAtoms)
    deriv = np.zeros((b.nAtoms, 3))
    from pdgpu import _abi as A
    A.check(A.lib().pdgpu_sasa_lcpo_get(b.ctx.ptr, b._id, A.dptr(area), A.dptr(deriv)))
    for s, (ws, (a1, d1), f1, e1) in enumerate(wss):
        lo, hi = b.offsets[s], b.offsets[s + 1]
        assert np.array_equal(area[lo:hi], a1)
        assert np.array_equal(deriv[lo:hi], d1)
        assert e[s][A.ENE_SURF] == pytest.approx(e1[A.ENE_SURF], rel=1e-13)
    b.close()


def test_lcpo_large_system(gpu_ctx):
    """The 20,566-atom system with the term, against the reference's
    forces and surface energy (its list is too large to keep, so the oracle
    runs on the device's exported list)."""
    import pdgpu
    a, meta = load_fixture("c2_16x80_s2")
    ws = pdgpu.WorkSpace(pdgpu.SystemSpec(a, meta), gpu_ctx)
    ff = pdgpu.Forcefield(ws)
    ff.add(pdgpu.FF_Bonded(ws))
    gb = pdgpu.FF_GeneralizedBorn_Still(ws)
    gb.Cutoff, gb.InnerCutoff = float(meta["cutoff"]), float(meta["inner"])
    gb.VdwCutoff, gb.VdwInnerCutoff = float(meta["vdwcut"]), float(meta["vdwinner"])
    ff.add(gb)
    sasa = pdgpu.FF_SASA_LCPO(ws)
    sasa.GlobalASP = float(a["lcpo_cfg"][0])
    ff.add(sasa)
    ws.nlist().calcNewList()
    ff.calcForces()
    assert rel_rms(ws.cur.f, a["lcpo_f_total"]) <= 1e-5
    assert ws.ene.epot_surf == pytest.approx(a["lcpo_ene_total"][10], rel=1e-12)
    area, deriv = sasa.sasa()
    ptr, data = ws.nlist().getData(shadow=True)
    o_area, o_deriv, _, _ = O.lcpo(a["pos"], ptr, data, a["lcpo_radius"], a["lcpo_p"], float(a["lcpo_cfg"][0]),
                                   a["lcpo_use"])
    assert np.array_equal(area, o_area)
    assert np.array_equal(deriv, o_deriv)
    ws.close()
