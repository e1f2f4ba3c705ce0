"""GPU parity of the stand-alone LJ/Coulomb component and of the GB
component with FastMode off, against the reference's own FP64 results
(tests/golden/nb_pep24_s7.npz, made by the compiled reference).

FF_NonBonded alone (forcefields/nonbonded.cpp:548-893, modes as calcForces
selects them at :1205-1229): force switching (its default), energy
switching, plain Coulomb, the DDDielectric flag (not consulted there: the
same results as force switching), dielectric 4, and the long-range VdW
correction (:845-857).  FF_GeneralizedBorn_Still with FastMode off:
FF_NonBonded::calcForces + calcBornForces (gbff.cpp:168-180, 1172-1400),
with FF_Bonded and alone, on both pair layouts.

Tolerances: relative force RMS 1e-5; energies relative 1e-5 or 1e-3
kcal/mol; the virial relative 1e-4 or 1e-3 kcal/mol.
"""
import numpy as np
import pytest

from conftest import load_fixture, rel_rms

pytestmark = pytest.mark.gpu

J2K = (1.0 / 4184.0) * 6.0221418e23
A_, M_ = load_fixture("nb_pep24_s7")
MODES = ["nbfs_", "nbes_", "nbnorm_", "nbddd_", "nbdiel4_", "nbvdwcor_"]


def close(got_J, ref_J, rel=1e-5, abs_kcal=1e-3):
    return abs(got_J - ref_J) * J2K <= max(rel * abs(ref_J) * J2K, abs_kcal)


@pytest.mark.parametrize("path", [0, 1])
@pytest.mark.parametrize("mode", MODES)
def test_nonbonded_mode(mode, path, gpu_ctx):
    import pdgpu
    cfg = A_[mode + "cfg"]
    ws = pdgpu.WorkSpace(pdgpu.SystemSpec(A_, M_), gpu_ctx)
    ff = pdgpu.Forcefield(ws)
    nb = pdgpu.FF_NonBonded(ws)
    nb.Cutoff, nb.InnerCutoff = float(cfg[0]), float(cfg[1])
    nb.VdwCutoff, nb.VdwInnerCutoff = float(cfg[0]), float(cfg[1])
    nb.ForceSwitch, nb.EnergySwitch, nb.DDDielectric = bool(cfg[2]), bool(cfg[3]), bool(cfg[4])
    nb.Dielectric = float(cfg[5])
    nb.VdwCor = bool(cfg[6])
    nb.VdwCorDensity, nb.VdwCorEpsilon, nb.VdwCorRadius, nb.VdwCorCutoff = (float(x) for x in cfg[7:11])
    ff.add(nb)
    ff.ensuresetup()
    ws.setPairPath(path)
    ws.nlist().calcNewList()
    ff.calcForces()
    assert rel_rms(ws.cur.f, A_[mode + "f"]) <= 1e-5
    e, et = ws.ene, A_[mode + "ene"]
    for field, idx in (("epot", 0), ("epot_vdw", 1), ("epot_elec", 2)):
        assert close(getattr(e, field), et[idx]), (mode, field, getattr(e, field) * J2K, et[idx] * J2K)
    assert close(e.InternalVirial, et[9], rel=1e-4), (mode, e.InternalVirial * J2K, et[9] * J2K)
    ws.close()


def _gb_slow(ctx, path, with_bonded):
    import pdgpu
    ws = pdgpu.WorkSpace(pdgpu.SystemSpec(A_, M_), ctx)
    ff = pdgpu.Forcefield(ws)
    if with_bonded:
        ff.add(pdgpu.FF_Bonded(ws))
    gb = pdgpu.FF_GeneralizedBorn_Still(ws)
    gb.Cutoff, gb.InnerCutoff = float(M_["cutoff"]), float(M_["inner"])
    gb.VdwCutoff, gb.VdwInnerCutoff = float(M_["vdwcut"]), float(M_["vdwinner"])
    gb.FastMode = False
    ff.add(gb)
    ff.ensuresetup()
    ws.setPairPath(path)
    ws.nlist().calcNewList()
    ff.calcForces()
    return ws


@pytest.mark.parametrize("path", [0, 1])
def test_gb_fastmode_off(path, gpu_ctx):
    ws = _gb_slow(gpu_ctx, path, True)
    born = ws.born_radii()
    assert np.max(np.abs(born - A_["gbslow_born"]) / np.abs(A_["gbslow_born"])) <= 2e-6
    assert rel_rms(ws.cur.f, A_["gbslow_f_total"]) <= 1e-5
    e, et = ws.ene, A_["gbslow_ene_total"]
    for field, idx in (("epot", 0), ("epot_vdw", 1), ("epot_elec", 2), ("epot_pol", 3), ("epot_pol_cross", 4),
                       ("epot_pol_self", 5)):
        assert close(getattr(e, field), et[idx]), (field, getattr(e, field) * J2K, et[idx] * J2K)
    for field, idx in (("epot_bond", 6), ("epot_angle", 7), ("epot_torsion", 8)):
        assert getattr(e, field) == pytest.approx(et[idx], rel=1e-9), field
    ws.close()
    # the component alone
    ws = _gb_slow(gpu_ctx, path, False)
    assert rel_rms(ws.cur.f, A_["gbslow_f_gb"]) <= 1e-5
    eg = A_["gbslow_ene_gb"]
    assert close(ws.ene.epot, eg[0])
    ws.close()


def test_gb_fastmode_off_md_runs(gpu_ctx):
    """A few Langevin steps with FastMode off stay finite and keep the
    temperature near its target (the step loop takes the same path)."""
    import ctypes
    from pdgpu import _abi as A
    ws = _gb_slow(gpu_ctx, 1, True)
    p = A.md_params_default()
    p.Integrator, p.UpdateNList, p.UseGraph = A.INTEGRATOR_LANGEVIN, 10, 1
    p.Timestep, p.FricCoeff, p.TargetTemp, p.Seed = 1e-15, 1e12, 300.0, 9
    A.check(A.lib().pdgpu_md_init_velocities(gpu_ctx.ptr, ws._sys, 300.0, 9))
    hist = np.zeros((30, 3))
    A.check(A.lib().pdgpu_md_run(gpu_ctx.ptr, ws._sys, ctypes.byref(p), 0, 30, 30, A.dptr(hist)))
    assert np.all(np.isfinite(hist))
    ws.close()
