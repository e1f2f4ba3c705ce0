"""GPU parity: libpdgpu (through its C ABI) against the reference's own FP64
results (tests/golden/, produced by the compiled reference) and the oracle.

Tolerances (stated per quantity, against the FP64 reference):
  neighbour list        bit-exact (sorted pair sets and bond-order bits)
  Born radii            relative 2e-6 (FP32 terms, each added in 64-bit fixed
                        point; FP64 inversion)
  forces                relative force RMS 1e-5 (FP32 pair arithmetic)
  pair energies         relative 1e-5 of the term, or 1e-3 kcal/mol
  bonded forces/energy  relative 1e-9 (FP64 terms, fixed-point scatter)
"""
import numpy as np
import pytest

from conftest import fixture_names, load_fixture, rel_rms

import oracle as O

pytestmark = pytest.mark.gpu

SMALL = fixture_names()
J2K = (1.0 / 4184.0) * 6.0221418e23


def make(name, ctx, with_bonded=True):
    import pdgpu
    arrays, meta = load_fixture(name)
    spec = pdgpu.SystemSpec(arrays, meta)
    ws = pdgpu.WorkSpace(spec, ctx)
    ff = pdgpu.Forcefield(ws)
    if with_bonded:
        ff.add(pdgpu.FF_Bonded(ws))
    gb = pdgpu.FF_GeneralizedBorn_Still(ws)
    gb.Cutoff = float(meta["cutoff"])
    gb.InnerCutoff = float(meta["inner"])
    gb.VdwCutoff = float(meta["vdwcut"])
    gb.VdwInnerCutoff = float(meta["vdwinner"])
    ff.add(gb)
    ff.ensuresetup()
    return ws, ff, arrays, meta


def energy_close(got_J, ref_J, rel=1e-5, abs_kcal=1e-3):
    return abs(got_J - ref_J) * J2K <= max(rel * abs(ref_J) * J2K, abs_kcal)


@pytest.mark.parametrize("name", SMALL)
def test_neighbour_list_bit_exact(name, gpu_ctx):
    ws, ff, a, _ = make(name, gpu_ctx)
    ws.nlist().calcNewList()
    ptr, data = ws.nlist().getData(shadow=True)
    assert np.array_equal(ptr, a["nl_ptr"])
    assert np.array_equal(data, a["nl_data"])
    # the half list the reference builds without CalcShadow (limit = i)
    S = O.System(a, cutoff=float(ws.spec.meta["cutoff"]))
    hp, hd = S.nlist(a["pos"], shadow=False)
    p2, d2 = ws.nlist().getData(shadow=False)
    assert np.array_equal(p2, hp) and np.array_equal(d2, hd)


@pytest.mark.parametrize("name", SMALL)
def test_gb_bonded_forces_and_energies(name, gpu_ctx):
    ws, ff, a, _ = make(name, gpu_ctx)
    ws.nlist().calcNewList()
    ff.calcForces()
    born = ws.born_radii()
    assert np.max(np.abs(born - a["born"]) / np.abs(a["born"])) <= 2e-6
    assert rel_rms(ws.cur.f, a["f_total"]) <= 1e-5
    et = a["ene_total"]
    e = ws.ene
    for field, idx in (("epot_vdw", 1), ("epot_elec", 2), ("epot_pol", 3), ("epot_pol_cross", 4),
                       ("epot_pol_self", 5), ("epot", 0)):
        assert energy_close(getattr(e, field), et[idx]), (field, getattr(e, field) * J2K, et[idx] * J2K)
    for field, idx in (("epot_bond", 6), ("epot_angle", 7), ("epot_torsion", 8)):
        assert getattr(e, field) == pytest.approx(et[idx], rel=1e-9), field


@pytest.mark.parametrize("name", SMALL)
def test_gb_component_alone(name, gpu_ctx):
    ws, ff, a, _ = make(name, gpu_ctx, with_bonded=False)
    ws.nlist().calcNewList()
    ff.calcForces()
    assert rel_rms(ws.cur.f, a["f_gb"]) <= 1e-5
    # Newton's third law: the pair forces cancel to FP32 rounding
    assert np.linalg.norm(ws.cur.f.sum(0)) <= 1e-5 * np.abs(ws.cur.f).sum()


@pytest.mark.parametrize("name", SMALL)
def test_energy_only_path(name, gpu_ctx):
    import pdgpu
    ws, ff, a, _ = make(name, gpu_ctx, with_bonded=False)
    ws.nlist().calcNewList()
    ff.calcEnergies()
    ep = a["ene_energypath"]
    e = np.zeros(16)
    from pdgpu import _abi as A
    A.check(A.lib().pdgpu_get_energies(ws.ctx.ptr, ws._sys, A.dptr(e), 16))
    assert energy_close(e[A.ENE_VDW], ep[1])
    assert energy_close(e[A.ENE_ELEC], ep[2])
    assert energy_close(e[A.ENE_GB_COMPONENT], ep[10])
    assert energy_close(e[A.ENE_EPOT], ep[0])
    assert energy_close(e[A.ENE_VIRIAL], ep[9])
    # the energy path applies the vacuum LJ/Coulomb forces, as the reference
    assert rel_rms(ws.cur.f, a["f_energypath"]) <= 1e-5


@pytest.mark.parametrize("name", SMALL)
def test_bit_reproducible(name, gpu_ctx):
    ws, ff, a, _ = make(name, gpu_ctx)
    ws.nlist().calcNewList()
    ff.calcForces()
    f1, e1 = ws.cur.f.copy(), ws.ene.epot
    ws.nlist().calcNewList()
    ff.calcForces()
    assert np.array_equal(f1, ws.cur.f) and e1 == ws.ene.epot


@pytest.mark.parametrize("name", ["pep8_s1", "pep20_s2"])
@pytest.mark.parametrize("kind,integ", [("mdlv_", 3), ("mdvv_", 1), ("mdbm_", 2)])
def test_integrator_steps_with_reference_normals(name, kind, integ, gpu_ctx):
    """Each step starts from the reference's own state; forces are the GPU's."""
    from pdgpu import _abi as A
    import ctypes
    ws, ff, a, _ = make(name, gpu_ctx)
    K = a[kind + "x"].shape[0]
    p = A.md_params_default()
    p.Integrator, p.FricCoeff, p.Timestep, p.TargetTemp = integ, 1e12, 1e-15, 300.0
    x, v = a[kind + "x0"], a[kind + "v0"]
    fold = np.zeros_like(x)
    for s in range(K):
        ws.cur.p[:] = x
        ws._push_positions()
        ws.cur.v[:] = v
        ws._push_velocities()
        if integ == 2:  # Beeman keeps the previous force
            pass
        ws.nlist().calcNewList()
        ff.calcForces()
        normals = A.cd(a[kind + "normals"][s])
        A.check(A.lib().pdgpu_md_step_with_normals(ws.ctx.ptr, ws._sys, ctypes.byref(p), s, K,
                                                   A.dptr(normals)))
        ws._pull_positions()
        ws._pull_velocities()
        dx_ref = a[kind + "x"][s] - x
        dv_ref = a[kind + "v"][s] - v
        assert rel_rms(ws.cur.p - x, dx_ref) <= 1e-5
        assert rel_rms(ws.cur.v - v, dv_ref) <= 1e-5
        x, v = a[kind + "x"][s], a[kind + "v"][s]


@pytest.mark.parametrize("name", ["pep8_s1", "pep20_s2"])
@pytest.mark.parametrize("alg", ["sd", "cg"])
def test_minimiser_matches_reference(name, alg, gpu_ctx):
    import pdgpu
    ws, ff, a, _ = make(name, gpu_ctx)
    pre = "min%s_" % alg
    r = a[pre + "result"]
    ws.cur.p[:] = a[pre + "x0"]
    ws._pos_dirty = True
    m = pdgpu.Minimisation(ff)
    m.Algorithm = pdgpu.Minimisation.SteepestDescent if alg == "sd" else pdgpu.Minimisation.ConjugateGradients
    m.Steps = int(r[0])
    taken = m.run()
    assert taken == int(r[0])
    assert np.max(np.abs(ws.cur.p - a[pre + "x"])) <= 1e-4
    assert energy_close(ws.ene.epot, r[1], rel=1e-5)


def test_full_size_large_system(gpu_ctx):
    """The 16 x 80-residue, ~20.6k-atom, Rc 16 system: Born radii, forces and
    energies against the reference, and the full pair set against the
    oracle (the reference's O(N^2) list restated)."""
    ws, ff, a, meta = make("c2_16x80_s2", gpu_ctx)
    ws.nlist().calcNewList()
    ff.calcForces()
    born = ws.born_radii()
    assert np.max(np.abs(born - a["born"]) / np.abs(a["born"])) <= 2e-6
    assert rel_rms(ws.cur.f, a["f_total"]) <= 1e-5
    et = a["ene_total"]
    for field, idx in (("epot_vdw", 1), ("epot_elec", 2), ("epot_pol", 3), ("epot", 0)):
        assert energy_close(getattr(ws.ene, field), et[idx], abs_kcal=0.05), field
    ptr, data = ws.nlist().getData(shadow=True)
    S = O.System(a, cutoff=float(meta["cutoff"]))
    optr, odata = S.nlist(a["pos"])
    assert np.array_equal(ptr, optr) and np.array_equal(data, odata)


def test_md_graph_and_eager_agree(gpu_ctx):
    """The CUDA-graph step loop and the eager loop run the same kernels:
    identical trajectories bit for bit."""
    import pdgpu
    outs = []
    for use_graph in (True, False):
        ws, ff, a, _ = make("c1_pep64_s0", gpu_ctx)
        ws.setLanes((8, 8, 8))  # the same kernel variants in both runs
        md = pdgpu.MolecularDynamics(ff)
        md.Integrator = pdgpu.MolecularDynamics.Langevin
        md.FricCoeff = 1e12
        md.Steps = 40
        md.UpdateNList = 10
        md.UseGraph = use_graph
        md.Seed = 7
        md.run()
        outs.append((ws.cur.p.copy(), ws.cur.v.copy(), md.history.copy()))
        assert np.all(np.isfinite(md.history))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    bad = np.argwhere(outs[0][2] != outs[1][2])
    assert len(bad) == 0, (bad[:10].tolist(), outs[0][2][tuple(bad[0])], outs[1][2][tuple(bad[0])])


def test_langevin_temperature_is_sane(gpu_ctx):
    import pdgpu
    ws, ff, a, _ = make("c1_pep64_s0", gpu_ctx)
    md = pdgpu.MolecularDynamics(ff)
    md.Integrator = pdgpu.MolecularDynamics.Langevin
    md.FricCoeff = 1e13
    md.Steps = 200
    md.Seed = 3
    md.run()
    n = ws.nAtoms()
    kB = 1.38065e-23
    T = 2 * md.history[:, 1] / (3 * n * kB)
    assert 150 < T[-50:].mean() < 450
