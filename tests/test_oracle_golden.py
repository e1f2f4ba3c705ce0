"""CPU: pin the oracle (oracle/pd_oracle.c) against the reference's own
outputs.

The fixtures under tests/golden/ were produced by the reference library
compiled from its sources (oracle/Makefile) on seeded synthetic peptides
(tests/golden/make_golden.py).  The restatement follows the reference's
operation order and is built without fast-math, so every quantity here
matches to the last bit except where noted; the tolerances state that.
"""
import numpy as np
import pytest

from conftest import fixture_names, load_fixture, rel_rms

import oracle as O

SMALL = fixture_names()


def _system(name):
    arrays, meta = load_fixture(name)
    S = O.System(arrays, cutoff=float(meta["cutoff"]), inner=float(meta["inner"]))
    return S, arrays, meta


@pytest.mark.parametrize("name", SMALL)
def test_bondorder_matches_reference(name):
    S, a, _ = _system(name)
    assert S.mid == int(a["bo_mid"][0])
    assert np.array_equal(S.band, a["bo_band"])
    assert S.n_off == a["bo_offdiag"].shape[0]


@pytest.mark.parametrize("name", SMALL)
def test_still_fixed_terms_bit_exact(name):
    S, a, _ = _system(name)
    assert np.array_equal(S.vj, a["gb_vj"])
    assert np.array_equal(S.terms123, a["gb_terms123"])


@pytest.mark.parametrize("name", SMALL)
def test_neighbour_list_bit_exact(name):
    S, a, _ = _system(name)
    ptr, data = S.nlist(a["pos"])
    assert np.array_equal(ptr, a["nl_ptr"])
    assert np.array_equal(data, a["nl_data"])


@pytest.mark.parametrize("name", SMALL)
def test_gb_forces_and_energies(name):
    S, a, _ = _system(name)
    ptr, data = S.nlist(a["pos"])
    f, e, born = S.calc_forces(a["pos"], ptr, data)
    assert np.array_equal(born, a["born"])
    assert rel_rms(f, a["f_total"]) <= 1e-14
    et = a["ene_total"]
    # component sums are order-identical; the total sums components in a
    # different order than Forcefield::calcForces, hence the 1e-12 relative
    for k, idx in (("vdw", 1), ("elec", 2), ("pol", 3), ("pol_cross", 4), ("pol_self", 5),
                   ("bond", 6), ("angle", 7), ("torsion", 8)):
        assert e[k] == pytest.approx(et[idx], rel=1e-13, abs=1e-30), k
    assert e["epot"] == pytest.approx(et[0], rel=1e-12)
    fg, eg, _, _, _ = S.gb_forces(a["pos"], ptr, data)
    assert rel_rms(fg, a["f_gb"]) <= 1e-14
    fb, eb = S.bonded_forces(a["pos"])
    assert rel_rms(fb, a["f_bonded"]) <= 1e-14


@pytest.mark.parametrize("name", SMALL)
def test_energy_path(name):
    S, a, _ = _system(name)
    ptr, data = S.nlist(a["pos"])
    f, ene, epol, pol, _ = S.energies_path(a["pos"], ptr, data)
    ep = a["ene_energypath"]
    assert rel_rms(f, a["f_energypath"]) <= 1e-14
    assert ene[1] == pytest.approx(ep[1], rel=1e-13)
    assert ene[2] == pytest.approx(ep[2], rel=1e-13)
    assert epol == pytest.approx(ep[10], rel=1e-13)
    assert ene[3] == pytest.approx(ep[9], rel=1e-13)  # virial


@pytest.mark.parametrize("name", [n for n in SMALL if "md" in n or n in ("pep8_s1", "pep20_s2")])
@pytest.mark.parametrize("kind", ["mdlv_", "mdvv_", "mdbm_"])
def test_integrator_steps_bit_exact(name, kind):
    S, a, _ = _system(name)
    if kind + "x" not in a:
        pytest.skip("no MD record")
    x = a[kind + "x0"].reshape(-1)
    v = a[kind + "v0"].reshape(-1)
    fold = np.zeros_like(x)
    K = a[kind + "x"].shape[0]
    for s in range(K):
        fr = a[kind + "f"][s].reshape(-1)
        if kind == "mdlv_":
            x, v, ek = O.langevin_step(x, v, fr, S.mass, a[kind + "normals"][s].reshape(-1), 1e-15, 1e12, 300.0, s, K)
        elif kind == "mdvv_":
            x, v, ek = O.velocity_verlet_step(x, v, fr, S.mass, 1e-15)
        else:
            x, v, fold, ek = O.beeman_step(x, v, fr, fold, S.mass, 1e-15, s, K)
        assert np.array_equal(x, a[kind + "x"][s].reshape(-1))
        assert np.array_equal(v, a[kind + "v"][s].reshape(-1))
        assert ek == a[kind + "ekin"][s]


@pytest.mark.parametrize("name", ["pep8_s1", "pep20_s2"])
@pytest.mark.parametrize("alg", ["sd", "cg"])
def test_minimiser_trajectory_bit_exact(name, alg):
    S, a, _ = _system(name)
    pre = "min%s_" % alg
    r = a[pre + "result"]
    taken, x, e, mult = O.minimise(S, a[pre + "x0"], int(r[0]), alg)
    assert taken == int(r[0])
    assert np.array_equal(x, a[pre + "x"])
    assert mult == r[2]
    assert e["epot"] == pytest.approx(r[1], rel=1e-12)


def test_constants_match_reference_definitions():
    c = O.constants()
    # forcefield.cpp:18-38: econv is the Coulomb energy of two unit charges
    # at 1 A in kcal/mol
    assert c["econv"] == pytest.approx(332.0636, rel=1e-6)
    assert c["halfeconv"] == c["econv"] * 0.5


def test_off_diagonal_bond_order_correction():
    """The sparse (off-band) bond orders overwrite list entries in both rows
    of a shadow list and only the lower row of a half list
    (neighbourlist.cpp:162-203).  Synthetic case: no seeded peptide has
    off-band covalent partners."""
    n = 6
    pos = np.zeros((n, 3))
    pos[:, 0] = np.arange(n) * 1.0
    band = np.full(1 * (n - 1), 7, dtype=np.int8)  # mid = 1: the band is empty
    off = np.array([0, 5, 1, 1, 4, 3], dtype=np.int32)  # (0,5)=1-2 (1,4)=1-4
    ptr = np.zeros(n + 1, dtype=np.int32)
    data = np.zeros(64, dtype=np.int32)
    L = O.lib()
    cnt = L.pdo_nlist(n, O._d(O._cd(pos).reshape(-1)), 10.0, 0.5, 1, 1, O._b(band), 2, O._i(off),
                      O._i(ptr), O._i(data), 64)
    d = data[:cnt]
    bo = {}
    for i in range(n):
        for k in range(ptr[i], ptr[i + 1]):
            bo[(i, d[k] & 0xFFFFFF)] = (d[k] >> 24) & 7
    assert bo[(0, 5)] == 1 and bo[(5, 0)] == 1
    assert bo[(1, 4)] == 3 and bo[(4, 1)] == 3
    assert bo[(0, 1)] == 7 and bo[(2, 3)] == 7


@pytest.mark.parametrize("name", [n for n in SMALL if n in ("pep20_s2", "two_chain_s4")])
def test_trial_moves_match_reference(name):
    """Backbone phi/psi trial conformations: the oracle's bond-by-bond
    restatement of MoleculeBase::rotateBond reproduces the reference's
    setResiduePhiPsi results from the recorded angles.  Not bit-exact: the
    reference rotates with matrix3x3 products in its own order (~1e-13 A)."""
    arrays, meta = load_fixture(name)
    ax = O.backbone_axes(arrays["backbone_ncac"])
    assert ax.shape[0] == arrays["trial_angles"].shape[1]
    for t in range(arrays["trial_angles"].shape[0]):
        x = O.apply_torsions(arrays["pos"], arrays["cov12_ptr"], arrays["cov12_idx"], ax, arrays["trial_angles"][t])
        assert np.abs(x - arrays["trial_pos"][t]).max() < 1e-10
        assert np.abs(arrays["trial_pos"][t] - arrays["pos"]).max() > 1.0  # the move did something


@pytest.mark.parametrize("name", [n for n in SMALL if n in ("pep20_s2", "two_chain_s4")])
def test_trial_forces_match_oracle(name):
    """The reference's single-point forces of each trial conformation agree
    with the oracle's at the same positions."""
    S, arrays, meta = _system(name)
    for t in range(arrays["trial_pos"].shape[0]):
        x = arrays["trial_pos"][t]
        ptr, data = S.nlist(x)
        f, e, _ = S.calc_forces(x, ptr, data)
        assert rel_rms(f, arrays["trial_f"][t]) < 1e-12
        assert e["epot"] == pytest.approx(arrays["trial_ene"][t][0], rel=1e-12, abs=1e-30)


# ------------------------------------------------------------------ LCPO
LCPO = [n for n in SMALL if n.startswith("lcpo_")]


@pytest.mark.parametrize("name", LCPO)
@pytest.mark.parametrize("dense", [False, True])
def test_lcpo_bit_exact(name, dense):
    """FF_SASA_LCPO alone: calcForces at Step 0 (forces path) and
    calcEnergies (energies path), on the built chain and on the dense
    packing whose overlap lists the reference truncates at 80 partners."""
    a, _ = load_fixture(name)
    c = O.constants()
    sig = O.lcpo_sigma_J(float(a["lcpo_cfg"][0]))
    pre = "lcpo_dense_" if dense else "lcpo_"
    pos = a["lcpo_dense_pos"] if dense else a["pos"]
    ptr, data = (a["lcpo_dense_nl_ptr"], a["lcpo_dense_nl_data"]) if dense else (a["nl_ptr"], a["nl_data"])
    sasa, deriv, e, lost = O.lcpo(pos, ptr, data, a["lcpo_radius"], a["lcpo_p"], sig, a["lcpo_use"])
    assert (lost > 0) == dense
    assert np.array_equal(deriv * (1 / c["Angstrom"]), a[pre + "f"])
    assert e == a[pre + "ene"][10] and e == a[pre + "ene"][0]  # epot_surf, epot
    assert np.all(sasa[a["lcpo_use"] == 0] == 0)
    s2, _, e2, _ = O.lcpo(pos, ptr, data, a["lcpo_radius"], a["lcpo_p"], sig, a["lcpo_use"], energy_only=True)
    assert e2 == a[pre + "ene_energypath"][10]


@pytest.mark.parametrize("name", LCPO)
def test_lcpo_in_the_forcefield_and_update_cadence(name):
    """{FF_Bonded, GB, LCPO}: the single point, then each velocity-Verlet
    step's forces from the reference's own positions, with the surface
    term recomputed only when Step % UpdateSasa == 0 and its forces of that
    step reused in between (lcpo.cpp:176-190)."""
    S, a, _ = _system(name)
    c = O.constants()
    sig = O.lcpo_sigma_J(float(a["lcpo_cfg"][0]))
    update = int(a["lcpo_cfg"][1])
    to_N = 1 / c["Angstrom"]

    def forces(pos, step, held):
        ptr, data = S.nlist(pos)
        f, e, _ = S.calc_forces(pos, ptr, data)
        if step % update == 0:
            sasa, deriv, esurf, _ = O.lcpo(pos, ptr, data, a["lcpo_radius"], a["lcpo_p"], sig, a["lcpo_use"])
            held[:] = [deriv, esurf]
        return f + held[0] * to_N, e["epot"] + held[1], held[1]

    held = [None, None]
    f, epot, esurf = forces(a["pos"], 0, held)
    assert rel_rms(f, a["lcpo_f_total"]) <= 1e-14
    assert esurf == a["lcpo_ene_total"][10]
    assert epot == pytest.approx(a["lcpo_ene_total"][0], rel=1e-12)
    x = a["lcpo_mdvv_x0"]
    K = a["lcpo_mdvv_f"].shape[0]
    assert K > update
    for s in range(K):
        f, epot, _ = forces(x, s, held)
        assert rel_rms(f, a["lcpo_mdvv_f"][s]) <= 1e-13, s
        assert epot == pytest.approx(a["lcpo_mdvv_epot"][s], rel=1e-12), s
        x = a["lcpo_mdvv_x"][s]
