"""GPU: the cluster-pair tile layout of the three pair passes.

The tiles re-cut the neighbour list into 32 x 8 atom blocks; they must hold
exactly the list's pairs, and the tile passes must give the row passes'
results.  Tolerances:
  unordered pairs held by the tiles   exactly half the (full) list entries
  Born radii, tiles vs rows           bit-exact (the same FP32 terms, each
                                      added in 64-bit fixed point)
  forces, tiles vs rows               relative RMS 1e-6 (FP32 partial sums
                                      in another order)
  forces vs the reference             relative RMS 1e-5
  tiles alone vs in a batch           bit-exact (no lanes, per-system tiles)
"""
import numpy as np
import pytest

from conftest import build_workspace, fixture_names, load_fixture, load_library, rel_rms

pytestmark = pytest.mark.gpu

SMALL = fixture_names()
J2K = (1.0 / 4184.0) * 6.0221418e23


def _counts(ws):
    import ctypes
    import pdgpu
    c = np.zeros(5, dtype=np.int64)
    assert pdgpu.lib().pdgpu_pair_counts(ws.ctx.ptr, ws._sys, c.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))) == 0
    return c


@pytest.mark.parametrize("name", SMALL + ["c2_16x80_s2"])
def test_tiles_hold_the_list_pairs(name, gpu_ctx):
    arrays, meta = load_fixture(name)
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    ws.nlist().calcNewList()
    c = _counts(ws)
    assert c[2] % 2 == 0 and c[3] == c[2] // 2
    assert c[4] > 0 and c[3] <= 256 * c[4]


def _eval(ws, ff, path):
    assert ws.setPairPath(path) == path
    ws.nlist().calcNewList()
    ff.calcForces()
    import pdgpu
    ep = np.zeros(ws.nAtoms())
    import ctypes
    pdgpu.lib().pdgpu_get_atom_epot(ws.ctx.ptr, ws._sys, ep.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return ws.cur.f.copy(), ws._pull_energies(), ws.born_radii(), ep


@pytest.mark.parametrize("name", SMALL + ["c2_16x80_s2"])
def test_tiles_match_rows_and_reference(name, gpu_ctx):
    arrays, meta = load_fixture(name)
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    f_r, e_r, b_r, ep_r = _eval(ws, ff, 0)
    f_t, e_t, b_t, ep_t = _eval(ws, ff, 1)
    assert np.array_equal(b_t, b_r)
    assert rel_rms(f_t, f_r) <= 1e-6
    assert rel_rms(f_t, arrays["f_total"]) <= 1e-5
    for k in range(6):  # epot, vdw, elec, pol, pol_cross, pol_self
        assert abs(e_t[k] - e_r[k]) * J2K <= max(1e-6 * abs(e_r[k]) * J2K, 1e-4), k
    assert abs(e_t[0] - arrays["ene_total"][0]) * J2K <= max(1e-5 * abs(arrays["ene_total"][0]) * J2K, 1e-3)
    assert rel_rms(ep_t, ep_r) <= 1e-6


def test_tiles_batch_equals_alone_bitwise(gpu_ctx):
    import pdgpu
    members = [build_workspace(a, m, gpu_ctx) + (a, m) for a, m in load_library("lib16_amber_s3")[:8]]
    alone = []
    for ws, ff, a, m in members:
        one = pdgpu.Batch([ws])
        one.setPairPath(1)
        f, e = one.evaluate()
        alone.append((f, e[0], one.born_radii()))
        one.close()
    b = pdgpu.Batch([ws for ws, *_ in members])
    b.setPairPath(1)
    f, e = b.evaluate()
    born = b.born_radii()
    for s, (ws, ff, a, m) in enumerate(members):
        assert np.array_equal(b.split(f)[s], alone[s][0])
        assert np.array_equal(e[s], alone[s][1])
        assert np.array_equal(b.split(born)[s], alone[s][2])
        assert rel_rms(b.split(f)[s], a["f_total"]) <= 1e-5
    b.close()


def test_tiles_clashing_trial(gpu_ctx):
    """A trial structure with forces near 1e10 kcal/mol/A (the reference's
    recorded two-chain trial 0): the fixed-point j side keeps the range."""
    arrays, meta = load_fixture("two_chain_s4")
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    ws.setPairPath(1)
    ws.setTorsionMoves()
    ws.saveBasePositions()
    for t in range(arrays["trial_angles"].shape[0]):
        ws.perturbTorsions(angles=arrays["trial_angles"][t])
        ws.nlist().calcNewList()
        ff.calcForces()
        assert rel_rms(ws.cur.f, arrays["trial_f"][t]) <= 1e-5


def test_tiles_md_graph_and_eager_agree(gpu_ctx):
    import pdgpu
    arrays, meta = load_fixture("c1_pep64_s0")
    outs = []
    for use_graph in (True, False):
        ws, ff = build_workspace(arrays, meta, gpu_ctx)
        ws.setPairPath(1)
        md = pdgpu.MolecularDynamics(ff)
        md.Integrator = pdgpu.MolecularDynamics.Langevin
        md.FricCoeff = 1e12
        md.Steps = 40
        md.UpdateNList = 10
        md.UseGraph = use_graph
        md.Seed = 7
        md.run()
        outs.append((ws.cur.p.copy(), md.history.copy()))
        assert ws.setPairPath(-2) == 1
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


def _forces_energies(ws, ff):
    ff.calcForces()
    return ws.cur.f.copy(), ws._pull_energies().copy(), ws.born_radii().copy()


@pytest.mark.parametrize("name", SMALL + ["c2_16x80_s2"])
def test_tile_search_equals_tiles_from_the_list(name, gpu_ctx):
    """Tiles searched straight from the positions hold the same pairs as the
    tiles cut from the list: every result is bit-identical (all tile sums
    are fixed point, so the tiles' order does not matter)."""
    arrays, meta = load_fixture(name)
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    assert ws.setPairPath(0) == 0
    ws.nlist().calcNewList()           # the list
    assert ws.setPairPath(1) == 1      # tiles cut from it
    f_l, e_l, b_l = _forces_energies(ws, ff)
    ws.nlist().calcNewList()           # on the tile layout: the tile search
    f_s, e_s, b_s = _forces_energies(ws, ff)
    assert np.array_equal(b_s, b_l)
    assert np.array_equal(f_s, f_l)
    assert np.array_equal(e_s, e_l)
    c = _counts(ws)                    # the list, built now at the same positions
    assert c[3] == c[2] // 2


@pytest.mark.parametrize("name", SMALL)
def test_list_after_a_tile_search_is_the_list(name, gpu_ctx):
    """After a tile search the list is built when read, at the positions of
    the search: the same entries as a list build there."""
    arrays, meta = load_fixture(name)
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    ws.setPairPath(0)
    ws.nlist().calcNewList()
    ptr_r, data_r = ws.nlist().getData()
    ws.setPairPath(1)
    ws.nlist().calcNewList()           # tiles only
    ptr_s, data_s = ws.nlist().getData()
    assert np.array_equal(ptr_s, ptr_r)
    assert np.array_equal(data_s, data_r)


def test_tile_md_rebuilds_keep_list_and_tiles_consistent(gpu_ctx):
    """MD on the tile layout rebuilds by tile search; the list read
    afterwards (built at the last rebuild's positions) holds exactly the
    tiles' pairs, and the row passes then give the tile passes' forces."""
    import pdgpu
    arrays, meta = load_fixture("c1_pep64_s0")
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    ws.setPairPath(1)
    md = pdgpu.MolecularDynamics(ff)
    md.Integrator = pdgpu.MolecularDynamics.Langevin
    md.FricCoeff = 1e12
    md.Steps = 25
    md.UpdateNList = 10
    md.Seed = 3
    md.run()
    c = _counts(ws)
    assert c[3] == c[2] // 2 and c[4] > 0
    f_t, e_t, _ = _forces_energies(ws, ff)
    ws.setPairPath(0)
    f_r, e_r, _ = _forces_energies(ws, ff)
    assert rel_rms(f_t, f_r) <= 1e-6
