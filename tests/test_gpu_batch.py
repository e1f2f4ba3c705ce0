"""GPU: batches (many systems in one device pack) and backbone trial moves.

Each member of a batch must get the results it gets alone, and both must
match the reference.  Tolerances:
  neighbour list (per member)        bit-exact
  batch vs alone, same lanes per atom: forces, energies, Born radii,
      MD and minimiser trajectories   bit-exact
  batch vs alone, each autotuned     relative force RMS 1e-6 (the FP32
      per-lane partial sums of a row split over another number of lanes)
  batch vs reference forces          relative force RMS 1e-5
  trial positions vs reference       1e-9 A (rotation matrices composed in
      another order than the reference's bond-by-bond rotations)
  trial moves alone vs in a batch    bit-exact (same per-system arithmetic)
"""
import ctypes

import numpy as np
import pytest

from conftest import build_workspace, load_fixture, load_library, rel_rms

import oracle as O

pytestmark = pytest.mark.gpu

J2K = (1.0 / 4184.0) * 6.0221418e23


def _library(ctx, name, count=None):
    lib = load_library(name)[:count]
    return [build_workspace(a, m, ctx) + (a, m) for a, m in lib]


@pytest.mark.parametrize("lanes", [(8, 8, 8), (4, 16, 32), None])
def test_batch_matches_alone_and_reference(gpu_ctx, lanes):
    import pdgpu
    members = _library(gpu_ctx, "lib16_amber_s3", 8)
    alone_f, alone_e, alone_b = [], [], []
    for ws, ff, a, m in members:
        one = pdgpu.Batch([ws])  # the same evaluation call, one system
        if lanes:
            one.setLanes(lanes)
        f1, e1 = one.evaluate()
        alone_f.append(f1)
        alone_e.append(e1[0])
        alone_b.append(one.born_radii())
        one.close()
    b = pdgpu.Batch([ws for ws, *_ in members])
    if lanes:
        b.setLanes(lanes)
    f, e = b.evaluate()
    born = b.born_radii()
    for s, (ws, ff, a, m) in enumerate(members):
        fs = b.split(f)[s]
        if lanes:
            assert np.array_equal(fs, alone_f[s])
            assert np.array_equal(e[s], alone_e[s])
            assert np.array_equal(b.split(born)[s], alone_b[s])
        else:
            assert rel_rms(fs, alone_f[s]) <= 1e-6
            # Born sums add fixed-point terms: exact whatever the lane count
            assert np.array_equal(b.split(born)[s], alone_b[s])
        assert rel_rms(fs, a["f_total"]) <= 1e-5
        assert abs(e[s][0] - a["ene_total"][0]) * J2K <= max(1e-5 * abs(a["ene_total"][0]) * J2K, 1e-3)
    b.close()


def test_batch_neighbour_lists_per_member(gpu_ctx):
    import pdgpu
    members = _library(gpu_ctx, "lib16_amber_s3", 5)
    b = pdgpu.Batch([ws for ws, *_ in members])
    b.calcNewList()
    n = b.nAtoms
    ptr = np.zeros(n + 1, dtype=np.int32)
    cnt = ctypes.c_int64(0)
    L = pdgpu.lib()
    assert L.pdgpu_nlist_export(gpu_ctx.ptr, b._id, 1, ptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), None, 0,
                                ctypes.byref(cnt)) == 0
    data = np.zeros(cnt.value, dtype=np.int32)
    assert L.pdgpu_nlist_export(gpu_ctx.ptr, b._id, 1, ptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                data.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), cnt.value,
                                ctypes.byref(cnt)) == 0
    for s, (ws, ff, a, m) in enumerate(members):
        o0, o1 = b.offsets[s], b.offsets[s + 1]
        S = O.System(a, cutoff=float(m["cutoff"]))
        rp, rd = S.nlist(a["pos"], shadow=True)
        p = ptr[o0:o1 + 1] - ptr[o0]
        d = data[ptr[o0]:ptr[o1]]
        assert np.array_equal(p, rp)
        # entries hold packed-batch indices: back to member-local ones
        j = (d & 0xFFFFFF) - o0
        assert j.min() >= 0 and j.max() < o1 - o0
        assert np.array_equal(j | (d & ~0xFFFFFF), rd)
    b.close()


@pytest.mark.parametrize("name", ["pep20_s2", "two_chain_s4"])
def test_trial_moves_match_reference(name, gpu_ctx):
    arrays, meta = load_fixture(name)
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    nrot = ws.setTorsionMoves()
    assert nrot == arrays["trial_angles"].shape[1]
    ws.saveBasePositions()
    for t in range(arrays["trial_angles"].shape[0]):
        ws.perturbTorsions(angles=arrays["trial_angles"][t])
        assert np.abs(ws.cur.p - arrays["trial_pos"][t]).max() <= 1e-9
        ws.nlist().calcNewList()
        ff.calcForces()
        assert rel_rms(ws.cur.f, arrays["trial_f"][t]) <= 1e-5
        et = arrays["trial_ene"][t]
        assert abs(ws.ene.epot - et[0]) * J2K <= max(1e-5 * abs(et[0]) * J2K, 1e-3)


def test_trial_moves_batch_equals_alone(gpu_ctx):
    """Philox-drawn trial moves: a member draws the same angles alone and in
    a batch (its stream depends on its own key and the trial number only),
    and the moved structures' forces agree with the reference's forces of
    the library's recorded trials in distribution (the moves are real)."""
    import pdgpu
    members = _library(gpu_ctx, "lib16_amber_s3", 6)
    sigma = np.deg2rad(15.0)
    keys = np.arange(100, 106, dtype=np.uint64)
    alone = []
    for s, (ws, ff, a, m) in enumerate(members):
        ws.setTorsionMoves()
        ws.saveBasePositions()
    b = pdgpu.Batch([ws for ws, *_ in members])
    b.setSeeds(keys)
    b.saveBasePositions()
    for s, (ws, ff, a, m) in enumerate(members):
        one = pdgpu.Batch([ws])
        one.setSeeds(keys[s:s + 1])
        one.saveBasePositions()
        one.perturbTorsions(sigma=sigma, trial=7)
        alone.append(one.positions())
        one.close()
    b.perturbTorsions(sigma=sigma, trial=7)
    pos = b.positions()
    for s, (ws, ff, a, m) in enumerate(members):
        p = b.split(pos)[s]
        assert np.array_equal(p, alone[s])
        moved = np.abs(p - a["pos"]).max()
        assert 0.5 < moved < 500.0
    # a different trial number draws different angles
    b.perturbTorsions(sigma=sigma, trial=8)
    assert not np.array_equal(b.positions(), pos)
    b.close()


def test_batch_md_matches_alone(gpu_ctx):
    import pdgpu
    members = _library(gpu_ctx, "lib16_opls_s4", 4)
    p = pdgpu.md_params_default()
    p.Integrator = pdgpu.MolecularDynamics.Langevin
    p.FricCoeff = 1e12
    p.Timestep = 1e-15
    p.UpdateNList = 10
    keys = np.arange(7, 11, dtype=np.uint64)
    alone_pos, alone_hist = [], []
    for s, (ws, ff, a, m) in enumerate(members):
        one = pdgpu.Batch([ws])
        one.setSeeds(keys[s:s + 1])
        one.setLanes((8, 8, 8))
        one.calcNewList()
        h = one.runMD(p, 20, init_velocities=300.0)
        alone_pos.append(one.positions())
        alone_hist.append(h[:, 0, :])
        one.close()
    b = pdgpu.Batch([ws for ws, *_ in members])
    b.setSeeds(keys)
    b.setLanes((8, 8, 8))
    b.calcNewList()
    h = b.runMD(p, 20, init_velocities=300.0)
    pos = b.positions()
    for s in range(len(members)):
        assert np.array_equal(b.split(pos)[s], alone_pos[s])
        assert np.array_equal(h[:, s, :], alone_hist[s])
        # Langevin at 300 K keeps the kinetic energy near 3/2 N kB T
        n = b.offsets[s + 1] - b.offsets[s]
        ek_expected = 1.5 * n * 1.38065e-23 * 300.0
        assert 0.5 * ek_expected < h[-1, s, 1] < 1.5 * ek_expected
    b.close()


def test_batch_minimise_matches_alone(gpu_ctx):
    import pdgpu
    members = _library(gpu_ctx, "lib16_amber_s3", 4)
    p = pdgpu.min_params_default()
    p.Algorithm = pdgpu.Minimisation.SteepestDescent
    alone_taken, alone_pos = [], []
    for ws, ff, a, m in members:
        one = pdgpu.Batch([ws])
        one.setLanes((8, 8, 8))
        alone_taken.append(int(one.minimise(p, 30)[0]))
        alone_pos.append(one.positions())
        one.close()
    b = pdgpu.Batch([ws for ws, *_ in members])
    b.setLanes((8, 8, 8))
    taken = b.minimise(p, 30)
    pos = b.positions()
    for s in range(len(members)):
        assert taken[s] == alone_taken[s] == 30
        assert np.array_equal(b.split(pos)[s], alone_pos[s])
    b.close()
