"""Edge cases of the pair structures: systems with one atom, with no pair
inside the cutoff, with a single pair, and with pairs across the cutoff
edge, built from atom parameters of the reference-built library (no bonded
terms, so every pair is a non-bonded pair of bond order 7).  Each is
evaluated on both pair layouts and compared with the oracle's FP64
evaluation at the same coordinates: the same neighbour pairs, Born radii to
2e-6, relative force RMS to 1e-5 (absolute 1e-12 N where the forces are
zero), energies to 1e-5 relative or 1e-6 kcal/mol; a short MD run stays
finite."""
import numpy as np
import pytest

from conftest import build_workspace, load_library, rel_rms

import oracle as O

pytestmark = pytest.mark.gpu

J2K = (1.0 / 4184.0) * 6.0221418e23
_ATOM = ("charge", "radius", "epsilon", "gb_radius", "mass", "is_h")


def _system(pos, picks):
    """Atoms with the parameters of library atoms `picks`, at `pos`, with
    no bonds."""
    a, m = load_library("lib16_amber_s3")[3]
    n = len(pos)
    out = {f: np.asarray(a[f])[list(picks)].copy() for f in _ATOM}
    out["ir"] = np.arange(n, dtype=np.int32)
    out["pos"] = np.asarray(pos, dtype=np.float64)
    for c in ("cov12", "cov13", "cov14"):
        out[c + "_ptr"] = np.zeros(n + 1, dtype=np.int32)
        out[c + "_idx"] = np.zeros(0, dtype=np.int32)
    out["cov12_d"] = np.zeros(0)
    out["cov13_d"] = np.zeros(0)
    out["bond_ij"], out["bond_lk"] = np.zeros((0, 2), np.int32), np.zeros((0, 2))
    out["angle_iaj"], out["angle_kt"] = np.zeros((0, 3), np.int32), np.zeros((0, 2))
    for t in ("tors", "impr"):
        out[t + "_idx"] = np.zeros((0, 4), np.int32)
        out[t + "_terms"] = np.zeros(0, np.int32)
        out[t + "_par"] = np.zeros((0, 12))
    out["backbone_ncac"] = np.zeros((0, 3), np.int32)
    out["ff_params"] = np.asarray(a["ff_params"])
    meta = {k: m[k] for k in ("cutoff", "inner", "vdwcut", "vdwinner", "param")}
    meta["natoms"] = str(n)
    return out, meta


# heavy atoms of library peptide 3 with charges of both signs
_PICK = (4, 8, 12, 20, 27, 33)
CASES = {
    "one_atom": [[0.0, 0.0, 0.0]],
    "no_pair_in_cutoff": [[0.0, 0.0, 0.0], [30.0, 0.0, 0.0]],
    "one_pair": [[0.0, 0.0, 0.0], [4.5, 0.0, 0.0]],
    "across_the_edges": [[0.0, 0.0, 0.0], [3.8, 0.0, 0.0], [0.0, 9.5, 0.0], [0.0, 0.0, 11.9],
                         [12.4, 0.0, 0.0], [7.0, 7.0, 7.0]],
}


@pytest.mark.parametrize("path", [1, 0])
@pytest.mark.parametrize("case", sorted(CASES))
def test_small_systems_match_the_oracle(case, path, gpu_ctx):
    pos = CASES[case]
    arrays, meta = _system(pos, _PICK[:len(pos)])
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    assert ws.setPairPath(path) == path
    ws.nlist().calcNewList()
    ff.calcForces()
    S = O.System(arrays, cutoff=float(meta["cutoff"]), inner=float(meta["inner"]))
    ptr, data = S.nlist(arrays["pos"])
    gptr, gdata = ws.nlist().getData(shadow=True)
    assert np.array_equal(gptr, ptr) and np.array_equal(gdata, data)
    f_ref, e_ref, born_ref = S.calc_forces(arrays["pos"], ptr, data)
    born = ws.born_radii()
    assert np.max(np.abs(born - born_ref) / np.abs(born_ref)) <= 2e-6
    if np.any(f_ref != 0.0):
        assert rel_rms(ws.cur.f, f_ref) <= 1e-5
    else:
        assert np.max(np.abs(ws.cur.f)) <= 1e-12
    got, ref = ws.ene.epot * J2K, e_ref["epot"] * J2K
    assert abs(got - ref) <= max(1e-5 * abs(ref), 1e-6), (got, ref)
    ws.close()


def test_small_system_md_stays_finite(gpu_ctx):
    import pdgpu
    pos = CASES["across_the_edges"]
    arrays, meta = _system(pos, _PICK[:len(pos)])
    ws, ff = build_workspace(arrays, meta, gpu_ctx)
    assert ws.setPairPath(1) == 1
    md = pdgpu.MolecularDynamics(ff)
    md.Integrator = pdgpu.MolecularDynamics.Langevin
    md.FricCoeff = 1e12
    md.Steps = 30
    md.UpdateNList = 10
    md.Seed = 2
    md.run()
    assert np.all(np.isfinite(md.history)) and np.all(np.isfinite(ws.cur.p))
    ws.close()


def test_batch_with_tiny_members_equals_alone(gpu_ctx):
    """A batch holding a one-atom system, a pairless system, a peptide and a
    six-atom system: every member's forces and energies are the bits it
    gets alone."""
    import pdgpu
    a, m = load_library("lib16_amber_s3")[0]
    specs = [_system(CASES["one_atom"], _PICK[:1]), _system(CASES["no_pair_in_cutoff"], _PICK[:2]),
             (a, m), _system(CASES["across_the_edges"], _PICK)]
    alone = []
    for arrays, meta in specs:
        ws, ff = build_workspace(arrays, meta, gpu_ctx)
        ws.setPairPath(1)
        ws.nlist().calcNewList()
        ff.calcForces()
        alone.append((ws.cur.f.copy(), ws.ene.epot))
        ws.close()
    members = [build_workspace(arrays, meta, gpu_ctx)[0] for arrays, meta in specs]
    b = pdgpu.Batch(members)
    b.setPairPath(1)
    f, e = b.evaluate()
    for s, (fa, ea) in enumerate(alone):
        assert np.array_equal(b.split(f)[s], fa), s
        assert e[s][0] == ea, s
    b.close()
    for ws in members:
        ws.close()
