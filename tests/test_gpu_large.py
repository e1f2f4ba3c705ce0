"""Systems above the tile search's atom limit (65,536 atoms a system): the
cluster-pair tiles then come from the neighbour list (k_tile_build) at every
rebuild.  Four copies of the 20,566-atom, Rc 16 system, set apart by more
than the cutoff, make one 82,264-atom system whose copies do not interact,
so each copy's forces and Born radii must be the reference's for the single
system (tests/golden/c2_16x80_s2.npz, made by the compiled reference) and
its pair energies four times the reference's.

Tolerances (those of the single-system parity test):
  Born radii            relative 2e-6
  forces                relative force RMS 1e-5 per copy
  pair energies         relative 1e-5, or 0.2 kcal/mol (4 x 0.05)
"""
import numpy as np
import pytest

from conftest import build_workspace, load_fixture, rel_rms

pytestmark = pytest.mark.gpu

J2K = (1.0 / 4184.0) * 6.0221418e23
COPIES = 4

_INDEX = ("bond_ij", "angle_iaj", "tors_idx", "impr_idx")
_PARAMS = ("bond_lk", "angle_kt", "tors_terms", "tors_par", "impr_terms", "impr_par")
_ATOM = ("charge", "radius", "epsilon", "gb_radius", "mass", "is_h")


def _copies(a, shift, n):
    """n translated copies of one system as one system."""
    N = a["charge"].shape[0]
    out = {f: np.concatenate([a[f]] * n) for f in _ATOM + _PARAMS + ("cov12_d", "cov13_d")}
    out["pos"] = np.concatenate([a["pos"] + k * shift for k in range(n)])
    out["ir"] = np.concatenate([a["ir"] + k * (int(a["ir"].max()) + 1) for k in range(n)]).astype(np.int32)
    for f in _INDEX:
        out[f] = np.concatenate([a[f] + k * N for k in range(n)]).astype(np.int32)
    bb = a["backbone_ncac"]
    out["backbone_ncac"] = np.concatenate([np.where(bb >= 0, bb + k * N, -1) for k in range(n)]).astype(np.int32)
    for c in ("cov12", "cov13", "cov14"):
        ptr, idx = a[c + "_ptr"], a[c + "_idx"]
        out[c + "_ptr"] = np.concatenate([ptr[:1]] + [ptr[1:] + k * ptr[-1] for k in range(n)]).astype(np.int32)
        out[c + "_idx"] = np.concatenate([idx + k * N for k in range(n)]).astype(np.int32)
    out["ff_params"] = a["ff_params"]
    return out


@pytest.mark.parametrize("path", [1, 0])
def test_system_above_the_tile_search_limit(path, gpu_ctx):
    a, meta = load_fixture("c2_16x80_s2")
    N = a["charge"].shape[0]
    ext = a["pos"].max(axis=0) - a["pos"].min(axis=0)
    shift = np.array([ext[0] + 2.0 * float(meta["cutoff"]) + 10.0, 0.0, 0.0])
    big = _copies(a, shift, COPIES)
    assert big["charge"].shape[0] == COPIES * N > 65536
    ws, ff = build_workspace(big, dict(meta, natoms=str(COPIES * N)), gpu_ctx)
    assert ws.setPairPath(path) == path
    ws.nlist().calcNewList()
    ff.calcForces()
    born = ws.born_radii().reshape(COPIES, N)
    f = ws.cur.f.reshape(COPIES, N, 3)
    for k in range(COPIES):
        assert np.max(np.abs(born[k] - a["born"]) / np.abs(a["born"])) <= 2e-6
        assert rel_rms(f[k], a["f_total"]) <= 1e-5
    et = a["ene_total"]
    for field, idx in (("epot_vdw", 1), ("epot_elec", 2), ("epot_pol", 3), ("epot", 0)):
        got, ref = getattr(ws.ene, field) * J2K, COPIES * et[idx] * J2K
        assert abs(got - ref) <= max(1e-5 * abs(ref), 0.2), (field, got, ref)
    ws.close()


def test_md_above_the_tile_search_limit(gpu_ctx):
    """The MD loop on the tile layout rebuilds its tiles from the list when
    the system is above the limit: 30 Langevin steps (three list periods,
    replayed from graphs) stay finite and near 300 K."""
    import pdgpu
    a, meta = load_fixture("c2_16x80_s2")
    N = a["charge"].shape[0]
    ext = a["pos"].max(axis=0) - a["pos"].min(axis=0)
    big = _copies(a, np.array([ext[0] + 42.0, 0.0, 0.0]), COPIES)
    ws, ff = build_workspace(big, dict(meta, natoms=str(COPIES * N)), gpu_ctx)
    assert ws.setPairPath(1) == 1
    md = pdgpu.MolecularDynamics(ff)
    md.Integrator = pdgpu.MolecularDynamics.Langevin
    md.FricCoeff = 1e12
    md.TargetTemp = 300.0
    md.Steps = 30
    md.UpdateNList = 10
    md.Seed = 5
    md.run()
    assert np.all(np.isfinite(md.history)) and np.all(np.isfinite(ws.cur.p))
    T = 2 * md.history[:, 1] / (3 * COPIES * N * 1.38065e-23)
    assert 150.0 < T[-10:].mean() < 450.0
    ws.nlist().calcNewList()  # a single point at the final positions
    ff.calcForces()
    assert np.isfinite(ws.ene.epot)
    ws.close()
