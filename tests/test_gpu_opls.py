"""GPU parity on OPLS-AA (param/oplsaal.ff): the 16 reference-built OPLS
peptides of the batched-MD library against the reference's own FP64 forces
and energies (tests/golden/lib16_opls_s4.npz, made by the compiled
reference), alone on both pair layouts and packed into one batch.

Tolerances (the same as the AMBER99 parity tests):
  Born radii            relative 2e-6
  forces                relative force RMS 1e-5
  pair energies         relative 1e-5 of the term, or 1e-3 kcal/mol
  bonded energies       relative 1e-9
"""
import numpy as np
import pytest

from conftest import build_workspace, load_library, rel_rms

pytestmark = pytest.mark.gpu

J2K = (1.0 / 4184.0) * 6.0221418e23
LIB = load_library("lib16_opls_s4")


def energy_close(got_J, ref_J, rel=1e-5, abs_kcal=1e-3):
    return abs(got_J - ref_J) * J2K <= max(rel * abs(ref_J) * J2K, abs_kcal)


def _check(ws, a):
    born = ws.born_radii()
    assert np.max(np.abs(born - a["born"]) / np.abs(a["born"])) <= 2e-6
    assert rel_rms(ws.cur.f, a["f_total"]) <= 1e-5
    et, e = a["ene_total"], ws.ene
    for field, idx in (("epot_vdw", 1), ("epot_elec", 2), ("epot_pol", 3), ("epot_pol_cross", 4),
                       ("epot_pol_self", 5), ("epot", 0)):
        assert energy_close(getattr(e, field), et[idx]), (field, getattr(e, field) * J2K, et[idx] * J2K)
    for field, idx in (("epot_bond", 6), ("epot_angle", 7), ("epot_torsion", 8)):
        assert getattr(e, field) == pytest.approx(et[idx], rel=1e-9), field


@pytest.mark.parametrize("path", [0, 1])
@pytest.mark.parametrize("k", range(len(LIB)))
def test_opls_member_matches_reference(k, path, gpu_ctx):
    a, m = LIB[k]
    assert m["param"] == "oplsaal.ff"
    ws, ff = build_workspace(a, m, gpu_ctx)
    assert ws.setPairPath(path) == path
    ws.nlist().calcNewList()
    ff.calcForces()
    _check(ws, a)
    ws.close()


def test_opls_batch_matches_reference(gpu_ctx):
    import pdgpu
    members = [build_workspace(a, m, gpu_ctx) + (a, m) for a, m in LIB]
    b = pdgpu.Batch([ws for ws, *_ in members])
    b.setPairPath(1)
    f, e = b.evaluate()
    for s, (ws, ff, a, m) in enumerate(members):
        assert rel_rms(b.split(f)[s], a["f_total"]) <= 1e-5
        assert energy_close(e[s][0], a["ene_total"][0])
    b.close()
    for ws, *_ in members:
        ws.close()
