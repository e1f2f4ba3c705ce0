"""Spliced peptides (pdgpu.peptides) as device workloads: after relaxation
by the device minimiser, a batch of seeded spliced AMBER99 and OPLS-AA
peptides (2 to 90 residues) has finite energies, its neighbour lists equal
the oracle's pair sets, and its forces and Born radii agree with the
oracle's FP64 evaluation at the same coordinates (relative force RMS 1e-5,
Born radii 2e-6)."""
import numpy as np
import pytest

from conftest import build_workspace, load_library, rel_rms

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lib_name", ["lib16_amber_s3", "lib16_opls_s4"])
def test_spliced_peptides_relax_and_match_the_oracle(lib_name, gpu_ctx):
    import pdgpu
    from pdgpu import _abi as A
    from pdgpu.peptides import ResidueLibrary
    lib = load_library(lib_name)
    R = ResidueLibrary(lib)
    rng = np.random.default_rng(21)
    built = []
    for nres in (2, 22, 47, 90):  # a dipeptide: the smallest chain, one i-cluster
        arrays = R.build(R.draw_sequence(rng, nres))
        meta = dict(lib[0][1], natoms=str(len(arrays["charge"])))
        ws, ff = build_workspace(arrays, meta, gpu_ctx)
        built.append((ws, ff, arrays, meta))
    b = pdgpu.Batch([ws for ws, *_ in built])
    mp = A.min_params_default()
    mp.Algorithm = A.MIN_STEEPEST_DESCENT
    taken = b.minimise(mp, 300)
    assert np.all(taken > 0)
    pos = b.split(b.positions())
    e = b.energies()
    b.close()
    for (ws, ff, arrays, meta), p, es in zip(built, pos, e):
        assert np.all(np.isfinite(es))
        ws.cur.p[:] = p
        ws._push_positions()
        ws.nlist().calcNewList()
        ff.calcForces()
        S = O.System(arrays, cutoff=float(meta["cutoff"]), inner=float(meta["inner"]))
        ptr, data = S.nlist(p)
        gptr, gdata = ws.nlist().getData(shadow=True)
        assert np.array_equal(gptr, ptr) and np.array_equal(gdata, data)
        f_ref, e_ref, born_ref = S.calc_forces(p, ptr, data)
        assert rel_rms(ws.cur.f, f_ref) <= 1e-5
        born = ws.born_radii()
        assert np.max(np.abs(born - born_ref) / born_ref) <= 2e-6
        # relaxed: no clash left (a negative total potential energy)
        assert ws.ene.epot < 0.0
        ws.close()
