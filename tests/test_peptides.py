"""The peptide splicer (pdgpu.peptides) against the reference's own builds.

Every library peptide (tests/golden/lib16_amber_s3.npz, lib16_opls_s4.npz,
built by the reference's NewProtein) is spliced again from its sequence with
the library's templates, and the result is compared with the reference's
arrays: per-atom parameters, residue indices, backbone atoms, bonds,
torsions and impropers (with their multiplicity) and the 1-2 / 1-3 / 1-4
lists exactly; angles exactly in their atoms and force constants.  The
reference takes the equilibrium angle of a few atom-type triples that its
parameter set lacks from the built geometry, so those angles (and the 1-3
distances formed from them) carry the template residue's value: fewer than
1 % of the angles may differ, by at most 0.16 rad.
"""
import collections

import numpy as np
import pytest

from conftest import load_library

from pdgpu import peptides as P

LIBS = ("lib16_amber_s3", "lib16_opls_s4")


@pytest.fixture(scope="module", params=LIBS)
def library(request):
    members = [(a, m) for a, m in load_library(request.param)]
    return members, P.ResidueLibrary(members)


def _rows(idx, *pars, canon=True):
    out = collections.Counter()
    for r in range(len(idx)):
        q = tuple(int(x) for x in idx[r])
        if canon:
            q = min(q, q[::-1])
        out[(q,) + tuple(tuple(np.atleast_1d(p[r]).tolist()) for p in pars)] += 1
    return out


def _csr_sets(a, name):
    ptr, idx = a[name + "_ptr"], a[name + "_idx"]
    return [set(idx[ptr[i]:ptr[i + 1]].tolist()) for i in range(len(ptr) - 1)]


def _csr_d(a, name):
    ptr, idx, d = a[name + "_ptr"], a[name + "_idx"], a[name + "_d"]
    return {(i, int(idx[k])): float(d[k]) for i in range(len(ptr) - 1) for k in range(ptr[i], ptr[i + 1])}


def test_spliced_library_peptides_match_the_reference_builds(library):
    members, lib = library
    angles_total = angles_off = 0
    for a, m in members:
        o = lib.build(m["chain"][0])
        for f in P._ATOM_FIELDS + ("ir", "backbone_ncac", "ff_params"):
            assert np.array_equal(o[f], a[f]), f
        assert _rows(o["bond_ij"], o["bond_lk"]) == _rows(a["bond_ij"], a["bond_lk"])
        assert _rows(o["tors_idx"], o["tors_terms"], o["tors_par"]) == _rows(a["tors_idx"], a["tors_terms"],
                                                                            a["tors_par"])
        assert _rows(o["impr_idx"], o["impr_terms"], o["impr_par"], canon=False) == \
            _rows(a["impr_idx"], a["impr_terms"], a["impr_par"], canon=False)
        for c in ("cov12", "cov13", "cov14"):
            assert _csr_sets(o, c) == _csr_sets(a, c), c
        assert _csr_d(o, "cov12") == _csr_d(a, "cov12")
        ka = {(min(i, j), c, max(i, j)): kt for (i, c, j), kt in zip(a["angle_iaj"], a["angle_kt"])}
        ko = {(min(i, j), c, max(i, j)): kt for (i, c, j), kt in zip(o["angle_iaj"], o["angle_kt"])}
        assert ka.keys() == ko.keys() and len(ka) == len(a["angle_iaj"])
        for k in ka:
            assert ka[k][0] == ko[k][0]
            angles_total += 1
            if ka[k][1] != ko[k][1]:
                angles_off += 1
                assert abs(ka[k][1] - ko[k][1]) <= 0.16
        d13a, d13o = _csr_d(a, "cov13"), _csr_d(o, "cov13")
        assert d13a.keys() == d13o.keys()
        assert max(abs(d13a[k] - d13o[k]) for k in d13a) <= 0.12
    assert angles_off <= 0.01 * angles_total


def test_new_sequences_are_complete_and_seeded(library):
    members, lib = library

    def draw(seed):
        rng = np.random.default_rng(seed)
        return [lib.draw_sequence(rng, n) for n in (20, 57, 140)]

    seqs = draw(11)
    assert seqs == draw(11) and seqs != draw(12)
    for seq in seqs:
        o = lib.build(seq)
        n = len(o["charge"])
        assert o["ir"].max() + 1 == len(seq) and o["pos"].shape == (n, 3)
        assert np.all(np.isfinite(o["pos"]))
        # one peptide bond per junction, every bond near its equilibrium length
        bl = np.linalg.norm(o["pos"][o["bond_ij"][:, 0]] - o["pos"][o["bond_ij"][:, 1]], axis=1)
        assert np.all(np.abs(bl - o["bond_lk"][:, 0]) < 0.35)
        span = np.ptp(o["ir"][o["bond_ij"]], axis=1)
        assert int((span == 1).sum()) == len(seq) - 1 and span.max() == 1
        # every atom has a bonded partner, and the net charge is whole
        assert np.all(np.diff(o["cov12_ptr"]) > 0)
        assert abs(o["charge"].sum() - round(o["charge"].sum())) < 1e-6
