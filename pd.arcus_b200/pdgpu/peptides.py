"""Seeded peptide systems spliced from residue templates.

The batched workloads ask for hundreds of distinct peptides (512 AMBER99
peptides of 20-200 residues; 256 OPLS-AA peptides of 30-150 residues).  The
reference builds a peptide with ``NewProtein`` (system/genpolymer.cpp) from
its parameter set and the residue definitions in it; this module does not
read the reference's parameter files.  It takes its residue templates from
peptides the reference itself built (the library fixtures, made by the
reference's builder and pre-minimised by its minimiser) and splices new
sequences from them:

- every residue of a library peptide is a template, keyed by its one-letter
  code and its place in the chain (N-terminal, inside, C-terminal): its
  atoms with their per-atom parameters (charge, LJ radius and well depth,
  GB radius, mass, hydrogen flag, force-field type), their coordinates and
  every bonded term inside the residue with its parameters;
- the bonded terms that cross a residue junction (the peptide bond C-N, the
  angles and torsions through it) are generated from the bond graph, and
  their parameters are looked up by the atom types of the term in the
  library, where every typed term has one parameter set (checked);
- the impropers that cross a junction belong to one residue and reach one
  atom of the neighbour, its peptide-bond atom (checked), so they are kept
  with their residue's template;
- the 1-2 / 1-3 / 1-4 lists and their equilibrium distances follow from the
  graph and, by type, from the library.

A spliced copy of a library peptide reproduces that peptide's topology and
parameters exactly (tests/test_peptides.py).  Coordinates: an ideal extended
backbone (phi = psi = omega = 180 degrees) with each residue's template
superposed on its N, CA and C atoms; the caller relaxes the clashes with the
device minimiser before use.
"""
from __future__ import annotations

import numpy as np

# ideal backbone geometry of an extended chain (Angstrom, degrees)
_N_CA, _CA_C, _C_N = 1.458, 1.525, 1.329
_ANG_N_CA_C, _ANG_CA_C_N, _ANG_C_N_CA = 111.2, 116.2, 121.7

_ATOM_FIELDS = ("charge", "radius", "epsilon", "gb_radius", "mass", "is_h", "fftype")


def _canon(types):
    t = tuple(int(x) for x in types)
    r = t[::-1]
    return t if t <= r else r


class _Template:
    """One residue: its atoms, coordinates and the bonded terms inside it."""

    def __init__(self, arrays, s, e, r, bb_global):
        self.n = e - s
        self.atoms = {f: np.asarray(arrays[f][s:e]).copy() for f in _ATOM_FIELDS}
        self.pos = np.asarray(arrays["pos"][s:e], dtype=np.float64).copy()
        self.bb = np.asarray(bb_global[r], dtype=np.int64) - s  # local N, CA, C

        def inside(idx):
            return np.all((idx >= s) & (idx < e), axis=1)

        bij = np.asarray(arrays["bond_ij"])
        m = inside(bij)
        self.bonds = (bij[m] - s, np.asarray(arrays["bond_lk"])[m])
        ang = np.asarray(arrays["angle_iaj"])
        m = inside(ang)
        self.angles = (ang[m] - s, np.asarray(arrays["angle_kt"])[m])
        tor = np.asarray(arrays["tors_idx"])
        m = inside(tor)
        self.tors = (tor[m] - s, np.asarray(arrays["tors_terms"])[m], np.asarray(arrays["tors_par"])[m])
        imp = np.asarray(arrays["impr_idx"])
        m = inside(imp)
        self.impr_inside = (imp[m] - s, np.asarray(arrays["impr_terms"])[m], np.asarray(arrays["impr_par"])[m])
        self.impr = []  # (((offset, local) x 4), terms, par): offset -1/+1 = the neighbour's link atom
        # equilibrium 1-2 and 1-3 distances inside the residue, by local pair
        self.d = {}
        for name in ("cov12", "cov13"):
            ptr, idx, dd = (np.asarray(arrays[name + "_ptr"]), np.asarray(arrays[name + "_idx"]),
                            np.asarray(arrays[name + "_d"]))
            loc = {}
            for i in range(s, e):
                for k in range(ptr[i], ptr[i + 1]):
                    j = int(idx[k])
                    if s <= j < e:
                        loc[(i - s, j - s)] = float(dd[k])
            self.d[name] = loc


class ResidueLibrary:
    """Residue templates and typed junction parameters of a set of
    reference-built peptides of one parameter set."""

    def __init__(self, members):
        """members: (arrays, meta) pairs of single-chain peptides (the library
        fixtures' layout), all built with the same parameter set."""
        self.templates = {}
        self.bond_p, self.angle_p, self.tors_p = {}, {}, {}
        self.tors_absent = set()
        self.d12, self.d13 = {}, {}
        self.ff_params = None
        for arrays, meta in members:
            self._add_member(arrays, meta)
        clash = set(self.tors_p) & self.tors_absent
        if clash:
            raise ValueError("torsions are not set by atom types alone: %d typed paths both with and without "
                             "a torsion" % len(clash))
        self.n_term = sorted(k[0] for k in self.templates if k[1] == "N")
        self.c_term = sorted(k[0] for k in self.templates if k[1] == "C")
        self.inner = sorted(k[0] for k in self.templates if k[1] == "M")

    @staticmethod
    def _put(d, key, val, what):
        val = np.asarray(val)
        old = d.get(key)
        if old is None:
            d[key] = val.copy()
        elif old.shape != val.shape or not np.array_equal(old, val):
            raise ValueError("%s %s has two parameter sets in the library" % (what, key))

    def _add_member(self, a, meta):
        chains = [meta["chain"]] if isinstance(meta["chain"], str) else list(meta["chain"])
        if len(chains) != 1:
            raise ValueError("library members must be single chains")
        chain = chains[0]
        ff = np.asarray(a["ff_params"])
        if self.ff_params is None:
            self.ff_params = ff.copy()
        elif not np.array_equal(ff, self.ff_params):
            raise ValueError("library members use different force-field settings")
        ir = np.asarray(a["ir"])
        if np.any(np.diff(ir) < 0) or ir.max() + 1 != len(chain):
            raise ValueError("residues must be contiguous and match the sequence")
        starts = np.searchsorted(ir, np.arange(len(chain) + 1))
        bb = np.asarray(a["backbone_ncac"])
        ft = np.asarray(a["fftype"])
        nres = len(chain)
        fresh = set()  # residues of this member that made a new template
        for r, code in enumerate(chain):
            var = "N" if r == 0 else ("C" if r == nres - 1 else "M")
            s, e = int(starts[r]), int(starts[r + 1])
            key = (code, var)
            t = _Template(a, s, e, r, bb)
            own = self.templates.get(key)
            if own is None:
                self.templates[key] = own = t
                fresh.add(r)
            elif own.n != t.n or any(not np.array_equal(own.atoms[f], t.atoms[f]) for f in _ATOM_FIELDS):
                raise ValueError("residue %s (%s) has two different templates" % key)
        # junction impropers: owned by the residue holding three of the atoms
        for q, terms, par in zip(np.asarray(a["impr_idx"]), np.asarray(a["impr_terms"]), np.asarray(a["impr_par"])):
            rs = ir[q]
            vals, cnt = np.unique(rs, return_counts=True)
            own_r = int(vals[np.argmax(cnt)])
            if len(vals) == 1 or own_r not in fresh:
                continue  # inside the template already, or the template came from another residue
            refs = []
            for atom in q:
                rr = int(ir[atom])
                if rr == own_r:
                    refs.append((0, int(atom - starts[own_r])))
                elif rr == own_r - 1 and atom == bb[rr][2]:
                    refs.append((-1, 0))
                elif rr == own_r + 1 and atom == bb[rr][0]:
                    refs.append((+1, 0))
                else:
                    raise ValueError("a junction improper reaches a neighbour atom other than its link atom")
            var = "N" if own_r == 0 else ("C" if own_r == nres - 1 else "M")
            tmpl = self.templates[(chain[own_r], var)]
            # every one, in order (the reference's builder can list one twice)
            tmpl.impr.append((tuple(refs), int(terms), np.asarray(par).copy()))
        # typed parameters of the terms that cross a junction (a new
        # junction's terms are looked up here; the terms inside a residue,
        # some of whose parameters depend on the built geometry, stay with
        # their template)
        def spans(q):
            return ir[q].min() != ir[q].max()

        for (i, j), lk in zip(np.asarray(a["bond_ij"]), np.asarray(a["bond_lk"])):
            if spans([i, j]):
                self._put(self.bond_p, _canon((ft[i], ft[j])), lk, "bond")
        for (i, c, j), kt in zip(np.asarray(a["angle_iaj"]), np.asarray(a["angle_kt"])):
            if spans([i, c, j]):
                self._put(self.angle_p, _canon((ft[i], ft[c], ft[j])), kt, "angle")
        tors = set()
        for q, n, par in zip(np.asarray(a["tors_idx"]), np.asarray(a["tors_terms"]), np.asarray(a["tors_par"])):
            tors.add(_canon(q))
            if spans(q):
                self._put(self.tors_p, _canon(ft[q]), np.concatenate([[n], par]), "torsion")
        adj = _adjacency(len(ir), np.asarray(a["bond_ij"]))
        for path in _paths3(adj):
            if _canon(path) not in tors and spans(list(path)):
                self.tors_absent.add(_canon(ft[list(path)]))
        for name, dk in (("cov12", self.d12), ("cov13", self.d13)):
            ptr, idx, d = (np.asarray(a[name + "_ptr"]), np.asarray(a[name + "_idx"]), np.asarray(a[name + "_d"]))
            for i in range(len(ptr) - 1):
                for k in range(ptr[i], ptr[i + 1]):
                    j = int(idx[k])
                    if ir[i] == ir[j]:
                        continue
                    key = (int(ft[i]), int(ft[j])) if name == "cov12" else self._key13(adj, ft, i, j)
                    self._put(dk, _canon(key), d[k], name + " distance")

    @staticmethod
    def _key13(adj, ft, i, j):
        mid = sorted(set(adj[i]) & set(adj[j]))
        return (int(ft[i]), int(ft[mid[0]]), int(ft[j]))

    # ------------------------------------------------------------ building
    def draw_sequence(self, rng, nres):
        """A seeded sequence: the first and last residues drawn uniformly from
        the library's terminal templates, the others from its inner ones."""
        if nres < 2:
            raise ValueError("a peptide needs at least two residues")
        seq = [self.n_term[rng.integers(len(self.n_term))]]
        seq += [self.inner[k] for k in rng.integers(len(self.inner), size=nres - 2)]
        seq.append(self.c_term[rng.integers(len(self.c_term))])
        return "".join(seq)

    def build(self, seq):
        """The arrays of a system (SystemSpec's layout) for one sequence."""
        nres = len(seq)
        tm = []
        for r, code in enumerate(seq):
            var = "N" if r == 0 else ("C" if r == nres - 1 else "M")
            if (code, var) not in self.templates:
                raise KeyError("no template for residue %s at a %s position" % (code, var))
            tm.append(self.templates[(code, var)])
        off = np.cumsum([0] + [t.n for t in tm])
        n = int(off[-1])
        out = {f: np.concatenate([t.atoms[f] for t in tm]) for f in _ATOM_FIELDS}
        out["ir"] = np.repeat(np.arange(nres, dtype=np.int32), [t.n for t in tm])
        bb = np.array([t.bb + off[r] for r, t in enumerate(tm)], dtype=np.int32)
        out["backbone_ncac"] = bb
        ft = out["fftype"]
        links = [(int(bb[r][2]), int(bb[r + 1][0])) for r in range(nres - 1)]
        # bonds
        bij = [t.bonds[0] + off[r] for r, t in enumerate(tm)]
        blk = [t.bonds[1] for t in tm]
        jb = np.array(links, dtype=np.int64).reshape(-1, 2)
        bij.append(jb)
        blk.append(np.array([self._get(self.bond_p, (ft[i], ft[j]), "bond") for i, j in links]).reshape(-1, 2))
        out["bond_ij"] = np.concatenate(bij).astype(np.int32)
        out["bond_lk"] = np.concatenate(blk).astype(np.float64)
        adj = _adjacency(n, out["bond_ij"])
        # angles and torsions: the templates' plus those through each junction
        ang = [t.angles[0] + off[r] for r, t in enumerate(tm)]
        akt = [t.angles[1] for t in tm]
        tor = [t.tors[0] + off[r] for r, t in enumerate(tm)]
        tn = [t.tors[1] for t in tm]
        tp = [t.tors[2] for t in tm]
        ja, jk, jt, jn, jp = [], [], [], [], []
        for c, nn in links:
            for x in adj[c]:
                if x != nn:
                    ja.append((x, c, nn))
            for y in adj[nn]:
                if y != c:
                    ja.append((c, nn, y))
            for path in _paths_through(adj, c, nn):
                key = _canon(ft[list(path)])
                if key in self.tors_p:
                    v = self.tors_p[key]
                    jt.append(path)
                    jn.append(int(v[0]))
                    jp.append(v[1:])
                elif key not in self.tors_absent:
                    raise KeyError("no torsion parameters for atom types %s" % (key,))
        for i, c, j in ja:
            jk.append(self._get(self.angle_p, (ft[i], ft[c], ft[j]), "angle"))
        ang.append(np.array(ja, dtype=np.int64).reshape(-1, 3))
        akt.append(np.array(jk, dtype=np.float64).reshape(-1, 2))
        tor.append(np.array(jt, dtype=np.int64).reshape(-1, 4))
        tn.append(np.array(jn, dtype=np.int32))
        tp.append(np.array(jp, dtype=np.float64).reshape(-1, 12))
        out["angle_iaj"] = np.concatenate(ang).astype(np.int32)
        out["angle_kt"] = np.concatenate(akt)
        out["tors_idx"] = np.concatenate(tor).astype(np.int32)
        out["tors_terms"] = np.concatenate(tn).astype(np.int32)
        out["tors_par"] = np.concatenate(tp)
        # impropers: the templates' own, the junction ones resolved to the link atoms
        ii, it, ip = [], [], []
        for r, t in enumerate(tm):
            for q, terms, par in t.impr:
                idx = []
                for o, loc in q:
                    if o == 0:
                        idx.append(off[r] + loc)
                    elif o == -1:
                        if r == 0:
                            break
                        idx.append(bb[r - 1][2])
                    else:
                        if r == nres - 1:
                            break
                        idx.append(bb[r + 1][0])
                else:
                    ii.append(idx)
                    it.append(terms)
                    ip.append(par)
        impr_inside = _template_impropers(tm, off)
        out["impr_idx"] = np.concatenate([impr_inside[0], np.array(ii, dtype=np.int64).reshape(-1, 4)]).astype(np.int32)
        out["impr_terms"] = np.concatenate([impr_inside[1], np.array(it, dtype=np.int32)]).astype(np.int32)
        out["impr_par"] = np.concatenate([impr_inside[2], np.array(ip, dtype=np.float64).reshape(-1, 12)])
        # 1-2, 1-3, 1-4 lists (ascending) with the equilibrium distances
        n12 = [sorted(adj[i]) for i in range(n)]
        n13 = []
        n14 = []
        for i in range(n):
            one = set(adj[i])
            two = set()
            for j in adj[i]:
                two.update(adj[j])
            two -= one | {i}
            # the far ends of three-bond paths, 1-3 partners of a ring included
            three = set()
            for j in adj[i]:
                for k in adj[j]:
                    if k == i:
                        continue
                    for q in adj[k]:
                        if q != j and q != i:
                            three.add(q)
            three -= one
            n13.append(sorted(two))
            n14.append(sorted(three))
        for name, lists in (("cov12", n12), ("cov13", n13), ("cov14", n14)):
            ptr = np.zeros(n + 1, dtype=np.int32)
            ptr[1:] = np.cumsum([len(x) for x in lists])
            out[name + "_ptr"] = ptr
            out[name + "_idx"] = np.array([j for x in lists for j in x], dtype=np.int32)
        ir = out["ir"]

        def dist(name, i, j):
            r = ir[i]
            if r == ir[j]:
                return tm[r].d[name][(i - off[r], j - off[r])]
            key = (ft[i], ft[j]) if name == "cov12" else self._key13(adj, ft, i, j)
            return float(self._get(self.d12 if name == "cov12" else self.d13, key, name + " distance"))

        out["cov12_d"] = np.array([dist("cov12", i, j) for i in range(n) for j in n12[i]], dtype=np.float64)
        out["cov13_d"] = np.array([dist("cov13", i, j) for i in range(n) for j in n13[i]], dtype=np.float64)
        out["ff_params"] = self.ff_params.copy()
        out["pos"] = self._place(tm, off, n)
        return out

    def _get(self, d, key, what):
        k = _canon(key)
        if k not in d:
            raise KeyError("no %s parameters for atom types %s" % (what, k))
        return d[k]

    @staticmethod
    def _place(tm, off, n):
        """Template coordinates superposed on an ideal extended backbone."""
        bbpos = _extended_backbone(len(tm))
        pos = np.zeros((n, 3))
        for r, t in enumerate(tm):
            src = t.pos[t.bb]
            rot, shift = _superpose(src, bbpos[r])
            pos[off[r]:off[r + 1]] = t.pos @ rot.T + shift
        return pos


def _template_impropers(tm, off):
    idx, terms, par = [], [], []
    for r, t in enumerate(tm):
        ti = t.impr_inside
        idx.append(ti[0] + off[r])
        terms.append(ti[1])
        par.append(ti[2])
    if not idx:
        return np.zeros((0, 4), np.int64), np.zeros(0, np.int32), np.zeros((0, 12))
    return np.concatenate(idx), np.concatenate(terms), np.concatenate(par)


def _adjacency(n, bonds):
    adj = [[] for _ in range(n)]
    for i, j in np.asarray(bonds):
        adj[int(i)].append(int(j))
        adj[int(j)].append(int(i))
    return adj


def _paths3(adj):
    """Every path of three bonds a-b-c-d (a != d), once per orientation pair."""
    for b in range(len(adj)):
        for c in adj[b]:
            if c <= b:
                continue
            for a in adj[b]:
                if a == c:
                    continue
                for d in adj[c]:
                    if d != b and d != a:
                        yield (a, b, c, d)


def _paths_through(adj, c, nn):
    """Paths of three bonds that hold the bond c-nn, once each."""
    seen = set()
    for a in adj[c]:  # the bond in the middle
        if a == nn:
            continue
        for d in adj[nn]:
            if d != c and d != a:
                seen.add(_canon((a, c, nn, d)))
    for x in adj[nn]:  # the bond at one end: c-nn-x-y
        if x == c:
            continue
        for y in adj[x]:
            if y != nn and y != c:
                seen.add(_canon((c, nn, x, y)))
    for x in adj[c]:  # ... or the other: y-x-c-nn
        if x == nn:
            continue
        for y in adj[x]:
            if y != c and y != nn:
                seen.add(_canon((y, x, c, nn)))
    return sorted(seen)


def _place_atom(a, b, c, bond, angle, torsion):
    """Position of d with |cd| = bond, angle bcd and torsion abcd (degrees)."""
    bc = c - b
    bc /= np.linalg.norm(bc)
    nrm = np.cross(b - a, bc)
    nrm /= np.linalg.norm(nrm)
    m = np.cross(nrm, bc)
    th, ph = np.deg2rad(angle), np.deg2rad(torsion)
    d = np.array([-bond * np.cos(th), bond * np.sin(th) * np.cos(ph), bond * np.sin(th) * np.sin(ph)])
    return c + d[0] * bc + d[1] * m + d[2] * nrm


def _extended_backbone(nres):
    """N, CA, C of every residue of an extended chain."""
    out = np.zeros((nres, 3, 3))
    n0 = np.zeros(3)
    ca0 = np.array([_N_CA, 0.0, 0.0])
    th = np.deg2rad(180.0 - _ANG_N_CA_C)
    c0 = ca0 + _CA_C * np.array([np.cos(th), np.sin(th), 0.0])
    out[0] = (n0, ca0, c0)
    if nres == 1:
        return out
    n1 = _place_atom(n0, ca0, c0, _C_N, _ANG_CA_C_N, 180.0)
    ca1 = _place_atom(ca0, c0, n1, _N_CA, _ANG_C_N_CA, 180.0)
    c1 = _place_atom(c0, n1, ca1, _CA_C, _ANG_N_CA_C, 180.0)
    out[1] = (n1, ca1, c1)
    # every residue repeats the one before it by the same rigid motion
    rot, shift = _superpose(out[0], out[1])
    for r in range(2, nres):
        out[r] = out[r - 1] @ rot.T + shift
    return out


def _superpose(src, dst):
    """Rotation and shift that best map the points src onto dst (Kabsch)."""
    cs, cd = src.mean(0), dst.mean(0)
    h = (src - cs).T @ (dst - cd)
    u, _, vt = np.linalg.svd(h)
    dd = np.sign(np.linalg.det(vt.T @ u.T))
    rot = vt.T @ np.diag([1.0, 1.0, dd]) @ u.T
    return rot, cd - cs @ rot.T


def library_members(npz):
    """(arrays, meta) of every member of a library fixture file."""
    import json
    meta = json.loads(bytes(npz["meta_json"]).decode())
    out = []
    for k, m in enumerate(meta["members"]):
        pre = "p%02d_" % k
        out.append(({f[len(pre):]: npz[f] for f in npz.files if f.startswith(pre)}, m))
    return out
