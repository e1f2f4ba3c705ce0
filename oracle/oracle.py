"""Python face of the CPU test oracle (oracle/pd_oracle.c) -- TEST ONLY.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module, and only as the checker: nothing on the product path
does.  The protocol loops here (minimisation, MD) restate the reference's
control flow in Python over the C restatement's kernels:

* ``minimise``     protocols/minimise.cpp:99-318 (runcore, SD and CG steps)
* ``md_run``       protocols/md.cpp:202-267 run_core with Langevin / VV / Beeman
* ``calc_forces``  forcefields/forcefield.cpp:220-247 (zero, then each component)
* ``lcpo``         forcefields/lcpo.cpp: FF_SASA_LCPO's forces and energies paths

Units follow the reference: Angstrom, J, N, kg.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libpd_oracle.so")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_B = ctypes.POINTER(ctypes.c_int8)


class Params(ctypes.Structure):
    """pdo_params: FF_NonBonded + FF_GeneralizedBorn_Still public settings."""

    _fields_ = [(n, ctypes.c_double) for n in (
        "cutoff", "inner_cutoff", "vdw_cutoff", "vdw_inner_cutoff", "vdw14", "elec14",
        "dielectric", "diel_solute", "diel_solvent", "still_cutoff", "exp_thresh",
        "diel_offset", "born_offset", "P1", "P2", "P3", "P4", "P5")] + [
        (n, ctypes.c_int) for n in (
            "energy_switch", "force_switch", "ddd", "do_vdw", "do_elec", "vdwcor")] + [
        (n, ctypes.c_double) for n in (
            "ddd_alpha", "vdwcor_density", "vdwcor_eps", "vdwcor_radius", "vdwcor_cutoff")]


def gb_params(cutoff=12.0, inner=None, vdw14=0.5, elec14=0.8333333333333334, P=None):
    """Settings of a FF_GeneralizedBorn_Still as constructed (gbff.cpp:17-38)
    plus FF_NonBonded defaults (nonbonded.cpp:968-1004), with the cutoffs set
    the way the synthetic workloads set them (inner = cutoff - 3)."""
    if inner is None:
        inner = cutoff - 3.0
    P = P if P is not None else (0.073, 0.921, 6.211, 15.236, 1.254)
    p = Params()
    p.cutoff, p.inner_cutoff = cutoff, inner
    p.vdw_cutoff, p.vdw_inner_cutoff = cutoff, inner
    p.vdw14, p.elec14 = vdw14, elec14
    p.dielectric, p.diel_solute, p.diel_solvent = 1.0, 1.0, 80.0
    p.still_cutoff, p.exp_thresh, p.diel_offset, p.born_offset = 10.0, -4.0, -0.090, 0.0
    p.P1, p.P2, p.P3, p.P4, p.P5 = P
    p.energy_switch, p.force_switch, p.ddd, p.do_vdw, p.do_elec, p.vdwcor = 1, 0, 0, 1, 1, 0
    p.ddd_alpha = 1.0
    return p


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])
        L = ctypes.CDLL(LIB_PATH)
        L.pdo_constants.argtypes = [_D]
        L.pdo_bondorder.argtypes = [ctypes.c_int, _I, _I, _I, _I, _I, _I, _I, _B,
                                    ctypes.c_long, _I, ctypes.c_int, _I]
        L.pdo_bondorder.restype = ctypes.c_int
        L.pdo_nlist.argtypes = [ctypes.c_int, _D, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                ctypes.c_int, _B, ctypes.c_int, _I, _I, _I, ctypes.c_long]
        L.pdo_nlist.restype = ctypes.c_long
        L.pdo_gb_fixed_terms.argtypes = [ctypes.c_int, _D, _I, _I, _D, _I, _I, _D,
                                         ctypes.POINTER(Params), _D, _D]
        L.pdo_born_radii.argtypes = [ctypes.c_int, _D, _I, _I, _D, _D, _D,
                                     ctypes.POINTER(Params), _D]
        L.pdo_gb_forces.argtypes = [ctypes.c_int, _D, _I, _I, _D, _D, _D, _D, _D, _D,
                                    ctypes.POINTER(Params), _D, _D, _D, _D]
        L.pdo_born_energy.argtypes = [ctypes.c_int, _D, _I, _I, _D, _D,
                                      ctypes.POINTER(Params), _D]
        L.pdo_born_energy.restype = ctypes.c_double
        L.pdo_nonbonded.argtypes = [ctypes.c_int, _D, _I, _I, _D, _D, _D,
                                    ctypes.POINTER(Params), _D, _D]
        L.pdo_bonded.argtypes = [ctypes.c_int, _D, ctypes.c_int, _I, _D, ctypes.c_int, _I, _D,
                                 ctypes.c_int, _I, _I, _D, ctypes.c_int, _I, _I, _D, _D, _D]
        L.pdo_langevin_step.argtypes = [ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_double,
                                        ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int]
        L.pdo_langevin_step.restype = ctypes.c_double
        L.pdo_velocity_verlet_step.argtypes = [ctypes.c_int, _D, _D, _D, _D, ctypes.c_double]
        L.pdo_velocity_verlet_step.restype = ctypes.c_double
        L.pdo_beeman_step.argtypes = [ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_int]
        L.pdo_beeman_step.restype = ctypes.c_double
        L.pdo_lcpo.argtypes = [ctypes.c_int, _D, _I, _I, _D, _D, _D, _B, ctypes.c_int, _D, _D,
                               ctypes.POINTER(ctypes.c_long)]
        L.pdo_lcpo.restype = ctypes.c_double
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_D)


def _i(a):
    return a.ctypes.data_as(_I)


def _b(a):
    return a.ctypes.data_as(_B)


def _cd(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ci(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def constants():
    out = np.zeros(8)
    lib().pdo_constants(_d(out))
    keys = ("kcal2J", "J2kcal", "Na", "kB", "Angstrom", "econv", "econv_joule", "halfeconv")
    return dict(zip(keys, out))


KCAL_PER_J = None


def j2kcal():
    c = constants()
    return c["J2kcal"] * c["Na"]


class System:
    """A system as the fixtures store it (arrays named as the reference
    driver dumps them) plus the oracle's derived per-system data."""

    def __init__(self, arrays, cutoff=12.0, inner=None, padding=0.5):
        a = {k: np.asarray(v) for k, v in arrays.items()}
        self.a = a
        self.n = int(a["charge"].shape[0])
        self.q = _cd(a["charge"])
        self.radius = _cd(a["radius"])
        self.eps = _cd(a["epsilon"])
        self.mass = _cd(a["mass"])
        self.gbr = _cd(a["gb_radius"])
        self.ir = _ci(a["ir"])
        self.c12p, self.c12i, self.c12d = _ci(a["cov12_ptr"]), _ci(a["cov12_idx"]), _cd(a["cov12_d"])
        self.c13p, self.c13i, self.c13d = _ci(a["cov13_ptr"]), _ci(a["cov13_idx"]), _cd(a["cov13_d"])
        self.c14p, self.c14i = _ci(a["cov14_ptr"]), _ci(a["cov14_idx"])
        self.params = gb_params(cutoff, inner)
        if "ff_params" in a:
            fp = a["ff_params"]
            self.params.P1, self.params.P2, self.params.P3, self.params.P4, self.params.P5 = fp[:5]
            self.params.vdw14, self.params.elec14 = fp[5], fp[6]
        self.padding = padding
        self.bondorder()
        self.fixed_terms()
        self.bonded = dict(
            bij=_ci(a["bond_ij"]).reshape(-1), blk=_cd(a["bond_lk"]).reshape(-1),
            aiaj=_ci(a["angle_iaj"]).reshape(-1), akt=_cd(a["angle_kt"]).reshape(-1),
            tidx=_ci(a["tors_idx"]).reshape(-1), tterms=_ci(a["tors_terms"]),
            tpar=_cd(a["tors_par"]).reshape(-1),
            iidx=_ci(a["impr_idx"]).reshape(-1), iterms=_ci(a["impr_terms"]),
            ipar=_cd(a["impr_par"]).reshape(-1))

    # -- setup-time pieces
    def bondorder(self):
        n = self.n
        cap = 64 * max(n, 1)
        band = np.zeros(cap, dtype=np.int8)
        off = np.zeros(3 * 4096, dtype=np.int32)
        noff = ctypes.c_int(0)
        mid = lib().pdo_bondorder(n, _i(self.ir), _i(self.c12p), _i(self.c12i), _i(self.c13p),
                                  _i(self.c13i), _i(self.c14p), _i(self.c14i), _b(band), cap,
                                  _i(off), 4096, ctypes.byref(noff))
        if mid < 0:
            raise RuntimeError("bond-order band too wide for the oracle buffer")
        self.mid = mid
        self.band = band[: mid * (n - 1)].copy()
        self.off = off[: 3 * noff.value].copy()
        self.n_off = noff.value

    def fixed_terms(self):
        self.vj = np.zeros(self.n)
        self.terms123 = np.zeros(self.n)
        lib().pdo_gb_fixed_terms(self.n, _d(self.gbr), _i(self.c12p), _i(self.c12i), _d(self.c12d),
                                 _i(self.c13p), _i(self.c13i), _d(self.c13d),
                                 ctypes.byref(self.params), _d(self.vj), _d(self.terms123))

    # -- per-step pieces
    def nlist(self, pos, shadow=True, cutoff=None):
        pos = _cd(pos).reshape(-1)
        c = self.params.cutoff if cutoff is None else cutoff
        c = max(c, self.params.vdw_cutoff)
        cap = 1 << 16
        while True:
            ptr = np.zeros(self.n + 1, dtype=np.int32)
            data = np.zeros(cap, dtype=np.int32)
            cnt = lib().pdo_nlist(self.n, _d(pos), c, self.padding, int(shadow), self.mid,
                                  _b(self.band), self.n_off, _i(self.off) if self.n_off else None,
                                  _i(ptr), _i(data), cap)
            if cnt >= 0:
                return ptr, data[:cnt].copy()
            cap *= 4

    def born_radii(self, pos, ptr, data):
        born = np.zeros(self.n)
        lib().pdo_born_radii(self.n, _d(_cd(pos).reshape(-1)), _i(ptr), _i(data), _d(self.gbr),
                             _d(self.vj), _d(self.terms123), ctypes.byref(self.params), _d(born))
        return born

    def gb_forces(self, pos, ptr, data, born=None):
        """GB component calcForces (FastMode): radii then fused pass."""
        pos = _cd(pos).reshape(-1)
        if born is None:
            born = self.born_radii(pos, ptr, data)
        f = np.zeros(3 * self.n)
        ene = np.zeros(6)
        aep = np.zeros(self.n)
        deda = np.zeros(self.n)
        lib().pdo_gb_forces(self.n, _d(pos), _i(ptr), _i(data), _d(self.q), _d(self.radius),
                            _d(self.eps), _d(self.gbr), _d(self.vj), _d(born),
                            ctypes.byref(self.params), _d(f), _d(ene), _d(aep), _d(deda))
        return f.reshape(-1, 3), ene, born, deda, aep

    def born_energy(self, pos, ptr, data, born):
        pol = np.zeros(3)
        e = lib().pdo_born_energy(self.n, _d(_cd(pos).reshape(-1)), _i(ptr), _i(data), _d(self.q),
                                  _d(born), ctypes.byref(self.params), _d(pol))
        return e, pol

    def nonbonded(self, pos, ptr, data, params=None):
        f = np.zeros(3 * self.n)
        ene = np.zeros(4)
        p = self.params if params is None else params
        lib().pdo_nonbonded(self.n, _d(_cd(pos).reshape(-1)), _i(ptr), _i(data), _d(self.q),
                            _d(self.radius), _d(self.eps), ctypes.byref(p), _d(f), _d(ene))
        return f.reshape(-1, 3), ene

    def bonded_forces(self, pos):
        b = self.bonded
        f = np.zeros(3 * self.n)
        ene = np.zeros(5)
        lib().pdo_bonded(self.n, _d(_cd(pos).reshape(-1)),
                         len(b["blk"]) // 2, _i(b["bij"]), _d(b["blk"]),
                         len(b["akt"]) // 2, _i(b["aiaj"]), _d(b["akt"]),
                         len(b["tterms"]), _i(b["tidx"]), _i(b["tterms"]), _d(b["tpar"]),
                         len(b["iterms"]), _i(b["iidx"]), _i(b["iterms"]), _d(b["ipar"]),
                         _d(f), _d(ene))
        return f.reshape(-1, 3), ene

    def energies_path(self, pos, ptr, data):
        """GB component calcEnergies (gbff.cpp:161-166): radii, then the
        stand-alone LJ/Coulomb kernel at the solute dielectric (forces are
        applied as a side effect, as in the reference), then the Born energy."""
        born = self.born_radii(pos, ptr, data)
        p = gb_params()
        ctypes.pointer(p)[0] = self.params
        p.dielectric = p.diel_solute
        f, ene = self.nonbonded(pos, ptr, data, p)
        epol, pol = self.born_energy(pos, ptr, data, born)
        return f, ene, epol, pol, born

    def calc_forces(self, pos, ptr, data, with_bonded=True):
        """Forcefield::calcForces with {FF_Bonded, FF_GeneralizedBorn_Still}.
        Returns forces (N) and the energy record (J)."""
        f = np.zeros((self.n, 3))
        e = dict.fromkeys(("epot", "vdw", "elec", "pol", "pol_cross", "pol_self", "bond",
                           "angle", "torsion", "virial"), 0.0)
        if with_bonded:
            fb, eb = self.bonded_forces(pos)
            f += fb
            e["bond"], e["angle"], e["torsion"], e["virial"] = eb[0], eb[1], eb[2], eb[3]
            e["epot"] += eb[4]
        fg, eg, born, deda, aep = self.gb_forces(pos, ptr, data)
        f += fg
        e["epot"] += eg[0]
        e["vdw"], e["elec"], e["pol"], e["pol_cross"], e["pol_self"] = eg[1:6]
        return f, e, born


def lcpo(pos, ptr, data, radius, p, sigma, use, energy_only=False):
    """FF_SASA_LCPO over the neighbour list (ptr, data as the reference
    packs it): (per-atom SASA in A^2, SASAderiv [n, 3] in sigma units per A
    (None on the energies path), epot_cav in sigma units, partners that did
    not fit in the 80-entry overlap lists)."""
    n = len(radius)
    sasa = np.zeros(n)
    deriv = None if energy_only else np.zeros((n, 3))
    lost = ctypes.c_long(0)
    sig = np.broadcast_to(np.asarray(sigma, dtype=np.float64), (n,))
    e = lib().pdo_lcpo(n, _d(_cd(pos)), _i(_ci(ptr)), _i(_ci(data)), _d(_cd(radius)), _d(_cd(p)),
                       _d(_cd(sig)), _b(np.ascontiguousarray(use, dtype=np.int8)), int(bool(energy_only)),
                       _d(sasa), None if deriv is None else _d(deriv), ctypes.byref(lost))
    return sasa, deriv, e, lost.value


def lcpo_sigma_J(asp_kcal):
    """The solvation parameter FF_SASA_LCPO::setup forms from GlobalASP
    (kcal/mol/A^2 -> J/A^2 per molecule, lcpo.cpp:44-47)."""
    c = constants()
    return asp_kcal / c["Na"] / c["J2kcal"]


def langevin_step(x, v, f, mass, normals, dt, gamma, temp, step, steps):
    x, v = _cd(x).copy(), _cd(v).copy()
    ek = lib().pdo_langevin_step(len(mass), _d(x), _d(v), _d(_cd(f)), _d(_cd(mass)),
                                 _d(_cd(normals)), dt, gamma, temp, step, steps)
    return x, v, ek


def velocity_verlet_step(x, v, f, mass, dt):
    x, v = _cd(x).copy(), _cd(v).copy()
    ek = lib().pdo_velocity_verlet_step(len(mass), _d(x), _d(v), _d(_cd(f)), _d(_cd(mass)), dt)
    return x, v, ek


def beeman_step(x, v, f, fold, mass, dt, step, steps):
    x, v, fold = _cd(x).copy(), _cd(v).copy(), _cd(fold).copy()
    ek = lib().pdo_beeman_step(len(mass), _d(x), _d(v), _d(_cd(f)), _d(fold), _d(_cd(mass)),
                               dt, step, steps)
    return x, v, fold, ek


def minimise(sysm, pos, steps, algorithm="sd", step_size=2e5, update_nlist=1,
             slope_cutoff=-1.0, strictness=0.0):
    """Minimisation::runcore (minimise.cpp:99-179) with doSteepestDescentStep
    (:181-235) / doConjugateGradientStep (:237-318), UpdateNList = 1."""
    c = constants()
    x = _cd(pos).reshape(-1, 3).copy()
    n = sysm.n
    mult = 1.0
    ptr, data = sysm.nlist(x)  # setup-time list (a full list; see module docs)
    f, e, _ = sysm.calc_forces(x, ptr, data)
    old_energy = e["epot"]
    best_x = x.copy()  # WorkSpace::old = cur
    op = x.copy()
    of = f.copy()
    ov = np.zeros_like(x)
    vdir = np.zeros_like(x)
    nl_counter = 0
    taken = 0
    for step in range(steps):
        if update_nlist > 0 and nl_counter % update_nlist == 0:
            ptr, data = sysm.nlist(x)
        nl_counter += 1
        f, e, _ = sysm.calc_forces(x, ptr, data)
        epot = e["epot"]
        if not np.isfinite(epot):
            return -1, x, e
        if algorithm == "sd":
            if step != 0:
                if epot <= old_energy:
                    mult *= 1.2
                    op = x.copy()
                    of = f.copy()
                    old_energy = epot
                else:
                    mult *= 0.5 / 1.2
                    x = op.copy()
                    f = of.copy()
                    old_energy += 1
                    taken = step + 1
                    best_x = op  # the "old" snapshot is the saved position
                    continue
            else:
                op = x.copy()
                of = f.copy()
                old_energy = epot
            x = x + f * (step_size * mult)
        else:
            if step != 0:
                if (mult < 0.05 and (epot - old_energy) < strictness * c["kcal2J"] / c["Na"]) or \
                        epot < old_energy:
                    mult *= 1.2
                    fmagold = float(np.sum(of * of))
                    fmagnew = float(np.sum((of - f) * f))
                    gamma = fmagnew / fmagold if fmagold != 0 else 0.0
                    if gamma < 0:
                        gamma = 0.0
                    vdir = ov * gamma + f
                    op = x.copy()
                    of = f.copy()
                    ov = vdir.copy()
                    old_energy = epot
                else:
                    mult *= 0.5 / 1.2
                    x = op.copy()
            else:
                op = x.copy()
                of = f.copy()
                ov = f.copy()
                vdir = f.copy()
                old_energy = epot
            x = x + vdir * (step_size * mult)
        taken = step + 1
        best_x = op
    x = best_x.copy()
    ptr2, data2 = ptr, data
    f, e, _ = sysm.calc_forces(x, ptr2, data2)
    return taken, x, e, mult


def load_system_dir(path):
    """Load a reference-driver dump directory (``*.npy`` + ``meta.txt``)."""
    arrays = {}
    for fn in os.listdir(path):
        if fn.endswith(".npy"):
            arrays[fn[:-4]] = np.load(os.path.join(path, fn))
    meta = {}
    chains = []
    with open(os.path.join(path, "meta.txt")) as fh:
        for line in fh:
            k, v = line.split(None, 1)
            if k == "chain":
                chains.append(v.strip())
            else:
                meta[k] = v.strip()
    meta["chains"] = chains
    return arrays, meta


# ------------------------------------------------------------------ trial moves
def backbone_axes(backbone_ncac):
    """Rotation bonds of every residue's phi then psi, residues in order, as
    MoleculeBase::setResiduePhiPsi applies them (system/molecule.cpp:702-711):
    (N, CA) then (CA, C).  Returns an (R, 2) int array."""
    bb = np.asarray(backbone_ncac).reshape(-1, 3)
    ax = []
    for n, ca, c in bb:
        ax.append((n, ca))
        ax.append((ca, c))
    return np.asarray(ax, dtype=np.int32)


def moved_atoms(cov12_ptr, cov12_idx, bi, bj):
    """Atoms MoleculeBase::rotateBond(bi, bj) moves (molecule.cpp:1099-1175):
    the covalent graph walked from bj without stepping onto bi."""
    seen = {bi, bj}
    queue = [bj]
    for a in queue:
        for nb in cov12_idx[cov12_ptr[a]:cov12_ptr[a + 1]]:
            nb = int(nb)
            if nb not in seen:
                seen.add(nb)
                queue.append(nb)
    return np.asarray(queue, dtype=np.int64)


def axis_rotation(axis, angle):
    """matrix3x3::setToAxisRot (maths/maths_matrix3x3.cpp:161-185): the
    right-handed rotation by `angle` about `axis`, applied to column vectors."""
    u = np.asarray(axis, dtype=np.float64) / np.linalg.norm(axis)
    c, s, t = np.cos(angle), np.sin(angle), 1.0 - np.cos(angle)
    x, y, z = u
    return np.array([[t * x * x + c, t * x * y - s * z, t * x * z + s * y],
                     [t * x * y + s * z, t * y * y + c, t * y * z - s * x],
                     [t * x * z - s * y, t * y * z + s * x, t * z * z + c]])


def apply_torsions(pos, cov12_ptr, cov12_idx, axes, angles):
    """Rotate the bonds one by one in list order, each about its current
    axis (rotateBond: translate to bi, rotate, translate back)."""
    x = np.array(pos, dtype=np.float64).reshape(-1, 3)
    for (bi, bj), th in zip(axes, angles):
        m = moved_atoms(cov12_ptr, cov12_idx, int(bi), int(bj))
        R = axis_rotation(x[bj] - x[bi], th)
        x[m] = (x[m] - x[bi]) @ R.T + x[bi]
    return x
