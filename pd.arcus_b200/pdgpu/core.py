"""Host-side mirror of the reference's Python surface for the GB/SA path.

The reference exposes its C++ classes to Python under their own names
through SWIG (src/pd/pd.i:44-166).  The classes here keep those names and
public attributes for the hot path -- WorkSpace, NeighbourList, Forcefield,
FF_Bonded, FF_NonBonded, FF_GeneralizedBorn_Still, Energy, Minimisation,
MolecularDynamics -- and run every evaluation through libpdgpu on the GPU.
System construction (FFParamSet, NewProtein) is not part of this path: a
WorkSpace is built from a ``SystemSpec``, the per-atom parameters and
topology the reference's WorkSpace holds after setup.

Units are the reference's: Angstrom, J, N, kg, s.
"""
from __future__ import annotations

import ctypes
import json

import numpy as np

from . import _abi as A

J2KCAL_NA = (1.0 / 4184.0) * 6.0221418e23  # J/molecule -> kcal/mol (forcefield.cpp:18-20)


# ------------------------------------------------------------------ context
class Context:
    """One device context (CUDA stream + resident systems)."""

    _default = None

    def __init__(self, device=0):
        self.ptr = A._CTX()
        A.check(A.lib().pdgpu_ctx_create(device, ctypes.byref(self.ptr)))

    @classmethod
    def default(cls):
        if cls._default is None:
            cls._default = Context(0)
        return cls._default

    def mem_used(self):
        b = ctypes.c_int64(0)
        A.check(A.lib().pdgpu_ctx_mem_used(self.ptr, ctypes.byref(b)))
        return b.value

    def last_run_ms(self):
        ms = ctypes.c_double(0)
        A.check(A.lib().pdgpu_last_run_ms(self.ptr, ctypes.byref(ms)))
        return ms.value

    def close(self):
        if self.ptr:
            A.lib().pdgpu_ctx_destroy(self.ptr)
            self.ptr = A._CTX()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ system
class SystemSpec:
    """Per-atom parameters, topology and coordinates of one WorkSpace, named
    as the reference's Particle / FF_Bonded fields (fundamentals.h:150-180,
    ffbonded.h).  ``from_arrays`` reads the layout the fixture generator
    writes (tests/golden/make_golden.py)."""

    def __init__(self, arrays, meta=None):
        a = {k: np.asarray(v) for k, v in arrays.items()}
        self.arrays = a
        self.meta = meta or {}
        self.natoms = int(a["charge"].shape[0])

    @classmethod
    def from_npz(cls, path):
        z = np.load(path)
        arrays = {k: z[k] for k in z.files}
        meta = json.loads(bytes(arrays.pop("meta_json")).decode()) if "meta_json" in arrays else {}
        return cls(arrays, meta)

    def __getitem__(self, k):
        return self.arrays[k]

    def __contains__(self, k):
        return k in self.arrays


class Hamiltonian:
    """The energy record (workspace/hamiltonian.h:23-49), J."""

    FIELDS = {"epot": A.ENE_EPOT, "epot_vdw": A.ENE_VDW, "epot_elec": A.ENE_ELEC, "epot_pol": A.ENE_POL,
              "epot_pol_cross": A.ENE_POL_CROSS, "epot_pol_self": A.ENE_POL_SELF,
              "epot_bond": A.ENE_BOND, "epot_angle": A.ENE_ANGLE, "epot_torsion": A.ENE_TORSION,
              "InternalVirial": A.ENE_VIRIAL, "ekin": A.ENE_EKIN, "etot": A.ENE_ETOT,
              "epot_surf": A.ENE_SURF}

    def __init__(self):
        self.zero()

    def zero(self):
        for k in self.FIELDS:
            setattr(self, k, 0.0)

    def load(self, vec):
        for k, i in self.FIELDS.items():
            setattr(self, k, float(vec[i]))

    def kcal(self, field):
        return getattr(self, field) * J2KCAL_NA


class SnapShot:
    """cur / old atom state (snapshot.h:16-22): p (A), f (N), v (m/s)."""

    def __init__(self, n):
        self.p = np.zeros((n, 3))
        self.f = np.zeros((n, 3))
        self.v = np.zeros((n, 3))


class WorkSpace:
    """A system resident on the device plus its host-side state mirror."""

    def __init__(self, spec: SystemSpec, ctx: Context | None = None):
        self.spec = spec
        self.ctx = ctx or Context.default()
        n = spec.natoms
        self.cur = SnapShot(n)
        self.old = SnapShot(n)
        if "pos" in spec:
            self.cur.p[:] = spec["pos"]
        self.ene = Hamiltonian()
        self.Step = 0
        self._sys = None
        self._params_key = None
        self._nlist = NeighbourList(self)
        self._pos_dirty = True
        self._ff = None  # the Forcefield whose components set this workspace up
        self._lcpo_set = False  # the device system has the LCPO term

    def nAtoms(self):
        return self.spec.natoms

    def nlist(self):
        return self._nlist

    # -- device plumbing
    def _ensure_device(self, params: A.FFParams, with_bonded: bool):
        key = (bytes(params), with_bonded)
        L, s = A.lib(), self.spec
        if self._sys is None:
            sid = ctypes.c_int32(0)
            A.check(L.pdgpu_system_create(
                self.ctx.ptr, s.natoms, A.dptr(A.cd(s["charge"])), A.dptr(A.cd(s["radius"])),
                A.dptr(A.cd(s["epsilon"])), A.dptr(A.cd(s["mass"])), A.dptr(A.cd(s["gb_radius"])),
                A.iptr(A.ci(s["ir"])), A.iptr(A.ci(s["cov12_ptr"])), A.iptr(A.ci(s["cov12_idx"])),
                A.dptr(A.cd(s["cov12_d"])), A.iptr(A.ci(s["cov13_ptr"])), A.iptr(A.ci(s["cov13_idx"])),
                A.dptr(A.cd(s["cov13_d"])), A.iptr(A.ci(s["cov14_ptr"])), A.iptr(A.ci(s["cov14_idx"])),
                ctypes.byref(params), ctypes.byref(sid)))
            self._sys = sid.value
            if with_bonded:
                self._set_bonded()
            if "is_h" in s:
                h = np.ascontiguousarray(s["is_h"], dtype=np.int8)
                A.check(L.pdgpu_system_set_hydrogens(self.ctx.ptr, self._sys, h.ctypes.data_as(A._I8)))
            self._params_key = key
            self._pos_dirty = True
        elif key != self._params_key:
            A.check(L.pdgpu_system_set_params(self.ctx.ptr, self._sys, ctypes.byref(params)))
            if with_bonded and not self._params_key[1]:
                self._set_bonded()
            self._params_key = key
            self._pos_dirty = True

    def _set_bonded(self):
        s = self.spec
        b = lambda k: A.ci(s[k]).reshape(-1)
        d = lambda k: A.cd(s[k]).reshape(-1)
        A.check(A.lib().pdgpu_system_set_bonded(
            self.ctx.ptr, self._sys, len(s["bond_lk"]), A.iptr(b("bond_ij")), A.dptr(d("bond_lk")),
            len(s["angle_kt"]), A.iptr(b("angle_iaj")), A.dptr(d("angle_kt")),
            len(s["tors_terms"]), A.iptr(b("tors_idx")), A.iptr(b("tors_terms")), A.dptr(d("tors_par")),
            len(s["impr_terms"]), A.iptr(b("impr_idx")), A.iptr(b("impr_terms")), A.dptr(d("impr_par"))))

    def _push_positions(self):
        A.check(A.lib().pdgpu_set_positions(self.ctx.ptr, self._sys, A.dptr(A.cd(self.cur.p))))
        self._pos_dirty = False

    def _pull_positions(self):
        p = np.zeros((self.nAtoms(), 3))
        A.check(A.lib().pdgpu_get_positions(self.ctx.ptr, self._sys, A.dptr(p)))
        self.cur.p[:] = p

    def _push_velocities(self):
        A.check(A.lib().pdgpu_set_velocities(self.ctx.ptr, self._sys, A.dptr(A.cd(self.cur.v))))

    def _pull_velocities(self):
        v = np.zeros((self.nAtoms(), 3))
        A.check(A.lib().pdgpu_get_velocities(self.ctx.ptr, self._sys, A.dptr(v)))
        self.cur.v[:] = v

    def _pull_forces(self):
        f = np.zeros((self.nAtoms(), 3))
        A.check(A.lib().pdgpu_get_forces(self.ctx.ptr, self._sys, A.dptr(f)))
        return f

    def _pull_energies(self):
        e = np.zeros(A.ENE_COUNT)
        A.check(A.lib().pdgpu_get_energies(self.ctx.ptr, self._sys, A.dptr(e), A.ENE_COUNT))
        return e

    def _pull_step(self):
        """WorkSpace::Step as the last protocol left it."""
        st = ctypes.c_int32(0)
        A.check(A.lib().pdgpu_get_step(self.ctx.ptr, self._sys, ctypes.byref(st)))
        self.Step = st.value

    def born_radii(self):
        b = np.zeros(self.nAtoms())
        A.check(A.lib().pdgpu_get_born_radii(self.ctx.ptr, self._sys, A.dptr(b)))
        return b

    def zeroForces(self):
        self.cur.f[:] = 0
        self.ene.zero()

    # -- backbone phi/psi trial moves (MoleculeBase::setResiduePhiPsi,
    #    system/molecule.cpp:702-711, applied as increments)
    def _device(self):
        if self._sys is None and self._ff is not None:
            self._ff.ensuresetup()
        if self._sys is None:
            raise A.PdgpuError(A.ERR_STATE, "add a forcefield component to this workspace first")
        if self._pos_dirty:
            self._push_positions()
        return self._sys

    def setLanes(self, lpa=None):
        """Fix the lanes per atom of the Born, fused and chain kernels
        (None: autotune at the next evaluation)."""
        arr = None if lpa is None else A.iptr(np.ascontiguousarray(lpa, dtype=np.int32))
        A.check(A.lib().pdgpu_set_lanes(self.ctx.ptr, self._device(), arr))

    def setPairPath(self, path):
        """Pair-pass layout: 0 neighbour-list rows, 1 cluster-pair tiles,
        -1 autotune, -2 report only; returns the layout in use."""
        cur = ctypes.c_int32(0)
        A.check(A.lib().pdgpu_pair_path(self.ctx.ptr, self._device(), int(path), ctypes.byref(cur)))
        return cur.value

    def setEvalMode(self, mode):
        """Launch form of an evaluation on the tile layout: 1 one
        cooperative launch, 0 three launches, 2 (the default) cooperative
        except inside MD step blocks, -1 report only; returns the form in
        use."""
        cur = ctypes.c_int32(0)
        A.check(A.lib().pdgpu_eval_mode(self.ctx.ptr, self._device(), int(mode), ctypes.byref(cur)))
        return cur.value

    def backboneAxes(self):
        """(N, CA) then (CA, C) of every residue in order: the bonds
        setResiduePhiPsi turns for phi and psi."""
        bb = np.asarray(self.spec["backbone_ncac"]).reshape(-1, 3)
        ax = []
        for n, ca, c in bb:
            if n >= 0 and ca >= 0:
                ax.append((n, ca))
            if ca >= 0 and c >= 0:
                ax.append((ca, c))
        return np.asarray(ax, dtype=np.int32).reshape(-1, 2)

    def setTorsionMoves(self, axes=None):
        """Register the rotatable bonds of trial moves (default: every
        residue's phi and psi); returns the rotation count."""
        sid = self._device()
        ax = self.backboneAxes() if axes is None else np.asarray(axes, dtype=np.int32).reshape(-1, 2)
        ax = np.ascontiguousarray(ax, dtype=np.int32)
        A.check(A.lib().pdgpu_system_set_torsions(self.ctx.ptr, sid, len(ax), A.iptr(ax)))
        self.nRotations = len(ax)
        return len(ax)

    def saveBasePositions(self):
        A.check(A.lib().pdgpu_save_base_positions(self.ctx.ptr, self._device()))

    def perturbTorsions(self, sigma=0.0, trial=0, angles=None):
        """Positions = base with rotation k turned by angles[k] (rad), or by
        sigma * N(0,1) from the counter-based RNG (key: Seed, counter: trial)."""
        sid = self._device()
        ang = None if angles is None else A.dptr(A.cd(angles))
        A.check(A.lib().pdgpu_perturb_torsions(self.ctx.ptr, sid, float(sigma), int(trial), ang))
        self._pull_positions()

    def close(self):
        if self._sys is not None and self.ctx.ptr:
            A.lib().pdgpu_system_destroy(self.ctx.ptr, self._sys)
        self._sys = None


class NeighbourList:
    """NeighbourList (workspace/neighbourlist.h:37-180) on the device: a
    cell-list rebuild with the reference's exact pair set and packed
    (index | bondorder<<24) entries.  The device list is always the full
    ('shadow') list; getData() returns the half list unless calcShadow(True)."""

    def __init__(self, ws: WorkSpace):
        self.ws = ws
        self.CalcShadow = False
        self.Cutoff = 0.0
        self.Padding = 0.5
        self._count = 0

    def calcShadow(self, enabled):
        self.CalcShadow = bool(enabled)

    def requestCutoff(self, c):
        if c > self.Cutoff:
            self.Cutoff = float(c)

    def getFullUpdateCount(self):
        return self._count

    def calcNewList(self):
        ws = self.ws
        if ws._sys is None and ws._ff is not None:
            ws._ff.ensuresetup()
        if ws._sys is None:
            raise A.PdgpuError(A.ERR_STATE, "add a forcefield component to this workspace first")
        if ws._pos_dirty:
            ws._push_positions()
        A.check(A.lib().pdgpu_nlist_build(ws.ctx.ptr, ws._sys))
        self._count += 1

    def getData(self, shadow=None):
        """(ptr[n+1], data) with the reference's packed entries."""
        ws = self.ws
        sh = self.CalcShadow if shadow is None else shadow
        n = ws.nAtoms()
        ptr = np.zeros(n + 1, dtype=np.int32)
        cnt = ctypes.c_int64(0)
        A.check(A.lib().pdgpu_nlist_export(ws.ctx.ptr, ws._sys, int(sh), A.iptr(ptr), None, 0,
                                           ctypes.byref(cnt)))
        data = np.zeros(max(cnt.value, 1), dtype=np.int32)
        A.check(A.lib().pdgpu_nlist_export(ws.ctx.ptr, ws._sys, int(sh), A.iptr(ptr), A.iptr(data),
                                           cnt.value, ctypes.byref(cnt)))
        return ptr, data[: cnt.value]


# ------------------------------------------------------------------ forcefields
class ForcefieldBase:
    name = "Forcefield component"

    def __init__(self, wspace: WorkSpace):
        self.wspace = wspace
        self.Active = True

    def getWSpace(self):
        return self.wspace


class FF_Bonded(ForcefieldBase):
    """Bonds, angles, torsions, impropers (forcefields/ffbonded.*); the
    term lists are the ones FF_Bonded::setup assembles (SystemSpec)."""

    name = "Bonded Forcefield"

    def __init__(self, wspace):
        super().__init__(wspace)
        self.DoBonds = self.DoAngles = self.DoTorsions = self.DoImpropers = True


class FF_NonBonded(ForcefieldBase):
    """LJ 12-6 + Coulomb with cutoffs (forcefields/nonbonded.h:55-126);
    defaults from FF_NonBonded::settodefault (nonbonded.cpp:968-1004)."""

    name = "Non-Bonded Forcefield"

    def __init__(self, wspace):
        super().__init__(wspace)
        self.fast = 0
        self.AutoScaling14 = True
        self.Cutoff = 15.0
        self.InnerCutoff = 12.0
        self.DoVdw = True
        self.VdwCutoff = self.Cutoff
        self.VdwInnerCutoff = self.InnerCutoff
        self.Vdw14Scaling = 1.0
        self.VdwAttenuator = 1.0
        self.VdwCor = False
        self.VdwCorDensity = self.VdwCorEpsilon = self.VdwCorRadius = self.VdwCorCutoff = 0.0
        self.DoElec = True
        self.Elec14Scaling = 1.0
        self.ElecAttenuator = 1.0
        self.Dielectric = 1.0
        self.DDDielectric = False
        self.DDDielectricAlpha = 1.0
        self.ForceSwitch = True
        self.EnergySwitch = False
        self.UsePartialRecalc = False
        self.IgnoreIntraResidue = False

    def _params(self):
        p = A.ff_params_default()
        for k in ("Cutoff", "InnerCutoff", "VdwCutoff", "VdwInnerCutoff", "Vdw14Scaling", "Elec14Scaling",
                  "Dielectric", "DDDielectricAlpha", "VdwCorDensity", "VdwCorEpsilon", "VdwCorRadius",
                  "VdwCorCutoff"):
            setattr(p, k, float(getattr(self, k)))
        for k in ("EnergySwitch", "ForceSwitch", "DDDielectric", "DoVdw", "DoElec", "VdwCor"):
            setattr(p, k, int(bool(getattr(self, k))))
        p.Padding = self.wspace.nlist().Padding
        sp = self.wspace.spec
        if self.AutoScaling14 and "ff_params" in sp:
            # FF_NonBonded::setup takes the 1-4 scalings from the parameter set
            p.Vdw14Scaling, p.Elec14Scaling = float(sp["ff_params"][5]), float(sp["ff_params"][6])
        p.FastMode = 0
        return p


class FF_GeneralizedBorn_Still(FF_NonBonded):
    """Still GB/SA implicit solvent (forcefields/gbff.h:120-200), FastMode
    computing GB + vacuum LJ/Coulomb in one pass by default."""

    name = "Generalised Born Forcefield"

    def __init__(self, wspace):
        super().__init__(wspace)
        # gbff.cpp:17-38
        self.FastMode = True
        self.DielectricSolvent = 80.0
        self.DielectricSolute = 1.0
        self.GbsaStillCutoff = 10.0
        self.ExpApproxThreshold = -4.0
        self.DielectricOffset = -0.090
        self.BornRadiusOffset = 0.0
        self.ForceSwitch = False
        self.EnergySwitch = True

    def _params(self):
        p = super()._params()
        for k in ("DielectricSolvent", "DielectricSolute", "GbsaStillCutoff", "ExpApproxThreshold",
                  "DielectricOffset", "BornRadiusOffset"):
            setattr(p, k, float(getattr(self, k)))
        sp = self.wspace.spec
        if "ff_params" in sp:  # SOLVATION_GENERALISED_BORN GENERALPARAMETERS
            p.P1, p.P2, p.P3, p.P4, p.P5 = (float(x) for x in sp["ff_params"][:5])
        p.Dielectric = self.DielectricSolute  # setup(): Dielectric = DielectricSolute
        p.FastMode = int(bool(self.FastMode))
        return p


class FF_SASA_LCPO(ForcefieldBase):
    """The LCPO surface-area term (forcefields/lcpo.h; Weiser, Shenkin &
    Still 1999): epot_surf = sum of SASA_i * sigma_i over the heavy atoms.

    The per-atom LCPO parameters (type radius + 1.4, P1..P4, use) are the
    ones FF_SASA_LCPO::setup assigns from the parameter file's
    LCPOSASAPARAMETERS section; the SystemSpec carries them (lcpo_radius,
    lcpo_p, lcpo_use).  sigma is GlobalASP (kcal/mol/A^2) on every atom, as
    on the reference's default path, unless ASP holds one value per atom.
    UpdateSasa: inside MD and minimisation the term is recomputed when
    WorkSpace.Step % UpdateSasa == 0 and otherwise reuses the forces of its
    last evaluation (lcpo.cpp:176-190)."""

    name = "LCPO SASA"
    LIST_CUTOFF = 7.0  # FF_SASA_LCPO::setup requests a 7 A neighbour list (lcpo.cpp:20)

    def __init__(self, wspace):
        super().__init__(wspace)
        self.ASPsection_name = ""
        self.GlobalASP = 0.0
        self.UpdateSasa = 5
        self.ASP = None
        self._key = None

    def _sigma(self):
        n = self.wspace.nAtoms()
        if self.ASP is not None:
            sig = np.ascontiguousarray(self.ASP, dtype=np.float64).reshape(-1)
            if sig.shape[0] != n:
                raise ValueError("ASP must hold one value per atom")
            return sig
        return np.full(n, float(self.GlobalASP))

    def _setup(self):
        ws, sp = self.wspace, self.wspace.spec
        if self.ASPsection_name:
            raise A.PdgpuError(A.ERR_ARG, "ASP sections are not read; give per-atom values in ASP")
        for k in ("lcpo_radius", "lcpo_p", "lcpo_use"):
            if k not in sp:
                raise A.PdgpuError(A.ERR_ARG, "the system spec has no LCPO parameters (%s)" % k)
        if int(self.UpdateSasa) < 1:
            raise ValueError("UpdateSasa must be >= 1")
        sig = self._sigma()
        key = (sig.tobytes(), int(self.UpdateSasa), bool(self.Active))
        if key == self._key and ws._lcpo_set:
            return
        use = np.ascontiguousarray(sp["lcpo_use"], dtype=np.uint8)
        A.check(A.lib().pdgpu_sasa_lcpo_set(
            ws.ctx.ptr, ws._sys, A.dptr(A.cd(sp["lcpo_radius"])), A.dptr(A.cd(sp["lcpo_p"]).reshape(-1)),
            A.dptr(sig), use.ctypes.data_as(A._U8), int(self.UpdateSasa) if self.Active else 0))
        self._key = key
        ws._lcpo_set = bool(self.Active)

    def sasa(self):
        """Per-atom SASA (A^2) of the last evaluation and SASAderiv of the
        last full one (kcal/mol/A, [n, 3])."""
        ws = self.wspace
        n = ws.nAtoms()
        a, d = np.zeros(n), np.zeros((n, 3))
        A.check(A.lib().pdgpu_sasa_lcpo_get(ws.ctx.ptr, ws._sys, A.dptr(a), A.dptr(d)))
        return a, d


class Forcefield:
    """The component container (forcefield.h:266-319): calcForces zeroes the
    workspace and runs every component (forcefield.cpp:220-247)."""

    def __init__(self, wspace: WorkSpace):
        self.wspace = wspace
        self.components = []
        self.max_force = -1.0

    def add(self, comp):
        if comp.getWSpace() is not self.wspace:
            raise ValueError("You cannot add this force field component because they use different workspaces.")
        self.components.append(comp)
        self.wspace._ff = self

    def getWSpace(self):
        return self.wspace

    def _nb(self, required=True):
        nb = [c for c in self.components if isinstance(c, FF_NonBonded) and c.Active]
        if len(nb) > 1 or (required and not nb):
            raise A.PdgpuError(A.ERR_ARG, "the GPU path needs exactly one FF_NonBonded / "
                                          "FF_GeneralizedBorn_Still component")
        return nb[0] if nb else None

    def _has_bonded(self):
        return any(isinstance(c, FF_Bonded) and c.Active for c in self.components)

    def _lcpo(self):
        lc = [c for c in self.components if isinstance(c, FF_SASA_LCPO)]
        if len(lc) > 1:
            raise A.PdgpuError(A.ERR_ARG, "more than one FF_SASA_LCPO component")
        return lc[0] if lc else None

    def ensuresetup(self, wspace=None):
        lc = self._lcpo()
        nb = self._nb(required=lc is None)
        ws = self.wspace
        if nb is not None:
            ws.nlist().requestCutoff(max(nb.Cutoff, nb.VdwCutoff))
            if isinstance(nb, FF_GeneralizedBorn_Still):
                ws.nlist().calcShadow(True)
            params = nb._params()
            if lc is not None and lc.Active and max(nb.Cutoff, nb.VdwCutoff) < lc.LIST_CUTOFF:
                raise A.PdgpuError(A.ERR_ARG, "FF_SASA_LCPO needs a neighbour list of at least 7 A: "
                                              "set the non-bonded Cutoff >= 7")
        else:
            # the surface term alone: a 7 A list and no pair passes
            ws.nlist().requestCutoff(lc.LIST_CUTOFF)
            params = A.ff_params_default()
            params.Cutoff = params.VdwCutoff = lc.LIST_CUTOFF
            params.InnerCutoff = params.VdwInnerCutoff = lc.LIST_CUTOFF - 3.0
            params.Padding = ws.nlist().Padding
        ws._ensure_device(params, self._has_bonded())
        if lc is not None:
            lc._setup()
        elif ws._lcpo_set:
            A.check(A.lib().pdgpu_sasa_lcpo_set(ws.ctx.ptr, ws._sys, None, None, None, None, 0))
            ws._lcpo_set = False
        return 0

    def _lcpo_active(self):
        lc = self._lcpo()
        return lc is not None and lc.Active

    def _sync_in(self):
        ws = self.wspace
        if ws._pos_dirty:
            ws._push_positions()

    def _sync_out(self, with_forces=True):
        ws = self.wspace
        if with_forces:
            ws.cur.f[:] = ws._pull_forces()
        ws.ene.load(ws._pull_energies())

    def calcForces(self):
        self.ensuresetup()
        self._sync_in()
        nb = self._nb(required=self._lcpo() is None)
        ws, L = self.wspace, A.lib()
        if self.wspace.nlist().getFullUpdateCount() == 0:
            self.wspace.nlist().calcNewList()
        A.check(L.pdgpu_zero_forces(ws.ctx.ptr, ws._sys))
        if self._has_bonded():
            A.check(L.pdgpu_bonded_forces(ws.ctx.ptr, ws._sys))
        if isinstance(nb, FF_GeneralizedBorn_Still):
            A.check(L.pdgpu_gb_forces(ws.ctx.ptr, ws._sys))
        elif nb is not None:
            A.check(L.pdgpu_nonbonded_forces(ws.ctx.ptr, ws._sys))
        if self._lcpo_active():
            A.check(L.pdgpu_sasa_lcpo_forces(ws.ctx.ptr, ws._sys, int(ws.Step)))
        self._sync_out()
        if not np.isfinite(ws.ene.epot_vdw) or not np.isfinite(ws.ene.epot_elec):
            ws.ene.epot = float("nan")

    def calcEnergies(self):
        self.ensuresetup()
        self._sync_in()
        nb = self._nb(required=self._lcpo() is None)
        ws, L = self.wspace, A.lib()
        if self.wspace.nlist().getFullUpdateCount() == 0:
            self.wspace.nlist().calcNewList()
        A.check(L.pdgpu_zero_forces(ws.ctx.ptr, ws._sys))
        if self._has_bonded():
            A.check(L.pdgpu_bonded_forces(ws.ctx.ptr, ws._sys))
        if isinstance(nb, FF_GeneralizedBorn_Still):
            A.check(L.pdgpu_gb_energies(ws.ctx.ptr, ws._sys))
        elif nb is not None:
            A.check(L.pdgpu_nonbonded_forces(ws.ctx.ptr, ws._sys))
        if self._lcpo_active():
            A.check(L.pdgpu_sasa_lcpo_energies(ws.ctx.ptr, ws._sys))
        self._sync_out()

    def printEnergySummary(self):
        self.ensuresetup()
        self.wspace.nlist().calcNewList()
        self.calcForces()
        e = self.wspace.ene
        print(" VdW:           %10.3f kcal/mol" % e.kcal("epot_vdw"))
        print(" Electrostatic: %10.3f kcal/mol" % e.kcal("epot_elec"))
        print(" GB:            %10.3f kcal/mol" % e.kcal("epot_pol"))
        if self._lcpo_active():
            print(" SASA Energy:   %10.3f kcal/mol" % e.kcal("epot_surf"))
        print(" Total energy: %10.3f kcal/mol" % e.kcal("epot"))


# ------------------------------------------------------------------ protocols
class ProtocolBase:
    """protocols/protocolbase.h: Steps, UpdateNList and the run() contract."""

    def __init__(self, ff: Forcefield):
        self.ff = ff
        self.Steps = 0
        self.UpdateScr = 0
        self.UpdateTra = 0
        self.UpdateMon = 1
        self.UpdateNList = 1
        self.OutputLevel = 0

    def getWSpace(self):
        return self.ff.getWSpace()

    def run(self):
        if self.Steps == 0:
            raise ValueError("You must set the number of steps before starting your simulation")
        self.ff.ensuresetup()
        return self.runcore()


class Energy(ProtocolBase):
    """Single point: list refresh + calcEnergies (energy.cpp:14-20)."""

    def __init__(self, ff):
        super().__init__(ff)
        self.Steps = 1

    def runcore(self):
        self.ff.ensuresetup()
        self.ff._sync_in()
        self.getWSpace().nlist().calcNewList()
        self.ff.calcEnergies()
        return 1


class Minimisation(ProtocolBase):
    """Steepest descent / conjugate gradients with the reference's adaptive
    step multiplier and restore-on-increase (minimise.cpp:99-318), run with
    its control flow on the device."""

    SteepestDescent = A.MIN_STEEPEST_DESCENT
    ConjugateGradients = A.MIN_CONJUGATE_GRADIENTS

    def __init__(self, ff):
        super().__init__(ff)
        d = A.min_params_default()
        self.Algorithm = d.Algorithm
        self.StepSize = d.StepSize
        self.SlopeCutoff = d.SlopeCutoff
        self.Strictness = d.Strictness
        self.Step = 0

    def runcore(self):
        ws = self.getWSpace()
        self.ff.ensuresetup()
        self.ff._sync_in()
        p = A.MinParams()
        p.Algorithm, p.UpdateNList = int(self.Algorithm), int(self.UpdateNList)
        p.StepSize, p.SlopeCutoff, p.Strictness = self.StepSize, self.SlopeCutoff, self.Strictness
        taken = ctypes.c_int32(0)
        st = A.lib().pdgpu_minimise_run(ws.ctx.ptr, ws._sys, ctypes.byref(p), int(self.Steps),
                                        ctypes.byref(taken))
        if st == A.ERR_UNSTABLE:
            return -1
        A.check(st)
        ws._pull_positions()
        self.ff._sync_out()
        self.Step = taken.value
        ws._pull_step()
        return taken.value


class MonteCarlo(ProtocolBase):
    """MonteCarlo (protocols/montecarlo.h:36-125) with backbone phi/psi moves
    of every residue (sigma Sigma rad each) as the move set and the
    forcefield's calcForces after a list rebuild as the evaluator, run on the
    device (pdgpu_mc_run).  Temperature is constant (K); FinalState is Last,
    LastAcc (default) or LowestEpot, as in the reference.  After run():
    acceptances and lowest (the lowest accepted epot, J)."""

    Last, LastAcc, LowestEpot = A.MC_LAST, A.MC_LAST_ACC, A.MC_LOWEST_EPOT

    def __init__(self, ff):
        super().__init__(ff)
        d = A.mc_params_default()
        self.Temperature = d.Temperature
        self.Sigma = d.Sigma
        self.FinalState = d.FinalState
        self.Seed = 0
        self.acceptances = 0
        self.lowest = float("nan")

    def runcore(self):
        ws = self.getWSpace()
        self.ff.ensuresetup()
        self.ff._sync_in()
        if getattr(ws, "nRotations", 0) == 0:
            ws.setTorsionMoves()
        p = A.mc_params_default()
        p.Steps, p.FinalState = int(self.Steps), int(self.FinalState)
        p.Temperature, p.Sigma, p.Seed = float(self.Temperature), float(self.Sigma), int(self.Seed)
        acc = np.zeros(1, dtype=np.int32)
        low = np.zeros(1)
        A.check(A.lib().pdgpu_mc_run(ws.ctx.ptr, ws._sys, ctypes.byref(p), A.iptr(acc), A.dptr(low)))
        self.acceptances, self.lowest = int(acc[0]), float(low[0])
        ws._pull_positions()
        self.ff._sync_out()
        ws._pull_step()
        return int(self.Steps)


def read_trajectory(ctx, handle, natoms, max_frames):
    """Frames recorded since the last read: (frames[n][natoms][3] in A,
    steps[n]) and the number overwritten before they were read."""
    frames = np.zeros((max_frames, natoms, 3))
    steps = np.zeros(max_frames, dtype=np.int64)
    n, dropped = ctypes.c_int32(0), ctypes.c_int32(0)
    A.check(A.lib().pdgpu_md_read_trajectory(ctx.ptr, handle, A.dptr(frames),
                                             steps.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                             int(max_frames), ctypes.byref(n), ctypes.byref(dropped)))
    return (frames[: n.value].copy(), steps[: n.value].copy()), dropped.value


class MolecularDynamics(ProtocolBase):
    """MD protocol (protocols/md.h:84-128; md.cpp:202-267) with the step loop
    on the device: list rebuild every UpdateNList steps, forces, integrator,
    the UpdateNList-step blocks captured in a CUDA graph."""

    Verlet = A.INTEGRATOR_VERLET
    VelocityVerlet = A.INTEGRATOR_VELOCITY_VERLET
    Beeman = A.INTEGRATOR_BEEMAN
    Langevin = A.INTEGRATOR_LANGEVIN

    def __init__(self, ff):
        super().__init__(ff)
        d = A.md_params_default()
        self.Integrator = d.Integrator
        self.Timestep = d.Timestep
        self.RandVel = True
        self.TargetTemp = d.TargetTemp
        self.FricCoeff = d.FricCoeff
        self.LangevinOnHydrogens = True
        self.UpdateNList = d.UpdateNList
        self.UseGraph = True
        self.Seed = 0
        self.UpdateTra = 0            # record a frame every UpdateTra steps (0: none)
        self.TrajectoryCapacity = 1000
        self.history = None
        self.frames = None            # (frames[n][natoms][3] A, steps[n]) of the last run
        self.dropped = 0

    def _params(self):
        p = A.md_params_default()
        p.Integrator, p.UpdateNList = int(self.Integrator), int(self.UpdateNList)
        p.LangevinOnHydrogens, p.UseGraph = int(bool(self.LangevinOnHydrogens)), int(bool(self.UseGraph))
        p.Timestep, p.FricCoeff, p.TargetTemp = self.Timestep, self.FricCoeff, float(self.TargetTemp)
        p.Seed = int(self.Seed)
        return p

    def runcore(self):
        ws = self.getWSpace()
        self.ff.ensuresetup()
        self.ff._sync_in()
        L = A.lib()
        if self.RandVel:
            A.check(L.pdgpu_md_init_velocities(ws.ctx.ptr, ws._sys, float(self.TargetTemp), int(self.Seed)))
        else:
            ws._push_velocities()
        hist = np.zeros(3 * int(self.Steps))
        every = int(self.UpdateTra)
        cap = max(1, int(self.TrajectoryCapacity))
        A.check(L.pdgpu_md_set_trajectory(ws.ctx.ptr, ws._sys, every, cap))
        st = L.pdgpu_md_run(ws.ctx.ptr, ws._sys, ctypes.byref(self._params()), 0, int(self.Steps),
                            int(self.Steps), A.dptr(hist))
        self.history = hist.reshape(-1, 3)
        if st == A.ERR_UNSTABLE:
            raise A.UnstableError(st, A.last_error())
        A.check(st)
        self.frames, self.dropped = None, 0
        if every > 0:
            self.frames, self.dropped = read_trajectory(ws.ctx, ws._sys, ws.nAtoms(), cap)
            A.check(L.pdgpu_md_set_trajectory(ws.ctx.ptr, ws._sys, 0, 0))
        ws._pull_positions()
        ws._pull_velocities()
        self.ff._sync_out()
        ws._pull_step()
        return int(self.Steps)
