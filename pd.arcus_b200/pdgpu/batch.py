"""Batches: many independent WorkSpaces evaluated together.

No reference counterpart (the reference evaluates one WorkSpace per call).
A ``Batch`` packs the member systems' atoms into one device pack behind
per-system offset tables (``pdgpu_batch_create``), so that one launch of
each kernel covers every member: neighbour lists, Born radii, the fused GB
pass, the chain-rule pass, bonded terms, integrator and minimiser steps.
Each member's results equal the ones it gets alone: lists, reductions and
RNG streams are per system.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi as A


class Batch:
    """Members are WorkSpaces whose forcefield is set up (their positions,
    velocities and settings are taken at construction)."""

    def __init__(self, workspaces, ctx=None):
        self.members = list(workspaces)
        if not self.members:
            raise ValueError("a batch needs at least one workspace")
        self.ctx = ctx or self.members[0].ctx
        ids = []
        for ws in self.members:
            if ws.ctx is not self.ctx:
                raise ValueError("all members must live on the batch's context")
            ids.append(ws._device())
        ids = np.asarray(ids, dtype=np.int32)
        bid = ctypes.c_int32(0)
        A.check(A.lib().pdgpu_batch_create(self.ctx.ptr, A.iptr(ids), len(ids), ctypes.byref(bid)))
        self._id = bid.value
        off = np.zeros(len(ids) + 1, dtype=np.int32)
        A.check(A.lib().pdgpu_batch_info(self.ctx.ptr, self._id, None, A.iptr(off)))
        self.offsets = off
        self.nAtoms = int(off[-1])
        self.nSystems = len(ids)
        self.history = None

    # -- layout helpers
    def split(self, arr):
        """Per-member views of a packed per-atom array."""
        return [arr[self.offsets[s]:self.offsets[s + 1]] for s in range(self.nSystems)]

    def _get3(self, fn):
        out = np.zeros((self.nAtoms, 3))
        A.check(fn(self.ctx.ptr, self._id, A.dptr(out)))
        return out

    # -- state
    def positions(self):
        return self._get3(A.lib().pdgpu_get_positions)

    def setPositions(self, pos):
        p = np.concatenate([np.asarray(x, dtype=np.float64).reshape(-1, 3) for x in pos]) \
            if isinstance(pos, (list, tuple)) else np.asarray(pos, dtype=np.float64).reshape(-1, 3)
        A.check(A.lib().pdgpu_set_positions(self.ctx.ptr, self._id, A.dptr(A.cd(p))))

    def velocities(self):
        return self._get3(A.lib().pdgpu_get_velocities)

    def forces(self):
        return self._get3(A.lib().pdgpu_get_forces)

    def born_radii(self):
        b = np.zeros(self.nAtoms)
        A.check(A.lib().pdgpu_get_born_radii(self.ctx.ptr, self._id, A.dptr(b)))
        return b

    def energies(self):
        """(nSystems, ENE_COUNT) energy records, J."""
        e = np.zeros(self.nSystems * A.ENE_COUNT)
        A.check(A.lib().pdgpu_get_energies(self.ctx.ptr, self._id, A.dptr(e), len(e)))
        return e.reshape(self.nSystems, A.ENE_COUNT)

    def setLanes(self, lpa=None):
        """Fix the lanes per atom of the Born, fused and chain kernels
        (None: autotune)."""
        arr = None if lpa is None else A.iptr(np.ascontiguousarray(lpa, dtype=np.int32))
        A.check(A.lib().pdgpu_set_lanes(self.ctx.ptr, self._id, arr))

    def setPairPath(self, path):
        """0: neighbour-list rows, 1: cluster-pair tiles, -1: autotune;
        returns the layout in use."""
        cur = ctypes.c_int32(0)
        A.check(A.lib().pdgpu_pair_path(self.ctx.ptr, self._id, int(path), ctypes.byref(cur)))
        return cur.value

    def setEvalMode(self, mode):
        """Launch form of an evaluation on the tile layout: 1 one
        cooperative launch, 0 three launches, 2 (the default) cooperative
        except inside MD step blocks, -1 report only."""
        cur = ctypes.c_int32(0)
        A.check(A.lib().pdgpu_eval_mode(self.ctx.ptr, self._id, int(mode), ctypes.byref(cur)))
        return cur.value

    def setSeeds(self, seeds=None):
        if seeds is None:
            A.check(A.lib().pdgpu_set_seeds(self.ctx.ptr, self._id, None))
            return
        k = np.ascontiguousarray(seeds, dtype=np.uint64)
        if k.shape != (self.nSystems,):
            raise ValueError("one seed per member")
        A.check(A.lib().pdgpu_set_seeds(self.ctx.ptr, self._id,
                                        k.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))))

    # -- evaluation
    def calcNewList(self):
        A.check(A.lib().pdgpu_nlist_build(self.ctx.ptr, self._id))

    def calcForces(self):
        """Forcefield::calcForces for every member (list must be current)."""
        A.check(A.lib().pdgpu_calc_forces(self.ctx.ptr, self._id))

    def evaluate(self):
        """List rebuild + forces; returns (forces, energies)."""
        self.calcNewList()
        self.calcForces()
        return self.forces(), self.energies()

    # -- trial moves
    def saveBasePositions(self):
        A.check(A.lib().pdgpu_save_base_positions(self.ctx.ptr, self._id))

    def perturbTorsions(self, sigma=0.0, trial=0, angles=None):
        ang = None if angles is None else A.dptr(A.cd(np.concatenate([np.ravel(a) for a in angles])
                                                      if isinstance(angles, (list, tuple)) else angles))
        A.check(A.lib().pdgpu_perturb_torsions(self.ctx.ptr, self._id, float(sigma), int(trial), ang))

    # -- protocols
    def runMC(self, steps, temperature=300.0, sigma=None, final_state=None, seed=0):
        """MonteCarlo for every member on the device (pdgpu_mc_run): phi/psi
        moves, list rebuild + forces as the evaluator, the Metropolis test.
        Returns (acceptances per member, lowest accepted epot per member, J)."""
        p = A.mc_params_default()
        p.Steps, p.Temperature, p.Seed = int(steps), float(temperature), int(seed)
        if sigma is not None:
            p.Sigma = float(sigma)
        if final_state is not None:
            p.FinalState = int(final_state)
        acc = np.zeros(self.nSystems, dtype=np.int32)
        low = np.zeros(self.nSystems)
        A.check(A.lib().pdgpu_mc_run(self.ctx.ptr, self._id, ctypes.byref(p), A.iptr(acc), A.dptr(low)))
        return acc, low

    def runMD(self, params: A.MDParams, steps, first_step=0, total_steps=None, init_velocities=None):
        """MolecularDynamics::run_core for every member at once; returns the
        (steps, nSystems, 3) history of epot, ekin, etot (J)."""
        L = A.lib()
        if init_velocities is not None:
            A.check(L.pdgpu_md_init_velocities(self.ctx.ptr, self._id, float(init_velocities), int(params.Seed)))
        total = steps if total_steps is None else total_steps
        hist = np.zeros(3 * steps * self.nSystems)
        st = L.pdgpu_md_run(self.ctx.ptr, self._id, ctypes.byref(params), int(first_step), int(steps), int(total),
                            A.dptr(hist))
        self.history = hist.reshape(steps, self.nSystems, 3)
        A.check(st)
        return self.history

    def minimise(self, params: A.MinParams, steps):
        """Minimisation::runcore for every member; returns the steps each
        member took (-1: NaN energy)."""
        taken = np.zeros(self.nSystems, dtype=np.int32)
        A.check(A.lib().pdgpu_minimise_run(self.ctx.ptr, self._id, ctypes.byref(params), int(steps),
                                           A.iptr(taken)))
        return taken

    def last_run_ms(self):
        return self.ctx.last_run_ms()

    def close(self):
        if self._id is not None and self.ctx.ptr:
            A.lib().pdgpu_system_destroy(self.ctx.ptr, self._id)
        self._id = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
