"""Serving: a request loop for single-point, minimisation and MD jobs.

No reference counterpart (the reference runs one protocol on one WorkSpace
at a time).  ``Server`` wraps ``pdgpu_serve_*``: a worker thread inside
libpdgpu admits jobs against an HBM budget, keeps each admitted job's state
on the device on its own stream, and overlaps the jobs' kernels.  Jobs name
a WorkSpace whose forcefield is set up (topology and settings) and carry
their own start positions.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi as A


class Server:
    ENERGY, MINIMISE, MD = A.JOB_ENERGY, A.JOB_MINIMISE, A.JOB_MD

    ARRIVAL, LEAST_WORK = 0, 1

    def __init__(self, ctx, hbm_budget=None, max_active=None, lanes=(8, 8, 8), tiles=True, policy=1, group=True,
                 batch_ms=None):
        self.ctx = ctx
        p = A.ServeParams()
        A.lib().pdgpu_serve_params_default(ctypes.byref(p))
        if hbm_budget is not None:
            p.hbm_budget = int(hbm_budget)
        if max_active is not None:
            p.max_active = int(max_active)
        for q in range(3):
            p.lanes[q] = int(lanes[q])
        p.tiles = int(bool(tiles))
        p.policy = int(policy)
        p.group = int(bool(group))
        if batch_ms is not None:
            p.batch_ms = int(batch_ms)
        self.params = p
        self.ptr = ctypes.c_void_p()
        A.check(A.lib().pdgpu_serve_create(ctx.ptr, ctypes.byref(p), ctypes.byref(self.ptr)))
        self._natoms = {}
        self._kind = {}

    @staticmethod
    def job(kind, steps=0, md=None, minimiser=None, init_temp=300.0):
        j = A.Job()
        j.kind, j.steps = int(kind), int(steps)
        j.md = md if md is not None else A.md_params_default()
        j.min = minimiser if minimiser is not None else A.min_params_default()
        j.init_temp = float(init_temp)
        return j

    def submit(self, ws, job, positions=None):
        """Queue `job` on WorkSpace `ws` (from `positions`, default ws.cur.p)."""
        sid = ws._device()
        x = np.ascontiguousarray(ws.cur.p if positions is None else positions, dtype=np.float64).reshape(-1, 3)
        jid = ctypes.c_int64(0)
        A.check(A.lib().pdgpu_serve_submit(self.ptr, sid, ctypes.byref(job), A.dptr(x), ctypes.byref(jid)))
        self._natoms[jid.value] = x.shape[0]
        self._kind[jid.value] = (job.kind, job.steps)
        return jid.value

    def wait(self, jid, timeout=-1.0):
        return A.lib().pdgpu_serve_wait(self.ptr, int(jid), float(timeout))

    def info(self, jid):
        i = A.JobInfo()
        A.check(A.lib().pdgpu_serve_info(self.ptr, int(jid), ctypes.byref(i)))
        return {k: getattr(i, k) for k, _ in A.JobInfo._fields_ if not k.startswith("_")}

    def result(self, jid):
        n = self._natoms[jid]
        kind, steps = self._kind[jid]
        x, f, e = np.zeros((n, 3)), np.zeros((n, 3)), np.zeros(A.ENE_COUNT)
        h = np.zeros(3 * max(steps, 1)) if kind == A.JOB_MD else None
        A.check(A.lib().pdgpu_serve_result(self.ptr, int(jid), A.dptr(x), A.dptr(f), A.dptr(e),
                                           A.dptr(h) if h is not None else None))
        out = {"positions": x, "forces": f, "energies": e}
        if h is not None:
            out["history"] = h.reshape(-1, 3)
        return out

    def release(self, jid):
        A.check(A.lib().pdgpu_serve_release(self.ptr, int(jid)))
        self._natoms.pop(jid, None)
        self._kind.pop(jid, None)

    def stats(self):
        s = A.ServeStats()
        A.check(A.lib().pdgpu_serve_get_stats(self.ptr, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in A.ServeStats._fields_ if not k.startswith("_")}

    def close(self):
        if self.ptr:
            A.lib().pdgpu_serve_destroy(self.ptr)
            self.ptr = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
