"""GPU: the request loop (pdgpu_serve_*).

A served job must give the same results alone and in a mix of overlapping
jobs -- bit for bit, since every job runs the same kernels (list rows with
fixed lanes per atom, or the cluster-pair tiles) on its own device state --
and the same results as the plain calls (pdgpu_nlist_build +
pdgpu_calc_forces, pdgpu_minimise_run, pdgpu_md_run) on that layout.
Single-point forces also match the reference's FP64 forces (relative force
RMS 1e-5).
"""
import numpy as np
import pytest

from conftest import build_workspace, load_library, rel_rms

pytestmark = pytest.mark.gpu

LANES = (8, 8, 8)


def _members(ctx, count):
    return [build_workspace(a, m, ctx) + (a, m) for a, m in load_library("lib16_amber_s3")[:count]]


def _jobs(pdgpu):
    S = pdgpu.Server
    md = pdgpu.md_params_default()
    md.Integrator = pdgpu.MolecularDynamics.Langevin
    md.FricCoeff = 1e12
    md.UpdateNList = 10
    mn = pdgpu.min_params_default()
    mn.Algorithm = pdgpu.Minimisation.SteepestDescent
    jobs = []
    for k in range(6):
        if k % 3 == 0:
            jobs.append(S.job(S.ENERGY))
        elif k % 3 == 1:
            jobs.append(S.job(S.MINIMISE, 30, minimiser=mn))
        else:
            m = pdgpu.md_params_default()
            ctypes_copy(m, md)
            m.Seed = 100 + k
            jobs.append(S.job(S.MD, 40, md=m, init_temp=300.0))
    return jobs


def ctypes_copy(dst, src):
    for name, _ in type(src)._fields_:
        setattr(dst, name, getattr(src, name))


def _run(server, members, jobs, together):
    ids = []
    if together:
        ids = [server.submit(ws, j) for (ws, *_), j in zip(members, jobs)]
        for jid in ids:
            assert server.wait(jid, 120.0) == 0
    else:
        for (ws, *_), j in zip(members, jobs):
            jid = server.submit(ws, j)
            assert server.wait(jid, 120.0) == 0
            ids.append(jid)
    out = [server.result(jid) for jid in ids]
    infos = [server.info(jid) for jid in ids]
    for jid in ids:
        server.release(jid)
    return out, infos


@pytest.mark.parametrize("tiles", [False, True])
def test_serve_alone_equals_mixed(gpu_ctx, tiles):
    import pdgpu
    members = _members(gpu_ctx, 6)
    jobs = _jobs(pdgpu)
    srv = pdgpu.Server(gpu_ctx, max_active=8, lanes=LANES, tiles=tiles)
    alone, _ = _run(srv, members, jobs, together=False)
    mixed, infos = _run(srv, members, jobs, together=True)
    st = srv.stats()
    srv.close()
    assert st["peak_active"] >= 2  # the mix really overlapped on the device
    assert st["failed"] == 0 and st["completed"] == 12
    for a, b, info in zip(alone, mixed, infos):
        for key in a:
            assert np.array_equal(a[key], b[key]), key
        assert info["state"] == 2  # PDGPU_JOB_DONE
        assert info["t_total_ms"] >= info["t_run_ms"] >= 0.0


@pytest.mark.parametrize("tiles", [True, False])
def test_serve_matches_plain_calls_and_reference(gpu_ctx, tiles):
    import pdgpu
    members = _members(gpu_ctx, 6)
    jobs = _jobs(pdgpu)
    srv = pdgpu.Server(gpu_ctx, max_active=8, lanes=LANES, tiles=tiles)
    served, infos = _run(srv, members, jobs, together=True)
    srv.close()
    for (ws, ff, a, m), job, res, info in zip(members, jobs, served, infos):
        one = pdgpu.Batch([ws])
        # the server's layout: tiles, or list rows with these lanes
        if tiles:
            one.setPairPath(1)
        else:
            one.setLanes(LANES)
        if job.kind == pdgpu.Server.ENERGY:
            f, e = one.evaluate()
            assert np.array_equal(res["forces"], f)
            assert np.array_equal(res["energies"], e[0])
            assert rel_rms(res["forces"], a["f_total"]) <= 1e-5
            assert info["steps_done"] == 1
        elif job.kind == pdgpu.Server.MINIMISE:
            taken = one.minimise(job.min, job.steps)
            assert info["steps_done"] == taken[0] == job.steps
            assert np.array_equal(res["positions"], one.positions())
            assert np.array_equal(res["forces"], one.forces())
            assert np.array_equal(res["energies"], one.energies()[0])
        else:
            one.calcNewList()
            h = one.runMD(job.md, job.steps, init_velocities=job.init_temp)
            assert np.array_equal(res["positions"], one.positions())
            assert np.array_equal(res["history"], h[:, 0, :])
            assert info["steps_done"] == job.steps
        one.close()


def test_serve_budget_admission(gpu_ctx):
    import pdgpu
    members = _members(gpu_ctx, 6)
    ws = max(members, key=lambda m: m[0].nAtoms())[0]
    n = ws.nAtoms()
    nsc, njc = (n + 31) // 32, (n + 7) // 8
    tiles = sum(njc - 4 * k for k in range(nsc))
    # the server's admission estimate (include/pdgpu.h, pdgpu_serve_submit)
    est = n * (1024 + 256 * 4) + tiles * 48 + nsc * 16 * 64 + 4 * 1024 * 1024
    budget = int(2.5 * est)  # room for two such jobs at a time
    srv = pdgpu.Server(gpu_ctx, hbm_budget=budget, max_active=8, lanes=LANES)
    job = pdgpu.Server.job(pdgpu.Server.MINIMISE, 20)
    ids = [srv.submit(ws, job) for _ in range(6)]
    for jid in ids:
        assert srv.wait(jid, 120.0) == 0
    st = srv.stats()
    assert st["completed"] == len(ids)
    assert st["peak_bytes"] <= budget
    assert st["peak_active"] <= 2
    # a job that cannot fit at all is refused at submission
    tiny = pdgpu.Server(gpu_ctx, hbm_budget=1024 * 1024, max_active=2, lanes=LANES)
    with pytest.raises(pdgpu.PdgpuError):
        tiny.submit(members[0][0], job)
    tiny.close()
    srv.close()


def test_serve_failed_job_does_not_disturb_others(gpu_ctx):
    """A job whose energy turns NaN fails alone (assertStability,
    protocolbase.cpp:104-110); the jobs running beside it are unaffected."""
    import pdgpu
    members = _members(gpu_ctx, 3)
    srv = pdgpu.Server(gpu_ctx, max_active=4, lanes=LANES)
    md = pdgpu.md_params_default()
    md.Integrator = pdgpu.MolecularDynamics.Langevin
    md.FricCoeff = 1e12
    job = pdgpu.Server.job(pdgpu.Server.MD, 20, md=md)
    ref_ids = [srv.submit(ws, job) for ws, *_ in members[1:]]
    ref = [srv.result(j) if srv.wait(j, 120.0) == 0 else None for j in ref_ids]
    bad_pos = members[0][0].cur.p.copy()
    bad_pos[5] = np.nan
    bad = srv.submit(members[0][0], job, positions=bad_pos)
    ok_ids = [srv.submit(ws, job) for ws, *_ in members[1:]]
    assert srv.wait(bad, 120.0) == pdgpu._abi.ERR_UNSTABLE
    for j, r in zip(ok_ids, ref):
        assert srv.wait(j, 120.0) == 0
        got = srv.result(j)
        assert np.array_equal(got["positions"], r["positions"])
    assert srv.info(bad)["state"] == 3
    srv.close()


def _md_job(pdgpu, seed, steps=30):
    md = pdgpu.md_params_default()
    md.Integrator = pdgpu.MolecularDynamics.Langevin
    md.FricCoeff = 1e12
    md.UpdateNList = 10
    md.Seed = seed
    return pdgpu.Server.job(pdgpu.Server.MD, steps, md=md)


@pytest.mark.parametrize("kind", ["energy", "minimise", "md"])
def test_serve_group_equals_alone(gpu_ctx, kind):
    """Jobs that queue behind a busy slot are admitted as one group (one
    pack, one launch sequence); each member's results are the bits it gets
    served alone (MD members each with their own seed)."""
    import pdgpu
    members = _members(gpu_ctx, 8)
    S = pdgpu.Server
    mn = pdgpu.min_params_default()
    mn.Algorithm = pdgpu.Minimisation.SteepestDescent
    if kind == "energy":
        jobs = lambda: [S.job(S.ENERGY) for _ in members]
    elif kind == "minimise":
        jobs = lambda: [S.job(S.MINIMISE, 40, minimiser=mn) for _ in members]
    else:
        jobs = lambda: [_md_job(pdgpu, 100 + k) for k in range(len(members))]
    srv = pdgpu.Server(gpu_ctx, max_active=1, lanes=LANES, tiles=True)
    alone, _ = _run(srv, members, jobs(), together=False)
    grouped, infos = _run(srv, members, jobs(), together=True)
    st = srv.stats()
    srv.close()
    assert st["groups"] >= 1  # the queued jobs shared a pack
    for a, g, (ws, ff, arr, m) in zip(alone, grouped, members):
        for key in a:
            assert np.array_equal(a[key], g[key]), key
        if kind == "energy":
            assert rel_rms(g["forces"], arr["f_total"]) <= 1e-5
    for ws, *_ in members:
        ws.close()


def test_serve_md_group_member_nan(gpu_ctx):
    """An MD group goes on past a member whose energy turns NaN: that member
    fails (UNSTABLE), the others give the bits they get served alone."""
    import pdgpu
    members = _members(gpu_ctx, 4)
    srv = pdgpu.Server(gpu_ctx, max_active=1, lanes=LANES, tiles=True)
    alone, _ = _run(srv, members[1:], [_md_job(pdgpu, 200 + k) for k in range(1, 4)], together=False)
    # a busy slot first, so the four queue and are admitted together
    blocker = srv.submit(members[0][0], _md_job(pdgpu, 7, steps=60))
    bad_pos = members[0][0].cur.p.copy()
    bad_pos[5] = np.nan
    bad = srv.submit(members[0][0], _md_job(pdgpu, 200), positions=bad_pos)
    ok = [srv.submit(ws, _md_job(pdgpu, 200 + k)) for k, (ws, *_) in enumerate(members[1:], start=1)]
    assert srv.wait(blocker, 120.0) == 0
    assert srv.wait(bad, 120.0) == pdgpu._abi.ERR_UNSTABLE
    assert srv.info(bad)["state"] == 3
    for jid, a in zip(ok, alone):
        assert srv.wait(jid, 120.0) == 0
        got = srv.result(jid)
        for key in a:
            assert np.array_equal(a[key], got[key]), key
    st = srv.stats()
    srv.close()
    assert st["groups"] >= 1
    for ws, *_ in members:
        ws.close()
