"""GB MD throughput on one large system, B200, plus the batched workloads.

Headline workload (the reference's single-large-system configuration): 16
seeded 80-residue peptides on a 4x4 grid 25 A apart, 20,566 atoms, built by
the reference's own builder and pre-minimised (tests/golden/c2_16x80_s2.npz),
AMBER99 + Still GB (FastMode) + bonded terms, Rc 16 A (inner 13 A),
neighbour list rebuilt every 10 steps, Langevin dynamics at 1 fs, 300 K,
friction 1/ps.  A "step" is one MD step: list refresh (every 10th), bonded +
Born radii + fused GB/LJ/Coulomb + chain-rule forces, integrator.

Extra keys of the same JSON line:
  plain_small the plain small method: one 64-residue peptide (1,001 atoms),
              Rc 12 A, 1,000 Langevin steps at 1 fs (friction 1e13/s, the
              reference's default), ns/day beside the reference's own CPU MD
              on one core.
  batched_sp  512 distinct AMBER99 peptides, lengths log-uniform 20-200
              residues: the 16 reference-built peptides of
              tests/golden/lib16_amber_s3.npz and 496 seeded ones spliced from
              their residue templates (pdgpu.peptides) and relaxed with 500
              steepest-descent steps on the device; each with its own RNG key,
              x 64 backbone phi/psi trials (sigma 15 deg) drawn on the device:
              32,768 energy+force evaluations, Rc 12 A, in 64 batched
              evaluations of all 512 systems; against the plain path (one
              system per launch sequence) on a sample.  device_mc: the same
              batch through the whole Monte Carlo protocol on the device
              (64 steps, Metropolis at 300 K, pdgpu_mc_run).
  batched_md  256 distinct OPLS-AA peptides of 30-150 residues (the 16 of
              tests/golden/lib16_opls_s4.npz and 240 spliced as above),
              Langevin 1 fs, gamma 1/ps, 300 K, Rc 12 A, list every 10 steps,
              all systems in one CUDA-graph step loop; aggregate ns/day against
              one system alone.
  lcpo        the headline system with the LCPO surface-area term added
              (FF_SASA_LCPO, GlobalASP 0.005 kcal/mol/A^2, UpdateSasa 5):
              parity against the reference, the device time of the term's
              two launches against the nominal FP64 roof, and MD ns/day with
              the term (same protocol as the headline).
  serving     a seeded Poisson request stream (200 requests/s) of jobs on
              systems of 500-30,000 atoms (log-uniform; multi-chain systems
              composed from the AMBER99 library peptides, chain axes along z
              on a 25 A grid): 60% single-point, 30% 200-step steepest-descent
              minimisation, 10% 2,000-step Langevin MD at 1 fs, Rc 12 A,
              through the request loop with a 120 GB HBM budget; p50/p99
              latency and jobs/s beside the plain sequential GPU path (the
              same jobs one after another through the plain calls).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU: independent replicas, one per rank (the path does not shard one
system); value = simulated ns of all ranks / the slowest rank's time.
"""
import argparse
import ctypes
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(ROOT, "tests", "golden", "c2_16x80_s2.npz")
LIB_SP = os.path.join(ROOT, "tests", "golden", "lib16_amber_s3.npz")
LIB_MD = os.path.join(ROOT, "tests", "golden", "lib16_opls_s4.npz")
REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver_timing")
REF_PARAM = os.path.join(ROOT, "oracle", "_ref", "param")
DT_FS = 1.0
BLOCK = 10  # list period = one timed iteration (L2 flushed between them)
METRIC = "GB MD ns/day"
# DRAM bytes (read + write) of one evaluation (the evaluation kernel's three
# one-phase launches of one MD step) on this workload, from one ncu capture
# of the 20,566-atom MD workload (dram__bytes_read.sum + dram__bytes_write.sum,
# cold caches: 1,924,864 + 3,327,488 + 3,181,312 bytes read, nothing written);
# ncu cannot run inside the timed bench, so the figure is carried here
NCU_TRAFFIC_EVAL = 8433664
# warp instructions the same three launches executed (smsp__inst_executed.sum
# of that capture: phases A, B, C), for the issue roof beside the FP32/SFU one
NCU_INST_EVAL = (5630203, 14581779, 6049203)


def rank_info():
    r = int(os.environ.get("RANK", "0"))
    w = int(os.environ.get("WORLD_SIZE", "1"))
    lr = int(os.environ.get("LOCAL_RANK", str(r)))
    return r, w, lr


def check_world(gpus, world):
    """The number of GPUs the job runs on: the ranks the launcher started.
    Each rank is one replica on its own GPU, so asking for more GPUs than
    there are ranks would count work nobody did; that is refused."""
    if gpus > world:
        raise SystemExit("bench.py: --gpus %d needs %d ranks (one process per GPU): launch it with "
                         "python -m torch.distributed.run --nproc-per-node %d bench.py --gpus %d "
                         "(WORLD_SIZE is %d)" % (gpus, gpus, gpus, gpus, world))
    return world


def warmup_plan(warmup, steps, block=BLOCK):
    """Warm-up blocks of the headline MD run: at least max(3, warmup) steps,
    rounded up to whole list periods so the timed region starts on a period
    boundary, plus (when the timed steps end inside a period) one partial
    period and the rest of it, so every step-block graph the timed region
    replays is captured before it starts.  Returns the block lengths."""
    w = max(3, warmup)
    plan = [block] * ((w + block - 1) // block)
    tail = steps % block
    if tail:
        plan += [tail, block - tail]
    return plan


def headline_config(n_atoms, n_gpus):
    """The workload description both arms print (same keys, same values)."""
    return {"workload": "16x80-residue chains, 20566 atoms, AMBER99 + Still GB + bonded, Rc 16 A, "
                        "Langevin 1 fs 300 K gamma 1/ps, list every 10 steps",
            "atoms": n_atoms, "forcefield": "amber99aa: FF_Bonded + FF_GeneralizedBorn_Still (FastMode)",
            "parallelism": "replicas" if n_gpus > 1 else "single",
            "l2": "flushed (256 MiB write) before every 10-step timed block"}


def max_over_ranks(value, dist, device):
    """The largest of the ranks' values, on every rank (the value itself
    without a process group).  Replicas: each rank times its own copy of the
    workload and the job takes as long as the slowest."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_ns_per_day(n_ranks, steps_per_rank, seconds):
    """Aggregate simulated time of all replicas per day of wall time."""
    return n_ranks * steps_per_rank * DT_FS * 1e-6 / seconds * 86400.0


def load_fixture():
    z = np.load(FIXTURE)
    arrays = {k: z[k] for k in z.files}
    meta = json.loads(bytes(arrays.pop("meta_json")).decode())
    return arrays, meta


def load_library(path):
    z = np.load(path)
    meta = json.loads(bytes(z["meta_json"]).decode())
    out = []
    for k, m in enumerate(meta["members"]):
        pre = "p%02d_" % k
        out.append(({f[len(pre):]: z[f] for f in z.files if f.startswith(pre)}, m))
    return out


def make_ws(pdgpu, arrays, meta, ctx):
    """WorkSpace + {FF_Bonded, FF_GeneralizedBorn_Still} at the fixture's cutoffs."""
    ws = pdgpu.WorkSpace(pdgpu.SystemSpec(arrays, meta), ctx)
    ff = pdgpu.Forcefield(ws)
    ff.add(pdgpu.FF_Bonded(ws))
    gb = pdgpu.FF_GeneralizedBorn_Still(ws)
    gb.Cutoff, gb.InnerCutoff = float(meta["cutoff"]), float(meta["inner"])
    gb.VdwCutoff, gb.VdwInnerCutoff = float(meta["vdwcut"]), float(meta["vdwinner"])
    ff.add(gb)
    ff.ensuresetup()
    return ws, ff


def spliced_members(pdgpu, A, ctx, lib, lengths, seed, premin=500):
    """Distinct seeded peptides of the given lengths, spliced from the
    library's reference-built residue templates (pdgpu.peptides) and relaxed
    with `premin` steepest-descent steps of the device minimiser (all of them
    as one batch).  Returns (ws, ff, arrays, meta) per peptide and the
    seconds the splicing and the minimisation took."""
    from pdgpu.peptides import ResidueLibrary
    t0 = time.perf_counter()
    R = ResidueLibrary(lib)
    rng = np.random.default_rng(seed)
    out = []
    for nres in lengths:
        seq = R.draw_sequence(rng, int(nres))
        arrays = R.build(seq)
        meta = dict(lib[0][1], chain=[seq], natoms=str(len(arrays["charge"])), premin=str(premin),
                    seed=str(seed), spliced="1")
        ws, ff = make_ws(pdgpu, arrays, meta, ctx)
        out.append((ws, ff, arrays, meta))
    t_build = time.perf_counter() - t0
    b = pdgpu.Batch([ws for ws, *_ in out])
    mp = A.min_params_default()
    mp.Algorithm = A.MIN_STEEPEST_DESCENT
    taken = b.minimise(mp, premin)
    if np.any(taken < 0):
        raise RuntimeError("a spliced peptide's energy turned NaN during its relaxation")
    for (ws, ff, arrays, meta), pos in zip(out, b.split(b.positions())):
        arrays["pos"] = pos.copy()
        ws.cur.p[:] = pos
        ws._push_positions()
    b.close()
    return out, {"splice_s": t_build, "minimise_s": time.perf_counter() - t0 - t_build, "premin_sd_steps": premin}


def eval_roofline(A, ctx, sid, peaks):
    """The evaluation kernel's FP32/SFU roofline fraction on handle `sid`
    (a system or a batch on the tile layout; None otherwise): the same work
    counts and measured peaks as the headline's, over the three one-phase
    launches and over the cooperative launch."""
    L = A.lib()
    if peaks is None or L.pdgpu_pair_path(ctx.ptr, sid, -2, None) != 0:
        return None
    cur = ctypes.c_int32(0)
    A.check(L.pdgpu_pair_path(ctx.ptr, sid, -2, ctypes.byref(cur)))
    if cur.value != 1:
        return None
    counts = np.zeros(5, dtype=np.int64)
    A.check(L.pdgpu_pair_counts(ctx.ptr, sid, counts.ctypes.data_as(A._I64)))
    ems = np.zeros(4)
    A.check(L.pdgpu_profile_eval(ctx.ptr, sid, 10, A.dptr(ems), None))
    P_B, P_H, entries, held, tiles = (int(c) for c in counts)
    F32, SFU = peaks
    t_roof = max((57.0 * P_B + 90.0 * P_H) / F32, (7.0 * P_B + 5.0 * P_H) / SFU)
    t3, t1 = sum(float(x) for x in ems[:3]) / 1e3, float(ems[3]) / 1e3
    return {"frac": t_roof / t3, "frac_one_cooperative_launch": t_roof / t1,
            "kernel_ms": {"three_launches": 1e3 * t3, "one_cooperative_launch": 1e3 * t1},
            "pairs": {"P_B": P_B, "P_H": P_H}, "tiles": tiles,
            "slot_occupancy": held / max(1, 256 * tiles)}


def pctl(xs, q):
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else None


# ---------------------------------------------------------------- batched workloads
def bench_batched_sp(pdgpu, A, ctx, torch, n_systems=512, trials=64, plain_trials=2, peaks=None):
    """Batched single-point evaluations of Monte Carlo trial conformations."""
    lib = load_library(LIB_SP)
    L = A.lib()
    sigma = np.deg2rad(15.0)
    members = []
    for k, (a, m) in enumerate(lib):
        ws, ff = make_ws(pdgpu, a, m, ctx)
        members.append((ws, ff, a, m))
    # the other peptides: lengths log-uniform in 20-200 residues (seeded)
    rng = np.random.default_rng(3003)
    lens = np.floor(np.exp(rng.uniform(np.log(20), np.log(200), n_systems - len(lib)))).astype(int)
    extra, prep = spliced_members(pdgpu, A, ctx, lib, lens, seed=3004)
    members += extra
    members = [(ws, ff, a, m, s) for s, (ws, ff, a, m) in enumerate(members)]
    for ws, *_ in members:
        ws.setTorsionMoves()
    nsys = len(members)
    b = pdgpu.Batch([ws for ws, *_ in members])
    b.setSeeds(np.array([1_000_003 * (s + 1) for *_, s in members], dtype=np.uint64))
    b.saveBasePositions()
    # parity: the reference's first recorded trial of every peptide
    ang = [a["trial_angles"][0] if "trial_angles" in a else np.zeros(ws.nRotations) for ws, ff, a, m, s in members]
    b.perturbTorsions(angles=ang)
    f, e = b.evaluate()
    worst = 0.0
    for s, (ws, ff, a, m, _) in enumerate(members[:len(lib)]):
        fs = b.split(f)[s]
        ref = a["trial_f"][0]
        worst = max(worst, float(np.sqrt(np.sum((fs - ref) ** 2) / np.sum(ref ** 2))))
    roof = eval_roofline(A, ctx, b._id, peaks)
    lat = []
    lc0 = ctypes.c_int64(0)
    L.pdgpu_launch_count(ctx.ptr, ctypes.byref(lc0))
    torch.cuda.synchronize()
    t_wall = time.perf_counter()
    for t in range(trials):
        t0 = time.perf_counter()
        b.perturbTorsions(sigma=sigma, trial=t)
        b.calcNewList()
        b.calcForces()
        e = b.energies()
        lat.append(time.perf_counter() - t0)
    t_all = time.perf_counter() - t_wall
    lc1 = ctypes.c_int64(0)
    L.pdgpu_launch_count(ctx.ptr, ctypes.byref(lc1))
    evals = nsys * trials
    # the whole Monte Carlo protocol on the device (moves, list, forces,
    # Metropolis at 300 K per system; one host read per 16 steps)
    b.setPositions(b.positions())
    torch.cuda.synchronize()
    t_mc = time.perf_counter()
    acc, low = b.runMC(trials, temperature=300.0, sigma=sigma)
    t_mc = time.perf_counter() - t_mc
    mc = {"metric": "device Monte Carlo evals/s (pdgpu_mc_run)", "value": nsys * trials / t_mc, "unit": "evals/s",
          "steps": trials, "acceptance": float(acc.sum()) / (nsys * trials),
          "device_ms": ctx.last_run_ms(), "timing": "wall clock around the call"}
    # plain path: one system per launch sequence (perturb, list, forces,
    # read); an untimed first evaluation per system tunes its kernels
    plain = []
    torch.cuda.synchronize()
    t_plain = 0.0
    n_plain = 0
    for ws, ff, a, m, s in members:
        sid = ws._sys
        A.check(L.pdgpu_save_base_positions(ctx.ptr, sid))
        A.check(L.pdgpu_nlist_build(ctx.ptr, sid))
        A.check(L.pdgpu_calc_forces(ctx.ptr, sid))
        for t in range(plain_trials):
            t0 = time.perf_counter()
            A.check(L.pdgpu_perturb_torsions(ctx.ptr, sid, sigma, t, None))
            A.check(L.pdgpu_nlist_build(ctx.ptr, sid))
            A.check(L.pdgpu_calc_forces(ctx.ptr, sid))
            ebuf = np.zeros(A.ENE_COUNT)
            A.check(L.pdgpu_get_energies(ctx.ptr, sid, A.dptr(ebuf), A.ENE_COUNT))
            plain.append(time.perf_counter() - t0)
            t_plain += plain[-1]
            n_plain += 1
    atoms = int(b.nAtoms)
    b.close()
    for ws, *_ in members:
        ws.close()
    # the CPU baseline: the reference's list rebuild + calcForces on every
    # library peptide, one process per host core
    cpu = None
    if os.path.exists(REF_DRIVER):
        cores = host_cores()
        jobs = []
        for a, m in lib:
            nat = a["charge"].shape[0]
            k = int(max(3, min(60, 0.8 / (2.7e-3 * (nat / 1000.0) ** 2 + 5e-4))))
            jobs.append((a, m, "evals", ["--steps", k, "--warmup", 1]))
        res, wall = run_ref_jobs(jobs, cores)
        t = [r["seconds"] / r["evals"] for r in res if r]
        if t:
            v = cores / float(np.mean(t))
            cpu = {"value": v, "unit": "evals/s", "cores": cores, "kind": "reference",
                   "sample": "NeighbourList::calcNewList + Forcefield::calcForces of each of the %d library peptides "
                             "(3-60 evaluations each), concurrent processes on %d cores; aggregate = cores / mean "
                             "evaluation time" % (len(t), cores)}
    return {"metric": "batched GB evals/s", "value": evals / t_all, "unit": "evals/s", "cpu_baseline": cpu,
            "evals": evals, "systems": nsys, "trials_per_system": trials, "atoms_packed": atoms,
            "systems_made": dict(prep, reference_built=len(lib), spliced=nsys - len(lib),
                                 how="16 library peptides built by the reference's NewProtein, and distinct seeded "
                                     "peptides (lengths log-uniform 20-200 residues) spliced from their residue "
                                     "templates and relaxed by the device minimiser"),
            "batch_latency_ms": {"p50": 1e3 * pctl(lat, 50), "p99": 1e3 * pctl(lat, 99)},
            "plain_one_system_per_launch": {"value": n_plain / t_plain, "unit": "evals/s", "sample_evals": n_plain,
                                            "latency_ms": {"p50": 1e3 * pctl(plain, 50), "p99": 1e3 * pctl(plain, 99)}},
            "speedup_vs_plain": (evals / t_all) / (n_plain / t_plain),
            "device_mc": dict(mc, speedup_vs_plain=(nsys * trials / t_mc) / (n_plain / t_plain)),
            "gpu_launches": int(lc1.value - lc0.value), "roofline": roof,
            "parity": {"force_rel_rms_vs_fp64_max": worst,
                       "case": "reference trial 0 of each of the 16 peptides, angles from the reference run"},
            "timing": "wall clock around perturb + list + forces + energies read-back, per batched evaluation"}


def bench_batched_md(pdgpu, A, ctx, torch, n_systems=256, steps=5000, plain_steps=200, drift_steps=1000,
                     peaks=None):
    """All systems advanced together in one CUDA-graph step loop."""
    lib = load_library(LIB_MD)
    L = A.lib()
    members = []
    for k, (a, m) in enumerate(lib):
        ws, ff = make_ws(pdgpu, a, m, ctx)
        members.append((ws, ff, a, m))
    # the other peptides: lengths uniform in 30-150 residues (seeded)
    lens = np.random.default_rng(4003).integers(30, 151, n_systems - len(lib))
    extra, prep = spliced_members(pdgpu, A, ctx, lib, lens, seed=4004)
    members += extra
    nsys = len(members)
    p = A.md_params_default()
    p.Integrator, p.UpdateNList, p.UseGraph = A.INTEGRATOR_LANGEVIN, 10, 1
    p.Timestep, p.FricCoeff, p.TargetTemp, p.Seed = 1e-15, 1e12, 300.0, 77
    b = pdgpu.Batch([ws for ws, *_ in members])
    b.calcNewList()
    total = steps + 20
    A.check(L.pdgpu_md_init_velocities(ctx.ptr, b._id, 300.0, 77))
    hist = np.zeros(3 * 20 * nsys)
    A.check(L.pdgpu_md_run(ctx.ptr, b._id, ctypes.byref(p), 0, 20, total, A.dptr(hist)))  # warm-up + graph
    lc0 = ctypes.c_int64(0)
    L.pdgpu_launch_count(ctx.ptr, ctypes.byref(lc0))
    hist = np.zeros(3 * steps * nsys)
    A.check(L.pdgpu_md_run(ctx.ptr, b._id, ctypes.byref(p), 20, steps, total, A.dptr(hist)))
    ms = ctx.last_run_ms()
    lc1 = ctypes.c_int64(0)
    L.pdgpu_launch_count(ctx.ptr, ctypes.byref(lc1))
    roof = eval_roofline(A, ctx, b._id, peaks)  # after the run: its launches are not counted
    h = hist.reshape(steps, nsys, 3) * pdgpu.J2KCAL_NA
    nat = np.diff(b.offsets)
    ek_per_atom = h[-100:, :, 1].mean(axis=0) / nat  # kcal/mol per atom
    t_kin = ek_per_atom / (1.5 * 0.0019872041)        # K
    agg = nsys * steps * 1e-6 / (ms / 1e3) * 86400.0
    # one system alone (the plain path), the median-sized peptide
    order = np.argsort([a["charge"].shape[0] for ws, ff, a, m in members[:len(lib)]])
    ws, ff, a, m = members[int(order[len(order) // 2])]
    one = pdgpu.Batch([ws])
    one.calcNewList()
    A.check(L.pdgpu_md_init_velocities(ctx.ptr, one._id, 300.0, 78))
    A.check(L.pdgpu_md_run(ctx.ptr, one._id, ctypes.byref(p), 0, 20, plain_steps + 20, None))
    A.check(L.pdgpu_md_run(ctx.ptr, one._id, ctypes.byref(p), 20, plain_steps, plain_steps + 20, None))
    ms1 = ctx.last_run_ms()
    one_nsday = plain_steps * 1e-6 / (ms1 / 1e3) * 86400.0
    atoms = int(b.nAtoms)
    one.close()
    b.close()
    for ws, *_ in members:
        ws.close()
    # per-system total-energy drift (the reference's least-squares slope,
    # md.cpp:182-189, 236-240) over the timed steps, and beside it the
    # reference's own FP64 MD on a sample of members (same start, its own
    # random draws: the two drifts agree statistically, not step by step)
    abs_steps = np.arange(20, 20 + steps)
    drifts = np.array([ls_drift(abs_steps, h[:, s, 2], total) for s in range(nsys)], dtype=np.float64)
    drift = {"unit": "kcal/mol per 1000 steps",
             "gpu_all_systems": {"median": float(np.median(drifts)), "p10": float(np.percentile(drifts, 10)),
                                 "p90": float(np.percentile(drifts, 90)),
                                 "median_abs": float(np.median(np.abs(drifts)))},
             "method": "least-squares slope of etot sampled every max(1, Steps/1000) steps after step 50 "
                       "(MolecularDynamics::run_core)"}
    cpu = None
    if os.path.exists(REF_DRIVER):
        cores = host_cores()
        sample = list(range(min(len(lib), 2)))
        opls = [(a, dict(m, param="oplsaal.ff")) for a, m in lib]
        jobs = [(opls[k][0], opls[k][1], "time", ["--steps", drift_steps, "--warmup", 0, "--nlist-every", 10,
                                                   "--drift"]) for k in sample]
        jobs += [(a, m, "time", ["--steps", 30, "--warmup", 10, "--nlist-every", 10]) for a, m in opls]
        res, wall = run_ref_jobs(jobs, cores)
        rows = []
        for k, r in zip(sample, res[:len(sample)]):
            if not r:
                continue
            hk = hist.reshape(steps, nsys, 3)[:drift_steps - 20, k, 2] * pdgpu.J2KCAL_NA
            rows.append({"member": k, "atoms": int(r["natoms"]), "reference": r.get("drift_kcal_per_1000"),
                         "gpu": ls_drift(np.arange(20, drift_steps), hk, drift_steps)})
        drift["vs_reference"] = rows
        drift["reference_sample"] = ("%d Langevin steps (1/ps, 300 K) of members %s from the fixture coordinates; the "
                                     "GPU figure is the same member's steps 20-%d of the batched run"
                                     % (drift_steps, sample, drift_steps))
        # the CPU baseline: one reference process per host core; each of the
        # 16 library members timed over 30 MD steps, and a core advancing
        # the library's mix at the mean step time
        t = [r["seconds"] / 30 for r in res[len(sample):] if r]
        if t:
            cpu = {"value": cores * DT_FS * 1e-6 / float(np.mean(t)) * 86400.0, "unit": "ns/day", "cores": cores,
                   "kind": "reference",
                   "sample": "30 reference MD steps (after 10) of each of the %d OPLS-AA library members, run as "
                             "concurrent processes on %d cores; aggregate = cores x 1 fs / mean step time" % (len(t),
                                                                                                        cores)}
    return {"metric": "batched GB MD aggregate ns/day", "value": agg, "unit": "ns/day", "systems": nsys,
            "drift": drift, "cpu_baseline": cpu, "roofline": roof,
            "systems_made": dict(prep, reference_built=len(lib), spliced=nsys - len(lib),
                                 how="16 library peptides built by the reference's NewProtein, and distinct seeded "
                                     "peptides (lengths uniform 30-150 residues) spliced from their residue templates "
                                     "and relaxed by the device minimiser"),
            "steps": steps, "atoms_packed": atoms, "ms_per_step": ms / steps,
            "plain_one_system": {"value": one_nsday, "unit": "ns/day", "atoms": int(a["charge"].shape[0]),
                                 "steps": plain_steps},
            "speedup_vs_plain_sequential": agg / one_nsday,
            "kinetic_temperature_K": {"median": float(np.median(t_kin)), "min": float(t_kin.min()),
                                      "max": float(t_kin.max())},
            "finite": bool(np.all(np.isfinite(h))),
            "gpu_launches": int(lc1.value - lc0.value),
            "timing": "CUDA events around the device step loop (pdgpu_last_run_ms)"}


def bench_plain_small(pdgpu, A, ctx, torch, steps=1000, cpu_steps=200):
    """The plain small method: one seeded 64-residue peptide (1,001 atoms,
    tests/golden/c1_pep64_s0.npz), AMBER99 + Still GB + bonded, Rc 12 A, list
    every 10 steps, Langevin at 1 fs and 300 K with the reference's default
    friction (1e13 /s), 1,000 steps; beside it the reference's own CPU MD on
    one core (a bounded sample)."""
    L = A.lib()
    path = os.path.join(ROOT, "tests", "golden", "c1_pep64_s0.npz")
    z = np.load(path)
    arrays = {k: z[k] for k in z.files}
    meta = json.loads(bytes(arrays.pop("meta_json")).decode())
    ws, ff = make_ws(pdgpu, arrays, meta, ctx)
    n = ws.nAtoms()
    ws.nlist().calcNewList()
    ff.calcForces()
    f_rms = float(np.sqrt(np.sum((ws.cur.f - arrays["f_total"]) ** 2) / np.sum(arrays["f_total"] ** 2)))
    de = float(abs(ws.ene.epot - arrays["ene_total"][0]) * pdgpu.J2KCAL_NA)
    p = A.md_params_default()
    p.Integrator, p.UpdateNList, p.UseGraph = A.INTEGRATOR_LANGEVIN, BLOCK, 1
    p.Timestep, p.FricCoeff, p.TargetTemp, p.Seed = 1e-15, 1e13, 300.0, 0
    A.check(L.pdgpu_md_init_velocities(ctx.ptr, ws._sys, 300.0, 0))
    total = steps + 2 * BLOCK
    A.check(L.pdgpu_md_run(ctx.ptr, ws._sys, ctypes.byref(p), 0, 2 * BLOCK, total, None))  # warm-up + graphs
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    hist = np.zeros(3 * steps)
    A.check(L.pdgpu_md_run(ctx.ptr, ws._sys, ctypes.byref(p), 2 * BLOCK, steps, total, A.dptr(hist)))
    wall = time.perf_counter() - t0
    ms = ctx.last_run_ms()
    h = hist.reshape(steps, 3) * pdgpu.J2KCAL_NA
    nsday = steps * DT_FS * 1e-6 / (ms / 1e3) * 86400.0
    out = {"metric": "GB MD ns/day", "value": nsday, "unit": "ns/day", "atoms": n, "steps": steps,
           "ms_per_step": ms / steps,
           "wall_clock_ns_per_day": steps * DT_FS * 1e-6 / wall * 86400.0,
           "parity": {"force_rel_rms_vs_fp64": f_rms, "epot_abs_err_kcal": de},
           "finite": bool(np.all(np.isfinite(h))),
           "drift_kcal_per_1000_steps": ls_drift(np.arange(2 * BLOCK, 2 * BLOCK + steps), h[:, 2], total),
           "workload": "64-residue peptide, AMBER99 + Still GB + bonded, Rc 12 A, Langevin 1 fs 300 K, "
                       "friction 1e13/s, list every 10 steps",
           "timing": "CUDA events around the device step loop (pdgpu_last_run_ms)"}
    # energy conservation without a thermostat (a friction of 1e3 /s: gamma dt
    # is below 1e-5, where both codes run velocity Verlet: the Langevin
    # integrator's fallback, md.cpp:906-1042) from
    # the fixture's coordinates at 300 K, against the
    # reference's own run of the same length (its own initial velocities:
    # the drifts agree statistically, not step by step)
    ws2, _ = make_ws(pdgpu, arrays, meta, ctx)
    ws2.nlist().calcNewList()
    q = A.md_params_default()
    q.Integrator, q.UpdateNList, q.UseGraph = A.INTEGRATOR_LANGEVIN, BLOCK, 1
    q.Timestep, q.FricCoeff, q.TargetTemp, q.Seed = 1e-15, 1e3, 300.0, 0
    A.check(L.pdgpu_md_init_velocities(ctx.ptr, ws2._sys, 300.0, 0))
    hv = np.zeros(3 * steps)
    A.check(L.pdgpu_md_run(ctx.ptr, ws2._sys, ctypes.byref(q), 0, steps, steps, A.dptr(hv)))
    ws2.close()
    hv = hv.reshape(steps, 3) * pdgpu.J2KCAL_NA
    out["nve_drift"] = {"unit": "kcal/mol per 1000 steps", "steps": steps,
                        "gpu": ls_drift(np.arange(steps), hv[:, 2], steps),
                        "etot_start_kcal": float(hv[0, 2]),
                        "method": "least-squares slope of etot (MolecularDynamics::run_core), velocity Verlet "
                                  "(Langevin at 1e3 /s falls back to it), 1 fs, list every 10 steps, initial "
                                  "velocities at 300 K"}
    if os.path.exists(REF_DRIVER):
        jobs = [(arrays, meta, "time", ["--steps", cpu_steps, "--warmup", 10, "--nlist-every", 10, "--fric", "1e13"]),
                (arrays, meta, "time", ["--steps", steps, "--warmup", 0, "--nlist-every", 10, "--fric", "1e3",
                                        "--drift"])]
        res, _ = run_ref_jobs(jobs, 2)
        if res[0]:
            v = cpu_steps * DT_FS * 1e-6 / res[0]["seconds"] * 86400.0
            out["cpu_baseline"] = {"value": v, "unit": "ns/day", "cores": 1, "kind": "reference",
                                   "sample": "%d MD steps after 10 warm-up, reference MolecularDynamics step loop"
                                             % cpu_steps}
            out["speedup_vs_cpu"] = nsday / v
        if res[1]:
            out["nve_drift"]["reference"] = res[1].get("drift_kcal_per_1000")
    return out


# FP64 operations of one (atom, partner, partner's partner) triple of the
# LCPO inner loop (lcpo.cpp:823-872, sqrt and divide counted as one each):
# the full body when the third atom overlaps the first, else the distance
# test alone
LCPO_FLOP_OVERLAP = 58
LCPO_FLOP_TEST = 10


def bench_lcpo(pdgpu, A, ctx, torch, arrays, meta, f_max, sms, steps=500):
    """FF_SASA_LCPO on the headline system."""
    L = A.lib()
    ws = pdgpu.WorkSpace(pdgpu.SystemSpec(arrays, meta), ctx)
    ff = pdgpu.Forcefield(ws)
    ff.add(pdgpu.FF_Bonded(ws))
    gb = pdgpu.FF_GeneralizedBorn_Still(ws)
    gb.Cutoff, gb.InnerCutoff = float(meta["cutoff"]), float(meta["inner"])
    gb.VdwCutoff, gb.VdwInnerCutoff = float(meta["vdwcut"]), float(meta["vdwinner"])
    ff.add(gb)
    sasa = pdgpu.FF_SASA_LCPO(ws)
    sasa.GlobalASP = float(arrays["lcpo_cfg"][0])
    sasa.UpdateSasa = 5
    ff.add(sasa)
    ws.nlist().calcNewList()
    ff.calcForces()
    f_ref = arrays["lcpo_f_total"]
    rms = float(np.sqrt(np.sum((ws.cur.f - f_ref) ** 2) / np.sum(f_ref ** 2)))
    esurf_rel = float(abs(ws.ene.epot_surf - arrays["lcpo_ene_total"][10]) / abs(arrays["lcpo_ene_total"][10]))
    prof = np.zeros(5)
    A.check(L.pdgpu_profile_lcpo(ctx.ptr, ws._sys, 20, A.dptr(prof)))
    t_list, t_eval = prof[0] / 1e3, prof[1] / 1e3
    pairs, triples, overl = prof[2], prof[3], prof[4]
    flop = LCPO_FLOP_OVERLAP * overl + LCPO_FLOP_TEST * (triples - overl)
    f64_peak = sms * 128 * f_max  # 64 FP64 FMA per SM per clock
    # MD with the term: the headline protocol
    p = A.md_params_default()
    p.Integrator, p.UpdateNList, p.UseGraph = A.INTEGRATOR_LANGEVIN, BLOCK, 1
    p.Timestep, p.FricCoeff, p.TargetTemp, p.Seed = 1e-15, 1e12, 300.0, 5
    A.check(L.pdgpu_md_init_velocities(ctx.ptr, ws._sys, 300.0, 5))
    total = steps + 20
    A.check(L.pdgpu_md_run(ctx.ptr, ws._sys, ctypes.byref(p), 0, 20, total, None))
    lc0 = ctypes.c_int64(0)
    L.pdgpu_launch_count(ctx.ptr, ctypes.byref(lc0))
    A.check(L.pdgpu_md_run(ctx.ptr, ws._sys, ctypes.byref(p), 20, steps, total, None))
    ms = ctx.last_run_ms()
    lc1 = ctypes.c_int64(0)
    L.pdgpu_launch_count(ctx.ptr, ctypes.byref(lc1))
    ws.close()
    return {"metric": "GB/SA (LCPO) MD ns/day", "value": steps * DT_FS * 1e-6 / (ms / 1e3) * 86400.0,
            "unit": "ns/day", "steps": steps, "ms_per_step": ms / steps,
            "gpu_launches": int(lc1.value - lc0.value),
            "parity": {"force_rel_rms_vs_fp64": rms, "epot_surf_rel_err": esurf_rel},
            "kernels": {"k_lcpo_list_ms": t_list * 1e3, "k_lcpo_eval_ms": t_eval * 1e3,
                        "overlap_partners": int(pairs), "inner_triples": int(triples),
                        "overlapping_triples": int(overl)},
            "roofline": {"kernel": "k_lcpo_eval (areas and derivatives, FP64)", "bound": "fp64",
                         "achieved": flop / t_eval / 1e12, "peak": f64_peak / 1e12, "unit": "TFLOP/s",
                         "frac": flop / t_eval / f64_peak,
                         "peak_source": "nominal %d SMs x 128 FP64 flop/clk at sm_max_mhz %.0f" % (
                             sms, f_max / 1e6),
                         "work": "%d flop per overlapping triple, %d per distance test" % (
                             LCPO_FLOP_OVERLAP, LCPO_FLOP_TEST)},
            "amortised_ms_per_step": (t_list + t_eval) * 1e3 / 5}


# ---------------------------------------------------------------- serving
PER_ATOM = ("charge", "radius", "epsilon", "mass", "gb_radius", "is_h")


def compose(parts, spacing=25.0):
    """One multi-chain system from several library peptides: per-atom arrays
    concatenated, index arrays shifted, each chain's principal axis turned
    onto z and the chains set on a square grid `spacing` apart in x-y."""
    out = {k: [] for k in PER_ATOM + ("ir", "pos", "cov12_d", "cov13_d", "bond_lk", "angle_kt", "tors_terms",
                                      "tors_par", "impr_terms", "impr_par", "backbone_ncac", "bond_ij",
                                      "angle_iaj", "tors_idx", "impr_idx")}
    csr = {k: ([0], []) for k in ("cov12", "cov13", "cov14")}
    g = int(np.ceil(np.sqrt(len(parts))))
    off = 0
    res_off = 0
    for k, a in enumerate(parts):
        n = a["charge"].shape[0]
        for f in PER_ATOM:
            out[f].append(a[f])
        out["ir"].append(a["ir"] + res_off)
        p = a["pos"] - a["pos"].mean(axis=0)
        _, _, vt = np.linalg.svd(p, full_matrices=False)
        ax = vt[0]
        # rotation taking the principal axis onto z
        z = np.array([0.0, 0.0, 1.0])
        v = np.cross(ax, z)
        c = float(np.dot(ax, z))
        if np.linalg.norm(v) < 1e-12:
            R = np.eye(3) if c > 0 else np.diag([1.0, -1.0, -1.0])
        else:
            vx = np.array([[0, -v[2], v[1]], [v[2], 0, -v[0]], [-v[1], v[0], 0]])
            R = np.eye(3) + vx + vx @ vx * (1.0 / (1.0 + c))
        out["pos"].append(p @ R.T + np.array([(k % g) * spacing, (k // g) * spacing, 0.0]))
        for name in ("cov12", "cov13", "cov14"):
            ptr, idx = csr[name]
            ptr.extend((a[name + "_ptr"][1:] + ptr[-1]).tolist())
            idx.append(a[name + "_idx"] + off)
        out["cov12_d"].append(a["cov12_d"])
        out["cov13_d"].append(a["cov13_d"])
        for f in ("bond_ij", "angle_iaj", "tors_idx", "impr_idx"):
            out[f].append(a[f] + off)
        for f in ("bond_lk", "angle_kt", "tors_terms", "tors_par", "impr_terms", "impr_par"):
            out[f].append(a[f])
        bb = a["backbone_ncac"].copy()
        out["backbone_ncac"].append(np.where(bb >= 0, bb + off, -1))
        off += n
        res_off += int(a["ir"].max()) + 1
    res = {k: np.concatenate(v) for k, v in out.items()}
    for name in ("cov12", "cov13", "cov14"):
        ptr, idx = csr[name]
        res[name + "_ptr"] = np.asarray(ptr, dtype=np.int32)
        res[name + "_idx"] = np.concatenate(idx).astype(np.int32)
    res["ff_params"] = parts[0]["ff_params"]
    return res


def bench_serving(pdgpu, A, ctx, torch, n_requests=300, rate=200.0, budget=120e9, max_active=16, seed=5,
                  policy=1, tiles=True, batch_ms=60):
    lib = load_library(LIB_SP)
    meta = lib[0][1]
    rng = np.random.default_rng(seed)
    # templates: sizes log-uniform in [500, 30000]
    n_tmpl = 24
    targets = np.exp(np.linspace(np.log(500), np.log(30000), n_tmpl))
    templates, tmpl_inputs = [], []
    for t in targets:
        parts, tot = [], 0
        while tot < 0.9 * t:
            a, am = lib[int(rng.integers(len(lib)))]
            if parts and tot + a["charge"].shape[0] > 1.15 * t:
                cand = [(x, xm) for x, xm in lib if tot + x["charge"].shape[0] <= 1.15 * t]
                if not cand:
                    break
                a, am = cand[int(rng.integers(len(cand)))]
            parts.append((a, am))
            tot += a["charge"].shape[0]
        arrays = compose([a for a, _ in parts])
        ws, ff = make_ws(pdgpu, arrays, meta, ctx)
        ws.setLanes((8, 8, 8))
        templates.append(ws)
        # the template for the reference driver: its chains and coordinates
        chains = [c for _, am in parts for c in (am["chain"] if isinstance(am["chain"], list) else [am["chain"]])]
        tmpl_inputs.append(({"pos": arrays["pos"]}, dict(meta, chains=chains)))
    sizes = np.array([ws.nAtoms() for ws in templates])
    # the request stream
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    want = np.exp(rng.uniform(np.log(500), np.log(30000), n_requests))
    tmpl = [int(np.argmin(np.abs(np.log(sizes) - np.log(w)))) for w in want]
    u = rng.uniform(size=n_requests)
    kinds = np.where(u < 0.6, A.JOB_ENERGY, np.where(u < 0.9, A.JOB_MINIMISE, A.JOB_MD))
    md = A.md_params_default()
    md.Integrator, md.UpdateNList, md.UseGraph = A.INTEGRATOR_LANGEVIN, 10, 1
    md.Timestep, md.FricCoeff, md.TargetTemp = 1e-15, 1e12, 300.0
    mn = A.min_params_default()
    mn.Algorithm = A.MIN_STEEPEST_DESCENT
    S = pdgpu.Server
    jobs = []
    for k in range(n_requests):
        if kinds[k] == A.JOB_ENERGY:
            jobs.append(S.job(S.ENERGY))
        elif kinds[k] == A.JOB_MINIMISE:
            jobs.append(S.job(S.MINIMISE, 200, minimiser=mn))
        else:
            m = A.md_params_default()
            for name, _ in A.MDParams._fields_:
                setattr(m, name, getattr(md, name))
            m.Seed = 1000 + k
            jobs.append(S.job(S.MD, 2000, md=m, init_temp=300.0))
    L = A.lib()
    # served: submit at the arrival times, the worker overlaps the jobs
    srv = pdgpu.Server(ctx, hbm_budget=budget, max_active=max_active, lanes=(8, 8, 8), tiles=tiles,
                       policy=policy, batch_ms=batch_ms)
    lc0 = L_count(L, ctx)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ids = []
    for k in range(n_requests):
        while time.perf_counter() - t0 < arrivals[k]:
            time.sleep(min(2e-4, max(0.0, arrivals[k] - (time.perf_counter() - t0))))
        ids.append(srv.submit(templates[tmpl[k]], jobs[k]))
    for jid in ids:
        A.check(srv.wait(jid, 600.0))
    makespan = time.perf_counter() - t0
    lc1 = L_count(L, ctx)
    lat = [srv.info(j)["t_total_ms"] for j in ids]
    st = srv.stats()
    for jid in ids:
        srv.release(jid)
    srv.close()
    by_kind = {}
    for k, name in ((A.JOB_ENERGY, "energy"), (A.JOB_MINIMISE, "minimise_200"), (A.JOB_MD, "md_2000")):
        sel = [lat[i] for i in range(n_requests) if kinds[i] == k]
        by_kind[name] = {"count": len(sel), "p50_ms": pctl(sel, 50), "p99_ms": pctl(sel, 99)}
    # plain sequential path: the same jobs, one after another, plain calls
    ebuf = np.zeros(A.ENE_COUNT)
    plat = []
    t0 = time.perf_counter()
    for k in range(n_requests):
        now = time.perf_counter() - t0
        if now < arrivals[k]:
            time.sleep(arrivals[k] - now)
        ws = templates[tmpl[k]]
        sid = ws._sys
        A.check(L.pdgpu_set_positions(ctx.ptr, sid, A.dptr(A.cd(ws.cur.p))))
        j = jobs[k]
        if j.kind == A.JOB_ENERGY:
            A.check(L.pdgpu_nlist_build(ctx.ptr, sid))
            A.check(L.pdgpu_calc_forces(ctx.ptr, sid))
        elif j.kind == A.JOB_MINIMISE:
            taken = np.zeros(1, dtype=np.int32)
            A.check(L.pdgpu_minimise_run(ctx.ptr, sid, ctypes.byref(j.min), j.steps, A.iptr(taken)))
        else:
            A.check(L.pdgpu_md_init_velocities(ctx.ptr, sid, j.init_temp, j.md.Seed))
            A.check(L.pdgpu_md_run(ctx.ptr, sid, ctypes.byref(j.md), 0, j.steps, j.steps, None))
        A.check(L.pdgpu_get_energies(ctx.ptr, sid, A.dptr(ebuf), A.ENE_COUNT))
        plat.append(1e3 * ((time.perf_counter() - t0) - arrivals[k]))
    plain_makespan = time.perf_counter() - t0
    for ws in templates:
        ws.close()
    cpu = serving_cpu_estimate(tmpl_inputs, sizes, kinds, tmpl, A) if os.path.exists(REF_DRIVER) else None
    return {"metric": "served GB jobs/s", "value": n_requests / makespan, "unit": "jobs/s", "cpu_baseline": cpu,
            "requests": n_requests, "arrival_rate_per_s": rate,
            "latency_ms": {"p50": pctl(lat, 50), "p99": pctl(lat, 99)}, "by_kind": by_kind,
            "plain_sequential": {"value": n_requests / plain_makespan, "unit": "jobs/s",
                                 "latency_ms": {"p50": pctl(plat, 50), "p99": pctl(plat, 99)}},
            "speedup_jobs_per_s_vs_plain": (n_requests / makespan) / (n_requests / plain_makespan),
            "system_atoms": {"min": int(sizes.min()), "max": int(sizes.max()), "templates": n_tmpl},
            "hbm_budget_bytes": int(budget), "max_active": max_active, "batch_window_ms": batch_ms,
            "groups": st["groups"], "peak_active": st["peak_active"],
            "admission": "least work first" if policy == 1 else "arrival order",
            "pair_path": "tiles" if tiles else "rows (8 lanes per atom)",
            "device_max_connections": os.environ.get("CUDA_DEVICE_MAX_CONNECTIONS"),
            "peak_bytes": st["peak_bytes"], "failed": st["failed"], "gpu_launches": int(lc1 - lc0),
            "timing": "wall clock: latency = finish - arrival per job; jobs/s = requests / makespan"}


def serving_cpu_estimate(tmpl_inputs, sizes, kinds, tmpl, A):
    """The reference's CPU time for the served job stream, from timed
    samples: on the smallest, the median and the largest template, the
    reference's list rebuild + calcForces (a single point, and a
    steepest-descent step, which rebuilds the list every step) and its MD
    step (list every 10 steps), each as its own process on the host's cores;
    a quadratic in the atom count through the three (the reference's list is
    O(N^2)) gives every job's time, and the stream's jobs/s assumes every
    core busy with one job after another (an upper bound for the CPU)."""
    cores = host_cores()
    order = np.argsort(sizes)
    pick = [int(order[0]), int(order[len(order) // 2]), int(order[-1])]
    jobs = []
    for t in pick:
        a, m = tmpl_inputs[t]
        k = 2 if sizes[t] > 10000 else 6
        jobs.append((a, m, "evals", ["--steps", k, "--warmup", 1]))
        jobs.append((a, m, "time", ["--steps", k, "--warmup", 1, "--nlist-every", 10]))
    res, wall = run_ref_jobs(jobs, cores)
    if any(r is None for r in res):
        return None
    n = np.array([float(sizes[t]) for t in pick])
    t_eval = np.array([res[2 * q]["seconds"] / res[2 * q]["evals"] for q in range(3)])
    t_md = np.array([res[2 * q + 1]["seconds"] / res[2 * q + 1]["steps"] for q in range(3)])
    X = np.stack([n, n * n], axis=1)
    ce = np.linalg.lstsq(X, t_eval, rcond=None)[0]
    cm = np.linalg.lstsq(X, t_md, rcond=None)[0]
    total = 0.0
    for k, kind in enumerate(kinds):
        N = float(sizes[tmpl[k]])
        te, tm = max(ce[0] * N + ce[1] * N * N, 0.0), max(cm[0] * N + cm[1] * N * N, 0.0)
        total += te if kind == A.JOB_ENERGY else (200 * te if kind == A.JOB_MINIMISE else 2000 * tm)
    return {"value": len(kinds) / (total / cores), "unit": "jobs/s", "cores": cores, "kind": "reference",
            "estimate": True, "sample_seconds": wall,
            "sample": "the reference's single point (list + calcForces) and MD step timed on the smallest, "
                      "median and largest templates (%d, %d, %d atoms); job times from a quadratic in N through "
                      "them; %d cores each running jobs back to back" % (sizes[pick[0]], sizes[pick[1]],
                                                                          sizes[pick[2]], cores)}


def L_count(L, ctx):
    c = ctypes.c_int64(0)
    L.pdgpu_launch_count(ctx.ptr, ctypes.byref(c))
    return c.value


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """SM clocks and clock-event (throttle) reasons sampled during the timed
    region: NVML read-only queries every 10 ms on a thread (the timed
    region of the default run is a fraction of a second), or nvidia-smi at
    its 200 ms floor where NVML cannot be loaded."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.nvml = None
        self.lines = []
        self.samples = []  # (sm_mhz, max_mhz, reasons) from NVML
        self.stop_ev = threading.Event()

    def _nvml_handle(self):
        import pynvml as N
        N.nvmlInit()
        try:
            pr = torch.cuda.get_device_properties(self.device)
            bus = "%08x:%02x:%02x.0" % (pr.pci_domain_id, pr.pci_bus_id, pr.pci_device_id)
            h = N.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            h = N.nvmlDeviceGetHandleByIndex(self.device)
        return N, h

    def start(self):
        try:
            N, h = self._nvml_handle()
            bits = {"hw_slowdown": N.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": N.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": N.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": N.nvmlClocksEventReasonSwPowerCap}
            mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
            self.nvml = N

            def poll():
                while not self.stop_ev.is_set():
                    try:
                        sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                        r = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((float(sm), float(mx), [k for k, b in bits.items() if r & b]))
                    except Exception:
                        pass
                    self.stop_ev.wait(0.01)
            self.t = threading.Thread(target=poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        if not shutil.which("nvidia-smi"):
            return
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        self.t = threading.Thread(target=self._read, daemon=True)
        self.t.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.stop_ev.set()
            self.t.join(timeout=2)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
            sm = [x[0] for x in self.samples]
            reasons = sorted({r for x in self.samples for r in x[2]})
            return {"sm_mhz": statistics.median(sm) if sm else None,
                    "sm_max_mhz": self.samples[0][1] if self.samples else None,
                    "reasons": reasons, "samples": len(sm), "source": "NVML, 10 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(self.NAMES):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}


# ---------------------------------------------------------------- reference CPU baselines
def host_cores():
    """Host cores this process may use (the CPU baselines run one reference
    process per core)."""
    try:
        return len(os.sched_getaffinity(0))
    except (AttributeError, OSError):
        return os.cpu_count() or 1


def _ref_input(arrays, meta):
    """A directory the reference driver reads: coordinates and the chains'
    sequences (it rebuilds the topology with the reference's own builder)."""
    tmp = tempfile.mkdtemp(prefix="pdref_")
    np.save(os.path.join(tmp, "pos.npy"), arrays["pos"])
    chains = meta.get("chains") or meta.get("chain") or []
    if isinstance(chains, str):
        chains = [chains]
    with open(os.path.join(tmp, "meta.txt"), "w") as fh:
        for c in chains:
            fh.write("chain %s\n" % c)
    return tmp


def run_ref_jobs(jobs, cores):
    """Run reference-driver jobs, at most `cores` at a time.  jobs: list of
    (arrays, meta, mode, extra args).  Returns the parsed JSON line of each
    job (None where the driver failed) and the wall time."""
    env = dict(os.environ, PD_PARAM_PATH=REF_PARAM)
    pending = list(enumerate(jobs))
    running, out = [], [None] * len(jobs)
    t0 = time.perf_counter()
    while pending or running:
        while pending and len(running) < cores:
            k, (arrays, meta, mode, extra) = pending.pop(0)
            d = _ref_input(arrays, meta)
            cmd = [REF_DRIVER, mode, "--in", d, "--cutoff", str(meta["cutoff"]), "--inner", str(meta["inner"]),
                   "--param", meta.get("param", "amber99aa.ff")] + [str(x) for x in extra]
            pr = subprocess.Popen(cmd, env=env, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            running.append((k, pr, d))
        still = []
        for k, pr, d in running:
            if pr.poll() is None:
                still.append((k, pr, d))
                continue
            txt = pr.stdout.read()
            shutil.rmtree(d, ignore_errors=True)
            try:
                out[k] = json.loads(txt.strip().splitlines()[-1])
            except (ValueError, IndexError):
                out[k] = None
        running = still
        if running:
            time.sleep(0.01)
    return out, time.perf_counter() - t0


def ls_drift(steps, etot_kcal, total_steps):
    """MolecularDynamics::run_core's total-energy drift (md.cpp:206,
    236-240, 182-189): etot sampled every max(1, Steps/1000) steps after
    step 50, least-squares slope, kcal/mol per 1000 steps."""
    freq = max(1, total_steps // 1000)
    steps = np.asarray(steps)
    keep = (steps > 50) & (steps % freq == 0)
    x, y = steps[keep].astype(np.float64), np.asarray(etot_kcal)[keep]
    if len(x) < 2:
        return None
    mx, my = x.mean(), y.mean()
    return 1000.0 * float(np.sum((x - mx) * (y - my)) / np.sum((x - mx) ** 2))


# ---------------------------------------------------------------- reference arm
def run_reference(args, n_gpus):
    """The reference's own CPU MD (compiled from its sources with its own
    flags, oracle/_ref/ref_driver_timing), single-threaded as the reference
    is, on a bounded sample of the same workload; else the oracle port."""
    arrays, meta = load_fixture()
    n = arrays["charge"].shape[0]
    steps = max(1, min(args.steps, args.ref_steps))
    warm = sum(warmup_plan(args.warmup, args.steps))  # the same warm-up as the device arm
    if os.path.exists(REF_DRIVER):
        tmp = tempfile.mkdtemp(prefix="pdref_")
        try:
            np.save(os.path.join(tmp, "pos.npy"), arrays["pos"])
            with open(os.path.join(tmp, "meta.txt"), "w") as fh:
                for c in meta["chains"]:
                    fh.write("chain %s\n" % c)
            env = dict(os.environ, PD_PARAM_PATH=REF_PARAM)
            out = subprocess.check_output(
                [REF_DRIVER, "time", "--in", tmp, "--cutoff", meta["cutoff"], "--inner", meta["inner"],
                 "--steps", str(steps), "--warmup", str(warm), "--nlist-every", "10"],
                env=env, stderr=subprocess.DEVNULL, text=True)
            res = json.loads(out.strip().splitlines()[-1])
            secs = res["seconds"]
            kind = "reference"
        finally:
            shutil.rmtree(tmp, ignore_errors=True)
    else:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        S = O.System(arrays, cutoff=float(meta["cutoff"]), inner=float(meta["inner"]))
        x = arrays["pos"].reshape(-1).copy()
        v = np.zeros_like(x)
        rng = np.random.default_rng(0)
        t0 = None
        ptr = data = None
        for s in range(warm + steps):
            if s == warm:
                t0 = time.perf_counter()
            if s % 10 == 0:
                ptr, data = S.nlist(x)
            f, e, _ = S.calc_forces(x, ptr, data)
            x, v, _ = O.langevin_step(x, v, f.reshape(-1), S.mass, rng.standard_normal(6 * n), 1e-15, 1e12,
                                      300.0, s, warm + steps + 1)
        secs = time.perf_counter() - t0
        kind = "port"
    ns_day = steps * DT_FS * 1e-6 / secs * 86400.0
    sample = "%d MD steps (1 list rebuild per 10) of the %d-atom workload after %d warm-up" % (steps, n, warm)
    return {"value": ns_day, "kind": kind, "cores": 1, "sample": sample, "seconds": secs, "steps": steps,
            "warmup": warm}


# ---------------------------------------------------------------- ours
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=100)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--ref-steps", type=int, default=60, help="bounded CPU sample (steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched workloads")
    ap.add_argument("--pair-path", default="auto", choices=["auto", "rows", "tiles"],
                    help="pair-pass layout of the headline run (default: the autotuner's choice)")
    ap.add_argument("--batched-md-steps", type=int, default=5000)
    ap.add_argument("--serve-requests", type=int, default=300)
    ap.add_argument("--serve-policy", type=int, default=1, help="0 arrival order, 1 least work first")
    ap.add_argument("--serve-max-active", type=int, default=16)
    ap.add_argument("--serve-batch-ms", type=int, default=60,
                    help="queue time a minimisation / MD job waits for like jobs to share its pack")
    ap.add_argument("--serve-rows", action="store_true", help="serve on the list-row pair passes")
    args = ap.parse_args()
    rank, world, local = rank_info()
    n_gpus = check_world(args.gpus, world)

    if args.impl == "reference":
        if rank != 0:
            return 0
        r = run_reference(args, n_gpus)
        cfg = headline_config(int(load_fixture()[0]["charge"].shape[0]), n_gpus)
        line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": "ns/day",
                "n_gpus": n_gpus, "steps": r["steps"], "warmup": r["warmup"],
                "ms_per_step": 1e3 * r["seconds"] / r["steps"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": cfg,
                "cpu_baseline": {"value": r["value"], "unit": "ns/day", "cores": 1, "kind": r["kind"],
                                 "sample": r["sample"]},
                "e2e": {"value": r["value"], "unit": "ns/day", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    device = torch.cuda.current_device()

    sys.path.insert(0, os.path.join(ROOT, "pd.arcus_b200"))
    import pdgpu
    from pdgpu import _abi as A

    arrays, meta = load_fixture()
    ctx = pdgpu.Context(device)
    ws = pdgpu.WorkSpace(pdgpu.SystemSpec(arrays, meta), ctx)
    ff = pdgpu.Forcefield(ws)
    ff.add(pdgpu.FF_Bonded(ws))
    gb = pdgpu.FF_GeneralizedBorn_Still(ws)
    gb.Cutoff, gb.InnerCutoff = float(meta["cutoff"]), float(meta["inner"])
    gb.VdwCutoff, gb.VdwInnerCutoff = float(meta["vdwcut"]), float(meta["vdwinner"])
    ff.add(gb)
    n = ws.nAtoms()

    # parity at the start coordinates (against the reference's FP64 forces)
    ws.nlist().calcNewList()
    ff.calcForces()
    f_ref = arrays["f_total"]
    force_rms = float(np.sqrt(np.sum((ws.cur.f - f_ref) ** 2) / np.sum(f_ref ** 2)))
    de_kcal = float(abs(ws.ene.epot - arrays["ene_total"][0]) * pdgpu.J2KCAL_NA)

    # roofline inputs: pair counts and per-kernel device times (CUDA events)
    counts = np.zeros(5, dtype=np.int64)
    A.check(A.lib().pdgpu_pair_counts(ctx.ptr, ws._sys, counts.ctypes.data_as(A._I64)))
    lpa = np.zeros(3, dtype=np.int32)
    A.check(A.lib().pdgpu_autotune(ctx.ptr, ws._sys, A.iptr(lpa)))
    if args.pair_path != "auto":  # a fixed layout (profiling runs)
        ws.setPairPath(1 if args.pair_path == "tiles" else 0)
    path = ws.setPairPath(-2)  # the layout in use (the autotuner's choice by default)
    kms = np.zeros(3)
    A.check(A.lib().pdgpu_profile_pair_kernels(ctx.ptr, ws._sys, 20, A.dptr(kms)))
    ems, ecnt = np.zeros(4), np.zeros(5, dtype=np.int64)
    if path == 1:  # the evaluation kernel: three phases as three launches, then one launch
        A.check(A.lib().pdgpu_profile_eval(ctx.ptr, ws._sys, 20, A.dptr(ems), ecnt.ctypes.data_as(A._I64)))
    # the FP32 (FMA) and special-function (MUFU) pipes' throughput on this device
    pipes = np.zeros(3)
    A.check(A.lib().pdgpu_measure_pipe_peaks(ctx.ptr, A.dptr(pipes)))

    p = A.md_params_default()
    p.Integrator, p.UpdateNList, p.UseGraph = A.INTEGRATOR_LANGEVIN, BLOCK, 1
    p.Timestep, p.FricCoeff, p.TargetTemp, p.Seed = 1e-15, 1e12, 300.0, 1000 + rank
    A.check(A.lib().pdgpu_md_init_velocities(ctx.ptr, ws._sys, 300.0, 1000 + rank))
    L = A.lib()
    # the end-to-end leg continues the same run (same total, so it replays the
    # graphs the timed region captured): one untimed period realigns it to
    # a list-period boundary and warms its host path, then whole periods,
    # at least 100 steps, are timed
    e2e_steps = max(10 * BLOCK, -(-min(args.steps, 1000) // BLOCK) * BLOCK)
    total = sum(warmup_plan(args.warmup, args.steps)) + args.steps + 2 * BLOCK + e2e_steps + BLOCK
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")  # > 126 MB L2

    def run_block(step0, k):
        st = L.pdgpu_md_run(ctx.ptr, ws._sys, ctypes.byref(p), step0, k, total, None)
        A.check(st)
        return ctx.last_run_ms()

    plan = warmup_plan(args.warmup, args.steps)
    warm = sum(plan)
    s = 0
    for k in plan:
        run_block(s, k)
        s += k
    # timed: K steps in list-period blocks, L2 flushed before each block
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    lc0 = ctypes.c_int64(0)
    L.pdgpu_launch_count(ctx.ptr, ctypes.byref(lc0))
    clocks = ClockSampler(device)
    clocks.start()
    dev_ms = 0.0
    done = 0
    while done < args.steps:
        k = min(BLOCK, args.steps - done)
        flush.zero_()
        torch.cuda.synchronize()
        dev_ms += run_block(s, k)
        s += k
        done += k
    torch.cuda.synchronize()
    clk = clocks.stop()
    lc1 = ctypes.c_int64(0)
    L.pdgpu_launch_count(ctx.ptr, ctypes.byref(lc1))
    if dist:
        dist.barrier()
    t_max = max_over_ranks(dev_ms / 1e3, dist, "cuda")
    value = whole_job_ns_per_day(n_gpus, args.steps, t_max)

    # end to end through the public API: per list period, host -> device
    # state (pinned), 10 steps, device -> host state + energies
    e2e = None
    if not args.no_e2e:
        x_h = torch.empty((n, 3), dtype=torch.float64).pin_memory()
        v_h = torch.empty((n, 3), dtype=torch.float64).pin_memory()
        e_h = torch.empty(A.ENE_COUNT, dtype=torch.float64).pin_memory()
        xp = ctypes.cast(x_h.data_ptr(), A._D)
        vp = ctypes.cast(v_h.data_ptr(), A._D)
        ep = ctypes.cast(e_h.data_ptr(), A._D)
        A.check(L.pdgpu_get_positions(ctx.ptr, ws._sys, xp))
        A.check(L.pdgpu_get_velocities(ctx.ptr, ws._sys, vp))
        s2 = s
        for k in ((BLOCK - s2 % BLOCK) % BLOCK, BLOCK):  # untimed: realign, warm the host path
            if k:
                A.check(L.pdgpu_md_run_io(ctx.ptr, ws._sys, ctypes.byref(p), s2, k, total, xp, vp, xp, vp, ep))
                s2 += k
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        done = 0
        while done < e2e_steps:
            k = min(BLOCK, e2e_steps - done)
            A.check(L.pdgpu_md_run_io(ctx.ptr, ws._sys, ctypes.byref(p), s2, k, total, xp, vp, xp, vp, ep))
            s2 += k
            done += k
        torch.cuda.synchronize()
        te = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
        e2e = {"value": whole_job_ns_per_day(n_gpus, e2e_steps, te), "unit": "ns/day",
               "h2d_bytes_per_step": int(2 * n * 24 / BLOCK),
               "d2h_bytes_per_step": int((2 * n * 24 + A.ENE_COUNT * 8) / BLOCK),
               "steps": e2e_steps, "api": "pdgpu_md_run_io: host positions and velocities in, 10 steps, positions, velocities and energies out"}

    # roofline of the pair kernels (FP32/SFU; nominal peaks at the max SM clock)
    P_B, P_H, entries, tile_pairs, n_tiles = (int(c) for c in counts)
    f_max = (clk.get("sm_max_mhz") or 1965.0) * 1e6
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    F32_nom, SFU_nom = sms * 256 * f_max, sms * 16 * f_max
    F32 = float(pipes[0]) if pipes[0] > 0 else F32_nom
    SFU = float(pipes[1]) if pipes[1] > 0 else SFU_nom
    t2, t3, t4 = (float(x) / 1e3 for x in kms)
    all_flop, all_sfu = 57.0 * P_B + 90.0 * P_H, 7.0 * P_B + 5.0 * P_H
    peak_note = ("measured on this device (pdgpu_measure_pipe_peaks: FP32 FMA and MUFU ex2 chains on every SM): "
                 "%.1f TFLOP/s FP32, %.2f Top/s MUFU; nominal %d SMs x 256 flop / 16 MUFU per clk at sm_max_mhz "
                 "%.0f: %.1f / %.2f (%%s)" % (F32 / 1e12, SFU / 1e12, sms, f_max / 1e6, F32_nom / 1e12,
                                                SFU_nom / 1e12))
    tiles_info = {"tiles": n_tiles, "pair_slots": 256 * n_tiles, "list_pairs_held": tile_pairs,
                  "slot_occupancy": tile_pairs / max(1, 256 * n_tiles)}
    if path == 1:
        # the dominant kernel is the evaluation kernel k_eval_tiles: the Born
        # sums, the GB + LJ + Coulomb pass and the chain rule; the MD step
        # launches it once per phase (its default inside step blocks), so
        # its device time per evaluation is the three phases' sum, and its
        # algorithmic work is all three passes
        tA, tB, tC, tF = (float(x) / 1e3 for x in ems)
        tE = tA + tB + tC
        fr32, frsfu = (all_flop / tE) / F32, (all_sfu / tE) / SFU
        bound = "fp32" if fr32 >= frsfu else "sfu"
        roof = {"kernel": "k_eval_tiles (Born sums, fused GB/LJ/Coulomb, chain rule on 32x8 cluster-pair tiles; "
                          "three one-phase launches per MD step)",
                "bound": bound, "pair_path": "tiles", "tiles": tiles_info,
                "achieved": (all_flop / tE / 1e12) if bound == "fp32" else (all_sfu / tE / 1e12),
                "peak": (F32 if bound == "fp32" else SFU) / 1e12,
                "unit": "TFLOP/s" if bound == "fp32" else "Top/s (MUFU)",
                "frac": max(fr32, frsfu),
                "work": "57 flop + 7 MUFU per P_B pair (Born sum 21+3, chain rule 36+4), 90 flop + 5 MUFU per "
                        "P_H pair (fused GB/LJ/Coulomb); FMA = 2 flop",
                "traffic": NCU_TRAFFIC_EVAL if NCU_TRAFFIC_EVAL else None,
                "traffic_unit": "bytes per evaluation (ncu dram__bytes_read.sum + dram__bytes_write.sum of the "
                                "three one-phase launches on this workload)",
                "peak_source": peak_note % ("the binding pipe: " + ("FP32" if bound == "fp32" else "MUFU")),
                "pairs": {"P_B": P_B, "P_H": P_H, "list_entries": entries},
                "kernel_ms": {"three_launches": tE * 1e3, "phase_born": tA * 1e3, "phase_pair": tB * 1e3,
                              "phase_chain": tC * 1e3, "one_cooperative_launch": tF * 1e3},
                "phase_frac": {"born": max(21.0 * P_B / F32, 3.0 * P_B / SFU) / tA,
                               "pair": max(90.0 * P_H / F32, 5.0 * P_H / SFU) / tB,
                               "chain": max(36.0 * P_B / F32, 4.0 * P_B / SFU) / tC,
                               "one_cooperative_launch": max(all_flop / F32, all_sfu / SFU) / tF},
                "chain_phase_tiles": {"visited": int(ecnt[1]), "of": int(ecnt[0])},
                "careful_tiles": {"born": int(ecnt[2]), "pair": int(ecnt[3]), "chain": int(ecnt[4])},
                "three_pass_form_ms": {"born_K2": t2 * 1e3, "pair_K3": t3 * 1e3, "chain_K4": t4 * 1e3,
                                       "frac_of_roof": max(all_flop / F32, all_sfu / SFU) / (t2 + t3 + t4)},
                "pair_kernels_frac_of_roof": max(all_flop / F32, all_sfu / SFU) / tE,
                "issue_roof": {
                    "warp_instructions": sum(NCU_INST_EVAL),
                    "per_phase": list(NCU_INST_EVAL),
                    "roof_ms": 1e3 * sum(NCU_INST_EVAL) / (sms * 4 * f_max),
                    "frac": (sum(NCU_INST_EVAL) / (sms * 4 * f_max)) / tE,
                    "frac_one_cooperative_launch": (sum(NCU_INST_EVAL) / (sms * 4 * f_max)) / tF,
                    "note": "the instructions the kernel executes (ncu, this workload) at one warp instruction "
                            "per scheduler per clock (4 a SM); the FP32/SFU roof counts only the algorithmic "
                            "operations of the pairs inside the cutoffs"}}
    else:
        k3_flop, k3_sfu = 90.0 * P_H, 5.0 * P_H
        k3_frac_fp32 = (k3_flop / t3) / F32
        k3_frac_sfu = (k3_sfu / t3) / SFU
        t_pair = t2 + t3 + t4
        t_roof = max(all_flop / F32, all_sfu / SFU)
        bound = "fp32" if k3_frac_fp32 >= k3_frac_sfu else "sfu"
        roof = {"kernel": "k_gb_pair (fused GB + LJ + Coulomb on neighbour-list rows, K3)", "bound": bound,
                "pair_path": "rows", "tiles": tiles_info,
                "achieved": (k3_flop / t3 / 1e12) if bound == "fp32" else (k3_sfu / t3 / 1e12),
                "peak": (F32 if bound == "fp32" else SFU) / 1e12,
                "unit": "TFLOP/s" if bound == "fp32" else "Top/s (MUFU)",
                "frac": max(k3_frac_fp32, k3_frac_sfu), "traffic": None,
                "peak_source": peak_note % ("the binding pipe: " + ("FP32" if bound == "fp32" else "MUFU")),
                "pairs": {"P_B": P_B, "P_H": P_H, "list_entries": entries},
                "kernel_ms": {"born_K2": t2 * 1e3, "pair_K3": t3 * 1e3, "chain_K4": t4 * 1e3},
                "lanes_per_atom": {"born_K2": int(lpa[0]), "pair_K3": int(lpa[1]), "chain_K4": int(lpa[2])},
                "pair_kernels_frac_of_roof": t_roof / t_pair}

    line = {"metric": METRIC, "value": value, "unit": "ns/day", "n_gpus": n_gpus, "steps": args.steps,
            "warmup": warm, "ms_per_step": 1e3 * t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 pair / f64 state",
            "data": "synthetic (seeded peptides built by the reference's NewProtein)",
            "config": headline_config(n, n_gpus),
            "parity": {"force_rel_rms_vs_fp64": force_rms, "epot_abs_err_kcal": de_kcal},
            "gpu_launches": int(lc1.value - lc0.value),
            "clocks": clk, "roofline": roof, "e2e": e2e}
    if not args.no_batched:
        line["plain_small"] = bench_plain_small(pdgpu, A, ctx, torch)
        line["lcpo"] = bench_lcpo(pdgpu, A, ctx, torch, arrays, meta, f_max, sms)
        line["batched_sp"] = bench_batched_sp(pdgpu, A, ctx, torch, peaks=(F32, SFU))
        line["batched_md"] = bench_batched_md(pdgpu, A, ctx, torch, steps=args.batched_md_steps,
                                              peaks=(F32, SFU))
        line["serving"] = bench_serving(pdgpu, A, ctx, torch, n_requests=args.serve_requests,
                                        policy=args.serve_policy, max_active=args.serve_max_active,
                                        tiles=not args.serve_rows, batch_ms=args.serve_batch_ms)
    if rank == 0 and n_gpus == 1 and not args.no_cpu_baseline:
        try:
            cb = run_reference(args, 1)
            line["cpu_baseline"] = {"value": cb["value"], "unit": "ns/day", "cores": cb["cores"],
                                    "kind": cb["kind"], "sample": cb["sample"]}
        except Exception as exc:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "error": str(exc)[:200]}
    if rank == 0:
        print(json.dumps(line))
    ws.close()
    ctx.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
