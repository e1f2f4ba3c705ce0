"""Generate the golden fixtures under tests/golden/ from the reference itself.

Runs oracle/_ref/ref_driver (the reference library compiled from its own
sources by ``make -C oracle ref``) on seeded synthetic peptide systems and
packs its FP64 outputs into compressed ``.npz`` files.  Needs the reference
tree (REF, default /root/reference) only through that build; the fixtures
themselves are self-contained and are what the tests read.

    python tests/golden/make_golden.py            # all fixtures
    python tests/golden/make_golden.py pep8_s1    # one

Systems (extended builds from the reference's NewProtein, sequences drawn
uniformly from the 20 standard residues with the stated seed, pre-minimised
with 500 steepest-descent steps at Rc 12 A unless noted):
  pep8_s1       8 residues, Rc 12, + 3 MD steps per integrator, 20 SD/CG steps
  pep20_s2      20 residues, Rc 12, + 2 MD steps per integrator, 10 SD/CG steps,
                4 phi/psi trial conformations (sigma 15 deg) with their forces
  pep30_s3_rc16 30 residues, Rc 16 (the large-system cutoff)
  two_chain_s4  two 12-residue chains 12 A apart, Rc 10 (inter-chain pairs),
                3 phi/psi trial conformations
  c1_pep64_s0   the 64-residue, seed-0 chain of the small plain-MD workload, Rc 12
  lcpo_pep24_s5 24 residues, Rc 12, with the LCPO surface-area term (FF_SASA_LCPO,
                GlobalASP 0.005 kcal/mol/A^2, UpdateSasa 5): its per-atom parameters,
                its forces and energies alone and with {FF_Bonded, GB}, and 12
                velocity-Verlet and 12 steepest-descent steps of the whole forcefield
  nb_pep24_s7   24 residues, Rc 12: FF_NonBonded alone in each calcForces mode
                (force switch -- its default --, energy switch, plain Coulomb,
                DDDielectric set, dielectric 4, the long-range VdW correction)
                at the GB cutoffs, and the GB component with FastMode off
                (FF_NonBonded::calcForces + calcBornForces)
  c2_16x80_s2   16 x 80-residue chains on a 4x4 grid 25 A apart (~20.6k atoms),
                Rc 16: inputs plus reference forces, Born radii and energies
                (no neighbour list: too large to store), and the LCPO term's
                parameters, forces and energies (GlobalASP 0.005, no dense case)
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "ref_driver")
PARAM = os.path.join(ROOT, "oracle", "_ref", "param")

SYSTEMS = {
    "pep8_s1": dict(nres=[8], seed=1, cutoff=12, premin=500, md=3, min=20),
    "pep20_s2": dict(nres=[20], seed=2, cutoff=12, premin=500, md=2, min=10, trials=4),
    "pep30_s3_rc16": dict(nres=[30], seed=3, cutoff=16, premin=500),
    "two_chain_s4": dict(nres=[12, 12], seed=4, cutoff=10, premin=500, grid=(2, 12), trials=3),
    "c1_pep64_s0": dict(nres=[64], seed=0, cutoff=12, premin=500),
    "lcpo_pep24_s5": dict(nres=[24], seed=5, cutoff=12, premin=500, lcpo=(0.005, 5, 12),
                          drop=("lcpo_mdvv_normals",)),
    "c2_16x80_s2": dict(nres=[80] * 16, seed=2, cutoff=16, premin=500, grid=(4, 25), drop_nl=True,
                        lcpo=(0.005, 5, 0, 0)),
    "nb_pep24_s7": dict(nres=[24], seed=7, cutoff=12, premin=500, nbmodes=True),
}

# arrays kept for the large system (inputs + a few reference results)
LARGE_KEEP = None  # everything except the neighbour list


def build(name, spec, keep_dir=None):
    if not os.path.exists(DRIVER):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", "-j8"])
    out = keep_dir or tempfile.mkdtemp(prefix="pdgold_")
    cmd = [DRIVER, "build", "--out", out, "--nres", ",".join(map(str, spec["nres"])),
           "--seed", str(spec["seed"]), "--cutoff", str(spec["cutoff"]),
           "--premin", str(spec.get("premin", 500))]
    if "grid" in spec:
        cmd += ["--grid", "%d,%d" % spec["grid"]]
    if spec.get("md"):
        cmd += ["--md", str(spec["md"])]
    if spec.get("min"):
        cmd += ["--min", str(spec["min"])]
    if spec.get("trials"):
        cmd += ["--trials", str(spec["trials"]), "--trial-sigma", "15"]
    if spec.get("nbmodes"):
        cmd += ["--nbmodes"]
    if spec.get("lcpo"):
        asp, update, steps = spec["lcpo"][:3]
        dense = spec["lcpo"][3] if len(spec["lcpo"]) > 3 else 1
        cmd += ["--lcpo-asp", repr(asp), "--lcpo", "%d,%d,%d" % (update, steps, dense)]
    env = dict(os.environ, PD_PARAM_PATH=PARAM)
    subprocess.check_call(cmd, env=env, stdout=subprocess.DEVNULL)
    arrays = {}
    for fn in sorted(os.listdir(out)):
        if fn.endswith(".npy"):
            arrays[fn[:-4]] = np.load(os.path.join(out, fn))
    meta = {}
    chains = []
    with open(os.path.join(out, "meta.txt")) as fh:
        for line in fh:
            k, v = line.split(None, 1)
            if k == "chain":
                chains.append(v.strip())
            else:
                meta[k] = v.strip()
    meta["chains"] = chains
    meta["name"] = name
    if spec.get("drop_nl"):
        for k in list(arrays):
            if k.startswith("nl_") or k in ("f_energypath", "ene_energypath", "atom_epot"):
                del arrays[k]
    for k in spec.get("drop", ()):
        del arrays[k]
    arrays["meta_json"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    if keep_dir is None:
        shutil.rmtree(out)
    return os.path.join(HERE, name + ".npz")


# Peptide libraries for the batched workloads: separate single-chain systems
# stored in one file, arrays prefixed "pNN_".  Lengths are drawn with numpy's
# seeded generator; each peptide is pre-minimised with 200 SD steps.
#   lib16_amber_s3  16 peptides, lengths floor(exp(U(ln 20, ln 200))), amber99aa, Rc 12,
#                   2 phi/psi trial conformations each (sigma 15 deg) with their forces
#   lib16_opls_s4   16 peptides, lengths U{30..150}, oplsaal, Rc 12
LIBRARIES = {
    "lib16_amber_s3": dict(n=16, seed=3, dist="loguniform", lo=20, hi=200, param="amber99aa.ff", trials=2),
    "lib16_opls_s4": dict(n=16, seed=4, dist="uniform", lo=30, hi=150, param="oplsaal.ff"),
}
LIB_KEEP_OUT = ("nl_", "f_energypath", "ene_energypath", "atom_epot", "f_gb", "ene_gb", "f_bonded", "ene_bonded")


def _lib_member(args):
    name, k, nres, seed, param, trials = args
    out = tempfile.mkdtemp(prefix="pdlib_")
    cmd = [DRIVER, "build", "--out", out, "--nres", str(nres), "--seed", str(seed), "--cutoff", "12",
           "--premin", "200", "--param", param]
    if trials:
        cmd += ["--trials", str(trials), "--trial-sigma", "15"]
    env = dict(os.environ, PD_PARAM_PATH=PARAM)
    subprocess.check_call(cmd, env=env, stdout=subprocess.DEVNULL)
    arrays = {}
    for fn in sorted(os.listdir(out)):
        if fn.endswith(".npy") and not fn.startswith(LIB_KEEP_OUT):
            arrays["p%02d_%s" % (k, fn[:-4])] = np.load(os.path.join(out, fn))
    meta = {}
    with open(os.path.join(out, "meta.txt")) as fh:
        for line in fh:
            kk, v = line.split(None, 1)
            meta.setdefault(kk, []).append(v.strip()) if kk == "chain" else meta.__setitem__(kk, v.strip())
    shutil.rmtree(out)
    return k, arrays, meta


def build_library(name, spec):
    import multiprocessing as mp
    if not os.path.exists(DRIVER):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", "-j8"])
    rng = np.random.default_rng(spec["seed"])
    if spec["dist"] == "loguniform":
        lens = np.floor(np.exp(rng.uniform(np.log(spec["lo"]), np.log(spec["hi"]), spec["n"]))).astype(int)
    else:
        lens = rng.integers(spec["lo"], spec["hi"] + 1, spec["n"])
    jobs = [(name, k, int(lens[k]), spec["seed"] * 100 + k, spec["param"], spec.get("trials", 0))
            for k in range(spec["n"])]
    arrays, metas = {}, {}
    with mp.get_context("spawn").Pool(min(8, os.cpu_count() or 1)) as pool:
        for k, a, m in pool.imap_unordered(_lib_member, jobs):
            arrays.update(a)
            metas[k] = m
    meta = {"name": name, "members": [metas[k] for k in range(spec["n"])], "param": spec["param"]}
    arrays["meta_json"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)
    return os.path.join(HERE, name + ".npz")


def main(argv):
    names = argv[1:] or (list(SYSTEMS) + list(LIBRARIES))
    for n in names:
        p = build(n, SYSTEMS[n]) if n in SYSTEMS else build_library(n, LIBRARIES[n])
        print("%-16s %8.1f KB" % (n, os.path.getsize(p) / 1024.0))


if __name__ == "__main__":
    main(sys.argv)
