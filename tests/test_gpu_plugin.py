"""GPU: the drop-in components FF_GeneralizedBorn_Still_GPU and
FF_SASA_LCPO_GPU (pd.arcus_b200/plugin) driven by the reference's own C++
protocols.

oracle/_ref/ref_driver_gpu is the reference driver (oracle/ref_driver.cpp,
linked with the reference library compiled from its sources) built with
the B200 components in place of FF_GeneralizedBorn_Still and FF_SASA_LCPO;
oracle/_ref/ref_driver is the same driver with the reference's own.  Both
replay one fixture system: single-point forces and energies through
Forcefield::calcForces / calcEnergies, two integrator steps, 10 SD and 10
CG steps through Minimisation::runcore, and 20 Langevin steps through
MolecularDynamics::runcore.  Tolerances:
  forces (relative RMS)               1e-5 against the FP64 reference
  Born radii                          relative 2e-6
  pair energies                       relative 1e-5 or 1e-3 kcal/mol
  integrator / minimiser positions    1e-4 A (the reference's own protocol
                                      decisions on FP32-level force sums)
"""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import ROOT, load_fixture, rel_rms

pytestmark = pytest.mark.gpu

J2K = (1.0 / 4184.0) * 6.0221418e23
REF = os.path.join(ROOT, "oracle", "_ref")


def energy_close(got_J, ref_J, rel=1e-5, abs_kcal=1e-3):
    return abs(got_J - ref_J) * J2K <= max(rel * abs(ref_J) * J2K, abs_kcal)


def _replay(binary, name, out, extra=None):
    arrays, meta = load_fixture(name)
    src = tempfile.mkdtemp(prefix="pdplug_in_")
    try:
        np.save(os.path.join(src, "pos.npy"), arrays["pos"])
        with open(os.path.join(src, "meta.txt"), "w") as fh:
            for c in meta["chains"]:
                fh.write("chain %s\n" % c)
        env = dict(os.environ, PD_PARAM_PATH=os.path.join(REF, "param"))
        args = extra if extra is not None else ["--md", "2", "--min", "10", "--steps", "20", "--nlist-every", "10"]
        subprocess.run([os.path.join(REF, binary), "replay", "--in", src, "--out", out, "--cutoff", meta["cutoff"],
                        "--inner", meta["inner"], "--param", meta["param"]] + args, env=env, check=True,
                       capture_output=True, timeout=600)
    finally:
        shutil.rmtree(src, ignore_errors=True)
    return {f[:-4]: np.load(os.path.join(out, f)) for f in os.listdir(out) if f.endswith(".npy")}, arrays


@pytest.fixture(scope="module")
def replays():
    if not os.path.exists(os.path.join(REF, "ref_driver_gpu")):
        pytest.fail("oracle/_ref/ref_driver_gpu is not built (make -C oracle ref-gpu)")
    tmp = tempfile.mkdtemp(prefix="pdplug_")
    try:
        gpu, arrays = _replay("ref_driver_gpu", "pep20_s2", os.path.join(tmp, "gpu"))
        cpu, _ = _replay("ref_driver", "pep20_s2", os.path.join(tmp, "cpu"))
        yield gpu, cpu, arrays
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def test_component_single_point(replays):
    gpu, cpu, a = replays
    assert np.array_equal(gpu["nl_ptr"], a["nl_ptr"]) and np.array_equal(gpu["nl_data"], a["nl_data"])
    assert rel_rms(gpu["f_total"], a["f_total"]) <= 1e-5
    assert rel_rms(gpu["f_gb"], a["f_gb"]) <= 1e-5
    assert np.max(np.abs(gpu["born"] - a["born"]) / np.abs(a["born"])) <= 2e-6
    for k in range(6):  # epot, vdw, elec, pol, pol_cross, pol_self
        assert energy_close(gpu["ene_total"][k], a["ene_total"][k]), k
    assert rel_rms(gpu["atom_epot"], a["atom_epot"]) <= 1e-5
    # the energy path (calcEnergies): forces and energies
    assert rel_rms(gpu["f_energypath"], a["f_energypath"]) <= 1e-5
    for k in (0, 1, 2, 10):
        assert energy_close(gpu["ene_energypath"][k], a["ene_energypath"][k]), k
    # the replaying CPU driver reproduces its own fixture
    assert rel_rms(cpu["f_total"], a["f_total"]) <= 1e-12


def test_component_in_protocols(replays):
    gpu, cpu, a = replays
    for pre in ("mdlv_", "mdvv_"):
        assert np.max(np.abs(gpu[pre + "x"] - a[pre + "x"])) <= 1e-4, pre
    for pre in ("minsd_", "mincg_"):
        assert np.max(np.abs(gpu[pre + "x"] - a[pre + "x"])) <= 1e-4, pre
        assert gpu[pre + "result"][0] == a[pre + "result"][0]  # steps taken
    # MolecularDynamics::runcore, 20 Langevin steps: the same random draws,
    # so the trajectories differ by the force rounding only
    assert int(gpu["proto_md_ene"][-1]) == int(cpu["proto_md_ene"][-1]) == 20
    assert np.max(np.abs(gpu["proto_md_x"] - cpu["proto_md_x"])) <= 1e-4
    assert energy_close(gpu["proto_md_ene"][0], cpu["proto_md_ene"][0], rel=1e-4)


def test_lcpo_component_in_protocols():
    """{FF_Bonded, GB, LCPO} with both B200 components: the single point at
    step 0, 12 velocity-Verlet steps and 12 steepest-descent steps
    (UpdateSasa 5: the held forces on the steps between), against the
    reference's own run of the same (tests/golden/lcpo_pep24_s5.npz)."""
    tmp = tempfile.mkdtemp(prefix="pdplug_lcpo_")
    try:
        gpu, a = _replay("ref_driver_gpu", "lcpo_pep24_s5", os.path.join(tmp, "gpu"),
                         ["--lcpo-asp", "0.005", "--lcpo", "5,12"])
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    assert rel_rms(gpu["lcpo_f_total"], a["lcpo_f_total"]) <= 1e-5
    for k in (0, 10):  # epot, epot_surf
        assert energy_close(gpu["lcpo_ene_total"][k], a["lcpo_ene_total"][k]), k
    assert np.max(np.abs(gpu["lcpo_mdvv_x"] - a["lcpo_mdvv_x"])) <= 1e-4
    # steps taken, final energy, step multiplier (the accept / reject record)
    res = (gpu["lcpo_minsd_result"].tolist(), a["lcpo_minsd_result"].tolist())
    assert gpu["lcpo_minsd_result"][0] == a["lcpo_minsd_result"][0], res
    assert np.max(np.abs(gpu["lcpo_minsd_x"] - a["lcpo_minsd_x"])) <= 1e-4, res
