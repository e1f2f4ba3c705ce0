"""ctypes binding of libpdgpu.so (the C ABI declared in include/pdgpu.h).

The library is built in-tree (``python pd.arcus_b200/build.py``) into
``pd.arcus_b200/pdgpu/_lib/libpdgpu.so``.  There is no CPU fallback: if the
library is missing or no CUDA device is usable, every entry point raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libpdgpu.so")

OK = 0
ERR_ARG, ERR_CUDA, ERR_NOMEM, ERR_UNSTABLE, ERR_STATE, ERR_BUDGET, ERR_NODEVICE = -1, -2, -3, -4, -5, -6, -7

ENE_EPOT, ENE_VDW, ENE_ELEC, ENE_POL, ENE_POL_CROSS, ENE_POL_SELF = 0, 1, 2, 3, 4, 5
ENE_BOND, ENE_ANGLE, ENE_TORSION, ENE_VIRIAL, ENE_EKIN, ENE_ETOT = 6, 7, 8, 9, 10, 11
ENE_GB_COMPONENT = 12
ENE_SURF = 15
ENE_COUNT = 16

INTEGRATOR_VERLET, INTEGRATOR_VELOCITY_VERLET, INTEGRATOR_BEEMAN, INTEGRATOR_LANGEVIN = 0, 1, 2, 3
MIN_STEEPEST_DESCENT, MIN_CONJUGATE_GRADIENTS = 0, 1


class PdgpuError(RuntimeError):
    """A non-zero status from libpdgpu (the reference maps its C++
    exceptions to RuntimeError in the SWIG layer, src/pd/pd.i:16-19)."""

    def __init__(self, status, msg):
        super().__init__("pdgpu status %d: %s" % (status, msg))
        self.status = status


class UnstableError(PdgpuError):
    """NaN energy: the reference's ProcedureException('Simulation unstable')."""


class FFParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "Cutoff", "InnerCutoff", "VdwCutoff", "VdwInnerCutoff", "Vdw14Scaling", "Elec14Scaling",
        "Dielectric", "DielectricSolute", "DielectricSolvent", "GbsaStillCutoff",
        "ExpApproxThreshold", "DielectricOffset", "BornRadiusOffset", "P1", "P2", "P3", "P4", "P5",
        "DDDielectricAlpha", "VdwCorDensity", "VdwCorEpsilon", "VdwCorRadius", "VdwCorCutoff",
        "Padding")] + [(n, ctypes.c_int32) for n in (
            "FastMode", "EnergySwitch", "ForceSwitch", "DDDielectric", "DoVdw", "DoElec", "VdwCor",
            "_reserved")]


class MDParams(ctypes.Structure):
    _fields_ = [("Integrator", ctypes.c_int32), ("UpdateNList", ctypes.c_int32),
                ("LangevinOnHydrogens", ctypes.c_int32), ("UseGraph", ctypes.c_int32),
                ("Timestep", ctypes.c_double), ("FricCoeff", ctypes.c_double),
                ("TargetTemp", ctypes.c_double), ("Seed", ctypes.c_uint64)]


class MinParams(ctypes.Structure):
    _fields_ = [("Algorithm", ctypes.c_int32), ("UpdateNList", ctypes.c_int32),
                ("StepSize", ctypes.c_double), ("SlopeCutoff", ctypes.c_double),
                ("Strictness", ctypes.c_double)]


class MCParams(ctypes.Structure):
    _fields_ = [("Steps", ctypes.c_int32), ("FinalState", ctypes.c_int32), ("Temperature", ctypes.c_double),
                ("Sigma", ctypes.c_double), ("Seed", ctypes.c_uint64)]


MC_LAST, MC_LAST_ACC, MC_LOWEST_EPOT = 0, 1, 2


class ServeParams(ctypes.Structure):
    _fields_ = [("hbm_budget", ctypes.c_int64), ("max_active", ctypes.c_int32), ("lanes", ctypes.c_int32 * 3),
                ("tiles", ctypes.c_int32), ("policy", ctypes.c_int32), ("group", ctypes.c_int32),
                ("batch_ms", ctypes.c_int32)]


class Job(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("steps", ctypes.c_int32), ("md", MDParams), ("min", MinParams),
                ("init_temp", ctypes.c_double)]


class JobInfo(ctypes.Structure):
    _fields_ = [("state", ctypes.c_int32), ("status", ctypes.c_int32), ("kind", ctypes.c_int32),
                ("natoms", ctypes.c_int32), ("steps_done", ctypes.c_int32), ("_reserved", ctypes.c_int32),
                ("t_queue_ms", ctypes.c_double), ("t_run_ms", ctypes.c_double), ("t_total_ms", ctypes.c_double)]


class ServeStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
                ("active", ctypes.c_int32), ("queued", ctypes.c_int32), ("peak_active", ctypes.c_int32),
                ("groups", ctypes.c_int32), ("bytes_in_use", ctypes.c_int64), ("peak_bytes", ctypes.c_int64)]


JOB_ENERGY, JOB_MINIMISE, JOB_MD = 0, 1, 2
JOB_QUEUED, JOB_RUNNING, JOB_DONE, JOB_FAILED = 0, 1, 2, 3

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int32)
_I8 = ctypes.POINTER(ctypes.c_int8)
_U8 = ctypes.POINTER(ctypes.c_uint8)
_I64 = ctypes.POINTER(ctypes.c_int64)
_CTX = ctypes.c_void_p

# name -> (restype, argtypes)
PROTOTYPES = {
    "pdgpu_ff_params_default": (None, [ctypes.POINTER(FFParams)]),
    "pdgpu_md_params_default": (None, [ctypes.POINTER(MDParams)]),
    "pdgpu_min_params_default": (None, [ctypes.POINTER(MinParams)]),
    "pdgpu_mc_params_default": (None, [ctypes.POINTER(MCParams)]),
    "pdgpu_mc_run": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.POINTER(MCParams), _I, _D]),
    "pdgpu_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_CTX)]),
    "pdgpu_ctx_destroy": (ctypes.c_int, [_CTX]),
    "pdgpu_last_error": (ctypes.c_char_p, []),
    "pdgpu_ctx_mem_used": (ctypes.c_int, [_CTX, _I64]),
    "pdgpu_system_create": (ctypes.c_int, [_CTX, ctypes.c_int32, _D, _D, _D, _D, _D, _I, _I, _I, _D,
                                           _I, _I, _D, _I, _I, ctypes.POINTER(FFParams), _I]),
    "pdgpu_system_destroy": (ctypes.c_int, [_CTX, ctypes.c_int32]),
    "pdgpu_system_set_params": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.POINTER(FFParams)]),
    "pdgpu_system_set_bonded": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.c_int32, _I, _D,
                                               ctypes.c_int32, _I, _D, ctypes.c_int32, _I, _I, _D,
                                               ctypes.c_int32, _I, _I, _D]),
    "pdgpu_system_set_hydrogens": (ctypes.c_int, [_CTX, ctypes.c_int32, _I8]),
    "pdgpu_sasa_lcpo_set": (ctypes.c_int, [_CTX, ctypes.c_int32, _D, _D, _D, _U8, ctypes.c_int32]),
    "pdgpu_set_step": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.c_int32]),
    "pdgpu_get_step": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]),
    "pdgpu_batch_create": (ctypes.c_int, [_CTX, _I, ctypes.c_int32, _I]),
    "pdgpu_batch_info": (ctypes.c_int, [_CTX, ctypes.c_int32, _I, _I]),
    "pdgpu_set_seeds": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64)]),
    "pdgpu_system_set_torsions": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.c_int32, _I]),
    "pdgpu_save_base_positions": (ctypes.c_int, [_CTX, ctypes.c_int32]),
    "pdgpu_perturb_torsions": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.c_double, ctypes.c_uint64, _D]),
    "pdgpu_set_positions": (ctypes.c_int, [_CTX, ctypes.c_int32, _D]),
    "pdgpu_get_positions": (ctypes.c_int, [_CTX, ctypes.c_int32, _D]),
    "pdgpu_set_velocities": (ctypes.c_int, [_CTX, ctypes.c_int32, _D]),
    "pdgpu_get_velocities": (ctypes.c_int, [_CTX, ctypes.c_int32, _D]),
    "pdgpu_get_forces": (ctypes.c_int, [_CTX, ctypes.c_int32, _D]),
    "pdgpu_get_born_radii": (ctypes.c_int, [_CTX, ctypes.c_int32, _D]),
    "pdgpu_get_atom_epot": (ctypes.c_int, [_CTX, ctypes.c_int32, _D]),
    "pdgpu_get_energies": (ctypes.c_int, [_CTX, ctypes.c_int32, _D, ctypes.c_int32]),
    "pdgpu_zero_forces": (ctypes.c_int, [_CTX, ctypes.c_int32]),
    "pdgpu_nlist_build": (ctypes.c_int, [_CTX, ctypes.c_int32]),
    "pdgpu_nlist_export": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.c_int32, _I, _I, ctypes.c_int64,
                                          _I64]),
    "pdgpu_gb_forces": (ctypes.c_int, [_CTX, ctypes.c_int32]),
    "pdgpu_gb_energies": (ctypes.c_int, [_CTX, ctypes.c_int32]),
    "pdgpu_nonbonded_forces": (ctypes.c_int, [_CTX, ctypes.c_int32]),
    "pdgpu_bonded_forces": (ctypes.c_int, [_CTX, ctypes.c_int32]),
    "pdgpu_sasa_lcpo_forces": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.c_int32]),
    "pdgpu_sasa_lcpo_energies": (ctypes.c_int, [_CTX, ctypes.c_int32]),
    "pdgpu_sasa_lcpo_get": (ctypes.c_int, [_CTX, ctypes.c_int32, _D, _D]),
    "pdgpu_profile_lcpo": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.c_int32, _D]),
    "pdgpu_calc_forces": (ctypes.c_int, [_CTX, ctypes.c_int32]),
    "pdgpu_md_run": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.POINTER(MDParams), ctypes.c_int32,
                                    ctypes.c_int32, ctypes.c_int32, _D]),
    "pdgpu_md_run_io": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.POINTER(MDParams), ctypes.c_int32,
                                       ctypes.c_int32, ctypes.c_int32, _D, _D, _D, _D, _D]),
    "pdgpu_md_set_trajectory": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "pdgpu_md_read_trajectory": (ctypes.c_int, [_CTX, ctypes.c_int32, _D, ctypes.POINTER(ctypes.c_int64),
                                                ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                                ctypes.POINTER(ctypes.c_int32)]),
    "pdgpu_md_step_with_normals": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.POINTER(MDParams),
                                                  ctypes.c_int32, ctypes.c_int32, _D]),
    "pdgpu_md_init_velocities": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.c_double, ctypes.c_uint64]),
    "pdgpu_minimise_run": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.POINTER(MinParams),
                                          ctypes.c_int32, _I]),
    "pdgpu_last_run_ms": (ctypes.c_int, [_CTX, _D]),
    "pdgpu_pair_counts": (ctypes.c_int, [_CTX, ctypes.c_int32, _I64]),
    "pdgpu_profile_pair_kernels": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.c_int32, _D]),
    "pdgpu_profile_eval": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.c_int32, _D, _I64]),
    "pdgpu_measure_pipe_peaks": (ctypes.c_int, [_CTX, _D]),
    "pdgpu_eval_mode": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.c_int32, _I]),
    "pdgpu_launch_count": (ctypes.c_int, [_CTX, _I64]),
    "pdgpu_graph_replays": (ctypes.c_int, [_CTX, ctypes.c_int32, _I64]),
    "pdgpu_autotune": (ctypes.c_int, [_CTX, ctypes.c_int32, _I]),
    "pdgpu_set_lanes": (ctypes.c_int, [_CTX, ctypes.c_int32, _I]),
    "pdgpu_pair_path": (ctypes.c_int, [_CTX, ctypes.c_int32, ctypes.c_int32, _I]),
    "pdgpu_serve_params_default": (None, [ctypes.POINTER(ServeParams)]),
    "pdgpu_serve_create": (ctypes.c_int, [_CTX, ctypes.POINTER(ServeParams), ctypes.POINTER(ctypes.c_void_p)]),
    "pdgpu_serve_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(Job), _D, _I64]),
    "pdgpu_serve_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double]),
    "pdgpu_serve_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.POINTER(JobInfo)]),
    "pdgpu_serve_result": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, _D, _D, _D, _D]),
    "pdgpu_serve_release": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64]),
    "pdgpu_serve_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServeStats)]),
    "pdgpu_serve_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "pdgpu_nlist_build_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, _I64,
                                                 ctypes.c_void_p]),
}

_lib = None


def lib():
    """Load libpdgpu.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libpdgpu.so not built (%s); run `python pd.arcus_b200/build.py`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error():
    m = lib().pdgpu_last_error()
    return m.decode() if m else ""


def check(status):
    if status != OK:
        cls = UnstableError if status == ERR_UNSTABLE else PdgpuError
        raise cls(status, last_error())
    return status


def dptr(a):
    return a.ctypes.data_as(_D)


def iptr(a):
    return a.ctypes.data_as(_I)


def cd(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def ci(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def ff_params_default():
    p = FFParams()
    lib().pdgpu_ff_params_default(ctypes.byref(p))
    return p


def md_params_default():
    p = MDParams()
    lib().pdgpu_md_params_default(ctypes.byref(p))
    return p


def min_params_default():
    p = MinParams()
    lib().pdgpu_min_params_default(ctypes.byref(p))
    return p


def mc_params_default():
    p = MCParams()
    lib().pdgpu_mc_params_default(ctypes.byref(p))
    return p
