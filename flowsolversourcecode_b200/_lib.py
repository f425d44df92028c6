"""ctypes binding of libfsb200.so (the C ABI declared in include/fsb200.h).

The library is built in-tree by ``flowsolversourcecode_b200.build``.  There is
no fallback: if the shared library is missing or a CUDA device is absent the
calls fail with an exception, never silently on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfsb200.so")

FS_MAX_PATCHES = 32

# status codes
FS_OK, FS_E_ARG, FS_E_CUDA, FS_E_NOMEM, FS_E_NAN, FS_E_DIVERGED, FS_E_TIMEOUT, FS_E_MESH, FS_E_UNSUPPORTED = (
    0, -1, -2, -3, -4, -5, -6, -7, -8)
FS_E_TOO_LARGE = -9
FS_NOALLOC_MAX_ROWS = 262144
FS_NN_NPARAM = 33665
# variable ids (GetNFfromVariable)
VAR_U, VAR_V, VAR_W, VAR_PC, VAR_MASS, VAR_TEMP = 1, 2, 3, 4, 5, 6
VAR_TKE, VAR_TED, VAR_RHOK, VAR_P = 8, 9, 10, 20
# boundary types
(BC_WALL_NOSLIP, BC_WALL_SLIP, BC_SYMMETRY, BC_INLET_VEL, BC_OUTLET_FD, BC_OUTLET_SP, BC_INLET_MASS, BC_INLET_SP,
 BC_OUTLET_MASS, BC_OUTLET_ASP, BC_OUTLET_RES, BC_INLET_STAG) = range(12)
# thermal boundary types (fs_tbc)
TBC = {"default": 0, "dirichlet": 1, "vonneumann": 2, "robin": 3, "statictemperature": 4,
       "stagnationtemperature": 5, "fullydevelopedenergy": 6, "symmetry": 7}
TRANSIENT = {"euler": 0, "cranknicolson1": 1, "cranknicolson2": 2, "adamsmoulton": 3}
# gradient interpolation
GI_AVERAGE, GI_UPWIND, GI_DOWNWIND, GI_AVERAGECORRECTED = 0, 1, 2, 3
HR_NONE, HR_TVD = 0, 1
TVD = {n: i for i, n in enumerate(["upwind", "downwind", "fromm", "sou", "cd", "quick", "superbee", "minmod",
                                    "osher", "vanleer", "muscl", "smart", "hquick", "umist", "charm"])}
SOLVER = {"sor": 0, "bicgs": 1, "amg": 2, "amg_bicgs": 3, "amg32_bicgs": 4, "gmres": 5, "ilu": 6, "amg32gs_bicgs": 7, "pbcg": 8}
SIMPLE, SIMPLEC = 0, 1

FIELDS = ["u", "v", "w", "p", "pc", "mdot", "bu", "bv", "bw", "bp", "bpc", "bmdot", "ac", "bc", "anb",
          "du1", "dv1", "dw1", "du2", "dv2", "dw2", "ugrad", "vgrad", "wgrad", "pgrad", "pcgrad",
          "volume", "xc", "gfactor", "sf", "gdiff", "ft", "bsf", "dphi",
          "tke", "ted", "mut", "btke", "bted", "bmut", "kx", "utau", "yplus",
          "old", "oldold", "bold", "temp", "btemp", "tgrad"]
FIELD_ID = {n: i for i, n in enumerate(FIELDS)}


class FsCase(C.Structure):
    _fields_ = [
        ("rho", C.c_double), ("mu", C.c_double), ("algorithm", C.c_int), ("relax_momentum", C.c_int),
        ("urf_momentum", C.c_double), ("urf_pressure", C.c_double),
        ("method_grad_mom", C.c_int), ("method_grad_cont", C.c_int),
        ("niter_grad_mom", C.c_int), ("niter_grad_cont", C.c_int),
        ("grad_interp_mom", C.c_int), ("grad_interp_cont", C.c_int),
        ("method_decompose_s", C.c_int), ("hr_framework", C.c_int), ("conv_scheme", C.c_int),
        ("niter_start_hr", C.c_int), ("bleed", C.c_double),
        ("solver_mom", C.c_int), ("solver_cont", C.c_int),
        ("rrf_mom", C.c_double), ("rrf_cont", C.c_double),
        ("itmax_mom", C.c_int), ("itmax_cont", C.c_int),
        ("nstop_type", C.c_int), ("max_residual", C.c_double),
        ("ref_pressure_cell", C.c_int), ("set_reference_pressure", C.c_int), ("inviscid", C.c_int),
        ("mg_cycle", C.c_int), ("mg_pre", C.c_int), ("mg_post", C.c_int), ("mg_max_cycles", C.c_int),
        ("mg_min_parents", C.c_int), ("mg_max_levels", C.c_int), ("mg_rrf", C.c_double),
        ("krylov_maxit", C.c_int), ("krylov_tol", C.c_double),
        ("n_patches", C.c_int), ("patch_type", C.c_int * FS_MAX_PATCHES),
        ("patch_vel", (C.c_double * 3) * FS_MAX_PATCHES),
        ("batched_momentum", C.c_int),
        ("mass_flow_fraction", C.c_double * FS_MAX_PATCHES),
        ("turbulence", C.c_int), ("solver_turb", C.c_int),
        ("rrf_tke", C.c_double), ("rrf_ted", C.c_double),
        ("itmax_tke", C.c_int), ("itmax_ted", C.c_int),
        ("urf_tke", C.c_double), ("urf_ted", C.c_double), ("urf_tvisc", C.c_double),
        ("max_visc_ratio", C.c_double), ("limit_production", C.c_int),
        ("conv_scheme_tke", C.c_int), ("conv_scheme_ted", C.c_int),
        ("inlet_intensity", C.c_double * FS_MAX_PATCHES), ("inlet_length", C.c_double * FS_MAX_PATCHES),
        ("wall_function", C.c_int),
        ("patch_pressure", C.c_double * FS_MAX_PATCHES),
        ("unsteady", C.c_int), ("transient_scheme", C.c_int), ("dt", C.c_double),
        ("patch_mass_flow", C.c_double * FS_MAX_PATCHES),
        ("patch_resistance", C.c_double * FS_MAX_PATCHES),
        ("energy", C.c_int), ("cp", C.c_double), ("conductivity", C.c_double), ("temp_init", C.c_double),
        ("solver_energy", C.c_int), ("rrf_energy", C.c_double), ("itmax_energy", C.c_int),
        ("relax_energy", C.c_int), ("urf_energy", C.c_double), ("conv_scheme_energy", C.c_int),
        ("bleed_energy", C.c_double), ("method_grad_energy", C.c_int), ("niter_grad_energy", C.c_int),
        ("grad_interp_energy", C.c_int), ("gamma_interp_energy", C.c_int),
        ("energy_sc", C.c_double), ("energy_sb", C.c_double),
        ("limit_temperature", C.c_int), ("temp_min", C.c_double), ("temp_max", C.c_double),
        ("sigma_t", C.c_double), ("energy_wall_function", C.c_int),
        ("patch_thermal", C.c_int * FS_MAX_PATCHES), ("patch_temperature", C.c_double * FS_MAX_PATCHES),
        ("patch_heat_flux", C.c_double * FS_MAX_PATCHES), ("patch_h_inf", C.c_double * FS_MAX_PATCHES),
        ("pc_history", C.c_int), ("pc_refresh", C.c_int),
    ]


class FsMeshIn(C.Structure):
    _fields_ = [
        ("n_nodes", C.c_int32), ("points", C.POINTER(C.c_double)),
        ("n_faces", C.c_int32), ("face_ptr", C.POINTER(C.c_int32)), ("face_nodes", C.POINTER(C.c_int32)),
        ("owner", C.POINTER(C.c_int32)), ("n_internal", C.c_int32), ("neighbour", C.POINTER(C.c_int32)),
        ("n_patches", C.c_int32), ("patch_start", C.POINTER(C.c_int32)), ("patch_size", C.POINTER(C.c_int32)),
        ("cell_face_ptr", C.POINTER(C.c_int32)), ("cell_faces", C.POINTER(C.c_int32)),
        ("cell_node_ptr", C.POINTER(C.c_int32)), ("cell_nodes", C.POINTER(C.c_int32)),
    ]


class FsNeuIn(C.Structure):
    _fields_ = [
        ("n_elements", C.c_int32), ("type", C.POINTER(C.c_int32)), ("node_ptr", C.POINTER(C.c_int32)),
        ("nodes", C.POINTER(C.c_int32)), ("n_sets", C.c_int32), ("set_size", C.POINTER(C.c_int32)),
        ("bc_element", C.POINTER(C.c_int32)), ("bc_face", C.POINTER(C.c_int32)),
    ]


class FsResiduals(C.Structure):
    _fields_ = [
        ("abs_", C.c_double * 5), ("max_", C.c_double * 5), ("rms", C.c_double * 5), ("scaled", C.c_double * 5),
        ("overall_imbalance", C.c_double), ("imax_imbalance", C.c_int), ("lin_iters", C.c_int * 5),
        ("source", C.c_double),
        ("turb_abs", C.c_double * 2), ("turb_max", C.c_double * 2), ("turb_rms", C.c_double * 2),
        ("turb_scaled", C.c_double * 2), ("turb_lin_iters", C.c_int * 2),
        ("temp_abs", C.c_double), ("temp_max", C.c_double), ("temp_rms", C.c_double), ("temp_scaled", C.c_double),
        ("temp_lin_iters", C.c_int),
    ]

    def as_dict(self) -> dict:
        return {"abs": list(self.abs_), "max": list(self.max_), "rms": list(self.rms), "scaled": list(self.scaled),
                "overall_imbalance": self.overall_imbalance, "imax_imbalance": self.imax_imbalance,
                "lin_iters": list(self.lin_iters), "source": self.source,
                "turb_abs": list(self.turb_abs), "turb_max": list(self.turb_max), "turb_rms": list(self.turb_rms),
                "turb_scaled": list(self.turb_scaled), "turb_lin_iters": list(self.turb_lin_iters),
                "temp_abs": self.temp_abs, "temp_max": self.temp_max, "temp_rms": self.temp_rms,
                "temp_scaled": self.temp_scaled, "temp_lin_iters": self.temp_lin_iters}


# every entry point of include/fsb200.h with its argument types
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int32)
_V = C.c_void_p
PROTOTYPES = {
    "fs_create": (C.c_int, [C.POINTER(FsMeshIn), C.POINTER(FsCase), C.c_int, C.POINTER(C.c_void_p)]),
    "fs_destroy": (C.c_int, [_V]),
    "fs_sizes": (C.c_int, [_V, _I, _I, _I, _I]),
    "fs_last_error": (C.c_char_p, [_V]),
    "fs_solve_momentum": (C.c_int, [_V, C.c_int]),
    "fs_solve_continuity": (C.c_int, [_V]),
    "fs_solve_energy": (C.c_int, [_V]),
    "fs_set_pc_history": (C.c_int, [_V, C.c_int]),
    "fs_simple_iteration": (C.c_int, [_V, C.POINTER(FsResiduals)]),
    "fs_simple_iteration_host": (C.c_int, [_V, _D, _D, _D, _D, _D, _D, _D, _D, _D, _D, C.POINTER(FsResiduals)]),
    "fs_assemble_momentum": (C.c_int, [_V, C.c_int]),
    "fs_assemble_continuity": (C.c_int, [_V]),
    "fs_correct_continuity": (C.c_int, [_V]),
    "fs_set_iteration": (C.c_int, [_V, C.c_int]),
    "fs_initialize_mdot": (C.c_int, [_V]),
    "fs_advance_time": (C.c_int, [_V, C.c_double]),
    "fs_adaptive_time_step": (C.c_int, [_V, C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double)]),
    "fs_neu_connectivity": (C.c_int, [C.POINTER(FsNeuIn)] + [C.POINTER(C.c_int32)] * 8),
    "fs_get_time": (C.c_int, [_V, C.POINTER(C.c_double), C.POINTER(C.c_int32)]),
    "fs_set_time": (C.c_int, [_V, C.POINTER(C.c_double), C.c_int32]),
    "fs_gradient": (C.c_int, [_V, C.c_int, C.c_int, C.c_int]),
    "fs_gradient_host": (C.c_int, [_V, C.c_int, C.c_int, C.c_int, _D, _D, _D, _D]),
    "fs_under_relax": (C.c_int, [_V, C.c_double]),
    "fs_solve_equation": (C.c_int, [_V, C.c_int, C.c_double, C.c_int, C.c_int]),
    "fs_solve_system_host": (C.c_int, [_V, _D, _D, _D, _D, C.c_double, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "fs_residuals_get": (C.c_int, [_V, C.POINTER(FsResiduals)]),
    "fs_get_field": (C.c_int, [_V, C.c_int, _D, C.c_size_t]),
    "fs_set_field": (C.c_int, [_V, C.c_int, _D, C.c_size_t]),
    "fs_get_connectivity": (C.c_int, [_V, _I, _I, _I, _I, _I]),
    "fs_mg_levels": (C.c_int, [_V, _I, _I, C.c_int]),
    "fs_mg_parents": (C.c_int, [_V, C.c_int, _I, C.c_size_t]),
    "fs_mg_info": (C.c_int, [_V, _I, C.c_int, _I, _I]),
    "fs_mg_coarse_matrix": (C.c_int, [_V, C.c_int, _D, _I, _I, _D, C.c_size_t, C.c_size_t]),
    "fs_solver_kernel_ms": (C.c_int, [_V, C.POINTER(C.c_float)]),
    "fs_nn_create": (C.c_int, [_V, C.c_int, C.c_uint64]),
    "fs_nn_mode": (C.c_int, [_V, C.c_int, C.c_int]),
    "fs_nn_snapshots": (C.c_int, [_V, _I]),
    "fs_nn_train": (C.c_int, [_V, C.c_int, C.c_float, C.c_uint64, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "fs_nn_params": (C.c_int, [_V, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_size_t]),
    "fs_nn_eval_host": (C.c_int, [_V] + [C.POINTER(C.c_float)] * 6),
    "fs_nn_stats": (C.c_int, [_V, _I, _I]),
    "fs_nn_policy": (C.c_int, [_V, _D, _D, _I]),
    "fs_set_launch_shape": (C.c_int, [_V, C.c_int]),
    "fs_test_wait_timeout": (C.c_int, [_V, C.c_int]),
    "fs_ensemble_run": (C.c_int, [C.POINTER(_V), C.c_int, C.c_int, C.c_int, _D, _I, C.POINTER(C.c_float)]),
    "fs_ensemble_run_batched": (C.c_int, [C.POINTER(_V), C.c_int, C.c_int, C.c_int, _D, _I, C.POINTER(C.c_float)]),
    "fs_ensemble_split": (C.c_int, [_V, C.c_double]),
    "fs_phase_times": (C.c_int, [_V, C.POINTER(C.c_float)]),
    "fs_timer_start": (C.c_int, [_V]),
    "fs_timer_stop": (C.c_int, [_V, C.POINTER(C.c_float)]),
    "fs_solver_stats": (C.c_int, [_V, C.POINTER(C.c_float), _I, _I, C.c_int]),
    "fs_launch_count": (C.c_int64, [_V]),
    "fs_sync": (C.c_int, [_V]),
    "fs_bicgstab_noalloc": (C.c_int, [C.c_int32, C.c_int32, _V, _V, _V, _V, _V, _V, C.c_int32, C.c_double, _V, _V]),
}

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libfsb200.so (building nothing): raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: run flowsolversourcecode_b200.build.build() first")
    lib = C.CDLL(path)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I)


def fptr(a):
    if a is None:
        return None
    assert a.dtype == np.float32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_float))


class FsError(RuntimeError):
    """A non-zero status of a C-ABI call; `status` holds the FS_E_* code."""

    def __init__(self, message: str, status: int = 0):
        super().__init__(message)
        self.status = status


def check(rc: int, ctx=None, what: str = "") -> None:
    if rc != FS_OK:
        msg = ""
        if ctx is not None and _lib is not None:
            m = _lib.fs_last_error(ctx)
            msg = m.decode() if m else ""
        raise FsError(f"{what} failed with status {rc}: {msg}", rc)


def mesh_struct(mesh) -> tuple[FsMeshIn, list]:
    """FsMeshIn view of a PolyMesh (keeps the numpy arrays alive in `keep`)."""
    pts = np.ascontiguousarray(mesh.points, np.float64).reshape(-1)
    fp = np.ascontiguousarray(mesh.face_ptr, np.int32)
    fn = np.ascontiguousarray(mesh.face_nodes, np.int32)
    ow = np.ascontiguousarray(mesh.owner, np.int32)
    nb = np.ascontiguousarray(mesh.neighbour, np.int32)
    ps = np.ascontiguousarray(mesh.patch_start, np.int32)
    pz = np.ascontiguousarray(mesh.patch_size, np.int32)
    keep = [pts, fp, fn, ow, nb, ps, pz]
    m = FsMeshIn(n_nodes=pts.shape[0] // 3, points=dptr(pts), n_faces=ow.shape[0], face_ptr=iptr(fp),
                 face_nodes=iptr(fn), owner=iptr(ow), n_internal=nb.shape[0], neighbour=iptr(nb),
                 n_patches=ps.shape[0], patch_start=iptr(ps), patch_size=iptr(pz))
    # element-local face order and element node order of a neutral-file mesh
    for name in ("cell_face_ptr", "cell_faces", "cell_node_ptr", "cell_nodes"):
        a = getattr(mesh, name, None)
        if a is not None:
            a = np.ascontiguousarray(a, np.int32)
            keep.append(a)
            setattr(m, name, iptr(a))
    return m, keep
