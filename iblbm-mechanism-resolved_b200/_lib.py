"""ctypes binding of ``libiblbm_b200.so`` (declarations in include/iblbm_b200.h).

The library is built in-tree by ``build.py``.  Loading fails loudly when it is
missing: there is no CPU fallback for any operation of this package.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libiblbm_b200.so")

COLL_IDS = {"BGK": 0, "TRT": 1, "CM_MRT": 2}
BC_IDS = {"dirichlet_neumann": 0, "open_boundary": 1, "settling_channel": 2, "velocity_inlet": 3,
          "tg_analytical": 4}
IBM_IDS = {"NONE": 0, "DF": 1, "MDF": 2, "DFC": 3}
DELTA_IDS = {"peskin4pt": 0, "hat": 1}
DELTA_RADIUS = {"peskin4pt": 2, "hat": 1}

_vp = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double


class Geom(ctypes.Structure):
    _fields_ = [("nx", _i), ("ny", _i), ("pitch", _i), ("qstride", ctypes.c_longlong)]


class Case(ctypes.Structure):
    _fields_ = [("collision", _i), ("bc", _i), ("incompressible", _i), ("tau", _d), ("dt", _d),
                ("s_minus", _d), ("S", _d * 9), ("inflow_u", _d), ("dens", _d), ("tg_face", _vp),
                ("tg_decay", _vp)]


class BandView(ctypes.Structure):
    _fields_ = [("box", _vp), ("map", _vp), ("fib", _vp), ("df", _vp)]


class DenseArgs(ctypes.Structure):
    _fields_ = [("g", Geom), ("c", Case), ("ibm", _i), ("fpost_prev", _vp), ("fpost_next", _vp),
                ("uring_prev", _vp), ("uring_next", _vp), ("band", BandView), ("ro_out", _vp),
                ("U_out", _vp), ("fstar_out", _vp), ("skip_box", _vp), ("only_box", _vp), ("box_blocks", _i)]


class IbmArgs(ctypes.Structure):
    _fields_ = [("g", Geom), ("c", Case), ("method", _i), ("delta_type", _i), ("rebuild", _i),
                ("n_particles", _i), ("lb_total", _i), ("moff", _vp), ("Lx", _vp), ("Ly", _vp),
                ("dvel", _vp), ("larea", _vp), ("dx", _d), ("dy", _d), ("Lx_c", _vp), ("Ly_c", _vp),
                ("xt_table", _vp), ("step_counter", _vp), ("xt_len", _i), ("mdf_iterations", _i),
                ("mdf_min_iterations", _i), ("mdf_coupled", _i), ("mdf_omega", _d), ("mdf_tol", _d),
                ("mdf_omega_max", _d), ("lambda_", _vp), ("lambda_valid", _vp), ("dfc_cache_lambda", _i),
                ("correction_scale", _d), ("fpost_prev", _vp), ("uring_prev", _vp), ("box", _vp),
                ("map", _vp), ("band_nodes", _vp), ("band_count", _vp), ("list_cache", _vp), ("excl_cur", _vp),
                ("excl_next", _vp), ("band_capacity", _i),
                ("box_capacity", _i), ("band_fib", _vp), ("band_df", _vp), ("band_fib_part", _vp),
                ("scratch", _vp), ("iscratch", _vp), ("Lux", _vp), ("Luy", _vp), ("Lfx", _vp),
                ("Lfy", _vp), ("dfc_force", _vp), ("stats", _vp), ("dstats", _vp), ("field_ro", _vp),
                ("field_ux", _vp), ("field_uy", _vp), ("field_fstar", _vp), ("field_ustride", _i),
                ("dvel_scale", _vp), ("dfc_rho_f", _d), ("wait_limit", ctypes.c_longlong), ("test_skip_copy", _i),
                ("cluster_plan", _vp), ("cluster_size", _i), ("df_given_force", _i)]


# The FP32 structs have the FP64 ones' fields in the same order (only pointee
# types differ) and add their own at the end: the learned warm start for the
# band step, the tile choice for the dense pass.
class Ibm32Args(ctypes.Structure):
    _fields_ = IbmArgs._fields_ + [("mlp_mode", _i), ("mlp_uref", ctypes.c_float), ("mlp_re", ctypes.c_float),
                                   ("mlp_params", _vp), ("mlp_features", _vp), ("mlp_targets", _vp)]


class Dense32Args(ctypes.Structure):
    _fields_ = DenseArgs._fields_ + [("tile", _i), ("status", _vp), ("wait_limit", ctypes.c_longlong),
                                     ("test_skip_copy", _i)]


TILES = {"pipe4x2": 0, "node": 1, "pipe8x2": 2, "rows2": 3, "rows4": 4}

class ParticlesArgs(ctypes.Structure):
    _fields_ = [("n_particles", _i), ("phase", _i), ("model", _i), ("fib_f32", _i), ("moff", _vp), ("Lx_c", _vp),
                ("Ly_c", _vp), ("Lx", _vp), ("Ly", _vp), ("dvel", _vp), ("state", _vp), ("consts", _vp),
                ("dt", _d), ("dx", _d), ("band_fib_part", _vp), ("band_count", _vp), ("band_capacity", _i),
                ("forces_out", _vp), ("n_nodes", _i), ("band_nodes", _vp), ("pw_leaves", _i), ("pw_internal", _i),
                ("pw_levels", _i), ("pw_leaf", _vp), ("pw_node", _vp), ("pw_level", _vp), ("pw_lut", _vp),
                ("pw_span", _vp), ("pw_scratch", _vp), ("rotation", _i), ("semi_implicit", _i),
                ("euler_trapezoidal", _i), ("nx", _i), ("dy", _d), ("rho", _vp), ("U", _vp), ("moments_f32", _i),
                ("ny", _i), ("lint_scratch", _vp), ("lint_capacity", _i), ("lagrangian", _i), ("Lfx", _vp),
                ("Lfy", _vp), ("dfc_force", _vp), ("half_kick_omega", _i),
                ("prescribed", _i), ("prescribed_velocity", _d * 2)]


PARTICLE_STATE, PARTICLE_CONSTS = 22, 10  # doubles per particle (IBLBM_PARTICLE_STATE / _CONSTS)


INERTIA_IDS = {"none": 0, "explicit_history": 1, "feng_b2": 2}


class ForceCoeffArgs(ctypes.Structure):
    _fields_ = [("ro", _vp), ("n_nodes", _i), ("f32", _i), ("method", _i), ("band_fib", _vp), ("band_count", _vp),
                ("dfc_force", _vp), ("lb_total", _i), ("u_ref", _d), ("lattice_r", _d), ("partials", _vp),
                ("ticket", _vp), ("ring", _vp), ("ring_len", _i), ("ring_pos", _vp)]


class VelocityChangeArgs(ctypes.Structure):
    _fields_ = [("U", _vp), ("U_prev", _vp), ("n_nodes", _i), ("f32", _i), ("partials", _vp), ("ticket", _vp),
                ("out", _vp)]

# entry point -> argtypes (all return int status)
_SIGS = {
    "iblbm_dense_step_f64": [ctypes.POINTER(DenseArgs), _vp],
    "iblbm_ibm_step_f64": [ctypes.POINTER(IbmArgs), _vp],
    "iblbm_ibm_step_f64_noalloc": [ctypes.POINTER(IbmArgs), _vp],
    "iblbm_ibm_scratch_doubles": [_i, _i, _i],
    "iblbm_ibm_scratch_ints": [_i, _i, _i],
    "iblbm_ibm_list_cache_ints": [_i, _i, _i],
    "iblbm_ibm_cluster_plan_ints": [_i, _i, _i],
    "iblbm_ibm_smem_bytes": [_i, _i, _i],
    "iblbm_feq": [_vp, _vp, _i, _i, _vp, _vp],
    "iblbm_macroscopic": [_vp, _i, _i, _vp, _vp, _vp],
    "iblbm_collision_bgk": [_vp, _vp, _vp, _vp, _i, _d, _d, _vp, _vp],
    "iblbm_collision_trt": [_vp, _vp, _vp, _vp, _i, _d, _d, _d, _vp, _vp],
    "iblbm_collision_cm_mrt": [_vp, _vp, _vp, _i, ctypes.POINTER(_d), _d, _vp, _vp],
    "iblbm_streaming": [_vp, _vp, _i, _i, _vp, _vp],
    "iblbm_velocity_correction": [_vp, _vp, _vp, _i, _d, _i, _vp],
    "iblbm_dense_step_f32": [ctypes.POINTER(Dense32Args), _vp],
    "iblbm_ibm_step_f32": [ctypes.POINTER(Ibm32Args), _vp],
    "iblbm_ibm_step_f32_batch": [ctypes.POINTER(Ibm32Args), _vp, _i, _vp],
    "iblbm_mlp_param_count": [],
    "iblbm_mlp_infer": [_vp, _vp, _i, _vp, _vp],
    "iblbm_mlp_grad_floats": [_i],
    "iblbm_mlp_train_step": [_vp, _vp, _vp, _vp, _vp, _vp, _i, ctypes.c_float, _i, _vp, _i, _vp],
    "iblbm_dense_step_f32_batch": [ctypes.POINTER(Dense32Args), _i, _vp],
    "iblbm_dense_step_f64_batch": [ctypes.POINTER(DenseArgs), _i, _vp],
    "iblbm_ibm_step_f64_batch": [ctypes.POINTER(IbmArgs), _vp, _i, _vp],
    "iblbm_ibm32_list_cache_ints": [_i, _i, _i],
    "iblbm_ibm32_smem_bytes": [_i, _i, _i],
    "iblbm_to_shifted_f32": [_vp, Geom, _vp, _vp],
    "iblbm_from_shifted_f32": [_vp, Geom, _vp, _vp],
    "iblbm_particles_step_f64": [ctypes.POINTER(ParticlesArgs), _vp],
    "iblbm_force_coeffs": [ctypes.POINTER(ForceCoeffArgs), _vp],
    "iblbm_velocity_change": [ctypes.POINTER(VelocityChangeArgs), _vp],
    "iblbm_diag_partials": [_i],
    "iblbm_aos_to_soa": [_vp, Geom, _vp, _vp],
    "iblbm_soa_to_aos": [_vp, Geom, _vp, _vp],
}

ERRORS = {-1: "invalid argument", -2: "CUDA launch error", -3: "capacity exceeded"}

_lib = None


def lib() -> ctypes.CDLL:
    """Load the CUDA library; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python {HERE}/build.py` "
                               "(this package has no CPU fallback)")
        _lib = ctypes.CDLL(LIB_PATH)
        for name, argtypes in _SIGS.items():
            fn = getattr(_lib, name)
            fn.argtypes = argtypes
            fn.restype = ctypes.c_int
    return _lib


def check(rc: int, what: str) -> None:
    if rc != 0:
        raise RuntimeError(f"{what} failed: {ERRORS.get(rc, rc)}")


def ptr(t) -> int:
    """Device pointer of a torch tensor (None -> NULL)."""
    return 0 if t is None else t.data_ptr()
