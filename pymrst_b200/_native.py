"""ctypes binding of libpymrst_b200.so (declarations in include/pymrst_b200.h).

The library is loaded from this package's folder.  There is no fallback: if
it is missing or a CUDA device is absent, the calls that need it raise.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libpymrst_b200.so"

PMB_OK = 0
ERROR_NAMES = {1: "CUDA error", 2: "invalid argument", 3: "non-finite value", 4: "zero pivot",
               5: "no convergence", 6: "allocation failure", 7: "internal error"}

c_int = C.c_int32
c_i64 = C.c_int64
c_dbl = C.c_double
c_vp = C.c_void_p
P_i32 = C.POINTER(C.c_int32)
P_i64 = C.POINTER(C.c_int64)
P_dbl = C.POINTER(C.c_double)


class OWDesc(C.Structure):
    _fields_ = [
        ("nc", c_int), ("nf", c_int), ("nw", c_int),
        ("h_N", P_i32), ("h_T", P_dbl), ("h_gdz", P_dbl), ("h_pv", P_dbl),
        ("mu", c_dbl * 2), ("rhoS", c_dbl * 2), ("n_exp", c_dbl * 2), ("c", c_dbl * 2),
        ("b0", c_dbl * 2), ("sl", c_dbl * 2), ("su", c_dbl * 2), ("p_ref", c_dbl),
        ("h_perf_ptr", P_i32), ("h_perf_cell", P_i32), ("h_perf_WI", P_dbl), ("h_perf_dZ", P_dbl),
        ("h_compi", P_dbl), ("h_well_type", P_i32), ("h_well_val", P_dbl),
        ("gravity", c_dbl),
        ("tol_cnv", c_dbl), ("tol_mb", c_dbl), ("tol_well", c_dbl), ("ds_max", c_dbl),
        ("dp_max_rel", c_dbl),
        ("h_line_face", P_i32),
    ]


class CPROpts(C.Structure):
    _fields_ = [
        ("rtol", c_dbl), ("maxiter", c_int), ("restart", c_int), ("precision", c_int),
        ("use_pressure_stage", c_int), ("local_sweeps", c_int), ("amg_smoother_degree", c_int),
        ("amg_cycle", c_int), ("amg_theta", c_dbl), ("amg_coarse_size", c_int),
        ("amg_rebuild_interval", c_int), ("inner_rtol", c_dbl), ("replay_graph", c_int),
        ("amg_coarse_degree", c_int),
    ]


class TpfaDesc(C.Structure):
    _fields_ = [
        ("nc", c_int), ("nf", c_int), ("nhf", c_int), ("dim", c_int),
        ("h_face_pos", P_i32), ("h_cell_faces", P_i32), ("h_neighbors", P_i32),
        ("h_cell_centroids", P_dbl), ("h_face_centroids", P_dbl),
        ("nw", c_int), ("h_perf_ptr", P_i32), ("h_perf_cell", P_i32), ("h_well_rate", P_i32),
        ("use_trans", c_int),
    ]


class TpfaForces(C.Structure):
    _fields_ = [
        ("d_T", c_vp), ("d_mob", c_vp), ("nph", c_int), ("h_rho", P_dbl),
        ("gravity", c_dbl * 3), ("well_gravity", c_dbl),
        ("nbc", c_int), ("h_bc_face", P_i32), ("h_bc_type", P_i32), ("h_bc_value", P_dbl),
        ("nsrc", c_int), ("h_src_cell", P_i32), ("h_src_rate", P_dbl),
        ("h_well_val", P_dbl), ("d_perf_WI", c_vp), ("d_perf_dZ", c_vp),
        ("ncompi", c_int), ("h_compi", P_dbl), ("h_injector", P_i32),
    ]


class BODesc(C.Structure):
    _fields_ = [
        ("nc", c_int), ("nf", c_int), ("nw", c_int),
        ("h_N", P_i32), ("h_T", P_dbl), ("h_gdz", P_dbl), ("h_pv", P_dbl),
        ("rhoS", c_dbl * 3), ("pvtw", c_dbl * 4), ("rock", c_dbl * 2), ("swcon", c_dbl),
        ("n_gas", c_int), ("h_gas_p", P_dbl), ("h_gas_b", P_dbl), ("h_gas_mu", P_dbl),
        ("n_rssat", c_int), ("h_rssat_p", P_dbl), ("h_rssat_rs", P_dbl),
        ("n_key", c_int), ("h_key", P_dbl), ("h_branch_ptr", P_i32), ("h_branch_p", P_dbl),
        ("h_branch_b", P_dbl), ("h_branch_mu", P_dbl),
        ("n_sw", c_int), ("h_sw", P_dbl), ("h_krw", P_dbl), ("h_pcow", P_dbl),
        ("n_sow", c_int), ("h_sow", P_dbl), ("h_krow", P_dbl),
        ("n_sg", c_int), ("h_sg", P_dbl), ("h_krg", P_dbl), ("h_pcog", P_dbl),
        ("n_sog", c_int), ("h_sog", P_dbl), ("h_krog", P_dbl),
        ("h_perf_ptr", P_i32), ("h_perf_cell", P_i32), ("h_perf_WI", P_dbl), ("h_well_type", P_i32),
        ("h_well_val", P_dbl), ("h_compi", P_dbl),
        ("tol_cnv", c_dbl), ("tol_mb", c_dbl), ("tol_well", c_dbl), ("ds_max", c_dbl),
    ]


# name -> (restype, argtypes)
SIGNATURES = {
    "pmb_last_error": (C.c_char_p, []),
    "pmb_version": (c_int, []),
    "pmb_launch_count": (c_int, [P_i64]),
    "pmb_profile_report": (c_int, [C.c_char_p, c_int, c_int]),
    "pmb_compute_trans": (c_int, [c_i64, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_int, c_vp, c_vp]),
    "pmb_compute_geometry3d": (c_int, [c_int, c_int] + [c_vp] * 13),
    "pmb_face_trans": (c_int, [c_i64, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_dense_inverse": (c_int, [c_int, c_vp, c_vp, c_vp]),
    "pmb_ow_create": (c_int, [C.POINTER(OWDesc), c_vp, C.POINTER(c_vp)]),
    "pmb_ow_destroy": (c_int, [c_vp]),
    "pmb_ow_sizes": (c_int, [c_vp, P_i64]),
    "pmb_ow_pattern": (c_int, [c_vp, P_i32, P_i32]),
    "pmb_ow_compute_cdp": (c_int, [c_vp, c_vp, c_vp]),
    "pmb_ow_reset_cdp": (c_int, [c_vp]),
    "pmb_ow_set_controls": (c_int, [c_vp, P_dbl]),
    "pmb_ow_prev_jacobian_tmul": (c_int, [c_vp, c_vp, c_dbl, c_vp, c_vp]),
    "pmb_ow_csr_values": (c_int, [c_vp, c_vp, c_vp, c_i64, c_vp, c_vp, c_vp]),
    "pmb_ow_perm_contract": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_ow_get_last_cdp": (c_int, [c_vp, c_vp, P_i32]),
    "pmb_ow_set_last_cdp": (c_int, [c_vp, c_vp]),
    "pmb_ow_fluxes": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_ow_assemble": (c_int, [c_vp, c_vp, c_vp, c_dbl, c_vp, c_vp, c_vp, c_vp, c_int]),
    "pmb_ow_spmv": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_ow_convergence": (c_int, [c_vp, c_vp, c_vp, c_dbl, P_dbl]),
    "pmb_ow_update": (c_int, [c_vp, c_vp, c_vp, c_dbl]),
    "pmb_ow_cnv_mb_noalloc": (c_int, [c_int, c_vp, c_vp, c_vp, c_dbl, P_dbl, c_dbl, c_vp, c_vp]),
    "pmb_cpr_default_opts": (c_int, [C.POINTER(CPROpts)]),
    "pmb_cpr_create": (c_int, [c_vp, C.POINTER(CPROpts), C.POINTER(c_vp)]),
    "pmb_cpr_destroy": (c_int, [c_vp]),
    "pmb_cpr_setup": (c_int, [c_vp, c_vp, c_vp, c_vp]),
    "pmb_cpr_solve": (c_int, [c_vp, c_vp, c_vp, P_dbl]),
    "pmb_cpr_levels": (c_int, [c_vp, c_int, P_i64, P_i32]),
    "pmb_cpr_bytes": (c_int, [c_vp, P_dbl]),
    "pmb_cpr_time_stage": (c_int, [c_vp, c_int, c_vp, c_vp, c_int, P_dbl]),
    "pmb_cpr_time_level": (c_int, [c_vp, c_int, c_int, P_dbl, P_i64]),
    "pmb_ow_step": (c_int, [c_vp, c_vp, c_vp, c_dbl, c_int, P_dbl]),
    "pmb_ow_step_members": (c_int, [c_vp, c_vp, c_vp, c_dbl, c_int, c_int, P_i32, P_i32, P_i32, P_i32, P_dbl]),
    "pmb_csr_cpr_create": (c_int, [c_int, c_int, c_int, P_i32, P_i32, c_int, C.POINTER(CPROpts), c_vp,
                                   C.POINTER(c_vp)]),
    "pmb_csr_cpr_destroy": (c_int, [c_vp]),
    "pmb_csr_cpr_setup": (c_int, [c_vp, c_vp, P_dbl]),
    "pmb_csr_cpr_solve": (c_int, [c_vp, c_vp, c_vp, P_dbl]),
    "pmb_csr_cpr_set_cell_weights": (c_int, [c_vp, c_int]),
    "pmb_csr_spmv": (c_int, [c_vp, c_vp, c_vp, c_vp]),
    "pmb_csr_row_scale": (c_int, [c_int, c_vp, c_vp, c_vp, c_vp]),
    "pmb_csr_cpr_levels": (c_int, [c_vp, c_int, P_i64, P_i32]),
    "pmb_pcg_create": (c_int, [c_int, P_i32, P_i32, c_dbl, c_int, c_vp, C.POINTER(c_vp)]),
    "pmb_pcg_destroy": (c_int, [c_vp]),
    "pmb_pcg_setup": (c_int, [c_vp, c_vp]),
    "pmb_pcg_solve": (c_int, [c_vp, c_vp, c_vp, c_dbl, c_int, P_dbl]),
    "pmb_pcg_levels": (c_int, [c_vp, c_int, P_i64, P_i32]),
    "pmb_tpfa_create": (c_int, [C.POINTER(TpfaDesc), c_vp, C.POINTER(c_vp)]),
    "pmb_tpfa_destroy": (c_int, [c_vp]),
    "pmb_tpfa_sizes": (c_int, [c_vp, P_i64]),
    "pmb_tpfa_pattern": (c_int, [c_vp, P_i32, P_i32]),
    "pmb_tpfa_assemble": (c_int, [c_vp, C.POINTER(TpfaForces), c_vp, c_vp]),
    "pmb_tpfa_solve": (c_int, [c_vp, c_vp, c_vp, c_vp, c_dbl, c_int, P_dbl]),
    "pmb_tpfa_reconstruct": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "pmb_tpfa_levels": (c_int, [c_vp, c_int, P_i64, P_i32]),
    "pmb_transport_create": (c_int, [c_int, c_int, P_i32, P_dbl, c_vp, C.POINTER(c_vp)]),
    "pmb_transport_destroy": (c_int, [c_vp]),
    "pmb_transport_pattern": (c_int, [c_vp, P_i64, P_i32, P_i32]),
    "pmb_transport_set_flow": (c_int, [c_vp, c_vp, c_vp, c_vp, P_dbl]),
    "pmb_transport_residual": (c_int, [c_vp, c_vp, c_vp, c_dbl, c_vp, P_dbl]),
    "pmb_transport_jacobian": (c_int, [c_vp, c_vp, c_dbl, c_vp]),
    "pmb_transport_explicit": (c_int, [c_vp, c_vp, c_dbl, c_dbl, c_dbl, c_dbl, c_dbl, c_dbl, P_dbl]),
    "pmb_transport_implicit": (c_int, [c_vp, c_vp, c_dbl, c_dbl, c_int, c_int, c_int, c_dbl,
                                       C.POINTER(CPROpts), P_dbl]),
    "pmb_bo_create": (c_int, [C.POINTER(BODesc), c_vp, C.POINTER(c_vp)]),
    "pmb_bo_destroy": (c_int, [c_vp]),
    "pmb_bo_sizes": (c_int, [c_vp, P_i64]),
    "pmb_bo_pattern": (c_int, [c_vp, P_i32, P_i32]),
    "pmb_bo_assemble": (c_int, [c_vp, c_vp, c_vp, c_dbl, c_vp, c_vp]),
    "pmb_bo_convergence": (c_int, [c_vp, c_vp, c_vp, c_dbl, P_dbl]),
    "pmb_bo_update": (c_int, [c_vp, c_vp, c_vp]),
    "pmb_bo_step": (c_int, [c_vp, c_vp, c_dbl, c_int, C.POINTER(CPROpts), P_dbl]),
    "pmb_bo_pvt_points": (c_int, [c_vp, c_int, c_vp, c_vp, c_vp, c_vp]),
    "pmb_bo_relperm_points": (c_int, [c_vp, c_int, c_vp, c_vp, c_vp]),
    "pmb_amg_hierarchy_host": (c_int, [c_int, P_i32, P_i32, P_dbl, c_dbl, c_int, c_int, P_i64, P_i32]),
}

_lib = None


def lib():
    """The loaded library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH.name} is not built; run `python -m pymrst_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class PMBError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERROR_NAMES.get(code, 'error')} ({code}): {msg}")
        self.code = code


def check(rc: int) -> None:
    if rc != PMB_OK:
        msg = lib().pmb_last_error().decode(errors="replace")
        raise PMBError(rc, msg)


def launch_count() -> int:
    v = C.c_int64()
    check(lib().pmb_launch_count(C.byref(v)))
    return int(v.value)


def profile_report(reset: bool = True) -> dict:
    """{phase: (total_ms, count)} collected under PMB_PROFILE=1."""
    buf = C.create_string_buffer(1 << 16)
    check(lib().pmb_profile_report(buf, len(buf), int(reset)))
    out = {}
    for line in buf.value.decode().splitlines():
        name, ms, cnt = line.split()
        out[name] = (float(ms), int(cnt))
    return out


def ptr(t) -> int:
    """Device (or host) address of a torch tensor / numpy array, as int."""
    if t is None:
        return 0
    if hasattr(t, "data_ptr"):
        return int(t.data_ptr())
    return int(t.ctypes.data)


def as_p(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype))
