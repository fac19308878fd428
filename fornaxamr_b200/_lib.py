"""ctypes bindings of libfornax_b200.so (declarations in include/fornax_b200.h).

The library is loaded from the package directory; there is no fallback: if
the native library is missing, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

from .layout import NG

HERE = os.path.dirname(os.path.abspath(__file__))
# the build with the ghost layers of this process (FX_NGHOST)
LIB_PATH = os.path.join(HERE, "libfornax_b200.so" if NG == 2 else f"libfornax_b200_ng{NG}.so")

FX_SUCCESS, FX_EINVAL, FX_ECUDA, FX_ENOMESH, FX_EPHYSICS, FX_ENOMEM, FX_ETOOBIG, FX_ECOMM = range(8)
NOALLOC_MAX_BLOCKS = 65536
DUMP_METADATA_SIZE = 639
BRANCH_OFF, BRANCH_RECORD, BRANCH_REPLAY = 0, 1, 2
FORM_PLAIN, FORM_BATCHED = 0, 1
BC_OUTFLOW, BC_REFLECT, BC_USER, BC_PERIODIC = 0, 1, 2, 3
ARR_W, ARR_EOSVAR, ARR_RHS, ARR_FLUX, ARR_VRIEMANN, ARR_GRAV, ARR_BF, ARR_BV1, ARR_BV2, ARR_EMF = (
    0, 1, 3, 4, 5, 6, 7, 8, 9, 10)


class FxSlot(C.Structure):
    _fields_ = [
        ("id", C.c_int32),
        ("rel_level", C.c_int32),
        ("type", C.c_int32),
        ("send_loc_start", C.c_int8 * 3),
        ("send_loc_end", C.c_int8 * 3),
        ("recv_loc_start", C.c_int8 * 3),
        ("recv_loc_end", C.c_int8 * 3),
    ]


class FxBlockDesc(C.Structure):
    _fields_ = [
        ("id", C.c_int32),
        ("level", C.c_int32),
        ("active", C.c_int32),
        ("rank", C.c_int32),
        ("xmin", C.c_double * 3),
        ("xmax", C.c_double * 3),
        ("dx", C.c_double * 3),
        ("vol", C.c_double),
        ("area", C.c_double * 3),
        ("slot", FxSlot * 56),
        ("parent", C.c_int32),
        ("children", C.c_int32 * 8),
        ("can_refine", C.c_int32),
    ]


class FxConfig(C.Structure):
    _fields_ = [
        ("mhd", C.c_int32),
        ("gravity", C.c_int32),
        ("gamma", C.c_double),
        ("coord", C.c_double * 6),
        ("bc", C.c_int32 * 6),
        ("mhd_eta", C.c_double),
        ("recon", C.c_int32),
        ("integrator", C.c_int32),
        ("use_bj", C.c_int32),
        ("pad", C.c_int32),
    ]


RECON_MC, RECON_WENO3, RECON_WENO7 = 0, 1, 2
INT_RK2, INT_ESSPRK10_4 = 0, 1

AMR_N = 4
AMR_LOEHNER, AMR_VELOCITY, AMR_PRESSURE_SCALE_HEIGHT, AMR_FRACTIONAL_JUMP = 0, 1, 2, 3
AMR_VAR_DENSITY, AMR_VAR_PRESSURE, AMR_VAR_TEMPERATURE = 0, 1, 2


class FxAmrCriterion(C.Structure):
    _fields_ = [
        ("set", C.c_int32),
        ("estimator", C.c_int32),
        ("lohner_var", C.c_int32),
        ("jump_var", C.c_int32),
        ("refine_thresh", C.c_double),
        ("derefine_thresh", C.c_double),
        ("lohner_eps", C.c_double),
    ]


class FxAmrConfig(C.Structure):
    _fields_ = [
        ("root_nx", C.c_int32 * 3),
        ("max_level", C.c_int32),
        ("max_blocks", C.c_int32),
        ("pad", C.c_int32),
        ("min_dx", C.c_double),
        ("reach_density", C.c_double),
        ("E_floor", C.c_double),
        ("crit", FxAmrCriterion * AMR_N),
    ]


# every entry point declared in include/fornax_b200.h
EXPORTS = [
    "fx_create", "fx_destroy", "fx_last_error", "fx_sync", "fx_stream", "fx_set_mesh",
    "fx_upload_block", "fx_download_block", "fx_upload_all", "fx_download_all",
    "fx_download_array", "fx_flux_update", "fx_mhd_update_emf", "fx_mhd_update_bf",
    "fx_update_cells", "fx_riemann_flux_send", "fx_mhd_emf_send", "fx_eos_fill_active_cells",
    "fx_eos_fill_mesh", "fx_boundary_fill_ghosts_and_bf", "fx_calc_dt", "fx_stage", "fx_step",
    "fx_run", "fx_plan_export", "fx_time_phase", "fx_info", "fx_upload_state", "fx_download_state",
    "fx_autotune", "fx_calc_dt_noalloc", "fx_mesh_slot_geometry", "fx_branch_trace", "fx_dump_gather", "fx_dump_metadata",
    "fx_upload_state_active", "fx_download_state_active", "fx_face_eval_host", "fx_face_vjp_host",
    "fx_adjoint_forward", "fx_adjoint_backward", "fx_adjoint_time", "fx_set_flux_shape",
    "fx_amr_configure", "fx_amr_tag", "fx_amr_adapt", "fx_get_mesh", "fx_amr_energy_injected",
    "fx_amr_remesh_host", "fx_amr_timings", "fx_shard_export", "fx_shard_set_mesh",
    "fx_shard_group_create", "fx_shard_group_destroy", "fx_shard_attach_group", "fx_nccl_unique_id",
    "fx_shard_attach_nccl", "fx_shard_info", "fx_ghost_layers",
]
PHASE_FLUX, PHASE_EMF, PHASE_CT, PHASE_CELLS, PHASE_GHOST, PHASE_STEP = range(6)


def load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m fornaxamr_b200.build` "
            "(the package has no CPU fallback)")
    L = C.CDLL(LIB_PATH, mode=C.RTLD_LOCAL)
    L.fx_ghost_layers.argtypes = []
    if L.fx_ghost_layers() != NG:
        raise ImportError(f"{LIB_PATH} was built with {L.fx_ghost_layers()} ghost layers, FX_NGHOST is {NG}")
    vp = C.c_void_p
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int32)
    dpp3 = C.POINTER(dp)
    L.fx_create.argtypes = [C.c_int, C.POINTER(FxConfig), C.POINTER(vp)]
    L.fx_destroy.argtypes = [vp]
    L.fx_destroy.restype = None
    L.fx_last_error.argtypes = [vp, C.c_char_p, C.c_size_t]
    L.fx_sync.argtypes = [vp]
    L.fx_stream.argtypes = [vp, C.POINTER(vp)]
    L.fx_set_mesh.argtypes = [vp, C.c_int, C.POINTER(FxBlockDesc)]
    L.fx_upload_block.argtypes = [vp, C.c_int, dp, dpp3, dpp3]
    L.fx_download_block.argtypes = [vp, C.c_int, dp, dp, dpp3]
    L.fx_upload_all.argtypes = [vp, dp, dp]
    L.fx_download_all.argtypes = [vp, dp, dp]
    L.fx_upload_state.argtypes = [vp, dp, dp]
    L.fx_download_state.argtypes = [vp, dp, dp]
    L.fx_download_array.argtypes = [vp, C.c_int, C.c_int, C.c_int, dp]
    L.fx_flux_update.argtypes = [vp, C.c_int, C.c_int, C.c_int]
    L.fx_mhd_update_emf.argtypes = [vp, C.c_int, C.c_int]
    L.fx_mhd_update_bf.argtypes = [vp, C.c_int, C.c_int, C.c_double]
    L.fx_update_cells.argtypes = [vp, C.c_int, C.c_int, C.c_double, dp]
    L.fx_riemann_flux_send.argtypes = [vp]
    L.fx_mhd_emf_send.argtypes = [vp]
    L.fx_eos_fill_active_cells.argtypes = [vp, C.c_int]
    L.fx_eos_fill_mesh.argtypes = [vp, C.c_int]
    L.fx_boundary_fill_ghosts_and_bf.argtypes = [vp, C.c_int, C.c_int]
    L.fx_calc_dt.argtypes = [vp, C.c_double, dp]
    L.fx_stage.argtypes = [vp, C.c_int, C.c_int, C.c_double, dp]
    L.fx_step.argtypes = [vp, C.c_int, C.c_double, dp]
    L.fx_run.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, dp]
    L.fx_plan_export.argtypes = [C.POINTER(FxConfig), C.c_int, C.POINTER(FxBlockDesc), C.c_int,
                                 ip, C.POINTER(C.c_int), ip, C.POINTER(C.c_int)]
    L.fx_shard_export.argtypes = [C.POINTER(FxConfig), C.c_int, C.POINTER(FxBlockDesc), ip, C.c_int,
                                  C.c_int, C.c_int, ip, C.POINTER(C.c_int), ip, C.POINTER(C.c_int)]
    L.fx_shard_set_mesh.argtypes = [vp, C.c_int, C.POINTER(FxBlockDesc), ip, C.c_int, C.c_int]
    L.fx_shard_group_create.argtypes = [C.c_int]
    L.fx_shard_group_create.restype = vp
    L.fx_shard_group_destroy.argtypes = [vp]
    L.fx_shard_group_destroy.restype = None
    L.fx_shard_attach_group.argtypes = [vp, vp]
    L.fx_nccl_unique_id.argtypes = [C.POINTER(C.c_ubyte)]
    L.fx_shard_attach_nccl.argtypes = [vp, C.POINTER(C.c_ubyte)]
    L.fx_shard_info.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_longlong)]
    L.fx_time_phase.argtypes = [vp, C.c_int, C.c_int, C.c_double, dp]
    L.fx_info.argtypes = [vp, C.c_int, C.POINTER(C.c_longlong)]
    L.fx_autotune.argtypes = [vp, dp, C.c_int, C.POINTER(C.c_int)]
    L.fx_set_flux_shape.argtypes = [vp, C.c_int]
    # device pointers (W, dx, blocks, dt) and the stream pass as plain addresses
    L.fx_branch_trace.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_ulonglong)]
    L.fx_upload_state_active.argtypes = [vp, vp, vp]
    L.fx_download_state_active.argtypes = [vp, vp, vp]
    L.fx_dump_gather.argtypes = [vp, vp, vp, vp]
    L.fx_dump_metadata.argtypes = [C.c_int, C.POINTER(FxBlockDesc), vp]
    L.fx_mesh_slot_geometry.argtypes = [C.c_int, C.POINTER(FxBlockDesc)]
    L.fx_calc_dt_noalloc.argtypes = [vp, C.c_int, C.c_int, vp, C.c_int, vp, C.c_int, C.c_double, C.c_double, vp, vp]
    L.fx_adjoint_forward.argtypes = [vp, C.c_int, C.c_double]
    L.fx_adjoint_backward.argtypes = [vp, dp, dp, dp, dp, C.c_int]
    L.fx_adjoint_time.argtypes = [vp, dp]
    L.fx_face_eval_host.argtypes = [dp, C.c_double, C.c_double, dp]
    L.fx_face_vjp_host.argtypes = [dp, C.c_double, C.c_double, dp, dp, dp]
    L.fx_amr_configure.argtypes = [vp, C.POINTER(FxAmrConfig)]
    L.fx_amr_tag.argtypes = [vp, ip]
    L.fx_amr_adapt.argtypes = [vp, C.POINTER(C.c_int)]
    L.fx_get_mesh.argtypes = [vp, C.c_int, C.POINTER(FxBlockDesc), C.POINTER(C.c_int)]
    L.fx_amr_energy_injected.argtypes = [vp, dp]
    L.fx_amr_timings.argtypes = [vp, dp]
    L.fx_amr_remesh_host.argtypes = [C.POINTER(FxConfig), C.POINTER(FxAmrConfig), C.c_int, C.POINTER(FxBlockDesc),
                                     ip, ip, C.c_int, C.POINTER(FxBlockDesc), C.POINTER(C.c_int)]
    return L
