"""ctypes binding of the native library (``libkelpcuda.so``, C ABI in
``include/kelp_cuda.h``).

There is no fallback: if the library is missing or a CUDA device cannot be
opened, every entry point raises.  Loading the library needs no GPU (the host
routine ``kc_node_xyz_fill`` runs anywhere); creating a context does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libkelpcuda.so")

KC_OK, KC_ERR_ARG, KC_ERR_CUDA, KC_ERR_STATE, KC_ERR_DEVICE = 0, 1, 2, 3, 4
KC_F32, KC_F64, KC_F16 = 0, 1, 2
KC_PLAIN, KC_MIXED = 0, 1
ABI_VERSION = 14
KC_EULER, KC_RK2, KC_RK4 = 0, 1, 2

#: every symbol include/kelp_cuda.h declares
EXPORTS = ("kc_abi_version", "kc_node_xyz_fill", "kc_create", "kc_destroy", "kc_last_error",
           "kc_synchronize", "kc_mesh_upload", "kc_depth_points_upload", "kc_field_upload", "kc_particles_upload", "kc_field_upload_az",
           "kc_particles_download", "kc_coastal_upload", "kc_beach_state_upload",
           "kc_beach_state_download", "kc_beach", "kc_step", "kc_step_host", "kc_step_range", "kc_run_fused",
           "kc_particles_set_realization", "kc_elem_neighbors_upload", "kc_elem_centers_upload", "kc_field_upload_async", "kc_particles_set_elem",
           "kc_particles_get_elem", "kc_find_elements_walk", "kc_find_elements", "kc_sigma_upload", "kc_field_upload_eta", "kc_cgrid_upload",
           "kc_set_fused_block", "kc_run", "kc_sort", "kc_find_nearest", "kc_find_nearest_noalloc", "kc_rng_normals", "kc_rng_domain_digests", "kc_grid_hash_build", "kc_grid_cell_stats", "kc_sample_field", "kc_sample_field_sigma", "kc_beach_surface", "kc_sigma_surfaces", "kc_sigma_surface_slots",
           "kc_device_errors",
           "kc_event_record", "kc_event_elapsed", "kc_l2_flush", "kc_host_alloc", "kc_host_free")


#: device error word bits (kc_device_errors)
ERR_SEARCH_CAP, ERR_BAD_ANCHOR = 1, 2


def describe_device_errors(word: int) -> str:
    parts = []
    if word & ERR_SEARCH_CAP:
        parts.append("a device-side search iteration cap was hit")
    if word & ERR_BAD_ANCHOR:
        parts.append("a particle's nearest_node lies outside [-n_nodes, n_nodes)")
    return "; ".join(parts) or f"device error word {word:#x}"


class KcError(RuntimeError):
    """A C-ABI call returned a non-zero code."""

    def __init__(self, code, msg):
        super().__init__(f"kelp_cuda error {code}: {msg}")
        self.code = code


class MeshDesc(C.Structure):
    _fields_ = [("n_nodes", C.c_longlong), ("n_elems", C.c_longlong),
                ("max_v", C.c_int), ("max_conn", C.c_int),
                ("nodes_lon", C.c_void_p), ("nodes_lat", C.c_void_p), ("depth", C.c_void_p),
                ("elem_nodes", C.c_void_p), ("node_to_elems", C.c_void_p),
                ("node_to_elems_count", C.c_void_p), ("gh_offsets", C.c_void_p),
                ("gh_node_ids", C.c_void_p), ("node_xyz", C.c_void_p),
                ("gh_cell_size", C.c_double), ("gh_lon_min", C.c_double), ("gh_lat_min", C.c_double),
                ("gh_nx", C.c_int), ("gh_ny", C.c_int), ("gh_wrap_lon", C.c_int), ("gh_far_rows", C.c_int),
                ("exact_nearest", C.c_int), ("r_earth", C.c_double),
                ("z_levels", C.c_void_p), ("n_levels", C.c_int)]


class StepArgs(C.Structure):
    _fields_ = [("scheme", C.c_int), ("dims", C.c_int),
                ("slot_a", C.c_int), ("slot_b", C.c_int), ("slot_t", C.c_int),
                ("alpha0", C.c_double), ("alpha_k", C.c_double * 4),
                ("dt", C.c_double), ("time_dir", C.c_double),
                ("w_code", C.c_int), ("uv_vertical", C.c_int), ("kick", C.c_int),
                ("kh_x", C.c_double), ("kh_y", C.c_double),
                ("seed", C.c_ulonglong), ("real_id", C.c_ulonglong),
                ("step_i", C.c_ulonglong), ("pid_offset", C.c_ulonglong),
                ("global_step", C.c_longlong), ("precision", C.c_int),
                ("az_kick", C.c_int), ("az_field", C.c_int), ("az_const", C.c_double),
                ("Dmin", C.c_double), ("z0b_min", C.c_double), ("alpha_end", C.c_double),
                ("pchip", C.c_int), ("slot_d", C.c_int), ("pchip_t", C.c_double * 4),
                ("uv_lsq", C.c_int)]


class BeachArgs(C.Structure):
    _fields_ = [("use_depth", C.c_int), ("use_coastal", C.c_int), ("use_stochastic", C.c_int),
                ("on_failure", C.c_int), ("resuspension", C.c_int), ("min_wet_steps", C.c_int),
                ("depth_min", C.c_double), ("zone_depth", C.c_double), ("rewet_hysteresis", C.c_double),
                ("p_beach", C.c_double), ("p_resusp", C.c_double),
                ("seed", C.c_ulonglong), ("real_id", C.c_ulonglong),
                ("step_i", C.c_ulonglong), ("pid_offset", C.c_ulonglong)]


class CgridDesc(C.Structure):
    _fields_ = [("ny", C.c_int), ("nx", C.c_int), ("K", C.c_int), ("partial_shrunk", C.c_int),
                ("corners", C.c_void_p), ("elem_ji", C.c_void_p), ("nlev", C.c_void_p), ("nlev_raster", C.c_void_p),
                ("e2u", C.c_void_p), ("e1v", C.c_void_p), ("area", C.c_void_p), ("zw", C.c_void_p),
                ("e3b", C.c_void_p), ("kbu", C.c_void_p), ("e3u", C.c_void_p), ("kbv", C.c_void_p),
                ("e3v", C.c_void_p)]


class HostParticles(C.Structure):
    _fields_ = [("lon", C.c_void_p), ("lat", C.c_void_p), ("z", C.c_void_p), ("status", C.c_void_p),
                ("nearest_node", C.c_void_p), ("failure_reason", C.c_void_p),
                ("u", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p),
                ("pid", C.c_void_p), ("real_id", C.c_void_p), ("release_step", C.c_void_p),
                ("elem", C.c_void_p)]


_lib = None


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m kelp_b200.build` "
                              "(the CUDA path has no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        vp, ll, i, d = C.c_void_p, C.c_longlong, C.c_int, C.c_double
        L.kc_abi_version.restype = i
        L.kc_node_xyz_fill.argtypes = [vp, vp, ll, vp]
        L.kc_create.argtypes = [i, C.POINTER(vp)]
        L.kc_destroy.argtypes = [vp]
        L.kc_destroy.restype = None
        L.kc_last_error.argtypes = [vp, C.c_char_p, i]
        L.kc_synchronize.argtypes = [vp]
        L.kc_mesh_upload.argtypes = [vp, C.POINTER(MeshDesc)]
        L.kc_field_upload.argtypes = [vp, i, i, ll, i, vp, vp, i, vp]
        L.kc_field_upload_async.argtypes = [vp, i, i, ll, i, vp, vp, i, vp]
        L.kc_depth_points_upload.argtypes = [vp, i, vp, vp, vp]
        L.kc_field_upload_az.argtypes = [vp, i, i, ll, i, vp]
        L.kc_particles_upload.argtypes = [vp, ll, vp, vp, vp, vp, vp, vp, vp, vp]
        L.kc_particles_download.argtypes = [vp, ll, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        L.kc_coastal_upload.argtypes = [vp, vp]
        L.kc_beach_state_upload.argtypes = [vp, vp, vp]
        L.kc_beach_state_download.argtypes = [vp, vp]
        L.kc_beach.argtypes = [vp, C.POINTER(BeachArgs)]
        L.kc_step.argtypes = [vp, C.POINTER(StepArgs)]
        L.kc_step_range.argtypes = [vp, C.POINTER(StepArgs), ll, ll]
        L.kc_run_fused.argtypes = [vp, C.POINTER(StepArgs), i, C.c_void_p, i]
        L.kc_particles_set_realization.argtypes = [vp, vp]
        L.kc_elem_neighbors_upload.argtypes = [vp, i, vp]
        L.kc_elem_centers_upload.argtypes = [vp, vp, vp]
        L.kc_particles_set_elem.argtypes = [vp, vp]
        L.kc_particles_get_elem.argtypes = [vp, ll, vp]
        L.kc_find_elements_walk.argtypes = [vp, ll, vp, vp, vp, vp]
        L.kc_find_elements.argtypes = [vp, ll, vp, vp, vp, vp]
        L.kc_sigma_upload.argtypes = [vp, i, vp]
        L.kc_field_upload_eta.argtypes = [vp, i, ll, vp]
        L.kc_cgrid_upload.argtypes = [vp, C.POINTER(CgridDesc)]
        L.kc_set_fused_block.argtypes = [vp, i]
        L.kc_step_host.argtypes = [vp, C.POINTER(StepArgs), ll, C.POINTER(HostParticles), C.POINTER(HostParticles),
                                   ll]
        L.kc_run.argtypes = [vp, C.POINTER(StepArgs), i]
        L.kc_sort.argtypes = [vp]
        L.kc_find_nearest.argtypes = [vp, ll, vp, vp, vp]
        L.kc_beach_surface.argtypes = [vp, vp, vp]
        L.kc_sigma_surfaces.argtypes = [vp, vp, vp, i]
        L.kc_sigma_surface_slots.argtypes = [vp, i, i, vp, C.c_double, vp, C.c_double, i]
        L.kc_sample_field.argtypes = [vp, vp, C.c_int, vp, ll, vp, vp, vp, vp, vp, C.c_int, vp]
        L.kc_sample_field_sigma.argtypes = [vp, vp, C.c_int, vp, C.c_double, ll, vp, vp, vp, vp, vp, C.c_int, vp]
        L.kc_find_nearest_noalloc.argtypes = [vp, ll, vp, vp, vp]
        L.kc_rng_normals.argtypes = [vp, ll, C.c_ulonglong, C.c_ulonglong, C.c_ulonglong, C.c_ulonglong,
                                     C.c_ulonglong, vp]
        L.kc_rng_domain_digests.argtypes = [vp, i, vp]
        L.kc_grid_hash_build.argtypes = [vp, ll, vp, vp, C.c_double, C.c_double, C.c_double, i, i, i, vp, vp]
        L.kc_grid_cell_stats.argtypes = [vp, ll, vp, C.c_double, C.c_double, C.c_double, i, i, i, ll, vp, vp, vp, vp,
                                         vp, vp, vp]
        L.kc_device_errors.argtypes = [vp, C.POINTER(i)]
        L.kc_event_record.argtypes = [vp, i]
        L.kc_event_elapsed.argtypes = [vp, i, i, C.POINTER(C.c_float)]
        L.kc_l2_flush.argtypes = [vp, ll]
        L.kc_host_alloc.argtypes = [ll, C.POINTER(vp)]
        L.kc_host_free.argtypes = [vp]
        for name in EXPORTS:
            fn = getattr(L, name)
            if name != "kc_destroy" and fn.restype is not None and fn.restype != i:
                fn.restype = i
        _lib = L
    return _lib


def ptr(a):
    """Data pointer of a C-contiguous numpy array (None passes NULL)."""
    if a is None:
        return None
    if not a.flags.c_contiguous:
        raise ValueError("array must be C-contiguous")
    return a.ctypes.data


def node_xyz_fill(lon: np.ndarray, lat: np.ndarray, out: np.ndarray) -> None:
    rc = lib().kc_node_xyz_fill(ptr(lon), ptr(lat), lon.shape[0], ptr(out))
    if rc:
        raise KcError(rc, "kc_node_xyz_fill")


def check(ctx, rc: int, what: str) -> None:
    if rc:
        buf = C.create_string_buffer(512)
        if ctx:
            lib().kc_last_error(ctx, buf, 512)
        raise KcError(rc, f"{what}: {buf.value.decode(errors='replace')}")
