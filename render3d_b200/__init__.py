"""Python bindings (ctypes) for libr3d_b200.so, the sm_100a volume raycaster.

The library is C: CUDA kernels behind the C-ABI in include/r3d_cuda.h, the
headless render3d interface in include/r3d_render.h and host helpers in
include/r3d_host.h.  This module mirrors those calls for tests, benchmarks
and Python callers.  It never falls back to another implementation: if the
shared library is missing or fails to load, importing it raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libr3d_b200.so")
ROOT = os.path.dirname(HERE)

R3D_OK = 0
ERRORS = {-1: "R3D_E_INVALID", -2: "R3D_E_CUDA", -3: "R3D_E_NOMEM", -4: "R3D_E_UNSUPPORTED",
          -5: "R3D_E_STATE", -6: "R3D_E_DEVICE", -7: "R3D_E_TIMEOUT"}

MODE_FULL, MODE_MIP, MODE_DEPTH, MODE_HEATMAP, MODE_RAYDIR, MODE_FLAT = range(6)
QUALITY_FULL, QUALITY_FAST = 0, 1
VIEW_ORTHO, VIEW_SURF, VIEW_OBLIQUE, VIEW_STRETCH, VIEW_CROP, VIEW_HALF = 1, 2, 4, 8, 16, 32
BRICK_LOD_FLAG = 0x20000


def VIEW_AXIS(a: int) -> int:
    """Bricks slab axis bits of view_flags: 0 = z, 1 = x, 2 = y."""
    return (a & 3) << 8


class FrameParams(C.Structure):
    """r3d_frame_params: 248 bytes, the reference's layout
    (src/render/render_types.h:47-94)."""
    _fields_ = [
        ("cam_origin", C.c_float * 3), ("step_voxels", C.c_float),
        ("cam_right", C.c_float * 3), ("density", C.c_float),
        ("cam_up", C.c_float * 3), ("lod_bias", C.c_float),
        ("cam_forward", C.c_float * 3), ("max_mip", C.c_float),
        ("viewport", C.c_uint32 * 2), ("mode", C.c_uint32), ("frame_index", C.c_uint32),
        ("threshold", C.c_float), ("slab_grid", C.c_uint32), ("slab_wz", C.c_uint32),
        ("slab_z0", C.c_float), ("slab_nx", C.c_float), ("slab_ny", C.c_float),
        ("slab_px", C.c_float), ("slab_py", C.c_float), ("slab_depth", C.c_uint32),
        ("clip_valid", C.c_uint32), ("clip_orig", (C.c_float * 2) * 6),
        ("vol_r0", C.c_float * 3), ("vol_tx", C.c_float),
        ("vol_r1", C.c_float * 3), ("vol_ty", C.c_float),
        ("vol_r2", C.c_float * 3), ("vol_tz", C.c_float),
        ("brick_mode", C.c_uint32), ("skip_gate", C.c_float),
        ("slab_x0", C.c_float), ("slab_y0", C.c_float),
        ("view_org", C.c_uint32), ("view_flags", C.c_uint32),
        ("overlay_gain", C.c_float), ("overlay_flags", C.c_uint32),
    ]

    def copy(self) -> "FrameParams":
        p = FrameParams()
        C.memmove(C.byref(p), C.byref(self), C.sizeof(FrameParams))
        return p


assert C.sizeof(FrameParams) == 248


class VolumeDesc(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32),
                ("brick_dim", C.c_uint32), ("voxel_um", C.c_float)]


class CudaAux(C.Structure):
    _fields_ = [("steps", C.c_void_p), ("mip_index", C.c_void_p),
                ("total_steps", C.c_void_p), ("counters", C.c_void_p)]


class Schedule(C.Structure):
    """r3d_cuda_schedule: forward launch scheduling (results never change)."""
    _fields_ = [("persistent", C.c_uint32), ("refill_min", C.c_uint32),
                ("tile_shape", C.c_uint32), ("unroll", C.c_uint32),
                ("blocks_per_sm", C.c_uint32), ("shade_group", C.c_uint32),
                ("staging", C.c_uint32)]


class SceneRequest(C.Structure):
    _fields_ = [("view", FrameParams), ("rgba", C.c_void_p), ("scene", C.c_void_p)]


class Request(C.Structure):
    _fields_ = [("view", FrameParams), ("rgba", C.c_void_p)]


class DiffScene(C.Structure):
    _fields_ = [("density", C.c_void_p), ("nx", C.c_uint32), ("ny", C.c_uint32),
                ("nz", C.c_uint32), ("lut", C.c_void_p)]


class Grads(C.Structure):
    _fields_ = [("density", C.c_void_p), ("lut", C.c_void_p), ("density_scale", C.c_void_p)]


class PhantomDesc(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("pitch", C.c_float), ("radius", C.c_float),
                ("r0", C.c_float), ("sheet_half", C.c_float), ("in_mean", C.c_float),
                ("in_sd", C.c_float), ("air_mean", C.c_float), ("air_sd", C.c_float),
                ("noise_sd", C.c_float)]


class HostCamera(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("yaw", C.c_float), ("pitch", C.c_float),
                ("fov_y", C.c_float), ("target", C.c_float * 3), ("dist", C.c_float)]


class RenderConfig(C.Structure):
    _fields_ = [("validate", C.c_bool), ("vsync", C.c_bool), ("spv_dir", C.c_char_p),
                ("gpu_budget_bytes", C.c_uint64), ("headless", C.c_bool),
                ("headless_w", C.c_uint32), ("headless_h", C.c_uint32)]


class FrameStats(C.Structure):
    _fields_ = [("gpu_ns", C.c_uint64), ("gpu_raycast_ns", C.c_uint64),
                ("gpu_blit_ns", C.c_uint64), ("gpu_gui_ns", C.c_uint64),
                ("panes_drawn", C.c_uint32), ("cpu_wait_ns", C.c_uint64),
                ("cpu_acquire_ns", C.c_uint64), ("cpu_record_ns", C.c_uint64),
                ("cpu_submit_ns", C.c_uint64)]


class StreamView(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("fwd", C.c_float * 3), ("half_tan", C.c_float),
                ("pixel_cone", C.c_float), ("slice_z0", C.c_uint32), ("slice_depth", C.c_uint32),
                ("gate", C.c_float), ("budget", C.c_uint32)]


class StreamStats(C.Structure):
    _fields_ = [("desired", C.c_uint32), ("requested", C.c_uint32), ("uploaded", C.c_uint32),
                ("evicted", C.c_uint32), ("resident", C.c_uint32)]


class StreamCand(C.Structure):
    _fields_ = [("d2", C.c_float), ("brick", C.c_uint32), ("priority", C.c_uint32)]


GEN_FN = C.CFUNCTYPE(C.c_uint32, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32)
FETCH_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                       C.POINTER(C.c_uint8))


class BrickSrc(C.Structure):
    """r3d_brick_src / r3d_label_src: per-brick content generation and fetch."""
    _fields_ = [("gen", GEN_FN), ("fetch", FETCH_FN), ("user", C.c_void_p)]


def brick_src(gen, fetch) -> BrickSrc:
    """A source from Python callables gen(level, bx, by, bz) -> int and
    fetch(level, bx, by, bz) -> (128, 128, 128) u8 array.  Keep the
    returned object alive while it is attached."""
    def g(_u, l, x, y, z):
        return int(gen(l, x, y, z)) & 0xFFFFFFFF

    def f(_u, l, x, y, z, out):
        a = np.ascontiguousarray(fetch(l, x, y, z), np.uint8).reshape(-1)
        assert a.size == 128 ** 3
        C.memmove(out, a.ctypes.data, a.size)
    s = BrickSrc(GEN_FN(g), FETCH_FN(f), None)
    s._keep = (g, f)
    return s


class VslabLayout(C.Structure):
    _fields_ = [("nx", C.c_uint64), ("ny", C.c_uint64), ("nz", C.c_uint64),
                ("W", C.c_uint32), ("H", C.c_uint32), ("D", C.c_uint32),
                ("px", C.c_uint32), ("wz", C.c_uint32), ("z_margin", C.c_uint32),
                ("x0", C.c_int64), ("y0", C.c_int64), ("z0", C.c_int64),
                ("s", C.c_uint32 * 5), ("gx", C.c_uint32 * 5), ("gy", C.c_uint32 * 5),
                ("base", C.c_uint32 * 5), ("ntiles", C.c_uint32)]


class VslabCell(C.Structure):
    _fields_ = [("cx", C.c_int64), ("cy", C.c_int64), ("za", C.c_int64), ("zb", C.c_int64)]


class VslabJob(C.Structure):
    _fields_ = [("cx", C.c_int64), ("cy", C.c_int64), ("zs0", C.c_int64), ("nz", C.c_uint32),
                ("prio", C.c_uint32)]


class VslabStats(C.Structure):
    _fields_ = [("jobs", C.c_uint32), ("slices", C.c_uint32), ("pending", C.c_uint32),
                ("pad", C.c_uint32), ("origin", C.c_int64 * 3)]


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run python render3d_b200/build.py")
    lib = C.CDLL(LIB_PATH)
    P, U32, F, I = C.c_void_p, C.c_uint32, C.c_float, C.c_int
    sig = {
        "r3d_cuda_create": (I, [I, C.POINTER(P)]),
        "r3d_cuda_destroy": (None, [P]),
        "r3d_cuda_last_error": (C.c_char_p, [P]),
        "r3d_cuda_stream": (P, [P]),
        "r3d_cuda_status": (I, [P, C.POINTER(U32), I]),
        "r3d_cuda_upload_volume": (I, [P, C.POINTER(VolumeDesc), P]),
        "r3d_cuda_set_transfer": (I, [P, P]),
        "r3d_cuda_set_quality": (I, [P, U32]),
        "r3d_cuda_set_alpha_cutoff": (I, [P, F]),
        "r3d_cuda_bricks_build": (I, [P, C.POINTER(VolumeDesc), P, U32, U32]),
        "r3d_cuda_bricks_load": (I, [P, P, U32, P, U32]),
        "r3d_cuda_brick_mode": (U32, [P]),
        "r3d_cuda_bricks_info": (I, [P, C.POINTER(U32), C.POINTER(U32), P, C.POINTER(U32)]),
        "r3d_cuda_bricks_read": (I, [P, P, P]),
        "r3d_cuda_cube_read": (I, [P, I, P, P]),
        "r3d_cuda_shard_build": (I, [P, U32, P, U32, P]),
        "r3d_cuda_bricks_overlay_load": (I, [P, U32, P]),
        "r3d_cuda_slab_build": (I, [P, C.POINTER(VolumeDesc), P, U32, U32]),
        "r3d_cuda_clip_build": (I, [P, C.POINTER(VolumeDesc), P, U32]),
        "r3d_cuda_clip_frame": (I, [P, C.c_double, C.c_double, C.c_uint64, P]),
        "r3d_cuda_clip_params": (None, [P, P]),
        "r3d_cuda_clip_read": (I, [P, U32, U32, P]),
        "r3d_cuda_surf_begin": (I, [P, U32, U32, P, P]),
        "r3d_cuda_surfvol_begin": (I, [P, U32, U32, U32, U32, F, F]),
        "r3d_cuda_surfvol_window": (I, [P, C.c_double, C.c_double, F, F]),
        "r3d_cuda_surfvol_overlay": (I, [P, I]),
        "r3d_cuda_surfvol_mark": (I, [P]),
        "r3d_cuda_surfvol_inkpred": (I, [P, P, U32, U32, F, F, F]),
        "r3d_cuda_bricks_postfilter": (I, [P, U32, F, U32]),
        "r3d_cuda_bricks_refilter": (I, [P]),
        "r3d_cuda_bricks_overlay_read": (I, [P, U32, P]),
        "r3d_cuda_bricks_atlas_attach": (I, [P, U32, C.POINTER(BrickSrc)]),
        "r3d_cuda_bricks_atlas_sync": (I, [P, U32, U32, C.POINTER(C.c_uint32)]),
        "r3d_cuda_bricks_atlas_detach": (I, [P, U32]),
        "r3d_host_brick_locate": (I, [P, U32, C.POINTER(U32), C.POINTER(U32), C.POINTER(U32),
                                      C.POINTER(U32)]),
        "r3d_host_atlas_pick": (U32, [P, P, U32, P, C.POINTER(BrickSrc), U32, P, P, P]),
        "r3d_cuda_surfvol_params": (None, [P, P]),
        "r3d_cuda_surfvol_read": (I, [P, P]),
        "r3d_cuda_surfmask": (I, [P, P, U32, U32]),
        "r3d_cuda_vslab_begin": (I, [P, C.POINTER(VolumeDesc), P, U32, U32, U32, U32]),
        "r3d_cuda_vslab_frame": (I, [P, C.c_double, C.c_double, C.c_int64, U32, P, P]),
        "r3d_cuda_vslab_params": (None, [P, P]),
        "r3d_cuda_vslab_layout": (I, [P, P]),
        "r3d_cuda_vslab_read": (I, [P, U32, P]),
        "r3d_cuda_vslab_table": (I, [P, P]),
        "r3d_host_vslab_init": (I, [P, C.c_uint64, C.c_uint64, C.c_uint64, U32, U32, U32, U32]),
        "r3d_host_vslab_zrange": (None, [P, C.c_int64, P, P]),
        "r3d_host_vslab_range": (None, [P, U32, C.c_int64, C.c_uint64, U32, P, P]),
        "r3d_host_vslab_plan": (U32, [P, P, C.c_double, C.c_double, C.c_int64, U32, P, U32]),
        "r3d_host_vslab_apply": (U32, [P, P, P, C.c_int64]),
        "r3d_host_vslab_key": (U32, [C.c_int64, C.c_int64]),
        "r3d_cuda_slab_window": (I, [P, U32]),
        "r3d_cuda_slab_params": (None, [P, P]),
        "r3d_cuda_slab_read": (I, [P, U32, U32, P, P]),
        "r3d_cuda_stream_begin": (I, [P, C.POINTER(VolumeDesc), P, U32, U32]),
        "r3d_cuda_stream_update": (I, [P, C.POINTER(StreamView), C.POINTER(StreamStats)]),
        "r3d_cuda_stream_view_of": (None, [P, P, U32, C.POINTER(StreamView)]),
        "r3d_host_stream_desired": (U32, [P, U32, P, P, F, F, U32, U32, F, P, P, U32]),
        "r3d_host_stream_box": (U32, [P, U32, P, P, F, F, P, P, U32, U32]),
        "r3d_host_stream_point": (U32, [P, U32, P, U32, F, P, P, U32, U32]),
        "r3d_host_stream_sort": (None, [P, U32]),
        "r3d_cuda_stream_collect_begin": (I, [P]),
        "r3d_cuda_stream_collect_view": (I, [P, C.POINTER(StreamView)]),
        "r3d_cuda_stream_collect_box": (I, [P, P, P, F, F]),
        "r3d_cuda_stream_collect_point": (I, [P, P, U32, F]),
        "r3d_cuda_stream_submit": (I, [P, U32, C.POINTER(StreamStats)]),
        "r3d_cuda_bricks_overlay_build": (I, [P, U32, C.POINTER(VolumeDesc), P]),
        "r3d_cuda_shard_mode": (U32, [P]),
        "r3d_cuda_shard_read": (I, [P, I, P, P, P]),
        "r3d_cuda_raycast_fwd": (I, [P, P, U32, P, U32, U32, C.POINTER(CudaAux), P]),
        "r3d_cuda_raycast_rows": (I, [P, P, P, U32, U32, U32, U32, P]),
        "r3d_cuda_last_kernel_ns": (I, [P, C.POINTER(C.c_uint64)]),
        "r3d_cuda_fmath_eval": (I, [P, P, P, P, U32]),
        "r3d_cuda_elide_counts": (None, [P, F, P]),
        "r3d_cuda_set_schedule": (I, [P, C.POINTER(Schedule)]),
        "r3d_cuda_l2_read_probe": (I, [P, C.c_size_t, U32, C.POINTER(F)]),
        "r3d_cuda_set_slot_trace": (I, [P, P]),
        "r3d_cuda_fill_rgba": (I, [P, P, C.c_size_t, P, P]),
        "r3d_cuda_raycast_fwd_noalloc": (I, [P, P, U32, P, U32, U32, P]),
        "r3d_cuda_diff_forward": (I, [P, C.POINTER(DiffScene), P, U32, P, P, P]),
        "r3d_cuda_diff_forward_tape": (I, [P, C.POINTER(DiffScene), P, U32, P, P, P]),
        "r3d_cuda_batch_create_scenes": (I, [P, P, U32, C.POINTER(P)]),
        "r3d_cuda_raycast_batch": (I, [P, P, U32, P, P]),
        "r3d_cuda_batch_create": (I, [P, P, U32, C.POINTER(P)]),
        "r3d_cuda_batch_destroy": (None, [P]),
        "r3d_cuda_batch_set_schedule": (I, [P, C.POINTER(Schedule)]),
        "r3d_cuda_batch_get_schedule": (I, [P, C.POINTER(Schedule)]),
        "r3d_cuda_batch_launch": (I, [P, P, P]),
        "r3d_cuda_batch_capture": (I, [P, P, P]),
        "r3d_cuda_batch_replay": (I, [P, P]),
        "r3d_cuda_batch_autotune": (I, [P, U32, C.POINTER(Schedule), C.POINTER(F)]),
        "r3d_cuda_raycast_bwd": (I, [P, C.POINTER(DiffScene), P, U32, P, C.POINTER(Grads), U32,
                                     I, P]),
        "r3d_cuda_get_schedule": (I, [P, C.POINTER(Schedule)]),
        "r3d_create": (I, [P, C.POINTER(RenderConfig), C.POINTER(P)]),
        "r3d_destroy": (None, [P]),
        "r3d_upload_volume": (I, [P, C.POINTER(VolumeDesc), P]),
        "r3d_set_transfer": (I, [P, P]),
        "r3d_set_quality": (None, [P, U32]),
        "r3d_set_alpha_cutoff": (I, [P, F]),
        "r3d_renderer_cuda": (P, [P]),
        "r3d_bricks_begin_volume": (I, [P, C.POINTER(VolumeDesc), P, U32, U32]),
        "r3d_bricks_begin_shard": (I, [P, P, U32, U32]),
        "r3d_bricks_end": (I, [P]),
        "r3d_bricks_params": (None, [P, C.POINTER(FrameParams)]),
        "r3d_bricks_extent": (None, [P, P]),
        "r3d_bricks_shape": (None, [P, P]),
        "r3d_slab_init": (I, [P, P]),
        "r3d_slab_window": (I, [P, P, U32]),
        "r3d_slab_params": (None, [P, P]),
        "r3d_clip_begin_volume": (I, [P, P, U32]),
        "r3d_clip_frame": (I, [P, C.c_double, C.c_double, C.c_uint64, P]),
        "r3d_bricks_begin_stream": (I, [P, C.POINTER(VolumeDesc), P, U32, U32]),
        "r3d_bricks_stream": (None, [P, P, P, F, F, U32, U32, F, U32]),
        "r3d_bricks_stream_begin": (C.c_bool, [P]),
        "r3d_bricks_stream_box": (None, [P, P, P, F, F]),
        "r3d_bricks_stream_point": (None, [P, P, U32, F]),
        "r3d_bricks_stream_submit": (None, [P, U32]),
        "r3d_bricks_get_stats": (None, [P, P]),
        "r3d_bricks_flush": (None, [P]),
        "r3d_bricks_overlay_volume": (I, [P, U32, C.POINTER(VolumeDesc), P]),
        "r3d_vslab_begin_volume": (I, [P, P, P]),
        "r3d_vslab_frame": (None, [P, C.c_double, C.c_double, C.c_int64, U32, P]),
        "r3d_vslab_get": (None, [P, P, P]),
        "r3d_vslab_resident_pending": (U32, [P]),
        "r3d_surf_begin": (I, [P, U32, U32, P, P]),
        "r3d_surf_swap": (I, [P, U32, U32, P, P, F, F]),
        "r3d_surfvol_begin": (I, [P, U32, U32, U32, U32, F, F]),
        "r3d_surfvol_window": (None, [P, C.c_double, C.c_double, F, F]),
        "r3d_surfvol_visible": (None, [P, U32, U32, U32, U32, U32, U32]),
        "r3d_surfvol_mark": (None, [P]),
        "r3d_surfvol_overlay_enable": (None, [P, C.c_bool]),
        "r3d_surfvol_regtap": (None, [P, C.c_bool]),
        "r3d_bricks_postfilter": (None, [P, U32, F, U32]),
        "r3d_bricks_labels": (I, [P, C.POINTER(BrickSrc)]),
        "r3d_bricks_labels_sync": (None, [P, U32]),
        "r3d_bricks_regatlas": (I, [P, C.POINTER(BrickSrc)]),
        "r3d_bricks_regatlas_sync": (None, [P, U32]),
        "r3d_bricks_regatlas_detach": (None, [P]),
        "r3d_bricks_refilter": (None, [P]),
        "r3d_surfvol_inkpred": (I, [P, P, U32, U32, F, F, F]),
        "r3d_surfvol_inkpred_clear": (None, [P]),
        "r3d_surfvol_params": (None, [P, P]),
        "r3d_surfmask": (I, [P, P, U32, U32]),
        "r3d_surfmask_clear": (None, [P]),
        "r3d_max_dim3d": (U32, [P]),
        "r3d_frame": (I, [P, C.POINTER(FrameParams), C.POINTER(FrameStats)]),
        "r3d_frame_views": (I, [P, P, U32, C.POINTER(FrameStats)]),
        "r3d_read_frame": (I, [P, P, C.POINTER(U32), C.POINTER(U32)]),
        "r3d_host_camera_init": (None, [C.POINTER(HostCamera), P]),
        "r3d_host_camera_look": (None, [C.POINTER(HostCamera), F, F]),
        "r3d_host_camera_move": (None, [C.POINTER(HostCamera), P, F]),
        "r3d_host_camera_orbit_set": (None, [C.POINTER(HostCamera), P, F]),
        "r3d_host_camera_orbit_drag": (None, [C.POINTER(HostCamera), F, F]),
        "r3d_host_camera_orbit_zoom": (None, [C.POINTER(HostCamera), F]),
        "r3d_host_camera_basis": (None, [C.POINTER(HostCamera), F, P, P, P]),
        "r3d_host_m3_ypr": (None, [F, F, F, P]),
        "r3d_host_tf_build": (None, [P, P, U32, P]),
        "r3d_host_tf_preset": (U32, [U32, P]),
        "r3d_host_tf_min_visible": (F, [P]),
        "r3d_host_skip_gate": (F, [F, P]),
        "r3d_host_lod_pick": (U32, [F, F, F, U32]),
        "r3d_host_lod_fallback": (U32, [U32, U32, U32]),
        "r3d_host_orbit_view": (None, [C.POINTER(FrameParams), F, P, U32, U32, F, F, F, U32,
                                       U32, F, P]),
        "r3d_host_phantom_default": (None, [U32, C.c_uint64, C.POINTER(PhantomDesc)]),
        "r3d_host_phantom": (I, [P, U32, U32, U32, C.POINTER(PhantomDesc), I]),
        "r3d_cuda_phantom": (I, [P, C.POINTER(PhantomDesc), U32, U32, U32, P, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()


class R3DError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def _ptr(a) -> int:
    """Address of a numpy array or a torch tensor (host or device)."""
    if a is None:
        return 0
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    return int(a.data_ptr())


# ------------------------------------------------------------------ host

def stream_desired(page: np.ndarray, eye, fwd, half_tan: float, pixel_cone: float,
                   gate: float = 0.0, slice_z0: int = 0, slice_depth: int = 0) -> np.ndarray:
    """The streamer's request set (r3d_host_stream_desired) as a structured
    array of (d2, brick, priority), sorted."""
    page = np.ascontiguousarray(page, np.uint32)
    mark = np.zeros(page.size, np.uint8)
    out = (StreamCand * page.size)()
    e3 = (C.c_float * 3)(*eye)
    f3 = (C.c_float * 3)(*fwd)
    n = lib.r3d_host_stream_desired(_ptr(page), page.size, e3, f3, half_tan, pixel_cone,
                                    slice_z0, slice_depth, gate, _ptr(mark), out, page.size)
    a = np.ctypeslib.as_array(out)[:n]
    return a.copy()


class StreamCollect:
    """One frame's request set built on the host from any number of cone,
    box and point collects (r3d_host_stream_desired / _box / _point), as
    the context's collect calls build it."""

    def __init__(self, page: np.ndarray):
        self.page = np.ascontiguousarray(page, np.uint32)
        self.mark = np.zeros(self.page.size, np.uint8)
        self.out = (StreamCand * self.page.size)()
        self.n = 0

    def box(self, lo, hi, pixel_cone: float, gate: float = 0.0) -> None:
        self.n = lib.r3d_host_stream_box(_ptr(self.page), self.page.size, (C.c_float * 3)(*lo),
                                         (C.c_float * 3)(*hi), pixel_cone, gate, _ptr(self.mark),
                                         self.out, self.page.size, self.n)

    def point(self, p, level: int, gate: float = 0.0) -> None:
        self.n = lib.r3d_host_stream_point(_ptr(self.page), self.page.size, (C.c_float * 3)(*p),
                                           level, gate, _ptr(self.mark), self.out,
                                           self.page.size, self.n)

    def cone(self, eye, fwd, half_tan: float, pixel_cone: float, gate: float = 0.0,
             slice_z0: int = 0, slice_depth: int = 0) -> None:
        tail = C.cast(C.addressof(self.out) + self.n * C.sizeof(StreamCand), C.c_void_p)
        self.n += lib.r3d_host_stream_desired(_ptr(self.page), self.page.size,
                                              (C.c_float * 3)(*eye), (C.c_float * 3)(*fwd),
                                              half_tan, pixel_cone, slice_z0, slice_depth, gate,
                                              _ptr(self.mark), tail, self.page.size - self.n)

    def sorted(self) -> np.ndarray:
        lib.r3d_host_stream_sort(self.out, self.n)
        return np.ctypeslib.as_array(self.out)[:self.n].copy()


class VslabHost:
    """The virtual slab's host layout and fill scheduler (r3d_host_vslab_*):
    a layout, its ledger of base tiles and one frame's plan + ledger update,
    without a device."""

    def __init__(self, nx, ny, nz, W, H, D, z_margin=0):
        self.v = VslabLayout()
        if lib.r3d_host_vslab_init(C.byref(self.v), nx, ny, nz, W, H, D, z_margin) != 0:
            raise ValueError("vslab layout")
        n = self.v.gx[0] * self.v.gy[0]
        self.cells = (VslabCell * n)()
        for c in self.cells:
            c.cx = c.cy = -(1 << 63)

    def frame(self, fx, fy, z0, budget):
        """Plans one frame, records its jobs as finished; returns them as
        (cx, cy, zs0, nz) tuples."""
        jobs = (VslabJob * 112)()
        n = lib.r3d_host_vslab_plan(C.byref(self.v), self.cells, fx, fy, z0, budget, jobs, 112)
        out = []
        for j in jobs[:n]:
            lib.r3d_host_vslab_apply(C.byref(self.v), self.cells, C.byref(j), self.v.z0)
            out.append((j.cx, j.cy, j.zs0, j.nz))
        return out


def tf_preset(idx: int) -> np.ndarray:
    lut = np.zeros((256, 4), np.uint8)
    if lib.r3d_host_tf_preset(idx, _ptr(lut)) != idx:
        raise ValueError(f"no TF preset {idx}")
    return lut


def tf_build(points: list[tuple[int, tuple[int, int, int, int]]]) -> np.ndarray:
    vals = np.array([p[0] for p in points], np.uint8)
    cols = np.array([p[1] for p in points], np.uint8).reshape(-1, 4)
    lut = np.zeros((256, 4), np.uint8)
    lib.r3d_host_tf_build(_ptr(vals), _ptr(cols), len(points), _ptr(lut))
    return lut


def grey_ramp() -> np.ndarray:
    return np.repeat(np.arange(256, dtype=np.uint8)[:, None], 4, axis=1).copy()


def scroll_ramp_tf() -> np.ndarray:
    """The benchmark TF: alpha 0 below 40, rising to 0.9 (230) at 200 and
    flat to 255, grey RGB ramp."""
    return tf_build([(0, (0, 0, 0, 0)), (40, (40, 40, 40, 0)), (200, (200, 200, 200, 230)),
                     (255, (255, 255, 255, 230))])


def skip_gate(low_cut: float, lut: np.ndarray) -> float:
    return float(lib.r3d_host_skip_gate(low_cut, _ptr(np.ascontiguousarray(lut))))


def phantom(n: int | tuple[int, int, int], seed: int = 1234, threads: int = 0,
            desc: PhantomDesc | None = None) -> np.ndarray:
    """Seeded scroll phantom as a (nz, ny, nx) u8 array."""
    nx, ny, nz = (n, n, n) if isinstance(n, int) else n
    if desc is None:
        desc = PhantomDesc()
        lib.r3d_host_phantom_default(max(nx, ny, nz), seed, C.byref(desc))
    vol = np.empty((nz, ny, nx), np.uint8)
    if threads <= 0:
        threads = os.cpu_count() or 8
    if lib.r3d_host_phantom(_ptr(vol), nx, ny, nz, C.byref(desc), threads) != 0:
        raise ValueError("phantom: bad parameters")
    return vol


def orbit_view(ph: float, w: int, h: int, lut: np.ndarray, target=(0.5, 0.5, 0.5),
               step_voxels: float = 1.0, density: float = 1.0, lod_bias: float = 0.0,
               mode: int = MODE_FULL, frame_index: int = 0, low_cut: float = 0.0
               ) -> FrameParams:
    """View of the scripted orbit benchmark at phase ph (src/main.c:3932-3946)."""
    p = FrameParams()
    t = (C.c_float * 3)(*target)
    lib.r3d_host_orbit_view(C.byref(p), ph, t, w, h, step_voxels, density, lod_bias, mode,
                            frame_index, low_cut, _ptr(np.ascontiguousarray(lut)))
    return p


def camera_view(yaw: float, pitch: float, dist: float, w: int, h: int, lut: np.ndarray,
                target=(0.5, 0.5, 0.5), step_voxels: float = 1.0, density: float = 1.0,
                lod_bias: float = 0.0, mode: int = MODE_FULL, frame_index: int = 0,
                low_cut: float = 0.0, max_mip: float = 10.0) -> FrameParams:
    """Turntable orbit view at (yaw, pitch) radians; pitch < 0 looks down."""
    cam = HostCamera()
    lib.r3d_host_camera_init(C.byref(cam), (C.c_float * 3)(0.5, 0.5, -1.5))
    cam.yaw, cam.pitch = yaw, pitch
    lib.r3d_host_camera_orbit_set(C.byref(cam), (C.c_float * 3)(*target), dist)
    p = FrameParams()
    p.cam_origin[:] = cam.pos[:]
    lib.r3d_host_camera_basis(C.byref(cam), C.c_float(w / h), p.cam_right, p.cam_up,
                              p.cam_forward)
    p.step_voxels, p.density, p.lod_bias, p.max_mip = step_voxels, density, lod_bias, max_mip
    p.viewport[0], p.viewport[1] = w, h
    p.mode, p.frame_index = mode, frame_index
    p.threshold = low_cut / 255.0
    p.skip_gate = skip_gate(low_cut, lut)
    p.vol_r0[:] = (1.0, 0.0, 0.0)
    p.vol_r1[:] = (0.0, 1.0, 0.0)
    p.vol_r2[:] = (0.0, 0.0, 1.0)
    return p


def set_rotation(p: FrameParams, yaw: float, pitch: float, roll: float,
                 t=(0.0, 0.0, 0.0)) -> None:
    m = (C.c_float * 9)()
    lib.r3d_host_m3_ypr(yaw, pitch, roll, m)
    p.vol_r0[:] = m[0:3]
    p.vol_r1[:] = m[3:6]
    p.vol_r2[:] = m[6:9]
    p.vol_tx, p.vol_ty, p.vol_tz = t


# ---------------------------------------------------------------- device

class Context:
    """An r3d_cuda_ctx: scene state on one GPU plus the forward raycast."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        rc = lib.r3d_cuda_create(device, C.byref(h))
        if rc != R3D_OK:
            raise R3DError(rc, "r3d_cuda_create failed (no CUDA device?)")
        self.h = h

    def close(self) -> None:
        if self.h:
            lib.r3d_cuda_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        if rc != R3D_OK:
            raise R3DError(rc, lib.r3d_cuda_last_error(self.h).decode())

    @property
    def stream(self) -> int:
        return lib.r3d_cuda_stream(self.h) or 0

    def upload_volume(self, vol) -> None:
        nz, ny, nx = vol.shape
        d = VolumeDesc(nx, ny, nz, 128, 1.0)
        self._check(lib.r3d_cuda_upload_volume(self.h, C.byref(d), _ptr(vol)))

    def set_transfer(self, lut: np.ndarray) -> None:
        lut = np.ascontiguousarray(lut, dtype=np.uint8)
        assert lut.shape == (256, 4)
        self._check(lib.r3d_cuda_set_transfer(self.h, _ptr(lut)))

    def set_quality(self, q: int) -> None:
        self._check(lib.r3d_cuda_set_quality(self.h, q))

    def set_alpha_cutoff(self, c: float) -> None:
        self._check(lib.r3d_cuda_set_alpha_cutoff(self.h, c))

    def bricks_build(self, vol, nlev: int, min_max: int = 0) -> None:
        nz, ny, nx = vol.shape
        d = VolumeDesc(nx, ny, nz, 128, 1.0)
        self._check(lib.r3d_cuda_bricks_build(self.h, C.byref(d), _ptr(vol), nlev, min_max))

    def bricks_load(self, page: np.ndarray, slots: np.ndarray) -> None:
        page = np.ascontiguousarray(page, np.uint32)
        slots = np.ascontiguousarray(slots, np.uint8)
        nslots = slots.size // (128 ** 3)
        self._check(lib.r3d_cuda_bricks_load(self.h, _ptr(page), page.size, _ptr(slots), nslots))

    @property
    def brick_mode(self) -> int:
        return int(lib.r3d_cuda_brick_mode(self.h))

    def bricks_info(self) -> dict:
        w, n, nl = C.c_uint32(), C.c_uint32(), C.c_uint32()
        shape = (C.c_uint32 * 3)()
        self._check(lib.r3d_cuda_bricks_info(self.h, C.byref(w), C.byref(n), shape,
                                             C.byref(nl)))
        return {"page_words": w.value, "nslots": n.value, "shape": tuple(shape),
                "nlev": nl.value}

    def bricks_read(self, slots: bool = True) -> tuple[np.ndarray, np.ndarray | None]:
        info = self.bricks_info()
        page = np.empty(info["page_words"], np.uint32)
        pool = np.empty(info["nslots"] * 128 ** 3, np.uint8) if slots else None
        self._check(lib.r3d_cuda_bricks_read(self.h, _ptr(page), _ptr(pool)))
        return page, pool

    def cube_read(self, level: int) -> np.ndarray:
        dims = (C.c_uint32 * 3)()
        self._check(lib.r3d_cuda_cube_read(self.h, level, None, dims))
        out = np.empty((dims[2], dims[1], dims[0]), np.uint8)
        self._check(lib.r3d_cuda_cube_read(self.h, level, _ptr(out), dims))
        return out

    def stream_begin(self, vol, nlev: int, nslots: int) -> None:
        """Streaming LOD cache: the whole pyramid in pinned host memory,
        nslots device slots filled by stream_update."""
        nz, ny, nx = vol.shape
        d = VolumeDesc(nx, ny, nz, 128, 1.0)
        self._check(lib.r3d_cuda_stream_begin(self.h, C.byref(d), _ptr(vol), nlev, nslots))

    def stream_update(self, p: "FrameParams", budget: int, ext=(1.0, 1.0, 1.0)) -> dict:
        """One pump update for view p; returns its statistics."""
        v = StreamView()
        e = (C.c_float * 3)(*ext)
        lib.r3d_cuda_stream_view_of(C.byref(p), e, budget, C.byref(v))
        st = StreamStats()
        self._check(lib.r3d_cuda_stream_update(self.h, C.byref(v), C.byref(st)))
        return {k: getattr(st, k) for k, _ in StreamStats._fields_}

    def stream_collect_begin(self) -> None:
        self._check(lib.r3d_cuda_stream_collect_begin(self.h))

    def stream_collect_view(self, p: "FrameParams", ext=(1.0, 1.0, 1.0)) -> None:
        v = StreamView()
        lib.r3d_cuda_stream_view_of(C.byref(p), (C.c_float * 3)(*ext), 0, C.byref(v))
        self._check(lib.r3d_cuda_stream_collect_view(self.h, C.byref(v)))

    def stream_collect_box(self, lo, hi, pixel_cone: float, gate: float = 0.0) -> None:
        self._check(lib.r3d_cuda_stream_collect_box(self.h, (C.c_float * 3)(*lo),
                                                    (C.c_float * 3)(*hi), pixel_cone, gate))

    def stream_collect_point(self, p, level: int, gate: float = 0.0) -> None:
        self._check(lib.r3d_cuda_stream_collect_point(self.h, (C.c_float * 3)(*p), level, gate))

    def stream_submit(self, budget: int) -> dict:
        st = StreamStats()
        self._check(lib.r3d_cuda_stream_submit(self.h, budget, C.byref(st)))
        return {k: getattr(st, k) for k, _ in StreamStats._fields_}

    def clip_build(self, vol, depth_max: int) -> None:
        nz, ny, nx = vol.shape
        d = VolumeDesc(nx, ny, nz, 128, 1.0)
        self._check(lib.r3d_cuda_clip_build(self.h, C.byref(d), _ptr(vol), depth_max))

    def clip_frame(self, fx: float, fy: float, z0: int, p: "FrameParams | None" = None) -> None:
        self._check(lib.r3d_cuda_clip_frame(self.h, fx, fy, z0,
                                            C.byref(p) if p is not None else None))

    def clip_params(self, p: "FrameParams") -> None:
        lib.r3d_cuda_clip_params(self.h, C.byref(p))

    def surf_begin(self, coords, normals) -> None:
        """Segment grids: (gh, gw, 4) float32 surface points (xyz, valid) and
        normals, host arrays or device tensors."""
        gh, gw = coords.shape[:2]
        self._check(lib.r3d_cuda_surf_begin(self.h, gw, gh, _ptr(coords), _ptr(normals)))

    def surfvol_begin(self, W: int, H: int, L: int, nback: int, sx: float, sy: float) -> None:
        self._check(lib.r3d_cuda_surfvol_begin(self.h, W, H, L, nback, sx, sy))

    def surfvol_window(self, u0: float, v0: float, step: float, zoff0: float) -> None:
        self._check(lib.r3d_cuda_surfvol_window(self.h, u0, v0, step, zoff0))

    def surfvol_overlay(self, atlas: int) -> None:
        self._check(lib.r3d_cuda_surfvol_overlay(self.h, atlas))

    def surfvol_mark(self) -> None:
        self._check(lib.r3d_cuda_surfvol_mark(self.h))

    def surfvol_params(self, p: "FrameParams") -> None:
        lib.r3d_cuda_surfvol_params(self.h, C.byref(p))

    def surfvol_read(self) -> np.ndarray:
        p = FrameParams()
        lib.r3d_cuda_surfvol_params(self.h, C.byref(p))
        out = np.empty((p.slab_wz, int(p.slab_ny), int(p.slab_nx), 2), np.uint8)
        self._check(lib.r3d_cuda_surfvol_read(self.h, _ptr(out)))
        return out

    def bricks_postfilter(self, mode: int, amount: float = 0.0, targets: int = 1) -> None:
        """The display filter for bricks landing in slots from now on."""
        self._check(lib.r3d_cuda_bricks_postfilter(self.h, mode, amount, targets))

    def bricks_refilter(self) -> None:
        self._check(lib.r3d_cuda_bricks_refilter(self.h))

    def atlas_attach(self, which: int, src: BrickSrc) -> None:
        self._check(lib.r3d_cuda_bricks_atlas_attach(self.h, which, C.byref(src)))
        self._srcs = getattr(self, "_srcs", {})
        self._srcs[which] = src

    def atlas_sync(self, which: int, budget: int = 0) -> int:
        n = C.c_uint32()
        self._check(lib.r3d_cuda_bricks_atlas_sync(self.h, which, budget, C.byref(n)))
        return n.value

    def atlas_detach(self, which: int) -> None:
        self._check(lib.r3d_cuda_bricks_atlas_detach(self.h, which))

    def overlay_read(self, which: int) -> np.ndarray:
        """Overlay atlas `which` as (nslots, 128, 128, 128) u8."""
        n = self.bricks_info()["nslots"]
        out = np.empty((n, 128, 128, 128), np.uint8)
        self._check(lib.r3d_cuda_bricks_overlay_read(self.h, which, _ptr(out)))
        return out

    def surfvol_inkpred(self, pred, g0u: float = 0.0, g0v: float = 0.0,
                        px_per_grid: float = 1.0) -> None:
        """Live 2.5D ink prediction, (h, w) float32; None drops it."""
        if pred is None:
            self._check(lib.r3d_cuda_surfvol_inkpred(self.h, None, 0, 0, 0.0, 0.0, 0.0))
            return
        pred = np.ascontiguousarray(pred, np.float32)
        self._check(lib.r3d_cuda_surfvol_inkpred(self.h, _ptr(pred), pred.shape[1], pred.shape[0],
                                                 g0u, g0v, px_per_grid))

    def surfmask(self, m) -> None:
        if m is None:
            self._check(lib.r3d_cuda_surfmask(self.h, None, 0, 0))
        else:
            m = np.ascontiguousarray(m, np.uint8)
            self._check(lib.r3d_cuda_surfmask(self.h, _ptr(m), m.shape[1], m.shape[0]))

    def raycast_rows(self, p: "FrameParams", out, out_w: int, out_h: int, row0: int, row1: int,
                     stream: int = 0) -> None:
        """Dispatch rows [row0, row1) of one view into a device image."""
        self._check(lib.r3d_cuda_raycast_rows(self.h, C.byref(p), _ptr(out), out_w, out_h, row0,
                                              row1, stream or None))

    def vslab_begin(self, vol, W: int, H: int, D: int, z_margin: int = 0) -> None:
        nz, ny, nx = vol.shape
        d = VolumeDesc(nx, ny, nz, 128, 1.0)
        self._check(lib.r3d_cuda_vslab_begin(self.h, C.byref(d), _ptr(vol), W, H, D, z_margin))

    def vslab_frame(self, fx: float, fy: float, z0: int, budget: int,
                    p: "FrameParams | None" = None) -> dict:
        st = VslabStats()
        self._check(lib.r3d_cuda_vslab_frame(self.h, fx, fy, z0, budget,
                                             C.byref(p) if p is not None else None,
                                             C.byref(st)))
        return {"jobs": st.jobs, "slices": st.slices, "pending": st.pending,
                "origin": tuple(st.origin)}

    def vslab_params(self, p: "FrameParams") -> None:
        lib.r3d_cuda_vslab_params(self.h, C.byref(p))

    def vslab_layout(self) -> VslabLayout:
        v = VslabLayout()
        self._check(lib.r3d_cuda_vslab_layout(self.h, C.byref(v)))
        return v

    def vslab_read(self, tile: int) -> np.ndarray:
        v = self.vslab_layout()
        out = np.empty((v.wz, v.px + 2, v.px + 2), np.uint8)
        self._check(lib.r3d_cuda_vslab_read(self.h, tile, _ptr(out)))
        return out

    def vslab_table(self) -> np.ndarray:
        v = self.vslab_layout()
        out = np.empty((v.gx[0] * v.gy[0], 4), np.uint32)
        self._check(lib.r3d_cuda_vslab_table(self.h, _ptr(out)))
        return out

    def clip_read(self, level: int, layer: int) -> np.ndarray:
        out = np.empty((2048, 2048), np.uint8)
        self._check(lib.r3d_cuda_clip_read(self.h, level, layer, _ptr(out)))
        return out

    def slab_build(self, vol, wz: int, z0: int = 0) -> None:
        """Tiled slab over a (nz, ny, nx) volume: a ring of wz slices from z0."""
        nz, ny, nx = vol.shape
        d = VolumeDesc(nx, ny, nz, 128, 1.0)
        self._check(lib.r3d_cuda_slab_build(self.h, C.byref(d), _ptr(vol), wz, z0))

    def slab_window(self, z0: int) -> None:
        self._check(lib.r3d_cuda_slab_window(self.h, z0))

    def slab_params(self, p: "FrameParams") -> None:
        lib.r3d_cuda_slab_params(self.h, C.byref(p))

    def slab_read(self, level: int, tile: int) -> np.ndarray:
        dims = (C.c_uint32 * 3)()
        self._check(lib.r3d_cuda_slab_read(self.h, level, tile, None, dims))
        out = np.empty((dims[2], dims[1], dims[0]), np.uint8)
        self._check(lib.r3d_cuda_slab_read(self.h, level, tile, _ptr(out), dims))
        return out

    def overlay_load(self, which: int, slots) -> None:
        """Overlay atlas `which` (0 ink, 1 3D ink, 2 labels, 3 registration)
        from slot contents in the CT pool's order, or None to remove it."""
        if slots is not None and isinstance(slots, np.ndarray):
            slots = np.ascontiguousarray(slots, np.uint8)
        self._check(lib.r3d_cuda_bricks_overlay_load(self.h, which, _ptr(slots)))

    def overlay_build(self, which: int, vol) -> None:
        """Overlay atlas `which` cut from a raw volume of the cache's shape."""
        nz, ny, nx = vol.shape
        d = VolumeDesc(nx, ny, nz, 128, 1.0)
        self._check(lib.r3d_cuda_bricks_overlay_build(self.h, which, C.byref(d), _ptr(vol)))

    def shard_build(self, vol, abpa: int | None = None, slot_of=None) -> None:
        """Single-level brick atlas from a cubic volume of edge bpa * 128
        (z, y, x order); slot_of[b] is brick b's slot or 0xFFFFFFFF."""
        e = vol.shape[0]
        assert tuple(vol.shape) == (e, e, e)
        bpa = e // 128
        if slot_of is not None:
            slot_of = np.ascontiguousarray(slot_of, np.uint32)
            assert slot_of.size == bpa ** 3
        self._check(lib.r3d_cuda_shard_build(self.h, e, _ptr(vol), abpa or bpa,
                                             _ptr(slot_of)))

    @property
    def shard_mode(self) -> int:
        return int(lib.r3d_cuda_shard_mode(self.h))

    def shard_read(self, level: int = 0) -> tuple[np.ndarray, np.ndarray]:
        """(page table, atlas mip `level` or, for -1, the occupancy grid)."""
        dims = (C.c_uint32 * 3)()
        self._check(lib.r3d_cuda_shard_read(self.h, level, None, None, dims))
        bpa = self.shard_mode & 0xFF
        page = np.empty(bpa ** 3, np.uint32)
        out = np.empty((dims[2], dims[1], dims[0]), np.uint8)
        self._check(lib.r3d_cuda_shard_read(self.h, level, _ptr(page), _ptr(out), dims))
        return page, out

    def status(self, clear: bool = True) -> int:
        b = C.c_uint32()
        self._check(lib.r3d_cuda_status(self.h, C.byref(b), int(clear)))
        return b.value

    def raycast(self, views, out_w: int, out_h: int, out=None, steps=None, mip_index=None,
                total=None, counters=None, stream: int = 0):
        """Raycasts views into out (host numpy (h, w, 4) u8 or a device tensor);
        returns out.  steps / mip_index: same kind, (h, w) u32; total: one
        u64 counter, counters: four u64 counters (samples, TF lookups,
        shaded samples, page walks), both accumulated."""
        if isinstance(views, FrameParams):
            views = [views]
        arr = (FrameParams * len(views))(*views)
        if out is None:
            out = np.zeros((out_h, out_w, 4), np.uint8)
        aux = None
        if any(a is not None for a in (steps, mip_index, total, counters)):
            aux = CudaAux(_ptr(steps) or None, _ptr(mip_index) or None, _ptr(total) or None,
                          _ptr(counters) or None)
        self._check(lib.r3d_cuda_raycast_fwd(self.h, arr, len(views), _ptr(out), out_w, out_h,
                                             C.byref(aux) if aux else None, stream or None))
        return out

    def diff_forward(self, density, lut, views, rgb_out, total=None, stream: int = 0,
                     tape: bool = False):
        """Differentiable render (device tensors): density (nz, ny, nx) f32,
        lut (256, 4) f32, rgb_out f32 of sum(w*h*3) over the views.  tape:
        record the tape a raycast_bwd(tape=True) over the same views reads."""
        if isinstance(views, FrameParams):
            views = [views]
        arr = (FrameParams * len(views))(*views)
        nz, ny, nx = density.shape
        sc = DiffScene(_ptr(density), nx, ny, nz, _ptr(lut))
        fn = lib.r3d_cuda_diff_forward_tape if tape else lib.r3d_cuda_diff_forward
        self._check(fn(self.h, C.byref(sc), arr, len(views), _ptr(rgb_out), _ptr(total) or None,
                       stream or None))

    def raycast_bwd(self, density, lut, views, dl_drgb, g_density, g_lut, g_scale,
                    ckpt_k: int = 32, deterministic: bool = False, stream: int = 0,
                    tape: bool = False):
        """Adjoint of diff_forward into the given device gradient buffers."""
        if isinstance(views, FrameParams):
            views = [views]
        arr = (FrameParams * len(views))(*views)
        nz, ny, nx = density.shape
        sc = DiffScene(_ptr(density), nx, ny, nz, _ptr(lut))
        gr = Grads(_ptr(g_density), _ptr(g_lut), _ptr(g_scale))
        self._check(lib.r3d_cuda_raycast_bwd(self.h, C.byref(sc), arr, len(views),
                                             _ptr(dl_drgb), C.byref(gr), ckpt_k,
                                             int(deterministic) | (2 if tape else 0),
                                             stream or None))

    def phantom(self, shape, seed: int = 1234, out=None):
        """Seeded scroll phantom generated on the device: a (nz, ny, nx) uint8
        CUDA tensor (allocated with torch when out is None)."""
        import torch
        nx, ny, nz = (shape, shape, shape) if isinstance(shape, int) else shape
        d = PhantomDesc()
        lib.r3d_host_phantom_default(max(nx, ny, nz), seed, C.byref(d))
        if out is None:
            out = torch.empty((nz, ny, nx), dtype=torch.uint8, device="cuda")
        self._check(lib.r3d_cuda_phantom(self.h, C.byref(d), nx, ny, nz, _ptr(out), None))
        return out

    def fmath_eval(self, x: np.ndarray, y: np.ndarray) -> np.ndarray:
        """Device log2, exp2, pow and x^24 of the inputs, (n, 4) float32."""
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        out = np.empty((x.size, 4), np.float32)
        self._check(lib.r3d_cuda_fmath_eval(self.h, _ptr(x), _ptr(y), _ptr(out), x.size))
        return out

    def set_schedule(self, persistent: int = 3, refill_min: int = 16, tile_shape: int = 0,
                     unroll: int = 1, blocks_per_sm: int = 0, shade_group: int = 0,
                     staging: int = 0) -> None:
        self._check(lib.r3d_cuda_set_schedule(
            self.h, C.byref(Schedule(persistent, refill_min, tile_shape, unroll, blocks_per_sm,
                                     shade_group, staging))))

    def schedule(self) -> dict:
        sc = Schedule()
        self._check(lib.r3d_cuda_get_schedule(self.h, C.byref(sc)))
        return {f: getattr(sc, f) for f, _ in Schedule._fields_}

    def raycast_batch(self, views, images, total=None, stream: int = 0) -> None:
        """r3d_cuda_raycast_batch: each view into its own device image."""
        arr = (Request * len(views))(*[Request(v, _ptr(im)) for v, im in zip(views, images)])
        self._check(lib.r3d_cuda_raycast_batch(self.h, arr, len(views), _ptr(total) or None,
                                               stream or None))

    def set_slot_trace(self, bits=None) -> None:
        """Counting launches mark the slots they read in bits (device u32)."""
        self._check(lib.r3d_cuda_set_slot_trace(self.h, _ptr(bits) if bits is not None else None))

    def l2_read_probe(self, nbytes: int = 48 << 20, passes: int = 40) -> float:
        """GB/s of an L2-resident read sweep (r3d_cuda_l2_read_probe)."""
        g = C.c_float()
        self._check(lib.r3d_cuda_l2_read_probe(self.h, nbytes, passes, C.byref(g)))
        return g.value

    def last_kernel_ns(self) -> int:
        ns = C.c_uint64()
        self._check(lib.r3d_cuda_last_kernel_ns(self.h, C.byref(ns)))
        return ns.value


class Batch:
    """r3d_cuda_batch: many views with their own device images (tensors);
    scenes (optional): per view the Context whose scene it samples (None:
    ctx's)."""

    def __init__(self, ctx: Context, views, images, scenes=None):
        h = C.c_void_p()
        if scenes is None:
            arr = (Request * len(views))(*[Request(v, _ptr(im)) for v, im in zip(views, images)])
            ctx._check(lib.r3d_cuda_batch_create(ctx.h, arr, len(views), C.byref(h)))
        else:
            arr = (SceneRequest * len(views))(*[
                SceneRequest(v, _ptr(im), sc.h if sc is not None else None)
                for v, im, sc in zip(views, images, scenes)])
            ctx._check(lib.r3d_cuda_batch_create_scenes(ctx.h, arr, len(views), C.byref(h)))
        self.ctx, self.h = ctx, h

    def close(self) -> None:
        if self.h:
            lib.r3d_cuda_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_schedule(self, **kw) -> None:
        sc = Schedule(kw.get("persistent", 1), kw.get("refill_min", 16), kw.get("tile_shape", 0),
                      kw.get("unroll", 1), kw.get("blocks_per_sm", 0), kw.get("shade_group", 0),
                      kw.get("staging", 0))
        self.ctx._check(lib.r3d_cuda_batch_set_schedule(self.h, C.byref(sc)))

    def schedule(self) -> dict:
        sc = Schedule()
        self.ctx._check(lib.r3d_cuda_batch_get_schedule(self.h, C.byref(sc)))
        return {f: getattr(sc, f) for f, _ in Schedule._fields_}

    def launch(self, total=None, stream: int = 0) -> None:
        self.ctx._check(lib.r3d_cuda_batch_launch(self.h, _ptr(total) or None, stream or None))

    def capture(self, total=None, stream: int = 0) -> None:
        self.ctx._check(lib.r3d_cuda_batch_capture(self.h, _ptr(total) or None, stream or None))

    def replay(self, stream: int = 0) -> None:
        self.ctx._check(lib.r3d_cuda_batch_replay(self.h, stream or None))

    def autotune(self, reps: int = 3) -> tuple[dict, float]:
        sc = Schedule()
        ms = C.c_float()
        self.ctx._check(lib.r3d_cuda_batch_autotune(self.h, reps, C.byref(sc), C.byref(ms)))
        return {f: getattr(sc, f) for f, _ in Schedule._fields_}, ms.value


class Volume(C.Structure):
    """r3d_volume: a raw u8 volume held by the caller."""
    _fields_ = [("voxels", C.c_void_p), ("nx", C.c_uint32), ("ny", C.c_uint32),
                ("nz", C.c_uint32), ("nbytes", C.c_size_t), ("voxel_um", C.c_float)]


class SlabDesc(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32), ("wz", C.c_uint32)]


class VslabDesc(C.Structure):
    _fields_ = [("nx", C.c_uint32), ("ny", C.c_uint32), ("nz", C.c_uint32), ("W", C.c_uint32),
                ("H", C.c_uint32), ("D", C.c_uint32), ("cache_dir", C.c_char_p),
                ("shard_url", C.c_char_p), ("z_prefetch", C.c_uint32),
                ("prefetch_slots", C.c_uint32), ("prefetch_threads", C.c_uint32)]


class BricksStats(C.Structure):
    _fields_ = [("nb", C.c_uint32), ("hot", C.c_uint32), ("hot_cap", C.c_uint32),
                ("warm_bricks", C.c_uint32), ("warm_bytes", C.c_uint64), ("warm_cap", C.c_uint64),
                ("inflight", C.c_uint32), ("decoded", C.c_uint64), ("jobs", C.c_uint64),
                ("stream_ns", C.c_uint64), ("failures", C.c_uint32), ("nlevels", C.c_uint32),
                ("lod_wanted", C.c_uint32 * 8), ("lod_requests", C.c_uint64 * 8),
                ("net_pending", C.c_uint32), ("net_fetched", C.c_uint64),
                ("net_encoded", C.c_uint64)]


def _volume(vol) -> Volume:
    nz, ny, nx = vol.shape
    return Volume(_ptr(vol), nx, ny, nz, nx * ny * nz, 0.0)


class Renderer:
    """The headless render3d interface (r3d_render.h)."""

    def __init__(self, w: int, h: int):
        cfg = RenderConfig(False, False, None, 0, True, w, h)
        r = C.c_void_p()
        if lib.r3d_create(None, C.byref(cfg), C.byref(r)) != 0:
            raise RuntimeError("r3d_create failed")
        self.r = r
        self.w, self.h = w, h

    def close(self) -> None:
        if self.r:
            lib.r3d_destroy(self.r)
            self.r = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, rc: int, what: str) -> None:
        if rc != 0:
            raise RuntimeError(f"{what} failed ({rc})")

    def upload_volume(self, vol) -> None:
        nz, ny, nx = vol.shape
        self._ok(lib.r3d_upload_volume(self.r, C.byref(VolumeDesc(nx, ny, nz, 128, 1.0)),
                                       _ptr(vol)), "r3d_upload_volume")

    def bricks_begin_volume(self, vol, nlev: int, min_max: int = 0) -> None:
        nz, ny, nx = vol.shape
        self._ok(lib.r3d_bricks_begin_volume(self.r, C.byref(VolumeDesc(nx, ny, nz, 128, 1.0)),
                                             _ptr(vol), nlev, min_max), "r3d_bricks_begin")

    def bricks_begin_shard(self, vol, pool_bpa: int = 0) -> None:
        self._ok(lib.r3d_bricks_begin_shard(self.r, _ptr(vol), vol.shape[0], pool_bpa),
                 "r3d_bricks_begin_shard")

    def bricks_params(self, p: FrameParams) -> None:
        lib.r3d_bricks_params(self.r, C.byref(p))

    # section modes and flattened views, with render.h's names
    def slab_init(self, shape, wz: int) -> None:
        nz, ny, nx = shape
        self._ok(lib.r3d_slab_init(self.r, C.byref(SlabDesc(nx, ny, nz, wz))), "r3d_slab_init")

    def slab_window(self, vol, z0: int) -> None:
        self._ok(lib.r3d_slab_window(self.r, C.byref(_volume(vol)), z0), "r3d_slab_window")

    def slab_params(self, p: FrameParams) -> None:
        lib.r3d_slab_params(self.r, C.byref(p))

    def clip_begin_volume(self, vol, depth_max: int) -> None:
        self._ok(lib.r3d_clip_begin_volume(self.r, C.byref(_volume(vol)), depth_max),
                 "r3d_clip_begin_volume")

    def clip_frame(self, fx: float, fy: float, z0: int, p: FrameParams) -> None:
        self._ok(lib.r3d_clip_frame(self.r, fx, fy, z0, C.byref(p)), "r3d_clip_frame")

    def bricks_begin_stream(self, vol, nlev: int, nslots: int) -> None:
        nz, ny, nx = vol.shape
        self._ok(lib.r3d_bricks_begin_stream(self.r, C.byref(VolumeDesc(nx, ny, nz, 128, 1.0)),
                                             _ptr(vol), nlev, nslots), "r3d_bricks_begin_stream")

    def bricks_stream(self, view: "StreamView") -> None:
        lib.r3d_bricks_stream(self.r, view.eye, view.fwd, view.half_tan, view.pixel_cone,
                              view.slice_z0, view.slice_depth, view.gate, view.budget)

    def bricks_postfilter(self, mode: int, amount: float = 0.0, targets: int = 1) -> None:
        lib.r3d_bricks_postfilter(self.r, mode, amount, targets)

    def bricks_labels(self, src: BrickSrc) -> None:
        self._srcs = getattr(self, "_srcs", {})
        self._srcs[2] = src
        self._ok(lib.r3d_bricks_labels(self.r, C.byref(src)), "r3d_bricks_labels")

    def bricks_labels_sync(self, budget: int = 0) -> None:
        lib.r3d_bricks_labels_sync(self.r, budget)

    def bricks_regatlas(self, src: BrickSrc) -> None:
        self._srcs = getattr(self, "_srcs", {})
        self._srcs[3] = src
        self._ok(lib.r3d_bricks_regatlas(self.r, C.byref(src)), "r3d_bricks_regatlas")

    def bricks_regatlas_sync(self, budget: int = 0) -> None:
        lib.r3d_bricks_regatlas_sync(self.r, budget)

    def bricks_regatlas_detach(self) -> None:
        lib.r3d_bricks_regatlas_detach(self.r)

    def bricks_refilter(self) -> None:
        lib.r3d_bricks_refilter(self.r)

    def bricks_stream_begin(self) -> bool:
        return bool(lib.r3d_bricks_stream_begin(self.r))

    def bricks_stream_box(self, lo, hi, pixel_cone: float, gate: float = 0.0) -> None:
        lib.r3d_bricks_stream_box(self.r, (C.c_float * 3)(*lo), (C.c_float * 3)(*hi), pixel_cone,
                                  gate)

    def bricks_stream_point(self, p, level: int, gate: float = 0.0) -> None:
        lib.r3d_bricks_stream_point(self.r, (C.c_float * 3)(*p), level, gate)

    def bricks_stream_submit(self, budget: int) -> None:
        lib.r3d_bricks_stream_submit(self.r, budget)

    def bricks_stats(self) -> BricksStats:
        st = BricksStats()
        lib.r3d_bricks_get_stats(self.r, C.byref(st))
        return st

    def bricks_overlay_volume(self, which: int, vol) -> None:
        nz, ny, nx = vol.shape
        self._ok(lib.r3d_bricks_overlay_volume(self.r, which,
                                               C.byref(VolumeDesc(nx, ny, nz, 128, 1.0)),
                                               _ptr(vol)), "r3d_bricks_overlay_volume")

    def vslab_begin_volume(self, vol, W: int, H: int, D: int, z_prefetch: int = 0) -> None:
        nz, ny, nx = vol.shape
        d = VslabDesc(nx, ny, nz, W, H, D, None, None, z_prefetch, 0, 0)
        self._ok(lib.r3d_vslab_begin_volume(self.r, C.byref(d), _ptr(vol)),
                 "r3d_vslab_begin_volume")

    def vslab_frame(self, fx: float, fy: float, z0: int, budget: int, p: FrameParams) -> None:
        lib.r3d_vslab_frame(self.r, fx, fy, z0, budget, C.byref(p))

    def vslab_get(self) -> tuple[tuple[int, int, int], int]:
        o = (C.c_int64 * 3)()
        pending = C.c_uint32()
        lib.r3d_vslab_get(self.r, o, C.byref(pending))
        return tuple(o), pending.value

    def surf_begin(self, coords, normals) -> None:
        gh, gw = coords.shape[:2]
        self._ok(lib.r3d_surf_begin(self.r, gw, gh, _ptr(coords), _ptr(normals)),
                 "r3d_surf_begin")

    def surf_swap(self, coords, normals, sx: float, sy: float) -> None:
        gh, gw = coords.shape[:2]
        self._ok(lib.r3d_surf_swap(self.r, gw, gh, _ptr(coords), _ptr(normals), sx, sy),
                 "r3d_surf_swap")

    def surfvol_begin(self, W: int, H: int, L: int, nback: int, sx: float, sy: float) -> None:
        self._ok(lib.r3d_surfvol_begin(self.r, W, H, L, nback, sx, sy), "r3d_surfvol_begin")

    def surfvol_window(self, u0: float, v0: float, step: float, zoff0: float) -> None:
        lib.r3d_surfvol_window(self.r, u0, v0, step, zoff0)

    def surfvol_overlay_enable(self, on: bool) -> None:
        lib.r3d_surfvol_overlay_enable(self.r, on)

    def surfvol_regtap(self, on: bool) -> None:
        lib.r3d_surfvol_regtap(self.r, on)

    def surfvol_inkpred(self, pred, g0u: float, g0v: float, px_per_grid: float) -> None:
        pred = np.ascontiguousarray(pred, np.float32)
        self._ok(lib.r3d_surfvol_inkpred(self.r, _ptr(pred), pred.shape[1], pred.shape[0], g0u,
                                         g0v, px_per_grid), "r3d_surfvol_inkpred")

    def surfvol_inkpred_clear(self) -> None:
        lib.r3d_surfvol_inkpred_clear(self.r)

    def surfvol_params(self, p: FrameParams) -> None:
        lib.r3d_surfvol_params(self.r, C.byref(p))

    def set_transfer(self, lut: np.ndarray) -> None:
        self._ok(lib.r3d_set_transfer(self.r, _ptr(np.ascontiguousarray(lut, np.uint8))),
                 "r3d_set_transfer")

    def set_quality(self, q: int) -> None:
        lib.r3d_set_quality(self.r, q)

    def set_alpha_cutoff(self, c: float) -> None:
        self._ok(lib.r3d_set_alpha_cutoff(self.r, c), "r3d_set_alpha_cutoff")

    def frame(self, p: FrameParams, stats: FrameStats | None = None) -> None:
        self._ok(lib.r3d_frame(self.r, C.byref(p), C.byref(stats) if stats else None),
                 "r3d_frame")

    def frame_views(self, views, stats: FrameStats | None = None) -> None:
        arr = (FrameParams * len(views))(*views)
        self._ok(lib.r3d_frame_views(self.r, arr, len(views),
                                     C.byref(stats) if stats else None), "r3d_frame_views")

    def read_frame(self, out=None):
        w, h = C.c_uint32(), C.c_uint32()
        if out is None:  # the size first (rgba NULL queries it)
            lib.r3d_read_frame(self.r, None, C.byref(w), C.byref(h))
            out = np.empty((h.value, w.value, 4), np.uint8)
        elif out.nbytes < self.w * self.h * 4:
            raise ValueError("read_frame: the buffer is smaller than the frame")
        self._ok(lib.r3d_read_frame(self.r, _ptr(out), C.byref(w), C.byref(h)),
                 "r3d_read_frame")
        return out

    @property
    def cuda(self) -> int:
        return lib.r3d_renderer_cuda(self.r)
