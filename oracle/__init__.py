"""ctypes bindings for the CPU oracle (liboracle.so) and for the reference's
own host code compiled from the reference tree (_ref/libr3dref.so).

Test infrastructure: only the test suite, the smoke check and the CPU
baseline of the benchmark import this package.  The oracle restates the
reference raycast on the CPU in FP32 (r3d_oracle.c); the renderer library
never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libr3dref.so")
REF_TEST_GPU = os.path.join(HERE, "_ref", "test_gpu")
CLI_PATH = os.path.join(HERE, "r3d_oracle_cli")


def build() -> None:
    """Builds liboracle.so, the oracle CLI and (when the reference tree is
    present) _ref/ with the system gcc."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


class Cube(C.Structure):
    _fields_ = [("nlevels", C.c_uint32), ("dim", (C.c_uint32 * 3) * 16),
                ("level", C.c_void_p * 16), ("occ", C.c_void_p), ("odim", C.c_uint32 * 3)]


class Slab(C.Structure):
    _fields_ = [("wz", C.c_uint32), ("nlev", C.c_uint32), ("ovs", C.c_uint32), ("nx", C.c_uint32),
                ("ny", C.c_uint32), ("z0", C.c_uint32), ("lev", (C.c_uint32 * 4) * 8),
                ("tiles", C.c_void_p * 8)]


class Clip(C.Structure):
    _fields_ = [("wzl", C.c_uint32 * 6), ("lev", C.c_void_p * 6), ("ox", C.c_float * 6),
                ("oy", C.c_float * 6), ("valid", C.c_uint32), ("nx", C.c_uint32),
                ("z0", C.c_uint32)]


class VSlab(C.Structure):
    _fields_ = [("px", C.c_uint32), ("wz", C.c_uint32), ("ntiles", C.c_uint32),
                ("gx", C.c_uint32 * 5), ("gy", C.c_uint32 * 5), ("base", C.c_uint32 * 5),
                ("tiles", C.c_void_p), ("table", C.c_void_p)]


class Surf(C.Structure):
    _fields_ = [("coords", C.c_void_p), ("normals", C.c_void_p), ("gw", C.c_uint32),
                ("gh", C.c_uint32), ("vol", C.c_void_p), ("W", C.c_uint32), ("H", C.c_uint32),
                ("L", C.c_uint32), ("mask", C.c_void_p), ("mw", C.c_uint32), ("mh", C.c_uint32),
                ("pred", C.c_void_p), ("pw", C.c_uint32), ("ph", C.c_uint32), ("pg0u", C.c_float),
                ("pg0v", C.c_float), ("pppg", C.c_float)]


class Bricks(C.Structure):
    _fields_ = [("page", C.c_void_p), ("page_words", C.c_uint32), ("pool", C.c_void_p),
                ("nslots", C.c_uint32), ("atlas", C.c_void_p), ("ovl", C.c_void_p * 4),
                ("slab", C.c_void_p), ("clip", C.c_void_p), ("vslab", C.c_void_p),
                ("surf", C.c_void_p)]


class Opts(C.Structure):
    _fields_ = [("alpha_cutoff", C.c_float), ("quality", C.c_uint32), ("threads", C.c_int)]


class Aux(C.Structure):
    _fields_ = [("steps", C.c_void_p), ("mip_index", C.c_void_p),
                ("total_steps", C.c_uint64), ("status", C.c_uint32)]


def _load():
    if not os.path.exists(LIB_PATH):
        build()
    lib = C.CDLL(LIB_PATH)
    P, U32, F = C.c_void_p, C.c_uint32, C.c_float
    lib.orc_render_view.restype = C.c_int
    lib.orc_render_view.argtypes = [P, C.POINTER(Cube), C.POINTER(Bricks), P, C.POINTER(Opts), P,
                                    U32, U32, C.POINTER(Aux)]
    lib.orc_render_pixels.restype = C.c_int
    lib.orc_render_pixels.argtypes = [P, C.POINTER(Cube), C.POINTER(Bricks), P, C.POINTER(Opts),
                                      P, U32, P, P, P]
    lib.orc_mip_levels.restype = U32
    lib.orc_mip_levels.argtypes = [U32, U32, U32, P]
    lib.orc_downsample.restype = None
    lib.orc_downsample.argtypes = [P, U32, U32, U32, P, U32, U32, U32]
    lib.orc_occupancy.restype = None
    lib.orc_occupancy.argtypes = [P, U32, U32, U32, P]
    lib.orc_build_lod_bricks.restype = C.c_int64
    lib.orc_build_lod_bricks.argtypes = [P, U32, U32, U32, U32, U32, P, U32, P, C.c_uint64]
    lib.orc_slab_layout.restype = U32
    lib.orc_slab_layout.argtypes = [U32, U32, P, P]
    lib.orc_slab_fill.restype = None
    lib.orc_slab_fill.argtypes = [P, U32, U32, U32, U32, U32, C.c_void_p * 8]
    lib.orc_postfilter.restype = None
    lib.orc_postfilter.argtypes = [P, U32, U32, F]
    lib.orc_surf_bake.restype = None
    lib.orc_surf_bake.argtypes = [P, P, F, F, F, F, F, F, U32, C.c_int]
    lib.orc_vslab_fill.restype = None
    lib.orc_vslab_fill.argtypes = [P, P, U32, U32, C.c_int64, C.c_int64, C.c_int64, U32]
    lib.orc_clip_fill.restype = None
    lib.orc_clip_fill.argtypes = [P, U32, U32, U32, U32, U32, P, C.c_void_p * 6]
    lib.orc_build_lod_overlay.restype = C.c_int
    lib.orc_build_lod_overlay.argtypes = [P, U32, U32, U32, P, U32, C.c_int, P, U32]
    lib.orc_build_shard.restype = C.c_int
    lib.orc_build_shard.argtypes = [P, U32, U32, P, P, P]
    lib.orc_shard_occupancy.restype = None
    lib.orc_shard_occupancy.argtypes = [P, U32, P, U32, P]
    lib.orc_lod_page_words.restype = U32
    lib.orc_lod_page_words.argtypes = [U32, U32, U32, U32]
    lib.orc_camera_basis.restype = None
    lib.orc_camera_basis.argtypes = [F, F, F, F, P, P, P]
    lib.orc_orbit_pos.restype = None
    lib.orc_orbit_pos.argtypes = [F, F, P, F, P]
    lib.orc_tf_build.restype = None
    lib.orc_tf_build.argtypes = [P, P, U32, P]
    lib.orc_lod_pick.restype = U32
    lib.orc_lod_pick.argtypes = [F, F, F, U32]
    lib.orc_lod_fallback.restype = U32
    lib.orc_lod_fallback.argtypes = [U32, U32, U32]
    lib.orc_diff_forward32.restype = C.c_int
    lib.orc_diff_forward32.argtypes = [P, P, P, P, F, P, P, C.c_int]
    lib.orc_diff_grad64.restype = C.c_int
    lib.orc_diff_grad64.argtypes = [P, P, P, P, F, P, C.c_int, P, P, P, P, P, P, C.c_int]
    lib.orc_fmath_eval.restype = None
    lib.orc_fmath_eval.argtypes = [P, P, P, U32]
    lib.orc_m3_ypr.restype = None
    lib.orc_m3_ypr.argtypes = [F, F, F, P]
    lib.orc_orbit_view.restype = None
    lib.orc_orbit_view.argtypes = [P, F, P, U32, U32, F, F, F, U32, U32, F, P]
    lib.orc_phantom.restype = C.c_int
    lib.orc_phantom.argtypes = [P, U32, U32, U32, C.c_uint64, C.c_int]
    return lib


lib = _load()


# r3d_frame_params (include/r3d_types.h; the reference's 248-byte layout,
# src/render/render_types.h:47-94), declared here too so that the CPU
# baseline builds its views without loading the library under test
class FrameParams(C.Structure):
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


assert C.sizeof(FrameParams) == 248
BRICK_LOD_FLAG = 0x20000  # brick_mode's LOD flag (src/vk/vkbackend.c:4511-4517)


def _p(a):
    return None if a is None else a.ctypes.data


class CubeScene:
    """A cube volume with the oracle's own mip chain and occupancy grid."""

    def __init__(self, vol: np.ndarray):
        vol = np.ascontiguousarray(vol, np.uint8)
        nz, ny, nx = vol.shape
        self.c = Cube()
        dims = ((C.c_uint32 * 3) * 16)()
        self.c.nlevels = lib.orc_mip_levels(nx, ny, nz, dims)
        self.levels = [vol]
        for m in range(1, self.c.nlevels):
            d = tuple(dims[m])
            dst = np.empty((d[2], d[1], d[0]), np.uint8)
            s = self.levels[-1]
            lib.orc_downsample(_p(s), s.shape[2], s.shape[1], s.shape[0], _p(dst), *d)
            self.levels.append(dst)
        for m, lv in enumerate(self.levels):
            self.c.dim[m][:] = (lv.shape[2], lv.shape[1], lv.shape[0])
            self.c.level[m] = lv.ctypes.data
        od = ((nx + 7) // 8, (ny + 7) // 8, (nz + 7) // 8)
        self.occ = np.empty((od[2], od[1], od[0]), np.uint8)
        lib.orc_occupancy(_p(vol), nx, ny, nz, _p(self.occ))
        self.c.occ = self.occ.ctypes.data
        self.c.odim[:] = od


class BrickScene:
    """A LOD brick cache: page table + slot pool (x fastest), and optional
    slot-parallel overlay atlases (ink, 3D ink, labels, registration)."""

    def __init__(self, page: np.ndarray, pool: np.ndarray):
        self.page = np.ascontiguousarray(page, np.uint32)
        self.pool = np.ascontiguousarray(pool, np.uint8)
        self.b = Bricks(self.page.ctypes.data, self.page.size, self.pool.ctypes.data,
                        self.pool.size // 128 ** 3)
        self.ovl = [None] * 4

    def set_overlay(self, which: int, slots: np.ndarray | None) -> None:
        self.ovl[which] = None if slots is None else np.ascontiguousarray(slots, np.uint8)
        self.b.ovl[which] = None if slots is None else self.ovl[which].ctypes.data

    def build_overlay(self, which: int, vol: np.ndarray) -> np.ndarray:
        """Overlay slot contents cut from a raw volume (labels: which == 2)."""
        vol = np.ascontiguousarray(vol, np.uint8)
        nz, ny, nx = vol.shape
        pool = np.zeros(self.pool.size, np.uint8)
        if lib.orc_build_lod_overlay(_p(vol), nx, ny, nz, _p(self.page), self.page.size,
                                     int(which == 2), _p(pool), self.b.nslots) != 0:
            raise ValueError("orc_build_lod_overlay failed")
        self.set_overlay(which, pool)
        return pool

    @classmethod
    def build(cls, vol: np.ndarray, nlev: int, min_max: int = 0) -> "BrickScene":
        vol = np.ascontiguousarray(vol, np.uint8)
        nz, ny, nx = vol.shape
        words = lib.orc_lod_page_words(nx, ny, nz, nlev)
        page = np.empty(words, np.uint32)
        n = lib.orc_build_lod_bricks(_p(vol), nx, ny, nz, nlev, min_max, _p(page), words, None, 0)
        if n < 0:
            raise ValueError("orc_build_lod_bricks failed")
        pool = np.empty(max(n, 1) * 128 ** 3, np.uint8)
        n2 = lib.orc_build_lod_bricks(_p(vol), nx, ny, nz, nlev, min_max, _p(page), words,
                                      _p(pool), n)
        assert n2 == n
        return cls(page, pool[: n * 128 ** 3] if n else pool[:0])


class ShardScene:
    """A single-level brick atlas: page table (bpa^3 entries) and atlas
    level 0 ((abpa * 128)^3), with the oracle's own mips and world-indexed
    occupancy grid."""

    def __init__(self, page: np.ndarray, atlas0: np.ndarray, bpa: int, abpa: int):
        self.page = np.ascontiguousarray(page, np.uint32)
        assert self.page.size == bpa ** 3
        a = abpa * 128
        self.levels = [np.ascontiguousarray(atlas0, np.uint8).reshape(a, a, a)]
        for m in range(1, 4):
            s, d = a >> (m - 1), a >> m
            dst = np.empty((d, d, d), np.uint8)
            lib.orc_downsample(_p(self.levels[-1]), s, s, s, _p(dst), d, d, d)
            self.levels.append(dst)
        od = bpa * 16
        self.occ = np.empty((od, od, od), np.uint8)
        lib.orc_shard_occupancy(_p(self.levels[0]), abpa, _p(self.page), bpa, _p(self.occ))
        self.atlas = Cube()
        self.atlas.nlevels = 4
        for m, lv in enumerate(self.levels):
            self.atlas.dim[m][:] = (lv.shape[2], lv.shape[1], lv.shape[0])
            self.atlas.level[m] = lv.ctypes.data
        self.atlas.occ = self.occ.ctypes.data
        self.atlas.odim[:] = (od, od, od)
        self.bpa, self.abpa = bpa, abpa
        self.identity = abpa == bpa and all(
            (int(e) & 0xFFFFFF) == b and int(e) != 0xFFFFFFFF for b, e in enumerate(self.page))
        self.b = Bricks(self.page.ctypes.data, self.page.size, None, abpa ** 3,
                        C.addressof(self.atlas))

    @property
    def brick_mode(self) -> int:
        return self.bpa | (self.abpa << 8) | (0x10000 if self.identity else 0)

    @classmethod
    def build(cls, vol: np.ndarray, abpa: int | None = None, slot_of=None) -> "ShardScene":
        vol = np.ascontiguousarray(vol, np.uint8)
        e = vol.shape[0]
        bpa = e // 128
        abpa = abpa or bpa
        page = np.empty(bpa ** 3, np.uint32)
        atlas0 = np.empty((abpa * 128,) * 3, np.uint8)
        so = None if slot_of is None else np.ascontiguousarray(slot_of, np.uint32)
        if lib.orc_build_shard(_p(vol), e, abpa, _p(so), _p(page), _p(atlas0)) < 0:
            raise ValueError("orc_build_shard failed")
        return cls(page, atlas0, bpa, abpa)


class SlabScene:
    """The tiled slab of a (nz, ny, nx) volume for the window [z0, z0 + wz),
    assembled the reference's way."""

    def __init__(self, vol: np.ndarray, wz: int, z0: int):
        vol = np.ascontiguousarray(vol, np.uint8)
        nz, ny, nx = vol.shape
        lev = ((C.c_uint32 * 4) * 8)()
        ovs = C.c_uint32()
        nl = lib.orc_slab_layout(nx, ny, lev, C.byref(ovs))
        if not nl:
            raise ValueError("slab layout")
        self.s = Slab()
        self.s.wz, self.s.nlev, self.s.ovs, self.s.nx, self.s.ny, self.s.z0 = wz, nl, ovs.value, nx, ny, z0
        self.tiles = []
        ptrs = (C.c_void_p * 8)()
        for l in range(nl):
            gx, gy, px, py = lev[l]
            self.s.lev[l][:] = (gx, gy, px, py)
            t = np.zeros((gx * gy, wz, py + 2, px + 2), np.uint8)
            self.tiles.append(t)
            ptrs[l] = t.ctypes.data
            self.s.tiles[l] = t.ctypes.data
        lib.orc_slab_fill(_p(vol), nx, ny, nz, wz, z0, ptrs)
        self.b = Bricks()
        self.b.slab = C.addressof(self.s)


CLIP_LEVELS, CLIP_TEX, CLIP_PAYLOAD, CLIP_SNAP = 6, 2048, 2046, 16


def _clip_snap(v: int, q: int) -> int:
    """src/core/clip.h:38-42: round toward minus infinity to a multiple of q."""
    return v // q * q if v >= 0 else -((-v + q - 1) // q) * q


def clip_origins(nx: int, ny: int, fx: float, fy: float, prev=None):
    """Level origins after a frame focused on (fx, fy) voxels: each level
    recentres (src/core/clip.h:48-66) on the first frame and whenever the
    focus drifted more than a quarter of its coverage from its centre, unless
    the coverage spans the whole volume (clip.h:98-108; vkclip.c:320-346
    passes the truncated focus)."""
    fx, fy = int(fx), int(fy)
    out = []
    for l in range(CLIP_LEVELS):
        s = 1 << l
        cov = CLIP_PAYLOAD * s
        if prev is not None:
            ox, oy = prev[l]
            cx, cy = ox + cov // 2, oy + cov // 2
            if (cov >= nx and cov >= ny) or not (abs(fx - cx) > cov // 4 or abs(fy - cy) > cov // 4):
                out.append((ox, oy))
                continue
        snap = CLIP_SNAP * s
        ox, oy = _clip_snap(fx - cov // 2, snap), _clip_snap(fy - cov // 2, snap)
        ox, oy = max(ox, 0), max(oy, 0)
        if ox + cov > nx:
            ox = _clip_snap(nx - cov, snap)
        if oy + cov > ny:
            oy = _clip_snap(ny - cov, snap)
        out.append((max(ox, 0), max(oy, 0)))
    return out


class ClipScene:
    """The XY clipmap of a (nz, ny, nx) volume for the window from z0 with
    the given level origins (clip_origins), every level valid."""

    def __init__(self, vol: np.ndarray, depth_max: int, origins, z0: int):
        vol = np.ascontiguousarray(vol, np.uint8)
        nz, ny, nx = vol.shape
        self.c = Clip()
        self.tex = []
        ptrs = (C.c_void_p * 6)()
        orig = (C.c_float * 12)()
        for l in range(CLIP_LEVELS):
            wzl = max(depth_max // (1 << l) + 3, 4)
            t = np.zeros((wzl, CLIP_TEX, CLIP_TEX), np.uint8)
            self.tex.append(t)
            ptrs[l] = t.ctypes.data
            self.c.wzl[l] = wzl
            self.c.lev[l] = t.ctypes.data
            self.c.ox[l], self.c.oy[l] = float(origins[l][0]), float(origins[l][1])
            orig[2 * l], orig[2 * l + 1] = float(origins[l][0]), float(origins[l][1])
        self.c.valid, self.c.nx, self.c.z0 = (1 << CLIP_LEVELS) - 1, nx, z0
        self.ny, self.depth = ny, depth_max
        lib.orc_clip_fill(_p(vol), nx, ny, nz, depth_max, z0, C.addressof(orig), ptrs)
        self.b = Bricks()
        self.b.clip = C.addressof(self.c)

    def params(self, p) -> None:
        """The view fields of a clip frame (vkclip.c:428-455), slab_depth the
        whole window."""
        p.slab_nx, p.slab_ny, p.slab_z0 = float(self.c.nx), float(self.ny), float(self.c.z0)
        p.slab_wz = p.slab_depth = self.depth
        for l in range(CLIP_LEVELS):
            p.clip_orig[l][0], p.clip_orig[l][1] = self.c.ox[l], self.c.oy[l]
        p.clip_valid, p.slab_grid, p.brick_mode = self.c.valid, 0, 0


VS_SCALE = (1, 4, 8, 16, 32)


def vslab_layout(nx, ny, nz, W, H, D, z_margin=0):
    """Window layout (src/core/vslab.h:55-105) as a dict, or None for a
    window that does not fit."""
    ring = D + 2 + 2 * z_margin
    if W < 64 or H < 64 or W > nx or H > ny or D < 2 or D > 2044 or D > nz or ring > 2046 \
            or ring > nz:
        return None
    m = max(W, H)
    px = min(max((m // 8 + 31) & ~31, 64), 2016)
    while px > 64 and (px + 2) ** 2 * ring > 3 << 30:
        px -= 32
    ex, ey = (2 if W < nx else 0), (2 if H < ny else 0)
    gx, gy, base, nt = [], [], [], 0
    for l, s in enumerate(VS_SCALE):
        cs = px * s
        base.append(nt)
        if l and m // s < 1024:
            gx.append(0)
            gy.append(0)
            continue
        gx.append(-(-W // cs) + ex)
        gy.append(-(-H // cs) + ey)
        nt += gx[-1] * gy[-1]
    return dict(nx=nx, ny=ny, nz=nz, W=W, H=H, D=D, px=px, wz=ring, z_margin=z_margin,
                gx=gx, gy=gy, base=base, ntiles=nt, x0=-1, y0=-1, z0=-1)


def _vs_zrange(v, z0):
    za = max(z0 - v["z_margin"], 0)
    zb = za + v["wz"]
    if zb > v["nz"]:
        zb = v["nz"]
        za = max(zb - v["wz"], 0)
    return za, zb


def _vs_range(v, o, n, span):
    cs = v["px"]
    return max(o // cs, 0), min((o + span - 1) // cs, (n - 1) // cs)


def _cdiv(a, b):
    """C integer division (truncating toward zero)."""
    q = abs(a) // abs(b)
    return q if (a >= 0) == (b > 0) else -q


def vslab_plan(v, cells, fx, fy, z0, budget):
    """One frame of the virtual slab's fill scheduler (vkbackend.c:6390-6620)
    with every queued fill finishing within the frame: returns the jobs
    (cx, cy, zs0, nz) in order and moves the window.  cells: slot ->
    [cx, cy, za, zb] (cx None: empty)."""
    px0, py0, pz0 = v["x0"], v["y0"], v["z0"]
    W, H, D, px = v["W"], v["H"], v["D"], v["px"]
    x0, y0 = int(fx) - W // 2, int(fy) - H // 2
    x0 = 0 if x0 < 0 else x0 & ~15
    y0 = 0 if y0 < 0 else y0 & ~15
    mx, my = max(v["nx"] - W, 0), max(v["ny"] - H, 0)
    x0 = mx & ~15 if x0 > mx else x0
    y0 = my & ~15 if y0 > my else y0
    z0 = min(max(z0, 0), max(v["nz"] - D, 0))
    za_w, zb_w = _vs_zrange(v, z0)
    vis_end = min(z0 + D + 2, v["nz"])
    up = pz0 < 0 or z0 >= pz0
    v["x0"], v["y0"], v["z0"] = x0, y0, z0
    cx0, cx1 = _vs_range(v, x0, v["nx"], W)
    cy0, cy1 = _vs_range(v, y0, v["ny"], H)
    gx, gy = v["gx"][0], v["gy"][0]
    ccx, ccy = (x0 + W // 2) // px, (y0 + H // 2) // px
    mchunks = (v["z_margin"] + 15) // 16
    jobs = []
    for cy in range(cy0, cy1 + 1):
        for cx in range(cx0, cx1 + 1):
            if len(jobs) >= 64:
                break
            c = cells[(cy % gy) * gx + cx % gx]
            held = c[0] == cx and c[1] == cy
            s0, s1, prio = z0, vis_end, 0
            if held:
                za, zb = c[2], c[3]
                if za <= za_w and zb >= zb_w:
                    continue
                visible = za <= z0 and zb >= vis_end
                if not visible and za < vis_end and zb > z0:
                    if za > z0:
                        s1 = min(za, vis_end)
                    else:
                        s0 = max(zb, z0)
                elif visible:
                    if up and zb < zb_w:
                        grow, extra = True, 0
                    elif not up and za > za_w:
                        grow, extra = False, 0
                    elif za > za_w:
                        grow, extra = False, mchunks
                    else:
                        grow, extra = True, mchunks
                    if grow:
                        s0, s1, filled = zb, min(zb + 16, zb_w), zb - vis_end
                    else:
                        s1, s0, filled = za, max(za - 16, za_w), z0 - za
                    prio = 1 + extra + (filled // 16 if filled > 0 else 0)
            jobs.append([prio, (cx - ccx) ** 2 + (cy - ccy) ** 2, cx, cy, s0, s1 - s0])
        if len(jobs) >= 64:
            break
    n = len(jobs)
    for a in range(n - 1):  # the reference's exchange sort
        for b in range(a + 1, n):
            if jobs[b][0] < jobs[a][0] or (jobs[b][0] == jobs[a][0] and jobs[b][1] < jobs[a][1]):
                jobs[a], jobs[b] = jobs[b], jobs[a]
    out = [tuple(j[2:]) for j in jobs[:budget]]
    if px0 >= 0 and (x0 != px0 or y0 != py0):
        pf = []
        mxc, myc = (v["nx"] - 1) // px, (v["ny"] - 1) // px
        if x0 != px0:
            cxc = cx1 + 1 if x0 > px0 else cx0 - 1
            if 0 <= cxc <= mxc and cx1 - cx0 + 2 <= gx:
                pf += [(cxc, cy) for cy in range(cy0, cy1 + 1)][:48]
        if y0 != py0:
            cyc = cy1 + 1 if y0 > py0 else cy0 - 1
            if 0 <= cyc <= myc and cy1 - cy0 + 2 <= gy:
                pf += [(cx, cyc) for cx in range(cx0, cx1 + 1)][:48 - len(pf)]
        for cx, cy in pf:
            if len(out) >= budget:
                break
            c = cells[(cy % gy) * gx + cx % gx]
            if c[0] == cx and c[1] == cy and c[2] <= za_w and c[3] >= zb_w:
                continue
            if any(j[0] == cx and j[1] == cy for j in out):
                continue
            out.append((cx, cy, za_w, zb_w - za_w))
    return out


def vslab_apply(v, cells, job):
    """A finished fill in the ledger (vkbackend.c:6408-6430); returns the slot."""
    cx, cy, zs0, nz = job
    za_w, zb_w = _vs_zrange(v, v["z0"])
    slot = (cy % v["gy"][0]) * v["gx"][0] + cx % v["gx"][0]
    c = cells[slot]
    if c[0] != cx or c[1] != cy:
        c[2], c[3] = zs0, zs0 + nz
    else:
        c[2], c[3] = min(c[2], zs0), max(c[3], zs0 + nz)
    c[0], c[1] = cx, cy
    c[2] = max(c[2], za_w)
    c[3] = max(min(c[3], zb_w), c[2])
    return slot


class VSlabScene:
    """The virtual slab of a (nz, ny, nx) volume, driven frame by frame with
    the scheduler restated above; the tiles are filled by the oracle's
    restatement of the reference's fill."""

    def __init__(self, vol: np.ndarray, W: int, H: int, D: int, z_margin: int = 0):
        self.vol = np.ascontiguousarray(vol, np.uint8)
        nz, ny, nx = self.vol.shape
        self.v = vslab_layout(nx, ny, nz, W, H, D, z_margin)
        if self.v is None:
            raise ValueError("vslab layout")
        v = self.v
        T = v["px"] + 2
        self.tiles = np.zeros((v["ntiles"], v["wz"], T, T), np.uint8)
        nslot = v["gx"][0] * v["gy"][0]
        self.table = np.zeros((nslot, 4), np.uint32)
        self.cells = [[None, None, 0, 0] for _ in range(nslot)]
        self.s = VSlab()
        self.s.px, self.s.wz, self.s.ntiles = v["px"], v["wz"], v["ntiles"]
        for l in range(5):
            self.s.gx[l], self.s.gy[l], self.s.base[l] = v["gx"][l], v["gy"][l], v["base"][l]
        self.s.tiles, self.s.table = self.tiles.ctypes.data, self.table.ctypes.data
        self.b = Bricks()
        self.b.vslab = C.addressof(self.s)

    def frame(self, fx, fy, z0, budget):
        """Plans and runs one frame's fills; returns the jobs."""
        nz, ny, nx = self.vol.shape
        jobs = vslab_plan(self.v, self.cells, fx, fy, z0, budget)
        for j in jobs:
            cx, cy, zs0, n = j
            if n:
                lib.orc_vslab_fill(C.byref(self.s), _p(self.vol), nx, ny, cx, cy, zs0, n)
            slot = vslab_apply(self.v, self.cells, j)
            c = self.cells[slot]
            self.table[slot] = ((c[0] & 1023) | ((c[1] & 1023) << 10) | 0x80000000, c[2], c[3], 0)
        return jobs

    def params(self, p) -> None:
        """The view fields of the frame (vkbackend.c:6628-6645)."""
        v = self.v
        p.slab_grid = v["gx"][0] | (v["gy"][0] << 6) | (1 << 24)
        p.brick_mode = sum((v["gx"][l] | (v["gy"][l] << 4)) << ((l - 1) * 8) for l in range(1, 5))
        p.slab_wz, p.slab_z0 = v["wz"], float(max(v["z0"], 0))
        p.slab_nx, p.slab_ny = float(v["W"]), float(v["H"])
        p.slab_px = p.slab_py = float(v["px"])
        p.slab_depth = v["D"]
        p.slab_x0, p.slab_y0 = float(max(v["x0"], 0)), float(max(v["y0"], 0))
        p.clip_valid = 0


class SurfScene:
    """A flattened segment over a LOD brick cache (BrickScene): the grids
    (gh, gw, 4) float32 of surface points (xyz, valid) and normals, a
    W x H x L flattened volume baked by the oracle's restatement of the
    reference's bake, and an optional supervision mask (mh, mw) u8."""

    def __init__(self, bricks: "BrickScene", coords, normals, W: int, H: int, L: int,
                 nback: int, sx: float, sy: float, mask=None):
        self.bricks = bricks
        self.coords = np.ascontiguousarray(coords, np.float32)
        self.normals = np.ascontiguousarray(normals, np.float32)
        gh, gw = self.coords.shape[:2]
        self.vol = np.zeros((L, H, W, 2), np.uint8)
        self.nback = nback if nback < L else L // 2
        self.sx, self.sy = sx, sy
        self.mask = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        self.s = Surf(self.coords.ctypes.data, self.normals.ctypes.data, gw, gh,
                      self.vol.ctypes.data, W, H, L,
                      None if self.mask is None else self.mask.ctypes.data,
                      0 if self.mask is None else self.mask.shape[1],
                      0 if self.mask is None else self.mask.shape[0])
        self.b = Bricks()
        C.memmove(C.addressof(self.b), C.addressof(bricks.b), C.sizeof(Bricks))
        self.b.surf = C.addressof(self.s)
        self.window = None

    def inkpred(self, pred, g0u: float, g0v: float, px_per_grid: float) -> None:
        """Live 2.5D ink prediction for later bakes: (ph, pw) float32
        probabilities, texel (0, 0) at grid coordinates (g0u, g0v);
        pred None drops it (vkbackend.c:1900-1968)."""
        if pred is None:
            self.pred = None
            self.s.pred, self.s.pw, self.s.ph = None, 0, 0
            return
        self.pred = np.ascontiguousarray(pred, np.float32)
        self.s.pred = self.pred.ctypes.data
        self.s.ph, self.s.pw = self.pred.shape
        self.s.pg0u, self.s.pg0v, self.s.pppg = g0u, g0v, px_per_grid

    def bake(self, u0: float, v0: float, step: float, zoff0: float, ovl: int = -1) -> None:
        lib.orc_surf_bake(C.byref(self.s), C.byref(self.bricks.b), u0, v0, step, zoff0,
                          self.sx, self.sy, self.nback, ovl)
        self.window = (np.float32(u0), np.float32(v0), np.float32(step), np.float32(zoff0))

    def params(self, p) -> None:
        """View fields of the baked window (vkbackend.c:2054-2066)."""
        u0, v0, step, zoff0 = self.window
        p.slab_x0, p.slab_y0, p.slab_px = float(u0), float(v0), float(step)
        p.slab_nx, p.slab_ny, p.slab_wz = float(self.s.W), float(self.s.H), self.s.L
        p.slab_grid, p.max_mip = self.nback, float(zoff0)
        p.vol_tx, p.vol_ty = float(np.float32(self.sx)), float(np.float32(self.sy))
        p.view_flags |= 2


def _scene_args(scene):
    cube = C.byref(scene.c) if isinstance(scene, CubeScene) else None
    br = (C.byref(scene.b)
          if isinstance(scene, (BrickScene, ShardScene, SlabScene, ClipScene, VSlabScene,
                                SurfScene))
          else None)
    return cube, br


def render(params, scene, lut: np.ndarray, img_w: int, img_h: int, cutoff: float = 0.98,
           quality: int = 0, threads: int = 0, img: np.ndarray | None = None,
           want_aux: bool = True):
    """Renders one view; returns (img (h, w, 4) u8, steps, mip_index, total, status)."""
    if img is None:
        img = np.zeros((img_h, img_w, 4), np.uint8)
    lut = np.ascontiguousarray(lut, np.uint8)
    steps = np.zeros((img_h, img_w), np.uint32) if want_aux else None
    mipi = np.zeros((img_h, img_w), np.uint32) if want_aux else None
    aux = Aux(_p(steps), _p(mipi), 0, 0)
    cube, br = _scene_args(scene)
    rc = lib.orc_render_view(C.byref(params), cube, br, _p(lut), C.byref(Opts(cutoff, quality,
                             threads)), _p(img), img_w, img_h, C.byref(aux))
    if rc != 0:
        raise ValueError("orc_render_view rejected the view")
    return img, steps, mipi, aux.total_steps, aux.status


def render_pixels(params, scene, lut: np.ndarray, xy: np.ndarray, cutoff: float = 0.98,
                  quality: int = 0, threads: int = 0):
    """Rays of the listed dispatch-thread coordinates xy (n, 2); returns
    (rgba (n, 4), steps (n,), mip_index (n,))."""
    xy = np.ascontiguousarray(xy, np.uint32)
    n = xy.shape[0]
    rgba = np.zeros((n, 4), np.uint8)
    steps = np.zeros(n, np.uint32)
    mipi = np.zeros(n, np.uint32)
    lut = np.ascontiguousarray(lut, np.uint8)
    cube, br = _scene_args(scene)
    rc = lib.orc_render_pixels(C.byref(params), cube, br, _p(lut),
                               C.byref(Opts(cutoff, quality, threads)), _p(xy), n, _p(rgba),
                               _p(steps), _p(mipi))
    if rc != 0:
        raise ValueError("orc_render_pixels rejected the view")
    return rgba, steps, mipi


def fmath_eval(x: np.ndarray, y: np.ndarray) -> np.ndarray:
    """CPU log2, exp2, pow and x^24 of the shared header, (n, 4) float32."""
    x = np.ascontiguousarray(x, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    out = np.empty((x.size, 4), np.float32)
    lib.orc_fmath_eval(_p(x), _p(y), _p(out), x.size)
    return out


def diff_forward32(params, dens: np.ndarray, lut: np.ndarray, cutoff: float = 0.98,
                   threads: int = 0):
    """FP32 differentiable render of one view: (rgb (h, w, 3) float32, steps)."""
    dens = np.ascontiguousarray(dens, np.float32)
    lut = np.ascontiguousarray(lut, np.float32)
    n = np.array(dens.shape[::-1], np.uint32)
    w, h = params.viewport[0], params.viewport[1]
    rgb = np.zeros((h, w, 3), np.float32)
    steps = np.zeros((h, w), np.uint32)
    rc = lib.orc_diff_forward32(C.byref(params), _p(dens), _p(n), _p(lut), cutoff, _p(rgb),
                                _p(steps), threads)
    if rc != 0:
        raise ValueError("orc_diff_forward32 rejected the view")
    return rgb, steps


def diff_grad64(params, dens: np.ndarray, lut: np.ndarray, dl_drgb: np.ndarray,
                cutoff: float = 0.98, decisions32: bool = True, threads: int = 0,
                dec_dens: np.ndarray | None = None, dec_lut: np.ndarray | None = None):
    """FP64 render and gradients: (rgb64, g_dens, g_lut (256, 4), g_density).
    With decisions32, the contributing samples and termination come from the
    FP32 render of (dec_dens, dec_lut) when given (frozen decisions)."""
    if dec_dens is not None:
        dec_dens = np.ascontiguousarray(dec_dens, np.float32)
    if dec_lut is not None:
        dec_lut = np.ascontiguousarray(dec_lut, np.float32)
    dens = np.ascontiguousarray(dens, np.float32)
    lut = np.ascontiguousarray(lut, np.float32)
    g = np.ascontiguousarray(dl_drgb, np.float32)
    n = np.array(dens.shape[::-1], np.uint32)
    w, h = params.viewport[0], params.viewport[1]
    rgb = np.zeros((h, w, 3), np.float64)
    gd = np.zeros(dens.shape, np.float64)
    gl = np.zeros((256, 4), np.float64)
    gs = np.zeros(1, np.float64)
    rc = lib.orc_diff_grad64(C.byref(params), _p(dens), _p(n), _p(lut), cutoff, _p(g),
                             int(decisions32), _p(dec_dens), _p(dec_lut), _p(gd), _p(gl),
                             _p(gs), _p(rgb), threads)
    if rc != 0:
        raise ValueError("orc_diff_grad64 rejected the view")
    return rgb, gd, gl, float(gs[0])


def ref_lib():
    """The reference's camera.c / transfer.c / lod.h / mathx.h, or None when
    _ref/ has not been built (no reference tree at build time)."""
    if not os.path.exists(REF_LIB_PATH):
        return None
    r = C.CDLL(REF_LIB_PATH)
    return r


def postfilter(slots, mode: int, amount: float = 0.0) -> np.ndarray:
    """The display filter (orc_postfilter) of (n, 128, 128, 128) u8 slots,
    returned as a filtered copy."""
    out = np.array(slots, np.uint8, order="C", copy=True).reshape(-1, 128, 128, 128)
    lib.orc_postfilter(out.ctypes.data, out.shape[0], mode, amount)
    return out


def tf_build(points) -> np.ndarray:
    """r3d_tf_build (src/core/transfer.c:5-23) of [(value, (r, g, b, a)), ...]."""
    vals = np.array([q[0] for q in points], np.uint8)
    cols = np.array([q[1] for q in points], np.uint8).reshape(-1, 4)
    lut = np.zeros((256, 4), np.uint8)
    lib.orc_tf_build(_p(vals), _p(cols), len(points), _p(lut))
    return lut


def scroll_ramp_tf() -> np.ndarray:
    """The benchmark TF: alpha 0 below 40, rising to 230 at 200 and flat to
    255, grey RGB ramp."""
    return tf_build([(0, (0, 0, 0, 0)), (40, (40, 40, 40, 0)), (200, (200, 200, 200, 230)),
                     (255, (255, 255, 255, 230))])


def orbit_view(ph: float, w: int, h: int, lut: np.ndarray, target=(0.5, 0.5, 0.5),
               step_voxels: float = 1.0, density: float = 1.0, lod_bias: float = 0.0,
               mode: int = 0, frame_index: int = 0, low_cut: float = 0.0) -> FrameParams:
    """The benchmark's scripted orbit view at phase ph (orc_orbit_view)."""
    p = FrameParams()
    lib.orc_orbit_view(C.byref(p), ph, _p(np.array(target, np.float32)), w, h, step_voxels,
                       density, lod_bias, mode, frame_index, low_cut,
                       _p(np.ascontiguousarray(lut, np.uint8)))
    return p


def phantom(n, seed: int = 1234, threads: int = 0) -> np.ndarray:
    """The seeded scroll phantom (orc_phantom) as a (nz, ny, nx) u8 array."""
    nx, ny, nz = (n, n, n) if isinstance(n, int) else n
    vol = np.empty((nz, ny, nx), np.uint8)
    if lib.orc_phantom(_p(vol), nx, ny, nz, seed, threads) != 0:
        raise ValueError("orc_phantom: bad arguments")
    return vol
