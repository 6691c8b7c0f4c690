"""Generates tests/golden/ref_host.npz from the reference's own host code.

The reference's src/core/camera.c and src/core/transfer.c, and the inline
helpers of src/core/lod.h and src/core/mathx.h, are compiled unmodified from
the reference tree into oracle/_ref/libr3dref.so (oracle/Makefile).  This
script calls them on a grid of inputs and stores the outputs, so that the
oracle and the library's host helpers can be pinned to the reference without
the reference tree present:

    python tests/golden/make_golden.py        # needs oracle/_ref built

Also stored: oracle renders of two small scenes (the 64^3 "shells" volume of
the reference's tests/test_gpu.c and a 96^3 scroll phantom), as regression
fixtures of the oracle itself.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


class RefCamera(C.Structure):
    """r3d_camera of src/core/camera.h:11-19."""
    _fields_ = [("pos", C.c_float * 3), ("yaw", C.c_float), ("pitch", C.c_float),
                ("fov_y", C.c_float), ("target", C.c_float * 3), ("dist", C.c_float)]


class RefTfPoint(C.Structure):
    _fields_ = [("value", C.c_uint8), ("rgba", C.c_uint8 * 4)]


class RefTf(C.Structure):
    _fields_ = [("pts", RefTfPoint * 16), ("npts", C.c_uint32)]


class V3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


def ref_lib():
    import oracle
    lib = oracle.ref_lib()
    if lib is None:
        raise SystemExit("oracle/_ref/libr3dref.so is not built (needs the reference tree)")
    lib.r3d_camera_init.argtypes = [C.POINTER(RefCamera), V3]
    lib.r3d_camera_basis.argtypes = [C.POINTER(RefCamera), C.c_float, C.POINTER(V3),
                                     C.POINTER(V3), C.POINTER(V3)]
    lib.r3d_camera_orbit_set.argtypes = [C.POINTER(RefCamera), V3, C.c_float]
    lib.r3d_tf_build.argtypes = [C.POINTER(RefTf), C.c_void_p]
    lib.r3d_tf_preset.argtypes = [C.c_uint32, C.POINTER(RefTf)]
    lib.r3d_tf_preset.restype = C.c_uint32
    lib.ref_lod_pick.argtypes = [C.c_float, C.c_float, C.c_float, C.c_uint32]
    lib.ref_lod_pick.restype = C.c_uint32
    lib.ref_lod_fallback.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
    lib.ref_lod_fallback.restype = C.c_uint32
    lib.ref_m3_ypr.argtypes = [C.c_float, C.c_float, C.c_float, C.c_void_p]
    return lib


def camera_cases():
    rng = np.random.default_rng(11)
    yaw = np.concatenate([[0.0, math.pi / 2, math.pi, 1.0], rng.uniform(-7, 7, 60)])
    pitch = np.concatenate([[0.0, 0.0, -0.6108652, 1.55], rng.uniform(-1.6, 1.6, 60)])
    aspect = np.concatenate([[1.0, 16 / 9, 2.0, 0.5], rng.uniform(0.3, 3.0, 60)])
    return yaw.astype(np.float32), pitch.astype(np.float32), aspect.astype(np.float32)


def tf_cases():
    rng = np.random.default_rng(12)
    cases = []
    for _ in range(40):
        n = int(rng.integers(2, 9))
        vals = np.sort(rng.choice(np.arange(1, 255), n - 2, replace=False))
        vals = np.concatenate([[0], vals, [255]]).astype(np.uint8)
        cols = rng.integers(0, 256, (n, 4)).astype(np.uint8)
        cases.append((vals, cols))
    return cases


def main() -> None:
    lib = ref_lib()
    out: dict[str, np.ndarray] = {}
    # camera bases and orbit positions (src/core/camera.c)
    yaw, pitch, aspect = camera_cases()
    basis = np.zeros((yaw.size, 3, 3), np.float32)
    orbit = np.zeros((yaw.size, 3), np.float32)
    for i in range(yaw.size):
        cam = RefCamera()
        lib.r3d_camera_init(C.byref(cam), V3(0.5, 0.5, -1.5))
        cam.yaw, cam.pitch = float(yaw[i]), float(pitch[i])
        r, u, f = V3(), V3(), V3()
        lib.r3d_camera_basis(C.byref(cam), float(aspect[i]), C.byref(r), C.byref(u), C.byref(f))
        basis[i] = [[r.x, r.y, r.z], [u.x, u.y, u.z], [f.x, f.y, f.z]]
        lib.r3d_camera_orbit_set(C.byref(cam), V3(0.5, 0.5, 0.5), 2.0)
        orbit[i] = cam.pos[:]
    out.update(cam_yaw=yaw, cam_pitch=pitch, cam_aspect=aspect, cam_basis=basis,
               cam_orbit=orbit)
    # TF presets and random point sets (src/core/transfer.c)
    presets = np.zeros((3, 256, 4), np.uint8)
    for k in range(3):
        tf = RefTf()
        assert lib.r3d_tf_preset(k, C.byref(tf)) == k
        lib.r3d_tf_build(C.byref(tf), presets[k].ctypes.data)
    out["tf_presets"] = presets
    cases = tf_cases()
    vals = np.zeros((len(cases), 16), np.uint8)
    cols = np.zeros((len(cases), 16, 4), np.uint8)
    npts = np.zeros(len(cases), np.uint32)
    luts = np.zeros((len(cases), 256, 4), np.uint8)
    for i, (v, c) in enumerate(cases):
        tf = RefTf()
        tf.npts = v.size
        for k in range(v.size):
            tf.pts[k].value = int(v[k])
            tf.pts[k].rgba[:] = [int(x) for x in c[k]]
        lib.r3d_tf_build(C.byref(tf), luts[i].ctypes.data)
        vals[i, :v.size], cols[i, :v.size], npts[i] = v, c, v.size
    out.update(tf_vals=vals, tf_cols=cols, tf_npts=npts, tf_luts=luts)
    # LOD policy (src/core/lod.h)
    rng = np.random.default_rng(13)
    lp = np.stack([rng.uniform(0, 200, 300), 10 ** rng.uniform(-5, -1, 300),
                   rng.choice([256.0, 1024.0, 8192.0, 43000.0], 300),
                   rng.integers(0, 12, 300)], axis=1).astype(np.float32)
    out["lod_args"] = lp
    out["lod_pick"] = np.array([lib.ref_lod_pick(float(a), float(b), float(c), int(d))
                                for a, b, c, d in lp], np.uint32)
    fb = []
    for d in range(0, 8):
        for o in range(0, 9):
            fb.append((d, o, 8, lib.ref_lod_fallback(d, o, 8)))
    out["lod_fallback"] = np.array(fb, np.uint32)
    # volume rotation (src/core/mathx.h:34-43)
    ypr = rng.uniform(-4, 4, (50, 3)).astype(np.float32)
    rows = np.zeros((50, 9), np.float32)
    for i, (a, b, c) in enumerate(ypr):
        lib.ref_m3_ypr(float(a), float(b), float(c), rows[i].ctypes.data)
    out.update(ypr=ypr, ypr_rows=rows)

    # oracle regression renders
    import oracle
    import render3d_b200 as rb
    n = 64
    g = np.linspace(-1, 1, n, dtype=np.float32)
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    r = np.sqrt(x * x + y * y + z * z)
    s = 0.5 + 0.5 * np.sin(r * 40.0)
    shells = np.where(r < 0.9, 255.0 * s * s, 0).astype(np.uint8)
    out["shells"] = shells
    sc = oracle.CubeScene(shells)
    ramp = rb.grey_ramp()
    imgs = []
    for mode in (5, 0, 1, 3):
        p = rb.camera_view(0.0, 0.0, 2.0, 96, 64, ramp, mode=mode)
        imgs.append(oracle.render(p, sc, ramp, 96, 64)[0])
    out["shells_renders"] = np.stack(imgs)
    vol = rb.phantom(96, seed=3)
    out["phantom96_sum"] = np.array([int(vol.astype(np.uint64).sum())], np.uint64)
    lut = rb.scroll_ramp_tf()
    sc = oracle.CubeScene(vol)
    p = rb.camera_view(0.6, -35 * math.pi / 180, 2.0, 96, 96, lut, step_voxels=0.5)
    img, steps, _, _, _ = oracle.render(p, sc, lut, 96, 96)
    out["phantom96_render"] = img
    out["phantom96_steps"] = steps
    np.savez_compressed(os.path.join(HERE, "ref_host.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_host.npz"))


if __name__ == "__main__":
    main()
