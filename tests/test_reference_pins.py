"""CPU pins of the oracle and of the library's host helpers against the
reference: its own conformance test (tests/test_gpu.c, built unmodified),
its host code (camera.c, transfer.c, lod.h, mathx.h) through the committed
golden outputs, and the known answers of its tests/test_quick.c."""
import ctypes as C
import math
import os
import subprocess

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_host.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLDEN)


def test_reference_test_gpu_accepts_oracle(orc):
    """tests/test_gpu.c of the reference (64^3 shells, FLAT mode, default
    orbit camera, identity TF) against the oracle: mean <= 2, max <= 64 LSB."""
    if not os.path.exists(orc.REF_TEST_GPU):
        pytest.skip("oracle/_ref/test_gpu not built (needs the reference tree at build time)")
    r = subprocess.run([orc.REF_TEST_GPU, orc.CLI_PATH], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "test_gpu: ok" in r.stdout
    line = [ln for ln in r.stdout.splitlines() if "mean err" in ln][0]
    mean = float(line.split("mean err")[1].split()[0])
    assert mean <= 0.5  # far inside the reference's 2 LSB budget


def test_camera_basis_bits(rb, orc, gold):
    for i in range(gold["cam_yaw"].size):
        yaw, pitch, asp = (float(gold[k][i]) for k in ("cam_yaw", "cam_pitch", "cam_aspect"))
        want = gold["cam_basis"][i]
        r, u, f = (C.c_float * 3)(), (C.c_float * 3)(), (C.c_float * 3)()
        orc.lib.orc_camera_basis(yaw, pitch, 1.04719755, asp, r, u, f)
        assert np.array_equal(np.array([r[:], u[:], f[:]], np.float32), want), i
        cam = rb.HostCamera()
        rb.lib.r3d_host_camera_init(C.byref(cam), (C.c_float * 3)(0.5, 0.5, -1.5))
        cam.yaw, cam.pitch = yaw, pitch
        rb.lib.r3d_host_camera_basis(C.byref(cam), asp, r, u, f)
        assert np.array_equal(np.array([r[:], u[:], f[:]], np.float32), want), i


def test_orbit_positions_bits(rb, orc, gold):
    for i in range(gold["cam_yaw"].size):
        yaw, pitch = float(gold["cam_yaw"][i]), float(gold["cam_pitch"][i])
        want = gold["cam_orbit"][i]
        pos = (C.c_float * 3)()
        orc.lib.orc_orbit_pos(yaw, pitch, (C.c_float * 3)(0.5, 0.5, 0.5), 2.0, pos)
        assert np.array_equal(np.array(pos[:], np.float32), want)
        cam = rb.HostCamera()
        rb.lib.r3d_host_camera_init(C.byref(cam), (C.c_float * 3)(0.5, 0.5, -1.5))
        cam.yaw, cam.pitch = yaw, pitch
        rb.lib.r3d_host_camera_orbit_set(C.byref(cam), (C.c_float * 3)(0.5, 0.5, 0.5), 2.0)
        assert np.array_equal(np.array(cam.pos[:], np.float32), want)


def test_tf_luts_bits(rb, orc, gold):
    for k in range(3):
        assert np.array_equal(rb.tf_preset(k), gold["tf_presets"][k]), k
    for i in range(gold["tf_npts"].size):
        n = int(gold["tf_npts"][i])
        vals = np.ascontiguousarray(gold["tf_vals"][i, :n])
        cols = np.ascontiguousarray(gold["tf_cols"][i, :n])
        want = gold["tf_luts"][i]
        got = rb.tf_build([(int(vals[j]), tuple(int(c) for c in cols[j])) for j in range(n)])
        assert np.array_equal(got, want), i
        lut = np.zeros((256, 4), np.uint8)
        orc.lib.orc_tf_build(vals.ctypes.data, cols.ctypes.data, n, lut.ctypes.data)
        assert np.array_equal(lut, want), i


def test_lod_policy_bits(rb, orc, gold):
    for (a, b, c, d), want in zip(gold["lod_args"], gold["lod_pick"]):
        assert orc.lib.orc_lod_pick(float(a), float(b), float(c), int(d)) == want
        assert rb.lib.r3d_host_lod_pick(float(a), float(b), float(c), int(d)) == want
    for d, o, n, want in gold["lod_fallback"]:
        assert orc.lib.orc_lod_fallback(int(d), int(o), int(n)) == want
        assert rb.lib.r3d_host_lod_fallback(int(d), int(o), int(n)) == want


def test_volume_rotation_bits(rb, orc, gold):
    for (a, b, c), want in zip(gold["ypr"], gold["ypr_rows"]):
        m = (C.c_float * 9)()
        orc.lib.orc_m3_ypr(float(a), float(b), float(c), m)
        assert np.array_equal(np.array(m[:], np.float32), want)
        rb.lib.r3d_host_m3_ypr(float(a), float(b), float(c), m)
        assert np.array_equal(np.array(m[:], np.float32), want)


def test_quick_known_answers(rb):
    """Known answers of the reference's tests/test_quick.c:64-151."""
    lut = rb.tf_preset(0)
    assert lut[0][0] == 0 and lut[0][3] == 0 and lut[255][0] == 255 and lut[255][3] == 255
    assert lut[128][0] == 128
    assert rb.lib.r3d_host_tf_preset(0xFFFFFFFF, None) == 3
    lut = rb.tf_preset(1)
    assert lut[20][3] == 0 and lut[255][3] == 255 and lut[100][3] >= lut[60][3]
    assert rb.lib.r3d_host_lod_pick(0.0, 0.001, 8192.0, 8) == 0
    assert rb.lib.r3d_host_lod_pick(1.0, 0.001, 8192.0, 8) == 3
    assert rb.lib.r3d_host_lod_pick(100.0, 0.01, 8192.0, 8) == 7
    assert [rb.lib.r3d_host_lod_fallback(2, i, 5) for i in range(5)] == [2, 3, 4, 1, 0]
    assert rb.lib.r3d_host_lod_fallback(2, 5, 5) == 0xFFFFFFFF
    cam = rb.HostCamera()
    rb.lib.r3d_host_camera_init(C.byref(cam), (C.c_float * 3)(0, 0, 0))
    r, u, f = (C.c_float * 3)(), (C.c_float * 3)(), (C.c_float * 3)()
    rb.lib.r3d_host_camera_basis(C.byref(cam), 2.0, r, u, f)
    assert abs(f[2] - 1) < 1e-6 and abs(f[0]) < 1e-6 and abs(f[1]) < 1e-6
    assert abs(sum(a * b for a, b in zip(r, f))) < 1e-6
    assert abs(math.sqrt(sum(a * a for a in u)) - math.tan(cam.fov_y / 2)) < 1e-6
    assert abs(math.sqrt(sum(a * a for a in r)) - 2 * math.tan(cam.fov_y / 2)) < 1e-6
    rb.lib.r3d_host_camera_orbit_set(C.byref(cam), (C.c_float * 3)(0.5, 0.5, 0.5), 2.0)
    assert abs(cam.pos[0] - 0.5) < 1e-6 and abs(cam.pos[2] + 1.5) < 1e-6
    rb.lib.r3d_host_camera_orbit_zoom(C.byref(cam), 0.5)
    assert abs(cam.dist - 1.0) < 1e-6 and abs(cam.pos[2] + 0.5) < 1e-6
    rb.lib.r3d_host_camera_orbit_drag(C.byref(cam), math.pi / 2, 0.0)
    assert abs(cam.pos[0] + 0.5) < 1e-5 and abs(cam.pos[2] - 0.5) < 1e-5
    rb.lib.r3d_host_camera_look(C.byref(cam), 0.0, 10.0)
    assert cam.pitch < 1.5708


def test_oracle_regression_renders(rb, orc, gold):
    """The oracle's renders of two small scenes are stable (regression of
    the oracle itself, generated by tests/golden/make_golden.py)."""
    shells = gold["shells"]
    sc = orc.CubeScene(shells)
    ramp = rb.grey_ramp()
    for k, mode in enumerate((5, 0, 1, 3)):
        p = rb.camera_view(0.0, 0.0, 2.0, 96, 64, ramp, mode=mode)
        assert np.array_equal(orc.render(p, sc, ramp, 96, 64)[0], gold["shells_renders"][k])
    vol = rb.phantom(96, seed=3)
    assert int(vol.astype(np.uint64).sum()) == int(gold["phantom96_sum"][0])
    lut = rb.scroll_ramp_tf()
    p = rb.camera_view(0.6, -35 * math.pi / 180, 2.0, 96, 96, lut, step_voxels=0.5)
    img, steps, _, _, _ = orc.render(p, orc.CubeScene(vol), lut, 96, 96)
    assert np.array_equal(img, gold["phantom96_render"])
    assert np.array_equal(steps, gold["phantom96_steps"])
