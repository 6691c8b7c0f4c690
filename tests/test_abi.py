"""The C-ABI boundary: r3d_frame_params layout (the reference's 248-byte
block, src/render/render_types.h:47-94), and every function declared in
include/*.h exported by the built library (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# offsets of the reference layout (checked with gcc against render_types.h)
OFFSETS = {"cam_origin": 0, "step_voxels": 12, "cam_right": 16, "density": 28, "cam_up": 32,
           "lod_bias": 44, "cam_forward": 48, "max_mip": 60, "viewport": 64, "mode": 72,
           "frame_index": 76, "threshold": 80, "slab_grid": 84, "slab_wz": 88,
           "slab_z0": 92, "slab_nx": 96, "slab_ny": 100, "slab_px": 104, "slab_py": 108,
           "slab_depth": 112, "clip_valid": 116, "clip_orig": 120, "vol_r0": 168,
           "vol_tx": 180, "vol_r1": 184, "vol_ty": 196, "vol_r2": 200, "vol_tz": 212,
           "brick_mode": 216, "skip_gate": 220, "slab_x0": 224, "slab_y0": 228,
           "view_org": 232, "view_flags": 236, "overlay_gain": 240, "overlay_flags": 244}


def test_frame_params_layout(rb, orc):
    for fp in (rb.FrameParams, orc.FrameParams):  # the library's and the oracle's bindings
        assert C.sizeof(fp) == 248
        for name, off in OFFSETS.items():
            assert getattr(fp, name).offset == off, name


def test_c_header_layout_with_gcc(tmp_path):
    """The C header compiles as C23 and places every field at the
    reference's offset."""
    src = tmp_path / "lay.c"
    body = "\n".join(f'  printf("{k} %zu\\n", offsetof(r3d_frame_params, {k}));'
                     for k in OFFSETS)
    src.write_text('#include <stddef.h>\n#include <stdio.h>\n#include "r3d_types.h"\n'
                   "int main(void) {\n" + body + '\n  printf("size %zu\\n", '
                   "sizeof(r3d_frame_params));\n  return 0;\n}\n")
    exe = tmp_path / "lay"
    subprocess.run(["/usr/bin/gcc", "-std=c2x", "-I" + os.path.join(ROOT, "include"), str(src),
                    "-o", str(exe)], check=True)
    out = dict(ln.split() for ln in subprocess.run([str(exe)], capture_output=True, text=True,
                                                   check=True).stdout.splitlines())
    assert int(out["size"]) == 248
    for k, off in OFFSETS.items():
        assert int(out[k]) == off, k


def _declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h") or h == "r3d_fmath.h":
            continue
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[a-zA-Z_][\w \*]*?\b(r3d_\w+)\s*\(", text, flags=re.M):
            if "typedef" not in m.group(0) and "#define" not in m.group(0):
                names.add(m.group(1))
    return names


def test_library_exports_every_declared_function(rb):
    names = _declared_functions()
    assert len(names) > 40
    missing = [n for n in sorted(names) if not hasattr(rb.lib, n)]
    assert not missing, missing
