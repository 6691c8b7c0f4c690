"""Generates tests/golden/ref_layout.npz from the reference's own layout
math of the section modes: src/core/slab.h (tiled slab grid, payload,
overview pyramid), src/core/clip.h (clipmap ring depths, level origins and
the recentre policy as src/vk/vkclip.c:320-346 applies it) and
src/core/vslab.h (virtual-slab payload, grids, tile bases, cell and z
ranges).  The headers are compiled unmodified from the reference tree into
oracle/_ref/libr3dref.so through oracle/ref_glue.c; this script calls them on
seeded random inputs and stores the outputs, so that the library's host
code and the oracle are pinned to the reference without the reference tree
present:

    python tests/golden/make_layout_golden.py     # needs oracle/_ref built
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def main() -> None:
    import oracle
    lib = oracle.ref_lib()
    if lib is None:
        raise SystemExit("oracle/_ref/libr3dref.so is not built (needs the reference tree)")
    U32, U64, I64, P = C.c_uint32, C.c_uint64, C.c_int64, C.c_void_p
    lib.ref_slab_layout.argtypes = [U32, U32, U32, U32, P]
    lib.ref_slab_layout.restype = C.c_int
    lib.ref_clip_sequence.argtypes = [U64, U64, U64, U32, U32, P, P, P]
    lib.ref_clip_sequence.restype = None
    lib.ref_vslab_layout.argtypes = [U64, U64, U64, U32, U32, U32, U32, P]
    lib.ref_vslab_layout.restype = C.c_int
    lib.ref_vslab_ranges.argtypes = [U64, U64, U64, U32, U32, U32, U32, I64, I64, P]
    lib.ref_vslab_ranges.restype = None
    rng = np.random.default_rng(21)
    out: dict[str, np.ndarray] = {}

    # tiled slab: random planes from 1 to 46000 voxels a side
    sides = np.concatenate([[1024, 2046, 2047, 4092, 4093, 8184, 8185, 16368, 43008, 45012,
                             45013], 10 ** rng.uniform(0, np.log10(46000), 300)]).astype(np.int64)
    args = np.stack([sides, np.roll(sides, 7)], 1)
    res = np.zeros((len(args), 31), np.int64)
    for i, (nx, ny) in enumerate(args):
        o = np.zeros(30, np.uint32)
        res[i, 0] = lib.ref_slab_layout(int(nx), int(ny), 64, 16, o.ctypes.data)
        res[i, 1:] = o
    out.update(slab_args=args, slab_out=res)

    # clipmap: volumes up to 43008 a side, 10-frame focus walks
    nclip = 60
    cargs = np.zeros((nclip, 4), np.int64)
    cfocus = np.zeros((nclip, 10, 2), np.int64)
    corig = np.zeros((nclip, 10, 6, 2), np.int64)
    cwzl = np.zeros((nclip, 6), np.int64)
    for i in range(nclip):
        nx, ny = (int(v) for v in 10 ** rng.uniform(2, np.log10(43008), 2))
        depth = int(rng.integers(1, 65))
        cargs[i] = (nx, ny, 500, depth)
        f = np.cumsum(rng.normal(0, 0.25 * max(nx, ny), (10, 2)), 0) + rng.uniform(0, 1, 2) * (nx, ny)
        f = np.clip(f, -2000, max(nx, ny) + 2000).astype(np.int64)
        cfocus[i] = f
        o = np.zeros((10, 6, 2), np.int64)
        w = np.zeros(6, np.uint32)
        lib.ref_clip_sequence(nx, ny, 500, depth, 10, f.ctypes.data, o.ctypes.data, w.ctypes.data)
        corig[i], cwzl[i] = o, w
    out.update(clip_args=cargs, clip_focus=cfocus, clip_origins=corig, clip_wzl=cwzl)

    # virtual slab: layouts (valid and rejected) and ranges
    nvs = 300
    vargs = np.zeros((nvs, 7), np.int64)
    vout = np.zeros((nvs, 19), np.int64)
    vrng = np.zeros((nvs, 6), np.int64)
    for i in range(nvs):
        nx, ny = (int(v) for v in 10 ** rng.uniform(1.5, np.log10(43008), 2))
        nz = int(10 ** rng.uniform(0.5, 4.8))
        W = int(rng.integers(32, nx + 80)) if rng.uniform() < 0.8 else nx
        H = int(rng.integers(32, ny + 80)) if rng.uniform() < 0.8 else ny
        D = int(10 ** rng.uniform(0, 3.4))
        zm = int(rng.integers(0, 40)) if rng.uniform() < 0.5 else 0
        vargs[i] = (nx, ny, nz, W, H, D, zm)
        o = np.zeros(18, np.uint32)
        vout[i, 0] = lib.ref_vslab_layout(nx, ny, nz, W, H, D, zm, o.ctypes.data)
        vout[i, 1:] = o
        org, z0 = int(rng.integers(-100, nx + 100)), int(rng.integers(-50, nz + 50))
        r = np.zeros(4, np.int64)
        if vout[i, 0] == 0:
            lib.ref_vslab_ranges(nx, ny, nz, W, H, D, zm, org, z0, r.ctypes.data)
        vrng[i] = (org, z0, *r)
    out.update(vslab_args=vargs, vslab_out=vout, vslab_ranges=vrng)
    np.savez_compressed(os.path.join(HERE, "ref_layout.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_layout.npz"),
          "vslab valid", int((vout[:, 0] == 0).sum()), "slab valid", int((res[:, 0] == 0).sum()))


if __name__ == "__main__":
    main()
