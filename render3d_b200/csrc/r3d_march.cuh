// Device-side ray march shared by the forward, batched and adjoint kernels.
//
// Restates render3d's raycast compute shader (src/shaders/raycast.slang) for
// sm_100a: one thread per ray, trilinear u8 sampling in FP32 in software, the
// 256-entry TF from shared memory, ray-cone LOD, empty-space skipping, six-
// or four-tap gradient shading and front-to-back compositing.  Arithmetic is
// fixed operation by operation (explicit fmaf, compiled with -fmad=false,
// IEEE division and square root, project-written log2/exp2/pow) so that the
// CPU restatement used as the test oracle reproduces every bit, including
// the early-termination step counts and MIP indices.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "r3d_cuda.h"
#include "r3d_fmath.h"
#include "r3d_types.h"

namespace r3d {

constexpr int kMaxLevels = 16;
constexpr uint32_t kMaxSteps = 4096u;  // raycast.slang:123
constexpr float kInv255 = 1.0f / 255.0f;

enum Path {
  PATH_CUBE = 0,
  PATH_LOD_BRICKS = 1,
  PATH_SHARD = 2,
  PATH_SLAB = 3,
  PATH_CLIP = 4,
  PATH_VSLAB = 5
};
constexpr int kNumPaths = 6;
// slab_grid bit of a virtual-slab view (vkbackend.c:6629); a tiled slab's
// slab_grid stops at bit 23 (its overview scale, at most 32, in bits 16..23)
constexpr uint32_t kVslabGrid = 1u << 24;

// Sampling path of a view: the clipmap when clip_valid is set, the virtual
// slab or the tiled slab by slab_grid, else by its brick_mode word
// (raycast.slang:134-140,157-160)
__host__ __device__ inline int path_of(uint32_t brick_mode) {
  return brick_mode == 0u ? PATH_CUBE
                          : (brick_mode & R3D_BRICK_LOD_FLAG) ? PATH_LOD_BRICKS : PATH_SHARD;
}
__host__ __device__ inline int path_of_view(const r3d_frame_params &pc) {
  return pc.clip_valid                 ? PATH_CLIP
         : (pc.slab_grid & kVslabGrid) ? PATH_VSLAB
         : pc.slab_grid                ? PATH_SLAB
                                       : path_of(pc.brick_mode);
}

struct DevCube {
  const uint8_t *lev[kMaxLevels];
  uint32_t dim[kMaxLevels][3];
  uint32_t nlevels;
  uint32_t maxdim;
  const uint8_t *occ;
  uint32_t odim[3];
};

// LOD brick cache.  The page-table header is validated and decoded on the
// host when the cache is loaded; entries are read from device memory.
struct DevBricks {
  const uint32_t *page;
  uint32_t page_words;
  const uint8_t *pool;  // slot s at pool + s * 128^3, x fastest
  // per slot, 16^3 entries: max of voxels [8b, 8b+8] per axis (clamped to
  // the slot), an upper bound of any trilinear sample whose base texel lies
  // in block b
  const uint8_t *bmax;
  // per slot, 128^3 words: bytes (x, y), (x1, y), (x, y1), (x1, y1) of the
  // texel's z plane, x1 = min(x + 1, 127) and y1 likewise
  const uint32_t *quad;
  // slot-parallel overlay atlases in the same quad form: ink, 3D ink,
  // labels, registration (nullptr: not loaded)
  const uint32_t *ovl[4];
  uint32_t nslots;
  uint32_t nlev;
  float bs[3];     // base shape
  float bs_hi[3];  // max(bs - 0.001, 0): upper clamp of base-level coordinates
  float md;        // max(base shape)
  uint32_t off[kMaxLevels];
  uint32_t bd[kMaxLevels][3];
  uint32_t scale[kMaxLevels];
  float inv_scale[kMaxLevels];  // exact: scales are powers of two
};

// Single-level brick atlas: render3d's bricks mode without the LOD flag
// (a shard of bpa^3 bricks of 128^3; src/shaders/raycast.slang:163-180,
// 284-288,800-822,829-860).  The atlas is one texture of (abpa * 128)^3
// texels with 4 box-filtered mips in which slot s occupies the 128^3 region
// at (s % abpa, s / abpa % abpa, s / abpa^2) * 128; atlas.occ is the
// world-indexed dilated 8^3 occupancy grid ((bpa * 16)^3, absent bricks 0).
struct DevShard {
  DevCube atlas;
  const uint32_t *page;  // bpa^3 entries: slot | max << 24, or 0xFFFFFFFF
  uint32_t bpa, abpa;
  float n;         // bpa * 128: voxels per axis of the shard
  float inv_adim;  // 1 / (abpa * 128)
  uint32_t identity;  // every brick in its own slot: sample the atlas directly
};

// Tiled slab (raycast.slang:423-455, src/core/slab.h): a wide, thin window
// of a volume as a grid of tiles of (px + 2) x (py + 2) x wz texels -- the
// payload plus a 1-texel apron copied from the neighbours (clamped at the
// volume's edges) -- whose z is a ring: world slice s in layer s % wz.
// Level 0 is the base grid, levels 1.. the overview pyramid at scales
// 4 << (level - 1); tile (i, j) of a level starts at off + (j * gx + i) *
// (px + 2) * (py + 2) * wz bytes of the pool.
struct DevSlabLevel {
  uint32_t gx, gy, px, py;
  size_t off;
};
constexpr int kSlabLevels = 8;
struct DevSlab {
  const uint8_t *pool;
  uint32_t wz, nlev;  // ring depth; levels (base + overview)
  uint32_t ovs;       // overview downscale of the coarsest level
  float nx, ny, px, py, z0;  // the frame parameters slab_nx/ny/px/py/z0 of the window
  DevSlabLevel lev[kSlabLevels];
  // per-view constants of vs_sample's overview branch (raycast.slang:430-446),
  // evaluated once with the shader's own float expressions: the number of
  // overview levels, and per level k the grid and payload gxl, gyl, pxl, pyl
  int nov;
  float ov[kSlabLevels][4];
};

// XY clipmap (raycast.slang:357-408, src/core/clip.h): 6 nested levels of
// spacing 2^l, each a 2048 x 2048 x wzl texture (2046 payload texels and a
// 1-texel apron) whose texel (tx, ty) holds level voxel (ox / 2^l - 1 + tx,
// oy / 2^l - 1 + ty) and whose z is a ring of level slices.
constexpr int kClipLevels = 6;
struct DevClip {
  const uint8_t *lev[kClipLevels];
  uint32_t wzl[kClipLevels];
  float ox[kClipLevels], oy[kClipLevels];  // clip_orig of the frame parameters
  uint32_t valid;                          // clip_valid
  float nx, z0;                            // slab_nx, slab_z0
};

// Virtual slab (raycast.slang:321-367, src/core/vslab.h): world-anchored
// toroidal tile grids.  Level l (spacing 1, 4, 8, 16, 32) has gx x gy tiles
// of (px + 2)^2 texels by a ring of wz slices; level cell (cx, cy) lives in
// tile base + (cy mod gy) * gx + (cx mod gx), texel t of the tile holding
// level texel cx * px - 1 + t.  gx = 0: level absent.  table holds four
// words per base tile: the key of the cell it holds (0: none) and the world
// slices [za, zb) it holds.
constexpr int kVsLevels = 5;
struct DevVslab {
  const uint8_t *tiles;
  const uint32_t *table;
  size_t tile_bytes;
  uint32_t px, wz;
  uint32_t gx[kVsLevels], gy[kVsLevels], base[kVsLevels];
  float x0, y0, z0, nx;  // the frame parameters slab_x0/y0/z0 and slab_nx (= W)
};

// Byte-valued thresholds of the fetch elision.  A block maximum m (a byte)
// bounds a sample by vub = (float)m * kInv255.  Every decision the elision
// takes on vub -- below the threshold, below the skip gate, inside the TF's
// clear prefix, at most the depth mode's hit level -- is monotone in m, so
// it holds exactly for the m below a count n.  The counts of a view are
// found on the host for each launch (a guess from the inverse, settled by
// the same float expressions the device evaluates) and reach the kernels
// as launch parameters.
struct ElideCounts {
  // m < n_void: known void (below the threshold or the skip gate); m <
  // n_dec: the mode's outcome is known (FULL/FLAT: below the threshold or
  // TF-clear; DEPTH: below the threshold or at most the hit level; MIP:
  // below the threshold); raw_dec: 2^23 + n_dec, for bytes taken as
  // 2^23 + byte (qraw)
  uint32_t n_void, n_dec;
  float raw_dec;
};
__host__ __device__ inline float vub_of(uint32_t m) { return (float)m * kInv255; }
// The number of m in 0..255 whose vub satisfies pred, for a pred that holds
// on a prefix of 0..255, from a guess g: kind 0: vub < x, 1: vub <= x, 2:
// the TF coordinate of vub lies below x (the TF's clear prefix).
__host__ __device__ inline bool vub_pred(int kind, float v, float x) {
  if (kind == 0) return v < x;
  if (kind == 1) return v <= x;
  return fminf(fmaxf(fmaf(v, 256.0f, -0.5f), 0.0f), 255.0f) < x;
}
__host__ __device__ inline uint32_t vub_prefix(int kind, float x, float g) {
  int n = g >= 256.0f ? 256 : (g > 0.0f ? (int)g : 0);  // NaN: 0
  while (n > 0 && !vub_pred(kind, vub_of((uint32_t)n - 1u), x)) n--;
  while (n < 256 && vub_pred(kind, vub_of((uint32_t)n), x)) n++;
  return (uint32_t)n;
}
// The counts of a LOD-brick view (threshold, skip gate and mode from pc; the
// scene's TF-clear coordinate tf_zero_t).  The gates follow view_const.
__host__ __device__ inline ElideCounts elide_counts(const r3d_frame_params &pc, float tf_zero_t) {
  const float bgate = fmaxf(fmaxf(pc.skip_gate, 0.5f / 255.0f), 4.5f / 255.0f);
  const uint32_t n_cut = vub_prefix(0, pc.threshold, ceilf(pc.threshold * 255.0f));
  const uint32_t n_bg = vub_prefix(0, bgate, ceilf(bgate * 255.0f));
  ElideCounts e;
  e.n_void = n_cut > n_bg ? n_cut : n_bg;
  e.n_dec = n_cut;
  uint32_t n2 = 0;
  if (pc.mode == R3D_MODE_FULL || pc.mode == R3D_MODE_FLAT)
    n2 = vub_prefix(2, tf_zero_t, ceilf((tf_zero_t + 0.5f) * (255.0f / 256.0f)));
  else if (pc.mode == R3D_MODE_DEPTH)
    n2 = vub_prefix(1, 0.05f, floorf(0.05f * 255.0f) + 1.0f);
  if (n2 > e.n_dec) e.n_dec = n2;
  e.raw_dec = 8388608.0f + (float)e.n_dec;
  return e;
}

struct DevScene {
  DevCube cube;
  DevBricks br;
  DevShard sh;
  DevSlab sl;
  DevClip cl;
  DevVslab vs;
  uint32_t *status;
  float alpha_cutoff;
  float tf_zero_t;  // TF coordinates below this have alpha exactly 0
  // counting launches: bit s set when slot s's voxels are read (nullptr: off)
  uint32_t *slot_bits;
  // one-view launches (grid, staged): the view's elision counts
  ElideCounts el;
};

struct RayResult {
  float rgb[3];
  uint32_t steps;
  uint32_t mip_index;
  uint32_t n_tf;    // composited TF lookups
  uint32_t n_grad;  // gradient-shaded samples
  uint32_t n_walk;  // page-table walks
};

__device__ __forceinline__ float lerp_(float a, float b, float t) { return fmaf(t, b - a, a); }
__device__ __forceinline__ float clamp_(float x, float lo, float hi) {
  return fminf(fmaxf(x, lo), hi);
}
__device__ __forceinline__ float sat_(float x) { return clamp_(x, 0.0f, 1.0f); }
__device__ __forceinline__ float dot3(float3 a, float3 b) {
  return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x));
}
__device__ __forceinline__ float3 norm3(float3 a) {
  float inv = 1.0f / sqrtf(dot3(a, a));
  return make_float3(a.x * inv, a.y * inv, a.z * inv);
}

// common.slang:57-61
__device__ __forceinline__ float hash12(uint32_t px, uint32_t py, uint32_t frame) {
  uint32_t h = px * 374761393u + py * 668265263u + frame * 2246822519u;
  h = (h ^ (h >> 13)) * 1274126177u;
  return (float)(h >> 8) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ uint8_t unorm8(float x) {
  return (uint8_t)(int)fmaf(sat_(x), 255.0f, 0.5f);
}

// floor of t in [0, 2^23) as an integer and its fraction, without the
// conversion unit: adding 2^23 with truncation leaves floor(t) in the
// mantissa.  Equal to (uint32_t)t and t - (float)(uint32_t)t.
__device__ __forceinline__ uint32_t floor_frac(float t, float &frac) {
  float r = __fadd_rz(t, 8388608.0f);
  frac = t - (r - 8388608.0f);
  return __float_as_uint(r) & 0x7fffffu;
}

// Bytes taken as the float 2^23 + byte (bits assembled, no conversion
// unit).  The difference of two such floats is the bytes' difference
// exactly, and one subtraction of 2^23 gives the first byte, so
// lerp_raw(2^23 + a, 2^23 + b, t) is lerp_(a, b, t) = fmaf(t, b - a, a) in
// the same bits, with one instruction fewer.
__device__ __forceinline__ float raw_u8(const uint8_t *p) {
  return __uint_as_float(0x4B000000u | (uint32_t)__ldg(p));
}
__device__ __forceinline__ float lerp_raw(float ra, float rb, float t) {
  return fmaf(t, rb - ra, ra - 8388608.0f);
}

// Clamp-to-edge trilinear at texel centres on a u8 grid: x, then y, then z
// lerps in 0..255 space, scaled by 1/255 at the end.
__device__ __forceinline__ float tri_u8(const uint8_t *__restrict__ g, uint32_t dx, uint32_t dy,
                                        uint32_t dz, float tx, float ty, float tz) {
  tx = clamp_(tx, 0.0f, (float)(dx - 1u));
  ty = clamp_(ty, 0.0f, (float)(dy - 1u));
  tz = clamp_(tz, 0.0f, (float)(dz - 1u));
  float fx, fy, fz;
  const uint32_t x0 = floor_frac(tx, fx), y0 = floor_frac(ty, fy), z0 = floor_frac(tz, fz);
  uint32_t x1 = min(x0 + 1u, dx - 1u), y1 = min(y0 + 1u, dy - 1u), z1 = min(z0 + 1u, dz - 1u);
  size_t sy = dx, sz = (size_t)dx * dy;
  const uint8_t *r00 = g + (size_t)y0 * sy + (size_t)z0 * sz;
  const uint8_t *r10 = g + (size_t)y1 * sy + (size_t)z0 * sz;
  const uint8_t *r01 = g + (size_t)y0 * sy + (size_t)z1 * sz;
  const uint8_t *r11 = g + (size_t)y1 * sy + (size_t)z1 * sz;
  float c00 = lerp_raw(raw_u8(r00 + x0), raw_u8(r00 + x1), fx);
  float c10 = lerp_raw(raw_u8(r10 + x0), raw_u8(r10 + x1), fx);
  float c01 = lerp_raw(raw_u8(r01 + x0), raw_u8(r01 + x1), fx);
  float c11 = lerp_raw(raw_u8(r11 + x0), raw_u8(r11 + x1), fx);
  float e0 = lerp_(c00, c10, fy), e1 = lerp_(c01, c11, fy);
  return lerp_(e0, e1, fz) * kInv255;
}

// volumes[0].SampleLevel(p, lod): trilinear within a level, linear between
// floor(lod) and floor(lod)+1 (raycast.slang:409-416, vkbackend.c:1058-1069)
__device__ __forceinline__ float cube_sample(const DevCube &c, float3 p, float lod) {
  float fl = floorf(lod);
  uint32_t m0 = min((uint32_t)fl, c.nlevels - 1u);
  float fr = lod - fl;
  float v = tri_u8(c.lev[m0], c.dim[m0][0], c.dim[m0][1], c.dim[m0][2],
                   fmaf(p.x, (float)c.dim[m0][0], -0.5f), fmaf(p.y, (float)c.dim[m0][1], -0.5f),
                   fmaf(p.z, (float)c.dim[m0][2], -0.5f));
  if (fr > 0.0f && m0 + 1u < c.nlevels) {
    uint32_t m1 = m0 + 1u;
    float v1 = tri_u8(c.lev[m1], c.dim[m1][0], c.dim[m1][1], c.dim[m1][2],
                      fmaf(p.x, (float)c.dim[m1][0], -0.5f),
                      fmaf(p.y, (float)c.dim[m1][1], -0.5f),
                      fmaf(p.z, (float)c.dim[m1][2], -0.5f));
    v = lerp_(v, v1, fr);
  }
  return v;
}

// occ.SampleLevel(p, 0) with a nearest sampler
__device__ __forceinline__ float occ_sample(const DevCube &c, float3 p) {
  float q[3] = {floorf(p.x * (float)c.odim[0]), floorf(p.y * (float)c.odim[1]),
                floorf(p.z * (float)c.odim[2])};
  uint32_t i[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    float m = (float)(c.odim[a] - 1u);
    i[a] = !(q[a] >= 0.0f) ? 0u : (q[a] > m ? c.odim[a] - 1u : (uint32_t)q[a]);
  }
  return (float)__ldg(c.occ + ((size_t)i[2] * c.odim[1] + i[1]) * c.odim[0] + i[0]) * kInv255;
}

struct BrickCtx {  // raycast.slang:144-152
  bool ok;
  float maxv;
  float3 bl;
  uint32_t slot;
  float grad_vox;
  float world_brick;
};

struct LodCache {  // raycast.slang:190-196 (the cached brick is kept as the
                   // float origin lo = 128 * bc of its coordinates)
  int desired;
  float inv_scale;
  // (uint)lv >> 7 == bc  <=>  lo <= lv < lo + 128, for lv >= 0; an empty
  // cache (no brick found, or none looked up yet) holds lo = +inf, which no
  // coordinate reaches
  float lo[3];
  BrickCtx c;
};

__device__ __forceinline__ uint32_t page_entry(const DevScene &s, uint32_t i) {
  if (i >= s.br.page_words) {
    atomicOr(s.status, R3D_STATUS_PAGE_RANGE);
    return 0xFFFFFFFFu;
  }
  return __ldcg(s.br.page + i);  // page table through L2
}

// bricks_lod_locate_ex, raycast.slang:198-247 (header pre-decoded)
__device__ __forceinline__ BrickCtx lod_locate_ex(const DevScene &s, float3 p, float lod,
                                               LodCache &lc, int desired) {
  const DevBricks &b = s.br;
  BrickCtx c;
  c.ok = false;
  c.maxv = 0.0f;
  c.bl = make_float3(0.0f, 0.0f, 0.0f);
  c.slot = 0;
  c.grad_vox = 1.0f;
  c.world_brick = (128.0f * (float)(1u << (b.nlev - 1u))) / b.md;
  float base_v[3] = {clamp_(p.x * b.md, 0.0f, b.bs_hi[0]), clamp_(p.y * b.md, 0.0f, b.bs_hi[1]),
                     clamp_(p.z * b.md, 0.0f, b.bs_hi[2])};
  int last = (int)b.nlev - 1;
  float inv_out = 1.0f;
  uint32_t bco[3] = {0u, 0u, 0u};
  for (uint32_t step = 0; step < 4u; step++) {
    int li = step < 3u ? desired + (int)step : last;
    if (li < 0 || li > last || (step == 3u && li <= desired + 2)) continue;
    float inv = b.inv_scale[li];
    float lv[3];
    uint32_t bc[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
      lv[a] = base_v[a] * inv;
      bc[a] = min((uint32_t)lv[a] >> 7, b.bd[li][a] - 1u);
    }
    uint32_t bi = b.off[li] + (bc[2] * b.bd[li][1] + bc[1]) * b.bd[li][0] + bc[0];
    uint32_t e = page_entry(s, bi);
    if (e == 0xFFFFFFFFu) continue;
    uint32_t slot = e & 0xFFFFFFu;
    if (slot >= b.nslots) {
      atomicOr(s.status, R3D_STATUS_PAGE_RANGE);
      continue;
    }
    c.ok = true;
    c.maxv = (float)(e >> 24) / 255.0f;
    c.slot = slot;
    c.bl = make_float3(lv[0] - (float)(bc[0] << 7), lv[1] - (float)(bc[1] << 7),
                       lv[2] - (float)(bc[2] << 7));
    c.grad_vox = r3d_exp2f(lod) * inv;
    c.world_brick = (128.0f * (float)b.scale[li]) / b.md;
    inv_out = inv;
    bco[0] = bc[0];
    bco[1] = bc[1];
    bco[2] = bc[2];
    break;
  }
  lc.desired = desired;
  lc.inv_scale = inv_out;
  lc.lo[0] = c.ok ? (float)(bco[0] << 7) : R3D_FM_INF;
  lc.lo[1] = c.ok ? (float)(bco[1] << 7) : R3D_FM_INF;
  lc.lo[2] = c.ok ? (float)(bco[2] << 7) : R3D_FM_INF;
  lc.c = c;
  return c;
}

// The hit test of bricks_lod_locate_cached (raycast.slang:255-279): true,
// with the brick context in out, when the desired level and the brick under
// p are the cached ones.  The test runs on bl = lv - lo: rounding keeps the
// sign of a difference, and for lo <= lv < lo + 128 the difference is exact
// (lo = 0, or lv <= 2 lo), so bl >= 0 && bl < 128 decides exactly what
// lo <= lv < lo + 128 does, and an empty cache (lo = +inf) never hits.
__device__ __forceinline__ bool lod_cache_hit(const DevScene &s, float3 p, int desired,
                                              const LodCache &lc, BrickCtx &out) {
  const DevBricks &b = s.br;
  if (lc.desired == desired) {
    float bl[3];
    bool same = true;
    float pv[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int a = 0; a < 3; a++) {
      float base_v = clamp_(pv[a] * b.md, 0.0f, b.bs_hi[a]);
      bl[a] = base_v * lc.inv_scale - lc.lo[a];
      same = same && bl[a] >= 0.0f && bl[a] < 128.0f;
    }
    if (same) {
      out = lc.c;
      out.bl = make_float3(bl[0], bl[1], bl[2]);
      return true;
    }
  }
  return false;
}

// Slot-local texel coordinates of bricks_fetch (clamped, minus 0.5) and
// their base texel.
struct SlotCoord {
  float fx, fy, fz;  // fractions
  uint32_t x0, y0, z0;
};

// One axis of bricks_fetch's coordinate: clamp to [0.5, 127.5] inside the
// brick, texel-centre shift, floor and fraction.  The shift rides on the
// truncating add: c + (2^23 - 0.5) is 2^23 + (c - 0.5) exactly before the
// truncation, so r holds 2^23 + floor(c - 0.5); r - (2^23 - 0.5) =
// floor + 0.5 and c - (floor + 0.5) are exact, so the floor and the
// fraction are the bits of floor_frac(c - 0.5).
__device__ __forceinline__ uint32_t slot_axis(float b, float &frac) {
  const float c = clamp_(b, 0.5f, 127.5f);
  const float r = __fadd_rz(c, 8388607.5f);
  frac = c - (r - 8388607.5f);
  return __float_as_uint(r) & 0x7fffffu;
}

__device__ __forceinline__ SlotCoord slot_coord(float3 bl) {
  SlotCoord q;
  q.x0 = slot_axis(bl.x, q.fx);
  q.y0 = slot_axis(bl.y, q.fy);
  q.z0 = slot_axis(bl.z, q.fz);
  return q;
}

// byte k of w as a float without the conversion unit: the byte permute
// assembles the bits of 2^23 + byte, and subtracting 2^23 is exact
__device__ __forceinline__ float qbyte(uint32_t w, uint32_t k) {
  return __uint_as_float(__byte_perm(w, 0x4B000000u, k | 0x7540u)) - 8388608.0f;
}

// Trilinear inside one 128^3 slot at a clamped slot coordinate, on the quad
// pool: the word of texel (x, y, z) holds the bytes at (x, y), (x1, y),
// (x, y1), (x1, y1) of its z plane (x1, y1 clamped to the slot), so a
// sample is two 4-byte loads; z1 is clamped the same way.  The lerps run
// in 0..255 space, x then y then z, as on the byte grid.
// The trilinear value of the quad words w0 (plane z0) and w1 (plane z1).
// The x lerps take the bytes as 2^23 + byte (the permute alone; lerp_raw).
__device__ __forceinline__ float qraw(uint32_t w, uint32_t k) {
  return __uint_as_float(__byte_perm(w, 0x4B000000u, k | 0x7540u));
}
// The eight bytes of two quad words, as 2^23 + byte.
struct RawBytes {
  float r[8];
};
__device__ __forceinline__ RawBytes raw_bytes(uint32_t w0, uint32_t w1) {
  return {{qraw(w0, 0), qraw(w0, 1), qraw(w0, 2), qraw(w0, 3), qraw(w1, 0), qraw(w1, 1),
           qraw(w1, 2), qraw(w1, 3)}};
}
// 2^23 + the largest of the eight bytes
__device__ __forceinline__ float raw_max(const RawBytes &b) {
  return fmaxf(fmaxf(fmaxf(b.r[0], b.r[1]), fmaxf(b.r[2], b.r[3])),
               fmaxf(fmaxf(b.r[4], b.r[5]), fmaxf(b.r[6], b.r[7])));
}
__device__ __forceinline__ float tri_raw(const RawBytes &b, const SlotCoord &q) {
  const float c00 = lerp_raw(b.r[0], b.r[1], q.fx);
  const float c10 = lerp_raw(b.r[2], b.r[3], q.fx);
  const float c01 = lerp_raw(b.r[4], b.r[5], q.fx);
  const float c11 = lerp_raw(b.r[6], b.r[7], q.fx);
  const float e0 = lerp_(c00, c10, q.fy), e1 = lerp_(c01, c11, q.fy);
  return lerp_(e0, e1, q.fz) * kInv255;
}
__device__ __forceinline__ float tri_words(uint32_t w0, uint32_t w1, const SlotCoord &q) {
  return tri_raw(raw_bytes(w0, w1), q);
}

__device__ __forceinline__ float tri_slot_q(const uint32_t *__restrict__ g, const SlotCoord &q) {
  const uint32_t dz1 = q.z0 < 127u ? 16384u : 0u;
  const uint32_t *r = g + ((q.z0 << 14) | (q.y0 << 7) | q.x0);
  return tri_words(__ldg(r), __ldg(r + dz1), q);
}

__device__ __forceinline__ float slot_sample(const DevScene &s, uint32_t slot, const SlotCoord &q) {
  return tri_slot_q(s.br.quad + (size_t)slot * (128u * 128u * 128u), q);
}

// A box of one slot's bytes staged in shared memory by TMA (the staged
// kernel, r3d_staged.cu): kBoxX x kBoxY x kBoxZ texels from (bx, by, bz) of
// slot `slot` (-1: nothing staged), x fastest.
constexpr uint32_t kBoxX = 32, kBoxY = 17, kBoxZ = 17;
constexpr uint32_t kBoxBytes = kBoxX * kBoxY * kBoxZ;
struct StageBox {
  const uint8_t *data;
  int slot, bx, by, bz;
};

// Whether the 2x2x2 texels of a sample (base q, neighbours clamped to the
// slot as in the quad pool) all lie in the staged box.
__device__ __forceinline__ bool box_has(const StageBox &b, uint32_t slot, const SlotCoord &q) {
  const int x1 = q.x0 < 127u ? (int)q.x0 + 1 : 127, y1 = q.y0 < 127u ? (int)q.y0 + 1 : 127,
            z1 = q.z0 < 127u ? (int)q.z0 + 1 : 127;
  return (int)slot == b.slot && (int)q.x0 >= b.bx && x1 < b.bx + (int)kBoxX &&
         (int)q.y0 >= b.by && y1 < b.by + (int)kBoxY && (int)q.z0 >= b.bz &&
         z1 < b.bz + (int)kBoxZ;
}

// tri_slot_q on the staged bytes: the same texels, the same lerps in the
// same order, so the same bits.
__device__ __forceinline__ float box_sample(const StageBox &b, const SlotCoord &q) {
  const uint8_t *p =
      b.data + (((int)q.z0 - b.bz) * (int)kBoxY + ((int)q.y0 - b.by)) * (int)kBoxX + ((int)q.x0 - b.bx);
  const int dx = q.x0 < 127u ? 1 : 0, dy = q.y0 < 127u ? (int)kBoxX : 0,
            dz = q.z0 < 127u ? (int)(kBoxX * kBoxY) : 0;
  const float c00 = lerp_((float)p[0], (float)p[dx], q.fx);
  const float c10 = lerp_((float)p[dy], (float)p[dy + dx], q.fx);
  const float c01 = lerp_((float)p[dz], (float)p[dz + dx], q.fx);
  const float c11 = lerp_((float)p[dz + dy], (float)p[dz + dy + dx], q.fx);
  const float e0 = lerp_(c00, c10, q.fy), e1 = lerp_(c01, c11, q.fy);
  return lerp_(e0, e1, q.fz) * kInv255;
}

// overlay_flags (raycast.slang:45-49): the four slot-parallel atlases
constexpr uint32_t kOvlInk = 1u, kOvlInk3d = 4u, kOvlLabels = 8u, kOvlReg = 16u;
constexpr uint32_t kOvlAtlases = kOvlInk | kOvlInk3d | kOvlLabels | kOvlReg;

// paint-label palette, class id 1..8 (raycast.slang:52-61)
static __constant__ float kLabelPal[8][3] = {
    {0.82f, 0.66f, 0.43f}, {0.95f, 0.20f, 0.85f}, {0.20f, 0.80f, 0.80f}, {0.30f, 0.90f, 0.30f},
    {1.00f, 0.55f, 0.15f}, {0.35f, 0.45f, 0.90f}, {0.95f, 0.90f, 0.20f}, {0.90f, 0.90f, 0.90f}};

// bricks_fetch of overlay atlas i (ink, 3D ink, registration) at the
// sample's clamped slot coordinate (raycast.slang:87-97,105-111)
__device__ __forceinline__ float ovl_fetch(const DevScene &s, int i, uint32_t slot,
                                           const SlotCoord &q) {
  return tri_slot_q(s.br.ovl[i] + (size_t)slot * (128u * 128u * 128u), q);
}

// bricks_fetch_label (raycast.slang:99-104): the texel under bl, snapped
// to its centre so that class ids never blend
__device__ __forceinline__ float ovl_label(const DevScene &s, uint32_t slot, float3 bl) {
  const uint32_t x = (uint32_t)(clamp_(floorf(bl.x) + 0.5f, 0.5f, 127.5f) - 0.5f);
  const uint32_t y = (uint32_t)(clamp_(floorf(bl.y) + 0.5f, 0.5f, 127.5f) - 0.5f);
  const uint32_t z = (uint32_t)(clamp_(floorf(bl.z) + 0.5f, 0.5f, 127.5f) - 0.5f);
  const uint32_t w =
      __ldg(s.br.ovl[2] + (size_t)slot * (128u * 128u * 128u) + ((z << 14) | (y << 7) | x));
  return qbyte(w, 0) * kInv255;
}

// label_color (raycast.slang:63-66)
__device__ __forceinline__ float3 label_color(float v) {
  uint32_t c = (uint32_t)floorf(fmaf(v, 255.0f, 0.5f));
  c = c < 1u ? 1u : (c > 8u ? 8u : c);
  return make_float3(kLabelPal[c - 1u][0], kLabelPal[c - 1u][1], kLabelPal[c - 1u][2]);
}

// bricks_fetch at atlas lod 0 (raycast.slang:284-288): clamp to
// [0.5, 127.5] inside the brick, no cross-brick filtering
__device__ __forceinline__ float brick_fetch(const DevScene &s, uint32_t slot, float3 bl) {
  return slot_sample(s, slot, slot_coord(bl));
}

// Texel origin of a single-level atlas slot (raycast.slang:176-177)
__device__ __forceinline__ float3 shard_slot_org(const DevShard &h, uint32_t slot) {
  const uint32_t sx = slot % h.abpa, sy = (slot / h.abpa) % h.abpa, sz = slot / (h.abpa * h.abpa);
  return make_float3((float)sx * 128.0f, (float)sy * 128.0f, (float)sz * 128.0f);
}

// bricks_fetch of the single-level atlas (raycast.slang:284-288): the
// brick-local position clamped to [inset, 128 - inset] with
// inset = max(0.5 * 2^lod, 0.5), then the atlas sampled at lod like a cube
// texture.  e2 = r3d_exp2f(lod).
__device__ __forceinline__ float shard_fetch(const DevShard &h, float3 org, float3 bl, float lod,
                                             float e2) {
  const float inset = fmaxf(0.5f * e2, 0.5f), hi = 128.0f - inset;
  const float3 u = make_float3((org.x + clamp_(bl.x, inset, hi)) * h.inv_adim,
                               (org.y + clamp_(bl.y, inset, hi)) * h.inv_adim,
                               (org.z + clamp_(bl.z, inset, hi)) * h.inv_adim);
  return cube_sample(h.atlas, u, lod);
}

// A slab tile sampled at normalized (u, v, w) like the slab sampler
// (src/vk/vkbackend.c:2203-2211): linear, clamp to edge in x and y (the
// apron makes tiles seamless), REPEAT in w so the z ring wraps.
__device__ __forceinline__ float tex_wrapz(const uint8_t *__restrict__ g, uint32_t tw, uint32_t th,
                                           uint32_t wz, float u, float v, float w) {
  const float tx = clamp_(fmaf(u, (float)tw, -0.5f), 0.0f, (float)(tw - 1u));
  const float ty = clamp_(fmaf(v, (float)th, -0.5f), 0.0f, (float)(th - 1u));
  const float tz = fmaf(w, (float)wz, -0.5f);
  float fx, fy;
  const uint32_t x0 = floor_frac(tx, fx), y0 = floor_frac(ty, fy);
  const float zf = floorf(tz), fz = tz - zf;
  // w is a fraction in [0, 1), so floor(tz) lies in [-1, wz - 1] and its
  // ring layer is one conditional away (the modulo of the restatement)
  const int zi = (int)zf;
  const uint32_t z0 = zi < 0 ? wz - 1u : min((uint32_t)zi, wz - 1u);
  const uint32_t z1 = z0 + 1u < wz ? z0 + 1u : 0u;
  const uint32_t x1 = min(x0 + 1u, tw - 1u), y1 = min(y0 + 1u, th - 1u);
  const size_t sy = tw, sz = (size_t)tw * th;
  const uint8_t *r00 = g + y0 * sy + z0 * sz, *r10 = g + y1 * sy + z0 * sz;
  const uint8_t *r01 = g + y0 * sy + z1 * sz, *r11 = g + y1 * sy + z1 * sz;
  const float c00 = lerp_raw(raw_u8(r00 + x0), raw_u8(r00 + x1), fx);
  const float c10 = lerp_raw(raw_u8(r10 + x0), raw_u8(r10 + x1), fx);
  const float c01 = lerp_raw(raw_u8(r01 + x0), raw_u8(r01 + x1), fx);
  const float c11 = lerp_raw(raw_u8(r11 + x0), raw_u8(r11 + x1), fx);
  return lerp_(lerp_(c00, c10, fy), lerp_(c01, c11, fy), fz) * kInv255;
}

__device__ __forceinline__ float slab_tile(const DevSlab &sl, int L, uint32_t k, float u, float v,
                                           float w) {
  const DevSlabLevel &lv = sl.lev[L];
  const uint32_t tw = lv.px + 2u, th = lv.py + 2u, wz = sl.wz;
  return tex_wrapz(sl.pool + lv.off + (size_t)k * tw * th * wz, tw, th, wz, u, v, w);
}

// sample_clip_level (raycast.slang:360-376): level l's texture at p, its z
// ring wrapping in level slices
// (divisions by the powers of two 2^l and 2048 are exact as products)
__device__ __forceinline__ float clip_level(const DevClip &cl, int l, float3 p) {
  const float is = 1.0f / (float)(1u << l);
  const float wx = p.x * cl.nx, wy = p.y * cl.nx;
  const float zw = (cl.z0 + 0.5f) + p.z * cl.nx;
  const float u = fmaf(wx - cl.ox[l], is, 1.0f) * (1.0f / 2048.0f);
  const float v = fmaf(wy - cl.oy[l], is, 1.0f) * (1.0f / 2048.0f);
  const float zq = (zw * is) / (float)cl.wzl[l];
  return tex_wrapz(cl.lev[l], 2048u, 2048u, cl.wzl[l], u, v, zq - floorf(zq));
}

// pick_clip_level (raycast.slang:380-395): the finest valid level holding
// p from the desired one (coarser first once past the top), or -1
__device__ __forceinline__ int clip_pick(const DevClip &cl, float3 p, float lod) {
  const float wx = p.x * cl.nx, wy = p.y * cl.nx;
  const int desired = (int)clamp_(lod, 0.0f, 5.0f);
  for (int step = 0; step < 6; step++) {
    int li = desired + step;
    if (li > 5) li = 5 - step;
    if (li < 0) continue;
    if (!(cl.valid & (1u << li))) continue;
    const float is = 1.0f / (float)(1u << li);  // exact: a power of two
    const float tx = fmaf(wx - cl.ox[li], is, 1.0f), ty = fmaf(wy - cl.oy[li], is, 1.0f);
    if (tx < 1.0f || tx >= 2047.0f || ty < 1.0f || ty >= 2047.0f) continue;
    return li;
  }
  return -1;
}

// vs_sample (raycast.slang:331-367): the base cell under p must be the one
// its tile holds and hold the sample's slice span; then the pyramid level
// whose prefilter (4 << level) matches the footprint, stepping down past
// absent levels, or the base tile.  Cells convert through int so that the
// key of a cell left of the volume is defined.
__device__ __forceinline__ float vs_sample(const DevVslab &v, float3 p, float lod) {
  const float P = (float)v.px, T = P + 2.0f;
  const uint32_t Tu = v.px + 2u;
  const float wx = v.x0 + p.x * v.nx, wy = v.y0 + p.y * v.nx;
  const float zc = (v.z0 + 0.5f) + p.z * v.nx;
  const float zq = zc / (float)v.wz, w = zq - floorf(zq);
  const float gx0 = (float)v.gx[0], gy0 = (float)v.gy[0];
  const float cbx = floorf(wx / P), cby = floorf(wy / P);
  const float pbx = cbx - floorf(cbx / gx0) * gx0, pby = cby - floorf(cby / gy0) * gy0;
  const uint32_t want = ((uint32_t)(int32_t)cbx & 1023u) |
                        (((uint32_t)(int32_t)cby & 1023u) << 10) | 0x80000000u;
  const uint32_t slot = (uint32_t)(pby * gx0 + pbx);
  const uint4 e = __ldg(reinterpret_cast<const uint4 *>(v.table) + slot);
  if (e.x != want) return 0.0f;  // not resident
  if (zc - 0.5f < (float)e.y || zc + 0.5f > (float)e.z) return 0.0f;
  int lev = min((int)floorf(lod) - 2, 3);
  while (lev >= 0 && v.gx[lev + 1] == 0u) lev--;
  if (lev < 0) {
    const float lx = (wx - cbx * P) + 1.0f, ly = (wy - cby * P) + 1.0f;
    return tex_wrapz(v.tiles + (size_t)slot * v.tile_bytes, Tu, Tu, v.wz, lx / T, ly / T, w);
  }
  const int L = lev + 1;
  const float isc = 1.0f / (float)(4 << lev);  // exact: a power of two
  const float gxl = (float)v.gx[L], gyl = (float)v.gy[L];
  const float tx = wx * isc, ty = wy * isc;
  const float cx = floorf(tx / P), cy = floorf(ty / P);
  const float qx = cx - floorf(cx / gxl) * gxl, qy = cy - floorf(cy / gyl) * gyl;
  const float lx = (tx - cx * P) + 1.0f, ly = (ty - cy * P) + 1.0f;
  const uint32_t k = v.base[L] + (uint32_t)(qy * gxl + qx);
  return tex_wrapz(v.tiles + (size_t)k * v.tile_bytes, Tu, Tu, v.wz, lx / T, ly / T, w);
}

// vol_sample in clip mode (raycast.slang:400-403)
__device__ __forceinline__ float clip_sample(const DevClip &cl, float3 p, float lod) {
  const int l = clip_pick(cl, p, lod);
  return l < 0 ? 0.0f : clip_level(cl, l, p);
}

// vol_sample of the tiled slab (raycast.slang:423-455): voxel coordinates
// of p, the ring coordinate, then the overview level whose prefilter
// (4 << level) matches the footprint, or the base tile under p.
__device__ __forceinline__ float slab_sample(const DevSlab &sl, float3 p, float lod) {
  const float wx = p.x * sl.nx, wy = p.y * sl.nx;
  const float zc = (sl.z0 + 0.5f) + p.z * sl.nx;
  const float zq = zc / (float)sl.wz;
  const float w = zq - floorf(zq);  // frac: the ring wraps
  int lev = (int)floorf(lod) - 2;
  if (lev >= 0) {
    lev = min(lev, sl.nov - 1);
    const float gxl = sl.ov[lev][0], gyl = sl.ov[lev][1], pxl = sl.ov[lev][2], pyl = sl.ov[lev][3];
    // division by the power of two 4 << lev is exact as a product
    const float isc = 1.0f / (float)(4 << lev);
    const float wxl = wx * isc, wyl = wy * isc;
    const float oix = fminf(floorf(fmaxf(wxl, 0.0f) / pxl), gxl - 1.0f);
    const float oiy = fminf(floorf(fmaxf(wyl, 0.0f) / pyl), gyl - 1.0f);
    const float ou = ((wxl - oix * pxl) + 1.0f) / (pxl + 2.0f);
    const float ov = ((wyl - oiy * pyl) + 1.0f) / (pyl + 2.0f);
    return slab_tile(sl, lev + 1, (uint32_t)(oiy * gxl + oix), ou, ov, w);
  }
  const uint32_t gx = sl.lev[0].gx, gy = sl.lev[0].gy;
  const uint32_t ix = min((uint32_t)(fmaxf(wx, 0.0f) / sl.px), gx - 1u);
  const uint32_t iy = min((uint32_t)(fmaxf(wy, 0.0f) / sl.py), gy - 1u);
  const float u = ((wx - (float)ix * sl.px) + 1.0f) / (sl.px + 2.0f);
  const float v = ((wy - (float)iy * sl.py) + 1.0f) / (sl.py + 2.0f);
  return slab_tile(sl, 0, iy * gx + ix, u, v, w);
}

// Page entry of brick bi of the shard (raycast.slang:813-821); a slot
// outside the atlas is treated as absent and flagged.
__device__ __forceinline__ void shard_entry(const DevScene &s, uint32_t bi, BrickCtx &c) {
  const uint32_t e = __ldg(s.sh.page + bi);
  c.ok = e != 0xFFFFFFFFu;
  c.slot = e & 0xFFFFFFu;
  if (c.ok && c.slot >= s.sh.abpa * s.sh.abpa * s.sh.abpa) {
    atomicOr(s.status, R3D_STATUS_PAGE_RANGE);
    c.ok = false;
  }
  c.maxv = c.ok ? (float)(e >> 24) / 255.0f : 0.0f;
}

// TF lookup (raycast.slang:894) from raw 0..255 RGBA values in shared memory
__device__ __forceinline__ float4 tf_sample(const float4 *tf, float t) {
  float f;
  const uint32_t i0 = floor_frac(t, f);
  const uint32_t i1 = min(i0 + 1u, 255u);
  float4 a = tf[i0], b = tf[i1];
  return make_float4(lerp_(a.x, b.x, f) * kInv255, lerp_(a.y, b.y, f) * kInv255,
                     lerp_(a.z, b.z, f) * kInv255, lerp_(a.w, b.w, f) * kInv255);
}

// (float)m for a byte m without the conversion unit (exact: the byte
// permute assembles the bits of 2^23 + m)
__device__ __forceinline__ float byte_float(uint32_t m) {
  return __uint_as_float(__byte_perm(m, 0x4B000000u, 0x7650u)) - 8388608.0f;
}

#ifndef R3D_BYTE_ELIDE
#define R3D_BYTE_ELIDE 1
#endif

// Per-view constants of the march (raycast.slang:647-683,722-762).
struct ViewConst {
  float voxel, vox_inv, max_lod, cone, dt, bs, occ_gate, bgate, opac_k;
  float lod_bias, threshold, density;
  float3 ext;
  bool ortho, lod_on;
  // overlays (raycast.slang:45-49,67-73): atlas bits, ink gain, the
  // registration fuse weight and the ink tint
  uint32_t ovl;
  float ovl_gain, reg_alpha;
  float3 ovl_col;
  ElideCounts el;  // LOD bricks: the fetch elision's counts
};

template <int PATH>
__device__ __forceinline__ ViewConst view_const(const r3d_frame_params &pc, const DevScene &s,
                                                const ElideCounts &el) {
  ViewConst v;
  v.el = el;
  if (PATH == PATH_LOD_BRICKS) {
    v.voxel = 1.0f / s.br.md;
    v.vox_inv = s.br.md;
    v.max_lod = (float)(s.br.nlev - 1u);
    v.ext = make_float3(s.br.bs[0] / s.br.md, s.br.bs[1] / s.br.md, s.br.bs[2] / s.br.md);
  } else if (PATH == PATH_SHARD) {  // raycast.slang:659-661: the atlas has 4 mips
    v.voxel = 1.0f / s.sh.n;
    v.vox_inv = s.sh.n;
    v.max_lod = 3.0f;
    v.ext = make_float3(1.0f, 1.0f, 1.0f);
  } else if (PATH == PATH_CLIP) {  // raycast.slang:651-654,305-314
    v.voxel = 1.0f / pc.slab_nx;
    v.vox_inv = pc.slab_nx;
    v.max_lod = 7.0f;
    v.ext = make_float3(1.0f, pc.slab_ny / pc.slab_nx, (float)pc.slab_depth / pc.slab_nx);
  } else if (PATH == PATH_VSLAB) {  // raycast.slang:661-671,305-314
    v.voxel = 1.0f / pc.slab_nx;
    v.vox_inv = pc.slab_nx;
    v.max_lod = 3.0f;  // +2 past the coarsest present pyramid level
    for (int l = 3; l >= 0; l--)
      if (((pc.brick_mode >> (8 * l)) & 0xffu) != 0u) {
        v.max_lod = (float)l + 4.0f;
        break;
      }
    v.ext = make_float3(1.0f, pc.slab_ny / pc.slab_nx, (float)pc.slab_depth / pc.slab_nx);
  } else if (PATH == PATH_SLAB) {  // raycast.slang:672-677,305-314
    v.voxel = 1.0f / pc.slab_nx;
    v.vox_inv = pc.slab_nx;
    v.max_lod = r3d_log2f((float)((pc.slab_grid >> 16) & 0xffu)) + 2.0f;
    v.ext = make_float3(1.0f, pc.slab_ny / pc.slab_nx, (float)pc.slab_depth / pc.slab_nx);
  } else {
    v.voxel = 1.0f / (float)s.cube.maxdim;
    v.vox_inv = (float)s.cube.maxdim;
    v.max_lod = fminf(pc.max_mip, (float)(s.cube.nlevels - 1u));
    v.ext = make_float3(1.0f, 1.0f, 1.0f);
  }
  const float3 up = make_float3(pc.cam_up[0], pc.cam_up[1], pc.cam_up[2]);
  v.cone = (2.0f * sqrtf(dot3(up, up))) / (float)pc.viewport[1];
  v.dt = pc.step_voxels * v.voxel;
  v.bs = 8.0f * v.voxel;
  v.occ_gate = fmaxf(pc.skip_gate, 0.5f / 255.0f);
  v.bgate = fmaxf(v.occ_gate, 4.5f / 255.0f);
  v.opac_k = pc.density * pc.step_voxels;
  v.lod_bias = pc.lod_bias;
  v.threshold = pc.threshold;
  v.density = pc.density;
  v.ortho = (pc.view_flags & R3D_VIEW_ORTHO) != 0u;
  // with a zero LOD ceiling the clamp pins lod to 0 whatever log2 returns
  v.lod_on = v.max_lod != 0.0f;
  v.ovl = pc.overlay_flags & kOvlAtlases;
  v.ovl_gain = pc.overlay_gain;
  v.reg_alpha = (float)((pc.overlay_flags >> 16) & 0xffu) * (1.0f / 255.0f);
  v.ovl_col = ((pc.overlay_flags >> 8) & 0xffu) == 1u ? make_float3(0.3f, 0.72f, 1.0f)
                                                      : make_float3(0.25f, 1.0f, 0.55f);
  return v;
}
// A one-view launch: the counts travel in the scene parameter.
template <int PATH>
__device__ __forceinline__ ViewConst view_const(const r3d_frame_params &pc, const DevScene &s) {
  return view_const<PATH>(pc, s, s.el);
}

enum { kStepDone = 0, kStepCont = 1, kStepShade = 2 };

// A contributing sample waiting for gradient shading and compositing.
struct Pending {
  float3 p;
  float lod, lod_step, a;
  float4 sm;  // TF sample
  uint32_t slot;
  float3 bl;
  float grad_vox;
  float4 rs;  // overlays: TF sample of the registration atlas
  bool reg_live;
};

// State of one ray between march steps.
struct RayState {
  float3 ro, dir;  // volume space
  float t, tf_, span_step;
  bool span_dom;  // span_step >= every exp2(lod): lod_step is span_step
  // LOD bricks: for t in [lod_tlo, lod_thi) the desired level is
  // lc.desired and lod_step is span_step (empty range: unknown)
  float lod_tlo, lod_thi;
  float slab_cap;  // tiled slab: at least 4 samples across the box (raycast.slang:778-779)
  uint32_t steps, mip_index;
  float mip_max, first_hit;
  float acc_r, acc_g, acc_b, acc_a;
  float ink_max, ink2_max, lbl_max, reg_max;  // overlay MIP maxima (raycast.slang:731-734)
  LodCache lc;
  uint32_t n_tf, n_grad, n_walk;
};

// Ray setup of raycast.slang main() (:640-762) for dispatch thread (px, py)
// (half mode already applied).  Returns false when the ray needs no march:
// out.rgb then holds its final colour (ray-direction mode or background).
template <int PATH, int MODE>
__device__ __forceinline__ bool ray_begin(const r3d_frame_params &pc, const DevScene &s,
                                          const ViewConst &vc, uint32_t px, uint32_t py,
                                          RayState &st, RayResult &out) {
  constexpr bool kLod = PATH == PATH_LOD_BRICKS;
  constexpr bool kShaded = MODE == R3D_MODE_FULL;
  out.steps = 0;
  out.mip_index = 0;
  out.n_tf = out.n_grad = out.n_walk = 0;

  // pix_ndc / ray_dir / ray_origin (raycast.slang:469-486)
  float ux = ((float)px + 0.5f) / (float)pc.viewport[0];
  float uy = ((float)py + 0.5f) / (float)pc.viewport[1];
  float nx = ux * 2.0f - 1.0f, ny = 1.0f - uy * 2.0f;
  float3 fwd = make_float3(pc.cam_forward[0], pc.cam_forward[1], pc.cam_forward[2]);
  float3 rt = make_float3(pc.cam_right[0], pc.cam_right[1], pc.cam_right[2]);
  float3 up = make_float3(pc.cam_up[0], pc.cam_up[1], pc.cam_up[2]);
  float3 dir;
  if (vc.ortho)
    dir = norm3(fwd);
  else
    dir = norm3(make_float3(fmaf(ny, up.x, fmaf(nx, rt.x, fwd.x)),
                            fmaf(ny, up.y, fmaf(nx, rt.y, fwd.y)),
                            fmaf(ny, up.z, fmaf(nx, rt.z, fwd.z))));
  if (MODE == R3D_MODE_RAYDIR) {
    out.rgb[0] = fmaf(dir.x, 0.5f, 0.5f);
    out.rgb[1] = fmaf(dir.y, 0.5f, 0.5f);
    out.rgb[2] = fmaf(dir.z, 0.5f, 0.5f);
    return false;
  }
  float3 org = make_float3(pc.cam_origin[0], pc.cam_origin[1], pc.cam_origin[2]);
  if (vc.ortho)
    org = make_float3(fmaf(ny, up.x, fmaf(nx, rt.x, org.x)), fmaf(ny, up.y, fmaf(nx, rt.y, org.y)),
                      fmaf(ny, up.z, fmaf(nx, rt.z, org.z)));

  // model transform (common.slang:45-52)
  const float3 ext = vc.ext;
  float3 c = make_float3(ext.x * 0.5f, ext.y * 0.5f, ext.z * 0.5f);
  float3 r0 = make_float3(pc.vol_r0[0], pc.vol_r0[1], pc.vol_r0[2]);
  float3 r1 = make_float3(pc.vol_r1[0], pc.vol_r1[1], pc.vol_r1[2]);
  float3 r2 = make_float3(pc.vol_r2[0], pc.vol_r2[1], pc.vol_r2[2]);
  float3 q = make_float3((org.x - pc.vol_tx) - c.x, (org.y - pc.vol_ty) - c.y,
                         (org.z - pc.vol_tz) - c.z);
  float3 ro = make_float3(fmaf(r2.x, q.z, fmaf(r1.x, q.y, r0.x * q.x)) + c.x,
                          fmaf(r2.y, q.z, fmaf(r1.y, q.y, r0.y * q.x)) + c.y,
                          fmaf(r2.z, q.z, fmaf(r1.z, q.y, r0.z * q.x)) + c.z);
  dir = make_float3(fmaf(r2.x, dir.z, fmaf(r1.x, dir.y, r0.x * dir.x)),
                    fmaf(r2.y, dir.z, fmaf(r1.y, dir.y, r0.y * dir.x)),
                    fmaf(r2.z, dir.z, fmaf(r1.z, dir.y, r0.z * dir.x)));

  // clip boxes and t range (raycast.slang:686-714)
  float lo[3] = {0.0f, 0.0f, 0.0f}, hi[3] = {ext.x, ext.y, ext.z};
  float t_lo = 0.0f, t_hi = 1e30f;
  if (kLod) {
    float md = s.br.md;
    if ((pc.view_flags & R3D_VIEW_CROP) != 0u) {
      float clo[3] = {pc.slab_x0 / md, pc.slab_y0 / md, pc.slab_z0 / md};
      float cx[3] = {pc.slab_px / md, pc.slab_py / md, pc.slab_nx / md};
#pragma unroll
      for (int a = 0; a < 3; a++) {
        lo[a] = clamp_(clo[a], 0.0f, hi[a]);
        hi[a] = clamp_(clo[a] + cx[a], lo[a], hi[a]);
      }
    } else if (pc.slab_depth > 0u) {
      if ((pc.view_flags & R3D_VIEW_OBLIQUE) != 0u) {
        t_lo = pc.slab_z0 / md;
        t_hi = (pc.slab_z0 + (float)pc.slab_depth) / md;
      } else {
        uint32_t axc = (pc.view_flags >> 8) & 3u;
        int a = axc == 1u ? 0 : (axc == 2u ? 1 : 2);
        float e = a == 0 ? hi[0] : (a == 1 ? hi[1] : hi[2]);
        float nlo = clamp_(pc.slab_z0 / md, 0.0f, e);
        float nhi = clamp_((pc.slab_z0 + (float)pc.slab_depth) / md, nlo, e);
        if (a == 0) { lo[0] = nlo; hi[0] = nhi; }
        if (a == 1) { lo[1] = nlo; hi[1] = nhi; }
        if (a == 2) { lo[2] = nlo; hi[2] = nhi; }
      }
    }
  }
  // box_hit (raycast.slang:489-495)
  float dv[3] = {dir.x, dir.y, dir.z}, ov[3] = {ro.x, ro.y, ro.z};
  float tmn[3], tmx[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    float inv = 1.0f / dv[a];
    float t0 = (lo[a] - ov[a]) * inv, t1 = (hi[a] - ov[a]) * inv;
    tmn[a] = fminf(t0, t1);
    tmx[a] = fmaxf(t0, t1);
  }
  float tn = fmaxf(fmaxf(fmaxf(tmn[0], tmn[1]), tmn[2]), t_lo);
  float tf_ = fminf(fminf(fminf(tmx[0], tmx[1]), tmx[2]), t_hi);
  if (tn >= tf_) {
    out.rgb[0] = 0.02f;
    out.rgb[1] = 0.02f;
    out.rgb[2] = 0.03f;
    return false;
  }

  // jitter, budget (raycast.slang:726-744)
  const uint32_t ray_budget = kLod ? (kShaded ? 192u : 256u) : kMaxSteps;
  st.ro = ro;
  st.dir = dir;
  st.t = fmaf(hash12(px, py, pc.frame_index), vc.dt, tn);
  st.tf_ = tf_;
  st.span_step = fmaxf((tf_ - tn) / ((float)ray_budget * vc.dt), 1.0f);
  st.slab_cap = fmaxf(1.0f, (tf_ - tn) / (4.0f * vc.dt));
  // exp2(lod) <= 2^ceil(max_lod) for every lod the clamp admits (powers of
  // two are exact and the margin covers the approximation), so beyond this
  // bound max(exp2(lod), span_step) is span_step without evaluating exp2
  st.span_dom = st.span_step >= r3d_exp2f(ceilf(vc.max_lod)) * 1.001f;
  st.lod_tlo = R3D_FM_INF;
  st.lod_thi = 0.0f;
  st.steps = 0;
  st.mip_index = 0;
  st.mip_max = 0.0f;
  st.first_hit = -1.0f;
  st.acc_r = st.acc_g = st.acc_b = st.acc_a = 0.0f;
  st.ink_max = st.ink2_max = st.lbl_max = st.reg_max = 0.0f;
  st.lc.desired = -1;
  st.lc.inv_scale = 1.0f;
  st.lc.lo[0] = st.lc.lo[1] = st.lc.lo[2] = R3D_FM_INF;
  st.lc.c.ok = false;
  st.lc.c.maxv = 0.0f;
  st.lc.c.slot = 0;
  st.lc.c.grad_vox = 1.0f;
  st.lc.c.world_brick = 128.0f * vc.voxel;
  st.lc.c.bl = make_float3(0.0f, 0.0f, 0.0f);
  st.n_tf = st.n_grad = st.n_walk = 0;
  return true;
}

// Block jump of the empty-space skip (raycast.slang:864-868).
__device__ __forceinline__ float skip_block(const RayState &st, float3 p, float bsz) {
  float pv[3] = {p.x, p.y, p.z}, dv[3] = {st.dir.x, st.dir.y, st.dir.z},
        ov[3] = {st.ro.x, st.ro.y, st.ro.z};
  float tex[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    float nextp = (floorf(pv[a] / bsz) + (dv[a] > 0.0f ? 1.0f : 0.0f)) * bsz;
    tex[a] = fabsf(dv[a]) > 1e-8f ? (nextp - ov[a]) / dv[a] : 1e30f;
  }
  return fmaxf(fminf(fminf(tex[0], tex[1]), tex[2]), st.t) + bsz * 0.01f;
}

// A gradient tap: the tiled slab's vol_sample; in clip mode the level the
// sample picked (or, without one, vol_sample; raycast.slang:942-946,
// 967-974); else a cube-like texture.
template <int PATH>
__device__ __forceinline__ float tap_sample(const DevScene &s, const DevCube &tex, float3 p,
                                            float lod, int clip_l) {
  if (PATH == PATH_SLAB) return slab_sample(s.sl, p, lod);
  if (PATH == PATH_VSLAB) return vs_sample(s.vs, p, lod);
  if (PATH == PATH_CLIP) return clip_l >= 0 ? clip_level(s.cl, clip_l, p) : clip_sample(s.cl, p, lod);
  return cube_sample(tex, p, lod);
}

// Colour of a contributing sample: the TF colour, gradient shading (FULL
// mode, raycast.slang:919-998) and the overlay tints (:1000-1014).
template <int PATH, int MODE, bool FAST, bool COUNT, bool OVL = false>
__device__ __forceinline__ float3 sample_color(const DevScene &s, const ViewConst &vc,
                                               RayState &st, const Pending &q) {
  constexpr bool kLod = PATH == PATH_LOD_BRICKS;
  constexpr bool kShard = PATH == PATH_SHARD;
  constexpr bool kShaded = MODE == R3D_MODE_FULL;
  const float3 dir = st.dir;
  float col_r = q.sm.x, col_g = q.sm.y, col_b = q.sm.z;
  if (OVL && q.reg_live) {  // green/magenta fuse in TF space, before shading (:910-914)
    const float3 wl = make_float3(0.333f, 0.334f, 0.333f);
    const float lm = dot3(make_float3(q.rs.x, q.rs.y, q.rs.z), wl);
    const float lf = dot3(make_float3(col_r, col_g, col_b), wl);
    col_r = lerp_(col_r, lm, vc.reg_alpha);
    col_g = lerp_(col_g, lf, vc.reg_alpha);
    col_b = lerp_(col_b, lm, vc.reg_alpha);
  }
  // taps sampled like a cube texture: the cube, or the identity shard atlas
  const DevCube &tex = kShard ? s.sh.atlas : s.cube;
  constexpr bool kSlab = PATH == PATH_SLAB;
  // non-identity shard: taps at lod_step voxels through the slot
  // (raycast.slang:937-940,972-979)
  const bool slot_taps = kShard && !s.sh.identity;
  constexpr bool kSection = PATH == PATH_SLAB || PATH == PATH_CLIP || PATH == PATH_VSLAB;
  if (kShaded) {
    if (COUNT) st.n_grad++;
    float g0, g1, g2;
    if (FAST) {  // raycast.slang:919-955
      const float ir3 = 0.57735026919f, renorm = 0.86602540378f;
      float q0, q1, q2, q3;
      if (kLod) {  // the eight quad words are loaded before any is used
        float ev = q.grad_vox * ir3;
        float3 u = q.bl;
        const SlotCoord t[4] = {slot_coord(make_float3(u.x + ev, u.y - ev, u.z - ev)),
                                slot_coord(make_float3(u.x - ev, u.y - ev, u.z + ev)),
                                slot_coord(make_float3(u.x - ev, u.y + ev, u.z - ev)),
                                slot_coord(make_float3(u.x + ev, u.y + ev, u.z + ev))};
        const uint32_t *g = s.br.quad + (size_t)q.slot * (128u * 128u * 128u);
        uint32_t w[8];
#pragma unroll
        for (int k = 0; k < 4; k++) {
          const uint32_t *r = g + ((t[k].z0 << 14) | (t[k].y0 << 7) | t[k].x0);
          w[2 * k] = __ldg(r);
          w[2 * k + 1] = __ldg(r + (t[k].z0 < 127u ? 16384u : 0u));
        }
        q0 = tri_words(w[0], w[1], t[0]);
        q1 = tri_words(w[2], w[3], t[1]);
        q2 = tri_words(w[4], w[5], t[2]);
        q3 = tri_words(w[6], w[7], t[3]);
      } else if (slot_taps) {
        const float ev = q.lod_step * ir3;
        const float3 u = q.bl, org = shard_slot_org(s.sh, q.slot);
        const float e2 = r3d_exp2f(q.lod);
        q0 = shard_fetch(s.sh, org, make_float3(u.x + ev, u.y - ev, u.z - ev), q.lod, e2);
        q1 = shard_fetch(s.sh, org, make_float3(u.x - ev, u.y - ev, u.z + ev), q.lod, e2);
        q2 = shard_fetch(s.sh, org, make_float3(u.x - ev, u.y + ev, u.z - ev), q.lod, e2);
        q3 = shard_fetch(s.sh, org, make_float3(u.x + ev, u.y + ev, u.z + ev), q.lod, e2);
      } else if (kSection) {
        // one inlined copy of the section lookup, looped over the taps, so
        // that the kernel stays in the instruction cache
        const float ee = (vc.voxel * q.lod_step) * ir3;
        q0 = q1 = q2 = q3 = 0.0f;
#pragma unroll 1
        for (int k = 0; k < 4; k++) {  // signs (+--), (--+), (-+-), (+++)
          const float dx = (k == 0 || k == 3) ? ee : -ee, dy = k >= 2 ? ee : -ee;
          const float dz = (k & 1) ? ee : -ee;
          const float t = tap_sample<PATH>(s, tex, make_float3(q.p.x + dx, q.p.y + dy, q.p.z + dz),
                                           q.lod, (int)q.slot);
          if (k == 0) q0 = t;
          else if (k == 1) q1 = t;
          else if (k == 2) q2 = t;
          else q3 = t;
        }
      } else {
        float ee = (vc.voxel * q.lod_step) * ir3;
        q0 = tap_sample<PATH>(s, tex, make_float3(q.p.x + ee, q.p.y - ee, q.p.z - ee), q.lod, (int)q.slot);
        q1 = tap_sample<PATH>(s, tex, make_float3(q.p.x - ee, q.p.y - ee, q.p.z + ee), q.lod, (int)q.slot);
        q2 = tap_sample<PATH>(s, tex, make_float3(q.p.x - ee, q.p.y + ee, q.p.z - ee), q.lod, (int)q.slot);
        q3 = tap_sample<PATH>(s, tex, make_float3(q.p.x + ee, q.p.y + ee, q.p.z + ee), q.lod, (int)q.slot);
      }
      g0 = (((q0 - q1) - q2) + q3) * renorm;
      g1 = (((-q0 - q1) + q2) + q3) * renorm;
      g2 = (((-q0 + q1) - q2) + q3) * renorm;
    } else {  // raycast.slang:957-986
      if (kLod) {
        // each tap moves one axis; the other two keep the sample's own
        // clamped coordinates.  The twelve quad words of the six taps are
        // loaded before any of them is used, so their latencies overlap.
        const float ev = q.grad_vox;
        const float3 u = q.bl;
        const SlotCoord c = slot_coord(u);
        SlotCoord t[6];
#pragma unroll
        for (int k = 0; k < 6; k++) t[k] = c;
        t[0].x0 = slot_axis(u.x + ev, t[0].fx);
        t[1].x0 = slot_axis(u.x - ev, t[1].fx);
        t[2].y0 = slot_axis(u.y + ev, t[2].fy);
        t[3].y0 = slot_axis(u.y - ev, t[3].fy);
        t[4].z0 = slot_axis(u.z + ev, t[4].fz);
        t[5].z0 = slot_axis(u.z - ev, t[5].fz);
        const uint32_t *g = s.br.quad + (size_t)q.slot * (128u * 128u * 128u);
        uint32_t w[12];
#pragma unroll
        for (int k = 0; k < 6; k++) {
          const uint32_t *r = g + ((t[k].z0 << 14) | (t[k].y0 << 7) | t[k].x0);
          w[2 * k] = __ldg(r);
          w[2 * k + 1] = __ldg(r + (t[k].z0 < 127u ? 16384u : 0u));
        }
        float v[6];
#pragma unroll
        for (int k = 0; k < 6; k++) v[k] = tri_words(w[2 * k], w[2 * k + 1], t[k]);
        g0 = v[0] - v[1];
        g1 = v[2] - v[3];
        g2 = v[4] - v[5];
      } else if (slot_taps) {
        const float ev = q.lod_step;
        const float3 u = q.bl, org = shard_slot_org(s.sh, q.slot);
        const float e2 = r3d_exp2f(q.lod);
        g0 = shard_fetch(s.sh, org, make_float3(u.x + ev, u.y, u.z), q.lod, e2) -
             shard_fetch(s.sh, org, make_float3(u.x - ev, u.y, u.z), q.lod, e2);
        g1 = shard_fetch(s.sh, org, make_float3(u.x, u.y + ev, u.z), q.lod, e2) -
             shard_fetch(s.sh, org, make_float3(u.x, u.y - ev, u.z), q.lod, e2);
        g2 = shard_fetch(s.sh, org, make_float3(u.x, u.y, u.z + ev), q.lod, e2) -
             shard_fetch(s.sh, org, make_float3(u.x, u.y, u.z - ev), q.lod, e2);
      } else if (kSection) {  // looped taps, as above
        const float e = vc.voxel * q.lod_step;
        float plus = 0.0f;
        g0 = g1 = g2 = 0.0f;
#pragma unroll 1
        for (int k = 0; k < 6; k++) {  // +x, -x, +y, -y, +z, -z
          const int ax = k >> 1;
          const float d = (k & 1) ? -e : e;
          const float t = tap_sample<PATH>(
              s, tex,
              make_float3(ax == 0 ? q.p.x + d : q.p.x, ax == 1 ? q.p.y + d : q.p.y,
                          ax == 2 ? q.p.z + d : q.p.z),
              q.lod, (int)q.slot);
          if (!(k & 1)) {
            plus = t;
          } else {
            const float g = plus - t;
            if (ax == 0) g0 = g;
            else if (ax == 1) g1 = g;
            else g2 = g;
          }
        }
      } else {
        float e = vc.voxel * q.lod_step;
        g0 = tap_sample<PATH>(s, tex, make_float3(q.p.x + e, q.p.y, q.p.z), q.lod, (int)q.slot) -
             tap_sample<PATH>(s, tex, make_float3(q.p.x - e, q.p.y, q.p.z), q.lod, (int)q.slot);
        g1 = tap_sample<PATH>(s, tex, make_float3(q.p.x, q.p.y + e, q.p.z), q.lod, (int)q.slot) -
             tap_sample<PATH>(s, tex, make_float3(q.p.x, q.p.y - e, q.p.z), q.lod, (int)q.slot);
        g2 = tap_sample<PATH>(s, tex, make_float3(q.p.x, q.p.y, q.p.z + e), q.lod, (int)q.slot) -
             tap_sample<PATH>(s, tex, make_float3(q.p.x, q.p.y, q.p.z - e), q.lod, (int)q.slot);
      }
    }
    float3 gv = make_float3(g0, g1, g2);
    float gm = sqrtf(dot3(gv, gv));
    if (gm > 1e-4f) {  // raycast.slang:988-998
      // key light, headlight l = -dir and its half vector normalize(l - dir)
      const float3 key = norm3(make_float3(0.4f, 0.8f, -0.4f));
      const float3 l = make_float3(-dir.x, -dir.y, -dir.z);
      const float3 hv = norm3(make_float3(l.x - dir.x, l.y - dir.y, l.z - dir.z));
      float inv = 1.0f / gm;
      float3 n = make_float3(gv.x * inv, gv.y * inv, gv.z * inv);
      float diff = fmaf(0.3f, fabsf(dot3(n, key)), 0.7f * fabsf(dot3(n, l)));
      float spec = r3d_powi24f(fabsf(dot3(n, hv))) * 0.3f;
      float lit = fmaf(0.75f, diff, 0.25f);
      float w = sat_(gm * 6.0f);
      float lm = fmaf(w, lit - 1.0f, 1.0f);
      float sw = spec * w;
      col_r = fmaf(col_r, lm, sw);
      col_g = fmaf(col_g, lm, sw);
      col_b = fmaf(col_b, lm, sw);
    }
  }
  if (OVL) {  // overlay tints after shading (raycast.slang:1000-1014)
    const SlotCoord c = slot_coord(q.bl);
    if (vc.ovl & kOvlInk) {
      const float k = sat_(ovl_fetch(s, 0, q.slot, c) * vc.ovl_gain);
      col_r = lerp_(col_r, vc.ovl_col.x, k);
      col_g = lerp_(col_g, vc.ovl_col.y, k);
      col_b = lerp_(col_b, vc.ovl_col.z, k);
    }
    if (vc.ovl & kOvlInk3d) {
      const float k = sat_(ovl_fetch(s, 1, q.slot, c) * vc.ovl_gain);
      col_r = lerp_(col_r, 1.0f, k);
      col_g = lerp_(col_g, 0.30f, k);
      col_b = lerp_(col_b, 0.22f, k);
    }
    if (vc.ovl & kOvlLabels) {
      const float k = ovl_label(s, q.slot, q.bl);
      if (k > 0.0f) {
        const float3 lc = label_color(k);
        col_r = lerp_(col_r, lc.x, 0.65f);
        col_g = lerp_(col_g, lc.y, 0.65f);
        col_b = lerp_(col_b, lc.z, 0.65f);
      }
    }
  }
  return make_float3(col_r, col_g, col_b);
}

// Gradient shading and front-to-back compositing (raycast.slang:1015-1017)
// of a contributing sample, then the step advance (:1020).  Returns false
// when the opacity cutoff ends the ray.
template <int PATH, int MODE, bool FAST, bool COUNT, bool OVL = false>
__device__ __forceinline__ bool composite_sample(const DevScene &s, const ViewConst &vc,
                                                 RayState &st, const Pending &q) {
  const float3 col = sample_color<PATH, MODE, FAST, COUNT, OVL>(s, vc, st, q);
  float wgt = (1.0f - st.acc_a) * q.a;
  st.acc_r = fmaf(wgt, col.x, st.acc_r);
  st.acc_g = fmaf(wgt, col.y, st.acc_g);
  st.acc_b = fmaf(wgt, col.z, st.acc_b);
  st.acc_a = st.acc_a + wgt;
  if (st.acc_a >= s.alpha_cutoff) return false;
  st.t = fmaf(vc.dt, q.lod_step, st.t);
  return true;
}

// Shading later (LOD bricks, FULL mode).  The opacity a ray accumulates, and
// so its termination and step positions, never depend on sample colours:
// only the colour sums do, through rgb <- fma(w_i, c_i, rgb) in sample
// order.  So the march can keep, for each contributing sample, its weight
// w_i = (1 - A) a, its TF coordinate and its brick position, and leave the
// shading (six brick taps, normal, lighting) for later.  A warp shades the
// kept samples of all its rays together once every ray has ended, instead
// of one or two lanes at a time inside divergent steps, and folds them into
// the sums in the same order with the same operations: the image is
// bit-identical.  A ray that keeps kShadeCap samples shades them at once.
#ifndef R3D_SHADE_CAP
#define R3D_SHADE_CAP 4
#endif
constexpr uint32_t kShadeCap = R3D_SHADE_CAP;
struct ShadeEntry {
  float wgt, tt, bx, by, bz, grad_vox;
  uint32_t slot;
};
struct ShadeBuf {
  ShadeEntry e[kShadeCap];
  uint32_t n;
};

template <int PATH, int MODE, bool FAST, bool COUNT>
__device__ __forceinline__ void shade_flush(const DevScene &s, const ViewConst &vc,
                                            const float4 *tf, RayState &st, ShadeBuf &sb) {
#pragma unroll 1
  for (uint32_t k = 0; k < sb.n; k++) {
    const ShadeEntry e = sb.e[k];
    Pending q;
    q.sm = tf_sample(tf, e.tt);
    q.slot = e.slot;
    q.bl = make_float3(e.bx, e.by, e.bz);
    q.grad_vox = e.grad_vox;
    const float3 col = sample_color<PATH, MODE, FAST, COUNT>(s, vc, st, q);
    st.acc_r = fmaf(e.wgt, col.x, st.acc_r);
    st.acc_g = fmaf(e.wgt, col.y, st.acc_g);
    st.acc_b = fmaf(e.wgt, col.z, st.acc_b);
  }
  sb.n = 0;
}

// The footprint ratio of a sample at t (raycast.slang:772-774).
__device__ __forceinline__ float lod_y(const ViewConst &vc, float t) {
  const float foot = vc.ortho ? vc.cone : t * vc.cone;
  return fmaxf(foot * vc.vox_inv, 1.0f);
}

// The samples whose LOD decisions are known without log2 / exp2, after the
// exact lod at some t gave desired level d.  lod = clamp(log2(y) + bias, 0,
// max_lod) has floor d for every footprint ratio y in [2^(d - bias),
// 2^(d + 1 - bias)) (open at the ends for d = 0 and the top level), narrowed
// by 2^-12 relative at each end -- 3.5e-4 in log2, far above the error of
// r3d_log2f plus the rounding of the bias add -- and when span_step >=
// 1.001 * 2^(d + 1) (2^max_lod at the top), lod_step is span_step for every
// lod of the level.  Otherwise the range is empty.  The range is kept as an
// interval of t: y(t) = max(fl(fl(t cone) vox_inv), 1) lies within a
// factor (1 +- 2^-24)^2 of t * cone * vox_inv, so the ends divided by that
// product and moved inwards by 2^-20 relative (far above those roundings
// and the ones of the division) bound t values whose y is certainly inside.
// A sample between the certain interval and the range's true ends takes the
// exact path (log2), which decides the same level and step.
__device__ __forceinline__ void lod_range(RayState &st, const ViewConst &vc, int d, int top) {
  const float hi_lod = d >= top ? vc.max_lod : (float)(d + 1);
  st.lod_tlo = R3D_FM_INF;
  st.lod_thi = 0.0f;
  if (!(st.span_step >= r3d_exp2f(hi_lod) * 1.001f)) return;
  const float ylo = d == 0 ? 0.0f : r3d_exp2f((float)d - vc.lod_bias) * (1.0f + 0x1p-12f);
  const float yhi = d >= top ? R3D_FM_INF : r3d_exp2f((float)(d + 1) - vc.lod_bias) * (1.0f - 0x1p-12f);
  if (vc.ortho) {  // y does not depend on t
    const float y = lod_y(vc, 0.0f);
    if (y >= ylo && y < yhi) {
      st.lod_tlo = -R3D_FM_INF;
      st.lod_thi = R3D_FM_INF;
    }
    return;
  }
  const float k = vc.cone * vc.vox_inv;
  if (!(k >= 0x1p-60f && k <= 0x1p60f) || !(yhi > 1.0f)) return;  // y >= 1: never below yhi <= 1
  st.lod_tlo = ylo <= 1.0f ? -R3D_FM_INF : (ylo / k) * (1.0f + 0x1p-20f);
  st.lod_thi = yhi == R3D_FM_INF ? R3D_FM_INF : (yhi / k) * (1.0f - 0x1p-20f);
}

// One iteration of the hot loop (raycast.slang:767-1021).  Returns
// kStepDone when the ray is finished (loop condition failed, saturation or
// opacity cutoff) and kStepCont otherwise.  With DEFER, a sample that needs
// gradient shading stops before it: the sample is left in pend and
// kStepShade returned; composite_sample(pend) completes the iteration.
template <int PATH, int MODE, bool FAST, bool COUNT, bool DEFER = false, bool OVL = false,
          bool LATER = false, bool STAGE = false>
__device__ __forceinline__ int ray_step(const DevScene &s, const ViewConst &vc, const float4 *tf,
                                        RayState &st, Pending &pend, ShadeBuf *sb = nullptr,
                                        const StageBox *box = nullptr) {
  constexpr bool kLod = PATH == PATH_LOD_BRICKS;
  constexpr bool kShard = PATH == PATH_SHARD;
  constexpr bool kSlab = PATH == PATH_SLAB;
  constexpr bool kClip = PATH == PATH_CLIP;
  constexpr bool kVslab = PATH == PATH_VSLAB;
  constexpr bool kComposite = MODE == R3D_MODE_FULL || MODE == R3D_MODE_FLAT;
  constexpr bool kShaded = MODE == R3D_MODE_FULL;
  constexpr uint32_t ray_budget = kLod ? (kShaded ? 192u : 256u) : kMaxSteps;
  if (!(st.t < st.tf_ && st.steps < ray_budget)) return kStepDone;
  st.steps++;
  const float t = st.t;
  // LOD and step (raycast.slang:772-779)
  float lod = 0.0f;
  bool lod_known = true;
  if (vc.lod_on) {
    if (kLod && t >= st.lod_tlo && t < st.lod_thi)
      lod_known = false;  // level and lod_step known (lod_range)
    else
      lod = clamp_(r3d_log2f(lod_y(vc, t)) + vc.lod_bias, 0.0f, vc.max_lod);
  }
  float lod_step =
      !lod_known || st.span_dom ? st.span_step
                                : fmaxf(lod == 0.0f ? 1.0f : r3d_exp2f(lod), st.span_step);
  if (kSlab || kClip || kVslab) lod_step = fminf(lod_step, st.slab_cap);
  const float3 dir = st.dir;
  const float3 p =
      make_float3(fmaf(t, dir.x, st.ro.x), fmaf(t, dir.y, st.ro.y), fmaf(t, dir.z, st.ro.z));

  float v = 0.0f;
  BrickCtx b;
  if (kLod) {
    const int top = (int)s.br.nlev - 1;
    int desired = st.lc.desired;
    if (lod_known) {
      desired = (int)clamp_(floorf(lod), 0.0f, (float)top);
      if (desired != st.lc.desired) lod_range(st, vc, desired, top);
    }
    if (!lod_cache_hit(s, p, desired, st.lc, b)) {  // walk the page table
      if (!lod_known) lod = clamp_(r3d_log2f(lod_y(vc, t)) + vc.lod_bias, 0.0f, vc.max_lod);
      if (COUNT) st.n_walk++;
      b = lod_locate_ex(s, p, lod, st.lc, desired);
    }
    if (b.ok) {
      // Exact fetch elision: vub bounds the trilinear value from above
      // (every tap lies in the dilated block and rounding is monotone).
      // When vub already fixes every decision the sample feeds, the outcome
      // equals the fetched one and the 8 loads are skipped.  The decisions
      // on vub are taken on its byte m against the view's counts.
      const SlotCoord q = slot_coord(b.bl);
      const uint32_t m = __ldg(s.br.bmax + (size_t)b.slot * 4096u +
                               (((q.z0 >> 3) << 8) | ((q.y0 >> 3) << 4) | (q.x0 >> 3)));
      const bool brick_lit = b.maxv >= vc.bgate;
      const bool void_known = brick_lit || m < vc.el.n_void;
      bool elide;
      if (MODE == R3D_MODE_MIP)
        elide = b.maxv <= st.mip_max ||
                (void_known && (m < vc.el.n_dec || byte_float(m) * kInv255 <= st.mip_max));
      else if (MODE == R3D_MODE_DEPTH)
        elide = void_known && (st.first_hit >= 0.0f || m < vc.el.n_dec);
      else if (MODE == R3D_MODE_HEATMAP)
        elide = void_known;
      else
        elide = void_known && m < vc.el.n_dec;
      // overlays read every sample (MIP maxima, registration opacity)
      if (!OVL && elide) {  // the sample changes nothing but the march position
        if ((MODE == R3D_MODE_MIP && b.maxv <= st.mip_max) || b.maxv < vc.bgate) {
          st.t = skip_block(st, p, b.world_brick);
          return kStepCont;
        }
        st.t = fmaf(vc.dt, lod_step, t);
        return kStepCont;
      }
      if (COUNT && s.slot_bits) {  // the unique slots a frame reads (test first: few atomics)
        const uint32_t m = 1u << (b.slot & 31u);
        if (!(__ldcg(s.slot_bits + (b.slot >> 5)) & m)) atomicOr(s.slot_bits + (b.slot >> 5), m);
      }
      if (STAGE && box_has(*box, b.slot, q)) {
        v = box_sample(*box, q);
      } else {
        const uint32_t *g = s.br.quad + (size_t)b.slot * (128u * 128u * 128u) +
                            ((q.z0 << 14) | (q.y0 << 7) | q.x0);
        const uint32_t w0 = __ldg(g), w1 = __ldg(g + (q.z0 < 127u ? 16384u : 0u));
        // The same elision on the sample's own eight bytes: their maximum
        // bounds the trilinear value too, so in a lit brick (known void) the
        // outcome is fixed when every byte is below n_dec.
        constexpr bool kByteElide = R3D_BYTE_ELIDE && !OVL &&
            (MODE == R3D_MODE_FULL || MODE == R3D_MODE_FLAT || MODE == R3D_MODE_DEPTH);
        const RawBytes rb = raw_bytes(w0, w1);
        if (kByteElide && brick_lit && raw_max(rb) < vc.el.raw_dec) {
          st.t = fmaf(vc.dt, lod_step, t);
          return kStepCont;
        }
        v = tri_raw(rb, q);
      }
    }
  } else if (kShard) {
    const DevShard &h = s.sh;
    if (h.identity) {  // atlas layout == world layout (raycast.slang:800-805)
      v = cube_sample(h.atlas, p, lod);
    } else {
      // page entry cached until the brick changes (raycast.slang:806-822)
      const float3 vp = make_float3(sat_(p.x) * h.n, sat_(p.y) * h.n, sat_(p.z) * h.n);
      const uint32_t bx = min((uint32_t)vp.x >> 7, h.bpa - 1u);
      const uint32_t by = min((uint32_t)vp.y >> 7, h.bpa - 1u);
      const uint32_t bz = min((uint32_t)vp.z >> 7, h.bpa - 1u);
      const uint32_t bi = (bz * h.bpa + by) * h.bpa + bx;
      if ((int)bi != st.lc.desired) {
        st.lc.desired = (int)bi;
        shard_entry(s, bi, st.lc.c);
        if (COUNT) st.n_walk++;
      }
      b = st.lc.c;
      b.bl = make_float3(vp.x - (float)(bx << 7), vp.y - (float)(by << 7), vp.z - (float)(bz << 7));
      v = b.ok ? shard_fetch(h, shard_slot_org(h, b.slot), b.bl, lod,
                             lod == 0.0f ? 1.0f : r3d_exp2f(lod))
               : 0.0f;
    }
  } else if (kSlab) {
    v = slab_sample(s.sl, p, lod);
  } else if (kVslab) {
    v = vs_sample(s.vs, p, lod);
  } else if (kClip) {  // the level is picked once; taps reuse it (raycast.slang:785-787)
    const int cl = clip_pick(s.cl, p, lod);
    b.slot = (uint32_t)cl;
    v = cl < 0 ? 0.0f : clip_level(s.cl, cl, p);
  } else {
    v = cube_sample(s.cube, p, lod);
  }
  const bool cut = v < vc.threshold;  // raycast.slang:826-827
  if (cut) v = 0.0f;

  // empty-space skip (raycast.slang:829-869)
  if (kLod) {
    // MIP early-out only without overlays: ink can live where CT is dim
    if ((MODE == R3D_MODE_MIP && !OVL && b.ok && b.maxv <= st.mip_max) ||
        (v < vc.bgate && b.maxv < vc.bgate)) {
      st.t = skip_block(st, p, b.world_brick);
      return kStepCont;
    }
  } else if (kShard) {
    if (v < vc.bgate) {
      if (s.sh.identity) {  // 8^3 occupancy only
        if (occ_sample(s.sh.atlas, p) < vc.bgate) {
          st.t = skip_block(st, p, vc.bs);
          return kStepCont;
        }
      } else if (b.maxv < vc.bgate) {  // whole brick (cached page entry)
        st.t = skip_block(st, p, 128.0f * vc.voxel);
        return kStepCont;
      } else if (occ_sample(s.sh.atlas, p) < vc.bgate) {  // 8^3 block
        st.t = skip_block(st, p, vc.bs);
        return kStepCont;
      }
    }
  } else if (!kSlab && !kClip && !kVslab && v < vc.occ_gate &&
             occ_sample(s.cube, p) < vc.occ_gate) {
    st.t = skip_block(st, p, vc.bs);  // (no empty-space skip in slab mode: raycast.slang:861)
    return kStepCont;
  }

  // the running maximum and its step, for MIP views (their MIP index aux
  // output); LOD-brick views of other modes without overlays skip it
  constexpr bool kTrackMip = MODE == R3D_MODE_MIP || !kLod || OVL;
  if (kTrackMip && v > st.mip_max) {
    st.mip_max = v;
    st.mip_index = st.steps;
  }
  if (OVL && MODE == R3D_MODE_MIP && b.ok) {  // overlay maxima (raycast.slang:872-887)
    const SlotCoord c = slot_coord(b.bl);
    if (vc.ovl & kOvlInk) {
      const float k = ovl_fetch(s, 0, b.slot, c);
      if (k > st.ink_max) st.ink_max = k;
    }
    if (vc.ovl & kOvlInk3d) {
      const float k = ovl_fetch(s, 1, b.slot, c);
      if (k > st.ink2_max) st.ink2_max = k;
    }
    if (vc.ovl & kOvlLabels) {
      const float k = ovl_label(s, b.slot, b.bl);
      if (k > st.lbl_max) st.lbl_max = k;
    }
    if (vc.ovl & kOvlReg) {
      float k = ovl_fetch(s, 3, b.slot, c);
      if (k < vc.threshold) k = 0.0f;
      if (k > st.reg_max) st.reg_max = k;
    }
  }
  if (MODE == R3D_MODE_MIP && !OVL && st.mip_max >= 0.999f) return kStepDone;
  if (MODE == R3D_MODE_DEPTH && st.first_hit < 0.0f && v > 0.05f) st.first_hit = t;

  if (kComposite && !cut) {
    float tt = clamp_(fmaf(v, 256.0f, -0.5f), 0.0f, 255.0f);
    const bool reg_live = OVL && (vc.ovl & kOvlReg) && b.ok;
    // below tf_zero_t both TF texels have alpha 0, so the opacity is
    // exactly 0 and the sample cannot contribute (unless the registration
    // scan lends it opacity)
    if (tt >= s.tf_zero_t || reg_live) {
      if (COUNT) st.n_tf++;
      float4 sm = tf_sample(tf, tt);
      float4 rs = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      if (reg_live) {  // the moving scan through the same TF (raycast.slang:895-905)
        float rv = ovl_fetch(s, 3, b.slot, slot_coord(b.bl));
        if (rv < vc.threshold) rv = 0.0f;
        rs = tf_sample(tf, clamp_(fmaf(rv, 256.0f, -0.5f), 0.0f, 255.0f));
        sm.w = fmaxf(sm.w, rs.w * vc.reg_alpha);
      }
      float a = 1.0f - r3d_powf(1.0f - sm.w, vc.opac_k * lod_step);
      if (LATER && a > 0.003f) {  // keep the sample; its colour comes later
        const float wgt = (1.0f - st.acc_a) * a;
        st.acc_a = st.acc_a + wgt;
        sb->e[sb->n] = {wgt, tt, b.bl.x, b.bl.y, b.bl.z, b.grad_vox, b.slot};
        if (++sb->n == kShadeCap) shade_flush<PATH, MODE, FAST, COUNT>(s, vc, tf, st, *sb);
        if (st.acc_a >= s.alpha_cutoff) return kStepDone;
        st.t = fmaf(vc.dt, lod_step, t);
        return kStepCont;
      }
      if (a > 0.003f) {
        const Pending q = {p, lod, lod_step, a, sm, b.slot, b.bl, b.grad_vox, rs, reg_live};
        if (DEFER && kShaded) {  // shading runs later, grouped across the warp
          pend = q;
          return kStepShade;
        }
        return composite_sample<PATH, MODE, FAST, COUNT, OVL>(s, vc, st, q) ? kStepCont
                                                                           : kStepDone;
      }
    }
  }
  st.t = fmaf(vc.dt, lod_step, t);  // raycast.slang:1020
  return kStepCont;
}

// Final colour of a marched ray (raycast.slang:1023-1038).
template <int MODE, bool OVL = false>
__device__ __forceinline__ void ray_end(const ViewConst &vc, const RayState &st, RayResult &out) {
  constexpr bool kComposite = MODE == R3D_MODE_FULL || MODE == R3D_MODE_FLAT;
  out.steps = st.steps;
  out.mip_index = st.mip_index;
  out.n_tf = st.n_tf;
  out.n_grad = st.n_grad;
  out.n_walk = st.n_walk;
  if (MODE == R3D_MODE_HEATMAP) {
    float x = (float)st.steps / 1024.0f;
    out.rgb[0] = x;
    out.rgb[1] = 1.0f - fabsf(x - 0.5f) * 2.0f;
    out.rgb[2] = 1.0f - x;
  } else if (MODE == R3D_MODE_DEPTH) {
    float d = st.first_hit < 0.0f ? 0.0f : 1.0f - sat_(st.first_hit * 0.5f);
    out.rgb[0] = out.rgb[1] = out.rgb[2] = d;
  } else if (kComposite) {
    float tr = 1.0f - st.acc_a;
    out.rgb[0] = fmaf(tr, 0.02f, st.acc_r);
    out.rgb[1] = fmaf(tr, 0.02f, st.acc_g);
    out.rgb[2] = fmaf(tr, 0.03f, st.acc_b);
  } else {
    float m = st.mip_max * vc.density;
    out.rgb[0] = out.rgb[1] = out.rgb[2] = m;
    if (OVL) {  // overlay MIP tints (raycast.slang:1032-1036)
      float r = m, g = m, b = m;
      if (vc.ovl & kOvlReg) {  // reg_fuse (raycast.slang:113-116)
        const float mr = st.reg_max * vc.density;
        const float lum = dot3(make_float3(r, g, b), make_float3(0.333f, 0.334f, 0.333f));
        r = lerp_(r, mr, vc.reg_alpha);
        g = lerp_(g, lum, vc.reg_alpha);
        b = lerp_(b, mr, vc.reg_alpha);
      }
      if (vc.ovl & kOvlInk) {
        const float k = sat_(st.ink_max * vc.ovl_gain);
        r = lerp_(r, vc.ovl_col.x, k);
        g = lerp_(g, vc.ovl_col.y, k);
        b = lerp_(b, vc.ovl_col.z, k);
      }
      if (vc.ovl & kOvlInk3d) {
        const float k = sat_(st.ink2_max * vc.ovl_gain);
        r = lerp_(r, 1.0f, k);
        g = lerp_(g, 0.30f, k);
        b = lerp_(b, 0.22f, k);
      }
      if ((vc.ovl & kOvlLabels) && st.lbl_max > 0.0f) {
        const float3 lc = label_color(st.lbl_max);
        r = lerp_(r, lc.x, 0.65f);
        g = lerp_(g, lc.y, 0.65f);
        b = lerp_(b, lc.z, 0.65f);
      }
      out.rgb[0] = r;
      out.rgb[1] = g;
      out.rgb[2] = b;
    }
  }
}

// One ray start to finish: raycast.slang main() for dispatch thread (px, py).
template <int PATH, int MODE, bool FAST, bool COUNT = false, bool OVL = false>
__device__ __forceinline__ void march(const r3d_frame_params &pc, const DevScene &s,
                                      const ViewConst &vc, const float4 *tf, uint32_t px,
                                      uint32_t py, RayResult &out) {
  RayState st;
  Pending pend;
  if (!ray_begin<PATH, MODE>(pc, s, vc, px, py, st, out)) return;
  while (ray_step<PATH, MODE, FAST, COUNT, false, OVL>(s, vc, tf, st, pend) != kStepDone) {
  }
  ray_end<MODE, OVL>(vc, st, out);
}

// Whether a kernel instantiation shades later (see shade_flush).
#ifndef R3D_SHADE_LATER
#define R3D_SHADE_LATER 0
#endif
template <int PATH, int MODE, bool OVL>
constexpr bool kShadesLater =
    R3D_SHADE_LATER && PATH == PATH_LOD_BRICKS && MODE == R3D_MODE_FULL && !OVL;

// march() for every lane of a warp (all 32 lanes call it; `inside` says
// whether the lane has a ray): with shading later, the rays march, the warp
// reconverges, and the kept samples of all its rays are shaded together.
template <int PATH, int MODE, bool FAST, bool COUNT = false, bool OVL = false>
__device__ __forceinline__ void march_warp(const r3d_frame_params &pc, const DevScene &s,
                                           const ViewConst &vc, const float4 *tf, uint32_t px,
                                           uint32_t py, bool inside, RayResult &out) {
  if constexpr (kShadesLater<PATH, MODE, OVL>) {
    RayState st;
    Pending pend;
    ShadeBuf sb;
    sb.n = 0;
    const bool marched = inside && ray_begin<PATH, MODE>(pc, s, vc, px, py, st, out);
    if (marched)
      while (ray_step<PATH, MODE, FAST, COUNT, false, false, true>(s, vc, tf, st, pend, &sb) !=
             kStepDone) {
      }
    __syncwarp();
    if (marched) {
      shade_flush<PATH, MODE, FAST, COUNT>(s, vc, tf, st, sb);
      ray_end<MODE>(vc, st, out);
    }
  } else {
    if (inside) march<PATH, MODE, FAST, COUNT, OVL>(pc, s, vc, tf, px, py, out);
  }
}

}  // namespace r3d
