/* CPU oracle for the volume raycast (test infrastructure; see r3d_oracle.h).
 *
 * Build with -ffp-contract=off: every multiply-add that is fused is written
 * as fmaf, every other operation rounds on its own, in the order written.
 * Line references are to the reference tree (src/shaders/raycast.slang
 * unless another file is named). */
#include "r3d_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "r3d_fmath.h"

/* ---------------------------------------------------------------- helpers */

typedef struct v3f {
  float x, y, z;
} v3f;

static inline v3f mk3(float x, float y, float z) {
  v3f r = {x, y, z};
  return r;
}
/* dot product, evaluated as fma(z, fma(y, x*x)) */
static inline float dot3(v3f a, v3f b) { return fmaf(a.z, b.z, fmaf(a.y, b.y, a.x * b.x)); }
static inline float lerpf_(float a, float b, float t) { return fmaf(t, b - a, a); }
static inline float clampf_(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
static inline float satf(float x) { return clampf_(x, 0.0f, 1.0f); }
static inline v3f norm3(v3f a) {
  float inv = 1.0f / sqrtf(dot3(a, a));
  return mk3(a.x * inv, a.y * inv, a.z * inv);
}

#define INV255 (1.0f / 255.0f)
#define MAX_STEPS 4096u   /* :123 */
#define OCC_BLOCK 8.0f    /* :125 */
#define BR_SLOT 128.0f    /* :156 */

static const float BG_R = 0.02f, BG_G = 0.02f, BG_B = 0.03f; /* :716 */

/* hash12, src/shaders/common.slang:57-61 */
static float hash12(uint32_t px, uint32_t py, uint32_t frame) {
  uint32_t h = px * 374761393u + py * 668265263u + frame * 2246822519u;
  h = (h ^ (h >> 13)) * 1274126177u;
  return (float)(h >> 8) * (1.0f / 16777216.0f);
}

static inline uint8_t unorm8(float x) { return (uint8_t)(int)fmaf(satf(x), 255.0f, 0.5f); }

/* ------------------------------------------------------------ sampling */

/* clamp-to-edge trilinear at texel centres on one u8 grid; the 8 taps are
 * blended in 0..255 space (x, then y, then z) and scaled by 1/255 */
static float tri_u8(const uint8_t *g, uint32_t dx, uint32_t dy, uint32_t dz, float tx, float ty,
                    float tz) {
  tx = clampf_(tx, 0.0f, (float)(dx - 1u));
  ty = clampf_(ty, 0.0f, (float)(dy - 1u));
  tz = clampf_(tz, 0.0f, (float)(dz - 1u));
  uint32_t x0 = (uint32_t)tx, y0 = (uint32_t)ty, z0 = (uint32_t)tz;
  float fx = tx - (float)x0, fy = ty - (float)y0, fz = tz - (float)z0;
  uint32_t x1 = x0 + 1u < dx ? x0 + 1u : dx - 1u;
  uint32_t y1 = y0 + 1u < dy ? y0 + 1u : dy - 1u;
  uint32_t z1 = z0 + 1u < dz ? z0 + 1u : dz - 1u;
  size_t sx = 1, sy = dx, sz = (size_t)dx * dy;
  const uint8_t *b = g;
#define T(X, Y, Z) ((float)b[(size_t)(X) * sx + (size_t)(Y) * sy + (size_t)(Z) * sz])
  float c00 = lerpf_(T(x0, y0, z0), T(x1, y0, z0), fx);
  float c10 = lerpf_(T(x0, y1, z0), T(x1, y1, z0), fx);
  float c01 = lerpf_(T(x0, y0, z1), T(x1, y0, z1), fx);
  float c11 = lerpf_(T(x0, y1, z1), T(x1, y1, z1), fx);
#undef T
  float c0 = lerpf_(c00, c10, fy), c1 = lerpf_(c01, c11, fy);
  return lerpf_(c0, c1, fz) * INV255;
}

/* volumes[0].SampleLevel(p, lod) with the trilinear + linear-mip sampler of
 * src/vk/vkbackend.c:1058-1069 (:409-416) */
static float cube_sample(const orc_cube *c, v3f p, float lod) {
  float fl = floorf(lod);
  uint32_t m0 = (uint32_t)fl;
  if (m0 > c->nlevels - 1u) m0 = c->nlevels - 1u;
  float fr = lod - fl;
  const uint32_t *d = c->dim[m0];
  float v = tri_u8(c->level[m0], d[0], d[1], d[2], fmaf(p.x, (float)d[0], -0.5f),
                   fmaf(p.y, (float)d[1], -0.5f), fmaf(p.z, (float)d[2], -0.5f));
  if (fr > 0.0f && m0 + 1u < c->nlevels) {
    const uint32_t *e = c->dim[m0 + 1u];
    float v1 = tri_u8(c->level[m0 + 1u], e[0], e[1], e[2], fmaf(p.x, (float)e[0], -0.5f),
                      fmaf(p.y, (float)e[1], -0.5f), fmaf(p.z, (float)e[2], -0.5f));
    v = lerpf_(v, v1, fr);
  }
  return v;
}

/* occ.SampleLevel(p, 0) with the nearest sampler */
static float occ_sample(const uint8_t *occ, const uint32_t od[3], v3f p) {
  float q[3] = {floorf(p.x * (float)od[0]), floorf(p.y * (float)od[1]), floorf(p.z * (float)od[2])};
  uint32_t i[3];
  for (int a = 0; a < 3; a++) {
    float m = (float)(od[a] - 1u);
    i[a] = !(q[a] >= 0.0f) ? 0u : (q[a] > m ? od[a] - 1u : (uint32_t)q[a]);
  }
  return (float)occ[((size_t)i[2] * od[1] + i[1]) * od[0] + i[0]] * INV255;
}

/* tf.SampleLevel(v, 0): 256-texel linear sampler, clamp (:894) */
static void tf_sample(const uint8_t lut[256][4], float v, float s[4]) {
  float t = clampf_(fmaf(v, 256.0f, -0.5f), 0.0f, 255.0f);
  uint32_t i0 = (uint32_t)t;
  uint32_t i1 = i0 + 1u < 256u ? i0 + 1u : 255u;
  float f = t - (float)i0;
  for (int c = 0; c < 4; c++) s[c] = lerpf_((float)lut[i0][c], (float)lut[i1][c], f) * INV255;
}

/* ------------------------------------------------------------- bricks */

typedef struct brick_ctx { /* BrickCtx, :144-152 */
  int ok;
  float maxv;
  v3f bl;
  uint32_t slot;
  float grad_vox;
  float world_brick;
} brick_ctx;

typedef struct lod_cache { /* LodCache, :190-196 */
  int valid;
  int desired;
  uint32_t scale;
  uint32_t bc[3];
  brick_ctx c;
} lod_cache;

typedef struct scene {
  const orc_cube *cube;
  const orc_bricks *br;
  uint32_t *status;
  const r3d_frame_params *pc; /* the view */
} scene;

static inline uint32_t page_rd(const scene *s, uint32_t i) {
  if (i >= s->br->page_words) {
    *s->status |= 1u;
    return 0xFFFFFFFFu;
  }
  return s->br->page[i];
}

/* bricks_lod_locate_ex, :198-247 */
static brick_ctx lod_locate_ex(const scene *s, v3f p, float lod, uint32_t *scale_out,
                               uint32_t bc_out[3]) {
  brick_ctx c;
  *scale_out = 1u;
  bc_out[0] = bc_out[1] = bc_out[2] = 0u;
  c.ok = 0;
  c.maxv = 0.0f;
  c.bl = mk3(0, 0, 0);
  c.slot = 0;
  c.grad_vox = 1.0f;
  uint32_t nlev = page_rd(s, 0);
  float bs[3] = {(float)page_rd(s, 1), (float)page_rd(s, 2), (float)page_rd(s, 3)};
  float md = fmaxf(bs[0], fmaxf(bs[1], bs[2]));
  c.world_brick = (BR_SLOT * (float)(1u << (nlev - 1u))) / md;
  float base_v[3] = {clampf_(p.x * md, 0.0f, fmaxf(bs[0] - 0.001f, 0.0f)),
                     clampf_(p.y * md, 0.0f, fmaxf(bs[1] - 0.001f, 0.0f)),
                     clampf_(p.z * md, 0.0f, fmaxf(bs[2] - 0.001f, 0.0f))};
  int desired = (int)clampf_(floorf(lod), 0.0f, (float)(nlev - 1u));
  int last = (int)nlev - 1;
  for (uint32_t step = 0; step < 4u; step++) {
    int li = step < 3u ? desired + (int)step : last;
    if (li < 0 || li > last || (step == 3u && li <= desired + 2)) continue;
    uint32_t h = 4u + (uint32_t)li * 4u;
    uint32_t off = page_rd(s, h), packed = page_rd(s, h + 1u), scale = page_rd(s, h + 2u);
    uint32_t bd[3] = {packed & 1023u, (packed >> 10) & 1023u, packed >> 20};
    float lv[3];
    uint32_t bc[3];
    for (int a = 0; a < 3; a++) {
      lv[a] = base_v[a] / (float)scale;
      uint32_t q = (uint32_t)lv[a] >> 7;
      bc[a] = q < bd[a] - 1u ? q : bd[a] - 1u;
    }
    uint32_t bi = off + (bc[2] * bd[1] + bc[1]) * bd[0] + bc[0];
    uint32_t e = page_rd(s, bi);
    if (e == 0xFFFFFFFFu) continue;
    uint32_t slot = e & 0xFFFFFFu;
    if (slot >= s->br->nslots) {
      *s->status |= 1u;
      continue;
    }
    c.ok = 1;
    c.maxv = (float)(e >> 24) / 255.0f;
    c.slot = slot;
    c.bl = mk3(lv[0] - (float)(bc[0] << 7), lv[1] - (float)(bc[1] << 7),
               lv[2] - (float)(bc[2] << 7));
    c.grad_vox = r3d_exp2f(lod) / (float)scale;
    c.world_brick = (BR_SLOT * (float)scale) / md;
    *scale_out = scale;
    bc_out[0] = bc[0];
    bc_out[1] = bc[1];
    bc_out[2] = bc[2];
    return c;
  }
  return c;
}

/* bricks_lod_locate_cached, :255-279 */
static brick_ctx lod_locate_cached(const scene *s, v3f p, float lod, lod_cache *lc) {
  uint32_t nlev = page_rd(s, 0);
  int desired = (int)clampf_(floorf(lod), 0.0f, (float)(nlev - 1u));
  if (lc->valid && lc->desired == desired) {
    float bs[3] = {(float)page_rd(s, 1), (float)page_rd(s, 2), (float)page_rd(s, 3)};
    float md = fmaxf(bs[0], fmaxf(bs[1], bs[2]));
    float pv[3] = {p.x, p.y, p.z};
    float lv[3];
    uint32_t bc[3];
    for (int a = 0; a < 3; a++) {
      float base_v = clampf_(pv[a] * md, 0.0f, fmaxf(bs[a] - 0.001f, 0.0f));
      lv[a] = base_v / (float)lc->scale;
      bc[a] = (uint32_t)lv[a] >> 7;
    }
    if (bc[0] == lc->bc[0] && bc[1] == lc->bc[1] && bc[2] == lc->bc[2]) {
      brick_ctx c = lc->c;
      c.bl = mk3(lv[0] - (float)(bc[0] << 7), lv[1] - (float)(bc[1] << 7),
                 lv[2] - (float)(bc[2] << 7));
      return c;
    }
  }
  uint32_t scale, bc[3];
  brick_ctx c = lod_locate_ex(s, p, lod, &scale, bc);
  lc->valid = c.ok;
  lc->desired = desired;
  lc->scale = scale;
  lc->bc[0] = bc[0];
  lc->bc[1] = bc[1];
  lc->bc[2] = bc[2];
  lc->c = c;
  return c;
}

/* bricks_fetch at atlas lod 0 (:284-288): clamp to [0.5, 127.5] inside the
 * brick (no cross-brick filtering), trilinear in the slot */
static float brick_fetch(const scene *s, uint32_t slot, v3f bl) {
  const uint8_t *g = s->br->pool + (size_t)slot * (128u * 128u * 128u);
  float lx = clampf_(bl.x, 0.5f, 127.5f), ly = clampf_(bl.y, 0.5f, 127.5f),
        lz = clampf_(bl.z, 0.5f, 127.5f);
  return tri_u8(g, 128u, 128u, 128u, lx - 0.5f, ly - 0.5f, lz - 0.5f);
}

/* bricks_fetch of the single-level atlas (:284-288): the brick-local
 * position clamped to [inset, 128 - inset], inset = max(0.5 * 2^lod, 0.5),
 * then the atlas sampled at lod like a cube texture at
 * (slot origin + clamped position) / (abpa * 128) */
static float shard_fetch(const orc_cube *atlas, float inv_adim, v3f org, v3f bl, float lod) {
  float inset = fmaxf(0.5f * r3d_exp2f(lod), 0.5f), hi = 128.0f - inset;
  v3f u = mk3((org.x + clampf_(bl.x, inset, hi)) * inv_adim,
              (org.y + clampf_(bl.y, inset, hi)) * inv_adim,
              (org.z + clampf_(bl.z, inset, hi)) * inv_adim);
  return cube_sample(atlas, u, lod);
}

/* overlay atlas i at the sample's brick coordinate: ink / 3D ink /
 * registration like bricks_fetch (:87-97,105-111), labels at the texel
 * centre under bl (:99-104) */
static float ovl_fetch(const scene *s, int i, uint32_t slot, v3f bl) {
  const uint8_t *g = s->br->ovl[i] + (size_t)slot * (128u * 128u * 128u);
  if (i == 2) {
    float lx = clampf_(floorf(bl.x) + 0.5f, 0.5f, 127.5f),
          ly = clampf_(floorf(bl.y) + 0.5f, 0.5f, 127.5f),
          lz = clampf_(floorf(bl.z) + 0.5f, 0.5f, 127.5f);
    return tri_u8(g, 128u, 128u, 128u, lx - 0.5f, ly - 0.5f, lz - 0.5f);
  }
  float lx = clampf_(bl.x, 0.5f, 127.5f), ly = clampf_(bl.y, 0.5f, 127.5f),
        lz = clampf_(bl.z, 0.5f, 127.5f);
  return tri_u8(g, 128u, 128u, 128u, lx - 0.5f, ly - 0.5f, lz - 0.5f);
}

/* label_color, :63-66 (palette :52-61) */
static void label_color(float v, float c[3]) {
  static const float pal[8][3] = {{0.82f, 0.66f, 0.43f}, {0.95f, 0.20f, 0.85f},
                                  {0.20f, 0.80f, 0.80f}, {0.30f, 0.90f, 0.30f},
                                  {1.00f, 0.55f, 0.15f}, {0.35f, 0.45f, 0.90f},
                                  {0.95f, 0.90f, 0.20f}, {0.90f, 0.90f, 0.90f}};
  uint32_t k = (uint32_t)floorf(fmaf(v, 255.0f, 0.5f));
  k = k < 1u ? 1u : (k > 8u ? 8u : k);
  for (int j = 0; j < 3; j++) c[j] = pal[k - 1u][j];
}

static void lerp3(float c[3], float r, float g, float b, float t) {
  c[0] = lerpf_(c[0], r, t);
  c[1] = lerpf_(c[1], g, t);
  c[2] = lerpf_(c[2], b, t);
}

/* a tw x th x wz texture at normalized (u, v, w): linear, clamp to edge in
 * x and y, REPEAT in w (the slab sampler, vkbackend.c:2203-2211) */
static float tex_wrapz(const uint8_t *g, uint32_t tw, uint32_t th, uint32_t wz, float u, float v,
                       float w) {
  float tx = clampf_(fmaf(u, (float)tw, -0.5f), 0.0f, (float)(tw - 1u));
  float ty = clampf_(fmaf(v, (float)th, -0.5f), 0.0f, (float)(th - 1u));
  float tz = fmaf(w, (float)wz, -0.5f);
  uint32_t x0 = (uint32_t)tx, y0 = (uint32_t)ty;
  float fx = tx - (float)x0, fy = ty - (float)y0;
  float zf = floorf(tz), fz = tz - zf;
  int zi = (int)zf % (int)wz;
  if (zi < 0) zi += (int)wz;
  uint32_t z0 = (uint32_t)zi, z1 = z0 + 1u < wz ? z0 + 1u : 0u;
  uint32_t x1 = x0 + 1u < tw ? x0 + 1u : tw - 1u, y1 = y0 + 1u < th ? y0 + 1u : th - 1u;
  size_t sy = tw, sz = (size_t)tw * th;
#define T(X, Y, Z) ((float)g[(size_t)(X) + (size_t)(Y) * sy + (size_t)(Z) * sz])
  float c00 = lerpf_(T(x0, y0, z0), T(x1, y0, z0), fx);
  float c10 = lerpf_(T(x0, y1, z0), T(x1, y1, z0), fx);
  float c01 = lerpf_(T(x0, y0, z1), T(x1, y0, z1), fx);
  float c11 = lerpf_(T(x0, y1, z1), T(x1, y1, z1), fx);
#undef T
  return lerpf_(lerpf_(c00, c10, fy), lerpf_(c01, c11, fy), fz) * INV255;
}

/* slab tile k of level L */
static float slab_tile(const orc_slab *sl, int L, uint32_t k, float u, float v, float w) {
  uint32_t tw = sl->lev[L][2] + 2u, th = sl->lev[L][3] + 2u, wz = sl->wz;
  return tex_wrapz(sl->tiles[L] + (size_t)k * tw * th * wz, tw, th, wz, u, v, w);
}

/* vol_sample of the tiled slab (raycast.slang:423-455) */
static float slab_sample(const orc_slab *sl, v3f p, float lod) {
  float nx = (float)sl->nx, ny = (float)sl->ny, px = (float)sl->lev[0][2],
        py = (float)sl->lev[0][3];
  float wx = p.x * nx, wy = p.y * nx;
  float zc = ((float)sl->z0 + 0.5f) + p.z * nx;
  float zq = zc / (float)sl->wz;
  float w = zq - floorf(zq);
  int lev = (int)floorf(lod) - 2;
  if (lev >= 0) {
    int nl = (int)(r3d_log2f((float)sl->ovs) + 0.5f) - 1;
    if (lev > nl - 1) lev = nl - 1;
    float sc = (float)(4 << lev);
    float vnx = ceilf(nx / sc), vny = ceilf(ny / sc);
    float gxl = ceilf(vnx / 2046.0f), gyl = ceilf(vny / 2046.0f);
    float pxl = ceilf(vnx / gxl), pyl = ceilf(vny / gyl);
    float wxl = wx / sc, wyl = wy / sc;
    float oix = fminf(floorf(fmaxf(wxl, 0.0f) / pxl), gxl - 1.0f);
    float oiy = fminf(floorf(fmaxf(wyl, 0.0f) / pyl), gyl - 1.0f);
    float ou = ((wxl - oix * pxl) + 1.0f) / (pxl + 2.0f);
    float ov = ((wyl - oiy * pyl) + 1.0f) / (pyl + 2.0f);
    return slab_tile(sl, lev + 1, (uint32_t)(oiy * gxl + oix), ou, ov, w);
  }
  uint32_t gx = sl->lev[0][0], gy = sl->lev[0][1];
  uint32_t ix = (uint32_t)(fmaxf(wx, 0.0f) / px), iy = (uint32_t)(fmaxf(wy, 0.0f) / py);
  if (ix > gx - 1u) ix = gx - 1u;
  if (iy > gy - 1u) iy = gy - 1u;
  float u = ((wx - (float)ix * px) + 1.0f) / (px + 2.0f);
  float v = ((wy - (float)iy * py) + 1.0f) / (py + 2.0f);
  return slab_tile(sl, 0, iy * gx + ix, u, v, w);
}

/* vs_sample, :331-367: the base cell under p must be the one its tile
 * holds, with the sample's slice span; then the pyramid level matching the
 * footprint (stepping down past absent levels) or the base tile.  Cells
 * convert through int for the key. */
static float vs_sample(const orc_vslab *v, const r3d_frame_params *pc, v3f p, float lod) {
  float P = pc->slab_px, T = P + 2.0f;
  uint32_t Tu = v->px + 2u;
  size_t tb = (size_t)Tu * Tu * v->wz;
  float wx = pc->slab_x0 + p.x * pc->slab_nx;
  float wy = pc->slab_y0 + p.y * pc->slab_nx;
  float zc = (pc->slab_z0 + 0.5f) + p.z * pc->slab_nx;
  float zq = zc / (float)pc->slab_wz, w = zq - floorf(zq);
  float gx0 = (float)(pc->slab_grid & 63u), gy0 = (float)((pc->slab_grid >> 6) & 63u);
  float cbx = floorf(wx / P), cby = floorf(wy / P);
  float pbx = cbx - floorf(cbx / gx0) * gx0, pby = cby - floorf(cby / gy0) * gy0;
  uint32_t want = ((uint32_t)(int32_t)cbx & 1023u) | (((uint32_t)(int32_t)cby & 1023u) << 10) |
                  0x80000000u;
  uint32_t s4 = (uint32_t)(pby * gx0 + pbx) * 4u;
  if (v->table[s4] != want) return 0.0f;
  if (zc - 0.5f < (float)v->table[s4 + 1] || zc + 0.5f > (float)v->table[s4 + 2]) return 0.0f;
  int lev = (int)floorf(lod) - 2;
  if (lev > 3) lev = 3;
  while (lev >= 0 && ((pc->brick_mode >> (8u * (uint32_t)lev)) & 0xffu) == 0u) lev--;
  if (lev < 0) {
    float lx = (wx - cbx * P) + 1.0f, ly = (wy - cby * P) + 1.0f;
    return tex_wrapz(v->tiles + (size_t)(s4 / 4u) * tb, Tu, Tu, v->wz, lx / T, ly / T, w);
  }
  float sc = (float)(4 << lev);
  uint32_t gp = pc->brick_mode >> (8u * (uint32_t)lev);
  float gxl = (float)(gp & 15u), gyl = (float)((gp >> 4) & 15u);
  uint32_t bse = (pc->slab_grid & 63u) * ((pc->slab_grid >> 6) & 63u);
  for (int k = 0; k < lev; k++) {
    uint32_t gk = pc->brick_mode >> (8u * (uint32_t)k);
    bse += (gk & 15u) * ((gk >> 4) & 15u);
  }
  float tx = wx / sc, ty = wy / sc;
  float cx = floorf(tx / P), cy = floorf(ty / P);
  float qx = cx - floorf(cx / gxl) * gxl, qy = cy - floorf(cy / gyl) * gyl;
  float lx = (tx - cx * P) + 1.0f, ly = (ty - cy * P) + 1.0f;
  uint32_t k = bse + (uint32_t)(qy * gxl + qx);
  return tex_wrapz(v->tiles + (size_t)k * tb, Tu, Tu, v->wz, lx / T, ly / T, w);
}

/* sample_clip_level, :360-376 */
static float clip_level(const orc_clip *cl, int l, v3f p) {
  float s = (float)(1u << l), nx = (float)cl->nx;
  float wx = p.x * nx, wy = p.y * nx;
  float zw = ((float)cl->z0 + 0.5f) + p.z * nx;
  float u = ((wx - cl->ox[l]) / s + 1.0f) / 2048.0f;
  float v = ((wy - cl->oy[l]) / s + 1.0f) / 2048.0f;
  float zq = (zw / s) / (float)cl->wzl[l];
  return tex_wrapz(cl->lev[l], 2048u, 2048u, cl->wzl[l], u, v, zq - floorf(zq));
}

/* pick_clip_level, :380-395 */
static int clip_pick(const orc_clip *cl, v3f p, float lod) {
  float nx = (float)cl->nx, wx = p.x * nx, wy = p.y * nx;
  int desired = (int)clampf_(lod, 0.0f, 5.0f);
  for (int step = 0; step < 6; step++) {
    int li = desired + step;
    if (li > 5) li = 5 - step;
    if (li < 0) continue;
    if (!(cl->valid & (1u << li))) continue;
    float s = (float)(1u << li);
    float tx = (wx - cl->ox[li]) / s + 1.0f, ty = (wy - cl->oy[li]) / s + 1.0f;
    if (tx < 1.0f || tx >= 2047.0f || ty < 1.0f || ty >= 2047.0f) continue;
    return li;
  }
  return -1;
}

/* a gradient tap by sampling path: the slab's vol_sample; clip mode's
 * picked level (or vol_sample without one, :942-946,967-974); the virtual
 * slab's vol_sample; else a cube-like texture */
enum { TAP_TEX, TAP_SLAB, TAP_CLIP, TAP_VSLAB };
static float tap_sample(const scene *s, int kind, const orc_cube *tex, v3f p, float lod,
                        int cl_l) {
  switch (kind) {
    case TAP_SLAB: return slab_sample(s->br->slab, p, lod);
    case TAP_VSLAB: return vs_sample(s->br->vslab, s->pc, p, lod);
    case TAP_CLIP:
      if (cl_l >= 0) return clip_level(s->br->clip, cl_l, p);
      cl_l = clip_pick(s->br->clip, p, lod);
      return cl_l < 0 ? 0.0f : clip_level(s->br->clip, cl_l, p);
    default: return cube_sample(tex, p, lod);
  }
}

/* ------------------------------------------------------------ the march */

typedef struct ray_out {
  float rgb[3];
  uint32_t steps;
  uint32_t mip_index;
  int store; /* 0: pixel outside the viewport */
} ray_out;

/* ------------------------------------------------- flattened segment */

/* GLSL mix(x, y, a) = x (1 - a) + y a */
static inline float mixf_(float x, float y, float a) { return fmaf(y, a, x * (1.0f - a)); }

/* bricks_sample_c, surfvol.comp:54-96, with its per-column brick cache */
typedef struct surf_cache {
  int valid;
  uint32_t scale, bc[3], slot;
} surf_cache;

static void surf_brick_sample(const scene *s, uint32_t lod, int ovl, v3f wp, v3f shape,
                              surf_cache *c, float out[2]) {
  float bv[3] = {clampf_(wp.x, 0.0f, fmaxf(shape.x - 0.001f, 0.0f)),
                 clampf_(wp.y, 0.0f, fmaxf(shape.y - 0.001f, 0.0f)),
                 clampf_(wp.z, 0.0f, fmaxf(shape.z - 0.001f, 0.0f))};
  uint32_t nlev = page_rd(s, 0);
  if (c->valid) {
    float lv[3];
    uint32_t bc[3];
    for (int a = 0; a < 3; a++) lv[a] = bv[a] / (float)c->scale, bc[a] = (uint32_t)lv[a] >> 7;
    if (bc[0] == c->bc[0] && bc[1] == c->bc[1] && bc[2] == c->bc[2]) {
      v3f bl = mk3(lv[0] - (float)(bc[0] << 7), lv[1] - (float)(bc[1] << 7), lv[2] - (float)(bc[2] << 7));
      out[0] = brick_fetch(s, c->slot, bl);
      out[1] = ovl >= 0 ? ovl_fetch(s, ovl, c->slot, bl) : 0.0f;
      return;
    }
  }
  int desired = (int)(lod < nlev - 1u ? lod : nlev - 1u), last = (int)nlev - 1;
  for (int stp = 0; stp < 4; stp++) {
    int li = stp < 3 ? desired + stp : last;
    if (li > last || (stp == 3 && li <= desired + 2)) continue;
    uint32_t h = 4u + (uint32_t)li * 4u;
    uint32_t off = page_rd(s, h), packed = page_rd(s, h + 1u), scale = page_rd(s, h + 2u);
    uint32_t bd[3] = {packed & 1023u, (packed >> 10) & 1023u, packed >> 20};
    float lv[3];
    uint32_t bc[3];
    for (int a = 0; a < 3; a++) {
      lv[a] = bv[a] / (float)scale;
      bc[a] = (uint32_t)lv[a] >> 7;
      if (bc[a] > bd[a] - 1u) bc[a] = bd[a] - 1u;
    }
    uint32_t e = page_rd(s, off + (bc[2] * bd[1] + bc[1]) * bd[0] + bc[0]);
    if (e == 0xFFFFFFFFu) continue;
    c->valid = 1;
    c->scale = scale;
    memcpy(c->bc, bc, sizeof bc);
    c->slot = e & 0xFFFFFFu;
    v3f bl = mk3(lv[0] - (float)(bc[0] << 7), lv[1] - (float)(bc[1] << 7), lv[2] - (float)(bc[2] << 7));
    out[0] = brick_fetch(s, c->slot, bl);
    out[1] = ovl >= 0 ? ovl_fetch(s, ovl, c->slot, bl) : 0.0f;
    return;
  }
  c->valid = 0;
  out[0] = out[1] = 0.0f;
}

/* the prediction texture, clamp-to-edge bilinear at texel-space position
 * (px, py) sampled as textureLod(inkpred, (pp + 0.5) / size) */
static float pred_sample(const orc_surf *sf, float px, float py) {
  float u = (px + 0.5f) / (float)sf->pw, v = (py + 0.5f) / (float)sf->ph;
  float tx = clampf_(fmaf(u, (float)sf->pw, -0.5f), 0.0f, (float)(sf->pw - 1u));
  float ty = clampf_(fmaf(v, (float)sf->ph, -0.5f), 0.0f, (float)(sf->ph - 1u));
  uint32_t x0 = (uint32_t)tx, y0 = (uint32_t)ty;
  uint32_t x1 = x0 + 1u < sf->pw ? x0 + 1u : sf->pw - 1u, y1 = y0 + 1u < sf->ph ? y0 + 1u : sf->ph - 1u;
  float fx = tx - (float)x0, fy = ty - (float)y0;
  const float *r0 = sf->pred + (size_t)y0 * sf->pw, *r1 = sf->pred + (size_t)y1 * sf->pw;
  return lerpf_(lerpf_(r0[x0], r0[x1], fx), lerpf_(r1[x0], r1[x1], fx), fy);
}

void orc_surf_bake(orc_surf *sf, const orc_bricks *br, float u0, float v0, float step,
                   float zoff0, float sx, float sy, uint32_t nback, int ovl) {
  uint32_t st = 0;
  scene s = {NULL, br, &st, NULL};
  uint32_t nlev = br->page[0], lod = 0;
  for (float sc = step; sc >= 2.0f && lod + 1u < nlev; sc *= 0.5f) lod++; /* vkbackend.c:7013 */
  v3f shape = mk3((float)br->page[1], (float)br->page[2], (float)br->page[3]);
  const uint32_t gw = sf->gw, gh = sf->gh;
#pragma omp parallel for schedule(dynamic, 4)
  for (uint32_t y = 0; y < sf->H; y++)
    for (uint32_t x = 0; x < sf->W; x++) {
      float fu = fmaf((float)x + 0.5f, step, u0), fv = fmaf((float)y + 0.5f, step, v0);
      float gx = fu * sx, gy = fv * sy;
      int ok = 0;
      v3f wp0 = mk3(0, 0, 0), nrm = mk3(0, 0, 0);
      if (gx >= 0.0f && gy >= 0.0f && gx <= (float)(gw - 1u) && gy <= (float)(gh - 1u)) {
        uint32_t ix = (uint32_t)gx, iy = (uint32_t)gy;
        if (ix > gw - 2u) ix = gw - 2u;
        if (iy > gh - 2u) iy = gh - 2u;
        float fx = gx - (float)ix, fy = gy - (float)iy;
        const float *c00 = sf->coords + 4u * ((size_t)iy * gw + ix), *c10 = c00 + 4,
                    *c01 = c00 + 4u * gw, *c11 = c01 + 4;
        if (fminf(fminf(c00[3], c10[3]), fminf(c01[3], c11[3])) >= 0.5f) {
          const float *n00 = sf->normals + 4u * ((size_t)iy * gw + ix), *n10 = n00 + 4,
                      *n01 = n00 + 4u * gw, *n11 = n01 + 4;
          float w[3], n[3];
          for (int a = 0; a < 3; a++) {
            w[a] = mixf_(mixf_(c00[a], c10[a], fx), mixf_(c01[a], c11[a], fx), fy);
            n[a] = mixf_(mixf_(n00[a], n10[a], fx), mixf_(n01[a], n11[a], fx), fy);
          }
          wp0 = mk3(w[0], w[1], w[2]);
          nrm = mk3(n[0], n[1], n[2]);
          float nl = sqrtf(dot3(nrm, nrm));
          if (nl > 1e-4f) {
            nrm = mk3(nrm.x / nl, nrm.y / nl, nrm.z / nl);
            ok = 1;
          }
        }
      }
      /* one prediction per column, over every layer (surfvol.comp:127-150) */
      float pred = -1.0f;
      if (sf->pred) {
        float px = (gx - sf->pg0u) * sf->pppg, py = (gy - sf->pg0v) * sf->pppg;
        if (px >= 0.0f && py >= 0.0f && px < (float)sf->pw && py < (float)sf->ph)
          pred = pred_sample(sf, px, py);
      }
      surf_cache c = {0, 1u, {0, 0, 0}, 0};
      for (uint32_t z = 0; z < sf->L; z++) {
        float v[2] = {0.0f, 0.0f};
        if (ok) {
          float k = fmaf((float)z - (float)nback, 1.0f, zoff0);
          v3f wp = mk3(fmaf(nrm.x, k, wp0.x), fmaf(nrm.y, k, wp0.y), fmaf(nrm.z, k, wp0.z));
          if (wp.x >= 0.0f && wp.y >= 0.0f && wp.z >= 0.0f && wp.x < shape.x && wp.y < shape.y &&
              wp.z < shape.z)
            surf_brick_sample(&s, lod, ovl, wp, shape, &c, v);
        }
        if (pred >= 0.0f) v[1] = pred;
        uint8_t *o = sf->vol + (((size_t)z * sf->H + y) * sf->W + x) * 2u;
        o[0] = unorm8(v[0]);
        o[1] = unorm8(v[1]);
      }
    }
}

/* the flattened volume, clamp-to-edge trilinear at normalized uvw */
static void surf_tex(const orc_surf *sf, float u, float v, float t, float out[2]) {
  float tx = clampf_(fmaf(u, (float)sf->W, -0.5f), 0.0f, (float)(sf->W - 1u));
  float ty = clampf_(fmaf(v, (float)sf->H, -0.5f), 0.0f, (float)(sf->H - 1u));
  float tz = clampf_(fmaf(t, (float)sf->L, -0.5f), 0.0f, (float)(sf->L - 1u));
  uint32_t x0 = (uint32_t)tx, y0 = (uint32_t)ty, z0 = (uint32_t)tz;
  float fx = tx - (float)x0, fy = ty - (float)y0, fz = tz - (float)z0;
  uint32_t x1 = x0 + 1u < sf->W ? x0 + 1u : sf->W - 1u, y1 = y0 + 1u < sf->H ? y0 + 1u : sf->H - 1u,
           z1 = z0 + 1u < sf->L ? z0 + 1u : sf->L - 1u;
  for (int ch = 0; ch < 2; ch++) {
#define T(X, Y, Z) ((float)sf->vol[(((size_t)(Z) * sf->H + (Y)) * sf->W + (X)) * 2u + ch])
    float a = lerpf_(lerpf_(T(x0, y0, z0), T(x1, y0, z0), fx), lerpf_(T(x0, y1, z0), T(x1, y1, z0), fx), fy);
    float b = lerpf_(lerpf_(T(x0, y0, z1), T(x1, y0, z1), fx), lerpf_(T(x0, y1, z1), T(x1, y1, z1), fx), fy);
#undef T
    out[ch] = lerpf_(a, b, fz) * INV255;
  }
}

/* flat_overlay_color, :76-81 */
static void flat_overlay_color(uint32_t f, float c[3]) {
  float r = 0.25f, g = 1.0f, b = 0.55f;
  if (f & 16u) r = 1.0f, g = 0.25f, b = 1.0f;
  else if (f & 2u) r = 0.25f, g = 1.0f, b = 0.55f;
  else if (f & 4u) r = 1.0f, g = 0.30f, b = 0.22f;
  else if (((f >> 8) & 0xffu) == 1u) r = 0.3f, g = 0.72f, b = 1.0f;
  c[0] = r, c[1] = g, c[2] = b;
}

/* the surf branch of main(), :515-638, for pixel (px, py) */
static void surf_pixel(const r3d_frame_params *pc, const orc_surf *sf, const uint8_t lut[256][4],
                       const orc_opts *o, uint32_t px, uint32_t py, float rgb[3]) {
  const float bg[3] = {0.02f, 0.02f, 0.03f};
  memcpy(rgb, bg, sizeof bg);
  float ux = ((float)px + 0.5f) / (float)pc->viewport[0];
  float uy = ((float)py + 0.5f) / (float)pc->viewport[1];
  float nx = ux * 2.0f - 1.0f, ny = 1.0f - uy * 2.0f;
  float fu = fmaf(ny, pc->cam_up[0], fmaf(nx, pc->cam_right[0], pc->cam_origin[0]));
  float fv = fmaf(ny, pc->cam_up[1], fmaf(nx, pc->cam_right[1], pc->cam_origin[1]));
  float tx = (fu - pc->slab_x0) / pc->slab_px, ty = (fv - pc->slab_y0) / pc->slab_px;
  if (tx < 0.0f || ty < 0.0f || tx >= pc->slab_nx || ty >= pc->slab_ny) return;
  float L = (float)pc->slab_wz;
  float center = (pc->slab_z0 - pc->max_mip) + (float)(pc->slab_grid & 0xffffu);
  float halfd = 0.5f * fmaxf((float)pc->slab_depth, 1.0f);
  float lo = clampf_(center - halfd, 0.0f, L), hi = clampf_(center + halfd, 0.0f, L);
  if (lo >= hi) return;
  float ix = 1.0f / pc->slab_nx, iy = 1.0f / pc->slab_ny, iz = 1.0f / L;
  float vk[2];
  if (pc->view_flags & R3D_VIEW_STRETCH) { /* distortion heatmap, :540-570 */
    float gx = fu * pc->vol_tx, gy = fv * pc->vol_ty;
    int gix = (int)clampf_(gx, 1.0f, (float)sf->gw - 2.0f);
    int giy = (int)clampf_(gy, 1.0f, (float)sf->gh - 2.0f);
    const float *cu0 = sf->coords + 4u * ((size_t)giy * sf->gw + gix - 1);
    const float *cu1 = sf->coords + 4u * ((size_t)giy * sf->gw + gix + 1);
    const float *cv0 = sf->coords + 4u * ((size_t)(giy - 1) * sf->gw + gix);
    const float *cv1 = sf->coords + 4u * ((size_t)(giy + 1) * sf->gw + gix);
    if (fminf(fminf(cu0[3], cu1[3]), fminf(cv0[3], cv1[3])) < 0.5f) return;
    v3f du = mk3(cu1[0] - cu0[0], cu1[1] - cu0[1], cu1[2] - cu0[2]);
    v3f dv = mk3(cv1[0] - cv0[0], cv1[1] - cv0[1], cv1[2] - cv0[2]);
    float su = sqrtf(dot3(du, du)) * 0.5f * pc->vol_tx;
    float sv = sqrtf(dot3(dv, dv)) * 0.5f * pc->vol_ty;
    float x = clampf_(r3d_log2f(fmaxf(0.5f * (su + sv), 1e-4f)) / 0.35f, -1.0f, 1.0f);
    float m = r3d_powf(fabsf(x), 0.6f);
    float tint[3] = {1.0f, 0.15f, 0.0f};
    if (x < 0.0f) tint[0] = 0.0f, tint[1] = 0.35f, tint[2] = 1.0f;
    surf_tex(sf, tx * ix, ty * iy, clampf_(center, lo, hi) * iz, vk);
    float k = fmaf(0.5f, vk[0], 0.5f);
    for (int c = 0; c < 3; c++) rgb[c] = lerpf_(0.95f, tint[c], m) * k;
    return;
  }
  float dt = fmaxf(pc->step_voxels, 0.25f);
  float t = fmaf(hash12(px, py, pc->frame_index), dt, lo);
  float mip_max = 0.0f, ink_max = 0.0f, acc[4] = {0, 0, 0, 0};
  int composite = pc->mode != R3D_MODE_MIP, ovl = (pc->overlay_flags & 1u) != 0u;
  float oc[3];
  flat_overlay_color(pc->overlay_flags, oc);
  float opac_k = pc->density * pc->step_voxels;
  for (uint32_t k = 0; k < 512u && t < hi; k++, t += dt) {
    float u = tx * ix, w = ty * iy, z = t * iz;
    surf_tex(sf, u, w, z, vk);
    float v = vk[0];
    if (ovl && vk[1] > ink_max) ink_max = vk[1];
    if (v < pc->threshold) continue;
    if (v > mip_max) mip_max = v;
    if (!composite) continue;
    float sm[4];
    tf_sample(lut, v, sm);
    float a = 1.0f - r3d_powf(1.0f - sm[3], opac_k);
    if (a <= 0.003f) continue;
    float col[3] = {sm[0], sm[1], sm[2]};
    if (pc->mode == R3D_MODE_FULL) { /* gradients in flattened space */
      float p1[2], m1[2];
      surf_tex(sf, u + ix, w, z, p1), surf_tex(sf, u - ix, w, z, m1);
      float g0 = p1[0] - m1[0];
      surf_tex(sf, u, w + iy, z, p1), surf_tex(sf, u, w - iy, z, m1);
      float g1 = p1[0] - m1[0];
      surf_tex(sf, u, w, z + iz, p1), surf_tex(sf, u, w, z - iz, m1);
      float g2 = p1[0] - m1[0];
      float gm = sqrtf(fmaf(g2, g2, fmaf(g1, g1, g0 * g0)));
      if (gm > 1e-4f) {
        float diff = fmaf(0.7f, fabsf(g2 / gm), 0.3f);
        float lit = fmaf(0.75f, diff, 0.25f);
        float lm = lerpf_(1.0f, lit, satf(gm * 6.0f));
        for (int c = 0; c < 3; c++) col[c] *= lm;
      }
    }
    if (ovl) {
      float kk = satf(vk[1] * pc->overlay_gain);
      for (int c = 0; c < 3; c++) col[c] = lerpf_(col[c], oc[c], kk);
    }
    float wgt = (1.0f - acc[3]) * a;
    for (int c = 0; c < 3; c++) acc[c] = fmaf(wgt, col[c], acc[c]);
    acc[3] = acc[3] + wgt;
    if (acc[3] >= o->alpha_cutoff) break;
  }
  if (composite) {
    float tr = 1.0f - acc[3];
    for (int c = 0; c < 3; c++) rgb[c] = fmaf(tr, bg[c], acc[c]);
  } else {
    float m = mip_max * pc->density;
    float kk = satf(ink_max * pc->overlay_gain);
    for (int c = 0; c < 3; c++) rgb[c] = ovl ? lerpf_(m, oc[c], kk) : m;
  }
  if ((pc->overlay_flags & 32u) && sf->mask) { /* supervision mask, :619-635 */
    float gx = fu * pc->vol_tx, gy = fv * pc->vol_ty;
    float upx = (float)sf->mw / fmaxf((float)sf->gw - 1.0f, 1.0f);
    float upy = (float)sf->mh / fmaxf((float)sf->gh - 1.0f, 1.0f);
    float mxf = gx * upx, myf = gy * upy;
    if (mxf > -1.0f && myf > -1.0f && mxf < (float)sf->mw && myf < (float)sf->mh) {
      uint32_t mc = sf->mask[(size_t)(int)myf * sf->mw + (size_t)(int)mxf];
      const float blue[3] = {0.25f, 0.45f, 1.0f}, orange[3] = {1.0f, 0.55f, 0.10f};
      for (int c = 0; c < 3; c++) {
        if (mc == 1u) rgb[c] = lerpf_(rgb[c], blue[c], 0.45f);
        else if (mc >= 2u) rgb[c] = lerpf_(rgb[c], orange[c], 0.55f);
      }
    }
  }
}

/* main(), :505-1038, for one dispatch thread (tx, ty) of the view */
static void march(const r3d_frame_params *pc, const scene *s, const uint8_t lut[256][4],
                  const orc_opts *o, uint32_t tx, uint32_t ty, ray_out *out) {
  int half = (pc->view_flags & R3D_VIEW_HALF) != 0u;
  uint32_t px = half ? tx * 2u : tx, py = half ? ty * 2u : ty;
  out->steps = 0;
  out->mip_index = 0;
  out->store = 0;
  if (px >= pc->viewport[0] || py >= pc->viewport[1]) return;
  out->store = 1;
  if (pc->view_flags & R3D_VIEW_SURF) {
    surf_pixel(pc, s->br->surf, lut, o, px, py, out->rgb);
    return;
  }
  int ortho = (pc->view_flags & R3D_VIEW_ORTHO) != 0u;
  int vslab = pc->clip_valid == 0u && (pc->slab_grid & (1u << 24)) != 0u;
  int bricks = !vslab && pc->brick_mode != 0u; /* a virtual slab's brick_mode packs its grids */
  int lodb = bricks && (pc->brick_mode & R3D_BRICK_LOD_FLAG) != 0u;
  int clip = pc->clip_valid != 0u;
  int slab = !clip && !vslab && pc->slab_grid != 0u;
  int tk = clip ? TAP_CLIP : vslab ? TAP_VSLAB : slab ? TAP_SLAB : TAP_TEX;
  int shard = bricks && !lodb && !slab && !clip;
  uint32_t sh_bpa = pc->brick_mode & 0xffu, sh_abpa = (pc->brick_mode >> 8) & 0xffu;
  int sh_ident = (pc->brick_mode & R3D_BRICK_IDENTITY_FLAG) != 0u;
  const orc_cube *atlas = shard ? s->br->atlas : NULL;

  /* pix_ndc / ray_dir / ray_origin, :469-486 */
  float ux = ((float)px + 0.5f) / (float)pc->viewport[0];
  float uy = ((float)py + 0.5f) / (float)pc->viewport[1];
  float nx = ux * 2.0f - 1.0f, ny = 1.0f - uy * 2.0f;
  v3f fwd = mk3(pc->cam_forward[0], pc->cam_forward[1], pc->cam_forward[2]);
  v3f rt = mk3(pc->cam_right[0], pc->cam_right[1], pc->cam_right[2]);
  v3f up = mk3(pc->cam_up[0], pc->cam_up[1], pc->cam_up[2]);
  v3f dir;
  if (ortho)
    dir = norm3(fwd);
  else
    dir = norm3(mk3(fmaf(ny, up.x, fmaf(nx, rt.x, fwd.x)), fmaf(ny, up.y, fmaf(nx, rt.y, fwd.y)),
                    fmaf(ny, up.z, fmaf(nx, rt.z, fwd.z))));
  if (pc->mode == R3D_MODE_RAYDIR) {
    out->rgb[0] = fmaf(dir.x, 0.5f, 0.5f);
    out->rgb[1] = fmaf(dir.y, 0.5f, 0.5f);
    out->rgb[2] = fmaf(dir.z, 0.5f, 0.5f);
    return;
  }
  v3f org = mk3(pc->cam_origin[0], pc->cam_origin[1], pc->cam_origin[2]);
  if (ortho)
    org = mk3(fmaf(ny, up.x, fmaf(nx, rt.x, org.x)), fmaf(ny, up.y, fmaf(nx, rt.y, org.y)),
              fmaf(ny, up.z, fmaf(nx, rt.z, org.z)));

  /* voxel pitch, LOD ceiling, extent (:647-683, :305-314); the ray-cone
   * footprint is measured in voxels by multiplying with vox_inv = 1/voxel */
  float voxel, vox_inv, max_lod;
  v3f ext = mk3(1.0f, 1.0f, 1.0f);
  uint32_t nlev = 0;
  float md = 0.0f; /* bricks: largest base dimension */
  if (lodb) {
    nlev = page_rd(s, 0);
    float bs[3] = {(float)page_rd(s, 1), (float)page_rd(s, 2), (float)page_rd(s, 3)};
    md = fmaxf(bs[0], fmaxf(bs[1], bs[2]));
    voxel = 1.0f / md;
    vox_inv = md;
    max_lod = (float)(nlev - 1u);
    ext = mk3(bs[0] / md, bs[1] / md, bs[2] / md);
  } else if (vslab) { /* :661-671, :305-314 */
    voxel = 1.0f / pc->slab_nx;
    vox_inv = pc->slab_nx;
    max_lod = 3.0f; /* +2 past the coarsest present pyramid level */
    for (int l = 3; l >= 0; l--)
      if (((pc->brick_mode >> (8u * (uint32_t)l)) & 0xffu) != 0u) {
        max_lod = (float)l + 4.0f;
        break;
      }
    ext = mk3(1.0f, pc->slab_ny / pc->slab_nx, (float)pc->slab_depth / pc->slab_nx);
  } else if (clip) { /* :651-654, :305-314 */
    voxel = 1.0f / pc->slab_nx;
    vox_inv = pc->slab_nx;
    max_lod = 7.0f;
    ext = mk3(1.0f, pc->slab_ny / pc->slab_nx, (float)pc->slab_depth / pc->slab_nx);
  } else if (slab) { /* :672-677, :305-314 */
    const orc_slab *sl = s->br->slab;
    voxel = 1.0f / pc->slab_nx;
    vox_inv = pc->slab_nx;
    max_lod = r3d_log2f((float)((pc->slab_grid >> 16) & 0xffu)) + 2.0f;
    ext = mk3(1.0f, pc->slab_ny / pc->slab_nx, (float)pc->slab_depth / pc->slab_nx);
    (void)sl;
  } else if (shard) { /* :659-661 */
    voxel = 1.0f / (float)(sh_bpa * 128u);
    vox_inv = (float)(sh_bpa * 128u);
    max_lod = 3.0f;
  } else {
    const uint32_t *d = s->cube->dim[0];
    uint32_t cm = d[0] > d[1] ? d[0] : d[1];
    if (d[2] > cm) cm = d[2];
    voxel = 1.0f / (float)cm;
    vox_inv = (float)cm;
    max_lod = fminf(pc->max_mip, (float)(s->cube->nlevels - 1u));
  }
  /* model transform, common.slang:45-52 */
  v3f c = mk3(ext.x * 0.5f, ext.y * 0.5f, ext.z * 0.5f);
  v3f r0 = mk3(pc->vol_r0[0], pc->vol_r0[1], pc->vol_r0[2]);
  v3f r1 = mk3(pc->vol_r1[0], pc->vol_r1[1], pc->vol_r1[2]);
  v3f r2 = mk3(pc->vol_r2[0], pc->vol_r2[1], pc->vol_r2[2]);
  v3f q = mk3((org.x - pc->vol_tx) - c.x, (org.y - pc->vol_ty) - c.y, (org.z - pc->vol_tz) - c.z);
  v3f ro = mk3(fmaf(r2.x, q.z, fmaf(r1.x, q.y, r0.x * q.x)) + c.x,
               fmaf(r2.y, q.z, fmaf(r1.y, q.y, r0.y * q.x)) + c.y,
               fmaf(r2.z, q.z, fmaf(r1.z, q.y, r0.z * q.x)) + c.z);
  dir = mk3(fmaf(r2.x, dir.z, fmaf(r1.x, dir.y, r0.x * dir.x)),
            fmaf(r2.y, dir.z, fmaf(r1.y, dir.y, r0.y * dir.x)),
            fmaf(r2.z, dir.z, fmaf(r1.z, dir.y, r0.z * dir.x)));

  /* clip boxes and t range, :686-714 */
  float lo[3] = {0.0f, 0.0f, 0.0f}, hi[3] = {ext.x, ext.y, ext.z};
  float t_lo = 0.0f, t_hi = 1e30f;
  if (lodb && (pc->view_flags & R3D_VIEW_CROP) != 0u) {
    float clo[3] = {pc->slab_x0 / md, pc->slab_y0 / md, pc->slab_z0 / md};
    float cx[3] = {pc->slab_px / md, pc->slab_py / md, pc->slab_nx / md};
    for (int a = 0; a < 3; a++) {
      lo[a] = clampf_(clo[a], 0.0f, hi[a]);
      hi[a] = clampf_(clo[a] + cx[a], lo[a], hi[a]);
    }
  } else if (lodb && pc->slab_depth > 0u) {
    if ((pc->view_flags & R3D_VIEW_OBLIQUE) != 0u) {
      t_lo = pc->slab_z0 / md;
      t_hi = (pc->slab_z0 + (float)pc->slab_depth) / md;
    } else {
      uint32_t axc = (pc->view_flags >> 8) & 3u;
      int a = axc == 1u ? 0 : (axc == 2u ? 1 : 2);
      float e = hi[a];
      lo[a] = clampf_(pc->slab_z0 / md, 0.0f, e);
      hi[a] = clampf_((pc->slab_z0 + (float)pc->slab_depth) / md, lo[a], e);
    }
  }
  /* box_hit, :489-495 */
  float dv[3] = {dir.x, dir.y, dir.z}, ov[3] = {ro.x, ro.y, ro.z};
  float tmn[3], tmx[3];
  for (int a = 0; a < 3; a++) {
    float inv = 1.0f / dv[a];
    float t0 = (lo[a] - ov[a]) * inv, t1 = (hi[a] - ov[a]) * inv;
    tmn[a] = fminf(t0, t1);
    tmx[a] = fmaxf(t0, t1);
  }
  float hx = fmaxf(fmaxf(tmn[0], tmn[1]), tmn[2]);
  float hy = fminf(fminf(tmx[0], tmx[1]), tmx[2]);
  float tn = fmaxf(hx, t_lo), tf_ = fminf(hy, t_hi);
  if (tn >= tf_) {
    out->rgb[0] = BG_R;
    out->rgb[1] = BG_G;
    out->rgb[2] = BG_B;
    return;
  }

  /* cone, step, jitter, budget, gates (:722-762) */
  float cone = (2.0f * sqrtf(dot3(up, up))) / (float)pc->viewport[1];
  float dt = pc->step_voxels * voxel;
  float jitter = hash12(px, py, pc->frame_index);
  float t = fmaf(jitter, dt, tn);
  float mip_max = 0.0f, first_hit = -1.0f;
  float acc[4] = {0, 0, 0, 0};
  uint32_t steps = 0, mip_index = 0;
  int composite = pc->mode == R3D_MODE_FULL || pc->mode == R3D_MODE_FLAT;
  /* overlays (:45-49,67-73) */
  uint32_t ovl = lodb ? pc->overlay_flags & 0x1Du : 0u;
  float reg_alpha = (float)((pc->overlay_flags >> 16) & 0xffu) * (1.0f / 255.0f);
  int pal1 = ((pc->overlay_flags >> 8) & 0xffu) == 1u;
  float ovl_col[3] = {pal1 ? 0.3f : 0.25f, pal1 ? 0.72f : 1.0f, pal1 ? 1.0f : 0.55f};
  float ink_max = 0.0f, ink2_max = 0.0f, lbl_max = 0.0f, reg_max = 0.0f;
  int shaded = pc->mode == R3D_MODE_FULL;
  uint32_t ray_budget = lodb ? (shaded ? 192u : 256u) : MAX_STEPS;
  float span_step = fmaxf((tf_ - tn) / ((float)ray_budget * dt), 1.0f);
  float slab_cap = fmaxf(1.0f, (tf_ - tn) / (4.0f * dt)); /* :778-779 */
  float bs = OCC_BLOCK * voxel;
  float occ_gate = fmaxf(pc->skip_gate, 0.5f / 255.0f);
  float opac_k = pc->density * pc->step_voxels;

  /* shading constants (:988-998): key light, headlight l = -dir and its
   * half vector normalize(l - dir) are per-ray constants */
  v3f key = norm3(mk3(0.4f, 0.8f, -0.4f));
  v3f l = mk3(-dir.x, -dir.y, -dir.z);
  v3f hv = norm3(mk3(l.x - dir.x, l.y - dir.y, l.z - dir.z));

  lod_cache lc;
  memset(&lc, 0, sizeof lc);
  lc.valid = 0;
  lc.desired = -1;
  lc.scale = 1u;
  lc.bc[0] = lc.bc[1] = lc.bc[2] = 0u;
  brick_ctx b;
  memset(&b, 0, sizeof b);
  b.world_brick = 128.0f * voxel;
  /* single-level page cache (:752-760) */
  uint32_t b_last = 0xFFFFFFFFu;
  float sh_n = (float)(sh_bpa * 128u);
  float sh_inv = 1.0f / ((float)sh_abpa * 128.0f);
  v3f sh_org = mk3(0.0f, 0.0f, 0.0f);

  while (t < tf_ && steps < ray_budget) {
    steps++;
    /* LOD and step (:772-779) */
    float foot = ortho ? cone : t * cone;
    float lod = clampf_(r3d_log2f(fmaxf(foot * vox_inv, 1.0f)) + pc->lod_bias, 0.0f, max_lod);
    float lod_step = fmaxf(r3d_exp2f(lod), span_step);
    if (slab || clip || vslab) lod_step = fminf(lod_step, slab_cap);
    v3f p = mk3(fmaf(t, dir.x, ro.x), fmaf(t, dir.y, ro.y), fmaf(t, dir.z, ro.z));

    float v;
    int cl_lvl = -1; /* clip: the level picked once per sample (:782) */
    if (lodb) {
      b = lod_locate_cached(s, p, lod, &lc);
      v = b.ok ? brick_fetch(s, b.slot, b.bl) : 0.0f;
    } else if (clip) { /* :785-787 */
      cl_lvl = clip_pick(s->br->clip, p, lod);
      v = cl_lvl < 0 ? 0.0f : clip_level(s->br->clip, cl_lvl, p);
    } else if (slab) {
      v = slab_sample(s->br->slab, p, lod);
    } else if (vslab) {
      v = vs_sample(s->br->vslab, pc, p, lod);
    } else if (shard && sh_ident) { /* :800-805 */
      v = cube_sample(atlas, p, lod);
    } else if (shard) { /* :806-822 */
      float vp[3] = {satf(p.x) * sh_n, satf(p.y) * sh_n, satf(p.z) * sh_n};
      uint32_t bc[3];
      for (int a = 0; a < 3; a++) {
        bc[a] = (uint32_t)vp[a] >> 7;
        if (bc[a] > sh_bpa - 1u) bc[a] = sh_bpa - 1u;
      }
      uint32_t bi = (bc[2] * sh_bpa + bc[1]) * sh_bpa + bc[0];
      if (bi != b_last) {
        b_last = bi;
        uint32_t e = page_rd(s, bi);
        b.ok = e != 0xFFFFFFFFu;
        b.slot = e & 0xFFFFFFu;
        if (b.ok && b.slot >= sh_abpa * sh_abpa * sh_abpa) {
          *s->status |= 1u;
          b.ok = 0;
        }
        b.maxv = b.ok ? (float)(e >> 24) / 255.0f : 0.0f;
        sh_org = mk3((float)(b.slot % sh_abpa) * 128.0f, (float)((b.slot / sh_abpa) % sh_abpa) * 128.0f,
                     (float)(b.slot / (sh_abpa * sh_abpa)) * 128.0f);
      }
      b.bl = mk3(vp[0] - (float)(bc[0] << 7), vp[1] - (float)(bc[1] << 7),
                 vp[2] - (float)(bc[2] << 7));
      v = b.ok ? shard_fetch(atlas, sh_inv, sh_org, b.bl, lod) : 0.0f;
    } else {
      v = cube_sample(s->cube, p, lod);
    }
    int cut = v < pc->threshold; /* :826-827 */
    if (cut) v = 0.0f;

    /* empty-space skip (:829-869) */
    int void_blk = 0;
    float bsz = bs;
    if (lodb) {
      float bgate = fmaxf(occ_gate, 4.5f / 255.0f);
      if (pc->mode == R3D_MODE_MIP && !ovl && b.ok && b.maxv <= mip_max) {
        void_blk = 1;
        bsz = b.world_brick;
      } else if (v < bgate && b.maxv < bgate) {
        void_blk = 1;
        bsz = b.world_brick;
      }
    } else if (shard) { /* :848-860 */
      float bgate = fmaxf(occ_gate, 4.5f / 255.0f);
      if (v < bgate) {
        if (sh_ident) {
          if (occ_sample(atlas->occ, atlas->odim, p) < bgate) void_blk = 1;
        } else if (b.maxv < bgate) {
          void_blk = 1;
          bsz = 128.0f * voxel;
        } else if (occ_sample(atlas->occ, atlas->odim, p) < bgate) {
          void_blk = 1;
        }
      }
    } else if (!slab && !clip && !vslab && v < occ_gate &&
               occ_sample(s->cube->occ, s->cube->odim, p) < occ_gate) {
      void_blk = 1;
    }
    if (void_blk) {
      float pv[3] = {p.x, p.y, p.z};
      float tex[3];
      for (int a = 0; a < 3; a++) {
        float nextp = (floorf(pv[a] / bsz) + (dv[a] > 0.0f ? 1.0f : 0.0f)) * bsz;
        tex[a] = fabsf(dv[a]) > 1e-8f ? (nextp - ov[a]) / dv[a] : 1e30f;
      }
      t = fmaxf(fminf(fminf(tex[0], tex[1]), tex[2]), t) + bsz * 0.01f;
      continue;
    }

    if (v > mip_max) { /* :871 */
      mip_max = v;
      mip_index = steps;
    }
    if (ovl && pc->mode == R3D_MODE_MIP && b.ok) { /* :872-887 */
      float k;
      if ((ovl & 1u) && (k = ovl_fetch(s, 0, b.slot, b.bl)) > ink_max) ink_max = k;
      if ((ovl & 4u) && (k = ovl_fetch(s, 1, b.slot, b.bl)) > ink2_max) ink2_max = k;
      if ((ovl & 8u) && (k = ovl_fetch(s, 2, b.slot, b.bl)) > lbl_max) lbl_max = k;
      if (ovl & 16u) {
        k = ovl_fetch(s, 3, b.slot, b.bl);
        if (k < pc->threshold) k = 0.0f;
        if (k > reg_max) reg_max = k;
      }
    }
    if (pc->mode == R3D_MODE_MIP && !ovl && mip_max >= 0.999f) break; /* :888 */
    if (first_hit < 0.0f && v > 0.05f) first_hit = t;         /* :891 */

    if (composite && !cut) {
      float sm[4], rs[4] = {0, 0, 0, 0};
      tf_sample(lut, v, sm);
      int reg_live = (ovl & 16u) && b.ok;
      if (reg_live) { /* the moving scan through the same TF (:895-905) */
        float rv = ovl_fetch(s, 3, b.slot, b.bl);
        if (rv < pc->threshold) rv = 0.0f;
        tf_sample(lut, rv, rs);
        sm[3] = fmaxf(sm[3], rs[3] * reg_alpha);
      }
      /* opacity correction (:906) */
      float a = 1.0f - r3d_powf(1.0f - sm[3], opac_k * lod_step);
      if (a > 0.003f) {
        float col[3] = {sm[0], sm[1], sm[2]};
        if (reg_live) { /* green/magenta fuse before shading (:910-914) */
          v3f wl = mk3(0.333f, 0.334f, 0.333f);
          float lm = dot3(mk3(rs[0], rs[1], rs[2]), wl);
          float lf = dot3(mk3(col[0], col[1], col[2]), wl);
          lerp3(col, lm, lf, lm, reg_alpha);
        }
        if (shaded) {
          float g[3];
          if (o->quality == R3D_QUALITY_FAST) { /* :919-955 */
            const float ir3 = 0.57735026919f, renorm = 0.86602540378f;
            float q0, q1, q2, q3;
            if (lodb) {
              float ev = b.grad_vox * ir3;
              q0 = brick_fetch(s, b.slot, mk3(b.bl.x + ev, b.bl.y - ev, b.bl.z - ev));
              q1 = brick_fetch(s, b.slot, mk3(b.bl.x - ev, b.bl.y - ev, b.bl.z + ev));
              q2 = brick_fetch(s, b.slot, mk3(b.bl.x - ev, b.bl.y + ev, b.bl.z - ev));
              q3 = brick_fetch(s, b.slot, mk3(b.bl.x + ev, b.bl.y + ev, b.bl.z + ev));
            } else if (shard && !sh_ident) { /* :937-940 */
              float ev = lod_step * ir3;
              v3f u = b.bl;
              q0 = shard_fetch(atlas, sh_inv, sh_org, mk3(u.x + ev, u.y - ev, u.z - ev), lod);
              q1 = shard_fetch(atlas, sh_inv, sh_org, mk3(u.x - ev, u.y - ev, u.z + ev), lod);
              q2 = shard_fetch(atlas, sh_inv, sh_org, mk3(u.x - ev, u.y + ev, u.z - ev), lod);
              q3 = shard_fetch(atlas, sh_inv, sh_org, mk3(u.x + ev, u.y + ev, u.z + ev), lod);
            } else {
              const orc_cube *tex = shard ? atlas : s->cube;
              float ee = (voxel * lod_step) * ir3;
              q0 = tap_sample(s, tk, tex, mk3(p.x + ee, p.y - ee, p.z - ee), lod, cl_lvl);
              q1 = tap_sample(s, tk, tex, mk3(p.x - ee, p.y - ee, p.z + ee), lod, cl_lvl);
              q2 = tap_sample(s, tk, tex, mk3(p.x - ee, p.y + ee, p.z - ee), lod, cl_lvl);
              q3 = tap_sample(s, tk, tex, mk3(p.x + ee, p.y + ee, p.z + ee), lod, cl_lvl);
            }
            g[0] = (((q0 - q1) - q2) + q3) * renorm;
            g[1] = (((-q0 - q1) + q2) + q3) * renorm;
            g[2] = (((-q0 + q1) - q2) + q3) * renorm;
          } else { /* :957-986 */
            if (lodb) {
              float ev = b.grad_vox;
              v3f u = b.bl;
              g[0] = brick_fetch(s, b.slot, mk3(u.x + ev, u.y, u.z)) -
                     brick_fetch(s, b.slot, mk3(u.x - ev, u.y, u.z));
              g[1] = brick_fetch(s, b.slot, mk3(u.x, u.y + ev, u.z)) -
                     brick_fetch(s, b.slot, mk3(u.x, u.y - ev, u.z));
              g[2] = brick_fetch(s, b.slot, mk3(u.x, u.y, u.z + ev)) -
                     brick_fetch(s, b.slot, mk3(u.x, u.y, u.z - ev));
            } else if (shard && !sh_ident) { /* :972-979 */
              float ev = lod_step;
              v3f u = b.bl;
              g[0] = shard_fetch(atlas, sh_inv, sh_org, mk3(u.x + ev, u.y, u.z), lod) -
                     shard_fetch(atlas, sh_inv, sh_org, mk3(u.x - ev, u.y, u.z), lod);
              g[1] = shard_fetch(atlas, sh_inv, sh_org, mk3(u.x, u.y + ev, u.z), lod) -
                     shard_fetch(atlas, sh_inv, sh_org, mk3(u.x, u.y - ev, u.z), lod);
              g[2] = shard_fetch(atlas, sh_inv, sh_org, mk3(u.x, u.y, u.z + ev), lod) -
                     shard_fetch(atlas, sh_inv, sh_org, mk3(u.x, u.y, u.z - ev), lod);
            } else {
              const orc_cube *tex = shard ? atlas : s->cube;
              float e = voxel * lod_step;
              g[0] = tap_sample(s, tk, tex, mk3(p.x + e, p.y, p.z), lod, cl_lvl) -
                     tap_sample(s, tk, tex, mk3(p.x - e, p.y, p.z), lod, cl_lvl);
              g[1] = tap_sample(s, tk, tex, mk3(p.x, p.y + e, p.z), lod, cl_lvl) -
                     tap_sample(s, tk, tex, mk3(p.x, p.y - e, p.z), lod, cl_lvl);
              g[2] = tap_sample(s, tk, tex, mk3(p.x, p.y, p.z + e), lod, cl_lvl) -
                     tap_sample(s, tk, tex, mk3(p.x, p.y, p.z - e), lod, cl_lvl);
            }
          }
          v3f gv = mk3(g[0], g[1], g[2]);
          float gm = sqrtf(dot3(gv, gv));
          if (gm > 1e-4f) { /* :988-998 */
            float inv = 1.0f / gm;
            v3f n = mk3(gv.x * inv, gv.y * inv, gv.z * inv);
            float diff = fmaf(0.3f, fabsf(dot3(n, key)), 0.7f * fabsf(dot3(n, l)));
            float spec = r3d_powi24f(fabsf(dot3(n, hv))) * 0.3f;
            float lit = fmaf(0.75f, diff, 0.25f);
            float w = satf(gm * 6.0f);
            float lm = fmaf(w, lit - 1.0f, 1.0f);
            float sw = spec * w;
            for (int k = 0; k < 3; k++) col[k] = fmaf(col[k], lm, sw);
          }
        }
        if (ovl & 1u) /* tints after shading (:1000-1014) */
          lerp3(col, ovl_col[0], ovl_col[1], ovl_col[2],
                satf(ovl_fetch(s, 0, b.slot, b.bl) * pc->overlay_gain));
        if (ovl & 4u)
          lerp3(col, 1.0f, 0.30f, 0.22f, satf(ovl_fetch(s, 1, b.slot, b.bl) * pc->overlay_gain));
        if (ovl & 8u) {
          float k = ovl_fetch(s, 2, b.slot, b.bl);
          if (k > 0.0f) {
            float lc[3];
            label_color(k, lc);
            lerp3(col, lc[0], lc[1], lc[2], 0.65f);
          }
        }
        /* front-to-back compositing and early termination (:1015-1017) */
        float wgt = (1.0f - acc[3]) * a;
        for (int k = 0; k < 3; k++) acc[k] = fmaf(wgt, col[k], acc[k]);
        acc[3] = acc[3] + wgt;
        if (acc[3] >= o->alpha_cutoff) break;
      }
    }
    t = fmaf(dt, lod_step, t); /* :1020 */
  }

  /* finalize (:1023-1038) */
  out->steps = steps;
  out->mip_index = mip_index;
  if (pc->mode == R3D_MODE_HEATMAP) {
    float x = (float)steps / 1024.0f;
    out->rgb[0] = x;
    out->rgb[1] = 1.0f - fabsf(x - 0.5f) * 2.0f;
    out->rgb[2] = 1.0f - x;
  } else if (pc->mode == R3D_MODE_DEPTH) {
    float d = first_hit < 0.0f ? 0.0f : 1.0f - satf(first_hit * 0.5f);
    out->rgb[0] = out->rgb[1] = out->rgb[2] = d;
  } else if (composite) {
    float tr = 1.0f - acc[3];
    out->rgb[0] = fmaf(tr, BG_R, acc[0]);
    out->rgb[1] = fmaf(tr, BG_G, acc[1]);
    out->rgb[2] = fmaf(tr, BG_B, acc[2]);
  } else {
    float m = mip_max * pc->density;
    float c[3] = {m, m, m};
    if (ovl & 16u) { /* reg_fuse, :113-116 */
      float mr = reg_max * pc->density;
      float lum = dot3(mk3(c[0], c[1], c[2]), mk3(0.333f, 0.334f, 0.333f));
      lerp3(c, mr, lum, mr, reg_alpha);
    }
    if (ovl & 1u) lerp3(c, ovl_col[0], ovl_col[1], ovl_col[2], satf(ink_max * pc->overlay_gain));
    if (ovl & 4u) lerp3(c, 1.0f, 0.30f, 0.22f, satf(ink2_max * pc->overlay_gain));
    if ((ovl & 8u) && lbl_max > 0.0f) {
      float lc[3];
      label_color(lbl_max, lc);
      lerp3(c, lc[0], lc[1], lc[2], 0.65f);
    }
    out->rgb[0] = c[0];
    out->rgb[1] = c[1];
    out->rgb[2] = c[2];
  }
}

static int check_view(const r3d_frame_params *p, const orc_cube *cube, const orc_bricks *br) {
  if (p->view_flags & R3D_VIEW_SURF) { /* flattened segment: the baked window */
    const orc_surf *sf = br ? br->surf : NULL;
    if (!sf || !sf->vol || sf->gw < 3u || sf->gh < 3u || p->slab_nx != (float)sf->W ||
        p->slab_ny != (float)sf->H || p->slab_wz != sf->L || !(p->slab_px > 0.0f) ||
        p->mode >= R3D_MODE_COUNT)
      return -1;
    return 0;
  }
  if ((p->overlay_flags & 0x1Du) &&
      (!(p->brick_mode & R3D_BRICK_LOD_FLAG) || !br || ((p->overlay_flags & 1u) && !br->ovl[0]) ||
       ((p->overlay_flags & 4u) && !br->ovl[1]) || ((p->overlay_flags & 8u) && !br->ovl[2]) ||
       ((p->overlay_flags & 16u) && !br->ovl[3])))
    return -1;
  int vslab = !p->clip_valid && (p->slab_grid & (1u << 24)) != 0u;
  if (vslab) { /* virtual-slab views must describe the loaded grids */
    const orc_vslab *v = br ? br->vslab : NULL;
    uint32_t bm = 0;
    if (v)
      for (int l = 1; l < 5; l++) bm |= (v->gx[l] | (v->gy[l] << 4)) << (8 * (l - 1));
    if (!v || p->slab_grid != (v->gx[0] | (v->gy[0] << 6) | (1u << 24)) || p->brick_mode != bm ||
        p->slab_wz != v->wz || p->slab_px != (float)v->px || p->slab_nx < 1.0f ||
        p->slab_depth < 1u || (p->overlay_flags & 0x1Du))
      return -1;
  }
  if (p->slab_grid && !vslab && !p->clip_valid) { /* slab views: the slab's window */
    const orc_slab *sl = br ? br->slab : NULL;
    if (!sl || p->brick_mode || p->slab_wz != sl->wz || p->slab_z0 != (float)sl->z0 ||
        p->slab_nx != (float)sl->nx || p->slab_ny != (float)sl->ny ||
        p->slab_px != (float)sl->lev[0][2] || p->slab_py != (float)sl->lev[0][3] ||
        p->slab_grid != (sl->lev[0][0] | (sl->lev[0][1] << 8) | (sl->ovs << 16)) ||
        p->slab_depth < 1u || p->slab_depth > sl->wz - 1u)
      return -1;
  }
  if (p->clip_valid) { /* clip views must describe the loaded levels */
    const orc_clip *cl = br ? br->clip : NULL;
    if (!cl || p->clip_valid != cl->valid || p->brick_mode || p->slab_grid ||
        p->slab_nx != (float)cl->nx || p->slab_z0 != (float)cl->z0 ||
        p->slab_wz != cl->wzl[0] - 3u || p->slab_depth < 1u || p->slab_depth > p->slab_wz ||
        (p->overlay_flags & 0x1Du))
      return -1;
    for (int l = 0; l < 6; l++)
      if (p->clip_orig[l][0] != cl->ox[l] || p->clip_orig[l][1] != cl->oy[l]) return -1;
  }
  if (p->mode >= R3D_MODE_COUNT) return -1;
  if (vslab) {
    /* brick_mode packs the pyramid grids (checked above) */
  } else if (p->brick_mode & R3D_BRICK_LOD_FLAG) {
    if (!br || !br->page || br->page_words < 64u) return -1;
    uint32_t nlev = br->page[0];
    if (nlev < 1u || nlev > 15u) return -1;
  } else if (p->brick_mode) { /* single-level atlas */
    uint32_t bpa = p->brick_mode & 0xffu, abpa = (p->brick_mode >> 8) & 0xffu;
    const orc_cube *a = br ? br->atlas : NULL;
    if (!bpa || !abpa || abpa > bpa || !br || !br->page || br->page_words != bpa * bpa * bpa || !a ||
        a->nlevels != 4u || !a->occ)
      return -1;
    for (int k = 0; k < 3; k++)
      if (a->dim[0][k] != abpa * 128u || a->odim[k] != bpa * 16u) return -1;
  } else if (!vslab && !p->slab_grid && !p->clip_valid &&
             (!cube || !cube->nlevels || !cube->occ)) {
    return -1;
  }
  return 0;
}

int orc_render_view(const r3d_frame_params *p, const orc_cube *cube, const orc_bricks *bricks,
                    const uint8_t lut[256][4], const orc_opts *o, uint8_t *img, uint32_t img_w,
                    uint32_t img_h, orc_aux *aux) {
  if (check_view(p, cube, bricks) != 0) return -1;
  uint32_t vw = p->viewport[0], vh = p->viewport[1];
  uint32_t ox = p->view_org & 0xffffu, oy = p->view_org >> 16;
  if (ox + vw > img_w || oy + vh > img_h) return -1;
  int half = (p->view_flags & R3D_VIEW_HALF) != 0u;
  uint32_t gw = half ? (vw + 1u) / 2u : vw, gh = half ? (vh + 1u) / 2u : vh;
  uint64_t total = 0;
  uint32_t status = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) reduction(| : status) \
    num_threads(o->threads > 0 ? o->threads : omp_get_max_threads())
  for (uint32_t ty = 0; ty < gh; ty++) {
    uint32_t st = 0;
    scene s = {cube, bricks, &st, p};
    for (uint32_t tx = 0; tx < gw; tx++) {
      ray_out r;
      march(p, &s, lut, o, tx, ty, &r);
      if (!r.store) continue;
      total += r.steps;
      uint32_t lx = half ? tx * 2u : tx, ly = half ? ty * 2u : ty;
      uint8_t px[4] = {unorm8(r.rgb[0]), unorm8(r.rgb[1]), unorm8(r.rgb[2]), 255};
      for (uint32_t k = 0; k < (half ? 4u : 1u); k++) {
        uint32_t ax = lx + (k & 1u), ay = ly + (k >> 1);
        if (ax >= vw || ay >= vh) continue;
        size_t i = (size_t)(oy + ay) * img_w + (ox + ax);
        memcpy(img + i * 4u, px, 4);
        if (aux && aux->steps) aux->steps[i] = r.steps;
        if (aux && aux->mip_index) aux->mip_index[i] = r.mip_index;
      }
    }
    status |= st;
  }
  if (aux) {
    aux->total_steps = total;
    aux->status = status;
  }
  return 0;
}

int orc_render_pixels(const r3d_frame_params *p, const orc_cube *cube, const orc_bricks *bricks,
                      const uint8_t lut[256][4], const orc_opts *o, const uint32_t *xy,
                      uint32_t n, uint8_t *out_rgba, uint32_t *steps, uint32_t *mip_index) {
  if (check_view(p, cube, bricks) != 0) return -1;
#pragma omp parallel for schedule(dynamic, 16) \
    num_threads(o->threads > 0 ? o->threads : omp_get_max_threads())
  for (uint32_t i = 0; i < n; i++) {
    uint32_t st = 0;
    scene s = {cube, bricks, &st, p};
    ray_out r;
    march(p, &s, lut, o, xy[2 * i], xy[2 * i + 1], &r);
    uint8_t px[4] = {0, 0, 0, 0};
    if (r.store) {
      px[0] = unorm8(r.rgb[0]);
      px[1] = unorm8(r.rgb[1]);
      px[2] = unorm8(r.rgb[2]);
      px[3] = 255;
    }
    memcpy(out_rgba + (size_t)i * 4u, px, 4);
    if (steps) steps[i] = r.steps;
    if (mip_index) mip_index[i] = r.mip_index;
  }
  return 0;
}

/* log2 / exp2 / pow / x^24 of the shared header, for the device bit check */
void orc_fmath_eval(const float *x, const float *y, float *out, uint32_t n) {
  for (uint32_t i = 0; i < n; i++) {
    out[4 * i + 0] = r3d_log2f(x[i]);
    out[4 * i + 1] = r3d_exp2f(x[i]);
    out[4 * i + 2] = r3d_powf(x[i], y[i]);
    out[4 * i + 3] = r3d_powi24f(x[i]);
  }
}

/* ------------------------------------------------------- data builders */

uint32_t orc_mip_levels(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t dims[][3]) {
  uint32_t maxdim = nx > ny ? nx : ny;
  if (nz > maxdim) maxdim = nz;
  uint32_t mips = 1;
  while ((maxdim >> mips) >= 1u && mips < 16u) mips++;
  for (uint32_t m = 0; m < mips; m++) {
    dims[m][0] = nx >> m ? nx >> m : 1u;
    dims[m][1] = ny >> m ? ny >> m : 1u;
    dims[m][2] = nz >> m ? nz >> m : 1u;
  }
  return mips;
}

void orc_downsample(const uint8_t *src, uint32_t sx, uint32_t sy, uint32_t sz, uint8_t *dst,
                    uint32_t dx, uint32_t dy, uint32_t dz) {
  for (uint32_t z = 0; z < dz; z++)
    for (uint32_t y = 0; y < dy; y++)
      for (uint32_t x = 0; x < dx; x++) {
        uint32_t sum = 4u;
        for (uint32_t k = 0; k < 8u; k++) {
          uint32_t xx = 2u * x + (k & 1u), yy = 2u * y + ((k >> 1) & 1u), zz = 2u * z + (k >> 2);
          if (xx >= sx) xx = sx - 1u;
          if (yy >= sy) yy = sy - 1u;
          if (zz >= sz) zz = sz - 1u;
          sum += src[((size_t)zz * sy + yy) * sx + xx];
        }
        dst[((size_t)z * dy + y) * dx + x] = (uint8_t)(sum / 8u);
      }
}

void orc_occupancy(const uint8_t *vox, uint32_t nx, uint32_t ny, uint32_t nz, uint8_t *out) {
  uint32_t ox = (nx + 7u) / 8u, oy = (ny + 7u) / 8u, oz = (nz + 7u) / 8u;
  size_t n = (size_t)ox * oy * oz;
  uint8_t *raw = malloc(n);
  if (!raw) return;
  for (uint32_t bz = 0; bz < oz; bz++)
    for (uint32_t by = 0; by < oy; by++)
      for (uint32_t bx = 0; bx < ox; bx++) {
        uint8_t m = 0;
        for (uint32_t z = bz * 8u; z < bz * 8u + 8u && z < nz; z++)
          for (uint32_t y = by * 8u; y < by * 8u + 8u && y < ny; y++)
            for (uint32_t x = bx * 8u; x < bx * 8u + 8u && x < nx; x++) {
              uint8_t v = vox[((size_t)z * ny + y) * nx + x];
              if (v > m) m = v;
            }
        raw[((size_t)bz * oy + by) * ox + bx] = m;
      }
  for (uint32_t z = 0; z < oz; z++)
    for (uint32_t y = 0; y < oy; y++)
      for (uint32_t x = 0; x < ox; x++) {
        uint8_t m = 0;
        for (int dz = -1; dz <= 1; dz++)
          for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
              int zz = (int)z + dz, yy = (int)y + dy, xx = (int)x + dx;
              if (zz < 0 || yy < 0 || xx < 0 || zz >= (int)oz || yy >= (int)oy || xx >= (int)ox)
                continue;
              uint8_t v = raw[((size_t)zz * oy + (size_t)yy) * ox + (size_t)xx];
              if (v > m) m = v;
            }
        out[((size_t)z * oy + y) * ox + x] = m;
      }
  free(raw);
}

static uint32_t ceil_div(uint32_t a, uint32_t b) { return (a + b - 1u) / b; }

static int slab_layout1(uint32_t nx, uint32_t ny, uint32_t out[4]) { /* slab.h:42-62 */
  uint32_t maxp = 2046u;
  out[0] = (nx + maxp - 1u) / maxp;
  out[1] = (ny + maxp - 1u) / maxp;
  if (out[0] > 22u || out[1] > 22u) return -1;
  out[2] = (nx + out[0] - 1u) / out[0];
  out[3] = (ny + out[1] - 1u) / out[1];
  return 0;
}

uint32_t orc_slab_layout(uint32_t nx, uint32_t ny, uint32_t lev[8][4], uint32_t *ovs) {
  if (slab_layout1(nx, ny, lev[0]) != 0) return 0;
  uint32_t o = 4u;
  while ((nx + o - 1u) / o > 2046u || (ny + o - 1u) / o > 2046u) o <<= 1;
  uint32_t nov = 1u;
  for (uint32_t s = 4u; s < o; s <<= 1) nov++;
  if (nov + 1u > 8u) return 0;
  for (uint32_t l = 1; l <= nov; l++) {
    uint32_t s = 4u << (l - 1u);
    slab_layout1((nx + s - 1u) / s, (ny + s - 1u) / s, lev[l]);
  }
  if (ovs) *ovs = o;
  return nov + 1u;
}

/* vkbackend.c:2128-2144: truncating n x n box average, clipped at the edges */
static void slab_down(const uint8_t *src, uint32_t nx, uint32_t ny, uint32_t n, uint8_t *dst) {
  uint32_t ox = (nx + n - 1u) / n, oy = (ny + n - 1u) / n;
  for (uint32_t y = 0; y < oy; y++)
    for (uint32_t x = 0; x < ox; x++) {
      uint32_t x0 = x * n, x1 = x0 + n > nx ? nx : x0 + n;
      uint32_t y0 = y * n, y1 = y0 + n > ny ? ny : y0 + n;
      uint32_t sum = 0;
      for (uint32_t yy = y0; yy < y1; yy++)
        for (uint32_t xx = x0; xx < x1; xx++) sum += src[(size_t)yy * nx + xx];
      dst[(size_t)y * ox + x] = (uint8_t)(sum / ((y1 - y0) * (x1 - x0)));
    }
}

/* tile slices of one level from a plane into ring `layer` (vkbackend.c:2148-2164) */
static void slab_tiles(const uint8_t *plane, uint32_t nx, uint32_t ny, const uint32_t L[4],
                       uint32_t wz, uint32_t layer, uint8_t *tiles) {
  uint32_t tw = L[2] + 2u, th = L[3] + 2u;
  size_t tb = (size_t)tw * th * wz;
  for (uint32_t j = 0; j < L[1]; j++)
    for (uint32_t i = 0; i < L[0]; i++)
      for (uint32_t ty = 0; ty < th; ty++)
        for (uint32_t tx = 0; tx < tw; tx++) {
          int64_t cx = (int64_t)i * L[2] - 1 + tx, cy = (int64_t)j * L[3] - 1 + ty;
          cx = cx < 0 ? 0 : (cx >= (int64_t)nx ? (int64_t)nx - 1 : cx);
          cy = cy < 0 ? 0 : (cy >= (int64_t)ny ? (int64_t)ny - 1 : cy);
          tiles[(size_t)(j * L[0] + i) * tb + (size_t)layer * tw * th + (size_t)ty * tw + tx] =
              plane[(size_t)cy * nx + (size_t)cx];
        }
}

/* truncating N x N box of a w x h plane (row pitch stride), vkbackend.c:5682-5696 */
static void vs_box(const uint8_t *src, uint32_t stride, uint32_t w, uint32_t h, uint32_t N,
                   uint8_t *dst) {
  for (uint32_t y = 0; y < h / N; y++)
    for (uint32_t x = 0; x < w / N; x++) {
      uint32_t sum = 0;
      for (uint32_t yy = 0; yy < N; yy++)
        for (uint32_t xx = 0; xx < N; xx++) sum += src[(size_t)(y * N + yy) * stride + x * N + xx];
      dst[(size_t)y * (w / N) + x] = (uint8_t)(sum / (N * N));
    }
}

void orc_vslab_fill(orc_vslab *v, const uint8_t *vox, uint32_t nx, uint32_t ny, int64_t cx,
                    int64_t cy, int64_t zs0, uint32_t nz) {
  const uint32_t P = v->px, T = P + 2u;
  const size_t plane = (size_t)T * T, tb = plane * v->wz;
  const uint32_t slot = (uint32_t)(cy % v->gy[0]) * v->gx[0] + (uint32_t)(cx % v->gx[0]);
  uint8_t *box = malloc(plane), *ds[5] = {0};
  for (uint32_t l = 1; l < 5; l++) ds[l] = malloc((size_t)(P / 4u) * (P / 4u));
  if (!box || !ds[4]) goto out;
  static const uint32_t scale[5] = {1u, 4u, 8u, 16u, 32u};
  for (uint32_t k = 0; k < nz; k++) {
    const int64_t z = zs0 + k;
    const size_t layer = (size_t)(z % v->wz) * plane;
    /* the decoded cell box: near edges duplicated, far edges zero */
    for (uint32_t ty = 0; ty < T; ty++)
      for (uint32_t tx = 0; tx < T; tx++) {
        int64_t wx = cx * (int64_t)P - 1 + tx, wy = cy * (int64_t)P - 1 + ty;
        uint8_t val = 0;
        if (wx < (int64_t)nx && wy < (int64_t)ny)
          val = vox[((size_t)z * ny + (size_t)(wy < 0 ? 0 : wy)) * nx + (size_t)(wx < 0 ? 0 : wx)];
        box[(size_t)ty * T + tx] = val;
      }
    memcpy(v->tiles + (size_t)(v->base[0] + slot) * tb + layer, box, plane);
    if (!v->gx[1]) continue;
    /* pyramid strips: 4x from the payload, then 2x chains */
    vs_box(box + T + 1u, T, P, P, 4u, ds[1]);
    for (uint32_t l = 2; l < 5 && v->gx[l]; l++)
      vs_box(ds[l - 1], P / scale[l - 1], P / scale[l - 1], P / scale[l - 1], 2u, ds[l]);
    for (uint32_t l = 1; l < 5 && v->gx[l]; l++) {
      const int64_t n = P / scale[l], t0x = cx * n, t0y = cy * n, Pi = P;
      int64_t p0x = (t0x - 1) / Pi, p1x = (t0x + n) / Pi;
      int64_t p0y = (t0y - 1) / Pi, p1y = (t0y + n) / Pi;
      if (p0x < 0) p0x = 0;
      if (p0y < 0) p0y = 0;
      for (int64_t qy = p0y; qy <= p1y; qy++)
        for (int64_t qx = p0x; qx <= p1x; qx++) {
          int64_t ax = t0x > qx * Pi - 1 ? t0x : qx * Pi - 1;
          int64_t bx = t0x + n < qx * Pi + Pi + 1 ? t0x + n : qx * Pi + Pi + 1;
          int64_t ay = t0y > qy * Pi - 1 ? t0y : qy * Pi - 1;
          int64_t by = t0y + n < qy * Pi + Pi + 1 ? t0y + n : qy * Pi + Pi + 1;
          if (ax >= bx || ay >= by) continue;
          uint32_t ti = v->base[l] + (uint32_t)(qy % v->gy[l]) * v->gx[l] + (uint32_t)(qx % v->gx[l]);
          uint8_t *dst = v->tiles + (size_t)ti * tb + layer;
          for (int64_t y = ay; y < by; y++)
            for (int64_t x = ax; x < bx; x++)
              dst[(size_t)(y - qy * Pi + 1) * T + (size_t)(x - qx * Pi + 1)] =
                  ds[l][(size_t)(y - t0y) * n + (size_t)(x - t0x)];
        }
    }
  }
out:
  free(box);
  for (uint32_t l = 1; l < 5; l++) free(ds[l]);
}

/* tight 2^3 box, truncating (tools/mkpyramid/main.c:53-69): dst is
 * (sx/2, sy/2, sz/2) */
static void clip_down2(const uint8_t *src, uint32_t sx, uint32_t sy, uint32_t sz, uint8_t *dst) {
  uint32_t hx = sx / 2u, hy = sy / 2u, hz = sz / 2u;
  for (uint32_t z = 0; z < hz; z++)
    for (uint32_t y = 0; y < hy; y++)
      for (uint32_t x = 0; x < hx; x++) {
        uint32_t v = 0;
        for (uint32_t k = 0; k < 8u; k++)
          v += src[((size_t)(2u * z + (k >> 2)) * sy + 2u * y + ((k >> 1) & 1u)) * sx + 2u * x +
                   (k & 1u)];
        dst[((size_t)z * hy + y) * hx + x] = (uint8_t)(v / 8u);
      }
}

static int64_t clampi64(int64_t v, int64_t lo, int64_t hi) { return v < lo ? lo : v > hi ? hi : v; }

void orc_clip_fill(const uint8_t *vox, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t depth_max,
                   uint32_t z0, const float orig[6][2], uint8_t *const tex[6]) {
  const uint32_t T = 2048u;
  uint8_t *pyr[6] = {0};
  uint32_t pd[6][3];
  pd[0][0] = nx, pd[0][1] = ny, pd[0][2] = nz;
  for (int l = 1; l < 6; l++)
    for (int a = 0; a < 3; a++) pd[l][a] = pd[l - 1][a] / 2u;
  /* the pyramid: half = down2(volume), level l = down2(level l-1) */
  const uint8_t *prev = vox;
  for (int l = 1; l < 6; l++) {
    size_t n = (size_t)pd[l][0] * pd[l][1] * pd[l][2];
    pyr[l] = malloc(n ? n : 1u);
    if (!pyr[l]) goto out;
    if (n) clip_down2(prev, pd[l - 1][0], pd[l - 1][1], pd[l - 1][2], pyr[l]);
    prev = pyr[l];
  }
  for (int l = 0; l < 6; l++) {
    uint32_t wzl = depth_max / (1u << l) + 3u;
    if (wzl < 4u) wzl = 4u;
    int64_t s = (int64_t)1 << l;
    int64_t ox = (int64_t)orig[l][0], oy = (int64_t)orig[l][1];
    int64_t vx0 = ox / s - 1, vy0 = oy / s - 1; /* texel 0 in level voxels */
    for (uint32_t k = 0; k < wzl; k++) {
      int64_t ls = (int64_t)(z0 >> l) + k;
      uint8_t *dst = tex[l] + (size_t)(ls % wzl) * T * T;
      for (uint32_t ty = 0; ty < T; ty++)
        for (uint32_t tx = 0; tx < T; tx++) {
          uint32_t v = 0;
          if (l == 0) { /* produce_slice level 0: decode_region_clamped (vkclip.c:138-176) */
            if (ls < (int64_t)nz)
              v = vox[((size_t)ls * ny + (size_t)clampi64(vy0 + ty, 0, ny - 1)) * nx +
                      (size_t)clampi64(vx0 + tx, 0, nx - 1)];
          } else if (l == 1) { /* full-resolution 2^3 box (vkclip.c:181-199) */
            for (uint32_t q = 0; q < 8u; q++) {
              int64_t z = 2 * ls + (q >> 2);
              if (z >= (int64_t)nz) continue;
              int64_t x = clampi64(2 * (vx0 + tx) + (q & 1u), 0, nx - 1);
              int64_t y = clampi64(2 * (vy0 + ty) + ((q >> 1) & 1u), 0, ny - 1);
              v += vox[((size_t)z * ny + (size_t)y) * nx + (size_t)x];
            }
            v /= 8u;
          } else if (ls < (int64_t)pd[l][2] && pd[l][0] && pd[l][1]) {
            /* produce_from_pyramid (vkclip.c:101-132): rows and columns
             * clamped at the level's extent */
            int64_t x = clampi64(vx0 + tx, 0, pd[l][0] - 1);
            int64_t y = clampi64(vy0 + ty, 0, pd[l][1] - 1);
            v = pyr[l][((size_t)ls * pd[l][1] + (size_t)y) * pd[l][0] + (size_t)x];
          }
          dst[(size_t)ty * T + tx] = (uint8_t)v;
        }
    }
  }
out:
  for (int l = 1; l < 6; l++) free(pyr[l]);
}

void orc_slab_fill(const uint8_t *vox, uint32_t nx, uint32_t ny, uint32_t nz, uint32_t wz,
                   uint32_t z0, uint8_t *const tiles[8]) {
  uint32_t lev[8][4], ovs = 0;
  uint32_t nl = orc_slab_layout(nx, ny, lev, &ovs);
  if (!nl || z0 + wz > nz) return;
  uint8_t *a = malloc((size_t)nx * ny), *b = malloc((size_t)nx * ny);
  if (!a || !b) goto out;
  for (uint32_t s = z0; s < z0 + wz; s++) {
    const uint8_t *slice = vox + (size_t)s * nx * ny;
    uint32_t layer = s % wz;
    slab_tiles(slice, nx, ny, lev[0], wz, layer, tiles[0]);
    const uint8_t *prev = slice;
    uint32_t pnx = nx, pny = ny;
    for (uint32_t l = 1; l < nl; l++) {
      uint8_t *dst = (l & 1u) ? a : b;
      uint32_t f = l == 1u ? 4u : 2u;
      slab_down(prev, pnx, pny, f, dst);
      pnx = (pnx + f - 1u) / f;
      pny = (pny + f - 1u) / f;
      slab_tiles(dst, pnx, pny, lev[l], wz, layer, tiles[l]);
      prev = dst;
    }
  }
out:
  free(a);
  free(b);
}

int orc_build_lod_overlay(const uint8_t *vox, uint32_t nx, uint32_t ny, uint32_t nz,
                          const uint32_t *page, uint32_t page_words, int labels, uint8_t *pool,
                          uint32_t nslots) {
  if (page_words < R3D_BRICK_PAGE_HEADER || page[1] != nx || page[2] != ny || page[3] != nz)
    return -1;
  uint32_t nlev = page[0];
  if (nlev < 1u || nlev > 15u || page_words != orc_lod_page_words(nx, ny, nz, nlev)) return -1;
  uint32_t bd[16][3], E[16][3];
  uint8_t *lev[16] = {0};
  for (uint32_t l = 0; l < nlev; l++) {
    uint32_t sc = 1u << l;
    bd[l][0] = ceil_div(ceil_div(nx, sc), 128u);
    bd[l][1] = ceil_div(ceil_div(ny, sc), 128u);
    bd[l][2] = ceil_div(ceil_div(nz, sc), 128u);
    for (int a = 0; a < 3; a++) E[l][a] = bd[l][a] * 128u;
  }
#define L0(X, Y, Z) \
  ((X) < nx && (Y) < ny && (Z) < nz ? vox[((size_t)(Z) * ny + (Y)) * nx + (X)] : (uint8_t)0)
  for (uint32_t l = 1; l < nlev; l++) {
    lev[l] = malloc((size_t)E[l][0] * E[l][1] * E[l][2]);
    if (!lev[l]) goto fail;
    for (uint32_t z = 0; z < E[l][2]; z++)
      for (uint32_t y = 0; y < E[l][1]; y++)
        for (uint32_t x = 0; x < E[l][0]; x++) {
          uint8_t v;
          if (labels) {
            uint64_t X = (uint64_t)x << l, Y = (uint64_t)y << l, Z = (uint64_t)z << l;
            v = X < nx && Y < ny && Z < nz ? vox[(Z * ny + Y) * nx + X] : 0;
          } else {
            uint32_t sum = 4u;
            for (uint32_t k = 0; k < 8u; k++) {
              uint32_t xx = 2u * x + (k & 1u), yy = 2u * y + ((k >> 1) & 1u),
                       zz = 2u * z + (k >> 2);
              if (l == 1u)
                sum += L0(xx, yy, zz);
              else if (xx < E[l - 1][0] && yy < E[l - 1][1] && zz < E[l - 1][2])
                sum += lev[l - 1][((size_t)zz * E[l - 1][1] + yy) * E[l - 1][0] + xx];
            }
            v = (uint8_t)(sum / 8u);
          }
          lev[l][((size_t)z * E[l][1] + y) * E[l][0] + x] = v;
        }
  }
  for (uint32_t l = 0; l < nlev; l++) {
    uint32_t off = page[4u + l * 4u];
    for (uint32_t bz = 0; bz < bd[l][2]; bz++)
      for (uint32_t by = 0; by < bd[l][1]; by++)
        for (uint32_t bx = 0; bx < bd[l][0]; bx++) {
          uint32_t e = page[off + (bz * bd[l][1] + by) * bd[l][0] + bx];
          if (e == R3D_BRICK_ABSENT || (e & 0xFFFFFFu) >= nslots) continue;
          uint8_t *dst = pool + (size_t)(e & 0xFFFFFFu) * (128u * 128u * 128u);
          for (uint32_t z = 0; z < 128u; z++)
            for (uint32_t y = 0; y < 128u; y++)
              for (uint32_t x = 0; x < 128u; x++) {
                uint32_t X = bx * 128u + x, Y = by * 128u + y, Z = bz * 128u + z;
                dst[((size_t)z * 128u + y) * 128u + x] =
                    l == 0u ? L0(X, Y, Z) : lev[l][((size_t)Z * E[l][1] + Y) * E[l][0] + X];
              }
        }
  }
#undef L0
  for (uint32_t l = 1; l < nlev; l++) free(lev[l]);
  return 0;
fail:
  for (uint32_t l = 1; l < nlev; l++) free(lev[l]);
  return -1;
}

int orc_build_shard(const uint8_t *vox, uint32_t edge, uint32_t abpa, const uint32_t *slot_of,
                    uint32_t *page, uint8_t *atlas0) {
  if (!vox || !page || !edge || edge % 128u || edge / 128u > 255u) return -1;
  uint32_t bpa = edge / 128u, nb = bpa * bpa * bpa;
  if (!abpa || abpa > bpa || (!slot_of && abpa != bpa)) return -1;
  uint32_t ns = abpa * abpa * abpa, a = abpa * 128u;
  int identity = abpa == bpa;
  if (atlas0) memset(atlas0, 0, (size_t)a * a * a);
  for (uint32_t b = 0; b < nb; b++) {
    uint32_t s = slot_of ? slot_of[b] : b;
    identity = identity && s == b;
    if (s == 0xFFFFFFFFu) {
      page[b] = 0xFFFFFFFFu;
      continue;
    }
    if (s >= ns) return -1;
    uint32_t bx = b % bpa, by = (b / bpa) % bpa, bz = b / (bpa * bpa);
    uint32_t sx = s % abpa, sy = (s / abpa) % abpa, sz = s / (abpa * abpa);
    uint8_t m = 0;
    for (uint32_t z = 0; z < 128u; z++)
      for (uint32_t y = 0; y < 128u; y++) {
        const uint8_t *src = vox + ((size_t)(bz * 128u + z) * edge + (by * 128u + y)) * edge +
                             bx * 128u;
        for (uint32_t x = 0; x < 128u; x++)
          if (src[x] > m) m = src[x];
        if (atlas0)
          memcpy(atlas0 + ((size_t)(sz * 128u + z) * a + (sy * 128u + y)) * a + sx * 128u, src,
                 128u);
      }
    page[b] = s | ((uint32_t)m << 24);
  }
  return identity ? 1 : 0;
}

void orc_shard_occupancy(const uint8_t *atlas0, uint32_t abpa, const uint32_t *page, uint32_t bpa,
                         uint8_t *out) {
  uint32_t od = bpa * 16u, a = abpa * 128u;
  size_t n = (size_t)od * od * od;
  uint8_t *raw = malloc(n);
  if (!raw) return;
  for (uint32_t wz = 0; wz < od; wz++)
    for (uint32_t wy = 0; wy < od; wy++)
      for (uint32_t wx = 0; wx < od; wx++) {
        uint32_t e = page[((wz >> 4) * bpa + (wy >> 4)) * bpa + (wx >> 4)];
        uint8_t m = 0;
        if (e != 0xFFFFFFFFu) {
          uint32_t s = e & 0xFFFFFFu;
          uint32_t x0 = (s % abpa) * 128u + (wx & 15u) * 8u;
          uint32_t y0 = ((s / abpa) % abpa) * 128u + (wy & 15u) * 8u;
          uint32_t z0 = (s / (abpa * abpa)) * 128u + (wz & 15u) * 8u;
          for (uint32_t z = z0; z < z0 + 8u; z++)
            for (uint32_t y = y0; y < y0 + 8u; y++)
              for (uint32_t x = x0; x < x0 + 8u; x++) {
                uint8_t v = atlas0[((size_t)z * a + y) * a + x];
                if (v > m) m = v;
              }
        }
        raw[((size_t)wz * od + wy) * od + wx] = m;
      }
  for (uint32_t z = 0; z < od; z++)
    for (uint32_t y = 0; y < od; y++)
      for (uint32_t x = 0; x < od; x++) {
        uint8_t m = 0;
        for (int dz = -1; dz <= 1; dz++)
          for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
              int zz = (int)z + dz, yy = (int)y + dy, xx = (int)x + dx;
              if (zz < 0 || yy < 0 || xx < 0 || zz >= (int)od || yy >= (int)od || xx >= (int)od)
                continue;
              uint8_t v = raw[((size_t)zz * od + (size_t)yy) * od + (size_t)xx];
              if (v > m) m = v;
            }
        out[((size_t)z * od + y) * od + x] = m;
      }
  free(raw);
}

uint32_t orc_lod_page_words(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t nlev) {
  uint32_t w = R3D_BRICK_PAGE_HEADER;
  for (uint32_t l = 0; l < nlev; l++) {
    uint32_t s = 1u << l;
    w += ceil_div(ceil_div(nx, s), 128u) * ceil_div(ceil_div(ny, s), 128u) *
         ceil_div(ceil_div(nz, s), 128u);
  }
  return w;
}

int64_t orc_build_lod_bricks(const uint8_t *vox, uint32_t nx, uint32_t ny, uint32_t nz,
                             uint32_t nlev, uint32_t min_max, uint32_t *page,
                             uint32_t page_words, uint8_t *pool, uint64_t pool_slots) {
  if (nlev < 1u || nlev > 15u || page_words != orc_lod_page_words(nx, ny, nz, nlev)) return -1;
  /* padded level grids: E[l] = 128 * bricks per axis; level 0 reads vox */
  uint32_t bd[16][3], E[16][3];
  uint8_t *lev[16] = {0};
  for (uint32_t l = 0; l < nlev; l++) {
    uint32_t s = 1u << l;
    bd[l][0] = ceil_div(ceil_div(nx, s), 128u);
    bd[l][1] = ceil_div(ceil_div(ny, s), 128u);
    bd[l][2] = ceil_div(ceil_div(nz, s), 128u);
    for (int a = 0; a < 3; a++) E[l][a] = bd[l][a] * 128u;
  }
#define L0(X, Y, Z) \
  ((X) < nx && (Y) < ny && (Z) < nz ? vox[((size_t)(Z) * ny + (Y)) * nx + (X)] : (uint8_t)0)
  for (uint32_t l = 1; l < nlev; l++) {
    lev[l] = malloc((size_t)E[l][0] * E[l][1] * E[l][2]);
    if (!lev[l]) goto fail;
    for (uint32_t z = 0; z < E[l][2]; z++)
      for (uint32_t y = 0; y < E[l][1]; y++)
        for (uint32_t x = 0; x < E[l][0]; x++) {
          uint32_t sum = 4u;
          for (uint32_t k = 0; k < 8u; k++) {
            uint32_t xx = 2u * x + (k & 1u), yy = 2u * y + ((k >> 1) & 1u),
                     zz = 2u * z + (k >> 2);
            if (l == 1u)
              sum += L0(xx, yy, zz);
            else if (xx < E[l - 1][0] && yy < E[l - 1][1] && zz < E[l - 1][2])
              sum += lev[l - 1][((size_t)zz * E[l - 1][1] + yy) * E[l - 1][0] + xx];
          }
          lev[l][((size_t)z * E[l][1] + y) * E[l][0] + x] = (uint8_t)(sum / 8u);
        }
  }
  memset(page, 0, R3D_BRICK_PAGE_HEADER * sizeof *page);
  page[0] = nlev;
  page[1] = nx;
  page[2] = ny;
  page[3] = nz;
  uint32_t off = 0;
  int64_t slot = 0;
  for (uint32_t l = 0; l < nlev; l++) {
    page[4u + l * 4u] = R3D_BRICK_PAGE_HEADER + off;
    page[5u + l * 4u] = bd[l][0] | (bd[l][1] << 10) | (bd[l][2] << 20);
    page[6u + l * 4u] = 1u << l;
    for (uint32_t bz = 0; bz < bd[l][2]; bz++)
      for (uint32_t by = 0; by < bd[l][1]; by++)
        for (uint32_t bx = 0; bx < bd[l][0]; bx++) {
          uint32_t m = 0;
          for (uint32_t z = 0; z < 128u; z++)
            for (uint32_t y = 0; y < 128u; y++)
              for (uint32_t x = 0; x < 128u; x++) {
                uint32_t X = bx * 128u + x, Y = by * 128u + y, Z = bz * 128u + z;
                uint32_t v = l == 0u ? L0(X, Y, Z)
                                     : lev[l][((size_t)Z * E[l][1] + Y) * E[l][0] + X];
                if (v > m) m = v;
              }
          uint32_t idx = R3D_BRICK_PAGE_HEADER + off + (bz * bd[l][1] + by) * bd[l][0] + bx;
          if (m >= min_max) {
            page[idx] = (uint32_t)slot | (m << 24);
            if (pool && (uint64_t)slot < pool_slots) {
              uint8_t *dst = pool + (size_t)slot * (128u * 128u * 128u);
              for (uint32_t z = 0; z < 128u; z++)
                for (uint32_t y = 0; y < 128u; y++)
                  for (uint32_t x = 0; x < 128u; x++) {
                    uint32_t X = bx * 128u + x, Y = by * 128u + y, Z = bz * 128u + z;
                    dst[((size_t)z * 128u + y) * 128u + x] =
                        l == 0u ? L0(X, Y, Z) : lev[l][((size_t)Z * E[l][1] + Y) * E[l][0] + X];
                  }
            }
            slot++;
          } else {
            page[idx] = R3D_BRICK_ABSENT;
          }
        }
    off += bd[l][0] * bd[l][1] * bd[l][2];
  }
#undef L0
  for (uint32_t l = 1; l < nlev; l++) free(lev[l]);
  return slot;
fail:
  for (uint32_t l = 1; l < nlev; l++) free(lev[l]);
  return -1;
}

/* ------------------------------------------------- host-side helpers */

/* forward_of + r3d_camera_basis, src/core/camera.c:12-15,65-75 */
void orc_camera_basis(float yaw, float pitch, float fov_y, float aspect, float right[3],
                      float up[3], float fwd[3]) {
  float cp = cosf(pitch);
  float f[3] = {sinf(yaw) * cp, sinf(pitch), cosf(yaw) * cp};
  /* cross(f, (0,1,0)) = (-f.z, 0, f.x) */
  float r[3] = {f[1] * 0.0f - f[2] * 1.0f, f[2] * 0.0f - f[0] * 0.0f, f[0] * 1.0f - f[1] * 0.0f};
  float rl = sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
  if (rl > 0.0f) {
    float inv = 1.0f / rl;
    r[0] *= inv, r[1] *= inv, r[2] *= inv;
  } else {
    r[0] = r[1] = r[2] = 0.0f;
  }
  if (sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]) == 0.0f) {
    r[0] = 1.0f;
    r[1] = r[2] = 0.0f;
  }
  float u[3] = {r[1] * f[2] - r[2] * f[1], r[2] * f[0] - r[0] * f[2], r[0] * f[1] - r[1] * f[0]};
  float t = tanf(fov_y * 0.5f);
  for (int a = 0; a < 3; a++) {
    right[a] = r[a] * (t * aspect);
    up[a] = u[a] * t;
    fwd[a] = f[a];
  }
}

/* orbit_sync, src/core/camera.c:32-34 */
void orc_orbit_pos(float yaw, float pitch, const float target[3], float dist, float pos[3]) {
  float cp = cosf(pitch);
  float f[3] = {sinf(yaw) * cp, sinf(pitch), cosf(yaw) * cp};
  for (int a = 0; a < 3; a++) pos[a] = target[a] - f[a] * dist;
}

/* r3d_tf_build, src/core/transfer.c:5-23 */
void orc_tf_build(const uint8_t *values, const uint8_t (*rgba)[4], uint32_t npts,
                  uint8_t lut[256][4]) {
  for (uint32_t i = 0; i < 256u; i++) {
    uint32_t lo = 0, hi = npts - 1u;
    for (uint32_t k = 0; k + 1u < npts; k++)
      if (values[k] <= i && i <= values[k + 1u]) {
        lo = k;
        hi = k + 1u;
        break;
      }
    uint32_t span = (uint32_t)(values[hi] - values[lo]);
    uint32_t tn = span ? i - values[lo] : 0u, td = span ? span : 1u;
    for (int c = 0; c < 4; c++)
      lut[i][c] = (uint8_t)(((uint32_t)rgba[lo][c] * (td - tn) + (uint32_t)rgba[hi][c] * tn) / td);
  }
}

/* r3d_lod_pick / r3d_lod_fallback, src/core/lod.h:8-26 */
uint32_t orc_lod_pick(float distance, float pixel_cone, float base_voxels, uint32_t nlevels) {
  if (!nlevels) return 0;
  float fp = fmaxf(distance * pixel_cone * base_voxels, 1.0f);
  int level = (int)floorf(log2f(fp));
  if (level < 0) level = 0;
  if (level >= (int)nlevels) level = (int)nlevels - 1;
  return (uint32_t)level;
}

uint32_t orc_lod_fallback(uint32_t desired, uint32_t ordinal, uint32_t nlevels) {
  if (!nlevels || desired >= nlevels || ordinal >= nlevels) return UINT32_MAX;
  uint32_t coarse = nlevels - desired;
  if (ordinal < coarse) return desired + ordinal;
  return desired - 1u - (ordinal - coarse);
}

/* m3_ypr, src/core/mathx.h:34-43 (rows; M = Ry * Rx * Rz) */
void orc_m3_ypr(float yaw, float pitch, float roll, float rows[3][3]) {
  float cy = cosf(yaw), sy = sinf(yaw), cp = cosf(pitch), sp = sinf(pitch), cr = cosf(roll),
        sr = sinf(roll);
  rows[0][0] = cy * cr + sy * sp * sr;
  rows[0][1] = -cy * sr + sy * sp * cr;
  rows[0][2] = sy * cp;
  rows[1][0] = cp * sr;
  rows[1][1] = cp * cr;
  rows[1][2] = -sp;
  rows[2][0] = -sy * cr + cy * sp * sr;
  rows[2][1] = sy * sr + cy * sp * cr;
  rows[2][2] = cy * cp;
}

/* ------------------------------------------------- benchmark inputs */

/* The benchmark's scripted orbit view at phase ph (src/main.c:3932-3946 and
 * the frame set-up of src/main.c:6788-6824): turntable camera from the
 * reference's default position, yaw = ph * tau, pitch = 0.5 sin(2 ph tau),
 * orbiting `target` at distance 2, 60 degree field of view; camera basis of
 * src/core/camera.c:65-75, skip gate of src/main.c:1238-1242, identity
 * volume rotation (src/core/mathx.h:34-43 at zero angles). */
void orc_orbit_view(r3d_frame_params *p, float ph, const float target[3], uint32_t w, uint32_t h,
                    float step_voxels, float density, float lod_bias, uint32_t mode,
                    uint32_t frame_index, float low_cut, const uint8_t lut[256][4]) {
  const float tau = 6.2831853f;
  const float yaw = ph * tau, pitch = 0.5f * sinf(ph * tau * 2.0f);
  memset(p, 0, sizeof *p);
  orc_orbit_pos(yaw, pitch, target, 2.0f, p->cam_origin);
  orc_camera_basis(yaw, pitch, 1.04719755f, (float)w / (float)h, p->cam_right, p->cam_up,
                   p->cam_forward);
  p->step_voxels = step_voxels;
  p->density = density;
  p->lod_bias = lod_bias;
  p->max_mip = 10.0f;
  p->viewport[0] = w;
  p->viewport[1] = h;
  p->mode = mode;
  p->frame_index = frame_index;
  p->threshold = low_cut / 255.0f;
  float vis = 255.0f;
  for (uint32_t i = 0; i < 256u; i++)
    if (lut[i][3] != 0) {
      vis = (float)i;
      break;
    }
  p->skip_gate = fmaxf(low_cut, vis - 0.5f) / 255.0f;
  float m[3][3];
  orc_m3_ypr(0.0f, 0.0f, 0.0f, m);
  memcpy(p->vol_r0, m[0], 12);
  memcpy(p->vol_r1, m[1], 12);
  memcpy(p->vol_r2, m[2], 12);
}

static uint64_t orc_splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

/* The seeded scroll phantom (the benchmark's synthetic volume): an
 * Archimedean spiral of papyrus sheets about the z axis through the volume
 * centre, r = r0 + pitch * theta / 2pi with r0 = 8, a voxel papyrus when its
 * radial distance to the nearest wrap is below 3 (6-voxel sheets) and
 * r0 <= r < radius; pitch 14 up to an edge of 256, else 18; radius 110/256 of
 * the largest edge.  Papyrus ~N(130, 15), air ~N(12, 4), plus N(0, 6) noise,
 * rounded and clamped to 0..255.  Voxel i draws its two normals by
 * Box-Muller from splitmix64(seed ^ 2i) and splitmix64(seed ^ (2i + 1)).
 * vox is (nz, ny, nx), x fastest. */
int orc_phantom(uint8_t *vox, uint32_t nx, uint32_t ny, uint32_t nz, uint64_t seed, int threads) {
  if (!vox || !nx || !ny || !nz) return -1;
  uint32_t n = nx > ny ? nx : ny;
  n = n > nz ? n : nz;
  const double pitch = n <= 256u ? 14.0 : 18.0, radius = (double)(110.0f * (float)n / 256.0f);
  const double r0 = 8.0, half = 3.0, two_pi = 6.283185307179586;
  uint8_t *mask = malloc((size_t)nx * ny);
  if (!mask) return -1;
  const double cx = 0.5 * nx, cy = 0.5 * ny;
  for (uint32_t y = 0; y < ny; y++)
    for (uint32_t x = 0; x < nx; x++) {
      double dx = x + 0.5 - cx, dy = y + 0.5 - cy;
      double r = sqrt(dx * dx + dy * dy), th = atan2(dy, dx);
      if (th < 0.0) th += two_pi;
      double m = fmod(r - r0 - pitch * th / two_pi, pitch);
      if (m < 0.0) m += pitch;
      double dist = m < pitch - m ? m : pitch - m;
      mask[(size_t)y * nx + x] = dist < half && r >= r0 && r < radius;
    }
  const int nt = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(static) num_threads(nt)
  for (int64_t z = 0; z < (int64_t)nz; z++)
    for (uint32_t y = 0; y < ny; y++)
      for (uint32_t x = 0; x < nx; x++) {
        const uint64_t i = ((uint64_t)z * ny + y) * nx + x;
        const uint64_t h1 = orc_splitmix64(seed ^ (i * 2u)), h2 = orc_splitmix64(seed ^ (i * 2u + 1u));
        const double u1 = ((double)(h1 >> 11) + 1.0) * 0x1.0p-53, u2 = (double)(h2 >> 11) * 0x1.0p-53;
        const double rad = sqrt(-2.0 * log(u1));
        const int pap = mask[(size_t)y * nx + x];
        double v = (pap ? 130.0 : 12.0) + (pap ? 15.0 : 4.0) * (rad * cos(two_pi * u2)) +
                   6.0 * (rad * sin(two_pi * u2));
        v = floor(v + 0.5);
        vox[i] = (uint8_t)(v < 0.0 ? 0.0 : (v > 255.0 ? 255.0 : v));
      }
  free(mask);
  return 0;
}

/* ---- post-decode display filter (src/shaders/postfilt.comp) ---- */

/* texelFetch of the slot at l + d, clamped to the slot (postfilt.comp:27-29) */
static float pf_fetch(const uint8_t *slot, int x, int y, int z, int dx, int dy, int dz) {
  int cx = x + dx, cy = y + dy, cz = z + dz;
  cx = cx < 0 ? 0 : cx > 127 ? 127 : cx;
  cy = cy < 0 ? 0 : cy > 127 ? 127 : cy;
  cz = cz < 0 ? 0 : cz > 127 ? 127 : cz;
  return (float)slot[((size_t)cz * 128 + cy) * 128 + cx] / 255.0f;
}

/* one voxel of shader mode m (1 median 27, 2 unsharp, 3 median 125, 4 max
 * 27, 5 max 125), postfilt.comp:31-104 */
static float pf_voxel(const uint8_t *s, int x, int y, int z, int m, float amount) {
  if (m == 1) { /* partial selection up to rank 13 */
    float v[27];
    int n = 0;
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) v[n++] = pf_fetch(s, x, y, z, dx, dy, dz);
    for (int i = 0; i <= 13; i++) {
      int mi = i;
      for (int j = i + 1; j < 27; j++)
        if (v[j] < v[mi]) mi = j;
      float t = v[i];
      v[i] = v[mi];
      v[mi] = t;
    }
    return v[13];
  }
  if (m == 2) { /* centre pushed off the box mean */
    float sum = 0.0f;
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) sum += pf_fetch(s, x, y, z, dx, dy, dz);
    float center = pf_fetch(s, x, y, z, 0, 0, 0);
    return clampf_(center + amount * (center - sum / 27.0f), 0.0f, 1.0f);
  }
  if (m == 3) { /* u8 histogram, 4 high bits then 4 low bits */
    int cnt[16] = {0}, rank = 62, coarse = 15, acc = 0;
    for (int dz = -2; dz <= 2; dz++)
      for (int dy = -2; dy <= 2; dy++)
        for (int dx = -2; dx <= 2; dx++) {
          int q = (int)rintf(pf_fetch(s, x, y, z, dx, dy, dz) * 255.0f);
          cnt[q >> 4]++;
        }
    for (int i = 0; i < 16; i++) {
      if (acc + cnt[i] > rank) {
        coarse = i;
        break;
      }
      acc += cnt[i];
    }
    int rank2 = rank - acc, fine = 15;
    memset(cnt, 0, sizeof cnt);
    for (int dz = -2; dz <= 2; dz++)
      for (int dy = -2; dy <= 2; dy++)
        for (int dx = -2; dx <= 2; dx++) {
          int q = (int)rintf(pf_fetch(s, x, y, z, dx, dy, dz) * 255.0f);
          if ((q >> 4) == coarse) cnt[q & 15]++;
        }
    acc = 0;
    for (int i = 0; i < 16; i++) {
      if (acc + cnt[i] > rank2) {
        fine = i;
        break;
      }
      acc += cnt[i];
    }
    return (float)(coarse * 16 + fine) / 255.0f;
  }
  int rr = m == 4 ? 1 : 2; /* max pool */
  float o = 0.0f;
  for (int dz = -rr; dz <= rr; dz++)
    for (int dy = -rr; dy <= rr; dy++)
      for (int dx = -rr; dx <= rr; dx++) o = fmaxf(o, pf_fetch(s, x, y, z, dx, dy, dz));
  return o;
}

void orc_postfilter(uint8_t *slots, uint32_t n, uint32_t mode, float amount) {
  static const int prim2shader[5] = {0, 1, 3, 4, 5}; /* vkbackend.c:3411-3417 */
  const uint32_t prim = mode & 0xFFu;
  const size_t sb = (size_t)128 * 128 * 128;
  uint8_t *tmp = malloc(sb);
  if (!tmp) return;
  for (uint32_t k = 0; k < n; k++) {
    uint8_t *s = slots + k * sb;
    for (int pass = 0; pass < 2; pass++) {
      int m = pass == 0 ? (prim < 5u ? prim2shader[prim] : 0) : (mode & 0x100u ? 2 : 0);
      if (!m) continue;
#pragma omp parallel for schedule(static)
      for (int z = 0; z < 128; z++)
        for (int y = 0; y < 128; y++)
          for (int x = 0; x < 128; x++)
            tmp[((size_t)z * 128 + y) * 128 + x] = unorm8(pf_voxel(s, x, y, z, m, amount));
      memcpy(s, tmp, sb);
    }
  }
  free(tmp);
}
