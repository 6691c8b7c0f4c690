// Flattened-segment (surf) views: render3d's segment pane.  A segment is a
// grid of surface points (xyz + valid) and unit normals; the bake resamples
// the LOD brick cache into a W x H x L "flattened volume" over (u, v,
// layer): texel (x, y, l) holds the volume at surface(u, v) + normal(u, v) *
// (zoff0 + (l - nback) * lstep) (src/shaders/surfvol.comp), R = CT, G = an
// overlay atlas.  The surf raycast then marches each pixel's column of
// layers (src/shaders/raycast.slang:515-638): composite or MIP, gradient
// shading in flattened space, overlay tint, the flattening-distortion
// heatmap and the supervision-mask tint.  The reference bakes in row bands
// spread over frames and shifts the window in place on integer moves; here
// a bake covers the whole window in one launch on the context's stream.
#include <string.h>

#include "r3d_internal.h"

namespace r3d {

// GLSL mix(x, y, a) = x * (1 - a) + y * a
__device__ __forceinline__ float mixf(float x, float y, float a) {
  return fmaf(y, a, x * (1.0f - a));
}

struct SurfBake {
  const float4 *coords, *normals;  // gw x gh grids, row-major
  uint32_t gw, gh;
  float u0, v0, step, zoff0, sx, sy, lstep;
  uint32_t W, H, L, nback, lod;
  int ovl;       // overlay atlas baked into G, or -1
  uint8_t *vol;  // W x H x L texels of (R, G), x fastest
  const float *pred;  // live ink prediction, pw x ph, or null
  uint32_t pw, ph;
  float pg0u, pg0v, pppg;  // texel (0, 0) in grid coordinates; texels per grid unit
};

// The prediction texture, clamp-to-edge bilinear at texel-space position
// (px, py), sampled as textureLod(inkpred, (pp + 0.5) / size)
// (surfvol.comp:131-136).
__device__ __forceinline__ float pred_sample(const SurfBake &b, float px, float py) {
  const float u = (px + 0.5f) / (float)b.pw, v = (py + 0.5f) / (float)b.ph;
  const float tx = clamp_(fmaf(u, (float)b.pw, -0.5f), 0.0f, (float)(b.pw - 1u));
  const float ty = clamp_(fmaf(v, (float)b.ph, -0.5f), 0.0f, (float)(b.ph - 1u));
  const uint32_t x0 = (uint32_t)tx, y0 = (uint32_t)ty;
  const uint32_t x1 = min(x0 + 1u, b.pw - 1u), y1 = min(y0 + 1u, b.ph - 1u);
  const float fx = tx - (float)x0, fy = ty - (float)y0;
  const float *r0 = b.pred + (size_t)y0 * b.pw, *r1 = b.pred + (size_t)y1 * b.pw;
  return lerp_(lerp_(__ldg(r0 + x0), __ldg(r0 + x1), fx), lerp_(__ldg(r1 + x0), __ldg(r1 + x1), fx), fy);
}

// Per-column brick cache of the bake (surfvol.comp:40-52)
struct ColCache {
  bool valid;
  uint32_t scale, bx, by, bz, slot;
};

// bricks_sample_c (surfvol.comp:54-96): the brick under the clamped
// position at the column's level, else the next two coarser levels, else
// the coarsest; the cached brick is reused while the position stays in it.
__device__ __forceinline__ float2 surf_brick_sample(const DevScene &s, const SurfBake &b,
                                                   float3 wp, float3 shape, ColCache &c) {
  const uint32_t *page = s.br.page;
  const uint32_t nlev = __ldg(page);
  const float3 bv = make_float3(clamp_(wp.x, 0.0f, fmaxf(shape.x - 0.001f, 0.0f)),
                                clamp_(wp.y, 0.0f, fmaxf(shape.y - 0.001f, 0.0f)),
                                clamp_(wp.z, 0.0f, fmaxf(shape.z - 0.001f, 0.0f)));
  if (c.valid) {
    const float sc = (float)c.scale;
    const float3 lv = make_float3(bv.x / sc, bv.y / sc, bv.z / sc);
    const uint32_t bx = (uint32_t)lv.x >> 7, by = (uint32_t)lv.y >> 7, bz = (uint32_t)lv.z >> 7;
    if (bx == c.bx && by == c.by && bz == c.bz) {
      const SlotCoord q = slot_coord(make_float3(lv.x - (float)(bx << 7), lv.y - (float)(by << 7),
                                                 lv.z - (float)(bz << 7)));
      return make_float2(slot_sample(s, c.slot, q), b.ovl >= 0 ? ovl_fetch(s, b.ovl, c.slot, q) : 0.0f);
    }
  }
  const int desired = (int)min(b.lod, nlev - 1u), last = (int)nlev - 1;
  for (int stp = 0; stp < 4; stp++) {
    const int li = stp < 3 ? desired + stp : last;
    if (li > last || (stp == 3 && li <= desired + 2)) continue;
    const uint32_t h = 4u + (uint32_t)li * 4u;
    const uint32_t off = __ldg(page + h), packed = __ldg(page + h + 1u), scale = __ldg(page + h + 2u);
    const uint32_t dx = packed & 1023u, dy = (packed >> 10) & 1023u, dz = packed >> 20;
    const float sc = (float)scale;
    const float3 lv = make_float3(bv.x / sc, bv.y / sc, bv.z / sc);
    const uint32_t bx = min((uint32_t)lv.x >> 7, dx - 1u), by = min((uint32_t)lv.y >> 7, dy - 1u),
                   bz = min((uint32_t)lv.z >> 7, dz - 1u);
    const uint32_t e = __ldg(page + off + (bz * dy + by) * dx + bx);
    if (e == 0xFFFFFFFFu) continue;
    c.valid = true;
    c.scale = scale;
    c.bx = bx, c.by = by, c.bz = bz;
    c.slot = e & 0xFFFFFFu;
    const SlotCoord q = slot_coord(make_float3(lv.x - (float)(bx << 7), lv.y - (float)(by << 7),
                                               lv.z - (float)(bz << 7)));
    return make_float2(slot_sample(s, c.slot, q), b.ovl >= 0 ? ovl_fetch(s, b.ovl, c.slot, q) : 0.0f);
  }
  c.valid = false;
  return make_float2(0.0f, 0.0f);
}

// One thread per (u, v) column of the band [z0, z1) (surfvol.comp:98-153).
__global__ void k_surf_bake(const __grid_constant__ DevScene s, const __grid_constant__ SurfBake b,
                            uint32_t z0, uint32_t z1) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= b.W || y >= b.H) return;
  const float fu = fmaf((float)x + 0.5f, b.step, b.u0), fv = fmaf((float)y + 0.5f, b.step, b.v0);
  const float gx = fu * b.sx, gy = fv * b.sy;  // grid coordinates
  bool ok = false;
  float3 wp0 = make_float3(0.0f, 0.0f, 0.0f), nrm = wp0;
  if (gx >= 0.0f && gy >= 0.0f && gx <= (float)(b.gw - 1u) && gy <= (float)(b.gh - 1u)) {
    const uint32_t ix = min((uint32_t)gx, b.gw - 2u), iy = min((uint32_t)gy, b.gh - 2u);
    const float fx = gx - (float)ix, fy = gy - (float)iy;
    const size_t i00 = (size_t)iy * b.gw + ix;
    const float4 c00 = b.coords[i00], c10 = b.coords[i00 + 1], c01 = b.coords[i00 + b.gw],
                 c11 = b.coords[i00 + b.gw + 1];
    if (fminf(fminf(c00.w, c10.w), fminf(c01.w, c11.w)) >= 0.5f) {
      wp0 = make_float3(mixf(mixf(c00.x, c10.x, fx), mixf(c01.x, c11.x, fx), fy),
                        mixf(mixf(c00.y, c10.y, fx), mixf(c01.y, c11.y, fx), fy),
                        mixf(mixf(c00.z, c10.z, fx), mixf(c01.z, c11.z, fx), fy));
      const float4 n00 = b.normals[i00], n10 = b.normals[i00 + 1], n01 = b.normals[i00 + b.gw],
                   n11 = b.normals[i00 + b.gw + 1];
      nrm = make_float3(mixf(mixf(n00.x, n10.x, fx), mixf(n01.x, n11.x, fx), fy),
                        mixf(mixf(n00.y, n10.y, fx), mixf(n01.y, n11.y, fx), fy),
                        mixf(mixf(n00.z, n10.z, fx), mixf(n01.z, n11.z, fx), fy));
      const float nl = sqrtf(dot3(nrm, nrm));
      if (nl > 1e-4f) {
        nrm = make_float3(nrm.x / nl, nrm.y / nl, nrm.z / nl);
        ok = true;
      }
    }
  }
  const float3 shape = make_float3((float)__ldg(s.br.page + 1), (float)__ldg(s.br.page + 2),
                                   (float)__ldg(s.br.page + 3));
  // one prediction per column, painted over every layer (surfvol.comp:127-150)
  float pred = -1.0f;
  if (b.pred) {
    const float px = (gx - b.pg0u) * b.pppg, py = (gy - b.pg0v) * b.pppg;
    if (px >= 0.0f && py >= 0.0f && px < (float)b.pw && py < (float)b.ph) pred = pred_sample(b, px, py);
  }
  ColCache c = {false, 1u, 0u, 0u, 0u, 0u};
  for (uint32_t z = z0; z < z1; z++) {
    float2 v = make_float2(0.0f, 0.0f);
    if (ok) {
      const float k = fmaf((float)z - (float)b.nback, b.lstep, b.zoff0);
      const float3 wp = make_float3(fmaf(nrm.x, k, wp0.x), fmaf(nrm.y, k, wp0.y), fmaf(nrm.z, k, wp0.z));
      if (wp.x >= 0.0f && wp.y >= 0.0f && wp.z >= 0.0f && wp.x < shape.x && wp.y < shape.y &&
          wp.z < shape.z)
        v = surf_brick_sample(s, b, wp, shape, c);
    }
    if (pred >= 0.0f) v.y = pred;
    uint8_t *o = b.vol + (((size_t)z * b.H + y) * b.W + x) * 2u;
    o[0] = unorm8(v.x);
    o[1] = unorm8(v.y);
  }
}

struct DevSurfView {
  const uint8_t *vol;  // W x H x L (R, G) texels
  uint32_t W, H, L;
  const float4 *coords;  // segment grid (heatmap taps)
  uint32_t gw, gh;
  const uint8_t *mask;  // supervision mask, or null
  uint32_t mw, mh;
};

// Clamp-to-edge trilinear of the (R, G) volume at normalized uvw.
__device__ __forceinline__ float2 surf_tex(const DevSurfView &v, float u, float w_, float t) {
  const float tx = clamp_(fmaf(u, (float)v.W, -0.5f), 0.0f, (float)(v.W - 1u));
  const float ty = clamp_(fmaf(w_, (float)v.H, -0.5f), 0.0f, (float)(v.H - 1u));
  const float tz = clamp_(fmaf(t, (float)v.L, -0.5f), 0.0f, (float)(v.L - 1u));
  const uint32_t x0 = (uint32_t)tx, y0 = (uint32_t)ty, z0 = (uint32_t)tz;
  const float fx = tx - (float)x0, fy = ty - (float)y0, fz = tz - (float)z0;
  const uint32_t x1 = min(x0 + 1u, v.W - 1u), y1 = min(y0 + 1u, v.H - 1u), z1 = min(z0 + 1u, v.L - 1u);
  const uchar2 *g = reinterpret_cast<const uchar2 *>(v.vol);
  const size_t sy = v.W, sz = (size_t)v.W * v.H;
  const uchar2 a00 = __ldg(g + z0 * sz + y0 * sy + x0), a10 = __ldg(g + z0 * sz + y0 * sy + x1);
  const uchar2 a01 = __ldg(g + z0 * sz + y1 * sy + x0), a11 = __ldg(g + z0 * sz + y1 * sy + x1);
  const uchar2 b00 = __ldg(g + z1 * sz + y0 * sy + x0), b10 = __ldg(g + z1 * sz + y0 * sy + x1);
  const uchar2 b01 = __ldg(g + z1 * sz + y1 * sy + x0), b11 = __ldg(g + z1 * sz + y1 * sy + x1);
  const float r = lerp_(lerp_(lerp_(a00.x, a10.x, fx), lerp_(a01.x, a11.x, fx), fy),
                        lerp_(lerp_(b00.x, b10.x, fx), lerp_(b01.x, b11.x, fx), fy), fz);
  const float gch = lerp_(lerp_(lerp_(a00.y, a10.y, fx), lerp_(a01.y, a11.y, fx), fy),
                          lerp_(lerp_(b00.y, b10.y, fx), lerp_(b01.y, b11.y, fx), fy), fz);
  return make_float2(r * kInv255, gch * kInv255);
}

// flat_overlay_color (raycast.slang:76-81)
__device__ __forceinline__ float3 flat_overlay_color(uint32_t f) {
  if (f & 16u) return make_float3(1.0f, 0.25f, 1.0f);
  if (f & 2u) return make_float3(0.25f, 1.0f, 0.55f);
  if (f & 4u) return make_float3(1.0f, 0.30f, 0.22f);
  return ((f >> 8) & 0xffu) == 1u ? make_float3(0.3f, 0.72f, 1.0f) : make_float3(0.25f, 1.0f, 0.55f);
}

// The surf branch of the raycast (raycast.slang:515-638) for one pixel.
__device__ float3 surf_pixel(const r3d_frame_params &pc, const DevSurfView &v, const float4 *tf,
                             float alpha_cutoff, uint32_t px, uint32_t py) {
  const float3 bg = make_float3(0.02f, 0.02f, 0.03f);
  const float ux = ((float)px + 0.5f) / (float)pc.viewport[0];
  const float uy = ((float)py + 0.5f) / (float)pc.viewport[1];
  const float nx = ux * 2.0f - 1.0f, ny = 1.0f - uy * 2.0f;
  const float fu = fmaf(ny, pc.cam_up[0], fmaf(nx, pc.cam_right[0], pc.cam_origin[0]));
  const float fv = fmaf(ny, pc.cam_up[1], fmaf(nx, pc.cam_right[1], pc.cam_origin[1]));
  const float tx = (fu - pc.slab_x0) / pc.slab_px, ty = (fv - pc.slab_y0) / pc.slab_px;
  if (tx < 0.0f || ty < 0.0f || tx >= pc.slab_nx || ty >= pc.slab_ny) return bg;
  const float L = (float)pc.slab_wz;
  const float center = (pc.slab_z0 - pc.max_mip) + (float)(pc.slab_grid & 0xffffu);
  const float halfd = 0.5f * fmaxf((float)pc.slab_depth, 1.0f);
  const float lo = clamp_(center - halfd, 0.0f, L), hi = clamp_(center + halfd, 0.0f, L);
  if (lo >= hi) return bg;
  const float ix = 1.0f / pc.slab_nx, iy = 1.0f / pc.slab_ny, iz = 1.0f / L;
  if (pc.view_flags & R3D_VIEW_STRETCH) {  // flattening-distortion heatmap (:540-570)
    const float gx = fu * pc.vol_tx, gy = fv * pc.vol_ty;
    const int gix = (int)clamp_(gx, 1.0f, (float)v.gw - 2.0f);
    const int giy = (int)clamp_(gy, 1.0f, (float)v.gh - 2.0f);
    const float4 cu0 = v.coords[(size_t)giy * v.gw + gix - 1], cu1 = v.coords[(size_t)giy * v.gw + gix + 1];
    const float4 cv0 = v.coords[(size_t)(giy - 1) * v.gw + gix], cv1 = v.coords[(size_t)(giy + 1) * v.gw + gix];
    if (fminf(fminf(cu0.w, cu1.w), fminf(cv0.w, cv1.w)) < 0.5f) return bg;
    const float3 du = make_float3(cu1.x - cu0.x, cu1.y - cu0.y, cu1.z - cu0.z);
    const float3 dv = make_float3(cv1.x - cv0.x, cv1.y - cv0.y, cv1.z - cv0.z);
    const float su = sqrtf(dot3(du, du)) * 0.5f * pc.vol_tx;
    const float sv = sqrtf(dot3(dv, dv)) * 0.5f * pc.vol_ty;
    const float x = clamp_(r3d_log2f(fmaxf(0.5f * (su + sv), 1e-4f)) / 0.35f, -1.0f, 1.0f);
    const float m = r3d_powf(fabsf(x), 0.6f);
    const float3 tint = x < 0.0f ? make_float3(0.0f, 0.35f, 1.0f) : make_float3(1.0f, 0.15f, 0.0f);
    const float ct = surf_tex(v, tx * ix, ty * iy, clamp_(center, lo, hi) * iz).x;
    const float k = fmaf(0.5f, ct, 0.5f);
    return make_float3(lerp_(0.95f, tint.x, m) * k, lerp_(0.95f, tint.y, m) * k,
                       lerp_(0.95f, tint.z, m) * k);
  }
  const float dt = fmaxf(pc.step_voxels, 0.25f);  // layers per step
  float t = fmaf(hash12(px, py, pc.frame_index), dt, lo);
  float mip_max = 0.0f, ink_max = 0.0f;
  float acc_r = 0.0f, acc_g = 0.0f, acc_b = 0.0f, acc_a = 0.0f;
  const bool composite = pc.mode != R3D_MODE_MIP;
  const bool ovl = (pc.overlay_flags & 1u) != 0u;
  const float3 oc = flat_overlay_color(pc.overlay_flags);
  const float opac_k = pc.density * pc.step_voxels;
  for (uint32_t k = 0; k < 512u && t < hi; k++, t += dt) {
    const float u = tx * ix, w = ty * iy, z = t * iz;
    const float2 vk = surf_tex(v, u, w, z);
    const float val = vk.x;
    if (ovl && vk.y > ink_max) ink_max = vk.y;
    if (val < pc.threshold) continue;
    if (val > mip_max) mip_max = val;
    if (!composite) continue;
    const float4 sm = tf_sample(tf, clamp_(fmaf(val, 256.0f, -0.5f), 0.0f, 255.0f));
    const float a = 1.0f - r3d_powf(1.0f - sm.w, opac_k);
    if (a <= 0.003f) continue;
    float cr = sm.x, cg = sm.y, cb = sm.z;
    if (pc.mode == R3D_MODE_FULL) {  // 1-texel taps in flattened space
      const float g0 = surf_tex(v, u + ix, w, z).x - surf_tex(v, u - ix, w, z).x;
      const float g1 = surf_tex(v, u, w + iy, z).x - surf_tex(v, u, w - iy, z).x;
      const float g2 = surf_tex(v, u, w, z + iz).x - surf_tex(v, u, w, z - iz).x;
      const float gm = sqrtf(fmaf(g2, g2, fmaf(g1, g1, g0 * g0)));
      if (gm > 1e-4f) {
        const float diff = fmaf(0.7f, fabsf(g2 / gm), 0.3f);  // headlight along the layers
        const float lit = fmaf(0.75f, diff, 0.25f);
        const float lm = lerp_(1.0f, lit, sat_(gm * 6.0f));
        cr *= lm, cg *= lm, cb *= lm;
      }
    }
    if (ovl) {
      const float kk = sat_(vk.y * pc.overlay_gain);
      cr = lerp_(cr, oc.x, kk), cg = lerp_(cg, oc.y, kk), cb = lerp_(cb, oc.z, kk);
    }
    const float wgt = (1.0f - acc_a) * a;
    acc_r = fmaf(wgt, cr, acc_r);
    acc_g = fmaf(wgt, cg, acc_g);
    acc_b = fmaf(wgt, cb, acc_b);
    acc_a = acc_a + wgt;
    if (acc_a >= alpha_cutoff) break;
  }
  float3 col;
  if (composite) {
    const float tr = 1.0f - acc_a;
    col = make_float3(fmaf(tr, bg.x, acc_r), fmaf(tr, bg.y, acc_g), fmaf(tr, bg.z, acc_b));
  } else {
    const float m = mip_max * pc.density;
    col = make_float3(m, m, m);
    if (ovl) {
      const float kk = sat_(ink_max * pc.overlay_gain);
      col = make_float3(lerp_(col.x, oc.x, kk), lerp_(col.y, oc.y, kk), lerp_(col.z, oc.z, kk));
    }
  }
  if ((pc.overlay_flags & 32u) && v.mask) {  // supervision mask, nearest (:619-635)
    const float gx = fu * pc.vol_tx, gy = fv * pc.vol_ty;
    const float upx = (float)v.mw / fmaxf((float)v.gw - 1.0f, 1.0f);
    const float upy = (float)v.mh / fmaxf((float)v.gh - 1.0f, 1.0f);
    const float mxf = gx * upx, myf = gy * upy;
    // int(g * up) truncates toward zero, so (-1, 0) lands on texel 0
    if (mxf > -1.0f && myf > -1.0f && mxf < (float)v.mw && myf < (float)v.mh) {
      const int mx = (int)mxf, my = (int)myf;
      {
        const uint32_t mc = v.mask[(size_t)my * v.mw + mx];
        if (mc == 1u)
          col = make_float3(lerp_(col.x, 0.25f, 0.45f), lerp_(col.y, 0.45f, 0.45f), lerp_(col.z, 1.0f, 0.45f));
        else if (mc >= 2u)
          col = make_float3(lerp_(col.x, 1.0f, 0.55f), lerp_(col.y, 0.55f, 0.55f), lerp_(col.z, 0.10f, 0.55f));
      }
    }
  }
  return col;
}

__global__ void __launch_bounds__(128) k_surf_raycast(const __grid_constant__ r3d_frame_params pc,
                                                      const __grid_constant__ DevSurfView v,
                                                      const uchar4 *__restrict__ lut,
                                                      float alpha_cutoff, uchar4 *__restrict__ img,
                                                      uint32_t out_w, uint32_t *__restrict__ steps_out,
                                                      uint32_t *__restrict__ mip_out) {
  __shared__ float4 tf[256];
  for (uint32_t i = threadIdx.y * blockDim.x + threadIdx.x; i < 256u; i += blockDim.x * blockDim.y) {
    const uchar4 u = lut[i];
    tf[i] = make_float4((float)u.x, (float)u.y, (float)u.z, (float)u.w);
  }
  __syncthreads();
  const bool half = (pc.view_flags & R3D_VIEW_HALF) != 0u;
  const uint32_t tx = blockIdx.x * blockDim.x + threadIdx.x, ty = blockIdx.y * blockDim.y + threadIdx.y;
  const uint32_t px = half ? tx * 2u : tx, py = half ? ty * 2u : ty;
  const uint32_t vw = pc.viewport[0], vh = pc.viewport[1];
  if (px >= vw || py >= vh) return;
  const float3 c = surf_pixel(pc, v, tf, alpha_cutoff, px, py);
  const uchar4 col = make_uchar4(unorm8(c.x), unorm8(c.y), unorm8(c.z), 255);
  const uint32_t ox = pc.view_org & 0xffffu, oy = pc.view_org >> 16;
  for (uint32_t k = 0; k < (half ? 4u : 1u); k++) {
    const uint32_t ax = px + (k & 1u), ay = py + (k >> 1);
    if (ax >= vw || ay >= vh) continue;
    const size_t i = (size_t)(oy + ay) * out_w + (ox + ax);
    img[i] = col;
    if (steps_out) steps_out[i] = 0u;  // no ray-march step counts in this view
    if (mip_out) mip_out[i] = 0u;
  }
}

cudaError_t launch_surf(const r3d_cuda_ctx *c, const r3d_frame_params &pc, uint8_t *img,
                        uint32_t out_w, uint32_t *steps, uint32_t *mip, cudaStream_t st) {
  DevSurfView v;
  v.vol = c->sv_vol;
  v.W = c->sv_W, v.H = c->sv_H, v.L = c->sv_L;
  v.coords = c->surf_coords;
  v.gw = c->surf_gw, v.gh = c->surf_gh;
  v.mask = c->surf_mask;
  v.mw = c->surf_mw, v.mh = c->surf_mh;
  const bool half = (pc.view_flags & R3D_VIEW_HALF) != 0u;
  const uint32_t gw = half ? (pc.viewport[0] + 1u) / 2u : pc.viewport[0];
  const uint32_t gh = half ? (pc.viewport[1] + 1u) / 2u : pc.viewport[1];
  const dim3 threads(16, 8), grid((gw + 15u) / 16u, (gh + 7u) / 8u);
  k_surf_raycast<<<grid, threads, 0, st>>>(pc, v, c->lut, c->alpha_cutoff, (uchar4 *)img, out_w,
                                           steps, mip);
  return cudaGetLastError();
}

}  // namespace r3d

using namespace r3d;

void surf_reset(r3d_cuda_ctx *c) {
  cudaFree(c->surf_coords);
  cudaFree(c->surf_normals);
  cudaFree(c->sv_vol);
  cudaFree(c->surf_mask);
  cudaFree(c->sv_pred);
  c->sv_pred = nullptr;
  c->sv_pw = c->sv_ph = 0;
  c->surf_coords = c->surf_normals = nullptr;
  c->sv_vol = nullptr;
  c->surf_mask = nullptr;
  c->surf_gw = c->surf_gh = c->surf_mw = c->surf_mh = 0;
  c->sv_W = c->sv_H = c->sv_L = 0;
  c->sv_step = 0.0f;
  c->sv_baked = false;
}

static int surf_bake(r3d_cuda_ctx *c) {
  if (!c->sv_vol || c->sv_step <= 0.0f) return R3D_OK;
  if (!c->have_bricks)
    return fail(c, R3D_E_STATE, "surfvol: the bake samples the LOD brick cache");
  if (c->sv_ovl >= 0 && !c->ovl_quad[c->sv_ovl])
    return fail(c, R3D_E_STATE, "surfvol: overlay atlas %d is not loaded", c->sv_ovl);
  SurfBake b;
  b.coords = c->surf_coords;
  b.normals = c->surf_normals;
  b.gw = c->surf_gw, b.gh = c->surf_gh;
  b.u0 = c->sv_u0, b.v0 = c->sv_v0, b.step = c->sv_step, b.zoff0 = c->sv_zoff0;
  b.sx = c->sv_sx, b.sy = c->sv_sy, b.lstep = 1.0f;  // depth stays native-res (vkbackend.c:7026)
  b.W = c->sv_W, b.H = c->sv_H, b.L = c->sv_L, b.nback = c->sv_nback;
  // level of the xy pitch: one per halving down to a 2-voxel step (:7013-7014)
  uint32_t lodq = 0;
  for (float s = c->sv_step; s >= 2.0f && lodq + 1u < c->br.nlev; s *= 0.5f) lodq++;
  b.lod = lodq;
  b.ovl = c->sv_ovl;
  b.vol = c->sv_vol;
  b.pred = c->sv_pred;
  b.pw = c->sv_pw, b.ph = c->sv_ph;
  b.pg0u = c->sv_pg0u, b.pg0v = c->sv_pg0v, b.pppg = c->sv_pppg;
  const dim3 threads(8, 8), grid((b.W + 7u) / 8u, (b.H + 7u) / 8u);
  k_surf_bake<<<grid, threads, 0, c->stream>>>(c->scene(), b, 0u, b.L);
  R3D_CUDA_TRY(c, cudaGetLastError());
  c->sv_baked = true;
  return R3D_OK;
}

extern "C" {

int r3d_cuda_surf_begin(r3d_cuda_ctx *c, uint32_t w, uint32_t h, const float *coords_rgba,
                        const float *normals_rgba) {
  if (!c || w < 3u || h < 3u || !coords_rgba || !normals_rgba)
    return fail(c, R3D_E_INVALID, "surf_begin: a grid of at least 3 x 3 points and both grids");
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  const size_t bytes = (size_t)w * h * sizeof(float4);
  float4 *cd = nullptr, *nd = nullptr;
  cudaError_t e = cudaMalloc(&cd, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&nd, bytes);
  if (e == cudaSuccess) e = copy_sync(c->stream, cd, coords_rgba, bytes);
  if (e == cudaSuccess) e = copy_sync(c->stream, nd, normals_rgba, bytes);
  if (e != cudaSuccess) {
    cudaFree(cd);
    cudaFree(nd);
    return cuda_fail(c, e, "surf_begin");
  }
  cudaFree(c->surf_coords);
  cudaFree(c->surf_normals);
  c->surf_coords = cd;
  c->surf_normals = nd;
  c->surf_gw = w, c->surf_gh = h;
  return surf_bake(c);  // a window already set re-bakes from the new grids
}

int r3d_cuda_surfvol_begin(r3d_cuda_ctx *c, uint32_t w, uint32_t h, uint32_t layers,
                           uint32_t nback, float sx, float sy) {
  if (!c || !w || !h || !layers || !(sx > 0.0f) || !(sy > 0.0f))
    return fail(c, R3D_E_INVALID, "surfvol_begin: bad arguments");
  if (!c->surf_coords) return fail(c, R3D_E_STATE, "surfvol_begin: no surface grids");
  if (w > 16384u || h > 16384u || layers > 2048u)
    return fail(c, R3D_E_INVALID, "surfvol_begin: %ux%ux%u window too large", w, h, layers);
  if (nback >= layers) nback = layers / 2u;  // vkbackend.c:1765
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  cudaFree(c->sv_vol);
  c->sv_vol = nullptr;
  const size_t bytes = (size_t)w * h * layers * 2u;
  R3D_CUDA_TRY(c, cudaMalloc(&c->sv_vol, bytes));
  R3D_CUDA_TRY(c, cudaMemsetAsync(c->sv_vol, 0, bytes, c->stream));
  c->sv_W = w, c->sv_H = h, c->sv_L = layers, c->sv_nback = nback;
  c->sv_sx = sx, c->sv_sy = sy;
  c->sv_step = 0.0f;  // no window yet
  c->sv_baked = false;
  return R3D_OK;
}

int r3d_cuda_surfvol_window(r3d_cuda_ctx *c, double u0, double v0, float step, float zoff0) {
  if (!c) return R3D_E_INVALID;
  if (!c->sv_vol) return fail(c, R3D_E_STATE, "surfvol_window: no surface volume");
  if (!(step > 0.0f)) return fail(c, R3D_E_INVALID, "surfvol_window: step must be > 0");
  cudaSetDevice(c->device);
  c->sv_u0 = (float)u0, c->sv_v0 = (float)v0, c->sv_step = step, c->sv_zoff0 = zoff0;
  return surf_bake(c);
}

int r3d_cuda_surfvol_overlay(r3d_cuda_ctx *c, int atlas) {
  if (!c || atlas < -1 || atlas > 3 || atlas == 2)
    return fail(c, R3D_E_INVALID, "surfvol_overlay: atlas %d (ink 0, 3D ink 1, registration 3, "
                                  "none -1)", atlas);
  cudaSetDevice(c->device);
  c->sv_ovl = atlas;
  return surf_bake(c);
}

int r3d_cuda_surfvol_inkpred(r3d_cuda_ctx *c, const float *pred, uint32_t w, uint32_t h, float g0u,
                             float g0v, float px_per_grid) {
  if (!c) return R3D_E_INVALID;
  if (!c->sv_vol) return fail(c, R3D_E_STATE, "surfvol_inkpred: no surface volume");
  cudaSetDevice(c->device);
  if (!pred) {  // clear (vkbackend.c:1963-1968): re-bake without it
    if (!c->sv_pred) return R3D_OK;
    R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    cudaFree(c->sv_pred);
    c->sv_pred = nullptr;
    c->sv_pw = c->sv_ph = 0;
    return surf_bake(c);
  }
  if (!w || !h || !(px_per_grid > 0.0f))
    return fail(c, R3D_E_INVALID, "surfvol_inkpred: a %ux%u prediction at %g texels per grid unit",
                w, h, (double)px_per_grid);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  const size_t bytes = (size_t)w * h * sizeof(float);
  if (c->sv_pw != w || c->sv_ph != h) {  // size change: a new buffer
    cudaFree(c->sv_pred);
    c->sv_pred = nullptr;
    c->sv_pw = c->sv_ph = 0;
    R3D_CUDA_TRY(c, cudaMalloc(&c->sv_pred, bytes));
  }
  R3D_CUDA_TRY(c, copy_sync(c->stream, c->sv_pred, pred, bytes));
  c->sv_pw = w, c->sv_ph = h;
  c->sv_pg0u = g0u, c->sv_pg0v = g0v, c->sv_pppg = px_per_grid;
  return surf_bake(c);  // repaint the window with the new probabilities
}

int r3d_cuda_surfvol_mark(r3d_cuda_ctx *c) {
  if (!c) return R3D_E_INVALID;
  cudaSetDevice(c->device);
  return surf_bake(c);
}

void r3d_cuda_surfvol_params(const r3d_cuda_ctx *c, r3d_frame_params *p) {
  if (!c || !p || !c->sv_vol) return;
  // vkbackend.c:2054-2066
  p->slab_x0 = c->sv_u0;
  p->slab_y0 = c->sv_v0;
  p->slab_px = c->sv_step;
  p->slab_nx = (float)c->sv_W;
  p->slab_ny = (float)c->sv_H;
  p->slab_wz = c->sv_L;
  p->slab_grid = c->sv_nback;
  p->max_mip = c->sv_zoff0;
  p->vol_tx = c->sv_sx;
  p->vol_ty = c->sv_sy;
  p->view_flags |= R3D_VIEW_SURF;
}

int r3d_cuda_surfvol_read(r3d_cuda_ctx *c, uint8_t *out) {
  if (!c || !out) return R3D_E_INVALID;
  if (!c->sv_vol) return fail(c, R3D_E_STATE, "surfvol_read: no surface volume");
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  R3D_CUDA_TRY(c, cudaMemcpy(out, c->sv_vol, (size_t)c->sv_W * c->sv_H * c->sv_L * 2u,
                             cudaMemcpyDeviceToHost));
  return R3D_OK;
}

int r3d_cuda_surfmask(r3d_cuda_ctx *c, const uint8_t *m, uint32_t w, uint32_t h) {
  if (!c) return R3D_E_INVALID;
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  cudaFree(c->surf_mask);
  c->surf_mask = nullptr;
  c->surf_mw = c->surf_mh = 0;
  if (!m || !w || !h) return R3D_OK;  // cleared
  R3D_CUDA_TRY(c, cudaMalloc(&c->surf_mask, (size_t)w * h));
  R3D_CUDA_TRY(c, copy_sync(c->stream, c->surf_mask, m, (size_t)w * h));
  c->surf_mw = w, c->surf_mh = h;
  return R3D_OK;
}

}  // extern "C"
