/* CPU oracle of the differentiable raycast (test infrastructure).
 *
 * The differentiable render is render3d's emission-absorption compositing
 * (the FLAT mode of src/shaders/raycast.slang:894-1017, no shading) over an
 * FP32 density grid and an FP32 256x4 transfer function: trilinear density
 * at texel centres (clamp to edge, level 0, no empty-space skip), TF lookup
 * at v*256-0.5, alpha clamped to [0, 1], opacity correction
 * a = 1 - (1 - alpha)^(density * step * lod_step), samples with a <= 0.003
 * ignored, front-to-back compositing with termination at the cutoff, then
 * the background.  Ray setup is the cube path of the plain raycast.
 *
 * orc_diff_forward32 evaluates it in FP32 exactly as the sm_100a kernel does.
 * orc_diff_grad64 evaluates the same render in FP64 and its exact adjoint
 * (reverse mode over the stored samples) for the loss gradient dL/drgb:
 * gradients with respect to every voxel, every LUT entry and the density
 * scale.  With decisions32 set, which samples contribute and where a ray
 * terminates are taken from the FP32 render (of dec_dens / dec_lut when
 * given, so finite differences can hold them fixed), and so is each sample's
 * piece of the piecewise-smooth render: its trilinear cell, its TF texel and
 * whether the TF coordinate and alpha lie inside their clamps.  The FP64
 * gradient is then that of the same branch and piece the FP32 kernel
 * differentiates: where a sample sits within rounding of a texel boundary,
 * FP32 and FP64 arithmetic can pick neighbouring texels, whose slopes differ
 * by the full LUT step; otherwise the FP64 render decides. */
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "r3d_fmath.h"
#include "r3d_oracle.h"

typedef struct dv3 {
  double x, y, z;
} dv3;

static inline float clampf_(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }
static inline float lerpf_(float a, float b, float t) { return fmaf(t, b - a, a); }
static inline float dot3f(const float a[3], const float b[3]) {
  return fmaf(a[2], b[2], fmaf(a[1], b[1], a[0] * b[0]));
}

static float hash12(uint32_t px, uint32_t py, uint32_t frame) {
  uint32_t h = px * 374761393u + py * 668265263u + frame * 2246822519u;
  h = (h ^ (h >> 13)) * 1274126177u;
  return (float)(h >> 8) * (1.0f / 16777216.0f);
}

/* ray setup of the cube path (raycast.slang:640-748), FP32 as the kernels */
typedef struct ray32 {
  float ro[3], dir[3];
  float t0, tf, dt, span;
  int hit;
} ray32;

static void setup32(const r3d_frame_params *pc, uint32_t nmax, uint32_t px, uint32_t py,
                    ray32 *r) {
  int ortho = (pc->view_flags & R3D_VIEW_ORTHO) != 0u;
  float ux = ((float)px + 0.5f) / (float)pc->viewport[0];
  float uy = ((float)py + 0.5f) / (float)pc->viewport[1];
  float nx = ux * 2.0f - 1.0f, ny = 1.0f - uy * 2.0f;
  const float *fw = pc->cam_forward, *rt = pc->cam_right, *up = pc->cam_up;
  float d[3];
  if (ortho) {
    d[0] = fw[0], d[1] = fw[1], d[2] = fw[2];
  } else {
    for (int a = 0; a < 3; a++) d[a] = fmaf(ny, up[a], fmaf(nx, rt[a], fw[a]));
  }
  float inv = 1.0f / sqrtf(dot3f(d, d));
  for (int a = 0; a < 3; a++) d[a] = d[a] * inv;
  float o[3] = {pc->cam_origin[0], pc->cam_origin[1], pc->cam_origin[2]};
  if (ortho)
    for (int a = 0; a < 3; a++) o[a] = fmaf(ny, up[a], fmaf(nx, rt[a], o[a]));
  const float c = 0.5f;
  float q[3] = {(o[0] - pc->vol_tx) - c, (o[1] - pc->vol_ty) - c, (o[2] - pc->vol_tz) - c};
  const float *r0 = pc->vol_r0, *r1 = pc->vol_r1, *r2 = pc->vol_r2;
  for (int a = 0; a < 3; a++) {
    r->ro[a] = fmaf(r2[a], q[2], fmaf(r1[a], q[1], r0[a] * q[0])) + c;
    r->dir[a] = fmaf(r2[a], d[2], fmaf(r1[a], d[1], r0[a] * d[0]));
  }
  float tmn[3], tmx[3];
  for (int a = 0; a < 3; a++) {
    float iv = 1.0f / r->dir[a];
    float t0 = (0.0f - r->ro[a]) * iv, t1 = (1.0f - r->ro[a]) * iv;
    tmn[a] = fminf(t0, t1);
    tmx[a] = fmaxf(t0, t1);
  }
  float tn = fmaxf(fmaxf(fmaxf(tmn[0], tmn[1]), tmn[2]), 0.0f);
  float tf = fminf(fminf(fminf(tmx[0], tmx[1]), tmx[2]), 1e30f);
  r->hit = !(tn >= tf);
  float voxel = 1.0f / (float)nmax;
  r->dt = pc->step_voxels * voxel;
  r->t0 = fmaf(hash12(px, py, pc->frame_index), r->dt, tn);
  r->tf = tf;
  r->span = fmaxf((tf - tn) / (4096.0f * r->dt), 1.0f);
}

/* FP32 trilinear of an FP32 grid; also returns the base texel / weights */
static float tri32(const float *g, const uint32_t n[3], const float p[3], uint32_t *idx8,
                   float *w8) {
  float t[3];
  uint32_t i0[3], i1[3];
  float f[3];
  for (int a = 0; a < 3; a++) {
    t[a] = clampf_(fmaf(p[a], (float)n[a], -0.5f), 0.0f, (float)(n[a] - 1u));
    i0[a] = (uint32_t)t[a];
    f[a] = t[a] - (float)i0[a];
    i1[a] = i0[a] + 1u < n[a] ? i0[a] + 1u : n[a] - 1u;
  }
  size_t sy = n[0], sz = (size_t)n[0] * n[1];
#define G(X, Y, Z) g[(size_t)(X) + (size_t)(Y)*sy + (size_t)(Z)*sz]
  float c00 = lerpf_(G(i0[0], i0[1], i0[2]), G(i1[0], i0[1], i0[2]), f[0]);
  float c10 = lerpf_(G(i0[0], i1[1], i0[2]), G(i1[0], i1[1], i0[2]), f[0]);
  float c01 = lerpf_(G(i0[0], i0[1], i1[2]), G(i1[0], i0[1], i1[2]), f[0]);
  float c11 = lerpf_(G(i0[0], i1[1], i1[2]), G(i1[0], i1[1], i1[2]), f[0]);
#undef G
  if (idx8) {
    for (int k = 0; k < 8; k++) {
      uint32_t X = k & 1 ? i1[0] : i0[0], Y = k & 2 ? i1[1] : i0[1], Z = k & 4 ? i1[2] : i0[2];
      idx8[k] = (uint32_t)(X + Y * sy + Z * sz);
      w8[k] = (k & 1 ? f[0] : 1.0f - f[0]) * (k & 2 ? f[1] : 1.0f - f[1]) *
              (k & 4 ? f[2] : 1.0f - f[2]);
    }
  }
  return lerpf_(lerpf_(c00, c10, f[1]), lerpf_(c01, c11, f[1]), f[2]);
}

/* One FP32 ray: colour and, if rec != NULL, the steps of the contributing
 * samples in order (returns their count). */
static uint32_t ray_fwd32(const r3d_frame_params *pc, const float *dens, const uint32_t n[3],
                          const float *lut, float cutoff, uint32_t px, uint32_t py,
                          float rgb[3], uint32_t *rec, uint32_t rec_cap, uint32_t *steps_out) {
  uint32_t nmax = n[0] > n[1] ? n[0] : n[1];
  if (n[2] > nmax) nmax = n[2];
  ray32 r;
  setup32(pc, nmax, px, py, &r);
  float acc[4] = {0, 0, 0, 0};
  uint32_t nrec = 0, steps = 0;
  if (r.hit) {
    const float k = pc->density * pc->step_voxels;
    float t = r.t0;
    while (t < r.tf && steps < 4096u) {
      steps++;
      float p[3] = {fmaf(t, r.dir[0], r.ro[0]), fmaf(t, r.dir[1], r.ro[1]),
                    fmaf(t, r.dir[2], r.ro[2])};
      float v = tri32(dens, n, p, NULL, NULL);
      if (!(v < pc->threshold)) {
        float tt = clampf_(fmaf(v, 256.0f, -0.5f), 0.0f, 255.0f);
        uint32_t i0 = (uint32_t)tt, i1 = i0 + 1u < 256u ? i0 + 1u : 255u;
        float f = tt - (float)i0;
        float s[4];
        for (int c = 0; c < 4; c++) s[c] = lerpf_(lut[i0 * 4 + c], lut[i1 * 4 + c], f);
        float alpha = clampf_(s[3], 0.0f, 1.0f);
        float a = 1.0f - r3d_powf(1.0f - alpha, k * r.span);
        if (a > 0.003f) {
          float w = (1.0f - acc[3]) * a;
          for (int c = 0; c < 3; c++) acc[c] = fmaf(w, s[c], acc[c]);
          acc[3] = acc[3] + w;
          if (rec && nrec < rec_cap) rec[nrec] = steps;
          nrec++;
          if (acc[3] >= cutoff) break;
        }
      }
      t = fmaf(r.dt, r.span, t);
    }
  }
  float tr = 1.0f - acc[3];
  rgb[0] = fmaf(tr, 0.02f, acc[0]);
  rgb[1] = fmaf(tr, 0.02f, acc[1]);
  rgb[2] = fmaf(tr, 0.03f, acc[2]);
  if (steps_out) *steps_out = steps;
  return nrec;
}

int orc_diff_forward32(const r3d_frame_params *pc, const float *dens, const uint32_t n[3],
                       const float *lut, float cutoff, float *rgb_out, uint32_t *steps_out,
                       int threads) {
  uint32_t w = pc->viewport[0], h = pc->viewport[1];
  if (!w || !h || pc->brick_mode || (pc->view_flags & ~R3D_VIEW_ORTHO)) return -1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (uint32_t y = 0; y < h; y++)
    for (uint32_t x = 0; x < w; x++)
      ray_fwd32(pc, dens, n, lut, cutoff, x, y, rgb_out + ((size_t)y * w + x) * 3, NULL, 0,
                steps_out ? steps_out + (size_t)y * w + x : NULL);
  return 0;
}

/* ----------------------------------------------------------- FP64 twin */

typedef struct samp64 {
  double tprev;  /* transmittance before the sample */
  double a, col[3], alpha, kk, kstep; /* kk = density * kstep */
  int alpha_free;  /* 0 < alpha < 1 (not clamped) */
  double tt;
  uint32_t i0, i1;
  double f;
  int tt_free;  /* 0 < tt < 255 */
  uint32_t idx8[8];
  double w8[8];
} samp64;

/* FP64 trilinear; cell0 (nullable) forces the base texel of each axis (the
 * FP32 sample's cell, whose piece of the piecewise-trilinear function is
 * then differentiated; the weights extend that piece linearly). */
static double tri64(const float *g, const uint32_t n[3], const double p[3],
                    const uint32_t *cell0, uint32_t *idx8, double *w8) {
  double t[3], f[3];
  uint32_t i0[3], i1[3];
  for (int a = 0; a < 3; a++) {
    t[a] = p[a] * (double)n[a] - 0.5;
    if (t[a] < 0.0) t[a] = 0.0;
    if (t[a] > (double)(n[a] - 1u)) t[a] = (double)(n[a] - 1u);
    i0[a] = cell0 ? cell0[a] : (uint32_t)t[a];
    f[a] = t[a] - (double)i0[a];
    i1[a] = i0[a] + 1u < n[a] ? i0[a] + 1u : n[a] - 1u;
  }
  size_t sy = n[0], sz = (size_t)n[0] * n[1];
  double v = 0.0;
  for (int k = 0; k < 8; k++) {
    uint32_t X = k & 1 ? i1[0] : i0[0], Y = k & 2 ? i1[1] : i0[1], Z = k & 4 ? i1[2] : i0[2];
    double wk = (k & 1 ? f[0] : 1.0 - f[0]) * (k & 2 ? f[1] : 1.0 - f[1]) *
                (k & 4 ? f[2] : 1.0 - f[2]);
    size_t id = X + Y * sy + Z * sz;
    v += wk * (double)g[id];
    idx8[k] = (uint32_t)id;
    w8[k] = wk;
  }
  return v;
}

/* The FP32 render's pieces at one sample: the trilinear cell, the TF texel
 * and whether the TF coordinate and alpha are inside their clamps (these
 * choose the smooth piece of the FP32 function the kernel differentiates). */
typedef struct piece32 {
  uint32_t cell[3], texel;
  int tt_free, alpha_free;
} piece32;

static void pieces32(const float *dens, const uint32_t n[3], const float *lut, const float p[3],
                     piece32 *o) {
  for (int a = 0; a < 3; a++)
    o->cell[a] = (uint32_t)clampf_(fmaf(p[a], (float)n[a], -0.5f), 0.0f, (float)(n[a] - 1u));
  const float v = tri32(dens, n, p, NULL, NULL);
  const float tu = fmaf(v, 256.0f, -0.5f), tt = clampf_(tu, 0.0f, 255.0f);
  o->texel = (uint32_t)tt;
  o->tt_free = tu > 0.0f && tu < 255.0f;
  const uint32_t i1 = o->texel + 1u < 256u ? o->texel + 1u : 255u;
  const float s3 = lerpf_(lut[o->texel * 4 + 3], lut[i1 * 4 + 3], tt - (float)o->texel);
  o->alpha_free = s3 > 0.0f && s3 < 1.0f;
}

/* Builds the FP64 sample list of one ray.  rec (decisions32): the
 * contributing steps from the FP32 render of (pdens, plut), whose pieces
 * (pieces32) the FP64 samples also keep; else everything is decided in FP64.
 * Returns count. */
static uint32_t ray_samples64(const r3d_frame_params *pc, const float *dens, const uint32_t n[3],
                              const float *lut, double density, float cutoff, uint32_t px,
                              uint32_t py, const uint32_t *rec, uint32_t nrec,
                              const float *pdens, const float *plut, samp64 *out,
                              uint32_t cap, double rgb[3]) {
  uint32_t nmax = n[0] > n[1] ? n[0] : n[1];
  if (n[2] > nmax) nmax = n[2];
  ray32 r; /* ray geometry and the step sequence are the FP32 ones */
  setup32(pc, nmax, px, py, &r);
  double A = 0.0, C[3] = {0, 0, 0};
  uint32_t ns = 0;
  if (r.hit) {
    double kstep = (double)pc->step_voxels * (double)r.span;
    double kk = density * kstep;
    float t = r.t0;
    uint32_t steps = 0, ri = 0;
    while (t < r.tf && steps < 4096u) {
      steps++;
      int consider = rec ? (ri < nrec && rec[ri] == steps) : 1;
      if (consider) {
        const float p32[3] = {fmaf(t, r.dir[0], r.ro[0]), fmaf(t, r.dir[1], r.ro[1]),
                              fmaf(t, r.dir[2], r.ro[2])};
        double p[3] = {(double)p32[0], (double)p32[1], (double)p32[2]};
        piece32 pc32;
        if (rec) pieces32(pdens, n, plut, p32, &pc32);
        samp64 s;
        double v = tri64(dens, n, p, rec ? pc32.cell : NULL, s.idx8, s.w8);
        int contrib = 0;
        if (rec || !(v < (double)pc->threshold)) {
          double tt = v * 256.0 - 0.5;
          s.tt_free = rec ? pc32.tt_free : (tt > 0.0 && tt < 255.0);
          if (tt < 0.0) tt = 0.0;
          if (tt > 255.0) tt = 255.0;
          s.i0 = rec ? pc32.texel : (uint32_t)tt;
          s.i1 = s.i0 + 1u < 256u ? s.i0 + 1u : 255u;
          s.f = tt - (double)s.i0;
          s.tt = tt;
          double sv[4];
          for (int c = 0; c < 4; c++)
            sv[c] = (double)lut[s.i0 * 4 + c] +
                    s.f * ((double)lut[s.i1 * 4 + c] - (double)lut[s.i0 * 4 + c]);
          double alpha = sv[3] < 0.0 ? 0.0 : (sv[3] > 1.0 ? 1.0 : sv[3]);
          s.alpha_free = rec ? pc32.alpha_free : (sv[3] > 0.0 && sv[3] < 1.0);
          s.alpha = alpha;
          s.kk = kk;
          s.kstep = kstep;
          s.a = 1.0 - pow(1.0 - alpha, kk);
          for (int c = 0; c < 3; c++) s.col[c] = sv[c];
          contrib = rec ? 1 : s.a > 0.003;
        }
        if (contrib) {
          if (rec) ri++;
          s.tprev = 1.0 - A;
          double w = s.tprev * s.a;
          for (int c = 0; c < 3; c++) C[c] += w * s.col[c];
          A += w;
          if (ns < cap) out[ns] = s;
          ns++;
          if (rec ? ri >= nrec : A >= (double)cutoff) break;
        }
      }
      t = fmaf(r.dt, r.span, t);
    }
  }
  double tr = 1.0 - A;
  rgb[0] = C[0] + tr * 0.02;
  rgb[1] = C[1] + tr * 0.02;
  rgb[2] = C[2] + tr * 0.03;
  return ns;
}

int orc_diff_grad64(const r3d_frame_params *pc, const float *dens, const uint32_t n[3],
                    const float *lut, float cutoff, const float *dl_drgb, int decisions32,
                    const float *dec_dens, const float *dec_lut, double *g_dens, double *g_lut,
                    double *g_density, double *rgb64_out, int threads) {
  uint32_t w = pc->viewport[0], h = pc->viewport[1];
  if (!w || !h || pc->brick_mode || (pc->view_flags & ~R3D_VIEW_ORTHO)) return -1;
  const double density = (double)pc->density;
  int nt = threads > 0 ? threads : omp_get_max_threads();
  size_t nvox = (size_t)n[0] * n[1] * n[2];
  int fail = 0;
#pragma omp parallel num_threads(nt)
  {
    samp64 *buf = malloc(sizeof(samp64) * 4096);
    uint32_t *rec = malloc(sizeof(uint32_t) * 4096);
    double *gl = calloc(256 * 4, sizeof(double));
    double gd = 0.0;
    if (!buf || !rec || !gl) fail = 1;
#pragma omp for schedule(dynamic, 1)
    for (uint32_t y = 0; y < h; y++) {
      if (fail) continue;
      for (uint32_t x = 0; x < w; x++) {
        size_t pix = (size_t)y * w + x;
        uint32_t nrec = 0;
        if (decisions32) {
          float rgb32[3];
          nrec = ray_fwd32(pc, dec_dens ? dec_dens : dens, n, dec_lut ? dec_lut : lut, cutoff, x,
                           y, rgb32, rec, 4096, NULL);
        }
        double rgb[3];
        uint32_t ns = ray_samples64(pc, dens, n, lut, density, cutoff, x, y,
                                    decisions32 ? rec : NULL, nrec, dec_dens ? dec_dens : dens,
                                    dec_lut ? dec_lut : lut, buf, 4096, rgb);
        if (rgb64_out)
          for (int c = 0; c < 3; c++) rgb64_out[pix * 3 + c] = rgb[c];
        const float *g = dl_drgb + pix * 3;
        double S[3] = {0.02, 0.02, 0.03};
        for (uint32_t i = ns; i-- > 0;) {
          const samp64 *s = &buf[i];
          double dc[3], da = 0.0;
          for (int c = 0; c < 3; c++) {
            dc[c] = (double)g[c] * s->tprev * s->a;
            da += (double)g[c] * s->tprev * (s->col[c] - S[c]);
          }
          for (int c = 0; c < 3; c++) S[c] = s->a * s->col[c] + (1.0 - s->a) * S[c];
          double dalpha = 0.0;
          if (s->alpha_free) dalpha = da * s->kk * pow(1.0 - s->alpha, s->kk - 1.0);
          if (s->alpha < 1.0) gd += da * (-(1.0 - s->a) * log(1.0 - s->alpha)) * s->kstep;
          double ds[4] = {dc[0], dc[1], dc[2], dalpha};
          double dv = 0.0;
          for (int c = 0; c < 4; c++) {
            gl[s->i0 * 4 + c] += ds[c] * (1.0 - s->f);
            gl[s->i1 * 4 + c] += ds[c] * s->f;
            if (s->tt_free) dv += ds[c] * ((double)lut[s->i1 * 4 + c] - (double)lut[s->i0 * 4 + c]) * 256.0;
          }
          if (dv != 0.0)
            for (int k = 0; k < 8; k++) {
              double add = dv * s->w8[k];
#pragma omp atomic
              g_dens[s->idx8[k]] += add;
            }
        }
      }
    }
#pragma omp critical
    {
      for (int i = 0; i < 256 * 4; i++) g_lut[i] += gl[i];
      *g_density += gd;
    }
    free(buf);
    free(rec);
    free(gl);
  }
  (void)nvox;
  return fail ? -1 : 0;
}
