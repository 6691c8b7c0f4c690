/* Host-side raycast inputs (camera, TF, LOD policy, bench orbit) and the
 * seeded scroll phantom.  Compiled with -ffp-contract=off so the float
 * results equal the reference core's (src/core/camera.c, transfer.c,
 * lod.h, mathx.h) bit for bit. */
#include "r3d_host.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ---- vector helpers in the evaluation order of src/core/mathx.h ---- */

static float dot3(const float a[3], const float b[3]) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static void cross3(const float a[3], const float b[3], float o[3]) {
  float x = a[1] * b[2] - a[2] * b[1], y = a[2] * b[0] - a[0] * b[2], z = a[0] * b[1] - a[1] * b[0];
  o[0] = x, o[1] = y, o[2] = z;
}
static void norm3(float a[3]) {
  float l = sqrtf(dot3(a, a));
  if (l > 0.0f) {
    float s = 1.0f / l;
    a[0] *= s, a[1] *= s, a[2] *= s;
  } else {
    a[0] = a[1] = a[2] = 0.0f;
  }
}
static float clampf_(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }

/* ---- camera (src/core/camera.c) ---- */

#define PITCH_LIMIT 1.55334303f /* pi/2 - 1 degree */

void r3d_host_camera_init(r3d_host_camera *c, const float pos[3]) {
  memset(c, 0, sizeof *c);
  memcpy(c->pos, pos, sizeof c->pos);
  c->fov_y = 1.04719755f; /* 60 degrees */
}

static void forward_of(const r3d_host_camera *c, float f[3]) {
  float cp = cosf(c->pitch);
  f[0] = sinf(c->yaw) * cp;
  f[1] = sinf(c->pitch);
  f[2] = cosf(c->yaw) * cp;
}

static void flat_right(const float fwd[3], float r[3]) {
  static const float wup[3] = {0.0f, 1.0f, 0.0f};
  cross3(fwd, wup, r);
  norm3(r);
  if (sqrtf(dot3(r, r)) == 0.0f) r[0] = 1.0f, r[1] = 0.0f, r[2] = 0.0f;
}

void r3d_host_camera_move(r3d_host_camera *c, const float local[3], float dist) {
  float f[3], r[3];
  forward_of(c, f);
  flat_right(f, r);
  for (int a = 0; a < 3; a++) {
    float up = a == 1 ? 1.0f : 0.0f;
    float d = (r[a] * local[0] + up * local[1]) + f[a] * local[2];
    c->pos[a] = c->pos[a] + d * dist;
  }
}

void r3d_host_camera_look(r3d_host_camera *c, float dyaw, float dpitch) {
  c->yaw += dyaw;
  c->pitch = clampf_(c->pitch + dpitch, -PITCH_LIMIT, PITCH_LIMIT);
}

static void orbit_sync(r3d_host_camera *c) {
  float f[3];
  forward_of(c, f);
  for (int a = 0; a < 3; a++) c->pos[a] = c->target[a] - f[a] * c->dist;
}

void r3d_host_camera_orbit_set(r3d_host_camera *c, const float target[3], float dist) {
  memcpy(c->target, target, sizeof c->target);
  c->dist = dist;
  orbit_sync(c);
}

void r3d_host_camera_orbit_drag(r3d_host_camera *c, float dyaw, float dpitch) {
  r3d_host_camera_look(c, dyaw, dpitch);
  orbit_sync(c);
}

void r3d_host_camera_orbit_zoom(r3d_host_camera *c, float factor) {
  c->dist = clampf_(c->dist * factor, 0.0005f, 20.0f);
  orbit_sync(c);
}

void r3d_host_camera_basis(const r3d_host_camera *c, float aspect, float right[3], float up[3],
                           float fwd[3]) {
  float f[3], r[3], u[3];
  forward_of(c, f);
  flat_right(f, r);
  cross3(r, f, u);
  float t = tanf(c->fov_y * 0.5f);
  float ta = t * aspect;
  for (int a = 0; a < 3; a++) {
    right[a] = r[a] * ta;
    up[a] = u[a] * t;
    fwd[a] = f[a];
  }
}

/* src/core/mathx.h:34-43 */
void r3d_host_m3_ypr(float yaw, float pitch, float roll, float m[3][3]) {
  float cy = cosf(yaw), sy = sinf(yaw), cp = cosf(pitch), sp = sinf(pitch), cr = cosf(roll),
        sr = sinf(roll);
  m[0][0] = cy * cr + sy * sp * sr;
  m[0][1] = -cy * sr + sy * sp * cr;
  m[0][2] = sy * cp;
  m[1][0] = cp * sr;
  m[1][1] = cp * cr;
  m[1][2] = -sp;
  m[2][0] = -sy * cr + cy * sp * sr;
  m[2][1] = sy * sr + cy * sp * cr;
  m[2][2] = cy * cp;
}

/* ---- transfer function (src/core/transfer.c) ---- */

void r3d_host_tf_build(const uint8_t *values, const uint8_t (*rgba)[4], uint32_t npts,
                       uint8_t lut[256][4]) {
  if (!npts) return;
  for (uint32_t i = 0; i < 256u; i++) {
    uint32_t lo = 0, hi = npts - 1u;
    for (uint32_t k = 0; k + 1u < npts; k++) {
      if (values[k] <= i && i <= values[k + 1u]) {
        lo = k;
        hi = k + 1u;
        break;
      }
    }
    uint32_t span = (uint32_t)values[hi] - (uint32_t)values[lo];
    uint32_t num = span ? i - values[lo] : 0u, den = span ? span : 1u;
    for (int ch = 0; ch < 4; ch++) {
      uint32_t a = rgba[lo][ch], b = rgba[hi][ch];
      lut[i][ch] = (uint8_t)((a * (den - num) + b * num) / den);
    }
  }
}

typedef struct preset_pt {
  uint8_t v, c[4];
} preset_pt;

static const preset_pt P_GREY[] = {{0, {0, 0, 0, 0}}, {255, {255, 255, 255, 255}}};
static const preset_pt P_SCROLL[] = {{0, {0, 0, 0, 0}},
                                     {40, {0, 0, 0, 0}},
                                     {90, {150, 110, 70, 40}},
                                     {160, {230, 190, 130, 160}},
                                     {255, {255, 250, 240, 255}}};
static const preset_pt P_HIGHPASS[] = {{0, {0, 0, 0, 0}},
                                       {120, {0, 0, 0, 0}},
                                       {180, {200, 200, 255, 120}},
                                       {255, {255, 255, 255, 255}}};

uint32_t r3d_host_tf_preset(uint32_t idx, uint8_t lut[256][4]) {
  const preset_pt *p;
  uint32_t n;
  switch (idx) {
    case 0: p = P_GREY, n = 2; break;
    case 1: p = P_SCROLL, n = 5; break;
    case 2: p = P_HIGHPASS, n = 4; break;
    default: return 3u;
  }
  uint8_t vals[8], cols[8][4];
  for (uint32_t k = 0; k < n; k++) {
    vals[k] = p[k].v;
    memcpy(cols[k], p[k].c, 4);
  }
  r3d_host_tf_build(vals, (const uint8_t(*)[4])cols, n, lut);
  return idx;
}

float r3d_host_tf_min_visible(const uint8_t lut[256][4]) {
  for (uint32_t i = 0; i < 256u; i++)
    if (lut[i][3] != 0) return (float)i;
  return 255.0f;
}

float r3d_host_skip_gate(float low_cut, const uint8_t lut[256][4]) {
  return fmaxf(low_cut, r3d_host_tf_min_visible(lut) - 0.5f) / 255.0f;
}

/* ---- LOD policy (src/core/lod.h) ---- */

uint32_t r3d_host_lod_pick(float distance, float pixel_cone, float base_voxels,
                           uint32_t nlevels) {
  if (!nlevels) return 0;
  float footprint = fmaxf(distance * pixel_cone * base_voxels, 1.0f);
  int level = (int)floorf(log2f(footprint));
  if (level < 0) level = 0;
  if (level >= (int)nlevels) level = (int)nlevels - 1;
  return (uint32_t)level;
}

uint32_t r3d_host_lod_fallback(uint32_t desired, uint32_t ordinal, uint32_t nlevels) {
  if (!nlevels || desired >= nlevels || ordinal >= nlevels) return UINT32_MAX;
  uint32_t coarse = nlevels - desired;
  if (ordinal < coarse) return desired + ordinal;
  return desired - 1u - (ordinal - coarse);
}

/* ---- scripted orbit view (src/main.c:3932-3946, 6788-6824) ---- */

void r3d_host_orbit_view(r3d_frame_params *p, float ph, const float target[3], uint32_t w,
                         uint32_t h, float step_voxels, float density, float lod_bias,
                         uint32_t mode, uint32_t frame_index, float low_cut,
                         const uint8_t lut[256][4]) {
  const float tau = 6.2831853f;
  static const float origin0[3] = {0.5f, 0.5f, -1.5f};
  r3d_host_camera cam;
  r3d_host_camera_init(&cam, origin0);
  cam.yaw = ph * tau;
  cam.pitch = 0.5f * sinf(ph * tau * 2.0f);
  r3d_host_camera_orbit_set(&cam, target, 2.0f);
  memset(p, 0, sizeof *p);
  memcpy(p->cam_origin, cam.pos, sizeof cam.pos);
  r3d_host_camera_basis(&cam, (float)w / (float)h, p->cam_right, p->cam_up, p->cam_forward);
  p->step_voxels = step_voxels;
  p->density = density;
  p->lod_bias = lod_bias;
  p->max_mip = 10.0f;
  p->viewport[0] = w;
  p->viewport[1] = h;
  p->mode = mode;
  p->frame_index = frame_index;
  p->threshold = low_cut / 255.0f;
  p->skip_gate = r3d_host_skip_gate(low_cut, lut);
  float m[3][3];
  r3d_host_m3_ypr(0.0f, 0.0f, 0.0f, m);
  memcpy(p->vol_r0, m[0], 12);
  memcpy(p->vol_r1, m[1], 12);
  memcpy(p->vol_r2, m[2], 12);
}

/* ---- seeded scroll phantom ---- */

void r3d_host_phantom_default(uint32_t n, uint64_t seed, r3d_phantom_desc *d) {
  memset(d, 0, sizeof *d);
  d->seed = seed;
  d->pitch = n <= 256u ? 14.0f : 18.0f;
  d->radius = 110.0f * (float)n / 256.0f;
  d->r0 = 8.0f;
  d->sheet_half = 3.0f;
  d->in_mean = 130.0f;
  d->in_sd = 15.0f;
  d->air_mean = 12.0f;
  d->air_sd = 4.0f;
  d->noise_sd = 6.0f;
}

static inline uint64_t splitmix64(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

typedef struct phantom_job {
  uint8_t *vox;
  const uint8_t *mask;
  uint32_t nx, ny, z0, z1;
  const r3d_phantom_desc *d;
} phantom_job;

static void *phantom_worker(void *arg) {
  phantom_job *j = arg;
  const r3d_phantom_desc *d = j->d;
  const double two_pi = 6.283185307179586;
  for (uint32_t z = j->z0; z < j->z1; z++)
    for (uint32_t y = 0; y < j->ny; y++)
      for (uint32_t x = 0; x < j->nx; x++) {
        uint64_t idx = ((uint64_t)z * j->ny + y) * j->nx + x;
        uint64_t h1 = splitmix64(d->seed ^ (idx * 2u));
        uint64_t h2 = splitmix64(d->seed ^ (idx * 2u + 1u));
        double u1 = ((double)(h1 >> 11) + 1.0) * 0x1.0p-53; /* (0, 1] */
        double u2 = (double)(h2 >> 11) * 0x1.0p-53;
        double rad = sqrt(-2.0 * log(u1));
        double g0 = rad * cos(two_pi * u2), g1 = rad * sin(two_pi * u2);
        int pap = j->mask[(size_t)y * j->nx + x];
        double mean = pap ? d->in_mean : d->air_mean, sd = pap ? d->in_sd : d->air_sd;
        double v = mean + sd * g0 + d->noise_sd * g1;
        v = floor(v + 0.5);
        j->vox[idx] = (uint8_t)(v < 0.0 ? 0.0 : (v > 255.0 ? 255.0 : v));
      }
  return NULL;
}

int r3d_host_phantom(uint8_t *vox, uint32_t nx, uint32_t ny, uint32_t nz,
                     const r3d_phantom_desc *d, int threads) {
  if (!vox || !d || !nx || !ny || !nz || !(d->pitch > 0.0f)) return -1;
  uint8_t *mask = malloc((size_t)nx * ny);
  if (!mask) return -1;
  /* papyrus mask of one z slice: the spiral is a prism along z */
  const double two_pi = 6.283185307179586;
  double cx = 0.5 * nx, cy = 0.5 * ny;
  for (uint32_t y = 0; y < ny; y++)
    for (uint32_t x = 0; x < nx; x++) {
      double dx = x + 0.5 - cx, dy = y + 0.5 - cy;
      double r = sqrt(dx * dx + dy * dy);
      double th = atan2(dy, dx);
      if (th < 0.0) th += two_pi;
      double m = fmod(r - d->r0 - d->pitch * th / two_pi, d->pitch);
      if (m < 0.0) m += d->pitch;
      double dist = m < d->pitch - m ? m : d->pitch - m;
      mask[(size_t)y * nx + x] = dist < d->sheet_half && r >= d->r0 && r < d->radius;
    }
  if (threads <= 0) threads = 8;
  if (threads > 256) threads = 256;
  if ((uint32_t)threads > nz) threads = (int)nz;
  pthread_t tid[256];
  phantom_job jobs[256];
  int live[256];
  for (int i = 0; i < threads; i++) {
    jobs[i] = (phantom_job){vox, mask, nx, ny, (uint32_t)((uint64_t)nz * (uint64_t)i / threads),
                            (uint32_t)((uint64_t)nz * (uint64_t)(i + 1) / threads), d};
    live[i] = pthread_create(&tid[i], NULL, phantom_worker, &jobs[i]) == 0;
    if (!live[i]) phantom_worker(&jobs[i]);
  }
  for (int i = 0; i < threads; i++)
    if (live[i]) pthread_join(tid[i], NULL);
  free(mask);
  return 0;
}

/* ------------------------------------------------- streamer request set */

static void stream_axis_bounds(float eye, float radius, float edge, uint32_t n, uint32_t *lo,
                               uint32_t *hi) {  // vkbackend.c:3096-3106
  int a = (int)ceilf((eye - radius) / edge - 0.5f);
  int b = (int)floorf((eye + radius) / edge - 0.5f) + 1;
  if (a < 0) a = 0;
  if (b < 0) b = 0;
  if (a > (int)n) a = (int)n;
  if (b > (int)n) b = (int)n;
  *lo = (uint32_t)a;
  *hi = (uint32_t)b;
}

static int stream_cand_cmp(const void *a, const void *b) {  // vkbackend.c:3075-3080
  const r3d_stream_cand *ca = a, *cb = b;
  if (ca->priority != cb->priority) return ca->priority < cb->priority ? -1 : 1;
  float d = ca->d2 - cb->d2;
  return d < 0.0f ? -1 : (d > 0.0f ? 1 : (ca->brick < cb->brick ? -1 : ca->brick > cb->brick));
}

uint32_t r3d_host_stream_desired(const uint32_t *page, uint32_t page_words, const float eye[3],
                                 const float fwd[3], float half_tan, float pixel_cone,
                                 uint32_t slice_z0, uint32_t slice_depth, float gate,
                                 uint8_t *mark, r3d_stream_cand *out, uint32_t cap) {
  if (!page || page_words < R3D_BRICK_PAGE_HEADER || !mark || !out) return 0;
  const uint32_t nlev = page[0];
  if (nlev < 1u || nlev > 15u) return 0;
  const float maxdim = (float)(page[1] > page[2] ? (page[1] > page[3] ? page[1] : page[3])
                                                 : (page[2] > page[3] ? page[2] : page[3]));
  const float tanw = half_tan * 1.15f + 1e-3f;
  int g8 = (int)(gate * 255.0f + 0.5f);
  if (g8 < 5) g8 = 5;  // decoded-air noise floor (vkbackend.c:2348)
  const float lod_factor = fmaxf(pixel_cone * maxdim, 1e-6f);
  uint32_t n = 0;
  for (uint32_t li = 0; li + 1u < nlev; li++) {
    const uint32_t off = page[4u + 4u * li], packed = page[5u + 4u * li],
                   scale = page[6u + 4u * li];
    const uint32_t bd[3] = {packed & 1023u, (packed >> 10) & 1023u, packed >> 20};
    const uint32_t poff = page[4u + 4u * (li + 1u)], ppacked = page[5u + 4u * (li + 1u)];
    const uint32_t pbd[2] = {ppacked & 1023u, (ppacked >> 10) & 1023u};
    const float edge = (float)(128u * scale) / maxdim;
    const float brad = 0.8660254f * edge;
    const float outer = exp2f((float)li + 1.0f) / lod_factor + brad;
    uint32_t x0, x1, y0, y1, z0, z1;
    stream_axis_bounds(eye[0], outer, edge, bd[0], &x0, &x1);
    stream_axis_bounds(eye[1], outer, edge, bd[1], &y0, &y1);
    stream_axis_bounds(eye[2], outer, edge, bd[2], &z0, &z1);
    if (slice_depth) {
      uint64_t zlast = (uint64_t)slice_z0 + slice_depth;
      if (zlast > page[3]) zlast = page[3];
      const uint32_t zbrick = 128u * scale;
      const uint32_t sz0 = slice_z0 / zbrick, sz1 = (uint32_t)((zlast + zbrick - 1u) / zbrick);
      if (z0 < sz0) z0 = sz0;
      if (z1 > sz1) z1 = sz1;
    }
    for (uint32_t bz = z0; bz < z1; bz++)
      for (uint32_t by = y0; by < y1; by++)
        for (uint32_t bx = x0; bx < x1; bx++) {
          const float cx = ((float)bx + 0.5f) * edge - eye[0];
          const float cy = ((float)by + 0.5f) * edge - eye[1];
          const float cz = ((float)bz + 0.5f) * edge - eye[2];
          const float d2 = cx * cx + cy * cy + cz * cz;
          const float along = cx * fwd[0] + cy * fwd[1] + cz * fwd[2];
          bool vis = d2 < (edge + brad) * (edge + brad);
          if (!vis && along > 0.0f) {
            const float perp2 = d2 - along * along;
            const float rad = along * tanw + brad;
            vis = perp2 < rad * rad;
          }
          if (!vis) continue;
          if (r3d_host_lod_pick(sqrtf(d2), pixel_cone, maxdim, nlev) != li) continue;
          const uint32_t cand[2] = {
              poff + ((bz >> 1) * pbd[1] + (by >> 1)) * pbd[0] + (bx >> 1),
              off + (bz * bd[1] + by) * bd[0] + bx};
          for (uint32_t k = 0; k < 2u; k++) {
            const uint32_t b = cand[k];
            if (b >= page_words || mark[b]) continue;
            const uint32_t e = page[b];
            if (e == R3D_BRICK_ABSENT || (int)(e >> 24) < g8) continue;
            mark[b] = 1;
            if (n < cap) out[n++] = (r3d_stream_cand){d2, b, k};
          }
        }
  }
  qsort(out, n, sizeof *out, stream_cand_cmp);
  return n;
}

void r3d_host_stream_sort(r3d_stream_cand *c, uint32_t n) {
  if (c && n > 1u) qsort(c, n, sizeof *c, stream_cand_cmp);
}

/* the brick of level li under voxel-normalized position coordinate v */
static uint32_t stream_level(const uint32_t *page, uint32_t li, uint32_t *off, uint32_t bd[3],
                             float *edge, float maxdim) {
  const uint32_t packed = page[5u + 4u * li];
  *off = page[4u + 4u * li];
  bd[0] = packed & 1023u, bd[1] = (packed >> 10) & 1023u, bd[2] = packed >> 20;
  *edge = (float)(128u * page[6u + 4u * li]) / maxdim;
  return page[6u + 4u * li];
}

/* appends brick b unless listed already, absent, or darker than g8 */
static uint32_t stream_add(const uint32_t *page, uint32_t page_words, uint32_t b, float d2,
                           uint32_t priority, int g8, uint8_t *mark, r3d_stream_cand *out,
                           uint32_t cap, uint32_t n) {
  if (b >= page_words || mark[b]) return n;
  const uint32_t e = page[b];
  if (e == R3D_BRICK_ABSENT || (int)(e >> 24) < g8) return n;
  mark[b] = 1;
  if (n < cap) out[n++] = (r3d_stream_cand){d2, b, priority};
  return n;
}

static int stream_gate8(float gate) {
  int g8 = (int)(gate * 255.0f + 0.5f);
  return g8 < 5 ? 5 : g8;  // decoded-air noise floor (vkbackend.c:2348)
}

static float stream_maxdim(const uint32_t *page) {
  return (float)(page[1] > page[2] ? (page[1] > page[3] ? page[1] : page[3])
                                   : (page[2] > page[3] ? page[2] : page[3]));
}

uint32_t r3d_host_stream_box(const uint32_t *page, uint32_t page_words, const float lo[3],
                             const float hi[3], float pixel_cone, float gate, uint8_t *mark,
                             r3d_stream_cand *out, uint32_t cap, uint32_t n) {
  if (!page || page_words < R3D_BRICK_PAGE_HEADER || !lo || !hi || !mark || !out) return n;
  const uint32_t nlev = page[0];
  if (nlev < 1u || nlev > 15u) return n;
  const int g8 = stream_gate8(gate);
  const float maxdim = stream_maxdim(page);
  const float vpp = fmaxf(pixel_cone * maxdim, 1.0f);  // base voxels per pixel
  uint32_t desired = (uint32_t)floorf(log2f(vpp));
  if (desired >= nlev) desired = nlev - 1u;
  uint32_t off, bd[3], rng[3][2];
  float edge;
  for (;;) {  // coarsen until the box holds at most 2048 bricks
    stream_level(page, desired, &off, bd, &edge, maxdim);
    uint64_t count = 1;
    for (int a = 0; a < 3; a++) {
      int64_t a0 = (int64_t)floorf(lo[a] / edge), a1 = (int64_t)floorf(hi[a] / edge) + 1;
      if (a0 < 0) a0 = 0;
      if (a1 > (int64_t)bd[a]) a1 = (int64_t)bd[a];
      if (a1 < a0) a1 = a0;
      rng[a][0] = (uint32_t)a0, rng[a][1] = (uint32_t)a1;
      count *= (uint64_t)(a1 - a0);
    }
    if (count <= 2048u || desired + 1u >= nlev) break;
    desired++;
  }
  const float cx0 = (lo[0] + hi[0]) * 0.5f, cy0 = (lo[1] + hi[1]) * 0.5f,
              cz0 = (lo[2] + hi[2]) * 0.5f;
  uint32_t poff = 0, pbd[3] = {0, 0, 0};
  float pedge;
  const int parent = desired + 1u < nlev;
  if (parent) stream_level(page, desired + 1u, &poff, pbd, &pedge, maxdim);
  for (uint32_t bz = rng[2][0]; bz < rng[2][1]; bz++)
    for (uint32_t by = rng[1][0]; by < rng[1][1]; by++)
      for (uint32_t bx = rng[0][0]; bx < rng[0][1]; bx++) {
        const float dx = ((float)bx + 0.5f) * edge - cx0;
        const float dy = ((float)by + 0.5f) * edge - cy0;
        const float dz = ((float)bz + 0.5f) * edge - cz0;
        const float d2 = dx * dx + dy * dy + dz * dz;
        if (parent)
          n = stream_add(page, page_words, poff + ((bz >> 1) * pbd[1] + (by >> 1)) * pbd[0] + (bx >> 1),
                         d2, 0u, g8, mark, out, cap, n);
        n = stream_add(page, page_words, off + (bz * bd[1] + by) * bd[0] + bx, d2, 1u, g8, mark, out,
                       cap, n);
      }
  return n;
}

uint32_t r3d_host_stream_point(const uint32_t *page, uint32_t page_words, const float p[3],
                               uint32_t level, float gate, uint8_t *mark, r3d_stream_cand *out,
                               uint32_t cap, uint32_t n) {
  if (!page || page_words < R3D_BRICK_PAGE_HEADER || !p || !mark || !out) return n;
  const uint32_t nlev = page[0];
  if (nlev < 1u || nlev > 15u) return n;
  const int g8 = stream_gate8(gate);
  const float maxdim = stream_maxdim(page);
  if (level >= nlev) level = nlev - 1u;
  uint32_t off, bd[3], bc[3];
  float edge;
  stream_level(page, level, &off, bd, &edge, maxdim);
  for (int a = 0; a < 3; a++) {
    int64_t i = (int64_t)(p[a] / edge);
    if (i < 0) i = 0;
    if (i >= (int64_t)bd[a]) i = (int64_t)bd[a] - 1;
    bc[a] = (uint32_t)i;
  }
  if (level + 1u < nlev) {
    uint32_t poff, pbd[3];
    float pedge;
    stream_level(page, level + 1u, &poff, pbd, &pedge, maxdim);
    n = stream_add(page, page_words,
                   poff + ((bc[2] >> 1) * pbd[1] + (bc[1] >> 1)) * pbd[0] + (bc[0] >> 1), 0.0f, 0u,
                   g8, mark, out, cap, n);
  }
  return stream_add(page, page_words, off + (bc[2] * bd[1] + bc[1]) * bd[0] + bc[0], 0.0f, 1u, g8,
                    mark, out, cap, n);
}

/* ---- CPU-sourced slot-parallel atlases ---- */

int r3d_host_brick_locate(const uint32_t *page, uint32_t b, uint32_t *level, uint32_t *bx,
                          uint32_t *by, uint32_t *bz) {
  if (!page) return -1;
  const uint32_t nlev = page[0];
  for (uint32_t l = 0; l < nlev && l < 15u; l++) {
    const uint32_t off = page[4u + 4u * l], packed = page[5u + 4u * l];
    const uint32_t dx = packed & 1023u, dy = (packed >> 10) & 1023u, dz = packed >> 20;
    if (b < off || b - off >= dx * dy * dz) continue;
    const uint32_t local = b - off;
    *level = l;
    *bx = local % dx;
    *by = (local / dx) % dy;
    *bz = local / (dx * dy);
    return 0;
  }
  return -1;
}

uint32_t r3d_host_atlas_pick(const uint32_t *page, const uint32_t *slot_brick, uint32_t nslots,
                             const uint64_t *keys, const r3d_brick_src *src, uint32_t budget,
                             uint32_t *sel_slot, uint32_t *sel_brick, uint64_t *sel_key) {
  if (!page || !slot_brick || !keys || !src || !src->gen) return 0;
  if (!budget || budget > 16u) budget = 16u;
  uint32_t n = 0;
  /* stale slots first: a slot given to another brick still shows the old
   * brick's content (vkbackend.c:4998-5020) */
  for (uint32_t s = 0; s < nslots && n < budget; s++) {
    const uint32_t b = slot_brick[s];
    if (b == R3D_BRICK_ABSENT) continue;
    const uint64_t key = keys[s];
    if (key == 0 || (uint32_t)(key >> 32) == b + 1u) continue;
    sel_slot[n] = s, sel_brick[n] = b, sel_key[n] = 0;
    n++;
  }
  if (n) return n;
  /* fill: content generations that changed (vkbackend.c:5022-5046) */
  for (uint32_t s = 0; s < nslots && n < budget; s++) {
    const uint32_t b = slot_brick[s];
    if (b == R3D_BRICK_ABSENT) continue;
    uint32_t l, bx, by, bz;
    if (r3d_host_brick_locate(page, b, &l, &bx, &by, &bz) != 0) continue;
    const uint32_t g = src->gen(src->user, l, bx, by, bz);
    const uint64_t want = g ? (((uint64_t)b + 1u) << 32) | g : 0u;
    if (keys[s] == want) continue;
    sel_slot[n] = s, sel_brick[n] = b, sel_key[n] = want;
    n++;
  }
  return n;
}

/* ---- virtual slab layout and fill planner ---- */

static const uint32_t vs_scale[R3D_VS_LEVELS] = {1u, 4u, 8u, 16u, 32u};

int r3d_host_vslab_init(r3d_vslab_layout *v, uint64_t nx, uint64_t ny, uint64_t nz, uint32_t W,
                        uint32_t H, uint32_t D, uint32_t z_margin) {
  const uint64_t ring = (uint64_t)D + 2u + 2u * (uint64_t)z_margin;
  if (!v || W < 64u || H < 64u || W > nx || H > ny || D < 2u || D > 2044u || D > nz ||
      ring > 2046u || ring > nz)
    return -1;
  memset(v, 0, sizeof *v);
  v->nx = nx, v->ny = ny, v->nz = nz;
  v->W = W, v->H = H, v->D = D;
  v->wz = (uint32_t)ring;
  v->z_margin = z_margin;
  const uint32_t m = W > H ? W : H;
  uint32_t px = (m / 8u + 31u) & ~31u;
  px = px < 64u ? 64u : (px > 2016u ? 2016u : px);
  while (px > 64u && (uint64_t)(px + 2u) * (px + 2u) * v->wz > (3ull << 30)) px -= 32u;
  v->px = px;
  /* a movable axis adds a straddle tile and a prefetch tile */
  const uint32_t ex = W < nx ? 2u : 0u, ey = H < ny ? 2u : 0u;
  uint32_t nt = 0;
  for (uint32_t l = 0; l < R3D_VS_LEVELS; l++) {
    const uint64_t cs = (uint64_t)px * vs_scale[l];
    v->s[l] = vs_scale[l];
    v->base[l] = nt;
    if (l && m / vs_scale[l] < 1024u) continue; /* pyramid level not needed */
    v->gx[l] = (uint32_t)((W + cs - 1u) / cs) + ex;
    v->gy[l] = (uint32_t)((H + cs - 1u) / cs) + ey;
    nt += v->gx[l] * v->gy[l];
  }
  v->ntiles = nt;
  v->x0 = v->y0 = v->z0 = -1;
  return 0;
}

void r3d_host_vslab_zrange(const r3d_vslab_layout *v, int64_t z0, int64_t *a, int64_t *b) {
  int64_t za = z0 - (int64_t)v->z_margin;
  if (za < 0) za = 0;
  int64_t zb = za + (int64_t)v->wz;
  if (zb > (int64_t)v->nz) {
    zb = (int64_t)v->nz;
    za = zb - (int64_t)v->wz;
    if (za < 0) za = 0;
  }
  *a = za, *b = zb;
}

void r3d_host_vslab_range(const r3d_vslab_layout *v, uint32_t l, int64_t o, uint64_t n,
                          uint32_t span, int64_t *c0, int64_t *c1) {
  const int64_t cs = (int64_t)v->px * (int64_t)v->s[l];
  int64_t a = o / cs, b = (o + (int64_t)span - 1) / cs;
  const int64_t last = ((int64_t)n - 1) / cs;
  *c0 = a < 0 ? 0 : a;
  *c1 = b > last ? last : b;
}

uint32_t r3d_host_vslab_key(int64_t cx, int64_t cy) {
  return ((uint32_t)cx & 1023u) | (((uint32_t)cy & 1023u) << 10) | 0x80000000u;
}

static uint32_t vs_slot(const r3d_vslab_layout *v, int64_t cx, int64_t cy) {
  return (uint32_t)(cy % v->gy[0]) * v->gx[0] + (uint32_t)(cx % v->gx[0]);
}

static int64_t vs_max0(uint64_t n, uint32_t span) {
  const int64_t m = (int64_t)n - (int64_t)span;
  return m < 0 ? 0 : m;
}

uint32_t r3d_host_vslab_plan(r3d_vslab_layout *v, const r3d_vslab_cell *cells, double fx,
                             double fy, int64_t z0, uint32_t budget, r3d_vslab_job *out,
                             uint32_t cap) {
  if (!v || !cells || (!out && cap)) return 0;
  const int64_t px0 = v->x0, py0 = v->y0, pz0 = v->z0;
  int64_t x0 = (int64_t)fx - v->W / 2, y0 = (int64_t)fy - v->H / 2;
  x0 = x0 < 0 ? 0 : (x0 & ~(int64_t)15);
  y0 = y0 < 0 ? 0 : (y0 & ~(int64_t)15);
  if (x0 > vs_max0(v->nx, v->W)) x0 = vs_max0(v->nx, v->W) & ~(int64_t)15;
  if (y0 > vs_max0(v->ny, v->H)) y0 = vs_max0(v->ny, v->H) & ~(int64_t)15;
  if (z0 < 0) z0 = 0;
  if (z0 > vs_max0(v->nz, v->D)) z0 = vs_max0(v->nz, v->D);
  int64_t za_want, zb_want;
  r3d_host_vslab_zrange(v, z0, &za_want, &zb_want);
  int64_t vis_end = z0 + (int64_t)v->D + 2;
  if (vis_end > (int64_t)v->nz) vis_end = (int64_t)v->nz;
  const int up = pz0 < 0 || z0 >= pz0; /* direction of z travel */
  v->x0 = x0, v->y0 = y0, v->z0 = z0;

  int64_t cx0, cx1, cy0, cy1;
  r3d_host_vslab_range(v, 0, x0, v->nx, v->W, &cx0, &cx1);
  r3d_host_vslab_range(v, 0, y0, v->ny, v->H, &cy0, &cy1);
  r3d_vslab_job jobs[64];
  uint64_t dist[64];
  uint32_t nj = 0;
  const int64_t ccx = (x0 + v->W / 2) / (int64_t)v->px, ccy = (y0 + v->H / 2) / (int64_t)v->px;
  const uint32_t mchunks = (v->z_margin + 15u) / 16u;
  for (int64_t cy = cy0; cy <= cy1 && nj < 64u; cy++)
    for (int64_t cx = cx0; cx <= cx1 && nj < 64u; cx++) {
      const r3d_vslab_cell *c = &cells[vs_slot(v, cx, cy)];
      r3d_vslab_job j = {cx, cy, z0, (uint32_t)(vis_end - z0), 0u};
      const int held = c->cx == cx && c->cy == cy;
      const int visible = held && c->za <= z0 && c->zb >= vis_end;
      if (held) {
        if (c->za <= za_want && c->zb >= zb_want) continue; /* whole range resident */
        int64_t s0 = z0, s1 = vis_end;
        if (!visible && c->za < vis_end && c->zb > z0) {
          /* finish the visible span around what is held */
          if (c->za > z0) {
            s1 = c->za < vis_end ? c->za : vis_end;
          } else {
            s0 = c->zb > z0 ? c->zb : z0;
          }
        } else if (visible) {
          /* grow the margin, 16 slices at a time, travel direction first */
          int grow_up;
          uint32_t extra;
          if (up && c->zb < zb_want) {
            grow_up = 1, extra = 0u;
          } else if (!up && c->za > za_want) {
            grow_up = 0, extra = 0u;
          } else if (c->za > za_want) {
            grow_up = 0, extra = mchunks;
          } else {
            grow_up = 1, extra = mchunks;
          }
          int64_t filled;
          if (grow_up) {
            s0 = c->zb;
            s1 = s0 + 16 < zb_want ? s0 + 16 : zb_want;
            filled = c->zb - vis_end;
          } else {
            s1 = c->za;
            s0 = s1 - 16 > za_want ? s1 - 16 : za_want;
            filled = z0 - c->za;
          }
          j.prio = 1u + extra + (uint32_t)(filled > 0 ? filled / 16 : 0);
        }
        j.zs0 = s0;
        j.nz = (uint32_t)(s1 - s0);
      }
      const int64_t dx = cx - ccx, dy = cy - ccy;
      dist[nj] = (uint64_t)(dx * dx + dy * dy);
      jobs[nj++] = j;
    }
  /* exchange sort by (priority, distance), the reference's order */
  for (uint32_t a = 0; a + 1u < nj; a++)
    for (uint32_t b = a + 1u; b < nj; b++)
      if (jobs[b].prio < jobs[a].prio || (jobs[b].prio == jobs[a].prio && dist[b] < dist[a])) {
        r3d_vslab_job t = jobs[a];
        jobs[a] = jobs[b], jobs[b] = t;
        uint64_t td = dist[a];
        dist[a] = dist[b], dist[b] = td;
      }
  uint32_t n = 0;
  for (uint32_t k = 0; k < nj && n < budget && n < cap; k++) out[n++] = jobs[k];
  /* prefetch the column / row past the window in the direction of motion */
  if (px0 >= 0 && (x0 != px0 || y0 != py0)) {
    int64_t pf[48][2];
    uint32_t npf = 0;
    const int64_t mxc = ((int64_t)v->nx - 1) / v->px, myc = ((int64_t)v->ny - 1) / v->px;
    if (x0 != px0) {
      const int64_t cxc = x0 > px0 ? cx1 + 1 : cx0 - 1;
      if (cxc >= 0 && cxc <= mxc && cx1 - cx0 + 2 <= (int64_t)v->gx[0])
        for (int64_t cy = cy0; cy <= cy1 && npf < 48u; cy++) pf[npf][0] = cxc, pf[npf++][1] = cy;
    }
    if (y0 != py0) {
      const int64_t cyc = y0 > py0 ? cy1 + 1 : cy0 - 1;
      if (cyc >= 0 && cyc <= myc && cy1 - cy0 + 2 <= (int64_t)v->gy[0])
        for (int64_t cx = cx0; cx <= cx1 && npf < 48u; cx++) pf[npf][0] = cx, pf[npf++][1] = cyc;
    }
    for (uint32_t k = 0; k < npf && n < budget && n < cap; k++) {
      const r3d_vslab_cell *c = &cells[vs_slot(v, pf[k][0], pf[k][1])];
      if (c->cx == pf[k][0] && c->cy == pf[k][1] && c->za <= za_want && c->zb >= zb_want)
        continue;
      int dup = 0; /* a cell listed twice (both axes moved) fills once */
      for (uint32_t m = 0; m < n; m++) dup |= out[m].cx == pf[k][0] && out[m].cy == pf[k][1];
      if (dup) continue;
      r3d_vslab_job j = {pf[k][0], pf[k][1], za_want, (uint32_t)(zb_want - za_want), 0u};
      out[n++] = j;
    }
  }
  return n;
}

uint32_t r3d_host_vslab_apply(const r3d_vslab_layout *v, r3d_vslab_cell *cells,
                              const r3d_vslab_job *j, int64_t z0) {
  int64_t za_want, zb_want;
  r3d_host_vslab_zrange(v, z0, &za_want, &zb_want);
  const uint32_t slot = vs_slot(v, j->cx, j->cy);
  r3d_vslab_cell *c = &cells[slot];
  const int64_t a = j->zs0, b = j->zs0 + (int64_t)j->nz;
  if (c->cx != j->cx || c->cy != j->cy) {
    c->za = a, c->zb = b;
  } else {
    if (a < c->za) c->za = a;
    if (b > c->zb) c->zb = b;
  }
  c->cx = j->cx, c->cy = j->cy;
  if (c->za < za_want) c->za = za_want;
  if (c->zb > zb_want) c->zb = zb_want;
  if (c->zb < c->za) c->zb = c->za;
  return slot;
}
