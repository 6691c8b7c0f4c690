/* Headless render3d-style command line on the CPU oracle (test
 * infrastructure).  Accepts the subset of render3d's flags that its
 * conformance test uses (reference tests/test_gpu.c:78-83):
 *   r3d_oracle_cli <vol.u8> <nx> <ny> <nz> [--frames N] [--mode M]
 *                  [--shot out.ppm] [--size W H] [--tf P] [--lowcut V]
 * and renders the last frame of the default turntable orbit (camera at
 * (0.5, 0.5, -1.5) looking +Z, reference src/main.c:2075,2860-2864) into a
 * binary PPM, the format of src/core/screenshot.c:6-28. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "r3d_oracle.h"

/* presets of src/core/transfer.c:25-50 as (value, r, g, b, a) rows */
static const uint8_t PRESET[3][5][5] = {
    {{0, 0, 0, 0, 0}, {255, 255, 255, 255, 255}},
    {{0, 0, 0, 0, 0}, {40, 0, 0, 0, 0}, {90, 150, 110, 70, 40}, {160, 230, 190, 130, 160},
     {255, 255, 250, 240, 255}},
    {{0, 0, 0, 0, 0}, {120, 0, 0, 0, 0}, {180, 200, 200, 255, 120}, {255, 255, 255, 255, 255}},
};
static const uint32_t PRESET_N[3] = {2, 5, 4};

int main(int argc, char **argv) {
  if (argc < 5) {
    fprintf(stderr, "usage: r3d_oracle_cli vol.u8 nx ny nz [flags]\n");
    return 2;
  }
  uint32_t nx = (uint32_t)atoi(argv[2]), ny = (uint32_t)atoi(argv[3]),
           nz = (uint32_t)atoi(argv[4]);
  uint32_t frames = 1, mode = 0, w = 1280, h = 720;
  int tf = -1;
  float lowcut = 0.0f;
  const char *shot = NULL;
  for (int i = 5; i < argc; i++) {
    if (i < argc - 1 && !strcmp(argv[i], "--frames")) frames = (uint32_t)atoi(argv[++i]);
    else if (i < argc - 1 && !strcmp(argv[i], "--mode")) mode = (uint32_t)atoi(argv[++i]) % 6u;
    else if (i < argc - 1 && !strcmp(argv[i], "--shot")) shot = argv[++i];
    else if (i < argc - 1 && !strcmp(argv[i], "--tf")) tf = atoi(argv[++i]);
    else if (i < argc - 1 && !strcmp(argv[i], "--lowcut")) lowcut = (float)atof(argv[++i]);
    else if (i < argc - 2 && !strcmp(argv[i], "--size")) {
      w = (uint32_t)atoi(argv[i + 1]);
      h = (uint32_t)atoi(argv[i + 2]);
      i += 2;
    }
  }
  size_t n = (size_t)nx * ny * nz;
  uint8_t *vol = malloc(n);
  FILE *f = fopen(argv[1], "rb");
  if (!vol || !f || fread(vol, 1, n, f) != n) {
    fprintf(stderr, "r3d_oracle_cli: cannot read %s\n", argv[1]);
    return 1;
  }
  fclose(f);

  orc_cube cube;
  memset(&cube, 0, sizeof cube);
  cube.nlevels = orc_mip_levels(nx, ny, nz, cube.dim);
  cube.level[0] = vol;
  for (uint32_t m = 1; m < cube.nlevels; m++) {
    uint8_t *d = malloc((size_t)cube.dim[m][0] * cube.dim[m][1] * cube.dim[m][2]);
    orc_downsample(cube.level[m - 1], cube.dim[m - 1][0], cube.dim[m - 1][1], cube.dim[m - 1][2],
                   d, cube.dim[m][0], cube.dim[m][1], cube.dim[m][2]);
    cube.level[m] = d;
  }
  for (int a = 0; a < 3; a++) cube.odim[a] = ((a == 0 ? nx : a == 1 ? ny : nz) + 7u) / 8u;
  uint8_t *occ = malloc((size_t)cube.odim[0] * cube.odim[1] * cube.odim[2]);
  orc_occupancy(vol, nx, ny, nz, occ);
  cube.occ = occ;

  uint8_t lut[256][4];
  float tf_min = 1.0f; /* default ramp: alpha nonzero from value 1 */
  if (tf >= 0 && tf < 3) {
    uint8_t vals[5], rgba[5][4];
    for (uint32_t k = 0; k < PRESET_N[tf]; k++) {
      vals[k] = PRESET[tf][k][0];
      memcpy(rgba[k], &PRESET[tf][k][1], 4);
    }
    orc_tf_build(vals, (const uint8_t(*)[4])rgba, PRESET_N[tf], lut);
    tf_min = 255.0f;
    for (int i = 0; i < 256; i++)
      if (lut[i][3]) {
        tf_min = (float)i;
        break;
      }
  } else {
    for (int i = 0; i < 256; i++) lut[i][0] = lut[i][1] = lut[i][2] = lut[i][3] = (uint8_t)i;
  }

  r3d_frame_params p;
  memset(&p, 0, sizeof p);
  float target[3] = {0.5f, 0.5f, 0.5f};
  orc_orbit_pos(0.0f, 0.0f, target, 2.0f, p.cam_origin);
  orc_camera_basis(0.0f, 0.0f, 1.04719755f, (float)w / (float)h, p.cam_right, p.cam_up,
                   p.cam_forward);
  p.step_voxels = 1.0f;
  p.density = 1.0f;
  p.max_mip = 10.0f;
  p.viewport[0] = w;
  p.viewport[1] = h;
  p.mode = mode;
  p.frame_index = frames ? frames - 1u : 0u;
  p.threshold = lowcut / 255.0f;
  p.skip_gate = (lowcut > tf_min - 0.5f ? lowcut : tf_min - 0.5f) / 255.0f;
  p.vol_r0[0] = p.vol_r1[1] = p.vol_r2[2] = 1.0f;

  uint8_t *img = calloc((size_t)w * h, 4);
  orc_opts o = {0.98f, R3D_QUALITY_FULL, 0};
  if (orc_render_view(&p, &cube, NULL, (const uint8_t(*)[4])lut, &o, img, w, h, NULL) != 0) {
    fprintf(stderr, "r3d_oracle_cli: render failed\n");
    return 1;
  }
  if (shot) {
    FILE *o2 = fopen(shot, "wb");
    if (!o2) return 1;
    fprintf(o2, "P6\n%u %u\n255\n", w, h);
    for (size_t i = 0; i < (size_t)w * h; i++) fwrite(img + i * 4, 1, 3, o2);
    fclose(o2);
  }
  return 0;
}
