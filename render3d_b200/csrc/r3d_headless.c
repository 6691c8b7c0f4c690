/* r3d_headless: render3d's headless capture path on the sm_100a library.
 *
 *   r3d_headless <vol.u8> <nx> <ny> <nz> [--frames N] [--mode M]
 *                [--shot out.ppm] [--size W H] [--tf P] [--lowcut V]
 *                [--quality full|fast]
 *
 * Same flags and defaults as the reference binary for this path
 * (src/main.c:2073-2083,2142-2221): 1280x720, turntable orbit at distance 2
 * around the volume centre with the camera starting at (0.5, 0.5, -1.5),
 * step 1 voxel, density 1, max_mip 10, the backend's grey-ramp TF, and a
 * binary PPM of the last frame (src/core/screenshot.c:6-28).  The
 * reference's GPU conformance test (tests/test_gpu.c) runs against it. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "r3d_host.h"
#include "r3d_render.h"

int main(int argc, char **argv) {
  if (argc < 5) {
    fprintf(stderr, "usage: r3d_headless vol.u8 nx ny nz [flags]\n");
    return 2;
  }
  uint32_t nx = (uint32_t)atoi(argv[2]), ny = (uint32_t)atoi(argv[3]),
           nz = (uint32_t)atoi(argv[4]);
  uint32_t frames = 1, mode = 0, w = 1280, h = 720, quality = R3D_QUALITY_FULL;
  int tf = -1;
  float lowcut = 0.0f;
  const char *shot = NULL;
  for (int i = 5; i < argc; i++) {
    if (i < argc - 1 && !strcmp(argv[i], "--frames")) frames = (uint32_t)atoi(argv[++i]);
    else if (i < argc - 1 && !strcmp(argv[i], "--mode")) mode = (uint32_t)atoi(argv[++i]) % 6u;
    else if (i < argc - 1 && !strcmp(argv[i], "--shot")) shot = argv[++i];
    else if (i < argc - 1 && !strcmp(argv[i], "--tf")) tf = atoi(argv[++i]);
    else if (i < argc - 1 && !strcmp(argv[i], "--lowcut")) lowcut = (float)atof(argv[++i]);
    else if (i < argc - 1 && !strcmp(argv[i], "--quality"))
      quality = !strcmp(argv[++i], "fast") ? R3D_QUALITY_FAST : R3D_QUALITY_FULL;
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
    fprintf(stderr, "r3d_headless: cannot read %s\n", argv[1]);
    return 1;
  }
  fclose(f);

  r3d_config cfg = {.headless = true, .headless_w = w, .headless_h = h};
  r3d_renderer *r = NULL;
  if (r3d_create(NULL, &cfg, &r) != 0) return 1;
  r3d_volume_desc d = {nx, ny, nz, 128, 1.0f};
  if (r3d_upload_volume(r, &d, vol) != 0) return 1;
  free(vol);
  r3d_set_quality(r, quality);
  uint8_t lut[256][4];
  for (int i = 0; i < 256; i++) lut[i][0] = lut[i][1] = lut[i][2] = lut[i][3] = (uint8_t)i;
  if (tf >= 0 && r3d_host_tf_preset((uint32_t)tf, lut) == (uint32_t)tf &&
      r3d_set_transfer(r, (const uint8_t(*)[4])lut) != 0)
    return 1;

  static const float origin0[3] = {0.5f, 0.5f, -1.5f}, target[3] = {0.5f, 0.5f, 0.5f};
  r3d_host_camera cam;
  r3d_host_camera_init(&cam, origin0);
  r3d_host_camera_orbit_set(&cam, target, 2.0f);
  float m[3][3];
  r3d_host_m3_ypr(0.0f, 0.0f, 0.0f, m);
  for (uint32_t fi = 0; fi < (frames ? frames : 1u); fi++) {
    r3d_frame_params p;
    memset(&p, 0, sizeof p);
    memcpy(p.cam_origin, cam.pos, sizeof cam.pos);
    r3d_host_camera_basis(&cam, (float)w / (float)h, p.cam_right, p.cam_up, p.cam_forward);
    p.step_voxels = 1.0f;
    p.density = 1.0f;
    p.max_mip = 10.0f;
    p.viewport[0] = w;
    p.viewport[1] = h;
    p.mode = mode;
    p.frame_index = fi;
    p.threshold = lowcut / 255.0f;
    p.skip_gate = r3d_host_skip_gate(lowcut, (const uint8_t(*)[4])lut);
    memcpy(p.vol_r0, m[0], 12);
    memcpy(p.vol_r1, m[1], 12);
    memcpy(p.vol_r2, m[2], 12);
    if (r3d_frame(r, &p, NULL) != 0) return 1;
  }
  if (shot) {
    uint32_t fw = 0, fh = 0;
    r3d_read_frame(r, NULL, &fw, &fh);
    uint8_t *img = malloc((size_t)fw * fh * 4);
    if (!img || r3d_read_frame(r, img, &fw, &fh) != 0) return 1;
    FILE *o = fopen(shot, "wb");
    if (!o) return 1;
    fprintf(o, "P6\n%u %u\n255\n", fw, fh);
    for (size_t i = 0; i < (size_t)fw * fh; i++) fwrite(img + i * 4, 1, 3, o);
    fclose(o);
    free(img);
  }
  r3d_destroy(r);
  return 0;
}
