// Streaming LOD brick cache: the brick residency pump.  The reference keeps
// a compressed warm tier in host memory and, once per frame, asks for the
// bricks of the view cone at their desired LOD, evicts the least recently
// used slots and decodes the requests into them, publishing page entries
// for the shader (src/vk/vkbackend.c:3075-3106,5208-5230,5256-5340,
// 5416-5590).  Here the warm tier is the whole decoded pyramid in pinned
// host memory, the request set comes from r3d_host_stream_desired, and an
// update copies the chosen bricks into their slots with one 2 MiB
// host-to-device copy each, rebuilds those slots' quad words and block
// maxima, and uploads the page table: all ordered on the context's stream
// after the frames already queued, so no rendered frame ever sees a slot
// change under it.
#include <string.h>

#include <algorithm>
#include <vector>

#include "r3d_host.h"
#include "r3d_internal.h"

namespace r3d {

constexpr uint32_t kSlotBytes = 128u * 128u * 128u;

// Quad words and dilated 8^3 block maxima of the listed slots (the per-slot
// tables of k_slot_quads / k_slot_blockmax).  Grid: (blocks, jobs).
__global__ void k_stream_fill(const uint8_t *__restrict__ pool, const uint32_t *__restrict__ jobs,
                              uint32_t *__restrict__ quad, uint8_t *__restrict__ bmax) {
  const uint32_t s = jobs[blockIdx.y];
  const uint8_t *g = pool + (size_t)s * kSlotBytes;
  uint32_t *q = quad + (size_t)s * kSlotBytes;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < kSlotBytes;
       i += gridDim.x * blockDim.x) {
    const uint32_t x = i & 127u, y = (i >> 7) & 127u;
    const uint32_t dx = x < 127u ? 1u : 0u, dy = y < 127u ? 128u : 0u;
    q[i] = (uint32_t)g[i] | ((uint32_t)g[i + dx] << 8) | ((uint32_t)g[i + dy] << 16) |
           ((uint32_t)g[i + dy + dx] << 24);
  }
  for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < 4096u;
       e += gridDim.x * blockDim.x) {
    const uint32_t bx = e & 15u, by = (e >> 4) & 15u, bz = e >> 8;
    uint32_t m = 0;
    for (uint32_t z = bz * 8u; z <= min(bz * 8u + 8u, 127u); z++)
      for (uint32_t y = by * 8u; y <= min(by * 8u + 8u, 127u); y++) {
        const uint8_t *row = g + ((size_t)z << 14) + ((size_t)y << 7);
        for (uint32_t x = bx * 8u; x <= min(bx * 8u + 8u, 127u); x++)
          m = max(m, (uint32_t)row[x]);
      }
    bmax[(size_t)s * 4096u + e] = (uint8_t)m;
  }
}


// Copies the listed (slot, store index) bricks in, refills their tables and
// publishes the page shadow.
static int stream_upload(r3d_cuda_ctx *c, const std::vector<uint32_t> &slots,
                         const std::vector<uint32_t> &src) {
  cudaStream_t st = c->stream;
  for (size_t i = 0; i < slots.size(); i++)
    R3D_CUDA_TRY(c, cudaMemcpyAsync(c->pool + (size_t)slots[i] * kSlotBytes,
                                    c->store + (size_t)src[i] * kSlotBytes, kSlotBytes,
                                    cudaMemcpyHostToDevice, st));
  // the display filter, before the slot tables
  const int frc = postfilter_slots(c, 0u, c->pool, slots.data(), (uint32_t)slots.size());
  if (frc != R3D_OK) return frc;
  for (size_t j0 = 0; j0 < slots.size(); j0 += 65535u) {
    const uint32_t nj = (uint32_t)std::min<size_t>(slots.size() - j0, 65535u);
    R3D_CUDA_TRY(c, cudaMemcpyAsync(c->stream_jobs + j0, slots.data() + j0, nj * 4u,
                                    cudaMemcpyHostToDevice, st));
    k_stream_fill<<<dim3(64, nj), 256, 0, st>>>(c->pool, c->stream_jobs + j0, c->quad, c->bmax);
    R3D_CUDA_TRY(c, cudaGetLastError());
    // the job list is reused by the next chunk: keep the kernel ahead of it
    if (j0 + nj < slots.size()) R3D_CUDA_TRY(c, cudaStreamSynchronize(st));
  }
  R3D_CUDA_TRY(c, cudaMemcpyAsync(c->page, c->page_shadow, (size_t)c->page_words * 4u,
                                  cudaMemcpyHostToDevice, st));
  R3D_CUDA_TRY(c, cudaEventRecord(c->page_ev, st));
  return R3D_OK;
}

}  // namespace r3d

using namespace r3d;

void stream_reset(r3d_cuda_ctx *c) {
  cudaFreeHost(c->store);
  cudaFreeHost(c->page_shadow);
  cudaFree(c->stream_jobs);
  c->store = nullptr;
  c->page_shadow = nullptr;
  c->stream_jobs = nullptr;
  c->store_page.clear();
  c->slot_brick.clear();
  c->slot_use.clear();
  c->brick_slot.clear();
  c->stream_cand.clear();
  c->stream_mark.clear();
  c->stream_open = false;
  c->streaming = false;
}

extern "C" {

int r3d_cuda_stream_begin(r3d_cuda_ctx *c, const r3d_volume_desc *d, const uint8_t *voxels,
                          uint32_t nlev, uint32_t nslots) {
  if (!c || !d || !voxels) return fail(c, R3D_E_INVALID, "stream_begin: bad arguments");
  // the full pyramid, every brick resident, on the device first
  c->defer_tables = true;  // the full pool only feeds the host store
  int rc = r3d_cuda_bricks_build(c, d, voxels, nlev, 0u);
  c->defer_tables = false;
  if (rc != R3D_OK) return rc;
  stream_reset(c);
  cudaSetDevice(c->device);
  const uint32_t words = c->page_words, nall = c->nslots;
  const uint32_t coarse_off = c->br.off[nlev - 1u];
  const uint32_t ncoarse = c->br.bd[nlev - 1u][0] * c->br.bd[nlev - 1u][1] * c->br.bd[nlev - 1u][2];
  if (nslots < ncoarse || nslots > nall || nslots >= (1u << 24)) {
    c->have_bricks = false;
    return fail(c, R3D_E_INVALID, "stream_begin: %u slots; the coarsest level alone needs %u and "
                                  "the whole pyramid has %u", nslots, ncoarse, nall);
  }
  if (!c->page_ev) R3D_CUDA_TRY(c, cudaEventCreateWithFlags(&c->page_ev, cudaEventDisableTiming));
  c->store_page.resize(words);
  R3D_CUDA_TRY(c, copy_sync(c->stream, c->store_page.data(), c->page, (size_t)words * 4u));
  cudaError_t e = cudaMallocHost(&c->store, (size_t)nall * kSlotBytes);
  if (e == cudaSuccess) e = cudaMallocHost(&c->page_shadow, (size_t)words * 4u);
  if (e == cudaSuccess) e = cudaMalloc(&c->stream_jobs, (size_t)std::min(nslots, 65535u) * 4u);
  if (e == cudaSuccess) e = copy_sync(c->stream, c->store, c->pool, (size_t)nall * kSlotBytes);
  if (e != cudaSuccess) {
    stream_reset(c);
    c->have_bricks = false;
    return cuda_fail(c, e, "stream_begin: host store");
  }
  // the device pool shrinks to nslots slots, all empty
  cudaFree(c->pool);
  c->pool = nullptr;
  e = cudaMalloc(&c->pool, (size_t)nslots * kSlotBytes);
  if (e == cudaSuccess) e = cudaMemsetAsync(c->pool, 0, (size_t)nslots * kSlotBytes, c->stream);
  if (e != cudaSuccess) {
    stream_reset(c);
    c->have_bricks = false;
    return cuda_fail(c, e, "stream_begin: slot pool");
  }
  c->nslots = nslots;
  c->abpa = atlas_bpa(nslots);
  c->br.pool = c->pool;
  c->br.nslots = nslots;
  rc = build_blockmax(c);
  if (rc != R3D_OK) {
    stream_reset(c);
    c->have_bricks = false;
    return rc;
  }
  c->slot_brick.assign(nslots, R3D_BRICK_ABSENT);
  c->slot_use.assign(nslots, 0u);
  c->brick_slot.assign(words, R3D_BRICK_ABSENT);
  memcpy(c->page_shadow, c->store_page.data(), R3D_BRICK_PAGE_HEADER * 4u);
  for (uint32_t w = R3D_BRICK_PAGE_HEADER; w < words; w++) c->page_shadow[w] = R3D_BRICK_ABSENT;
  // the coarsest level is resident from the start and never evicted
  // (vkbackend.c:5317-5327)
  c->stream_frame = 1;
  std::vector<uint32_t> slots, src;
  for (uint32_t i = 0; i < ncoarse; i++) {
    const uint32_t b = coarse_off + i, ent = c->store_page[b];
    c->slot_brick[i] = b;
    c->slot_use[i] = c->stream_frame;
    c->brick_slot[b] = i;
    c->page_shadow[b] = (ent >> 24) >= 5u ? i | (ent & 0xFF000000u) : R3D_BRICK_ABSENT;
    slots.push_back(i);
    src.push_back(ent & 0xFFFFFFu);
  }
  c->streaming = true;
  rc = stream_upload(c, slots, src);
  if (rc == R3D_OK) R3D_CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  return rc;
}

void r3d_cuda_stream_view_of(const r3d_frame_params *p, const float ext[3], uint32_t budget,
                             r3d_stream_view *v) {
  if (!p || !ext || !v) return;
  memset(v, 0, sizeof *v);
  const float c[3] = {ext[0] * 0.5f, ext[1] * 0.5f, ext[2] * 0.5f};
  const float t[3] = {p->vol_tx, p->vol_ty, p->vol_tz};
  float q[3];
  for (int a = 0; a < 3; a++) q[a] = (p->cam_origin[a] - t[a]) - c[a];
  for (int a = 0; a < 3; a++) {  // R^T q + c and R^T fwd (common.slang:45-52)
    v->eye[a] = fmaf(p->vol_r2[a], q[2], fmaf(p->vol_r1[a], q[1], p->vol_r0[a] * q[0])) + c[a];
    v->fwd[a] = fmaf(p->vol_r2[a], p->cam_forward[2],
                     fmaf(p->vol_r1[a], p->cam_forward[1], p->vol_r0[a] * p->cam_forward[0]));
  }
  const float up2 = p->cam_up[0] * p->cam_up[0] + p->cam_up[1] * p->cam_up[1] +
                    p->cam_up[2] * p->cam_up[2];
  const float rt2 = p->cam_right[0] * p->cam_right[0] + p->cam_right[1] * p->cam_right[1] +
                    p->cam_right[2] * p->cam_right[2];
  v->half_tan = sqrtf(up2 + rt2);  // right and up are pre-scaled by tan(fov/2)
  v->pixel_cone = 2.0f * sqrtf(up2) / (float)(p->viewport[1] ? p->viewport[1] : 1u) *
                  exp2f(p->lod_bias);
  if (p->slab_depth && !(p->view_flags & (R3D_VIEW_OBLIQUE | R3D_VIEW_CROP))) {
    v->slice_z0 = (uint32_t)p->slab_z0;
    v->slice_depth = p->slab_depth;
  }
  v->gate = p->skip_gate;
  v->budget = budget;
}

int r3d_cuda_stream_collect_begin(r3d_cuda_ctx *c) {
  if (!c) return R3D_E_INVALID;
  if (!c->streaming || !c->have_bricks)
    return fail(c, R3D_E_STATE, "stream_collect_begin: no streaming cache");
  cudaSetDevice(c->device);
  // the previous update's page upload reads the shadow: let it finish
  R3D_CUDA_TRY(c, cudaEventSynchronize(c->page_ev));
  const uint32_t nlev = c->br.nlev, frame = ++c->stream_frame;
  // pin the coarsest level's stamps
  const uint32_t coarse_off = c->br.off[nlev - 1u];
  const uint32_t ncoarse = c->br.bd[nlev - 1u][0] * c->br.bd[nlev - 1u][1] * c->br.bd[nlev - 1u][2];
  for (uint32_t i = 0; i < ncoarse; i++) {
    const uint32_t s = c->brick_slot[coarse_off + i];
    if (s != R3D_BRICK_ABSENT) c->slot_use[s] = frame;
  }
  c->stream_mark.assign(c->page_words, 0);
  c->stream_cand.clear();
  c->stream_cand.reserve(c->page_words);  // a brick is listed once
  c->stream_open = true;
  return R3D_OK;
}

static int collect_check(r3d_cuda_ctx *c, const char *what) {
  if (!c) return R3D_E_INVALID;
  if (!c->stream_open) return fail(c, R3D_E_STATE, "%s: no open collect (stream_collect_begin)", what);
  return R3D_OK;
}

}  // extern "C"

// grows the candidate list by what a collect appended into its tail
template <class F>
static void collect_into(r3d_cuda_ctx *c, F f) {
  const uint32_t n0 = (uint32_t)c->stream_cand.size(), cap = c->page_words;
  c->stream_cand.resize(cap);
  const uint32_t n = f(c->stream_cand.data(), cap, n0);
  c->stream_cand.resize(n);
}

extern "C" {

int r3d_cuda_stream_collect_view(r3d_cuda_ctx *c, const r3d_stream_view *v) {
  int rc = collect_check(c, "stream_collect_view");
  if (rc != R3D_OK) return rc;
  if (!v) return fail(c, R3D_E_INVALID, "stream_collect_view: no view");
  collect_into(c, [&](r3d_stream_cand *out, uint32_t cap, uint32_t n0) {
    return n0 + r3d_host_stream_desired(c->store_page.data(), c->page_words, v->eye, v->fwd,
                                        v->half_tan, v->pixel_cone, v->slice_z0, v->slice_depth,
                                        v->gate, c->stream_mark.data(), out + n0, cap - n0);
  });
  return R3D_OK;
}

int r3d_cuda_stream_collect_box(r3d_cuda_ctx *c, const float lo[3], const float hi[3],
                                float pixel_cone, float gate) {
  int rc = collect_check(c, "stream_collect_box");
  if (rc != R3D_OK) return rc;
  if (!lo || !hi) return fail(c, R3D_E_INVALID, "stream_collect_box: no box");
  collect_into(c, [&](r3d_stream_cand *out, uint32_t cap, uint32_t n0) {
    return r3d_host_stream_box(c->store_page.data(), c->page_words, lo, hi, pixel_cone, gate,
                               c->stream_mark.data(), out, cap, n0);
  });
  return R3D_OK;
}

int r3d_cuda_stream_collect_point(r3d_cuda_ctx *c, const float p[3], uint32_t level, float gate) {
  int rc = collect_check(c, "stream_collect_point");
  if (rc != R3D_OK) return rc;
  if (!p) return fail(c, R3D_E_INVALID, "stream_collect_point: no point");
  collect_into(c, [&](r3d_stream_cand *out, uint32_t cap, uint32_t n0) {
    return r3d_host_stream_point(c->store_page.data(), c->page_words, p, level, gate,
                                 c->stream_mark.data(), out, cap, n0);
  });
  return R3D_OK;
}

int r3d_cuda_stream_submit(r3d_cuda_ctx *c, uint32_t budget, r3d_stream_stats *out) {
  int rc = collect_check(c, "stream_submit");
  if (rc != R3D_OK) return rc;
  c->stream_open = false;
  cudaSetDevice(c->device);
  const uint32_t frame = c->stream_frame, n = (uint32_t)c->stream_cand.size();
  r3d_stream_cand *cand = c->stream_cand.data();
  r3d_host_stream_sort(cand, n);  // every collect's candidates, nearest first
  r3d_stream_stats stats;
  memset(&stats, 0, sizeof stats);
  stats.desired = n;
  std::vector<uint32_t> req;
  for (uint32_t k = 0; k < n; k++) {  // resident ones are touched, the rest requested
    const uint32_t b = cand[k].brick, s = c->brick_slot[b];
    if (s != R3D_BRICK_ABSENT)
      c->slot_use[s] = frame;
    else
      req.push_back(b);
  }
  stats.requested = (uint32_t)req.size();
  std::vector<uint32_t> slots, src;
  for (size_t k = 0; k < req.size() && slots.size() < budget; k++) {
    // free slot first, else the least recently used one not wanted this
    // frame (vkbackend.c:5320-5332); none left: stop rather than thrash
    uint32_t best = R3D_BRICK_ABSENT, bu = UINT32_MAX;
    for (uint32_t s = 0; s < c->nslots; s++) {
      if (c->slot_brick[s] == R3D_BRICK_ABSENT) {
        best = s;
        break;
      }
      if (c->slot_use[s] != frame && c->slot_use[s] < bu) {
        bu = c->slot_use[s];
        best = s;
      }
    }
    if (best == R3D_BRICK_ABSENT) break;
    const uint32_t old = c->slot_brick[best], b = req[k], ent = c->store_page[b];
    if (old != R3D_BRICK_ABSENT) {
      c->brick_slot[old] = R3D_BRICK_ABSENT;
      c->page_shadow[old] = R3D_BRICK_ABSENT;
      stats.evicted++;
    }
    c->slot_brick[best] = b;
    c->slot_use[best] = frame;
    c->brick_slot[b] = best;
    c->page_shadow[b] = (ent >> 24) >= 5u ? best | (ent & 0xFF000000u) : R3D_BRICK_ABSENT;
    slots.push_back(best);
    src.push_back(ent & 0xFFFFFFu);
  }
  stats.uploaded = (uint32_t)slots.size();
  for (uint32_t s = 0; s < c->nslots; s++) stats.resident += c->slot_brick[s] != R3D_BRICK_ABSENT;
  c->stream_cand.clear();
  if (!slots.empty()) rc = stream_upload(c, slots, src);
  if (out) *out = stats;
  return rc;
}

int r3d_cuda_bricks_refilter(r3d_cuda_ctx *c) {
  if (!c) return R3D_E_INVALID;
  if (!c->have_bricks) return fail(c, R3D_E_STATE, "bricks_refilter: no brick cache");
  if (!c->streaming)
    return fail(c, R3D_E_STATE, "bricks_refilter: a resident cache is filtered when it is built; "
                                "build it again to apply another filter");
  cudaSetDevice(c->device);
  R3D_CUDA_TRY(c, cudaEventSynchronize(c->page_ev));
  // every resident brick but the pinned coarsest level's, again from the
  // store through the current filter (vkbackend.c:4875-4906 invalidates
  // them to re-stream; here they are refilled within the call)
  const uint32_t nlev = c->br.nlev, c0 = c->br.off[nlev - 1u];
  const uint32_t c1 = c0 + c->br.bd[nlev - 1u][0] * c->br.bd[nlev - 1u][1] * c->br.bd[nlev - 1u][2];
  std::vector<uint32_t> slots, src;
  for (uint32_t s = 0; s < c->nslots; s++) {
    const uint32_t b = c->slot_brick[s];
    if (b == R3D_BRICK_ABSENT || (b >= c0 && b < c1)) continue;
    slots.push_back(s);
    src.push_back(c->store_page[b] & 0xFFFFFFu);
  }
  int rc = slots.empty() ? R3D_OK : stream_upload(c, slots, src);
  if (rc == R3D_OK) rc = r3d_cuda_surfvol_mark(c);  // a baked flattened window re-bakes
  return rc;
}

int r3d_cuda_stream_update(r3d_cuda_ctx *c, const r3d_stream_view *v, r3d_stream_stats *out) {
  if (!c || !v) return fail(c, R3D_E_INVALID, "stream_update: bad arguments");
  if (!c->streaming || !c->have_bricks)
    return fail(c, R3D_E_STATE, "stream_update: no streaming cache");
  int rc = r3d_cuda_stream_collect_begin(c);
  if (rc == R3D_OK) rc = r3d_cuda_stream_collect_view(c, v);
  if (rc == R3D_OK) rc = r3d_cuda_stream_submit(c, v->budget, out);
  c->stream_open = false;
  return rc;
}

}  // extern "C"
