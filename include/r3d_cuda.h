/* C-ABI of the sm_100a volume-raycast library (libr3d_b200.so).
 *
 * This is the layer beneath render3d's render-backend interface
 * (reference src/render/render.h): render3d's Vulkan backend records one
 * raycast dispatch per view (src/vk/vkbackend.c:7121-7173) of the compute
 * shader src/shaders/raycast.slang; this library replaces that dispatch and
 * the resources it samples with hand-written CUDA kernels.  r3d_render.h
 * builds the headless render.h subset on top of these calls.
 *
 * Conventions: every call returns R3D_OK (0) or a negative R3D_E_* code and
 * leaves a message in r3d_cuda_last_error(ctx); nothing aborts or throws.
 * Calls are stream-ordered on the stream passed (NULL = the context's own
 * stream); a context is used by one host thread at a time.  Output buffers
 * may be device pointers (asynchronous) or host pointers (the call copies to
 * them and synchronizes).  No CUDA types appear here: streams are void *. */
#ifndef R3D_CUDA_H
#define R3D_CUDA_H

#include <stddef.h>
#include <stdint.h>

#include "r3d_host.h"
#include "r3d_types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct r3d_cuda_ctx r3d_cuda_ctx;

enum {
  R3D_OK = 0,
  R3D_E_INVALID = -1,     /* bad argument */
  R3D_E_CUDA = -2,        /* CUDA runtime error (message names it) */
  R3D_E_NOMEM = -3,       /* device or host allocation failed */
  R3D_E_UNSUPPORTED = -4, /* a feature this library does not implement */
  R3D_E_STATE = -5,       /* no volume / bricks / TF uploaded yet */
  R3D_E_DEVICE = -6,      /* a kernel reported a data error (see status) */
  R3D_E_TIMEOUT = -7,     /* a bounded device wait ran out */
};

/* Device status bits (r3d_cuda_status). */
#define R3D_STATUS_PAGE_RANGE 1u  /* page word or slot index out of range */
#define R3D_STATUS_QUEUE 2u       /* batched queue descriptor rejected */
#define R3D_STATUS_WAIT 4u        /* a bounded spin-wait gave up */

/* --- context ----------------------------------------------------------- */

/* Creates a context on CUDA device `device` with its own stream. */
int r3d_cuda_create(int device, r3d_cuda_ctx **out);
void r3d_cuda_destroy(r3d_cuda_ctx *ctx);
const char *r3d_cuda_last_error(const r3d_cuda_ctx *ctx);
/* The context's stream (a cudaStream_t). */
void *r3d_cuda_stream(r3d_cuda_ctx *ctx);
/* Synchronizes, returns and (if clear) resets the device status bits. */
int r3d_cuda_status(r3d_cuda_ctx *ctx, uint32_t *bits, int clear);

/* --- scene state --------------------------------------------------------- */

/* Cube volume: copies nx*ny*nz u8 voxels (x fastest; host or device
 * pointer), builds the full mip chain (2x box, (sum+4)/8) and the dilated
 * 8^3 occupancy grid on the device.  Replaces r3d_upload_volume
 * (reference src/render/render.h:20, src/vk/vkbackend.c:1508-1672). */
int r3d_cuda_upload_volume(r3d_cuda_ctx *ctx, const r3d_volume_desc *d, const uint8_t *voxels);

/* 256-entry RGBA8 transfer function (reference src/render/render.h:240). */
int r3d_cuda_set_transfer(r3d_cuda_ctx *ctx, const uint8_t rgba[256][4]);

/* R3D_QUALITY_FULL (six-tap) or R3D_QUALITY_FAST (four-tap) gradients
 * (reference src/render/render.h:242). */
int r3d_cuda_set_quality(r3d_cuda_ctx *ctx, uint32_t quality);

/* Front-to-back termination opacity, default 0.98 (the reference's
 * ALPHA_CUTOFF constant, src/shaders/raycast.slang:124).  (0, 1]. */
int r3d_cuda_set_alpha_cutoff(r3d_cuda_ctx *ctx, float cutoff);

/* LOD brick cache built on the device from a raw volume: nlev levels of the
 * (sum+4)/8 box pyramid over 128^3 bricks, zero-padded at the far edges; a
 * brick is resident when its maximum is >= min_max (0: all resident).
 * Writes render3d's page table (64-word header + one word per brick, entry
 * = slot | max << 24, 0xFFFFFFFF absent; src/vk/vkbackend.c:4184-4206).
 * voxels may be a host or device pointer. */
int r3d_cuda_bricks_build(r3d_cuda_ctx *ctx, const r3d_volume_desc *d, const uint8_t *voxels,
                          uint32_t nlev, uint32_t min_max);

/* Brick cache from an existing page table and slot pool (host pointers):
 * page_words u32 words in render3d's LOD format and nslots 128^3 slots,
 * x fastest.  The header is validated; scales must be powers of two. */
int r3d_cuda_bricks_load(r3d_cuda_ctx *ctx, const uint32_t *page, uint32_t page_words,
                         const uint8_t *slots, uint32_t nslots);

/* brick_mode word for r3d_frame_params (abpa | nlev << 8 | 0x20000;
 * reference src/vk/vkbackend.c:4511-4517), 0 when no bricks are loaded. */
uint32_t r3d_cuda_brick_mode(const r3d_cuda_ctx *ctx);

/* Sizes of the loaded brick cache; and a copy of it (host pointers, either
 * may be NULL) for inspection and tests. */
int r3d_cuda_bricks_info(const r3d_cuda_ctx *ctx, uint32_t *page_words, uint32_t *nslots,
                         uint32_t shape[3], uint32_t *nlev);
int r3d_cuda_bricks_read(r3d_cuda_ctx *ctx, uint32_t *page, uint8_t *slots);

/* Streaming LOD brick cache: the brick residency pump of render3d's
 * streamed bricks mode (reference src/render/render.h:44-50 with a pool
 * smaller than the volume; src/vk/vkbackend.c:3075-3106,5208-5340,
 * 5416-5590).  _begin builds the whole LOD pyramid of a raw volume (as
 * r3d_cuda_bricks_build with min_max 0) into pinned host memory and keeps
 * only nslots device slots, of which the coarsest level takes its share for
 * good.  Each _update requests the bricks of the view cone at their desired
 * LOD (r3d_host_stream_desired), keeps the resident ones, and fills up to
 * `budget` requests, nearest first, into free or least-recently-used slots
 * not wanted this frame: one host-to-device copy per brick, then the slots'
 * tables and the page table, all on the context's stream.  Bricks whose
 * maximum is below 5 stay unpublished, like the reference's decoded air.
 * Renders on the context's stream after an update see its bricks; views
 * use r3d_cuda_brick_mode as for a resident cache. */
typedef struct r3d_stream_view {
  float eye[3], fwd[3]; /* volume-normalized camera position and direction */
  float half_tan;       /* tan(fov / 2) */
  float pixel_cone;     /* footprint of one pixel per unit distance */
  uint32_t slice_z0, slice_depth; /* z window in voxels (depth 0: none) */
  float gate;           /* bricks with max < gate * 255 are never requested */
  uint32_t budget;      /* bricks copied in by this update, at most */
} r3d_stream_view;
typedef struct r3d_stream_stats {
  uint32_t desired;   /* bricks of the request set (parents included) */
  uint32_t requested; /* of those, not resident */
  uint32_t uploaded;  /* copied in by this update */
  uint32_t evicted;   /* slots taken from other bricks */
  uint32_t resident;  /* occupied slots afterwards */
} r3d_stream_stats;
int r3d_cuda_stream_begin(r3d_cuda_ctx *ctx, const r3d_volume_desc *d, const uint8_t *voxels,
                          uint32_t nlev, uint32_t nslots);
/* The pump's inputs for a view, as render3d's main loop derives them
 * (src/main.c:6886-6900): the camera moved into volume space by the view's
 * model transform (ext = the volume's extent, r3d_bricks_extent), the
 * diagonal half-angle tan(fov/2) * sqrt(1 + aspect^2), the pixel cone
 * 2 tan(fov/2) / height * 2^lod_bias, the axis-slab z window and the
 * skip gate. */
void r3d_cuda_stream_view_of(const r3d_frame_params *p, const float ext[3], uint32_t budget,
                             r3d_stream_view *view);
int r3d_cuda_stream_update(r3d_cuda_ctx *ctx, const r3d_stream_view *view,
                           r3d_stream_stats *stats);
/* The multi-view pump (reference r3d_bricks_stream_begin / _box / _point /
 * _submit, src/render/render.h:128-139, src/vk/vkbackend.c:5244-5414,
 * 5519-5590): _collect_begin opens a frame's request set and pins the
 * coarsest level; _collect_view adds a view's cone (budget unused),
 * _collect_box a volume-normalized box at the level matching pixel_cone
 * (r3d_host_stream_box), _collect_point one brick of a level and its parent
 * (r3d_host_stream_point), each listing a brick at most once per frame;
 * _submit sorts them all (priority, then distance), touches the resident
 * ones and fills up to budget of the rest as _update does, which is begin +
 * view + submit.  Collects and submit without an open frame fail with
 * R3D_E_STATE. */
int r3d_cuda_stream_collect_begin(r3d_cuda_ctx *ctx);
int r3d_cuda_stream_collect_view(r3d_cuda_ctx *ctx, const r3d_stream_view *view);
int r3d_cuda_stream_collect_box(r3d_cuda_ctx *ctx, const float lo[3], const float hi[3],
                                float pixel_cone, float gate);
int r3d_cuda_stream_collect_point(r3d_cuda_ctx *ctx, const float p[3], uint32_t level, float gate);
int r3d_cuda_stream_submit(r3d_cuda_ctx *ctx, uint32_t budget, r3d_stream_stats *stats);

/* Tiled slab: render3d's slab mode for wide, thin windows (reference
 * src/core/slab.h, src/vk/vkbackend.c:2128-2335, sampled by
 * src/shaders/raycast.slang:423-455).  The volume (nx x ny x nz, x fastest,
 * host or device) is copied to the device; a window of wz slices (4 <= wz
 * <= nz) from z0 lives in a z ring of tiles of at most 2048 texels per axis,
 * each with a 1-texel apron copied from its neighbours (clamped at the
 * edges).  An overview pyramid at scales 4, 8, ... up to the scale that fits
 * the whole plane in 2046-texel tiles (4x box of the slice, then 2x chains,
 * truncating averages) serves far footprints.  Views set slab_grid and
 * the other slab fields with r3d_cuda_slab_params (slab_depth may be
 * lowered).  _window moves the window to z0 (clamped to nz - wz),
 * refilling only the ring layers of slices that enter it, after the frames
 * already queued on the context's stream. */
int r3d_cuda_slab_build(r3d_cuda_ctx *ctx, const r3d_volume_desc *d, const uint8_t *voxels,
                        uint32_t wz, uint32_t z0);
int r3d_cuda_slab_window(r3d_cuda_ctx *ctx, uint32_t z0);
void r3d_cuda_slab_params(const r3d_cuda_ctx *ctx, r3d_frame_params *p);
/* Copy of tile `tile` of level `level` (0 = base grid, 1.. overview, scale
 * 4 << (level - 1)): (px + 2) x (py + 2) x wz bytes; dims receives them. */
int r3d_cuda_slab_read(r3d_cuda_ctx *ctx, uint32_t level, uint32_t tile, uint8_t *out,
                       uint32_t dims[3]);

/* XY clipmap: render3d's clip mode for whole cross-sections (reference
 * src/core/clip.h, src/vk/vkclip.c, sampled by
 * src/shaders/raycast.slang:357-408).  Six nested levels of spacing 2^l
 * around a focus, each a 2048^2 texture (2046 payload texels and a 1-texel
 * apron) with a ring of depth_max / 2^l + 3 (at least 4) level slices.
 * Level 0 is the volume (nx x ny x nz, x fastest, host or device; copied to
 * the device), level 1 its 2^3 box with coordinates clamped at full
 * resolution, levels 2..5 the tight 2^3 box pyramid of tools/mkpyramid; all
 * boxes truncate.  _frame recentres the levels whose coverage the focus
 * (fx, fy in voxels) has drifted from by more than a quarter (origins
 * snapped to 16 level voxels), fills the ring layers of the window from z0
 * that are missing, on the context's stream, and writes the view fields
 * (slab_nx/ny/z0/wz/depth, clip_orig, clip_valid) into p when p is not
 * NULL. */
int r3d_cuda_clip_build(r3d_cuda_ctx *ctx, const r3d_volume_desc *d, const uint8_t *voxels,
                        uint32_t depth_max);
int r3d_cuda_clip_frame(r3d_cuda_ctx *ctx, double fx, double fy, uint64_t z0,
                        r3d_frame_params *p);
void r3d_cuda_clip_params(const r3d_cuda_ctx *ctx, r3d_frame_params *p);
/* Copy of ring layer `layer` of level `level` (2048^2 bytes). */
int r3d_cuda_clip_read(r3d_cuda_ctx *ctx, uint32_t level, uint32_t layer, uint8_t *out);

/* Virtual slab: render3d's vslab mode (reference src/render/render.h:161-191,
 * src/core/vslab.h, src/vk/vkbackend.c:5675-6660, sampled by
 * src/shaders/raycast.slang:321-367).  A W x H x D window anywhere in the
 * volume (nx x ny x nz, x fastest, host or device; copied to the device),
 * rendered from world-anchored toroidal tile grids laid out by
 * r3d_host_vslab_init with z_margin resident slices on each side.  The
 * reference streams cells from a shard store on a worker thread; here
 * _frame plans the frame's fills (r3d_host_vslab_plan, at most budget cell
 * fills), runs them on the context's stream, records them in the ledger,
 * publishes the validity table and writes the view fields (slab_grid with
 * bit 24 set, brick_mode = packed pyramid grids, slab_wz/z0/nx/ny/px/py/
 * depth/x0/y0) into p when p is not NULL.  Frames queued later on the
 * context's stream see the fills.  R3D_E_INVALID for a window
 * r3d_host_vslab_init rejects or whose grids do not fit the view fields
 * (base 63, pyramid 15 tiles per axis). */
typedef struct r3d_vslab_stats {
  uint32_t jobs;    /* cell fills this frame */
  uint32_t slices;  /* base slices written this frame */
  uint32_t pending; /* window cells whose visible span is still missing */
  uint32_t pad;
  int64_t origin[3]; /* window origin x0, y0, z0 (r3d_vslab_get) */
} r3d_vslab_stats;
int r3d_cuda_vslab_begin(r3d_cuda_ctx *ctx, const r3d_volume_desc *d, const uint8_t *voxels,
                         uint32_t W, uint32_t H, uint32_t D, uint32_t z_margin);
int r3d_cuda_vslab_frame(r3d_cuda_ctx *ctx, double fx, double fy, int64_t z0, uint32_t budget,
                         r3d_frame_params *p, r3d_vslab_stats *st);
void r3d_cuda_vslab_params(const r3d_cuda_ctx *ctx, r3d_frame_params *p);
/* The layout (origin included) of the loaded window. */
int r3d_cuda_vslab_layout(const r3d_cuda_ctx *ctx, r3d_vslab_layout *out);
/* Copy of tile `tile` ((px + 2)^2 * wz bytes, layer-major) and of the
 * validity table (4 words per base tile: key, za, zb, 0). */
int r3d_cuda_vslab_read(r3d_cuda_ctx *ctx, uint32_t tile, uint8_t *out);
int r3d_cuda_vslab_table(r3d_cuda_ctx *ctx, uint32_t *out);

/* Flattened-segment (surf) views: render3d's segment pane (reference
 * src/render/render.h:193-202 and 58-107, src/vk/vkbackend.c:1674-2066,
 * src/shaders/surfvol.comp, raycast.slang:515-638).
 * _surf_begin: the segment as two w x h RGBA32F grids (host or device),
 * surface points (xyz voxels + valid flag in w) and unit normals; w, h >= 3.
 * Replaces earlier grids (r3d_surf_begin and r3d_surf_swap).
 * _surfvol_begin: a w x h x layers flattened volume (two bytes a texel: CT
 * and overlay), nback layers behind the surface, grid scale (sx, sy) cells
 * per flattened voxel.  _surfvol_window: texel (x, y, l) samples the LOD
 * brick cache at surface(u, v) + normal(u, v) * (zoff0 + l - nback), u =
 * u0 + (x + 0.5) * step (v likewise), at the level of the xy pitch, and the
 * whole window is baked on the context's stream (the reference bakes row
 * bands over frames).  _surfvol_overlay selects the overlay atlas baked into
 * the second byte (0 ink, 1 3D ink, 3 registration, -1 none) and _mark
 * re-bakes after the brick cache or an overlay changed.  _surfvol_params
 * writes the view fields (slab_x0/y0 = u0/v0, slab_px = step, slab_nx/ny/wz
 * = window, slab_grid = nback, max_mip = zoff0, vol_tx/ty = grid scale) and
 * sets R3D_VIEW_SURF; the caller sets the view centre (cam_origin x, y),
 * half extents (cam_right x, cam_up y), slab_z0 (normal offset) and
 * slab_depth (marched layers).  _surfmask: a grid-space class image
 * (0 unlabeled, 1 background, 2 ink) tinted by overlay_flags bit 5; NULL
 * clears it. */
int r3d_cuda_surf_begin(r3d_cuda_ctx *ctx, uint32_t w, uint32_t h, const float *coords_rgba,
                        const float *normals_rgba);
int r3d_cuda_surfvol_begin(r3d_cuda_ctx *ctx, uint32_t w, uint32_t h, uint32_t layers,
                           uint32_t nback, float sx, float sy);
int r3d_cuda_surfvol_window(r3d_cuda_ctx *ctx, double u0, double v0, float step, float zoff0);
int r3d_cuda_surfvol_overlay(r3d_cuda_ctx *ctx, int atlas);
/* Live 2.5D ink prediction (reference r3d_surfvol_inkpred / _clear,
 * src/render/render.h:222-230, src/shaders/surfvol.comp:127-150): w x h
 * float probabilities, texel (0, 0) at grid coordinates (g0u, g0v),
 * px_per_grid texels per grid unit.  Each bake samples it (clamp-to-edge
 * bilinear) once per (u, v) column and writes it into G over every layer
 * where the column falls inside it, replacing the overlay atlas there.
 * Uploading re-bakes the window; pred NULL drops it and re-bakes. */
int r3d_cuda_surfvol_inkpred(r3d_cuda_ctx *ctx, const float *pred, uint32_t w, uint32_t h,
                             float g0u, float g0v, float px_per_grid);
int r3d_cuda_surfvol_mark(r3d_cuda_ctx *ctx);
void r3d_cuda_surfvol_params(const r3d_cuda_ctx *ctx, r3d_frame_params *p);
/* Copy of the flattened volume (w * h * layers * 2 bytes, x fastest). */
int r3d_cuda_surfvol_read(r3d_cuda_ctx *ctx, uint8_t *out);
int r3d_cuda_surfmask(r3d_cuda_ctx *ctx, const uint8_t *m, uint32_t w, uint32_t h);

/* Post-decode 3D display filter (reference r3d_bricks_postfilter /
 * r3d_bricks_refilter, src/render/render.h:62-73, src/shaders/postfilt.comp):
 * each brick that lands in a slot after the call is filtered once, with
 * its neighbourhoods clamped to the slot.  mode: low byte 1 median of 3^3,
 * 2 median of 5^3, 3 max of 3^3, 4 max of 5^3 (other values: none); bit 8
 * adds an unsharp pass after it, centre + amount * (centre - mean of 3^3)
 * clamped to [0, 1].  targets: bit 0 the CT bricks, bit 1 the ink overlay
 * atlas, bit 2 the 3D ink atlas (0: the CT bricks).  Applies to resident
 * builds, streamed uploads and overlay builds and loads; the settings
 * survive new builds.  Per-slot tables (block maxima, quads) derive from
 * the filtered bricks; page-table maxima stay those of the bricks as
 * built, as the reference keeps the decoder's.  _refilter (streaming
 * caches only; R3D_E_STATE for a resident cache) copies every resident
 * brick but the coarsest level's in again from the host store through the
 * current filter, and re-bakes a flattened window. */
int r3d_cuda_bricks_postfilter(r3d_cuda_ctx *ctx, uint32_t mode, float amount, uint32_t targets);
int r3d_cuda_bricks_refilter(r3d_cuda_ctx *ctx);

/* Slot-parallel overlay atlases of the LOD brick cache (reference
 * src/render/render.h:51-101; sampled by src/shaders/raycast.slang:45-115,
 * 872-914,1000-1014,1032-1036): which = 0 ink (overlay_flags bit 0, tinted
 * by the palette id in bits 8..15), 1 3D ink (bit 2), 2 paint labels,
 * class ids 1..8 (bit 3), 3 registered second scan (bit 4, fuse weight in
 * bits 16..23).  Each holds one 128^3 u8 brick per CT slot, in the CT
 * pool's slot order (absent = 0).  _load takes the slot contents (host or
 * device, nslots * 128^3 bytes; NULL removes the atlas); _build cuts them
 * from a raw volume of the cache's shape: the CT's (sum+4)/8 box pyramid,
 * or for labels the level-0 voxel at (x, y, z) << level
 * (src/core/labelvol.c:172-196).  Rebuilding or reloading the brick cache
 * removes every overlay. */
int r3d_cuda_bricks_overlay_load(r3d_cuda_ctx *ctx, uint32_t which, const uint8_t *slots);
/* CPU-sourced atlases (reference r3d_bricks_labels / _labels_sync,
 * r3d_bricks_regatlas / _sync / _detach, src/render/render.h:74-97,
 * src/vk/vkbackend.c:4908-5150): _attach gives atlas `which` a source of
 * per-brick content (r3d_brick_src); a missing atlas starts cleared, and
 * re-attaching (or attaching to one built or loaded) zeroes every slot
 * before refilling it.  Each _sync round picks up to budget slots (0 or
 * over 16: 16) by r3d_host_atlas_pick: stale slots zeroed first, else
 * slots whose brick's generation changed, fetched on the calling thread;
 * it uploads them on the context's stream and reports how many in
 * *synced.  _detach drops the source and keeps the atlas; a sync without a
 * source does nothing.  A new brick cache detaches every source. */
int r3d_cuda_bricks_atlas_attach(r3d_cuda_ctx *ctx, uint32_t which, const r3d_brick_src *src);
int r3d_cuda_bricks_atlas_sync(r3d_cuda_ctx *ctx, uint32_t which, uint32_t budget, uint32_t *synced);
int r3d_cuda_bricks_atlas_detach(r3d_cuda_ctx *ctx, uint32_t which);
/* Reads atlas `which` back as nslots 128^3 slots (the layout _load takes). */
int r3d_cuda_bricks_overlay_read(r3d_cuda_ctx *ctx, uint32_t which, uint8_t *slots);
int r3d_cuda_bricks_overlay_build(r3d_cuda_ctx *ctx, uint32_t which, const r3d_volume_desc *d,
                                  const uint8_t *voxels);

/* Copy of cube mip level `level` or (level == -1) the occupancy grid into a
 * host buffer; dims receives its size. */
int r3d_cuda_cube_read(r3d_cuda_ctx *ctx, int level, uint8_t *out, uint32_t dims[3]);

/* Single-level brick atlas: render3d's bricks mode without the LOD flag, the
 * decoded shard of a c5s volume (reference src/shaders/raycast.slang:163-180,
 * 284-288,800-860; residency and atlas upkeep src/vk/vkbackend.c:3241-3330,
 * 4060-4075,4236-4273).  The volume is a cube of edge = bpa * 128 voxels
 * (x fastest, host or device pointer, 1 <= bpa <= 255).  The atlas holds
 * abpa^3 slots of 128^3 (1 <= abpa <= bpa); slot s sits at texel
 * (s % abpa, s / abpa % abpa, s / abpa^2) * 128 of one (abpa * 128)^3
 * texture with 4 mips ((sum+4)/8 box), and a world-indexed 8^3 occupancy
 * grid ((bpa * 16)^3, block maxima of resident bricks, 0 elsewhere, then
 * 26-neighbour max dilation) serves the empty-space skip.  slot_of (host,
 * bpa^3 entries in brick order) gives each brick's slot, or 0xFFFFFFFF for
 * a brick that is not resident; NULL puts brick b in slot b and needs
 * abpa == bpa.  Page entries are slot | brick max << 24.  When every brick
 * sits in its own slot the atlas is laid out like the world and views
 * sample it directly (the identity bit of brick_mode). */
int r3d_cuda_shard_build(r3d_cuda_ctx *ctx, uint32_t edge, const uint8_t *voxels, uint32_t abpa,
                         const uint32_t *slot_of);

/* brick_mode word of the loaded atlas: bpa | abpa << 8 | 0x10000 when the
 * layout is the identity (reference src/vk/vkbackend.c:4511-4517); 0 when
 * none is loaded. */
uint32_t r3d_cuda_shard_mode(const r3d_cuda_ctx *ctx);

/* Copy of the atlas's page table (bpa^3 words, may be NULL) and of atlas
 * mip `level` (0..3) or, for level == -1, the occupancy grid (out may be
 * NULL); dims receives the copied grid's size. */
int r3d_cuda_shard_read(r3d_cuda_ctx *ctx, int level, uint32_t *page, uint8_t *out,
                        uint32_t dims[3]);

/* --- forward raycast ------------------------------------------------------ */

/* Optional per-pixel outputs of a forward raycast, in the same memory kind
 * (device or host) as the image. */
typedef struct r3d_cuda_aux {
  uint32_t *steps;     /* out_w*out_h: march iterations of the ray */
  uint32_t *mip_index; /* out_w*out_h: step at which the MIP max last rose; defined for
                        MIP views (LOD-brick views of other modes leave 0) */
  unsigned long long *total_steps; /* one counter: += sum of steps */
  /* R3D_COUNTERS counters, += per frame: samples (= steps), composited TF
   * lookups, gradient-shaded samples, page-table walks.  Counting runs a
   * separate kernel build; NULL for the plain one. */
  unsigned long long *counters;
} r3d_cuda_aux;
#define R3D_COUNTERS 4

/* Raycasts nviews (1..64) views into the RGBA8 image rgba_out of
 * out_w x out_h pixels (row-major, 4 bytes per pixel).  Each view renders
 * its viewport rect at view_org, clipped to the image like render3d's
 * r3d_frame_views sanitize pass (src/vk/vkbackend.c:6871-6900); views whose
 * rect is empty are skipped.  A cube view needs r3d_cuda_upload_volume, a
 * brick view (brick_mode != 0) r3d_cuda_bricks_*.  Replaces the per-view
 * vkCmdDispatch of src/vk/vkbackend.c:7121-7173. */
int r3d_cuda_raycast_fwd(r3d_cuda_ctx *ctx, const r3d_frame_params *views, uint32_t nviews,
                         uint8_t *rgba_out, uint32_t out_w, uint32_t out_h,
                         const r3d_cuda_aux *aux, void *stream);

/* Dispatch rows [row0, row1) of one view into the device image (rows of
 * the halved grid for half-resolution views; row0 is rounded down to a
 * multiple of 8).  No counterpart in the reference: the headless render
 * layer draws a frame as row bands on two streams so that each band's
 * device-to-host copy overlaps the bands still rendering (r3d_read_frame).
 * Every pixel equals the one r3d_cuda_raycast_fwd renders.  Surface views
 * are rejected (R3D_E_UNSUPPORTED). */
int r3d_cuda_raycast_rows(r3d_cuda_ctx *ctx, const r3d_frame_params *view, uint8_t *rgba_out,
                          uint32_t out_w, uint32_t out_h, uint32_t row0, uint32_t row1,
                          void *stream);

/* Writes one RGBA8 colour into npix pixels of the device image img,
 * stream-ordered.  The render layer's clear of the offscreen regions that no
 * view covers when the pane layout changes (the vkCmdClearColorImage of
 * src/vk/vkbackend.c:7079-7098). */
int r3d_cuda_fill_rgba(r3d_cuda_ctx *ctx, uint8_t *img, size_t npix, const uint8_t rgba[4],
                       void *stream);

/* Forward raycast that allocates no device memory.  No counterpart in the
 * reference: it exists for callers that must not let the library allocate
 * while they render -- applications that give the renderer a fixed device-
 * memory budget at start-up, or real-time render threads for which an
 * allocation (which can synchronize the device) is a frame hitch.  Same
 * views, image rules and results as r3d_cuda_raycast_fwd with a device
 * rgba_out (required here), without the auxiliary outputs.  It runs a
 * persistent queue-draining kernel under the context's schedule
 * (r3d_cuda_set_schedule): whole 8x4 tiles when its persistent field is 2,
 * else lane refill with its tile shape, refill threshold and unroll; blocks
 * per SM as set.  Its per-call scratch (the view table and tile
 * counters) lives in a 32 KiB array of device memory inside the library,
 * which every GPU that loads the library holds until the process exits; at
 * most 64 views fit, larger calls fail with R3D_E_INVALID.  The views reach
 * that array through kernel launch parameters, so no host buffer is read
 * after the call returns.  The first call on a device looks up that array's
 * device address, so make it before any stream capture; the lookup is not
 * repeated, so the entry point must not be used across a cudaDeviceReset.
 * All calls share the array and each overwrites it: calls queued on one
 * stream run one after the other, but calls that overlap on the GPU
 * (different streams, or different contexts on one device) race and must be
 * serialized by the caller. */
int r3d_cuda_raycast_fwd_noalloc(r3d_cuda_ctx *ctx, const r3d_frame_params *views,
                                 uint32_t nviews, uint8_t *rgba_out, uint32_t out_w,
                                 uint32_t out_h, void *stream);

/* How forward launches are scheduled.  persistent = 0: one thread per ray
 * (one grid per view).  persistent = 1: resident warps drain a queue of
 * 32-ray tiles covering all views of the call, refilling lanes whose rays
 * have ended whenever at least refill_min lanes are idle; tile_shape 0/1/2
 * = 8x4 / 16x2 / 32x1 rays; unroll = march steps between refill checks
 * (1 or 2).  persistent = 2: resident warps drain a queue of whole 8x4
 * tiles covering all views of the call (one launch per sampling path and
 * mode), each marching its 32 rays to the end before taking the next tile
 * (refill_min, tile_shape and unroll unused).  persistent = 3 (automatic,
 * a context's default): whole tiles for a call with two or more views to
 * render, one thread per ray for one view (a batch resolves it once, from
 * its view count).  blocks_per_sm = resident
 * 128-thread blocks per SM of a persistent launch (0: the occupancy
 * limit).  shade_group (FULL mode, one-thread-per-ray launches):
 * n > 0 lets lanes park a sample that needs gradient shading until n lanes
 * of the warp (or all its live lanes) wait, and shades them together (1:
 * each sample where its ray meets it); 0 picks the sampling path's default,
 * 16 for the tiled slab, clipmap and virtual slab, whose gradient taps are
 * whole section lookups, and ungrouped shading for the cube and brick
 * paths.  Results are identical under every schedule. */
typedef struct r3d_cuda_schedule {
  uint32_t persistent;
  uint32_t refill_min;
  uint32_t tile_shape;
  uint32_t unroll;
  uint32_t blocks_per_sm;
  uint32_t shade_group;
  /* 1: one-thread-per-ray launches of LOD-brick views in FULL or MIP mode
   * without overlays, auxiliary outputs or row ranges run the TMA-staged
   * kernel instead: blocks of 8x8 Morton ray tiles that copy the slot box
   * their next samples fall in (32 x 17 x 17 u8 texels) into shared memory
   * with cp.async.bulk.tensor, and sample it from there.  0: off. */
  uint32_t staging;
} r3d_cuda_schedule;

int r3d_cuda_set_schedule(r3d_cuda_ctx *ctx, const r3d_cuda_schedule *sched);
int r3d_cuda_get_schedule(const r3d_cuda_ctx *ctx, r3d_cuda_schedule *sched);

/* CUDA-event time of the last r3d_cuda_raycast_fwd's kernels in ns
 * (synchronizes the events). */
int r3d_cuda_last_kernel_ns(r3d_cuda_ctx *ctx, uint64_t *ns);

/* --- batched views ---------------------------------------------------------- */

/* One view of a batch, with its own image: viewport[0] x viewport[1] RGBA8
 * pixels in device memory, rows of viewport[0] pixels (view_org must be 0).
 * No counterpart in the reference, which renders at most R3D_MAX_VIEWS panes
 * into one offscreen image (src/vk/vkbackend.c:7121-7173). */
typedef struct r3d_cuda_request {
  r3d_frame_params view;
  uint8_t *rgba;
} r3d_cuda_request;

/* Raycasts n (1..64) requests, each into its own device image, on stream
 * (NULL: the context's), under the context's schedule: one grid per request
 * (persistent 0), or one queue-draining launch per sampling path and mode
 * over all of them (persistent 1 or 2).  total_steps (nullable, device)
 * += march iterations.  The batched form of the per-view dispatch loop of
 * src/vk/vkbackend.c:7121-7173 for views of any size; nothing is kept
 * between calls (r3d_cuda_batch_* plans a batch once for replay). */
int r3d_cuda_raycast_batch(r3d_cuda_ctx *ctx, const r3d_cuda_request *reqs, uint32_t n,
                           unsigned long long *total_steps, void *stream);

typedef struct r3d_cuda_batch r3d_cuda_batch;

/* One request of a batch whose views sample several scenes: a view, its
 * image and the context whose scene it samples (volume or brick cache, TF,
 * quality, cutoff; NULL: the batch's context).  No counterpart in the
 * reference, which renders one scene per frame. */
typedef struct r3d_cuda_scene_request {
  r3d_frame_params view;
  uint8_t *rgba;
  r3d_cuda_ctx *scene;
} r3d_cuda_scene_request;

/* Plans a batch of 1..64 requests over the context's scene (all views use
 * it; requests may differ in size, projection and mode).  The plan keeps
 * its view table and tile counters in device memory, so its launch reads no
 * host data: it can be captured into a CUDA graph and replayed. */
int r3d_cuda_batch_create(r3d_cuda_ctx *ctx, const r3d_cuda_request *reqs, uint32_t n,
                          r3d_cuda_batch **out);
/* Plans a batch over up to 4 scenes (contexts on the batch context's
 * device).  Under the whole-tile schedule (persistent 2, the default when
 * there are several scenes) one launch per sampling path, mode and quality
 * drains the tiles of every view of every scene; the lane-refill schedule
 * needs a batch of one scene.  Launches read each scene as it is when they
 * are enqueued, and a captured graph keeps the scenes as they were at
 * capture: capture again after changing a scene. */
int r3d_cuda_batch_create_scenes(r3d_cuda_ctx *ctx, const r3d_cuda_scene_request *reqs,
                                 uint32_t n, r3d_cuda_batch **out);
void r3d_cuda_batch_destroy(r3d_cuda_batch *batch);
/* Schedule of the batch's launches (default: lane refill with 8x4 tiles
 * for one scene, whole tiles for several). */
int r3d_cuda_batch_set_schedule(r3d_cuda_batch *batch, const r3d_cuda_schedule *sched);
int r3d_cuda_batch_get_schedule(const r3d_cuda_batch *batch, r3d_cuda_schedule *sched);
/* Enqueues the batch on stream (NULL: the context's): one persistent
 * launch per sampling path and mode present (per path, mode and quality
 * under whole tiles; one in the common single-mode batch) draining the
 * tiles of all its views, or one grid per view under a grid schedule.
 * total_steps (nullable, device) += march iterations. */
int r3d_cuda_batch_launch(r3d_cuda_batch *batch, unsigned long long *total_steps, void *stream);
/* Captures r3d_cuda_batch_launch into a CUDA graph owned by the batch
 * (replacing an earlier one), and launches that graph. */
int r3d_cuda_batch_capture(r3d_cuda_batch *batch, unsigned long long *total_steps, void *stream);
int r3d_cuda_batch_replay(r3d_cuda_batch *batch, void *stream);
/* Autotuner: times every candidate schedule (one thread per ray with
 * grouped shading off / 4 / 8 / 16; lane refill with tile 8x4 / 16x2 /
 * 32x1, refill threshold 8 / 16 / 24, 1 or 2 steps between refills, for a
 * batch of one scene; whole 8x4 tiles) over `reps` launches each after a
 * warm-up, keeps the fastest as the batch's schedule and returns it with
 * its time per launch.  Results are identical under every candidate. */
int r3d_cuda_batch_autotune(r3d_cuda_batch *batch, uint32_t reps, r3d_cuda_schedule *best,
                            float *best_ms);

/* --- differentiable render and adjoint --------------------------------------- */

/* No counterpart in the reference: render3d's emission-absorption
 * compositing (the FLAT mode of src/shaders/raycast.slang:894-1017) made
 * differentiable over an FP32 density grid and an FP32 256x4 TF.  The render
 * is the cube path at level 0 with no empty-space skip; alpha is clamped to
 * [0, 1]; density scale = r3d_frame_params.density; termination at the
 * context's alpha cutoff.  All pointers are device memory. */
typedef struct r3d_cuda_diff_scene {
  const float *density; /* nx*ny*nz, x fastest */
  uint32_t nx, ny, nz;
  const float *lut; /* 256 x RGBA, any real values (alpha is clamped) */
} r3d_cuda_diff_scene;

typedef struct r3d_cuda_grads {
  float *density;       /* nx*ny*nz: dL/dvoxel (overwritten) */
  float *lut;           /* 256*4: dL/dLUT (overwritten) */
  float *density_scale; /* 1: dL/ddensity (overwritten) */
} r3d_cuda_grads;

/* Renders nviews (1..64) views (explicit viewports, cube path, optionally
 * orthographic) into rgb_out: per view, viewport[0]*viewport[1]*3 floats,
 * views back to back.  total_steps (nullable) += march iterations. */
int r3d_cuda_diff_forward(r3d_cuda_ctx *ctx, const r3d_cuda_diff_scene *scene,
                          const r3d_frame_params *views, uint32_t nviews, float *rgb_out,
                          unsigned long long *total_steps, void *stream);

/* The same render, recording a tape for the backward: per ray, the first 64
 * contributing samples (march position and the opacity accumulated before
 * them) and their count, in a context-owned buffer of 516 bytes per ray.
 * A later r3d_cuda_raycast_bwd with R3D_BWD_TAPE over the same views and
 * scene (same buffers, sizes and cutoff) reads it instead of marching the
 * rays forward again; the grid and LUT contents must not change in
 * between, and the backward must be ordered after this call.  Each call
 * replaces the tape. */
int r3d_cuda_diff_forward_tape(r3d_cuda_ctx *ctx, const r3d_cuda_diff_scene *scene,
                               const r3d_frame_params *views, uint32_t nviews, float *rgb_out,
                               unsigned long long *total_steps, void *stream);

#define R3D_BWD_DETERMINISTIC 1u /* fixed-point accumulation */
#define R3D_BWD_TAPE 2u          /* use the tape of r3d_cuda_diff_forward_tape */

/* Adjoint of r3d_cuda_diff_forward: given dL/drgb in rgb_out's layout,
 * writes dL/dvoxel, dL/dLUT and dL/ddensity.  The march is recomputed in
 * reverse from checkpoints kept every ckpt_k (32, 64 or 128) samples.
 * deterministic (flags): without R3D_BWD_DETERMINISTIC, FP32 atomic
 * accumulation (last bits depend on the execution order); with it,
 * fixed-point accumulation (2^-32 resolution, int64), bit-identical from
 * run to run, using a context-owned buffer of 8 * (nvox + 1025) bytes.
 * R3D_BWD_TAPE: rays whose contributions are all on the tape of the
 * matching r3d_cuda_diff_forward_tape skip the forward sweep (same
 * gradients, bit for bit in deterministic mode); R3D_E_STATE when no such
 * tape exists. */
int r3d_cuda_raycast_bwd(r3d_cuda_ctx *ctx, const r3d_cuda_diff_scene *scene,
                         const r3d_frame_params *views, uint32_t nviews, const float *dl_drgb,
                         const r3d_cuda_grads *out, uint32_t ckpt_k, int deterministic,
                         void *stream);

/* --- diagnostics ----------------------------------------------------------- */

/* Slot trace of counting launches (those given aux->counters) of the LOD
 * brick path: bit s of the device bitmap `bits` (nslots bits, zeroed by the
 * caller) is set when a sample reads slot s's voxels; NULL turns it off.
 * The benchmark's compulsory-bytes figure (unique bricks a frame reads);
 * plain launches never test it.  No counterpart in the reference. */
int r3d_cuda_set_slot_trace(r3d_cuda_ctx *ctx, uint32_t *bits);

/* Read bandwidth of an L2-resident buffer of `bytes` (>= 1 MiB; pick it
 * well inside the 126 MB L2) swept `passes` times through L2 by every SM,
 * in GB/s from CUDA events: the L2 peak the raycast's algorithmic bytes are
 * compared with (its footprint is reused through L1 and L2).  Allocates
 * and frees its buffer; no counterpart in the reference. */
int r3d_cuda_l2_read_probe(r3d_cuda_ctx *ctx, size_t bytes, uint32_t passes, float *gbs);

/* Evaluates the raycast's log2, exp2, pow(x, y) and x^24 on the device for n
 * inputs (host pointers); out receives 4 floats per input in that order.
 * Used to check the device build of r3d_fmath.h bit for bit. */
int r3d_cuda_fmath_eval(r3d_cuda_ctx *ctx, const float *x, const float *y, float *out,
                        uint32_t n);

/* The byte counts the LOD-brick kernels' fetch elision compares a block
 * maximum m (and a fetched sample's bytes) with, for view p in a scene whose
 * TF is clear below tf_zero_t: out[0] = n_void (m < n_void: the sample is
 * below the threshold or the skip gate), out[1] = n_dec (m < n_dec: the
 * view's mode decides nothing on the sample).  Host code, the same function
 * the launches use; no device work.  Used to check the counts against all
 * 256 byte values; no counterpart in the reference. */
void r3d_cuda_elide_counts(const r3d_frame_params *p, float tf_zero_t, uint32_t out[2]);

#ifdef __cplusplus
}
#endif

#endif /* R3D_CUDA_H */
