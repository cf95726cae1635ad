/*
 * nefct_b200 -- C ABI of the B200 (sm_100a) projector library.
 *
 * Replaces the TensorFlow custom ops of bill52547/CT-NEF (package `nefct`)
 * on the projector hot path: the cone-beam ray-driven ("Siddon") forward
 * projector, its exact transpose, the reference's own backprojection, the
 * LOR projector pair, FDK filtering and voxel-driven backprojection, and the
 * trilinear deformation warp.
 *
 * Conventions (all entry points):
 *  - plain pointers and sizes; device pointers unless stated "host";
 *  - the caller owns every buffer; temporaries live in a caller-provided
 *    workspace whose size a *_workspace_bytes() query returns;
 *  - work is enqueued on `stream` (a cudaStream_t, NULL = legacy default
 *    stream) with no host synchronisation and no host round trip;
 *  - outputs are fully written (zeroed first where the op accumulates);
 *  - every call returns an nefct_status; nefct_last_error() gives the
 *    calling thread's message for the last failure.  No call aborts or traps;
 *  - volumes are float [nz][ny][nx] (x fastest), sinograms [nv][nb][na]
 *    (detector column a fastest), the reference's device layouts.
 */
#ifndef NEFCT_B200_H
#define NEFCT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t nefct_status;
#define NEFCT_OK              0
#define NEFCT_ERR_INVALID     1  /* bad argument, shape or geometry */
#define NEFCT_ERR_CUDA        2  /* a CUDA runtime call or launch failed */
#define NEFCT_ERR_WORKSPACE   3  /* workspace missing or too small */
#define NEFCT_ERR_TIMEOUT     4  /* a bounded device-side wait gave up */
#define NEFCT_ERR_UNSUPPORTED 5  /* valid request this build does not implement */

const char *nefct_version(void);
const char *nefct_status_string(nefct_status st);
const char *nefct_last_error(void);

/* Process-wide launch tuning used by the autotuner (nefct_b200/autotune.py).
 * No counterpart in the reference (its launch shapes are constants,
 * siddon.cu.cc:8-10).  Every value runs the same per-ray arithmetic in the
 * same order; the transpose sums with atomics, whose order is not fixed
 * under any setting.
 *   NEFCT_TUNE_CB_ROWS   detector rows per CTA of the cone-beam Siddon
 *                        kernels (1, 2, 4, 8; 32 columns per row); default 8
 *   NEFCT_TUNE_CB_ORDER  0: row bands outermost (default; keeps the volume
 *                        slab of the rows in flight in L2), 1: views outermost
 *   NEFCT_TUNE_CB_WALK   bit 0 forward, bit 1 transpose: column warps (FP32
 *                        slab walk with a workspace) -- each warp walks 32
 *                        rows of one detector column, which share their
 *                        transverse walk, over a z-fastest copy of the volume,
 *                        and NEFCT_TUNE_CB_ROWS counts columns per CTA; a
 *                        clear bit: one thread per ray.  Default 3 */
#define NEFCT_TUNE_CB_ROWS  0
#define NEFCT_TUNE_CB_ORDER 1
#define NEFCT_TUNE_CB_WALK  2
#define NEFCT_TUNE_COUNT    3
nefct_status nefct_tune_set(int32_t key, int32_t value);
int32_t nefct_tune_get(int32_t key);

/* Voxel grid: nx*ny*nz voxels of a box of extent (sx, sy, sz) centred on
 * (cx, cy, cz).  Same meaning as the reference ops' grid/center/size inputs
 * (nefct/cc/siddon_3d/siddon.cc:13-15; cpp/siddon/siddon_gpu.cc:14-16),
 * passed by value on the host instead of as device tensors that the
 * reference reads back with blocking copies (siddon.cu.cc:403-405). */
typedef struct nefct_grid {
    int32_t nx, ny, nz;
    float cx, cy, cz;
    float sx, sy, sz;
} nefct_grid;

#define NEFCT_DET_FLAT 0
#define NEFCT_DET_CYL  1

/* Circular cone-beam geometry, reference kernel convention
 * (nefct/cc/siddon_3d/siddon.cu.cc:341-353): at view angle phi the source
 * sits at (-src_iso cos phi, -src_iso sin phi, z_off) and detector cell
 * (ia, ib) at the rotation by phi of
 *   flat: (src_det - src_iso, a, b)
 *   cyl:  (src_det cos a - src_iso, src_det sin a, b)
 * with a = (ia + a_shift) da - na da / 2,  b = (ib + b_shift) db - nb db / 2
 * (+ z_off).  src_iso is the kernel's `SID`, src_det its `SAD` (the python
 * geometry names them the other way round, quirk Q12).  a_shift/b_shift are
 * the kernel's `ai`/`bi` (0.5 puts the cell centres symmetric about 0). */
typedef struct nefct_cb_geom {
    nefct_grid grid;
    int32_t nv;                /* views */
    const float *angles;       /* host, nv radians */
    const float *z_offsets;    /* host, nv, or NULL for none */
    float src_iso;             /* source -> rotation axis */
    float src_det;             /* source -> detector */
    int32_t na; float da; float a_shift;
    int32_t nb; float db; float b_shift;
    int32_t det_kind;          /* NEFCT_DET_FLAT / NEFCT_DET_CYL */
} nefct_cb_geom;

/* Walk switches.  With flags == 0 the forward reproduces siddon_3d's
 * project_device (siddon.cu.cc:12-321): x drives when |xd| >= |yd| and each
 * weight carries dx/L^2 (L = source-detector length in voxel units). */
#define NEFCT_TIE_GT        0x01u /* x drives only when |xd| > |yd| (backproject_device :480, cpp/siddon :42) */
#define NEFCT_SKIP_SHORT    0x02u /* skip rays with hypot(xd, yd) < 10 voxels (Q4: :472, cpp :33,:358) */
#define NEFCT_NO_INV_L2     0x04u /* weights without 1/L^2: plain line integrals (backproject_device :526) */
#define NEFCT_Q5            0x08u /* extra 1/L on y-driven three-voxel middle weights (cpp/siddon :292,:313);
                                     LOR calls only: the cone-beam calls refuse it (NEFCT_ERR_UNSUPPORTED) */
#define NEFCT_Q8_INDEX      0x10u /* cylindrical backprojection reads the sinogram at ia + iv*na + ib*na*nb (:830) */
#define NEFCT_NO_TRANSPOSE  0x20u /* x-driven rays read the x-fastest volume directly: no workspace, slower */
#define NEFCT_EXACT         0x80u /* classical exact Siddon instead of the reference's slab split: FP64 per-ray
                                     entry/exit and first crossings, FP32 stepping; exact transpose with the
                                     same flags.  No counterpart in the reference (its split is quirk Q1) */
#define NEFCT_DETERMINISTIC 0x40u /* backward: bitwise reproducible sums (64-bit fixed point, see nefct_cb_backward);
                                     the forward is deterministic anyway and ignores it */

/* presets */
#define NEFCT_REF_FORWARD        0u                                              /* siddon_3d project_device */
#define NEFCT_REF_BACKPROJECT    (NEFCT_TIE_GT | NEFCT_SKIP_SHORT | NEFCT_NO_INV_L2) /* siddon_3d backproject_device */
#define NEFCT_LINE_INTEGRAL      NEFCT_NO_INV_L2
#define NEFCT_LOR_REF_FORWARD    (NEFCT_TIE_GT | NEFCT_SKIP_SHORT | NEFCT_Q5)    /* cpp/siddon project_device */
#define NEFCT_LOR_REF_BACKPROJECT (NEFCT_TIE_GT | NEFCT_SKIP_SHORT | NEFCT_NO_INV_L2)

/* Bytes of workspace nefct_cb_forward / nefct_cb_backward need for this
 * geometry and flags (a y-fastest copy of the volume; 0 with
 * NEFCT_NO_TRANSPOSE; with NEFCT_DETERMINISTIC the backward's two 64-bit
 * accumulators).  FP64 calls need twice the non-deterministic size.
 * Host-only, no CUDA call. */
size_t nefct_cb_workspace_bytes(const nefct_cb_geom *g, uint32_t flags);

/* Cone-beam forward projection vol -> sino.  Replaces ProjectFlat /
 * ProjectCyli (nefct/cc/siddon_3d/siddon.cc:11-42, 114-224) and their host
 * entry points project_flat / project_cyli (siddon.cu.cc:392-448).  The
 * reference op passes da where db belongs (Q7, siddon.cc:155,211); callers
 * that want that pass db = da. */
nefct_status nefct_cb_forward(const nefct_cb_geom *g, const float *vol, float *sino, uint32_t flags,
                              void *workspace, size_t workspace_bytes, void *stream);

/* Cone-beam backprojection sino -> vol (vol is overwritten).  With the same
 * flags as a forward call it is that forward's exact transpose; with
 * NEFCT_REF_BACKPROJECT it reproduces BackProjectFlat / BackProjectCyli
 * (siddon.cc:44-80, 226-348; siddon.cu.cc:450-890).
 * Sums are float atomics (order not fixed) unless NEFCT_DETERMINISTIC: then
 * every contribution is scaled by a power of two chosen from max|sino| and a
 * bound on the weights (so no sum can exceed 2^61), rounded to a 64-bit
 * integer and reduced with integer atomics, and the sums are converted once
 * -- bitwise identical across runs, with rounding far below float sums.
 * Float32 only; NaN/Inf in sino are not supported in that mode. */
nefct_status nefct_cb_backward(const nefct_cb_geom *g, const float *sino, float *vol, uint32_t flags,
                               void *workspace, size_t workspace_bytes, void *stream);

/* Forward projection for callers that cannot allocate device memory: the
 * same kernels and bit-identical result as nefct_cb_forward (same flags,
 * same launch tuning), but its scratch (the volume copy the walk gathers
 * from) lives in a fixed 32 MiB array inside the library instead of a
 * caller workspace.  No counterpart in the reference.  It is for callers
 * that may not call cudaMalloc -- a service that reserves all GPU memory at
 * start-up, a host framework that owns the memory pool, a binding that only
 * receives device pointers.  It allocates nothing (no cudaMalloc/cudaFree,
 * no allocating library call) and rejects grids of more than 8 Mi voxels
 * (8388608) with NEFCT_ERR_INVALID.  Every GPU that loads the library holds
 * the 32 MiB until the process exits.  The first call in each CUDA context
 * (each device's primary context, a caller's own driver-API context, the new
 * primary context after cudaDeviceReset) looks up the array's device address
 * there (cudaGetSymbolAddress) and caches it by the context's ID; make that
 * first call before any stream capture.  All calls share
 * the one array: calls that overlap on the GPU (other streams, other host
 * threads) race on it and must be serialised by the caller.  Nothing in it
 * needs clearing: each call overwrites every element it reads. */
nefct_status nefct_cb_forward_noalloc(const nefct_cb_geom *g, const float *vol, float *sino, uint32_t flags,
                                      void *stream);

/* FP64 builds of the same two operators (finite-difference and adjoint
 * checks); geometry fields stay float. */
nefct_status nefct_cb_forward_f64(const nefct_cb_geom *g, const double *vol, double *sino, uint32_t flags,
                                  void *workspace, size_t workspace_bytes, void *stream);
nefct_status nefct_cb_backward_f64(const nefct_cb_geom *g, const double *sino, double *vol, uint32_t flags,
                                   void *workspace, size_t workspace_bytes, void *stream);

/* Number of ray-voxel contributions (intersections) the forward with these
 * flags makes, added into *count (device uint64).  No counterpart in the
 * reference; it defines the throughput metric. */
nefct_status nefct_cb_count_intersections(const nefct_cb_geom *g, uint32_t flags,
                                          unsigned long long *count, void *stream);

/* Batched cone-beam problems of uneven sizes: forward of every problem in
 * one persistent launch, transposes of every problem in another (or one
 * launch per problem, nefct_cb_batch_set_strategy).  No
 * counterpart in the reference (which projects one problem per op call,
 * e.g. project_t.py:153-160 even one view per call).  Work is tiled (32
 * detector columns x NEFCT_TUNE_CB_ROWS rows of one view), ordered longest
 * rays first and handed out through an atomic ticket; nothing waits, so the
 * launch cannot hang.  Per problem: vol -> sino (forward), grad -> back
 * (transpose, exact for the same flags). */
typedef struct nefct_cb_problem {
    nefct_cb_geom geom;        /* host geometry (angles/z_offsets read at plan time) */
    const float *vol;          /* device [nz][ny][nx], forward input */
    float *sino;               /* device [nv][nb][na], forward output */
    const float *grad;         /* device [nv][nb][na], transpose input (may be sino) */
    float *back;               /* device [nz][ny][nx], transpose output (overwritten) */
} nefct_cb_problem;
typedef struct nefct_cb_batch nefct_cb_batch;
/* Host-only: validates the problems (at most 96 per plan), builds the tile
 * order and returns the device workspace size (view tables and one volume
 * copy per problem; the problem descriptors travel as kernel parameters). */
nefct_status nefct_cb_batch_plan(const nefct_cb_problem *problems, int32_t n, uint32_t flags,
                                 nefct_cb_batch **plan, size_t *workspace_bytes);
/* Uploads the plan's tables into the caller's workspace (256-byte aligned)
 * and waits for that copy.  Call once, before forward/backward and before
 * capturing them in a CUDA graph; the buffers named in the problems must stay
 * valid while the plan is used. */
nefct_status nefct_cb_batch_bind(nefct_cb_batch *plan, void *workspace, size_t workspace_bytes, void *stream);
nefct_status nefct_cb_batch_forward(nefct_cb_batch *plan, void *stream);
nefct_status nefct_cb_batch_backward(nefct_cb_batch *plan, void *stream);
int64_t nefct_cb_batch_tiles(const nefct_cb_batch *plan);   /* work tiles per launch */
/* How forward/backward run the problems: one persistent launch over all
 * tiles (NEFCT_BATCH_PERSISTENT), or the single-problem kernels once per
 * problem (NEFCT_BATCH_PER_PROBLEM, the default: the persistent kernel holds
 * its per-problem constants in registers and runs at lower occupancy, which
 * only pays when problems are too small to fill the GPU). */
#define NEFCT_BATCH_PERSISTENT  0
#define NEFCT_BATCH_PER_PROBLEM 1
nefct_status nefct_cb_batch_set_strategy(nefct_cb_batch *plan, int32_t strategy);
/* Host-only: points the plan's problems at other buffers of the same shapes
 * (arrays of n pointers in the caller's problem order; a NULL array or a
 * NULL entry keeps the current buffer), so a caller can run the batch on
 * tensors it already holds instead of copying them into the bound ones.
 * Takes effect from the next forward / backward (their launches copy the
 * pointers when they are issued); a CUDA graph keeps the pointers it was
 * captured with.  The buffers must stay valid while the plan uses them.  No
 * counterpart in the reference. */
nefct_status nefct_cb_batch_set_buffers(nefct_cb_batch *plan, const float *const *vols, float *const *sinos,
                                        const float *const *grads, float *const *backs);
void nefct_cb_batch_destroy(nefct_cb_batch *plan);

/* LOR projector pair.  lors is [6][n] (rows x1 y1 z1 x2 y2 z2, each n
 * long), as the reference op slices it (cpp/siddon/siddon_gpu.cc:74-86).
 * Replace Projection / Backprojection (siddon_gpu.cc:11-35) and their host
 * entry points projection / backprojection (siddon_gpu.cu.cc:700-747).
 * nefct_lor_forward writes every out[i] (0 for rays the reference skips
 * without writing, Q4); nefct_lor_backward overwrites vol (the reference op
 * accumulates into an unzeroed buffer, Q6).  n = 0 is valid: the forward
 * writes nothing (its buffers may be NULL), the backward zeroes vol. */
nefct_status nefct_lor_forward(const nefct_grid *grid, const float *lors, int64_t n, const float *vol,
                               float *out, uint32_t flags, void *stream);
nefct_status nefct_lor_backward(const nefct_grid *grid, const float *lors, int64_t n, const float *vals,
                                float *vol, uint32_t flags, void *stream);
/* Walk order for large unsorted line lists (no counterpart in the reference,
 * whose kernels walk lines in list order).  nefct_lor_order_keys writes a
 * 31-bit key per line (driving axis, in-plane direction, distance from the
 * grid centre, z, z slope); a permutation that sorts the keys (any stable or
 * unstable sort) makes a warp's lines nearly parallel neighbours.  The
 * *_ordered walks visit lines in that order and write each result at the
 * line's own index: the same outputs as the unordered calls (the backward's
 * atomic summation order differs).  Fewer than 2^31 lines. */
nefct_status nefct_lor_order_keys(const nefct_grid *grid, const float *lors, int64_t n, int32_t *keys, void *stream);
nefct_status nefct_lor_forward_ordered(const nefct_grid *grid, const float *lors, int64_t n, const int32_t *order,
                                       const float *vol, float *out, uint32_t flags, void *stream);
nefct_status nefct_lor_backward_ordered(const nefct_grid *grid, const float *lors, int64_t n, const int32_t *order,
                                        const float *vals, float *vol, uint32_t flags, void *stream);

/* FDK.  Filter windows of mat_codes/filtering.m:63-88. */
#define NEFCT_WIN_RAM_LAK     0
#define NEFCT_WIN_SHEPP_LOGAN 1
#define NEFCT_WIN_COSINE      2
#define NEFCT_WIN_HAMMING     3
#define NEFCT_WIN_HANN        4

/* Cosine weight, optional Parker short-scan weight and ramp filtering of a
 * flat-detector sinogram [nv][nb][na] -> out (same shape; may not alias).
 * Follows mat_codes/filtering.m:5-48 and ParkerWeight.m:5-27 with DSD =
 * src_det, DSO = src_iso, du = da, dv = db, u along detector columns.
 * parker: 0 off, +1 / -1 on with ParkerWeight's `dir` = +1 / -1 (the view
 * step is taken from angles[1] - angles[0]).  Like the MATLAB code, each
 * row is zero-padded to L = max(64, 2^nextpow2(2 na)), transformed,
 * multiplied by the windowed filter response and transformed back (FP32
 * FFTs on the device, two rows per complex transform).  na <= 2048. */
nefct_status nefct_fdk_filter(const nefct_cb_geom *g, const float *sino, float *out, int32_t window,
                              int32_t parker, void *stream);

/* Voxel-driven bilinear backprojection filtered sino -> vol (overwritten):
 * the geometry and index semantics of nefct/cc/pixel_3d/pixel.cu.cc:12-146
 * (Q9-Q11; the grid is given by its centre here, the reference takes its
 * low corner, Q10) times the FDK weight (src_iso / (src_iso + x'))^2 of
 * mat_codes/backprojection.m:12.  NEFCT_FDK_NO_WEIGHT drops the weight,
 * reproducing BackProjectFlat/BackProjectCyli of pixel_3d/pixel.cc:11-47.
 * A voxel whose detector column or row lies within a few thousandths of a
 * cell of the flat detector's first or last (where Q11 keeps or drops it on
 * a rounding) is
 * decided with the reference's own operations, so the same voxels are kept;
 * elsewhere the weights differ from the reference's by a few ulp. */
#define NEFCT_FDK_NO_WEIGHT 0x100u
nefct_status nefct_fdk_backproject(const nefct_cb_geom *g, const float *filtered, float *vol, uint32_t flags,
                                   void *stream);
/* The same backprojection with a caller workspace (nefct_fdk_workspace_bytes,
 * 16-byte aligned; NULL gives nefct_fdk_backproject): each chunk of views
 * is first repacked into tap quads (the four bilinear taps of every detector
 * cell side by side) so a voxel reads its taps with one 16-byte load.  Same
 * arithmetic, bit-identical result.  The workspace holds one chunk: up to
 * 128 views, about 400 MB at most (16 bytes per detector cell and view).
 * No counterpart in the reference. */
size_t nefct_fdk_workspace_bytes(const nefct_cb_geom *g);
nefct_status nefct_fdk_backproject_ws(const nefct_cb_geom *g, const float *filtered, float *vol, uint32_t flags,
                                      void *ws, size_t ws_bytes, void *stream);

/* Trilinear warp of cpp/deform (DeformKernel deform.cu.cc:13-46, op Deform
 * deform.cc:12-22): out[i] = trilinear(img, i + m[i]), displacements in
 * voxels, 0 where the reference returns early (base index <= 0 or the
 * upper tap out of range, Q13).  All arrays [nz][ny][nx]. */
nefct_status nefct_warp_forward(const float *img, const float *mx, const float *my, const float *mz,
                                int32_t nx, int32_t ny, int32_t nz, float *out, void *stream);
/* Adjoint of nefct_warp_forward with respect to img: gimg (overwritten) =
 * W^T gout.  No counterpart in the reference (it has no gradients). */
nefct_status nefct_warp_adjoint(const float *gout, const float *mx, const float *my, const float *mz,
                                int32_t nx, int32_t ny, int32_t nz, float *gimg, void *stream);
/* Gradient of <gout, warp(img, m)> with respect to the displacement field:
 * gm* (overwritten).  No counterpart in the reference. */
nefct_status nefct_warp_grad_dvf(const float *img, const float *mx, const float *my, const float *mz,
                                 const float *gout, int32_t nx, int32_t ny, int32_t nz,
                                 float *gmx, float *gmy, float *gmz, void *stream);
/* Inverse of a displacement field by `iters` fixed-point passes (the
 * reference uses 30): replaces DeformInvert (nefct/cc/deform/deform_tex.cc:24,
 * deform_tex.cu.cc:78-99).  Fields are sampled trilinearly with
 * clamp-to-edge addressing in FP32 (the reference samples a linear-filtered
 * texture, whose weights carry 8 fractional bits). */
nefct_status nefct_warp_invert(const float *mx, const float *my, const float *mz, int32_t nx, int32_t ny, int32_t nz,
                               int32_t iters, float *ix, float *iy, float *iz, void *stream);
nefct_status nefct_warp_forward_f64(const double *img, const double *mx, const double *my, const double *mz,
                                    int32_t nx, int32_t ny, int32_t nz, double *out, void *stream);
nefct_status nefct_warp_adjoint_f64(const double *gout, const double *mx, const double *my, const double *mz,
                                    int32_t nx, int32_t ny, int32_t nz, double *gimg, void *stream);
nefct_status nefct_warp_grad_dvf_f64(const double *img, const double *mx, const double *my, const double *mz,
                                     const double *gout, int32_t nx, int32_t ny, int32_t nz,
                                     double *gmx, double *gmy, double *gmz, void *stream);


/* ---- distance-driven FDK backprojection ----
 * Replaces back_project_flat_fdk_gpu / back_project_cyli_fdk_gpu
 * (nefct/cc/distance_3d/dist_3d_back_fdk.cu.cc:257-298, kernel :17-255), the
 * detector-driven part of the dist_3d_mod library that the reference's
 * Project3D/BackProject3D load.  Geometry in voxel units with the grid centred
 * on the rotation axis, as there: source at distance src_iso from the axis
 * (the reference's SAD), detector at src_det from the source (its SID); bin
 * (ia, ib) sits at a = (ia + 0.5) * da + a_offset - na * da / 2 (radians for
 * det_kind NEFCT_DET_CYL), b likewise; per-view z offsets shift source and
 * detector (NULL = 0).  Each bin spreads value * (footprint overlap in the
 * transverse and z axes) * |p2 - p1| / |driving component| * the FDK weight
 * src_iso^2 / (src_iso + x cos + y sin)^2 over the voxels of every slab of
 * its driving axis.  vol ([nz][ny][nx]) is overwritten (the reference adds
 * into the caller's buffer).  Workspace: nefct_dd_workspace_bytes (one
 * volume, a z-fastest accumulator). */
typedef struct nefct_dd_geom {
    int32_t nx, ny, nz, nv;
    const float *angles;       /* host, nv */
    const float *z_offsets;    /* host, nv, or NULL */
    float src_iso, src_det;
    int32_t na;
    float da, a_offset;
    int32_t nb;
    float db, b_offset;
    int32_t det_kind;
} nefct_dd_geom;
size_t nefct_dd_workspace_bytes(const nefct_dd_geom *g);
nefct_status nefct_dd_backproject(const nefct_dd_geom *g, const float *proj, float *vol, void *ws, size_t ws_bytes,
                                  void *stream);

/* ---- distance-driven projector pair ----
 * The forward half of the dist_3d_mod family that the reference's
 * Project3D loads (project_flat_three / project_cyli_three,
 * nefct/functions/project.py:11-16, :95); its source is not in the
 * reference, so the forward is defined as the exact transpose of the
 * backprojection above: each bin (ia, ib, iv) sums voxel * weight over the
 * voxels and weights its backprojection would spread value into (same
 * geometry struct, same footprints).  flags: 0 keeps the FDK weight
 * src_iso^2 / (src_iso + x cos + y sin)^2 in the weight (the transpose of
 * nefct_dd_backproject); NEFCT_FDK_NO_WEIGHT drops it (footprint-weighted
 * line integrals, overlap fractions times |p2 - p1| / |driving component|).
 * nefct_dd_backward with the same flags is the transpose of nefct_dd_forward
 * (with flags 0 it is nefct_dd_backproject).  proj is [nv][nb][na], vol
 * [nz][ny][nx]; outputs are overwritten.  Workspace:
 * nefct_dd_workspace_bytes (a z-fastest volume copy / accumulator).  The
 * FP64 builds (adjoint and finite-difference checks) need no workspace. */
nefct_status nefct_dd_forward(const nefct_dd_geom *g, const float *vol, float *proj, uint32_t flags, void *ws,
                              size_t ws_bytes, void *stream);
nefct_status nefct_dd_backward(const nefct_dd_geom *g, const float *proj, float *vol, uint32_t flags, void *ws,
                               size_t ws_bytes, void *stream);
nefct_status nefct_dd_forward_f64(const nefct_dd_geom *g, const double *vol, double *proj, uint32_t flags,
                                  void *stream);
nefct_status nefct_dd_backward_f64(const nefct_dd_geom *g, const double *proj, double *vol, uint32_t flags,
                                   void *stream);

/* ---- ceiling probes (measurement; no counterpart in the reference) ----
 * The cone-beam walks read and reduce mostly L2-resident data, so their
 * rooflines are set by the L2 read bandwidth and the L2 reduction rate of
 * the GPU at hand.  nefct_probe_l2_read streams n floats of buf (16-byte
 * aligned, n a multiple of 4; size it to stay in L2) `reps` times with
 * 16-byte L2-only loads; nefct_probe_l2_red adds 1.0f to each of n floats of
 * buf `reps` times with coalesced red.global.add.f32.  Both run
 * blocks_per_sm x (SM count) CTAs of 256 threads; sink takes
 * nefct_probe_sink_floats(blocks_per_sm) floats.  Time them with events on
 * `stream`. */
size_t nefct_probe_sink_floats(int32_t blocks_per_sm);
nefct_status nefct_probe_l2_read(const float *buf, size_t n, int32_t reps, int32_t blocks_per_sm, float *sink,
                                 void *stream);
nefct_status nefct_probe_l2_red(float *buf, size_t n, int32_t reps, int32_t blocks_per_sm, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* NEFCT_B200_H */
