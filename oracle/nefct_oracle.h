/*
 * TEST INFRASTRUCTURE (oracle).  CPU restatement of the reference's
 * projector hot path (bill52547/CT-NEF), used only by tests/, the smoke
 * check and the benchmark's CPU-baseline leg.  Never part of the product.
 *
 * Parity pinning: tests/test_oracle.py compares every function here with the
 * reference's own device routines compiled as host code (oracle/_ref, built
 * by oracle/Makefile from the reference sources) on seeded inputs, and with
 * the committed golden fixtures under tests/golden/.
 */
#ifndef NEFCT_ORACLE_H
#define NEFCT_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nx, ny, nz;      /* grid; memory order x fastest: ix + iy*nx + iz*nx*ny */
    float cx, cy, cz;    /* volume centre */
    float sx, sy, sz;    /* volume extent */
} or_grid;

/* walk flags */
#define OR_TIE_GE       1u  /* x drives when |xd| >= |yd| (siddon_3d forward); else when > */
#define OR_SKIP_SHORT   2u  /* Q4: skip rays with hypot(xd, yd) < 10 voxels */
#define OR_INV_L2       4u  /* Q2: weights carry 1/L^2 (forward) */
#define OR_Q5_TRIPLE_L  8u  /* Q5: cpp/siddon forward, extra 1/L on y-driven middle weights */

/* reference-semantics presets */
#define OR_CB_FWD   (OR_TIE_GE | OR_INV_L2)              /* siddon_3d project_device */
#define OR_CB_BP    (OR_SKIP_SHORT)                      /* siddon_3d backproject_device */
#define OR_LOR_FWD  (OR_SKIP_SHORT | OR_INV_L2 | OR_Q5_TRIPLE_L)
#define OR_LOR_BP   (OR_SKIP_SHORT)

long long or_cb_forward_f32(const or_grid *g, const float *img, const float *cs, const float *sn,
                            const float *off, int nv, float src_iso, float src_det,
                            int na, float da, float ai, int nb, float db, float bi,
                            int cyl, unsigned flags, float *sino);
long long or_cb_forward_f64(const or_grid *g, const double *img, const double *cs, const double *sn,
                            const double *off, int nv, double src_iso, double src_det,
                            int na, double da, double ai, int nb, double db, double bi,
                            int cyl, unsigned flags, double *sino);
void or_cb_backward_f32(const or_grid *g, const float *sino, const float *cs, const float *sn,
                        const float *off, int nv, float src_iso, float src_det,
                        int na, float da, float ai, int nb, float db, float bi,
                        int cyl, unsigned flags, int q8, float *img);
void or_cb_backward_f64(const or_grid *g, const double *sino, const double *cs, const double *sn,
                        const double *off, int nv, double src_iso, double src_det,
                        int na, double da, double ai, int nb, double db, double bi,
                        int cyl, unsigned flags, int q8, double *img);
long long or_lor_forward_f32(const or_grid *g, const float *img, const float *lors, long long n,
                             unsigned flags, float *out);
void or_lor_backward_f32(const or_grid *g, const float *vals, const float *lors, long long n,
                         unsigned flags, float *img);

/* cos/sin table of the view angles: use_cosf=1 evaluates cosf/sinf in float
 * as the reference's kernels do; 0 rounds the double-precision values. */
void or_trig_f32(const float *angles, int nv, int use_cosf, float *cs, float *sn);

/* Exact FP64 radiological path (classical Siddon/Jacobs plane crossing) of
 * every cone-beam ray; inv_l2 != 0 divides by L^2 in x-pitch voxel units as
 * the reference forward does, so the result is comparable with it. */
void or_cb_exact_f64(const or_grid *g, const double *img, const double *angles, const double *off,
                     int nv, double src_iso, double src_det, int na, double da, double ai,
                     int nb, double db, double bi, int cyl, int inv_l2, double *sino);

/* Voxel-driven bilinear backprojection of nefct/cc/pixel_3d/pixel.cu.cc:12-146.
 * corner[3] is the reference's `center` argument (the grid's low corner, Q10).
 * fdk != 0 multiplies each view's tap sum by (src_iso / (src_iso + xc0))^2,
 * the weight of mat_codes/backprojection.m:12. */
void or_pixel_backproject_f32(const float *sino, const float *angles, int nv,
                              int nx, int ny, int nz, const float *corner, const float *size,
                              float src_iso, float src_det, int na, float da, float ai,
                              int nb, float db, float bi, int cyl, int fdk, float *img);
void or_pixel_backproject_f64(const double *sino, const double *angles, int nv,
                              int nx, int ny, int nz, const double *corner, const double *size,
                              double src_iso, double src_det, int na, double da, double ai,
                              int nb, double db, double bi, int cyl, int fdk, double *img);

/* Trilinear warp of cpp/deform/deform.cu.cc:13-46; voxels the reference
 * leaves unwritten (Q13) are written as 0. */
void or_deform_f32(const float *img, const float *mx, const float *my, const float *mz,
                   int nx, int ny, int nz, float *out);
void or_deform_f64(const double *img, const double *mx, const double *my, const double *mz,
                   int nx, int ny, int nz, double *out);

/* Displacement-field inversion of nefct/cc/deform/deform_tex.cu.cc:78-99
 * (FP32 trilinear, clamp-to-edge, Gauss-Seidel fixed point). */
void or_warp_invert_f32(const float *mx, const float *my, const float *mz, int nx, int ny, int nz, int iters,
                        float *ix, float *iy, float *iz);

/* Distance-driven FDK-weighted backprojection of
 * nefct/cc/distance_3d/dist_3d_back_fdk.cu.cc:17-298 (voxel units, grid
 * centred on the axis, SID = source-detector, SAD = source-axis); cs/sn are
 * the per-view cos/sin (or_trig_f32), off the per-view z offsets. */
void or_dd_backproject_f32(const float *proj, const float *cs, const float *sn, const float *off, int nv,
                           float SID, float SAD, int nx, int ny, int nz, int na, float da, float ai, int nb,
                           float db, float bi, int cyl, int use_cosf, float *img);

#ifdef __cplusplus
}
#endif
#endif
