/*
 * ctlab_b200.h — C ABI of the B200 Siddon projector (libctlab_b200.so).
 *
 * Every entry point takes raw device pointers, 64-bit sizes and a CUDA stream
 * (passed as void*, i.e. a cudaStream_t; NULL means the legacy default
 * stream), launches asynchronously on that stream and returns a status code.
 * Nothing is allocated: the caller owns every buffer, outputs included.
 * Errors never cross the ABI as exceptions; ctlab_last_error() returns the
 * message of the calling thread's most recent failure.
 *
 * Data layouts are the reference's (ct_laboratory, src/ct_projector_*.cu):
 *   volume   float32 [batch, n_x, n_y, n_z], C-contiguous (k fastest)
 *   image    float32 [batch, n_row, n_col], C-contiguous
 *   src, dst float32 [n_ray, 3] (3-D) or [n_ray, 2] (2-D), world coordinates
 *   sinogram float32 [batch, n_ray]
 *   M_inv    float32 [9] (3-D) or [4] (2-D), row-major inverse of the
 *            voxel-index -> world matrix M;   b float32 [3] / [2].
 *            Both live in device memory, exactly as the reference's kernels
 *            take them (ct_projector_3d.cu:21-36).
 *   tvals    float32 [n_ray, n_int], sorted plane parameters, +inf padded
 *   t_uint16 uint16  [n_ray, n_int] delta-encoded tvals (stored by the
 *            reference in a torch.int16 tensor), t_start / t_scale [n_ray].
 *
 * Adjoint entry points take `accumulate`: 0 zeroes `out` on the stream first
 * (the reference returns torch::zeros-initialised volumes), 1 adds into it.
 */
#ifndef CTLAB_B200_H
#define CTLAB_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CTLAB_OK 0
#define CTLAB_EINVAL 1  /* bad argument: null pointer, negative or oversized dimension */
#define CTLAB_ECUDA 2   /* a CUDA runtime call or kernel launch failed */
#define CTLAB_ETIMEOUT 3 /* a bounded device-side wait gave up */

#define CTLAB_ABI_VERSION 1

/* ABI version of the loaded library (CTLAB_ABI_VERSION). */
int ctlab_abi_version(void);

/* Message of the calling thread's last failed call ("" if none). */
const char* ctlab_last_error(void);

/* M_inv = M^-1 for a row-major n x n matrix (n = 2 or 3) in device memory,
 * computed on the stream by Gauss-Jordan elimination with partial pivoting.
 * Replaces the torch.inverse(M) calls of the reference's wrappers
 * (tomography/ct_projector_3d_cuda.py:42-48, ct_projector_2d_cuda.py:6-8)
 * without a host synchronisation.  A singular or non-finite M yields NaN
 * entries and, if `singular` is not NULL, *singular = 1 (device memory). */
int ctlab_invert_matrix(const float* M, int n, float* M_inv, int* singular, void* stream);

/*
 * Launch options of the on-the-fly projectors (the *_ex / *_siddon calls).
 *
 * Ray tiling: rays are addressed as a grid
 *     ray = view * view_stride + row * row_stride + col * col_stride
 * with n_view x n_row x n_col entries (n_view*n_row*n_col must equal n_ray).
 * One CTA covers `tile_rows` consecutive rows of (block_threads / tile_rows)
 * columns of one view, and the lanes of a warp run along rows.  For a cone-
 * beam scan ordered [view][det_v][det_u] (conebeam_projector_3d.py:84-94)
 * rows = det_v, cols = det_u puts adjacent lanes on vertically adjacent
 * detector cells: their rays share one x-y line, and with tile_rows a
 * multiple of 32 the 3-D kernels walk that line once per warp.
 *
 * Voxel rule: which voxel a segment between two consecutive plane crossings
 * is charged to.  CTLAB_VOXEL_MIDPOINT (the reference's rule,
 * ct_projector_3d.cu:982-996) rounds the segment's world-space midpoint;
 * CTLAB_VOXEL_CROSSING takes the voxel the two bounding crossings enclose
 * (exact topology, as an FP64 evaluation of the midpoint rule would).  They
 * differ only for segments whose extent across some plane family is below
 * the rounding noise of the midpoint (~1e-4 voxel), i.e. rays nearly
 * parallel to a plane family.
 *
 * A NULL options pointer means: flat run (n_view = 1, n_row = n_ray,
 * n_col = 1, 256 threads) with the midpoint rule.
 */
#define CTLAB_VOXEL_MIDPOINT 0
#define CTLAB_VOXEL_CROSSING 1
/* Walk: CTLAB_WALK_LANE walks each ray on its own lane.  CTLAB_WALK_COLUMN
 * (3-D, either voxel rule, detector-row tilings with tile_rows a multiple of
 * 32 or equal to 16, grid dimensions <= 65536) derives the merged x-y
 * crossings of a warp's shared line (or of each 16-lane group's) once and
 * splits each x-y cell per lane at its z planes.  Warps fall back to the
 * lane walk inside the same launch where their rays do not share their x-y
 * line; under the crossing rule also where a ray's z slope is steeper than
 * 3/4 of its x-y slope, and under the midpoint rule where M^-1 is not
 * diagonal.  The crossing rule's two walks give bitwise equal forward
 * projections; under the midpoint rule the column walk sums in another
 * order (equal to rounding).  CTLAB_WALK_AUTO takes the column walk
 * wherever it applies (the faster one measured) and the lane walk
 * elsewhere. */
#define CTLAB_WALK_AUTO 0
#define CTLAB_WALK_LANE 1
#define CTLAB_WALK_COLUMN 2
typedef struct ctlab_ray_opts {
    int64_t n_view, n_row, n_col;
    int64_t view_stride, row_stride, col_stride;
    int32_t tile_rows;     /* 1..block_threads, divides block_threads; 0 = 32 */
    int32_t block_threads; /* multiple of 32, <= 256; 0 = 256 */
    int32_t voxel_rule;    /* CTLAB_VOXEL_MIDPOINT or CTLAB_VOXEL_CROSSING */
    int32_t walk;          /* CTLAB_WALK_AUTO, CTLAB_WALK_LANE or CTLAB_WALK_COLUMN */
} ctlab_ray_opts;

/* ---------------------------------------------------------------------- */
/* 3-D, on the fly (no intersection table)                                 */
/* ---------------------------------------------------------------------- */

/* Replaces _C.forward_project_3d_on_the_fly_cuda (src/bindings.cpp:98;
 * host wrapper src/ct_projector_3d.cu:1018-1049, kernel :902-1012).
 * out[b, r] = sum over the ray's voxels of volume[b, voxel] * segment length. */
int ctlab_forward_project_3d_on_the_fly(const float* volume, int64_t batch, int64_t n_x, int64_t n_y,
                                        int64_t n_z, const float* src, const float* dst, int64_t n_ray,
                                        const float* M_inv, const float* b, float* out, void* stream);

/* Replaces _C.back_project_3d_on_the_fly_cuda (src/bindings.cpp:101;
 * src/ct_projector_3d.cu:1051-1079): the exact adjoint of the above, by
 * atomic scatter of sino[b, r] * segment length. */
int ctlab_back_project_3d_on_the_fly(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                     const float* dst, const float* M_inv, const float* b, int64_t n_x,
                                     int64_t n_y, int64_t n_z, float* out, int accumulate, void* stream);

/* The two calls above with launch options (NULL = flat, midpoint rule). */
int ctlab_forward_project_3d_on_the_fly_ex(const float* volume, int64_t batch, int64_t n_x, int64_t n_y,
                                           int64_t n_z, const float* src, const float* dst, int64_t n_ray,
                                           const float* M_inv, const float* b, float* out,
                                           const ctlab_ray_opts* tiling, void* stream);
int ctlab_back_project_3d_on_the_fly_ex(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                        const float* dst, const float* M_inv, const float* b, int64_t n_x,
                                        int64_t n_y, int64_t n_z, float* out, int accumulate,
                                        const ctlab_ray_opts* tiling, void* stream);

/* Active tiles.  A projector's geometry is fixed, while most of a scan's
 * rays may miss the volume (about two thirds on a cone-beam scan whose
 * detector overhangs the volume).  ctlab_active_tiles lists, once, the tiles
 * of `tiling` (the CTAs of the *_ex launches) that hold at least one ray the
 * walks charge: a ray is charged only if its end points are finite, its
 * direction is not degenerate and some of the box lies inside its [0, 1]
 * (ctlab_forward_project_3d_on_the_fly_ex applies exactly these tests to
 * every ray).  The *_tiles calls then launch only the listed tiles: the
 * forward zeroes its output first (every other ray projects to 0), the
 * adjoint adds nothing for them, so the results are those of the *_ex calls
 * with the same tiling.  `flags` is device workspace of ctlab_tile_count
 * bytes, `tiles_out` room for as many int32 entries, `*n_out` (device
 * memory) receives the count.  No counterpart in the reference, whose
 * kernels run every ray (src/ct_projector_3d.cu:1018-1049). */
int64_t ctlab_tile_count(int64_t n_ray, const ctlab_ray_opts* tiling);
int ctlab_active_tiles(const float* src, const float* dst, int64_t n_ray, const float* M_inv, const float* b,
                       int64_t n_x, int64_t n_y, int64_t n_z, const ctlab_ray_opts* tiling, uint8_t* flags,
                       int32_t* tiles_out, int64_t* n_out, void* stream);
int ctlab_forward_project_3d_on_the_fly_tiles(const float* volume, int64_t batch, int64_t n_x, int64_t n_y,
                                              int64_t n_z, const float* src, const float* dst, int64_t n_ray,
                                              const float* M_inv, const float* b, float* out,
                                              const ctlab_ray_opts* tiling, const int32_t* tiles, int64_t n_tiles,
                                              void* stream);
int ctlab_back_project_3d_on_the_fly_tiles(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                           const float* dst, const float* M_inv, const float* b, int64_t n_x,
                                           int64_t n_y, int64_t n_z, float* out, int accumulate,
                                           const ctlab_ray_opts* tiling, const int32_t* tiles, int64_t n_tiles,
                                           void* stream);

/*
 * One flat detector panel: a view whose cell centres form an affine grid
 *     dst(ju, jv) = origin + ju * du + jv * dv,   ray = first_ray + jv*v_stride + ju*u_stride
 * seen from one source point (a cone-beam view; a StaticCT module lit by one
 * source in one frame).  Stored with the dual basis eu, ev of (du, dv)
 * ((P - origin) . eu = ju for P in the panel plane) and the unit normal n.
 */
typedef struct ctlab_panel {
    float src[3], origin[3];
    float eu[3], ev[3];
    float n[3];
    int64_t first_ray, u_stride, v_stride;
    int32_t n_u, n_v;
} ctlab_panel;

/* Deterministic adjoint by gathering: every voxel sums y[b, r] * len(r, voxel)
 * over the rays of each panel that can reach it, in a fixed order, with
 * len the crossing-rule walk's parameter span (bitwise) times |v|.  It is bitwise
 * reproducible, and is the transpose of
 * ctlab_forward_project_3d_on_the_fly_ex with CTLAB_VOXEL_CROSSING.  No
 * counterpart in the reference (its adjoints all scatter with atomicAdd,
 * src/ct_projector_3d.cu:267, :374, :1005).  `M` is the voxel-index -> world
 * matrix (M_inv its inverse); panels live in device memory.  Writes out. */
int ctlab_back_project_3d_gather(const float* sino, int64_t batch, int64_t n_ray, const float* src, const float* dst,
                                 const float* M, const float* M_inv, const float* b, int64_t n_x, int64_t n_y,
                                 int64_t n_z, const ctlab_panel* panels, int64_t n_panel, float* out, void* stream);

/* ctlab_back_project_3d_gather with a caller-provided device workspace
 * `ray_table` of 32 * n_ray bytes, 16-byte aligned (NULL: as
 * ctlab_back_project_3d_gather): each ray's set-up (its source in index
 * space, 1/v and |v|) and its y are written into it once per sinogram
 * instead of recomputed by every voxel that the ray can reach.  The result
 * is bitwise the same. */
int ctlab_back_project_3d_gather_ws(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                    const float* dst, const float* M, const float* M_inv, const float* b, int64_t n_x,
                                    int64_t n_y, int64_t n_z, const ctlab_panel* panels, int64_t n_panel, float* out,
                                    void* ray_table, void* stream);

/* Reproducible scatter adjoint: the walk of ctlab_back_project_3d_on_the_fly_ex
 * (same rays, voxels and segment lengths under either voxel rule) with every
 * contribution y * len rounded once to a multiple of 2^-e and added as a
 * 64-bit integer.  Integer addition is associative, so the volume is the same
 * bits on every run, whatever the launch order or what else shares the GPU.
 * e is chosen per sinogram from max|y| * (the grid's longest world-space
 * diagonal) * n_ray <= 2^61, a bound on every voxel's sum; the result differs
 * from the float scatter by the rounding of n_ray terms, far below the float
 * adjoint's own order-dependence for any voxel a ray crosses more than a
 * hair.  A sinogram holding NaN or inf gives a NaN volume.  No counterpart
 * in the reference (its adjoints scatter with float atomicAdd,
 * src/ct_projector_3d.cu:1005).  `workspace` is device memory, 256-byte
 * aligned, of ctlab_back_project_3d_fixed_workspace_bytes bytes (one int64
 * volume per sinogram plus a header); it is cleared here.  `tiles` /
 * `n_tiles`: a list of active tiles of `tiling` (ctlab_active_tiles) to walk
 * only those, or NULL / -1 for every tile. */
int64_t ctlab_back_project_3d_fixed_workspace_bytes(int64_t batch, int64_t n_x, int64_t n_y, int64_t n_z);
int ctlab_back_project_3d_fixed(const float* sino, int64_t batch, int64_t n_ray, const float* src, const float* dst,
                                const float* M_inv, const float* b, int64_t n_x, int64_t n_y, int64_t n_z,
                                float* out, int accumulate, const ctlab_ray_opts* tiling, const int32_t* tiles,
                                int64_t n_tiles, void* workspace, int64_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------- */
/* Elementwise steps of a MAP iteration (the reconstruction server)        */
/* ---------------------------------------------------------------------- */

/* r[i] = y[i] - I0 exp(-p[i]) for i < n: the Beer-Lambert Poisson residual
 * of p = A x.  No counterpart in the reference, which forms it through
 * autograd (probability/random_variables/poisson.py:36-47). */
int ctlab_map_poisson_residual(const float* y, const float* p, float* r, int64_t n, float I0, void* stream);

/* g += w * sum_d D_d^T D_d x (D_d the forward difference along axis d of the
 * [n_x][n_y][n_z] volume, no wrap-around), then x -= lr * g: the quadratic
 * smoothness prior's gradient and the gradient step.  No counterpart in the
 * reference, which forms it through autograd (image_energies.py:18-29,
 * bayesian_estimation/map_estimator.py:102-117). */
int ctlab_map_smoothness_step(float* x, float* g, int64_t n_x, int64_t n_y, int64_t n_z, float w, float lr,
                              void* stream);

/* ---------------------------------------------------------------------- */
/* 3-D, precomputed intersections                                          */
/* ---------------------------------------------------------------------- */

/* Replaces _C.compute_intersections_3d (src/bindings.cpp:83;
 * src/ct_projector_3d.cu:42-96, 381-401).  t_out is [n_ray, n_int] with
 * n_int = (n_x+1)+(n_y+1)+(n_z+1): every x/y/z plane parameter in [0,1],
 * ascending, then +inf. */
int ctlab_compute_intersections_3d(int64_t n_x, int64_t n_y, int64_t n_z, const float* src, const float* dst,
                                   int64_t n_ray, const float* M_inv, const float* b, float* t_out,
                                   void* stream);

/* Replaces _C.forward_project_3d_cuda (src/bindings.cpp:85;
 * src/ct_projector_3d.cu:272-323, 403-433). */
int ctlab_forward_project_3d_tvals(const float* volume, int64_t batch, int64_t n_x, int64_t n_y, int64_t n_z,
                                   const float* tvals, int64_t n_int, const float* src, const float* dst,
                                   int64_t n_ray, const float* M_inv, const float* b, float* out, void* stream);

/* Replaces _C.back_project_3d_cuda (src/bindings.cpp:87;
 * src/ct_projector_3d.cu:326-376, 435-462). */
int ctlab_back_project_3d_tvals(const float* sino, int64_t batch, int64_t n_ray, const float* tvals,
                                int64_t n_int, const float* src, const float* dst, const float* M_inv,
                                const float* b, int64_t n_x, int64_t n_y, int64_t n_z, float* out, int accumulate,
                                void* stream);

/* Replaces _C.compress_tvals_3d_cuda (src/bindings.cpp:90;
 * src/ct_projector_3d.cu:160-212, 464-489).  Writes t_uint16 [n_ray, n_int],
 * t_start [n_ray] and t_scale [n_ray] exactly as the reference kernel does. */
int ctlab_compress_tvals_3d(const float* tvals, int64_t n_ray, int64_t n_int, const float* src,
                            const float* dst, float voxel_diag_len, uint16_t* t_uint16, float* t_start,
                            float* t_scale, void* stream);

/* The compressor with a choice of encoder.  The reference has two that
 * disagree: CTLAB_COMPRESS_CUDA is compress_tvals_3d_kernel
 * (src/ct_projector_3d.cu:160-212; what ctlab_compress_tvals_3d does);
 * CTLAB_COMPRESS_TORCH is compress_tvals_to_uint16
 * (tomography/ct_projector_3d_torch.py:4-65), which CTProjector3DModule uses
 * for its own precompute (ct_projector_3d_module.py:100-102): +inf becomes
 * 10.0, rounding is half to even and the running sum is a float. */
#define CTLAB_COMPRESS_CUDA 0
#define CTLAB_COMPRESS_TORCH 1
int ctlab_compress_tvals_3d_ex(const float* tvals, int64_t n_ray, int64_t n_int, const float* src, const float* dst,
                               float voxel_diag_len, uint16_t* t_uint16, float* t_start, float* t_scale, int mode,
                               void* stream);

/* Replaces _C.forward_project_3d_compressed_cuda (src/bindings.cpp:92;
 * src/ct_projector_3d.cu:99-157, 491-522). */
int ctlab_forward_project_3d_compressed(const float* volume, int64_t batch, int64_t n_x, int64_t n_y,
                                        int64_t n_z, const uint16_t* t_uint16, const float* t_start,
                                        const float* t_scale, int64_t n_int, const float* src, const float* dst,
                                        int64_t n_ray, const float* M_inv, const float* b, float* out,
                                        void* stream);

/* Replaces _C.back_project_3d_compressed_cuda (src/bindings.cpp:94;
 * src/ct_projector_3d.cu:215-269, 524-553). */
int ctlab_back_project_3d_compressed(const float* sino, int64_t batch, int64_t n_ray, const uint16_t* t_uint16,
                                     const float* t_start, const float* t_scale, int64_t n_int, const float* src,
                                     const float* dst, const float* M_inv, const float* b, int64_t n_x,
                                     int64_t n_y, int64_t n_z, float* out, int accumulate, void* stream);

/* ---------------------------------------------------------------------- */
/* 2-D                                                                     */
/* ---------------------------------------------------------------------- */

/* Replaces _C.compute_intersections_2d (src/bindings.cpp:67;
 * src/ct_projector_2d.cu:36-73, 158-177). n_int = (n_row+1)+(n_col+1). */
int ctlab_compute_intersections_2d(int64_t n_row, int64_t n_col, const float* src, const float* dst,
                                   int64_t n_ray, const float* M_inv, const float* b, float* t_out,
                                   void* stream);

/* Replaces _C.forward_project_2d_cuda (src/bindings.cpp:69;
 * src/ct_projector_2d.cu:76-114, 179-200). */
int ctlab_forward_project_2d_tvals(const float* image, int64_t batch, int64_t n_row, int64_t n_col,
                                   const float* tvals, int64_t n_int, const float* src, const float* dst,
                                   int64_t n_ray, const float* M_inv, const float* b, float* out, void* stream);

/* Replaces _C.back_project_2d_cuda (src/bindings.cpp:71;
 * src/ct_projector_2d.cu:117-155, 202-221). */
int ctlab_back_project_2d_tvals(const float* sino, int64_t batch, int64_t n_ray, const float* tvals,
                                int64_t n_int, const float* src, const float* dst, const float* M_inv,
                                const float* b, int64_t n_row, int64_t n_col, float* out, int accumulate,
                                void* stream);

/* Replaces _C.forward_project_2d_on_the_fly_cuda (src/bindings.cpp:75;
 * src/ct_projector_2d.cu:246-331, 416-440), keeping its incremental march
 * (t_next += dt) so results follow that kernel rather than the tvals path. */
int ctlab_forward_project_2d_on_the_fly(const float* image, int64_t batch, int64_t n_row, int64_t n_col,
                                        const float* src, const float* dst, int64_t n_ray, const float* M_inv,
                                        const float* b, float* out, void* stream);

/* Replaces _C.back_project_2d_on_the_fly_cuda (src/bindings.cpp:78;
 * src/ct_projector_2d.cu:334-413, 442-465). */
int ctlab_back_project_2d_on_the_fly(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                     const float* dst, const float* M_inv, const float* b, int64_t n_row,
                                     int64_t n_col, float* out, int accumulate, void* stream);

/* 2-D Siddon without an intersection table, with the per-plane parameter
 * arithmetic of the 3-D kernels (every plane parameter evaluated on its own,
 * no drift).  Used by the 2-D module in place of the reference's
 * precomputed-table path (ct_projector_2d_module.py:35-41, which stores
 * [n_ray, n_int] tables), with the same results within float rounding. */
int ctlab_forward_project_2d_siddon(const float* image, int64_t batch, int64_t n_row, int64_t n_col,
                                    const float* src, const float* dst, int64_t n_ray, const float* M_inv,
                                    const float* b, float* out, const ctlab_ray_opts* tiling, void* stream);
int ctlab_back_project_2d_siddon(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                 const float* dst, const float* M_inv, const float* b, int64_t n_row,
                                 int64_t n_col, float* out, int accumulate, const ctlab_ray_opts* tiling,
                                 void* stream);

/* ctlab_back_project_2d_siddon with scratch: `scratch` is NULL or device
 * memory of batch * n_row * n_col floats (not `out`; its contents are
 * overwritten).  Rays whose larger index-space direction component is
 * along the image's columns (its stride-1 axis) accumulate into the images'
 * transposes there, which are then added into `out`: neighbouring rays then
 * add into neighbouring addresses, and the L2 performs several times fewer
 * reduction operations.  Same segments and result, either voxel rule, up to
 * the order of the float additions.  No counterpart in the reference. */
int ctlab_back_project_2d_siddon_ws(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                    const float* dst, const float* M_inv, const float* b, int64_t n_row,
                                    int64_t n_col, float* out, int accumulate, const ctlab_ray_opts* tiling,
                                    float* scratch, void* stream);

/* ---------------------------------------------------------------------- */
/* Many scans in one launch                                                */
/* ---------------------------------------------------------------------- */

/*
 * One scan of a batch: its geometry, its voxel grid and the buffers a
 * forward and / or an adjoint pass read and write (batch size 1 per scan;
 * layouts as above).  The forward reads image_in and writes sino_out; the
 * adjoint reads sino_in and writes (or adds into) image_out.  Either pair may
 * be NULL when that pass is not run; a scan with n_ray = 0 may give NULL
 * sinogram pointers.  `opts` is the scan's ray tiling and
 * voxel rule as for the single-scan *_ex calls (n_view = 0: flat); every scan
 * of a batch has the same ndim and voxel rule, and opts.block_threads is 0 or
 * the batch's.  opts.walk is not used: 3-D crossing-rule scans take the
 * column walk in every warp whose rays share their x-y line and the per-lane
 * walk elsewhere, which give bitwise equal results.
 */
typedef struct ctlab_scan {
    const float* image_in;
    float* sino_out;
    const float* sino_in;
    float* image_out;
    const float* src;
    const float* dst;
    const float* M_inv;
    const float* b;
    int64_t n_ray;
    int64_t dims[3]; /* 2-D: n_row, n_col (dims[2] unused); 3-D: n_x, n_y, n_z (each <= 65536) */
    int32_t ndim;    /* 2 or 3 */
    int32_t reserved;
    ctlab_ray_opts opts;
    /* NULL or dims[0] * dims[1] floats of device memory for a 2-D adjoint:
     * the transposed accumulation of ctlab_back_project_2d_siddon_ws
     * (contents overwritten).  Ignored in 3-D. */
    float* image_scratch;
} ctlab_scan;

/* A plan: filled by ctlab_batch_plan, owned by the caller, read by the
 * launch calls.  `workspace` is the caller's device buffer that holds the
 * work counter and the resolved scan table. */
typedef struct ctlab_batch {
    void* workspace;
    int64_t total_tiles;
    int32_t n_scan, ndim, block_threads, voxel_rule;
    int32_t has_forward, has_adjoint;
    int32_t device;
    int32_t has_scratch; /* some scan's adjoint accumulates in image_scratch */
} ctlab_batch;

/* Bytes of device workspace a plan of n_scan scans needs (-1 if n_scan is
 * outside [1, 65535]). */
int64_t ctlab_batch_workspace_bytes(int32_t n_scan);

/* Validates the scans (host array) and copies their resolved table into
 * `workspace` (device memory, 256-byte aligned, at least
 * ctlab_batch_workspace_bytes(n_scan) bytes) on `stream`; fills *plan.  Every
 * scan is cut into tiles of block_threads rays (0 = 256); tiles are handed
 * out in scan order, so list the heaviest scans first.  The plan stays valid
 * while the workspace and every bound buffer stay allocated.  The table is
 * copied from pageable memory (the call waits for the stream), so call this
 * outside stream capture.
 *
 * No counterpart in the reference, whose projectors take one scan per call
 * (src/bindings.cpp:65-104); it batches the calls that
 * ctlab_forward_project_3d_on_the_fly_ex / ctlab_forward_project_2d_siddon
 * (and their adjoints) make one at a time, with their results: bitwise for
 * the forward, up to the order of the float atomic additions for the adjoint. */
int ctlab_batch_plan(const ctlab_scan* scans, int32_t n_scan, int32_t block_threads, void* workspace,
                     int64_t workspace_bytes, ctlab_batch* plan, void* stream);

/* One persistent launch of n_cta CTAs (0 = resident CTAs per SM x SMs) that
 * projects every scan of the plan: sino_out = A image_in.  Resets the
 * plan's work counter on the stream first (cudaMemsetAsync), so launches of
 * one plan on one stream may follow each other, and may be captured in a
 * CUDA graph; launches of one plan on two streams at once race. */
int ctlab_forward_project_batched(const ctlab_batch* plan, int32_t n_cta, void* stream);

/* image_out = A^T sino_in for every scan of the plan (accumulate = 0 zeroes
 * each image_out first, 1 adds into it); one zeroing launch (if any: image
 * outputs, scratch buffers), one persistent launch and, when scans have
 * image_scratch, one launch that adds the transposed parts back. */
int ctlab_back_project_batched(const ctlab_batch* plan, int accumulate, int32_t n_cta, void* stream);

/* Resident CTAs per SM x SMs of the current device for the batched kernel
 * of this kind (ndim, adjoint 0/1, voxel rule, block_threads). */
int ctlab_batch_default_ctas(int32_t ndim, int adjoint, int voxel_rule, int32_t block_threads, int32_t* n_cta);

/* The batched projector for callers that cannot allocate GPU memory: a
 * plugin whose host application's allocator owns the whole device, or a
 * real-time loop where an allocation could stall or fail mid-scan.  No
 * counterpart in the reference (it has no batched or allocation-free path).
 *
 * Projects every scan of a host array once: the forward (adjoint = 0:
 * sino_out = A image_in) or the adjoint (adjoint = 1: image_out = A^T sino_in,
 * zeroed first unless accumulate = 1), with the results of
 * ctlab_forward_project_batched / ctlab_back_project_batched.  The caller
 * still owns every input and output buffer; the scratch those calls keep in
 * a workspace (work counter, resolved scan table) lives instead in a fixed
 * array inside the library's device image, of at most 64 scans (about
 * 13 KB, held on every GPU that loads the library until the process
 * exits).  More than 64 scans is rejected with CTLAB_EINVAL.  No cudaMalloc,
 * cudaFree or other allocating call is made.
 *
 * The first call on each device looks up that array's device address (with
 * the device current) and caches it; make that first call before any
 * stream capture.  Each call copies the scan table in from host memory,
 * which waits for work already queued on `stream`, and clears the work
 * counter.  All calls share the one array, so calls whose work overlaps on
 * the GPU (other streams, other host threads) race and give wrong results:
 * issue them one after another.  block_threads (0 = 256) and n_cta
 * (0 = resident CTAs per SM x SMs) as for the planned calls. */
int ctlab_project_batched_noalloc(const ctlab_scan* scans, int32_t n_scan, int adjoint, int accumulate,
                                  int32_t block_threads, int32_t n_cta, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CTLAB_B200_H */
