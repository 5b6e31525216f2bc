/*
 * Siddon oracle body, included twice by siddon_oracle.c: once with
 * REAL=float (suffix _f32) and once with REAL=double (suffix _f64).
 *
 * TEST INFRASTRUCTURE ONLY.  This is a CPU restatement of the reference
 * ct_laboratory projector, used by tests/, by __graft_entry__.smoke() and by
 * bench.py's cpu_baseline / --impl reference legs as the checker and the CPU
 * baseline.  The product (ct_laboratory_b200) never links or calls it.
 *
 * Two families of routines live here:
 *
 *  1. "torch path" routines restate the reference's pure-PyTorch backend
 *     (ct_laboratory/tomography/ct_projector_{2d,3d}_torch.py) operation by
 *     operation, with every float operation rounded separately (the file is
 *     compiled with -ffp-contract=off) because each torch op materialises a
 *     rounded tensor.  These are what the golden fixtures pin.
 *
 *  2. "cuda path" routines restate the reference's CUDA kernels
 *     (src/ct_projector_{2d,3d}.cu): the on-the-fly plane-sort kernel, the 2-D
 *     on-the-fly DDA, the uint16 compressor and the compressed decode.  nvcc
 *     contracts a*b+c into one fused multiply-add by default; where the
 *     reference writes such an expression the restatement uses an explicit
 *     FMA (FMA_) so that the CPU arithmetic mirrors the GPU's.
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SUFFIX)

/* ------------------------------------------------------------------ */
/* small helpers                                                       */
/* ------------------------------------------------------------------ */

/* torch.round / __float2int_rn: round half to even (default FE_TONEAREST). */
static inline int64_t FN(rne_)(REAL v) { return (int64_t)NEARBYINT_(v); }

/* (src - b) @ M_inv^T, evaluated left to right without fusion
 * (ct_projector_3d_torch.py:100-104). */
static inline void FN(affine3_torch_)(const REAL* Mi, const REAL* b, REAL x, REAL y, REAL z,
                                      REAL* i, REAL* j, REAL* k) {
    REAL xs = x - b[0], ys = y - b[1], zs = z - b[2];
    *i = (Mi[0] * xs + Mi[1] * ys) + Mi[2] * zs;
    *j = (Mi[3] * xs + Mi[4] * ys) + Mi[5] * zs;
    *k = (Mi[6] * xs + Mi[7] * ys) + Mi[8] * zs;
}

/* apply_affine_inverse_3d (ct_projector_3d.cu:21-36) as nvcc contracts it:
 * a*b + c*d becomes fma(a, b, c*d), then + M2*z becomes fma(M2, z, .). */
static inline void FN(affine3_cuda_)(const REAL* Mi, const REAL* b, REAL x, REAL y, REAL z,
                                     REAL* i, REAL* j, REAL* k) {
    REAL xs = x - b[0], ys = y - b[1], zs = z - b[2];
    *i = FMA_(Mi[2], zs, FMA_(Mi[0], xs, Mi[1] * ys));
    *j = FMA_(Mi[5], zs, FMA_(Mi[3], xs, Mi[4] * ys));
    *k = FMA_(Mi[8], zs, FMA_(Mi[6], xs, Mi[7] * ys));
}

static inline void FN(affine2_torch_)(const REAL* Mi, const REAL* b, REAL x, REAL y, REAL* r, REAL* c) {
    REAL xs = x - b[0], ys = y - b[1];
    *r = Mi[0] * xs + Mi[1] * ys;
    *c = Mi[2] * xs + Mi[3] * ys;
}

/* apply_affine_inverse (ct_projector_2d.cu:18-30), contracted. */
static inline void FN(affine2_cuda_)(const REAL* Mi, const REAL* b, REAL x, REAL y, REAL* r, REAL* c) {
    REAL xs = x - b[0], ys = y - b[1];
    *r = FMA_(Mi[0], xs, Mi[1] * ys);
    *c = FMA_(Mi[2], xs, Mi[3] * ys);
}

static int FN(cmp_)(const void* a, const void* b) {
    REAL x = *(const REAL*)a, y = *(const REAL*)b;
    return (x > y) - (x < y);
}

/* ------------------------------------------------------------------ */
/* 1. torch path                                                        */
/* ------------------------------------------------------------------ */

/* One ray's sorted plane parameters, ct_projector_3d_torch.py:78-158
 * (3-D, zero rule |dir| < 1e-12) and ct_projector_2d_torch.py:4-65 (2-D,
 * zero rule dir == 0).  dims[0..ndim-1] are the grid sizes, s/d the
 * index-space endpoints.  Writes K = sum(dims+1) values to t. */
static void FN(isect_row_)(int ndim, const int* dims, const REAL* s, const REAL* d, int zero_exact,
                           int sort_mode, REAL* t) {
    int c = 0;
    for (int a = 0; a < ndim; ++a) {
        REAL dir = d[a] - s[a];
        int zero = zero_exact ? (dir == (REAL)0) : (FABS_(dir) < (REAL)1e-12);
        for (int p = 0; p <= dims[a]; ++p) {
            REAL plane = (REAL)p - (REAL)0.5;
            REAL tt = (plane - s[a]) / dir;
            if (zero) tt = (REAL)INFINITY;
            if (tt < (REAL)0 || tt > (REAL)1) tt = (REAL)INFINITY;
            t[c++] = tt;
        }
    }
    if (sort_mode) qsort(t, (size_t)c, sizeof(REAL), FN(cmp_));
}

/* compute_intersections_{2d,3d}_torch.  ndim is 2 or 3; Mi is M^-1 as
 * torch.inverse(M) produced it (row-major ndim x ndim). */
void FN(orc_isect_torch)(int ndim, const int* dims, const REAL* Mi, const REAL* b,
                         const REAL* src, const REAL* dst, int64_t n_ray, REAL* t_out) {
    int K = 0;
    for (int a = 0; a < ndim; ++a) K += dims[a] + 1;
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n_ray; ++r) {
        REAL s[3], d[3];
        if (ndim == 3) {
            FN(affine3_torch_)(Mi, b, src[3 * r], src[3 * r + 1], src[3 * r + 2], &s[0], &s[1], &s[2]);
            FN(affine3_torch_)(Mi, b, dst[3 * r], dst[3 * r + 1], dst[3 * r + 2], &d[0], &d[1], &d[2]);
        } else {
            FN(affine2_torch_)(Mi, b, src[2 * r], src[2 * r + 1], &s[0], &s[1]);
            FN(affine2_torch_)(Mi, b, dst[2 * r], dst[2 * r + 1], &d[0], &d[1]);
        }
        FN(isect_row_)(ndim, dims, s, d, ndim == 2, 1, t_out + (size_t)r * K);
    }
}

/* Per-segment work of forward_project_{2d,3d}_torch / back_project_*_torch
 * (ct_projector_3d_torch.py:219-271, ct_projector_2d_torch.py:89-161):
 * points s + t*dir, segment length sqrt of squared differences, midpoint
 * rounded to the nearest voxel (half to even).  Returns the flat voxel index
 * or -1 when the segment is masked; *len receives the segment length. */
static inline int64_t FN(seg_torch_)(int ndim, const int* dims, const REAL* Mi, const REAL* b,
                                     const REAL* sw, const REAL* vw, REAL t0, REAL t1, REAL* len) {
    REAL p0[3], p1[3];
    int inf = 0;
    for (int a = 0; a < ndim; ++a) {
        p0[a] = sw[a] + t0 * vw[a];
        p1[a] = sw[a] + t1 * vw[a];
        inf |= ISINF_(p0[a]) | ISINF_(p1[a]);
    }
    if (inf) return -1;
    REAL acc = 0;
    for (int a = 0; a < ndim; ++a) {
        REAL dd = p1[a] - p0[a];
        acc = (a == 0) ? dd * dd : acc + dd * dd;
    }
    *len = SQRT_(acc);
    REAL m[3], f[3];
    for (int a = 0; a < ndim; ++a) m[a] = (REAL)0.5 * (p0[a] + p1[a]);
    if (ndim == 3) FN(affine3_torch_)(Mi, b, m[0], m[1], m[2], &f[0], &f[1], &f[2]);
    else FN(affine2_torch_)(Mi, b, m[0], m[1], &f[0], &f[1]);
    int64_t flat = 0;
    for (int a = 0; a < ndim; ++a) {
        int64_t ix = FN(rne_)(f[a]);
        if (ix < 0 || ix >= dims[a]) return -1;
        flat = flat * dims[a] + ix;
    }
    return flat;
}

/* forward_project_{2d,3d}_torch with a float tvals table [n_ray, K]. */
void FN(orc_fwd_tvals_torch)(int ndim, const int* dims, const REAL* img, const REAL* tvals, int K,
                             const REAL* Mi, const REAL* b, const REAL* src, const REAL* dst,
                             int64_t n_ray, REAL* out) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t r = 0; r < n_ray; ++r) {
        REAL sw[3], vw[3];
        for (int a = 0; a < ndim; ++a) {
            sw[a] = src[ndim * r + a];
            vw[a] = dst[ndim * r + a] - sw[a];
        }
        const REAL* t = tvals + (size_t)r * K;
        double acc = 0.0;
        for (int i = 0; i < K - 1; ++i) {
            REAL len;
            int64_t v = FN(seg_torch_)(ndim, dims, Mi, b, sw, vw, t[i], t[i + 1], &len);
            if (v >= 0) acc += (double)(img[v] * len);
        }
        out[r] = (REAL)acc;
    }
}

/* back_project_{2d,3d}_torch with a float tvals table.  Accumulates into out
 * (caller zeroes) in ray-major order, as scatter_add_ does on the CPU. */
void FN(orc_back_tvals_torch)(int ndim, const int* dims, const REAL* sino, const REAL* tvals, int K,
                              const REAL* Mi, const REAL* b, const REAL* src, const REAL* dst,
                              int64_t n_ray, REAL* out) {
    for (int64_t r = 0; r < n_ray; ++r) {
        REAL sw[3], vw[3];
        for (int a = 0; a < ndim; ++a) {
            sw[a] = src[ndim * r + a];
            vw[a] = dst[ndim * r + a] - sw[a];
        }
        const REAL* t = tvals + (size_t)r * K;
        for (int i = 0; i < K - 1; ++i) {
            REAL len;
            int64_t v = FN(seg_torch_)(ndim, dims, Mi, b, sw, vw, t[i], t[i + 1], &len);
            if (v >= 0) out[v] += sino[r] * len;
        }
    }
}

/* The reference CPU "no precompute" path as its benchmark runs it
 * (benchmark/projector_timing_benchmark.py:171-190): intersections then the
 * tvals forward, one ray at a time so no [n_ray, K] table is materialised. */
void FN(orc_fwd_otf_torch)(int ndim, const int* dims, const REAL* img, const REAL* Mi, const REAL* b,
                           const REAL* src, const REAL* dst, int64_t n_ray, REAL* out) {
    int K = 0;
    for (int a = 0; a < ndim; ++a) K += dims[a] + 1;
#pragma omp parallel
    {
        REAL* t = (REAL*)malloc(sizeof(REAL) * (size_t)K);
#pragma omp for schedule(dynamic, 256)
        for (int64_t r = 0; r < n_ray; ++r) {
            REAL s[3], d[3], sw[3], vw[3];
            if (ndim == 3) {
                FN(affine3_torch_)(Mi, b, src[3 * r], src[3 * r + 1], src[3 * r + 2], &s[0], &s[1], &s[2]);
                FN(affine3_torch_)(Mi, b, dst[3 * r], dst[3 * r + 1], dst[3 * r + 2], &d[0], &d[1], &d[2]);
            } else {
                FN(affine2_torch_)(Mi, b, src[2 * r], src[2 * r + 1], &s[0], &s[1]);
                FN(affine2_torch_)(Mi, b, dst[2 * r], dst[2 * r + 1], &d[0], &d[1]);
            }
            FN(isect_row_)(ndim, dims, s, d, ndim == 2, 1, t);
            for (int a = 0; a < ndim; ++a) {
                sw[a] = src[ndim * r + a];
                vw[a] = dst[ndim * r + a] - sw[a];
            }
            double acc = 0.0;
            for (int i = 0; i < K - 1; ++i) {
                REAL len;
                int64_t v = FN(seg_torch_)(ndim, dims, Mi, b, sw, vw, t[i], t[i + 1], &len);
                if (v >= 0) acc += (double)(img[v] * len);
            }
            out[r] = (REAL)acc;
        }
        free(t);
    }
}

/* Adjoint of orc_fwd_otf_torch.  Each thread scatters into a private volume
 * and the partial volumes are summed at the end, so the summation order is
 * fixed for a given thread count. */
void FN(orc_back_otf_torch)(int ndim, const int* dims, const REAL* sino, const REAL* Mi, const REAL* b,
                            const REAL* src, const REAL* dst, int64_t n_ray, REAL* out) {
    int K = 0;
    size_t nvox = 1;
    for (int a = 0; a < ndim; ++a) {
        K += dims[a] + 1;
        nvox *= (size_t)dims[a];
    }
    int nth = 1;
#ifdef _OPENMP
    nth = omp_get_max_threads();
#endif
    REAL* part = (REAL*)calloc((size_t)nth * nvox, sizeof(REAL));
#pragma omp parallel
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        REAL* mine = part + (size_t)tid * nvox;
        REAL* t = (REAL*)malloc(sizeof(REAL) * (size_t)K);
#pragma omp for schedule(dynamic, 256)
        for (int64_t r = 0; r < n_ray; ++r) {
            REAL s[3], d[3], sw[3], vw[3];
            if (ndim == 3) {
                FN(affine3_torch_)(Mi, b, src[3 * r], src[3 * r + 1], src[3 * r + 2], &s[0], &s[1], &s[2]);
                FN(affine3_torch_)(Mi, b, dst[3 * r], dst[3 * r + 1], dst[3 * r + 2], &d[0], &d[1], &d[2]);
            } else {
                FN(affine2_torch_)(Mi, b, src[2 * r], src[2 * r + 1], &s[0], &s[1]);
                FN(affine2_torch_)(Mi, b, dst[2 * r], dst[2 * r + 1], &d[0], &d[1]);
            }
            FN(isect_row_)(ndim, dims, s, d, ndim == 2, 1, t);
            for (int a = 0; a < ndim; ++a) {
                sw[a] = src[ndim * r + a];
                vw[a] = dst[ndim * r + a] - sw[a];
            }
            for (int i = 0; i < K - 1; ++i) {
                REAL len;
                int64_t v = FN(seg_torch_)(ndim, dims, Mi, b, sw, vw, t[i], t[i + 1], &len);
                if (v >= 0) mine[v] += sino[r] * len;
            }
        }
        free(t);
#pragma omp for schedule(static)
        for (size_t v = 0; v < nvox; ++v) {
            REAL acc = 0;
            for (int k = 0; k < nth; ++k) acc += part[(size_t)k * nvox + v];
            out[v] += acc;
        }
    }
    free(part);
}

/* Longest voxel diagonal |M d| over the four body diagonals
 * (ct_projector_3d_torch.py:28-35, ct_projector_3d_cuda.py:97-104). */
REAL FN(orc_voxel_diag_len)(const REAL* M) {
    static const int dg[4][3] = {{1, 1, 1}, {1, 1, -1}, {1, -1, 1}, {-1, 1, 1}};
    REAL best = 0;
    for (int q = 0; q < 4; ++q) {
        REAL n2 = 0;
        for (int r = 0; r < 3; ++r) {
            REAL v = (M[3 * r] * (REAL)dg[q][0] + M[3 * r + 1] * (REAL)dg[q][1]) + M[3 * r + 2] * (REAL)dg[q][2];
            n2 = (r == 0) ? v * v : FMA_(v, v, n2);
        }
        REAL n = SQRT_(n2);
        if (n > best) best = n;
    }
    return best;
}

/* compress_tvals_to_uint16 (ct_projector_3d_torch.py:4-65).  scales may be
 * given (as torch computed them) or NULL, in which case they are computed
 * here from |dst-src|.  inf entries become 10.0 before encoding; deltas are
 * clamped to [0, 32000] and the running sum is kept in REAL. */
void FN(orc_compress_torch)(const REAL* tvals, int64_t n_ray, int K, const REAL* src, const REAL* dst,
                            REAL voxel_diag_len, const REAL* scales_in, uint16_t* u16, REAL* starts,
                            REAL* scales) {
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n_ray; ++r) {
        REAL sc;
        if (scales_in) {
            sc = scales_in[r];
        } else {
            REAL dx = dst[3 * r] - src[3 * r], dy = dst[3 * r + 1] - src[3 * r + 1], dz = dst[3 * r + 2] - src[3 * r + 2];
            /* torch.norm(dim=1) on the CPU accumulates the squares with fused
             * multiply-adds: sqrt(fma(z, z, fma(y, y, x*x))). */
            REAL len = SQRT_(FMA_(dz, dz, FMA_(dy, dy, dx * dx)));
            if (len < (REAL)1e-6) len = (REAL)1e-6;
            sc = (voxel_diag_len / (REAL)10000.0) / len;
        }
        scales[r] = sc;
        const REAL* t = tvals + (size_t)r * K;
        uint16_t* o = u16 + (size_t)r * K;
        REAL start = ISINF_(t[0]) ? (REAL)10.0 : t[0];
        starts[r] = start;
        REAL inv = (REAL)1.0 / sc;
        REAL prev = 0;
        o[0] = 0;
        for (int i = 1; i < K; ++i) {
            REAL ti = ISINF_(t[i]) ? (REAL)10.0 : t[i];
            REAL cur = NEARBYINT_((ti - start) * inv);
            REAL diff = cur - prev;
            if (diff < 0) diff = 0;
            if (diff > 32000) diff = 32000;
            o[i] = (uint16_t)(int)diff;
            prev += (REAL)o[i];
        }
    }
}

/* decompress_tvals_from_uint16 (ct_projector_3d_torch.py:68-75): REAL cumsum,
 * times scale, plus start, each rounded. */
void FN(orc_decompress_torch)(const uint16_t* u16, const REAL* starts, const REAL* scales, int64_t n_ray,
                              int K, REAL* t_out) {
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n_ray; ++r) {
        REAL cs = 0;
        for (int i = 0; i < K; ++i) {
            cs += (REAL)u16[(size_t)r * K + i];
            t_out[(size_t)r * K + i] = cs * scales[r] + starts[r];
        }
    }
}

/* ------------------------------------------------------------------ */
/* 2. cuda path                                                         */
/* ------------------------------------------------------------------ */

/* ray_kernel_plane_sort (ct_projector_3d.cu:902-1012) with collect_hits and
 * sort_in_place (:834-895): all plane hits in [0,1] via a reciprocal
 * multiply, plus the end points 0 and 1, sorted; segment length (t1-t0)*|v|;
 * voxel from the rounded world midpoint.  mode 0: forward (out[r] = sum),
 * mode 1: adjoint (out[voxel] += sino[r]*len, ray-major). */
static void FN(planesort_ray_)(int mode, const int* dims, const REAL* data, const REAL* Mi, const REAL* b,
                               const REAL* src, const REAL* dst, int64_t r, REAL* t, REAL* out) {
    REAL sx = src[3 * r], sy = src[3 * r + 1], sz = src[3 * r + 2];
    REAL dx = dst[3 * r], dy = dst[3 * r + 1], dz = dst[3 * r + 2];
    REAL vx = dx - sx, vy = dy - sy, vz = dz - sz;
    REAL ray_len = SQRT_(FMA_(vz, vz, FMA_(vx, vx, vy * vy)));
    if (ray_len < (REAL)1e-12) {
        if (mode == 0) out[r] = 0;
        return;
    }
    REAL s[3], d[3], v[3];
    FN(affine3_cuda_)(Mi, b, sx, sy, sz, &s[0], &s[1], &s[2]);
    FN(affine3_cuda_)(Mi, b, dx, dy, dz, &d[0], &d[1], &d[2]);
    for (int a = 0; a < 3; ++a) v[a] = d[a] - s[a];
    int n = 0;
    for (int a = 0; a < 3; ++a) {
        if (FABS_(v[a]) > (REAL)1e-12) {
            REAL inv = (REAL)1.0 / v[a];
            for (int p = 0; p <= dims[a]; ++p) {
                REAL tt = ((REAL)p - (REAL)0.5 - s[a]) * inv;
                if (tt >= (REAL)0 && tt <= (REAL)1) t[n++] = tt;
            }
        }
    }
    t[n++] = 0;
    t[n++] = 1;
    qsort(t, (size_t)n, sizeof(REAL), FN(cmp_));
    REAL acc = 0;
    REAL val = (mode == 1) ? data[r] : 0;
    for (int i = 0; i < n - 1; ++i) {
        REAL t0 = t[i], t1 = t[i + 1];
        if (t1 <= t0) continue;
        REAL tm = (REAL)0.5 * (t0 + t1);
        REAL mx = FMA_(tm, vx, sx), my = FMA_(tm, vy, sy), mz = FMA_(tm, vz, sz);
        REAL fi, fj, fk;
        FN(affine3_cuda_)(Mi, b, mx, my, mz, &fi, &fj, &fk);
        int64_t ii = FN(rne_)(fi), jj = FN(rne_)(fj), kk = FN(rne_)(fk);
        if (ii < 0 || ii >= dims[0] || jj < 0 || jj >= dims[1] || kk < 0 || kk >= dims[2]) continue;
        REAL len = (t1 - t0) * ray_len;
        size_t vi = ((size_t)ii * dims[1] + (size_t)jj) * dims[2] + (size_t)kk;
        if (mode == 0) acc = FMA_(data[vi], len, acc);
        else out[vi] += val * len;
    }
    if (mode == 0) out[r] = acc;
}

void FN(orc_fwd_planesort)(const int* dims, const REAL* vol, const REAL* Mi, const REAL* b, const REAL* src,
                           const REAL* dst, int64_t n_ray, REAL* out) {
    int K = dims[0] + dims[1] + dims[2] + 5;
#pragma omp parallel
    {
        REAL* t = (REAL*)malloc(sizeof(REAL) * (size_t)K);
#pragma omp for schedule(dynamic, 256)
        for (int64_t r = 0; r < n_ray; ++r) FN(planesort_ray_)(0, dims, vol, Mi, b, src, dst, r, t, out);
        free(t);
    }
}

void FN(orc_back_planesort)(const int* dims, const REAL* sino, const REAL* Mi, const REAL* b, const REAL* src,
                            const REAL* dst, int64_t n_ray, REAL* out) {
    int K = dims[0] + dims[1] + dims[2] + 5;
    REAL* t = (REAL*)malloc(sizeof(REAL) * (size_t)K);
    for (int64_t r = 0; r < n_ray; ++r) FN(planesort_ray_)(1, dims, sino, Mi, b, src, dst, r, t, out);
    free(t);
}

/* forward/back_project_2d_on_the_fly_kernel (ct_projector_2d.cu:246-413):
 * slab entry/exit, floor/ceil start pixel, incremental t_next += dt march,
 * segment (t_hit - t_cur)*|v| with |v| = hypot. */
static void FN(dda2_ray_)(int mode, const int* dims, const REAL* data, const REAL* Mi, const REAL* b,
                          const REAL* src, const REAL* dst, int64_t r, REAL* out) {
    int n_row = dims[0], n_col = dims[1];
    REAL sx = src[2 * r], sy = src[2 * r + 1], dx = dst[2 * r], dy = dst[2 * r + 1];
    REAL vx = dx - sx, vy = dy - sy;
    REAL ray_len = HYPOT_(vx, vy);
    if (ray_len < (REAL)1e-12) {
        if (mode == 0) out[r] = 0;
        return;
    }
    REAL sr, sc, dr, dc;
    FN(affine2_cuda_)(Mi, b, sx, sy, &sr, &sc);
    FN(affine2_cuda_)(Mi, b, dx, dy, &dr, &dc);
    REAL vr = dr - sr, vc = dc - sc;
    REAL inv_vr = (FABS_(vr) < (REAL)1e-12) ? (REAL)1e32 : (REAL)1.0 / vr;
    REAL inv_vc = (FABS_(vc) < (REAL)1e-12) ? (REAL)1e32 : (REAL)1.0 / vc;
    REAL t_r0 = ((REAL)-0.5 - sr) * inv_vr, t_r1 = ((REAL)n_row - (REAL)0.5 - sr) * inv_vr;
    REAL t_c0 = ((REAL)-0.5 - sc) * inv_vc, t_c1 = ((REAL)n_col - (REAL)0.5 - sc) * inv_vc;
    REAL t_enter = FMAX_(FMIN_(t_r0, t_r1), FMIN_(t_c0, t_c1));
    REAL t_exit = FMIN_(FMAX_(t_r0, t_r1), FMAX_(t_c0, t_c1));
    if (t_exit <= t_enter) {
        if (mode == 0) out[r] = 0;
        return;
    }
    t_enter = FMAX_(t_enter, (REAL)0);
    t_exit = FMIN_(t_exit, (REAL)1);
    REAL r_enter = FMA_(t_enter, vr, sr), c_enter = FMA_(t_enter, vc, sc);
    int64_t ri = (vr >= 0) ? (int64_t)FLOOR_(r_enter) : (int64_t)CEIL_(r_enter) - 1;
    int64_t ci = (vc >= 0) ? (int64_t)FLOOR_(c_enter) : (int64_t)CEIL_(c_enter) - 1;
    REAL t_next_r = (vr >= 0) ? FMA_(((REAL)ri + (REAL)0.5) - r_enter, inv_vr, t_enter)
                              : FMA_(((REAL)ri - (REAL)0.5) - r_enter, inv_vr, t_enter);
    REAL t_next_c = (vc >= 0) ? FMA_(((REAL)ci + (REAL)0.5) - c_enter, inv_vc, t_enter)
                              : FMA_(((REAL)ci - (REAL)0.5) - c_enter, inv_vc, t_enter);
    REAL dt_r = FABS_(inv_vr), dt_c = FABS_(inv_vc);
    REAL acc = 0, val = (mode == 1) ? data[r] : 0;
    REAL t_cur = t_enter;
    while (t_cur < t_exit) {
        int step_row = t_next_r < t_next_c;
        REAL t_hit = step_row ? t_next_r : t_next_c;
        t_hit = FMIN_(t_hit, t_exit);
        if (ri >= 0 && ri < n_row && ci >= 0 && ci < n_col) {
            REAL seg = (t_hit - t_cur) * ray_len;
            size_t idx = (size_t)ri * n_col + (size_t)ci;
            if (mode == 0) acc = FMA_(data[idx], seg, acc);
            else out[idx] += val * seg;
        }
        t_cur = t_hit;
        if (step_row) {
            t_next_r += dt_r;
            ri += (vr >= 0) ? 1 : -1;
        } else {
            t_next_c += dt_c;
            ci += (vc >= 0) ? 1 : -1;
        }
    }
    if (mode == 0) out[r] = acc;
}

void FN(orc_fwd_dda2)(const int* dims, const REAL* img, const REAL* Mi, const REAL* b, const REAL* src,
                      const REAL* dst, int64_t n_ray, REAL* out) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t r = 0; r < n_ray; ++r) FN(dda2_ray_)(0, dims, img, Mi, b, src, dst, r, out);
}

void FN(orc_back_dda2)(const int* dims, const REAL* sino, const REAL* Mi, const REAL* b, const REAL* src,
                       const REAL* dst, int64_t n_ray, REAL* out) {
    for (int64_t r = 0; r < n_ray; ++r) FN(dda2_ray_)(1, dims, sino, Mi, b, src, dst, r, out);
}

/* compress_tvals_3d_kernel (ct_projector_3d.cu:160-212): scale from the
 * world ray length, start = t[0] as stored (inf stays inf), inf entries
 * encode 0, k = roundf((t-start)*inv) (half away from zero), delta clamped
 * to [0, 32000], running sum unsigned. */
void FN(orc_compress_cuda)(const REAL* tvals, int64_t n_ray, int K, const REAL* src, const REAL* dst,
                           REAL voxel_diag_len, uint16_t* u16, REAL* starts, REAL* scales) {
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < n_ray; ++r) {
        REAL dx = dst[3 * r] - src[3 * r], dy = dst[3 * r + 1] - src[3 * r + 1], dz = dst[3 * r + 2] - src[3 * r + 2];
        REAL len = SQRT_(FMA_(dz, dz, FMA_(dx, dx, dy * dy)));
        len = FMAX_(len, (REAL)1e-6);
        REAL sc = (voxel_diag_len / (REAL)10000.0) / len;
        scales[r] = sc;
        const REAL* t = tvals + (size_t)r * K;
        uint16_t* o = u16 + (size_t)r * K;
        REAL start = t[0];
        starts[r] = start;
        o[0] = 0;
        REAL inv = (REAL)1.0 / sc;
        uint32_t prev = 0;
        for (int i = 1; i < K; ++i) {
            if (ISINF_(t[i])) {
                o[i] = 0;
                continue;
            }
            uint32_t cur = (uint32_t)ROUND_((t[i] - start) * inv);
            int diff = (int)cur - (int)prev;
            if (diff < 0) diff = 0;
            if (diff > 32000) diff = 32000;
            o[i] = (uint16_t)diff;
            prev += o[i];
        }
    }
}

/* forward/back_project_3d_compressed_kernel (ct_projector_3d.cu:99-157,
 * 215-269): t_i = start + (float)k_sum*scale (one fused multiply-add),
 * world-space segment, skipped when shorter than 1e-9. */
static void FN(comp_ray_)(int mode, const int* dims, const REAL* data, const uint16_t* u16, const REAL* starts,
                          const REAL* scales, int K, const REAL* Mi, const REAL* b, const REAL* src,
                          const REAL* dst, int64_t r, REAL* out) {
    REAL sx = src[3 * r], sy = src[3 * r + 1], sz = src[3 * r + 2];
    REAL vx = dst[3 * r] - sx, vy = dst[3 * r + 1] - sy, vz = dst[3 * r + 2] - sz;
    const uint16_t* q = u16 + (size_t)r * K;
    REAL start = starts[r], sc = scales[r];
    REAL acc = 0, val = (mode == 1) ? data[r] : 0;
    REAL t_prev = start;
    uint32_t ks = 0;
    for (int i = 0; i < K - 1; ++i) {
        ks += q[i + 1];
        REAL t1 = FMA_((REAL)ks, sc, start);
        REAL t0 = t_prev;
        t_prev = t1;
        REAL x0 = FMA_(t0, vx, sx), y0 = FMA_(t0, vy, sy), z0 = FMA_(t0, vz, sz);
        REAL x1 = FMA_(t1, vx, sx), y1 = FMA_(t1, vy, sy), z1 = FMA_(t1, vz, sz);
        REAL ddx = x1 - x0, ddy = y1 - y0, ddz = z1 - z0;
        REAL len = SQRT_(FMA_(ddz, ddz, FMA_(ddx, ddx, ddy * ddy)));
        if (len < (REAL)1e-9) continue;
        REAL mx = (REAL)0.5 * (x0 + x1), my = (REAL)0.5 * (y0 + y1), mz = (REAL)0.5 * (z0 + z1);
        REAL fi, fj, fk;
        FN(affine3_cuda_)(Mi, b, mx, my, mz, &fi, &fj, &fk);
        int64_t ii = FN(rne_)(fi), jj = FN(rne_)(fj), kk = FN(rne_)(fk);
        if (ii < 0 || ii >= dims[0] || jj < 0 || jj >= dims[1] || kk < 0 || kk >= dims[2]) continue;
        size_t vi = ((size_t)ii * dims[1] + (size_t)jj) * dims[2] + (size_t)kk;
        if (mode == 0) acc = FMA_(data[vi], len, acc);
        else out[vi] += val * len;
    }
    if (mode == 0) out[r] = acc;
}

void FN(orc_fwd_comp_cuda)(const int* dims, const REAL* vol, const uint16_t* u16, const REAL* starts,
                           const REAL* scales, int K, const REAL* Mi, const REAL* b, const REAL* src,
                           const REAL* dst, int64_t n_ray, REAL* out) {
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t r = 0; r < n_ray; ++r) FN(comp_ray_)(0, dims, vol, u16, starts, scales, K, Mi, b, src, dst, r, out);
}

void FN(orc_back_comp_cuda)(const int* dims, const REAL* sino, const uint16_t* u16, const REAL* starts,
                            const REAL* scales, int K, const REAL* Mi, const REAL* b, const REAL* src,
                            const REAL* dst, int64_t n_ray, REAL* out) {
    for (int64_t r = 0; r < n_ray; ++r) FN(comp_ray_)(1, dims, sino, u16, starts, scales, K, Mi, b, src, dst, r, out);
}

/* Number of in-volume segments per ray under the torch-path rules; used to
 * freeze the algorithmic byte count (sum over rays) of a workload. */
int64_t FN(orc_count_segments)(int ndim, const int* dims, const REAL* Mi, const REAL* b, const REAL* src,
                               const REAL* dst, int64_t n_ray) {
    int K = 0;
    for (int a = 0; a < ndim; ++a) K += dims[a] + 1;
    int64_t total = 0;
#pragma omp parallel reduction(+ : total)
    {
        REAL* t = (REAL*)malloc(sizeof(REAL) * (size_t)K);
#pragma omp for schedule(dynamic, 256)
        for (int64_t r = 0; r < n_ray; ++r) {
            REAL s[3], d[3], sw[3], vw[3];
            if (ndim == 3) {
                FN(affine3_torch_)(Mi, b, src[3 * r], src[3 * r + 1], src[3 * r + 2], &s[0], &s[1], &s[2]);
                FN(affine3_torch_)(Mi, b, dst[3 * r], dst[3 * r + 1], dst[3 * r + 2], &d[0], &d[1], &d[2]);
            } else {
                FN(affine2_torch_)(Mi, b, src[2 * r], src[2 * r + 1], &s[0], &s[1]);
                FN(affine2_torch_)(Mi, b, dst[2 * r], dst[2 * r + 1], &d[0], &d[1]);
            }
            FN(isect_row_)(ndim, dims, s, d, ndim == 2, 1, t);
            for (int a = 0; a < ndim; ++a) {
                sw[a] = src[ndim * r + a];
                vw[a] = dst[ndim * r + a] - sw[a];
            }
            for (int i = 0; i < K - 1; ++i) {
                REAL len;
                if (FN(seg_torch_)(ndim, dims, Mi, b, sw, vw, t[i], t[i + 1], &len) >= 0 && len > 0) total += 1;
            }
        }
        free(t);
    }
    return total;
}

#undef FN
#undef CAT
#undef CAT_
