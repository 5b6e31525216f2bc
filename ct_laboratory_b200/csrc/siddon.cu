// siddon.cu — on-the-fly Siddon forward projector and exact adjoint (2-D and
// 3-D) for sm_100a.
//
// The reference's on-the-fly 3-D kernel (src/ct_projector_3d.cu:902-1012)
// collects every plane hit of a ray into an 8 KB per-thread array, insertion-
// sorts it and then walks the sorted list.  The x-, y- and z-plane parameters
// of a ray are each already monotone, so their sorted union is a three-way
// merge.  This kernel walks that merge directly (a DDA): it keeps the next
// plane parameter of every axis in registers, repeatedly takes the smallest,
// and evaluates each plane's parameter on its own with the reference's
// formula t = (p - s) * (1/v), so the segment end points are the very floats
// the reference sorts.  Only segments inside the volume are visited (those
// outside map to out-of-range voxels, which the reference skips).  The voxel
// of a segment comes from which planes were crossed rather than from rounding
// the segment midpoint; the two agree except for segments of rounding-noise
// length, which contribute rounding-noise amounts.
//
// Memory behaviour: the volume is read through the read-only path (__ldg)
// and, at the benchmark size (256^3 fp32 = 64 MiB), stays resident in the
// 126 MB L2.  A CTA covers `tile_rows` detector rows x (threads/tile_rows)
// columns, with warp lanes along rows, so that for a cone-beam scan the 32
// lanes of a warp trace 32 vertically adjacent rays: they share the same x-y
// path and touch neighbouring k (fastest-varying) voxels, so a warp's gather
// hits a few 32-byte sectors instead of 32.  The adjoint scatters with
// red.global.add.f32 (atomicAdd with an unused result).
#include <type_traits>

#include "common.cuh"

namespace ctlab {

template <int NDIM>
using AffineT = typename std::conditional<NDIM == 3, Affine3, Affine2>::type;

template <int NDIM>
struct GridDims {
    int n[NDIM];
    int stride[NDIM];
};

// One Siddon traversal.  ADJ=false: returns sum of in[voxel]*len.
// ADJ=true: scatters y*len into out[voxel].
template <int NDIM, bool ADJ>
__device__ __forceinline__ float traverse(const float* __restrict__ vol, float* __restrict__ out, float y,
                                          const float* sw, const float* dw, const GridDims<NDIM>& G,
                                          const AffineT<NDIM>& A, unsigned nvox) {
    // World direction and length: ct_projector_3d.cu:941-942 (fused as nvcc
    // contracts vx*vx + vy*vy + vz*vz).
    float vw[NDIM];
#pragma unroll
    for (int a = 0; a < NDIM; ++a) vw[a] = __fsub_rn(dw[a], sw[a]);
    float len2;
    if constexpr (NDIM == 3) len2 = sumsq3(vw[0], vw[1], vw[2]);
    else len2 = sumsq2(vw[0], vw[1]);
    const float ray_len = sqrtf(len2);
    if (!(ray_len >= 1e-12f)) return 0.f;

    // Endpoints in index space.
    float s[NDIM], d[NDIM];
    if constexpr (NDIM == 3) {
        world_to_index3(A, sw[0], sw[1], sw[2], s[0], s[1], s[2]);
        world_to_index3(A, dw[0], dw[1], dw[2], d[0], d[1], d[2]);
    } else {
        world_to_index2(A, sw[0], sw[1], s[0], s[1]);
        world_to_index2(A, dw[0], dw[1], d[0], d[1]);
    }

    float inv[NDIM], tn[NDIM], pn[NDIM], ps[NDIM];
    int ds[NDIM];
    float t_enter = 0.f, t_exit = 1.f;
    int idx = 0;
    bool live = true;
#pragma unroll
    for (int a = 0; a < NDIM; ++a) {
        const float va = __fsub_rn(d[a], s[a]);
        const float nf = (float)G.n[a];
        live = live && isfinite(s[a]) && isfinite(va);
        if (fabsf(va) > 1e-12f) {
            // collect_hits (ct_projector_3d.cu:865-870): inv = 1/v.
            inv[a] = __frcp_rn(va);
            const float lo = va > 0.f ? -0.5f : nf - 0.5f;
            const float hi = va > 0.f ? nf - 0.5f : -0.5f;
            t_enter = fmaxf(t_enter, plane_t(lo, s[a], inv[a]));
            t_exit = fminf(t_exit, plane_t(hi, s[a], inv[a]));
            ps[a] = va > 0.f ? 1.f : -1.f;
            ds[a] = va > 0.f ? G.stride[a] : -G.stride[a];
        } else {
            // No planes of this axis are hit: the ray keeps one index along
            // it, the rounded coordinate (the reference rounds the midpoint).
            inv[a] = 0.f;
            const int i = __float2int_rn(s[a]);
            live = live && (i >= 0) && (i < G.n[a]);
            idx += i * G.stride[a];
            tn[a] = __int_as_float(0x7f800000);  // +inf
            pn[a] = 0.f;
            ps[a] = 0.f;
            ds[a] = 0;
        }
    }
    live = live && (t_enter < t_exit);
    if (!live) return 0.f;

    // Starting voxel: for each crossing axis, the slab whose behind-plane
    // parameter is <= t_enter and whose ahead-plane parameter is > t_enter,
    // found from an estimate and fixed up with the exact plane formula.
#pragma unroll
    for (int a = 0; a < NDIM; ++a) {
        if (inv[a] == 0.f) continue;
        const float va = __fsub_rn(d[a], s[a]);
        const float c = __fmaf_rn(t_enter, va, s[a]);
        int i = __float2int_rd(c + 0.5f);
        if (va > 0.f) {
#pragma unroll 1
            for (int k = 0; k < 4 && plane_t((float)i + 0.5f, s[a], inv[a]) <= t_enter; ++k) ++i;
#pragma unroll 1
            for (int k = 0; k < 4 && plane_t((float)i - 0.5f, s[a], inv[a]) > t_enter; ++k) --i;
        } else {
#pragma unroll 1
            for (int k = 0; k < 4 && plane_t((float)i - 0.5f, s[a], inv[a]) <= t_enter; ++k) --i;
#pragma unroll 1
            for (int k = 0; k < 4 && plane_t((float)i + 0.5f, s[a], inv[a]) > t_enter; ++k) ++i;
        }
        i = min(max(i, 0), G.n[a] - 1);
        idx += i * G.stride[a];
        pn[a] = (float)i + 0.5f * ps[a];
        tn[a] = plane_t(pn[a], s[a], inv[a]);
    }

    // The merge walk.  Every plane is crossed at most once, which bounds the
    // loop even for non-finite input.
    int max_it = 3;
#pragma unroll
    for (int a = 0; a < NDIM; ++a) max_it += G.n[a];
    float acc = 0.f;
    float t_cur = t_enter;
#pragma unroll 1
    for (int it = 0; it < max_it; ++it) {
        float tm = tn[0];
#pragma unroll
        for (int a = 1; a < NDIM; ++a) tm = fminf(tm, tn[a]);
        const bool fin = !(tm < t_exit);
        const float t1 = fin ? t_exit : tm;
        if (t1 > t_cur && (unsigned)idx < nvox) {
            // Segment length (t1 - t0) * |v| (ct_projector_3d.cu:998).
            const float seg = __fmul_rn(__fsub_rn(t1, t_cur), ray_len);
            if constexpr (ADJ) {
                atomicAdd(out + idx, __fmul_rn(y, seg));
            } else {
                acc = __fmaf_rn(__ldg(vol + idx), seg, acc);
            }
        }
        if (fin) break;
        t_cur = t1;
        // Advance the axis that owns tm (x before y before z on ties, the
        // order in which equal values leave the reference's sort).
        if (tn[0] == tm) {
            idx += ds[0];
            pn[0] += ps[0];
            tn[0] = plane_t(pn[0], s[0], inv[0]);
        } else if (NDIM == 2 || tn[1] == tm) {
            idx += ds[1];
            pn[1] += ps[1];
            tn[1] = plane_t(pn[1], s[1], inv[1]);
        } else {
            idx += ds[NDIM - 1];
            pn[NDIM - 1] += ps[NDIM - 1];
            tn[NDIM - 1] = plane_t(pn[NDIM - 1], s[NDIM - 1], inv[NDIM - 1]);
        }
    }
    return acc;
}

template <int NDIM, bool ADJ>
__global__ void __launch_bounds__(256) siddon_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                     const float* __restrict__ src, const float* __restrict__ dst,
                                                     int64_t n_ray, const float* __restrict__ M_inv,
                                                     const float* __restrict__ bvec, GridDims<NDIM> G,
                                                     int64_t nvox, Tiling T) {
    const int64_t r = tile_ray(T);
    if (r < 0) return;
    const int64_t bi = blockIdx.y;
    AffineT<NDIM> aff;
    if constexpr (NDIM == 3) {
        aff = load_affine3(M_inv, bvec);
    } else {
        aff = load_affine2(M_inv, bvec);
    }
    float sw[NDIM], dw[NDIM];
#pragma unroll
    for (int a = 0; a < NDIM; ++a) {
        sw[a] = __ldg(src + r * NDIM + a);
        dw[a] = __ldg(dst + r * NDIM + a);
    }
    if constexpr (ADJ) {
        const float y = __ldg(in + bi * n_ray + r);
        if (y == 0.f) return;  // contributes exactly nothing
        traverse<NDIM, true>(nullptr, out + bi * nvox, y, sw, dw, G, aff, (unsigned)nvox);
    } else {
        out[bi * n_ray + r] = traverse<NDIM, false>(in + bi * nvox, nullptr, 0.f, sw, dw, G, aff, (unsigned)nvox);
    }
}

// ----------------------------------------------------------------------------
// host side
// ----------------------------------------------------------------------------

template <int NDIM, bool ADJ>
static int launch_siddon(const char* what, const float* in, float* out, int64_t batch, const int64_t* dims,
                         const float* src, const float* dst, int64_t n_ray, const float* M_inv, const float* b,
                         int accumulate, const ctlab_ray_tiling* tiling, void* stream) {
    CTLAB_REQUIRE(batch >= 1 && batch <= 65535, "%s: batch must be in [1, 65535], got %lld", what, (long long)batch);
    CTLAB_REQUIRE(n_ray >= 0, "%s: n_ray must be >= 0", what);
    GridDims<NDIM> G;
    int64_t nvox = 1;
    for (int a = 0; a < NDIM; ++a) {
        CTLAB_REQUIRE(dims[a] >= 1 && dims[a] < (1 << 24), "%s: grid dimension %d out of range (%lld)", what, a,
                      (long long)dims[a]);
        nvox *= dims[a];
    }
    CTLAB_REQUIRE(nvox < (1LL << 31), "%s: a volume of %lld voxels exceeds 2^31", what, (long long)nvox);
    int64_t st = 1;
    for (int a = NDIM - 1; a >= 0; --a) {
        G.n[a] = (int)dims[a];
        G.stride[a] = (int)st;
        st *= dims[a];
    }
    CTLAB_REQUIRE(in && out && M_inv && b, "%s: null data pointer", what);
    CTLAB_REQUIRE(n_ray == 0 || (src && dst), "%s: null src/dst", what);
    cudaStream_t s = as_stream(stream);
    if (ADJ && !accumulate) {
        CTLAB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float) * (size_t)(batch * nvox), s));
    }
    if (n_ray == 0) return CTLAB_OK;
    Tiling T;
    int rc = resolve_tiling(tiling, n_ray, T);
    if (rc) return rc;
    CTLAB_REQUIRE(T.tile_rows * T.tile_cols <= 256, "%s: block_threads must be <= 256", what);
    CTLAB_REQUIRE(T.n_blocks <= kMaxGrid, "%s: too many rays for one launch", what);
    dim3 grid((unsigned)T.n_blocks, (unsigned)batch);
    siddon_kernel<NDIM, ADJ><<<grid, T.tile_rows * T.tile_cols, 0, s>>>(in, out, src, dst, n_ray, M_inv, b, G,
                                                                        nvox, T);
    return launch_status(what);
}

}  // namespace ctlab

using namespace ctlab;

extern "C" int ctlab_forward_project_3d_on_the_fly_ex(const float* volume, int64_t batch, int64_t n_x, int64_t n_y,
                                                      int64_t n_z, const float* src, const float* dst,
                                                      int64_t n_ray, const float* M_inv, const float* b, float* out,
                                                      const ctlab_ray_tiling* tiling, void* stream) {
    clear_error();
    const int64_t dims[3] = {n_x, n_y, n_z};
    return launch_siddon<3, false>("forward_project_3d_on_the_fly", volume, out, batch, dims, src, dst, n_ray,
                                   M_inv, b, 0, tiling, stream);
}

extern "C" int ctlab_back_project_3d_on_the_fly_ex(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                                   const float* dst, const float* M_inv, const float* b, int64_t n_x,
                                                   int64_t n_y, int64_t n_z, float* out, int accumulate,
                                                   const ctlab_ray_tiling* tiling, void* stream) {
    clear_error();
    const int64_t dims[3] = {n_x, n_y, n_z};
    return launch_siddon<3, true>("back_project_3d_on_the_fly", sino, out, batch, dims, src, dst, n_ray, M_inv, b,
                                  accumulate, tiling, stream);
}

extern "C" int ctlab_forward_project_3d_on_the_fly(const float* volume, int64_t batch, int64_t n_x, int64_t n_y,
                                                   int64_t n_z, const float* src, const float* dst, int64_t n_ray,
                                                   const float* M_inv, const float* b, float* out, void* stream) {
    return ctlab_forward_project_3d_on_the_fly_ex(volume, batch, n_x, n_y, n_z, src, dst, n_ray, M_inv, b, out,
                                                  nullptr, stream);
}

extern "C" int ctlab_back_project_3d_on_the_fly(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                                const float* dst, const float* M_inv, const float* b, int64_t n_x,
                                                int64_t n_y, int64_t n_z, float* out, int accumulate, void* stream) {
    return ctlab_back_project_3d_on_the_fly_ex(sino, batch, n_ray, src, dst, M_inv, b, n_x, n_y, n_z, out,
                                               accumulate, nullptr, stream);
}

extern "C" int ctlab_forward_project_2d_siddon(const float* image, int64_t batch, int64_t n_row, int64_t n_col,
                                               const float* src, const float* dst, int64_t n_ray,
                                               const float* M_inv, const float* b, float* out,
                                               const ctlab_ray_tiling* tiling, void* stream) {
    clear_error();
    const int64_t dims[2] = {n_row, n_col};
    return launch_siddon<2, false>("forward_project_2d_siddon", image, out, batch, dims, src, dst, n_ray, M_inv, b,
                                   0, tiling, stream);
}

extern "C" int ctlab_back_project_2d_siddon(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                            const float* dst, const float* M_inv, const float* b, int64_t n_row,
                                            int64_t n_col, float* out, int accumulate, const ctlab_ray_tiling* tiling,
                                            void* stream) {
    clear_error();
    const int64_t dims[2] = {n_row, n_col};
    return launch_siddon<2, true>("back_project_2d_siddon", sino, out, batch, dims, src, dst, n_ray, M_inv, b,
                                  accumulate, tiling, stream);
}
