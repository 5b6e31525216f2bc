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

// Round half to even to int without a conversion instruction: adding
// 1.5*2^23 leaves the rounded integer in the low mantissa bits (exact for
// |x| < 2^22); outside that range (and for NaN / inf) the result is an
// integer >= 2^22 or negative, which every grid bound check (n <= 2^22)
// rejects.
__device__ __forceinline__ int rne_int(float x) {
    return __float_as_int(__fadd_rn(x, 12582912.0f)) - 0x4B400000;
}

// Voxel of a segment [t0, t1] under the reference's rule: the world-space
// midpoint s + t_mid*v mapped to index space and rounded half to even
// (ct_projector_3d.cu:982-996).  Returns the flat index or -1 (outside).
template <int NDIM>
__device__ __forceinline__ int midpoint_voxel(const AffineT<NDIM>& A, const float* sw, const float* vw, float t0,
                                              float t1, const GridDims<NDIM>& G) {
    const float tm = __fmul_rn(0.5f, __fadd_rn(t0, t1));
    float m[NDIM], f[NDIM];
#pragma unroll
    for (int a = 0; a < NDIM; ++a) m[a] = __fmaf_rn(tm, vw[a], sw[a]);
    if constexpr (NDIM == 3) world_to_index3(A, m[0], m[1], m[2], f[0], f[1], f[2]);
    else world_to_index2(A, m[0], m[1], f[0], f[1]);
    int flat = 0;
    bool ok = true;
#pragma unroll
    for (int a = 0; a < NDIM; ++a) {
        const int i = rne_int(f[a]);
        ok = ok && (unsigned)i < (unsigned)G.n[a];
        flat += i * G.stride[a];
    }
    return ok ? flat : -1;
}

// One Siddon traversal.  ADJ=false: returns sum of in[voxel]*len.
// ADJ=true: scatters y*len into out[voxel].  MID selects the voxel of each
// segment: true = the reference's rounded world midpoint, false = the voxel
// between the two crossings that bound the segment (exact topology).
template <int NDIM, bool ADJ, bool MID>
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

    // The merge walk.  Each step ends the current segment at the nearest
    // next plane (or at t_exit) and then steps every axis whose next plane
    // lies exactly there: equal plane parameters of two axes only ever bound
    // a zero-length segment, which the reference skips and which would add
    // nothing here, so stepping them together gives the same segments.  The
    // steps are predicated, not branched, so the lanes of a warp never
    // diverge inside the walk.
    //
    // The voxel index never leaves the grid: an axis is stepped across its
    // last plane only when that plane's parameter (>= t_exit, which is the
    // minimum over the axes' exit planes) is below t_exit, which cannot
    // happen.  Every plane is crossed at most once, which bounds the loop
    // even for non-finite input.
    int max_it = 3;
#pragma unroll
    for (int a = 0; a < NDIM; ++a) max_it += G.n[a];
    (void)nvox;
    float t_cur = t_enter;
    if constexpr (!ADJ) {
        // Forward: four steps, then their four gathers back to back (four
        // loads in flight per lane), accumulated in walk order; zero-length
        // segments (ties, and the padding after the exit) are not added.
        float acc = 0.f;
        bool done = false;
#pragma unroll 1
        for (int it = 0; it < max_it && !done; it += 4) {
            int vq[4];
            float sq[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float tm = tn[0];
#pragma unroll
                for (int a = 1; a < NDIM; ++a) tm = fminf(tm, tn[a]);
                const float t1 = fminf(tm, t_exit);
                float seg = done ? 0.f : __fmul_rn(__fsub_rn(t1, t_cur), ray_len);
                int v = idx;
                if constexpr (MID) {
                    const int m = midpoint_voxel<NDIM>(A, sw, vw, t_cur, t1, G);
                    v = m < 0 ? 0 : m;
                    seg = m < 0 ? 0.f : seg;
                }
                vq[q] = v;
                sq[q] = seg;
                done = done || !(tm < t_exit);
                t_cur = t1;
#pragma unroll
                for (int a = 0; a < NDIM; ++a) {
                    if (!done && tn[a] == tm) {
                        idx += ds[a];
                        pn[a] += ps[a];
                        tn[a] = plane_t(pn[a], s[a], inv[a]);
                    }
                }
            }
            float vv[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) vv[q] = __ldg(vol + vq[q]);
#pragma unroll
            for (int q = 0; q < 4; ++q) acc = sq[q] > 0.f ? __fmaf_rn(vv[q], sq[q], acc) : acc;
        }
        return acc;
    } else {
#pragma unroll 1
        for (int it = 0; it < max_it; ++it) {
            float tm = tn[0];
#pragma unroll
            for (int a = 1; a < NDIM; ++a) tm = fminf(tm, tn[a]);
            const float t1 = fminf(tm, t_exit);
            // Segment length (t1 - t0) * |v| (ct_projector_3d.cu:998).
            const float seg = __fmul_rn(__fsub_rn(t1, t_cur), ray_len);
            const int v = MID ? midpoint_voxel<NDIM>(A, sw, vw, t_cur, t1, G) : idx;
            if (seg > 0.f && v >= 0) atomicAdd(out + v, __fmul_rn(y, seg));
            if (!(tm < t_exit)) break;
            t_cur = t1;
#pragma unroll
            for (int a = 0; a < NDIM; ++a) {
                if (tn[a] == tm) {
                    idx += ds[a];
                    pn[a] += ps[a];
                    tn[a] = plane_t(pn[a], s[a], inv[a]);
                }
            }
        }
        return 0.f;
    }
}

template <int NDIM, bool ADJ, bool MID>
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
        traverse<NDIM, true, MID>(nullptr, out + bi * nvox, y, sw, dw, G, aff, (unsigned)nvox);
    } else {
        out[bi * n_ray + r] =
            traverse<NDIM, false, MID>(in + bi * nvox, nullptr, 0.f, sw, dw, G, aff, (unsigned)nvox);
    }
}

// ----------------------------------------------------------------------------
// Column-coherent 3-D traversal.
//
// When the 32 lanes of a warp trace rays that share their x-y line (same
// source, same detector column of a detector whose columns run along z: the
// cone-beam and StaticCT rings), every x- and y-plane parameter is bitwise
// the same for all lanes; only the z planes differ.  The per-lane merge walk
// above then diverges at almost every step (some lane always takes a z step)
// and the lanes drift apart along the x-y path.  Here the warp walks the x-y
// cells together (warp-uniform state) and each lane splits a cell only at its
// own z planes.  The segment end points are the same floats and they are
// accumulated in the same order as in traverse(), so results are bitwise those
// of the general walk; the gathers (forward) and reductions (adjoint) of a
// warp now address one voxel column (i, j, k..k+~32) at a time.
// A warp whose lanes do not share the x-y line falls back to traverse().
// ----------------------------------------------------------------------------
constexpr unsigned kFullMask = 0xffffffffu;

struct LaneRay {
    float s[3], inv[3], ray_len, t_enter, t_exit;
    bool live;
};

// Per-lane set-up, identical arithmetic to the start of traverse<3>.
__device__ __forceinline__ void lane_setup(LaneRay& R, const float* sw, const float* dw, const GridDims<3>& G,
                                           const Affine3& A, int& fixed_idx, bool& z_parallel) {
    float vw[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) vw[a] = __fsub_rn(dw[a], sw[a]);
    R.ray_len = sqrtf(sumsq3(vw[0], vw[1], vw[2]));
    R.live = R.ray_len >= 1e-12f;
    float d[3];
    world_to_index3(A, sw[0], sw[1], sw[2], R.s[0], R.s[1], R.s[2]);
    world_to_index3(A, dw[0], dw[1], dw[2], d[0], d[1], d[2]);
    R.t_enter = 0.f;
    R.t_exit = 1.f;
    fixed_idx = 0;
    z_parallel = false;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float va = __fsub_rn(d[a], R.s[a]);
        const float nf = (float)G.n[a];
        R.live = R.live && isfinite(R.s[a]) && isfinite(va);
        if (fabsf(va) > 1e-12f) {
            R.inv[a] = __frcp_rn(va);
            const float lo = va > 0.f ? -0.5f : nf - 0.5f;
            const float hi = va > 0.f ? nf - 0.5f : -0.5f;
            R.t_enter = fmaxf(R.t_enter, plane_t(lo, R.s[a], R.inv[a]));
            R.t_exit = fminf(R.t_exit, plane_t(hi, R.s[a], R.inv[a]));
        } else {
            R.inv[a] = 0.f;
            const int i = __float2int_rn(R.s[a]);
            R.live = R.live && (i >= 0) && (i < G.n[a]);
            fixed_idx += i * G.stride[a];
            if (a == 2) z_parallel = true;
        }
    }
    R.live = R.live && (R.t_enter < R.t_exit);
}

// Slab index of a crossing axis at time t: behind-plane parameter <= t and
// ahead-plane parameter > t (the fix-up of traverse), clamped into the grid.
__device__ __forceinline__ int slab_at(float t, float s, float inv, int n) {
    const float va_sign = inv;  // same sign as v
    const float c = __fmaf_rn(t, __frcp_rn(inv), s);
    int i = __float2int_rd(c + 0.5f);
    if (va_sign > 0.f) {
#pragma unroll 1
        for (int k = 0; k < 4 && plane_t((float)i + 0.5f, s, inv) <= t; ++k) ++i;
#pragma unroll 1
        for (int k = 0; k < 4 && plane_t((float)i - 0.5f, s, inv) > t; ++k) --i;
    } else {
#pragma unroll 1
        for (int k = 0; k < 4 && plane_t((float)i - 0.5f, s, inv) <= t; ++k) --i;
#pragma unroll 1
        for (int k = 0; k < 4 && plane_t((float)i + 0.5f, s, inv) > t; ++k) ++i;
    }
    return min(max(i, 0), n - 1);
}

template <bool ADJ, bool MID>
__global__ void __launch_bounds__(256) siddon3d_column_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                              const float* __restrict__ src,
                                                              const float* __restrict__ dst, int64_t n_ray,
                                                              const float* __restrict__ M_inv,
                                                              const float* __restrict__ bvec, GridDims<3> G,
                                                              int64_t nvox, Tiling T) {
    const int64_t r = tile_ray(T);
    const int64_t bi = blockIdx.y;
    const Affine3 A = load_affine3(M_inv, bvec);
    float sw[3] = {0.f, 0.f, 0.f}, dw[3] = {0.f, 0.f, 0.f};
    if (r >= 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            sw[a] = __ldg(src + r * 3 + a);
            dw[a] = __ldg(dst + r * 3 + a);
        }
    }
    float y = 0.f;
    if constexpr (ADJ) {
        if (r >= 0) y = __ldg(in + bi * n_ray + r);
    }
    LaneRay R;
    int fixed_idx;
    bool z_par;
    lane_setup(R, sw, dw, G, A, fixed_idx, z_par);
    R.live = R.live && (r >= 0) && (!ADJ || y != 0.f);

    // Do the live lanes share their x-y line?  (Inactive lanes do not vote.)
    const unsigned live_mask = __ballot_sync(kFullMask, R.live);
    if (live_mask == 0u) {
        if (!ADJ && r >= 0) out[bi * n_ray + r] = 0.f;
        return;
    }
    const int leader = __ffs(live_mask) - 1;
    const float s0 = __shfl_sync(kFullMask, R.s[0], leader), s1 = __shfl_sync(kFullMask, R.s[1], leader);
    const float i0 = __shfl_sync(kFullMask, R.inv[0], leader), i1 = __shfl_sync(kFullMask, R.inv[1], leader);
    const bool same = !R.live || (__float_as_uint(R.s[0]) == __float_as_uint(s0) &&
                                  __float_as_uint(R.s[1]) == __float_as_uint(s1) &&
                                  __float_as_uint(R.inv[0]) == __float_as_uint(i0) &&
                                  __float_as_uint(R.inv[1]) == __float_as_uint(i1));
    if (!__all_sync(kFullMask, same)) {
        // lanes do not share the x-y line: per-lane merge walk
        if (r < 0) return;
        if constexpr (ADJ) {
            if (R.live) traverse<3, true, MID>(nullptr, out + bi * nvox, y, sw, dw, G, A, (unsigned)nvox);
        } else {
            out[bi * n_ray + r] =
                R.live ? traverse<3, false, MID>(in + bi * nvox, nullptr, 0.f, sw, dw, G, A, (unsigned)nvox) : 0.f;
        }
        return;
    }

    // ---- warp-uniform x-y walk (every lane holds the same values) ----------
    const float nx = (float)G.n[0], ny = (float)G.n[1];
    float txy_in = 0.f, txy_out = 1.f;
    bool xy_ok = true;
    int col = 0;  // flat index of the current (i, j) column, k = 0
    float tnx = __int_as_float(0x7f800000), tny = tnx, pnx = 0.f, pny = 0.f, psx = 0.f, psy = 0.f;
    int dsx = 0, dsy = 0;
    if (i0 != 0.f) {
        const bool pos = i0 > 0.f;
        txy_in = fmaxf(txy_in, plane_t(pos ? -0.5f : nx - 0.5f, s0, i0));
        txy_out = fminf(txy_out, plane_t(pos ? nx - 0.5f : -0.5f, s0, i0));
    } else {
        const int i = __float2int_rn(s0);
        xy_ok = xy_ok && i >= 0 && i < G.n[0];
        col += i * G.stride[0];
    }
    if (i1 != 0.f) {
        const bool pos = i1 > 0.f;
        txy_in = fmaxf(txy_in, plane_t(pos ? -0.5f : ny - 0.5f, s1, i1));
        txy_out = fminf(txy_out, plane_t(pos ? ny - 0.5f : -0.5f, s1, i1));
    } else {
        const int j = __float2int_rn(s1);
        xy_ok = xy_ok && j >= 0 && j < G.n[1];
        col += j * G.stride[1];
    }
    // Every live lane's own interval [t_enter, t_exit] lies inside
    // [txy_in, txy_out]; walk only the union of the lanes' intervals.
    float te = R.live ? R.t_enter : __int_as_float(0x7f800000);
    float tx = R.live ? R.t_exit : __int_as_float(0xff800000);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        te = fminf(te, __shfl_xor_sync(kFullMask, te, o));
        tx = fmaxf(tx, __shfl_xor_sync(kFullMask, tx, o));
    }
    txy_in = fmaxf(txy_in, te);
    txy_out = fminf(txy_out, tx);
    xy_ok = xy_ok && txy_in < txy_out;
    if (i0 != 0.f) {
        const int i = slab_at(txy_in, s0, i0, G.n[0]);
        col += i * G.stride[0];
        psx = i0 > 0.f ? 1.f : -1.f;
        dsx = i0 > 0.f ? G.stride[0] : -G.stride[0];
        pnx = (float)i + 0.5f * psx;
        tnx = plane_t(pnx, s0, i0);
    }
    if (i1 != 0.f) {
        const int j = slab_at(txy_in, s1, i1, G.n[1]);
        col += j * G.stride[1];
        psy = i1 > 0.f ? 1.f : -1.f;
        dsy = i1 > 0.f ? G.stride[1] : -G.stride[1];
        pny = (float)j + 0.5f * psy;
        tny = plane_t(pny, s1, i1);
    }

    // ---- per-lane z state, started at the lane's own entry ----------------
    float tnz = __int_as_float(0x7f800000), pnz = 0.f, psz = 0.f;
    int kz = 0, dsz = 0;
    if (R.live) {
        if (!z_par) {
            const int k = slab_at(R.t_enter, R.s[2], R.inv[2], G.n[2]);
            kz = k * G.stride[2];
            psz = R.inv[2] > 0.f ? 1.f : -1.f;
            dsz = R.inv[2] > 0.f ? G.stride[2] : -G.stride[2];
            pnz = (float)k + 0.5f * psz;
            tnz = plane_t(pnz, R.s[2], R.inv[2]);
        } else {
            kz = fixed_idx - (fixed_idx / G.stride[1]) * G.stride[1];  // the k part of the fixed index
        }
    }
    const float* vol = in + bi * nvox;
    float* vout = out + bi * nvox;
    float acc = 0.f;
    const int max_xy = G.n[0] + G.n[1] + 3;
    const int max_z = G.n[2] + 3;
    int zsteps = 0;
    float ta = txy_in;
#pragma unroll 1
    for (int it = 0; it < max_xy && xy_ok; ++it) {
        const float tm = fminf(tnx, tny);
        const bool last = !(tm < txy_out);
        const float tb = last ? txy_out : tm;
        if (R.live) {
            float t0 = fmaxf(ta, R.t_enter);
            const float tend = fminf(tb, R.t_exit);
#pragma unroll 1
            while (t0 < tend && zsteps < max_z) {
                if (tnz <= t0) {  // a z plane at or before t0 has been crossed
                    kz += dsz;
                    pnz += psz;
                    tnz = plane_t(pnz, R.s[2], R.inv[2]);
                    ++zsteps;
                    continue;
                }
                const float t1 = fminf(tend, tnz);
                int idx = col + kz;
                if constexpr (MID) {
                    float vw[3];
#pragma unroll
                    for (int a = 0; a < 3; ++a) vw[a] = __fsub_rn(dw[a], sw[a]);
                    idx = midpoint_voxel<3>(A, sw, vw, t0, t1, G);
                }
                if ((unsigned)idx < (unsigned)nvox) {
                    const float seg = __fmul_rn(__fsub_rn(t1, t0), R.ray_len);
                    if constexpr (ADJ) atomicAdd(vout + idx, __fmul_rn(y, seg));
                    else acc = __fmaf_rn(__ldg(vol + idx), seg, acc);
                }
                t0 = t1;
            }
        }
        if (last) break;
        ta = tb;
        if (tnx == tm) {
            col += dsx;
            pnx += psx;
            tnx = plane_t(pnx, s0, i0);
        } else {
            col += dsy;
            pny += psy;
            tny = plane_t(pny, s1, i1);
        }
    }
    if constexpr (!ADJ) {
        if (r >= 0) out[bi * n_ray + r] = acc;
    }
}

// ----------------------------------------------------------------------------
// host side
// ----------------------------------------------------------------------------

template <int NDIM, bool ADJ>
static int launch_siddon(const char* what, const float* in, float* out, int64_t batch, const int64_t* dims,
                         const float* src, const float* dst, int64_t n_ray, const float* M_inv, const float* b,
                         int accumulate, const ctlab_ray_opts* tiling, void* stream) {
    CTLAB_REQUIRE(batch >= 1 && batch <= 65535, "%s: batch must be in [1, 65535], got %lld", what, (long long)batch);
    CTLAB_REQUIRE(n_ray >= 0, "%s: n_ray must be >= 0", what);
    GridDims<NDIM> G;
    int64_t nvox = 1;
    for (int a = 0; a < NDIM; ++a) {
        CTLAB_REQUIRE(dims[a] >= 1 && dims[a] <= (1 << 22), "%s: grid dimension %d out of range (%lld)", what, a,
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
    // Buffers of zero elements may be NULL (torch gives empty tensors a null
    // data pointer); the volume side is never empty.
    const bool vol_ok = ADJ ? (out != nullptr) : (in != nullptr);
    const bool ray_ok = n_ray == 0 || (src && dst && (ADJ ? in != nullptr : out != nullptr));
    CTLAB_REQUIRE(vol_ok && M_inv && b, "%s: null data pointer", what);
    CTLAB_REQUIRE(ray_ok, "%s: null src/dst/sinogram", what);
    cudaStream_t s = as_stream(stream);
    if (ADJ && !accumulate) {
        CTLAB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float) * (size_t)(batch * nvox), s));
    }
    if (n_ray == 0) return CTLAB_OK;
    Tiling T;
    int rc = resolve_tiling(tiling, n_ray, T);
    if (rc) return rc;
    CTLAB_REQUIRE(T.n_blocks <= kMaxGrid, "%s: too many rays for one launch", what);
    dim3 grid((unsigned)T.n_blocks, (unsigned)batch);
    const int threads = T.tile_rows * T.tile_cols;
    const bool mid = tiling == nullptr || tiling->voxel_rule == CTLAB_VOXEL_MIDPOINT;
    const bool flat = tiling == nullptr || tiling->n_view == 0;
    const int walk = tiling == nullptr ? CTLAB_WALK_AUTO : tiling->walk;
    if constexpr (NDIM == 3) {
        // Detector-row tilings (a warp = 32 rows of one column) may take the
        // column-coherent walk; it checks per warp that the lanes share their
        // x-y line and otherwise runs the per-lane walk.
        if (!flat && T.tile_rows % 32 == 0 && walk == CTLAB_WALK_COLUMN) {
            if (mid)
                siddon3d_column_kernel<ADJ, true>
                    <<<grid, threads, 0, s>>>(in, out, src, dst, n_ray, M_inv, b, G, nvox, T);
            else
                siddon3d_column_kernel<ADJ, false>
                    <<<grid, threads, 0, s>>>(in, out, src, dst, n_ray, M_inv, b, G, nvox, T);
            return launch_status(what);
        }
    }
    if (mid)
        siddon_kernel<NDIM, ADJ, true><<<grid, threads, 0, s>>>(in, out, src, dst, n_ray, M_inv, b, G, nvox, T);
    else
        siddon_kernel<NDIM, ADJ, false><<<grid, threads, 0, s>>>(in, out, src, dst, n_ray, M_inv, b, G, nvox, T);
    return launch_status(what);
}

}  // namespace ctlab

using namespace ctlab;

extern "C" int ctlab_forward_project_3d_on_the_fly_ex(const float* volume, int64_t batch, int64_t n_x, int64_t n_y,
                                                      int64_t n_z, const float* src, const float* dst,
                                                      int64_t n_ray, const float* M_inv, const float* b, float* out,
                                                      const ctlab_ray_opts* tiling, void* stream) {
    clear_error();
    const int64_t dims[3] = {n_x, n_y, n_z};
    return launch_siddon<3, false>("forward_project_3d_on_the_fly", volume, out, batch, dims, src, dst, n_ray,
                                   M_inv, b, 0, tiling, stream);
}

extern "C" int ctlab_back_project_3d_on_the_fly_ex(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                                   const float* dst, const float* M_inv, const float* b, int64_t n_x,
                                                   int64_t n_y, int64_t n_z, float* out, int accumulate,
                                                   const ctlab_ray_opts* tiling, void* stream) {
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
                                               const ctlab_ray_opts* tiling, void* stream) {
    clear_error();
    const int64_t dims[2] = {n_row, n_col};
    return launch_siddon<2, false>("forward_project_2d_siddon", image, out, batch, dims, src, dst, n_ray, M_inv, b,
                                   0, tiling, stream);
}

extern "C" int ctlab_back_project_2d_siddon(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                            const float* dst, const float* M_inv, const float* b, int64_t n_row,
                                            int64_t n_col, float* out, int accumulate, const ctlab_ray_opts* tiling,
                                            void* stream) {
    clear_error();
    const int64_t dims[2] = {n_row, n_col};
    return launch_siddon<2, true>("back_project_2d_siddon", sino, out, batch, dims, src, dst, n_ray, M_inv, b,
                                  accumulate, tiling, stream);
}
