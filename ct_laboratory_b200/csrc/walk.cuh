#pragma once
// walk.cuh — device side of the Siddon walks (sm_100a), shared by the
// single-scan kernels (siddon.cu) and the multi-scan persistent kernels
// (batched.cu): the on-the-fly Siddon forward projector and its exact adjoint,
// 2-D and 3-D.
//
// The reference's on-the-fly 3-D kernel (src/ct_projector_3d.cu:902-1012)
// collects every plane hit of a ray into an 8 KB per-thread array, insertion-
// sorts it and then walks the sorted list.  The x-, y- and z-plane parameters
// of a ray are each already monotone, so their sorted union is a three-way
// merge.  The walk here takes that merge directly (a DDA): it keeps the next
// plane parameter of every axis in registers, repeatedly takes the smallest,
// and evaluates each plane's parameter on its own with the reference's
// formula t = (p - s) * (1/v), so the segment end points are the very floats
// the reference sorts.  Only segments inside the volume are visited (those
// outside map to out-of-range voxels, which the reference skips).  The voxel
// of a segment comes from which planes were crossed rather than from rounding
// the segment midpoint; the two agree except for segments of rounding-noise
// length, which contribute rounding-noise amounts.
//
// Memory behaviour: the volume is read through the read-only path with an
// L2 evict-last policy and the ray geometry and sinogram stream through with
// evict-first, so that a volume the size of the benchmark's (256^3 fp32 =
// 64 MiB) stays resident in the 126 MB L2.  A CTA covers `tile_rows` detector rows x (threads/tile_rows)
// columns, with warp lanes along rows, so that for a cone-beam scan the 32
// lanes of a warp trace 32 vertically adjacent rays: they share the same x-y
// path and touch neighbouring k (fastest-varying) voxels, so a warp's gather
// hits a few 32-byte sectors instead of 32.  The adjoint scatters with
// red.global.add.f32 (atomicAdd with an unused result).
#include <type_traits>

#include "common.cuh"

namespace ctlab {

constexpr unsigned kFullMask = 0xffffffffu;

// The column walk's merge ranks from an estimate checked against two lanes
// (falling back to the binary search) rather than the binary search alone.
#ifndef CTLAB_XY_RANK_EST
#define CTLAB_XY_RANK_EST 1
#endif

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

// midpoint_voxel for a diagonal M^-1 (every off-diagonal entry zero): each
// index from its own axis, i_a = rne(m_aa (fma(tm, v_a, s_a) - b_a)).
// world_to_index3 adds only exact zeros to these products (0 * x = +-0, and
// x + +-0 = x for x != 0; a zero sum rounds to index 0 either way), so the
// voxel is the same as midpoint_voxel's.
__device__ __forceinline__ int midpoint_voxel_diag(const Affine3& A, const float* sw, const float* vw, float t0,
                                                   float t1, const GridDims<3>& G) {
    const float tm = __fmul_rn(0.5f, __fadd_rn(t0, t1));
    int flat = 0;
    bool ok = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int i = rne_int(__fmul_rn(A.m[4 * a], __fsub_rn(__fmaf_rn(tm, vw[a], sw[a]), A.b[a])));
        ok = ok && (unsigned)i < (unsigned)G.n[a];
        flat += i * G.stride[a];
    }
    return ok ? flat : -1;
}

// Segments next to the grid under the midpoint rule.  The reference forms a
// segment between every two consecutive plane hits in [0, 1] (the end points
// 0 and 1 included, ct_projector_3d.cu:889-891) and charges it to the voxel
// its rounded float midpoint falls in (:982-996).  Segments before the entry
// or after the exit lie outside the grid, but one thinner than the rounding
// noise of the midpoint (about 1e-4 voxel at scanner coordinates) can have
// its midpoint rounded onto a face voxel.  This finds the segments the
// reference forms next to the entry (DIR = -1, from t_edge = t_enter
// backwards) or the exit (DIR = +1, from t_edge = t_exit onwards): the
// neighbouring hits are the next in-range plane of each axis beyond the
// edge, or the end point (DIAG: M^-1 is diagonal, midpoint_voxel_diag).
// It records up to kEdge of them, nearest first,
// and stops at the first whose midpoint rounds outside the grid.  p0[a] is a
// plane of axis a at or beyond the edge (its parameter on the far side of
// t_edge or equal to it).
constexpr int kEdge = 2;

template <int NDIM, int DIR, bool DIAG = false>
__device__ __forceinline__ int edge_segments(const AffineT<NDIM>& A, const float* sw, const float* vw,
                                             const float* s, const float* inv, const float* ps, const float* p0,
                                             float t_edge, float ray_len, const GridDims<NDIM>& G, int* vox,
                                             float* len) {
    const float kFar = DIR > 0 ? __int_as_float(0x7f800000) : -__int_as_float(0x7f800000);
#pragma unroll
    for (int k = 0; k < kEdge; ++k) {
        vox[k] = 0;
        len[k] = 0.f;
    }
    float q[NDIM], tq[NDIM];
#pragma unroll
    for (int a = 0; a < NDIM; ++a) {
        q[a] = p0[a];
        tq[a] = kFar;
        if (inv[a] == 0.f) continue;
        tq[a] = plane_t(q[a], s[a], inv[a]);
        // a plane at the edge itself bounds no segment on this side: step past it
#pragma unroll 1
        for (int k = 0; k < 2 && (DIR > 0 ? tq[a] <= t_edge : tq[a] >= t_edge); ++k) {
            q[a] += (float)DIR * ps[a];
            tq[a] = plane_t(q[a], s[a], inv[a]);
        }
        const bool in = q[a] >= -0.5f && q[a] <= (float)G.n[a] - 0.5f;
        if (!in || (DIR > 0 ? tq[a] <= t_edge : tq[a] >= t_edge)) tq[a] = kFar;
    }
    int n = 0;
    float t_near = t_edge;
#pragma unroll
    for (int k = 0; k < kEdge; ++k) {
        if (DIR > 0 ? !(t_near < 1.f) : !(t_near > 0.f)) break;
        float t_far = DIR > 0 ? 1.f : 0.f;
#pragma unroll
        for (int a = 0; a < NDIM; ++a) t_far = DIR > 0 ? fminf(t_far, tq[a]) : fmaxf(t_far, tq[a]);
        const float lo = DIR > 0 ? t_near : t_far, hi = DIR > 0 ? t_far : t_near;
        int m;
        if constexpr (DIAG && NDIM == 3) m = midpoint_voxel_diag(A, sw, vw, lo, hi, G);
        else m = midpoint_voxel<NDIM>(A, sw, vw, lo, hi, G);
        if (m < 0) break;
        vox[n] = m;
        len[n] = __fmul_rn(__fsub_rn(hi, lo), ray_len);
        ++n;
#pragma unroll
        for (int a = 0; a < NDIM; ++a) {
            if (tq[a] == t_far) {
                q[a] += (float)DIR * ps[a];
                const bool in = q[a] >= -0.5f && q[a] <= (float)G.n[a] - 0.5f;
                tq[a] = in ? plane_t(q[a], s[a], inv[a]) : kFar;
            }
        }
        t_near = t_far;
    }
    return n;
}

// Forward steps walked per group of the per-lane walk: their gathers are
// issued together (kLaneSteps loads in flight per lane); 8 against 4: the
// 64-scan 2-D batch's forward 3.65 against 3.80 ms, the midpoint-rule
// cone-beam forward 17.69 against 17.96 ms.
#ifndef CTLAB_LANE_STEPS
#define CTLAB_LANE_STEPS 8
#endif
constexpr int kLaneSteps = CTLAB_LANE_STEPS;

// One Siddon traversal.  ADJ=false: returns sum of in[voxel]*len.
// ADJ=true: scatters y*len into out[voxel].  MID selects the voxel of each
// segment: true = the reference's rounded world midpoint, false = the voxel
// between the two crossings that bound the segment (exact topology).
// `acc` accumulates the adjoint's contributions (RedF32 float atomics, or
// RedFixed integer sums; `out` is then the int64 volume).
template <int NDIM, bool ADJ, bool MID, class Acc = RedF32>
__device__ __forceinline__ float traverse(const float* __restrict__ vol, float* __restrict__ out, float y,
                                          const float* sw, const float* dw, const GridDims<NDIM>& G,
                                          const AffineT<NDIM>& A, unsigned nvox, const Acc& acc = Acc()) {
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
        const uint64_t pol = l2_policy_keep();
        if constexpr (MID) {
            // segments just before the entry, added in ascending order
            float pb[NDIM], el[kEdge];
            int ev[kEdge];
#pragma unroll
            for (int a = 0; a < NDIM; ++a) pb[a] = pn[a] - ps[a];
            const int ne = edge_segments<NDIM, -1>(A, sw, vw, s, inv, ps, pb, t_enter, ray_len, G, ev, el);
#pragma unroll
            for (int k = kEdge - 1; k >= 0; --k)
                if (k < ne && el[k] > 0.f) acc = __fmaf_rn(ld_keep(vol + (unsigned)ev[k], pol), el[k], acc);
        }
#pragma unroll 1
        for (int it = 0; it < max_it && !done; it += kLaneSteps) {
            int vq[kLaneSteps];
            float sq[kLaneSteps];
#pragma unroll
            for (int q = 0; q < kLaneSteps; ++q) {
                float tm = tn[0];
#pragma unroll
                for (int a = 1; a < NDIM; ++a) tm = fminf(tm, tn[a]);
                const float t1 = fminf(tm, t_exit);
                // crossing rule: parameter spans, scaled by |v| once per ray
                float seg = done ? 0.f : (MID ? __fmul_rn(__fsub_rn(t1, t_cur), ray_len) : __fsub_rn(t1, t_cur));
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
            float vv[kLaneSteps];
#pragma unroll
            for (int q = 0; q < kLaneSteps; ++q) vv[q] = ld_keep(vol + (unsigned)vq[q], pol);
#pragma unroll
            for (int q = 0; q < kLaneSteps; ++q) acc = sq[q] > 0.f ? __fmaf_rn(vv[q], sq[q], acc) : acc;
        }
        if constexpr (MID) {
            // segments just after the exit
            float el[kEdge];
            int ev[kEdge];
            const int ne = edge_segments<NDIM, 1>(A, sw, vw, s, inv, ps, pn, t_exit, ray_len, G, ev, el);
#pragma unroll
            for (int k = 0; k < kEdge; ++k)
                if (k < ne && el[k] > 0.f) acc = __fmaf_rn(ld_keep(vol + (unsigned)ev[k], pol), el[k], acc);
        }
        return MID ? acc : __fmul_rn(acc, ray_len);
    } else {
        if constexpr (MID) {
            float pb[NDIM], el[kEdge];
            int ev[kEdge];
#pragma unroll
            for (int a = 0; a < NDIM; ++a) pb[a] = pn[a] - ps[a];
            const int ne = edge_segments<NDIM, -1>(A, sw, vw, s, inv, ps, pb, t_enter, ray_len, G, ev, el);
#pragma unroll
            for (int k = 0; k < kEdge; ++k) acc.add(out, (unsigned)ev[k], __fmul_rn(y, el[k]), k < ne && el[k] > 0.f);
        }
        // Segment length (t1 - t0) * |v| (ct_projector_3d.cu:998) times y;
        // the crossing rule multiplies y * |v| once by each span t1 - t0.
        const float yl = MID ? y : __fmul_rn(y, ray_len);
#pragma unroll 1
        for (int it = 0; it < max_it; ++it) {
            float tm = tn[0];
#pragma unroll
            for (int a = 1; a < NDIM; ++a) tm = fminf(tm, tn[a]);
            const float t1 = fminf(tm, t_exit);
            const float span = __fsub_rn(t1, t_cur);
            const float seg = MID ? __fmul_rn(span, ray_len) : span;
            const int v = MID ? midpoint_voxel<NDIM>(A, sw, vw, t_cur, t1, G) : idx;
            acc.add(out, (unsigned)v, __fmul_rn(yl, seg), seg > 0.f && v >= 0);
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
        if constexpr (MID) {
            float el[kEdge];
            int ev[kEdge];
            const int ne = edge_segments<NDIM, 1>(A, sw, vw, s, inv, ps, pn, t_exit, ray_len, G, ev, el);
#pragma unroll
            for (int k = 0; k < kEdge; ++k) acc.add(out, (unsigned)ev[k], __fmul_rn(y, el[k]), k < ne && el[k] > 0.f);
        }
        return 0.f;
    }
}

// 2-D, crossing rule: the major-axis walk.  Each step crosses one slab of
// the ray's major axis (the axis with the larger |v|: a pixel row for a
// steep ray) and splits it at the minor-axis plane that falls inside, if
// any:
//     te = min(next major plane, t_exit)     ts = min(next minor plane, te)
//     segment A = [t_cur, ts] in the current pixel, segment B = [ts, te] in
//     the pixel past the minor plane (empty unless a minor plane lies inside)
// These are the segments of traverse<2, ADJ, false> in the same order (the
// same plane parameters, ties stepping both axes), so the results are
// bitwise equal, with fewer steps.  A slab holds at most one minor plane
// when |v_minor| <= kMajorRatio |v_major|: with |s|, |d| <= 4096 and grid
// sides <= 4096 every plane parameter is within 0.002 index units of exact
// (p - s rounds by at most 2^-11, 1/v and the product by 2^-24 relative), so
// minor planes lie at least 1/0.97 - 0.007 > 1 major slab apart.  Other rays
// take traverse<2>.
// Neighbouring rays of a fan (the lanes of a warp) that enter the image at
// the same row stay on the same row step by step, so their scattered
// additions fall into neighbouring pixels of one row.
#ifndef CTLAB_MAJOR2_RATIO
#define CTLAB_MAJOR2_RATIO 0.97f
#endif
constexpr float kMajorRatio = CTLAB_MAJOR2_RATIO;

// State of one lane's major-axis walk: the major axis's next plane, the
// minor axis's next plane, the current pixel index.
struct Major2 {
    float ray_len, t_cur, t_exit;
    float sM, iM, psM, pnM, tnM;  // major axis: start, 1/v, step sign, next plane, its parameter
    float sm, im, psm, pnm, tnm;  // minor axis (tnm = +inf when the ray crosses none)
    int idx, dsM, dsm;            // pixel index and its steps in the buffer walked
    int n_major, start_major;     // major-axis size; slab index at the entry
    bool major_axis1, transposed;
    float sw[2], vw[2];           // world start and direction (midpoint rule)
};

// Set-up of the major-axis walk, the arithmetic of traverse<2>'s start.
// Returns 0 when the ray contributes nothing, 2 when it is outside the walk's
// bound (the caller takes traverse<2>), 1 to walk.  With `transpose_fast`,
// a ray whose major axis is the image's stride-1 axis indexes the image's
// transpose (column-major: minor axis at stride 1, major at n_minor), so
// that neighbouring rays stepping through the same major slab touch
// neighbouring addresses.
__device__ __forceinline__ int major2_setup(Major2& W, const float* sw, const float* dw, const GridDims<2>& G,
                                            const Affine2& A, bool transpose_fast) {
    float* vw = W.vw;
    vw[0] = __fsub_rn(dw[0], sw[0]);
    vw[1] = __fsub_rn(dw[1], sw[1]);
    W.sw[0] = sw[0];
    W.sw[1] = sw[1];
    W.ray_len = sqrtf(sumsq2(vw[0], vw[1]));
    if (!(W.ray_len >= 1e-12f)) return 0;
    float s[2], d[2];
    world_to_index2(A, sw[0], sw[1], s[0], s[1]);
    world_to_index2(A, dw[0], dw[1], d[0], d[1]);
    float va[2], inv[2];
    float t_enter = 0.f, t_exit = 1.f;
    bool live = true;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        va[a] = __fsub_rn(d[a], s[a]);
        live = live && isfinite(s[a]) && isfinite(va[a]);
        inv[a] = 0.f;
        if (fabsf(va[a]) > 1e-12f) {
            inv[a] = __frcp_rn(va[a]);
            const float nf = (float)G.n[a];
            const float lo = va[a] > 0.f ? -0.5f : nf - 0.5f;
            const float hi = va[a] > 0.f ? nf - 0.5f : -0.5f;
            t_enter = fmaxf(t_enter, plane_t(lo, s[a], inv[a]));
            t_exit = fminf(t_exit, plane_t(hi, s[a], inv[a]));
        }
    }
    // (selects, not indexing by the major axis: the arrays stay in registers)
    const bool M = fabsf(va[1]) > fabsf(va[0]);
    const float aM = fabsf(M ? va[1] : va[0]), am = fabsf(M ? va[0] : va[1]);
    const bool fits = (M ? inv[1] : inv[0]) != 0.f && am <= kMajorRatio * aM &&
                      fmaxf(fmaxf(fabsf(s[0]), fabsf(s[1])), fmaxf(fabsf(d[0]), fabsf(d[1]))) <= 4096.f &&
                      G.n[0] <= 4096 && G.n[1] <= 4096;
    if (!fits) return 2;
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        if (inv[a] == 0.f) {  // no planes of this axis: the ray keeps one index along it
            const int i = __float2int_rn(s[a]);
            live = live && i >= 0 && i < G.n[a];
        }
    }
    live = live && (t_enter < t_exit);
    if (!live) return 0;

    W.major_axis1 = M;
    W.transposed = transpose_fast && (M ? G.stride[1] : G.stride[0]) == 1;
    int stride[2];
    stride[0] = W.transposed ? 1 : G.stride[0];  // transposed: (i0, i1) at i0 + i1 * n0
    stride[1] = W.transposed ? G.n[0] : G.stride[1];
    // start slabs at t_enter, as in traverse
    int idx = 0, slab[2];
    float pn[2], tn[2], ps[2];
    int ds[2];
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        if (inv[a] == 0.f) {
            slab[a] = __float2int_rn(s[a]);
            idx += slab[a] * stride[a];
            pn[a] = 0.f;
            ps[a] = 0.f;
            ds[a] = 0;
            tn[a] = __int_as_float(0x7f800000);
            continue;
        }
        const float c = __fmaf_rn(t_enter, va[a], s[a]);
        int i = __float2int_rd(c + 0.5f);
        if (va[a] > 0.f) {
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
        slab[a] = i;
        idx += i * stride[a];
        ps[a] = va[a] > 0.f ? 1.f : -1.f;
        ds[a] = va[a] > 0.f ? stride[a] : -stride[a];
        pn[a] = (float)i + 0.5f * ps[a];
        tn[a] = plane_t(pn[a], s[a], inv[a]);
    }
    W.sM = M ? s[1] : s[0];
    W.iM = M ? inv[1] : inv[0];
    W.psM = M ? ps[1] : ps[0];
    W.pnM = M ? pn[1] : pn[0];
    W.tnM = M ? tn[1] : tn[0];
    W.sm = M ? s[0] : s[1];
    W.im = M ? inv[0] : inv[1];
    W.psm = M ? ps[0] : ps[1];
    W.pnm = M ? pn[0] : pn[1];
    W.tnm = M ? tn[0] : tn[1];
    W.dsM = M ? ds[1] : ds[0];
    W.dsm = M ? ds[0] : ds[1];
    W.n_major = M ? G.n[1] : G.n[0];
    W.start_major = M ? slab[1] : slab[0];
    W.idx = idx;
    W.t_cur = t_enter;
    W.t_exit = t_exit;
    return 1;
}

// One step of the adjoint walk: the rest of the current major slab, split at
// the minor plane inside it (if any), scattered as y * length.  MID: each
// segment's voxel is the reference's rounded world midpoint, indexed with
// Gt's strides (the buffer walked), and `y` is y; otherwise `y` is
// y * |v|, multiplied by each parameter span.  Returns whether the walk is
// done.
template <bool MID>
__device__ __forceinline__ bool major2_adj_step(Major2& W, float* __restrict__ o, float y, const Affine2& A,
                                                const GridDims<2>& Gt) {
    const float te = fminf(W.tnM, W.t_exit);
    const float ts = fminf(W.tnm, te);
    const float da = __fsub_rn(ts, W.t_cur);
    const float sa = MID ? __fmul_rn(da, W.ray_len) : da;
    int va = W.idx;
    bool pa = sa > 0.f;
    if constexpr (MID) {
        va = midpoint_voxel<2>(A, W.sw, W.vw, W.t_cur, ts, Gt);
        pa = pa && va >= 0;
    }
    red_add_if(o + (unsigned)va, __fmul_rn(y, sa), pa);
    if (W.tnm <= te) {
        W.idx += W.dsm;
        W.pnm += W.psm;
        W.tnm = plane_t(W.pnm, W.sm, W.im);
    }
    const float db = __fsub_rn(te, ts);
    const float sb = MID ? __fmul_rn(db, W.ray_len) : db;
    int vb = W.idx;
    bool pb = sb > 0.f;
    if constexpr (MID) {
        vb = midpoint_voxel<2>(A, W.sw, W.vw, ts, te, Gt);
        pb = pb && vb >= 0;
    }
    red_add_if(o + (unsigned)vb, __fmul_rn(y, sb), pb);
    W.t_cur = te;
    const bool done = !(W.tnM < W.t_exit);
    if (!done) {
        W.idx += W.dsM;
        W.pnM += W.psM;
        W.tnM = plane_t(W.pnM, W.sM, W.iM);
    }
    return done;
}

// Midpoint rule: the segments the reference forms just outside the grid
// (edge_segments) next to the entry (DIR = -1, from the walk's start state)
// or the exit (DIR = +1, from its end state), scattered into o with Gt's
// strides.
template <int DIR>
__device__ __forceinline__ void major2_edge_adj(const Major2& W, float* __restrict__ o, float y, const Affine2& A,
                                                const GridDims<2>& Gt) {
    const bool M = W.major_axis1;
    float s[2], inv[2], ps[2], p0[2];
    s[0] = M ? W.sm : W.sM;
    s[1] = M ? W.sM : W.sm;
    inv[0] = M ? W.im : W.iM;
    inv[1] = M ? W.iM : W.im;
    ps[0] = M ? W.psm : W.psM;
    ps[1] = M ? W.psM : W.psm;
    // entry: the planes behind the start slabs; exit: the next planes ahead
    const float pM = DIR < 0 ? W.pnM - W.psM : W.pnM, pm = DIR < 0 ? W.pnm - W.psm : W.pnm;
    p0[0] = M ? pm : pM;
    p0[1] = M ? pM : pm;
    float el[kEdge];
    int ev[kEdge];
    const int ne = edge_segments<2, DIR>(A, W.sw, W.vw, s, inv, ps, p0, DIR < 0 ? W.t_cur : W.t_exit, W.ray_len,
                                         Gt, ev, el);
#pragma unroll
    for (int k = 0; k < kEdge; ++k) red_add_if(o + (unsigned)ev[k], __fmul_rn(y, el[k]), k < ne && el[k] > 0.f);
}

template <bool ADJ>
__device__ __forceinline__ float traverse_major2(const float* __restrict__ vol, float* __restrict__ out, float y,
                                                 const float* sw, const float* dw, const GridDims<2>& G,
                                                 const Affine2& A) {
    Major2 W;
    const int kind = major2_setup(W, sw, dw, G, A, false);
    if (kind == 0) return 0.f;
    if (kind == 2) return traverse<2, ADJ, false>(vol, out, y, sw, dw, G, A, 0u);
    // Every step crosses one major plane; the walk ends at the slab holding
    // the exit, so it takes at most n_major + 1 steps.
    const int max_it = W.n_major + 2;
    bool done = false;
    if constexpr (!ADJ) {
        float acc = 0.f;
        const uint64_t pol = l2_policy_keep();
#pragma unroll 1
        for (int it = 0; it < max_it && !done; it += 4) {
            float sa[4], sb[4];
            int ia[4], ib[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const float te = fminf(W.tnM, W.t_exit);
                const float ts = fminf(W.tnm, te);
                sa[q] = done ? 0.f : __fsub_rn(ts, W.t_cur);
                ia[q] = W.idx;
                if (!done && W.tnm <= te) {
                    W.idx += W.dsm;
                    W.pnm += W.psm;
                    W.tnm = plane_t(W.pnm, W.sm, W.im);
                }
                sb[q] = done ? 0.f : __fsub_rn(te, ts);
                ib[q] = W.idx;
                W.t_cur = te;
                done = done || !(W.tnM < W.t_exit);
                if (!done) {
                    W.idx += W.dsM;
                    W.pnM += W.psM;
                    W.tnM = plane_t(W.pnM, W.sM, W.iM);
                }
            }
            float v[8];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (sa[q] > 0.f) v[q] = ld_keep(vol + (unsigned)ia[q], pol);
                if (sb[q] > 0.f) v[4 + q] = ld_keep(vol + (unsigned)ib[q], pol);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                if (sa[q] > 0.f) acc = __fmaf_rn(v[q], sa[q], acc);
                if (sb[q] > 0.f) acc = __fmaf_rn(v[4 + q], sb[q], acc);
            }
        }
        return __fmul_rn(acc, W.ray_len);
    } else {
        const float yl = __fmul_rn(y, W.ray_len);
#pragma unroll 1
        for (int it = 0; it < max_it && !done; ++it) done = major2_adj_step<false>(W, out, yl, A, G);
        return 0.f;
    }
}

// The 2-D adjoint of one warp's rays, row-aligned: called by all 32 lanes
// together (r = -1: the lane has no ray).  When every walking lane has the
// same major axis and direction, the lanes start their walks staggered so
// that at every step they all stand in the same major slab (a lane whose ray
// enters the image later along the walk waits for the others to reach its
// entry slab): a fan's neighbouring rays then scatter into neighbouring
// pixels of one image row in the same instruction, a few 32-byte sectors
// instead of one per lane.  With outT (an image-sized buffer holding the
// image's transpose, zeroed), rays whose major axis is the image's stride-1
// axis scatter there; the caller adds it back.  The segments and their
// values are those of traverse<2, true, MID> (MID: the reference's midpoint
// voxel rule, with its segments just outside the grid); only the order of
// the additions differs.
template <bool MID>
__device__ __forceinline__ void major2_adjoint_warp(const float* __restrict__ in, float* __restrict__ out,
                                                    float* __restrict__ outT, const float* __restrict__ src,
                                                    const float* __restrict__ dst, int64_t n_ray,
                                                    const Affine2& A, const GridDims<2>& G, int64_t nvox,
                                                    int64_t r, int64_t bi) {
    float sw[2] = {0.f, 0.f}, dw[2] = {0.f, 0.f}, y = 0.f;
    if (r >= 0) {
        y = ld_stream(in + bi * n_ray + r);
#pragma unroll
        for (int a = 0; a < 2; ++a) {
            sw[a] = ld_stream(src + r * 2 + a);
            dw[a] = ld_stream(dst + r * 2 + a);
        }
    }
    Major2 W;
    const int kind = (r >= 0 && y != 0.f) ? major2_setup(W, sw, dw, G, A, outT != nullptr) : 0;
    const bool walk = kind == 1;
    // walking lanes with one major axis and direction: align them by slab
    const int key = walk ? (W.major_axis1 ? 2 : 0) + (W.psM > 0.f ? 1 : 0) : -1;
    const unsigned walkers = __ballot_sync(kFullMask, walk);
    int delay = 0;
    if (walkers != 0u) {
        const int key0 = __shfl_sync(kFullMask, key, __ffs(walkers) - 1);
        if (__all_sync(kFullMask, !walk || key == key0)) {
            // position of the entry slab along the walk direction
            int pos = walk ? (W.psM > 0.f ? W.start_major : -W.start_major) : 0x7fffffff;
            int lo = pos;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) lo = min(lo, __shfl_xor_sync(kFullMask, lo, o));
            delay = walk ? pos - lo : 0;
        }
    }
    const bool tr = walk && W.transposed;
    float* o = (tr ? outT : out) + bi * nvox;
    GridDims<2> Gt = G;  // the strides of the buffer walked
    if (tr) {
        Gt.stride[0] = 1;
        Gt.stride[1] = G.n[0];
    }
    if constexpr (MID) {
        if (walk) major2_edge_adj<-1>(W, o, y, A, Gt);
    }
    bool done = !walk;
    // every step crosses one major plane: at most n_major + 1 steps per lane
    // (a walk ends by itself before `last`; the bound only guards the loop)
    const int last = walk ? delay + W.n_major + 1 : 0;
    const float ys = MID || !walk ? y : __fmul_rn(y, W.ray_len);  // the step's scale (major2_adj_step)
#pragma unroll 1
    for (int it = 0;; ++it) {
        if (!done && it >= delay) done = major2_adj_step<MID>(W, o, ys, A, Gt) || it >= last;
        if (__all_sync(kFullMask, done)) break;
    }
    if constexpr (MID) {
        if (walk) major2_edge_adj<1>(W, o, y, A, Gt);
    }
    if (kind == 2) traverse<2, true, MID>(nullptr, out + bi * nvox, y, sw, dw, G, A, (unsigned)nvox);
}

// 2-D crossing-rule rays walk by major-axis slabs (traverse_major2):
// 0 = never, 1 = adjoint only, 2 = forward and adjoint.
#ifndef CTLAB_MAJOR2
#define CTLAB_MAJOR2 1
#endif
// The 2-D adjoint kernels take the row-aligned warp walk
// (major2_adjoint_warp).
#ifndef CTLAB_MAJOR2_WARP
#define CTLAB_MAJOR2_WARP 1
#endif

// Per-thread body of the per-lane walk: ray r (>= 0) of batch item bi.
template <int NDIM, bool ADJ, bool MID, class Acc = RedF32>
__device__ __forceinline__ void lane_ray(const float* __restrict__ in, float* __restrict__ out,
                                         const float* __restrict__ src, const float* __restrict__ dst, int64_t n_ray,
                                         const AffineT<NDIM>& aff, const GridDims<NDIM>& G, int64_t nvox, int64_t r,
                                         int64_t bi, const Acc& acc = Acc()) {
    float sw[NDIM], dw[NDIM];
#pragma unroll
    for (int a = 0; a < NDIM; ++a) {
        sw[a] = ld_stream(src + r * NDIM + a);
        dw[a] = ld_stream(dst + r * NDIM + a);
    }
    if constexpr (ADJ) {
        const float y = ld_stream(in + bi * n_ray + r);
        if (y == 0.f) return;  // contributes exactly nothing
        if constexpr (NDIM == 2 && !MID && CTLAB_MAJOR2 >= 1)
            traverse_major2<true>(nullptr, out + bi * nvox, y, sw, dw, G, aff);
        else
            traverse<NDIM, true, MID, Acc>(nullptr, acc.at(out, bi * nvox), y, sw, dw, G, aff, (unsigned)nvox, acc);
    } else {
        float v;
        if constexpr (NDIM == 2 && !MID && CTLAB_MAJOR2 >= 2)
            v = traverse_major2<false>(in + bi * nvox, nullptr, 0.f, sw, dw, G, aff);
        else
            v = traverse<NDIM, false, MID>(in + bi * nvox, nullptr, 0.f, sw, dw, G, aff, (unsigned)nvox);
        st_stream(out + bi * n_ray + r, v);
    }
}

// ----------------------------------------------------------------------------
// Shared x-y walk for detector columns (3-D, crossing rule).
//
// When the 32 lanes of a warp trace rays that share their x-y line (one
// source, one detector column whose cells run along z: cone-beam views tiled
// with 32 detector rows per warp), every x- and y-plane parameter is bitwise
// the same for all lanes and only the z planes differ.  (Detectors with 16
// rows per column, such as StaticCT modules, run the same walk in two
// 16-lane groups per warp: shared_xy_ray's W below.)
// The per-lane walk then spends most of its compare / select work deriving
// the same x-y crossings 32 times over.  Here the warp derives the merged x-y
// crossing sequence once, 32 crossings per round: lane l evaluates the l-th
// next x plane and the l-th next y plane, a rank search across the warp
// places each in merged order, and the first 32 go to a per-warp shared
// buffer together with the x-y column each one ends.  Every lane then walks
// the buffer cell by cell (the same cell on all lanes, a broadcast read) and
// splits the cell at its own next z plane when one falls inside it:
//     te = min(t_cell_end, t_exit)      ts = min(t_next_z, te)
//     segment A = [t_cur, ts] in (column, k)
//     segment B = [ts, te]    in (column, k +- 1), empty unless a z plane lies inside
// Segments are the parameter spans t1 - t0 over the same plane parameters as
// the per-lane walk, taken in the same order, zero-length ones skipped and
// |v| applied once per ray as there, so the results are bitwise those of
// traverse<3, ADJ, false>.
//
// At most one z plane per cell: a cell spans at most the x or y plane
// spacing in t, 1 / max(|v_x|, |v_y|), and z planes are 1 / |v_z| apart.  A
// warp takes this walk only when every live lane has |v_z| <= 0.75 max(|v_x|,
// |v_y|) and |s| <= 2^17 (with every grid dimension <= 2^16, checked on the
// host), so |p - s| < 2^18 and float rounding of a plane parameter (< 2^-6 of
// a spacing) cannot close the 25 % margin.  Other warps run the per-lane walk.
// ----------------------------------------------------------------------------
constexpr int kChunk = 32;  // x-y crossings produced per round, one per lane
// Cells walked per inner step (both divide kChunk): the forward issues the
// gathers of 8 cells together (up to 16 loads in flight per lane), the
// adjoint's reductions need no results and walk 4 at a time (measured
// fastest for each on the cone-beam benchmark scan).
#ifndef CTLAB_XY_GROUP_FWD
#define CTLAB_XY_GROUP_FWD 8
#endif
#ifndef CTLAB_XY_GROUP_ADJ
#define CTLAB_XY_GROUP_ADJ 4
#endif
constexpr int kGroupFwd = CTLAB_XY_GROUP_FWD;
constexpr int kGroupAdj = CTLAB_XY_GROUP_ADJ;

// Walk warps whose lanes all enter and leave together without per-lane clipping.
#ifndef CTLAB_XY_UNIFORM
#define CTLAB_XY_UNIFORM 1
#endif

struct XYCell {
    float t;  // parameter of the crossing that ends the cell
    int col;  // flat index of the cell's (i, j) column at k = 0
};

// Per-lane set-up, the arithmetic of the start of traverse<3>.
struct LaneRay {
    float s[3], va[3], inv[3], ray_len, t_enter, t_exit;
    bool live;
};

__device__ __forceinline__ void lane_setup(LaneRay& R, const float* sw, const float* dw, const GridDims<3>& G,
                                           const Affine3& A) {
    float vw[3], d[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) vw[a] = __fsub_rn(dw[a], sw[a]);
    R.ray_len = sqrtf(sumsq3(vw[0], vw[1], vw[2]));
    R.live = R.ray_len >= 1e-12f;
    world_to_index3(A, sw[0], sw[1], sw[2], R.s[0], R.s[1], R.s[2]);
    world_to_index3(A, dw[0], dw[1], dw[2], d[0], d[1], d[2]);
    R.t_enter = 0.f;
    R.t_exit = 1.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float va = __fsub_rn(d[a], R.s[a]);
        const float nf = (float)G.n[a];
        R.va[a] = va;
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
        }
    }
    R.live = R.live && (R.t_enter < R.t_exit);
}

// Slab of a crossing axis at parameter t: behind-plane parameter <= t and
// ahead-plane parameter > t, from an estimate fixed up with the exact plane
// formula (the start rule of traverse), clamped into the grid.
__device__ __forceinline__ int slab_at(float t, float s, float va, float inv, int n) {
    int i = __float2int_rd(__fmaf_rn(t, va, s) + 0.5f);
    if (va > 0.f) {
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

// Number of lanes m whose `sorted` value (non-decreasing over the lanes) is
// below `key` (INCLUSIVE: at or below): a branch-free binary search.
// W: the lanes searched are the caller's group of W lanes (W = 32: the warp;
// W = 16: its half), lane indices relative to the group.
template <bool INCLUSIVE, int W = 32>
__device__ __forceinline__ int warp_rank(float sorted, float key) {
    int c = 0;
#pragma unroll
    for (int step = W / 2; step > 0; step >>= 1) {
        const float v = __shfl_sync(kFullMask, sorted, c + step - 1, W);
        c += (INCLUSIVE ? v <= key : v < key) ? step : 0;
    }
    // c counts lanes 0..W-2; lane W-1 is the one left to test
    const float v = __shfl_sync(kFullMask, sorted, c, W);
    return c + ((INCLUSIVE ? v <= key : v < key) ? 1 : 0);
}

// Merged positions of a round's x and y crossings: lane l holds the l-th next
// x crossing tx and the l-th next y crossing ty (each non-decreasing over the
// lanes of its group of W); on equal parameters the x crossing comes first:
//     ky = #{k : ty_k < tx},   kx = #{k : tx_k <= ty}.
// With CTLAB_XY_RANK_EST (32-lane groups crossing both axes) the counts are
// estimated from the plane coordinate each parameter falls at (the y index
// reached at tx, the x index reached at ty) and checked against the two
// neighbouring lanes: a count is exact when the lane below is on the near
// side and the lane at the count on the far side.  Any miss in the warp: the
// binary search (warp_rank).  16-lane groups always search (two steps
// shorter there, and measured faster than the estimate).  `both` must be
// warp-uniform.
template <int W>
__device__ __forceinline__ void xy_merge_ranks(float tx, float ty, bool both, float s0, float s1, float va0,
                                               float va1, float pnx, float pny, float psx, float psy, int& kx,
                                               int& ky) {
#if CTLAB_XY_RANK_EST
    if (W == 32 && both) {
        const float by = psy * __fmaf_rn(tx, va1, __fsub_rn(s1, pny));
        const float bx = psx * __fmaf_rn(ty, va0, __fsub_rn(s0, pnx));
        ky = min(max(__float2int_ru(by), 0), W);
        kx = min(max(__float2int_rd(bx) + 1, 0), W);
        const float ylo = __shfl_sync(kFullMask, ty, max(ky - 1, 0), W);
        const float yhi = __shfl_sync(kFullMask, ty, min(ky, W - 1), W);
        const float xlo = __shfl_sync(kFullMask, tx, max(kx - 1, 0), W);
        const float xhi = __shfl_sync(kFullMask, tx, min(kx, W - 1), W);
        const bool ok = (ky == 0 || ylo < tx) && (ky == W || !(yhi < tx)) && (kx == 0 || xlo <= ty) &&
                        (kx == W || !(xhi <= ty));
        if (__all_sync(kFullMask, ok)) return;
    }
#endif
    ky = warp_rank<false, W>(ty, tx);
    kx = warp_rank<true, W>(tx, ty);
}

// Per-lane z state of the shared x-y walk.
struct ZWalk {
    float t_cur, t_end, len, tnz, pnz, psz, s2, i2;
    int kz, dsz;
};

// NG cells of the buffer from position q: segment A = [t_cur, ts] in
// (column, k), segment B = [ts, te] in (column, k') after a z step, as
// parameter spans t1 - t0; the caller scales by |v| (the reference's length
// (t1 - t0) * |v|, ct_projector_3d.cu:998) once per ray: the forward
// multiplies its sum, the adjoint its y.
template <int NG>
struct CellGroup {
    float sa[NG], sb[NG];
    unsigned ia[NG], ib[NG];  // voxel indices, valid where the segment is positive
};

// UNI: every lane of the warp enters and leaves the grid at the warp's
// t_start / t_stop (and the round's cell ends are clipped to t_stop when the
// buffer is written), so a cell's end needs no clipping to the lane's exit
// and t_cur only moves forward: two operations per cell fewer, the same
// segments.
template <int NG, bool UNI>
__device__ __forceinline__ void walk_group(const XYCell* buf, int q, CellGroup<NG>& g, ZWalk& Z) {
#pragma unroll
    for (int u = 0; u < NG; ++u) {
        const XYCell c = buf[q + u];
        const float te = UNI ? c.t : fminf(c.t, Z.t_end);
        const float ts = fminf(Z.tnz, te);
        g.sa[u] = __fsub_rn(ts, Z.t_cur);
        g.ia[u] = (unsigned)(c.col + Z.kz);
        if (Z.tnz <= te) {  // a z plane inside the cell (or ending it)
            Z.kz += Z.dsz;
            Z.pnz += Z.psz;
            Z.tnz = plane_t(Z.pnz, Z.s2, Z.i2);
        }
        g.sb[u] = __fsub_rn(te, ts);
        g.ib[u] = (unsigned)(c.col + Z.kz);
        Z.t_cur = UNI ? te : fmaxf(Z.t_cur, te);
    }
}

// A positive segment lies inside the lane's [t_enter, t_exit] and between
// crossed planes only, so its voxel is inside the grid; zero-length ones
// (before entry, after exit, ties) are neither read nor added.
template <int NG>
__device__ __forceinline__ void gather_group(const float* vol, const CellGroup<NG>& g, float* v, uint64_t pol) {
#pragma unroll
    for (int u = 0; u < NG; ++u) {
        if (g.sa[u] > 0.f) v[u] = ld_keep(vol + g.ia[u], pol);
        if (g.sb[u] > 0.f) v[NG + u] = ld_keep(vol + g.ib[u], pol);
    }
}

template <int NG>
__device__ __forceinline__ float accumulate_group(const CellGroup<NG>& g, const float* v, float acc) {
#pragma unroll
    for (int u = 0; u < NG; ++u) {
        if (g.sa[u] > 0.f) acc = __fmaf_rn(v[u], g.sa[u], acc);
        if (g.sb[u] > 0.f) acc = __fmaf_rn(v[NG + u], g.sb[u], acc);
    }
    return acc;
}

// Per-thread body of the shared x-y walk for ray r (r = -1: the thread has no
// ray but still takes part in the warp's collective steps) and the nb <= NB
// batch items b0 .. b0+nb-1: the walk is done once and every segment gathers
// from (forward) or reduces into (adjoint) all nb volumes.  All 32 lanes of
// the warp call it together; `buf` is the warp's kChunk-entry shared-memory
// cell buffer.
//
// W = 16 splits the warp into two groups of 16 lanes, each walking its own
// x-y line with 16 crossings per round (detectors with 16 rows per column,
// such as StaticCT modules, tiled 16 rows x 2 columns per warp).  The two
// groups keep step round by round (the rank search shuffles within each
// half, with all 32 lanes taking part), a group that has left the volume
// idling until the other is done; every decision that branches around a
// collective step is taken for the whole warp.
template <bool ADJ, int NB, int W = 32, class Acc = RedF32>
__device__ __forceinline__ void shared_xy_ray(const float* __restrict__ in, float* __restrict__ out,
                                              const float* __restrict__ src, const float* __restrict__ dst,
                                              int64_t n_ray, const Affine3& A, const GridDims<3>& G,
                                              int64_t nvox, int64_t r, int64_t b0, int nb, XYCell* buf,
                                              const Acc& acc = Acc()) {
    static_assert(W == 32 || W == 16, "group width must be 32 or 16");
    const int wlane = threadIdx.x & 31;
    const int lane = wlane & (W - 1);  // lane within the group
    const unsigned gmask = W == 32 ? kFullMask : (0xffffu << (wlane & 16));
    buf += wlane & (32 - W);  // the group's part of the warp's buffer
    float sw[3] = {0.f, 0.f, 0.f}, dw[3] = {0.f, 0.f, 0.f};
    if (r >= 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            sw[a] = ld_stream(src + r * 3 + a);
            dw[a] = ld_stream(dst + r * 3 + a);
        }
    }
    float y[NB];
    bool any_y = false;
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        y[j] = 0.f;
        if constexpr (ADJ) {
            if (r >= 0 && j < nb) y[j] = ld_stream(in + (b0 + j) * n_ray + r);
        }
        any_y = any_y || y[j] != 0.f;
    }
    LaneRay R;
    lane_setup(R, sw, dw, G, A);
    R.live = R.live && (r >= 0) && (!ADJ || any_y);

    const unsigned warp_live = __ballot_sync(kFullMask, R.live);
    const unsigned live_mask = warp_live & gmask;
    if (warp_live == 0u) {
        if (!ADJ && r >= 0) {
#pragma unroll
            for (int j = 0; j < NB; ++j)
                if (j < nb) st_stream(out + (b0 + j) * n_ray + r, 0.f);
        }
        return;
    }
    // Do the live lanes share their x-y line, and is every live lane's z
    // slope inside the one-z-plane-per-cell bound?  (Dead lanes do not vote.)
    // (a group without live lanes reads its first lane; nothing it walks has length)
    const int leader = live_mask ? __ffs(live_mask) - 1 : (wlane & (32 - W));
    const float s0 = __shfl_sync(kFullMask, R.s[0], leader), s1 = __shfl_sync(kFullMask, R.s[1], leader);
    const float va0 = __shfl_sync(kFullMask, R.va[0], leader), va1 = __shfl_sync(kFullMask, R.va[1], leader);
    const float i0 = __shfl_sync(kFullMask, R.inv[0], leader), i1 = __shfl_sync(kFullMask, R.inv[1], leader);
    const float vxy = fmaxf(i0 != 0.f ? fabsf(va0) : 0.f, i1 != 0.f ? fabsf(va1) : 0.f);
    const bool ok = !R.live || (__float_as_uint(R.s[0]) == __float_as_uint(s0) &&
                                __float_as_uint(R.s[1]) == __float_as_uint(s1) &&
                                __float_as_uint(R.va[0]) == __float_as_uint(va0) &&
                                __float_as_uint(R.va[1]) == __float_as_uint(va1) &&
                                fabsf(R.va[2]) <= 0.75f * vxy && fabsf(R.s[0]) <= 131072.f &&
                                fabsf(R.s[1]) <= 131072.f && fabsf(R.s[2]) <= 131072.f);
    if (!__all_sync(kFullMask, ok && (live_mask == 0u || vxy != 0.f))) {
        if (r < 0) return;
#pragma unroll 1
        for (int j = 0; j < nb; ++j) {  // the per-lane walk, once per volume
            const int64_t b = b0 + j;
            if constexpr (ADJ) {
                const float yj = ld_stream(in + b * n_ray + r);
                if (R.live && yj != 0.f)
                    traverse<3, true, false, Acc>(nullptr, acc.at(out, b * nvox), yj, sw, dw, G, A, (unsigned)nvox,
                                                  acc);
            } else {
                st_stream(out + b * n_ray + r,
                          R.live ? traverse<3, false, false>(in + b * nvox, nullptr, 0.f, sw, dw, G, A, (unsigned)nvox)
                                 : 0.f);
            }
        }
        return;
    }

    // ---- x-y start, warp-uniform: the slabs at the earliest lane entry ----
    const float kInf = __int_as_float(0x7f800000);
    float t_start = R.live ? R.t_enter : kInf, t_stop = R.live ? R.t_exit : -kInf;
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) {
        t_start = fminf(t_start, __shfl_xor_sync(kFullMask, t_start, o));
        t_stop = fmaxf(t_stop, __shfl_xor_sync(kFullMask, t_stop, o));
    }
    int col = 0, dsx = 0, dsy = 0;
    float pnx = 0.f, pny = 0.f, psx = 0.f, psy = 0.f;
    if (i0 != 0.f) {
        const int i = slab_at(t_start, s0, va0, i0, G.n[0]);
        psx = va0 > 0.f ? 1.f : -1.f;
        dsx = va0 > 0.f ? G.stride[0] : -G.stride[0];
        pnx = (float)i + 0.5f * psx;
        col += i * G.stride[0];
    } else {
        col += __float2int_rn(s0) * G.stride[0];
    }
    if (i1 != 0.f) {
        const int j = slab_at(t_start, s1, va1, i1, G.n[1]);
        psy = va1 > 0.f ? 1.f : -1.f;
        dsy = va1 > 0.f ? G.stride[1] : -G.stride[1];
        pny = (float)j + 0.5f * psy;
        col += j * G.stride[1];
    } else {
        col += __float2int_rn(s1) * G.stride[1];
    }

    // ---- per-lane z state at the lane's own entry ------------------------
    // Dead lanes keep t_cur = t_end = 0 and no z plane: every segment they
    // form has zero length.
    ZWalk Z;
    Z.s2 = R.s[2];
    Z.i2 = R.inv[2];
    Z.t_cur = 0.f;
    Z.t_end = 0.f;
    Z.len = 0.f;
    Z.tnz = kInf;
    Z.pnz = 0.f;
    Z.psz = 0.f;
    Z.kz = 0;
    Z.dsz = 0;
    if (R.live) {
        Z.t_cur = R.t_enter;
        Z.t_end = R.t_exit;
        Z.len = R.ray_len;
        if (Z.i2 != 0.f) {
            const int k = slab_at(Z.t_cur, Z.s2, R.va[2], Z.i2, G.n[2]);
            Z.psz = R.va[2] > 0.f ? 1.f : -1.f;
            Z.dsz = R.va[2] > 0.f ? G.stride[2] : -G.stride[2];
            Z.pnz = (float)k + 0.5f * Z.psz;
            Z.tnz = plane_t(Z.pnz, Z.s2, Z.i2);
            Z.kz = k * G.stride[2];
        } else {
            Z.kz = __float2int_rn(Z.s2) * G.stride[2];
        }
    }

    // ---- rounds of 32 x-y crossings ---------------------------------------
    // Each round consumes 32 crossings of the x-y sequence; after
    // n_x + n_y + 2 of them both exit planes lie behind, so the bound below
    // is never the reason the loop ends.  Volumes past nb alias the last
    // valid one (their results are not stored, their reductions predicated
    // off), so every address stays inside the batch.
    const float* vol[NB];
    float* vout[NB];
    float sum[NB], yl[NB];
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        const int64_t b = b0 + (j < nb ? j : nb - 1);
        vol[j] = ADJ ? nullptr : pin_ptr(in + b * nvox);
        vout[j] = ADJ ? pin_ptr(acc.at(out, b * nvox)) : nullptr;
        sum[j] = 0.f;
        yl[j] = __fmul_rn(y[j], Z.len);  // adjoint: y * |v| (0 on dead lanes)
    }
    const uint64_t pol = l2_policy_keep();
    const float fl = (float)lane;
    const int max_rounds = (G.n[0] + G.n[1] + 2) / W + 2;
    // forward: cells per step so that every step has 2 * kGroupFwd gathers in flight
    constexpr int kGF = kGroupFwd / NB > 0 ? kGroupFwd / NB : 1;
    // Do all 32 lanes trace live rays entering and leaving at the warp's
    // t_start / t_stop?  (Most warps of a cone-beam scan: their rays cross the
    // volume's side faces, not its top or bottom.)
    const bool uniform = __all_sync(kFullMask, R.live && R.t_enter == t_start && R.t_exit == t_stop);
    auto rounds = [&](auto uni_tag) {
        constexpr bool UNI = decltype(uni_tag)::value;
        bool fin = false;  // W = 16: this group has walked its last cell
#pragma unroll 1
        for (int round = 0; round < max_rounds; ++round) {
            // lane l: the l-th next x plane and the l-th next y plane (plane
            // coordinates are exact: |p| < 2^17 in steps of 1)
            float tx = i0 != 0.f ? plane_t(__fmaf_rn(fl, psx, pnx), s0, i0) : kInf;
            float ty = i1 != 0.f ? plane_t(__fmaf_rn(fl, psy, pny), s1, i1) : kInf;
            // merged positions (x first on equal parameters)
            int ky, kx;
            xy_merge_ranks<W>(tx, ty, i0 != 0.f && i1 != 0.f, s0, s1, va0, va1, pnx, pny, psx, psy, kx, ky);
            const int rx = lane + ky;
            const int ry = lane + kx;
            if (UNI) {  // cell ends past the common exit are the exit
                tx = fminf(tx, t_stop);
                ty = fminf(ty, t_stop);
            }
            if (rx < W) buf[rx] = XYCell{tx, col + lane * dsx + (rx - lane) * dsy};
            if (ry < W) buf[ry] = XYCell{ty, col + (ry - lane) * dsx + lane * dsy};
            const int n_x = __popc(__ballot_sync(kFullMask, rx < W) & gmask);
            __syncwarp();
            // cells up to and including the one that ends at or after t_stop
            const int n_in = __popc(__ballot_sync(kFullMask, buf[lane].t < t_stop) & gmask);
            const int n_cells = (W == 16 && fin) ? 0 : min(n_in + 1, W);
            if constexpr (ADJ) {
                // y * |v| once per lane, times each parameter span (the
                // forward applies |v| once to its sum of spans instead)
#pragma unroll 1
                for (int q = 0; q < n_cells; q += kGroupAdj) {
                    CellGroup<kGroupAdj> g;
                    walk_group<kGroupAdj, UNI>(buf, q, g, Z);
#pragma unroll
                    for (int j = 0; j < NB; ++j) {
#pragma unroll
                        for (int u = 0; u < kGroupAdj; ++u) {
                            const bool vj = NB == 1 || j < nb;  // one volume: always valid
                            acc.add(vout[j], g.ia[u], __fmul_rn(yl[j], g.sa[u]), g.sa[u] > 0.f && vj);
                            acc.add(vout[j], g.ib[u], __fmul_rn(yl[j], g.sb[u]), g.sb[u] > 0.f && vj);
                        }
                    }
                }
            } else {
                // the step's gathers are issued together, then accumulated in
                // walk order, volume by volume
#pragma unroll 1
                for (int q = 0; q < n_cells; q += kGF) {
                    CellGroup<kGF> g;
                    walk_group<kGF, UNI>(buf, q, g, Z);
                    float v[NB][2 * kGF];
#pragma unroll
                    for (int j = 0; j < NB; ++j) gather_group<kGF>(vol[j], g, v[j], pol);
#pragma unroll
                    for (int j = 0; j < NB; ++j) sum[j] = accumulate_group<kGF>(g, v[j], sum[j]);
                }
            }
            if constexpr (W == 32) {
                if (n_in < W) break;
            } else {
                fin = fin || n_in < W;
                if (__all_sync(kFullMask, fin)) break;
            }
            __syncwarp();  // every lane is done with this round's cells
            if (W == 32 || !fin) {
                col += n_x * dsx + (W - n_x) * dsy;
                pnx = __fmaf_rn((float)n_x, psx, pnx);
                pny = __fmaf_rn((float)(W - n_x), psy, pny);
            }
        }
    };
#if CTLAB_XY_UNIFORM
    if (uniform) rounds(std::true_type{});
    else
#else
    (void)uniform;
#endif
        rounds(std::false_type{});
    if constexpr (!ADJ) {
        if (r >= 0) {
#pragma unroll
            for (int j = 0; j < NB; ++j)
                if (j < nb) st_stream(out + (b0 + j) * n_ray + r, __fmul_rn(sum[j], Z.len));
        }
    }
}

// ----------------------------------------------------------------------------
// Shared x-y walk under the reference's midpoint rule (3-D).
//
// The reference charges each segment [t0, t1] to the voxel of its rounded
// world-space midpoint s + tm v, tm = 0.5 (t0 + t1) (ct_projector_3d.cu:
// 982-996).  With a diagonal M^-1 (every off-diagonal entry exactly zero, as
// standard_image_transform_3d builds it) each index depends on its own axis
// only: i = rne(m00 (fma(tm, v_x, s_x) - b_x)), and likewise j and k, because
// the zero products of world_to_index3 add exact zeros.
//
// Lanes that share their world x-y line (one source, one detector column)
// share every x- and y-plane parameter, and for a segment that is a whole x-y
// cell [c0, c1] they share its midpoint tm and its (i, j).  The warp derives
// the merged x-y crossings 32 per round as in shared_xy_ray and, one lane per
// cell, a record: the cell's end, tm, span c1 - c0 and the flat (i, j) offset
// of the rounded midpoint (or -1 when that is outside the grid).  Each round
// is then walked in two passes:
//
//  pass 1, all lanes in step, one broadcast record per cell: the whole cell
//    is one segment in voxel (i, j, k(tm)), k evaluated by each lane with the
//    reference's arithmetic.  This is the reference's segment for every cell
//    that holds none of the lane's z planes (and lies inside the lane's own
//    [t_enter, t_exit]);
//  pass 2, per lane: each cell that holds one of the lane's z planes, or its
//    own entry or exit, strictly inside is walked again: its segments (split
//    at the z planes, clipped to [t_enter, t_exit]) each get the voxel of
//    their own rounded midpoint (midpoint_voxel_diag), and the whole-cell
//    term pass 1 added for it, if any, is taken back out.  The forward folds
//    it into the charge of the first piece in the same voxel (length -
//    span), so a cell split in two costs two gathers, not three (1 % on the
//    cone256 scan; the adjoint measured 0.4 % slower folded and keeps the
//    separate reduction).
//
// Every segment of the reference inside the grid is thus charged to the
// reference's voxel with the reference's parameter span; the segments just
// outside the grid whose midpoint rounds onto a face voxel are added from
// edge_segments, as in traverse<3, ADJ, true>.  Spans are scaled by |v| once
// per ray (the forward multiplies its sum, the adjoint its y), and the
// forward sums in pass order, so results equal the reference's to rounding,
// not bitwise (the per-lane walk, traverse<3, false, true>, is bitwise).
// Warps whose lanes do not share their x-y line, or whose M^-1 is not
// diagonal, run traverse<3, ADJ, true> per lane.
// ----------------------------------------------------------------------------
struct __align__(16) MidCell {
    float t;     // end of the cell: the crossing that ends it (clipped to the warp's exit when uniform)
    int col;     // flat (i, j) offset of the cell's rounded midpoint (k = 0); -1 when outside in x or y
    float tm;    // the cell's midpoint parameter, 0.5 (c0 + c1) as the reference forms it
    float span;  // c1 - c0
};

__device__ __forceinline__ bool affine_is_diagonal(const Affine3& A) {
    return A.m[1] == 0.f && A.m[2] == 0.f && A.m[3] == 0.f && A.m[5] == 0.f && A.m[6] == 0.f && A.m[7] == 0.f;
}

// Per-lane slab-plane coordinates at parameter t for the edge segments:
// behind (DIR = -1) or ahead (DIR = +1) of the slab holding t, per axis.
template <int DIR>
__device__ __forceinline__ void edge_planes(const LaneRay& R, float t, const GridDims<3>& G, float* p, float* ps) {
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        ps[a] = R.inv[a] == 0.f ? 0.f : (R.va[a] > 0.f ? 1.f : -1.f);
        p[a] = 0.f;
        if (R.inv[a] != 0.f) {
            const int i = slab_at(t, R.s[a], R.va[a], R.inv[a], G.n[a]);
            p[a] = (float)i + 0.5f * (float)DIR * ps[a];
        }
    }
}

// Number of the W sorted values v[0..W-1] that are <= key (a branch-free
// binary search over this lane's own key; v in shared memory).
template <int W>
__device__ __forceinline__ int count_le(const float* v, float key) {
    int c = 0;
#pragma unroll
    for (int step = W / 2; step > 0; step >>= 1) c += v[c + step - 1] <= key ? step : 0;
    return c + (v[c] <= key ? 1 : 0);
}

// Cells per pass-1 step (forward: gathers in flight per lane).  On the
// cone256 scan the forward measured 9.67 ms with 4 against 9.77 with 8 and
// 10.04 with 16; the adjoint 9.33 ms with 4 against 9.52 with 2 and 9.94
// with 8.
#ifndef CTLAB_MID_GROUP_FWD
#define CTLAB_MID_GROUP_FWD 4
#endif
// The same for 16-lane groups (the StaticCT ring's 16-row modules): 8
// cells measured 2.46 ms per static512 forward against 2.54 with 4.
#ifndef CTLAB_MID_GROUP_FWD16
#define CTLAB_MID_GROUP_FWD16 8
#endif
#ifndef CTLAB_MID_GROUP_ADJ
#define CTLAB_MID_GROUP_ADJ 4
#endif

// Per-thread body; arguments as shared_xy_ray.  `raw` is the warp's kChunk
// floats of crossing parameters, `rec` its kChunk cell records.
template <bool ADJ, int NB, int W = 32, class Acc = RedF32>
__device__ __forceinline__ void shared_xy_ray_mid(const float* __restrict__ in, float* __restrict__ out,
                                                  const float* __restrict__ src, const float* __restrict__ dst,
                                                  int64_t n_ray, const Affine3& A, const GridDims<3>& G,
                                                  int64_t nvox, int64_t r, int64_t b0, int nb, float* raw,
                                                  MidCell* rec, const Acc& acc = Acc()) {
    static_assert(W == 32 || W == 16, "group width must be 32 or 16");
    const int wlane = threadIdx.x & 31;
    const int lane = wlane & (W - 1);
    const unsigned gmask = W == 32 ? kFullMask : (0xffffu << (wlane & 16));
    raw += wlane & (32 - W);
    rec += wlane & (32 - W);
    float sw[3] = {0.f, 0.f, 0.f}, dw[3] = {0.f, 0.f, 0.f};
    if (r >= 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            sw[a] = ld_stream(src + r * 3 + a);
            dw[a] = ld_stream(dst + r * 3 + a);
        }
    }
    float y[NB];
    bool any_y = false;
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        y[j] = 0.f;
        if constexpr (ADJ) {
            if (r >= 0 && j < nb) y[j] = ld_stream(in + (b0 + j) * n_ray + r);
        }
        any_y = any_y || y[j] != 0.f;
    }
    LaneRay R;
    lane_setup(R, sw, dw, G, A);
    R.live = R.live && (r >= 0) && (!ADJ || any_y);

    const unsigned warp_live = __ballot_sync(kFullMask, R.live);
    const unsigned live_mask = warp_live & gmask;
    if (warp_live == 0u) {
        if (!ADJ && r >= 0) {
#pragma unroll
            for (int j = 0; j < NB; ++j)
                if (j < nb) st_stream(out + (b0 + j) * n_ray + r, 0.f);
        }
        return;
    }
    // Do the live lanes share their world x-y line (source and detector cell
    // in x and y), and is M^-1 diagonal?  (Dead lanes do not vote.)
    const int leader = live_mask ? __ffs(live_mask) - 1 : (wlane & (32 - W));
    const float sx = __shfl_sync(kFullMask, sw[0], leader), sy = __shfl_sync(kFullMask, sw[1], leader);
    const float dx = __shfl_sync(kFullMask, dw[0], leader), dy = __shfl_sync(kFullMask, dw[1], leader);
    const float s0 = __shfl_sync(kFullMask, R.s[0], leader), s1 = __shfl_sync(kFullMask, R.s[1], leader);
    const float va0 = __shfl_sync(kFullMask, R.va[0], leader), va1 = __shfl_sync(kFullMask, R.va[1], leader);
    const float i0 = __shfl_sync(kFullMask, R.inv[0], leader), i1 = __shfl_sync(kFullMask, R.inv[1], leader);
    const float vxy = fmaxf(i0 != 0.f ? fabsf(va0) : 0.f, i1 != 0.f ? fabsf(va1) : 0.f);
    const bool ok = !R.live || (__float_as_uint(sw[0]) == __float_as_uint(sx) &&
                                __float_as_uint(sw[1]) == __float_as_uint(sy) &&
                                __float_as_uint(dw[0]) == __float_as_uint(dx) &&
                                __float_as_uint(dw[1]) == __float_as_uint(dy));
    if (!affine_is_diagonal(A) || !__all_sync(kFullMask, ok && (live_mask == 0u || vxy != 0.f))) {
        if (r < 0) return;
#pragma unroll 1
        for (int j = 0; j < nb; ++j) {  // the per-lane walk, once per volume
            const int64_t b = b0 + j;
            if constexpr (ADJ) {
                const float yj = ld_stream(in + b * n_ray + r);
                if (R.live && yj != 0.f)
                    traverse<3, true, true, Acc>(nullptr, acc.at(out, b * nvox), yj, sw, dw, G, A, (unsigned)nvox,
                                                 acc);
            } else {
                st_stream(out + b * n_ray + r,
                          R.live ? traverse<3, false, true>(in + b * nvox, nullptr, 0.f, sw, dw, G, A, (unsigned)nvox)
                                 : 0.f);
            }
        }
        return;
    }
    float vw[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) vw[a] = __fsub_rn(dw[a], sw[a]);

    // ---- x-y start, warp-uniform: the next planes after the earliest entry
    const float kInf = __int_as_float(0x7f800000);
    float t_start = R.live ? R.t_enter : kInf, t_stop = R.live ? R.t_exit : -kInf;
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) {
        t_start = fminf(t_start, __shfl_xor_sync(kFullMask, t_start, o));
        t_stop = fmaxf(t_stop, __shfl_xor_sync(kFullMask, t_stop, o));
    }
    float pnx = 0.f, pny = 0.f, psx = 0.f, psy = 0.f;
    if (i0 != 0.f) {
        psx = va0 > 0.f ? 1.f : -1.f;
        pnx = (float)slab_at(t_start, s0, va0, i0, G.n[0]) + 0.5f * psx;
    }
    if (i1 != 0.f) {
        psy = va1 > 0.f ? 1.f : -1.f;
        pny = (float)slab_at(t_start, s1, va1, i1, G.n[1]) + 0.5f * psy;
    }
    // (i, j) of a world midpoint on the shared x-y line (diagonal M^-1)
    const float lvx = __fsub_rn(dx, sx), lvy = __fsub_rn(dy, sy);

    // ---- per-lane state: own entry / exit, next z plane, k(tm) constants --
    float t_enter = 0.f, t_exit = 0.f, tnz = kInf, pnz = 0.f, psz = 0.f;
    if (R.live) {
        t_enter = R.t_enter;
        t_exit = R.t_exit;
        if (R.inv[2] != 0.f) {
            psz = R.va[2] > 0.f ? 1.f : -1.f;
            pnz = (float)slab_at(t_enter, R.s[2], R.va[2], R.inv[2], G.n[2]) + 0.5f * psz;
            tnz = plane_t(pnz, R.s[2], R.inv[2]);
        }
    }
    const float s2 = R.s[2], i2 = R.inv[2];
    const float zs0 = sw[2], zv = vw[2], zb = A.b[2], zm = A.m[8];
    const unsigned nz = (unsigned)G.n[2];
    const float len = R.ray_len;
    // Without the uniform walk's clipping of the cell ends, pass 2 also
    // walks the cell holding a lane's own entry (when it enters after the
    // first cell's start, t_start) and the one holding its exit (for every
    // live lane: the last cell may end past even the latest exit).
    bool pend_enter = R.live && t_enter > t_start, pend_exit = R.live;

    const float* vol[NB];
    float* vout[NB];
    float sum[NB], yl[NB];
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        const int64_t b = b0 + (j < nb ? j : nb - 1);
        vol[j] = ADJ ? nullptr : pin_ptr(in + b * nvox);
        vout[j] = ADJ ? pin_ptr(acc.at(out, b * nvox)) : nullptr;
        sum[j] = 0.f;
        yl[j] = __fmul_rn(y[j], len);  // adjoint: y * |v|, times each parameter span
    }
    const uint64_t pol = l2_policy_keep();
    // one segment of voxel v and parameter span w into every volume
    auto charge = [&](int v, float w, bool use) {
#pragma unroll
        for (int j = 0; j < NB; ++j) {
            if constexpr (ADJ) {
                acc.add(vout[j], (unsigned)v, __fmul_rn(yl[j], w), use && (NB == 1 || j < nb));
            } else {
                if (use) sum[j] = __fmaf_rn(ld_keep(vol[j] + (unsigned)v, pol), w, sum[j]);
            }
        }
    };
    // k of the rounded midpoint at tm (this lane's z line)
    auto k_at = [&](float tm) { return rne_int(__fmul_rn(zm, __fsub_rn(__fmaf_rn(tm, zv, zs0), zb))); };

    // ---- segments just before the entry (spans: edge_segments with |v| = 1)
    if (R.live) {
        float p0[3], ps[3], el[kEdge];
        int ev[kEdge];
        edge_planes<-1>(R, t_enter, G, p0, ps);
        const int ne = edge_segments<3, -1, true>(A, sw, vw, R.s, R.inv, ps, p0, t_enter, 1.f, G, ev, el);
#pragma unroll
        for (int k = kEdge - 1; k >= 0; --k) charge(ev[k], el[k], k < ne && el[k] > 0.f);
    }

    const float fl = (float)lane;
    const int max_rounds = (G.n[0] + G.n[1] + 2) / W + 2;
    const int max_steps = W + G.n[2] + 4;  // pass-2 cells of a round: at most one per z plane, entry and exit
    constexpr int kGF = W == 16 ? CTLAB_MID_GROUP_FWD16 : CTLAB_MID_GROUP_FWD;
    constexpr int kNG = ADJ ? CTLAB_MID_GROUP_ADJ : (kGF / NB > 0 ? kGF / NB : 1);
    static_assert(W % kNG == 0, "pass-1 steps must tile the round's cells");
    const bool uniform = __all_sync(kFullMask, R.live && R.t_enter == t_start && R.t_exit == t_stop);
    float carry = t_start;  // start of the round's first cell
    auto rounds = [&](auto uni_tag) {
        constexpr bool UNI = decltype(uni_tag)::value;
        bool fin = false;  // W = 16: this group has walked its last cell
#pragma unroll 1
        for (int round = 0; round < max_rounds; ++round) {
            float tx = i0 != 0.f ? plane_t(__fmaf_rn(fl, psx, pnx), s0, i0) : kInf;
            float ty = i1 != 0.f ? plane_t(__fmaf_rn(fl, psy, pny), s1, i1) : kInf;
            int ky, kx;
            xy_merge_ranks<W>(tx, ty, i0 != 0.f && i1 != 0.f, s0, s1, va0, va1, pnx, pny, psx, psy, kx, ky);
            const int rx = lane + ky;
            const int ry = lane + kx;
            if (UNI) {  // cell ends past the common exit are the exit
                tx = fminf(tx, t_stop);
                ty = fminf(ty, t_stop);
            }
            if (rx < W) raw[rx] = tx;
            if (ry < W) raw[ry] = ty;
            const int n_x = __popc(__ballot_sync(kFullMask, rx < W) & gmask);
            __syncwarp();
            const float c1 = raw[lane];
            const float r0 = carry;
            const float c0 = lane == 0 ? r0 : raw[lane - 1];
            const int n_in = __popc(__ballot_sync(kFullMask, c1 < t_stop) & gmask);
            const int n_cells = (W == 16 && fin) ? 0 : min(n_in + 1, W);
            carry = __shfl_sync(kFullMask, c1, (wlane & (32 - W)) + W - 1);
            {  // the record of this lane's cell
                const float tm = __fmul_rn(0.5f, __fadd_rn(c0, c1));
                const int i = rne_int(__fmul_rn(A.m[0], __fsub_rn(__fmaf_rn(tm, lvx, sx), A.b[0])));
                const int j = rne_int(__fmul_rn(A.m[4], __fsub_rn(__fmaf_rn(tm, lvy, sy), A.b[1])));
                // (cells past the round's last walk nothing: col -1 for them too)
                const bool in = (unsigned)i < (unsigned)G.n[0] && (unsigned)j < (unsigned)G.n[1] && lane < n_cells;
                rec[lane] = MidCell{c1, in ? i * G.stride[0] + j * G.stride[1] : -1, tm, __fsub_rn(c1, c0)};
            }
            __syncwarp();
            // ---- pass 1: whole cells, in step -------------------------------
            float p0 = r0;  // start of the step's first cell
#pragma unroll 1
            for (int q = 0; q < n_cells; q += kNG) {
                int vq[kNG];
                float wq[kNG];
                bool uq[kNG];
#pragma unroll
                for (int u = 0; u < kNG; ++u) {
                    const MidCell c = rec[q + u];  // q + u < W: kNG divides W
                    const int k = k_at(c.tm);
                    bool use = c.col >= 0 && (unsigned)k < nz;
                    if (!UNI) use = use && p0 >= t_enter && c.t <= t_exit;
                    // index and span are read only where `use` holds (an unused
                    // cell's span may be inf - inf; no select is spent on it)
                    vq[u] = (int)((unsigned)c.col + (unsigned)k);
                    wq[u] = c.span;
                    uq[u] = use;
                    p0 = c.t;
                }
                if constexpr (ADJ) {
#pragma unroll
                    for (int u = 0; u < kNG; ++u) charge(vq[u], wq[u], uq[u]);
                } else {
                    float vv[NB][kNG];
#pragma unroll
                    for (int j = 0; j < NB; ++j)
#pragma unroll
                        for (int u = 0; u < kNG; ++u) vv[j][u] = uq[u] ? ld_keep(vol[j] + (unsigned)vq[u], pol) : 0.f;
#pragma unroll
                    for (int j = 0; j < NB; ++j)
#pragma unroll
                        for (int u = 0; u < kNG; ++u) sum[j] = uq[u] ? __fmaf_rn(vv[j][u], wq[u], sum[j]) : sum[j];
                }
            }
            // ---- pass 2: this lane's cells with a z plane, entry or exit inside
            // (the loop and its vote are taken by the whole warp: with W = 16
            // a finished group has no cells, an empty range and no work)
            {
                const float r1 = n_cells > 0 ? raw[n_cells - 1] : -kInf;  // end of the round's last cell
#pragma unroll 1
                for (int it = 0; it < max_steps; ++it) {
                    float bp = tnz < t_exit ? tnz : kInf;
                    if (!UNI) {
                        bp = pend_enter ? fminf(bp, t_enter) : bp;
                        bp = pend_exit ? fminf(bp, t_exit) : bp;
                    }
                    const bool work = bp < r1;
                    if (!__any_sync(kFullMask, work)) break;
                    if (work) {
                        const int q = count_le<W>(raw, bp);  // the cell holding bp: c0 <= bp < c1
                        const float e0 = q == 0 ? r0 : raw[q - 1], e1 = raw[q];
                        const float lo = UNI ? e0 : fmaxf(e0, t_enter), hi = UNI ? e1 : fminf(e1, t_exit);
                        // pass 1's whole-cell term of this cell, if it charged one
                        // (the forward looks it up first, to fold it into a piece)
                        auto cell_term = [&](MidCell& c) {
                            c = rec[q];
                            const int k = k_at(c.tm);
                            bool f = c.col >= 0 && (unsigned)k < nz;
                            if (!UNI) f = f && e0 >= t_enter && e1 <= t_exit;
                            return f ? c.col + k : -1;
                        };
                        MidCell c;
                        int v_cell = -1;
                        if constexpr (!ADJ) v_cell = cell_term(c);
                        bool full = v_cell >= 0;
                        // the cell's segments: split at the z planes inside, the last one ending at hi
                        float t = lo;
#pragma unroll 1
                        for (int zs = 0; zs < max_steps; ++zs) {
                            const bool zin = tnz < hi;
                            const float e = zin ? tnz : hi;
                            if (e > t) {
                                const int v = midpoint_voxel_diag(A, sw, vw, t, e, G);
                                const float d = __fsub_rn(e, t);
                                // forward: the take-back folded into this piece's charge
                                const bool back = !ADJ && full && v == v_cell;
                                charge(v, back ? __fsub_rn(d, c.span) : d, v >= 0);
                                full = full && !back;
                                t = e;
                            }
                            if (!zin) break;
                            pnz += psz;
                            tnz = plane_t(pnz, s2, i2);
                        }
                        // take back pass 1's whole-cell term (if not folded)
                        if constexpr (ADJ) {
                            v_cell = cell_term(c);
                            full = v_cell >= 0;
                        }
                        charge(full ? v_cell : 0, -c.span, full);
                        if (!UNI) {
                            pend_enter = pend_enter && !(t_enter < e1);
                            pend_exit = pend_exit && !(t_exit <= e1);
                        }
                    }
                }
            }
            if constexpr (W == 32) {
                if (n_in < W) break;
            } else {
                fin = fin || n_in < W;
                if (__all_sync(kFullMask, fin)) break;
            }
            __syncwarp();  // every lane is done with this round's records
            if (W == 32 || !fin) {
                pnx = __fmaf_rn((float)n_x, psx, pnx);
                pny = __fmaf_rn((float)(W - n_x), psy, pny);
            }
        }
    };
#if CTLAB_XY_UNIFORM
    if (uniform) rounds(std::true_type{});
    else
#else
    (void)uniform;
#endif
        rounds(std::false_type{});

    // ---- segments just after the exit ----------------------------------------
    if (R.live) {
        float p0[3], ps[3], el[kEdge];
        int ev[kEdge];
        edge_planes<1>(R, t_exit, G, p0, ps);
        const int ne = edge_segments<3, 1, true>(A, sw, vw, R.s, R.inv, ps, p0, t_exit, 1.f, G, ev, el);
#pragma unroll
        for (int k = 0; k < kEdge; ++k) charge(ev[k], el[k], k < ne && el[k] > 0.f);
    }
    if constexpr (!ADJ) {
        if (r >= 0) {
#pragma unroll
            for (int j = 0; j < NB; ++j)
                if (j < nb) st_stream(out + (b0 + j) * n_ray + r, __fmul_rn(sum[j], len));
        }
    }
}

}  // namespace ctlab
