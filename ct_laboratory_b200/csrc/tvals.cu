// tvals.cu — projectors driven by an intersection table, the table builders,
// the uint16 compressor and the 2-D incremental-march kernels.
//
// Layout: the reference's tables are row-major [n_ray, n_int]
// (ct_projector_3d.cu:117, :290), one row per ray, and its kernels give each
// thread a whole row; the projectors here do the same (one lane per ray, the
// row read front to back through the L1, segments added in the reference's
// order), but skip the entries past a row's last hit at the cost of a load
// and a compare each, and take the row in blocks of kTableBlock entries:
// the block's loads are in flight together and, in the forward, so are its
// volume gathers, added afterwards in the row's order (block 8 against 1:
// 7.1 against 11.3 ms for the uint16 forward below, bitwise the same).  A warp that owned one ray, its lanes taking
// consecutive segments (coalesced row loads, a warp scan for the uint16
// decode, a warp reduction for the sum), measured slower on a 2.9 M-ray
// StaticCT scan (14.2 / 12.4 ms against 10.0 / 10.3 ms forward / adjoint from
// the uint16 table): its 32 lanes gather from 32 voxels strung along one ray,
// where neighbouring lanes on neighbouring detector rows share most of their
// x-y path.  The table builders keep a warp per ray.
#include "common.cuh"

namespace ctlab {

constexpr int kWarpsPerBlock = 8;

// Per-segment work of the reference's table kernels: world end points
// s + t*v, world segment length, rounded midpoint voxel
// (3-D: ct_projector_3d.cu:297-313; 2-D: ct_projector_2d.cu:99-108, whose
// length is hypotf).  Returns the flat voxel index or -1.
template <int NDIM>
__device__ __forceinline__ int seg_world(const float* sw, const float* vw, float t0, float t1, const int* n,
                                         const Affine3& A3, const Affine2& A2, float& len) {
    float p0[NDIM], p1[NDIM];
#pragma unroll
    for (int a = 0; a < NDIM; ++a) {
        p0[a] = __fmaf_rn(t0, vw[a], sw[a]);
        p1[a] = __fmaf_rn(t1, vw[a], sw[a]);
    }
    float f[NDIM];
    if constexpr (NDIM == 3) {
        len = sqrtf(sumsq3(__fsub_rn(p1[0], p0[0]), __fsub_rn(p1[1], p0[1]), __fsub_rn(p1[2], p0[2])));
        world_to_index3(A3, __fmul_rn(0.5f, __fadd_rn(p0[0], p1[0])), __fmul_rn(0.5f, __fadd_rn(p0[1], p1[1])),
                        __fmul_rn(0.5f, __fadd_rn(p0[2], p1[2])), f[0], f[1], f[2]);
    } else {
        len = hypotf(__fsub_rn(p1[0], p0[0]), __fsub_rn(p1[1], p0[1]));
        world_to_index2(A2, __fmul_rn(0.5f, __fadd_rn(p0[0], p1[0])), __fmul_rn(0.5f, __fadd_rn(p0[1], p1[1])),
                        f[0], f[1]);
    }
    int flat = 0;
#pragma unroll
    for (int a = 0; a < NDIM; ++a) {
        const int i = __float2int_rn(f[a]);
        if (i < 0 || i >= n[a]) return -1;
        flat = flat * n[a] + i;
    }
    return flat;
}

struct Dims {
    int n[3];
};

// ----------------------------------------------------------------------------
// Lane-per-ray table projectors.  Each lane walks its own row front to back,
// as the reference's kernels do (ct_projector_3d.cu:117-160, :290-330), and
// adds its segments in the reference's order.  The row entries past the last
// hit cost next to nothing: a float row ends at its first +inf (rows are
// sorted, so the rest is +inf too); a uint16 delta of 0 (an +inf entry or a
// tie) leaves t unchanged, a zero-length segment the reference skips as well,
// so the lane moves straight to the next entry.  Rows are read through the
// L1 (each lane's 32-byte sector serves 8 float or 16 uint16 entries), and a
// lane's gathers / reductions are those of one ray.
// ----------------------------------------------------------------------------
// Row entries loaded (and, in the forward, volume gathers issued) per block.
#ifndef CTLAB_TABLE_BLOCK
#define CTLAB_TABLE_BLOCK 8
#endif
constexpr int kTableBlock = CTLAB_TABLE_BLOCK;
// The compressed kernels load the next block's deltas before working the
// current block (their latency hidden behind its arithmetic; the static
// ring's uint16 forward 6.94 against 7.12 ms): 1, or each block when it is
// reached: 0.
#ifndef CTLAB_TABLE_PREFETCH
#define CTLAB_TABLE_PREFETCH 1
#endif

template <int NDIM, bool ADJ>
__global__ void __launch_bounds__(256) tvals_lane_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                         const float* __restrict__ tvals, int n_int,
                                                         const float* __restrict__ src,
                                                         const float* __restrict__ dst, int64_t n_ray,
                                                         const float* __restrict__ M_inv,
                                                         const float* __restrict__ bvec, Dims D, int64_t nvox) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_ray) return;
    const int64_t bi = blockIdx.y;
    Affine3 A3;
    Affine2 A2;
    if constexpr (NDIM == 3) A3 = load_affine3(M_inv, bvec);
    else A2 = load_affine2(M_inv, bvec);
    float sw[NDIM], vw[NDIM];
#pragma unroll
    for (int a = 0; a < NDIM; ++a) {
        sw[a] = __ldg(src + r * NDIM + a);
        vw[a] = __fsub_rn(__ldg(dst + r * NDIM + a), sw[a]);
    }
    float y = 0.f;
    if constexpr (ADJ) {
        y = __ldg(in + bi * n_ray + r);
        if (y == 0.f) return;
    }
    const float* row = tvals + r * n_int;
    const float* vol = in + bi * nvox;
    float* vout = out + bi * nvox;
    float acc = 0.f;
    float t0 = __ldg(row);
    bool more = !isinf(t0);
    // A block's entries are loaded together (kTableBlock loads in flight).
    // The next block is loaded at the end of an iteration, where its loads
    // do not wait for this block's accumulation (the static ring's forward:
    // 6.64 ms, against 7.25 with the next block loaded before the current
    // one is worked and about 7.4 with each block loaded at the top of its
    // iteration).
    auto load_block = [&](int i, float* tb) {
#pragma unroll
        for (int q = 0; q < kTableBlock; ++q) tb[q] = (i + q < n_int) ? __ldg(row + i + q) : __int_as_float(0x7f800000);
    };
    float tb[kTableBlock];
    load_block(1, tb);
#pragma unroll 1
    for (int i0 = 1; i0 < n_int && more; i0 += kTableBlock) {
        int vq[kTableBlock];
        float lq[kTableBlock];
#pragma unroll
        for (int q = 0; q < kTableBlock; ++q) {
            // a row is sorted: past its first +inf there is nothing left
            const bool ok = more && !isinf(tb[q]);
            more = ok;
            lq[q] = 0.f;
            vq[q] = -1;
            if (ok) {
                vq[q] = seg_world<NDIM>(sw, vw, t0, tb[q], D.n, A3, A2, lq[q]);
                t0 = tb[q];
            }
        }
        if constexpr (ADJ) {
#pragma unroll
            for (int q = 0; q < kTableBlock; ++q)
                if (vq[q] >= 0) atomicAdd(vout + vq[q], __fmul_rn(y, lq[q]));
        } else {
            float g[kTableBlock];
#pragma unroll
            for (int q = 0; q < kTableBlock; ++q)
                if (vq[q] >= 0) g[q] = __ldg(vol + vq[q]);
#pragma unroll
            for (int q = 0; q < kTableBlock; ++q)
                if (vq[q] >= 0) acc = __fmaf_rn(g[q], lq[q], acc);
        }
        load_block(i0 + kTableBlock, tb);
    }
    if constexpr (!ADJ) out[bi * n_ray + r] = acc;
}

template <bool ADJ>
__global__ void __launch_bounds__(256) compressed_lane_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                              const uint16_t* __restrict__ tq,
                                                              const float* __restrict__ t_start,
                                                              const float* __restrict__ t_scale, int n_int,
                                                              const float* __restrict__ src,
                                                              const float* __restrict__ dst, int64_t n_ray,
                                                              const float* __restrict__ M_inv,
                                                              const float* __restrict__ bvec, Dims D, int64_t nvox) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_ray) return;
    const int64_t bi = blockIdx.y;
    const Affine3 A = load_affine3(M_inv, bvec);
    float sw[3], vw[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        sw[a] = __ldg(src + r * 3 + a);
        vw[a] = __fsub_rn(__ldg(dst + r * 3 + a), sw[a]);
    }
    float y = 0.f;
    if constexpr (ADJ) {
        y = __ldg(in + bi * n_ray + r);
        if (y == 0.f) return;
    }
    const float start = __ldg(t_start + r), scale = __ldg(t_scale + r);
    const uint16_t* row = tq + r * n_int;
    const float* vol = in + bi * nvox;
    float* vout = out + bi * nvox;
    float acc = 0.f;
    // world point of the current segment start: t0 = start (ct_projector_3d.cu:129)
    float p0[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) p0[a] = __fmaf_rn(start, vw[a], sw[a]);
    unsigned k = 0;  // running sum of the deltas, in unsigned int as the reference
    // a block's deltas are loaded together (kTableBlock loads in flight)
    auto load_block = [&](int i, unsigned* d) {
#pragma unroll
        for (int q = 0; q < kTableBlock; ++q) d[q] = (i + q < n_int) ? (unsigned)__ldg(row + i + q) : 0u;
    };
    unsigned d[kTableBlock];
    load_block(1, d);
#pragma unroll 1
    for (int i0 = 1; i0 < n_int; i0 += kTableBlock) {
#if CTLAB_TABLE_PREFETCH
        unsigned dn[kTableBlock];
        load_block(i0 + kTableBlock, dn);
#endif
        unsigned any = 0u;
#pragma unroll
        for (int q = 0; q < kTableBlock; ++q) any |= d[q];
        // any == 0: t unchanged over the block (past the last hit), nothing to add
        if (any != 0u) {
        int vq[kTableBlock];
        float lq[kTableBlock];
#pragma unroll
        for (int q = 0; q < kTableBlock; ++q) {
            vq[q] = -1;
            lq[q] = 0.f;
            if (d[q] == 0u) continue;  // t1 == t0: a zero-length segment
            k += d[q];
            const float t1 = __fmaf_rn(__uint2float_rn(k), scale, start);
            float p1[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) p1[a] = __fmaf_rn(t1, vw[a], sw[a]);
            const float len =
                sqrtf(sumsq3(__fsub_rn(p1[0], p0[0]), __fsub_rn(p1[1], p0[1]), __fsub_rn(p1[2], p0[2])));
            if (len >= 1e-9f) {  // ct_projector_3d.cu:137
                float f[3];
                world_to_index3(A, __fmul_rn(0.5f, __fadd_rn(p0[0], p1[0])),
                                __fmul_rn(0.5f, __fadd_rn(p0[1], p1[1])), __fmul_rn(0.5f, __fadd_rn(p0[2], p1[2])),
                                f[0], f[1], f[2]);
                const int ii = __float2int_rn(f[0]), jj = __float2int_rn(f[1]), kk = __float2int_rn(f[2]);
                if ((unsigned)ii < (unsigned)D.n[0] && (unsigned)jj < (unsigned)D.n[1] &&
                    (unsigned)kk < (unsigned)D.n[2]) {
                    vq[q] = (ii * D.n[1] + jj) * D.n[2] + kk;
                    lq[q] = len;
                }
            }
#pragma unroll
            for (int a = 0; a < 3; ++a) p0[a] = p1[a];
        }
        if constexpr (ADJ) {
#pragma unroll
            for (int q = 0; q < kTableBlock; ++q)
                if (vq[q] >= 0) atomicAdd(vout + vq[q], __fmul_rn(y, lq[q]));
        } else {
            // gathers issued together, then added in the row's order
            float g[kTableBlock];
#pragma unroll
            for (int q = 0; q < kTableBlock; ++q)
                if (vq[q] >= 0) g[q] = __ldg(vol + vq[q]);
#pragma unroll
            for (int q = 0; q < kTableBlock; ++q)
                if (vq[q] >= 0) acc = __fmaf_rn(g[q], lq[q], acc);
        }
        }
#if CTLAB_TABLE_PREFETCH
#pragma unroll
        for (int q = 0; q < kTableBlock; ++q) d[q] = dn[q];
#else
        load_block(i0 + kTableBlock, d);
#endif
    }
    if constexpr (!ADJ) out[bi * n_ray + r] = acc;
}

// ----------------------------------------------------------------------------
// Intersection tables (one warp per ray).  The reference computes every plane
// parameter t = (p - s)/dir with a true division (ct_projector_3d.cu:68),
// maps those outside [0,1] to +inf and bubble-sorts the row (:90-95), which
// is stable: equal values keep x, y, z order.  Each axis's in-range planes
// form one contiguous run whose parameters are monotone, so the sorted row
// is a stable merge of at most three runs.  Each lane takes elements of the
// runs, computes the element's merged position (its rank in its own run plus
// the number of elements of the other runs before it, found by binary
// search) and stores it there; the tail is filled with +inf.
// ----------------------------------------------------------------------------
struct Run {
    float s, dir;  // index-space start and direction of this axis
    int first;     // plane index of the run's first (smallest-t) element
    int step;      // +1 or -1: plane index step along ascending t
    int count;     // number of elements
};

__device__ __forceinline__ float run_t(const Run& R, int q) {
    const float p = (float)(R.first + q * R.step) - 0.5f;
    return __fdiv_rn(__fsub_rn(p, R.s), R.dir);
}

// Elements of run R with t <= x (inclusive) or t < x.
__device__ __forceinline__ int run_count(const Run& R, float x, bool inclusive) {
    int lo = 0, hi = R.count;  // answer in [lo, hi]
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const float t = run_t(R, mid);
        const bool before = inclusive ? (t <= x) : (t < x);
        if (before) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ Run make_run(float s, float d, int n) {
    Run R;
    R.s = s;
    R.dir = __fsub_rn(d, s);
    R.count = 0;
    R.first = 0;
    R.step = 1;
    if (!(fabsf(R.dir) >= 1e-12f)) return R;  // ct_projector_3d.cu:66 (and NaN)
    // Planes p_k = k - 0.5, k = 0..n; t_k monotone in k.  In-range k form a
    // contiguous interval; find its ends from estimates plus exact checks.
    auto tk = [&](int k) { return __fdiv_rn(__fsub_rn((float)k - 0.5f, R.s), R.dir); };
    auto ok = [&](int k) {
        const float t = tk(k);
        return !(t < 0.f || t > 1.f);
    };
    // Coordinates spanned by t in [0,1]: [min(s,d), max(s,d)].
    const float cmin = fminf(s, d), cmax = fmaxf(s, d);
    int klo = (int)fmaxf(0.f, fminf((float)n, floorf(cmin + 0.5f)));
    int khi = (int)fmaxf(0.f, fminf((float)n, floorf(cmax + 0.5f)));
    // widen by one on each side, then shrink to exactly the valid set
    klo = max(klo - 1, 0);
    khi = min(khi + 1, n);
    int guard = 0;
    while (klo <= khi && !ok(klo) && guard++ < 8) ++klo;
    guard = 0;
    while (khi >= klo && !ok(khi) && guard++ < 8) --khi;
    if (klo > khi || !ok(klo) || !ok(khi)) return R;
    // extend outwards in case the estimate was short
    guard = 0;
    while (klo > 0 && ok(klo - 1) && guard++ < 8) --klo;
    guard = 0;
    while (khi < n && ok(khi + 1) && guard++ < 8) ++khi;
    R.count = khi - klo + 1;
    if (R.dir > 0.f) {
        R.first = klo;
        R.step = 1;
    } else {
        R.first = khi;
        R.step = -1;
    }
    return R;
}

template <int NDIM>
__global__ void __launch_bounds__(256) intersections_kernel(const float* __restrict__ src,
                                                            const float* __restrict__ dst, int64_t n_ray,
                                                            const float* __restrict__ M_inv,
                                                            const float* __restrict__ bvec, Dims D, int n_int,
                                                            float* __restrict__ t_out) {
    const int lane = threadIdx.x & 31;
    const int64_t r = (int64_t)blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
    if (r >= n_ray) return;
    float s[3] = {0.f, 0.f, 0.f}, d[3] = {0.f, 0.f, 0.f};
    if constexpr (NDIM == 3) {
        const Affine3 A = load_affine3(M_inv, bvec);
        world_to_index3(A, __ldg(src + 3 * r), __ldg(src + 3 * r + 1), __ldg(src + 3 * r + 2), s[0], s[1], s[2]);
        world_to_index3(A, __ldg(dst + 3 * r), __ldg(dst + 3 * r + 1), __ldg(dst + 3 * r + 2), d[0], d[1], d[2]);
    } else {
        const Affine2 A = load_affine2(M_inv, bvec);
        world_to_index2(A, __ldg(src + 2 * r), __ldg(src + 2 * r + 1), s[0], s[1]);
        world_to_index2(A, __ldg(dst + 2 * r), __ldg(dst + 2 * r + 1), d[0], d[1]);
    }
    Run R[NDIM];
    int offs[NDIM + 1];
    offs[0] = 0;
#pragma unroll
    for (int a = 0; a < NDIM; ++a) {
        R[a] = make_run(s[a], d[a], D.n[a]);
        offs[a + 1] = offs[a] + R[a].count;
    }
    const int total = offs[NDIM];
    float* row = t_out + r * n_int;
    for (int e = lane; e < total; e += 32) {
        int a = 0;
#pragma unroll
        for (int q = 1; q < NDIM; ++q)
            if (e >= offs[q]) a = q;
        const int q = e - offs[a];
        const float t = run_t(R[a], q);
        int rank = q;
#pragma unroll
        for (int bx = 0; bx < NDIM; ++bx) {
            if (bx == a) continue;
            rank += run_count(R[bx], t, bx < a);
        }
        row[rank] = t;
    }
    const float kInf = __int_as_float(0x7f800000);
    for (int e = total + lane; e < n_int; e += 32) row[e] = kInf;
}

// ----------------------------------------------------------------------------
// uint16 compressor (thread per ray).  Two encoders exist in the reference
// and they disagree, so both are provided:
//  mode 0: compress_tvals_3d_kernel (ct_projector_3d.cu:160-212): start = t[0]
//          as stored, inf entries encode 0, k = roundf (half away from 0),
//          running sum in unsigned int;
//  mode 1: compress_tvals_to_uint16 (ct_projector_3d_torch.py:4-65): inf is
//          replaced by 10.0 first (start included), k = round half to even,
//          running sum in float.  The length |dst-src| is fused as the CPU
//          torch.norm computes it, sqrt(fma(z,z,fma(y,y,x*x))).
// Both: scale = (voxel_diag/10000)/max(|dst-src|, 1e-6), delta clamped to
// [0, 32000].
// ----------------------------------------------------------------------------
template <int MODE>
__global__ void __launch_bounds__(256) compress_kernel(const float* __restrict__ tvals, int64_t n_ray, int n_int,
                                                       const float* __restrict__ src,
                                                       const float* __restrict__ dst, float voxel_diag_len,
                                                       uint16_t* __restrict__ tq, float* __restrict__ t_start,
                                                       float* __restrict__ t_scale) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_ray) return;
    const float dx = __fsub_rn(__ldg(dst + 3 * r), __ldg(src + 3 * r));
    const float dy = __fsub_rn(__ldg(dst + 3 * r + 1), __ldg(src + 3 * r + 1));
    const float dz = __fsub_rn(__ldg(dst + 3 * r + 2), __ldg(src + 3 * r + 2));
    const float len2 = MODE == 0 ? sumsq3(dx, dy, dz) : __fmaf_rn(dz, dz, __fmaf_rn(dy, dy, __fmul_rn(dx, dx)));
    const float ray_len = fmaxf(sqrtf(len2), 1e-6f);
    const float scale = __fdiv_rn(__fdiv_rn(voxel_diag_len, 10000.0f), ray_len);
    t_scale[r] = scale;
    const float* row = tvals + r * n_int;
    uint16_t* q = tq + r * n_int;
    float start = __ldg(row);
    if (MODE == 1 && isinf(start)) start = 10.0f;
    t_start[r] = start;
    q[0] = 0;
    const float inv = __frcp_rn(scale);
    unsigned prev = 0;
    float prev_f = 0.f;
    for (int i = 1; i < n_int; ++i) {
        float t = __ldg(row + i);
        if constexpr (MODE == 0) {
            if (isinf(t)) {
                q[i] = 0;
                continue;
            }
            const unsigned cur = __float2uint_rz(roundf(__fmul_rn(__fsub_rn(t, start), inv)));
            int diff = (int)cur - (int)prev;
            diff = min(max(diff, 0), 32000);
            q[i] = (uint16_t)diff;
            prev += (unsigned)diff;
        } else {
            if (isinf(t)) t = 10.0f;
            const float cur = rintf(__fmul_rn(__fsub_rn(t, start), inv));
            const float diff = fminf(fmaxf(__fsub_rn(cur, prev_f), 0.f), 32000.f);
            const uint16_t dq = (uint16_t)__float2int_rz(diff);
            q[i] = dq;
            prev_f = __fadd_rn(prev_f, (float)dq);
        }
    }
}

// ----------------------------------------------------------------------------
// 2-D incremental march (thread per ray), the reference's on-the-fly 2-D
// kernels (ct_projector_2d.cu:246-413): slab entry/exit, floor/ceil start
// pixel, t_next += dt, hypot length.  Kept as written there so the `_C`
// entry points behave like the reference's.
// ----------------------------------------------------------------------------
template <bool ADJ>
__global__ void __launch_bounds__(256) march2d_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                      const float* __restrict__ src, const float* __restrict__ dst,
                                                      int64_t n_ray, const float* __restrict__ M_inv,
                                                      const float* __restrict__ bvec, int n_row, int n_col) {
    const int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_ray) return;
    const int64_t bi = blockIdx.y;
    const int64_t npix = (int64_t)n_row * n_col;
    const float sx = __ldg(src + 2 * r), sy = __ldg(src + 2 * r + 1);
    const float vx = __fsub_rn(__ldg(dst + 2 * r), sx), vy = __fsub_rn(__ldg(dst + 2 * r + 1), sy);
    const float ray_len = hypotf(vx, vy);
    float acc = 0.f;
    float y = 0.f;
    if constexpr (ADJ) {
        y = __ldg(in + bi * n_ray + r);
        if (y == 0.f) return;
    }
    if (ray_len >= 1e-12f) {
        const Affine2 A = load_affine2(M_inv, bvec);
        float sr, sc, dr, dc;
        world_to_index2(A, sx, sy, sr, sc);
        world_to_index2(A, __ldg(dst + 2 * r), __ldg(dst + 2 * r + 1), dr, dc);
        const float vr = __fsub_rn(dr, sr), vc = __fsub_rn(dc, sc);
        const float inv_r = (fabsf(vr) < 1e-12f) ? 1e32f : __frcp_rn(vr);
        const float inv_c = (fabsf(vc) < 1e-12f) ? 1e32f : __frcp_rn(vc);
        const float tr0 = __fmul_rn(__fsub_rn(-0.5f, sr), inv_r);
        const float tr1 = __fmul_rn(__fsub_rn((float)n_row - 0.5f, sr), inv_r);
        const float tc0 = __fmul_rn(__fsub_rn(-0.5f, sc), inv_c);
        const float tc1 = __fmul_rn(__fsub_rn((float)n_col - 0.5f, sc), inv_c);
        float t_enter = fmaxf(fminf(tr0, tr1), fminf(tc0, tc1));
        float t_exit = fminf(fmaxf(tr0, tr1), fmaxf(tc0, tc1));
        if (t_exit > t_enter) {
            t_enter = fmaxf(t_enter, 0.f);
            t_exit = fminf(t_exit, 1.f);
            const float r_en = __fmaf_rn(t_enter, vr, sr), c_en = __fmaf_rn(t_enter, vc, sc);
            int ri = (vr >= 0.f) ? (int)floorf(r_en) : (int)ceilf(r_en) - 1;
            int ci = (vc >= 0.f) ? (int)floorf(c_en) : (int)ceilf(c_en) - 1;
            float tnr = __fmaf_rn(__fsub_rn((float)ri + (vr >= 0.f ? 0.5f : -0.5f), r_en), inv_r, t_enter);
            float tnc = __fmaf_rn(__fsub_rn((float)ci + (vc >= 0.f ? 0.5f : -0.5f), c_en), inv_c, t_enter);
            const float dtr = fabsf(inv_r), dtc = fabsf(inv_c);
            const int sr_step = vr >= 0.f ? 1 : -1, sc_step = vc >= 0.f ? 1 : -1;
            float t_cur = t_enter;
            const float* img = in + bi * npix;
            float* iout = out + bi * npix;
            // The march ends when t reaches t_exit; the pixel count bounds it.
            const int max_it = n_row + n_col + 4;
            for (int it = 0; it < max_it && t_cur < t_exit; ++it) {
                const bool step_row = tnr < tnc;
                const float t_hit = fminf(step_row ? tnr : tnc, t_exit);
                if (ri >= 0 && ri < n_row && ci >= 0 && ci < n_col) {
                    const float seg = __fmul_rn(__fsub_rn(t_hit, t_cur), ray_len);
                    const int idx = ri * n_col + ci;
                    if constexpr (ADJ) atomicAdd(iout + idx, __fmul_rn(y, seg));
                    else acc = __fmaf_rn(__ldg(img + idx), seg, acc);
                }
                t_cur = t_hit;
                if (step_row) {
                    tnr = __fadd_rn(tnr, dtr);
                    ri += sr_step;
                } else {
                    tnc = __fadd_rn(tnc, dtc);
                    ci += sc_step;
                }
            }
        }
    }
    if constexpr (!ADJ) out[bi * n_ray + r] = acc;
}

// ----------------------------------------------------------------------------
// host side
// ----------------------------------------------------------------------------
static int check_grid(const char* what, int ndim, const int64_t* dims, Dims& D, int64_t& nvox) {
    nvox = 1;
    for (int a = 0; a < ndim; ++a) {
        CTLAB_REQUIRE(dims[a] >= 1 && dims[a] <= (1 << 22), "%s: grid dimension %d out of range (%lld)", what, a,
                      (long long)dims[a]);
        D.n[a] = (int)dims[a];
        nvox *= dims[a];
    }
    for (int a = ndim; a < 3; ++a) D.n[a] = 1;
    CTLAB_REQUIRE(nvox < (1LL << 31), "%s: %lld voxels exceed 2^31", what, (long long)nvox);
    return CTLAB_OK;
}

constexpr int kLaneThreads = 128;

// One thread per ray, kLaneThreads per block.
static int lane_grid(const char* what, int64_t n_ray, int64_t batch, dim3& grid) {
    CTLAB_REQUIRE(n_ray >= 0, "%s: n_ray must be >= 0", what);
    CTLAB_REQUIRE(batch >= 1 && batch <= 65535, "%s: batch must be in [1, 65535]", what);
    const int64_t blocks = (n_ray + kLaneThreads - 1) / kLaneThreads;
    CTLAB_REQUIRE(blocks <= kMaxGrid, "%s: too many rays", what);
    grid = dim3((unsigned)blocks, (unsigned)batch);
    return CTLAB_OK;
}

static int warp_grid(const char* what, int64_t n_ray, int64_t batch, dim3& grid) {
    CTLAB_REQUIRE(n_ray >= 0, "%s: n_ray must be >= 0", what);
    CTLAB_REQUIRE(batch >= 1 && batch <= 65535, "%s: batch must be in [1, 65535]", what);
    const int64_t blocks = (n_ray + kWarpsPerBlock - 1) / kWarpsPerBlock;
    CTLAB_REQUIRE(blocks <= kMaxGrid, "%s: too many rays", what);
    grid = dim3((unsigned)blocks, (unsigned)batch);
    return CTLAB_OK;
}

template <int NDIM, bool ADJ>
static int run_tvals(const char* what, const float* in, float* out, int64_t batch, const int64_t* dims,
                     const float* tvals, int64_t n_int, const float* src, const float* dst, int64_t n_ray,
                     const float* M_inv, const float* b, int accumulate, void* stream) {
    Dims D;
    int64_t nvox;
    int rc = check_grid(what, NDIM, dims, D, nvox);
    if (rc) return rc;
    dim3 grid;
    rc = lane_grid(what, n_ray, batch, grid);
    if (rc) return rc;
    CTLAB_REQUIRE(n_int >= 1 && n_int < (1LL << 30), "%s: n_int out of range", what);
    CTLAB_REQUIRE((ADJ ? out : in) && M_inv && b, "%s: null data pointer", what);
    CTLAB_REQUIRE(n_ray == 0 || (tvals && src && dst && (ADJ ? in : out)), "%s: null tvals/src/dst/sinogram", what);
    cudaStream_t s = as_stream(stream);
    if (ADJ && !accumulate) CTLAB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float) * (size_t)(batch * nvox), s));
    if (n_ray == 0) return CTLAB_OK;
    tvals_lane_kernel<NDIM, ADJ><<<grid, kLaneThreads, 0, s>>>(in, out, tvals, (int)n_int, src, dst, n_ray, M_inv, b,
                                                               D, nvox);
    return launch_status(what);
}

template <bool ADJ>
static int run_compressed(const char* what, const float* in, float* out, int64_t batch, const int64_t* dims,
                          const uint16_t* tq, const float* t_start, const float* t_scale, int64_t n_int,
                          const float* src, const float* dst, int64_t n_ray, const float* M_inv, const float* b,
                          int accumulate, void* stream) {
    Dims D;
    int64_t nvox;
    int rc = check_grid(what, 3, dims, D, nvox);
    if (rc) return rc;
    dim3 grid;
    rc = lane_grid(what, n_ray, batch, grid);
    if (rc) return rc;
    CTLAB_REQUIRE(n_int >= 1 && n_int < (1LL << 30), "%s: n_int out of range", what);
    CTLAB_REQUIRE((ADJ ? out : in) && M_inv && b, "%s: null data pointer", what);
    CTLAB_REQUIRE(n_ray == 0 || (tq && t_start && t_scale && src && dst && (ADJ ? in : out)),
                  "%s: null table/src/dst/sinogram", what);
    cudaStream_t s = as_stream(stream);
    if (ADJ && !accumulate) CTLAB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float) * (size_t)(batch * nvox), s));
    if (n_ray == 0) return CTLAB_OK;
    compressed_lane_kernel<ADJ><<<grid, kLaneThreads, 0, s>>>(in, out, tq, t_start, t_scale, (int)n_int, src, dst,
                                                              n_ray, M_inv, b, D, nvox);
    return launch_status(what);
}

template <int NDIM>
static int run_intersections(const char* what, const int64_t* dims, const float* src, const float* dst,
                             int64_t n_ray, const float* M_inv, const float* b, float* t_out, void* stream) {
    Dims D;
    int64_t nvox;
    int rc = check_grid(what, NDIM, dims, D, nvox);
    if (rc) return rc;
    dim3 grid;
    rc = warp_grid(what, n_ray, 1, grid);
    if (rc) return rc;
    int64_t n_int = 0;
    for (int a = 0; a < NDIM; ++a) n_int += dims[a] + 1;
    CTLAB_REQUIRE(M_inv && b && (n_ray == 0 || (src && dst && t_out)), "%s: null pointer", what);
    if (n_ray == 0) return CTLAB_OK;
    intersections_kernel<NDIM><<<grid, 32 * kWarpsPerBlock, 0, as_stream(stream)>>>(src, dst, n_ray, M_inv, b, D,
                                                                                   (int)n_int, t_out);
    return launch_status(what);
}

template <bool ADJ>
static int run_march2d(const char* what, const float* in, float* out, int64_t batch, int64_t n_row, int64_t n_col,
                       const float* src, const float* dst, int64_t n_ray, const float* M_inv, const float* b,
                       int accumulate, void* stream) {
    Dims D;
    int64_t nvox;
    const int64_t dims[2] = {n_row, n_col};
    int rc = check_grid(what, 2, dims, D, nvox);
    if (rc) return rc;
    CTLAB_REQUIRE(n_ray >= 0 && batch >= 1 && batch <= 65535, "%s: bad n_ray/batch", what);
    CTLAB_REQUIRE((ADJ ? out : in) && M_inv && b && (n_ray == 0 || (src && dst && (ADJ ? in : out))),
                  "%s: null pointer", what);
    cudaStream_t s = as_stream(stream);
    if (ADJ && !accumulate) CTLAB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float) * (size_t)(batch * nvox), s));
    if (n_ray == 0) return CTLAB_OK;
    const int64_t blocks = (n_ray + 255) / 256;
    CTLAB_REQUIRE(blocks <= kMaxGrid, "%s: too many rays", what);
    march2d_kernel<ADJ><<<dim3((unsigned)blocks, (unsigned)batch), 256, 0, s>>>(in, out, src, dst, n_ray, M_inv, b,
                                                                               (int)n_row, (int)n_col);
    return launch_status(what);
}

}  // namespace ctlab

using namespace ctlab;

extern "C" int ctlab_compute_intersections_3d(int64_t n_x, int64_t n_y, int64_t n_z, const float* src,
                                              const float* dst, int64_t n_ray, const float* M_inv, const float* b,
                                              float* t_out, void* stream) {
    clear_error();
    const int64_t dims[3] = {n_x, n_y, n_z};
    return run_intersections<3>("compute_intersections_3d", dims, src, dst, n_ray, M_inv, b, t_out, stream);
}

extern "C" int ctlab_compute_intersections_2d(int64_t n_row, int64_t n_col, const float* src, const float* dst,
                                              int64_t n_ray, const float* M_inv, const float* b, float* t_out,
                                              void* stream) {
    clear_error();
    const int64_t dims[2] = {n_row, n_col};
    return run_intersections<2>("compute_intersections_2d", dims, src, dst, n_ray, M_inv, b, t_out, stream);
}

extern "C" int ctlab_forward_project_3d_tvals(const float* volume, int64_t batch, int64_t n_x, int64_t n_y,
                                              int64_t n_z, const float* tvals, int64_t n_int, const float* src,
                                              const float* dst, int64_t n_ray, const float* M_inv, const float* b,
                                              float* out, void* stream) {
    clear_error();
    const int64_t dims[3] = {n_x, n_y, n_z};
    return run_tvals<3, false>("forward_project_3d_tvals", volume, out, batch, dims, tvals, n_int, src, dst, n_ray,
                               M_inv, b, 0, stream);
}

extern "C" int ctlab_back_project_3d_tvals(const float* sino, int64_t batch, int64_t n_ray, const float* tvals,
                                           int64_t n_int, const float* src, const float* dst, const float* M_inv,
                                           const float* b, int64_t n_x, int64_t n_y, int64_t n_z, float* out,
                                           int accumulate, void* stream) {
    clear_error();
    const int64_t dims[3] = {n_x, n_y, n_z};
    return run_tvals<3, true>("back_project_3d_tvals", sino, out, batch, dims, tvals, n_int, src, dst, n_ray, M_inv,
                              b, accumulate, stream);
}

extern "C" int ctlab_forward_project_2d_tvals(const float* image, int64_t batch, int64_t n_row, int64_t n_col,
                                              const float* tvals, int64_t n_int, const float* src, const float* dst,
                                              int64_t n_ray, const float* M_inv, const float* b, float* out,
                                              void* stream) {
    clear_error();
    const int64_t dims[2] = {n_row, n_col};
    return run_tvals<2, false>("forward_project_2d_tvals", image, out, batch, dims, tvals, n_int, src, dst, n_ray,
                               M_inv, b, 0, stream);
}

extern "C" int ctlab_back_project_2d_tvals(const float* sino, int64_t batch, int64_t n_ray, const float* tvals,
                                           int64_t n_int, const float* src, const float* dst, const float* M_inv,
                                           const float* b, int64_t n_row, int64_t n_col, float* out, int accumulate,
                                           void* stream) {
    clear_error();
    const int64_t dims[2] = {n_row, n_col};
    return run_tvals<2, true>("back_project_2d_tvals", sino, out, batch, dims, tvals, n_int, src, dst, n_ray, M_inv,
                              b, accumulate, stream);
}

extern "C" int ctlab_compress_tvals_3d_ex(const float* tvals, int64_t n_ray, int64_t n_int, const float* src,
                                          const float* dst, float voxel_diag_len, uint16_t* t_uint16,
                                          float* t_start, float* t_scale, int mode, void* stream) {
    clear_error();
    CTLAB_REQUIRE(n_ray >= 0 && n_int >= 1 && n_int < (1LL << 30), "compress_tvals_3d: bad n_ray/n_int");
    CTLAB_REQUIRE(mode == CTLAB_COMPRESS_CUDA || mode == CTLAB_COMPRESS_TORCH, "compress_tvals_3d: bad mode %d",
                  mode);
    CTLAB_REQUIRE(n_ray == 0 || (tvals && src && dst && t_uint16 && t_start && t_scale),
                  "compress_tvals_3d: null pointer");
    if (n_ray == 0) return CTLAB_OK;
    const int64_t blocks = (n_ray + 255) / 256;
    CTLAB_REQUIRE(blocks <= kMaxGrid, "compress_tvals_3d: too many rays");
    if (mode == CTLAB_COMPRESS_CUDA)
        compress_kernel<0><<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(tvals, n_ray, (int)n_int, src, dst,
                                                                            voxel_diag_len, t_uint16, t_start,
                                                                            t_scale);
    else
        compress_kernel<1><<<(unsigned)blocks, 256, 0, as_stream(stream)>>>(tvals, n_ray, (int)n_int, src, dst,
                                                                            voxel_diag_len, t_uint16, t_start,
                                                                            t_scale);
    return launch_status("compress_tvals_3d");
}

extern "C" int ctlab_compress_tvals_3d(const float* tvals, int64_t n_ray, int64_t n_int, const float* src,
                                       const float* dst, float voxel_diag_len, uint16_t* t_uint16, float* t_start,
                                       float* t_scale, void* stream) {
    return ctlab_compress_tvals_3d_ex(tvals, n_ray, n_int, src, dst, voxel_diag_len, t_uint16, t_start, t_scale,
                                      CTLAB_COMPRESS_CUDA, stream);
}

extern "C" int ctlab_forward_project_3d_compressed(const float* volume, int64_t batch, int64_t n_x, int64_t n_y,
                                                   int64_t n_z, const uint16_t* t_uint16, const float* t_start,
                                                   const float* t_scale, int64_t n_int, const float* src,
                                                   const float* dst, int64_t n_ray, const float* M_inv,
                                                   const float* b, float* out, void* stream) {
    clear_error();
    const int64_t dims[3] = {n_x, n_y, n_z};
    return run_compressed<false>("forward_project_3d_compressed", volume, out, batch, dims, t_uint16, t_start,
                                 t_scale, n_int, src, dst, n_ray, M_inv, b, 0, stream);
}

extern "C" int ctlab_back_project_3d_compressed(const float* sino, int64_t batch, int64_t n_ray,
                                                const uint16_t* t_uint16, const float* t_start, const float* t_scale,
                                                int64_t n_int, const float* src, const float* dst,
                                                const float* M_inv, const float* b, int64_t n_x, int64_t n_y,
                                                int64_t n_z, float* out, int accumulate, void* stream) {
    clear_error();
    const int64_t dims[3] = {n_x, n_y, n_z};
    return run_compressed<true>("back_project_3d_compressed", sino, out, batch, dims, t_uint16, t_start, t_scale,
                                n_int, src, dst, n_ray, M_inv, b, accumulate, stream);
}

extern "C" int ctlab_forward_project_2d_on_the_fly(const float* image, int64_t batch, int64_t n_row, int64_t n_col,
                                                   const float* src, const float* dst, int64_t n_ray,
                                                   const float* M_inv, const float* b, float* out, void* stream) {
    clear_error();
    return run_march2d<false>("forward_project_2d_on_the_fly", image, out, batch, n_row, n_col, src, dst, n_ray,
                              M_inv, b, 0, stream);
}

extern "C" int ctlab_back_project_2d_on_the_fly(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                                const float* dst, const float* M_inv, const float* b, int64_t n_row,
                                                int64_t n_col, float* out, int accumulate, void* stream) {
    clear_error();
    return run_march2d<true>("back_project_2d_on_the_fly", sino, out, batch, n_row, n_col, src, dst, n_ray, M_inv,
                             b, accumulate, stream);
}
