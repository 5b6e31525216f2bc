// gather.cu — deterministic voxel-driven adjoint (A^T y by gathering).
//
// The atomic adjoint scatters y_r * len(r, v) from every ray into its voxels;
// the order of the float additions then depends on scheduling.  Here every
// voxel instead gathers its own sum: for each detector panel (a view whose
// cells form a flat grid: a cone-beam view, a fan-beam view, a StaticCT
// module lit by one source in one frame), the voxel is projected from the
// panel's source onto the panel plane, the cells whose rays can pass through
// it are enumerated, and for each such ray the voxel's intersection length is
// evaluated with the arithmetic of the forward walk:
//     t_in  = max(t_enter, behind-plane parameters of the voxel)
//     t_out = min(t_exit,  ahead-plane parameters of the voxel)
//     len   = (t_out - t_in) * |v|      (0 when t_out <= t_in)
// with every plane parameter t = (p - s) * (1/v) and the per-ray set-up
// (s, 1/v, |v|) computed exactly as the walks in walk.cuh compute them (t_enter
// and t_exit need not be: see RaySetup).
// These are the crossing-rule walk's parameter spans (bitwise) times |v|
// (the atomic adjoint scatters (y * |v|) * span, the forward applies |v| to
// each ray's sum of spans: rounding-level differences), so the result is the
// transpose of that forward, accumulated in a fixed order (panel, then row,
// then column): bitwise reproducible from run to run.
//
// Candidate cells come from projecting the voxel's eight corners (a cell is
// a candidate when its centre lies in the bounding box of the projected
// corners, widened by a small margin); the exact length test then discards
// rays that miss, so the margin only costs time.
#include <algorithm>
#include <cstdint>

#include "common.cuh"

namespace ctlab {

struct PanelDev {
    float src[3], origin[3];
    float eu[3], ev[3];  // dual basis: (P - origin) . eu = continuous column index
    float n[3];          // panel normal
    int64_t first_ray, u_stride, v_stride;
    int n_u, n_v;
};

// The per-ray values of lane_setup in walk.cuh that a voxel's length needs,
// computed with the same arithmetic.  The ray's entry and exit parameters are
// not: along every crossed axis the voxel's own behind / ahead plane lies
// inside the grid's, and t = (p - s) * (1/v) is monotone in p under
// round-to-nearest, so max(t_enter, voxel behind-planes) equals
// max(0, voxel behind-planes) bitwise, and likewise for the exit with 1.  A
// ray that misses the grid gets an empty interval for every voxel the same
// way.
struct RaySetup {
    float s[3], inv[3], ray_len;
    int fixed[3];  // index along an axis the ray does not cross, else -1
    bool live;
};

__device__ __forceinline__ RaySetup ray_setup(const float* __restrict__ src, const float* __restrict__ dst,
                                              int64_t r, const Affine3& A) {
    RaySetup R;
    float sw[3], dw[3], vw[3], d[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        sw[a] = __ldg(src + 3 * r + a);
        dw[a] = __ldg(dst + 3 * r + a);
        vw[a] = __fsub_rn(dw[a], sw[a]);
    }
    R.ray_len = sqrtf(sumsq3(vw[0], vw[1], vw[2]));
    R.live = R.ray_len >= 1e-12f;
    world_to_index3(A, sw[0], sw[1], sw[2], R.s[0], R.s[1], R.s[2]);
    world_to_index3(A, dw[0], dw[1], dw[2], d[0], d[1], d[2]);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float va = __fsub_rn(d[a], R.s[a]);
        R.live = R.live && isfinite(R.s[a]) && isfinite(va);
        if (fabsf(va) > 1e-12f) {
            R.inv[a] = __frcp_rn(va);
            R.fixed[a] = -1;
        } else {
            R.inv[a] = 0.f;
            R.fixed[a] = __float2int_rn(R.s[a]);
        }
    }
    return R;
}

// Intersection length of a set-up ray with voxel (i, j, k).
__device__ __forceinline__ float voxel_len(const RaySetup& R, const int* ijk) {
    float t_in = 0.f, t_out = 1.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (R.inv[a] != 0.f) {
            const float p0 = (float)ijk[a] - 0.5f, p1 = (float)ijk[a] + 0.5f;
            const float ta = plane_t(p0, R.s[a], R.inv[a]), tb = plane_t(p1, R.s[a], R.inv[a]);
            const bool pos = R.inv[a] > 0.f;
            t_in = fmaxf(t_in, pos ? ta : tb);
            t_out = fminf(t_out, pos ? tb : ta);
        } else if (R.fixed[a] != ijk[a]) {
            return 0.f;
        }
    }
    return t_out > t_in ? __fmul_rn(__fsub_rn(t_out, t_in), R.ray_len) : 0.f;
}

// The ray table: per ray s[3] and |v| (0 for a ray the walk skips), then
// 1/v[3] (0 along an axis the ray does not cross, where s rounds to the
// fixed index) and y (for a single sinogram; 0 for a skipped ray), 32 bytes,
// one sector, read as two float4.
struct __align__(16) RayRow {
    float s[3], ray_len;
    float inv[3], y;
};
static_assert(sizeof(RayRow) == 32, "ray table row");

__global__ void __launch_bounds__(256) gather_ray_table_kernel(const float* __restrict__ src,
                                                               const float* __restrict__ dst, int64_t n_ray,
                                                               const float* __restrict__ M_inv,
                                                               const float* __restrict__ bvec,
                                                               const float* __restrict__ y, RayRow* __restrict__ tab) {
    const Affine3 A = load_affine3(M_inv, bvec);
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n_ray; r += (int64_t)gridDim.x * blockDim.x) {
        const RaySetup R = ray_setup(src, dst, r, A);
        RayRow row;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            row.s[a] = R.s[a];
            row.inv[a] = R.inv[a];
        }
        row.ray_len = R.live ? R.ray_len : 0.f;
        row.y = (y != nullptr && R.live) ? __ldg(y + r) : 0.f;
        tab[r] = row;
    }
}

__device__ __forceinline__ float voxel_len_row(const float4 a, const float4 b, const int* ijk) {
    const float s[3] = {a.x, a.y, a.z}, inv[3] = {b.x, b.y, b.z};
    float t_in = 0.f, t_out = 1.f;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (inv[k] != 0.f) {
            const float p0 = (float)ijk[k] - 0.5f, p1 = (float)ijk[k] + 0.5f;
            const float ta = plane_t(p0, s[k], inv[k]), tb = plane_t(p1, s[k], inv[k]);
            const bool pos = inv[k] > 0.f;
            t_in = fmaxf(t_in, pos ? ta : tb);
            t_out = fminf(t_out, pos ? tb : ta);
        } else if (__float2int_rn(s[k]) != ijk[k]) {
            return 0.f;
        }
    }
    return t_out > t_in ? __fmul_rn(__fsub_rn(t_out, t_in), a.w) : 0.f;
}

// What the corner projection needs of a panel, derived once per launch
// block: with q = X - S for a point X,
//     u(X) = base_u + lam * (q . eu),  v(X) = base_v + lam * (q . ev),
//     lam  = nd / (q . n),  nd = n . (O - S),
// and q . e over the eight corners X = centre +- h0 +- h1 +- h2 (h_a the
// half voxel edges in world space) is (centre - S) . e +- h0.e +- h1.e +- h2.e.
// Packed in 16-byte fields: a warp reads each with one broadcast.
struct __align__(16) PanelProj {
    float4 s_nd;   // S, nd
    float4 n_bu;   // n, base_u
    float4 eu_bv;  // eu, base_v
    float4 ev;     // ev, 0
    float4 hn, hu, hv;
    int4 dims;            // n_u, n_v
    longlong2 first_us;   // first_ray, u_stride
    longlong2 vs;         // v_stride
};

constexpr int kPanelChunk = 64;

__device__ __forceinline__ void panel_proj(const PanelDev& P, const float* __restrict__ M, PanelProj& Q) {
    float so[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) so[r] = P.src[r] - P.origin[r];
    const float nd = -(so[0] * P.n[0] + so[1] * P.n[1] + so[2] * P.n[2]);
    const float bu = so[0] * P.eu[0] + so[1] * P.eu[1] + so[2] * P.eu[2];
    const float bv = so[0] * P.ev[0] + so[1] * P.ev[1] + so[2] * P.ev[2];
    Q.s_nd = make_float4(P.src[0], P.src[1], P.src[2], nd);
    Q.n_bu = make_float4(P.n[0], P.n[1], P.n[2], bu);
    Q.eu_bv = make_float4(P.eu[0], P.eu[1], P.eu[2], bv);
    Q.ev = make_float4(P.ev[0], P.ev[1], P.ev[2], 0.f);
    float hn[3], hu[3], hv[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float h[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) h[r] = 0.5f * __ldg(M + 3 * r + a);
        hn[a] = h[0] * P.n[0] + h[1] * P.n[1] + h[2] * P.n[2];
        hu[a] = h[0] * P.eu[0] + h[1] * P.eu[1] + h[2] * P.eu[2];
        hv[a] = h[0] * P.ev[0] + h[1] * P.ev[1] + h[2] * P.ev[2];
    }
    Q.hn = make_float4(hn[0], hn[1], hn[2], 0.f);
    Q.hu = make_float4(hu[0], hu[1], hu[2], 0.f);
    Q.hv = make_float4(hv[0], hv[1], hv[2], 0.f);
    Q.dims = make_int4(P.n_u, P.n_v, 0, 0);
    Q.first_us = make_longlong2(P.first_ray, P.u_stride);
    Q.vs = make_longlong2(P.v_stride, 0);
}

// The eight corner values x0 +- h0 +- h1 +- h2.
__device__ __forceinline__ void corner_values(float x0, const float4 h, float* out) {
    const float a0 = x0 - h.x, a1 = x0 + h.x;
    const float b0 = a0 - h.y, b1 = a1 - h.y, b2 = a0 + h.y, b3 = a1 + h.y;
    out[0] = b0 - h.z;
    out[1] = b1 - h.z;
    out[2] = b2 - h.z;
    out[3] = b3 - h.z;
    out[4] = b0 + h.z;
    out[5] = b1 + h.z;
    out[6] = b2 + h.z;
    out[7] = b3 + h.z;
}

// One thread per voxel (z fastest, so a warp holds 32 neighbours along z,
// whose footprints share detector columns).  The panels are taken in chunks
// staged in shared memory; every thread of the block takes part in staging,
// voxels past the grid included (with no candidates).
// TAB: the rays' set-up and y come from the ray table (tab, built for the
// sinogram gathered), so a candidate is one 32-byte sector; else the set-up
// is recomputed for every candidate.  The lengths are the same bitwise.  (Staging a warp's candidate rows in shared memory first, read
// coalesced along detector rows, measured slower: 97.8 against 82.8 ms on
// the cone256 scan; each row is read by every warp whose voxels it crosses
// either way.)
template <bool TAB>
__global__ void __launch_bounds__(256, TAB ? 4 : 3) gather3d_kernel(const float* __restrict__ sino, float* __restrict__ out,
                                                       const float* __restrict__ src, const float* __restrict__ dst,
                                                       int64_t n_ray, const float* __restrict__ M_inv,
                                                       const float* __restrict__ bvec, const float* __restrict__ M,
                                                       int nx, int ny, int nz, const PanelDev* __restrict__ panels,
                                                       int n_panel, float margin, const float4* __restrict__ tab) {
    __shared__ PanelProj sp[kPanelChunk];
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nvox = (int64_t)nx * ny * nz;
    const bool active = v < nvox;
    const int64_t bi = blockIdx.y;
    const int64_t vc = active ? v : 0;
    const int ijk[3] = {(int)(vc / ((int64_t)ny * nz)), (int)((vc / nz) % ny), (int)(vc % nz)};
    const Affine3 A = load_affine3(M_inv, bvec);
    (void)A;
    // voxel centre in world space: x = M (ijk) + b
    float c[3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        c[r] = __ldg(bvec + r);
#pragma unroll
        for (int a = 0; a < 3; ++a) c[r] = __fmaf_rn(__ldg(M + 3 * r + a), (float)ijk[a], c[r]);
    }
    const float* y = sino + bi * n_ray;
    float acc = 0.f;
    for (int p0 = 0; p0 < n_panel; p0 += kPanelChunk) {
        const int np = min(kPanelChunk, n_panel - p0);
        __syncthreads();  // the previous chunk is no longer read
        if ((int)threadIdx.x < np) panel_proj(panels[p0 + threadIdx.x], M, sp[threadIdx.x]);
        __syncthreads();
#pragma unroll 1
        for (int p = 0; p < np; ++p) {
            const float4 s_nd = sp[p].s_nd, n_bu = sp[p].n_bu, eu_bv = sp[p].eu_bv, ev = sp[p].ev;
            const float q0[3] = {c[0] - s_nd.x, c[1] - s_nd.y, c[2] - s_nd.z};
            float cn[8], cu[8], cv[8];
            corner_values(q0[0] * n_bu.x + q0[1] * n_bu.y + q0[2] * n_bu.z, sp[p].hn, cn);
            corner_values(q0[0] * eu_bv.x + q0[1] * eu_bv.y + q0[2] * eu_bv.z, sp[p].hu, cu);
            corner_values(q0[0] * ev.x + q0[1] * ev.y + q0[2] * ev.z, sp[p].hv, cv);
            float umin = 3.0e38f, umax = -3.0e38f, vmin = 3.0e38f, vmax = -3.0e38f;
            bool behind = false;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                // a corner at or behind the source plane: the footprint is unbounded
                behind = behind || !(cn[k] * s_nd.w > 0.f);
                const float lam = __fdividef(s_nd.w, cn[k]);
                const float u = __fmaf_rn(lam, cu[k], n_bu.w);
                const float w = __fmaf_rn(lam, cv[k], eu_bv.w);
                umin = fminf(umin, u);
                umax = fmaxf(umax, u);
                vmin = fminf(vmin, w);
                vmax = fmaxf(vmax, w);
            }
            const int4 dims = sp[p].dims;
            const longlong2 fu = sp[p].first_us;
            const int64_t v_stride = sp[p].vs.x;
            int u0, u1, v0, v1;
            if (!active) {  // no voxel: no candidates
                u0 = 0;
                u1 = -1;
                v0 = 0;
                v1 = -1;
            } else if (behind) {
                u0 = 0;
                u1 = dims.x - 1;
                v0 = 0;
                v1 = dims.y - 1;
            } else {
                u0 = max(0, (int)ceilf(umin - margin));
                u1 = min(dims.x - 1, (int)floorf(umax + margin));
                v0 = max(0, (int)ceilf(vmin - margin));
                v1 = min(dims.y - 1, (int)floorf(vmax + margin));
            }
            for (int jv = v0; jv <= v1; ++jv) {
                for (int ju = u0; ju <= u1; ++ju) {
                    const int64_t r = fu.x + (int64_t)jv * v_stride + (int64_t)ju * fu.y;
                    float yr, len;
                    if constexpr (TAB) {
                        const float4 ra = __ldg(tab + 2 * r), rb = __ldg(tab + 2 * r + 1);
                        yr = rb.w;  // 0 for a skipped ray
                        if (yr == 0.f) continue;
                        len = voxel_len_row(ra, rb, ijk);
                    } else {
                        yr = __ldg(y + r);
                        if (yr == 0.f) continue;
                        const RaySetup R = ray_setup(src, dst, r, A);
                        if (!R.live) continue;
                        len = voxel_len(R, ijk);
                    }
                    if (len > 0.f) acc = __fmaf_rn(yr, len, acc);
                }
            }
        }
    }
    if (active) out[bi * nvox + v] = acc;
}

}  // namespace ctlab

using namespace ctlab;

namespace {

int gather_entry(const char* what, const float* sino, int64_t batch, int64_t n_ray, const float* src, const float* dst,
                 const float* M, const float* M_inv, const float* b, int64_t n_x, int64_t n_y, int64_t n_z,
                 const ctlab_panel* panels, int64_t n_panel, float* out, void* ray_table, void* stream) {
    clear_error();
    CTLAB_REQUIRE(batch >= 1 && batch <= 65535, "%s: batch must be in [1, 65535]", what);
    CTLAB_REQUIRE(n_ray >= 0 && n_panel >= 0 && n_panel < (1LL << 31), "%s: bad n_ray/n_panel", what);
    CTLAB_REQUIRE(n_x >= 1 && n_y >= 1 && n_z >= 1 && n_x <= (1 << 22) && n_y <= (1 << 22) && n_z <= (1 << 22),
                  "%s: bad grid", what);
    const int64_t nvox = n_x * n_y * n_z;
    CTLAB_REQUIRE(nvox < (1LL << 31), "%s: volume too large", what);
    CTLAB_REQUIRE(out && M && M_inv && b && (n_panel == 0 || panels) && (n_ray == 0 || (sino && src && dst)),
                  "%s: null pointer", what);
    CTLAB_REQUIRE(((uintptr_t)ray_table & 15) == 0, "%s: ray_table must be 16-byte aligned", what);
    const int64_t blocks = (nvox + 255) / 256;
    static_assert(sizeof(ctlab_panel) == sizeof(PanelDev), "panel layout");
    cudaStream_t st = as_stream(stream);
    const PanelDev* pd = reinterpret_cast<const PanelDev*>(panels);
    if (ray_table && n_ray > 0) {
        // sinogram by sinogram: its y goes into the table with the rays'
        // set-up (rebuilt per sinogram, about 1 % of a gather), so that a
        // candidate ray is one sector
        const int64_t tb = std::min<int64_t>((n_ray + 255) / 256, 148 * 64);
        const float4* tab = static_cast<const float4*>(ray_table);
        for (int64_t k = 0; k < batch; ++k) {
            gather_ray_table_kernel<<<(unsigned)tb, 256, 0, st>>>(src, dst, n_ray, M_inv, b, sino + k * n_ray,
                                                                  static_cast<RayRow*>(ray_table));
            gather3d_kernel<true><<<dim3((unsigned)blocks, 1), 256, 0, st>>>(
                sino + k * n_ray, out + k * nvox, src, dst, n_ray, M_inv, b, M, (int)n_x, (int)n_y, (int)n_z, pd,
                (int)n_panel, 0.05f, tab);
        }
    } else {
        gather3d_kernel<false><<<dim3((unsigned)blocks, (unsigned)batch), 256, 0, st>>>(
            sino, out, src, dst, n_ray, M_inv, b, M, (int)n_x, (int)n_y, (int)n_z, pd, (int)n_panel, 0.05f, nullptr);
    }
    return launch_status(what);
}

}  // namespace

extern "C" int ctlab_back_project_3d_gather(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                            const float* dst, const float* M, const float* M_inv, const float* b,
                                            int64_t n_x, int64_t n_y, int64_t n_z, const ctlab_panel* panels,
                                            int64_t n_panel, float* out, void* stream) {
    return gather_entry("back_project_3d_gather", sino, batch, n_ray, src, dst, M, M_inv, b, n_x, n_y, n_z, panels,
                        n_panel, out, nullptr, stream);
}

extern "C" int ctlab_back_project_3d_gather_ws(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                               const float* dst, const float* M, const float* M_inv, const float* b,
                                               int64_t n_x, int64_t n_y, int64_t n_z, const ctlab_panel* panels,
                                               int64_t n_panel, float* out, void* ray_table, void* stream) {
    return gather_entry("back_project_3d_gather_ws", sino, batch, n_ray, src, dst, M, M_inv, b, n_x, n_y, n_z,
                        panels, n_panel, out, ray_table, stream);
}
