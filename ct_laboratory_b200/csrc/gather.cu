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
// (t_enter, t_exit, 1/v, |v|) computed exactly as the walks in walk.cuh compute them.
// These are the crossing-rule walk's segment spans times |v|, bitwise the
// lengths the atomic adjoint scatters with (the forward applies |v| to each
// ray's sum instead, a rounding-level difference), so the result is the
// transpose of that forward, accumulated in a fixed order (panel, then row,
// then column): bitwise reproducible from run to run.
//
// Candidate cells come from projecting the voxel's eight corners (a cell is
// a candidate when its centre lies in the bounding box of the projected
// corners, widened by a small margin); the exact length test then discards
// rays that miss, so the margin only costs time.
#include "common.cuh"

namespace ctlab {

struct PanelDev {
    float src[3], origin[3];
    float eu[3], ev[3];  // dual basis: (P - origin) . eu = continuous column index
    float n[3];          // panel normal
    int64_t first_ray, u_stride, v_stride;
    int n_u, n_v;
};

// Same set-up as lane_setup / traverse in walk.cuh.
struct RaySetup {
    float s[3], inv[3], ray_len, t_enter, t_exit;
    int fixed[3];  // index along an axis the ray does not cross, else -1
    bool live;
};

__device__ __forceinline__ RaySetup ray_setup(const float* __restrict__ src, const float* __restrict__ dst,
                                              int64_t r, const Affine3& A, const int* n) {
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
    R.t_enter = 0.f;
    R.t_exit = 1.f;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float va = __fsub_rn(d[a], R.s[a]);
        const float nf = (float)n[a];
        R.live = R.live && isfinite(R.s[a]) && isfinite(va);
        if (fabsf(va) > 1e-12f) {
            R.inv[a] = __frcp_rn(va);
            R.fixed[a] = -1;
            const float lo = va > 0.f ? -0.5f : nf - 0.5f;
            const float hi = va > 0.f ? nf - 0.5f : -0.5f;
            R.t_enter = fmaxf(R.t_enter, plane_t(lo, R.s[a], R.inv[a]));
            R.t_exit = fminf(R.t_exit, plane_t(hi, R.s[a], R.inv[a]));
        } else {
            R.inv[a] = 0.f;
            R.fixed[a] = __float2int_rn(R.s[a]);
            R.live = R.live && R.fixed[a] >= 0 && R.fixed[a] < n[a];
        }
    }
    R.live = R.live && (R.t_enter < R.t_exit);
    return R;
}

// Intersection length of a set-up ray with voxel (i, j, k).
__device__ __forceinline__ float voxel_len(const RaySetup& R, const int* ijk) {
    float t_in = R.t_enter, t_out = R.t_exit;
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

__global__ void __launch_bounds__(256) gather3d_kernel(const float* __restrict__ sino, float* __restrict__ out,
                                                       const float* __restrict__ src, const float* __restrict__ dst,
                                                       int64_t n_ray, const float* __restrict__ M_inv,
                                                       const float* __restrict__ bvec, const float* __restrict__ M,
                                                       int nx, int ny, int nz, const PanelDev* __restrict__ panels,
                                                       int n_panel, float margin) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t nvox = (int64_t)nx * ny * nz;
    if (v >= nvox) return;
    const int64_t bi = blockIdx.y;
    const int n[3] = {nx, ny, nz};
    const int ijk[3] = {(int)(v / ((int64_t)ny * nz)), (int)((v / nz) % ny), (int)(v % nz)};
    const Affine3 A = load_affine3(M_inv, bvec);
    // voxel centre and half-edge vectors in world space: x = M (ijk) + b
    float c[3], h[3][3];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        c[r] = __ldg(bvec + r);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float m = __ldg(M + 3 * r + a);
            c[r] = __fmaf_rn(m, (float)ijk[a], c[r]);
            h[a][r] = 0.5f * m;
        }
    }
    const float* y = sino + bi * n_ray;
    float acc = 0.f;
    for (int p = 0; p < n_panel; ++p) {
        const PanelDev& P = panels[p];
        // project the eight corners: u = ((S - O) + lam (X - S)) . eu with
        // lam = n.(O - S) / n.(X - S)
        float so[3], q0[3];
#pragma unroll
        for (int r = 0; r < 3; ++r) {
            so[r] = P.src[r] - P.origin[r];
            q0[r] = c[r] - P.src[r];
        }
        const float nd = -(so[0] * P.n[0] + so[1] * P.n[1] + so[2] * P.n[2]);
        const float base_u = so[0] * P.eu[0] + so[1] * P.eu[1] + so[2] * P.eu[2];
        const float base_v = so[0] * P.ev[0] + so[1] * P.ev[1] + so[2] * P.ev[2];
        float umin = 3.0e38f, umax = -3.0e38f, vmin = 3.0e38f, vmax = -3.0e38f;
        bool behind = false;
#pragma unroll
        for (int corner = 0; corner < 8; ++corner) {
            float q[3];
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                q[r] = q0[r];
#pragma unroll
                for (int a = 0; a < 3; ++a) q[r] += ((corner >> a) & 1 ? h[a][r] : -h[a][r]);
            }
            const float qn = q[0] * P.n[0] + q[1] * P.n[1] + q[2] * P.n[2];
            // a corner at or behind the source plane: the footprint is unbounded
            behind = behind || !(qn * nd > 0.f);
            const float lam = nd / qn;
            const float u = base_u + lam * (q[0] * P.eu[0] + q[1] * P.eu[1] + q[2] * P.eu[2]);
            const float w = base_v + lam * (q[0] * P.ev[0] + q[1] * P.ev[1] + q[2] * P.ev[2]);
            umin = fminf(umin, u);
            umax = fmaxf(umax, u);
            vmin = fminf(vmin, w);
            vmax = fmaxf(vmax, w);
        }
        int u0, u1, v0, v1;
        if (behind) {
            u0 = 0;
            u1 = P.n_u - 1;
            v0 = 0;
            v1 = P.n_v - 1;
        } else {
            u0 = max(0, (int)ceilf(umin - margin));
            u1 = min(P.n_u - 1, (int)floorf(umax + margin));
            v0 = max(0, (int)ceilf(vmin - margin));
            v1 = min(P.n_v - 1, (int)floorf(vmax + margin));
        }
        for (int jv = v0; jv <= v1; ++jv) {
            for (int ju = u0; ju <= u1; ++ju) {
                const int64_t r = P.first_ray + (int64_t)jv * P.v_stride + (int64_t)ju * P.u_stride;
                const float yr = __ldg(y + r);
                if (yr == 0.f) continue;
                const RaySetup R = ray_setup(src, dst, r, A, n);
                if (!R.live) continue;
                const float len = voxel_len(R, ijk);
                if (len > 0.f) acc = __fmaf_rn(yr, len, acc);
            }
        }
    }
    out[bi * nvox + v] = acc;
}

}  // namespace ctlab

using namespace ctlab;

extern "C" int ctlab_back_project_3d_gather(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                            const float* dst, const float* M, const float* M_inv, const float* b,
                                            int64_t n_x, int64_t n_y, int64_t n_z, const ctlab_panel* panels,
                                            int64_t n_panel, float* out, void* stream) {
    clear_error();
    const char* what = "back_project_3d_gather";
    CTLAB_REQUIRE(batch >= 1 && batch <= 65535, "%s: batch must be in [1, 65535]", what);
    CTLAB_REQUIRE(n_ray >= 0 && n_panel >= 0 && n_panel < (1LL << 31), "%s: bad n_ray/n_panel", what);
    CTLAB_REQUIRE(n_x >= 1 && n_y >= 1 && n_z >= 1 && n_x <= (1 << 22) && n_y <= (1 << 22) && n_z <= (1 << 22),
                  "%s: bad grid", what);
    const int64_t nvox = n_x * n_y * n_z;
    CTLAB_REQUIRE(nvox < (1LL << 31), "%s: volume too large", what);
    CTLAB_REQUIRE(out && M && M_inv && b && (n_panel == 0 || panels) && (n_ray == 0 || (sino && src && dst)),
                  "%s: null pointer", what);
    const int64_t blocks = (nvox + 255) / 256;
    static_assert(sizeof(ctlab_panel) == sizeof(PanelDev), "panel layout");
    gather3d_kernel<<<dim3((unsigned)blocks, (unsigned)batch), 256, 0, as_stream(stream)>>>(
        sino, out, src, dst, n_ray, M_inv, b, M, (int)n_x, (int)n_y, (int)n_z,
        reinterpret_cast<const PanelDev*>(panels), (int)n_panel, 0.05f);
    return launch_status(what);
}
