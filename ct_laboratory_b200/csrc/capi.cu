// capi.cu — ABI-level helpers of libctlab_b200.so: per-thread error strings,
// ray-tiling validation and the version query.
#include "common.cuh"

namespace ctlab {

static thread_local char g_last_error[512] = "";

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

void clear_error() { g_last_error[0] = '\0'; }

int resolve_tiling(const ctlab_ray_opts* t, int64_t n_ray, Tiling& T) {
    const bool flat = t == nullptr || (t->n_view == 0 && t->n_row == 0 && t->n_col == 0);
    int threads = 256, rows = 256;
    if (t != nullptr) {
        CTLAB_REQUIRE(t->voxel_rule == CTLAB_VOXEL_MIDPOINT || t->voxel_rule == CTLAB_VOXEL_CROSSING,
                      "ray options: unknown voxel_rule %d", t->voxel_rule);
        CTLAB_REQUIRE(t->walk == CTLAB_WALK_AUTO || t->walk == CTLAB_WALK_LANE || t->walk == CTLAB_WALK_COLUMN,
                      "ray options: unknown walk %d", t->walk);
        threads = t->block_threads ? t->block_threads : 256;
        rows = t->tile_rows ? t->tile_rows : (flat ? threads : 32);
        CTLAB_REQUIRE(threads >= 32 && threads <= 256 && threads % 32 == 0,
                      "ray tiling: block_threads must be a multiple of 32 in [32, 256] (got %d)", threads);
        CTLAB_REQUIRE(rows >= 1 && rows <= threads && threads % rows == 0,
                      "ray tiling: tile_rows must divide block_threads (got %d, %d)", rows, threads);
    }
    if (flat) {
        T.n_view = 1;
        T.n_row = n_ray;
        T.n_col = 1;
        T.view_stride = n_ray;
        T.row_stride = 1;
        T.col_stride = 1;
        T.tile_rows = threads;
        T.tile_cols = 1;
    } else {
        CTLAB_REQUIRE(t->n_view >= 1 && t->n_row >= 1 && t->n_col >= 1, "ray tiling: empty grid");
        CTLAB_REQUIRE(t->n_view * t->n_row * t->n_col == n_ray,
                      "ray tiling: n_view*n_row*n_col (%lld) must equal n_ray (%lld)",
                      (long long)(t->n_view * t->n_row * t->n_col), (long long)n_ray);
        // Every grid position must map into [0, n_ray).
        const int64_t last = (t->n_view - 1) * t->view_stride + (t->n_row - 1) * t->row_stride +
                             (t->n_col - 1) * t->col_stride;
        CTLAB_REQUIRE(t->view_stride >= 0 && t->row_stride >= 0 && t->col_stride >= 0 && last < n_ray,
                      "ray tiling: strides address rays outside [0, n_ray)");
        T.n_view = t->n_view;
        T.n_row = t->n_row;
        T.n_col = t->n_col;
        T.view_stride = t->view_stride;
        T.row_stride = t->row_stride;
        T.col_stride = t->col_stride;
        T.tile_rows = rows;
        T.tile_cols = threads / rows;
    }
    T.tiles_r = (T.n_row + T.tile_rows - 1) / T.tile_rows;
    T.tiles_c = (T.n_col + T.tile_cols - 1) / T.tile_cols;
    T.n_blocks = T.n_view * T.tiles_r * T.tiles_c;
    T.tiles = nullptr;
    T.n_full = T.n_blocks;
    return CTLAB_OK;
}

}  // namespace ctlab

extern "C" int ctlab_abi_version(void) { return CTLAB_ABI_VERSION; }

extern "C" const char* ctlab_last_error(void) { return ctlab::g_last_error; }

// ----------------------------------------------------------------------------
// M -> M^-1 on the device (one thread), so that callers holding M on the GPU
// need neither a host round trip nor torch.inverse's singularity check (which
// synchronises).  Gauss-Jordan elimination with partial pivoting, the same
// elimination LU-based inversion performs; for the diagonal M the geometry
// classes build (standard_image_transform.py:3-50) every entry is the
// correctly rounded reciprocal 1/s, as with torch.inverse.
// ----------------------------------------------------------------------------
namespace ctlab {
__global__ void invert_kernel(const float* __restrict__ M, int n, float* __restrict__ out,
                              int* __restrict__ singular) {
    float a[3][6];
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < 2 * n; ++c) a[r][c] = (c < n) ? M[r * n + c] : (c - n == r ? 1.f : 0.f);
    int bad = 0;
    for (int col = 0; col < n; ++col) {
        int piv = col;
        for (int r = col + 1; r < n; ++r)
            if (fabsf(a[r][col]) > fabsf(a[piv][col])) piv = r;
        if (piv != col)
            for (int c = 0; c < 2 * n; ++c) {
                const float t = a[col][c];
                a[col][c] = a[piv][c];
                a[piv][c] = t;
            }
        const float p = a[col][col];
        if (!(p != 0.f) || !isfinite(p)) {
            bad = 1;
            break;
        }
        for (int c = 0; c < 2 * n; ++c) a[col][c] = __fdiv_rn(a[col][c], p);
        for (int r = 0; r < n; ++r) {
            if (r == col) continue;
            const float f = a[r][col];
            if (f == 0.f) continue;
            for (int c = 0; c < 2 * n; ++c) a[r][c] = __fsub_rn(a[r][c], __fmul_rn(f, a[col][c]));
        }
    }
    for (int r = 0; r < n; ++r)
        for (int c = 0; c < n; ++c) out[r * n + c] = bad ? __int_as_float(0x7fc00000) : a[r][n + c];
    if (singular) *singular = bad;
}
}  // namespace ctlab

extern "C" int ctlab_invert_matrix(const float* M, int n, float* M_inv, int* singular, void* stream) {
    ctlab::clear_error();
    CTLAB_REQUIRE(n == 2 || n == 3, "invert_matrix: n must be 2 or 3 (got %d)", n);
    CTLAB_REQUIRE(M && M_inv, "invert_matrix: null pointer");
    ctlab::invert_kernel<<<1, 1, 0, ctlab::as_stream(stream)>>>(M, n, M_inv, singular);
    return ctlab::launch_status("invert_matrix");
}
