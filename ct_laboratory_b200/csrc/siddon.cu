// siddon.cu — single-scan kernels and C entry points of the on-the-fly
// Siddon forward projector and exact adjoint (2-D and 3-D), sm_100a.  The
// walks themselves are in walk.cuh.
#include "walk.cuh"

namespace ctlab {

template <int NDIM, bool ADJ, bool MID>
__global__ void __launch_bounds__(256) siddon_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                     const float* __restrict__ src, const float* __restrict__ dst,
                                                     int64_t n_ray, const float* __restrict__ M_inv,
                                                     const float* __restrict__ bvec, GridDims<NDIM> G,
                                                     int64_t nvox, Tiling T, float* __restrict__ outT) {
    const int64_t r = tile_ray(T);
    if constexpr (NDIM == 2 && ADJ && CTLAB_MAJOR2_WARP) {
        // warp-cooperative: every lane takes part, with or without a ray
        major2_adjoint_warp<MID>(in, out, outT, src, dst, n_ray, load_affine2(M_inv, bvec), G, nvox, r,
                                 blockIdx.y);
        return;
    }
    if (r < 0) return;
    AffineT<NDIM> aff;
    if constexpr (NDIM == 3) {
        aff = load_affine3(M_inv, bvec);
    } else {
        aff = load_affine2(M_inv, bvec);
    }
    lane_ray<NDIM, ADJ, MID>(in, out, src, dst, n_ray, aff, G, nvox, r, blockIdx.y);
}

// out[b][i0][i1] += T[b][i1][i0] for a batch of n0 x n1 images (row-major)
// and their transposes T: 32 x 32 tiles through shared memory, so that both
// the reads of T and the read-modify-writes of out are coalesced.  Tiles are
// taken grid-stride: blockIdx.x strides over the tiles of image b =
// blockIdx.y.
__global__ void __launch_bounds__(256) add_transposed_kernel(float* __restrict__ out, const float* __restrict__ T,
                                                             int n0, int n1, int64_t nvox) {
    __shared__ float tile[32][33];
    const int64_t b = blockIdx.y;
    const int t0 = (n0 + 31) >> 5, t1 = (n1 + 31) >> 5;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int k = blockIdx.x; k < t0 * t1; k += gridDim.x) {
        const int i0b = (k / t1) << 5, i1b = (k % t1) << 5;
        __syncthreads();  // the previous tile has been read out
#pragma unroll
        for (int r = ty; r < 32; r += 8) {
            const int i1 = i1b + r, i0 = i0b + tx;
            if (i1 < n1 && i0 < n0) tile[r][tx] = T[b * nvox + (int64_t)i1 * n0 + i0];
        }
        __syncthreads();
#pragma unroll
        for (int r = ty; r < 32; r += 8) {
            const int i0 = i0b + r, i1 = i1b + tx;
            if (i0 < n0 && i1 < n1) out[b * nvox + (int64_t)i0 * n1 + i1] += tile[tx][r];
        }
    }
}

// Resident CTAs per SM the register allocation of the column walk targets.
#ifndef CTLAB_XY_MIN_BLOCKS
#define CTLAB_XY_MIN_BLOCKS 4
#endif

// blockIdx.y covers batch items NB at a time: the walk of a tile is done once
// for NB volumes (a batch of B volumes costs B / NB walks, not B).
template <bool ADJ, int NB, int W = 32>
__global__ void __launch_bounds__(256, NB == 1 ? CTLAB_XY_MIN_BLOCKS : 3)
    siddon3d_shared_xy_kernel(const float* __restrict__ in, float* __restrict__ out, const float* __restrict__ src,
                              const float* __restrict__ dst, int64_t n_ray, const float* __restrict__ M_inv,
                              const float* __restrict__ bvec, GridDims<3> G, int64_t nvox, Tiling T, int batch) {
    __shared__ XYCell cells[256 / 32][kChunk];
    const Affine3 A = load_affine3(M_inv, bvec);
    const int64_t b0 = (int64_t)blockIdx.y * NB;
    const int nb = min(NB, batch - (int)b0);
    shared_xy_ray<ADJ, NB, W>(in, out, src, dst, n_ray, A, G, nvox, tile_ray(T), b0, nb, cells[threadIdx.x >> 5]);
}

// The same launch shape under the reference's midpoint rule
// (shared_xy_ray_mid): per warp the round's crossing parameters and its
// certified cell records.
template <bool ADJ, int NB, int W = 32>
__global__ void __launch_bounds__(256, NB == 1 ? CTLAB_XY_MIN_BLOCKS : 3)
    siddon3d_shared_xy_mid_kernel(const float* __restrict__ in, float* __restrict__ out,
                                  const float* __restrict__ src, const float* __restrict__ dst, int64_t n_ray,
                                  const float* __restrict__ M_inv, const float* __restrict__ bvec, GridDims<3> G,
                                  int64_t nvox, Tiling T, int batch) {
    __shared__ float raw[256 / 32][kChunk];
    __shared__ MidCell rec[256 / 32][kChunk];
    const Affine3 A = load_affine3(M_inv, bvec);
    const int64_t b0 = (int64_t)blockIdx.y * NB;
    const int nb = min(NB, batch - (int)b0);
    shared_xy_ray_mid<ADJ, NB, W>(in, out, src, dst, n_ray, A, G, nvox, tile_ray(T), b0, nb, raw[threadIdx.x >> 5],
                                  rec[threadIdx.x >> 5]);
}

template <bool ADJ, bool MID, int NB, int W>
static void launch_column(dim3 g, int threads, cudaStream_t s, const float* in, float* out, const float* src,
                          const float* dst, int64_t n_ray, const float* M_inv, const float* b, const GridDims<3>& G,
                          int64_t nvox, const Tiling& T, int batch) {
    if constexpr (MID)
        siddon3d_shared_xy_mid_kernel<ADJ, NB, W><<<g, threads, 0, s>>>(in, out, src, dst, n_ray, M_inv, b, G, nvox,
                                                                         T, batch);
    else
        siddon3d_shared_xy_kernel<ADJ, NB, W><<<g, threads, 0, s>>>(in, out, src, dst, n_ray, M_inv, b, G, nvox, T,
                                                                     batch);
}

// The column-walk kernel for nb volumes per walk and 32- or 16-row columns.
template <bool ADJ, bool MID>
static void launch_column_nb(int nb, int rows, dim3 g, int threads, cudaStream_t s, const float* in, float* out,
                             const float* src, const float* dst, int64_t n_ray, const float* M_inv, const float* b,
                             const GridDims<3>& G, int64_t nvox, const Tiling& T, int batch) {
    if (rows == 16) {  // 16 detector rows per column: two 16-lane groups per warp
        if (nb == 4) launch_column<ADJ, MID, 4, 16>(g, threads, s, in, out, src, dst, n_ray, M_inv, b, G, nvox, T, batch);
        else if (nb == 2) launch_column<ADJ, MID, 2, 16>(g, threads, s, in, out, src, dst, n_ray, M_inv, b, G, nvox, T, batch);
        else launch_column<ADJ, MID, 1, 16>(g, threads, s, in, out, src, dst, n_ray, M_inv, b, G, nvox, T, batch);
        return;
    }
    if (nb == 4) launch_column<ADJ, MID, 4, 32>(g, threads, s, in, out, src, dst, n_ray, M_inv, b, G, nvox, T, batch);
    else if (nb == 2) launch_column<ADJ, MID, 2, 32>(g, threads, s, in, out, src, dst, n_ray, M_inv, b, G, nvox, T, batch);
    else launch_column<ADJ, MID, 1, 32>(g, threads, s, in, out, src, dst, n_ray, M_inv, b, G, nvox, T, batch);
}


// ----------------------------------------------------------------------------
// host side
// ----------------------------------------------------------------------------

template <int NDIM, bool ADJ>
static int launch_siddon(const char* what, const float* in, float* out, int64_t batch, const int64_t* dims,
                         const float* src, const float* dst, int64_t n_ray, const float* M_inv, const float* b,
                         int accumulate, const ctlab_ray_opts* tiling, void* stream, float* scratch = nullptr) {
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
        // Detector-row tilings (a warp = 32 rows of one column, or two groups
        // of 16) take the shared x-y walk under either voxel rule; it checks
        // per warp that the lanes share their x-y line (and, under the
        // midpoint rule, that M^-1 is diagonal) and otherwise runs the
        // per-lane walk.
        const bool small_grid = G.n[0] <= 65536 && G.n[1] <= 65536 && G.n[2] <= 65536;
        if (!flat && small_grid && (T.tile_rows % 32 == 0 || T.tile_rows == 16) &&
            (walk == CTLAB_WALK_COLUMN || walk == CTLAB_WALK_AUTO)) {
            const int nb = batch >= 4 ? 4 : (batch >= 2 ? 2 : 1);
            const dim3 g((unsigned)T.n_blocks, (unsigned)((batch + nb - 1) / nb));
            const int rows = T.tile_rows == 16 ? 16 : 32;
            if (mid)
                launch_column_nb<ADJ, true>(nb, rows, g, threads, s, in, out, src, dst, n_ray, M_inv, b, G, nvox, T,
                                            (int)batch);
            else
                launch_column_nb<ADJ, false>(nb, rows, g, threads, s, in, out, src, dst, n_ray, M_inv, b, G, nvox, T,
                                             (int)batch);
            return launch_status(what);
        }
    }
    // 2-D adjoint with scratch: rays whose major axis is the image's column
    // axis scatter into the transpose held in `scratch`, which is then added
    // back (major2_adjoint_warp).
    float* outT = (NDIM == 2 && ADJ && CTLAB_MAJOR2_WARP) ? scratch : nullptr;
    if (outT) CTLAB_CUDA_TRY(cudaMemsetAsync(outT, 0, sizeof(float) * (size_t)(batch * nvox), s));
    if (mid)
        siddon_kernel<NDIM, ADJ, true><<<grid, threads, 0, s>>>(in, out, src, dst, n_ray, M_inv, b, G, nvox, T, outT);
    else
        siddon_kernel<NDIM, ADJ, false><<<grid, threads, 0, s>>>(in, out, src, dst, n_ray, M_inv, b, G, nvox, T, outT);
    if (outT) {
        int rc = launch_status(what);
        if (rc) return rc;
        const int tiles = ((G.n[0] + 31) / 32) * ((G.n[1] + 31) / 32);
        add_transposed_kernel<<<dim3((unsigned)(tiles < 1024 ? tiles : 1024), (unsigned)batch), 256, 0, s>>>(
            out, outT, G.n[0], G.n[1], nvox);
    }
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

extern "C" int ctlab_back_project_2d_siddon_ws(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                               const float* dst, const float* M_inv, const float* b, int64_t n_row,
                                               int64_t n_col, float* out, int accumulate,
                                               const ctlab_ray_opts* tiling, float* scratch, void* stream) {
    clear_error();
    const int64_t dims[2] = {n_row, n_col};
    CTLAB_REQUIRE(scratch == nullptr || scratch != out, "back_project_2d_siddon_ws: scratch must not be the output");
    return launch_siddon<2, true>("back_project_2d_siddon_ws", sino, out, batch, dims, src, dst, n_ray, M_inv, b,
                                  accumulate, tiling, stream, scratch);
}
