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
// The midpoint walk's adjoint (one volume) targets 3: with up to 85
// registers a thread it measured 8.91 ms on the cone256 scan against 9.31
// at 4 (64 registers), while its forward and the crossing-rule adjoint are
// faster at 4 (9.67 against 10.71 ms; 8.43 against 8.53 ms).
#ifndef CTLAB_XY_MIN_BLOCKS_ADJ
#define CTLAB_XY_MIN_BLOCKS_ADJ CTLAB_XY_MIN_BLOCKS
#endif
#ifndef CTLAB_MID_MIN_BLOCKS_ADJ
#define CTLAB_MID_MIN_BLOCKS_ADJ 3
#endif

// blockIdx.y covers batch items NB at a time: the walk of a tile is done once
// for NB volumes (a batch of B volumes costs B / NB walks, not B).
template <bool ADJ, int NB, int W = 32>
__global__ void __launch_bounds__(256, NB == 1 ? (ADJ ? CTLAB_XY_MIN_BLOCKS_ADJ : CTLAB_XY_MIN_BLOCKS) : 3)
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
__global__ void __launch_bounds__(256, NB == 1 ? (ADJ ? CTLAB_MID_MIN_BLOCKS_ADJ : CTLAB_XY_MIN_BLOCKS) : 3)
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
                         int accumulate, const ctlab_ray_opts* tiling, void* stream, float* scratch = nullptr,
                         const int32_t* tiles = nullptr, int64_t n_tiles = -1) {
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
    if (n_tiles >= 0) {
        // only the listed tiles run: the rays of every other tile must be
        // ones the walks do not charge (ctlab_active_tiles), so the forward
        // zeroes its output first and the adjoint adds nothing for them
        CTLAB_REQUIRE(n_tiles <= T.n_blocks, "%s: %lld tiles listed, the tiling has %lld", what,
                      (long long)n_tiles, (long long)T.n_blocks);
        CTLAB_REQUIRE(n_tiles == 0 || tiles != nullptr, "%s: null tile list", what);
        if (!ADJ) CTLAB_CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float) * (size_t)(batch * n_ray), s));
        if (n_tiles == 0) return CTLAB_OK;
        T.tiles = tiles;
        T.n_full = T.n_blocks;
        T.n_blocks = n_tiles;
    }
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

// ----------------------------------------------------------------------------
// Reproducible 3-D adjoint: the walks' contributions added as 64-bit
// integers (RedFixed), then converted to float once per voxel.
// ----------------------------------------------------------------------------

// The column walks (either voxel rule) over one sinogram per blockIdx.y,
// into its int64 volume.
template <bool MID, int W>
__global__ void __launch_bounds__(256, MID ? CTLAB_MID_MIN_BLOCKS_ADJ : CTLAB_XY_MIN_BLOCKS_ADJ)
    siddon3d_fixed_column_kernel(const float* __restrict__ in, float* __restrict__ sums,
                                 const float* __restrict__ src, const float* __restrict__ dst, int64_t n_ray,
                                 const float* __restrict__ M_inv, const float* __restrict__ bvec, GridDims<3> G,
                                 int64_t nvox, Tiling T, const float* __restrict__ scale) {
    const Affine3 A = load_affine3(M_inv, bvec);
    const RedFixed acc{scale[blockIdx.y]};
    if constexpr (MID) {
        __shared__ float raw[256 / 32][kChunk];
        __shared__ MidCell rec[256 / 32][kChunk];
        shared_xy_ray_mid<true, 1, W, RedFixed>(in, sums, src, dst, n_ray, A, G, nvox, tile_ray(T), blockIdx.y, 1,
                                                raw[threadIdx.x >> 5], rec[threadIdx.x >> 5], acc);
    } else {
        __shared__ XYCell cells[256 / 32][kChunk];
        shared_xy_ray<true, 1, W, RedFixed>(in, sums, src, dst, n_ray, A, G, nvox, tile_ray(T), blockIdx.y, 1,
                                            cells[threadIdx.x >> 5], acc);
    }
}

// The per-lane walk (flat or irregular ray lists).
template <bool MID>
__global__ void __launch_bounds__(256) siddon3d_fixed_lane_kernel(
    const float* __restrict__ in, float* __restrict__ sums, const float* __restrict__ src,
    const float* __restrict__ dst, int64_t n_ray, const float* __restrict__ M_inv, const float* __restrict__ bvec,
    GridDims<3> G, int64_t nvox, Tiling T, const float* __restrict__ scale) {
    const int64_t r = tile_ray(T);
    if (r < 0) return;
    lane_ray<3, true, MID, RedFixed>(in, sums, src, dst, n_ray, load_affine3(M_inv, bvec), G, nvox, r, blockIdx.y,
                                     RedFixed{scale[blockIdx.y]});
}

// max |y| of each sinogram (blockIdx.y) as float bits: for non-negative
// floats the bit patterns order as the values do, so an unsigned atomicMax
// gives the same result in any order.
__global__ void __launch_bounds__(256) abs_max_kernel(const float* __restrict__ y, int64_t n_ray,
                                                      unsigned* __restrict__ out) {
    const int64_t b = blockIdx.y;
    unsigned m = 0u;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_ray; i += (int64_t)gridDim.x * blockDim.x)
        m = max(m, __float_as_uint(fabsf(y[b * n_ray + i])));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m != 0u) atomicMax(out + b, m);
}

// scale = 2^e per sinogram, e the largest integer with B * 2^e <= 2^61 for
// B = max|y| * L * n_ray, L the longest chord through the grid (the longest
// of the four world-space body diagonals of the box, M (+-n_x, +-n_y, n_z),
// with M the inverse of M^-1).  Every contribution |y| * (segment length) is
// at most max|y| * L and every voxel's sum at most B, so each contribution
// converts to an int64 below 2^61 and every sum stays below 2^61.  A
// sinogram holding NaN or inf gets a NaN scale (its volume comes out NaN).
// The sums are exact modulo 2^64: a partial sum that wraps past 2^63 on the
// way (pass 1's whole-cell terms before pass 2 takes them back) still ends
// at the exact final sum.
__global__ void fixed_scale_kernel(const unsigned* __restrict__ maxbits, int batch, const float* __restrict__ M_inv,
                                   GridDims<3> G, int64_t n_ray, float* __restrict__ scale) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= batch) return;
    double a[9];
    for (int i = 0; i < 9; ++i) a[i] = M_inv[i];
    const double c0 = a[4] * a[8] - a[5] * a[7], c1 = a[5] * a[6] - a[3] * a[8], c2 = a[3] * a[7] - a[4] * a[6];
    const double det = a[0] * c0 + a[1] * c1 + a[2] * c2;
    // M = adj(M^-1) / det (columns of the adjugate as rows: M[r][c] = cof[c][r] / det)
    const double m[9] = {c0 / det, (a[2] * a[7] - a[1] * a[8]) / det, (a[1] * a[5] - a[2] * a[4]) / det,
                         c1 / det, (a[0] * a[8] - a[2] * a[6]) / det, (a[2] * a[3] - a[0] * a[5]) / det,
                         c2 / det, (a[1] * a[6] - a[0] * a[7]) / det, (a[0] * a[4] - a[1] * a[3]) / det};
    double L = 0.0;
    for (int sx = -1; sx <= 1; sx += 2)
        for (int sy = -1; sy <= 1; sy += 2) {
            const double v[3] = {sx * (double)G.n[0], sy * (double)G.n[1], (double)G.n[2]};
            double q = 0.0;
            for (int r = 0; r < 3; ++r) {
                const double w = m[3 * r] * v[0] + m[3 * r + 1] * v[1] + m[3 * r + 2] * v[2];
                q += w * w;
            }
            L = fmax(L, sqrt(q));
        }
    const float ymax = __uint_as_float(maxbits[b]);
    const double bound = (double)ymax * L * (double)(n_ray > 0 ? n_ray : 1) * (1.0 + 1e-6);
    float out = 1.f;
    if (!isfinite(ymax) || !isfinite(bound)) {
        out = __int_as_float(0x7fc00000);
    } else if (bound > 0.0) {
        const int e = 61 - (int)ceil(log2(bound));
        // a bound beyond 2^181 has no float scale: the volume comes out NaN
        out = e < -120 ? __int_as_float(0x7fc00000) : ldexpf(1.f, min(e, 120));
    }
    scale[b] = out;
}

// out = sums / scale (exact in double: scale is a power of 2), rounded to
// float once; accumulate adds it to out.
__global__ void __launch_bounds__(256) fixed_to_float_kernel(const long long* __restrict__ sums,
                                                             const float* __restrict__ scale, int64_t nvox,
                                                             int64_t total, float* __restrict__ out, int accumulate) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const float v = (float)((double)sums[i] / (double)scale[i / nvox]);
        out[i] = accumulate ? out[i] + v : v;
    }
}

// ----------------------------------------------------------------------------
// Active tiles: the tiles of a tiling holding at least one ray that the walks
// charge.  Every walk tests a ray with lane_setup's checks (finite end
// points, a non-degenerate direction, an interval of the box inside [0, 1];
// traverse applies the same ones) before it charges anything, so the rays
// of every other tile add nothing and project to 0.
// ----------------------------------------------------------------------------

__global__ void __launch_bounds__(256) tile_live_kernel(const float* __restrict__ src, const float* __restrict__ dst,
                                                        const float* __restrict__ M_inv, const float* __restrict__ bvec,
                                                        GridDims<3> G, Tiling T, uint8_t* __restrict__ flags) {
    const int64_t r = tile_ray_at(T, blockIdx.x, threadIdx.x);
    bool live = false;
    if (r >= 0) {
        float sw[3], dw[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            sw[a] = ld_stream(src + r * 3 + a);
            dw[a] = ld_stream(dst + r * 3 + a);
        }
        LaneRay R;
        lane_setup(R, sw, dw, G, load_affine3(M_inv, bvec));
        live = R.live;
    }
    live = __syncthreads_or(live);
    if (threadIdx.x == 0) flags[blockIdx.x] = live ? 1 : 0;
}

// The flagged tile indices in ascending order (the launch order of the full
// tiling, so a list launch keeps its locality), by one CTA of 1024 threads:
// per chunk of 1024 flags a warp-ballot and shared-memory prefix count.
__global__ void __launch_bounds__(1024) compact_tiles_kernel(const uint8_t* __restrict__ flags, int64_t n,
                                                             int32_t* __restrict__ tiles_out,
                                                             int64_t* __restrict__ n_out) {
    __shared__ int warp_base[32];
    __shared__ int chunk_total;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t base = 0;
    for (int64_t start = 0; start < n; start += 1024) {
        const int64_t i = start + threadIdx.x;
        const bool f = i < n && flags[i] != 0;
        const unsigned bal = __ballot_sync(kFullMask, f);
        if (lane == 0) warp_base[warp] = __popc(bal);
        __syncthreads();
        if (warp == 0) {  // exclusive prefix over the 32 warp counts
            const int c = warp_base[lane];
            int incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(kFullMask, incl, o);
                if (lane >= o) incl += v;
            }
            warp_base[lane] = incl - c;
            if (lane == 31) chunk_total = incl;
        }
        __syncthreads();
        if (f) tiles_out[base + warp_base[warp] + __popc(bal & ((1u << lane) - 1u))] = (int32_t)i;
        base += chunk_total;
        __syncthreads();  // warp_base and chunk_total are rewritten by the next chunk
    }
    if (threadIdx.x == 0) *n_out = base;
}

// Bytes of the reproducible adjoint's workspace: a 256-byte-aligned header
// (per sinogram its max |y| bits and its scale) and an int64 volume per
// sinogram.
static int64_t fixed_header_bytes(int64_t batch) { return ((batch * 8 + 255) / 256) * 256; }

}  // namespace ctlab

using namespace ctlab;

extern "C" int64_t ctlab_tile_count(int64_t n_ray, const ctlab_ray_opts* tiling) {
    clear_error();
    if (n_ray < 1) return -1;
    Tiling T;
    if (resolve_tiling(tiling, n_ray, T) != CTLAB_OK || T.n_blocks > kMaxGrid) return -1;
    return T.n_blocks;
}

extern "C" int ctlab_active_tiles(const float* src, const float* dst, int64_t n_ray, const float* M_inv,
                                  const float* b, int64_t n_x, int64_t n_y, int64_t n_z,
                                  const ctlab_ray_opts* tiling, uint8_t* flags, int32_t* tiles_out, int64_t* n_out,
                                  void* stream) {
    clear_error();
    const char* what = "active_tiles";
    CTLAB_REQUIRE(n_ray >= 1, "%s: n_ray must be >= 1", what);
    CTLAB_REQUIRE(src && dst && M_inv && b && flags && tiles_out && n_out, "%s: null pointer", what);
    const int64_t dims[3] = {n_x, n_y, n_z};
    GridDims<3> G;
    int64_t nvox = 1, st = 1;
    for (int a = 0; a < 3; ++a) {
        CTLAB_REQUIRE(dims[a] >= 1 && dims[a] <= (1 << 22), "%s: grid dimension %d out of range", what, a);
        nvox *= dims[a];
    }
    CTLAB_REQUIRE(nvox < (1LL << 31), "%s: a volume of %lld voxels exceeds 2^31", what, (long long)nvox);
    for (int a = 2; a >= 0; --a) {
        G.n[a] = (int)dims[a];
        G.stride[a] = (int)st;
        st *= dims[a];
    }
    Tiling T;
    int rc = resolve_tiling(tiling, n_ray, T);
    if (rc) return rc;
    CTLAB_REQUIRE(T.n_blocks <= kMaxGrid, "%s: too many tiles", what);
    cudaStream_t s = as_stream(stream);
    tile_live_kernel<<<(unsigned)T.n_blocks, T.tile_rows * T.tile_cols, 0, s>>>(src, dst, M_inv, b, G, T, flags);
    rc = launch_status(what);
    if (rc) return rc;
    compact_tiles_kernel<<<1, 1024, 0, s>>>(flags, T.n_blocks, tiles_out, n_out);
    return launch_status(what);
}

extern "C" int64_t ctlab_back_project_3d_fixed_workspace_bytes(int64_t batch, int64_t n_x, int64_t n_y,
                                                               int64_t n_z) {
    if (batch < 1 || n_x < 1 || n_y < 1 || n_z < 1) return -1;
    return fixed_header_bytes(batch) + batch * n_x * n_y * n_z * 8;
}

extern "C" int ctlab_back_project_3d_fixed(const float* sino, int64_t batch, int64_t n_ray, const float* src,
                                           const float* dst, const float* M_inv, const float* b, int64_t n_x,
                                           int64_t n_y, int64_t n_z, float* out, int accumulate,
                                           const ctlab_ray_opts* tiling, const int32_t* tiles, int64_t n_tiles,
                                           void* workspace, int64_t workspace_bytes, void* stream) {
    clear_error();
    const char* what = "back_project_3d_fixed";
    CTLAB_REQUIRE(batch >= 1 && batch <= 65535, "%s: batch must be in [1, 65535], got %lld", what, (long long)batch);
    CTLAB_REQUIRE(n_ray >= 0, "%s: n_ray must be >= 0", what);
    const int64_t dims[3] = {n_x, n_y, n_z};
    GridDims<3> G;
    int64_t nvox = 1, st = 1;
    for (int a = 0; a < 3; ++a) {
        CTLAB_REQUIRE(dims[a] >= 1 && dims[a] <= (1 << 22), "%s: grid dimension %d out of range (%lld)", what, a,
                      (long long)dims[a]);
        nvox *= dims[a];
    }
    CTLAB_REQUIRE(nvox < (1LL << 31), "%s: a volume of %lld voxels exceeds 2^31", what, (long long)nvox);
    for (int a = 2; a >= 0; --a) {
        G.n[a] = (int)dims[a];
        G.stride[a] = (int)st;
        st *= dims[a];
    }
    CTLAB_REQUIRE(out && M_inv && b, "%s: null data pointer", what);
    CTLAB_REQUIRE(n_ray == 0 || (src && dst && sino), "%s: null src/dst/sinogram", what);
    const int64_t need = ctlab_back_project_3d_fixed_workspace_bytes(batch, n_x, n_y, n_z);
    CTLAB_REQUIRE(workspace != nullptr && workspace_bytes >= need && ((uintptr_t)workspace & 255) == 0,
                  "%s: workspace must be 256-byte aligned and hold %lld bytes (got %lld)", what, (long long)need,
                  (long long)workspace_bytes);
    cudaStream_t s = as_stream(stream);
    unsigned* maxbits = reinterpret_cast<unsigned*>(workspace);
    float* scale = reinterpret_cast<float*>(maxbits + batch);
    long long* sums = reinterpret_cast<long long*>(reinterpret_cast<char*>(workspace) + fixed_header_bytes(batch));
    CTLAB_CUDA_TRY(cudaMemsetAsync(workspace, 0, (size_t)need, s));
    if (n_ray > 0) {
        const int64_t per = (n_ray + 255) / 256;
        abs_max_kernel<<<dim3((unsigned)(per < 4096 ? per : 4096), (unsigned)batch), 256, 0, s>>>(sino, n_ray, maxbits);
        int rc = launch_status(what);
        if (rc) return rc;
    }
    fixed_scale_kernel<<<(unsigned)((batch + 127) / 128), 128, 0, s>>>(maxbits, (int)batch, M_inv, G, n_ray, scale);
    int rc = launch_status(what);
    if (rc) return rc;
    if (n_ray > 0) {
        Tiling T;
        rc = resolve_tiling(tiling, n_ray, T);
        if (rc) return rc;
        CTLAB_REQUIRE(T.n_blocks <= kMaxGrid, "%s: too many rays for one launch", what);
        if (n_tiles >= 0) {  // only the listed tiles (ctlab_active_tiles); the others add nothing
            CTLAB_REQUIRE(n_tiles <= T.n_blocks && (n_tiles == 0 || tiles != nullptr),
                          "%s: bad tile list (%lld tiles of %lld)", what, (long long)n_tiles, (long long)T.n_blocks);
            T.tiles = tiles;
            T.n_full = T.n_blocks;
            T.n_blocks = n_tiles;
        }
        const int threads = T.tile_rows * T.tile_cols;
        const bool mid = tiling == nullptr || tiling->voxel_rule == CTLAB_VOXEL_MIDPOINT;
        const bool flat = tiling == nullptr || tiling->n_view == 0;
        const int walk = tiling == nullptr ? CTLAB_WALK_AUTO : tiling->walk;
        const bool small_grid = G.n[0] <= 65536 && G.n[1] <= 65536 && G.n[2] <= 65536;
        const dim3 g((unsigned)T.n_blocks, (unsigned)batch);
        float* o = reinterpret_cast<float*>(sums);
        if (T.n_blocks == 0) {
            // an empty tile list: nothing to walk (the sums stay zero)
        } else if (!flat && small_grid && (T.tile_rows % 32 == 0 || T.tile_rows == 16) &&
            (walk == CTLAB_WALK_COLUMN || walk == CTLAB_WALK_AUTO)) {
            if (T.tile_rows == 16) {
                if (mid) siddon3d_fixed_column_kernel<true, 16><<<g, threads, 0, s>>>(sino, o, src, dst, n_ray, M_inv, b, G, nvox, T, scale);
                else siddon3d_fixed_column_kernel<false, 16><<<g, threads, 0, s>>>(sino, o, src, dst, n_ray, M_inv, b, G, nvox, T, scale);
            } else {
                if (mid) siddon3d_fixed_column_kernel<true, 32><<<g, threads, 0, s>>>(sino, o, src, dst, n_ray, M_inv, b, G, nvox, T, scale);
                else siddon3d_fixed_column_kernel<false, 32><<<g, threads, 0, s>>>(sino, o, src, dst, n_ray, M_inv, b, G, nvox, T, scale);
            }
        } else if (mid) {
            siddon3d_fixed_lane_kernel<true><<<g, threads, 0, s>>>(sino, o, src, dst, n_ray, M_inv, b, G, nvox, T, scale);
        } else {
            siddon3d_fixed_lane_kernel<false><<<g, threads, 0, s>>>(sino, o, src, dst, n_ray, M_inv, b, G, nvox, T, scale);
        }
        rc = launch_status(what);
        if (rc) return rc;
    }
    const int64_t total = batch * nvox;
    const int64_t blocks = (total + 255) / 256;
    fixed_to_float_kernel<<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, s>>>(sums, scale, nvox, total,
                                                                                            out, accumulate);
    return launch_status(what);
}

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

extern "C" int ctlab_forward_project_3d_on_the_fly_tiles(const float* volume, int64_t batch, int64_t n_x,
                                                         int64_t n_y, int64_t n_z, const float* src, const float* dst,
                                                         int64_t n_ray, const float* M_inv, const float* b,
                                                         float* out, const ctlab_ray_opts* tiling,
                                                         const int32_t* tiles, int64_t n_tiles, void* stream) {
    clear_error();
    CTLAB_REQUIRE(n_tiles >= 0, "forward_project_3d_on_the_fly_tiles: n_tiles must be >= 0");
    const int64_t dims[3] = {n_x, n_y, n_z};
    return launch_siddon<3, false>("forward_project_3d_on_the_fly_tiles", volume, out, batch, dims, src, dst, n_ray,
                                   M_inv, b, 0, tiling, stream, nullptr, tiles, n_tiles);
}

extern "C" int ctlab_back_project_3d_on_the_fly_tiles(const float* sino, int64_t batch, int64_t n_ray,
                                                      const float* src, const float* dst, const float* M_inv,
                                                      const float* b, int64_t n_x, int64_t n_y, int64_t n_z,
                                                      float* out, int accumulate, const ctlab_ray_opts* tiling,
                                                      const int32_t* tiles, int64_t n_tiles, void* stream) {
    clear_error();
    CTLAB_REQUIRE(n_tiles >= 0, "back_project_3d_on_the_fly_tiles: n_tiles must be >= 0");
    const int64_t dims[3] = {n_x, n_y, n_z};
    return launch_siddon<3, true>("back_project_3d_on_the_fly_tiles", sino, out, batch, dims, src, dst, n_ray, M_inv,
                                  b, accumulate, tiling, stream, nullptr, tiles, n_tiles);
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
