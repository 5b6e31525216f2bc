// common.cuh — shared helpers of the B200 Siddon kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>

#include "ctlab_b200.h"

namespace ctlab {

// ----------------------------------------------------------------------------
// Host-side status plumbing
// ----------------------------------------------------------------------------

// Records a printf-style message as the calling thread's last error and
// returns `code`.
int set_error(int code, const char* fmt, ...);
void clear_error();

#define CTLAB_REQUIRE(cond, ...)                                  \
    do {                                                          \
        if (!(cond)) return ::ctlab::set_error(CTLAB_EINVAL, __VA_ARGS__); \
    } while (0)

#define CTLAB_CUDA_TRY(call)                                                              \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess)                                                            \
            return ::ctlab::set_error(CTLAB_ECUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

// After a launch: report configuration errors without synchronising.
inline int launch_status(const char* what) {
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_error(CTLAB_ECUDA, "%s launch failed: %s", what, cudaGetErrorString(e));
    }
    return CTLAB_OK;
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

constexpr int64_t kMaxGrid = 2147483647LL;

// ----------------------------------------------------------------------------
// Device helpers shared by every kernel.  Expressions the reference writes
// as a*b + c (which nvcc contracts into fused multiply-adds) are written here
// with explicit __fmaf_rn / __fmul_rn so the rounding is pinned and matches
// the reference's kernels, e.g. apply_affine_inverse_3d
// (ct_projector_3d.cu:21-36).
// ----------------------------------------------------------------------------

struct Affine3 {
    float m[9];
    float b[3];
};

struct Affine2 {
    float m[4];
    float b[2];
};

__device__ __forceinline__ Affine3 load_affine3(const float* __restrict__ M_inv, const float* __restrict__ b) {
    Affine3 a;
#pragma unroll
    for (int i = 0; i < 9; ++i) a.m[i] = __ldg(M_inv + i);
#pragma unroll
    for (int i = 0; i < 3; ++i) a.b[i] = __ldg(b + i);
    return a;
}

__device__ __forceinline__ Affine2 load_affine2(const float* __restrict__ M_inv, const float* __restrict__ b) {
    Affine2 a;
#pragma unroll
    for (int i = 0; i < 4; ++i) a.m[i] = __ldg(M_inv + i);
#pragma unroll
    for (int i = 0; i < 2; ++i) a.b[i] = __ldg(b + i);
    return a;
}

// a*b + c*d the way nvcc contracts it when both products have one use: the
// first product is fused, fma(a, b, c*d).  Set CTLAB_CONTRACT_FIRST=0 to fuse
// the second instead.
#ifndef CTLAB_CONTRACT_FIRST
#define CTLAB_CONTRACT_FIRST 1
#endif
__device__ __forceinline__ float mad2(float a, float b, float c, float d) {
#if CTLAB_CONTRACT_FIRST
    return __fmaf_rn(a, b, __fmul_rn(c, d));
#else
    return __fmaf_rn(c, d, __fmul_rn(a, b));
#endif
}

// x*x + y*y + z*z, left to right, contracted.
__device__ __forceinline__ float sumsq3(float x, float y, float z) { return __fmaf_rn(z, z, mad2(x, x, y, y)); }
__device__ __forceinline__ float sumsq2(float x, float y) { return mad2(x, x, y, y); }

__device__ __forceinline__ void world_to_index3(const Affine3& A, float x, float y, float z, float& i, float& j,
                                                float& k) {
    float xs = __fsub_rn(x, A.b[0]), ys = __fsub_rn(y, A.b[1]), zs = __fsub_rn(z, A.b[2]);
    i = __fmaf_rn(A.m[2], zs, mad2(A.m[0], xs, A.m[1], ys));
    j = __fmaf_rn(A.m[5], zs, mad2(A.m[3], xs, A.m[4], ys));
    k = __fmaf_rn(A.m[8], zs, mad2(A.m[6], xs, A.m[7], ys));
}

__device__ __forceinline__ void world_to_index2(const Affine2& A, float x, float y, float& r, float& c) {
    float xs = __fsub_rn(x, A.b[0]), ys = __fsub_rn(y, A.b[1]);
    r = mad2(A.m[0], xs, A.m[1], ys);
    c = mad2(A.m[2], xs, A.m[3], ys);
}

// Plane parameter of plane coordinate p along one axis: (p - s) * inv, the
// reciprocal-multiply form of collect_hits (ct_projector_3d.cu:866-868).
__device__ __forceinline__ float plane_t(float p, float s, float inv) { return __fmul_rn(__fsub_rn(p, s), inv); }

// Returns `p` as an opaque register value.  Inside a hot loop the compiler
// may otherwise re-derive a base pointer from the kernel parameters at every
// use (constant-bank loads plus 64-bit address arithmetic per access).
template <typename T>
__device__ __forceinline__ T* pin_ptr(T* p) {
    asm volatile("" : "+l"(p));
    return p;
}

// L2 eviction policies.  The volume is gathered over and over while the
// ray geometry and the sinogram stream through once; marking the volume
// evict-last and the streams evict-first keeps a volume of up to about half
// the 126 MB L2 resident while hundreds of MB of geometry pass by.
__device__ __forceinline__ uint64_t l2_policy_keep() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ float ld_keep(const float* p, uint64_t pol) {
    float v;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ void st_stream(float* p, float v) { __stcs(p, v); }

// red.global.add.f32 issued under a predicate: the reduction is one
// predicated instruction instead of a branch around an atomicAdd.
__device__ __forceinline__ void red_add_if(float* addr, float v, bool pred) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %2, 0;\n\t@p red.global.add.f32 [%0], %1;\n\t}" ::"l"(addr), "f"(v),
        "r"((int)pred)
        : "memory");
}

// red.global.add.u64 under a predicate (two's-complement: signed sums too).
__device__ __forceinline__ void red_add_u64_if(unsigned long long* addr, long long v, bool pred) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %2, 0;\n\t@p red.global.add.u64 [%0], %1;\n\t}" ::"l"(addr),
        "l"(v), "r"((int)pred)
        : "memory");
}

// How the 3-D adjoint walks accumulate a contribution v into voxel i of a
// volume: `at` offsets a volume base by `off` voxels, `add` adds.
//
// RedF32: float atomics into the float volume (the order of the additions,
// and so the last bits of a sum, depend on scheduling).
struct RedF32 {
    __device__ __forceinline__ float* at(float* base, int64_t off) const { return base + off; }
    __device__ __forceinline__ void add(float* p, unsigned i, float v, bool pred) const { red_add_if(p + i, v, pred); }
};

// RedFixed: every contribution rounded once to a multiple of 2^-e
// (v * scale, scale = 2^e, to the nearest integer) and added as a 64-bit
// integer.  Integer addition is associative, so a voxel's sum is the same
// bits in any order: the adjoint is reproducible run to run and whatever
// else shares the launch.  The volume base holds int64 sums (`p` is its
// address, typed as float* only to share the walks' signatures).
struct RedFixed {
    float scale;
    __device__ __forceinline__ float* at(float* base, int64_t off) const {
        return reinterpret_cast<float*>(reinterpret_cast<unsigned long long*>(base) + off);
    }
    __device__ __forceinline__ void add(float* p, unsigned i, float v, bool pred) const {
        red_add_u64_if(reinterpret_cast<unsigned long long*>(p) + i, __float2ll_rn(__fmul_rn(v, scale)), pred);
    }
};

// Ray tiling resolved on the host into plain integers for the kernels.
struct Tiling {
    int64_t n_view, n_row, n_col;
    int64_t view_stride, row_stride, col_stride;
    int tile_rows, tile_cols;       // tile_rows * tile_cols == blockDim.x
    int64_t tiles_r, tiles_c;       // tiles per view along rows / cols
    int64_t n_blocks;               // tiles launched: n_view * tiles_r * tiles_c, or the list's length
    const int32_t* tiles = nullptr; // optional list of the tiles to launch (device memory), block b -> tiles[b]
    int64_t n_full = 0;             // with a list: the tiling's n_view * tiles_r * tiles_c
};

// Validates `t` (may be NULL = flat) against n_ray and fills `out`.
int resolve_tiling(const ctlab_ray_opts* t, int64_t n_ray, Tiling& out);

// Ray handled by this thread, or -1 when the thread's slot is outside the grid.
//
// Blocks are numbered band-major: row tile outermost, then view, then column
// tile.  Blocks run roughly in index order, so the blocks resident at any
// moment share one band of detector rows across many views; for a cone-beam
// scan such a band sees a slab of the volume about tile_rows detector rows
// thick, and the volume voxels the whole GPU touches at a time stay a small,
// L2-resident fraction of the volume.  A scan has at most 2^31 - 1 tiles,
// so all tile coordinates fit 32-bit unsigned division.  `blk` is the tile
// index (the block index of a one-scan launch).
// `tid` is the thread's index within the tile (threadIdx.x for one tile per
// CTA; warp slot * 32 + lane when warps take tiles' slices on their own).
__device__ __forceinline__ int64_t tile_ray_at(const Tiling& T, unsigned blk, int tid) {
    const unsigned per_band = (unsigned)(T.n_view * T.tiles_c);
    const unsigned tr_u = blk / per_band;
    const unsigned rem = blk - tr_u * per_band;
    const unsigned view_u = rem / (unsigned)T.tiles_c;
    const int64_t view = view_u, tr = tr_u, tc = rem - view_u * (unsigned)T.tiles_c;
    const int lane_r = tid % T.tile_rows;
    const int lane_c = tid / T.tile_rows;
    int64_t row = tr * T.tile_rows + lane_r;
    int64_t col = tc * T.tile_cols + lane_c;
    if (row >= T.n_row || col >= T.n_col) return -1;
    return view * T.view_stride + row * T.row_stride + col * T.col_stride;
}

// The tile of this block: blockIdx.x, or its entry of the tile list (an
// entry outside the tiling gives no ray).
__device__ __forceinline__ int64_t tile_ray(const Tiling& T) {
    unsigned blk = blockIdx.x;
    if (T.tiles != nullptr) {
        const int32_t t = __ldg(T.tiles + blockIdx.x);
        if (t < 0 || (int64_t)t >= T.n_full) return -1;
        blk = (unsigned)t;
    }
    return tile_ray_at(T, blk, threadIdx.x);
}

}  // namespace ctlab
