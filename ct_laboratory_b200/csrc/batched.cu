// batched.cu — many scans in one persistent launch (sm_100a).
//
// A reconstruction service or a study with many small scans calls the
// projector once per scan: dozens of launches of a few hundred CTAs each,
// most of them too small to fill 148 SMs, each paying launch latency and a
// tail where the GPU drains.  Here the scans of a batch (uneven image sizes,
// view counts and geometries: fan-beam views, StaticCT rings, cone-beam
// scans) are cut into ray tiles, laid end to end, and one launch of
// persistent CTAs (resident CTAs per SM x SMs) works through them: every warp
// pulls its next slice of a tile from a device work counter until the batch
// is done.  Scans are listed heaviest first by the
// caller (the Python planner orders them), so the long tiles start early and
// the short ones fill the tail.
//
// Every tile is walked by the same device code as the single-scan kernels
// (walk.cuh): 2-D scans by the per-lane walk, 3-D crossing-rule scans by the
// shared x-y column walk (which falls back to the per-lane walk in warps
// whose rays do not share their x-y line), midpoint-rule scans by the
// per-lane midpoint walk.  Results are therefore those of the single-scan
// entry points: bitwise for the forward; for the adjoint up to the order of
// the float atomic additions.
//
// Scratch: a plan's workspace (device memory the caller allocates, size from
// ctlab_batch_workspace_bytes) holds the work counter and the scan
// descriptor table.  ctlab_batch_plan validates the scans on the host and
// copies the table in once; the launch entry points then only reset the
// counter (cudaMemsetAsync) and launch, so they can be replayed from a CUDA
// graph as long as the bound buffers stay where they are.
#include "walk.cuh"

#include <atomic>
#include <vector>

namespace ctlab {

// Resolved scan descriptor as the kernels read it.
struct ScanDev {
    const float* image_in;
    float* sino_out;
    const float* sino_in;
    float* image_out;
    const float* src;
    const float* dst;
    const float* M_inv;
    const float* b;
    int64_t n_ray;
    int64_t nvox;
    Tiling T;
    int64_t first_tile;  // first tile of this scan in the batch
    int n[3], stride[3];
    float* image_t;  // 2-D crossing-rule adjoint: transposed accumulation (or NULL)
};

struct BatchHeader {
    unsigned counter;  // next tile to hand out
    unsigned pad[63];  // keeps the descriptor table 256-byte aligned
};
static_assert(sizeof(BatchHeader) == 256, "header must be 256 bytes");

constexpr int64_t kMaxBatchScans = 65535;        // grid.y of the zeroing kernel
constexpr int64_t kMaxBatchTiles = 1LL << 31;    // the work counter is 32-bit

static int64_t table_bytes(int64_t n_scan) {
    return ((n_scan * (int64_t)sizeof(ScanDev) + 255) / 256) * 256;
}

// Scan index of tile t: the last scan whose first tile is <= t (scans with
// no tiles share their first tile with the next one and are skipped).
__device__ __forceinline__ int find_scan(const ScanDev* __restrict__ scans, int n_scan, unsigned t) {
    int lo = 0, hi = n_scan - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if ((unsigned)__ldg(&scans[mid].first_tile) <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Resident CTAs per SM the register allocation of the batched kernels targets.
// The 3-D forward targets 3: inside the persistent loop its column walk
// needs more than the 64 registers a thread gets at 4 (it spilled 228 bytes
// there and measured 9.98 ms on the cone256 scan, 9.69 ms at 3).
#ifndef CTLAB_BATCH_MIN_BLOCKS
#define CTLAB_BATCH_MIN_BLOCKS 4
#endif
#ifndef CTLAB_BATCH_MIN_BLOCKS_3D_FWD
#define CTLAB_BATCH_MIN_BLOCKS_3D_FWD 3
#endif

// Persistent warps: each warp takes the next work item -- one warp's slice
// (32 threads) of one tile -- from the device counter, walks its rays and
// repeats, with no CTA-wide barrier: a warp never waits for its CTA's other
// warps or for a tile hand-off.  Items are numbered tile-major (item = tile *
// warps_per_tile + warp slot), so the warps resident at a time work on
// neighbouring tiles.  MID selects the midpoint voxel rule for every scan of
// the batch.  The column walk's collective steps only need the warp itself.
template <int NDIM, bool ADJ, bool MID>
__global__ void __launch_bounds__(256, (NDIM == 3 && !ADJ) ? CTLAB_BATCH_MIN_BLOCKS_3D_FWD : CTLAB_BATCH_MIN_BLOCKS)
    batched_kernel(const ScanDev* __restrict__ scans, int n_scan, unsigned total_items, unsigned* __restrict__ counter) {
    __shared__ XYCell cells[256 / 32][kChunk];
    const int lane = threadIdx.x & 31;
    XYCell* buf = cells[threadIdx.x >> 5];
    const unsigned warps_per_tile = blockDim.x >> 5;
#pragma unroll 1
    for (;;) {
        unsigned item = 0;
        if (lane == 0) item = atomicAdd(counter, 1u);
        item = __shfl_sync(kFullMask, item, 0);
        if (item >= total_items) return;
        const unsigned t = item / warps_per_tile;
        const unsigned slot = item - t * warps_per_tile;
        const ScanDev* S = scans + find_scan(scans, n_scan, t);
        Tiling T;
        T.n_view = S->T.n_view;
        T.n_row = S->T.n_row;
        T.n_col = S->T.n_col;
        T.view_stride = S->T.view_stride;
        T.row_stride = S->T.row_stride;
        T.col_stride = S->T.col_stride;
        T.tile_rows = S->T.tile_rows;
        T.tile_cols = S->T.tile_cols;
        T.tiles_r = S->T.tiles_r;
        T.tiles_c = S->T.tiles_c;
        T.n_blocks = S->T.n_blocks;
        const int64_t r = tile_ray_at(T, t - (unsigned)S->first_tile, (int)(slot * 32 + lane));
        const float* in = ADJ ? S->sino_in : S->image_in;
        float* out = ADJ ? S->image_out : S->sino_out;
        const int64_t n_ray = S->n_ray, nvox = S->nvox;
        GridDims<NDIM> G;
#pragma unroll
        for (int a = 0; a < NDIM; ++a) {
            G.n[a] = S->n[a];
            G.stride[a] = S->stride[a];
        }
        if constexpr (NDIM == 3) {
            const Affine3 A = load_affine3(S->M_inv, S->b);
            if constexpr (MID) {
                if (r >= 0) lane_ray<3, ADJ, true>(in, out, S->src, S->dst, n_ray, A, G, nvox, r, 0);
            } else if (ADJ && T.tile_rows == 16) {
                // 16 rows per column (a warp-uniform branch: one scan per warp).  The
                // adjoint only: the forward with both walks inlined spills; a batch's
                // 3-D forward runs scan by scan by default, on the single-scan kernels.
                shared_xy_ray<ADJ, 1, 16>(in, out, S->src, S->dst, n_ray, A, G, nvox, r, 0, 1, buf);
            } else {
                shared_xy_ray<ADJ, 1>(in, out, S->src, S->dst, n_ray, A, G, nvox, r, 0, 1, buf);
            }
        } else {
            const Affine2 A = load_affine2(S->M_inv, S->b);
            if constexpr (ADJ && CTLAB_MAJOR2_WARP) {
                major2_adjoint_warp<MID>(in, out, S->image_t, S->src, S->dst, n_ray, A, G, nvox, r, 0);
            } else if (r >= 0) {
                lane_ray<2, ADJ, MID>(in, out, S->src, S->dst, n_ray, A, G, nvox, r, 0);
            }
        }
        __syncwarp();
    }
}

__device__ __forceinline__ void zero_span(float* p, int64_t n) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if ((reinterpret_cast<uintptr_t>(p) & 15u) == 0) {
        float4* q = reinterpret_cast<float4*>(p);
        const int64_t n4 = n >> 2;
        for (int64_t i = i0; i < n4; i += stride) q[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int64_t i = (n4 << 2) + i0; i < n; i += stride) p[i] = 0.f;
    } else {
        for (int64_t i = i0; i < n; i += stride) p[i] = 0.f;
    }
}

// Zeroes every scan's image_out (zero_out) and transposed scratch:
// blockIdx.y = scan, grid-stride in float4 where the buffer is 16-byte
// aligned.
__global__ void batched_zero_kernel(const ScanDev* __restrict__ scans, int zero_out) {
    const ScanDev* S = scans + blockIdx.y;
    if (zero_out && S->image_out != nullptr) zero_span(S->image_out, S->nvox);
    if (S->image_t != nullptr) zero_span(S->image_t, S->nvox);
}

// image_out[i0][i1] += image_t[i1][i0] for every scan with scratch
// (blockIdx.y = scan): 32 x 32 tiles through shared memory, grid-stride over
// the scan's tiles, so both sides are read and written coalesced.
__global__ void __launch_bounds__(256) batched_add_transposed_kernel(const ScanDev* __restrict__ scans) {
    __shared__ float tile[32][33];
    const ScanDev* S = scans + blockIdx.y;
    const float* __restrict__ T = S->image_t;
    float* __restrict__ out = S->image_out;
    if (T == nullptr || out == nullptr) return;
    const int n0 = S->n[0], n1 = S->n[1];
    const int t0 = (n0 + 31) >> 5, t1 = (n1 + 31) >> 5;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int k = blockIdx.x; k < t0 * t1; k += gridDim.x) {
        const int i0b = (k / t1) << 5, i1b = (k % t1) << 5;
        __syncthreads();  // the previous tile has been read out
#pragma unroll
        for (int r = ty; r < 32; r += 8) {
            const int i1 = i1b + r, i0 = i0b + tx;
            if (i1 < n1 && i0 < n0) tile[r][tx] = T[(int64_t)i1 * n0 + i0];
        }
        __syncthreads();
#pragma unroll
        for (int r = ty; r < 32; r += 8) {
            const int i0 = i0b + r, i1 = i1b + tx;
            if (i0 < n0 && i1 < n1) out[(int64_t)i0 * n1 + i1] += tile[tx][r];
        }
    }
}

// ----------------------------------------------------------------------------
// host side
// ----------------------------------------------------------------------------

// Validates one scan and resolves it into `D`; `what` names it in messages.
static int resolve_scan(const ctlab_scan& s, int64_t idx, int ndim, int block_threads, int voxel_rule, ScanDev& D) {
    CTLAB_REQUIRE(s.ndim == ndim, "batch: scan %lld has ndim %d, the batch's first scan has %d", (long long)idx,
                  s.ndim, ndim);
    CTLAB_REQUIRE(s.n_ray >= 0, "batch: scan %lld has n_ray < 0", (long long)idx);
    int64_t nvox = 1;
    for (int a = 0; a < ndim; ++a) {
        const int64_t lim = ndim == 3 ? 65536 : (1 << 22);
        CTLAB_REQUIRE(s.dims[a] >= 1 && s.dims[a] <= lim, "batch: scan %lld grid dimension %d out of range (%lld)",
                      (long long)idx, a, (long long)s.dims[a]);
        nvox *= s.dims[a];
    }
    CTLAB_REQUIRE(nvox < (1LL << 31), "batch: scan %lld has %lld voxels (limit 2^31)", (long long)idx,
                  (long long)nvox);
    CTLAB_REQUIRE(s.M_inv && s.b, "batch: scan %lld has a null M_inv or b", (long long)idx);
    CTLAB_REQUIRE(s.n_ray == 0 || (s.src && s.dst), "batch: scan %lld has null src/dst", (long long)idx);
    CTLAB_REQUIRE(s.image_in || s.sino_out || s.sino_in || s.image_out, "batch: scan %lld binds no buffer",
                  (long long)idx);
    // A pass binds its image and its sinogram together; the sinogram of a
    // scan without rays may be NULL (an empty buffer).
    const bool fwd = s.image_in || s.sino_out, adj = s.sino_in || s.image_out;
    CTLAB_REQUIRE(!fwd || (s.image_in && (s.sino_out || s.n_ray == 0)),
                  "batch: scan %lld: image_in and sino_out must be given together", (long long)idx);
    CTLAB_REQUIRE(!adj || (s.image_out && (s.sino_in || s.n_ray == 0)),
                  "batch: scan %lld: sino_in and image_out must be given together", (long long)idx);
    const int rule = s.opts.voxel_rule;
    CTLAB_REQUIRE(rule == voxel_rule, "batch: scan %lld has voxel_rule %d, the batch's first scan has %d",
                  (long long)idx, rule, voxel_rule);
    CTLAB_REQUIRE(s.opts.block_threads == 0 || s.opts.block_threads == block_threads,
                  "batch: scan %lld asks for %d threads per tile, the batch runs %d", (long long)idx,
                  s.opts.block_threads, block_threads);
    ctlab_ray_opts o = s.opts;
    o.block_threads = block_threads;
    Tiling T;
    int rc = resolve_tiling(&o, s.n_ray, T);
    if (rc) return rc;
    D.image_in = s.image_in;
    D.sino_out = s.sino_out;
    D.sino_in = s.sino_in;
    D.image_out = s.image_out;
    D.src = s.src;
    D.dst = s.dst;
    D.M_inv = s.M_inv;
    D.b = s.b;
    D.n_ray = s.n_ray;
    D.nvox = nvox;
    D.T = T;
    int64_t st = 1;
    for (int a = 2; a >= 0; --a) {
        D.n[a] = a < ndim ? (int)s.dims[a] : 1;
        D.stride[a] = a < ndim ? (int)st : 0;
        if (a < ndim) st *= s.dims[a];
    }
    if (s.n_ray == 0) D.T.n_blocks = 0;
    // transposed accumulation: 2-D adjoints only
    D.image_t = (ndim == 2 && CTLAB_MAJOR2_WARP && s.image_out) ? s.image_scratch : nullptr;
    CTLAB_REQUIRE(D.image_t == nullptr || (D.image_t != s.image_out && (const float*)D.image_t != s.image_in),
                  "batch: scan %lld: image_scratch must be a buffer of its own", (long long)idx);
    return CTLAB_OK;
}

template <int NDIM, bool ADJ, bool MID>
static const void* batched_fn() {
    return reinterpret_cast<const void*>(&batched_kernel<NDIM, ADJ, MID>);
}

static const void* pick_kernel(int ndim, bool adj, bool mid) {
    if (ndim == 2) {
        if (adj) return mid ? batched_fn<2, true, true>() : batched_fn<2, true, false>();
        return mid ? batched_fn<2, false, true>() : batched_fn<2, false, false>();
    }
    if (adj) return mid ? batched_fn<3, true, true>() : batched_fn<3, true, false>();
    return mid ? batched_fn<3, false, true>() : batched_fn<3, false, false>();
}

static int default_ctas(const void* fn, int block_threads, int* n_cta) {
    int dev = 0, sms = 0, per_sm = 0;
    CTLAB_CUDA_TRY(cudaGetDevice(&dev));
    CTLAB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    CTLAB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, block_threads, 0));
    *n_cta = (per_sm < 1 ? 1 : per_sm) * sms;
    return CTLAB_OK;
}

static int launch_batched(const ctlab_batch* plan, bool adj, int accumulate, int32_t n_cta, void* stream) {
    const char* what = adj ? "back_project_batched" : "forward_project_batched";
    CTLAB_REQUIRE(plan != nullptr && plan->workspace != nullptr, "%s: null plan", what);
    CTLAB_REQUIRE(plan->n_scan >= 1 && (plan->ndim == 2 || plan->ndim == 3), "%s: plan is not initialised", what);
    CTLAB_REQUIRE(adj ? plan->has_adjoint : plan->has_forward, "%s: the plan's scans bind no %s buffers", what,
                  adj ? "adjoint" : "forward");
    CTLAB_REQUIRE(n_cta >= 0, "%s: n_cta must be >= 0 (0 = resident CTAs per SM x SMs)", what);
    int dev = 0;
    CTLAB_CUDA_TRY(cudaGetDevice(&dev));
    CTLAB_REQUIRE(dev == plan->device, "%s: the plan was made on device %d, the current device is %d", what,
                  plan->device, dev);
    cudaStream_t s = as_stream(stream);
    char* ws = static_cast<char*>(plan->workspace);
    const ScanDev* table = reinterpret_cast<const ScanDev*>(ws + sizeof(BatchHeader));
    unsigned* counter = reinterpret_cast<unsigned*>(ws);
    const bool scratch = adj && plan->has_scratch;
    if (adj && (!accumulate || scratch)) {
        batched_zero_kernel<<<dim3(64, (unsigned)plan->n_scan), 256, 0, s>>>(table, accumulate ? 0 : 1);
        int rc = launch_status(what);
        if (rc) return rc;
    }
    if (plan->total_tiles == 0) return CTLAB_OK;
    const bool mid = plan->voxel_rule == CTLAB_VOXEL_MIDPOINT;
    const void* fn = pick_kernel(plan->ndim, adj, mid);
    int ctas = n_cta;
    if (ctas == 0) {
        int rc = default_ctas(fn, plan->block_threads, &ctas);
        if (rc) return rc;
    }
    CTLAB_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned), s));
    const unsigned total = (unsigned)(plan->total_tiles * (plan->block_threads / 32));
    const int n_scan = plan->n_scan;
    void* args[] = {(void*)&table, (void*)&n_scan, (void*)&total, (void*)&counter};
    CTLAB_CUDA_TRY(cudaLaunchKernel(fn, dim3((unsigned)ctas), dim3((unsigned)plan->block_threads), args, 0, s));
    if (scratch) {
        int rc = launch_status(what);
        if (rc) return rc;
        batched_add_transposed_kernel<<<dim3(256, (unsigned)plan->n_scan), 256, 0, s>>>(table);
    }
    return launch_status(what);
}

}  // namespace ctlab

using namespace ctlab;

extern "C" int64_t ctlab_batch_workspace_bytes(int32_t n_scan) {
    if (n_scan < 1 || n_scan > kMaxBatchScans) return -1;
    return (int64_t)sizeof(BatchHeader) + table_bytes(n_scan);
}

extern "C" int ctlab_batch_plan(const ctlab_scan* scans, int32_t n_scan, int32_t block_threads, void* workspace,
                                int64_t workspace_bytes, ctlab_batch* plan, void* stream) {
    clear_error();
    CTLAB_REQUIRE(scans != nullptr && plan != nullptr, "batch_plan: null scans or plan");
    CTLAB_REQUIRE(n_scan >= 1 && n_scan <= kMaxBatchScans, "batch_plan: n_scan must be in [1, %lld] (got %d)",
                  (long long)kMaxBatchScans, n_scan);
    if (block_threads == 0) block_threads = 256;
    CTLAB_REQUIRE(block_threads >= 32 && block_threads <= 256 && block_threads % 32 == 0,
                  "batch_plan: block_threads must be a multiple of 32 in [32, 256] (got %d)", block_threads);
    const int64_t need = ctlab_batch_workspace_bytes(n_scan);
    CTLAB_REQUIRE(workspace != nullptr && workspace_bytes >= need,
                  "batch_plan: workspace of %lld bytes is too small (%lld needed for %d scans)",
                  (long long)workspace_bytes, (long long)need, n_scan);
    CTLAB_REQUIRE((reinterpret_cast<uintptr_t>(workspace) & 255u) == 0, "batch_plan: workspace must be 256-byte aligned");
    const int ndim = scans[0].ndim;
    CTLAB_REQUIRE(ndim == 2 || ndim == 3, "batch_plan: ndim must be 2 or 3 (got %d)", ndim);
    const int rule = scans[0].opts.voxel_rule;
    CTLAB_REQUIRE(rule == CTLAB_VOXEL_MIDPOINT || rule == CTLAB_VOXEL_CROSSING, "batch_plan: unknown voxel_rule %d",
                  rule);
    std::vector<ScanDev> table((size_t)n_scan);
    int64_t tiles = 0;
    bool fwd = false, adj = false, has_scratch = false;
    for (int32_t i = 0; i < n_scan; ++i) {
        int rc = resolve_scan(scans[i], i, ndim, block_threads, rule, table[i]);
        if (rc) return rc;
        table[i].first_tile = tiles;
        tiles += table[i].T.n_blocks;
        CTLAB_REQUIRE(tiles * (block_threads / 32) < kMaxBatchTiles,
                      "batch_plan: more than 2^31 warp work items in one batch");
        fwd = fwd || scans[i].image_in != nullptr;
        adj = adj || scans[i].image_out != nullptr;
        has_scratch = has_scratch || table[i].image_t != nullptr;
    }
    int dev = 0;
    CTLAB_CUDA_TRY(cudaGetDevice(&dev));
    char* ws = static_cast<char*>(workspace);
    cudaStream_t s = as_stream(stream);
    CTLAB_CUDA_TRY(cudaMemsetAsync(ws, 0, sizeof(BatchHeader), s));
    // From pageable host memory: the call returns once the table has been
    // staged, so `table` may be released right after it.
    CTLAB_CUDA_TRY(cudaMemcpyAsync(ws + sizeof(BatchHeader), table.data(), sizeof(ScanDev) * (size_t)n_scan,
                                   cudaMemcpyHostToDevice, s));
    plan->workspace = workspace;
    plan->total_tiles = tiles;
    plan->n_scan = n_scan;
    plan->ndim = ndim;
    plan->block_threads = block_threads;
    plan->voxel_rule = rule;
    plan->has_forward = fwd ? 1 : 0;
    plan->has_adjoint = adj ? 1 : 0;
    plan->device = dev;
    plan->has_scratch = has_scratch ? 1 : 0;
    return CTLAB_OK;
}

extern "C" int ctlab_forward_project_batched(const ctlab_batch* plan, int32_t n_cta, void* stream) {
    clear_error();
    return launch_batched(plan, false, 0, n_cta, stream);
}

extern "C" int ctlab_back_project_batched(const ctlab_batch* plan, int accumulate, int32_t n_cta, void* stream) {
    clear_error();
    return launch_batched(plan, true, accumulate, n_cta, stream);
}

extern "C" int ctlab_batch_default_ctas(int32_t ndim, int adjoint, int voxel_rule, int32_t block_threads,
                                        int32_t* n_cta) {
    clear_error();
    CTLAB_REQUIRE(n_cta != nullptr, "batch_default_ctas: null output");
    CTLAB_REQUIRE(ndim == 2 || ndim == 3, "batch_default_ctas: ndim must be 2 or 3");
    CTLAB_REQUIRE(block_threads >= 32 && block_threads <= 256 && block_threads % 32 == 0,
                  "batch_default_ctas: block_threads must be a multiple of 32 in [32, 256]");
    int v = 0;
    int rc = default_ctas(pick_kernel(ndim, adjoint != 0, voxel_rule == CTLAB_VOXEL_MIDPOINT), block_threads, &v);
    if (rc) return rc;
    *n_cta = v;
    return CTLAB_OK;
}

// ----------------------------------------------------------------------------
// The batched projector for callers that cannot allocate device memory.
//
// Some programs that link this library must not call cudaMalloc: a plugin
// inside a host application whose own allocator owns all of the GPU's memory
// (a framework caching allocator, an inference server with a fixed memory
// budget), or a real-time acquisition loop where an allocation could block
// or fail in the middle of a scan.  ctlab_batch_plan asks such a caller for
// a workspace it cannot provide; this entry point keeps the same scratch (the
// work counter and the resolved scan table) in a fixed array that is part of
// the library's own device image instead.
// ----------------------------------------------------------------------------
namespace ctlab {

constexpr int kNoAllocMaxScans = 64;
constexpr size_t kNoAllocBytes = sizeof(BatchHeader) + (size_t)kNoAllocMaxScans * sizeof(ScanDev);

// Every GPU that loads the library holds this array (about 13 KB) until
// the process exits.  Calls share it: it keeps the last call's table and
// counter, so each call rewrites the table and clears the counter.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of g_noalloc_scratch per device.  In host code the array's
// name is a host-side stand-in, not a device address, so the address is
// looked up with cudaGetSymbolAddress, once per device with that device
// current (the first call on each device), and cached by device ordinal.
// The cache assumes each device's primary context (the one the runtime API
// and torch use): a caller that pushes other driver-API contexts of the same
// device would be handed the primary context's address.
constexpr int kNoAllocMaxDevices = 64;
static std::atomic<void*> g_noalloc_addr[kNoAllocMaxDevices];

static int noalloc_scratch(void** out) {
    int dev = 0;
    CTLAB_CUDA_TRY(cudaGetDevice(&dev));
    CTLAB_REQUIRE(dev >= 0 && dev < kNoAllocMaxDevices, "project_batched_noalloc: device %d beyond the %d supported",
                  dev, kNoAllocMaxDevices);
    void* p = g_noalloc_addr[dev].load(std::memory_order_acquire);
    if (p == nullptr) {
        CTLAB_CUDA_TRY(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        g_noalloc_addr[dev].store(p, std::memory_order_release);
    }
    *out = p;
    return CTLAB_OK;
}

}  // namespace ctlab

extern "C" int ctlab_project_batched_noalloc(const ctlab_scan* scans, int32_t n_scan, int adjoint, int accumulate,
                                             int32_t block_threads, int32_t n_cta, void* stream) {
    clear_error();
    const char* what = "project_batched_noalloc";
    CTLAB_REQUIRE(scans != nullptr, "%s: null scans", what);
    CTLAB_REQUIRE(n_scan >= 1 && n_scan <= kNoAllocMaxScans,
                  "%s: n_scan must be in [1, %d], got %d (the library's fixed scratch holds at most %d scans; "
                  "larger batches need ctlab_batch_plan with a caller-allocated workspace)",
                  what, kNoAllocMaxScans, n_scan, kNoAllocMaxScans);
    if (block_threads == 0) block_threads = 256;
    CTLAB_REQUIRE(block_threads >= 32 && block_threads <= 256 && block_threads % 32 == 0,
                  "%s: block_threads must be a multiple of 32 in [32, 256] (got %d)", what, block_threads);
    CTLAB_REQUIRE(n_cta >= 0, "%s: n_cta must be >= 0 (0 = resident CTAs per SM x SMs)", what);
    const int ndim = scans[0].ndim;
    CTLAB_REQUIRE(ndim == 2 || ndim == 3, "%s: ndim must be 2 or 3 (got %d)", what, ndim);
    const int rule = scans[0].opts.voxel_rule;
    CTLAB_REQUIRE(rule == CTLAB_VOXEL_MIDPOINT || rule == CTLAB_VOXEL_CROSSING, "%s: unknown voxel_rule %d", what,
                  rule);
    ScanDev table[kNoAllocMaxScans];  // host stack, copied into the scratch below
    int64_t tiles = 0;
    bool has_scratch = false;
    for (int32_t i = 0; i < n_scan; ++i) {
        int rc = resolve_scan(scans[i], i, ndim, block_threads, rule, table[i]);
        if (rc) return rc;
        has_scratch = has_scratch || (adjoint && table[i].image_t != nullptr);
        const bool bound = adjoint ? scans[i].image_out != nullptr : scans[i].image_in != nullptr;
        CTLAB_REQUIRE(bound, "%s: scan %d binds no %s buffers", what, i, adjoint ? "adjoint" : "forward");
        table[i].first_tile = tiles;
        tiles += table[i].T.n_blocks;
        CTLAB_REQUIRE(tiles * (block_threads / 32) < kMaxBatchTiles, "%s: more than 2^31 warp work items in one batch",
                      what);
    }
    void* base = nullptr;
    int rc = noalloc_scratch(&base);
    if (rc) return rc;
    char* ws = static_cast<char*>(base);
    const ScanDev* dtable = reinterpret_cast<const ScanDev*>(ws + sizeof(BatchHeader));
    unsigned* counter = reinterpret_cast<unsigned*>(ws);
    cudaStream_t s = as_stream(stream);
    // From pageable (stack) memory: the copy waits for the stream's earlier
    // work and has taken the table when it returns.
    CTLAB_CUDA_TRY(cudaMemcpyAsync(ws + sizeof(BatchHeader), table, sizeof(ScanDev) * (size_t)n_scan,
                                   cudaMemcpyHostToDevice, s));
    CTLAB_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned), s));
    if (adjoint && (!accumulate || has_scratch)) {
        batched_zero_kernel<<<dim3(64, (unsigned)n_scan), 256, 0, s>>>(dtable, accumulate ? 0 : 1);
        rc = launch_status(what);
        if (rc) return rc;
    }
    if (tiles == 0) return CTLAB_OK;
    const void* fn = pick_kernel(ndim, adjoint != 0, rule == CTLAB_VOXEL_MIDPOINT);
    int ctas = n_cta;
    if (ctas == 0) {
        rc = default_ctas(fn, block_threads, &ctas);
        if (rc) return rc;
    }
    const unsigned total = (unsigned)(tiles * (block_threads / 32));
    int n = n_scan;
    void* args[] = {(void*)&dtable, (void*)&n, (void*)&total, (void*)&counter};
    CTLAB_CUDA_TRY(cudaLaunchKernel(fn, dim3((unsigned)ctas), dim3((unsigned)block_threads), args, 0, s));
    if (has_scratch) {
        rc = launch_status(what);
        if (rc) return rc;
        batched_add_transposed_kernel<<<dim3(256, (unsigned)n_scan), 256, 0, s>>>(dtable);
    }
    return launch_status(what);
}
