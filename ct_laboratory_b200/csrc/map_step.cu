// map_step.cu — the elementwise steps of one MAP iteration, fused for the
// reconstruction server (sm_100a): the Beer-Lambert Poisson residual, and
// the quadratic smoothness prior's gradient with the gradient step.
//
// The reference forms these through autograd (its MAP estimator,
// bayesian_estimation/map_estimator.py:102-117, the Poisson likelihood,
// probability/random_variables/poisson.py:36-47, and the non-periodic
// quadratic smoothness energy, image_energies.py:18-29); written out, a job's
// iteration is
//     r = y - I0 exp(-p)                                   (p = A x)
//     g = A^T r + w sum_d D_d^T D_d x,   x <- x - lr g
// with D_d the forward difference along axis d (no wrap-around).  Each
// kernel makes one pass over its arrays instead of one pass per torch op.
#include "common.cuh"

namespace ctlab {

__global__ void __launch_bounds__(256) poisson_residual_kernel(const float* __restrict__ y,
                                                               const float* __restrict__ p, float* __restrict__ r,
                                                               int64_t n, float I0) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = __fadd_rn(__fmul_rn(-I0, expf(-p[i])), y[i]);
}

// g[v] += w * sum over the axes of (D^T D x)[v]: along an axis of length n
// at coordinate q, (x[v] - x[v - s]) when q >= 1 minus (x[v + s] - x[v])
// when q <= n - 2 (s the axis stride; the volume is [nx][ny][nz], z fastest).
// x is only read, so every thread sees the iteration's x.
__global__ void __launch_bounds__(256) smoothness_grad_kernel(const float* __restrict__ x, float* __restrict__ g,
                                                              int nx, int ny, int nz, float w) {
    const int64_t n = (int64_t)nx * ny * nz;
    const int64_t sy = nz, sx = (int64_t)ny * nz;
    for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(v % nz);
        const int64_t t = v / nz;
        const int b = (int)(t % ny);
        const int a = (int)(t / ny);
        const float xv = x[v];
        float acc = 0.f;
        if (a >= 1) acc = __fadd_rn(acc, __fsub_rn(xv, x[v - sx]));
        if (a <= nx - 2) acc = __fsub_rn(acc, __fsub_rn(x[v + sx], xv));
        if (b >= 1) acc = __fadd_rn(acc, __fsub_rn(xv, x[v - sy]));
        if (b <= ny - 2) acc = __fsub_rn(acc, __fsub_rn(x[v + sy], xv));
        if (c >= 1) acc = __fadd_rn(acc, __fsub_rn(xv, x[v - 1]));
        if (c <= nz - 2) acc = __fsub_rn(acc, __fsub_rn(x[v + 1], xv));
        g[v] = __fmaf_rn(w, acc, g[v]);
    }
}

__global__ void __launch_bounds__(256) gradient_step_kernel(float* __restrict__ x, const float* __restrict__ g,
                                                            int64_t n, float lr) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = __fmaf_rn(-lr, g[i], x[i]);
}

// Grid-stride launches: up to 8 CTAs of 256 threads per SM.
static unsigned elementwise_blocks(int64_t n) {
    const int64_t b = (n + 255) / 256;
    return (unsigned)(b < 148 * 8 ? (b > 0 ? b : 1) : 148 * 8);
}

}  // namespace ctlab

using namespace ctlab;

extern "C" int ctlab_map_poisson_residual(const float* y, const float* p, float* r, int64_t n, float I0,
                                          void* stream) {
    clear_error();
    CTLAB_REQUIRE(n >= 0, "map_poisson_residual: n must be >= 0");
    if (n == 0) return CTLAB_OK;
    CTLAB_REQUIRE(y && p && r, "map_poisson_residual: null data pointer");
    poisson_residual_kernel<<<elementwise_blocks(n), 256, 0, as_stream(stream)>>>(y, p, r, n, I0);
    return launch_status("map_poisson_residual");
}

extern "C" int ctlab_map_smoothness_step(float* x, float* g, int64_t n_x, int64_t n_y, int64_t n_z, float w,
                                         float lr, void* stream) {
    clear_error();
    CTLAB_REQUIRE(n_x >= 1 && n_y >= 1 && n_z >= 1 && n_x <= (1 << 22) && n_y <= (1 << 22) && n_z <= (1 << 22),
                  "map_smoothness_step: volume dimensions out of range (%lld, %lld, %lld)", (long long)n_x,
                  (long long)n_y, (long long)n_z);
    CTLAB_REQUIRE(x && g, "map_smoothness_step: null data pointer");
    const int64_t n = n_x * n_y * n_z;
    cudaStream_t s = as_stream(stream);
    smoothness_grad_kernel<<<elementwise_blocks(n), 256, 0, s>>>(x, g, (int)n_x, (int)n_y, (int)n_z, w);
    int rc = launch_status("map_smoothness_step");
    if (rc) return rc;
    gradient_step_kernel<<<elementwise_blocks(n), 256, 0, s>>>(x, g, n, lr);
    return launch_status("map_smoothness_step");
}
