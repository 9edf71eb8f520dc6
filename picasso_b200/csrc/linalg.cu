// Batched 3x3 determinant / inverse / inverse-times-vector, FP64, one thread
// per matrix with the 9 loads staged through shared memory so that the
// row-major array is read with unit-stride warp accesses.
#include "common.cuh"

namespace pb {

__global__ void __launch_bounds__(128)
mat3_inverse_kernel(int64_t n, const double* __restrict__ a, double* __restrict__ a_inv,
                    double* __restrict__ det, const double* __restrict__ x,
                    double* __restrict__ y)
{
    __shared__ double sa[128 * 9];
    __shared__ double sinv[128 * 9];
    for (int64_t base = (int64_t)blockIdx.x * 128; base < n; base += (int64_t)gridDim.x * 128) {
        const int cnt = (int)((n - base) < 128 ? (n - base) : 128);
        for (int e = threadIdx.x; e < cnt * 9; e += 128) sa[e] = a[base * 9 + e];
        __syncthreads();
        if (threadIdx.x < cnt) {
            const double* m = sa + threadIdx.x * 9;
            // BatchedLinearAlgebra.hpp:4344-4349
            const double dt = m[0] * m[4] * m[8] + m[1] * m[5] * m[6] + m[2] * m[3] * m[7] -
                              m[2] * m[4] * m[6] - m[1] * m[3] * m[8] - m[0] * m[5] * m[7];
            // BatchedLinearAlgebra.hpp:4637-4670
            const double r = 1.0 / dt;
            double inv[9];
            inv[0] = (m[4] * m[8] - m[5] * m[7]) * r;
            inv[1] = (m[2] * m[7] - m[1] * m[8]) * r;
            inv[2] = (m[1] * m[5] - m[2] * m[4]) * r;
            inv[3] = (m[5] * m[6] - m[3] * m[8]) * r;
            inv[4] = (m[0] * m[8] - m[2] * m[6]) * r;
            inv[5] = (m[2] * m[3] - m[0] * m[5]) * r;
            inv[6] = (m[3] * m[7] - m[4] * m[6]) * r;
            inv[7] = (m[1] * m[6] - m[0] * m[7]) * r;
            inv[8] = (m[0] * m[4] - m[1] * m[3]) * r;
            const int64_t b = base + threadIdx.x;
            if (det) det[b] = dt;
            if (x && y) {
                const double xv[3] = {x[3 * b], x[3 * b + 1], x[3 * b + 2]};
#pragma unroll
                for (int i = 0; i < 3; ++i) {
                    double s = 0.0;
#pragma unroll
                    for (int j = 0; j < 3; ++j) s += inv[3 * i + j] * xv[j];
                    y[3 * b + i] = s;
                }
            }
#pragma unroll
            for (int q = 0; q < 9; ++q) sinv[threadIdx.x * 9 + q] = inv[q];
        }
        __syncthreads();
        if (a_inv)
            for (int e = threadIdx.x; e < cnt * 9; e += 128) a_inv[base * 9 + e] = sinv[e];
        __syncthreads();
    }
}

}  // namespace pb

extern "C" picasso_status picasso_mat3_inverse(int64_t n, const double* a, double* a_inv,
                                               double* det, const double* x, double* y,
                                               const picasso_exec* exec)
{
    if (n < 0 || (n > 0 && !a)) return PICASSO_ERR_INVALID_ARGUMENT;
    if ((x == nullptr) != (y == nullptr)) return PICASSO_ERR_INVALID_ARGUMENT;
    if (n == 0) return PICASSO_OK;
    const unsigned blocks = pb::grid_for(n, 128);
    pb::mat3_inverse_kernel<<<blocks, 128, 0, pb::stream_of(exec)>>>(n, a, a_inv, det, x, y);
    return pb::check_launch();
}
