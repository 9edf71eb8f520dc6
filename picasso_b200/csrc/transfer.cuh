// Spline dispatch by arithmetic type and APIC constants shared by the plain
// and tiled transfer kernels.
#pragma once

#include <type_traits>

#include "common.cuh"

namespace pb {

// Storage / arithmetic form of a P2G call: all FP64 with FP64 atomics; FP32
// particles with 64-bit fixed-point grid; FP64 particles with fixed-point grid.
enum class Form { F64, F32Fixed, F64Fixed };

// FP64 arithmetic follows the oracle's expressions; reduced precision forms
// the weights from the in-cell fraction (see spline_eval_frac).
template <int ORDER, class R>
__device__ __forceinline__ void eval_spline(double x, double lo, double dx, double rdx,
                                            Spline1D<ORDER, R>& sp)
{
    if constexpr (std::is_same<R, double>::value)
        spline_eval_f64<ORDER>(x, lo, dx, rdx, sp);
    else
        spline_eval_frac<ORDER, R>(x, lo, dx, rdx, sp);
}

// APIC inertial tensor scaling D_p^-1 (Picasso_APIC.hpp:33-47): 4/dx^2 for
// quadratic, 3/dx^2 for cubic splines, from the first dimension's cell size.
template <int ORDER, class R>
__device__ __forceinline__ R inertial_scaling(double dx0)
{
    return (R)((ORDER == 2 ? 4.0 : 3.0) / (dx0 * dx0));
}

// Select element `sel` of a small register array without dynamic indexing.
template <int N, class R>
__device__ __forceinline__ R select(const R (&v)[N], int sel)
{
    R r = v[0];
#pragma unroll
    for (int q = 1; q < N; ++q)
        if (q == sel) r = v[q];
    return r;
}

}  // namespace pb
