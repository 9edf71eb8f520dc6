// picasso_b200.hpp -- C++ host interface with the names of Picasso's transfer
// API, over the C ABI of picasso_b200.h.
//
// A Picasso application calls, per particle inside a GridOperator loop,
//   APIC::p2g(m_p, c_p, m_i, mu_i, sd)      (src/Picasso_APIC.hpp:55-402)
//   APIC::g2p(u_i, c_p, sd)                 (src/Picasso_APIC.hpp:407-544)
//   PolyPIC::p2g(m_p, u_p, c_p, mu_i, m_i, dt, sd)  (src/Picasso_PolyPIC.hpp:39-229)
//   PolyPIC::g2p(u_i, c_p, sd)              (src/Picasso_PolyPIC.hpp:235-358)
// with sd = createSpline(Location(), InterpolationOrder<N>(), local_mesh, x_p,
// ...) (src/Picasso_ParticleInterpolation.hpp:88-105).  Here the same calls
// take whole particle members and grid arrays in device memory and run one
// kernel over all particles: the particle loop of GridOperator::apply
// (src/Picasso_GridOperator.hpp:612-642) moves inside the call.
//
// Errors are reported by throwing Picasso::B200::Error (the C ABI returns
// status codes; this header converts them).
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>

#include "picasso_b200.h"

namespace Picasso {

// ---------------------------------------------------------------------------
// locations, orders, spline members
// ---------------------------------------------------------------------------
namespace FieldLocation {
struct Node {
    static constexpr int value = PICASSO_NODE;
};
struct Cell {
    static constexpr int value = PICASSO_CELL;
};
template <int D>
struct Face {
    static_assert(D >= 0 && D < 3, "Face dimension out of bounds");
    static constexpr int value = PICASSO_FACE_I + D;
};
template <int D>
struct Edge {
    static_assert(D >= 0 && D < 3, "Edge dimension out of bounds");
    static constexpr int value = PICASSO_EDGE_I + D;
};
}  // namespace FieldLocation

template <int N>
struct InterpolationOrder {
    static_assert(N >= 1 && N <= 3, "interpolation order 1, 2 or 3");
    static constexpr int value = N;
};

// Spline members are computed inside the kernels; the tags are accepted so
// that call sites read as in Picasso.
struct SplineValue {};
struct SplineGradient {};
struct SplineDistance {};
struct SplineCellSize {};
struct SplineLogicalPosition {};

namespace B200 {

struct Error : std::runtime_error {
    picasso_status status;
    Error(picasso_status s, const std::string& where)
        : std::runtime_error(where + ": " + picasso_status_string(s) +
                             (s == PICASSO_ERR_CUDA ? std::string(" (") +
                                                          picasso_last_cuda_error() + ")"
                                                    : std::string())),
          status(s)
    {
    }
};

inline void check(picasso_status s, const char* where)
{
    if (s != PICASSO_OK) throw Error(s, where);
}

// ---------------------------------------------------------------------------
// device data descriptions
// ---------------------------------------------------------------------------
template <class T>
constexpr int32_t dtype_of();
template <>
constexpr int32_t dtype_of<double>()
{
    return PICASSO_F64;
}
template <>
constexpr int32_t dtype_of<float>()
{
    return PICASSO_F32;
}

// A particle member in device memory: n particles of `components` values.
struct ParticleMember {
    picasso_particle_field field;
    int64_t n;
    int32_t components;  // total values per particle (rows * cols)
    int32_t cols;        // columns of a matrix member (ncomp)

    // Plain array of structures: element (p, c) at data[p * components + c].
    template <class T>
    static ParticleMember aos(T* data, int64_t n, int32_t rows, int32_t cols)
    {
        ParticleMember m;
        m.field = {data, dtype_of<T>(), 0, (int64_t)rows * cols, 1};
        m.n = n;
        m.components = rows * cols;
        m.cols = cols;
        return m;
    }
    // Structure of arrays: element (p, c) at data[c * n + p].
    template <class T>
    static ParticleMember soa(T* data, int64_t n, int32_t rows, int32_t cols)
    {
        ParticleMember m;
        m.field = {data, dtype_of<T>(), 62, 0, n};
        m.n = n;
        m.components = rows * cols;
        m.cols = cols;
        return m;
    }
    // Cabana AoSoA member: `member` points at the member's first element,
    // `vector_length` (power of two) particles per SoA, `soa_elements` values
    // of T per SoA (the AoSoA stride).
    template <class T>
    static ParticleMember aosoa(T* member, int64_t n, int32_t rows, int32_t cols,
                                int32_t vector_length, int64_t soa_elements)
    {
        int32_t shift = 0;
        while ((1 << shift) < vector_length) ++shift;
        if ((1 << shift) != vector_length)
            throw Error(PICASSO_ERR_INVALID_ARGUMENT, "AoSoA vector length must be 2^k");
        ParticleMember m;
        m.field = {member, dtype_of<T>(), shift, soa_elements, vector_length};
        m.n = n;
        m.components = rows * cols;
        m.cols = cols;
        return m;
    }
};

// A grid array (i, j, k, component) in device memory with element strides.
struct GridArray {
    picasso_grid_field field;
    int32_t components;

    // Cabana::Grid layout: (nx, ny, nz, nc) row-major.
    template <class T>
    static GridArray layout_right(T* data, const int32_t ext[3], int32_t nc)
    {
        GridArray g;
        g.field = {data, dtype_of<T>(), 0,
                   {(int64_t)ext[1] * ext[2] * nc, (int64_t)ext[2] * nc, (int64_t)nc, 1}};
        g.components = nc;
        return g;
    }
    // 64-bit fixed-point accumulator (value = raw * 2^-bits).
    static GridArray fixed_layout_right(int64_t* data, const int32_t ext[3], int32_t nc,
                                        int32_t bits)
    {
        GridArray g;
        g.field = {data, PICASSO_I64_FIXED, bits,
                   {(int64_t)ext[1] * ext[2] * nc, (int64_t)ext[2] * nc, (int64_t)nc, 1}};
        g.components = nc;
        return g;
    }
    // One component of a multi-component array viewed as a scalar array.
    GridArray component(int32_t c) const
    {
        GridArray g = *this;
        const int64_t es = field.dtype == PICASSO_F32 ? 4 : 8;
        g.field.data = static_cast<char*>(field.data) + es * c * field.stride[3];
        g.components = 1;
        return g;
    }
};

// Execution context: stream, optional skipped-particle counter, optional
// sorted bins (see picasso_cell_sort).
struct Exec {
    picasso_exec exec{nullptr, nullptr, nullptr};
    explicit Exec(void* stream = nullptr, int32_t* error_count = nullptr,
                  const picasso_bins* bins = nullptr)
    {
        exec.stream = stream;
        exec.error_count = error_count;
        exec.bins = bins;
    }
};

template <class Location, class Order>
struct SplineData {
    picasso_spline spline;
    ParticleMember x;
    int64_t num_particles() const { return x.n; }
};

}  // namespace B200

// createSpline(Location, InterpolationOrder<N>, mesh, x, members...):
// `mesh` describes the local grid of the arrays passed to the transfers.
template <class Location, class Order, class... Members>
B200::SplineData<Location, Order> createSpline(Location, Order, const picasso_mesh& mesh,
                                               const B200::ParticleMember& x, Members...)
{
    B200::SplineData<Location, Order> sd;
    sd.spline.mesh = mesh;
    sd.spline.location = Location::value;
    sd.spline.order = Order::value;
    sd.x = x;
    return sd;
}

namespace APIC {

// APIC::p2g(m_p, c_p, m_i, mu_i, sd): adds into m_i / mu_i.
template <class Location, class Order>
void p2g(const B200::ParticleMember& m_p, const B200::ParticleMember& c_p,
         const B200::GridArray& m_i, const B200::GridArray& mu_i,
         const B200::SplineData<Location, Order>& sd, const B200::Exec& ex = B200::Exec())
{
    B200::check(picasso_apic_p2g(&sd.spline, sd.num_particles(), c_p.cols, sd.x.field,
                                 m_p.field, c_p.field, m_i.field, mu_i.field, &ex.exec),
                "APIC::p2g");
}

// APIC::g2p(u_i, c_p, sd): overwrites c_p.
template <class Location, class Order>
void g2p(const B200::GridArray& u_i, const B200::ParticleMember& c_p,
         const B200::SplineData<Location, Order>& sd, const B200::Exec& ex = B200::Exec())
{
    B200::check(picasso_apic_g2p(&sd.spline, sd.num_particles(), c_p.cols, sd.x.field,
                                 u_i.field, c_p.field, &ex.exec),
                "APIC::g2p");
}

// APIC::g2p followed by the position update x_p += dt * c_p(0, :) in one
// pass (collocated, 3 components; positions of sd.x are updated in place).
template <class Location, class Order>
void g2pAdvect(const B200::GridArray& u_i, const B200::ParticleMember& c_p,
               const B200::SplineData<Location, Order>& sd, double dt,
               const B200::Exec& ex = B200::Exec())
{
    B200::check(picasso_apic_g2p_advect(&sd.spline, sd.num_particles(), sd.x.field, u_i.field,
                                        c_p.field, dt, &ex.exec),
                "APIC::g2pAdvect");
}

// g2pAdvect that also writes key_out[p] (device), the cell-sort key of every
// moved particle for bins of shape `tile`: the input of
// picasso_cell_sort_keys for the next step.
template <class Location, class Order>
void g2pAdvect(const B200::GridArray& u_i, const B200::ParticleMember& c_p,
               const B200::SplineData<Location, Order>& sd, double dt, const int32_t tile[3],
               uint32_t* key_out, const B200::Exec& ex = B200::Exec())
{
    B200::check(picasso_apic_g2p_advect_keys(&sd.spline, sd.num_particles(), sd.x.field,
                                             u_i.field, c_p.field, dt, tile, key_out, &ex.exec),
                "APIC::g2pAdvect");
}

}  // namespace APIC

namespace PolyPIC {

// PolyPIC::p2g(m_p, u_p, c_p, mu_i, m_i, dt, sd) -- field before mass.
template <class Location, class Order>
void p2g(const B200::ParticleMember& m_p, const B200::ParticleMember& u_p,
         const B200::ParticleMember& c_p, const B200::GridArray& mu_i,
         const B200::GridArray& m_i, double dt, const B200::SplineData<Location, Order>& sd,
         const B200::Exec& ex = B200::Exec())
{
    B200::check(picasso_polypic_p2g(&sd.spline, sd.num_particles(), c_p.cols, sd.x.field,
                                    m_p.field, u_p.field, c_p.field, mu_i.field, m_i.field, dt,
                                    &ex.exec),
                "PolyPIC::p2g");
}

template <class Location, class Order>
void g2p(const B200::GridArray& u_i, const B200::ParticleMember& c_p,
         const B200::SplineData<Location, Order>& sd, const B200::Exec& ex = B200::Exec())
{
    B200::check(picasso_polypic_g2p(&sd.spline, sd.num_particles(), c_p.cols, sd.x.field,
                                    u_i.field, c_p.field, &ex.exec),
                "PolyPIC::g2p");
}

}  // namespace PolyPIC

namespace LinearAlgebra {

// Batched 3x3 determinant and inverse of n row-major FP64 matrices.
inline void inverse(int64_t n, const double* a, double* a_inv, double* det,
                    const B200::Exec& ex = B200::Exec())
{
    B200::check(picasso_mat3_inverse(n, a, a_inv, det, nullptr, nullptr, &ex.exec),
                "LinearAlgebra::inverse");
}

}  // namespace LinearAlgebra

namespace B200 {

// Field solve between P2G and G2P (doc/basic/explict_nearly_incompressible_flow.md):
// u_i = (mu_i + dt f_i) / m_i + dt g, then the wall conditions of `params`.
// `f_i.field.data == nullptr` means no force.
inline void gridUpdate(const picasso_mesh& mesh, const GridArray& m_i, const GridArray& mu_i,
                       const GridArray& f_i, const picasso_grid_update_params& params,
                       const GridArray& u_i, const Exec& ex = Exec())
{
    picasso_grid_field none{};
    check(picasso_grid_update(&mesh, m_i.field, mu_i.field, f_i.field, &params, u_i.field, none,
                              &ex.exec),
          "gridUpdate");
}

// Many independent APIC problems stepped together (picasso_batch_*); owns the
// batch handle.
class Batch {
  public:
    Batch(const picasso_batch_instance* instances, int32_t count,
          picasso_batch_mode mode = PICASSO_BATCH_PHASED)
    {
        check(picasso_batch_create(instances, count, mode, &b_), "Batch");
    }
    ~Batch() { picasso_batch_destroy(b_); }
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;
    void step(void* stream = nullptr, bool use_graph = true)
    {
        check(picasso_batch_step(b_, stream, use_graph ? 1 : 0), "Batch::step");
    }
    void stepSequential(void* stream = nullptr)
    {
        check(picasso_batch_step_sequential(b_, stream), "Batch::stepSequential");
    }
    void status(void* stream = nullptr) { check(picasso_batch_status(b_, stream), "Batch::status"); }

  private:
    picasso_batch* b_ = nullptr;
};

}  // namespace B200

}  // namespace Picasso
