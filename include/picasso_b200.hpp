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
#include <map>
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
// the particle loop of GridOperator::apply
struct Particle {};
}  // namespace FieldLocation

// Field value types: a field tag derives from one of these and gives a
// static label() (the tags of the reference's tests, tstAPIC.hpp:35-48).
namespace Field {
template <class T>
struct Scalar {
    using value_type = T;
    static constexpr int rows = 1, cols = 1, size = 1;
};
template <class T, int N>
struct Vector {
    using value_type = T;
    static constexpr int rows = 1, cols = N, size = N;
};
template <class T, int R, int C>
struct Matrix {
    using value_type = T;
    static constexpr int rows = R, cols = C, size = R * C;
};
}  // namespace Field

// A field at a mesh location (FieldLayout<Location, Tag>).
template <class Location, class Tag>
struct FieldLayout {
    using location = Location;
    using tag = Tag;
};

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
// sorted bins (see picasso_cell_sort), optional fixed-point overflow counter.
struct Exec {
    picasso_exec exec{nullptr, nullptr, nullptr, nullptr};
    explicit Exec(void* stream = nullptr, int32_t* error_count = nullptr,
                  const picasso_bins* bins = nullptr, int32_t* overflow_count = nullptr)
    {
        exec.stream = stream;
        exec.error_count = error_count;
        exec.bins = bins;
        exec.overflow_count = overflow_count;
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

// Launch knobs of the precision-form tiled step measured on the particles of
// sd (picasso_autotune): tile and chunk for picasso_cell_sort, p2g_lanes for
// the bins.  A set-up call: it allocates device memory and waits for the
// stream; m_i / mu_i / u_i serve as the step's grids.
template <class Location, class Order>
picasso_tune_result autotune(const SplineData<Location, Order>& sd, const ParticleMember& m_p,
                             const ParticleMember& c_p, const GridArray& m_i,
                             const GridArray& mu_i, const GridArray& u_i,
                             double mass_threshold = 1e-12, int32_t trials = 3,
                             const Exec& ex = Exec())
{
    picasso_tune_result r{};
    check(picasso_autotune(&sd.spline, sd.num_particles(), sd.x.field, m_p.field, c_p.field,
                           m_i.field, mu_i.field, u_i.field, mass_threshold, trials, &r,
                           &ex.exec),
          "autotune");
    return r;
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

// ---------------------------------------------------------------------------
// GridOperator-style bulk calls (src/Picasso_GridOperator.hpp:380-642,
// src/Picasso_FieldManager.hpp:66-140)
// ---------------------------------------------------------------------------
// In Picasso an application registers grid fields in a FieldManager, keeps
// particles in a Cabana ParticleList and calls
//   op.apply("p2g", FieldLocation::Particle(), exec, fm, pl, functor)
// with a device functor that calls APIC::p2g per particle.  Here the functor
// is one of the transfer descriptors below (it names the fields the transfer
// reads and writes), and apply() runs the transfer as one call over the
// particle list.  As in GridOperator::applyImpl, the scatter fields of a
// particle transfer start from zero.  Halo exchange between ranks is the
// caller's (picasso_b200.dist in Python); periodic meshes wrap on one rank.

// Grid fields in device memory, keyed by (location, tag label); the arrays
// are borrowed.  Each location carries the picasso_mesh its arrays index
// (extent with ghosts, owned range, low corner, cell size).
class FieldManager {
  public:
    template <class Location>
    void setMesh(Location, const picasso_mesh& mesh)
    {
        const int loc = Location::value;  // (no odr-use of the constant in C++14)
        meshes_[loc] = mesh;
    }
    template <class Location>
    const picasso_mesh& mesh(Location) const
    {
        const int loc = Location::value;
        auto it = meshes_.find(loc);
        if (it == meshes_.end())
            throw Error(PICASSO_ERR_INVALID_ARGUMENT, "FieldManager: no mesh for location");
        return it->second;
    }
    template <class Location, class Tag>
    void add(Location, Tag, const GridArray& array)
    {
        if (array.components != Tag::size)
            throw Error(PICASSO_ERR_INVALID_ARGUMENT,
                        "FieldManager::add: " + Tag::label() + " component count");
        fields_[key(Location::value, Tag::label())] = array;
    }
    template <class Layout>
    void add(Layout, const GridArray& array)
    {
        add(typename Layout::location(), typename Layout::tag(), array);
    }
    template <class Location, class Tag>
    const GridArray& array(Location, Tag) const
    {
        auto it = fields_.find(key(Location::value, Tag::label()));
        if (it == fields_.end())
            throw Error(PICASSO_ERR_INVALID_ARGUMENT, "FieldManager: no field " + Tag::label());
        return it->second;
    }
    template <class Layout>
    const GridArray& array(Layout) const
    {
        return array(typename Layout::location(), typename Layout::tag());
    }

  private:
    static std::string key(int location, const std::string& label)
    {
        return std::to_string(location) + "/" + label;
    }
    std::map<int, picasso_mesh> meshes_;
    std::map<std::string, GridArray> fields_;
};

// Particle members in device memory, keyed by tag label (borrowed), and the
// optional sorted bins of the current particle order (picasso_cell_sort
// followed by picasso_permute of every member).
class ParticleList {
  public:
    explicit ParticleList(int64_t n) : n_(n) {}
    int64_t size() const { return n_; }
    template <class Tag>
    void add(Tag, const ParticleMember& member)
    {
        if (member.n != n_ || member.components != Tag::size)
            throw Error(PICASSO_ERR_INVALID_ARGUMENT, "ParticleList::add: " + Tag::label());
        members_[Tag::label()] = member;
    }
    template <class Tag>
    const ParticleMember& get(Tag) const
    {
        auto it = members_.find(Tag::label());
        if (it == members_.end())
            throw Error(PICASSO_ERR_INVALID_ARGUMENT, "ParticleList: no member " + Tag::label());
        return it->second;
    }
    void setBins(const picasso_bins* bins) { bins_ = bins; }
    const picasso_bins* bins() const { return bins_; }

  private:
    int64_t n_;
    std::map<std::string, ParticleMember> members_;
    const picasso_bins* bins_ = nullptr;
};

// Transfer descriptors for GridOperator::apply over FieldLocation::Particle.
// Particle tags: Position (3 x FP64), Mass, Affine (4 x 3 APIC c_p) or
// Velocity / Modes (PolyPIC u_p, c_p); grid tags at `Location`.
template <class Location, class Order, class Position, class Mass, class Affine, class GridMass,
          class GridMomentum>
struct APICP2G {};
template <class Location, class Order, class Position, class Affine, class GridVelocity>
struct APICG2P {};
// G2P followed by x_p += dt u_p (collocated, 3 components)
template <class Location, class Order, class Position, class Affine, class GridVelocity>
struct APICG2PAdvect {
    double dt;
};
template <class Location, class Order, class Position, class Mass, class Velocity, class Modes,
          class GridMomentum, class GridMass>
struct PolyPICP2G {
    double dt;
};
template <class Location, class Order, class Position, class Modes, class GridVelocity>
struct PolyPICG2P {};

// Grid descriptors for GridOperator::apply over a mesh location.
template <class GridMass, class GridMomentum, class GridVelocity>
struct VelocityUpdate {  // u = mu / m where m > mass_threshold, else 0
    double mass_threshold;
};
template <class GridMass, class GridMomentum, class GridVelocity>
struct MomentumUpdate {  // picasso_grid_update without a force field
    picasso_grid_update_params params;
};

template <class FieldDependencies = void>
class GridOperator {
  public:
    // Fields are registered by the application (they are borrowed), so there
    // is nothing to add; kept for the call sequence of Picasso.
    void setup(FieldManager&) {}

    template <class Op>
    void apply(const std::string& label, FieldLocation::Particle, const Exec& exec,
               const FieldManager& fm, const ParticleList& pl, const Op& op) const
    {
        Exec ex = exec;
        if (!ex.exec.bins) ex.exec.bins = pl.bins();
        run(label, ex, fm, pl, op);
    }

    template <class Location, class Op>
    void apply(const std::string& label, Location loc, const Exec& exec, const FieldManager& fm,
               const Op& op) const
    {
        run_grid(label, loc, exec, fm, op);
    }

  private:
    template <class L, class O, class P, class M, class A, class GM, class GU>
    static void run(const std::string&, const Exec& ex, const FieldManager& fm,
                    const ParticleList& pl, const APICP2G<L, O, P, M, A, GM, GU>&)
    {
        const picasso_mesh& mesh = fm.mesh(L());
        const GridArray& m_i = fm.array(L(), GM());
        const GridArray& mu_i = fm.array(L(), GU());
        zero(mesh, m_i, ex);
        zero(mesh, mu_i, ex);
        auto sd = createSpline(L(), O(), mesh, pl.get(P()));
        APIC::p2g(pl.get(M()), pl.get(A()), m_i, mu_i, sd, ex);
    }
    template <class L, class O, class P, class A, class GV>
    static void run(const std::string&, const Exec& ex, const FieldManager& fm,
                    const ParticleList& pl, const APICG2P<L, O, P, A, GV>&)
    {
        auto sd = createSpline(L(), O(), fm.mesh(L()), pl.get(P()));
        APIC::g2p(fm.array(L(), GV()), pl.get(A()), sd, ex);
    }
    template <class L, class O, class P, class A, class GV>
    static void run(const std::string&, const Exec& ex, const FieldManager& fm,
                    const ParticleList& pl, const APICG2PAdvect<L, O, P, A, GV>& op)
    {
        auto sd = createSpline(L(), O(), fm.mesh(L()), pl.get(P()));
        APIC::g2pAdvect(fm.array(L(), GV()), pl.get(A()), sd, op.dt, ex);
    }
    template <class L, class O, class P, class M, class V, class C, class GU, class GM>
    static void run(const std::string&, const Exec& ex, const FieldManager& fm,
                    const ParticleList& pl, const PolyPICP2G<L, O, P, M, V, C, GU, GM>& op)
    {
        const picasso_mesh& mesh = fm.mesh(L());
        const GridArray& mu_i = fm.array(L(), GU());
        const GridArray& m_i = fm.array(L(), GM());
        zero(mesh, mu_i, ex);
        zero(mesh, m_i, ex);
        auto sd = createSpline(L(), O(), mesh, pl.get(P()));
        PolyPIC::p2g(pl.get(M()), pl.get(V()), pl.get(C()), mu_i, m_i, op.dt, sd, ex);
    }
    template <class L, class O, class P, class C, class GV>
    static void run(const std::string&, const Exec& ex, const FieldManager& fm,
                    const ParticleList& pl, const PolyPICG2P<L, O, P, C, GV>&)
    {
        auto sd = createSpline(L(), O(), fm.mesh(L()), pl.get(P()));
        PolyPIC::g2p(fm.array(L(), GV()), pl.get(C()), sd, ex);
    }

    template <class L, class GM, class GU, class GV>
    static void run_grid(const std::string&, L, const Exec& ex, const FieldManager& fm,
                         const VelocityUpdate<GM, GU, GV>& op)
    {
        const GridArray& mu_i = fm.array(L(), GU());
        picasso_grid_field none{};
        check(picasso_grid_velocity(&fm.mesh(L()), mu_i.components, fm.array(L(), GM()).field,
                                    mu_i.field, op.mass_threshold, fm.array(L(), GV()).field,
                                    none, &ex.exec),
              "GridOperator::apply(VelocityUpdate)");
    }
    template <class L, class GM, class GU, class GV>
    static void run_grid(const std::string&, L, const Exec& ex, const FieldManager& fm,
                         const MomentumUpdate<GM, GU, GV>& op)
    {
        gridUpdate(fm.mesh(L()), fm.array(L(), GM()), fm.array(L(), GU()), GridArray{},
                   op.params, fm.array(L(), GV()), ex);
    }

    // scatter fields start from zero (GridOperator.hpp:532-533)
    static void zero(const picasso_mesh& mesh, const GridArray& a, const Exec& ex)
    {
        check(picasso_grid_fill(&mesh, a.components, a.field, 0.0, &ex.exec),
              "GridOperator::apply (zero scatter field)");
    }
};

}  // namespace B200

}  // namespace Picasso
