// The reference's quadratic APIC known-answer fixture (tstAPIC.hpp:537-682:
// one particle, Cell location, polynomial grid field), written the way a
// Picasso application drives transfers: fields registered in a FieldManager,
// particle members in a ParticleList, and GridOperator::apply over
// FieldLocation::Particle with the G2P and P2G transfer descriptors.  Prints
// u_p, B_p and the p2g mass / momentum on the 27 stencil cells in the format
// of shim_golden.cpp.
#include <cuda_runtime_api.h>

#include <cmath>
#include <cstdio>
#include <vector>

#include "picasso_b200.hpp"

using namespace Picasso;

#define CUDA_OK(x)                                                                 \
    do {                                                                           \
        cudaError_t e = (x);                                                       \
        if (e != cudaSuccess) {                                                    \
            std::fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e));           \
            return 2;                                                              \
        }                                                                          \
    } while (0)

// field tags as an application defines them
struct ParticlePosition : Field::Vector<double, 3> {
    static std::string label() { return "particle_position"; }
};
struct ParticleMass : Field::Scalar<double> {
    static std::string label() { return "particle_mass"; }
};
struct ParticleVelocity : Field::Matrix<double, 4, 3> {
    static std::string label() { return "particle_velocity"; }
};
struct GridVelocity : Field::Vector<double, 3> {
    static std::string label() { return "grid_velocity"; }
};
struct GridMass : Field::Scalar<double> {
    static std::string label() { return "grid_mass"; }
};
struct GridMomentum : Field::Vector<double, 3> {
    static std::string label() { return "grid_momentum"; }
};

int main()
{
    const int ext[3] = {204, 204, 204};
    picasso_mesh mesh{};
    for (int d = 0; d < 3; ++d) {
        mesh.extent[d] = ext[d];
        mesh.own_begin[d] = 2;
        mesh.own_extent[d] = 200;
        mesh.periodic[d] = 0;
        mesh.low_corner[d] = -51.0;
        mesh.cell_size[d] = 0.5;
    }
    const int cx = 120, cy = 85, cz = 95;
    const size_t ncell = (size_t)ext[0] * ext[1] * ext[2];
    std::vector<double> grid(ncell * 3, 0.0);
    for (int i = cx - 4; i < cx + 5; ++i)
        for (int j = cy - 4; j < cy + 5; ++j)
            for (int k = cz - 4; k < cz + 5; ++k)
                for (int d = 0; d < 3; ++d) {
                    const double ic = i - 2, jc = j - 2, kc = k - 2;
                    grid[((size_t)(i * ext[1] + j) * ext[2] + k) * 3 + d] =
                        0.0000000001 * (d + 1) * std::pow(ic, 5) -
                        0.0000000012 * std::pow((d + 1) + jc * ic, 3) +
                        0.0000000001 * std::pow(ic * jc * kc, 2) + std::pow((d + 1), 2);
                }
    double *d_u, *d_mom, *d_mass, *d_x, *d_m, *d_c;
    CUDA_OK(cudaMalloc((void**)&d_u, ncell * 3 * sizeof(double)));
    CUDA_OK(cudaMalloc((void**)&d_mom, ncell * 3 * sizeof(double)));
    CUDA_OK(cudaMalloc((void**)&d_mass, ncell * sizeof(double)));
    CUDA_OK(cudaMalloc((void**)&d_x, 3 * sizeof(double)));
    CUDA_OK(cudaMalloc((void**)&d_m, sizeof(double)));
    CUDA_OK(cudaMalloc((void**)&d_c, 12 * sizeof(double)));
    // the scatter fields hold garbage: apply() must zero them first
    CUDA_OK(cudaMemset(d_mom, 0x7f, ncell * 3 * sizeof(double)));
    CUDA_OK(cudaMemset(d_mass, 0x7f, ncell * sizeof(double)));
    const double x[3] = {9.31, -8.28, -3.34}, m = 0.134;
    CUDA_OK(cudaMemcpy(d_u, grid.data(), ncell * 3 * sizeof(double), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_x, x, sizeof(x), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_m, &m, sizeof(m), cudaMemcpyHostToDevice));

    try {
        B200::FieldManager fm;
        fm.setMesh(FieldLocation::Cell(), mesh);
        fm.add(FieldLocation::Cell(), GridVelocity(), B200::GridArray::layout_right(d_u, ext, 3));
        fm.add(FieldLayout<FieldLocation::Cell, GridMass>(),
               B200::GridArray::layout_right(d_mass, ext, 1));
        fm.add(FieldLocation::Cell(), GridMomentum(),
               B200::GridArray::layout_right(d_mom, ext, 3));
        B200::ParticleList pl(1);
        pl.add(ParticlePosition(), B200::ParticleMember::aos(d_x, 1, 1, 3));
        pl.add(ParticleMass(), B200::ParticleMember::aos(d_m, 1, 1, 1));
        pl.add(ParticleVelocity(), B200::ParticleMember::aos(d_c, 1, 4, 3));
        using Cell = FieldLocation::Cell;
        using Q = InterpolationOrder<2>;
        B200::GridOperator<> op;
        op.setup(fm);
        op.apply("g2p", FieldLocation::Particle(), B200::Exec(), fm, pl,
                 B200::APICG2P<Cell, Q, ParticlePosition, ParticleVelocity, GridVelocity>());
        double c[12];
        CUDA_OK(cudaMemcpy(c, d_c, sizeof(c), cudaMemcpyDeviceToHost));
        for (int q = 0; q < 12; ++q) std::printf("c %d %.17g\n", q, c[q]);
        op.apply("p2g", FieldLocation::Particle(), B200::Exec(), fm, pl,
                 B200::APICP2G<Cell, Q, ParticlePosition, ParticleMass, ParticleVelocity,
                               GridMass, GridMomentum>());
    } catch (const B200::Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 3;
    }
    CUDA_OK(cudaMemcpy(grid.data(), d_mom, ncell * 3 * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<double> mass(ncell);
    CUDA_OK(cudaMemcpy(mass.data(), d_mass, ncell * sizeof(double), cudaMemcpyDeviceToHost));
    int n = 0;
    for (int i = cx - 1; i < cx + 2; ++i)
        for (int j = cy - 1; j < cy + 2; ++j)
            for (int k = cz - 1; k < cz + 2; ++k, ++n) {
                const size_t e = (size_t)(i * ext[1] + j) * ext[2] + k;
                std::printf("node %d %.17g %.17g %.17g %.17g\n", n, mass[e], grid[e * 3],
                            grid[e * 3 + 1], grid[e * 3 + 2]);
            }
    // nothing outside the stencil: the zeroing covered the whole array
    double outside = 0.0;
    for (size_t e = 0; e < ncell; ++e) {
        const int i = (int)(e / ((size_t)ext[1] * ext[2])), j = (int)(e / ext[2] % ext[1]);
        const int k = (int)(e % ext[2]);
        if (std::abs(i - cx) <= 1 && std::abs(j - cy) <= 1 && std::abs(k - cz) <= 1) continue;
        outside = std::fmax(outside, std::fabs(mass[e]));
        for (int d = 0; d < 3; ++d) outside = std::fmax(outside, std::fabs(grid[e * 3 + d]));
    }
    std::printf("outside %.17g\n", outside);
    return 0;
}
