// Runs the reference's quadratic APIC known-answer fixture (tstAPIC.hpp:537-682:
// one particle, Cell location, polynomial grid field) through the C++ drop-in
// header and prints u_p, B_p and the p2g mass / momentum on the 27 stencil
// cells, one value per line, for the test to compare with the golden values.
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

int main()
{
    // mesh of the reference test: [-50, 50]^3, cell 0.5, 2 halo cells, no
    // periodicity; Cell entities: 200 + 4 per dimension, node 0 at -51
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
    double *d_grid, *d_mass, *d_x, *d_m, *d_c;
    CUDA_OK(cudaMalloc((void**)&d_grid, ncell * 3 * sizeof(double)));
    CUDA_OK(cudaMalloc((void**)&d_mass, ncell * sizeof(double)));
    CUDA_OK(cudaMalloc((void**)&d_x, 3 * sizeof(double)));
    CUDA_OK(cudaMalloc((void**)&d_m, sizeof(double)));
    CUDA_OK(cudaMalloc((void**)&d_c, 12 * sizeof(double)));
    const double x[3] = {9.31, -8.28, -3.34}, m = 0.134;
    CUDA_OK(cudaMemcpy(d_grid, grid.data(), ncell * 3 * sizeof(double), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_x, x, sizeof(x), cudaMemcpyHostToDevice));
    CUDA_OK(cudaMemcpy(d_m, &m, sizeof(m), cudaMemcpyHostToDevice));

    auto xp = B200::ParticleMember::aos(d_x, 1, 1, 3);
    auto mp = B200::ParticleMember::aos(d_m, 1, 1, 1);
    auto cp = B200::ParticleMember::aos(d_c, 1, 4, 3);
    auto u_i = B200::GridArray::layout_right(d_grid, ext, 3);
    auto m_i = B200::GridArray::layout_right(d_mass, ext, 1);
    auto sd = createSpline(FieldLocation::Cell(), InterpolationOrder<2>(), mesh, xp,
                           SplineValue(), SplineDistance(), SplineCellSize());
    try {
        APIC::g2p(u_i, cp, sd);
        double c[12];
        CUDA_OK(cudaMemcpy(c, d_c, sizeof(c), cudaMemcpyDeviceToHost));
        for (int q = 0; q < 12; ++q) std::printf("c %d %.17g\n", q, c[q]);
        CUDA_OK(cudaMemset(d_grid, 0, ncell * 3 * sizeof(double)));
        CUDA_OK(cudaMemset(d_mass, 0, ncell * sizeof(double)));
        APIC::p2g(mp, cp, m_i, u_i, sd);
    } catch (const B200::Error& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 3;
    }
    CUDA_OK(cudaMemcpy(grid.data(), d_grid, ncell * 3 * sizeof(double), cudaMemcpyDeviceToHost));
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
    return 0;
}
