"""The C++ drop-in header (include/picasso_b200.hpp): it compiles on its own
(CPU), and a program written against it reproduces the reference's quadratic
APIC known answers on the GPU."""

import os
import subprocess

import numpy as np
import pytest

from helpers import golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
CUDA = "/usr/local/cuda"
SRC = os.path.join(ROOT, "tests", "cpp", "shim_golden.cpp")
CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def test_header_compiles_standalone(tmp_path):
    src = tmp_path / "inc.cpp"
    src.write_text('#include "picasso_b200.hpp"\nint main() { return 0; }\n')
    subprocess.run([CXX, "-std=c++14", "-Wall", "-Wextra", "-Werror", "-I", INC, str(src),
                    "-o", str(tmp_path / "inc")], check=True)


def test_header_wrappers_instantiate(tmp_path):
    """Every wrapper template of the header instantiates and links against
    the library's exported symbols (nothing is run)."""
    src = tmp_path / "inst.cpp"
    src.write_text(r'''
#include "picasso_b200.hpp"
using namespace Picasso;
int main(int argc, char**) {
    if (argc > 100) {  // never taken: only instantiation and linking are tested
        picasso_mesh mesh{};
        double* xd = nullptr; float* mf = nullptr; float* cf = nullptr;
        int32_t ext[3] = {8, 8, 8};
        auto x = B200::ParticleMember::aos(xd, 1, 1, 3);
        auto m = B200::ParticleMember::aos(mf, 1, 1, 1);
        auto c = B200::ParticleMember::aos(cf, 1, 4, 3);
        auto u = B200::GridArray::layout_right(cf, ext, 3);
        auto sd = createSpline(FieldLocation::Node(), InterpolationOrder<2>(), mesh, x);
        APIC::p2g(m, c, u, u, sd);
        APIC::g2p(u, c, sd);
        APIC::g2pAdvect(u, c, sd, 0.1);
        const int32_t tile[3] = {4, 8, 8};
        uint32_t* keys = nullptr;
        APIC::g2pAdvect(u, c, sd, 0.1, tile, keys);
        PolyPIC::g2p(u, c, sd);
        picasso_grid_update_params prm{};
        B200::gridUpdate(mesh, u, u, u, prm, u);
        B200::Batch batch(nullptr, 0);
        batch.step();
    }
    return 0;
}
''')
    lib = os.path.join(ROOT, "picasso_b200")
    subprocess.run([CXX, "-std=c++14", "-Wall", "-Wextra", "-Werror", "-Wno-unused-parameter",
                    "-I", INC, str(src), "-L", lib, "-lpicasso_b200", "-Wl,-rpath," + lib, "-o",
                    str(tmp_path / "inst")], check=True)


@pytest.mark.gpu
def test_shim_reproduces_golden(cuda, tmp_path):
    exe = str(tmp_path / "shim_golden")
    lib = os.path.join(ROOT, "picasso_b200")
    subprocess.run([CXX, "-std=c++17", "-O2", "-I", INC, "-I", CUDA + "/include", SRC, "-o", exe,
                    "-L", lib, "-lpicasso_b200", "-L", CUDA + "/lib64", "-lcudart",
                    "-Wl,-rpath," + lib + ":" + CUDA + "/lib64"], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    c = np.array([float(l.split()[2]) for l in out if l.startswith("c ")])
    nodes = np.array([[float(v) for v in l.split()[2:]] for l in out if l.startswith("node ")])
    ck = golden()["apic"]["checks"]["2"]
    np.testing.assert_allclose(c[0:3], ck["checkParticleVelocity"]["mathematica_u"], rtol=0,
                               atol=1e-11)
    b = c[3:].reshape(3, 3).T  # c_p(1 + a, d) -> B_p(d, a)
    np.testing.assert_allclose(b, ck["checkParticleVelocity"]["mathematica_b"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(nodes[:, 0], ck["checkGridMass"]["mathematica"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(nodes[:, 1:], ck["checkGridMomentum"]["mathematica"], rtol=0,
                               atol=1e-11)
