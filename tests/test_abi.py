"""CPU checks of the boundary: the library loads, exports every entry point
the public header declares, its descriptors have the layout the ctypes
mirror assumes, and invalid arguments are rejected on the host (no device
needed)."""

import ctypes as C
import os
import re
import subprocess

import pytest

from picasso_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "picasso_b200.h")


def _declared():
    names = set()
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            with open(os.path.join(ROOT, "include", h)) as f:
                names |= set(re.findall(r"PICASSO_API\s+[\w\s\*]*?\b(picasso_\w+)\s*\(", f.read()))
    return names


def test_library_exports_every_declared_symbol():
    lib = _abi.load_library()
    declared = _declared()
    assert len(declared) >= 14
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(picasso_\w+)", out))
    assert declared <= exported, declared - exported
    for name in declared:
        assert hasattr(lib, name)
    assert {s[0] for s in _abi.SIGNATURES} == declared
    assert lib.picasso_version().startswith(b"picasso_b200")


def test_descriptor_layout_matches_ctypes(tmp_path):
    structs = {
        "picasso_mesh": (_abi.Mesh, ["extent", "own_begin", "own_extent", "periodic",
                                     "low_corner", "cell_size"]),
        "picasso_spline": (_abi.Spline, ["mesh", "location", "order"]),
        "picasso_particle_field": (_abi.ParticleField, ["data", "dtype", "vector_shift",
                                                        "tile_stride", "comp_stride"]),
        "picasso_grid_field": (_abi.GridField, ["data", "dtype", "fixed_bits", "stride"]),
        "picasso_bins": (_abi.Bins, ["tile", "num_tiles", "bin_extent", "order", "location",
                                     "chunk", "p2g_lanes", "tile_offset", "tile_items"]),
        "picasso_exec": (_abi.Exec, ["stream", "error_count", "bins"]),
        "picasso_batch_instance": (_abi.BatchInstance, ["spline", "num_particles", "x_p", "m_p",
                                                        "c_p", "m_i", "mu_i", "u_i",
                                                        "mass_threshold", "bins",
                                                        "error_count"]),
        "picasso_batch_info": (_abi.BatchInfo, ["count", "precision_form", "grid_blocks",
                                                "smem_bytes", "items", "particles"]),
        "picasso_tune_result": (_abi.TuneResult, ["tile", "chunk", "p2g_lanes", "step_ms"]),
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "picasso_b200.h"',
             "int main(void) {"]
    for s, (_, fields) in structs.items():
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (s, s))
        for fld in fields:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (s, fld, s, fld))
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = dict(l.split() for l in subprocess.run([str(exe)], capture_output=True, text=True,
                                                 check=True).stdout.splitlines())
    for s, (cls, fields) in structs.items():
        assert int(got[s]) == C.sizeof(cls), s
        for fld in fields:
            assert int(got["%s.%s" % (s, fld)]) == getattr(cls, fld).offset, (s, fld)


def _spline(order=2, location=0, n=8):
    sp = _abi.Spline()
    for d in range(3):
        sp.mesh.extent[d] = n
        sp.mesh.own_begin[d] = 0
        sp.mesh.own_extent[d] = n
        sp.mesh.periodic[d] = 1
        sp.mesh.cell_size[d] = 1.0 / n
    sp.order = order
    sp.location = location
    return sp


def _pf(dtype=_abi.F64, data=16):
    f = _abi.ParticleField()
    f.data = data
    f.dtype = dtype
    f.vector_shift = 0
    f.tile_stride = 3
    f.comp_stride = 1
    return f


def _gf(dtype=_abi.F64, data=16):
    g = _abi.GridField()
    g.data = data
    g.dtype = dtype
    return g


@pytest.mark.parametrize("case", ["order", "location", "ncomp", "null", "dtype_mix", "mesh",
                                  "negative_n", "stag_ncomp", "fixed_bits"])
def test_invalid_arguments_rejected_on_host(case):
    lib = _abi.load_library()
    sp = _spline()
    n, ncomp = 10, 3
    x, m, c = _pf(), _pf(), _pf()
    gm, gmu = _gf(), _gf()
    if case == "order":
        sp.order = 4
    elif case == "location":
        sp.location = 9
    elif case == "ncomp":
        ncomp = 4
    elif case == "null":
        x.data = None
    elif case == "dtype_mix":
        m = _pf(_abi.F32)
    elif case == "mesh":
        sp.mesh.cell_size[1] = 0.0
    elif case == "negative_n":
        n = -1
    elif case == "stag_ncomp":
        sp.location = _abi.FACE_J
        ncomp = 1
    elif case == "fixed_bits":
        m, c = _pf(_abi.F32), _pf(_abi.F32)
        gm, gmu = _gf(_abi.I64_FIXED), _gf(_abi.I64_FIXED)
        gm.fixed_bits = 70
    st = lib.picasso_apic_p2g(C.byref(sp), n, ncomp, x, m, c, gm, gmu, None)
    assert st == _abi.ERR_INVALID_ARGUMENT


def test_unsupported_combinations():
    lib = _abi.load_library()
    sp = _spline(order=3)
    # PolyPIC has no cubic form
    st = lib.picasso_polypic_p2g(C.byref(sp), 1, 3, _pf(), _pf(), _pf(), _pf(), _gf(), _gf(),
                                 1e-3, None)
    assert st == _abi.ERR_UNSUPPORTED
    # quadratic staggered PolyPIC is not defined
    sp = _spline(order=2, location=_abi.EDGE_I)
    st = lib.picasso_polypic_g2p(C.byref(sp), 1, 3, _pf(), _gf(), _pf(), None)
    assert st == _abi.ERR_UNSUPPORTED


def test_zero_particles_is_a_no_op():
    lib = _abi.load_library()
    sp = _spline()
    assert lib.picasso_apic_p2g(C.byref(sp), 0, 3, _pf(), _pf(), _pf(), _gf(), _gf(), None) == 0
    assert lib.picasso_apic_g2p(C.byref(sp), 0, 3, _pf(), _gf(), _pf(), None) == 0


def test_sort_workspace_and_key_range():
    lib = _abi.load_library()
    sp = _spline(n=256)
    nbytes = C.c_int64()
    tile = (C.c_int32 * 3)(8, 8, 8)
    assert lib.picasso_cell_sort_workspace(C.byref(sp), 1 << 20, tile, C.byref(nbytes)) == 0
    assert nbytes.value >= 8 * (1 << 20)
    big = _spline(n=2048)  # 2048^3 bins do not fit 32-bit keys
    assert lib.picasso_cell_sort_workspace(C.byref(big), 10, tile, C.byref(nbytes)) == \
        _abi.ERR_OUT_OF_RANGE


def test_sort_keys_and_key_emission_reject_on_host():
    lib = _abi.load_library()
    sp = _spline(n=16)
    tile = (C.c_int32 * 3)(4, 4, 4)
    nbytes = C.c_int64()
    assert lib.picasso_cell_sort_workspace(C.byref(sp), 100, tile, C.byref(nbytes)) == 0
    ws, nb = 1 << 12, nbytes.value

    def sort_keys(key_in, key, n=100):
        return lib.picasso_cell_sort_keys(C.byref(sp), n, key_in, tile, 256, key, 1 << 20,
                                          1 << 21, 1 << 22, ws, nb, None, None)
    assert sort_keys(1 << 16, 1 << 16) == _abi.ERR_INVALID_ARGUMENT  # key_in is the output
    assert sort_keys(None, 1 << 16) == _abi.ERR_INVALID_ARGUMENT
    assert lib.picasso_cell_sort_keys(C.byref(sp), 100, 1 << 16, tile, 256, 1 << 17, 1 << 20,
                                      1 << 21, 1 << 22, ws, nb - 1, None, None) == \
        _abi.ERR_INVALID_ARGUMENT  # workspace too small
    x, c, u = _pf(), _pf(), _gf()
    c.tile_stride = 12
    bad = (C.c_int32 * 3)(0, 4, 4)
    assert lib.picasso_apic_g2p_advect_keys(C.byref(sp), 10, x, u, c, 0.1, None, 1 << 16,
                                            None) == _abi.ERR_INVALID_ARGUMENT
    assert lib.picasso_apic_g2p_advect_keys(C.byref(sp), 10, x, u, c, 0.1, bad, 1 << 16,
                                            None) == _abi.ERR_INVALID_ARGUMENT
    assert lib.picasso_apic_g2p_advect_keys(C.byref(sp), 10, x, u, c, 0.1, tile, None,
                                            None) == _abi.ERR_INVALID_ARGUMENT
    assert lib.picasso_apic_g2p_advect_keys(C.byref(sp), 0, x, u, c, 0.1, tile, None, None) == 0


def test_autotune_rejects_on_host():
    lib = _abi.load_library()
    sp = _spline(n=16)
    x, m, c = _pf(), _pf(_abi.F32), _pf(_abi.F32)
    m.tile_stride, c.tile_stride = 1, 12
    gm, gmu, gu = _gf(_abi.I64_FIXED), _gf(_abi.I64_FIXED), _gf(_abi.F32)
    gm.fixed_bits = gmu.fixed_bits = 36
    res = _abi.TuneResult()

    def tune(n=100, trials=3, out=True, mm=m, spl=sp):
        return lib.picasso_autotune(C.byref(spl), n, x, mm, c, gm, gmu, gu, 1e-12, trials,
                                    C.byref(res) if out else None, None)
    assert tune(out=False) == _abi.ERR_INVALID_ARGUMENT
    assert tune(n=0) == _abi.ERR_INVALID_ARGUMENT
    assert tune(trials=0) == _abi.ERR_INVALID_ARGUMENT
    assert tune(mm=_pf(_abi.F64)) == _abi.ERR_INVALID_ARGUMENT  # the FP32 form only
    assert tune(spl=_spline(location=_abi.FACE_I, n=16)) == _abi.ERR_UNSUPPORTED


def _batch_instance(f32=True):
    inst = _abi.BatchInstance()
    inst.spline = _spline()
    inst.num_particles = 10
    pt = _abi.F32 if f32 else _abi.F64
    gt = _abi.I64_FIXED if f32 else _abi.F64
    inst.x_p = _pf()
    inst.m_p = _pf(pt)
    inst.m_p.tile_stride = 1
    inst.c_p = _pf(pt)
    inst.c_p.tile_stride = 12
    inst.m_i, inst.mu_i, inst.u_i = _gf(gt), _gf(gt), _gf(pt)
    b = inst.bins
    for d in range(3):
        b.tile[d], b.num_tiles[d], b.bin_extent[d] = 4, 2, 8
    b.order, b.location, b.chunk = 2, 0, 256
    b.tile_offset, b.tile_items = 16, 16
    return inst


@pytest.mark.parametrize("case", ["count", "null_out", "location", "mixed_forms", "lanes",
                                  "bins_order", "layout", "mode"])
def test_batch_create_rejects_invalid_instances_on_host(case):
    lib = _abi.load_library()
    insts = (_abi.BatchInstance * 2)(_batch_instance(), _batch_instance())
    count, mode = 2, _abi.BATCH_FUSED
    out = C.c_void_p()
    out_ptr = C.byref(out)
    if case == "count":
        count = 0
    elif case == "null_out":
        out_ptr = None
    elif case == "location":
        insts[1].spline.location = _abi.CELL
        insts[1].bins.location = _abi.CELL
    elif case == "mixed_forms":
        insts[1] = _batch_instance(f32=False)
    elif case == "lanes":
        insts[0].spline.order = insts[0].bins.order = 3
        insts[0].bins.p2g_lanes = 1
    elif case == "bins_order":
        insts[0].bins.order = 1
    elif case == "layout":
        insts[1].c_p.tile_stride = 3
    elif case == "mode":
        mode = 7
    st = lib.picasso_batch_create(insts, count, mode, out_ptr)
    assert st == _abi.ERR_INVALID_ARGUMENT
    assert not out.value


def test_package_names():
    """The tuner module and the native tuner's wrapper are both reachable
    (the wrapper must not shadow the module)."""
    import picasso_b200 as pb
    from picasso_b200 import autotune
    assert hasattr(autotune, "Tuner")
    assert callable(pb.tune_tiled_step)
