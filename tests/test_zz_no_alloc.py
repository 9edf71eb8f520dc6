"""The cell sort that allocates nothing (picasso_cell_sort_static).

It exists for callers that cannot allocate device memory at the moment they
sort -- applications that give all GPU memory to their own pool at start-up,
plugins running inside such applications, loops that must not meet the
allocator's latency or out-of-memory path.  Its scratch is a fixed 32 MiB
array inside the library, shared by every call.

The test calls it twice in a row through the C ABI, on two different
particle sets, and checks every output against the workspace version
(integer outputs: bit-identical), then checks that a sort too large for the
array is refused before anything runs.  This file is named to be collected
last so that a stop at the first failure has run every other test first.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from particles import clustered_particles, periodic_mesh, uniform_particles
from picasso_b200 import FieldLocation, _abi, cell_sort, create_spline
from picasso_b200.api import particle_field

pytestmark = pytest.mark.gpu


def _static_sort(sd, tile, chunk):
    lib = _abi.load_library()
    n = sd.num_particles
    dev = sd.x.device
    key = torch.empty(n, dtype=torch.int32, device=dev)
    perm = torch.empty(n, dtype=torch.int32, device=dev)
    nt = 1
    m = sd.desc.mesh
    for d in range(3):
        nb = m.own_extent[d] if m.periodic[d] else m.extent[d]
        nt *= -(-nb // tile[d])
    off = torch.empty(nt + 1, dtype=torch.int64, device=dev)
    items = torch.empty(nt + 1, dtype=torch.int32, device=dev)
    bins = _abi.Bins()
    ex = _abi.Exec()
    ex.stream = torch.cuda.current_stream().cuda_stream
    st = lib.picasso_cell_sort_static(C.byref(sd.desc), n, particle_field(sd.x),
                                      (C.c_int32 * 3)(*tile), chunk, key.data_ptr(),
                                      perm.data_ptr(), off.data_ptr(), items.data_ptr(),
                                      C.byref(bins), C.byref(ex))
    return st, key, perm, off, items, bins


def test_static_sort_matches_workspace_sort_twice(cuda):
    tile, chunk = (4, 8, 8), 512
    sets = []
    mesh = periodic_mesh(32, halo=1)
    x1, _, _ = clustered_particles(mesh, 32 ** 3 * 8, nblob=4, sigma_cells=2.0, frac=0.7, seed=71)
    x2, _, _ = uniform_particles(mesh, 6, seed=72)
    sets = [x1, x2]
    for x in sets:  # two calls in a row share the static scratch
        sd = create_spline(FieldLocation.Node, 2, mesh,
                           torch.as_tensor(np.ascontiguousarray(x), device="cuda"))
        st, key, perm, off, items, bins = _static_sort(sd, tile, chunk)
        assert st == _abi.OK
        key_w, perm_w, bins_w = cell_sort(sd, tile, chunk=chunk)
        torch.cuda.synchronize()
        assert torch.equal(key, key_w)
        assert torch.equal(perm, perm_w)
        assert torch.equal(off, bins_w.tile_offset)
        assert torch.equal(items, bins_w.tile_items)
        for fld in ("tile", "num_tiles", "bin_extent"):
            assert list(getattr(bins, fld)) == list(getattr(bins_w.desc, fld))
        assert (bins.order, bins.location, bins.chunk) == (2, FieldLocation.Node, chunk)


def test_static_sort_refuses_sizes_beyond_its_scratch(cuda):
    mesh = periodic_mesh(64, halo=0)
    x = torch.zeros((5_000_000, 3), dtype=torch.float64, device="cuda")
    sd = create_spline(FieldLocation.Node, 2, mesh, x)
    st, *_ = _static_sort(sd, (4, 8, 8), 2048)
    assert st == _abi.ERR_OUT_OF_RANGE
