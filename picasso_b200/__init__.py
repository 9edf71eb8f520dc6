"""B200-native particle/grid transfers with Picasso's APIC / PolyPIC interface.

The compute path is the CUDA library ``libpicasso_b200.so`` (C ABI declared
in ``include/picasso_b200.h``); this package is the host-side mirror of the
reference's operator interface on top of it.  Importing the package does not
touch the GPU; the first transfer call loads the library and raises if it has
not been built.
"""

from ._abi import PicassoError, load_library  # noqa: F401
from .api import (  # noqa: F401
    APIC,
    Batch,
    BatchInstance,
    Bins,
    Exec,
    FieldLocation,
    FixedGrid,
    InterpolationOrder,
    PolyPIC,
    SortBuffers,
    Spline,
    UniformMesh,
    advect,
    cell_sort,
    create_spline,
    fixed_bits_for,
    grid_field,
    grid_fill,
    grid_update,
    grid_velocity,
    mat3_inverse,
    p2g_update_workspace,
    particle_field,
    permute,
    permute_members,
    sort_workspace,
    spline_records,
    tune_tiled_step,
)

__version__ = "0.1.0"
