"""ChysX cloth step, B200-native.

Drop-in for the reference package's cloth API (chysx/__init__.py of
caixiao-0725/Ai-Phyiscs): ``ClothMaterial`` and ``ClothSimulator`` with the
same constructor, method names, argument names and defaults.  The simulator
borrows raw CUDA device pointers (``tensor.data_ptr()`` or ``wp.array.ptr``)
to float3 position / velocity buffers and advances them in place::

    import chysx
    mat = chysx.ClothMaterial()
    mat.gx, mat.gy, mat.gz = 0.0, -9.81, 0.0
    sim = chysx.ClothSimulator()
    sim.set_material(mat)
    sim.set_external_buffers(pos_ptr, vel_ptr, n, inv_mass_ptr)
    sim.set_mesh(tris)
    sim.redistribute_mass_area_weighted(0.1, inv_mass_ptr, n)
    sim.build_springs_from_current_positions(1e3)
    sim.build_fem_stretch_from_current_positions(1e4)
    sim.set_pins(idx, targets)
    sim.step(1.0 / 60.0)

Importing fails loudly if the compiled extension is missing: there is no
CPU fallback.
"""
from __future__ import annotations

from . import _chysx_native

ClothMaterial = _chysx_native.ClothMaterial
ClothSimulator = _chysx_native.ClothSimulator
ClothVBDSolver = _chysx_native.ClothVBDSolver

__version__ = "0.1.0"

__all__ = ["ClothMaterial", "ClothSimulator", "ClothVBDSolver", "__version__"]
