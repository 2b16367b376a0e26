"""B200-native thermal lattice-Boltzmann time step (MRT D2Q9/D3Q19 + D2Q5/D3Q7
ISLBM on stretched grids): the drop-in for the time step of
zzhao0930/MPI-Multi-Process-Version, behind the C ABI in include/lbm_b200.h."""
from .lbm import (EXPORTS, GRID, MODE, NOALLOC_MAX_NODES, STORE, Batch, Cavity, LBMError, Mesh, check_noalloc,
                  fortran_e, kernel_launches, lbm_params, lib, mesh, mesh_box, output_ascii, run_main, sweep_specs,
                  write_tecplot)

from . import studies  # noqa: E402
from . import sharding  # noqa: E402
from . import slabs  # noqa: E402
from . import surrogate  # noqa: E402
from . import warmstart  # noqa: E402

__all__ = ["studies", "sharding", "surrogate", "warmstart", "EXPORTS", "GRID", "MODE", "NOALLOC_MAX_NODES", "STORE", "Batch", "Cavity", "LBMError", "Mesh",
           "check_noalloc", "sweep_specs", "mesh_box",
           "fortran_e", "kernel_launches", "lbm_params", "lib", "mesh", "output_ascii", "run_main", "write_tecplot"]
