"""psum_b200 -- B200 (sm_100a) electrostatic PIC step behind PSuM's plugin ABI.

Native library: ``libpsum_b200.so`` (built in-tree by ``psum_b200.build``),
exporting the solver plugin ABI of include/psum_field_solver.h, the
particle-kernel set of include/psum_pic.h and the B-spline interpolation of
include/psum_interp.h.  The Python modules are thin
ctypes mirrors of the reference interfaces; there is no CPU fallback.
"""
from ._lib import LIB_PATH, PROTOTYPES, PsumError, check, lib
from .field_solver import (Dirichlet_box, Dirichlet_box_rz, Dirichlet_func, Dirichlet_line, Dirichlet_nodes,
                           Dirichlet_plane, Dirichlet_point, Dirichlet_range, MixedBoundary, Neumann_line,
                           Neumann_plane, Neumann_point, Poisson_solver_1d, Poisson_solver_2d, Poisson_solver_3d,
                           Robin_Line, Robin_plane, Robin_point, assemble_poisson, assemble_poisson_1d,
                           assemble_poisson_2d, assemble_poisson_3d, registered_table, simple_grid, solver_backend)
from .interp import add_back_B_spline, interp_B_spline, interp_diff_B_spline
from .pic import BORIS, FP64, LEAPFROG, MIXED, ParticleContext

__all__ = ["LIB_PATH", "PROTOTYPES", "PsumError", "check", "lib", "Dirichlet_line", "Dirichlet_nodes",
           "Dirichlet_plane", "Dirichlet_box", "Dirichlet_box_rz", "Dirichlet_func", "Neumann_line", "Robin_Line",
           "Neumann_plane", "Robin_plane", "MixedBoundary", "Poisson_solver_2d", "Poisson_solver_3d",
           "assemble_poisson", "assemble_poisson_2d", "assemble_poisson_3d", "registered_table", "simple_grid",
           "solver_backend", "ParticleContext", "MIXED", "FP64", "LEAPFROG", "BORIS", "interp_B_spline",
           "interp_diff_B_spline", "add_back_B_spline", "Poisson_solver_1d", "Dirichlet_point", "Dirichlet_range",
           "Neumann_point", "Robin_point", "assemble_poisson_1d"]
