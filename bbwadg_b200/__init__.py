"""B200-native acoustic WADG time step on affine tetrahedra.

Drop-in for the time step of jlchan/bbwadg's cpp/ solver
(RK_step_WADG_subelem, cpp/src/WaveOKL3d.cpp:2084-2109) in its nodal and
Bernstein-Bezier variants.  The native library (libbbwadg_b200.so, C ABI in
include/bbwadg.h) holds the sm_100a kernels, the solver context and the host
setup; this package is a thin Python front end over it.
"""
from .mesh import kuhn_box, read_gmsh22, write_gmsh22  # noqa: F401
from .problem import (Problem, build_operators, cavity_mode, connect_and_geometry,  # noqa: F401
                      gaussian_pulse, make_problem)
from .solver import RK4A, RK4B, RK4C, WaveSolver  # noqa: F401

__all__ = ["kuhn_box", "read_gmsh22", "write_gmsh22", "Problem", "build_operators",
           "connect_and_geometry", "make_problem", "cavity_mode", "gaussian_pulse", "WaveSolver",
           "RK4A", "RK4B", "RK4C"]
