"""B200-native walk-on-spheres: the per-grid-point WoS estimator of
zhouzh721/walk-on-spheres as hand-written sm_100a CUDA kernels behind a C ABI
(include/wos_b200.h, libwos_b200.so), with the reference's equation registry,
OBJ input, --seed semantics and HDF5 result layout.

    from walk_on_spheres_b200 import Solver, meshes
    s = Solver(0).set_mesh(meshes.annulus())
    r = s.solve_grid("laplace", 64, 64, N_walks=10000, seed=12345)
"""
from .meshes import Mesh  # noqa: F401

__all__ = ["Solver", "registry", "peek_mesh_dim", "meshes", "h5lite", "Mesh"]


def __getattr__(name):
    # the CUDA binding loads lazily so mesh generation and file reading work
    # on machines without the built library
    if name in ("Solver", "registry", "peek_mesh_dim", "GridResult", "EQUATIONS"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)
