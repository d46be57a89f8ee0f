"""nmhd_b200: a B200-native (sm_100a) ideal-MHD time step with the solver
interface of nushio3/nmhd's ``MHDSolver``.

The compute path lives in ``libnmhd.so`` (C ABI, include/nmhd.h) built from
``nmhd_b200/csrc``; this package holds the host-side mirror of the reference
interface (:class:`~nmhd_b200.solver.MHDSolver`), problem setup and ``.bin`` I/O.
"""
from .config import SolverConfig  # noqa: F401
from .binio import read_bin, write_bin  # noqa: F401
