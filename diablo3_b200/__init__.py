"""diablo3_b200 -- DIABLO 3.0's channel RK substep (RKW3 + Crank-Nicolson)
on one B200, behind the C-ABI of include/diablo_b200.h.

The compute path is libdiablo_b200.so (CUDA, sm_100a); this package holds
the host-side mirror of the reference's driver interface: run parameters
(input.dat / input_chan.dat), the wall-normal grid (create_grid.m), initial
conditions (create_flow_chan) and the ``Channel`` wrapper.
"""
from .params import DbParams, make_params, read_inputs  # noqa: F401
from .grid import create_grid, metrics  # noqa: F401

__all__ = ["DbParams", "make_params", "read_inputs", "create_grid", "metrics", "Channel"]


def __getattr__(name):
    if name == "Channel":
        from .channel import Channel
        return Channel
    raise AttributeError(name)
