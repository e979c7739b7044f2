"""B200-native multilevel spectral bisection (HEC coarsening, coarse-graph
construction, Fiedler power iteration, median split) behind the sgpar.h
partition API of cmg (IPDPS 2021 graph coarsening).

The compute path is ``libsgpar_b200.so`` (hand-written sm_100a kernels, C ABI
in ``include/sgpar_b200.h``); this package only binds it.
"""
from .graphs import CSR  # noqa: F401

__all__ = ["CSR", "api", "graphs", "build"]
