"""ddg_b200: B200-native (sm_100a) matrix-free SIPG Poisson/Helmholtz solves
for 2D nodal-DG triangle meshes, a drop-in for ddg's ``dg2d.sipg`` /
``dg2d.multigrid`` solve path.  Host setup is numpy + C++; every operator
apply, Krylov iteration, preconditioner and load runs in the CUDA library
``ddg_b200/lib/libddg_sipg.so`` (build: ``python -m ddg_b200.build``).
"""

__version__ = "0.1.0"


def pinned_empty(shape, dtype="float64"):
    """A numpy array in page-locked host memory (a view of a pinned torch
    tensor, kept alive by the array).  Host fields in pinned memory are
    read and written by the GPU copy engines directly, e.g. by
    ``SipgOperator.apply_host``."""
    import numpy as np
    import torch
    t = torch.empty(tuple(shape), dtype=getattr(torch, np.dtype(dtype).name), pin_memory=True)
    return t.numpy()
