"""ddg_b200: B200-native (sm_100a) matrix-free SIPG Poisson/Helmholtz solves
for 2D nodal-DG triangle meshes, a drop-in for ddg's ``dg2d.sipg`` /
``dg2d.multigrid`` solve path.  Host setup is numpy + C++; every operator
apply, Krylov iteration, preconditioner and load runs in the CUDA library
``ddg_b200/lib/libddg_sipg.so`` (build: ``python -m ddg_b200.build``).
"""

__version__ = "0.1.0"
