"""B200-native CG2D free-surface pressure solver: a drop-in for mitgcm_jax's cg2d_fortran / cg2d_solve.

Importing the package does not touch the GPU; the CUDA library (libcg2d.so, built in-tree) is loaded on first use.
"""

from mit_jax_b200.layout import LLC90, LLC270, Layout  # noqa: F401

__version__ = "0.1.0"
