"""The mesh generator used by the tests: ndg_cuda_b200.meshgen."""
from ndg_cuda_b200.meshgen import *  # noqa: F401,F403
from ndg_cuda_b200.meshgen import flatten, hilbert_d2xy, su2_markers, uniform_zone, write_su2  # noqa: F401
