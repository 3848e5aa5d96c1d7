"""B200-native SIMP compliance minimisation with the Problem / mesh / Ke / YAML
interface of tomohiron907/toptimization.

Host code keeps every field in PyTorch CUDA tensors and calls the sm_100a
kernels of libtpo through its C ABI (`include/tpo.h`). There is no CPU path.
"""

from .problem import Problem, load_problem  # noqa: F401

__version__ = "0.1.0"
