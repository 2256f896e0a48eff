"""Device-array projector modules (ct_projector.projector.cupy of the reference).

Arrays are torch CUDA tensors (or any object with __cuda_array_interface__,
e.g. cupy arrays, which are returned as cupy arrays).
"""
from .ct_projector import ct_projector, set_device  # noqa: F401
