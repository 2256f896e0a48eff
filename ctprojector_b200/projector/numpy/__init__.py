"""Host-array projector modules (ct_projector.projector.numpy of the reference).

Each call copies its inputs to the GPU, runs the sm_100a kernel and copies the
result back (the c* entries of libctp.so), like the reference numpy modules.
"""
from .ct_projector import ct_projector, set_device  # noqa: F401
