"""sesmesh_b200: the SES mesh stage of sesmesh on one NVIDIA B200 (sm_100a).

`native` binds the C ABI of include/sesmesh_b200.h (device kernels and their
host runtime); `workloads` makes the seeded synthetic inputs.
"""
from . import native  # noqa: F401

__version__ = "0.1.0"
