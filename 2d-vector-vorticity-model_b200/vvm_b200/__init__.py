"""Host side of the B200 VVM time step.

* ``initial_state`` -- seeded synthetic states in the reference's layout.
* ``config``        -- the reference's key=value config reader.
* ``gpu``           -- ctypes binding of libvvmgpu.so (include/vvm_gpu.h).
* ``build``         -- nvcc build of libvvmgpu.so for sm_100a.
"""
from .config import config_from_file, vvm_read_config
from .initial_state import GridSpec, VVMState, base_state, random_state, warm_bubble

__all__ = ["GridSpec", "VVMState", "base_state", "random_state", "warm_bubble",
           "vvm_read_config", "config_from_file"]
