"""channel3d_parallel_b200 -- B200 (sm_100a) RK3 fractional-step path of channel3D.

A drop-in GPU implementation of the reference's ``compute_time_step_RK3``
(MetamaterialFSI/channel3D_parallel, src/time_integration.f90:86-213) and
everything it calls, behind the C-ABI of ``include/c3d.h`` (``libc3d.so``).
``Channel`` is the Python host mirror of the reference's module interfaces.
"""
from .lib import C3DError, load  # noqa: F401
from .channel import Channel, namelist_text, seeded_initial_state, laminar_perturbed_fields  # noqa: F401

__all__ = ["Channel", "C3DError", "load", "namelist_text", "seeded_initial_state",
           "laminar_perturbed_fields"]
