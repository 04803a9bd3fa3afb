"""B200 (sm_100a) implementation of CHAPSim's periodic-channel time step.

Host-side package: set-up restatement (:mod:`.mesh`), seeded fields and the
``.D`` file format (:mod:`.fields`), and the ctypes mirror of the reference's
subroutine interface over the C ABI of ``libchapsim_gpu.so`` (:mod:`.gpu`).
"""
from .mesh import ChannelSetup, channel_setup  # noqa: F401
from .fields import initial_field, bulk_velocity, read_dfile, write_dfile  # noqa: F401
