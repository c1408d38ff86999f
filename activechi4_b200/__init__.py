"""activechi4_b200 — B200-native (sm_100a) MD timestep for the active
Kob-Andersen glass, a drop-in for the reference's cell_list+forces.c,
active.c and time_evolve.c entry points.

The compute path is the in-tree CUDA library ``libactivechi4_b200.so`` (built
by ``activechi4_b200.build``) behind the C ABI in ``include/activechi4.h``.
"""
from .engine import Engine, default_params, footprint, observables_from_sums, qvectors  # noqa: F401
from .init import State, box_length, lattice_state, n_active, select_active  # noqa: F401

__all__ = ["Engine", "default_params", "footprint", "State", "box_length", "lattice_state",
           "n_active", "select_active"]
