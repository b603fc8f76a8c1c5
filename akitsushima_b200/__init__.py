"""akitsushima_b200: the many-body force path of akitsushima on B200 GPUs.

Neighbour list and Tersoff / Stillinger-Weber / alloy EAM (Zhou 2004,
setfl splines) energy + force + virial, evaluated by hand-written sm_100a
CUDA kernels in libmbforce.so (C ABI: include/mbforce.h), behind the
reference's own API: ``force_fn_from_config``, ``make_force_fn``,
``PotentialEngine``, the potential ``.compute()`` protocol and
``NeighbourList(backend='cuda')``.
"""
from .batched import BatchedEvaluator
from .eam import EAMPotential, continuous, read_setfl, zhou_cutoff, zhou_eam
from .force_fn import (PotentialEngine, accepts_need_stress, call_force_fn,
                       force_fn_from_config, make_force_fn)
from .neighbourlist import (DeviceNeighbourList, NeighbourList, NullNeighbourList,
                            clear_owned_neighbour_lists, neighbour_list_for,
                            owned_neighbour_list, uses_neighbour_list)
from .published_parameters import SW_SI_1985, TERSOFF_1989, TERSOFF_SI_1988, ZHOU_2004
from .spatial import SpatialForceFn, slab_partition
from .stillinger_weber import StillingerWeberPotential
from .system import Batch
from .tersoff import TersoffPotential, tersoff1989_to_triplets

__version__ = "0.1.0"

__all__ = [
    "Batch", "BatchedEvaluator", "DeviceNeighbourList", "EAMPotential", "NeighbourList", "NullNeighbourList",
    "PotentialEngine", "SpatialForceFn", "StillingerWeberPotential", "TersoffPotential", "accepts_need_stress",
    "call_force_fn", "clear_owned_neighbour_lists", "continuous", "force_fn_from_config",
    "make_force_fn", "neighbour_list_for", "owned_neighbour_list", "read_setfl", "slab_partition",
    "tersoff1989_to_triplets", "uses_neighbour_list", "zhou_cutoff", "zhou_eam",
    "SW_SI_1985", "TERSOFF_1989", "TERSOFF_SI_1988", "ZHOU_2004",
]
