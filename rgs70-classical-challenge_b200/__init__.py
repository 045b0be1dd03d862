"""B200-native graph-state probability and exact Born-sampling engine.

Drop-in for the scan-contraction and conditional-sampler path of
whyihaveyou/rgs70-classical-challenge.  Python host code calls hand-written
sm_100a CUDA kernels in ``librgs_b200.so`` through the C ABI of
``include/rgs_b200.h``; torch tensors are used only as device buffers.
"""
from . import _lib
from .plan import ScanPlan, Step, make_plan, future_masks, rank_profile, byte_tables, kernel_combos, \
    edges_from_graph, search_order
from .scan_oracle import ScanEngine, ScanOracle, pack_bits, amplitudes_from, PRECISIONS, capture_graph, autotune_tile, \
    max_batch_tile
from . import instances
from .samplers import ConditionalSampler, ShardedConditionalSampler, DrawRecorder, produce, fwht, product, block_mass
from .chain import ChainSampler, unpack_bits
from .batch import ResidentBatch
from . import batch
from . import frontend
from . import replicas
from . import proposal
from .proposal import MadeProposal, rejection_sample, capped_rejection, calibrate_envelope

__all__ = [
    "ScanPlan", "Step", "make_plan", "future_masks", "rank_profile", "byte_tables", "kernel_combos",
    "edges_from_graph", "search_order", "ScanEngine", "ScanOracle", "pack_bits", "amplitudes_from", "PRECISIONS", "capture_graph", "autotune_tile",
    "ConditionalSampler", "ShardedConditionalSampler", "DrawRecorder", "produce", "fwht", "product", "block_mass", "ChainSampler", "unpack_bits", "ResidentBatch",
    "MadeProposal", "rejection_sample", "capped_rejection", "calibrate_envelope",
]
