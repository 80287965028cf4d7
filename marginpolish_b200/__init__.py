"""B200-native (sm_100a) realignment engine for MarginPolish's banded pair-HMM
posterior pass. The compute path is the in-tree CUDA library libmpgpu.so
(C ABI in include/mpgpu.h); this package is its host-side interface."""
from . import _lib
from .params import AlignmentParams, PolishModel, StateModel, build_state_model, load_polish_model
from .realign import (DeviceBatch, Engine, Expectations, Jobs, Model, Pairs, compute_forward_probability,
                      expectations_batch, forward_batch, forward_pairs, forward_pairs_timing, match_pairs_reference, get_aligned_pairs_using_anchors,
                      get_aligned_pairs_with_indels_using_anchors, realign_batch,
                      realign_batch_pipelined)
from .rle import RleString, crop_range, rle_anchors
from .poa import PoaSet, PolishParams, merge_contig, merge_contig_threaded, polish

__all__ = [
    "AlignmentParams", "PolishModel", "StateModel", "build_state_model", "load_polish_model", "DeviceBatch",
    "Engine", "Jobs", "Model", "Pairs", "get_aligned_pairs_using_anchors",
    "get_aligned_pairs_with_indels_using_anchors", "realign_batch", "realign_batch_pipelined", "RleString", "crop_range", "rle_anchors",
    "compute_forward_probability", "forward_batch", "forward_pairs", "forward_pairs_timing", "match_pairs_reference", "expectations_batch", "Expectations", "PoaSet", "PolishParams",
    "polish", "merge_contig", "merge_contig_threaded",
]
