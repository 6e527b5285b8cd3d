"""msa_b200 — B200-native all-pairs Needleman-Wunsch and neighbor-joining with
the API surface of Museqa's pairwise and phylogeny modules.

The compute path is libmsa_b200.so (hand-written CUDA for sm_100a behind the C
ABI in include/msa_b200.h). This package is the Python face of that ABI.
"""
from . import pairwise, phylogeny, runtime
from .database import Database
from .pairwise import DistanceMatrix, ScoringTable
from .sequence import Sequence, encode

__all__ = ["Database", "DistanceMatrix", "ScoringTable", "Sequence", "encode", "pairwise", "phylogeny", "runtime"]
