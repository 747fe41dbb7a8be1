"""ordvec_b200: B200 (sm_100a) implementation of ordvec's compressed-scan path.

Device-resident indices and CUDA kernels behind the reference's C ABI
(include/ordvec_b200.h) with a Python mirror of the reference API.
"""
from ._lib import LIB_PATH, OrdvecError, lib
from .api import (Bitmap, CandidateBatch, MultiBucketBitmap, Rank, RankQuant, RankQuantFastscan,
                  SearchResults, Server, SignBitmap, Ticket, TwoStageCandidatePolicy, last_launch_count, load,
                  search_device, set_device, synth_docs, synth_queries, two_stage_profile, two_stage_search,
                  two_stage_search_device, search_mixed, mixed_plan_info)

__all__ = [
    "Bitmap", "CandidateBatch", "MultiBucketBitmap", "OrdvecError", "Rank", "RankQuant", "RankQuantFastscan",
    "SearchResults", "SignBitmap", "TwoStageCandidatePolicy", "LIB_PATH", "last_launch_count", "lib",
    "load", "search_device", "synth_docs", "synth_queries", "two_stage_search", "Server", "Ticket", "search_mixed", "mixed_plan_info",
]
