"""brp_b200 -- the BRP4 per-template search path (orbital resampling, mean
padding, packed real FFT, power spectrum, 1/2/4/8/16-harmonic summing,
candidate compaction, bank-wide toplist) on NVIDIA B200 (sm_100a).

Host side of the C ABI in include/brp_cuda.h.  ``GPU`` mirrors the
reference's brp::GPU, ``Bank`` runs a whole orbital bank in one CUDA graph,
``host`` holds the reference's host functions (template constants, search
parameters, toplist), ``synth`` the seeded synthetic workloads.
"""
from ._lib import (BANK_CANDIDATE, CANDIDATE, EXPORTS, BrpError, Params, STATUS_WAIT_TIMEOUT, STATUS_OVERFLOW,
                   STATUS_RESAMPLE_OOB, build, lib)
from .bank import Bank
from .gpu import GPU, Snapshot
from .host import Toplist, parameters, production, resampling_steps, search_parameters

__all__ = ["GPU", "Bank", "Snapshot", "Params", "Toplist", "BrpError", "parameters", "production",
           "resampling_steps", "search_parameters", "build", "lib", "CANDIDATE", "BANK_CANDIDATE", "EXPORTS",
           "STATUS_OVERFLOW", "STATUS_RESAMPLE_OOB", "STATUS_WAIT_TIMEOUT"]
