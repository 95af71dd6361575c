"""gnomon_b200 — B200-native (sm_100a) polygenic-score hot path.

Drop-in for the GPU slot of gnomon's ``score::pipeline`` (SauersML/gnomon):
packed PLINK .bed unpack fused with the missing-call rule, effect-allele flip
reconciliation and dosage x weight accumulation, returning per-person FP64
sums plus missing counts.  The compute lives in ``libgnomon_gpu.so`` (C ABI,
``include/gnomon_gpu.h``); this package is the host-side mirror.
"""
from . import _lib, prepare, synth  # noqa: F401

__all__ = ["_lib", "prepare", "synth"]
