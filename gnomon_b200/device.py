"""Device-resident scoring: a plan over genotypes that already live in HBM.

PyTorch supplies device memory and streams only; all arithmetic runs in
``libgnomon_gpu.so``.  ``DevicePlan`` wraps the ``gnm_plan_*`` entry points.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _lib
from .pipeline import prep_view
from .prepare import PreparationResult


def row_pitch(bytes_per_variant: int, align: int = 128) -> int:
    """Device row pitch: bytes per variant rounded up to ``align`` (a multiple of 16)."""
    return (bytes_per_variant + align - 1) // align * align


def _stream_ptr(stream: Optional[torch.cuda.Stream]) -> Optional[int]:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream or None


class DevicePlan:
    """Prepared weights on one device plus FP64 partial accumulators."""

    def __init__(self, prep: PreparationResult, engine: int = _lib.ENGINE_AUTO,
                 device: Optional[int] = None):
        self.lib = _lib.load()
        self.prep = prep
        self.device = torch.cuda.current_device() if device is None else device
        self._view = prep_view(prep)
        handle = C.c_void_p()
        err = _lib.gnm_error()
        st = self.lib.gnm_plan_create(C.byref(self._view), engine, self.device, C.byref(handle),
                                      C.byref(err))
        _lib.check(st, err)
        self.handle = handle

    def close(self):
        if getattr(self, "handle", None):
            self.lib.gnm_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def engine(self) -> int:
        return self.lib.gnm_plan_engine(self.handle)

    @property
    def launches(self) -> int:
        return int(self.lib.gnm_plan_launch_count(self.handle))

    @property
    def device_bytes(self) -> int:
        return int(self.lib.gnm_plan_device_bytes(self.handle))

    def _err(self):
        return _lib.gnm_error()

    def reset(self, stream=None):
        e = self._err()
        _lib.check(self.lib.gnm_plan_reset(self.handle, _stream_ptr(stream), C.byref(e)), e)

    def accumulate(self, rows: torch.Tensor, pitch: int, variant_begin: int,
                   variant_count: int, stream=None):
        assert rows.is_cuda and rows.dtype == torch.uint8
        e = self._err()
        _lib.check(self.lib.gnm_plan_accumulate_device(self.handle, rows.data_ptr(), pitch,
                                                       variant_begin, variant_count,
                                                       _stream_ptr(stream), C.byref(e)), e)

    def finalize(self, sums: torch.Tensor, counts: torch.Tensor, stream=None):
        e = self._err()
        _lib.check(self.lib.gnm_plan_finalize_device(self.handle, sums.data_ptr(),
                                                     counts.data_ptr(), _stream_ptr(stream),
                                                     C.byref(e)), e)

    def sync(self, stream=None):
        e = self._err()
        _lib.check(self.lib.gnm_plan_sync(self.handle, _stream_ptr(stream), C.byref(e)), e)

    def outputs(self):
        P, K = self.prep.num_people_to_score, self.prep.num_scores
        dev = torch.device("cuda", self.device)
        return (torch.empty(P * K, dtype=torch.float64, device=dev),
                torch.empty(P * K, dtype=torch.int32, device=dev))

    def score(self, rows: torch.Tensor, pitch: int, sums=None, counts=None, stream=None):
        """reset + accumulate(all rows) + finalize; returns device (sums f64, counts i32)."""
        if sums is None:
            sums, counts = self.outputs()
        e = self._err()
        _lib.check(self.lib.gnm_score_device(self.handle, rows.data_ptr(), pitch,
                                             sums.data_ptr(), counts.data_ptr(),
                                             _stream_ptr(stream), C.byref(e)), e)
        return sums, counts

    def autotune(self, rows: torch.Tensor, pitch: int, variant_count: Optional[int] = None,
                 stream=None) -> int:
        """Time candidate launch shapes on resident rows, keep the fastest; returns it."""
        n = self.prep.num_reconciled_variants if variant_count is None else variant_count
        e = self._err()
        _lib.check(self.lib.gnm_plan_autotune(self.handle, rows.data_ptr(), pitch, n,
                                              _stream_ptr(stream), C.byref(e)), e)
        return int(self.lib.gnm_plan_tuned_shape(self.handle))

    def set_shape(self, shape: int) -> None:
        """Pin a launch shape (a value ``autotune`` returned)."""
        e = self._err()
        _lib.check(self.lib.gnm_plan_set_shape(self.handle, int(shape), C.byref(e)), e)

    @property
    def shape(self) -> int:
        return int(self.lib.gnm_plan_tuned_shape(self.handle))

    def set_backward_limbs(self, bits: int) -> None:
        """dS limb width of ``backward``: 8 (default) or 16 (BF16)."""
        e = self._err()
        _lib.check(self.lib.gnm_plan_set_backward_limbs(self.handle, int(bits), C.byref(e)), e)

    def capture(self, rows: torch.Tensor, pitch: int, sums=None, counts=None):
        """Record one full scoring pass (reset + accumulate + finalize) into a CUDA
        graph; ``graph.replay()`` reruns it with no per-launch host work.  Returns
        (graph, sums, counts) — the output tensors the graph writes."""
        if sums is None:
            sums, counts = self.outputs()
        side = torch.cuda.Stream(rows.device)
        with torch.cuda.stream(side):     # warm-up outside capture (sets kernel attributes)
            self.score(rows, pitch, sums, counts, stream=side)
        side.synchronize()
        self.sync(side)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=side):
            self.score(rows, pitch, sums, counts, stream=torch.cuda.current_stream())
        return graph, sums, counts

    def backward(self, rows: torch.Tensor, pitch: int, grad_s: torch.Tensor,
                 grad_corr: bool = False, stream=None):
        """dW = G^T dS by re-unpacking the packed rows; returns dense [V, K] float32."""
        V, K = self.prep.num_reconciled_variants, self.prep.num_scores
        gs = grad_s.contiguous().to(torch.float32)
        gw = torch.empty(V * K, dtype=torch.float32, device=gs.device)
        gc = torch.empty(V * K, dtype=torch.float32, device=gs.device) if grad_corr else None
        e = self._err()
        _lib.check(self.lib.gnm_backward_dw_device(self.handle, rows.data_ptr(), pitch,
                                                   gs.data_ptr(), gw.data_ptr(),
                                                   gc.data_ptr() if gc is not None else None,
                                                   _stream_ptr(stream), C.byref(e)), e)
        return gw.view(V, K), (gc.view(V, K) if gc is not None else None)


def synth_fill(rows: torch.Tensor, pitch: int, variant_begin: int, num_variants: int,
               num_people: int, thresholds: np.ndarray, seed: int, stream=None,
               person_begin: int = 0):
    """Fill device rows with the deterministic HWE generator (gnomon_b200.synth).

    Column c holds cohort person ``person_begin + c``."""
    lib = _lib.load()
    thr = torch.from_numpy(np.ascontiguousarray(thresholds, dtype=np.uint32).view(np.int32)).to(
        rows.device)
    e = _lib.gnm_error()
    _lib.check(lib.gnm_synth_fill_device(rows.data_ptr(), pitch, variant_begin, num_variants,
                                         person_begin, num_people, thr.data_ptr(), seed,
                                         _stream_ptr(stream), C.byref(e)), e)
    return thr


def decode(rows: torch.Tensor, pitch: int, num_variants: int, num_people: int, stream=None):
    """Device decode to int8 {0,1,2,-1 missing} [V, P]."""
    lib = _lib.load()
    out = torch.empty(num_variants * max(num_people, 1), dtype=torch.int8, device=rows.device)
    e = _lib.gnm_error()
    _lib.check(lib.gnm_decode_device(rows.data_ptr(), pitch, num_variants, num_people,
                                     out.data_ptr(), num_people, _stream_ptr(stream),
                                     C.byref(e)), e)
    return out.view(num_variants, num_people)
