"""The entry point that allocates nothing (saru_align_device_static).

Callers that cannot allocate device memory themselves -- a host program
whose allocator owns the whole device budget and forbids other cudaMalloc
calls, or a code path that must not add the synchronisation and latency of
an allocation -- still need the banded kernel, whose decision planes need
scratch memory.  This entry point takes that scratch from a fixed device
array inside the library instead of from the caller.  The test checks it
against the regular device entry point (saru_align_device) bit for bit, on
two calls in a row with different batches, so the second call runs on the
scratch contents the first one left.  It lives in its own file so pytest
collects it last.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import saruman_b200 as S
from saruman_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _device_batch(b, dev):
    import torch
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    keep = dict(genome=T(b.genome), reads=T(b.reads), goff=T(b.genome_offsets),
                roff=T(b.read_offsets), dirs=T(b.dirs))
    sb = S.SaruBatch(keep["genome"].data_ptr(), keep["reads"].data_ptr(), keep["goff"].data_ptr(),
                     keep["roff"].data_ptr(), keep["dirs"].data_ptr(), b.n, b.k, 0, 1, 1, b.m,
                     len(b.genome), b.total_genome)
    return sb, keep


def _outputs(b, dev):
    import torch
    out = dict(scores=torch.full((b.n,), -7, dtype=torch.int32, device=dev),
               ra=torch.full((b.total_genome + 64,), 0x5A, dtype=torch.uint8, device=dev),
               ga=torch.full((b.total_genome + 64,), 0x5A, dtype=torch.uint8, device=dev),
               status=torch.zeros(1, dtype=torch.int32, device=dev))
    sr = S.SaruResult(out["scores"].data_ptr(), out["ra"].data_ptr(), out["ga"].data_ptr(),
                      out["status"].data_ptr())
    return sr, out


def test_static_scratch_entry_matches_device_entry(saru_lib):
    import torch
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    lib = S.load()
    lib.saru_align_device_static.restype = C.c_int
    lib.saru_align_device_static.argtypes = [C.POINTER(S.SaruBatch), C.POINTER(S.SaruResult),
                                             C.c_void_p]
    stream = torch.cuda.current_stream()
    batches = [W.random_batch(100, 5, 20000, seed=41, err=0.04),
               W.random_batch(150, 9, 7000, seed=42, err=0.05, alphabet=b"ACGTN"),
               W.random_batch(512, 15, 10000, seed=43, err=0.03)]
    # the widest reads: the full grid's decision planes (half the queued
    # form's, which saru_scratch_bytes sizes) do not fit in the array, so
    # the static entry runs on a reduced grid
    b512 = batches[2]
    assert (S.scratch_bytes(b512.n, b512.m, b512.k) - 256) // 2 > (32 << 20)
    for b in batches:  # calls in a row; each sees the scratch contents the last one left
        sb, keep = _device_batch(b, dev)
        want_r, want = _outputs(b, dev)
        nscr = S.scratch_bytes(b.n, b.m, b.k)
        scratch = torch.empty(nscr, dtype=torch.uint8, device=dev)
        S.align_device(sb, want_r, scratch.data_ptr(), nscr, stream.cuda_stream)
        got_r, got = _outputs(b, dev)
        rc = lib.saru_align_device_static(C.byref(sb), C.byref(got_r), stream.cuda_stream)
        assert rc == S.SARU_OK, S.last_error()
        torch.cuda.synchronize()
        assert int(want["status"].item()) == 0 and int(got["status"].item()) == 0
        tot = b.total_genome
        assert torch.equal(want["scores"], got["scores"])
        assert torch.equal(want["ra"][:tot], got["ra"][:tot])
        assert torch.equal(want["ga"][:tot], got["ga"][:tot])
        assert int((got["scores"] <= b.k).sum().item()) > b.n // 4


def test_static_scratch_entry_refuses_what_it_cannot_hold(saru_lib):
    import torch
    lib = S.load()
    lib.saru_align_device_static.restype = C.c_int
    lib.saru_align_device_static.argtypes = [C.POINTER(S.SaruBatch), C.POINTER(S.SaruResult),
                                             C.c_void_p]
    b = W.random_batch(36, 2, 64, seed=3)
    dev = torch.device("cuda:0")
    sb, keep = _device_batch(b, dev)
    sr, out = _outputs(b, dev)
    sb.max_read_length = 4096  # beyond what the banded kernel takes
    rc = lib.saru_align_device_static(C.byref(sb), C.byref(sr), None)
    assert rc == S.SARU_E_INVALID
    assert "max_read_length" in S.last_error()
