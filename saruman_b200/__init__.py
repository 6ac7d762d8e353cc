"""saruman_b200 -- B200 (sm_100a) alignment stage of SARUMAN behind its C ABI.

The product is libsaruman_b200.so (built in-tree by saruman_b200.build):
CUDA kernels plus the reference's four entry points (cuda_needleman_wunsch,
cuda_allocate_memory, cuda_free_memory, get_cuda_infos; see
include/saruman_b200.h).  This module is a thin ctypes view of that library
for Python callers (tests, bench, the serving loop).  There is no Python or
CPU implementation of the alignment: if the library is missing, loading
fails.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from pathlib import Path

import numpy as np

from .workloads import Batch

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libsaruman_b200.so"

SARU_OK, SARU_E_INVALID, SARU_E_CUDA, SARU_E_NOMEM, SARU_E_OVERFLOW = 0, 1, 2, 3, 4
SARU_E_TIMEOUT = 5
SARU_MAX_CALLS = 192
SARU_S_IRREGULAR, SARU_S_ALPHABET, SARU_S_OVERFLOW, SARU_S_GATHER = 1, 2, 4, 16

# symbols include/saruman_b200.h declares
ABI_FUNCTIONS = ("cuda_needleman_wunsch", "cuda_allocate_memory", "cuda_free_memory",
                 "get_cuda_infos", "saru_align_host", "saru_align_device", "saru_scratch_bytes",
                 "saru_format_tsv", "saru_last_error", "saru_kernel_launches",
                 "saru_int32_issue_probe", "saru_align_device_static",
                 "saru_align_multi_device", "saru_multi_scratch_bytes", "saru_server_create",
                 "saru_server_submit", "saru_server_wait", "saru_server_counters",
                 "saru_server_destroy", "saru_server_set_genome", "saru_gather_device",
                 "saru_tuning_set", "saru_tuning_get", "saru_tuning_clear",
                 "saru_mlp_param_count", "saru_mlp_work_floats", "saru_mlp_forward",
                 "saru_mlp_loss_grad", "saru_mlp_adam_step", "saru_compact_record_bytes",
                 "saru_align_device_compact", "saru_expand_compact", "saru_format_tsv_compact",
                 "saru_filter_create", "saru_filter_run", "saru_filter_results",
                 "saru_filter_last_ms", "saru_filter_genome", "saru_filter_destroy",
                 "saru_filter_set_chunk", "saru_align_host_compact",
                 "saru_reads_open", "saru_reads_next", "saru_reads_close", "saru_genome_open",
                 "saru_genome_next", "saru_genome_close", "saru_server_submit_reads",
                 "saru_server_read_results", "saru_server_release", "saru_tsv_to_sam",
                 "saru_align_multi_device_compact")
ABI_DATA = ("alignment_time",)


class SaruError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"saruman_b200 error {code}: {msg}")
        self.code = code


class SaruBatch(C.Structure):
    _fields_ = [("genome", C.c_void_p), ("reads", C.c_void_p), ("genome_offsets", C.c_void_p),
                ("read_offsets", C.c_void_p), ("dirs", C.c_void_p), ("n", C.c_int32),
                ("k", C.c_int32), ("match", C.c_int32), ("mismatch", C.c_int32),
                ("first_of_call", C.c_int32), ("max_read_length", C.c_int32),
                ("genome_bytes", C.c_int64), ("total_slots", C.c_int64)]


class SaruResult(C.Structure):
    _fields_ = [("scores", C.c_void_p), ("read_aln", C.c_void_p), ("genome_aln", C.c_void_p),
                ("status", C.c_void_p)]


class SaruTuning(C.Structure):
    _fields_ = [("warps_per_cta", C.c_int32), ("ctas_per_sm", C.c_int32),
                ("word_bits", C.c_int32)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("pipeline", C.c_int32),
                ("max_requests_per_launch", C.c_int32), ("max_inflight", C.c_int32),
                ("device_budget_bytes", C.c_int64), ("host_pool_bytes", C.c_int64)]


class SaruGatherCall(C.Structure):
    _fields_ = [("read_table", C.c_void_p), ("read_index", C.c_void_p), ("positions", C.c_void_p),
                ("dirs", C.c_void_p), ("genome_offsets", C.c_void_p), ("n", C.c_int32),
                ("nreads", C.c_int32), ("k", C.c_int32), ("match", C.c_int32),
                ("mismatch", C.c_int32), ("first_of_call", C.c_int32),
                ("read_length", C.c_int32), ("genome_bytes", C.c_int64),
                ("total_slots", C.c_int64)]


class SaruRequest(C.Structure):
    _fields_ = [("calls", C.POINTER(SaruBatch)), ("results", C.POINTER(SaruResult)),
                ("ncalls", C.c_int32), ("gather", C.POINTER(SaruGatherCall)),
                ("compact", C.c_int32)]


class RequestStats(C.Structure):
    _fields_ = [("submit_us", C.c_int64), ("admit_us", C.c_int64), ("done_us", C.c_int64),
                ("group", C.c_int32), ("redone_calls", C.c_int32)]


_lib = None


class SaruReadSet(C.Structure):
    _fields_ = [("reads", C.c_void_p), ("nreads", C.c_int32), ("read_length", C.c_int32),
                ("k", C.c_int32), ("chunk_value", C.c_uint32)]


class SaruReadResults(C.Structure):
    _fields_ = [("ncalls", C.c_int32), ("nperfect", C.c_int32), ("n", C.c_int64),
                ("call_begin", C.c_void_p), ("slot_begin", C.c_void_p),
                ("call_strand", C.c_void_p), ("ids", C.c_void_p), ("pos", C.c_void_p),
                ("dirs", C.c_void_p), ("scores", C.c_void_p), ("read_aln", C.c_void_p),
                ("genome_aln", C.c_void_p), ("records", C.c_void_p),
                ("record_bytes", C.c_int64), ("perfect_ids", C.c_void_p),
                ("perfect_pos", C.c_void_p), ("perfect_strand", C.c_void_p)]


def load(path: str | Path | None = None):
    """Loads libsaruman_b200.so (in-tree).  Raises if it is not built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is not built; run `python -m saruman_b200.build` "
                           "(there is no CPU fallback)")
    lib = C.CDLL(str(p))
    lib.saru_align_host.restype = C.c_int
    lib.saru_align_host.argtypes = [C.POINTER(SaruBatch), C.POINTER(SaruResult), C.c_int]
    lib.saru_align_device.restype = C.c_int
    lib.saru_align_device.argtypes = [C.POINTER(SaruBatch), C.POINTER(SaruResult), C.c_void_p,
                                      C.c_size_t, C.c_void_p]
    lib.saru_scratch_bytes.restype = C.c_size_t
    lib.saru_scratch_bytes.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int]
    lib.saru_format_tsv.restype = C.c_int64
    lib.saru_last_error.restype = C.c_char_p
    lib.saru_kernel_launches.restype = C.c_uint64
    lib.get_cuda_infos.restype = C.c_ulong
    lib.saru_align_multi_device.restype = C.c_int
    lib.saru_align_multi_device.argtypes = [C.POINTER(SaruBatch), C.POINTER(SaruResult), C.c_int32,
                                            C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
    lib.saru_align_multi_device_compact.restype = C.c_int
    lib.saru_align_multi_device_compact.argtypes = lib.saru_align_multi_device.argtypes
    lib.saru_multi_scratch_bytes.restype = C.c_size_t
    lib.saru_multi_scratch_bytes.argtypes = [C.POINTER(SaruBatch), C.c_int32]
    lib.saru_server_create.restype = C.c_void_p
    lib.saru_server_create.argtypes = [C.POINTER(ServerConfig)]
    lib.saru_server_submit.restype = C.c_int
    lib.saru_server_submit.argtypes = [C.c_void_p, C.POINTER(SaruRequest), C.POINTER(C.c_int64)]
    lib.saru_server_wait.restype = C.c_int
    lib.saru_server_wait.argtypes = [C.c_void_p, C.c_int64, C.c_int32, C.POINTER(RequestStats)]
    lib.saru_server_counters.restype = None
    lib.saru_server_counters.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.saru_server_destroy.restype = None
    lib.saru_server_set_genome.restype = C.c_int
    lib.saru_server_set_genome.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
    lib.saru_gather_device.restype = C.c_int
    lib.saru_gather_device.argtypes = [C.POINTER(SaruGatherCall), C.c_void_p, C.c_int64,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.POINTER(SaruBatch), C.c_void_p]
    lib.saru_server_destroy.argtypes = [C.c_void_p]
    lib.saru_server_submit_reads.restype = C.c_int
    lib.saru_server_submit_reads.argtypes = [C.c_void_p, C.POINTER(SaruReadSet), C.c_int32,
                                             C.c_int32, C.POINTER(C.c_int64)]
    lib.saru_server_read_results.restype = C.c_int
    lib.saru_server_read_results.argtypes = [C.c_void_p, C.c_int64, C.c_int32,
                                             C.POINTER(SaruReadResults)]
    lib.saru_server_release.restype = None
    lib.saru_server_release.argtypes = [C.c_void_p, C.c_int64]
    lib.saru_tuning_set.restype = C.c_int
    lib.saru_tuning_set.argtypes = [C.c_int32, C.c_int32, C.POINTER(SaruTuning)]
    lib.saru_tuning_get.restype = C.c_int
    lib.saru_tuning_get.argtypes = [C.c_int32, C.c_int32, C.POINTER(SaruTuning)]
    lib.saru_tuning_clear.restype = None
    I32P = C.POINTER(C.c_int32)
    lib.saru_mlp_param_count.restype = C.c_int64
    lib.saru_mlp_param_count.argtypes = [I32P, C.c_int32]
    lib.saru_mlp_work_floats.restype = C.c_int64
    lib.saru_mlp_work_floats.argtypes = [I32P, C.c_int32, C.c_int32]
    lib.saru_mlp_forward.restype = C.c_int
    lib.saru_mlp_forward.argtypes = [I32P, C.c_int32, C.c_void_p, C.c_void_p, C.c_int32,
                                     C.c_void_p, C.c_void_p, C.c_void_p]
    lib.saru_mlp_loss_grad.restype = C.c_int
    lib.saru_mlp_loss_grad.argtypes = [I32P, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.saru_mlp_adam_step.restype = C.c_int
    lib.saru_mlp_adam_step.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64,
                                       C.c_float, C.c_float, C.c_float, C.c_float, C.c_int32,
                                       C.c_void_p]
    lib.saru_compact_record_bytes.restype = C.c_int64
    lib.saru_compact_record_bytes.argtypes = [C.c_int32, C.c_int32]
    lib.saru_align_device_compact.restype = C.c_int
    lib.saru_align_device_compact.argtypes = [C.POINTER(SaruBatch), C.c_void_p, C.c_void_p,
                                              C.c_int64, C.c_void_p, C.c_void_p, C.c_size_t,
                                              C.c_void_p]
    lib.saru_expand_compact.restype = C.c_int
    lib.saru_expand_compact.argtypes = [C.POINTER(SaruBatch), C.c_void_p, C.c_void_p, C.c_int64,
                                        C.c_void_p, C.c_void_p, C.c_int32]
    lib.saru_format_tsv_compact.restype = C.c_int64
    lib.saru_format_tsv_compact.argtypes = [C.POINTER(SaruBatch), C.c_void_p, C.c_void_p,
                                            C.c_int64, C.c_void_p, C.c_void_p, C.c_int32,
                                            C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                                            C.c_int64, C.POINTER(C.c_int32),
                                            C.POINTER(C.c_int32), C.c_int32]
    lib.saru_filter_create.restype = C.c_void_p
    lib.saru_filter_create.argtypes = [C.c_void_p, C.c_int64, C.c_int32, C.c_int32, C.c_int32]
    lib.saru_filter_run.restype = C.c_int
    lib.saru_filter_run.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_uint32,
                                    C.c_void_p]
    lib.saru_filter_results.restype = C.c_int
    lib.saru_filter_results.argtypes = [C.c_void_p] + [C.c_void_p] * 6
    lib.saru_filter_last_ms.restype = C.c_double
    lib.saru_filter_last_ms.argtypes = [C.c_void_p]
    lib.saru_filter_genome.restype = C.c_void_p
    lib.saru_filter_genome.argtypes = [C.c_void_p]
    lib.saru_filter_destroy.restype = None
    lib.saru_filter_destroy.argtypes = [C.c_void_p]
    lib.saru_align_host_compact.restype = C.c_int
    lib.saru_align_host_compact.argtypes = [C.POINTER(SaruBatch), C.c_void_p, C.c_void_p,
                                            C.c_int64, C.c_int32]
    lib.saru_filter_set_chunk.restype = C.c_int
    lib.saru_filter_set_chunk.argtypes = [C.c_void_p, C.c_int64, C.c_int64]
    lib.saru_reads_open.restype = C.c_void_p
    lib.saru_reads_open.argtypes = [C.c_char_p, C.c_int32, C.c_int32, C.c_int32]
    lib.saru_reads_next.restype = C.c_int32
    lib.saru_reads_next.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                    C.POINTER(C.c_int32)]
    lib.saru_reads_close.restype = None
    lib.saru_reads_close.argtypes = [C.c_void_p]
    lib.saru_genome_open.restype = C.c_void_p
    lib.saru_genome_open.argtypes = [C.c_char_p, C.c_int64, C.c_int32]
    lib.saru_genome_next.restype = C.c_int32
    lib.saru_genome_next.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int64),
                                     C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.saru_genome_close.restype = None
    lib.saru_genome_close.argtypes = [C.c_void_p]
    lib.saru_int32_issue_probe.restype = C.c_double
    lib.saru_int32_issue_probe.argtypes = [C.c_int]
    if path is None:
        _lib = lib
    return lib


def last_error() -> str:
    return load().saru_last_error().decode(errors="replace")


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def host_batch(b: Batch, first_of_call: bool = True) -> tuple[SaruBatch, list]:
    """ctypes view of a host batch; the returned list keeps arrays alive."""
    keep = [np.ascontiguousarray(b.genome, np.uint8), np.ascontiguousarray(b.reads, np.uint8),
            np.ascontiguousarray(b.genome_offsets, np.int32),
            np.ascontiguousarray(b.read_offsets, np.int32), np.ascontiguousarray(b.dirs, np.int8)]
    sb = SaruBatch(_p(keep[0]), _p(keep[1]), _p(keep[2]), _p(keep[3]), _p(keep[4]), b.n, b.k,
                   b.match, b.mismatch, 1 if first_of_call else 0, b.m, len(b.genome),
                   b.total_genome)
    return sb, keep


@dataclasses.dataclass
class AlignResult:
    scores: np.ndarray      # int32, D[L][m] if <= k else k + 1
    read_aln: np.ndarray    # uint8, sum(L + k), reference slot layout
    genome_aln: np.ndarray  # uint8


def align_host(b: Batch, lane: int = 0, first_of_call: bool = True,
               out: AlignResult | None = None) -> AlignResult:
    """Host arrays in, host arrays out (saru_align_host)."""
    lib = load()
    sb, keep = host_batch(b, first_of_call)
    tot = b.total_genome
    if out is None:
        out = AlignResult(np.zeros(max(b.n, 1), np.int32), np.zeros(tot + 64, np.uint8),
                          np.zeros(tot + 64, np.uint8))
    res = SaruResult(_p(out.scores), _p(out.read_aln), _p(out.genome_aln), None)
    rc = lib.saru_align_host(C.byref(sb), C.byref(res), lane)
    if rc != SARU_OK:
        raise SaruError(rc, last_error())
    return AlignResult(out.scores[:b.n], out.read_aln[:tot], out.genome_aln[:tot])


def align_host_compact(b: Batch, lane: int = 0, first_of_call: bool = True,
                       out: tuple | None = None) -> tuple[np.ndarray, np.ndarray, int]:
    """Host arrays in, (scores, compact records, record bytes) out
    (saru_align_host_compact); `out` = (scores, records) to fill."""
    lib = load()
    sb, keep = host_batch(b, first_of_call)
    rb = compact_record_bytes(b.m, b.k)
    if out is None:
        out = (np.zeros(max(b.n, 1), np.int32), np.zeros(max(b.n, 1) * rb, np.uint8))
    rc = lib.saru_align_host_compact(C.byref(sb), _p(out[0]), _p(out[1]), rb, lane)
    if rc != SARU_OK:
        raise SaruError(rc, last_error())
    return out[0][:b.n], out[1][:b.n * rb], rb


def scratch_bytes(n: int, max_m: int, k: int) -> int:
    return int(load().saru_scratch_bytes(n, max_m, k, 1 if k > 7 else 0))


def align_device(batch: SaruBatch, result: SaruResult, scratch_ptr: int, scratch_len: int,
                 stream_ptr: int = 0) -> None:
    """Device pointers in and out, enqueued on a stream (saru_align_device)."""
    rc = load().saru_align_device(C.byref(batch), C.byref(result), scratch_ptr, scratch_len,
                                  stream_ptr)
    if rc != SARU_OK:
        raise SaruError(rc, last_error())


def name_table(names: dict[int, bytes] | list[bytes], stride: int = 60) -> np.ndarray:
    if isinstance(names, dict):
        n = max(names) + 1 if names else 1
        items = names.items()
    else:
        n = max(len(names), 1)
        items = enumerate(names)
    tab = np.zeros((n, stride), np.uint8)
    for i, nm in items:
        raw = nm[:stride - 1]
        tab[i, :len(raw)] = np.frombuffer(raw, np.uint8)
    return tab


def format_tsv(b: Batch, r: AlignResult, names: np.ndarray, read_length: int | None = None,
               first_of_call: bool = True) -> tuple[bytes, int, int]:
    """The reference writer's TSV for an aligned call (saru_format_tsv):
    (text, forward alignments, reverse alignments)."""
    lib = load()
    sb, keep = host_batch(b, first_of_call)
    scores = np.ascontiguousarray(r.scores, np.int32)
    ra = np.concatenate([np.ascontiguousarray(r.read_aln, np.uint8), np.zeros(64, np.uint8)])
    ga = np.concatenate([np.ascontiguousarray(r.genome_aln, np.uint8), np.zeros(64, np.uint8)])
    res = SaruResult(_p(scores), _p(ra), _p(ga), None)
    ids = np.ascontiguousarray(b.ids, np.int32)
    pos = np.ascontiguousarray(b.pos, np.int32)
    rl = b.m if read_length is None else read_length
    df, dr = C.c_int32(), C.c_int32()
    args = [C.byref(sb), C.byref(res), C.c_void_p(_p(ids)), C.c_void_p(_p(pos)), C.c_int32(rl),
            C.c_void_p(_p(names)), C.c_int32(names.shape[1]), C.c_int32(names.shape[0])]
    need = lib.saru_format_tsv(*args, None, C.c_int64(0), C.byref(df), C.byref(dr))
    buf = np.zeros(need + 1, np.uint8)
    lib.saru_format_tsv(*args, C.c_void_p(_p(buf)), C.c_int64(need + 1), C.byref(df), C.byref(dr))
    return buf[:need].tobytes(), df.value, dr.value


def kernel_launches() -> int:
    return int(load().saru_kernel_launches())


def int32_issue_peak(iters: int = 4096) -> float:
    """Measured 32-bit integer ops/s of the current GPU (see probe.cu)."""
    return float(load().saru_int32_issue_probe(iters))


def align_multi_device(batches: list[SaruBatch], results: list[SaruResult], status_ptr: int,
                       scratch_ptr: int, scratch_len: int, stream_ptr: int = 0) -> None:
    """Several calls (device pointers) in one launch (saru_align_multi_device)."""
    n = len(batches)
    arr_b = (SaruBatch * n)(*batches)
    arr_r = (SaruResult * n)(*results)
    rc = load().saru_align_multi_device(arr_b, arr_r, n, status_ptr, scratch_ptr, scratch_len,
                                        stream_ptr)
    if rc != SARU_OK:
        raise SaruError(rc, last_error())


def align_multi_device_compact(batches: list[SaruBatch], results: list[SaruResult],
                               status_ptr: int, scratch_ptr: int, scratch_len: int,
                               stream_ptr: int = 0) -> None:
    """saru_align_multi_device with compact records: results[i].read_aln is
    call i's records array (device)."""
    n = len(batches)
    rc = load().saru_align_multi_device_compact((SaruBatch * n)(*batches),
                                                (SaruResult * n)(*results), n, status_ptr,
                                                scratch_ptr, scratch_len, stream_ptr)
    if rc != SARU_OK:
        raise SaruError(rc, last_error())


def multi_scratch_bytes(batches: list[SaruBatch]) -> int:
    n = len(batches)
    return int(load().saru_multi_scratch_bytes((SaruBatch * n)(*batches), n))


class HostRequest:
    """Host arrays of one request for the server: the inputs of each call
    (copied from Batch objects) and output arrays of the reference layout.
    `alloc(nbytes)` gives the uint8 host buffers (pinned ones let the
    server's copies overlap its kernels); numpy by default."""

    def __init__(self, batches: list[Batch], first_of_call: list[bool] | None = None,
                 alloc=None, compact: bool = False):
        alloc = alloc or (lambda nbytes: np.zeros(nbytes, np.uint8))
        first = first_of_call or [True] * len(batches)
        self.compact = compact
        self.first = first

        def host(a: np.ndarray, dtype) -> np.ndarray:
            a = np.ascontiguousarray(a, dtype)
            buf = alloc(max(a.nbytes, 1)).view(np.uint8)[:max(a.nbytes, 1)]
            buf[:a.nbytes] = a.view(np.uint8).reshape(-1)
            return buf[:a.nbytes].view(dtype) if a.nbytes else buf[:0].view(dtype)

        self.batches = batches
        self.keep: list[np.ndarray] = []
        self.outs: list[AlignResult] = []
        calls, results = [], []
        for b, f in zip(batches, first):
            arrs = [host(b.genome, np.uint8), host(b.reads, np.uint8),
                    host(b.genome_offsets, np.int32), host(b.read_offsets, np.int32),
                    host(b.dirs, np.int8)]
            self.keep += arrs
            calls.append(SaruBatch(*[_p(a) if a.size else 0 for a in arrs], b.n, b.k, b.match,
                                   b.mismatch, 1 if f else 0, b.m, len(b.genome),
                                   b.total_genome))
            if compact:  # records in read_aln, genome_aln unused
                nrec = max(b.n, 1) * compact_record_bytes(b.m, b.k)
                out = AlignResult(alloc(4 * max(b.n, 1)).view(np.int32)[:max(b.n, 1)],
                                  alloc(nrec)[:nrec], np.zeros(0, np.uint8))
            else:
                out = AlignResult(alloc(4 * max(b.n, 1)).view(np.int32)[:max(b.n, 1)],
                                  alloc(b.total_genome + 64)[:b.total_genome + 64],
                                  alloc(b.total_genome + 64)[:b.total_genome + 64])
            self.outs.append(out)
            results.append(SaruResult(_p(out.scores), _p(out.read_aln),
                                      _p(out.genome_aln) if out.genome_aln.size else 0, None))
        n = len(batches)
        self.calls = (SaruBatch * n)(*calls)
        self.results = (SaruResult * n)(*results)
        self.req = SaruRequest(self.calls, self.results, n, None, 1 if compact else 0)

    def result(self, i: int) -> AlignResult:
        """Call i's scores and slot strings (compact records are expanded)."""
        b, o = self.batches[i], self.outs[i]
        if self.compact:
            return expand_compact(b, o.scores[:b.n], o.read_aln, compact_record_bytes(b.m, b.k),
                                  first_of_call=self.first[i])
        return AlignResult(o.scores[:b.n], o.read_aln[:b.total_genome],
                           o.genome_aln[:b.total_genome])


class GatherRequest(HostRequest):
    """A request of gather calls: per call the read table (reads as
    sequenced, `table` rows of m bytes) and per candidate its read's row,
    window start and flag; the server gathers windows and reads from its
    resident genome.  `batches` give the call shapes and the expected
    layout (their genome/reads arrays are not sent)."""

    def __init__(self, batches: list[Batch], tables: list[np.ndarray],
                 first_of_call: list[bool] | None = None, compact: bool = False):
        super().__init__(batches, first_of_call, compact=compact)
        first = first_of_call or [True] * len(batches)
        gcs = []
        for b, tab, f in zip(batches, tables, first):
            arrs = [np.ascontiguousarray(tab, np.uint8).reshape(-1),
                    np.ascontiguousarray(b.ids, np.int32), np.ascontiguousarray(b.pos, np.int32),
                    np.ascontiguousarray(b.dirs, np.int8),
                    np.ascontiguousarray(b.genome_offsets, np.int32)]
            self.keep += arrs
            gcs.append(SaruGatherCall(*[_p(a) if a.size else 0 for a in arrs], b.n,
                                      int(arrs[0].size // max(b.m, 1)), b.k, b.match, b.mismatch,
                                      1 if f else 0, b.m, len(b.genome), b.total_genome))
        n = len(batches)
        self.gcalls = (SaruGatherCall * n)(*gcs)
        self.req.gather = C.cast(self.gcalls, C.POINTER(SaruGatherCall))


def gather_device(call: SaruGatherCall, genome_ptr: int, genome_len: int, windows_ptr: int,
                  reads_ptr: int, read_offsets_ptr: int, status_ptr: int,
                  stream_ptr: int = 0) -> SaruBatch:
    """Windows and reads of a gather call built on the device
    (saru_gather_device); returns the saru_batch that views them."""
    out = SaruBatch()
    rc = load().saru_gather_device(C.byref(call), genome_ptr, genome_len, windows_ptr, reads_ptr,
                                   read_offsets_ptr, status_ptr, C.byref(out), stream_ptr)
    if rc != SARU_OK:
        raise SaruError(rc, last_error())
    return out


class Server:
    """Continuous-batching request server on one GPU (saru_server_*)."""

    def __init__(self, device: int = 0, pipeline: bool = True, max_requests_per_launch: int = 64,
                 max_inflight: int = 2, budget_bytes: int = 8 << 30, host_pool_bytes: int = 0):
        self._lib = load()
        cfg = ServerConfig(device, 1 if pipeline else 0, max_requests_per_launch, max_inflight,
                           budget_bytes, host_pool_bytes)
        self._h = self._lib.saru_server_create(C.byref(cfg))
        if not self._h:
            raise SaruError(SARU_E_CUDA, last_error())
        self._live: dict[int, HostRequest] = {}
        self._keep: dict[int, tuple] = {}  # reads-only requests' read arrays

    def set_genome(self, genome: np.ndarray) -> None:
        g = np.ascontiguousarray(genome, np.uint8)
        rc = self._lib.saru_server_set_genome(self._h, _p(g), g.size)
        if rc != SARU_OK:
            raise SaruError(rc, last_error())

    def submit(self, req: HostRequest) -> int:
        t = C.c_int64()
        rc = self._lib.saru_server_submit(self._h, C.byref(req.req), C.byref(t))
        if rc != SARU_OK:
            raise SaruError(rc, last_error())
        self._live[t.value] = req
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 600_000) -> tuple[int, RequestStats]:
        """(status code, stats) once the request is done; raises TimeoutError."""
        st = RequestStats()
        rc = self._lib.saru_server_wait(self._h, ticket, timeout_ms, C.byref(st))
        if rc == SARU_E_TIMEOUT:
            raise TimeoutError(f"request {ticket} not done after {timeout_ms} ms")
        self._live.pop(ticket, None)
        return rc, st

    def submit_reads(self, sets: list, compact: bool = False) -> int:
        """Queues a reads-only request: `sets` = [(reads (n, m) uint8 as
        sequenced, k, chunk_value or 0), ...].  The read arrays must stay
        alive until the request is waited for (they are kept on the ticket)."""
        arr = (SaruReadSet * len(sets))()
        keep = []
        for i, (reads, k, cv) in enumerate(sets):
            r = np.ascontiguousarray(reads, np.uint8)
            keep.append(r)
            arr[i] = SaruReadSet(_p(r) if r.size else 0, r.shape[0], r.shape[1], k, cv)
        t = C.c_int64()
        rc = self._lib.saru_server_submit_reads(self._h, arr, len(sets), 1 if compact else 0,
                                                C.byref(t))
        if rc != SARU_OK:
            raise SaruError(rc, last_error())
        self._keep[t.value] = (arr, keep)
        return t.value

    def read_results(self, ticket: int, s: int) -> dict:
        """Copies of set s's results of a finished reads-only request."""
        out = SaruReadResults()
        rc = self._lib.saru_server_read_results(self._h, ticket, s, C.byref(out))
        if rc != SARU_OK:
            raise SaruError(rc, last_error())

        def arr(ptr, n, dt):
            if n == 0 or not ptr:
                return np.zeros(0, dt)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dt))),
                                         shape=(n,)).copy()

        nc, n, npf = out.ncalls, out.n, out.nperfect
        slot_begin = arr(out.slot_begin, nc + 1, np.int64)
        tot = int(slot_begin[-1]) if nc else 0
        res = dict(call_begin=arr(out.call_begin, nc + 1, np.int64), slot_begin=slot_begin,
                   call_strand=arr(out.call_strand, nc, np.int8), ids=arr(out.ids, n, np.int32),
                   pos=arr(out.pos, n, np.int32), dirs=arr(out.dirs, n, np.int8),
                   scores=arr(out.scores, n, np.int32),
                   perfect_ids=arr(out.perfect_ids, npf, np.int32),
                   perfect_pos=arr(out.perfect_pos, npf, np.int32),
                   perfect_strand=arr(out.perfect_strand, npf, np.int8),
                   record_bytes=int(out.record_bytes))
        if out.records:
            res["records"] = arr(out.records, n * int(out.record_bytes), np.uint8)
        else:
            res["read_aln"] = arr(out.read_aln, tot, np.uint8)
            res["genome_aln"] = arr(out.genome_aln, tot, np.uint8)
        return res

    def release(self, ticket: int) -> None:
        self._lib.saru_server_release(self._h, ticket)
        self._keep.pop(ticket, None)

    def candidates(self, ticket: int) -> int:
        """Candidates the filter made for a finished reads-only request (all
        sets), without copying its results."""
        out = SaruReadResults()
        n = 0
        for i in range(len(self._keep.get(ticket, ((), []))[1])):
            if self._lib.saru_server_read_results(self._h, ticket, i, C.byref(out)) != SARU_OK:
                raise SaruError(SARU_E_INVALID, last_error())
            n += int(out.n)
        return n

    def counters(self) -> tuple[int, int]:
        g, l_ = C.c_int64(), C.c_int64()
        self._lib.saru_server_counters(self._h, C.byref(g), C.byref(l_))
        return g.value, l_.value

    def close(self) -> None:
        if self._h:
            self._lib.saru_server_destroy(self._h)
            self._h = None
            self._live.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def set_tuning(m: int, k: int, warps: int = 0, ctas_per_sm: int = 0, word_bits: int = 0) -> None:
    """Launch shape of the banded kernel for (read length, k) (saru_tuning_set)."""
    t = SaruTuning(warps, ctas_per_sm, word_bits)
    rc = load().saru_tuning_set(m, k, C.byref(t))
    if rc != SARU_OK:
        raise SaruError(rc, last_error())


def clear_tuning(m: int | None = None, k: int | None = None) -> None:
    if m is None:
        load().saru_tuning_clear()
    else:
        load().saru_tuning_set(m, k, None)


def get_tuning(m: int, k: int) -> tuple[int, int, int] | None:
    t = SaruTuning()
    if load().saru_tuning_get(m, k, C.byref(t)):
        return (t.warps_per_cta, t.ctas_per_sm, t.word_bits)
    return None


def compact_record_bytes(m: int, k: int) -> int:
    return int(load().saru_compact_record_bytes(m, k))


def align_device_compact(batch: SaruBatch, scores_ptr: int, records_ptr: int, record_bytes: int,
                         status_ptr: int, scratch_ptr: int, scratch_len: int,
                         stream_ptr: int = 0) -> None:
    """Device pointers; compact records instead of slot strings."""
    rc = load().saru_align_device_compact(C.byref(batch), scores_ptr, records_ptr, record_bytes,
                                          status_ptr, scratch_ptr, scratch_len, stream_ptr)
    if rc != SARU_OK:
        raise SaruError(rc, last_error())


def expand_compact(b: Batch, scores: np.ndarray, records: np.ndarray, record_bytes: int,
                   nthreads: int = 0, first_of_call: bool = True) -> AlignResult:
    """The reference slot strings rebuilt on the host from compact records."""
    sb, keep = host_batch(b, first_of_call)
    tot = b.total_genome
    ra = np.zeros(tot + 64, np.uint8)
    ga = np.zeros(tot + 64, np.uint8)
    sc = np.ascontiguousarray(scores, np.int32)
    rec = np.ascontiguousarray(records, np.uint8)
    rc = load().saru_expand_compact(C.byref(sb), _p(sc), _p(rec), record_bytes, _p(ra), _p(ga),
                                    nthreads)
    if rc != SARU_OK:
        raise SaruError(rc, last_error())
    return AlignResult(sc[:b.n], ra[:tot], ga[:tot])


def format_tsv_compact(b: Batch, scores: np.ndarray, records: np.ndarray, record_bytes: int,
                       names: np.ndarray, read_length: int | None = None,
                       first_of_call: bool = True, nthreads: int = 0) -> tuple[bytes, int, int]:
    """The reference writer's TSV straight from compact records
    (saru_format_tsv_compact): (text, forward alignments, reverse alignments)."""
    lib = load()
    sb, keep = host_batch(b, first_of_call)
    sc = np.ascontiguousarray(scores, np.int32)
    rec = np.ascontiguousarray(records, np.uint8)
    ids = np.ascontiguousarray(b.ids, np.int32)
    pos = np.ascontiguousarray(b.pos, np.int32)
    rl = b.m if read_length is None else read_length
    df, dr = C.c_int32(), C.c_int32()
    est = int((sc <= b.k).sum()) * (names.shape[1] + 2 * (b.m + 3 * b.k) + 64) + 64
    buf = np.zeros(est, np.uint8)
    need = lib.saru_format_tsv_compact(C.byref(sb), _p(sc), _p(rec), record_bytes, _p(ids),
                                       _p(pos), rl, _p(names), names.shape[1], names.shape[0],
                                       _p(buf), est, C.byref(df), C.byref(dr), nthreads)
    if need < 0:
        raise SaruError(SARU_E_INVALID, last_error())
    if need > est:  # the estimate was short: once more with the exact size
        buf = np.zeros(need, np.uint8)
        lib.saru_format_tsv_compact(C.byref(sb), _p(sc), _p(rec), record_bytes, _p(ids), _p(pos),
                                    rl, _p(names), names.shape[1], names.shape[0], _p(buf), need,
                                    C.byref(df), C.byref(dr), nthreads)
    return buf[:need].tobytes(), df.value, dr.value


@dataclasses.dataclass
class FilterCalls:
    """One strand's calls as the reference would submit them: call c holds
    candidates call_begin[c]..call_begin[c+1] (ids, pos, dirs); perfect hits
    (read id, 0-based start) are printed by the filter, not aligned."""
    call_begin: np.ndarray
    ids: np.ndarray
    pos: np.ndarray
    dirs: np.ndarray
    perfect_ids: np.ndarray
    perfect_pos: np.ndarray
    ms: float

    def call(self, genome: np.ndarray, reads: np.ndarray, m: int, k: int, c: int,
             offset: int = 0) -> Batch:
        """Call c in the reference's call layout (windows cut from the genome
        -- a chunk starting at genome position `offset` --, reads
        reverse-complemented for flags 4-7; pos stays the genome position)."""
        from .workloads import flank, make_batch, reverse_complement
        lo, hi = int(self.call_begin[c]), int(self.call_begin[c + 1])
        ids, pos, dirs = self.ids[lo:hi], self.pos[lo:hi], self.dirs[lo:hi]
        wins = []
        for p, d in zip(pos, dirs):
            so, eo = flank(int(d), k)
            at = int(p) - offset
            wins.append(genome[at:at + m + so + eo])
        rd = reads[ids].copy()
        rev = dirs > 3
        if rev.any():
            rd[rev] = reverse_complement(rd[rev])
        return make_batch(m, k, wins, rd, dirs, ids=ids, pos=pos)


class Filter:
    """The reference's q-gram pair filter on the device (saru_filter_*)."""

    def __init__(self, genome: np.ndarray, m: int, k: int, device: int = -1):
        """device -1: the calling thread's current CUDA device."""
        self._lib = load()
        g = np.ascontiguousarray(genome, np.uint8)
        self.m, self.k = m, k
        self._h = self._lib.saru_filter_create(_p(g), g.size, m, k, device)
        if not self._h:
            raise SaruError(SARU_E_INVALID, last_error())

    def set_chunk(self, offset: int, limit: int) -> None:
        """The genome as a chunk at genome position `offset`; windows must end
        by `limit` (saru_filter_set_chunk)."""
        rc = self._lib.saru_filter_set_chunk(self._h, offset, limit)
        if rc != SARU_OK:
            raise SaruError(rc, last_error())

    def run(self, reads: np.ndarray, do_reverse: int, chunk_value: int) -> FilterCalls:
        """One batch of reads (ids from 0), one strand (do_reverse 0 or 4)."""
        r = np.ascontiguousarray(reads, np.uint8).reshape(-1)
        n = r.size // self.m
        cnt = np.zeros(3, np.int64)
        rc = self._lib.saru_filter_run(self._h, _p(r) if r.size else 0, n, do_reverse,
                                       chunk_value, _p(cnt))
        if rc != SARU_OK:
            raise SaruError(rc, last_error())
        nc, na, npf = (int(x) for x in cnt)
        out = FilterCalls(np.zeros(nc + 1, np.int64), np.zeros(na, np.int32),
                          np.zeros(na, np.int32), np.zeros(na, np.int8),
                          np.zeros(npf, np.int32), np.zeros(npf, np.int32),
                          float(self._lib.saru_filter_last_ms(self._h)))
        self._lib.saru_filter_results(self._h, *[_p(a) if a.size else 0 for a in
                                                 (out.call_begin, out.ids, out.pos, out.dirs,
                                                  out.perfect_ids, out.perfect_pos)])
        return out

    def close(self) -> None:
        if self._h:
            self._lib.saru_filter_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


@dataclasses.dataclass
class ReadBatch:
    """One batch of reads as the reference's reader leaves it."""
    reads: np.ndarray   # uint8 (n, read_length), upper-case
    names: list         # bytes, one per read (read id = index)
    records: int        # records of the file this batch consumed (kept + dropped)


def read_batches(path, read_length: int, max_n: int, batch: int, fastq: bool = False):
    """Yields the reference's read batches of a FASTA/FASTQ file
    (saru_reads_*): up to `batch` records each, reads with more than `max_n`
    Ns or shorter than read_length dropped.  Like the reference, a batch
    whose records were all dropped is followed by the next one, and the
    batches stop after the first one that did not fill `batch` records."""
    lib = load()
    h = lib.saru_reads_open(str(path).encode(), 1 if fastq else 0, read_length, max_n)
    if not h:
        raise SaruError(SARU_E_INVALID, last_error())
    try:
        reads = np.zeros((batch, read_length), np.uint8)
        names = np.zeros((batch, 60), np.uint8)
        skipped = C.c_int32(0)
        while True:
            n = lib.saru_reads_next(h, batch, reads.ctypes.data, names.ctypes.data,
                                    C.byref(skipped))
            if n < 0:
                raise SaruError(SARU_E_INVALID, last_error())
            records = n + skipped.value
            if records == 0:
                return
            if n > 0:
                nm = [bytes(names[i]).split(b"\0", 1)[0] for i in range(n)]
                yield ReadBatch(reads[:n].copy(), nm, records)
            if records < batch:
                return
    finally:
        lib.saru_reads_close(h)


@dataclasses.dataclass
class GenomeChunk:
    """One genome chunk as the reference's chunk loop leaves it."""
    seq: np.ndarray  # uint8: the chunk's bases and its overhang
    offset: int      # genome position of seq[0]
    bases: int       # the chunk's own bases (without the overhang)
    total: int       # bases of all chunks so far: windows must end by it


def genome_chunks(path, chunk_value: int, read_length: int):
    """Yields the reference's genome chunks of a FASTA file (saru_genome_*)."""
    lib = load()
    h = lib.saru_genome_open(str(path).encode(), chunk_value, read_length)
    if not h:
        raise SaruError(SARU_E_INVALID, last_error())
    try:
        out = np.zeros(chunk_value + read_length + 1, np.uint8)
        ln, bases, total = C.c_int64(0), C.c_int64(0), C.c_int64(0)
        run = 0
        while True:
            rc = lib.saru_genome_next(h, out.ctypes.data, C.byref(ln), C.byref(bases),
                                      C.byref(total))
            if rc < 0:
                raise SaruError(SARU_E_INVALID, last_error())
            if rc == 0:
                return
            yield GenomeChunk(out[:ln.value].copy(), run * chunk_value, bases.value, total.value)
            run += 1
    finally:
        lib.saru_genome_close(h)
