"""ctypes bindings of the oracle build (oracle/_ref) for the tests.

Test infrastructure only.  Two checkers are exposed:

* `oracle_*`   our host C restatement (oracle/saru_oracle.c), always built;
* `ref_*`      the reference's own src/cuda-functions.cu compiled for the host
               (oracle/_ref/libref_emul.so), present only where the reference
               sources were available when the oracle was built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
from saruman_b200.workloads import Batch  # noqa: E402

REF_DIR = ROOT / "oracle" / "_ref"
NAME_STRIDE = 60


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True,
                   stdout=subprocess.DEVNULL)


def _ptr(a: np.ndarray, t=C.c_void_p):
    return C.cast(a.ctypes.data, t)


_oracle = None
_ref = None


def oracle_lib():
    global _oracle
    if _oracle is None:
        p = REF_DIR / "libsaru_oracle.so"
        if not p.exists():
            build_oracle()
        _oracle = C.CDLL(str(p))
        _oracle.saru_oracle_align.restype = C.c_int
        _oracle.saru_oracle_write_tsv.restype = C.c_long
    return _oracle


def have_ref() -> bool:
    return (REF_DIR / "libref_emul.so").exists()


def ref_lib():
    global _ref
    if _ref is None:
        _ref = C.CDLL(str(REF_DIR / "libref_emul.so"))
        _ref.ref_align_batch.restype = C.c_int
    return _ref


def _outputs(b: Batch):
    tot = b.total_genome
    return (np.zeros(max(b.n, 1), np.int32), np.zeros(tot + 1, np.uint8),
            np.zeros(tot + 1, np.uint8))


def oracle_align(b: Batch, nthreads: int = 1):
    lib = oracle_lib()
    sc, ra, ga = _outputs(b)
    st = lib.saru_oracle_align(
        C.c_int(b.match), C.c_int(b.mismatch), _ptr(b.genome), C.c_long(len(b.genome)),
        _ptr(b.reads), C.c_long(len(b.reads)), _ptr(b.genome_offsets), _ptr(b.read_offsets),
        _ptr(b.edit_offsets), C.c_int(b.n), _ptr(b.dirs), C.c_int(b.k), C.c_int(nthreads),
        _ptr(sc), _ptr(ra), _ptr(ga))
    tot = b.total_genome
    return sc[:b.n], ra[:tot], ga[:tot], st


def oracle_check(b: Batch, scores, read_aln, genome_aln, nthreads: int | None = None):
    """Checks another implementation's outputs for the whole call `b` (any
    size) against the oracle, in sub-calls led by their predecessor
    (saru_oracle_check).  Returns (candidates that differ, lowest such
    index or -1, oracle status bits)."""
    lib = oracle_lib()
    lib.saru_oracle_check.restype = C.c_long
    go = np.ascontiguousarray(b.genome_offsets, np.int64)
    ro = np.ascontiguousarray(b.read_offsets, np.int64)
    sc = np.ascontiguousarray(scores, np.int32)
    ra = np.ascontiguousarray(read_aln, np.uint8)
    ga = np.ascontiguousarray(genome_aln, np.uint8)
    assert len(sc) >= b.n and len(ra) >= b.total_genome and len(ga) >= b.total_genome
    first, st = C.c_long(-1), C.c_int(0)
    bad = lib.saru_oracle_check(
        C.c_int(b.match), C.c_int(b.mismatch), _ptr(b.genome), _ptr(b.reads), _ptr(go), _ptr(ro),
        C.c_long(b.n), _ptr(b.dirs), C.c_int(b.k), C.c_int(nthreads or os.cpu_count() or 1),
        _ptr(sc), _ptr(ra), _ptr(ga), C.byref(first), C.byref(st))
    return int(bad), int(first.value), int(st.value)


def ref_align(b: Batch, strict: bool = True, nthreads: int = 1, chunk: int = 512):
    lib = ref_lib()
    sc, ra, ga = _outputs(b)
    rc = lib.ref_align_batch(
        C.c_int(b.match), C.c_int(b.mismatch), _ptr(b.genome), _ptr(b.reads),
        _ptr(b.genome_offsets), _ptr(b.read_offsets), _ptr(b.edit_offsets), C.c_int(b.n),
        _ptr(b.dirs), C.c_int(b.k), C.c_size_t(b.total_genome), C.c_int(1 if strict else 0),
        C.c_int(nthreads), C.c_int(chunk), _ptr(sc), _ptr(ra), _ptr(ga))
    assert rc == 0
    tot = b.total_genome
    return sc[:b.n], ra[:tot], ga[:tot]


def name_table(names_by_id: dict[int, bytes] | list[bytes]) -> np.ndarray:
    if isinstance(names_by_id, dict):
        n = max(names_by_id) + 1 if names_by_id else 0
        items = names_by_id.items()
    else:
        n = len(names_by_id)
        items = enumerate(names_by_id)
    tab = np.zeros((max(n, 1), NAME_STRIDE), np.uint8)
    for i, nm in items:
        raw = nm[:NAME_STRIDE - 1]
        tab[i, :len(raw)] = np.frombuffer(raw, np.uint8)
    return tab


def oracle_tsv(b: Batch, scores, ra, ga, names: np.ndarray, read_length: int | None = None):
    """TSV bytes the reference writer prints for this call, plus the status
    bits and the (forward, reverse) alignment counts."""
    lib = oracle_lib()
    rl = b.m if read_length is None else read_length
    scores = np.ascontiguousarray(scores, np.int32)
    ra = np.ascontiguousarray(ra, np.uint8)
    ga = np.ascontiguousarray(ga, np.uint8)
    st, df, dr = C.c_int(), C.c_int(), C.c_int()
    args = [_ptr(scores), _ptr(ra), _ptr(ga), C.c_long(len(ra)), _ptr(b.genome_offsets),
            _ptr(b.pos), _ptr(b.dirs), _ptr(b.ids), C.c_int(b.n), C.c_int(b.k), C.c_int(rl),
            _ptr(names), C.c_int(NAME_STRIDE), C.c_int(names.shape[0])]
    need = lib.saru_oracle_write_tsv(*args, None, C.c_long(0), C.byref(st), C.byref(df),
                                     C.byref(dr))
    out = np.zeros(need + 1, np.uint8)
    lib.saru_oracle_write_tsv(*args, _ptr(out), C.c_long(need + 1), C.byref(st), C.byref(df),
                              C.byref(dr))
    return out[:need].tobytes(), st.value, (df.value, dr.value)


_REF_TSV_SCRIPT = r"""
import ctypes as C, sys, numpy as np
sys.path.insert(0, {tests!r})
from nwbio import read_nwb
b, names, do_rev, m = read_nwb({path!r})
lib = C.CDLL({lib!r})
P = lambda a: C.cast(a.ctypes.data, C.c_void_p)
n_ids = int(b.ids.max()) + 1 if b.n else 1
tab = np.zeros((n_ids, 60), np.uint8)
for i, nm in zip(b.ids, names):
    tab[i, :len(nm)] = np.frombuffer(nm, np.uint8)
lib.ref_set_read_length(C.c_int(m))
lib.ref_set_read_names(C.c_int(n_ids), P(tab), C.c_int(60))
lib.ref_alloc_output_control(C.c_int(n_ids))
need = b.total_edit * 2 + b.total_genome * 3 + b.n * 32 + (1 << 20)
lib.ref_set_memory_per_thread(C.c_ulong(need))
lib.cuda_allocate_memory(C.c_int(4 if do_rev else 0))
lib.cuda_needleman_wunsch(C.c_int(b.match), C.c_int(b.mismatch), P(b.genome), P(b.reads),
    P(b.genome_offsets), P(b.read_offsets), P(b.edit_offsets), C.c_int(b.n), P(b.ids), P(b.pos),
    P(b.dirs), C.c_int(b.k), C.c_size_t(b.total_genome), C.c_size_t(b.n * b.m),
    C.c_size_t(b.total_edit), C.c_int(do_rev))
libc = C.CDLL(None)
libc.fflush(None)
"""


def ref_module_tsv(nwb_path: str) -> bytes:
    """Runs the reference's own cuda_needleman_wunsch (host-emulated) on a
    captured batch in a child process and returns what it printed."""
    code = _REF_TSV_SCRIPT.format(tests=str(ROOT / "tests"), path=str(nwb_path),
                                  lib=str(REF_DIR / "libref_emul.so"))
    env = dict(os.environ)
    env.pop("SARU_CAPTURE_DIR", None)
    r = subprocess.run([sys.executable, "-c", code], stdout=subprocess.PIPE,
                       stderr=subprocess.PIPE, env=env, check=True)
    return r.stdout


def write_temp_nwb(b: Batch, names: list[bytes], do_rev: int) -> str:
    from nwbio import write_nwb
    fd, path = tempfile.mkstemp(suffix=".nwb")
    os.close(fd)
    write_nwb(path, b, names, do_rev)
    return path
