"""ctypes wrapper of the CPU oracle (oracle/cosine_greedy_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU baseline / reference arm, never by the cudams package.
See cosine_greedy_oracle.c for what is restated and from where.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import c_double, c_float, c_int, c_int64, c_void_p
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_lib = None


def build(force: bool = False) -> Path:
    if force or not LIB.exists() or LIB.stat().st_mtime < (HERE / "cosine_greedy_oracle.c").stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def _load():
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIB))
        p = c_void_p
        lib.oracle_cosine_greedy.restype = c_int
        lib.oracle_cosine_greedy.argtypes = [p, p, p, p, c_int64, p, p, p, p, c_int64, c_double,
                                             c_double, c_int, c_int, p, p, p, c_int64, c_int]
        lib.oracle_cosine_greedy_pairs.restype = c_int
        lib.oracle_cosine_greedy_pairs.argtypes = [p, p, p, p, p, p, p, p, p, p, c_int64,
                                                   c_double, c_double, c_int, c_int, p, p, p,
                                                   c_int]
        lib.oracle_modified_cosine.restype = c_int
        lib.oracle_modified_cosine.argtypes = [p, p, p, p, p, c_int64, p, p, p, p, p, c_int64,
                                               c_double, c_int, p, p, p, c_int64, c_int]
        lib.oracle_fingerprint.restype = c_int
        lib.oracle_fingerprint.argtypes = [c_int, p, p, c_int64, p, p, c_int64, c_int, c_float,
                                           p, c_int64, c_int]
        _lib = lib
    return _lib


def _ptr(a):
    return c_void_p(0) if a is None else c_void_p(a.ctypes.data)


def _side(s):
    """(mz f32, a f64|None, b f64, offsets i64) from a packed spectrum set."""
    mz = np.ascontiguousarray(s.mz, dtype=np.float32)
    a = None if s.a is None else np.ascontiguousarray(s.a, dtype=np.float64)
    b = np.ascontiguousarray(s.b, dtype=np.float64)
    off = np.ascontiguousarray(s.offsets, dtype=np.int64)
    return mz, a, b, off


def cosine_greedy(ref, qry, tolerance: float, shift: float, match_limit: int,
                  key_mode: int = 0, threads: int = 0):
    """Dense (score f32, matches i32, overflow u8) [n_ref, n_q].

    key_mode 0: matchms float64 semantics; 1: the reference CUDA kernel's
    float32 keys and window test."""
    rm, ra, rb, ro = _side(ref)
    qm, qa, qb, qo = _side(qry)
    nr, nq = ro.shape[0] - 1, qo.shape[0] - 1
    score = np.zeros((nr, nq), np.float32)
    matches = np.zeros((nr, nq), np.int32)
    overflow = np.zeros((nr, nq), np.uint8)
    rc = _load().oracle_cosine_greedy(_ptr(rm), _ptr(ra), _ptr(rb), _ptr(ro), nr, _ptr(qm),
                                      _ptr(qa), _ptr(qb), _ptr(qo), nq, float(tolerance),
                                      float(shift), int(match_limit), int(key_mode),
                                      _ptr(score), _ptr(matches), _ptr(overflow), nq,
                                      int(threads))
    if rc != 0:
        raise RuntimeError("oracle_cosine_greedy failed")
    return score, matches, overflow


def modified_cosine(ref, qry, ref_precursor, qry_precursor, tolerance: float, match_limit: int,
                    threads: int = 0):
    """Dense modified cosine (score f32, matches i32, overflow u8) [n_ref, n_q]:
    matchms ModifiedCosine restated (see cosine_greedy_oracle.c), float64."""
    rm, ra, rb, ro = _side(ref)
    qm, qa, qb, qo = _side(qry)
    rp = np.ascontiguousarray(ref_precursor, dtype=np.float64)
    qp = np.ascontiguousarray(qry_precursor, dtype=np.float64)
    nr, nq = ro.shape[0] - 1, qo.shape[0] - 1
    if rp.shape[0] != nr or qp.shape[0] != nq:
        raise ValueError("one precursor m/z per spectrum")
    score = np.zeros((nr, nq), np.float32)
    matches = np.zeros((nr, nq), np.int32)
    overflow = np.zeros((nr, nq), np.uint8)
    rc = _load().oracle_modified_cosine(_ptr(rm), _ptr(ra), _ptr(rb), _ptr(ro), _ptr(rp), nr,
                                        _ptr(qm), _ptr(qa), _ptr(qb), _ptr(qo), _ptr(qp), nq,
                                        float(tolerance), int(match_limit), _ptr(score),
                                        _ptr(matches), _ptr(overflow), nq, int(threads))
    if rc != 0:
        raise RuntimeError("oracle_modified_cosine failed")
    return score, matches, overflow


def cosine_greedy_symmetric(ref, qry, tolerance: float, shift: float, match_limit: int,
                            key_mode: int = 0, threads: int = 0):
    """matchms is_symmetric=True (matchms>=0.24 BaseSimilarity.matrix, the
    pin of requirements.txt:1; the reference accepts and ignores the flag,
    CudaCosineGreedy.py:131-132): pair (i, j) with i <= j is scored as
    (references[i], queries[j]) and (j, i) receives the same result."""
    full = cosine_greedy(ref, qry, tolerance, shift, match_limit, key_mode, threads)
    n = full[0].shape[0]
    if full[0].shape[1] != n:
        raise ValueError("symmetric scoring needs as many queries as references")
    lower = np.tril_indices(n, -1)
    out = []
    for a in full:
        a = a.copy()
        a[lower] = a.T[lower]
        out.append(a)
    return tuple(out)


def cosine_greedy_pairs(ref, qry, pair_r, pair_q, tolerance: float, shift: float,
                        match_limit: int, key_mode: int = 0, threads: int = 0):
    rm, ra, rb, ro = _side(ref)
    qm, qa, qb, qo = _side(qry)
    pr = np.ascontiguousarray(pair_r, dtype=np.int64)
    pq = np.ascontiguousarray(pair_q, dtype=np.int64)
    n = pr.shape[0]
    score = np.zeros(n, np.float32)
    matches = np.zeros(n, np.int32)
    overflow = np.zeros(n, np.uint8)
    rc = _load().oracle_cosine_greedy_pairs(_ptr(rm), _ptr(ra), _ptr(rb), _ptr(ro), _ptr(qm),
                                            _ptr(qa), _ptr(qb), _ptr(qo), _ptr(pr), _ptr(pq), n,
                                            float(tolerance), float(shift), int(match_limit),
                                            int(key_mode), _ptr(score), _ptr(matches),
                                            _ptr(overflow), int(threads))
    if rc != 0:
        raise RuntimeError("oracle_cosine_greedy_pairs failed")
    return score, matches, overflow


MEASURES = {"jaccard": 0, "dice": 1, "cosine": 2}


def fingerprint(measure: str, r_bits, r_valid, q_bits, q_valid, n_words: int, fill: float,
                threads: int = 0) -> np.ndarray:
    rb = np.ascontiguousarray(r_bits, dtype=np.uint32)
    qb = np.ascontiguousarray(q_bits, dtype=np.uint32)
    rv = None if r_valid is None else np.ascontiguousarray(r_valid, dtype=np.uint8)
    qv = None if q_valid is None else np.ascontiguousarray(q_valid, dtype=np.uint8)
    nr, nq = rb.shape[0], qb.shape[0]
    out = np.zeros((nr, nq), np.float32)
    rc = _load().oracle_fingerprint(MEASURES[measure], _ptr(rb), _ptr(rv), nr, _ptr(qb), _ptr(qv),
                                    nq, int(n_words), float(fill), _ptr(out), nq, int(threads))
    if rc != 0:
        raise RuntimeError("oracle_fingerprint failed")
    return out


def available_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
