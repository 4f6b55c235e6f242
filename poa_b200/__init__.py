"""poa_b200 - B200-native partial-order alignment (minipoa's hot path).

The product is the native library ``libpoa_b200.so`` (CUDA kernels for
sm_100a + the host driver in C++, behind the C ABI in include/poa_b200.h).
This module is a thin ctypes mirror of that ABI for Python callers, tests
and the benchmark. It never falls back to a CPU implementation: if the
library is missing or no GPU is present, the calls raise.

Mirrors the reference's operator interface (minipoa, src/main.cpp):
``Params`` holds the CLI options with the same defaults, ``Context.run``
is one minipoa invocation (consensus by default, row-column MSA with
``result=1``), returning exactly the text minipoa prints.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import List, Optional, Sequence, Tuple

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpoa_b200.so")

STATUS = {
    0: "ok", 1: "backtrack left the band", 2: "backtrack error", 3: "bad argument",
    4: "out of device memory", 5: "node in-degree above 510 within one window",
    6: "degenerate band or sub-window", 7: "window outgrew its device capacity",
    8: "CUDA error", 9: "unsupported option",
}


class PoaError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        super().__init__(f"poa status {status} ({STATUS.get(status, '?')}){': ' + msg if msg else ''}")
        self.status = status


class _CParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in (
        "match", "mismatch", "gap_open", "gap_ext", "band_b", "band_f", "ab_band", "seeding",
        "k", "mm_w", "poa_w", "thread", "result", "progressive", "verbose")]


@dataclass
class Params:
    """minipoa's options (src/main.cpp:16-33) with the same defaults."""
    match: int = 2          # -M
    mismatch: int = -4      # -X
    gap_open: int = -4      # -O
    gap_ext: int = -2       # -E
    band_b: int = 100       # -b
    band_f: int = 40        # -f
    ab_band: bool = False   # -B
    seeding: bool = False   # -S
    k: int = 19             # -k
    mm_w: int = 10          # -w
    poa_w: int = 0          # -W (minipoa reads it only when given; 0 = unset)
    thread: int = 1         # -t
    result: int = 0         # -r (0 consensus, 1 MSA, 2 GFA)
    progressive: bool = False  # -p
    verbose: int = 0        # -V

    def _c(self) -> _CParams:
        return _CParams(*[int(getattr(self, f[0])) for f in _CParams._fields_])

    @classmethod
    def from_cli(cls, opts: Sequence[str]) -> "Params":
        """Parse minipoa-style short options (``-B -r 1 -M 3 ...``)."""
        keys = {"-M": "match", "-X": "mismatch", "-O": "gap_open", "-E": "gap_ext", "-b": "band_b",
                "-f": "band_f", "-k": "k", "-w": "mm_w", "-W": "poa_w", "-t": "thread", "-r": "result",
                "-V": "verbose"}
        flags = {"-B": "ab_band", "-S": "seeding", "-p": "progressive"}
        p = cls()
        it = iter(opts)
        for o in it:
            if o == "-i":
                next(it)  # the graph file: see Context.run_gfa
            elif o in flags:
                setattr(p, flags[o], True)
            elif o in keys:
                setattr(p, keys[o], int(next(it)))
            else:
                raise ValueError(f"unknown option {o}")
        return p


_lib = None


def lib() -> ctypes.CDLL:
    """Load the native library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m poa_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    L.poa_params_init.argtypes = [ctypes.POINTER(_CParams)]
    L.poa_create.restype = ctypes.c_void_p
    L.poa_create.argtypes = [ctypes.c_int, ctypes.POINTER(_CParams)]
    L.poa_destroy.argtypes = [ctypes.c_void_p]
    L.poa_last_error.restype = ctypes.c_char_p
    L.poa_last_error.argtypes = [ctypes.c_void_p]
    L.poa_status_str.restype = ctypes.c_char_p
    L.poa_free.argtypes = [ctypes.c_void_p]
    L.poa_run.restype = ctypes.c_int
    L.poa_run.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_char_p),
                          ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_char_p),
                          ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t),
                          ctypes.POINTER(ctypes.c_int32)]
    L.poa_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]
    L.poa_run_gfa.restype = ctypes.c_int
    L.poa_run_gfa.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int32,
                              ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_int32),
                              ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_void_p),
                              ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int32)]
    _i64p, _i32p, _u8p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32), ctypes.c_void_p
    L.poa_batch_upload.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_int64, _i64p, _i32p, ctypes.c_int32, _i32p,
                                   ctypes.c_int32]
    L.poa_batch_run.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
    L.poa_batch_download.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, _i64p, _i32p]
    L.poa_batch_consensus.argtypes = [ctypes.c_void_p, _u8p, ctypes.c_int64, _i64p, _i32p, ctypes.c_int32, _i32p,
                                      ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64, _i64p, _i32p]
    L.poa_batch_stats.argtypes = [ctypes.c_void_p, _i64p]
    L.poa_set_timing.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.poa_batch_config.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64]
    L.poa_batch_read_stats.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
    L.poa_batch_plan.argtypes = [ctypes.c_void_p] * 5
    L.poa_batch_plan_get.argtypes = [ctypes.c_void_p, _i32p, _i64p, _i64p, ctypes.c_int32]
    L.poa_prop_create.restype = ctypes.c_void_p
    L.poa_prop_create.argtypes = [ctypes.c_int]
    L.poa_prop_destroy.argtypes = [ctypes.c_void_p]
    L.poa_prop_last_error.restype = ctypes.c_char_p
    L.poa_prop_last_error.argtypes = [ctypes.c_void_p]
    L.poa_prop_set_weights.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.poa_prop_get_weights.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.poa_prop_train.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int32,
                                 ctypes.c_int32, ctypes.c_float, ctypes.c_uint64, ctypes.c_void_p]
    L.poa_prop_predict.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]
    L.poa_prop_gradient.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                    ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]
    L.poa_batch_features.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]
    L.poa_batch_propose.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.poa_batch_use_proposer.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.poa_alloc_pinned.restype = ctypes.c_void_p
    L.poa_alloc_pinned.argtypes = [ctypes.c_size_t]
    L.poa_free_pinned.argtypes = [ctypes.c_void_p]
    L.poa_int_peak.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_double)]
    L.poa_batch_consensus_files.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int32,
                                            ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int64, _i64p,
                                            _i32p]
    L.poa_batch_partition.argtypes = [_i32p, _i32p, ctypes.c_int32, ctypes.c_int32, _i32p, _i64p]
    L.poa_batch_consensus_multi.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int32, _u8p, ctypes.c_int64,
                                            _i64p, _i32p, ctypes.c_int32, _i32p, ctypes.c_int32, ctypes.c_void_p,
                                            ctypes.c_int64, _i64p, _i32p]
    _lib = L
    return L


class Context:
    """One device context (CUDA stream + device arena) with fixed options."""

    def __init__(self, params: Optional[Params] = None, device: int = 0):
        self.params = params or Params()
        L = lib()
        self._cp = self.params._c()
        self._h = L.poa_create(device, ctypes.byref(self._cp))
        if not self._h:
            raise PoaError(8, "poa_create failed (no CUDA device or out of memory)")

    def close(self):
        if getattr(self, "_h", None):
            lib().poa_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int):
        if st != 0:
            raise PoaError(st, lib().poa_last_error(self._h).decode(errors="replace"))

    def run(self, seqs: Sequence[bytes], headers: Optional[Sequence[str]] = None) -> Tuple[bytes, List[int]]:
        """One minipoa run over ``seqs``; returns (stdout text, per-read score)."""
        n = len(seqs)
        arr = (ctypes.c_char_p * n)(*[bytes(s) for s in seqs])
        lens = (ctypes.c_int32 * n)(*[len(s) for s in seqs])
        hdr = None
        if headers is not None:
            hdr = (ctypes.c_char_p * n)(*[h.encode() for h in headers])
        out = ctypes.c_void_p()
        olen = ctypes.c_size_t()
        scores = (ctypes.c_int32 * max(n, 1))()
        st = lib().poa_run(self._h, n, arr, lens, hdr, ctypes.byref(out), ctypes.byref(olen), scores)
        self._check(st)
        text = ctypes.string_at(out.value, olen.value)
        lib().poa_free(out)
        return text, list(scores)[:n]

    def run_gfa(self, gfa: bytes, seqs: Sequence[bytes], headers: Optional[Sequence[str]] = None):
        """minipoa -i: extend the graph in ``gfa`` (GFA text) with ``seqs``; returns (text, scores)."""
        n = len(seqs)
        arr = (ctypes.c_char_p * max(n, 1))(*[bytes(s) for s in seqs])
        lens = (ctypes.c_int32 * max(n, 1))(*[len(s) for s in seqs])
        hdr = None
        if headers is not None:
            hdr = (ctypes.c_char_p * max(n, 1))(*[h.encode() for h in headers])
        out = ctypes.c_void_p()
        olen = ctypes.c_size_t()
        scores = (ctypes.c_int32 * max(n, 1))()
        g = bytes(gfa)
        st = lib().poa_run_gfa(self._h, g, len(g), n, arr, lens, hdr, ctypes.byref(out), ctypes.byref(olen), scores)
        self._check(st)
        text = ctypes.string_at(out.value, olen.value)
        lib().poa_free(out)
        return text, list(scores)[:n]

    # ---- batched windows -------------------------------------------------
    @staticmethod
    def _win_arrays(ws):
        import numpy as np
        seq = np.ascontiguousarray(ws.seq, dtype=np.uint8)
        roff = np.ascontiguousarray(ws.read_off, dtype=np.int64)
        rlen = np.ascontiguousarray(ws.read_len, dtype=np.int32)
        woff = np.ascontiguousarray(ws.win_off, dtype=np.int32)
        return seq, roff, rlen, woff

    def batch_upload(self, ws) -> None:
        """Copy a synth.WindowSet-like batch (seq, read_off, read_len, win_off) to the device."""
        seq, roff, rlen, woff = self._keep = self._win_arrays(ws)
        i64p, i32p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
        st = lib().poa_batch_upload(self._h, seq.ctypes.data, seq.shape[0], roff.ctypes.data_as(i64p),
                                    rlen.ctypes.data_as(i32p), rlen.shape[0], woff.ctypes.data_as(i32p),
                                    woff.shape[0] - 1)
        self._check(st)
        self._nwin = int(woff.shape[0] - 1)
        self._cons_cap = int(2 * (int(rlen.max()) if rlen.shape[0] else 0) + 64) * max(self._nwin, 1)

    def batch_run(self) -> float:
        """Run every uploaded window on the device; returns the device time (ms)."""
        ms = ctypes.c_double()
        self._check(lib().poa_batch_run(self._h, ctypes.byref(ms)))
        return ms.value

    def batch_download(self):
        """(consensus bytes per window, status per window) of the last run."""
        import numpy as np
        cons = ctypes.create_string_buffer(max(self._cons_cap, 1))
        off = np.zeros(self._nwin + 1, dtype=np.int64)
        st = np.zeros(max(self._nwin, 1), dtype=np.int32)
        self._check(lib().poa_batch_download(self._h, cons, self._cons_cap,
                                             off.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                             st.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        raw = cons.raw
        return [raw[off[w]:off[w + 1]] for w in range(self._nwin)], [int(x) for x in st[:self._nwin]]

    def batch_consensus(self, ws):
        """Upload + run + download through poa_batch_consensus (host buffers in, host buffers out)."""
        import numpy as np
        seq, roff, rlen, woff = self._win_arrays(ws)
        nwin = int(woff.shape[0] - 1)
        cap = int(2 * (int(rlen.max()) if rlen.shape[0] else 0) + 64) * max(nwin, 1)
        cons = ctypes.create_string_buffer(max(cap, 1))
        off = np.zeros(nwin + 1, dtype=np.int64)
        st = np.zeros(max(nwin, 1), dtype=np.int32)
        i64p, i32p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
        self._check(lib().poa_batch_consensus(self._h, seq.ctypes.data, seq.shape[0], roff.ctypes.data_as(i64p),
                                              rlen.ctypes.data_as(i32p), rlen.shape[0], woff.ctypes.data_as(i32p),
                                              nwin, cons, cap, off.ctypes.data_as(i64p), st.ctypes.data_as(i32p)))
        self._nwin = nwin
        raw = cons.raw
        return [raw[off[w]:off[w + 1]] for w in range(nwin)], [int(x) for x in st[:nwin]]

    def batch_consensus_files(self, paths, chunk: int = 20000, threads: int = 0, cons_cap: int = 0):
        """Windows from FASTA / FASTQ files (one window per file, plain or gzip),
        parsed on host threads while the device runs the previous chunk
        (poa_batch_consensus_files). Returns (consensus bytes, status) per file."""
        import numpy as np
        n = len(paths)
        arr = (ctypes.c_char_p * max(n, 1))(*[os.fsencode(p) for p in paths])
        if cons_cap <= 0:
            # a consensus is never longer than its window's bases (<= the file, or ~10x a gzip file)
            cons_cap = sum(os.path.getsize(p) * (10 if str(p).endswith(".gz") else 1) + 64 for p in paths) + 4096
        cons = ctypes.create_string_buffer(max(cons_cap, 1))
        off = np.zeros(n + 1, dtype=np.int64)
        st = np.zeros(max(n, 1), dtype=np.int32)
        i64p, i32p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
        self._check(lib().poa_batch_consensus_files(self._h, arr, n, chunk, threads, cons, cons_cap,
                                                    off.ctypes.data_as(i64p), st.ctypes.data_as(i32p)))
        raw = cons.raw
        return [raw[off[w]:off[w + 1]] for w in range(n)], [int(x) for x in st[:n]]

    def batch_read_stats(self):
        """int32 array [n_reads, 8] of the last run: widest row (blocks), cells, rows,
        nodes after fusion, record bytes, spilled row-store entries, edges after fusion, 0."""
        import numpy as np
        n = int(self._keep[2].shape[0]) if getattr(self, "_keep", None) is not None else 0
        out = np.zeros((max(n, 1), 8), dtype=np.int32)
        self._check(lib().poa_batch_read_stats(self._h, out.ctypes.data, out.size))
        return out[:n]

    def batch_plan_get(self):
        """(nodes, record bytes, spilled entries) per window of the last planned run."""
        import numpy as np
        n = int(self._nwin)
        nodes = np.zeros(max(n, 1), dtype=np.int32)
        tb = np.zeros(max(n, 1), dtype=np.int64)
        sp = np.zeros(max(n, 1), dtype=np.int64)
        i64p, i32p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
        self._check(lib().poa_batch_plan_get(self._h, nodes.ctypes.data_as(i32p), tb.ctypes.data_as(i64p),
                                             sp.ctypes.data_as(i64p), n))
        return nodes[:n], tb[:n], sp[:n]

    def batch_features(self, prop: "Proposer"):
        """float32 [n_reads, 32, 8] proposer features of the uploaded windows."""
        import numpy as np
        n = int(self._keep[2].shape[0]) if getattr(self, "_keep", None) is not None else 0
        X = np.zeros((max(n, 1), PROP_BINS, PROP_CIN), dtype=np.float32)
        self._check(lib().poa_batch_features(self._h, prop._h, X.ctypes.data, X.size))
        return X[:n]

    def batch_use_proposer(self, prop: Optional["Proposer"]) -> None:
        """Plan every following batch run with ``prop`` (None: no proposer)."""
        self._prop = prop  # keep it alive while the engine may use it
        self._check(lib().poa_batch_use_proposer(self._h, prop._h if prop is not None else None))

    def batch_propose(self, prop: "Proposer") -> None:
        """Plan the uploaded windows' slots with the proposer (see poa_batch_propose)."""
        self._check(lib().poa_batch_propose(self._h, prop._h))

    def batch_autotuned(self, workload: str) -> Optional[dict]:
        """Apply the launch shape poa_b200.autotune recorded for ``workload`` (if any); returns it."""
        from poa_b200 import autotune
        t = autotune.load(workload)
        if t:
            self.batch_config(blocks_per_sm=t["blocks_per_sm"], smem_per_warp=t["smem_per_warp"])
        return t

    def batch_config(self, blocks_per_sm=None, max_blocks=None, smem_per_warp=None):
        """Launch shape of the batch kernel (see poa_batch_config)."""
        for key, val in ((0, blocks_per_sm), (1, max_blocks), (2, smem_per_warp)):
            if val is not None:
                self._check(lib().poa_batch_config(self._h, key, int(val)))

    def batch_stats(self) -> dict:
        o = (ctypes.c_int64 * 19)()
        self._check(lib().poa_batch_stats(self._h, o))
        names = ("view", "fill", "backtrack", "fusion", "topsort", "consensus")
        return dict(cells=o[0], failed=o[1], slots=o[2], slot_bytes=o[3], h2d_bytes=o[4], d2h_bytes=o[5],
                    phase_cycles={names[k]: o[6 + k] for k in range(6)}, launches=o[12], retried=o[13],
                    fallback=o[14], kernel_us=o[15], run_us=o[16], plan_us=o[17], edge_cells=o[18])

    def batch_plan(self, nodes=None, tb_bytes=None, spill=None, cost=None):
        """Per-window resource plan (see poa_batch_plan); no arguments clears it."""
        import numpy as np
        if nodes is None:
            self._check(lib().poa_batch_plan(self._h, None, None, None, None))
            return
        n = np.ascontiguousarray(nodes, dtype=np.int32)
        t = np.ascontiguousarray(tb_bytes, dtype=np.int64)
        sp = np.ascontiguousarray(spill, dtype=np.int64)
        c = np.ascontiguousarray(cost, dtype=np.float32)
        if not (n.shape[0] == t.shape[0] == sp.shape[0] == c.shape[0] == self._nwin):
            raise ValueError("plan arrays need one value per uploaded window")
        self._check(lib().poa_batch_plan(self._h, n.ctypes.data, t.ctypes.data, sp.ctypes.data, c.ctypes.data))

    def set_timing(self, on: bool = True):
        lib().poa_set_timing(self._h, 1 if on else 0)

    def stats(self) -> dict:
        o = (ctypes.c_int64 * 6)()
        lib().poa_stats(self._h, o)
        return dict(launches=o[0], alignments=o[1], cells=o[2], kernel_us=o[3], h2d_bytes=o[4], d2h_bytes=o[5])


PROP_BINS, PROP_CIN, PROP_OUT = 32, 8, 4
PROP_WEIGHTS = os.path.join(_HERE, "proposer_weights.f32")


class Proposer:
    """The learned band proposer (poa_prop_* in include/poa_b200.h)."""

    def __init__(self, device: int = 0, weights: Optional[str] = None):
        self._h = lib().poa_prop_create(device)
        if not self._h:
            raise PoaError(8, "poa_prop_create failed (no CUDA device or out of memory)")
        if weights is not None:
            self.load(weights)

    @staticmethod
    def nweights() -> int:
        return int(lib().poa_prop_nweights())

    def close(self):
        if getattr(self, "_h", None):
            lib().poa_prop_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != 0:
            raise PoaError(st, lib().poa_prop_last_error(self._h).decode(errors="replace"))

    def get_weights(self):
        import numpy as np
        w = np.zeros(self.nweights(), dtype=np.float32)
        self._check(lib().poa_prop_get_weights(self._h, w.ctypes.data))
        return w

    def set_weights(self, w) -> None:
        import numpy as np
        w = np.ascontiguousarray(w, dtype=np.float32)
        if w.shape != (self.nweights(),):
            raise ValueError(f"expected {self.nweights()} weights, got {w.shape}")
        self._check(lib().poa_prop_set_weights(self._h, w.ctypes.data))

    def load(self, path: str = PROP_WEIGHTS) -> None:
        import numpy as np
        self.set_weights(np.fromfile(path, dtype="<f4"))

    def save(self, path: str) -> None:
        self.get_weights().astype("<f4").tofile(path)

    def train(self, X, Y, epochs: int = 30, batch: int = 256, lr: float = 1e-3, seed: int = 1):
        """Train on X [n,32,8] / raw targets Y [n,4]; returns the per-epoch losses."""
        import numpy as np
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        losses = np.zeros(epochs, dtype=np.float32)
        self._check(lib().poa_prop_train(self._h, X.ctypes.data, Y.ctypes.data, X.shape[0], epochs, batch, lr, seed,
                                         losses.ctypes.data))
        return losses

    def predict(self, X):
        import numpy as np
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.zeros((X.shape[0], PROP_OUT), dtype=np.float32)
        self._check(lib().poa_prop_predict(self._h, X.ctypes.data, X.shape[0], Y.ctypes.data))
        return Y

    def gradient(self, X, Y):
        """(loss, parameter gradient) of one batch (1..4096 reads), no update."""
        import numpy as np
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        g = np.zeros(self.nweights() - 12, dtype=np.float32)
        loss = ctypes.c_float()
        self._check(lib().poa_prop_gradient(self._h, X.ctypes.data, Y.ctypes.data, X.shape[0], g.ctypes.data,
                                            ctypes.byref(loss)))
        return loss.value, g


class PinnedArray:
    """A numpy array over page-locked host memory (released with close())."""

    def __init__(self, shape, dtype):
        import numpy as np
        self.dtype = np.dtype(dtype)
        n = int(np.prod(shape)) if shape else 1
        nbytes = max(n * self.dtype.itemsize, 1)
        self._p = lib().poa_alloc_pinned(nbytes)
        if not self._p:
            raise PoaError(4, "cudaMallocHost failed")
        buf = (ctypes.c_char * nbytes).from_address(self._p)
        self.array = np.frombuffer(buf, dtype=self.dtype, count=n).reshape(shape)

    def close(self):
        if self._p:
            self.array = None
            lib().poa_free_pinned(self._p)
            self._p = None


def pinned_copy(a):
    """Copy a numpy array into page-locked memory; returns (holder, array)."""
    h = PinnedArray(a.shape, a.dtype)
    h.array[...] = a
    return h, h.array


def partition(ws, n_parts: int):
    """Split a window set over n_parts devices by estimated cost
    (poa_batch_partition: longest processing time first). Returns (part of
    each window as an int32 array, summed cost of each part)."""
    import numpy as np
    rlen = np.ascontiguousarray(ws.read_len, dtype=np.int32)
    woff = np.ascontiguousarray(ws.win_off, dtype=np.int32)
    nwin = int(woff.shape[0] - 1)
    part = np.zeros(max(nwin, 1), dtype=np.int32)
    cost = np.zeros(n_parts, dtype=np.int64)
    i64p, i32p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
    st = lib().poa_batch_partition(rlen.ctypes.data_as(i32p), woff.ctypes.data_as(i32p), nwin, n_parts,
                                   part.ctypes.data_as(i32p), cost.ctypes.data_as(i64p))
    if st != 0:
        raise PoaError(st, "poa_batch_partition")
    return part[:nwin], cost


def batch_consensus_multi(contexts: Sequence["Context"], ws):
    """One window set over several devices (poa_batch_consensus_multi: a
    cost-balanced split, one context per device on its own host thread, the
    consensus gathered in input order). Returns (consensus bytes, status) per
    window, as Context.batch_consensus does."""
    import numpy as np
    seq, roff, rlen, woff = Context._win_arrays(ws)
    nwin = int(woff.shape[0] - 1)
    cap = int(2 * (int(rlen.max()) if rlen.shape[0] else 0) + 64) * max(nwin, 1)
    cons = ctypes.create_string_buffer(max(cap, 1))
    off = np.zeros(nwin + 1, dtype=np.int64)
    st = np.zeros(max(nwin, 1), dtype=np.int32)
    hs = (ctypes.c_void_p * len(contexts))(*[c._h for c in contexts])
    i64p, i32p = ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32)
    rc = lib().poa_batch_consensus_multi(hs, len(contexts), seq.ctypes.data, seq.shape[0], roff.ctypes.data_as(i64p),
                                         rlen.ctypes.data_as(i32p), rlen.shape[0], woff.ctypes.data_as(i32p), nwin,
                                         cons, cap, off.ctypes.data_as(i64p), st.ctypes.data_as(i32p))
    if rc != 0:
        raise PoaError(rc, "poa_batch_consensus_multi")
    raw = cons.raw
    return [raw[off[w]:off[w + 1]] for w in range(nwin)], [int(x) for x in st[:nwin]]


def int_peak(device: int = 0, iters: int = 200000) -> Tuple[float, float]:
    """Measured int32 add+max operations per second of `device` (the integer
    roofline's denominator) and the timed launch's milliseconds."""
    ops, ms = ctypes.c_double(), ctypes.c_double()
    st = lib().poa_int_peak(device, iters, ctypes.byref(ops), ctypes.byref(ms))
    if st != 0:
        raise PoaError(st, "poa_int_peak")
    return ops.value, ms.value


def run(seqs: Sequence[bytes], params: Optional[Params] = None, headers=None, device: int = 0) -> bytes:
    with Context(params, device) as ctx:
        return ctx.run(seqs, headers)[0]
