"""poa_align_noalloc against poa_align.

poa_align_noalloc is for callers that cannot allocate device memory when they
align (a framework that owns the device pool, or a service that forbids
cudaMalloc on its request path): the caller places the window rows and the
query in device memory it owns, and the library works in a fixed array it
holds on every GPU. This test builds a real POA graph, flattens it once, and
requires the no-allocation entry point to return exactly what poa_align
returns (same path, same score; both are bit-exact integer DP) on two calls
in a row, so the second call also runs on the scratch contents the first one
left behind. The test itself allocates its inputs and outputs with torch; only
the entry point is allocation-free.

The file name sorts last so that a run stopping at the first failure has
already run every other test.
"""
import ctypes
import os

import numpy as np
import pytest

import poa_b200
from poa_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_LIB = os.path.join(ROOT, "oracle", "build", "libpoa_oracle.so")

P32 = ctypes.POINTER(ctypes.c_int32)
PU8 = ctypes.POINTER(ctypes.c_uint8)


class GraphView(ctypes.Structure):
    _fields_ = [("n_nodes", ctypes.c_int32), ("base", PU8), ("rank", P32), ("par_id", P32), ("ind", P32),
                ("aligned", P32), ("in_ptr", P32), ("in_id", P32), ("in_weight", P32), ("out_ptr", P32),
                ("out_id", P32), ("n_ranks", ctypes.c_int32), ("rank_to_id", P32), ("hlen", P32), ("tlen", P32)]


class Res(ctypes.Structure):
    _fields_ = [("from_", ctypes.c_int32), ("base", ctypes.c_uint8), ("aligned_id", ctypes.c_int32)]


class DevWindow(ctypes.Structure):
    _fields_ = [("n_rows", ctypes.c_int32)] + [(f, ctypes.c_void_p) for f in (
        "in_ptr", "in_row", "in_weight", "in_base", "base", "ind", "hq", "hq_loc", "tq", "out_ptr", "out_row")]


class OParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("match", "mismatch", "gap_open1", "gap_ext1", "b", "f", "ab_band",
                                            "verbose")]


class ORes(ctypes.Structure):
    _fields_ = [("from_", ctypes.c_int), ("base", ctypes.c_uint8), ("aligned_id", ctypes.c_int)]


def _oracle():
    lib = ctypes.CDLL(ORACLE_LIB)
    lib.po_graph_new.restype = ctypes.c_void_p
    lib.po_graph_free.argtypes = [ctypes.c_void_p]
    lib.po_alignment.argtypes = [ctypes.c_void_p, ctypes.POINTER(OParams), PU8, ctypes.c_int,
                                 ctypes.POINTER(ctypes.POINTER(ORes)), ctypes.POINTER(ctypes.c_int),
                                 ctypes.POINTER(ctypes.c_int)]
    lib.po_add_path.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ORes), ctypes.c_int, ctypes.c_int]
    lib.po_topsort.argtypes = [ctypes.c_void_p, ctypes.POINTER(OParams), ctypes.c_int]
    lib.po_graph_sizes.argtypes = [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_int)] * 5
    lib.po_graph_export.argtypes = [ctypes.c_void_p, PU8] + [P32] * 12
    return lib


def build_graph(reads):
    """A POA graph of `reads` (default scoring, static band), flattened."""
    o = _oracle()
    libc = ctypes.CDLL(None)
    libc.free.argtypes = [ctypes.c_void_p]
    p = OParams(2, -4, -4, -2, 100, 40, 0, 0)
    g = o.po_graph_new()
    for i, r in enumerate(reads):
        q = np.frombuffer(bytes(r), dtype=np.uint8).copy()
        path = ctypes.POINTER(ORes)()
        plen, score = ctypes.c_int(), ctypes.c_int()
        assert o.po_alignment(g, ctypes.byref(p), q.ctypes.data_as(PU8), q.shape[0], ctypes.byref(path),
                              ctypes.byref(plen), ctypes.byref(score)) == 0
        o.po_add_path(g, i, path, plen.value, 1)
        libc.free(ctypes.cast(path, ctypes.c_void_p))
        o.po_topsort(g, ctypes.byref(p), 0)
    sz = [ctypes.c_int() for _ in range(5)]
    o.po_graph_sizes(g, *[ctypes.byref(x) for x in sz])
    nn, ni, no, nr, nl = [x.value for x in sz]
    a = dict(base=np.zeros(nn, np.uint8), rank=np.zeros(nn, np.int32), par=np.zeros(nn, np.int32),
             ind=np.zeros(nn, np.int32), aligned=np.zeros(5 * nn, np.int32), in_ptr=np.zeros(nn + 1, np.int32),
             in_id=np.zeros(max(ni, 1), np.int32), in_w=np.zeros(max(ni, 1), np.int32),
             out_ptr=np.zeros(nn + 1, np.int32), out_id=np.zeros(max(no, 1), np.int32),
             rank_to_id=np.zeros(nr, np.int32), hlen=np.zeros(max(nl, 1), np.int32),
             tlen=np.zeros(max(nl, 1), np.int32))
    o.po_graph_export(g, a["base"].ctypes.data_as(PU8), *[a[k].ctypes.data_as(P32) for k in (
        "rank", "par", "ind", "aligned", "in_ptr", "in_id", "in_w", "out_ptr", "out_id", "rank_to_id", "hlen",
        "tlen")])
    o.po_graph_free(g)
    return a


def graph_view(a):
    return GraphView(a["base"].shape[0], a["base"].ctypes.data_as(PU8), *[a[k].ctypes.data_as(P32) for k in (
        "rank", "par", "ind", "aligned", "in_ptr", "in_id", "in_w", "out_ptr", "out_id")],
        a["rank_to_id"].shape[0], a["rank_to_id"].ctypes.data_as(P32), a["hlen"].ctypes.data_as(P32),
        a["tlen"].ctypes.data_as(P32))


def window_rows(a, beg_id=0, end_id=1):
    """Rows of ranks [rank(beg), rank(end)] laid out as poa_dev_window wants."""
    rank, r2i = a["rank"], a["rank_to_id"]
    beg_i, end_i = int(rank[beg_id]), int(rank[end_id])
    n = end_i - beg_i + 1
    rows = dict(in_ptr=[0], in_row=[], in_weight=[], in_base=[], base=[], ind=[], hq=[], hq_loc=[], tq=[],
                out_ptr=[0], out_row=[])
    for r in range(n):
        u = int(r2i[beg_i + r])
        rows["base"].append(a["base"][u])
        rows["ind"].append(a["ind"][u])
        rows["hq"].append(a["hlen"][beg_i + r] - a["hlen"][beg_i])
        rows["hq_loc"].append(a["hlen"][r] - a["hlen"][beg_i])
        rows["tq"].append(a["tlen"][beg_i + r] - a["tlen"][end_i])
        for e in range(a["in_ptr"][u], a["in_ptr"][u + 1]):
            p = int(rank[a["in_id"][e]]) - beg_i
            if p < 0:
                continue
            rows["in_row"].append(p)
            rows["in_weight"].append(a["in_w"][e])
            rows["in_base"].append(4 if p == 0 else a["base"][a["in_id"][e]])
        rows["in_ptr"].append(len(rows["in_row"]))
        for e in range(a["out_ptr"][u], a["out_ptr"][u + 1]):
            s = int(rank[a["out_id"][e]]) - beg_i
            if s < n:
                rows["out_row"].append(s)
        rows["out_ptr"].append(len(rows["out_row"]))
    u8 = ("in_base", "base")
    return n, {k: np.array(v if v else [0], dtype=np.uint8 if k in u8 else np.int32) for k, v in rows.items()}


def moves_to_res(a, n_rows, moves):
    """Backtrack moves (backtrack order) -> forward path, as poa_align emits it."""
    r2i, beg_i = a["rank_to_id"], int(a["rank"][0])
    out = []
    for mv in reversed(moves):
        mv = int(mv) & 0xffffffff
        qc, kind, prow = mv & 7, (mv >> 3) & 3, mv >> 5
        if kind == 2:
            out.append((-1, qc, -1))
            continue
        pre = int(r2i[beg_i + prow])
        if kind == 0:
            out.append((pre, int(a["base"][pre]), -1))
        else:
            par = int(a["par"][pre])
            al = int(a["aligned"][5 * par + qc])
            out.append((al, qc, -1) if al != -1 else (-1, qc, par))
    return out


def _bind(L):
    L.poa_align.argtypes = [ctypes.c_void_p, ctypes.POINTER(GraphView), ctypes.c_int32, ctypes.c_int32, PU8,
                            ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(Res), ctypes.c_int32, P32, P32]
    L.poa_align_noalloc.argtypes = [ctypes.POINTER(DevWindow), ctypes.c_void_p, ctypes.c_int32,
                                    ctypes.POINTER(poa_b200._CParams), ctypes.c_int32, ctypes.c_void_p,
                                    ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
    return L


def oracle_alignment(reads, query, adaptive):
    """Score and path of the CPU restatement for `query` against the graph of
    `reads` (the graph built as build_graph builds it, static band)."""
    o = _oracle()
    libc = ctypes.CDLL(None)
    libc.free.argtypes = [ctypes.c_void_p]
    p_graph = OParams(2, -4, -4, -2, 100, 40, 0, 0)
    p_query = OParams(2, -4, -4, -2, 100, 40, int(adaptive), 0)
    g = o.po_graph_new()
    for i, r in enumerate(list(reads) + [query]):
        last = i == len(reads)
        q = np.frombuffer(bytes(r), dtype=np.uint8).copy()
        path = ctypes.POINTER(ORes)()
        plen, score = ctypes.c_int(), ctypes.c_int()
        assert o.po_alignment(g, ctypes.byref(p_query if last else p_graph), q.ctypes.data_as(PU8), q.shape[0],
                              ctypes.byref(path), ctypes.byref(plen), ctypes.byref(score)) == 0
        res = [(path[k].from_, path[k].base, path[k].aligned_id) for k in range(plen.value)]
        if not last:
            o.po_add_path(g, i, path, plen.value, 1)
            o.po_topsort(g, ctypes.byref(p_graph), 0)
        libc.free(ctypes.cast(path, ctypes.c_void_p))
    o.po_graph_free(g)
    return score.value, res


def noalloc_need(n_rows, qlen, adaptive):
    """Worst-case scratch bytes of a window, as the entry point computes them."""
    def up(x):
        return (x + 255) // 256 * 256
    m = qlen + 1
    blocks = m // 8 + 1
    need = up(((m // 8 + 3) * 8 + 15) // 16 * 16) + up(24 * n_rows)
    if adaptive:
        need += up(4 * 7 * n_rows)
    return need + up(4 * (n_rows * blocks * 16 + 16)) + up(n_rows * (blocks * 8 * 4 + 16) + 16)


SCRATCH = 64 << 20


def encode(seq):
    return np.array([{65: 0, 67: 1, 71: 2, 84: 3}.get(int(c), 4) for c in bytes(seq)], dtype=np.uint8)


def align_both_ways(L, torch, reads, query, adaptive, q_pad=0):
    """(score, path) of poa_align, and of two poa_align_noalloc calls in a row."""
    a = build_graph(reads)
    q_enc = encode(query)
    params = poa_b200.Params(ab_band=adaptive)
    cp = params._c()
    with poa_b200.Context(params) as ctx:
        gv = graph_view(a)
        out = (Res * (a["base"].shape[0] + q_enc.shape[0] + 8))()
        olen, score = ctypes.c_int32(), ctypes.c_int32()
        st = L.poa_align(ctypes.c_void_p(ctx._h), ctypes.byref(gv), 0, 1, q_enc.ctypes.data_as(PU8),
                         q_enc.shape[0], int(adaptive), out, len(out), ctypes.byref(olen), ctypes.byref(score))
        assert st == 0
        want = (score.value, [(out[k].from_, out[k].base, out[k].aligned_id) for k in range(olen.value)])
    n, rows = window_rows(a)
    dev = {k: torch.from_numpy(v).cuda() for k, v in rows.items()}
    dq = torch.zeros(q_enc.shape[0] + q_pad + 16, dtype=torch.uint8, device="cuda")
    dq[:q_enc.shape[0]] = torch.from_numpy(q_enc.copy()).cuda()
    cap = n + q_enc.shape[0] + q_pad + 8
    w = DevWindow(n, *[dev[k].data_ptr() for k in ("in_ptr", "in_row", "in_weight", "in_base", "base", "ind",
                                                   "hq", "hq_loc", "tq", "out_ptr", "out_row")])
    got = []
    for _ in range(2):
        dmoves = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
        dres = torch.full((4,), -7, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        st = L.poa_align_noalloc(ctypes.byref(w), dq.data_ptr(), q_enc.shape[0], ctypes.byref(cp), int(adaptive),
                                 dmoves.data_ptr(), cap, dres.data_ptr(), None)
        assert st == 0
        torch.cuda.synchronize()
        res = dres.cpu().tolist()
        assert res[0] == 0, res
        got.append((res[1], moves_to_res(a, n, dmoves[:res[2]].cpu().numpy())))
    return n, want, got, (w, dq, cap, cp)


def _cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def test_noalloc_matches_poa_align_and_oracle(oracle_bin):
    torch = _cuda()
    L = _bind(poa_b200.lib())
    ws = synth.windows(77, 2, (500, 600), (10, 12), 0.08)
    for w, adaptive in ((0, False), (1, True)):  # static band, then adaptive band
        reads = ws.window_reads(w)
        _, want, got, _ = align_both_ways(L, torch, reads[:6], reads[6], adaptive)
        assert got[0] == want and got[1] == want
        # and, independently of the CUDA entry points, the CPU restatement
        assert oracle_alignment(reads[:6], reads[6], adaptive) == want


def test_noalloc_window_at_the_scratch_limit(oracle_bin):
    """A window whose worst case just fits the fixed scratch runs and matches;
    a few query bases more and the call is refused before any launch."""
    torch = _cuda()
    L = _bind(poa_b200.lib())
    ws = synth.windows(78, 1, (600, 600), (7, 7), 0.08)
    reads = ws.window_reads(0)
    a = build_graph(reads[:6])
    n = int(a["rank"][1]) - int(a["rank"][0]) + 1
    qlen = 1
    while noalloc_need(n, qlen + 1, False) <= SCRATCH:
        qlen += 1
    assert noalloc_need(n, qlen, False) > SCRATCH - (1 << 20)  # within 1 MiB of the limit
    # the last read with a random insertion in its middle, up to qlen bases
    r = reads[6]
    rng = np.random.default_rng(79)
    ins = synth.to_ascii(synth.random_root(rng, qlen - len(r)))
    query = r[:len(r) // 2] + ins + r[len(r) // 2:]
    assert len(query) == qlen
    n2, want, got, (w, dq, cap, cp) = align_both_ways(L, torch, reads[:6], query, False, q_pad=64)
    assert n2 == n
    assert got[0] == want and got[1] == want
    assert oracle_alignment(reads[:6], query, False) == want
    # 8 more bases: one more block per row no longer fits; refused (POA_OOM), nothing launched
    assert noalloc_need(n, qlen + 8, False) > SCRATCH
    dres = torch.full((4,), -7, dtype=torch.int32, device="cuda")
    dmoves = torch.zeros(cap, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    st = L.poa_align_noalloc(ctypes.byref(w), dq.data_ptr(), qlen + 8, ctypes.byref(cp), 0, dmoves.data_ptr(),
                             cap, dres.data_ptr(), None)
    assert st == 4
    torch.cuda.synchronize()
    assert dres.cpu().tolist() == [-7, -7, -7, -7]


def test_noalloc_rejects_oversized_window():
    torch = _cuda()
    L = _bind(poa_b200.lib())
    # 20,000 rows x a 10 kb query needs far more than the fixed scratch: POA_OOM, nothing launched
    dummy = torch.zeros(16, dtype=torch.int32, device="cuda")
    p = dummy.data_ptr()
    w = DevWindow(20000, *([p] * 11))
    cp = poa_b200.Params()._c()
    st = L.poa_align_noalloc(ctypes.byref(w), p, 10000, ctypes.byref(cp), 0, p, 40000, p, None)
    assert st == 4
