"""ctypes binding of liboracle.so, the plain-C restatement of Vite's Louvain path,
plus readers for the reference harness's record files.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA product path. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg import this module.
"""
from __future__ import annotations

import ctypes as C
import os
import struct
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
HARNESS = os.path.join(REF_DIR, "vite_ref_harness")
FILE_CONVERT = os.path.join(REF_DIR, "fileConvert")
REF_MAIN = os.path.join(REF_DIR, "graphClustering")

_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)


class _VoGraph(C.Structure):
    _fields_ = [("nv", C.c_int64), ("ne", C.c_int64), ("rowptr", _i64p),
                ("tail", _i64p), ("weight", _f64p)]


class _VoPhase(C.Structure):
    _fields_ = [("lower", C.c_double), ("threshold", C.c_double), ("et_type", C.c_int),
                ("et_delta", C.c_double), ("ordering", C.c_int), ("num_color", C.c_int64)]


class _VoRun(C.Structure):
    _fields_ = [("threshold", C.c_double), ("coloring", C.c_int), ("vertex_order", C.c_int),
                ("max_colors", C.c_int), ("single_color_iter", C.c_int), ("et_type", C.c_int),
                ("et_delta", C.c_double), ("threshold_scaling", C.c_int), ("one_phase", C.c_int)]


def reference_dir() -> str:
    """Directory of the reference sources: $VITE_REFERENCE_DIR when set, else the
    default written in oracle/Makefile (the one place that names it)."""
    d = os.environ.get("VITE_REFERENCE_DIR")
    if d:
        return d
    res = subprocess.run(["make", "-s", "-C", HERE, "print-ref"], capture_output=True,
                         text=True)
    return res.stdout.strip()


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and, when the reference sources are present, oracle/_ref)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "restate"], check=True, stdout=out)
    ref = reference_dir()
    if ref and os.path.isdir(ref):
        subprocess.run(["make", "-C", HERE, "-j8", f"REF={ref}", "ref"], check=True, stdout=out)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        gp = C.POINTER(_VoGraph)
        L.vo_graph_free.argtypes = [gp]
        L.vo_rgg.argtypes = [C.c_int64, gp]
        L.vo_rgg_radius.argtypes = [C.c_int64]
        L.vo_rgg_radius.restype = C.c_double
        L.vo_lcg_drand.argtypes = [C.c_uint32, C.c_int64, _f64p]
        L.vo_seed_seq1.argtypes = [C.c_uint32]
        L.vo_seed_seq1.restype = C.c_uint32
        L.vo_add_random_edges.argtypes = [gp, C.c_double, C.c_uint64, gp]
        L.vo_add_random_edges.restype = C.c_int64
        L.vo_ba.argtypes = [C.c_int64, C.c_int64, C.c_uint64, gp]
        L.vo_er.argtypes = [C.c_int64, C.c_double, C.c_uint64, gp]
        L.vo_reweight.argtypes = [gp, C.c_int, C.c_uint64]
        L.vo_mix.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
        L.vo_mix.restype = C.c_uint64
        L.vo_vertex_degree.argtypes = [gp, _f64p]
        L.vo_vertex_degree.restype = C.c_double
        L.vo_louvain_phase.argtypes = [gp, C.POINTER(_VoPhase), _i64p, _i64p, _f64p,
                                       C.POINTER(C.c_int)]
        L.vo_color.argtypes = [gp, C.c_int64, C.c_int, C.c_int, _i64p]
        L.vo_color.restype = C.c_int64
        L.vo_color_hash.argtypes = [C.c_uint32, C.c_uint32]
        L.vo_color_hash.restype = C.c_uint32
        L.vo_rebuild.argtypes = [gp, _i64p, gp]
        L.vo_run.argtypes = [gp, C.POINTER(_VoRun), C.c_int, _i64p, _i64p,
                             C.POINTER(C.c_int), _f64p, _i64p, _f64p]
        L.vo_compare.argtypes = [C.c_int64, _i64p, _i64p, C.POINTER(CompareStats)]
        _lib = L
    return _lib


@dataclass
class Graph:
    """CSR in Vite's layout (graph.hpp:77-106): rowptr[nv+1], tail[ne], weight[ne]."""
    rowptr: np.ndarray
    tail: np.ndarray
    weight: np.ndarray

    @property
    def nv(self) -> int:
        return len(self.rowptr) - 1

    @property
    def ne(self) -> int:
        return len(self.tail)

    def _c(self):
        self.rowptr = np.ascontiguousarray(self.rowptr, dtype=np.int64)
        self.tail = np.ascontiguousarray(self.tail, dtype=np.int64)
        self.weight = np.ascontiguousarray(self.weight, dtype=np.float64)
        g = _VoGraph(self.nv, self.ne, self.rowptr.ctypes.data_as(_i64p),
                     self.tail.ctypes.data_as(_i64p), self.weight.ctypes.data_as(_f64p))
        return g

    def unit(self) -> "Graph":
        return Graph(self.rowptr.copy(), self.tail.copy(), np.ones_like(self.weight))


def _take(g: _VoGraph) -> Graph:
    nv, ne = g.nv, g.ne
    rp = np.ctypeslib.as_array(g.rowptr, shape=(nv + 1,)).copy()
    t = np.ctypeslib.as_array(g.tail, shape=(max(ne, 1),))[:ne].copy()
    w = np.ctypeslib.as_array(g.weight, shape=(max(ne, 1),))[:ne].copy()
    lib().vo_graph_free(C.byref(g))
    return Graph(rp, t, w)


def rgg(n: int) -> Graph:
    out = _VoGraph()
    if lib().vo_rgg(n, C.byref(out)):
        raise MemoryError("vo_rgg")
    return _take(out)


def rgg_radius(n: int) -> float:
    return lib().vo_rgg_radius(n)


def lcg_drand(seed: int, count: int) -> np.ndarray:
    out = np.empty(count, dtype=np.float64)
    lib().vo_lcg_drand(seed, count, out.ctypes.data_as(_f64p))
    return out


def add_random_edges(g: Graph, percent: float, seed: int) -> tuple[Graph, int]:
    out = _VoGraph()
    gi = g._c()
    added = lib().vo_add_random_edges(C.byref(gi), percent, seed, C.byref(out))
    return _take(out), int(added)


def ba(n: int, m: int, seed: int) -> Graph:
    out = _VoGraph()
    lib().vo_ba(n, m, seed, C.byref(out))
    return _take(out)


def er(n: int, avg_degree: float, seed: int) -> Graph:
    out = _VoGraph()
    lib().vo_er(n, avg_degree, seed, C.byref(out))
    return _take(out)


def reweight(g: Graph, mode: int, seed: int) -> Graph:
    h = Graph(g.rowptr.copy(), g.tail.copy(), g.weight.copy())
    gi = h._c()
    lib().vo_reweight(C.byref(gi), mode, seed)
    return h


def mix(seed: int, stream: int, k: int) -> int:
    return int(lib().vo_mix(seed, stream, k))


def vertex_degree(g: Graph) -> tuple[np.ndarray, float]:
    vd = np.empty(g.nv, dtype=np.float64)
    gi = g._c()
    c = lib().vo_vertex_degree(C.byref(gi), vd.ctypes.data_as(_f64p))
    return vd, c


def louvain_phase(g: Graph, threshold: float = 1e-6, lower: float = -1.0, et_type: int = 0,
                  et_delta: float = 1.0, ordering: int = 0, colors=None, num_color: int = 1):
    cv = np.empty(g.nv, dtype=np.int64)
    mod = C.c_double()
    iters = C.c_int()
    gi = g._c()
    p = _VoPhase(lower, threshold, et_type, et_delta, ordering, num_color)
    cp = None
    if colors is not None:
        colors = np.ascontiguousarray(colors, dtype=np.int64)
        cp = colors.ctypes.data_as(_i64p)
    lib().vo_louvain_phase(C.byref(gi), C.byref(p), cp, cv.ctypes.data_as(_i64p),
                           C.byref(mod), C.byref(iters))
    return cv, mod.value, iters.value


def color(g: Graph, n_hash: int, target_percent: int = 70, single: bool = False):
    out = np.empty(g.nv, dtype=np.int64)
    gi = g._c()
    nc = lib().vo_color(C.byref(gi), n_hash, target_percent, int(single),
                        out.ctypes.data_as(_i64p))
    return out, int(nc)


def color_hash(a: int, seed: int) -> int:
    return int(lib().vo_color_hash(a & 0xFFFFFFFF, seed & 0xFFFFFFFF))


class CompareStats(C.Structure):
    _fields_ = [("n", C.c_int64), ("nc1", C.c_int64), ("nc2", C.c_int64),
                ("same_same", C.c_int64), ("same_diff", C.c_int64), ("diff_same", C.c_int64),
                ("precision", C.c_double), ("recall", C.c_double), ("fscore", C.c_double),
                ("gini1", C.c_double), ("gini2", C.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


def compare(truth: np.ndarray, found: np.ndarray) -> dict:
    """compare_communities (compare.cpp:58-318): pair counts, precision, recall,
    F-score and Gini coefficients of two community vectors (truth first)."""
    a = np.ascontiguousarray(truth, dtype=np.int64)
    b = np.ascontiguousarray(found, dtype=np.int64)
    st = CompareStats()
    rc = lib().vo_compare(len(a), a.ctypes.data_as(_i64p), b.ctypes.data_as(_i64p), C.byref(st))
    if rc != 0:
        raise ValueError(f"vo_compare failed ({rc})")
    return st.as_dict()


def rebuild(g: Graph, cvect: np.ndarray) -> Graph:
    out = _VoGraph()
    gi = g._c()
    cv = np.ascontiguousarray(cvect, dtype=np.int64)
    lib().vo_rebuild(C.byref(gi), cv.ctypes.data_as(_i64p), C.byref(out))
    return _take(out)


@dataclass
class RunResult:
    level_nv: list = field(default_factory=list)
    level_ne: list = field(default_factory=list)
    level_iters: list = field(default_factory=list)
    level_mod: list = field(default_factory=list)
    level_colors: list = field(default_factory=list)
    seconds: float = 0.0


def run(g: Graph, threshold: float = 1e-6, coloring: bool = False, vertex_order: bool = False,
        max_colors: int = 8, single_color_iter: bool = False, et_type: int = 0,
        et_delta: float = 1.0, threshold_scaling: bool = False, one_phase: bool = False,
        max_levels: int = 256) -> RunResult:
    """The reference's phase loop (main.cpp:242-513) over the restatement."""
    rp = _VoRun(threshold, int(coloring), int(vertex_order), max_colors, int(single_color_iter),
                et_type, et_delta, int(threshold_scaling), int(one_phase))
    nv = np.zeros(max_levels, np.int64)
    ne = np.zeros(max_levels, np.int64)
    it = np.zeros(max_levels, np.int32)
    md = np.zeros(max_levels, np.float64)
    nc = np.zeros(max_levels, np.int64)
    sec = C.c_double()
    gi = g._c()
    n = lib().vo_run(C.byref(gi), C.byref(rp), max_levels, nv.ctypes.data_as(_i64p),
                     ne.ctypes.data_as(_i64p), it.ctypes.data_as(C.POINTER(C.c_int)),
                     md.ctypes.data_as(_f64p), nc.ctypes.data_as(_i64p), C.byref(sec))
    n = min(n, max_levels)
    return RunResult(list(nv[:n]), list(ne[:n]), list(it[:n]), list(md[:n]), list(nc[:n]),
                     sec.value)


# --------------------------------------------------------------------------------------
# Vite binary graph files (converters/convert.cpp:245-278, distgraph.cpp:1008-1061) and
# the reference harness's record files (oracle/ref_harness.cpp)

def write_vite_binary(path: str, g: Graph) -> None:
    edges = np.empty(g.ne, dtype=[("tail", "<i8"), ("weight", "<f8")])
    edges["tail"] = g.tail
    edges["weight"] = g.weight
    with open(path, "wb") as f:
        f.write(struct.pack("<qq", g.nv, g.ne))
        f.write(np.ascontiguousarray(g.rowptr, dtype="<i8").tobytes())
        f.write(edges.tobytes())


def read_vite_binary(path: str) -> Graph:
    with open(path, "rb") as f:
        nv, ne = struct.unpack("<qq", f.read(16))
        rp = np.frombuffer(f.read(8 * (nv + 1)), dtype="<i8").copy()
        e = np.frombuffer(f.read(16 * ne), dtype=[("tail", "<i8"), ("weight", "<f8")])
    return Graph(rp, e["tail"].copy(), e["weight"].copy())


@dataclass
class RefLevel:
    level: int
    nv: int
    ne: int
    iters: int
    mod: float
    num_colors: int
    seconds: float
    cvect: np.ndarray


@dataclass
class RefRecord:
    levels: list = field(default_factory=list)
    graphs: dict = field(default_factory=dict)
    colors: np.ndarray | None = None


def read_record(path: str) -> RefRecord:
    rec = RefRecord()
    with open(path, "rb") as f:
        if f.read(4) != b"VREC":
            raise ValueError("not a harness record file")
        f.read(4)
        while True:
            (tag,) = struct.unpack("<i", f.read(4))
            if tag == 0:
                break
            if tag == 1:
                level, nv, ne = struct.unpack("<qqq", f.read(24))
                (iters,) = struct.unpack("<i", f.read(4))
                mod, = struct.unpack("<d", f.read(8))
                ncol, = struct.unpack("<q", f.read(8))
                sc, sr = struct.unpack("<dd", f.read(16))
                cv = np.frombuffer(f.read(8 * nv), dtype="<i8").copy()
                rec.levels.append(RefLevel(level, nv, ne, iters, mod, ncol, sc, cv))
            elif tag == 2:
                level, nv, ne = struct.unpack("<qqq", f.read(24))
                rp = np.frombuffer(f.read(8 * (nv + 1)), dtype="<i8").copy()
                t = np.frombuffer(f.read(8 * ne), dtype="<i8").copy()
                w = np.frombuffer(f.read(8 * ne), dtype="<f8").copy()
                rec.graphs[level] = Graph(rp, t, w)
            elif tag == 3:
                nv, = struct.unpack("<q", f.read(8))
                rec.colors = np.frombuffer(f.read(8 * nv), dtype="<i8").copy()
            else:
                raise ValueError(f"bad record tag {tag}")
    return rec


def run_harness(args: list[str], record: str | None, threads: int = 1,
                timeout: float = 3600.0) -> str:
    """Run the reference harness (oracle/_ref) and return its stdout; `record` names the
    record file of the first run (None: no record)."""
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close")
    rec = ["-w", record] if record else []
    res = subprocess.run([HARNESS, *args, *rec], capture_output=True, text=True,
                         env=env, timeout=timeout, check=True)
    return res.stdout


def harness_totals(out: str) -> list[dict]:
    """The per-run totals a harness run printed (one line per run of the level loop)."""
    runs = []
    for line in out.splitlines():
        if line.startswith("HARNESS total_clustering_s"):
            f = line.split()
            runs.append({"clustering_s": float(f[2]), "rebuild_s": float(f[4]),
                         "total_s": float(f[6]), "levels": int(f[8]), "iterations": int(f[10]),
                         "final_mod": float(f[12])})
    return runs


def harness_read_seconds(out: str) -> float:
    for line in out.splitlines():
        if line.startswith("HARNESS graph_seconds"):
            return float(line.split()[2])
    return float("nan")


def output_map(levels: list, threshold: float = 1e-6) -> np.ndarray:
    """graphClustering's -o map (main.cpp:381-425) from a record's levels: every accepted
    level's communities renamed by sorted rank, composed into the level-0 map."""
    allmap = None
    prev = -1.0
    for lv in levels:
        if lv.level < 0 or not (lv.mod - prev) > threshold:
            break
        _, inv = np.unique(lv.cvect, return_inverse=True)
        allmap = inv.astype(np.int64) if allmap is None else inv[allmap].astype(np.int64)
        prev = lv.mod
    return allmap


@dataclass
class LevelResult:
    nv: int
    ne: int
    iters: int
    mod: float
    num_colors: int
    cvect: np.ndarray
    graph: Graph


def run_levels(g: Graph, threshold: float = 1e-6, coloring: bool = False,
               vertex_order: bool = False, max_colors: int = 8, single_color_iter: bool = False,
               et_type: int = 0, et_delta: float = 1.0, threshold_scaling: bool = False,
               one_phase: bool = False):
    """The reference's phase loop (main.cpp:242-513) over the restatement, keeping every
    level's graph and community vector. Returns (levels, colors of phase 0 or None)."""
    levels = []
    colors0 = None
    cur = g
    currMod, prevMod = -1.0, -1.0
    phase = short_phase = tot_iters = 0
    while True:
        if threshold_scaling and not one_phase:
            if short_phase > 12:
                short_phase = 0
            thr = (1e-3 if short_phase <= 2 else 1e-4 if short_phase <= 6
                   else 1e-5 if short_phase <= 9 else threshold)
        else:
            thr = threshold
        ncol = 0
        if (coloring or vertex_order) and phase == 0:
            colors0, ncol = color(cur, max_colors // 2, 70, single_color_iter)
            cv, currMod, iters = louvain_phase(cur, thr, currMod, et_type, et_delta,
                                               1 if coloring else 2, colors0, ncol + 1)
        else:
            cv, currMod, iters = louvain_phase(cur, thr, currMod, et_type, et_delta)
        tot_iters += iters
        levels.append(LevelResult(cur.nv, cur.ne, iters, currMod, ncol, cv, cur))
        if currMod - prevMod > thr:
            if not one_phase:
                cur = rebuild(cur, cv)
        else:
            if threshold_scaling and not one_phase and phase < 10:
                cv, currMod, iters = louvain_phase(cur, 1e-6, currMod)
                levels.append(LevelResult(cur.nv, cur.ne, iters, currMod, 0, cv, cur))
            break
        prevMod, currMod = currMod, -1.0
        phase += 1
        if one_phase:
            break
        if threshold_scaling and not one_phase:
            short_phase += 1
        if phase == 200 or tot_iters > 10000:
            break
    return levels, colors0


def flags_to_kwargs(flags: list[str]) -> dict:
    """graphClustering flags (main.cpp:609-708) -> keyword arguments of run/run_levels."""
    kw: dict = {}
    i = 0
    while i < len(flags):
        f = flags[i]
        if f in ("-c", "-d"):
            parts = flags[i + 1].split(" ")
            kw["max_colors"] = int(parts[0])
            if len(parts) > 1:
                kw["single_color_iter"] = parts[1].lower() in ("true", "1")
            kw["coloring" if f == "-c" else "vertex_order"] = True
            i += 2
        elif f == "-t":
            kw["et_type"] = int(flags[i + 1])
            i += 2
        elif f == "-a":
            kw["et_delta"] = float(flags[i + 1])
            i += 2
        elif f == "-h":
            kw["threshold"] = float(flags[i + 1])
            i += 2
        elif f == "-i":
            kw["threshold_scaling"] = True
            i += 1
        elif f == "-p":
            kw["one_phase"] = True
            i += 1
        else:
            raise ValueError(f"unsupported flag {f}")
    return kw


def golden_graph(entry: dict) -> Graph:
    """Rebuild the input graph of a golden case with the restatement's generators."""
    src = entry["source"]
    if src["kind"] == "reference_rgg":
        return rgg(int(src["n"]))
    kind, *rest = src["spec"].split(":")
    if kind == "file":
        base = {"rgg4k": 4096, "rgg64k": 65536}[rest[0]]
        g = rgg(base)
        return g.unit() if len(rest) > 1 and rest[1] == "unit" else g
    if kind == "ba":
        return ba(int(rest[0]), int(rest[1]), int(rest[2]))
    if kind == "er":
        return er(int(rest[0]), float(rest[1]), int(rest[2]))
    if kind == "rggx":
        return add_random_edges(rgg(int(rest[0])), float(rest[1]), int(rest[2]))[0]
    raise ValueError(src)


# --------------------------------------------------------------------------------------
# fileConvert's text readers (converters/convert.cpp:102-281): plain edge lists (-s,
# converters/simple.cpp:61-160), SNAP (-n, converters/snap.cpp:65-196) and Matrix Market
# (-m, converters/matrix-market.cpp:65-241), then processGraphData (utils.cpp:101-152)

import re as _re

_I64 = _re.compile(rb"[ \t\r\v\f]*([+-]?[0-9]+)")
_F64 = _re.compile(rb"[ \t\r\v\f]*([+-]?(?:[0-9]+\.?[0-9]*|\.[0-9]+)(?:[eE][+-]?[0-9]+)?)")


def _read_i64(line: bytes, pos: int):
    """operator>>(long long&) from pos: (value, new pos) or None."""
    m = _I64.match(line, pos)
    if not m:
        return None
    v = int(m.group(1))
    if not -(1 << 63) <= v < (1 << 63):
        return None
    return v, m.end()


def _read_f64(line: bytes, pos: int):
    """operator>>(double&): the correctly rounded value, or 0.0 when no number starts
    here (C++11 stores 0 on a failed read)."""
    m = _F64.match(line, pos)
    return float(m.group(1)) if m else 0.0


class _GenRandom:
    """genRandom(0.01, 1.0)'s stream, one weight per call (see gen_random_weights)."""

    def __init__(self):
        self.x = 1

    def __call__(self) -> float:
        M = 2147483647
        self.x = (self.x * 16807) % M
        x1 = self.x
        self.x = (self.x * 16807) % M
        x2 = self.x
        s = float(x1 - 1) * 1.0
        s = s + float(x2 - 1) * 2147483646.0
        c = s / float(2147483646 * 2147483646)
        if c >= 1.0:
            c = float(np.nextafter(1.0, 0.0))
        return c * (1.0 - 0.01) + 0.01


def gen_random_weights(count: int) -> np.ndarray:
    """genRandom(0.01, 1.0) (utils.cpp:93-99) called `count` times: a static
    std::default_random_engine (minstd_rand0, x <- 16807 x mod 2^31 - 1, seed 1) through
    std::uniform_real_distribution<double>, whose generate_canonical<double, 53> takes
    two draws (range r = 2^31 - 2): c = ((x1 - 1) + (x2 - 1) * r) / r^2, then
    0.01 + c * (1.0 - 0.01); restated from the C++ standard's definitions."""
    out = np.empty(count, dtype=np.float64)
    x = 1
    M = 2147483647
    r = 2147483646.0
    rr = float(2147483646 * 2147483646)
    for k in range(count):
        x = (x * 16807) % M
        x1 = x
        x = (x * 16807) % M
        x2 = x
        s = float(x1 - 1) * 1.0
        s = s + float(x2 - 1) * r
        c = s / rr
        if c >= 1.0:
            c = np.nextafter(1.0, 0.0)
        out[k] = c * (1.0 - 0.01) + 0.01
    return out


def _csr_from_list(nv: int, src, dst, w) -> Graph:
    """processGraphData: counts per source, entries sorted by (source, tail); equal pairs
    keep their list order (std::sort leaves them unspecified)."""
    src = np.asarray(src, dtype=np.int64)
    dst = np.asarray(dst, dtype=np.int64)
    w = np.asarray(w, dtype=np.float64)
    order = np.lexsort((dst, src)) if len(src) else np.zeros(0, np.int64)
    rp = np.zeros(nv + 1, dtype=np.int64)
    if len(src):
        np.add.at(rp, src + 1, 1)
    rp = np.cumsum(rp)
    return Graph(rp, dst[order], w[order])


def canonical_ties(g: Graph) -> np.ndarray:
    """The weights with every run of equal (row, tail) entries sorted by weight bits:
    std::sort leaves such runs in an unspecified order, so comparisons with the
    reference's converter output go through this."""
    rows = np.repeat(np.arange(g.nv, dtype=np.int64), np.diff(g.rowptr))
    order = np.lexsort((g.weight.view(np.int64), g.tail, rows))
    return g.weight[order]


def read_text(path: str, fmt: str, weights: str = "abs", one_based: bool = False) -> Graph:
    """fileConvert -s/-n/-m [-w|-i|-r] [-z] as a Graph. fmt: 'simple', 'snap' or 'mm';
    weights: 'abs' (default), 'orig' (-i), 'one' (-w), 'random' (-r)."""
    data = open(path, "rb").read()
    src, dst, w = [], [], []
    rnd = _GenRandom()

    def weight_of(x: float) -> float:
        if weights == "one":
            return 1.0
        if weights == "random":
            return rnd()
        return abs(x) if weights == "abs" else x

    if fmt == "simple":
        pieces = data.split(b"\n")  # the last piece is the text after the last newline
        read_w = weights in ("abs", "orig")
        mx = -1
        for k, line in enumerate(pieces):  # first pass: the largest id (simple.cpp:78-102)
            if line[:1] in (b"#", b"%"):
                continue
            a = _read_i64(line, 0)
            if a is None:
                v0 = 0 - (1 if one_based else 0)
                mx = max(mx, v0)
                continue
            b = _read_i64(line, a[1])
            v0 = a[0] - (1 if one_based else 0)
            v1 = b[0] - (1 if one_based else 0) if b else v0
            mx = max(mx, v0, v1)
        nv = mx + 1
        for k, line in enumerate(pieces[:-1]):  # second pass: every piece but the last
            if line[:1] in (b"#", b"%"):
                continue
            a = _read_i64(line, 0)
            b = _read_i64(line, a[1]) if a else None
            if a is None or b is None:
                raise ValueError(f"line {k + 1}: two ids expected")
            x = _read_f64(line, b[1]) if read_w else 0.0
            v0, v1 = a[0], b[0]
            if one_based:
                v0, v1 = v0 - 1, v1 - 1
            x = weight_of(x)
            src += [v0, v1]
            dst += [v1, v0]
            w += [x, x]
        return _csr_from_list(nv, src, dst, w)

    if fmt == "snap":
        pos = 0
        nv = ne = None
        lines = data.split(b"\n")
        i = 0
        while i < len(lines) and lines[i][:1] == b"#":
            line = lines[i].decode()
            if "Nodes" in line:
                nums = [int(_re.match(r"\s*([+-]?\d+)", part).group(1))
                        for part in line.split(":")[1:3]]
                nv, ne = nums
            pos += len(lines[i]) + 1
            i += 1
        toks = data[pos:].split()[: 2 * ne]
        if len(toks) < 2 * ne:
            raise ValueError("fewer ids than the header's edges")
        newid: dict = {}
        ids = []
        for t in toks:
            v = int(t)
            if v not in newid:
                newid[v] = len(newid)
            ids.append(newid[v])
        for k in range(ne):
            x = weight_of(1.0) if weights == "random" else 1.0
            u, v = ids[2 * k], ids[2 * k + 1]
            src += [u, v]
            dst += [v, u]
            w += [x, x]
        return _csr_from_list(nv, src, dst, w)

    if fmt == "mm":
        lines = data.split(b"\n")
        banner = lines[0].split()
        field, symm = banner[3].upper(), banner[4].upper()
        pattern = field == b"PATTERN"
        symmetric = symm == b"SYMMETRIC"
        i = 1
        while lines[i][:1] == b"%":
            i += 1
        ns, _, ne = (int(x) for x in lines[i].split()[:3])
        nv = ns
        read_w = not pattern and weights in ("abs", "orig")
        for k in range(ne):
            line = lines[i + 1 + k]
            a = _read_i64(line, 0)
            b = _read_i64(line, a[1])
            x = _read_f64(line, b[1]) if read_w else 1.0
            if weights == "abs" and not pattern:
                x = abs(x)
            if weights == "one":
                x = 1.0
            if weights == "random":
                x = weight_of(1.0)
            s, d = a[0] - 1, b[0] - 1
            if symmetric and s != d:
                src += [s, d]
                dst += [d, s]
                w += [x, x]
            else:
                src.append(s)
                dst.append(d)
                w.append(x)
        return _csr_from_list(nv, src, dst, w)
    raise ValueError(fmt)
