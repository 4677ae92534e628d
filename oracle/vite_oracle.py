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


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and, when the reference sources are present, oracle/_ref)."""
    out = subprocess.DEVNULL if quiet else None
    subprocess.run(["make", "-C", HERE, "restate"], check=True, stdout=out)
    if os.path.isdir("/root/reference"):
        subprocess.run(["make", "-C", HERE, "-j8", "ref"], check=True, stdout=out)


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


def run_harness(args: list[str], record: str, threads: int = 1, timeout: float = 3600.0) -> str:
    """Run the reference harness (oracle/_ref) and return its stdout."""
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="close")
    res = subprocess.run([HARNESS, *args, "-w", record], capture_output=True, text=True,
                         env=env, timeout=timeout, check=True)
    return res.stdout


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
