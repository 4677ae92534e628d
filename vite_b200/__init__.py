"""vite_b200: B200-native Louvain community detection (Vite's method) on one GPU.

Python view of the C ABI in include/vite_b200.h (libvite_b200.so, built in this
directory by ``make -C vite_b200/csrc``). The names follow the reference's
operators: ``louvain_phase`` is distLouvainMethod and its variants,
``color`` distColoringMultiHashMinMax, ``rebuild`` distbuildNextLevelGraph,
``generate_rgg`` generateInMemGraph, ``run`` the phase loop of graphClustering.

Importing this module loads the CUDA library; it raises if the library is
missing, and every call runs on the GPU (there is no CPU path).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libvite_b200.so")
HOST_LIB_PATH = os.path.join(HERE, "libvite_host.so")
CLI_PATH = os.path.join(HERE, "graphClustering")

EDGE_DTYPE = np.dtype([("tail", "<i8"), ("weight", "<f8")])

VG_OK, VG_ERR_ARG, VG_ERR_OOM, VG_ERR_CUDA, VG_ERR_TIMEOUT, VG_ERR_STATE = range(6)
_STATUS_NAMES = {0: "VG_OK", 1: "VG_ERR_ARG", 2: "VG_ERR_OOM", 3: "VG_ERR_CUDA",
                 4: "VG_ERR_TIMEOUT", 5: "VG_ERR_STATE"}

EXPORTED_SYMBOLS = [
    "vg_ctx_create", "vg_ctx_destroy", "vg_last_error", "vg_ctx_bytes_in_use", "vg_ctx_profile",
    "vg_ctx_stream", "vg_ctx_reserve",
    "vg_graph_upload", "vg_graph_info", "vg_graph_download", "vg_graph_free", "vg_vertex_degree",
    "vg_louvain_phase", "vg_color", "vg_set_colors", "vg_rebuild", "vg_louvain_run",
    "vg_generate_rgg", "vg_generate_ba", "vg_generate_er", "vg_graph_reweight",
    "vg_graph_reorder", "vg_vertex_degree_noalloc",
    "vg_batch_create", "vg_batch_destroy", "vg_batch_submit", "vg_batch_step", "vg_batch_poll",
    "vg_batch_result", "vg_batch_forget", "vg_batch_get_stats", "vg_compare_communities",
    "vg_ctx_get_tuning", "vg_ctx_set_tuning", "vg_autotune",
    "vg_graph_read_vite", "vg_graph_write_vite", "vg_graph_read_text",
]

# vg_text_format / vg_text_weights (fileConvert's -s/-n/-m and -w/-i/-r)
TEXT_FORMATS = {"simple": 1, "snap": 2, "mm": 3}
TEXT_WEIGHTS = {"abs": 0, "orig": 1, "one": 2, "random": 3}

VG_BATCH_TAKE = 1
VG_BATCH_COMM = 2


class VgError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{_STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class PhaseParams(C.Structure):
    _fields_ = [("lower", C.c_double), ("threshold", C.c_double), ("et_type", C.c_int32),
                ("et_delta", C.c_double), ("ordering", C.c_int32)]


class RunParams(C.Structure):
    _fields_ = [("threshold", C.c_double), ("coloring", C.c_int32), ("vertex_order", C.c_int32),
                ("max_colors", C.c_int32), ("single_color_iter", C.c_int32),
                ("et_type", C.c_int32), ("et_delta", C.c_double),
                ("threshold_scaling", C.c_int32), ("one_phase", C.c_int32),
                ("layout", C.c_int32)]


class LevelStat(C.Structure):
    _fields_ = [("nv", C.c_int64), ("ne", C.c_int64), ("iters", C.c_int32),
                ("modularity", C.c_double), ("num_colors", C.c_int64),
                ("seconds_color", C.c_double), ("seconds_phase", C.c_double),
                ("seconds_sweep", C.c_double), ("seconds_rebuild", C.c_double),
                ("edges_swept", C.c_int64), ("seconds_layout", C.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class CompareStats(C.Structure):
    _fields_ = [("n", C.c_int64), ("nc1", C.c_int64), ("nc2", C.c_int64),
                ("same_same", C.c_int64), ("same_diff", C.c_int64), ("diff_same", C.c_int64),
                ("precision", C.c_double), ("recall", C.c_double), ("fscore", C.c_double),
                ("gini1", C.c_double), ("gini2", C.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class TextParams(C.Structure):
    _fields_ = [("format", C.c_int32), ("weights", C.c_int32), ("one_based", C.c_int32)]


class Tuning(C.Structure):
    """vg_tuning: which sweep kernel takes each degree, and the tile grid."""
    _fields_ = [("t32", C.c_int32), ("ws_max", C.c_int32), ("wt_max", C.c_int32),
                ("ct_max", C.c_int32), ("tile_grid", C.c_int32)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class BatchStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("admitted", C.c_int64), ("completed", C.c_int64),
                ("rounds", C.c_int64), ("running", C.c_int64), ("queued", C.c_int64),
                ("running_bytes", C.c_size_t), ("seconds_phase", C.c_double),
                ("seconds_rebuild", C.c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_i64p = C.POINTER(C.c_int64)
_f64p = C.POINTER(C.c_double)
_lib = None


def library_path() -> str:
    return LIB_PATH


def lib() -> C.CDLL:
    """Load libvite_b200.so; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C vite_b200/csrc` "
                              "(or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.vg_ctx_create.argtypes = [C.c_int, C.c_size_t, C.POINTER(vp)]
        L.vg_ctx_destroy.argtypes = [vp]
        L.vg_last_error.argtypes = [vp]
        L.vg_last_error.restype = C.c_char_p
        L.vg_ctx_bytes_in_use.argtypes = [vp]
        L.vg_ctx_bytes_in_use.restype = C.c_size_t
        L.vg_ctx_profile.argtypes = [vp, C.c_int32, _f64p, _i64p, C.c_int32]
        L.vg_ctx_stream.argtypes = [vp, C.POINTER(vp)]
        L.vg_ctx_reserve.argtypes = [vp, C.c_size_t]
        L.vg_graph_upload.argtypes = [vp, C.c_int64, C.c_int64, _i64p, vp, C.POINTER(vp)]
        L.vg_graph_info.argtypes = [vp, _i64p, _i64p]
        L.vg_graph_download.argtypes = [vp, vp, _i64p, vp]
        L.vg_graph_free.argtypes = [vp, vp]
        L.vg_vertex_degree.argtypes = [vp, vp, _f64p, _f64p]
        L.vg_louvain_phase.argtypes = [vp, vp, C.POINTER(PhaseParams), _i64p, _f64p,
                                       C.POINTER(C.c_int32)]
        L.vg_color.argtypes = [vp, vp, C.c_int64, C.c_int32, C.c_int32, _i64p, _i64p]
        L.vg_set_colors.argtypes = [vp, vp, _i64p, C.c_int64]
        L.vg_rebuild.argtypes = [vp, vp, _i64p]
        L.vg_louvain_run.argtypes = [vp, vp, C.POINTER(RunParams), C.POINTER(LevelStat),
                                     C.c_int32, C.POINTER(C.c_int32), _i64p]
        L.vg_generate_rgg.argtypes = [vp, C.c_int64, C.c_double, C.c_uint64, C.POINTER(vp)]
        L.vg_generate_ba.argtypes = [vp, C.c_int64, C.c_int64, C.c_uint64, C.POINTER(vp)]
        L.vg_generate_er.argtypes = [vp, C.c_int64, C.c_double, C.c_uint64, C.POINTER(vp)]
        L.vg_graph_reweight.argtypes = [vp, vp, C.c_int32, C.c_uint64]
        L.vg_graph_reorder.argtypes = [vp, vp, C.c_int32]
        L.vg_vertex_degree_noalloc.argtypes = [C.c_int64, vp, vp, vp, _f64p, vp, C.c_char_p,
                                               C.c_size_t]
        L.vg_batch_create.argtypes = [vp, C.c_size_t, C.POINTER(vp)]
        L.vg_batch_destroy.argtypes = [vp]
        L.vg_batch_submit.argtypes = [vp, vp, C.POINTER(RunParams), C.c_int32, _i64p]
        L.vg_batch_step.argtypes = [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.vg_batch_poll.argtypes = [vp, _i64p, C.c_int32, C.POINTER(C.c_int32)]
        L.vg_batch_result.argtypes = [vp, C.c_int64, C.POINTER(LevelStat), C.c_int32,
                                      C.POINTER(C.c_int32), _i64p]
        L.vg_batch_forget.argtypes = [vp, C.c_int64]
        L.vg_batch_get_stats.argtypes = [vp, C.POINTER(BatchStats)]
        L.vg_compare_communities.argtypes = [vp, C.c_int64, _i64p, _i64p, C.POINTER(CompareStats)]
        L.vg_graph_read_vite.argtypes = [vp, C.c_char_p, C.POINTER(vp)]
        L.vg_graph_write_vite.argtypes = [vp, vp, C.c_char_p]
        L.vg_graph_read_text.argtypes = [vp, C.c_char_p, C.POINTER(TextParams), C.POINTER(vp)]
        L.vg_ctx_get_tuning.argtypes = [vp, C.POINTER(Tuning)]
        L.vg_ctx_set_tuning.argtypes = [vp, C.POINTER(Tuning)]
        L.vg_autotune.argtypes = [vp, C.POINTER(vp), C.c_int32, C.c_int32, C.POINTER(Tuning),
                                  _f64p, _f64p]
        for name in EXPORTED_SYMBOLS:
            if name not in ("vg_last_error", "vg_ctx_bytes_in_use"):
                getattr(L, name).restype = C.c_int
        _lib = L
    return _lib


def _ptr(a: np.ndarray | None, ty=_i64p):
    return None if a is None else a.ctypes.data_as(ty)


NOALLOC_MAX_VERTICES = 2048 * 65536


def vertex_degree_noalloc(nv: int, d_rowptr: int, d_weight: int, d_vdeg_out: int,
                          stream: int = 0) -> float:
    """vg_vertex_degree_noalloc: degrees into the caller's device buffer d_vdeg_out
    (device pointers as integers, e.g. torch tensor .data_ptr()); returns 1/(2m).
    Allocates no device memory; see include/vite_b200.h for the limits."""
    err = C.create_string_buffer(512)
    c = C.c_double()
    st = lib().vg_vertex_degree_noalloc(nv, d_rowptr, d_weight, d_vdeg_out, C.byref(c),
                                        stream or None, err, len(err))
    if st != VG_OK:
        raise VgError(st, err.value.decode())
    return c.value


@dataclass
class Levels:
    stats: list
    comm: np.ndarray | None


class Graph:
    """A CSR resident on the device (vg_graph)."""

    def __init__(self, ctx: "Context", handle: C.c_void_p):
        self.ctx = ctx
        self.handle = handle

    @property
    def nv(self) -> int:
        nv = C.c_int64()
        lib().vg_graph_info(self.handle, C.byref(nv), None)
        return nv.value

    @property
    def ne(self) -> int:
        ne = C.c_int64()
        lib().vg_graph_info(self.handle, None, C.byref(ne))
        return ne.value

    def download(self):
        """(rowptr int64[nv+1], tail int64[ne], weight float64[ne]) in Vite's layout."""
        nv, ne = self.nv, self.ne
        rp = np.empty(nv + 1, np.int64)
        edges = np.empty(ne, EDGE_DTYPE)
        self.ctx._check(lib().vg_graph_download(self.ctx.handle, self.handle, _ptr(rp),
                                                edges.ctypes.data if ne else None))
        return rp, edges["tail"].copy(), edges["weight"].copy()

    def free(self):
        if self.handle:
            self.ctx._check(lib().vg_graph_free(self.ctx.handle, self.handle))
            self.handle = None

    def __del__(self):
        try:
            if self.handle and self.ctx.handle:
                lib().vg_graph_free(self.ctx.handle, self.handle)
                self.handle = None
        except Exception:
            pass


class Context:
    """vg_ctx: one device, one stream, an optional device-memory budget."""

    def __init__(self, device: int = 0, mem_budget: int = 0):
        h = C.c_void_p()
        st = lib().vg_ctx_create(device, mem_budget, C.byref(h))
        if st != VG_OK:
            raise VgError(st, f"vg_ctx_create(device={device}) failed")
        self.handle = h
        self.device = device

    def close(self):
        if self.handle:
            lib().vg_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int):
        if st != VG_OK:
            raise VgError(st, lib().vg_last_error(self.handle).decode())

    @property
    def bytes_in_use(self) -> int:
        return int(lib().vg_ctx_bytes_in_use(self.handle))

    def reserve(self, nbytes: int) -> None:
        """Pre-grow the device memory pool (no mid-run mapping up to this working set)."""
        self._check(lib().vg_ctx_reserve(self.handle, int(nbytes)))

    @property
    def stream(self) -> int:
        """cudaStream_t of the context, as an integer handle."""
        s = C.c_void_p()
        self._check(lib().vg_ctx_stream(self.handle, C.byref(s)))
        return s.value or 0

    def profile(self, enable: bool, reset: bool = True) -> tuple[float, int]:
        ms = C.c_double()
        n = C.c_int64()
        self._check(lib().vg_ctx_profile(self.handle, int(enable), C.byref(ms), C.byref(n),
                                         int(reset)))
        return ms.value, n.value

    # graphs ---------------------------------------------------------------------------
    def upload(self, rowptr, tail, weight) -> Graph:
        rowptr = np.ascontiguousarray(rowptr, dtype=np.int64)
        nv = len(rowptr) - 1
        ne = len(tail)
        edges = np.empty(ne, EDGE_DTYPE)
        edges["tail"] = tail
        edges["weight"] = weight
        h = C.c_void_p()
        self._check(lib().vg_graph_upload(self.handle, nv, ne, _ptr(rowptr),
                                          edges.ctypes.data if ne else None, C.byref(h)))
        return Graph(self, h)

    def upload_edges(self, rowptr: np.ndarray, edges: np.ndarray) -> Graph:
        """Upload from a Vite Edge array (structured int64 tail / float64 weight)."""
        h = C.c_void_p()
        self._check(lib().vg_graph_upload(self.handle, len(rowptr) - 1, len(edges), _ptr(rowptr),
                                          edges.ctypes.data if len(edges) else None, C.byref(h)))
        return Graph(self, h)

    def generate_rgg(self, n: int, extra_percent: float = 0.0, seed: int = 0) -> Graph:
        h = C.c_void_p()
        self._check(lib().vg_generate_rgg(self.handle, n, extra_percent, seed, C.byref(h)))
        return Graph(self, h)

    def generate_ba(self, n: int, m: int, seed: int) -> Graph:
        h = C.c_void_p()
        self._check(lib().vg_generate_ba(self.handle, n, m, seed, C.byref(h)))
        return Graph(self, h)

    def generate_er(self, n: int, avg_degree: float, seed: int) -> Graph:
        h = C.c_void_p()
        self._check(lib().vg_generate_er(self.handle, n, avg_degree, seed, C.byref(h)))
        return Graph(self, h)

    def reorder(self, g: Graph, mode: int = 1) -> None:
        """Store g in the locality layout (mode 1) or back in reference order (mode 0)."""
        self._check(lib().vg_graph_reorder(self.handle, g.handle, mode))

    def reweight(self, g: Graph, mode: int, seed: int = 0) -> None:
        self._check(lib().vg_graph_reweight(self.handle, g.handle, mode, seed))

    # the Louvain path ---------------------------------------------------------------
    def vertex_degree(self, g: Graph):
        vd = np.empty(g.nv, np.float64)
        c = C.c_double()
        self._check(lib().vg_vertex_degree(self.handle, g.handle, _ptr(vd, _f64p), C.byref(c)))
        return vd, c.value

    def louvain_phase(self, g: Graph, threshold: float = 1e-6, lower: float = -1.0,
                      et_type: int = 0, et_delta: float = 1.0, ordering: int = 0,
                      want_cvect: bool = True):
        p = PhaseParams(lower, threshold, et_type, et_delta, ordering)
        cv = np.empty(g.nv, np.int64) if want_cvect else None
        mod = C.c_double()
        it = C.c_int32()
        self._check(lib().vg_louvain_phase(self.handle, g.handle, C.byref(p), _ptr(cv),
                                           C.byref(mod), C.byref(it)))
        return cv, mod.value, it.value

    def color(self, g: Graph, n_hash: int, target_percent: int = 70, single: bool = False):
        out = np.empty(g.nv, np.int64)
        nc = C.c_int64()
        self._check(lib().vg_color(self.handle, g.handle, n_hash, target_percent, int(single),
                                   _ptr(out), C.byref(nc)))
        return out, nc.value

    def set_colors(self, g: Graph, colors: np.ndarray, num_colors: int) -> None:
        colors = np.ascontiguousarray(colors, dtype=np.int64)
        self._check(lib().vg_set_colors(self.handle, g.handle, _ptr(colors), num_colors))

    def rebuild(self, g: Graph, cvect: np.ndarray | None = None) -> None:
        cv = None if cvect is None else np.ascontiguousarray(cvect, dtype=np.int64)
        self._check(lib().vg_rebuild(self.handle, g.handle, _ptr(cv)))

    def run(self, g: Graph, threshold: float = 1e-6, coloring: bool = False,
            vertex_order: bool = False, max_colors: int = 8, single_color_iter: bool = False,
            et_type: int = 0, et_delta: float = 1.0, threshold_scaling: bool = False,
            one_phase: bool = False, want_comm: bool = False, max_levels: int = 256,
            layout: int = 2, comm_out: np.ndarray | None = None) -> Levels:
        """graphClustering's phase loop (vg_louvain_run). With want_comm, or a caller's
        int64 buffer `comm_out` of nv entries (pinned memory copies fastest), the -o map
        of level-0 vertices to final communities is returned as Levels.comm."""
        p = RunParams(threshold, int(coloring), int(vertex_order), max_colors,
                      int(single_color_iter), et_type, et_delta, int(threshold_scaling),
                      int(one_phase), layout)
        stats = (LevelStat * max_levels)()
        n = C.c_int32()
        if comm_out is not None:
            if (comm_out.dtype != np.int64 or comm_out.shape != (g.nv,)
                    or not comm_out.flags.c_contiguous):
                raise VgError(VG_ERR_ARG, "comm_out must be a contiguous int64 array of nv entries")
            comm = comm_out
        else:
            comm = np.empty(g.nv, np.int64) if want_comm else None
        self._check(lib().vg_louvain_run(self.handle, g.handle, C.byref(p), stats, max_levels,
                                         C.byref(n), _ptr(comm)))
        return Levels([stats[i].as_dict() for i in range(min(n.value, max_levels))], comm)

    def compare_communities(self, truth: np.ndarray, found: np.ndarray) -> dict:
        """compare_communities (compare.cpp:58-318) on the device: pair counts,
        precision, recall, F-score and Gini coefficients (truth first)."""
        a = np.ascontiguousarray(truth, dtype=np.int64)
        b = np.ascontiguousarray(found, dtype=np.int64)
        if len(a) != len(b):
            raise VgError(VG_ERR_ARG, "both community vectors need one label per vertex")
        st = CompareStats()
        self._check(lib().vg_compare_communities(self.handle, len(a), _ptr(a), _ptr(b),
                                                 C.byref(st)))
        return st.as_dict()

    def read_vite(self, path: str) -> Graph:
        """A Vite binary graph file straight into a device graph (vg_graph_read_vite)."""
        h = C.c_void_p()
        self._check(lib().vg_graph_read_vite(self.handle, os.fsencode(path), C.byref(h)))
        return Graph(self, h)

    def read_text(self, path: str, fmt: str, weights: str = "abs",
                  one_based: bool = False) -> Graph:
        """A text edge list parsed on the device (vg_graph_read_text): fmt 'simple' (-s),
        'snap' (-n) or 'mm' (-m); weights 'abs' (default), 'orig' (-i), 'one' (-w),
        'random' (-r); one_based is -z."""
        p = TextParams(TEXT_FORMATS[fmt], TEXT_WEIGHTS[weights], int(one_based))
        h = C.c_void_p()
        self._check(lib().vg_graph_read_text(self.handle, os.fsencode(path), C.byref(p),
                                             C.byref(h)))
        return Graph(self, h)

    def write_vite(self, g: Graph, path: str) -> None:
        """Write g as a Vite binary graph file, reference vertex order (vg_graph_write_vite)."""
        self._check(lib().vg_graph_write_vite(self.handle, g.handle, os.fsencode(path)))

    @property
    def tuning(self) -> dict:
        """The sweep launch tuning in use (vg_ctx_get_tuning)."""
        t = Tuning()
        self._check(lib().vg_ctx_get_tuning(self.handle, C.byref(t)))
        return t.as_dict()

    @tuning.setter
    def tuning(self, value: dict) -> None:
        t = Tuning(**{**self.tuning, **value})
        self._check(lib().vg_ctx_set_tuning(self.handle, C.byref(t)))

    def autotune(self, graphs: list, sweeps: int = 2) -> dict:
        """vg_autotune over `graphs`: sets and returns the fastest tuning found, with the
        summed sweep times (ms) of it and of the tuning it started from."""
        arr = (C.c_void_p * len(graphs))(*[g.handle for g in graphs])
        t = Tuning()
        best, start = C.c_double(), C.c_double()
        self._check(lib().vg_autotune(self.handle, arr, len(graphs), sweeps, C.byref(t),
                                      C.byref(best), C.byref(start)))
        return {"tuning": t.as_dict(), "sweep_ms": best.value, "start_sweep_ms": start.value}

    def batch(self, budget: int = 0) -> "Batch":
        return Batch(self, budget)

    def run_batch(self, graphs: list, threshold: float = 1e-6, want_comm: bool = False,
                  one_phase: bool = False, layout: int = 2) -> list:
        """Run every graph to completion as one batch; one Levels per graph, in order."""
        with Batch(self) as b:
            ids = [b.submit(g, threshold=threshold, one_phase=one_phase, want_comm=want_comm,
                            layout=layout) for g in graphs]
            b.run_all()
            return [b.result(j, want_comm=want_comm) for j in ids]


class Batch:
    """vg_batch: many graphs run together (batched and served Louvain).

    ``submit`` queues a graph with its run parameters; every ``step`` is one round
    (admit what fits the budget, one phase for every graph in the batch, retire
    the graphs whose level loop ended, rebuild the rest); ``poll`` lists the
    graphs finished since the last poll and ``result`` returns what ``Context.run``
    would have returned for the graph alone.
    """

    def __init__(self, ctx: "Context", budget: int = 0):
        self.ctx = ctx
        h = C.c_void_p()
        ctx._check(lib().vg_batch_create(ctx.handle, budget, C.byref(h)))
        self.handle = h
        self._nv: dict[int, int] = {}
        self._held: dict[int, Graph] = {}

    def submit(self, g: Graph, threshold: float = 1e-6, one_phase: bool = False,
               want_comm: bool = False, take: bool = False, layout: int = 2) -> int:
        """Queue g. With take=True the batch frees g once packed (g is emptied);
        otherwise g must stay alive until it is packed (the batch keeps a
        reference until the graph's job is polled as finished)."""
        p = RunParams(threshold, 0, 0, 8, 0, 0, 1.0, 0, int(one_phase), layout)
        flags = (VG_BATCH_TAKE if take else 0) | (VG_BATCH_COMM if want_comm else 0)
        jid = C.c_int64()
        nv = g.nv
        self.ctx._check(lib().vg_batch_submit(self.handle, g.handle, C.byref(p), flags,
                                              C.byref(jid)))
        if take:
            g.handle = None
        else:
            self._held[jid.value] = g
        self._nv[jid.value] = nv
        return jid.value

    def step(self) -> tuple[int, int]:
        r, q = C.c_int32(), C.c_int32()
        self.ctx._check(lib().vg_batch_step(self.handle, C.byref(r), C.byref(q)))
        return r.value, q.value

    def poll(self, max_ids: int = 65536) -> list[int]:
        ids = np.empty(max_ids, np.int64)
        n = C.c_int32()
        self.ctx._check(lib().vg_batch_poll(self.handle, _ptr(ids), max_ids, C.byref(n)))
        done = [int(x) for x in ids[:n.value]]
        for j in done:  # packed long ago: the caller's graph may go
            self._held.pop(j, None)
        return done

    def result(self, jid: int, want_comm: bool = False, max_levels: int = 256) -> Levels:
        stats = (LevelStat * max_levels)()
        n = C.c_int32()
        comm = np.empty(self._nv[jid], np.int64) if want_comm else None
        self.ctx._check(lib().vg_batch_result(self.handle, jid, stats, max_levels, C.byref(n),
                                              _ptr(comm)))
        return Levels([stats[i].as_dict() for i in range(min(n.value, max_levels))], comm)

    def forget(self, jid: int) -> None:
        self.ctx._check(lib().vg_batch_forget(self.handle, jid))
        self._nv.pop(jid, None)

    def stats(self) -> dict:
        s = BatchStats()
        self.ctx._check(lib().vg_batch_get_stats(self.handle, C.byref(s)))
        return s.as_dict()

    def run_all(self) -> None:
        """Step until nothing is queued or running."""
        while True:
            r, q = self.step()
            if r == 0 and q == 0:
                break

    def close(self) -> None:
        if self.handle:
            self.ctx._check(lib().vg_batch_destroy(self.handle))
            self.handle = None
        self._held = {}

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            if self.handle:
                lib().vg_batch_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


@dataclass
class LevelOut:
    nv: int
    ne: int
    iters: int
    mod: float
    num_colors: int
    cvect: np.ndarray


def run_levels(ctx: Context, g: Graph, threshold: float = 1e-6, coloring: bool = False,
               vertex_order: bool = False, max_colors: int = 8, single_color_iter: bool = False,
               et_type: int = 0, et_delta: float = 1.0, threshold_scaling: bool = False,
               one_phase: bool = False) -> list[LevelOut]:
    """graphClustering's phase loop (main.cpp:242-513) driven from the host through the
    per-operator entry points, returning every level's community vector. The graph g is
    coarsened in place, as distbuildNextLevelGraph replaces the DistGraph it is given."""
    out: list[LevelOut] = []
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
        ordering = 0
        if (coloring or vertex_order) and phase == 0:
            _, ncol = ctx.color(g, max_colors // 2, 70, single_color_iter)
            ordering = 1 if coloring else 2
        nv, ne = g.nv, g.ne
        cv, currMod, iters = ctx.louvain_phase(g, thr, currMod, et_type, et_delta, ordering)
        tot_iters += iters
        out.append(LevelOut(nv, ne, iters, currMod, ncol, cv))
        if currMod - prevMod > thr:
            if not one_phase:
                ctx.rebuild(g)
        else:
            if threshold_scaling and not one_phase and phase < 10:
                cv, currMod, iters = ctx.louvain_phase(g, 1e-6, currMod)
                out.append(LevelOut(g.nv, g.ne, iters, currMod, 0, cv))
            break
        prevMod, currMod = currMod, -1.0
        phase += 1
        if one_phase:
            break
        if threshold_scaling and not one_phase:
            short_phase += 1
        if phase == 200 or tot_iters > 10000:
            break
    return out
