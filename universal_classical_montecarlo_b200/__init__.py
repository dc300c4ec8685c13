"""B200 engine for the local-update hot path of universal_monte_carlo.

The engine is ``libumc_b200.so`` (hand-written sm_100a CUDA behind the C ABI in
``include/umc_b200.h``).  This module binds that ABI with ctypes and mirrors the
reference's user-facing names so scripts read like the reference's tests:

=====================  ================================================
reference              here
=====================  ================================================
PairGraph(n, edges)    ``PairGraph(n, edges, symmetric=True)``
square_lattice(Lx,Ly)  ``square_lattice(Lx, Ly)``
(3D by hand)           ``cubic_lattice(Lx, Ly, Lz)``
CellComplex<4>         ``CellComplex(n_sites, cells)``
hypercubic_plaquettes  ``hypercubic_plaquettes(L)``
Ising / VectorSpin<N>  ``Ising(graph, J)`` / ``VectorSpin(N, graph, J)``
XY (angles, PairModel) ``XYAngle(graph, J)``
U1Gauge / SUGauge<N>   ``U1Gauge(cells, beta)`` / ``SUGauge(N, cells, beta)``
Metropolis<M,Q,R>      ``Metropolis(model, proposal, rng, beta)``
Wolff<M,A,R>           ``Wolff(model, axis, rng, beta)``
Pcg32(seed, stream)    ``Pcg32(seed, stream)`` (keys the counter streams)
=====================  ================================================

There is no CPU fallback: importing this module fails if the library was not
built, and creating a model fails (``UmcError``) on a host without a GPU.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libumc_b200.so")

if not os.path.isfile(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python universal_classical_montecarlo_b200/_build.py`"
    )
lib = C.CDLL(LIB_PATH)

# ------------------------------------------------------------------ constants
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_OUT_OF_RANGE = 2
ERR_OVERFLOW = 3
ERR_UNSUPPORTED = 4
ERR_CUDA = 5
ERR_DEVICE_TIMEOUT = 6
ERR_OUT_OF_MEMORY = 7
ERR_STATE = 8

MODEL_ISING = 1
MODEL_VECTOR = 2
MODEL_XY_ANGLE = 3
MODEL_U1 = 4
MODEL_SU = 5

PROPOSAL_FLIP = 1
PROPOSAL_SPHERE = 2
PROPOSAL_ROTATION = 3
PROPOSAL_U1SHIFT = 4
PROPOSAL_SUSHIFT = 5

AXIS_NONE = 0
AXIS_FIXED = 1
AXIS_SPHERE = 2

OBS_STRIDE = 8


class UmcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[umc status {code}] {msg}")
        self.code = code


def _exc(code: int, msg: str) -> Exception:
    # the reference builders' exception types
    if code == ERR_INVALID_ARGUMENT:
        return ValueError(msg)
    if code == ERR_OUT_OF_RANGE:
        return IndexError(msg)
    if code == ERR_OVERFLOW:
        return OverflowError(msg)
    return UmcError(code, msg)


_vp = C.c_void_p
_u32 = C.c_uint32
_u64 = C.c_uint64
_i32 = C.c_int32
_f64 = C.c_double
_int = C.c_int


class ChainDesc(C.Structure):
    _fields_ = [
        ("model", _i32),
        ("components", _i32),
        ("graph", _vp),
        ("cells", _vp),
        ("coupling", _f64),
        ("proposal", _i32),
        ("width", _f64),
        ("hits", _u32),
        ("wolff_axis", _i32),
        ("seed", _u64),
        ("device", _i32),
        ("stream", _vp),
        ("max_records", _u64),
    ]


def _decl(name, restype, *args):
    f = getattr(lib, name)
    f.restype = restype
    f.argtypes = list(args)
    return f


_last_error = _decl("umc_last_error", C.c_char_p)
_decl("umc_abi_version", _int)
_decl("umc_device_count", _int, C.POINTER(_int))
_decl("umc_graph_create", _int, _u64, _vp, _vp, _u64, _int, C.POINTER(_vp))
_decl("umc_graph_square", _int, _u64, _u64, C.POINTER(_vp))
_decl("umc_graph_cubic", _int, _u64, _u64, _u64, C.POINTER(_vp))
_decl("umc_graph_destroy", None, _vp)
_decl("umc_graph_sites", _u64, _vp)
_decl("umc_graph_slots", _u64, _vp)
_decl("umc_graph_csr", _int, _vp, _vp, _vp)
_decl("umc_graph_create_payload", _int, _u64, _vp, _vp, _u64, _int, _vp, _u32, C.POINTER(_vp))
_decl("umc_graph_payload_bytes", _u32, _vp)
_decl("umc_graph_payloads", _int, _vp, _vp)
_decl("umc_graph_slot_edges", _int, _vp, _vp)
_decl("umc_graph_colouring", _int, _vp, _vp, _vp, _vp)
_decl("umc_cells_create", _int, _u64, _u32, _vp, _u64, C.POINTER(_vp))
_decl("umc_cells_hypercubic", _int, _u64, C.POINTER(_vp))
_decl("umc_cells_square_plaquettes", _int, _u64, C.POINTER(_vp))
_decl("umc_cells_destroy", None, _vp)
_decl("umc_cells_sites", _u64, _vp)
_decl("umc_cells_count", _u64, _vp)
_decl("umc_cells_arity", _u32, _vp)
_decl("umc_cells_table", _int, _vp, _vp)
_decl("umc_cells_incidence", _int, _vp, _vp, _vp, _vp)
_decl("umc_cells_colouring", _int, _vp, _vp, _vp, _vp)
_decl("umc_chain_create", _int, C.POINTER(ChainDesc), C.POINTER(_vp))
_decl("umc_chain_destroy", _int, _vp)
_decl("umc_chain_set_field", _int, _vp, _vp)
_decl("umc_chain_get_field", _int, _vp, _vp)
_decl("umc_chain_upload_async", _int, _vp, _vp)
_decl("umc_batch_set_state", _int, _vp, _u64, _u64, _u64, _vp)
_decl("umc_chain_checkpoint_bytes", _int, _vp, C.POINTER(_u64))
_decl("umc_chain_checkpoint", _int, _vp, _vp, _u64)
_decl("umc_chain_restore", _int, _vp, _vp, _u64)
_decl("umc_chain_set_record_streaming", _int, _vp, _int)
_decl("umc_chain_randomize", _int, _vp, _u64)
_decl("umc_chain_set_proposal", _int, _vp, _i32, _f64, _u32)
_decl("umc_chain_set_wolff_axis", _int, _vp, _i32)
_decl("umc_chain_set_seed", _int, _vp, _u64)
_decl("umc_chain_counters", _int, _vp, C.POINTER(_u64), C.POINTER(_u64))
_decl("umc_chain_set_counters", _int, _vp, _u64, _u64)
_decl("umc_chain_stream", _vp, _vp)
_decl("umc_chain_sync", _int, _vp)
_decl("umc_chain_observe", _int, _vp, _vp)
_decl("umc_metropolis_run", _int, _vp, _f64, _u64, _vp)
_decl("umc_wolff_run", _int, _vp, _f64, _u64, _vp, _vp)
_decl("umc_hybrid_run", _int, _vp, _f64, _u64, _vp, _vp)
_decl("umc_metropolis_enqueue", _int, _vp, _f64, _u64)
_decl("umc_wolff_enqueue", _int, _vp, _f64, _u64)
_decl("umc_hybrid_enqueue", _int, _vp, _f64, _u64)
_decl("umc_chain_fetch", _int, _vp, _vp, _vp, _u64, C.POINTER(_u64))
_decl("umc_wolff_stats", _int, _vp, C.POINTER(_u64), C.POINTER(_f64))
_decl("umc_chain_set_timing", _int, _vp, _int)
_decl("umc_chain_set_fused", _int, _vp, _int)


class BatchDesc(C.Structure):
    _fields_ = [
        ("n_ladders", _u32),
        ("replicas", _u32),
        ("L", _vp),
        ("betas", _vp),
        ("coupling", _f64),
        ("width", _f64),
        ("sweeps_per_exchange", _u32),
        ("seed", _u64),
        ("device", _i32),
        ("stream", _vp),
        ("max_records", _u64),
        ("first_ladder", _u32),
    ]


_decl("umc_batch_create", _int, C.POINTER(BatchDesc), C.POINTER(_vp))
_decl("umc_batch_set_persistent", _int, _vp, _int)
_decl("umc_batch_set_persistent_config", _int, _vp, _u32, _u32)
_decl("umc_batch_persistent_info", _int, _vp, C.POINTER(_int), C.POINTER(_u32), C.POINTER(_u32), C.POINTER(_u32),
      C.POINTER(_u32), C.POINTER(_u32))
_decl("umc_batch_destroy", _int, _vp)
_decl("umc_batch_randomize", _int, _vp, _u64)
_decl("umc_batch_set_field", _int, _vp, _u32, _vp)
_decl("umc_batch_get_field", _int, _vp, _u32, _vp)
_decl("umc_batch_enqueue", _int, _vp, _u64)
_decl("umc_batch_fetch", _int, _vp, _vp, _u64, C.POINTER(_u64))
_decl("umc_batch_run", _int, _vp, _u64, _vp)
_decl("umc_batch_counters", _int, _vp, C.POINTER(_u64), C.POINTER(_u64), C.POINTER(_u64))
_decl("umc_batch_temperature_map", _int, _vp, _vp)
_decl("umc_batch_seeds", _int, _vp, _vp, _vp)
_decl("umc_batch_config", _int, _vp, _u32, C.POINTER(_u32), C.POINTER(_u32), C.POINTER(_u32))
_decl("umc_batch_sites", _int, _vp, C.POINTER(_u64), C.POINTER(_u64))
_decl("umc_batch_stream", _vp, _vp)
_decl("umc_chain_kernel_stats", _int, _vp, _vp, _vp, _int)

KERNEL_KINDS = ["metropolis", "wolff_union", "wolff_flip", "observe", "gauge", "batch", "learned", "other",
                "wolff_merge", "fused"]


def check(code: int) -> None:
    if code != OK:
        raise _exc(code, (_last_error() or b"").decode())


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_vp)


def device_count() -> int:
    n = _int(0)
    check(lib.umc_device_count(C.byref(n)))
    return n.value


# ================================================================== self-test
_decl("umc_selftest_barrier_timeout", _int, _i32, C.POINTER(_u32))


def selftest_barrier_timeout(device: int = 0):
    """Runs the engine's bounded grid barrier on a barrier that never completes.
    Returns (status code, status bits): ERR_DEVICE_TIMEOUT and bit 8 when the
    bound works."""
    bits = _u32(0)
    code = lib.umc_selftest_barrier_timeout(device, C.byref(bits))
    return code, bits.value


# ================================================================= statistics
_decl("umc_tau_int", _int, _vp, _u64, _f64, C.POINTER(_f64), C.POINTER(_f64), C.POINTER(_u64))
_decl("umc_binning_error", _int, _vp, _u64, _u64, C.POINTER(_f64), C.POINTER(_f64))


def tau_int(series, c: float = 6.0):
    """Integrated autocorrelation time with Sokal's automatic window.

    Returns ``(tau, tau_err, window)``; tau = 1/2 + sum_{t<=W} rho(t)."""
    x = np.ascontiguousarray(series, dtype=np.float64)
    t, e, w = _f64(), _f64(), _u64()
    check(lib.umc_tau_int(_ptr(x), x.size, c, C.byref(t), C.byref(e), C.byref(w)))
    return t.value, e.value, w.value


_decl("umc_tau_int_multi", _int, _vp, _u64, _u64, _f64, C.POINTER(_f64), C.POINTER(_f64), C.POINTER(_u64))


def tau_int_multi(series, c: float = 6.0):
    """Pooled tau_int of independent chains: ``series`` is (chains, length).
    Returns ``(tau, tau_err, window)``; window == length // 2 means the estimate
    did not converge inside the series."""
    x = np.ascontiguousarray(series, dtype=np.float64)
    if x.ndim != 2:
        raise ValueError("series must be (chains, length)")
    t, e, w = _f64(), _f64(), _u64()
    check(lib.umc_tau_int_multi(_ptr(x), x.shape[0], x.shape[1], c, C.byref(t), C.byref(e), C.byref(w)))
    return t.value, e.value, w.value


def binning_error(series, bin: int):
    """Mean and its standard error from bins of ``bin`` consecutive values."""
    x = np.ascontiguousarray(series, dtype=np.float64)
    m, e = _f64(), _f64()
    check(lib.umc_binning_error(_ptr(x), x.size, bin, C.byref(m), C.byref(e)))
    return m.value, e.value


_decl("umc_obs_stream_create", _int, C.c_char_p, _u32, _vp, _u64, _u64, _i32, _f64, C.POINTER(_vp))
_decl("umc_obs_stream_append", _int, _vp, _vp, _u64)
_decl("umc_obs_stream_close", _int, _vp)
_decl("umc_obs_stream_info", _int, C.c_char_p, C.POINTER(_u32), C.POINTER(_u64), C.POINTER(_u64), C.POINTER(_u64),
      C.POINTER(_i32), C.POINTER(_f64), _vp)
_decl("umc_obs_stream_read", _int, C.c_char_p, _u64, _u64, _vp)


class ObsStream:
    """umc_obs_stream_*: a per-sweep (or per-flip) FP64 observable series
    written to disk as it is produced, for offline tau_int of long runs.

        with ObsStream(path, ["E", "Mx", "My", "Mz"], seed=1, first=0) as s:
            s.append(chain.metropolis(beta, 1000)[:, :4])
        meta, data = read_obs_stream(path)
    """

    def __init__(self, path, names, seed: int = 0, first: int = 0, model: int = 0, beta: float = 0.0):
        self.columns = len(names)
        arr = (C.c_char_p * self.columns)(*[n.encode() for n in names])
        h = _vp()
        check(lib.umc_obs_stream_create(os.fspath(path).encode(), self.columns, C.cast(arr, _vp), seed, first, model,
                                        beta, C.byref(h)))
        self._h = h

    def append(self, records) -> None:
        r = np.ascontiguousarray(records, np.float64).reshape(-1, self.columns)
        check(lib.umc_obs_stream_append(self._h, _ptr(r), r.shape[0]))

    def close(self) -> None:
        if self._h:
            h, self._h = self._h, None
            check(lib.umc_obs_stream_close(h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        if getattr(self, "_h", None) and lib is not None:  # the library may be gone at interpreter exit
            lib.umc_obs_stream_close(self._h)
            self._h = None


def read_obs_stream(path, first: int = 0, n: int | None = None):
    """(meta, records): the stream's header fields and records [first, first + n)."""
    p = os.fspath(path).encode()
    cols, recs, seed, f0, beta, model = _u32(), _u64(), _u64(), _u64(), _f64(), _i32()
    check(lib.umc_obs_stream_info(p, C.byref(cols), C.byref(recs), C.byref(seed), C.byref(f0), C.byref(model),
                                  C.byref(beta), None))
    names = C.create_string_buffer(32 * cols.value)
    check(lib.umc_obs_stream_info(p, None, None, None, None, None, None, names))
    count = recs.value - first if n is None else n
    out = np.zeros((count, cols.value))
    check(lib.umc_obs_stream_read(p, first, count, _ptr(out)))
    raw = names.raw
    meta = {"names": [raw[32 * c:32 * (c + 1)].split(b"\0", 1)[0].decode() for c in range(cols.value)],
            "records": recs.value, "seed": seed.value, "first": f0.value, "model": model.value, "beta": beta.value}
    return meta, out


# ===================================================================== tables
class PairGraph:
    """PairGraph(n, edges, symmetric) -- lattice/pair_graph.hpp:49-83.

    payload: optional per-edge records (PairGraph<P>'s Edge::c), a numpy array
    with one row (or element) per edge, e.g. float64 couplings or a structured
    dtype; each is copied into both directed slots as the reference copies c."""

    def __init__(self, n_sites: int = 0, edges=None, symmetric: bool = True, payload=None, _handle=None):
        if _handle is not None:
            self._h = _handle
            self.payload_dtype = None
            return
        e = np.zeros((0, 2), np.uint32) if edges is None else np.asarray(edges)
        e = np.ascontiguousarray(e.reshape(-1, 2))
        if e.size and (e.min() < 0 or e.max() > 0xFFFFFFFF):
            raise IndexError("PairGraph: edge endpoint out of range")
        ei = np.ascontiguousarray(e[:, 0], np.uint32)
        ej = np.ascontiguousarray(e[:, 1], np.uint32)
        h = _vp()
        self.payload_dtype = None
        if payload is None:
            check(lib.umc_graph_create(n_sites, _ptr(ei), _ptr(ej), len(ei), int(symmetric), C.byref(h)))
        else:
            pay = np.ascontiguousarray(payload)
            if len(pay) != len(ei):
                raise ValueError("PairGraph: one payload record per edge")
            rec = pay.reshape(len(ei), -1) if pay.ndim > 1 else pay.reshape(len(ei))
            nbytes = rec.itemsize * (rec.shape[1] if rec.ndim > 1 else 1)
            self.payload_dtype = (pay.dtype, pay.shape[1:])
            check(lib.umc_graph_create_payload(n_sites, _ptr(ei), _ptr(ej), len(ei), int(symmetric), _ptr(rec),
                                               nbytes, C.byref(h)))
        self._h = h

    def payloads(self):
        """Bond<P>::c of every CSR slot, in umc_graph_csr's slot order."""
        if self.payload_dtype is None:
            raise ValueError("graph has no payload")
        dt, shape = self.payload_dtype
        out = np.zeros((int(lib.umc_graph_slots(self._h)),) + tuple(shape), dt)
        check(lib.umc_graph_payloads(self._h, _ptr(out)))
        return out

    def slot_edges(self):
        """The input edge of every CSR slot."""
        out = np.zeros(int(lib.umc_graph_slots(self._h)), np.uint32)
        check(lib.umc_graph_slot_edges(self._h, _ptr(out)))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:  # the library may be gone at interpreter exit
            lib.umc_graph_destroy(h)
            self._h = None

    def sites(self) -> int:
        return int(lib.umc_graph_sites(self._h))

    def csr(self):
        n = self.sites()
        off = np.zeros(n + 1, np.uint32)
        bonds = np.zeros(int(lib.umc_graph_slots(self._h)), np.uint32)
        check(lib.umc_graph_csr(self._h, _ptr(off), _ptr(bonds)))
        return off, bonds

    def degree(self, i: int) -> int:
        off, _ = self.csr()
        return int(off[i + 1] - off[i])

    def colouring(self):
        """(n_colours, colour[n], position[n]) of the colour passes."""
        n = self.sites()
        nc = _u32(0)
        col = np.zeros(n, np.uint32)
        pos = np.zeros(n, np.uint32)
        check(lib.umc_graph_colouring(self._h, C.byref(nc), _ptr(col), _ptr(pos)))
        return nc.value, col, pos


def square_lattice(Lx: int, Ly: int) -> PairGraph:
    """square_lattice(Lx, Ly) -- lattice/square.hpp:15-38."""
    h = _vp()
    check(lib.umc_graph_square(Lx, Ly, C.byref(h)))
    return PairGraph(_handle=h)


def cubic_lattice(Lx: int, Ly: int, Lz: int) -> PairGraph:
    """Periodic cubic lattice with square_lattice's conventions (no reference builder)."""
    h = _vp()
    check(lib.umc_graph_cubic(Lx, Ly, Lz, C.byref(h)))
    return PairGraph(_handle=h)


class CellComplex:
    """CellComplex<A>(sites, cells) -- lattice/cell_complex.hpp:36-63."""

    def __init__(self, n_sites: int = 0, cells=None, _handle=None):
        if _handle is not None:
            self._h = _handle
            return
        c = np.ascontiguousarray(np.asarray(cells), np.uint32)
        if c.ndim != 2:
            raise ValueError("cells must be (n_cells, arity)")
        h = _vp()
        check(lib.umc_cells_create(n_sites, c.shape[1], _ptr(c), c.shape[0], C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:  # the library may be gone at interpreter exit
            lib.umc_cells_destroy(h)
            self._h = None

    def sites(self) -> int:
        return int(lib.umc_cells_sites(self._h))

    def cells(self) -> int:
        return int(lib.umc_cells_count(self._h))

    def table(self):
        a = int(lib.umc_cells_arity(self._h))
        t = np.zeros((self.cells(), a), np.uint32)
        check(lib.umc_cells_table(self._h, _ptr(t)))
        return t

    def incidence(self):
        n = self.sites()
        tot = self.cells() * int(lib.umc_cells_arity(self._h))
        off = np.zeros(n + 1, np.uint64)
        ic = np.zeros(tot, np.uint32)
        iw = np.zeros(tot, np.uint8)
        check(lib.umc_cells_incidence(self._h, _ptr(off), _ptr(ic), _ptr(iw)))
        return off, ic, iw

    def colouring(self):
        n = self.sites()
        nc = _u32(0)
        col = np.zeros(n, np.uint32)
        pos = np.zeros(n, np.uint32)
        check(lib.umc_cells_colouring(self._h, C.byref(nc), _ptr(col), _ptr(pos)))
        return nc.value, col, pos


def hypercubic_plaquettes(L: int) -> CellComplex:
    """hypercubic_plaquettes(L) -- lattice/hypercubic.hpp:15-64."""
    h = _vp()
    check(lib.umc_cells_hypercubic(L, C.byref(h)))
    return CellComplex(_handle=h)


def square_plaquettes(L: int) -> CellComplex:
    """Periodic 2D plaquette complex with the hypercubic orientation rule."""
    h = _vp()
    check(lib.umc_cells_square_plaquettes(L, C.byref(h)))
    return CellComplex(_handle=h)


# ===================================================================== chains
class Chain:
    """One model's field on one GPU (the C ABI's umc_chain)."""

    def __init__(self, model: int, *, graph: PairGraph | None = None, cells: CellComplex | None = None,
                 components: int = 1, coupling: float = 1.0, proposal: int = 0, width: float = 0.0,
                 hits: int = 1, wolff_axis: int = AXIS_NONE, seed: int = 1, device: int = 0,
                 stream: int | None = None, max_records: int = 0):
        d = ChainDesc()
        d.model = model
        d.components = components
        d.graph = graph._h if graph is not None else None
        d.cells = cells._h if cells is not None else None
        d.coupling = coupling
        d.proposal = proposal
        d.width = width
        d.hits = hits
        d.wolff_axis = wolff_axis
        d.seed = seed
        d.device = device
        d.stream = stream
        d.max_records = max_records
        h = _vp()
        check(lib.umc_chain_create(C.byref(d), C.byref(h)))
        self._h = h
        self.model = model
        self.components = components
        self._graph = graph
        self._cells = cells
        if model == MODEL_ISING:
            self.dtype, self.comps = np.int8, 1
        elif model == MODEL_VECTOR:
            self.dtype, self.comps = np.float32, components
        elif model in (MODEL_XY_ANGLE, MODEL_U1):
            self.dtype, self.comps = np.float32, 1
        else:
            self.dtype, self.comps = np.float32, components * components * 2
        self.n = graph.sites() if graph is not None else cells.sites()
        self._inflight = []  # host arrays of uploads that may still be copying

    def close(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:  # module globals are gone at interpreter exit
            lib.umc_chain_destroy(h)
        self._h = None
        self._inflight = []

    def __del__(self):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_field(self, field) -> None:
        a = np.ascontiguousarray(np.asarray(field, self.dtype).reshape(-1))
        if a.size != self.n * self.comps:
            raise ValueError(f"field has {a.size} scalars, expected {self.n * self.comps}")
        check(lib.umc_chain_set_field(self._h, _ptr(a)))

    def upload_async(self, field) -> None:
        """umc_chain_upload_async: the array is kept alive until the next
        synchronising call; pinned memory (torch pin_memory) makes the copy
        asynchronous."""
        a = np.asarray(field)
        if a.dtype != self.dtype or not a.flags.c_contiguous:
            raise ValueError(f"upload_async needs a C-contiguous {np.dtype(self.dtype).name} array")
        if a.size != self.n * self.comps:
            raise ValueError(f"field has {a.size} scalars, expected {self.n * self.comps}")
        check(lib.umc_chain_upload_async(self._h, _ptr(a)))
        self._inflight.append(a)

    def checkpoint(self) -> bytes:
        """umc_chain_checkpoint: header + field; restore() continues the chain
        exactly, in this process or another."""
        n = _u64(0)
        check(lib.umc_chain_checkpoint_bytes(self._h, C.byref(n)))
        buf = np.zeros(n.value, np.uint8)
        check(lib.umc_chain_checkpoint(self._h, _ptr(buf), n.value))
        return buf.tobytes()

    def restore(self, image: bytes) -> None:
        buf = np.frombuffer(image, np.uint8)
        check(lib.umc_chain_restore(self._h, _ptr(buf), buf.size))

    def save(self, path) -> None:
        with open(path, "wb") as f:
            f.write(self.checkpoint())

    def load(self, path) -> None:
        with open(path, "rb") as f:
            self.restore(f.read())

    def set_record_streaming(self, enable: bool) -> None:
        check(lib.umc_chain_set_record_streaming(self._h, int(enable)))

    def get_field(self) -> np.ndarray:
        self._inflight = []
        a = np.zeros(self.n * self.comps, self.dtype)
        check(lib.umc_chain_get_field(self._h, _ptr(a)))
        return a.reshape(self.n, self.comps) if self.comps > 1 else a

    def randomize(self, seed: int) -> None:
        check(lib.umc_chain_randomize(self._h, seed))

    def set_proposal(self, proposal: int, width: float = 0.0, hits: int = 1) -> None:
        check(lib.umc_chain_set_proposal(self._h, proposal, width, hits))

    def set_wolff_axis(self, axis: int) -> None:
        check(lib.umc_chain_set_wolff_axis(self._h, axis))

    def set_seed(self, seed: int) -> None:
        check(lib.umc_chain_set_seed(self._h, seed))

    def counters(self):
        s, f = _u64(0), _u64(0)
        check(lib.umc_chain_counters(self._h, C.byref(s), C.byref(f)))
        return s.value, f.value

    def set_counters(self, sweeps: int, flips: int) -> None:
        check(lib.umc_chain_set_counters(self._h, sweeps, flips))

    def stream(self) -> int:
        return lib.umc_chain_stream(self._h) or 0

    def sync(self) -> None:
        check(lib.umc_chain_sync(self._h))
        self._inflight = []

    def observe(self) -> np.ndarray:
        r = np.zeros(OBS_STRIDE)
        check(lib.umc_chain_observe(self._h, _ptr(r)))
        return r

    def metropolis(self, beta: float, n: int, records: bool = True):
        rec = np.zeros((n, OBS_STRIDE)) if records else None
        check(lib.umc_metropolis_run(self._h, beta, n, _ptr(rec)))
        return rec

    def wolff(self, beta: float, n: int, records: bool = True):
        sizes = np.zeros(n, np.uint64)
        rec = np.zeros((n, OBS_STRIDE)) if records else None
        check(lib.umc_wolff_run(self._h, beta, n, _ptr(sizes), _ptr(rec)))
        return sizes, rec

    def hybrid(self, beta: float, n: int):
        sizes = np.zeros(n, np.uint64)
        rec = np.zeros((n, OBS_STRIDE))
        check(lib.umc_hybrid_run(self._h, beta, n, _ptr(sizes), _ptr(rec)))
        return sizes, rec

    def enqueue_metropolis(self, beta: float, n: int) -> None:
        check(lib.umc_metropolis_enqueue(self._h, beta, n))

    def enqueue_wolff(self, beta: float, n: int) -> None:
        check(lib.umc_wolff_enqueue(self._h, beta, n))

    def enqueue_hybrid(self, beta: float, n: int) -> None:
        check(lib.umc_hybrid_enqueue(self._h, beta, n))

    def fetch(self, capacity: int):
        rec = np.zeros((capacity, OBS_STRIDE))
        sizes = np.zeros(capacity, np.uint64)
        got = _u64(0)
        check(lib.umc_chain_fetch(self._h, _ptr(rec), _ptr(sizes), capacity, C.byref(got)))
        self._inflight = []
        return rec[: got.value], sizes[: got.value]

    def set_fused(self, enable: bool) -> None:
        check(lib.umc_chain_set_fused(self._h, int(enable)))

    def set_timing(self, enable: bool) -> None:
        check(lib.umc_chain_set_timing(self._h, int(enable)))

    def kernel_stats(self, reset: bool = False) -> dict:
        """{kind: (launches, device_ms)} for the chain's kernels."""
        n = np.zeros(len(KERNEL_KINDS), np.uint64)
        ms = np.zeros(len(KERNEL_KINDS))
        check(lib.umc_chain_kernel_stats(self._h, _ptr(n), _ptr(ms), int(reset)))
        return {k: (int(n[i]), float(ms[i])) for i, k in enumerate(KERNEL_KINDS)}

    def wolff_stats(self):
        f, s = _u64(0), _f64(0)
        check(lib.umc_wolff_stats(self._h, C.byref(f), C.byref(s)))
        return f.value, s.value


def shard_range(n_units: int, rank: int, world: int):
    """The contiguous range [lo, hi) of n_units independent units (ladders,
    chains) that rank `rank` of `world` owns: sizes differ by at most one,
    lower ranks take the larger shares."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    q, r = divmod(n_units, world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def gather_shards(local, group=None):
    """All ranks' arrays (e.g. the records of their shards, ladders or chains
    along axis 1) concatenated in rank order along axis 1, on every rank,
    through torch.distributed (gloo on CPU, NCCL on GPUs)."""
    import torch.distributed as dist

    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, np.asarray(local), group=group)
    return np.concatenate(parts, axis=1)


class SlabDesc(C.Structure):
    _fields_ = [
        ("model", _i32),
        ("components", _i32),
        ("Lx", _u32),
        ("Ly", _u32),
        ("Lz", _u32),
        ("first_plane", _u32),
        ("planes", _u32),
        ("coupling", _f64),
        ("proposal", _i32),
        ("width", _f64),
        ("seed", _u64),
        ("device", _i32),
    ]


_decl("umc_slab_create", _int, C.POINTER(SlabDesc), C.POINTER(_vp))
_decl("umc_slab_destroy", _int, _vp)
_decl("umc_slab_local_sites", _u64, _vp)
_decl("umc_slab_row_split", _u32, _vp)
_decl("umc_slab_pass", _int, _vp, _vp, _f64, _u64, _u32, _vp)
_decl("umc_slab_record", _int, _vp, _vp, _vp)
_decl("umc_slab_wolff_local", _int, _vp, _vp, _f64, _u64, _vp)
_decl("umc_slab_wolff_boundary", _int, _vp, _vp, _vp, _vp, _vp)
_decl("umc_slab_wolff_seed", _int, _vp, _u64, C.POINTER(_u32), C.POINTER(_u32), _vp)
_decl("umc_slab_wolff_merge", _int, _u32, _u32, _vp, _vp, _vp, _u32, _u32, _vp, _vp, _u32, _vp, C.POINTER(_u32))
_decl("umc_slab_wolff_flip", _int, _vp, _vp, _u64, _vp, _u32, C.POINTER(_u64), _vp)


class SlabChain:
    """One periodic Lx x Ly x Lz lattice (Lz = 1 in 2D) split into slabs over
    the ranks of a torch.distributed group, one process per GPU (umc_slab_*):
    this rank's planes along z (3D) or y (2D) plus a halo plane on each side
    live in a torch tensor on its GPU; each colour pass is followed by an
    exchange of the boundary planes with the two neighbouring ranks
    (batch_isend_irecv: NCCL device to device, gloo through host copies).
    Without a process group (world 1) the halos are the slab's own periodic
    planes.  The ranks together run exactly the single-GPU Chain of the same
    seed (keys of global site indices); records are summed over the ranks."""

    def __init__(self, model, dims, *, rank=0, world=1, group=None, components=1, coupling=1.0,
                 proposal=None, width=0.0, seed=1, device=0):
        import torch

        self.torch = torch
        Lx, Ly, Lz = (tuple(dims) + (1,))[:3]
        self.dims = (Lx, Ly, Lz)
        self.rank, self.world, self.group = rank, world, group
        total = Lz if Lz > 1 else Ly
        lo, hi = shard_range(total, rank, world)
        self.planes_range = (lo, hi)
        self.planes = hi - lo
        self.P = Lx * Ly if Lz > 1 else Lx
        self.model = model
        self.N = components if model == MODEL_VECTOR else 1
        if proposal is None:
            proposal = PROPOSAL_FLIP if model == MODEL_ISING else PROPOSAL_SPHERE
        d = SlabDesc()
        d.model, d.components, d.Lx, d.Ly, d.Lz = model, self.N, Lx, Ly, Lz
        d.first_plane, d.planes, d.coupling, d.proposal, d.width = lo, self.planes, coupling, proposal, width
        d.seed, d.device = seed, device
        h = _vp()
        check(lib.umc_slab_create(C.byref(d), C.byref(h)))
        self._h = h
        self.nloc = int(lib.umc_slab_local_sites(h))
        # 2D Ising with Lx / 2 a multiple of 16: each row stored split by colour
        self.row_split = bool(lib.umc_slab_row_split(h))
        self.device = torch.device("cuda", device)
        dt = torch.int8 if model == MODEL_ISING else torch.float32
        self.field = torch.zeros(self.N * self.nloc, dtype=dt, device=self.device)
        self.stream = torch.cuda.current_stream(self.device)
        self.sweeps = 0
        self.flips = 0

    def close(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:
            lib.umc_slab_destroy(h)
        self._h = None

    def __del__(self):
        self.close()

    def _local_planes(self):
        total = self.dims[2] if self.dims[2] > 1 else self.dims[1]
        lo, hi = self.planes_range
        return [(p % total) for p in range(lo - 1, hi + 1)]

    def set_field(self, full):
        """full: the whole lattice in natural site order ((z Ly + y) Lx + x),
        shape (sites,) or (sites, N); every rank passes the same array."""
        a = np.asarray(full).reshape(-1, self.N)
        planes = self._local_planes()
        if self.row_split:  # row y: its (x + y) even sites, then the odd ones
            loc = np.concatenate([np.concatenate([a[p * self.P + (p & 1)::2][: self.P // 2],
                                                  a[p * self.P + 1 - (p & 1)::2][: self.P // 2]]) for p in planes])
        else:
            loc = np.concatenate([a[p * self.P:(p + 1) * self.P] for p in planes])  # (nloc, N)
        soa = np.ascontiguousarray(loc.T).reshape(-1).astype(np.int8 if self.model == MODEL_ISING else np.float32)
        self.field.copy_(self.torch.from_numpy(soa).to(self.device))

    def get_field(self):
        """This rank's planes in natural order: (planes * plane sites, N)."""
        loc = self.field.cpu().numpy().reshape(self.N, self.nloc).T
        own = loc[self.P:(self.planes + 1) * self.P].copy()
        if self.row_split:  # back to x order
            lo = self.planes_range[0]
            h = self.P // 2
            out = np.empty_like(own)
            for r in range(self.planes):
                row, par = own[r * self.P:(r + 1) * self.P], (lo + r) & 1
                out[r * self.P + par:(r + 1) * self.P:2] = row[:h]
                out[r * self.P + 1 - par:(r + 1) * self.P:2] = row[h:]
            own = out
        return own

    def gather_field(self):
        """The whole lattice (natural order), on every rank."""
        if self.world == 1:
            return self.get_field()
        import torch.distributed as dist

        parts = [None] * self.world
        dist.all_gather_object(parts, self.get_field(), group=self.group)
        return np.concatenate(parts)

    def _plane(self, k):
        v = self.field.view(self.N, self.nloc)
        return v[:, k * self.P:(k + 1) * self.P]

    def _exchange(self):
        """Both halos from the neighbouring ranks' boundary planes."""
        if self.world == 1:
            self._plane(0).copy_(self._plane(self.planes))
            self._plane(self.planes + 1).copy_(self._plane(1))
            return
        import torch.distributed as dist

        prev, nxt = (self.rank - 1) % self.world, (self.rank + 1) % self.world
        cpu = dist.get_backend(self.group) == "gloo"
        mv = (lambda t: t.cpu()) if cpu else (lambda t: t.contiguous())
        last, first = mv(self._plane(self.planes)), mv(self._plane(1))
        lower = self.torch.empty_like(last)
        upper = self.torch.empty_like(first)
        # the same order on every rank: sends to next then prev, receives from
        # prev then next (tags for gloo; NCCL matches each pair's messages in order)
        ops = [dist.P2POp(dist.isend, last, nxt, self.group, 0), dist.P2POp(dist.isend, first, prev, self.group, 1),
               dist.P2POp(dist.irecv, lower, prev, self.group, 0), dist.P2POp(dist.irecv, upper, nxt, self.group, 1)]
        for w in dist.batch_isend_irecv(ops):
            w.wait()
        self._plane(0).copy_(lower.to(self.device))
        self._plane(self.planes + 1).copy_(upper.to(self.device))

    def sweep(self, beta):
        """One Metropolis sweep of the whole lattice; returns its record
        summed over the ranks ([E, M_0..M_{N-1}, .., accepted])."""
        s = self.stream.cuda_stream
        for colour in (0, 1):
            check(lib.umc_slab_pass(self._h, C.c_void_p(self.field.data_ptr()), beta, self.sweeps, colour, s))
            self._exchange()
        self.sweeps += 1
        rec = np.zeros(OBS_STRIDE)
        check(lib.umc_slab_record(self._h, _ptr(rec), s))
        if self.world > 1:
            import torch.distributed as dist

            t = self.torch.from_numpy(rec.copy())
            if dist.get_backend(self.group) != "gloo":
                t = t.to(self.device)
            dist.all_reduce(t, group=self.group)
            rec = t.cpu().numpy()
        return rec

    def metropolis(self, beta, n):
        """n sweeps; their records (n x OBS_STRIDE)."""
        self._exchange()
        return np.stack([self.sweep(beta) for _ in range(n)])

    def wolff_flip(self, beta):
        """One Wolff flip of the whole lattice (the single-GPU chain's flip of
        the same counter); returns the cluster size (summed over the ranks)."""
        h, s = self._h, self.stream.cuda_stream
        f = C.c_void_p(self.field.data_ptr())
        flip = self.flips
        self._exchange()
        check(lib.umc_slab_wolff_local(h, f, beta, flip, s))
        P = self.P
        first, last = np.zeros(P, np.uint32), np.zeros(P, np.uint32)
        up = np.zeros(P, np.uint8)
        check(lib.umc_slab_wolff_boundary(h, _ptr(first), _ptr(last), _ptr(up), s))
        nat, root = _u32(0), _u32(0)
        check(lib.umc_slab_wolff_seed(h, flip, C.byref(nat), C.byref(root), s))
        mine = (first, last, up, root.value)
        parts = [mine]
        if self.world > 1:
            import torch.distributed as dist

            parts = [None] * self.world
            dist.all_gather_object(parts, mine, group=self.group)
        seed_root = next(p[3] for p in parts if p[3] != 0xFFFFFFFF)
        firsts = np.ascontiguousarray(np.concatenate([p[0] for p in parts]))
        lasts = np.ascontiguousarray(np.concatenate([p[1] for p in parts]))
        ups = np.ascontiguousarray(np.concatenate([p[2] for p in parts]))
        roots = np.zeros(2 * P + 1, np.uint32)
        n_roots = _u32(0)
        check(lib.umc_slab_wolff_merge(self.world, P, _ptr(firsts), _ptr(lasts), _ptr(ups), seed_root, self.rank,
                                       _ptr(first), _ptr(last), root.value, _ptr(roots), C.byref(n_roots)))
        flipped = _u64(0)
        check(lib.umc_slab_wolff_flip(h, f, flip, _ptr(roots), n_roots.value, C.byref(flipped), s))
        size = flipped.value
        if self.world > 1:
            import torch.distributed as dist

            t = self.torch.tensor([size], dtype=self.torch.int64)
            if dist.get_backend(self.group) != "gloo":
                t = t.to(self.device)
            dist.all_reduce(t, group=self.group)
            size = int(t.item())
        self.flips = flip + 1
        self._exchange()
        return size

    def wolff(self, beta, n):
        """n Wolff flips; their cluster sizes."""
        return np.array([self.wolff_flip(beta) for _ in range(n)], np.uint64)


class GaugeSlabDesc(C.Structure):
    _fields_ = [
        ("model", _i32),
        ("N", _i32),
        ("cells", _vp),
        ("owner", _vp),
        ("rank", _u32),
        ("world", _u32),
        ("coupling", _f64),
        ("width", _f64),
        ("hits", _u32),
        ("seed", _u64),
        ("device", _i32),
    ]


_decl("umc_gslab_create", _int, C.POINTER(GaugeSlabDesc), C.POINTER(_vp))
_decl("umc_gslab_destroy", _int, _vp)
_decl("umc_gslab_info", _int, _vp, C.POINTER(_u32), C.POINTER(_u32), C.POINTER(_u32), C.POINTER(_u32))
_decl("umc_gslab_local_links", _int, _vp, _vp)
_decl("umc_gslab_exchange_counts", _int, _vp, _u32, _u32, C.POINTER(_u32), C.POINTER(_u32))
_decl("umc_gslab_pack", _int, _vp, _vp, _u32, _u32, _vp, _vp)
_decl("umc_gslab_unpack", _int, _vp, _vp, _u32, _u32, _vp, _vp)
_decl("umc_gslab_pass", _int, _vp, _vp, _f64, _u64, _u32, _vp)
_decl("umc_gslab_record", _int, _vp, _vp, _vp, _vp)


def slowest_axis_owner(cells, rank_count):
    """Link -> rank for hypercubic_plaquettes(L) (4D: link mu*L^4 + site,
    site = ((t L + z) L + y) L + x) or square_plaquettes(L) (2D: mu*L^2 + y L +
    x): ranks take contiguous ranges of the slowest coordinate (t, or y in 2D),
    sizes differing by at most one (shard_range)."""
    n = cells.sites()
    if n % 4 == 0 and round((n // 4) ** 0.25) ** 4 == n // 4:
        L = round((n // 4) ** 0.25)
        slow = (np.arange(n) % L**4) // L**3
    else:
        L = round((n // 2) ** 0.5)
        if 2 * L * L != n:
            raise ValueError("not a hypercubic or square plaquette complex")
        slow = (np.arange(n) % (L * L)) // L
    owner = np.zeros(n, np.uint32)
    for r in range(rank_count):
        lo, hi = shard_range(L, r, rank_count)
        owner[(slow >= lo) & (slow < hi)] = r
    return owner


class GaugeSlab:
    """One U(1) or SU(N) gauge chain split over the ranks of a
    torch.distributed group (umc_gslab_*), one process per GPU.  `owner`
    assigns every link (reference numbering) to a rank (slowest_axis_owner
    cuts the slowest coordinate).  This rank's owned links and the halo links
    their plaquettes touch live in a torch tensor on its GPU (comps planes x
    n_local); after each colour class the links just updated go to the ranks
    that hold them as halo (batch_isend_irecv: NCCL device to device, gloo
    through host copies).  The ranks together run exactly the single-GPU
    Chain of the same seed; records are summed over the ranks."""

    def __init__(self, model, cells, owner, *, rank=0, world=1, group=None, N=3, coupling=1.0, width=0.3, hits=1,
                 seed=1, device=0):
        import torch

        self.torch = torch
        self.rank, self.world, self.group = rank, world, group
        self.cells = cells
        owner = np.ascontiguousarray(owner, np.uint32)
        if owner.shape != (cells.sites(),):
            raise ValueError("owner needs one rank per link")
        d = GaugeSlabDesc()
        d.model, d.N, d.cells, d.owner = model, N, cells._h, owner.ctypes.data_as(_vp)
        d.rank, d.world, d.coupling, d.width, d.hits, d.seed, d.device = rank, world, coupling, width, hits, seed, device
        h = _vp()
        check(lib.umc_gslab_create(C.byref(d), C.byref(h)))
        self._h = h
        nl, no, nc, cp = _u32(0), _u32(0), _u32(0), _u32(0)
        check(lib.umc_gslab_info(h, C.byref(nl), C.byref(no), C.byref(nc), C.byref(cp)))
        self.n_local, self.n_owned, self.n_classes, self.comps = nl.value, no.value, nc.value, cp.value
        self.local_ref = np.zeros(self.n_local, np.uint32)
        check(lib.umc_gslab_local_links(h, _ptr(self.local_ref)))
        self.device = torch.device("cuda", device)
        self.field = torch.zeros(self.comps * self.n_local, dtype=torch.float32, device=self.device)
        self.stream = torch.cuda.current_stream(self.device)
        self.sweeps = 0
        # (peer, class) -> (links to send, links to receive)
        self.counts = {}
        for p in range(world):
            if p == rank:
                continue
            for c in range(self.n_classes):
                ns, nr = _u32(0), _u32(0)
                check(lib.umc_gslab_exchange_counts(h, p, c, C.byref(ns), C.byref(nr)))
                if ns.value or nr.value:
                    self.counts[(p, c)] = (ns.value, nr.value)

    def close(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:
            lib.umc_gslab_destroy(h)
        self._h = None

    def __del__(self):
        self.close()

    def set_field(self, full):
        """full: every link's scalars in the reference's layout, (links, comps);
        every rank passes the same array."""
        a = np.asarray(full, np.float32).reshape(-1, self.comps)
        soa = np.ascontiguousarray(a[self.local_ref].T).reshape(-1)
        self.field.copy_(self.torch.from_numpy(soa).to(self.device))

    def get_owned(self):
        """(reference ids, scalars) of this rank's owned links."""
        loc = self.field.cpu().numpy().reshape(self.comps, self.n_local).T
        return self.local_ref[: self.n_owned].copy(), loc[: self.n_owned].copy()

    def gather_field(self):
        """Every link's scalars (links, comps), on every rank."""
        parts = [self.get_owned()]
        if self.world > 1:
            import torch.distributed as dist

            parts = [None] * self.world
            dist.all_gather_object(parts, self.get_owned(), group=self.group)
        out = np.zeros((self.cells.sites(), self.comps), np.float32)
        for ids, vals in parts:
            out[ids] = vals
        return out

    def _exchange(self, colour):
        if self.world == 1:
            return
        import torch.distributed as dist

        cpu = dist.get_backend(self.group) == "gloo"
        s = self.stream.cuda_stream
        f = C.c_void_p(self.field.data_ptr())
        ops, recvs = [], []
        for p in range(self.world):
            ns, nr = self.counts.get((p, colour), (0, 0))
            if ns:
                buf = self.torch.empty(self.comps * ns, dtype=self.torch.float32, device=self.device)
                check(lib.umc_gslab_pack(self._h, f, p, colour, C.c_void_p(buf.data_ptr()), s))
                self.stream.synchronize()
                ops.append(dist.P2POp(dist.isend, buf.cpu() if cpu else buf, p, self.group, colour))
            if nr:
                buf = self.torch.empty(self.comps * nr, dtype=self.torch.float32, device="cpu" if cpu else self.device)
                ops.append(dist.P2POp(dist.irecv, buf, p, self.group, colour))
                recvs.append((p, buf))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        for p, buf in recvs:
            b = buf.to(self.device)
            check(lib.umc_gslab_unpack(self._h, f, p, colour, C.c_void_p(b.data_ptr()), s))
        self.stream.synchronize()

    def sweep(self, beta):
        """One sweep of every colour class; its record summed over the ranks
        ([S, <P>, Q, 0.., accepted])."""
        s = self.stream.cuda_stream
        f = C.c_void_p(self.field.data_ptr())
        for c in range(self.n_classes):
            check(lib.umc_gslab_pass(self._h, f, beta, self.sweeps, c, s))
            self._exchange(c)
        rec = np.zeros(OBS_STRIDE)
        check(lib.umc_gslab_record(self._h, f, _ptr(rec), s))
        self.sweeps += 1
        if self.world > 1:
            import torch.distributed as dist

            t = self.torch.from_numpy(rec.copy())
            if dist.get_backend(self.group) != "gloo":
                t = t.to(self.device)
            dist.all_reduce(t, group=self.group)
            rec = t.cpu().numpy()
        return rec

    def metropolis(self, beta, n):
        """n sweeps; their records (n x OBS_STRIDE)."""
        return np.stack([self.sweep(beta) for _ in range(n)])


class Batch:
    """Independent XY chains in replica-exchange ladders (umc_batch_*).

    first_ladder: global index of this batch's first ladder, for a shard of a
    larger batch (Batch.shard); its chains then run exactly as in the
    unsharded batch."""

    @classmethod
    def shard(cls, L, betas, rank, world, **kw):
        """The batch of rank `rank` of `world`: its contiguous range of the
        ladders (shard_range), keyed as in the whole batch."""
        lo, hi = shard_range(len(L), rank, world)
        b = cls(np.asarray(L)[lo:hi], np.asarray(betas)[lo:hi], first_ladder=lo, **kw)
        b.ladder_range = (lo, hi)
        return b

    def __init__(self, L, betas, *, coupling=1.0, width=1.0, sweeps_per_exchange=10, seed=1, device=0,
                 max_records=1024, first_ladder=0):
        L = np.ascontiguousarray(L, np.uint32)
        betas = np.ascontiguousarray(betas, np.float64)
        if betas.ndim != 2 or betas.shape[0] != len(L):
            raise ValueError("betas must be (n_ladders, replicas)")
        d = BatchDesc()
        d.n_ladders, d.replicas = betas.shape
        d.L = L.ctypes.data_as(_vp)
        d.betas = betas.ctypes.data_as(_vp)
        d.coupling, d.width = coupling, width
        d.sweeps_per_exchange = sweeps_per_exchange
        d.seed, d.device, d.stream, d.max_records = seed, device, None, max_records
        d.first_ladder = first_ladder
        h = _vp()
        check(lib.umc_batch_create(C.byref(d), C.byref(h)))
        self._h = h
        self.L = L.copy()
        self.betas = betas.copy()
        self.n_ladders, self.R = betas.shape
        self.n_chains = self.n_ladders * self.R
        self.sweeps_per_exchange = sweeps_per_exchange

    def close(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:  # module globals are gone at interpreter exit
            lib.umc_batch_destroy(h)
        self._h = None

    def __del__(self):
        self.close()

    def chain_side(self, c):
        return int(self.L[c // self.R])

    def randomize(self, seed):
        check(lib.umc_batch_randomize(self._h, seed))

    def set_field(self, chain, theta):
        a = np.ascontiguousarray(theta, np.float32).reshape(-1)
        if a.size != self.chain_side(chain) ** 2:
            raise ValueError("wrong field size")
        check(lib.umc_batch_set_field(self._h, chain, _ptr(a)))

    def get_field(self, chain):
        a = np.zeros(self.chain_side(chain) ** 2, np.float32)
        check(lib.umc_batch_get_field(self._h, chain, _ptr(a)))
        return a

    def run(self, n_segments):
        rec = np.zeros((n_segments, self.n_chains, OBS_STRIDE))
        check(lib.umc_batch_run(self._h, n_segments, _ptr(rec)))
        return rec.reshape(n_segments, self.n_ladders, self.R, OBS_STRIDE)

    def enqueue(self, n_segments):
        check(lib.umc_batch_enqueue(self._h, n_segments))

    def fetch(self, capacity):
        rec = np.zeros((capacity, self.n_chains, OBS_STRIDE))
        got = _u64(0)
        check(lib.umc_batch_fetch(self._h, _ptr(rec), capacity, C.byref(got)))
        return rec[: got.value].reshape(-1, self.n_ladders, self.R, OBS_STRIDE)

    def counters(self):
        s, r, w = _u64(0), _u64(0), _u64(0)
        check(lib.umc_batch_counters(self._h, C.byref(s), C.byref(r), C.byref(w)))
        return s.value, r.value, w.value

    def temperature_map(self):
        h = np.zeros(self.n_chains, np.uint32)
        check(lib.umc_batch_temperature_map(self._h, _ptr(h)))
        return h.reshape(self.n_ladders, self.R)

    def seeds(self):
        cs = np.zeros(self.n_chains, np.uint64)
        ls = np.zeros(self.n_ladders, np.uint64)
        check(lib.umc_batch_seeds(self._h, _ptr(cs), _ptr(ls)))
        return cs, ls

    def save(self, path) -> None:
        """Every chain's angles, the counters and the temperature map (.npz).
        load() into a batch made with the same description continues it
        exactly."""
        s, r, w = self.counters()
        cs, ls = self.seeds()
        fields = {f"theta{c}": self.get_field(c) for c in range(self.n_chains)}
        np.savez(path, counters=np.array([s, r, w], np.uint64), holder=self.temperature_map(), chain_seeds=cs,
                 ladder_seeds=ls, L=self.L, betas=self.betas, **fields)

    def load(self, path) -> None:
        z = np.load(path)
        cs, ls = self.seeds()
        if (not np.array_equal(z["L"], self.L) or not np.array_equal(z["betas"], self.betas)
                or not np.array_equal(z["chain_seeds"], cs) or not np.array_equal(z["ladder_seeds"], ls)):
            raise ValueError("checkpoint is of another batch (sides, betas or seed)")
        for c in range(self.n_chains):
            self.set_field(c, z[f"theta{c}"])
        s, r, w = (int(v) for v in z["counters"])
        holder = np.ascontiguousarray(z["holder"], np.uint32).reshape(-1)
        check(lib.umc_batch_set_state(self._h, s, r, w, _ptr(holder)))

    def config(self, L):
        a, b, c = _u32(0), _u32(0), _u32(0)
        check(lib.umc_batch_config(self._h, L, C.byref(a), C.byref(b), C.byref(c)))
        return {"chains_per_cta": a.value, "ctas_per_chain": b.value, "block": c.value}

    def sites(self):
        t, k = _u64(0), _u64(0)
        check(lib.umc_batch_sites(self._h, C.byref(t), C.byref(k)))
        return t.value, k.value

    def set_persistent(self, enable: bool) -> None:
        """One persistent kernel per segment, or one kernel per lattice-size
        group plus an exchange kernel.  Creation selects the form that
        measured faster on this batch; this overrides it."""
        check(lib.umc_batch_set_persistent(self._h, int(enable)))

    def set_persistent_config(self, cluster: int, ctas_per_sm: int) -> None:
        """The persistent form with this cluster size (1, 4, 8) and CTAs per
        SM (1, 2) instead of the tuned ones."""
        check(lib.umc_batch_set_persistent_config(self._h, cluster, ctas_per_sm))

    def persistent_info(self):
        e, g, nb, ni, kc, mb = _int(0), _u32(0), _u32(0), _u32(0), _u32(0), _u32(0)
        check(lib.umc_batch_persistent_info(self._h, C.byref(e), C.byref(g), C.byref(nb), C.byref(ni), C.byref(kc),
                                            C.byref(mb)))
        return {"enabled": bool(e.value), "grid": g.value, "big_items": nb.value, "items": ni.value,
                "cluster": kc.value, "ctas_per_sm": mb.value}

    def stream(self) -> int:
        return lib.umc_batch_stream(self._h) or 0


# ============================================== batched U(1), learned proposal
class U1BatchDesc(C.Structure):
    _fields_ = [
        ("n_chains", _u32),
        ("L", _u32),
        ("beta", _f64),
        ("width", _f64),
        ("seed", _u64),
        ("device", _i32),
        ("stream", _vp),
        ("max_records", _u64),
        ("first_chain", _u32),
    ]


class MlpDesc(C.Structure):
    _fields_ = [
        ("seed", _u64),
        ("device", _i32),
        ("stream", _vp),
        ("max_configs", _u64),
        ("L", _u32),
    ]


MLP_PARAMS = 5456
U1_RECORD = 4
_decl("umc_u1batch_create", _int, C.POINTER(U1BatchDesc), C.POINTER(_vp))
_decl("umc_u1batch_destroy", _int, _vp)
_decl("umc_u1batch_randomize", _int, _vp, _u64)
_decl("umc_u1batch_set_field", _int, _vp, _u32, _vp)
_decl("umc_u1batch_get_field", _int, _vp, _u32, _vp)
_decl("umc_u1batch_enqueue", _int, _vp, _u64, _vp)
_decl("umc_u1batch_fetch", _int, _vp, _vp, _u64, C.POINTER(_u64))
_decl("umc_u1batch_run", _int, _vp, _u64, _vp, _vp)
_decl("umc_u1batch_run_dump", _int, _vp, _vp, _vp)
_decl("umc_u1batch_counters", _int, _vp, C.POINTER(_u64), C.POINTER(_u64))
_decl("umc_u1batch_set_counter", _int, _vp, _u64)
_decl("umc_u1batch_seeds", _int, _vp, _vp)
_decl("umc_u1batch_config", _int, _vp, C.POINTER(_u32), C.POINTER(_u32))
_decl("umc_u1batch_stream", _vp, _vp)
_decl("umc_mlp_create", _int, C.POINTER(MlpDesc), C.POINTER(_vp))
_decl("umc_mlp_destroy", _int, _vp)
_decl("umc_mlp_set_params", _int, _vp, _vp)
_decl("umc_mlp_get_params", _int, _vp, _vp)
_decl("umc_mlp_forward", _int, _vp, _vp, _u64, _vp)
_decl("umc_mlp_loss_grad", _int, _vp, _vp, _vp, _u64, C.POINTER(_f64), _vp)
_decl("umc_mlp_apply_gradient", _int, _vp, _vp, _f64)
_decl("umc_mlp_add_configs", _int, _vp, _vp)
_decl("umc_mlp_configs", _int, _vp, C.POINTER(_u64))
_decl("umc_mlp_clear_configs", _int, _vp)
_decl("umc_mlp_train", _int, _vp, _u64, _u32, _f64, _vp)
_decl("umc_mlp_counters", _int, _vp, C.POINTER(_u64), C.POINTER(_u64))
_decl("umc_mlp_stream", _vp, _vp)


class ProposalNet:
    """The learned proposal's network (umc_mlp_*): staple features -> 4-component
    von Mises mixture, BF16 tensor-core forward/backward, Adam on FP32 masters.
    With max_configs > 0 it holds that many L x L training configurations."""

    def __init__(self, seed=1, *, device=0, max_configs=0, L=0):
        d = MlpDesc()
        d.seed, d.device, d.stream, d.max_configs, d.L = seed, device, None, max_configs, L
        h = _vp()
        check(lib.umc_mlp_create(C.byref(d), C.byref(h)))
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:  # module globals are gone at interpreter exit
            lib.umc_mlp_destroy(h)
        self._h = None

    def __del__(self):
        self.close()

    def save(self, path) -> None:
        """The network's parameters (.npy); load() sets them (and resets Adam)."""
        np.save(path, self.get_params())

    def load(self, path) -> None:
        self.set_params(np.load(path))

    def set_params(self, p):
        a = np.ascontiguousarray(p, np.float32)
        if a.size != MLP_PARAMS:
            raise ValueError("wrong parameter count")
        check(lib.umc_mlp_set_params(self._h, _ptr(a)))

    def get_params(self):
        a = np.zeros(MLP_PARAMS, np.float32)
        check(lib.umc_mlp_get_params(self._h, _ptr(a)))
        return a

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 3)
        out = np.zeros((x.shape[0], 16), np.float32)
        check(lib.umc_mlp_forward(self._h, _ptr(x), x.shape[0], _ptr(out)))
        return out

    def loss_grad(self, x, theta):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(theta, np.float32)
        g = np.zeros(MLP_PARAMS, np.float32)
        loss = _f64(0)
        check(lib.umc_mlp_loss_grad(self._h, _ptr(x), _ptr(t), x.shape[0], C.byref(loss), _ptr(g)))
        return loss.value, g

    def apply_gradient(self, g, lr):
        a = np.ascontiguousarray(g, np.float32)
        check(lib.umc_mlp_apply_gradient(self._h, _ptr(a), lr))

    def add_configs(self, batch: "U1Batch"):
        check(lib.umc_mlp_add_configs(self._h, batch._h))

    def configs(self) -> int:
        n = _u64(0)
        check(lib.umc_mlp_configs(self._h, C.byref(n)))
        return n.value

    def clear_configs(self):
        check(lib.umc_mlp_clear_configs(self._h))

    def train(self, steps, batch=8192, lr=1e-3):
        losses = np.zeros(steps)
        check(lib.umc_mlp_train(self._h, steps, batch, lr, _ptr(losses)))
        return losses

    def counters(self):
        s, k = _u64(0), _u64(0)
        check(lib.umc_mlp_counters(self._h, C.byref(s), C.byref(k)))
        return s.value, k.value


class U1Batch:
    """Independent 2D U(1) chains (umc_u1batch_*): plain U1Shift Metropolis, or
    Metropolis-Hastings with a ProposalNet.  Records per sweep and chain:
    [S, mean plaquette, Q, accepted]."""

    @classmethod
    def shard(cls, n_chains, L, beta, rank, world, **kw):
        """Rank `rank` of `world`'s contiguous range of n_chains chains
        (shard_range), keyed as in the whole batch."""
        lo, hi = shard_range(n_chains, rank, world)
        b = cls(hi - lo, L, beta, first_chain=lo, **kw)
        b.chain_range = (lo, hi)
        return b

    def __init__(self, n_chains, L, beta, *, width=0.5, seed=1, device=0, max_records=1024, first_chain=0):
        d = U1BatchDesc()
        d.n_chains, d.L, d.beta, d.width = n_chains, L, beta, width
        d.seed, d.device, d.stream, d.max_records = seed, device, None, max_records
        d.first_chain = first_chain
        h = _vp()
        check(lib.umc_u1batch_create(C.byref(d), C.byref(h)))
        self._h = h
        self.n_chains, self.L, self.beta, self.width = n_chains, L, beta, width
        self.max_records = max_records or 1024

    def close(self):
        h = getattr(self, "_h", None)
        if h and lib is not None:  # module globals are gone at interpreter exit
            lib.umc_u1batch_destroy(h)
        self._h = None

    def __del__(self):
        self.close()

    def randomize(self, seed):
        check(lib.umc_u1batch_randomize(self._h, seed))

    def set_field(self, chain, theta):
        a = np.ascontiguousarray(theta, np.float32).reshape(-1)
        if a.size != 2 * self.L * self.L:
            raise ValueError("wrong field size")
        check(lib.umc_u1batch_set_field(self._h, chain, _ptr(a)))

    def get_field(self, chain):
        a = np.zeros(2 * self.L * self.L, np.float32)
        check(lib.umc_u1batch_get_field(self._h, chain, _ptr(a)))
        return a

    def run(self, n_sweeps, net: ProposalNet | None = None, records=True):
        rec = np.zeros((n_sweeps, self.n_chains, U1_RECORD)) if records else None
        check(lib.umc_u1batch_run(self._h, n_sweeps, net._h if net else None, _ptr(rec)))
        return rec

    def enqueue(self, n_sweeps, net: ProposalNet | None = None):
        check(lib.umc_u1batch_enqueue(self._h, n_sweeps, net._h if net else None))

    def fetch(self, capacity=None):
        capacity = capacity or self.max_records
        rec = np.zeros((capacity, self.n_chains, U1_RECORD))
        got = _u64(0)
        check(lib.umc_u1batch_fetch(self._h, _ptr(rec), capacity, C.byref(got)))
        return rec[: got.value]

    def run_dump(self, net: ProposalNet):
        out = np.zeros((2 * self.L * self.L, 16), np.float32)
        check(lib.umc_u1batch_run_dump(self._h, net._h, _ptr(out)))
        return out

    def counters(self):
        s, k = _u64(0), _u64(0)
        check(lib.umc_u1batch_counters(self._h, C.byref(s), C.byref(k)))
        return s.value, k.value

    def save(self, path) -> None:
        """Every chain's angles, the sweep counter and the chain seeds (.npz).
        load() into a batch made with the same chains, L, beta, width and seed
        continues it exactly."""
        np.savez(path, theta=np.stack([self.get_field(c) for c in range(self.n_chains)]),
                 sweeps=np.uint64(self.counters()[0]), seeds=self.seeds(),
                 shape=np.array([self.n_chains, self.L], np.uint64), beta=np.float64(self.beta),
                 width=np.float64(self.width))

    def load(self, path) -> None:
        z = np.load(path)
        if (tuple(int(v) for v in z["shape"]) != (self.n_chains, self.L) or float(z["beta"]) != self.beta
                or float(z["width"]) != self.width or not np.array_equal(z["seeds"], self.seeds())):
            raise ValueError("checkpoint is of another batch (chains, L, beta, width or seed)")
        for c in range(self.n_chains):
            self.set_field(c, z["theta"][c])
        self.set_counter(int(z["sweeps"]))

    def set_counter(self, sweeps):
        check(lib.umc_u1batch_set_counter(self._h, sweeps))

    def seeds(self):
        s = np.zeros(self.n_chains, np.uint64)
        check(lib.umc_u1batch_seeds(self._h, _ptr(s)))
        return s

    def config(self):
        a, b = _u32(0), _u32(0)
        check(lib.umc_u1batch_config(self._h, C.byref(a), C.byref(b)))
        return {"plain_grid": a.value, "learned_grid": b.value}

    def stream(self) -> int:
        return lib.umc_u1batch_stream(self._h) or 0


# ========================================================= reference mirror
class Pcg32:
    """The driver's RNG argument: (seed, stream) choose the key seed of every
    counter-keyed stream the driver opens (rng.hpp:14-20 for the generator)."""

    def __init__(self, seed: int, stream: int = 0):
        self.seed = int(seed)
        self.stream = int(stream)

    @property
    def key(self) -> int:
        return (self.seed ^ ((self.stream * 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF)) & 0xFFFFFFFFFFFFFFFF


class Flip:
    """dof/ising.hpp:27-38."""
    kind = PROPOSAL_FLIP
    width = 0.0


class FixedAxis:
    """dof/ising.hpp:41-49."""
    axis = AXIS_FIXED


class UniformSphereN:
    """dof/vector.hpp:35-61 (also the Wolff axis for VectorSpin)."""
    kind = PROPOSAL_SPHERE
    axis = AXIS_SPHERE
    width = 0.0

    def __init__(self, N: int | None = None):
        self.N = N


class LocalRotation:
    """dof/vector.hpp:70-122."""
    kind = PROPOSAL_ROTATION

    def __init__(self, delta: float):
        self.width = float(delta)


class U1Shift:
    """dof/u1.hpp:35-50."""
    kind = PROPOSAL_U1SHIFT

    def __init__(self, width: float = 0.5):
        self.width = float(width)


class SUShift:
    """dof/sun.hpp:163-204."""
    kind = PROPOSAL_SUSHIFT

    def __init__(self, width: float = 0.3):
        self.width = float(width)


class _Model:
    _model = 0
    _components = 1

    def _chain(self, proposal=None, hits=1) -> Chain:
        if self.chain is None:
            kind = getattr(proposal, "kind", self._default_proposal)
            width = getattr(proposal, "width", 0.0)
            self.chain = Chain(self._model, graph=self._graph, cells=self._cells, components=self._components,
                               coupling=self._coupling, proposal=kind, width=width, hits=hits, device=self._device)
        return self.chain

    def data(self) -> np.ndarray:
        """The field in the reference's data() layout (forces a device copy)."""
        return self._chain().get_field()

    def update_all(self, field) -> None:
        self._chain().set_field(field)

    def sites(self) -> int:
        return self._chain().n

    def observe(self) -> np.ndarray:
        return self._chain().observe()


class Ising(_Model):
    """Ising(graph, J) -- example/ising.hpp:14-76 (cold start: all +1)."""
    _model = MODEL_ISING
    _default_proposal = PROPOSAL_FLIP

    def __init__(self, graph: PairGraph, J: int = 1, device: int = 0):
        self._graph, self._cells, self._coupling, self._device = graph, None, float(J), device
        self.chain = None


class VectorSpin(_Model):
    """VectorSpin<N>(graph, J) -- example/vector_spin.hpp:14-83 (FP32 state)."""
    _model = MODEL_VECTOR
    _default_proposal = PROPOSAL_SPHERE

    def __init__(self, N: int, graph: PairGraph, J: float = 1.0, device: int = 0):
        self._graph, self._cells, self._coupling, self._device = graph, None, float(J), device
        self._components = N
        self.chain = None


def XY(graph: PairGraph, J: float = 1.0, device: int = 0) -> VectorSpin:
    return VectorSpin(2, graph, J, device)


def Heisenberg(graph: PairGraph, J: float = 1.0, device: int = 0) -> VectorSpin:
    return VectorSpin(3, graph, J, device)


class XYAngle(_Model):
    """XY model on FP32 angles: PairModel<U1Dof, -J cos(ti - tj)> (model/pair.hpp)."""
    _model = MODEL_XY_ANGLE
    _default_proposal = PROPOSAL_U1SHIFT

    def __init__(self, graph: PairGraph, J: float = 1.0, device: int = 0):
        self._graph, self._cells, self._coupling, self._device = graph, None, float(J), device
        self.chain = None


class U1Gauge(_Model):
    """U(1) gauge theory on a plaquette complex (example/u1_gauge.hpp)."""
    _model = MODEL_U1
    _default_proposal = PROPOSAL_U1SHIFT

    def __init__(self, cells: CellComplex, beta: float = 1.0, device: int = 0):
        self._graph, self._cells, self._coupling, self._device = None, cells, float(beta), device
        self.chain = None


class SUGauge(_Model):
    """SU(N) gauge theory on a plaquette complex (example/sun_gauge.hpp)."""
    _model = MODEL_SU
    _default_proposal = PROPOSAL_SUSHIFT

    def __init__(self, N: int, cells: CellComplex, beta: float = 1.0, device: int = 0):
        self._graph, self._cells, self._coupling, self._device = None, cells, float(beta), device
        self._components = N
        self.chain = None


class Metropolis:
    """Metropolis(model, proposal, rng, beta) -- driver.hpp:17-68."""

    def __init__(self, model: _Model, proposal, rng: Pcg32, beta: float, hits: int = 1):
        self.model, self.proposal, self.rng, self.beta, self.hits = model, proposal, rng, float(beta), hits
        self.chain = model._chain(proposal, hits)

    def _arm(self):
        self.chain.set_proposal(self.proposal.kind, getattr(self.proposal, "width", 0.0), self.hits)
        self.chain.set_seed(self.rng.key)

    def sweep(self) -> None:
        self._arm()
        self.chain.metropolis(self.beta, 1, records=False)

    def run(self, sweeps: int) -> None:
        self._arm()
        self.chain.metropolis(self.beta, sweeps, records=False)

    def sample(self, sweeps: int, observe=None) -> np.ndarray:
        """Runs n sweeps; returns the per-sweep observable records and, if an
        observe callback is given, calls it once per sweep with the record."""
        self._arm()
        rec = self.chain.metropolis(self.beta, sweeps, records=True)
        if observe is not None:
            for r in rec:
                observe(r)
        return rec


class Wolff:
    """Wolff(model, axis, rng, beta) -- driver.hpp:92-210."""

    def __init__(self, model: _Model, axis, rng: Pcg32, beta: float):
        self.model, self.axis, self.rng, self.beta = model, axis, rng, float(beta)
        self.chain = model._chain()

    def _arm(self):
        self.chain.set_wolff_axis(self.axis.axis)
        self.chain.set_seed(self.rng.key)

    def flip(self) -> int:
        self._arm()
        sizes, _ = self.chain.wolff(self.beta, 1, records=False)
        return int(sizes[0])

    def sweep(self) -> None:
        self._arm()
        touched, n = 0, self.chain.n
        while touched < n:
            sizes, _ = self.chain.wolff(self.beta, 1, records=False)
            touched += int(sizes[0])

    def run(self, sweeps: int) -> None:
        for _ in range(sweeps):
            self.sweep()

    def sample(self, flips: int, observe=None):
        self._arm()
        sizes, rec = self.chain.wolff(self.beta, flips, records=True)
        if observe is not None:
            for r in rec:
                observe(r)
        return sizes, rec

    def mean_cluster_size(self) -> float:
        f, s = self.chain.wolff_stats()
        return 0.0 if f == 0 else s / f
