"""ctypes bindings for the CPU oracle (TEST INFRASTRUCTURE ONLY).

Two libraries live here:

* ``libumc_oracle.so`` -- the C restatement of the reference algorithms
  (``umc_oracle.c``); always built by ``make -C oracle oracle``.
* ``_ref/libumc_ref.so`` -- the reference library's own headers driven through
  project-written adapters (``ref_harness.cpp``); built where the reference tree
  is mounted and shipped with the repository snapshot otherwise.

Only tests, the package's smoke check and bench.py's CPU-baseline leg import this
module.  Every function works on numpy arrays and returns fresh arrays; none of
them touches a GPU.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libumc_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libumc_ref.so")
# the same harness built -O3 -march=x86-64-v3, for the timed CPU baselines
REF_FAST_SO = os.path.join(HERE, "_ref", "libumc_ref_fast.so")
_X86_64_V3 = {"avx", "avx2", "bmi1", "bmi2", "fma", "f16c", "lzcnt", "movbe", "xsave"}

TAG_BOND = 1
TAG_AXIS = 2
TAG_INIT = 3
TAG_SWAP = 4


def TAG_SITE(h: int = 0) -> int:
    return 0x100 + h


PROP_SPHERE = 0
PROP_ROTATION = 1

_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_vp = C.c_void_p
_u32 = C.c_uint32
_u64 = C.c_uint64
_i32 = C.c_int32
_f64 = C.c_double
_int = C.c_int


def build(reference_root: str | None = None) -> None:
    """Builds the oracle, and the reference harness where the reference tree
    exists: at ``reference_root``, else at $UMC_REFERENCE_ROOT, else wherever
    oracle/Makefile's REF default points (the Makefile skips the harness when
    no tree is there)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    root = reference_root or os.environ.get("UMC_REFERENCE_ROOT")
    if root:
        if os.path.isfile(os.path.join(root, "driver.hpp")):
            subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={root}"], check=True)
    else:
        subprocess.run(["make", "-s", "-C", HERE, "ref-if-present"], check=True)


def reference_root() -> str | None:
    """The reference tree: $UMC_REFERENCE_ROOT, else oracle/Makefile's REF
    default; None where no tree is there."""
    root = os.environ.get("UMC_REFERENCE_ROOT")
    if not root:
        with open(os.path.join(HERE, "Makefile")) as f:
            for line in f:
                if line.startswith("REF ?="):
                    root = line.split("=", 1)[1].strip()
                    break
    return root if root and os.path.isfile(os.path.join(root, "driver.hpp")) else None


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_vp)


class _Lib:
    def __init__(self, path: str, prefix: str):
        self.path = path
        self.lib = C.CDLL(path)
        self.prefix = prefix

    def fn(self, name, restype, *argtypes):
        f = getattr(self.lib, self.prefix + name)
        f.restype = restype
        f.argtypes = list(argtypes)
        return f


# --------------------------------------------------------------------- oracle
class Oracle:
    """The C restatement (``orc_*``)."""

    def __init__(self, path: str = ORACLE_SO):
        if not os.path.isfile(path):
            raise FileNotFoundError(f"oracle library not built: {path} (run make -C oracle oracle)")
        L = _Lib(path, "orc_")
        self._L = L
        self._key_draws = L.fn("key_draws", None, _u64, _u64, _u32, _u32, _u32, _vp)
        self._pcg_draws = L.fn("pcg32_draws", None, _u64, _u64, _u32, _vp)
        self._key_seed = L.fn("key_seed", _u64, _u64, _u64, _u32)
        self._stream_id = L.fn("stream_id", _u32, _u32)
        self._id_seed = L.fn("id_seed", _u64, _u64, _u32)
        self._pair_graph = L.fn("pair_graph", _int, _u64, _vp, _vp, _u64, _int, _vp, _vp, _vp)
        self._square = L.fn("square_edges", C.c_int64, _u64, _u64, _vp, _vp)
        self._cubic = L.fn("cubic_edges", C.c_int64, _u64, _u64, _u64, _vp, _vp)
        self._hyper = L.fn("hypercubic_cells", C.c_int64, _u64, _vp)
        self._plaq2 = L.fn("square_plaquette_cells", C.c_int64, _u64, _vp)
        self._incidence = L.fn("cell_incidence", _int, _u64, _u32, _vp, _u64, _vp, _vp, _vp)
        self._check_col = L.fn("check_colouring", _int, _u64, _vp, _vp, _vp)
        self._check_cell_col = L.fn("check_cell_colouring", _int, _u64, _u32, _vp, _u64, _vp)
        self._ising_metro = L.fn("ising_metropolis", None, _u64, _vp, _vp, _i32, _f64, _u64, _u64,
                                 _u64, _vp, _vp, _vp)
        self._ising_wolff = L.fn("ising_wolff", None, _u64, _vp, _vp, _vp, _i32, _f64, _u64, _u64,
                                 _u64, _vp, _vp, _vp, _vp)
        self._vec_metro = L.fn("vector_metropolis", None, _u32, _u64, _vp, _vp, _f64, _f64, _int,
                               _f64, _u64, _u64, _u64, _vp, _vp, _vp)
        self._vec_wolff = L.fn("vector_wolff", None, _u32, _u64, _vp, _vp, _vp, _f64, _f64, _u64,
                               _u64, _u64, _vp, _vp, _vp, _vp)
        self._wising_metro = L.fn("weighted_ising_metropolis", None, _u64, _vp, _vp, _vp, _f64, _u64, _u64, _u64,
                                  _vp, _vp, _vp)
        self._wising_wolff = L.fn("weighted_ising_wolff", None, _u64, _vp, _vp, _vp, _vp, _f64, _u64, _u64, _u64,
                                  _vp, _vp, _vp)
        self._xy_metro = L.fn("xy_metropolis", None, _u64, _vp, _vp, _f64, _f64, _f64, _u64, _u64,
                              _u64, _vp, _vp, _vp)
        self._u1_metro = L.fn("u1_metropolis", None, _u64, _vp, _u64, _vp, _vp, _vp, _f64, _f64,
                              _f64, _u32, _u64, _u64, _u64, _vp, _vp, _vp)
        self._u1_plaq = L.fn("u1_mean_plaquette", _f64, _u64, _vp, _vp)
        self._u1_q = L.fn("u1_topological_charge", _f64, _u64, _vp, _vp)
        self._su_metro = L.fn("su_metropolis", None, _u32, _u64, _vp, _u64, _vp, _vp, _vp, _f64,
                              _f64, _f64, _u32, _u64, _u64, _u64, _vp, _vp, _vp)
        self._su_plaq = L.fn("su_mean_plaquette", _f64, _u32, _u64, _vp, _vp)
        self._su_expm = L.fn("su_expm", None, _u32, _vp, _vp)
        self._su_unit = L.fn("su_unitarity_error", _f64, _u32, _vp)
        self._rex = L.fn("replica_exchange", _int, _u32, _vp, _vp, _vp, _u64, _u64, _u32, _vp)
        self._bf16 = L.fn("bf16", _f64, _f64)
        self._log_i0 = L.fn("log_i0", _f64, _f64)
        self._i1_i0 = L.fn("i1_over_i0", _f64, _f64)
        self._mlp_fwd = L.fn("mlp_forward", None, _vp, _u64, _vp, _int, _vp)
        self._mixture = L.fn("vm_mixture", None, _vp, _vp, _vp, _vp, _vp)
        self._mix_logpdf = L.fn("vm_mixture_logpdf", _f64, _vp, _vp, _vp, _vp, _f64)
        self._mlp_grad = L.fn("mlp_loss_grad", _f64, _vp, _u64, _vp, _vp, _int, _vp)
        self._adam = L.fn("adam_step", None, _u64, _vp, _vp, _vp, _vp, _u64, _f64, _f64, _f64, _f64)
        self._u1_learned = L.fn("u1_learned_metropolis", None, _u64, _vp, _u64, _vp, _vp, _vp, _vp,
                                _vp, _f64, _f64, _u64, _u64, _u64, _vp, _vp, _vp, _vp, _vp)
        self._vm_sample_keyed = L.fn("vm_sample", _int, _vp, _f64, _vp)
        self._key_open = L.fn("key_open", None, _vp, _u64, _u64, _u32, _u32)

    # ---- RNG
    def key_draws(self, seed, counter, tag, id_, n):
        out = np.zeros(n, np.uint32)
        self._key_draws(seed, counter, tag, id_, n, _ptr(out))
        return out

    def pcg32_draws(self, seed, stream, n):
        out = np.zeros(n, np.uint32)
        self._pcg_draws(seed, stream, n, _ptr(out))
        return out

    def key_seed(self, seed, counter, tag):
        return int(self._key_seed(seed, counter, tag))

    def stream_id(self, i):
        return int(self._stream_id(i))

    def id_seed(self, kseed, i):
        return int(self._id_seed(kseed, i))

    # ---- tables
    def pair_graph(self, n, ei, ej, symmetric=True):
        """CSR of PairGraph(n, edges, symmetric): (status, offset, bonds, slot_edge)."""
        ei = np.ascontiguousarray(ei, np.uint32)
        ej = np.ascontiguousarray(ej, np.uint32)
        offset = np.zeros(n + 1, np.uint32)
        st = self._pair_graph(n, _ptr(ei), _ptr(ej), len(ei), int(symmetric), _ptr(offset), None, None)
        if st != 0:
            return st, None, None, None
        bonds = np.zeros(int(offset[-1]), np.uint32)
        slot = np.zeros(int(offset[-1]), np.uint32)
        self._pair_graph(n, _ptr(ei), _ptr(ej), len(ei), int(symmetric), _ptr(offset), _ptr(bonds), _ptr(slot))
        return 0, offset, bonds, slot

    def square_edges(self, Lx, Ly):
        m = self._square(Lx, Ly, None, None)
        if m < 0:
            return m, None, None
        ei = np.zeros(m, np.uint32)
        ej = np.zeros(m, np.uint32)
        self._square(Lx, Ly, _ptr(ei), _ptr(ej))
        return 0, ei, ej

    def cubic_edges(self, Lx, Ly, Lz):
        m = self._cubic(Lx, Ly, Lz, None, None)
        if m < 0:
            return m, None, None
        ei = np.zeros(m, np.uint32)
        ej = np.zeros(m, np.uint32)
        self._cubic(Lx, Ly, Lz, _ptr(ei), _ptr(ej))
        return 0, ei, ej

    def hypercubic_cells(self, L):
        m = self._hyper(L, None)
        cells = np.zeros((m, 4), np.uint32)
        self._hyper(L, _ptr(cells))
        return cells

    def square_plaquette_cells(self, L):
        m = self._plaq2(L, None)
        cells = np.zeros((m, 4), np.uint32)
        self._plaq2(L, _ptr(cells))
        return cells

    def cell_incidence(self, n_sites, cells):
        cells = np.ascontiguousarray(cells, np.uint32)
        arity = cells.shape[1]
        offset = np.zeros(n_sites + 1, np.uint64)
        st = self._incidence(n_sites, arity, _ptr(cells), cells.shape[0], _ptr(offset), None, None)
        if st != 0:
            return st, None, None, None
        tot = int(offset[-1])
        inc_cell = np.zeros(tot, np.uint32)
        inc_which = np.zeros(tot, np.uint8)
        self._incidence(n_sites, arity, _ptr(cells), cells.shape[0], _ptr(offset), _ptr(inc_cell), _ptr(inc_which))
        return 0, offset, inc_cell, inc_which

    def check_colouring(self, offset, bonds, colour):
        colour = np.ascontiguousarray(colour, np.uint32)
        return bool(self._check_col(len(offset) - 1, _ptr(offset), _ptr(bonds), _ptr(colour)))

    def check_cell_colouring(self, n_sites, cells, colour):
        cells = np.ascontiguousarray(cells, np.uint32)
        colour = np.ascontiguousarray(colour, np.uint32)
        return bool(self._check_cell_col(n_sites, cells.shape[1], _ptr(cells), cells.shape[0], _ptr(colour)))

    # ---- Ising
    def ising_metropolis(self, offset, bonds, J, beta, seed, sweep0, n_sweeps, spins):
        s = np.array(spins, np.int8, copy=True)
        E = np.zeros(n_sweeps)
        M = np.zeros(n_sweeps)
        self._ising_metro(len(s), _ptr(offset), _ptr(bonds), J, beta, seed, sweep0, n_sweeps,
                          _ptr(s), _ptr(E), _ptr(M))
        return s, E, M

    def ising_wolff(self, offset, bonds, slot_edge, J, beta, seed, flip0, n_flips, spins):
        s = np.array(spins, np.int8, copy=True)
        sizes = np.zeros(n_flips, np.uint64)
        E = np.zeros(n_flips)
        M = np.zeros(n_flips)
        self._ising_wolff(len(s), _ptr(offset), _ptr(bonds), _ptr(slot_edge), J, beta, seed, flip0,
                          n_flips, _ptr(s), _ptr(sizes), _ptr(E), _ptr(M))
        return s, sizes, E, M

    # ---- weighted Ising (test/graph_check.cpp's IsingGraph on PairGraph<double>)
    def weighted_ising_metropolis(self, offset, bonds, c, beta, seed, sweep0, n_sweeps, spins):
        """c: the coupling of every CSR slot.  Returns spins, E per sweep and
        the last sweep's accept margins log(u) - log_p."""
        s = np.array(spins, np.float64, copy=True)
        c = np.ascontiguousarray(c, np.float64)
        E = np.zeros(n_sweeps)
        margin = np.zeros(len(s))
        self._wising_metro(len(s), _ptr(offset), _ptr(bonds), _ptr(c), beta, seed, sweep0, n_sweeps, _ptr(s),
                           _ptr(E), _ptr(margin))
        return s, E, margin

    def weighted_ising_wolff(self, offset, bonds, key, c, beta, seed, flip0, n_flips, spins):
        s = np.array(spins, np.float64, copy=True)
        c = np.ascontiguousarray(c, np.float64)
        key = np.ascontiguousarray(key, np.uint32)
        sizes = np.zeros(n_flips, np.uint64)
        E = np.zeros(n_flips)
        self._wising_wolff(len(s), _ptr(offset), _ptr(bonds), _ptr(key), _ptr(c), beta, seed, flip0, n_flips,
                           _ptr(s), _ptr(sizes), _ptr(E))
        return s, sizes, E

    # ---- VectorSpin
    def vector_metropolis(self, N, offset, bonds, J, beta, proposal, delta, seed, sweep0, n_sweeps, spins):
        s = np.array(spins, np.float64, copy=True).reshape(-1)
        n = s.size // N
        obs = np.zeros((n_sweeps, N + 1))
        margin = np.zeros(n)
        self._vec_metro(N, n, _ptr(offset), _ptr(bonds), J, beta, proposal, delta, seed, sweep0,
                        n_sweeps, _ptr(s), _ptr(obs), _ptr(margin))
        return s.reshape(n, N), obs, margin

    def vector_wolff(self, N, offset, bonds, slot_edge, J, beta, seed, flip0, n_flips, spins):
        s = np.array(spins, np.float64, copy=True).reshape(-1)
        n = s.size // N
        sizes = np.zeros(n_flips, np.uint64)
        obs = np.zeros((n_flips, N + 1))
        margin = np.zeros(n_flips)
        self._vec_wolff(N, n, _ptr(offset), _ptr(bonds), _ptr(slot_edge), J, beta, seed, flip0,
                        n_flips, _ptr(s), _ptr(sizes), _ptr(obs), _ptr(margin))
        return s.reshape(n, N), sizes, obs, margin

    def xy_metropolis(self, offset, bonds, J, beta, width, seed, sweep0, n_sweeps, theta):
        t = np.array(theta, np.float64, copy=True)
        obs = np.zeros((n_sweeps, 3))
        margin = np.zeros(t.size)
        self._xy_metro(t.size, _ptr(offset), _ptr(bonds), J, beta, width, seed, sweep0, n_sweeps,
                       _ptr(t), _ptr(obs), _ptr(margin))
        return t, obs, margin

    # ---- gauge
    def u1_metropolis(self, cells, inc, model_beta, driver_beta, width, hits, seed, sweep0,
                      n_sweeps, theta):
        cells = np.ascontiguousarray(cells, np.uint32)
        off, ic, iw = inc
        t = np.array(theta, np.float64, copy=True)
        obs = np.zeros((n_sweeps, 2))
        margin = np.zeros(t.size)
        self._u1_metro(t.size, _ptr(cells), cells.shape[0], _ptr(off), _ptr(ic), _ptr(iw),
                       model_beta, driver_beta, width, hits, seed, sweep0, n_sweeps, _ptr(t),
                       _ptr(obs), _ptr(margin))
        return t, obs, margin

    def u1_mean_plaquette(self, cells, theta):
        cells = np.ascontiguousarray(cells, np.uint32)
        theta = np.ascontiguousarray(theta, np.float64)
        return self._u1_plaq(cells.shape[0], _ptr(cells), _ptr(theta))

    def u1_topological_charge(self, cells, theta):
        cells = np.ascontiguousarray(cells, np.uint32)
        theta = np.ascontiguousarray(theta, np.float64)
        return self._u1_q(cells.shape[0], _ptr(cells), _ptr(theta))

    def su_metropolis(self, N, cells, inc, model_beta, driver_beta, width, hits, seed, sweep0,
                      n_sweeps, links):
        """links: complex array (n_links, N, N)."""
        cells = np.ascontiguousarray(cells, np.uint32)
        off, ic, iw = inc
        l = np.ascontiguousarray(np.array(links, np.complex128, copy=True))
        n_links = l.shape[0]
        obs = np.zeros((n_sweeps, 2))
        margin = np.zeros(n_links)
        self._su_metro(N, n_links, _ptr(cells), cells.shape[0], _ptr(off), _ptr(ic), _ptr(iw),
                       model_beta, driver_beta, width, hits, seed, sweep0, n_sweeps, _ptr(l),
                       _ptr(obs), _ptr(margin))
        return l, obs, margin

    def su_mean_plaquette(self, N, cells, links):
        cells = np.ascontiguousarray(cells, np.uint32)
        l = np.ascontiguousarray(links, np.complex128)
        return self._su_plaq(N, cells.shape[0], _ptr(cells), _ptr(l))

    def su_expm(self, N, a):
        a = np.ascontiguousarray(a, np.complex128)
        out = np.zeros((N, N), np.complex128)
        self._su_expm(N, _ptr(a), _ptr(out))
        return out

    def su_unitarity_error(self, N, u):
        u = np.ascontiguousarray(u, np.complex128)
        return self._su_unit(N, _ptr(u))

    # ---- learned proposal
    MLP_PARAMS = 5456
    TAG_LEARN = 5
    TAG_LEARNED = 6

    def bf16(self, v):
        return self._bf16(float(v))

    def log_i0(self, x):
        return self._log_i0(float(x))

    def i1_over_i0(self, x):
        return self._i1_i0(float(x))

    def mlp_forward(self, params, x, emulate=True):
        p = np.ascontiguousarray(params, np.float64)
        x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
        out = np.zeros((x.shape[0], 16))
        self._mlp_fwd(_ptr(p), x.shape[0], _ptr(x), int(emulate), _ptr(out))
        return out

    def vm_mixture(self, out16):
        o = np.ascontiguousarray(out16, np.float64)
        w, mu, k, li = (np.zeros(4) for _ in range(4))
        self._mixture(_ptr(o), _ptr(w), _ptr(mu), _ptr(k), _ptr(li))
        return w, mu, k, li

    def vm_mixture_logpdf(self, out16, theta):
        w, mu, k, li = self.vm_mixture(out16)
        return self._mix_logpdf(_ptr(w), _ptr(mu), _ptr(k), _ptr(li), float(theta))

    def vm_sample(self, kappa, seed, counter, tag, id_):
        """Best-Fisher sample around 0 from the keyed stream (None if all trials fail)."""
        g = (C.c_uint64 * 2)()
        self._key_open(g, seed, counter, tag, id_)
        a = C.c_double(0.0)
        ok = self._vm_sample_keyed(g, float(kappa), C.byref(a))
        return a.value if ok else None

    def mlp_loss_grad(self, params, x, theta, emulate=True, grad=True):
        p = np.ascontiguousarray(params, np.float64)
        x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
        t = np.ascontiguousarray(theta, np.float64)
        g = np.zeros(p.size) if grad else None
        loss = self._mlp_grad(_ptr(p), x.shape[0], _ptr(x), _ptr(t), int(emulate), _ptr(g))
        return loss, g

    def adam_step(self, p, g, m, v, t, lr, b1=0.9, b2=0.999, eps=1e-8):
        p, m, v = (np.array(a, np.float64, copy=True) for a in (p, m, v))
        g = np.ascontiguousarray(g, np.float64)
        self._adam(p.size, _ptr(p), _ptr(g), _ptr(m), _ptr(v), t, lr, b1, b2, eps)
        return p, m, v

    def u1_learned_metropolis(self, cells, inc, params, model_beta, driver_beta, seed, sweep0,
                              n_sweeps, theta, given_out=None):
        cells = np.ascontiguousarray(cells, np.uint32)
        off, ic, iw = inc
        t = np.array(theta, np.float64, copy=True)
        p = np.ascontiguousarray(params, np.float64)
        given = None if given_out is None else np.ascontiguousarray(given_out, np.float64)
        obs = np.zeros((n_sweeps, 3))
        margin = np.zeros(t.size)
        dump = np.zeros((t.size, 16))
        acc = np.zeros(t.size, np.uint8)
        self._u1_learned(t.size, _ptr(cells), cells.shape[0], _ptr(off), _ptr(ic), _ptr(iw),
                         _ptr(p), _ptr(given), model_beta, driver_beta, seed, sweep0, n_sweeps,
                         _ptr(t), _ptr(obs), _ptr(margin), _ptr(dump), _ptr(acc))
        return t, obs, margin, dump, acc

    def replica_exchange(self, betas, holder, energy, seed, round_, parity):
        """One exchange round: returns (new holder, accepted flags per slot)."""
        betas = np.ascontiguousarray(betas, np.float64)
        h = np.array(holder, np.uint32, copy=True)
        e = np.ascontiguousarray(energy, np.float64)
        acc = np.zeros(len(h), np.uint8)
        self._rex(len(h), _ptr(betas), _ptr(h), _ptr(e), seed, round_, parity, _ptr(acc))
        return h, acc


# ------------------------------------------------------------------ reference
class Reference:
    """The reference headers driven by ref_harness.cpp (``ref_*``)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.isfile(path):
            raise FileNotFoundError(f"reference harness not built: {path}")
        L = _Lib(path, "ref_")
        self._pcg_draws = L.fn("pcg32_draws", None, _u64, _u64, _u32, _vp)
        self._key_draws = L.fn("key_draws", None, _u64, _u64, _u32, _u32, _u32, _vp)
        self._pair_graph = L.fn("pair_graph", _int, _u64, _vp, _vp, _u64, _int, _vp, _vp)
        self._square = L.fn("square_lattice", _int, _u64, _u64, _vp, _vp)
        self._hyper = L.fn("hypercubic", _int, _u64, _vp, _vp, _vp, _vp)
        self._incidence = L.fn("cell_incidence", _int, _u64, _vp, _u64, _vp, _vp, _vp)
        self._ising_metro = L.fn("ising_metropolis", _int, _u64, _vp, _vp, _u64, _i32, _f64, _u64,
                                 _u64, _u64, _vp, _vp, _vp)
        self._ising_wolff = L.fn("ising_wolff", _int, _u64, _vp, _vp, _u64, _i32, _f64, _u64, _u64,
                                 _u64, _vp, _vp, _vp, _vp)
        self._vec_metro = L.fn("vector_metropolis", _int, _u32, _u64, _vp, _vp, _u64, _f64, _f64,
                               _int, _f64, _u64, _u64, _u64, _vp, _vp)
        self._vec_wolff = L.fn("vector_wolff", _int, _u32, _u64, _vp, _vp, _u64, _f64, _f64, _u64,
                               _u64, _u64, _vp, _vp, _vp)
        self._sphere = L.fn("sphere_sample", None, _u32, _u64, _u64, _u32, _u32, _vp)
        self._xy_metro = L.fn("xy_metropolis", _int, _u64, _vp, _vp, _u64, _f64, _f64, _f64, _u64,
                              _u64, _u64, _vp, _vp)
        self._u1_metro = L.fn("u1_metropolis", _int, _u64, _vp, _u64, _f64, _f64, _f64, _u32,
                              _u64, _u64, _u64, _vp, _vp)
        self._u1_learned = L.fn("u1_learned_metropolis", _int, _u64, _vp, _u64, _vp, _vp, _vp, _vp,
                                _f64, _f64, _u64, _u64, _u64, _vp, _vp)
        self._su_metro = L.fn("su_metropolis", _int, _u32, _u64, _vp, _u64, _f64, _f64, _f64, _u32,
                              _u64, _u64, _u64, _vp, _vp)
        self._su_expm = L.fn("su_expm", None, _u32, _vp, _vp)
        self._su_shift = L.fn("su_shift", None, _u32, _f64, _u64, _u64, _u32, _u32, _vp, _vp)
        self._bench_o3 = L.fn("bench_o3", _int, _u64, _f64, _u64, _u64, _u32, _u64, _vp, _vp)
        self._wising_metro = L.fn("weighted_ising_metropolis", _int, _u64, _vp, _vp, _vp, _u64, _f64, _u64, _u64,
                                  _u64, _vp, _vp)
        self._wising_wolff = L.fn("weighted_ising_wolff", _int, _u64, _vp, _vp, _vp, _u64, _vp, _f64, _u64, _u64,
                                  _u64, _vp, _vp, _vp)
        self._stock_o3 = L.fn("stock_o3_chain", _int, _u64, _f64, _u64, _u64, _u64, _vp)
        self._stock_o3_multi = L.fn("stock_o3_chains", _int, _u64, _f64, _u64, _u32, _vp, _u64, _u64, _vp)
        self._stock_su3 = L.fn("stock_su3_chain", _int, _u64, _f64, _f64, _u64, _u32, _u64, _u64, _vp)
        self._bench_ising = L.fn("bench_ising", _int, _u64, _f64, _u64, _u64, _u32, _u64, _vp, _vp)
        self._bench_xy = L.fn("bench_xy", _int, _u64, _f64, _f64, _u64, _u64, _u32, _u64, _vp, _vp)
        self._bench_pair_o3 = L.fn("bench_pair_o3", _int, _u64, _f64, _u64, _u64, _u32, _u64, _vp, _vp)
        self._bench_ising_wolff = L.fn("bench_ising_wolff", _int, _u64, _f64, _u64, _u64, _u32, _u64, _vp, _vp)
        self._bench_u1_cells = L.fn("bench_u1_cells", _int, _u64, _f64, _f64, _f64, _u64, _u64, _u32, _u64, _vp, _vp)
        self._bench_su3 = L.fn("bench_su3", _int, _u64, _f64, _f64, _u32, _u64, _u64, _u32, _u64, _vp, _vp)

    def pcg32_draws(self, seed, stream, n):
        out = np.zeros(n, np.uint32)
        self._pcg_draws(seed, stream, n, _ptr(out))
        return out

    def key_draws(self, seed, counter, tag, id_, n):
        out = np.zeros(n, np.uint32)
        self._key_draws(seed, counter, tag, id_, n, _ptr(out))
        return out

    def pair_graph(self, n, ei, ej, symmetric=True):
        ei = np.ascontiguousarray(ei, np.uint32)
        ej = np.ascontiguousarray(ej, np.uint32)
        offset = np.zeros(n + 1, np.uint32)
        st = self._pair_graph(n, _ptr(ei), _ptr(ej), len(ei), int(symmetric), _ptr(offset), None)
        if st != 0:
            return st, None, None
        bonds = np.zeros(int(offset[-1]), np.uint32)
        self._pair_graph(n, _ptr(ei), _ptr(ej), len(ei), int(symmetric), _ptr(offset), _ptr(bonds))
        return 0, offset, bonds

    def square_lattice(self, Lx, Ly):
        n = Lx * Ly
        offset = np.zeros(n + 1, np.uint32)
        st = self._square(Lx, Ly, _ptr(offset), None)
        if st != 0:
            return st, None, None
        bonds = np.zeros(int(offset[-1]), np.uint32)
        self._square(Lx, Ly, _ptr(offset), _ptr(bonds))
        return 0, offset, bonds

    def hypercubic(self, L):
        L4 = L ** 4
        cells = np.zeros((6 * L4, 4), np.uint32)
        offset = np.zeros(4 * L4 + 1, np.uint64)
        inc_cell = np.zeros(24 * L4, np.uint32)
        inc_which = np.zeros(24 * L4, np.uint8)
        st = self._hyper(L, _ptr(cells), _ptr(offset), _ptr(inc_cell), _ptr(inc_which))
        return st, cells, offset, inc_cell, inc_which

    def cell_incidence(self, n_sites, cells):
        cells = np.ascontiguousarray(cells, np.uint32)
        offset = np.zeros(n_sites + 1, np.uint64)
        tot = cells.size
        inc_cell = np.zeros(tot, np.uint32)
        inc_which = np.zeros(tot, np.uint8)
        st = self._incidence(n_sites, _ptr(cells), cells.shape[0], _ptr(offset), _ptr(inc_cell), _ptr(inc_which))
        return st, offset, inc_cell, inc_which

    def ising_metropolis(self, n, ei, ej, J, beta, seed, sweep0, n_sweeps, spins):
        ei = np.ascontiguousarray(ei, np.uint32)
        ej = np.ascontiguousarray(ej, np.uint32)
        s = np.array(spins, np.int8, copy=True)
        E = np.zeros(n_sweeps)
        M = np.zeros(n_sweeps)
        st = self._ising_metro(n, _ptr(ei), _ptr(ej), len(ei), J, beta, seed, sweep0, n_sweeps,
                               _ptr(s), _ptr(E), _ptr(M))
        assert st == 0, st
        return s, E, M

    def ising_wolff(self, n, ei, ej, J, beta, seed, flip0, n_flips, spins):
        ei = np.ascontiguousarray(ei, np.uint32)
        ej = np.ascontiguousarray(ej, np.uint32)
        s = np.array(spins, np.int8, copy=True)
        sizes = np.zeros(n_flips, np.uint64)
        E = np.zeros(n_flips)
        M = np.zeros(n_flips)
        st = self._ising_wolff(n, _ptr(ei), _ptr(ej), len(ei), J, beta, seed, flip0, n_flips,
                               _ptr(s), _ptr(sizes), _ptr(E), _ptr(M))
        assert st == 0, st
        return s, sizes, E, M

    def vector_metropolis(self, N, n, ei, ej, J, beta, proposal, delta, seed, sweep0, n_sweeps, spins):
        ei = np.ascontiguousarray(ei, np.uint32)
        ej = np.ascontiguousarray(ej, np.uint32)
        s = np.array(spins, np.float64, copy=True).reshape(-1)
        obs = np.zeros((n_sweeps, N + 1))
        st = self._vec_metro(N, n, _ptr(ei), _ptr(ej), len(ei), J, beta, proposal, delta, seed,
                             sweep0, n_sweeps, _ptr(s), _ptr(obs))
        assert st == 0, st
        return s.reshape(n, N), obs

    def vector_wolff(self, N, n, ei, ej, J, beta, seed, flip0, n_flips, spins):
        ei = np.ascontiguousarray(ei, np.uint32)
        ej = np.ascontiguousarray(ej, np.uint32)
        s = np.array(spins, np.float64, copy=True).reshape(-1)
        sizes = np.zeros(n_flips, np.uint64)
        obs = np.zeros((n_flips, N + 1))
        st = self._vec_wolff(N, n, _ptr(ei), _ptr(ej), len(ei), J, beta, seed, flip0, n_flips,
                             _ptr(s), _ptr(sizes), _ptr(obs))
        assert st == 0, st
        return s.reshape(n, N), sizes, obs

    def sphere_sample(self, N, seed, counter, tag, id_):
        out = np.zeros(N)
        self._sphere(N, seed, counter, tag, id_, _ptr(out))
        return out

    def xy_metropolis(self, n, ei, ej, J, beta, width, seed, sweep0, n_sweeps, theta):
        ei = np.ascontiguousarray(ei, np.uint32)
        ej = np.ascontiguousarray(ej, np.uint32)
        t = np.array(theta, np.float64, copy=True)
        obs = np.zeros((n_sweeps, 3))
        st = self._xy_metro(n, _ptr(ei), _ptr(ej), len(ei), J, beta, width, seed, sweep0, n_sweeps,
                            _ptr(t), _ptr(obs))
        assert st == 0, st
        return t, obs

    def u1_learned_metropolis(self, cells, inc, params, model_beta, driver_beta, seed, sweep0,
                              n_sweeps, theta):
        """Reference Metropolis driver with the learned proposal adapter; obs = mean plaquette."""
        cells = np.ascontiguousarray(cells, np.uint32)
        off, ic, iw = inc
        t = np.array(theta, np.float64, copy=True)
        p = np.ascontiguousarray(params, np.float64)
        obs = np.zeros(n_sweeps)
        st = self._u1_learned(t.size, _ptr(cells), cells.shape[0], _ptr(off), _ptr(ic), _ptr(iw),
                              _ptr(p), model_beta, driver_beta, seed, sweep0, n_sweeps, _ptr(t), _ptr(obs))
        assert st == 0, st
        return t, obs

    def u1_metropolis(self, cells, model_beta, driver_beta, width, hits, seed, sweep0, n_sweeps, theta):
        cells = np.ascontiguousarray(cells, np.uint32)
        t = np.array(theta, np.float64, copy=True)
        obs = np.zeros((n_sweeps, 2))
        st = self._u1_metro(t.size, _ptr(cells), cells.shape[0], model_beta, driver_beta, width,
                            hits, seed, sweep0, n_sweeps, _ptr(t), _ptr(obs))
        assert st == 0, st
        return t, obs

    def su_metropolis(self, N, cells, model_beta, driver_beta, width, hits, seed, sweep0, n_sweeps, links):
        cells = np.ascontiguousarray(cells, np.uint32)
        l = np.ascontiguousarray(np.array(links, np.complex128, copy=True))
        obs = np.zeros((n_sweeps, 2))
        st = self._su_metro(N, l.shape[0], _ptr(cells), cells.shape[0], model_beta, driver_beta,
                            width, hits, seed, sweep0, n_sweeps, _ptr(l), _ptr(obs))
        assert st == 0, st
        return l, obs

    def su_expm(self, N, a):
        a = np.ascontiguousarray(a, np.complex128)
        out = np.zeros((N, N), np.complex128)
        self._su_expm(N, _ptr(a), _ptr(out))
        return out

    def su_shift(self, N, width, seed, counter, tag, id_, cur):
        cur = np.ascontiguousarray(cur, np.complex128)
        out = np.zeros((N, N), np.complex128)
        self._su_shift(N, width, seed, counter, tag, id_, _ptr(cur), _ptr(out))
        return out

    def weighted_ising_metropolis(self, n, ei, ej, c, beta, seed, sweep0, n_sweeps, spins):
        """The reference Metropolis on the weighted Ising model of
        test/graph_check.cpp (c: per-edge couplings): spins and E per sweep."""
        ei = np.ascontiguousarray(ei, np.uint32)
        ej = np.ascontiguousarray(ej, np.uint32)
        c = np.ascontiguousarray(c, np.float64)
        s = np.array(spins, np.float64, copy=True)
        E = np.zeros(n_sweeps)
        st = self._wising_metro(n, _ptr(ei), _ptr(ej), _ptr(c), len(ei), beta, seed, sweep0, n_sweeps, _ptr(s),
                                _ptr(E))
        assert st == 0, st
        return s, E

    def weighted_ising_wolff(self, n, ei, ej, c, key, beta, seed, flip0, n_flips, spins):
        """The reference Wolff on the weighted Ising model; key: per CSR slot."""
        ei = np.ascontiguousarray(ei, np.uint32)
        ej = np.ascontiguousarray(ej, np.uint32)
        c = np.ascontiguousarray(c, np.float64)
        key = np.ascontiguousarray(key, np.uint32)
        s = np.array(spins, np.float64, copy=True)
        sizes = np.zeros(n_flips, np.uint64)
        E = np.zeros(n_flips)
        st = self._wising_wolff(n, _ptr(ei), _ptr(ej), _ptr(c), len(ei), _ptr(key), beta, seed, flip0, n_flips,
                                _ptr(s), _ptr(sizes), _ptr(E))
        assert st == 0, st
        return s, sizes, E

    def stock_o3_chain(self, L, beta, seed, warmup, steps):
        """The reference's own O(3) L^3 chain (plain Pcg32; 1 Wolff flip + 1
        sweep per step): per-step [E, Mx, My, Mz] after `warmup` steps."""
        obs = np.zeros((steps, 4))
        st = self._stock_o3(L, beta, seed, warmup, steps, _ptr(obs))
        assert st == 0, st
        return obs

    def stock_o3_chains(self, L, beta, seed, chains, warmup, steps, init=None):
        """Independent reference O(3) L^3 chains, one per thread (seed + c),
        chain c from init[c] (chains x n x 3, the natural site order) or its
        own random start: (chains, steps, 4) of per-step [E, Mx, My, Mz] after
        `warmup`."""
        obs = np.zeros((chains, steps, 4))
        ini = None
        if init is not None:
            ini = np.ascontiguousarray(init, np.float64)
            assert ini.shape == (chains, L**3, 3), ini.shape
            ini = ini.reshape(-1)
        st = self._stock_o3_multi(L, beta, seed, chains, _ptr(ini), warmup, steps, _ptr(obs))
        assert st == 0, st
        return obs

    def stock_su3_chain(self, L, beta, width, seed, chains, warmup, sweeps):
        """The reference's own SU(3) L^4 chains (SUGauge<3>, SUShift, 1 hit,
        plain Pcg32 seeded seed + c), one per thread: (chains, sweeps) mean
        plaquettes after `warmup`."""
        plaq = np.zeros((chains, sweeps))
        st = self._stock_su3(L, beta, width, seed, chains, warmup, sweeps, _ptr(plaq))
        assert st == 0, st
        return plaq

    def bench_o3(self, L, beta, warmup, steps, threads, seed=1):
        """Reference stock path, O(3) L^3 (1 Wolff flip + 1 sweep per step):
        (site-updates, seconds of the slowest thread)."""
        su = C.c_double()
        sec = C.c_double()
        st = self._bench_o3(L, beta, warmup, steps, threads, seed, C.byref(su), C.byref(sec))
        assert st == 0, st
        return su.value, sec.value

    def bench_ising(self, L, beta, warmup, sweeps, threads, seed=1):
        su = C.c_double()
        sec = C.c_double()
        st = self._bench_ising(L, beta, warmup, sweeps, threads, seed, C.byref(su), C.byref(sec))
        assert st == 0, st
        return su.value, sec.value


def _bench_xy(self, L, beta, width, warmup, sweeps, threads, seed=1):
    su = C.c_double()
    sec = C.c_double()
    st = self._bench_xy(L, beta, width, warmup, sweeps, threads, seed, C.byref(su), C.byref(sec))
    assert st == 0, st
    return su.value, sec.value


Reference.bench_xy = _bench_xy


def _bench_pair_o3(self, L, beta, warmup, sweeps, threads, seed=1):
    """Reference PairModel<VectorDof<3>, HeisenbergTerm<3>> Metropolis on L^3:
    (site-updates, seconds of the slowest thread)."""
    su = C.c_double()
    sec = C.c_double()
    st = self._bench_pair_o3(L, beta, warmup, sweeps, threads, seed, C.byref(su), C.byref(sec))
    assert st == 0, st
    return su.value, sec.value


Reference.bench_pair_o3 = _bench_pair_o3


def _bench_ising_wolff(self, L, beta, warmup, flips, threads, seed=1):
    """Reference Ising Wolff (FixedAxis) on L x L: (flipped sites of the timed
    flips over all threads, seconds of the slowest thread)."""
    su = C.c_double()
    sec = C.c_double()
    st = self._bench_ising_wolff(L, beta, warmup, flips, threads, seed, C.byref(su), C.byref(sec))
    assert st == 0, st
    return su.value, sec.value


Reference.bench_ising_wolff = _bench_ising_wolff


def _bench_u1_cells(self, L, model_beta, beta, width, warmup, sweeps, threads, seed=1):
    """Reference CellModel<U1Dof, U1PlaquetteTerm, CellComplex<4>> Metropolis on
    L^4: (link-updates, seconds of the slowest thread)."""
    su = C.c_double()
    sec = C.c_double()
    st = self._bench_u1_cells(L, model_beta, beta, width, warmup, sweeps, threads, seed, C.byref(su), C.byref(sec))
    assert st == 0, st
    return su.value, sec.value


Reference.bench_u1_cells = _bench_u1_cells


def _bench_su3(self, L, model_beta, width, hits, window, sweeps, threads, seed=1):
    """ref_bench_su3: the reference's stock SU(3) multi-hit Metropolis timed on
    a window of links per thread; returns (link-updates, seconds)."""
    su, sec = _f64(0), _f64(0)
    st = self._bench_su3(L, model_beta, width, hits, window, sweeps, threads, seed, C.byref(su), C.byref(sec))
    assert st == 0, st
    return su.value, sec.value


Reference.bench_su3 = _bench_su3


def have_reference() -> bool:
    return os.path.isfile(REF_SO)


def _host_has_x86_64_v3() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    # lzcnt is listed as abm on some kernels
                    return _X86_64_V3 <= (flags | ({"lzcnt"} if "abm" in flags else set()))
    except OSError:
        pass
    return False


def timing_reference():
    """(Reference, build) for the timed CPU baselines: the -O3 x86-64-v3 build
    of the harness when it exists and the host runs that instruction set, else
    the portable -O2 parity build.  None when neither was built."""
    if os.path.isfile(REF_FAST_SO) and _host_has_x86_64_v3():
        return Reference(REF_FAST_SO), "g++ -O3 -march=x86-64-v3"
    if os.path.isfile(REF_SO):
        return Reference(REF_SO), "g++ -O2 (portable parity build)"
    return None
