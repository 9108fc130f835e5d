"""ctypes binding of the CPU oracle (liboracle.so): TEST INFRASTRUCTURE ONLY.

The oracle restates the reference TPB path on the CPU (see sbd_oracle.h).  Tests, the smoke
check and the CPU-baseline leg of bench.py use it as the checker; the product never does.
Build it with ``make -C oracle oracle``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")


class Ham(C.Structure):
    _fields_ = [
        ("L", C.c_int),
        ("nelec", C.c_int),
        ("I0", C.c_double),
        ("I1", C.POINTER(C.c_double)),
        ("I2", C.POINTER(C.c_double)),
        ("n_I2", C.c_size_t),
        ("direct", C.POINTER(C.c_double)),
        ("exchange", C.POINTER(C.c_double)),
    ]


class Tables(C.Structure):
    _fields_ = [("na", C.c_size_t), ("nb", C.c_size_t)] + [
        (f"{k}_{f}", C.POINTER(t))
        for k in ("sa", "da", "sb", "db")
        for f, t in (("off", C.c_uint64), ("ket", C.c_uint64), ("cran", C.c_int32))
    ]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is not built (make -C oracle oracle)")
        L = C.CDLL(path)
        L.orc_load_fcidump.argtypes = [C.c_char_p, C.POINTER(Ham)]
        L.orc_ham_from_arrays.argtypes = [C.c_int, C.c_int, C.c_double, _f64p, _f64p, C.POINTER(Ham)]
        L.orc_free_ham.argtypes = [C.POINTER(Ham)]
        L.orc_load_strings.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]
        L.orc_load_strings_bin.argtypes = [C.c_char_p, C.c_int, C.c_void_p, C.c_size_t, C.POINTER(C.c_size_t)]
        L.orc_excitations.restype = C.c_size_t
        L.orc_excitations.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, C.c_int, C.c_int, C.c_int,
                                      _u64p, C.c_void_p, C.c_void_p]
        for name in ("orc_zero_excite",):
            getattr(L, name).restype = C.c_double
            getattr(L, name).argtypes = [C.c_uint64, C.c_uint64, C.POINTER(Ham)]
        L.orc_one_excite.restype = C.c_double
        L.orc_one_excite.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.POINTER(Ham)]
        L.orc_two_excite.restype = C.c_double
        L.orc_two_excite.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(Ham)]
        L.orc_hij.restype = C.c_double
        L.orc_hij.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, C.c_uint64, C.POINTER(Ham)]
        L.orc_diagonal.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, C.POINTER(Ham), _f64p]
        L.orc_build_tables.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, C.c_int, C.POINTER(Tables)]
        L.orc_free_tables.argtypes = [C.POINTER(Tables)]
        L.orc_sigma.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, C.POINTER(Tables), C.POINTER(Ham),
                                _f64p, _f64p, _f64p]
        L.orc_hash_vector.restype = C.c_double
        L.orc_hash_vector.argtypes = [C.c_size_t]
        L.orc_sigma_rows.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, C.POINTER(Tables), C.POINTER(Ham),
                                     C.c_void_p, C.c_void_p, C.c_size_t, _f64p]
        L.orc_davidson.restype = C.c_int
        L.orc_davidson.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, C.POINTER(Tables), C.POINTER(Ham),
                                   _f64p, _f64p, C.c_int, C.c_int, C.c_double, C.c_int,
                                   C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_rdm.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, C.POINTER(Tables), C.c_int, _f64p, _f64p, _f64p]
        L.orc_rdm_energy.argtypes = [C.POINTER(Ham), _f64p, _f64p, _f64p]
        L.orc_reorder_sign.restype = C.c_int
        L.orc_reorder_sign.argtypes = [C.c_uint64, C.c_uint64]
        L.orc_mlp_forward.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p,
                                      _f32p, _f32p, _f32p, _f32p]
        L.orc_lanczos.restype = C.c_int
        L.orc_lanczos.argtypes = [_u64p, C.c_size_t, _u64p, C.c_size_t, C.POINTER(Tables), C.POINTER(Ham),
                                  _f64p, _f64p, C.c_int, C.c_int, C.c_double, C.c_int,
                                  C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.orc_string_weights.argtypes = [_f64p, C.c_size_t, C.c_size_t, C.c_double, _f64p, _f64p, _u64p, _u64p,
                                         C.POINTER(C.c_double)]
        L.orc_carryover_select.restype = C.c_size_t
        L.orc_carryover_select.argtypes = [_f64p, C.c_size_t, C.c_double, C.c_double, _u64p,
                                           C.POINTER(C.c_double)]
        L.orc_singles_extend.restype = C.c_size_t
        L.orc_singles_extend.argtypes = [_u64p, C.c_size_t, C.c_int, _u64p]
        L.orc_mlp_backward.restype = C.c_double
        L.orc_mlp_backward.argtypes = [C.c_int, C.c_int, C.c_int, _f32p, _f32p, _f32p, _f32p, _f32p, _f32p,
                                       _f32p, _f32p, _f32p, _f32p, _f64p, _f64p, _f64p, _f64p, _f64p, _f64p]
        _LIB = L
    return _LIB


class Hamiltonian:
    """Owning wrapper around orc_ham."""

    def __init__(self, ham: Ham):
        self.h = ham

    @classmethod
    def from_fcidump(cls, path: str) -> "Hamiltonian":
        h = Ham()
        rc = lib().orc_load_fcidump(path.encode(), C.byref(h))
        if rc != 0:
            raise ValueError(f"orc_load_fcidump({path}) failed: {rc}")
        return cls(h)

    @classmethod
    def from_arrays(cls, L: int, nelec: int, I0: float, h1: np.ndarray, eri_packed: np.ndarray) -> "Hamiltonian":
        h = Ham()
        lib().orc_ham_from_arrays(L, nelec, I0, np.ascontiguousarray(h1, np.float64),
                                  np.ascontiguousarray(eri_packed, np.float64), C.byref(h))
        return cls(h)

    @property
    def L(self) -> int:
        return self.h.L

    @property
    def I0(self) -> float:
        return self.h.I0

    def h1(self) -> np.ndarray:
        L = self.L
        I1 = np.ctypeslib.as_array(self.h.I1, shape=(4 * L * L,)).reshape(2 * L, 2 * L)
        return I1[0::2, 0::2].copy()

    def eri_packed(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.h.I2, shape=(self.h.n_I2,)).copy()

    def __del__(self):
        try:
            lib().orc_free_ham(C.byref(self.h))
        except Exception:
            pass


def load_strings(path: str, L: int) -> np.ndarray:
    n = C.c_size_t(0)
    rc = lib().orc_load_strings(path.encode(), L, None, 0, C.byref(n))
    if rc != 0:
        raise ValueError(f"orc_load_strings({path}) failed: {rc}")
    out = np.zeros(n.value, np.uint64)
    lib().orc_load_strings(path.encode(), L, out.ctypes.data, n.value, C.byref(n))
    return out


def load_strings_bin(path: str, L: int) -> np.ndarray:
    """Sorted unique strings of a binary string file (orc_load_strings_bin)."""
    n = C.c_size_t(0)
    if lib().orc_load_strings_bin(path.encode(), L, None, 0, C.byref(n)) != 0:
        raise ValueError(f"orc_load_strings_bin({path}) failed")
    out = np.zeros(max(n.value, 1), np.uint64)
    lib().orc_load_strings_bin(path.encode(), L, out.ctypes.data, n.value, C.byref(n))
    return out[: n.value]


def excitations(bra: np.ndarray, ket: np.ndarray, L: int, ndiff: int, spin: int):
    bra = np.ascontiguousarray(bra, np.uint64)
    ket = np.ascontiguousarray(ket, np.uint64)
    off = np.zeros(len(bra) + 1, np.uint64)
    n = lib().orc_excitations(bra, len(bra), ket, len(ket), L, ndiff, spin, off, None, None)
    k = np.zeros(max(n, 1), np.uint64)
    c = np.zeros(max(n, 1) * (2 if ndiff == 2 else 4), np.int32)
    lib().orc_excitations(bra, len(bra), ket, len(ket), L, ndiff, spin, off, k.ctypes.data, c.ctypes.data)
    return off, k[:n], c[: n * (2 if ndiff == 2 else 4)]


def hash_vector(idx) -> np.ndarray:
    """The closed-form test vector at the given indices (same bits as orc_hash_vector)."""
    i = np.asarray(idx, dtype=np.uint64)
    return ((i * np.uint64(0x9E3779B97F4A7C15)) >> np.uint64(11)).astype(np.float64) * 2.0 ** -53 - 0.5


def random_start(n: int, seed: int, normalise: bool = True) -> np.ndarray:
    """The reference's seeded random start (BasisInitVector with init 1, tpb/davidson.h:138-141):
    element i = uniform in [-1, 1) from the splitmix64-style mix of (seed, i) of Randomize
    (framework/dm_vector.h:100-178), in the reference's determinant order and sign convention;
    normalised to unit length when asked (the reference's norm is a Kahan sum per thread, so its
    last bit can differ)."""
    i = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = np.uint64(seed) * np.uint64(6364136223846793005) + i * np.uint64(2862933555777941757)
        x ^= x >> np.uint64(30)
        x *= np.uint64(0xBF58476D1CE4E5B9)
        x ^= x >> np.uint64(27)
        x *= np.uint64(0x94D049BB133111EB)
        x ^= x >> np.uint64(31)
    w = (x >> np.uint64(11)).astype(np.float64) * (2.0 / 9007199254740992.0) - 1.0
    return w / np.sqrt(np.dot(w, w)) if normalise else w


class System:
    """Strings + Hamiltonian + tables: the oracle's view of one TPB problem."""

    def __init__(self, ham: Hamiltonian, astr: np.ndarray, bstr: np.ndarray):
        self.ham = ham
        self.astr = np.ascontiguousarray(astr, np.uint64)
        self.bstr = np.ascontiguousarray(bstr, np.uint64)
        self.t = Tables()
        lib().orc_build_tables(self.astr, len(self.astr), self.bstr, len(self.bstr), ham.L, C.byref(self.t))

    @property
    def na(self):
        return len(self.astr)

    @property
    def nb(self):
        return len(self.bstr)

    def table(self, kind: str):
        """(off, ket, cran) arrays for kind in sa/da/sb/db."""
        n = self.na if kind[1] == "a" else self.nb
        off = np.ctypeslib.as_array(getattr(self.t, kind + "_off"), shape=(n + 1,)).copy()
        nnz = int(off[-1])
        per = 2 if kind[0] == "s" else 4
        ket = np.ctypeslib.as_array(getattr(self.t, kind + "_ket"), shape=(max(nnz, 1),))[:nnz].copy()
        cran = np.ctypeslib.as_array(getattr(self.t, kind + "_cran"), shape=(max(nnz, 1) * per,))[: nnz * per].copy()
        return off, ket, cran

    def diagonal(self) -> np.ndarray:
        out = np.zeros(self.na * self.nb)
        lib().orc_diagonal(self.astr, self.na, self.bstr, self.nb, C.byref(self.ham.h), out)
        return out

    def sigma(self, C_: np.ndarray, hii: np.ndarray | None = None) -> np.ndarray:
        if hii is None:
            hii = self.diagonal()
        out = np.zeros(self.na * self.nb)
        lib().orc_sigma(self.astr, self.na, self.bstr, self.nb, C.byref(self.t), C.byref(self.ham.h),
                        np.ascontiguousarray(hii, np.float64), np.ascontiguousarray(C_, np.float64), out)
        return out

    def sigma_rows(self, rows, C_: np.ndarray | None = None) -> np.ndarray:
        """sigma at the determinant indices `rows` (orc_sigma_rows); C_ = None takes the closed-form
        vector hash_vector(index), so no N-vector is needed."""
        rows = np.ascontiguousarray(rows, np.uint64)
        out = np.zeros(len(rows))
        cptr = None
        if C_ is not None:
            C_ = np.ascontiguousarray(C_, np.float64)
            cptr = C_.ctypes.data
        lib().orc_sigma_rows(self.astr, self.na, self.bstr, self.nb, C.byref(self.t), C.byref(self.ham.h),
                             cptr, rows.ctypes.data, len(rows), out)
        return out

    def davidson(self, max_it=10, max_nb=10, eps=1e-8, verbose=False, W0=None):
        hii = self.diagonal()
        W = np.zeros(self.na * self.nb)
        if W0 is None:
            W[0] = 1.0
        else:
            W[:] = W0
        e = C.c_double(0)
        r = C.c_double(0)
        ns = lib().orc_davidson(self.astr, self.na, self.bstr, self.nb, C.byref(self.t), C.byref(self.ham.h),
                                hii, W, max_it, max_nb, eps, int(verbose), C.byref(e), C.byref(r))
        return e.value, W, ns, r.value

    def lanczos(self, max_it=10, num_block=10, eps=1e-8, verbose=False, W0=None):
        """(energy, W, sigma applications, printed lines, converged) of orc_lanczos from the first
        determinant (or W0)."""
        hii = self.diagonal()
        W = np.zeros(self.na * self.nb)
        if W0 is None:
            W[0] = 1.0
        else:
            W[:] = W0
        e, printed, conv = C.c_double(0), C.c_int(0), C.c_int(0)
        ns = lib().orc_lanczos(self.astr, self.na, self.bstr, self.nb, C.byref(self.t), C.byref(self.ham.h),
                               hii, W, max_it, num_block, eps, int(verbose), C.byref(e), C.byref(printed),
                               C.byref(conv))
        return e.value, W, ns, printed.value, bool(conv.value)

    def rdm(self, W: np.ndarray):
        L = self.ham.L
        one = np.zeros(2 * L * L)
        two = np.zeros(4 * L ** 4)
        lib().orc_rdm(self.astr, self.na, self.bstr, self.nb, C.byref(self.t), L,
                      np.ascontiguousarray(W, np.float64), one, two)
        return one, two

    def rdm_energy(self, one, two):
        out = np.zeros(3)
        lib().orc_rdm_energy(C.byref(self.ham.h), one, two, out)
        return out

    def hij(self, a, b, a2, b2) -> float:
        return lib().orc_hij(int(a), int(b), int(a2), int(b2), C.byref(self.ham.h))

    def __del__(self):
        try:
            lib().orc_free_tables(C.byref(self.t))
        except Exception:
            pass


def reorder_sign(a: int, b: int) -> int:
    return lib().orc_reorder_sign(int(a), int(b))


def string_weights(W: np.ndarray, na: int, nb: int, cutoff: float = 0.0):
    """(wa, wb, ca, cb, total): per-string weights of W and the counts/total above the cutoff
    (orc_string_weights)."""
    W = np.ascontiguousarray(W, np.float64).reshape(-1)
    wa, wb = np.zeros(na), np.zeros(nb)
    ca, cb = np.zeros(na, np.uint64), np.zeros(nb, np.uint64)
    t = C.c_double(0.0)
    lib().orc_string_weights(W, na, nb, float(cutoff), wa, wb, ca, cb, C.byref(t))
    return wa, wb, ca, cb, t.value


def carryover_select(w: np.ndarray, ratio: float, threshold: float):
    """(order[:kept], truncated weight) of the dominant strings (orc_carryover_select)."""
    w = np.ascontiguousarray(w, np.float64)
    order = np.zeros(len(w), np.uint64)
    t = C.c_double(0.0)
    k = lib().orc_carryover_select(w, len(w), float(ratio), float(threshold), order, C.byref(t))
    return order[:k].astype(np.int64), t.value


def singles_extend(s: np.ndarray, L: int) -> np.ndarray:
    """Strings plus all their single excitations, sorted and unique (orc_singles_extend)."""
    s = np.ascontiguousarray(s, np.uint64)
    if len(s) == 0:
        return s.copy()
    e = int(bin(int(s[0])).count("1"))
    out = np.zeros(len(s) * (1 + e * (L - e)), np.uint64)
    m = lib().orc_singles_extend(s, len(s), L, out)
    return out[:m].copy()


def carryover(W: np.ndarray, astr: np.ndarray, bstr: np.ndarray, L: int, kind: int, ratio: float,
              threshold: float):
    """Carry-over strings of W as the reference's sbd::tpb::diag computes them (tpb/sbdiag.h:690-736):
    kind 1 = dominant strings, 2 = dominant strings and their singles, 3 = singles of the strings in
    determinants with W^2 > threshold.  Returns (co_a, co_b, truncated_a, truncated_b, total)."""
    na, nb = len(astr), len(bstr)
    if kind in (1, 2):
        wa, wb, _, _, _ = string_weights(W, na, nb)
        oa, ta = carryover_select(wa, ratio, threshold)
        ob, tb = carryover_select(wb, ratio, threshold)
        co_a, co_b = np.asarray(astr, np.uint64)[oa], np.asarray(bstr, np.uint64)[ob]
        if kind == 2:
            co_a, co_b = singles_extend(co_a, L), singles_extend(co_b, L)
        return co_a, co_b, ta, tb, 0.0
    if kind == 3:
        _, _, ca, cb, total = string_weights(W, na, nb, threshold)
        co_a = singles_extend(np.asarray(astr, np.uint64)[ca > 0], L)
        co_b = singles_extend(np.asarray(bstr, np.uint64)[cb > 0], L)
        return co_a, co_b, 0.0, 0.0, total
    raise ValueError("carry-over kind must be 1, 2 or 3")


def _f32(x):
    return np.ascontiguousarray(x, np.float32)


def mlp_forward(x, W1, b1, W2, b2, w3, b3):
    """y of the preconditioner MLP (orc_mlp_forward), x [n, din]."""
    x, W1, b1, W2, b2, w3, b3 = (_f32(v) for v in (x, W1, b1, W2, b2, w3, b3))
    n, din = x.shape
    dh = W1.shape[0]
    h1 = np.zeros((n, dh), np.float32)
    h2 = np.zeros((n, dh), np.float32)
    y = np.zeros(n, np.float32)
    lib().orc_mlp_forward(n, din, dh, x, W1, b1, W2, b2, w3, b3, h1, h2, y)
    return y


def mlp_backward(x, a, b, w, W1, b1, W2, b2, w3, b3):
    """(loss, [gW1, gb1, gW2, gb2, gw3, gb3]) of the weighted preconditioner loss (orc_mlp_backward)."""
    x, a, b, w, W1, b1, W2, b2, w3, b3 = (_f32(v) for v in (x, a, b, w, W1, b1, W2, b2, w3, b3))
    n, din = x.shape
    dh = W1.shape[0]
    g = [np.zeros(W1.shape), np.zeros(dh), np.zeros(W2.shape), np.zeros(dh), np.zeros(dh), np.zeros(1)]
    loss = lib().orc_mlp_backward(n, din, dh, x, a, b, w, W1, b1, W2, b2, w3, b3, *g)
    return loss, g
