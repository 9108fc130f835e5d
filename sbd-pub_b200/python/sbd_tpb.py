"""ctypes binding of libsbdtpb (the C ABI in include/sbd_tpb.h).

Python-side mirror of the reference's one-rank TPB entry points: ``diag`` replaces
``sbd::tpb::diag`` (tpb/sbdiag.h:139-151) and ``Handle`` exposes the stages it is made of --
excitation tables (tpb/helper.h:185-323), the diagonal (tpb/qcham.h:290-340), sigma
(``MultBase::run``, basic/mult.h:94-102), Davidson (tpb/davidson.h:667-930) and the RDMs
(tpb/correlation.h:378-664).  Every call goes to the CUDA library; there is no CPU fallback:
loading raises when ``lib/libsbdtpb.so`` is missing and calls raise ``TpbError`` with the
library's message on any failure status.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libsbdtpb.so")

OK = 0
ERR_INVALID = -1
ERR_CUDA = -2
ERR_OOM = -3
ERR_NOT_CONVERGED = -4
ERR_STATE = -5
ERR_IO = -6
ERR_NO_DEVICE = -7
HOST, DEVICE = 0, 1
SINGLES_ALPHA, DOUBLES_ALPHA, SINGLES_BETA, DOUBLES_BETA = 0, 1, 2, 3
FP64, MIXED = 0, 1
METHOD_DAVIDSON, METHOD_LANCZOS = 0, 2
PRECOND_DIAGONAL, PRECOND_LEARNED = 0, 1

# Every function the header declares (the symbol test checks the library against this list).
EXPORTED = [
    "sbd_tpb_default_params", "sbd_tpb_diag", "sbd_tpb_diag_from", "sbd_tpb_last_error", "sbd_tpb_create",
    "sbd_tpb_destroy", "sbd_tpb_set_hamiltonian", "sbd_tpb_set_strings", "sbd_tpb_build_tables",
    "sbd_tpb_table_size", "sbd_tpb_get_table", "sbd_tpb_diagonal", "sbd_tpb_sigma",
    "sbd_tpb_sigma_f32", "sbd_tpb_sigma_device", "sbd_tpb_sigma_noalloc", "sbd_tpb_davidson", "sbd_tpb_rdm", "sbd_tpb_stream",
    "sbd_tpb_last_sigma_ms", "sbd_tpb_last_sigma_kernels", "sbd_tpb_kernel_launches", "sbd_tpb_release_work",
    "sbd_tpb_precond_create", "sbd_tpb_precond_destroy", "sbd_tpb_precond_collect",
    "sbd_tpb_precond_num_samples", "sbd_tpb_precond_train", "sbd_tpb_precond_evaluate",
    "sbd_tpb_precond_get_params", "sbd_tpb_precond_set_params", "sbd_tpb_precond_gradients",
    "sbd_tpb_precond_apply", "sbd_tpb_set_preconditioner", "sbd_tpb_carryover_strings",
    "sbd_tpb_carryover_capacity", "sbd_tpb_last_carryover_ms", "sbd_tpb_lanczos",
    "sbd_tpb_parse_strings", "sbd_tpb_read_strings", "sbd_tpb_last_parse_ms",
]
STRINGS_TEXT, STRINGS_BINARY = 0, 1
CARRYOVER_NONE, CARRYOVER_DOMINANT, CARRYOVER_DOMINANT_SINGLES, CARRYOVER_CUTOFF_SINGLES = 0, 1, 2, 3
ERR_CAPACITY = -8
MLP_HIDDEN, MLP_FEATURES, MLP_PARAMS = 256, 64, 82689


class TpbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"sbd_tpb error {code}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("max_it", C.c_int), ("max_nb", C.c_int), ("eps", C.c_double), ("max_time", C.c_double),
        ("init", C.c_int), ("do_rdm", C.c_int), ("precision", C.c_int), ("preconditioner", C.c_int),
        ("verbose", C.c_int), ("device", C.c_int), ("symmetry", C.c_int), ("method", C.c_int),
        ("seed", C.c_ulonglong),
    ]


class Hamiltonian(C.Structure):
    _fields_ = [
        ("norb", C.c_int), ("nelec", C.c_int), ("core_energy", C.c_double),
        ("h1", C.POINTER(C.c_double)), ("eri_packed", C.POINTER(C.c_double)),
        ("n_eri_packed", C.c_size_t),
    ]


class Carryover(C.Structure):
    _fields_ = [
        ("type", C.c_int), ("ratio", C.c_double), ("threshold", C.c_double),
        ("astr", C.POINTER(C.c_uint64)), ("acap", C.c_size_t), ("na", C.c_size_t),
        ("bstr", C.POINTER(C.c_uint64)), ("bcap", C.c_size_t), ("nb", C.c_size_t),
        ("truncated_a", C.c_double), ("truncated_b", C.c_double), ("total_weight", C.c_double),
    ]


class Result(C.Structure):
    _fields_ = [
        ("energy", C.c_double), ("residual", C.c_double), ("iterations", C.c_int),
        ("converged", C.c_int), ("ci_vector", C.POINTER(C.c_double)),
        ("density", C.POINTER(C.c_double)), ("one_rdm", C.POINTER(C.c_double)),
        ("two_rdm", C.POINTER(C.c_double)), ("seconds_tables", C.c_double),
        ("seconds_davidson", C.c_double), ("seconds_rdm", C.c_double),
        ("seconds_total", C.c_double), ("learned_steps", C.c_int), ("fallback_steps", C.c_int),
        ("carryover", C.POINTER(Carryover)),
    ]


_lib = None


def lib():
    """Load libsbdtpb.so (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C sbd-pub_b200`")
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    L.sbd_tpb_last_error.restype = C.c_char_p
    L.sbd_tpb_default_params.argtypes = [C.POINTER(Params)]
    L.sbd_tpb_diag.argtypes = [C.POINTER(Params), C.POINTER(Hamiltonian), vp, C.c_size_t, vp,
                               C.c_size_t, C.POINTER(Result)]
    L.sbd_tpb_diag_from.argtypes = [C.POINTER(Params), C.POINTER(Hamiltonian), vp, C.c_size_t, vp,
                                    C.c_size_t, vp, C.POINTER(Result)]
    L.sbd_tpb_create.argtypes = [C.c_int, C.POINTER(vp)]
    L.sbd_tpb_destroy.argtypes = [vp]
    L.sbd_tpb_set_hamiltonian.argtypes = [vp, C.POINTER(Hamiltonian)]
    L.sbd_tpb_set_strings.argtypes = [vp, vp, C.c_size_t, vp, C.c_size_t]
    L.sbd_tpb_build_tables.argtypes = [vp]
    L.sbd_tpb_table_size.argtypes = [vp, C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
    L.sbd_tpb_get_table.argtypes = [vp, C.c_int, vp, vp, vp]
    L.sbd_tpb_diagonal.argtypes = [vp, vp, C.c_int]
    L.sbd_tpb_sigma.argtypes = [vp, vp, vp, C.c_int, C.c_int]
    L.sbd_tpb_sigma_f32.argtypes = [vp, vp, vp, C.c_int, C.c_int]
    L.sbd_tpb_sigma_device.argtypes = [vp, vp, vp, C.c_int, C.c_int, C.c_int]
    L.sbd_tpb_sigma_noalloc.argtypes = [vp, vp, vp, C.c_int, C.c_int]
    L.sbd_tpb_davidson.argtypes = [vp, C.POINTER(Params), vp, C.POINTER(Result)]
    L.sbd_tpb_rdm.argtypes = [vp, vp, vp, vp, C.c_int]
    L.sbd_tpb_lanczos.argtypes = [vp, C.POINTER(Params), vp, C.POINTER(Result)]
    L.sbd_tpb_parse_strings.argtypes = [vp, vp, C.c_size_t, C.c_int, C.c_int, vp, C.c_size_t,
                                        C.POINTER(C.c_size_t)]
    L.sbd_tpb_read_strings.argtypes = [vp, C.c_char_p, C.c_int, vp, C.c_size_t, C.POINTER(C.c_size_t)]
    L.sbd_tpb_last_parse_ms.restype = C.c_double
    L.sbd_tpb_last_parse_ms.argtypes = [vp]
    L.sbd_tpb_stream.restype = vp
    L.sbd_tpb_stream.argtypes = [vp]
    L.sbd_tpb_last_sigma_ms.restype = C.c_double
    L.sbd_tpb_last_sigma_ms.argtypes = [vp]
    L.sbd_tpb_last_sigma_kernels.argtypes = [vp, C.POINTER(C.c_double), C.c_int]
    L.sbd_tpb_kernel_launches.restype = C.c_uint64
    L.sbd_tpb_kernel_launches.argtypes = [vp]
    L.sbd_tpb_release_work.argtypes = [vp]
    L.sbd_tpb_precond_create.argtypes = [C.c_int, C.c_uint64, C.POINTER(vp)]
    L.sbd_tpb_precond_destroy.argtypes = [vp]
    L.sbd_tpb_precond_collect.argtypes = [vp, vp, C.POINTER(Params), C.c_size_t, C.c_int,
                                          C.POINTER(C.c_double)]
    L.sbd_tpb_precond_num_samples.argtypes = [vp, C.c_int, C.POINTER(C.c_size_t)]
    L.sbd_tpb_precond_train.argtypes = [vp, C.c_int, C.c_int, C.c_double, C.POINTER(C.c_double)]
    L.sbd_tpb_precond_evaluate.argtypes = [vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.sbd_tpb_precond_get_params.argtypes = [vp, vp, C.c_size_t]
    L.sbd_tpb_precond_set_params.argtypes = [vp, vp, C.c_size_t]
    L.sbd_tpb_precond_gradients.argtypes = [vp, C.c_size_t, vp, vp, vp, vp, vp,
                                            C.POINTER(C.c_double), vp]
    L.sbd_tpb_precond_apply.argtypes = [vp, vp, vp, C.c_double, C.c_double, vp]
    L.sbd_tpb_set_preconditioner.argtypes = [vp, vp]
    L.sbd_tpb_carryover_strings.argtypes = [vp, vp, C.c_int, C.POINTER(Carryover)]
    L.sbd_tpb_carryover_capacity.restype = C.c_size_t
    L.sbd_tpb_carryover_capacity.argtypes = [vp, C.c_int, C.c_int]
    L.sbd_tpb_last_carryover_ms.argtypes = [vp, C.POINTER(C.c_double)]
    _lib = L
    return L


def _check(rc: int, allow=(OK,)):
    if rc not in allow:
        raise TpbError(rc, lib().sbd_tpb_last_error().decode(errors="replace"))
    return rc


def _ptr(a) -> int:
    """Address of a C-contiguous numpy array or a torch tensor."""
    if isinstance(a, np.ndarray):
        assert a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    return a.data_ptr()  # torch tensor (host or device)


def default_params(**kw) -> Params:
    p = Params()
    lib().sbd_tpb_default_params(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


@dataclass
class Problem:
    """An FCIDUMP-style Hamiltonian and its alpha/beta strings (host numpy arrays)."""
    norb: int
    nelec: int
    core: float
    h1: np.ndarray          # [L, L] float64
    eri_packed: np.ndarray  # packed 8-fold store, float64
    astr: np.ndarray        # uint64
    bstr: np.ndarray        # uint64

    def ham_struct(self) -> Hamiltonian:
        self._h1c = np.ascontiguousarray(self.h1, np.float64)
        self._eric = np.ascontiguousarray(self.eri_packed, np.float64)
        return Hamiltonian(self.norb, self.nelec, self.core,
                           self._h1c.ctypes.data_as(C.POINTER(C.c_double)),
                           self._eric.ctypes.data_as(C.POINTER(C.c_double)), self._eric.size)

    @property
    def ndet(self) -> int:
        return len(self.astr) * len(self.bstr)


class Handle:
    """One GPU, one problem: tables, diagonal, sigma, Davidson and RDMs (include/sbd_tpb.h)."""

    def __init__(self, device: int = 0):
        self.h = C.c_void_p()
        self.device = device
        _check(lib().sbd_tpb_create(device, C.byref(self.h)))
        self.problem: Problem | None = None

    def close(self):
        if self.h:
            lib().sbd_tpb_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_problem(self, prob: Problem, build: bool = True):
        self.problem = prob
        hs = prob.ham_struct()
        _check(lib().sbd_tpb_set_hamiltonian(self.h, C.byref(hs)))
        a = np.ascontiguousarray(prob.astr, np.uint64)
        b = np.ascontiguousarray(prob.bstr, np.uint64)
        _check(lib().sbd_tpb_set_strings(self.h, a.ctypes.data, len(a), b.ctypes.data, len(b)))
        if build:
            self.build_tables()

    def build_tables(self):
        _check(lib().sbd_tpb_build_tables(self.h))

    def table(self, kind: int):
        """(off[n+1] u64, ket[nnz] u64, cran[2|4 * nnz] i32) in the reference layout."""
        nrows, nnz = C.c_size_t(), C.c_size_t()
        _check(lib().sbd_tpb_table_size(self.h, kind, C.byref(nrows), C.byref(nnz)))
        per = 2 if kind in (SINGLES_ALPHA, SINGLES_BETA) else 4
        off = np.zeros(nrows.value + 1, np.uint64)
        ket = np.zeros(max(nnz.value, 1), np.uint64)
        cran = np.zeros(max(nnz.value, 1) * per, np.int32)
        _check(lib().sbd_tpb_get_table(self.h, kind, off.ctypes.data, ket.ctypes.data, cran.ctypes.data))
        return off, ket[: nnz.value], cran[: nnz.value * per]

    def diagonal(self) -> np.ndarray:
        out = np.zeros(self.problem.ndet)
        _check(lib().sbd_tpb_diagonal(self.h, out.ctypes.data, HOST))
        return out

    def diagonal_device(self):
        """H_ii as a torch float64 CUDA tensor on the handle's device (sbd_tpb_diagonal, device copy)."""
        import torch
        out = torch.empty(self.problem.ndet, dtype=torch.float64, device=f"cuda:{self.device}")
        _check(lib().sbd_tpb_diagonal(self.h, out.data_ptr(), DEVICE))
        return out

    def sigma(self, C_, out=None, accumulate: bool = False):
        """sigma (+)= H C for numpy (host) or torch CUDA (device) vectors, float64 or float32."""
        dev = not isinstance(C_, np.ndarray)
        if out is None:
            if dev:
                import torch
                out = torch.zeros_like(C_)
            else:
                out = np.zeros_like(C_)
        f32 = (C_.dtype == np.float32) if not dev else (str(C_.dtype) == "torch.float32")
        fn = lib().sbd_tpb_sigma_f32 if f32 else lib().sbd_tpb_sigma
        _check(fn(self.h, _ptr(C_), _ptr(out), int(accumulate), DEVICE if dev else HOST))
        return out

    def _device_pair(self, x, y) -> int:
        """dtype code (0 float64, 1 float32) of two torch CUDA N-vectors the device entry points
        may read and write: same dtype, one of the two, ndet elements, contiguous, on the
        handle's device, distinct buffers."""
        import torch
        if x.dtype not in (torch.float64, torch.float32) or y.dtype != x.dtype:
            raise TpbError(ERR_INVALID, f"sigma vectors must both be float64 or float32 (got {x.dtype}, {y.dtype})")
        for t in (x, y):
            if not t.is_cuda or t.device.index != self.device:
                raise TpbError(ERR_INVALID, f"sigma vectors must live on cuda:{self.device}")
            if not t.is_contiguous() or t.numel() != self.problem.ndet:
                raise TpbError(ERR_INVALID, f"sigma vectors must be contiguous with {self.problem.ndet} elements")
        if x.data_ptr() == y.data_ptr():
            raise TpbError(ERR_INVALID, "sigma input and output must be distinct buffers")
        return 1 if x.dtype == torch.float32 else 0

    def sigma_device(self, x, y, accumulate=False, separated=True, symmetric=False):
        """sigma on torch CUDA tensors; separated=True keeps the library's internal convention;
        symmetric=True (separated, exchange-symmetric x over identical string lists) takes the
        one-pass form (convention 2)."""
        dt = self._device_pair(x, y)
        conv = 2 if symmetric else (1 if separated else 0)
        _check(lib().sbd_tpb_sigma_device(self.h, x.data_ptr(), y.data_ptr(), dt, int(accumulate), conv))
        return y

    def sigma_noalloc(self, x, y, accumulate=False):
        """sigma into caller-owned torch CUDA tensors without any device allocation by the
        library (separated convention, fixed 16 MiB scratch; see sbd_tpb_sigma_noalloc)."""
        dt = self._device_pair(x, y)
        _check(lib().sbd_tpb_sigma_noalloc(self.h, x.data_ptr(), y.data_ptr(), dt, int(accumulate)))
        return y

    def last_sigma_ms(self) -> float:
        return lib().sbd_tpb_last_sigma_ms(self.h)

    def last_sigma_kernels(self):
        """Device ms of each stage of the last sigma: [alpha pass, beta pass, alpha-beta term]."""
        buf = (C.c_double * 8)()
        n = lib().sbd_tpb_last_sigma_kernels(self.h, buf, 8)
        _check(n if n < 0 else OK)
        return [buf[i] for i in range(n)]

    def kernel_launches(self) -> int:
        return int(lib().sbd_tpb_kernel_launches(self.h))

    def free_vectors(self):
        """Release the cached work memory (Davidson vectors, sigma staging): sbd_tpb_release_work."""
        _check(lib().sbd_tpb_release_work(self.h))

    def stream(self) -> int:
        return lib().sbd_tpb_stream(self.h) or 0

    def davidson(self, params: Params | None = None, W0: np.ndarray | None = None,
                 want_vector=True, want_rdm=False, carryover: tuple | None = None):
        """Davidson (or Lanczos when params.method == METHOD_LANCZOS) on the handle's problem;
        carryover = (type, ratio, threshold) also returns the carry-over strings of the final vector
        under "carryover"."""
        prob = self.problem
        params = params or default_params()
        res = Result()
        W = np.zeros(prob.ndet) if want_vector else None
        dens = np.zeros(2 * prob.norb)
        one = np.zeros(2 * prob.norb ** 2) if want_rdm else None
        two = np.zeros(4 * prob.norb ** 4) if want_rdm else None
        dp = C.POINTER(C.c_double)
        res.ci_vector = W.ctypes.data_as(dp) if W is not None else dp()
        res.density = dens.ctypes.data_as(dp)
        res.one_rdm = one.ctypes.data_as(dp) if one is not None else dp()
        res.two_rdm = two.ctypes.data_as(dp) if two is not None else dp()
        co = bufs = None
        if carryover is not None:
            co, bufs = self._carryover_record(*carryover)
            res.carryover = C.pointer(co)
        w0 = None if W0 is None else np.ascontiguousarray(W0, np.float64)
        solver = lib().sbd_tpb_lanczos if params.method == METHOD_LANCZOS else lib().sbd_tpb_davidson
        rc = solver(self.h, C.byref(params), w0.ctypes.data if w0 is not None else None, C.byref(res))
        _check(rc, allow=(OK, ERR_NOT_CONVERGED))
        return dict(energy=res.energy, residual=res.residual, iterations=res.iterations,
                    converged=bool(res.converged), W=W, density=dens, one=one, two=two,
                    seconds=res.seconds_davidson, learned_steps=res.learned_steps,
                    fallback_steps=res.fallback_steps,
                    carryover=self._carryover_result(co, bufs) if co is not None else None)

    def set_preconditioner(self, pc: "Precond | None"):
        """Attach a learned preconditioner (used when params.preconditioner == PRECOND_LEARNED)."""
        _check(lib().sbd_tpb_set_preconditioner(self.h, pc.p if pc is not None else None))
        self._pc = pc  # keep it alive while attached

    def _carryover_record(self, kind: int, ratio: float, threshold: float):
        co = Carryover(type=kind, ratio=ratio, threshold=threshold)
        bufs = []
        for spin, (pf, cf) in enumerate((("astr", "acap"), ("bstr", "bcap"))):
            cap = int(lib().sbd_tpb_carryover_capacity(self.h, kind, spin))
            buf = np.zeros(max(cap, 1), np.uint64)
            setattr(co, pf, buf.ctypes.data_as(C.POINTER(C.c_uint64)))
            setattr(co, cf, cap)
            bufs.append(buf)
        return co, bufs

    @staticmethod
    def _carryover_result(co, bufs):
        return dict(astr=bufs[0][:co.na].copy(), bstr=bufs[1][:co.nb].copy(), truncated_a=co.truncated_a,
                    truncated_b=co.truncated_b, total_weight=co.total_weight)

    def carryover(self, W, kind: int, ratio: float = 0.0, threshold: float = 0.01, mem: int = HOST):
        """Carry-over strings of W (sbd_tpb_carryover_strings): dict with astr, bstr, truncated_a/b,
        total_weight.  W is a host array or, with mem=DEVICE, a device tensor/pointer."""
        co, bufs = self._carryover_record(kind, ratio, threshold)
        if mem == HOST:
            w = np.ascontiguousarray(W, np.float64)
            assert w.size == self.problem.ndet
            ptr = w.ctypes.data
        else:
            ptr = W if isinstance(W, int) else W.data_ptr()
        _check(lib().sbd_tpb_carryover_strings(self.h, ptr, mem, C.byref(co)))
        return self._carryover_result(co, bufs)

    def parse_strings(self, data, norb: int, fmt: int = STRINGS_TEXT) -> np.ndarray:
        """Sorted unique strings of a string file's bytes, parsed on the GPU (sbd_tpb_parse_strings)."""
        buf = np.frombuffer(bytes(data), np.uint8) if not isinstance(data, np.ndarray) else data
        buf = np.ascontiguousarray(buf, np.uint8)
        cap = (len(buf) // ((norb + 7) // 8)) if fmt == STRINGS_BINARY else len(buf) // (norb + 1) + 1
        out = np.zeros(max(cap, 1), np.uint64)
        n = C.c_size_t(0)
        _check(lib().sbd_tpb_parse_strings(self.h, buf.ctypes.data if len(buf) else None, len(buf), fmt, norb,
                                           out.ctypes.data, len(out), C.byref(n)))
        return out[: n.value].copy()

    def read_strings(self, path: str, norb: int) -> np.ndarray:
        """Sorted unique strings of a .txt or .bin string file, parsed on the GPU (sbd_tpb_read_strings)."""
        size = os.path.getsize(path)
        cap = size // ((norb + 7) // 8) if path.endswith(".bin") else size // (norb + 1) + 1
        out = np.zeros(max(cap, 1), np.uint64)
        n = C.c_size_t(0)
        _check(lib().sbd_tpb_read_strings(self.h, path.encode(), norb, out.ctypes.data, len(out), C.byref(n)))
        return out[: n.value].copy()

    def last_parse_ms(self) -> float:
        return float(lib().sbd_tpb_last_parse_ms(self.h))

    def last_carryover_ms(self):
        """(weight pass ms, whole call ms) of the last carry-over on this handle."""
        ms = (C.c_double * 2)()
        _check(lib().sbd_tpb_last_carryover_ms(self.h, ms))
        return float(ms[0]), float(ms[1])

    def rdm(self, W: np.ndarray, two_body=True):
        L = self.problem.norb
        one = np.zeros(2 * L * L)
        two = np.zeros(4 * L ** 4) if two_body else None
        w = np.ascontiguousarray(W, np.float64)
        _check(lib().sbd_tpb_rdm(self.h, w.ctypes.data, one.ctypes.data,
                                 two.ctypes.data if two is not None else None, HOST))
        return one, two


class Precond:
    """Learned Davidson preconditioner (MLP, trained by the library's own kernels)."""

    def __init__(self, device: int = 0, seed: int = 1):
        self.p = C.c_void_p()
        _check(lib().sbd_tpb_precond_create(device, seed, C.byref(self.p)))

    def close(self):
        if self.p:
            lib().sbd_tpb_precond_destroy(self.p)
            self.p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def collect(self, handle: Handle, params: Params | None = None, samples_per_step=1 << 17,
                role=0) -> float:
        """Plain FP64 Davidson on the handle's problem; its steps become training pairs."""
        params = params or default_params(max_it=4, max_nb=10, eps=1e-8)
        e = C.c_double()
        _check(lib().sbd_tpb_precond_collect(self.p, handle.h, C.byref(params), samples_per_step,
                                             role, C.byref(e)))
        return e.value

    def num_samples(self, role=0) -> int:
        n = C.c_size_t()
        _check(lib().sbd_tpb_precond_num_samples(self.p, role, C.byref(n)))
        return n.value

    def train(self, epochs=3, batch=8192, lr=1e-3) -> float:
        loss = C.c_double()
        _check(lib().sbd_tpb_precond_train(self.p, epochs, batch, lr, C.byref(loss)))
        return loss.value

    def evaluate(self, role=1):
        """(learned, diagonal) weighted squared errors against the exact corrections of a set."""
        a, b = C.c_double(), C.c_double()
        _check(lib().sbd_tpb_precond_evaluate(self.p, role, C.byref(a), C.byref(b)))
        return a.value, b.value

    def get_params(self) -> np.ndarray:
        out = np.zeros(MLP_PARAMS, np.float32)
        _check(lib().sbd_tpb_precond_get_params(self.p, out.ctypes.data, out.size))
        return out

    def set_params(self, params: np.ndarray):
        x = np.ascontiguousarray(params, np.float32)
        _check(lib().sbd_tpb_precond_set_params(self.p, x.ctypes.data, x.size))

    def gradients(self, x, a, b, w):
        """One forward/backward pass of the training kernels: (grad, loss, y)."""
        x = np.ascontiguousarray(x, np.float32)
        a, b, w = (np.ascontiguousarray(v, np.float32) for v in (a, b, w))
        n = len(a)
        grad = np.zeros(MLP_PARAMS, np.float32)
        y = np.zeros(n, np.float32)
        loss = C.c_double()
        _check(lib().sbd_tpb_precond_gradients(self.p, n, x.ctypes.data, a.ctypes.data, b.ctypes.data,
                                               w.ctypes.data, grad.ctypes.data, C.byref(loss),
                                               y.ctypes.data))
        return grad, loss.value, y

    def apply(self, handle: Handle, d: np.ndarray, e0: float, rnorm: float) -> np.ndarray:
        """The fused inference kernel on the handle's determinants: t = d (1 + y)."""
        d = np.ascontiguousarray(d, np.float64)
        t = np.zeros_like(d)
        _check(lib().sbd_tpb_precond_apply(handle.h, self.p, d.ctypes.data, e0, rnorm, t.ctypes.data))
        return t


def mlp_unpack(params: np.ndarray):
    """Split the flat parameter vector into (W1 [256,64], b1, W2 [256,256], b2, w3, b3)."""
    H, F = MLP_HIDDEN, MLP_FEATURES
    o = 0
    W1 = params[o:o + H * F].reshape(H, F); o += H * F
    b1 = params[o:o + H]; o += H
    W2 = params[o:o + H * H].reshape(H, H); o += H * H
    b2 = params[o:o + H]; o += H
    w3 = params[o:o + H]; o += H
    b3 = params[o:o + 1]
    return W1, b1, W2, b2, w3, b3


def diag(prob: Problem, params: Params | None = None, want_rdm=False):
    """One-shot solve: sbd::tpb::diag for one rank (tpb/sbdiag.h:139-151)."""
    params = params or default_params()
    res = Result()
    W = np.zeros(prob.ndet)
    dens = np.zeros(2 * prob.norb)
    one = np.zeros(2 * prob.norb ** 2) if want_rdm else None
    two = np.zeros(4 * prob.norb ** 4) if want_rdm else None
    dp = C.POINTER(C.c_double)
    res.ci_vector = W.ctypes.data_as(dp)
    res.density = dens.ctypes.data_as(dp)
    res.one_rdm = one.ctypes.data_as(dp) if one is not None else dp()
    res.two_rdm = two.ctypes.data_as(dp) if two is not None else dp()
    params.do_rdm = int(want_rdm)
    hs = prob.ham_struct()
    a = np.ascontiguousarray(prob.astr, np.uint64)
    b = np.ascontiguousarray(prob.bstr, np.uint64)
    rc = lib().sbd_tpb_diag(C.byref(params), C.byref(hs), a.ctypes.data, len(a), b.ctypes.data,
                            len(b), C.byref(res))
    _check(rc, allow=(OK, ERR_NOT_CONVERGED))
    return dict(energy=res.energy, residual=res.residual, iterations=res.iterations,
                converged=bool(res.converged), W=W, density=dens, one=one, two=two,
                seconds_tables=res.seconds_tables, seconds_davidson=res.seconds_davidson,
                seconds_total=res.seconds_total)
