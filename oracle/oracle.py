"""TEST INFRASTRUCTURE ONLY — Python face of the oracle.

Three independent CPU references for the reference's CFFT/RFFT path:

* ``port``: the project's scalar C restatement of the reference algorithm
  (oracle/zlfft_oracle.c -> oracle/_build/libzloracle.so). Bit-identical to
  the reference's micro-only Stockham path when twiddle tables agree, and,
  inside ``hybrid()``, to its macro DIF path.
* ``ref``: the reference's own headers, unchanged, compiled against the
  project's Highway-API shim (oracle/ref_capi.cpp -> oracle/_ref/libzlref.so).
  Present only where it was built (the build reads the reference sources).
  A second build (oracle/_ref/libzlref_macro.so) links the same code with a
  sysconf() stand-in reporting a small-cache host (oracle/ref_sysconf_wrap.cpp),
  so that the reference's own switch sends orders >= 14 (float) / 13 (double)
  down its Cooley-Tukey DIF macro path (src/common/zldsp_fft_common_execute.hpp:174-272).
* ``fp64``: numpy.fft in complex128, scaled to the reference's unnormalised
  conventions: CFFT backward = N * ifft, RFFT backward = (N/2) * irfft
  (src/common/zldsp_fft_common_structure.hpp:47-135,
  src/common/zldsp_fft_common_execute.hpp:407-408).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module. The product library never imports it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PORT_SO = os.path.join(HERE, "_build", "libzloracle.so")
REF_SO = os.path.join(HERE, "_ref", "libzlref.so")
REF_MACRO_SO = os.path.join(HERE, "_ref", "libzlref_macro.so")
# (max_l1_order, switch_order) of the small-cache host that libzlref_macro.so
# reports (oracle/ref_sysconf_wrap.cpp), per precision
MACRO_HOST = {"f32": (10, 14), "f64": (9, 13)}

AOS, SOA = 0, 1
_c = ctypes
_sz = ctypes.c_size_t
_vp = ctypes.c_void_p

_port = None
_ref = {}


def _dtypes(prec):
    return (np.float32, np.complex64) if prec == "f32" else (np.float64, np.complex128)


def port_lib():
    """The C restatement (built by ``make -C oracle port``)."""
    global _port
    if _port is None:
        if not os.path.exists(PORT_SO):
            raise RuntimeError(f"oracle port not built: {PORT_SO} (run make -C oracle port)")
        lib = ctypes.CDLL(PORT_SO)
        for suf, f in (("f32", _c.c_float), ("f64", _c.c_double)):
            fp = _c.POINTER(f)
            getattr(lib, f"zlo_twiddles_{suf}").argtypes = [_sz, fp, fp]
            getattr(lib, f"zlo_rfft_twiddles_{suf}").argtypes = [_sz, fp, fp]
            getattr(lib, f"zlo_cfft_{suf}").argtypes = [_sz, _c.c_int, fp, fp, _sz, fp, fp, _sz]
            getattr(lib, f"zlo_cfft_batch_{suf}").argtypes = [
                _sz, _c.c_int, _c.c_int, fp, fp, _c.c_int, fp, fp, _sz, _c.c_int]
            getattr(lib, f"zlo_rfft_forward_{suf}").argtypes = [_sz, fp, _c.c_int, fp, fp, _sz]
            getattr(lib, f"zlo_rfft_backward_{suf}").argtypes = [_sz, fp, fp, _sz, fp]
            getattr(lib, f"zlo_set_hybrid_{suf}").argtypes = [_c.c_int, _c.c_int]
            getattr(lib, f"zlo_micro_order_{suf}").argtypes = [_sz]
            getattr(lib, f"zlo_micro_order_{suf}").restype = _c.c_int
        _port = lib
    return _port


def ref_available(macro: bool = False) -> bool:
    return os.path.exists(REF_MACRO_SO if macro else REF_SO)


def ref_lib(macro: bool = False):
    """The reference's own code compiled against the Highway-API shim; with
    macro, the build whose cache probe reports a small-cache host."""
    if macro not in _ref:
        path = REF_MACRO_SO if macro else REF_SO
        if not os.path.exists(path):
            raise RuntimeError(f"reference build absent: {path} (run make -C oracle ref)")
        lib = ctypes.CDLL(path)
        lib.zlref_plan_create.restype = _vp
        lib.zlref_plan_create.argtypes = [_c.c_int, _c.c_int, _sz, _sz]
        lib.zlref_plan_destroy.argtypes = [_c.c_int, _vp]
        lib.zlref_cfft_exec.argtypes = [_c.c_int, _vp, _c.c_int, _c.c_int, _vp, _vp, _c.c_int, _vp, _vp, _sz]
        lib.zlref_rfft_exec.argtypes = [_c.c_int, _vp, _c.c_int, _c.c_int, _vp, _vp, _vp, _vp, _sz]
        lib.zlref_switch_order.argtypes = [_c.c_int, _c.POINTER(_sz), _c.POINTER(_sz)]
        lib.zlref_cfft_roundtrip_repeat.argtypes = [_c.c_int, _vp, _vp, _vp, _vp, _sz]
        _ref[macro] = lib
    return _ref[macro]


def _ptr(a, f):
    return a.ctypes.data_as(ctypes.POINTER(f))


# ----------------------------------------------------------------- port (C)
class hybrid:
    """Context manager: the port follows the reference's algorithm switch with
    the given (max_l1_order, switch_order) (src/common/zldsp_fft_common_init.hpp:305-339):
    CFFTs of order >= switch_order, and RFFTs whose inner CFFT is that large,
    take the macro DIF path. Outside it the port is micro-only. Not thread-safe:
    the setting is process-wide for the precision."""

    def __init__(self, prec: str, max_l1_order: int, switch_order: int):
        self.prec, self.l1, self.sw = prec, max_l1_order, switch_order

    def __enter__(self):
        getattr(port_lib(), f"zlo_set_hybrid_{self.prec}")(self.l1, self.sw)
        return self

    def __exit__(self, *exc):
        getattr(port_lib(), f"zlo_set_hybrid_{self.prec}")(0, 1 << 30)
        return False


def macro_host(prec: str = "f32") -> hybrid:
    """hybrid() with the small-cache host that libzlref_macro.so reports."""
    return hybrid(prec, *MACRO_HOST[prec])


def micro_order(order: int, prec: str = "f32") -> int:
    """Micro order of the port's current switch for a CFFT of `order` (-1: micro-only)."""
    return getattr(port_lib(), f"zlo_micro_order_{prec}")(order)


def twiddles(order: int, prec: str = "f32") -> np.ndarray:
    """Unified twiddle table T[t] = exp(-2 pi i t / N), t < 3N/4, as the reference rounds it."""
    ft, ct = _dtypes(prec)
    f = _c.c_float if prec == "f32" else _c.c_double
    n = (3 * (1 << order)) // 4
    re = np.zeros(max(n, 1), ft)
    im = np.zeros(max(n, 1), ft)
    getattr(port_lib(), f"zlo_twiddles_{prec}")(order, _ptr(re, f), _ptr(im, f))
    return (re + 1j * im).astype(ct)[:n]


def rfft_twiddles(rfft_order: int, prec: str = "f32"):
    """(wc, ws) for k = 0..M/2 (index 0 unused), M = N/2."""
    ft, _ = _dtypes(prec)
    f = _c.c_float if prec == "f32" else _c.c_double
    m = (1 << rfft_order) // 2
    wc = np.zeros(m // 2 + 1, ft)
    ws = np.zeros(m // 2 + 1, ft)
    getattr(port_lib(), f"zlo_rfft_twiddles_{prec}")(rfft_order, _ptr(wc, f), _ptr(ws, f))
    return wc, ws


def cfft_port(x: np.ndarray, forward: bool = True) -> np.ndarray:
    """Batched complex FFT, x shape (batch, N) complex64/complex128 (AoS)."""
    x = np.ascontiguousarray(x)
    prec = "f32" if x.dtype == np.complex64 else "f64"
    ft, _ = _dtypes(prec)
    f = _c.c_float if prec == "f32" else _c.c_double
    if x.ndim == 1:
        return cfft_port(x[None, :], forward)[0]
    batch, n = x.shape
    order = n.bit_length() - 1
    assert 1 << order == n
    out = np.zeros_like(x)
    xf = x.view(ft)
    of = out.view(ft)
    getattr(port_lib(), f"zlo_cfft_batch_{prec}")(
        order, int(forward), AOS, _ptr(xf, f), _ptr(xf, f), AOS, _ptr(of, f), _ptr(of, f), batch,
        min(8, os.cpu_count() or 1))
    return out


def rfft_forward_port(x: np.ndarray, sqr_mag: bool = False) -> np.ndarray:
    """RFFT forward of real frames x (batch, N): complex bins (batch, N/2+1), or
    squared magnitudes (batch, N/2+1) when sqr_mag."""
    x = np.ascontiguousarray(x)
    prec = "f32" if x.dtype == np.float32 else "f64"
    ft, ct = _dtypes(prec)
    f = _c.c_float if prec == "f32" else _c.c_double
    if x.ndim == 1:
        return rfft_forward_port(x[None, :], sqr_mag)[0]
    batch, n = x.shape
    order = n.bit_length() - 1
    nb = n // 2 + 1
    fn = getattr(port_lib(), f"zlo_rfft_forward_{prec}")
    if sqr_mag:
        out = np.zeros((batch, nb), ft)
        for b in range(batch):
            ob = out[b]
            fn(order, _ptr(x[b], f), 1, _ptr(ob, f), _ptr(ob, f), 1)
        return out
    out = np.zeros((batch, nb), ct)
    for b in range(batch):
        ob = out[b].view(ft)
        fn(order, _ptr(x[b], f), 0, _ptr(ob, f), _ptr(ob[1:], f), 2)
    return out


def rfft_backward_port(X: np.ndarray) -> np.ndarray:
    """RFFT backward of bins X (batch, N/2+1) complex -> (batch, N) real, unnormalised."""
    X = np.ascontiguousarray(X)
    prec = "f32" if X.dtype == np.complex64 else "f64"
    ft, _ = _dtypes(prec)
    f = _c.c_float if prec == "f32" else _c.c_double
    if X.ndim == 1:
        return rfft_backward_port(X[None, :])[0]
    batch, nb = X.shape
    n = 2 * (nb - 1)
    order = n.bit_length() - 1
    out = np.zeros((batch, n), ft)
    fn = getattr(port_lib(), f"zlo_rfft_backward_{prec}")
    for b in range(batch):
        xb = X[b].view(ft)
        fn(order, _ptr(xb, f), _ptr(xb[1:], f), 2, _ptr(out[b], f))
    return out


def istft_port(X: np.ndarray, hop: int, filt=None, win=None) -> np.ndarray:
    """Inverse STFT with overlap-add, sequentially: bins X (frames, N/2+1) ->
    signal of (frames - 1) * hop + N reals, y[f*hop + n] += win[n] * x_f[n] for
    f = 0, 1, ... in order, x_f = RFFT backward (the port) of filt * X_f. Every
    product and sum is one operation in the bins' precision (numpy array
    arithmetic, so no fused multiply-adds)."""
    X = np.ascontiguousarray(X)
    ft = np.float32 if X.dtype == np.complex64 else np.float64
    if filt is not None:
        xr, xi = X.real.astype(ft), X.imag.astype(ft)
        hr, hi = filt.real.astype(ft), filt.imag.astype(ft)
        Y = np.empty_like(X)
        Y.real = xr * hr - xi * hi
        Y.imag = xr * hi + xi * hr
        X = Y
    x = rfft_backward_port(X)
    frames, n = x.shape
    if win is not None:
        x = x * np.asarray(win, ft)[None, :]
    y = np.zeros((frames - 1) * hop + n, ft)
    for f in range(frames):
        y[f * hop:f * hop + n] += x[f]
    return y


def istft_fp64(X: np.ndarray, hop: int, filt=None, win=None) -> np.ndarray:
    """The same overlap-add in float64 from numpy.fft (RFFT backward = (N/2) irfft)."""
    X = np.asarray(X, np.complex128)
    if filt is not None:
        X = X * np.asarray(filt, np.complex128)[None, :]
    x = rfft_backward_fp64(X)
    frames, n = x.shape
    if win is not None:
        x = x * np.asarray(win, np.float64)[None, :]
    y = np.zeros((frames - 1) * hop + n)
    for f in range(frames):
        y[f * hop:f * hop + n] += x[f]
    return y


# ----------------------------------------------------------------- reference (shim-built)
class RefPlan:
    """One reference CFFT/RFFT instance per thread (the reference is single-threaded)."""

    def __init__(self, kind: str, order: int, prec: str = "f32", threads: int = 1, macro: bool = False):
        self.lib = ref_lib(macro)
        self.prec = 0 if prec == "f32" else 1
        self.kind = kind
        self.order = order
        self.handle = self.lib.zlref_plan_create(self.prec, 0 if kind == "c2c" else 1, order, threads)

    def close(self):
        if self.handle:
            self.lib.zlref_plan_destroy(self.prec, self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def cfft_roundtrip_repeat(self, x, reps):
        """forward then backward of the single AoS transform x, reps times on
        one thread; returns the backward output of the last repetition."""
        x = np.ascontiguousarray(x)
        mid, out = np.empty_like(x), np.empty_like(x)
        self.lib.zlref_cfft_roundtrip_repeat(self.prec, self.handle, x.ctypes.data, mid.ctypes.data,
                                             out.ctypes.data, int(reps))
        return out

    def cfft(self, x, forward=True, in_layout=AOS, out_layout=AOS, out=None):
        """x: (batch, N) complex (AoS) or a pair (re, im) of (batch, N) real arrays (SoA)."""
        if in_layout == AOS:
            batch = x.shape[0]
            a0, a1 = x.ctypes.data, None
            ct = x.dtype
        else:
            batch = x[0].shape[0]
            a0, a1 = x[0].ctypes.data, x[1].ctypes.data
            ct = np.complex64 if x[0].dtype == np.float32 else np.complex128
        n = 1 << self.order
        if out is None:
            if out_layout == AOS:
                out = np.zeros((batch, n), ct)
            else:
                ft = np.float32 if ct == np.complex64 else np.float64
                out = (np.zeros((batch, n), ft), np.zeros((batch, n), ft))
        if out_layout == AOS:
            o0, o1 = out.ctypes.data, None
        else:
            o0, o1 = out[0].ctypes.data, out[1].ctypes.data
        self.lib.zlref_cfft_exec(self.prec, self.handle, int(forward), in_layout, a0, a1, out_layout, o0, o1, batch)
        return out

    def rfft_forward(self, x, layout=AOS, sqr_mag=False, out=None):
        batch, n = x.shape
        nb = n // 2 + 1
        ft = x.dtype
        ct = np.complex64 if ft == np.float32 else np.complex128
        if sqr_mag:
            out = np.zeros((batch, nb), ft) if out is None else out
            self.lib.zlref_rfft_exec(self.prec, self.handle, 1, AOS, x.ctypes.data, None, out.ctypes.data, None, batch)
            return out
        if layout == AOS:
            out = np.zeros((batch, nb), ct) if out is None else out
            self.lib.zlref_rfft_exec(self.prec, self.handle, 0, AOS, x.ctypes.data, None, out.ctypes.data, None, batch)
        else:
            out = (np.zeros((batch, nb), ft), np.zeros((batch, nb), ft)) if out is None else out
            self.lib.zlref_rfft_exec(self.prec, self.handle, 0, SOA, x.ctypes.data, None, out[0].ctypes.data,
                                     out[1].ctypes.data, batch)
        return out

    def rfft_backward(self, X, layout=AOS, out=None):
        if layout == AOS:
            batch, nb = X.shape
            a0, a1 = X.ctypes.data, None
            ft = np.float32 if X.dtype == np.complex64 else np.float64
        else:
            batch, nb = X[0].shape
            a0, a1 = X[0].ctypes.data, X[1].ctypes.data
            ft = X[0].dtype
        n = 2 * (nb - 1)
        out = np.zeros((batch, n), ft) if out is None else out
        self.lib.zlref_rfft_exec(self.prec, self.handle, 2, layout, a0, a1, out.ctypes.data, None, batch)
        return out


def ref_switch_order(prec: str = "f32", macro: bool = False):
    """(max_l1_order, switch_order) the reference derives from this host's caches
    (with macro: from the small-cache host of libzlref_macro.so)."""
    a, b = _sz(), _sz()
    ref_lib(macro).zlref_switch_order(0 if prec == "f32" else 1, ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


# ----------------------------------------------------------------- FP64 (numpy)
def cfft_fp64(x: np.ndarray, forward: bool = True) -> np.ndarray:
    x = np.asarray(x, np.complex128)
    n = x.shape[-1]
    return np.fft.fft(x, axis=-1) if forward else np.fft.ifft(x, axis=-1) * n


def rfft_fp64(x: np.ndarray) -> np.ndarray:
    return np.fft.rfft(np.asarray(x, np.float64), axis=-1)


def rfft_backward_fp64(X: np.ndarray) -> np.ndarray:
    X = np.asarray(X, np.complex128)
    n = 2 * (X.shape[-1] - 1)
    return np.fft.irfft(X, n=n, axis=-1) * (n / 2)


def rel_l2(y, ref) -> np.ndarray:
    """Per-transform relative L2 error along the last axis."""
    y = np.asarray(y, np.complex128)
    ref = np.asarray(ref, np.complex128)
    num = np.linalg.norm(y - ref, axis=-1)
    den = np.linalg.norm(ref, axis=-1)
    return num / np.where(den == 0, 1.0, den)


def tolerance(order: int, prec: str = "f32") -> float:
    """Relative-L2 bound 4 * log2(N) * eps (eps = 2^-24 for f32, 2^-53 for f64)."""
    eps = 2.0 ** -24 if prec == "f32" else 2.0 ** -53
    return 4.0 * max(order, 1) * eps
