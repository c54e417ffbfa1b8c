"""Python front end of libmpzmm_b200 over packed vectors.

Mirrors the reference's operator interface (alexp616/rforest
src/include/hwmpz.h): ``setup()`` ~ hw_mpz_setup, ``matmul`` ~
mpz_rmatrix_mult_fft for general m x k by k x n shapes, plus batches and
device-resident plans.  Every call goes through the C ABI; there is no
Python or CPU implementation of the product behind it.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from .packed import Packed, from_ints

ProductIn = Tuple[int, int, int, Packed, Packed]


def _ptr(a: np.ndarray, t):
    return a.ctypes.data_as(t)


def _stream_arg(stream) -> Optional[int]:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return int(getattr(stream, "cuda_stream"))  # torch.cuda.Stream


def setup(device: int = 0) -> None:
    _lib.check(_lib.lib().mpzmm_setup(device))


def set_contract_mode(mode: int) -> None:
    """0 automatic, 1 CUDA cores only, 2 tensor cores wherever the shape allows."""
    _lib.check(_lib.lib().mpzmm_set_option(_lib.MPZMM_OPT_CONTRACT, mode))


def autotune(stream=None):
    """Measure CUDA-core vs tensor-core contraction per size class; automatic
    mode then uses the faster one.  Returns {(k, m=n): (cuda_ms, tc_ms)}."""
    ms = (C.c_float * 40)()
    _lib.check(_lib.lib().mpzmm_autotune(_stream_arg(stream), ms))
    out = {}
    for bk, k in enumerate((8, 16, 32, 64)):
        for bm, mn in enumerate((4, 8, 16, 32, 64)):
            i = bk * 5 + bm
            out[(k, mn)] = (ms[2 * i], ms[2 * i + 1])
    return out


def set_chunk_limbs(limbs: int) -> None:
    """Input limbs per chunk of a pipelined one-shot batch (0 = automatic)."""
    _lib.check(_lib.lib().mpzmm_set_option(_lib.MPZMM_OPT_CHUNK_LIMBS, int(limbs)))


def chunk_limbs() -> int:
    return int(_lib.lib().mpzmm_get_option(_lib.MPZMM_OPT_CHUNK_LIMBS))


def batch_stats():
    """Last one-shot batch: host time in ms (plan, input copies, launch
    queueing, wait + results), chunk count, and bytes copied each way (with
    the parts that moved straight from / to pinned caller memory)."""
    ns = (C.c_int64 * 4)()
    nb = (C.c_int64 * 4)()
    chunks = C.c_int64()
    _lib.check(_lib.lib().mpzmm_batch_stats(ns, C.byref(chunks), nb))
    return {"plan_ms": ns[0] / 1e6, "inputs_ms": ns[1] / 1e6, "launch_ms": ns[2] / 1e6,
            "finish_ms": ns[3] / 1e6, "chunks": chunks.value,
            "h2d_bytes": nb[0], "d2h_bytes": nb[1],
            "h2d_direct_bytes": nb[2], "d2h_direct_bytes": nb[3]}


TIMELINE_FIELDS = ("plan_begin", "plan_end", "queue_begin", "queue_end", "h2d_begin",
                   "h2d_end", "kernels_end", "d2h_end", "h2d_bytes", "d2h_bytes")


def batch_timeline():
    """Last one-shot batch, one dict per chunk: host planning and queueing
    times and device copy / kernel event times in ms from the batch's start,
    and the bytes copied each way (mpzmm_batch_timeline)."""
    n = C.c_int()
    _lib.check(_lib.lib().mpzmm_batch_timeline(None, 0, C.byref(n)))
    rows = (C.c_double * (len(TIMELINE_FIELDS) * max(1, n.value)))()
    _lib.check(_lib.lib().mpzmm_batch_timeline(rows, n.value, C.byref(n)))
    F = len(TIMELINE_FIELDS)
    return [dict(zip(TIMELINE_FIELDS, rows[c * F:(c + 1) * F])) for c in range(n.value)]


def batch_chunks(limbs: Sequence[int], chunk_limbs: int = 0) -> List[int]:
    """Product-index bounds of the chunks mpzmm_matmul_batch would use for
    products with these input limb counts (chunk_limbs 0: automatic); the
    last bound is the product count."""
    arr = np.ascontiguousarray(np.asarray(limbs, dtype=np.int64).reshape(-1))
    n = C.c_int()
    bounds = np.zeros(arr.size + 2, dtype=np.int64)
    _lib.check(_lib.lib().mpzmm_batch_chunks(
        int(arr.size), arr.ctypes.data_as(C.POINTER(C.c_int64)), int(chunk_limbs),
        bounds.ctypes.data_as(C.POINTER(C.c_int64)), int(bounds.size), C.byref(n)))
    return [int(b) for b in bounds[:n.value + 1]]


class HostArena:
    """Pinned host memory from the library (mpzmm_host_alloc).  Transfers
    whose host side lies inside it go straight to and from the device."""

    def __init__(self, nbytes: int):
        self.nbytes = max(int(nbytes), 8)
        p = C.c_void_p()
        _lib.check(_lib.lib().mpzmm_host_alloc(self.nbytes, C.byref(p)))
        self.ptr = p.value
        self.used = 0

    def take(self, count: int, dtype) -> np.ndarray:
        """Next ``count`` elements of ``dtype`` (8-byte aligned) as a numpy view."""
        dt = np.dtype(dtype)
        off = (self.used + 7) & ~7
        nb = max(int(count), 1) * dt.itemsize
        if off + nb > self.nbytes:
            raise MemoryError("host arena exhausted")
        self.used = off + nb
        buf = (C.c_char * nb).from_address(self.ptr + off)
        return np.frombuffer(buf, dtype=dt, count=max(int(count), 1))

    def close(self) -> None:
        if self.ptr:
            _lib.check(_lib.lib().mpzmm_host_free(C.c_void_p(self.ptr)))
            self.ptr = None


def contract_mode() -> int:
    return int(_lib.lib().mpzmm_get_option(_lib.MPZMM_OPT_CONTRACT))


def device_available() -> bool:
    return bool(_lib.lib().mpzmm_device_available())


def choose_params(a_bits: int, b_bits: int, k: int) -> Tuple[int, int, int]:
    P, r, lg = C.c_int(), C.c_int(), C.c_int()
    _lib.check(_lib.lib().mpzmm_choose_params(a_bits, b_bits, k, C.byref(P), C.byref(r),
                                              C.byref(lg)))
    return P.value, r.value, lg.value


def output_limbs(k: int, a_bits: int, b_bits: int) -> int:
    return int(_lib.lib().mpzmm_output_limbs(k, a_bits, b_bits))


class _Holder:
    """Keeps the numpy arrays behind one mpzmm_product alive."""

    def __init__(self, m: int, k: int, n: int, A: Packed, B: Packed, bufs=None):
        """``bufs``: optional (a_limbs, b_limbs, c_limbs) arrays to use (for
        example views into a pinned arena); the inputs are copied into them."""
        if len(A) != m * k or len(B) != k * n:
            raise ValueError("entry counts do not match the dimensions")
        self.m, self.k, self.n = m, k, n
        if bufs is not None:
            self.al, self.bl = bufs[0], bufs[1]
            np.copyto(self.al[:A.limbs.size], A.limbs)
            np.copyto(self.bl[:B.limbs.size], B.limbs)
        else:
            self.al = np.ascontiguousarray(A.limbs, dtype=np.uint64)
            self.bl = np.ascontiguousarray(B.limbs, dtype=np.uint64)
        if self.al.size == 0:
            self.al = np.zeros(1, np.uint64)
        if self.bl.size == 0:
            self.bl = np.zeros(1, np.uint64)
        self.ao = np.ascontiguousarray(A.offs, dtype=np.int64)
        self.bo = np.ascontiguousarray(B.offs, dtype=np.int64)
        self.asz = np.ascontiguousarray(A.sizes, dtype=np.int32)
        self.bsz = np.ascontiguousarray(B.sizes, dtype=np.int32)
        cap = self.out_cap(k, A, B)
        self.caps = np.full(m * n, cap, dtype=np.int64)
        self.co = np.arange(m * n, dtype=np.int64) * cap
        if bufs is not None:
            self.cl = bufs[2]
        else:
            self.cl = np.zeros(max(m * n * cap, 1), dtype=np.uint64)
        self.csz = np.zeros(m * n, dtype=np.int32)
        self.struct = _lib.Product(
            m, k, n,
            _ptr(self.al, _lib.u64p), _ptr(self.ao, _lib.i64p), _ptr(self.asz, _lib.i32p),
            _ptr(self.bl, _lib.u64p), _ptr(self.bo, _lib.i64p), _ptr(self.bsz, _lib.i32p),
            _ptr(self.cl, _lib.u64p), _ptr(self.co, _lib.i64p), _ptr(self.caps, _lib.i64p),
            _ptr(self.csz, _lib.i32p))

    @staticmethod
    def out_cap(k: int, A: Packed, B: Packed) -> int:
        """The library's own bound for the product (exact operand bit
        lengths), so results fill the output array back to back."""
        return output_limbs(k, A.max_bits(), B.max_bits())

    def result(self) -> Packed:
        return Packed(self.cl, self.co, self.csz)

    def set_inputs(self, A: Packed, B: Packed) -> None:
        """Overwrite the input limbs in place (same sizes and signs)."""
        np.copyto(self.al[:A.limbs.size], A.limbs)
        np.copyto(self.bl[:B.limbs.size], B.limbs)


def matmul(m: int, k: int, n: int, A: Packed, B: Packed, stream=None) -> Packed:
    """Exact C = A * B (A m x k, B k x n, row-major packed vectors)."""
    return matmul_holder(_Holder(m, k, n, A, B), stream)


def holder(m: int, k: int, n: int, A: Packed, B: Packed) -> "_Holder":
    """The arrays of one product laid out for the C ABI (inputs, result
    arrays sized by the library's bound), reusable for repeated calls."""
    return _Holder(m, k, n, A, B)


def matmul_holder(h: "_Holder", stream=None) -> Packed:
    """mpzmm_matmul on a holder's arrays; the result is a view of them."""
    _lib.check(_lib.lib().mpzmm_matmul_batch(1, C.byref(h.struct), _stream_arg(stream)))
    return h.result()


class Batch:
    """Host-side arrays of a batch of products, reusable across calls.  Each
    ``run`` is one full pass through the C ABI (mpzmm_matmul_batch): plan,
    host->device copy of the inputs, all kernels, device->host copy of the
    results into the host output arrays."""

    def __init__(self, products: Sequence[ProductIn], pinned: bool = False):
        """With ``pinned`` the inputs are copied (once, here) into one pinned
        arena from the library and the outputs live there too, so every
        ``run`` moves them straight between that memory and the device.  The
        results of a pinned batch are views into the arena: valid until
        ``close``."""
        self.arena = None
        bufs = [None] * len(products)
        if pinned:
            caps = [_Holder.out_cap(p[1], p[3], p[4]) for p in products]
            nbytes = 64
            for (m, k, n, A, B), cap in zip(products, caps):
                nbytes += 8 * (max(A.limbs.size, 1) + max(B.limbs.size, 1)
                               + max(m * n * cap, 1)) + 24
            self.arena = HostArena(nbytes)
            # all inputs back to back (one copy run for the batch), then all
            # outputs
            ins = [(self.arena.take(A.limbs.size, np.uint64),
                    self.arena.take(B.limbs.size, np.uint64)) for (m, k, n, A, B) in products]
            outs = [self.arena.take(max(p[0] * p[2] * cap, 1), np.uint64)
                    for p, cap in zip(products, caps)]
            bufs = [(a, b, c) for (a, b), c in zip(ins, outs)]
        self.holders = [_Holder(*p, bufs=bb) for p, bb in zip(products, bufs)]
        self.arr = (_lib.Product * len(self.holders))(*[h.struct for h in self.holders])
        # the results are views of the output arrays: made once, valid after every run
        self.results = [h.result() for h in self.holders]

    def run(self, stream=None) -> List[Packed]:
        _lib.check(_lib.lib().mpzmm_matmul_batch(len(self.holders), self.arr,
                                                 _stream_arg(stream)))
        return self.results

    def close(self) -> None:
        self.holders = []
        self.results = []
        self.arr = None
        if self.arena is not None:
            self.arena.close()
            self.arena = None


def matmul_batch(products: Sequence[ProductIn], stream=None) -> List[Packed]:
    """Many independent products in one pass (one launch per stage)."""
    return Batch(products).run(stream)


def chain(mats: Sequence[Tuple[int, int, Packed]], stream=None) -> Packed:
    """M = X_0 X_1 ... X_{n-1} (each (rows, cols, packed row-major entries)),
    the running product kept in device memory between the steps."""
    keep = []
    arr = (_lib.Matrix * len(mats))()
    for i, (rows, cols, X) in enumerate(mats):
        if len(X) != rows * cols:
            raise ValueError("entry count does not match the dimensions")
        limbs = np.ascontiguousarray(X.limbs, dtype=np.uint64)
        if limbs.size == 0:
            limbs = np.zeros(1, np.uint64)
        offs = np.ascontiguousarray(X.offs, dtype=np.int64)
        sizes = np.ascontiguousarray(X.sizes, dtype=np.int32)
        keep += [limbs, offs, sizes]
        arr[i] = _lib.Matrix(rows, cols, _ptr(limbs, _lib.u64p), _ptr(offs, _lib.i64p),
                             _ptr(sizes, _lib.i32p))
    cap = int(_lib.lib().mpzmm_chain_output_limbs(len(mats), arr))
    if cap < 0:
        _lib.check(_lib.MPZMM_ERR_ARG)
    m, n = mats[0][0], mats[-1][1]
    cl = np.zeros(max(m * n * cap, 1), dtype=np.uint64)
    co = np.arange(m * n, dtype=np.int64) * cap
    caps = np.full(m * n, cap, dtype=np.int64)
    csz = np.zeros(m * n, dtype=np.int32)
    _lib.check(_lib.lib().mpzmm_chain(len(mats), arr, _ptr(cl, _lib.u64p), _ptr(co, _lib.i64p),
                                      _ptr(caps, _lib.i64p), _ptr(csz, _lib.i32p),
                                      _stream_arg(stream)))
    return Packed(cl, co, csz)


class Mod:
    """Reduction by a fixed modulus d > 0 (a Python int): ``reduce(X)`` gives
    x mod d in [0, d) for every entry of the packed vector X, for entries of
    up to ``max_bits`` bits.  Mirrors mpzfft_mod_init / mpzfft_mod_mod."""

    def __init__(self, d: int, max_bits: int):
        if d <= 0:
            raise ValueError("the modulus must be positive")
        self._d = from_ints([d])
        self._dl = np.ascontiguousarray(self._d.limbs, dtype=np.uint64)
        self.handle = C.c_void_p()
        _lib.check(_lib.lib().mpzmm_mod_create(C.byref(self.handle), _ptr(self._dl, _lib.u64p),
                                               int(self._d.sizes[0]), (int(max_bits) + 63) // 64))
        self.n = int(_lib.lib().mpzmm_mod_limbs(self.handle))

    def reduce(self, X: Packed, stream=None) -> Packed:
        count = len(X)
        xl = np.ascontiguousarray(X.limbs, dtype=np.uint64)
        if xl.size == 0:
            xl = np.zeros(1, np.uint64)
        xo = np.ascontiguousarray(X.offs, dtype=np.int64)
        xs = np.ascontiguousarray(X.sizes, dtype=np.int32)
        rl = np.zeros(max(count * self.n, 1), dtype=np.uint64)
        ro = np.arange(count, dtype=np.int64) * self.n
        rc = np.full(count, self.n, dtype=np.int64)
        rs = np.zeros(count, dtype=np.int32)
        _lib.check(_lib.lib().mpzmm_mod_batch(self.handle, count, _ptr(xl, _lib.u64p),
                                              _ptr(xo, _lib.i64p), _ptr(xs, _lib.i32p),
                                              _ptr(rl, _lib.u64p), _ptr(ro, _lib.i64p),
                                              _ptr(rc, _lib.i64p), _ptr(rs, _lib.i32p),
                                              _stream_arg(stream)))
        return Packed(rl, ro, rs)

    def close(self) -> None:
        if self.handle:
            _lib.lib().mpzmm_mod_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Plan:
    """A device-resident batch: inputs uploaded once, executed many times."""

    def __init__(self, products: Sequence[ProductIn], stream=None, fixed_b: bool = False):
        """fixed_b: keep B's transforms across executes (mpzmm_plan_create_fixed_b);
        set new A values with set_a() and upload_a()."""
        self.holders = [_Holder(*p) for p in products]
        self.arr = (_lib.Product * len(self.holders))(*[h.struct for h in self.holders])
        self.handle = C.c_void_p()
        create = (_lib.lib().mpzmm_plan_create_fixed_b if fixed_b
                  else _lib.lib().mpzmm_plan_create)
        _lib.check(create(C.byref(self.handle), len(self.holders), self.arr,
                          _stream_arg(stream)))

    def set_a(self, index: int, A: Packed) -> None:
        """New A values for product `index` with the same signed limb counts
        (the plan's descriptors hold sizes and signs), read by the next
        upload() or upload_a()."""
        h = self.holders[index]
        if not np.array_equal(np.asarray(A.sizes, dtype=np.int32), h.asz):
            raise ValueError("new A must have the same signed limb counts")
        np.copyto(h.al[:A.limbs.size], A.limbs)

    def upload_a(self, stream=None) -> None:
        _lib.check(_lib.lib().mpzmm_plan_upload_a(self.handle, _stream_arg(stream)))

    def execute(self, stream=None) -> None:
        _lib.check(_lib.lib().mpzmm_plan_execute(self.handle, _stream_arg(stream)))

    def upload(self, stream=None) -> None:
        _lib.check(_lib.lib().mpzmm_plan_upload(self.handle, _stream_arg(stream)))

    def download(self, stream=None) -> List[Packed]:
        _lib.check(_lib.lib().mpzmm_plan_download(self.handle, _stream_arg(stream)))
        return [h.result() for h in self.holders]

    def info(self, index: int = 0):
        launches, nbytes = C.c_int64(), C.c_int64()
        P, r, lg = C.c_int(), C.c_int(), C.c_int()
        _lib.check(_lib.lib().mpzmm_plan_info(self.handle, C.byref(launches), C.byref(nbytes),
                                              index, C.byref(P), C.byref(r), C.byref(lg)))
        return {"launches": launches.value, "device_bytes": nbytes.value,
                "P": P.value, "r": r.value, "lgN": lg.value}

    def set_graph(self, on: bool) -> None:
        """Capture the plan's launches into a CUDA graph on the next execute."""
        _lib.check(_lib.lib().mpzmm_plan_set_graph(self.handle, 1 if on else 0))

    def set_timing(self, on: bool) -> None:
        _lib.check(_lib.lib().mpzmm_plan_set_timing(self.handle, 1 if on else 0))

    def stage_times(self):
        """(ms per stage summed over timed executes, launches per stage per
        execute, timed executes); stages: fwd, contract, inv, crt."""
        ms = (C.c_float * 4)()
        launches = (C.c_int64 * 4)()
        ex = C.c_int64()
        _lib.check(_lib.lib().mpzmm_plan_stage_times(
            self.handle, ms, C.cast(launches, _lib.i64p), C.byref(ex)))
        return list(ms), list(launches), ex.value

    def close(self) -> None:
        if self.handle:
            _lib.lib().mpzmm_plan_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request server (mpzmm_server_* of the C ABI)."""

    def __init__(self, budget_bytes: int = 0, slots: int = 3, max_batch: int = 0,
                 window_us: Optional[int] = None):
        self.handle = C.c_void_p()
        _lib.check(_lib.lib().mpzmm_server_create(C.byref(self.handle), budget_bytes, slots,
                                                  max_batch))
        self.holders = {}
        if window_us is not None:
            self.set_admission_window(window_us)

    def set_admission_window(self, microseconds: int) -> None:
        _lib.check(_lib.lib().mpzmm_server_set_admission_window(self.handle, int(microseconds)))

    def submit(self, m: int, k: int, n: int, A: Packed, B: Packed) -> int:
        return self.submit_holder(_Holder(m, k, n, A, B))

    def submit_holder(self, h: "_Holder") -> int:
        """Queues a request whose arrays are already laid out (a holder made
        once and reused once its previous request has completed)."""
        t = C.c_uint64()
        _lib.check(_lib.lib().mpzmm_server_submit(self.handle, C.byref(h.struct), C.byref(t)))
        self.holders[t.value] = h
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> Packed:
        _lib.check(_lib.lib().mpzmm_server_wait(self.handle, ticket, timeout_ms))
        return self.holders[ticket].result()

    def done(self, ticket: int) -> bool:
        d = C.c_int()
        _lib.check(_lib.lib().mpzmm_server_poll(self.handle, ticket, C.byref(d)))
        return bool(d.value)

    def times(self, ticket: int):
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        _lib.check(_lib.lib().mpzmm_server_ticket_times(self.handle, ticket, C.byref(a),
                                                        C.byref(b), C.byref(c)))
        return a.value, b.value, c.value

    def release(self, ticket: int) -> None:
        _lib.check(_lib.lib().mpzmm_server_release(self.handle, ticket))
        self.holders.pop(ticket, None)

    def stats(self):
        b, p, f = C.c_int64(), C.c_int64(), C.c_int64()
        _lib.check(_lib.lib().mpzmm_server_stats(self.handle, C.byref(b), C.byref(p), C.byref(f)))
        return {"batches": b.value, "products": p.value, "max_in_flight": f.value}

    def phase_ms(self):
        ns = (C.c_int64 * 4)()
        _lib.check(_lib.lib().mpzmm_server_phase_ns(self.handle, C.cast(ns, _lib.i64p)))
        return dict(zip(("build", "upload", "launch", "download"), [x / 1e6 for x in ns]))

    def phase_max_ms(self):
        """The longest single batch in each phase since the previous call."""
        ns = (C.c_int64 * 4)()
        _lib.check(_lib.lib().mpzmm_server_phase_max_ns(self.handle, C.cast(ns, _lib.i64p)))
        return dict(zip(("build", "upload", "launch", "download"), [x / 1e6 for x in ns]))

    def close(self) -> None:
        if self.handle:
            _lib.lib().mpzmm_server_destroy(self.handle)
            self.handle = C.c_void_p()
            self.holders.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
