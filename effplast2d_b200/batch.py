"""Batched solving and the continuous-batching server (ep2d_batch_solve, ep2d_server_*).

A request is one RVE: the inputs of one run of the reference binary (grid, pa.dat
values, NL, initial load and load type, time steps).  Results are ep2d_result dicts
with the numerical and analytic moduli.
"""
import ctypes

from . import _abi
from .solver import _check, lib


def spec(n, pa, nl, n_time_steps, init_load_value, load_type, ny=None):
    return _abi.make_spec(n, ny or n, pa, nl, n_time_steps, init_load_value, load_type)


def footprint(s, precision=_abi.FP64):
    """device bytes an RVE holds while it is solved"""
    return int(lib().ep2d_rve_footprint(ctypes.byref(s), int(precision)))


def batch_solve(specs, niter=100000, eiter=1e-9, check_every=10000, precision=_abi.FP64, device=0, rows=0,
                graph_len=0, kernel=_abi.KERNEL_AUTO):
    """Solve every spec together; returns (list of result dicts, stats dict).  rows = 0
    lets the library time the kernel forms and rows on the first launches."""
    cfg = _abi.make_batch_config(niter, eiter, check_every, precision, device, rows, graph_len, kernel)
    n = len(specs)
    arr = (_abi.RveSpec * n)(*specs)
    res = (_abi.Result * n)()
    st = _abi.BatchStats()
    _check(lib().ep2d_batch_solve(ctypes.byref(cfg), arr, n, res, ctypes.byref(st)))
    return [r.as_dict() for r in res], st.as_dict()


class Server:
    """Continuous batching: submit() returns a ticket at once; the worker admits
    requests at checkpoint boundaries while device memory and the active-RVE cap allow,
    keeps each RVE resident until it converges, and wait() returns its result with the
    latency measured from submission."""

    def __init__(self, mem_budget_bytes, max_active=0, niter=100000, eiter=1e-9, check_every=10000,
                 precision=_abi.FP64, device=0, rows=0, graph_len=0, kernel=_abi.KERNEL_AUTO):
        self.cfg = _abi.make_batch_config(niter, eiter, check_every, precision, device, rows, graph_len, kernel)
        h = ctypes.c_void_p()
        _check(lib().ep2d_server_create(ctypes.byref(self.cfg), int(mem_budget_bytes), int(max_active),
                                        ctypes.byref(h)))
        self._h = h

    def submit(self, s):
        t = ctypes.c_uint64()
        _check(lib().ep2d_server_submit(self._h, ctypes.byref(s), ctypes.byref(t)))
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        """(result dict, latency_s, queue_s) or None if not finished within timeout_ms"""
        done = ctypes.c_int32()
        res = _abi.Result()
        lat = ctypes.c_double()
        q = ctypes.c_double()
        _check(lib().ep2d_server_wait(self._h, ctypes.c_uint64(ticket), int(timeout_ms), ctypes.byref(done),
                                      ctypes.byref(res), ctypes.byref(lat), ctypes.byref(q)))
        if not done.value:
            return None
        return res.as_dict(), lat.value, q.value

    def stats(self):
        sub, adm, fin, byt = (ctypes.c_int64() for _ in range(4))
        st = _abi.BatchStats()
        _check(lib().ep2d_server_stats(self._h, ctypes.byref(sub), ctypes.byref(adm), ctypes.byref(fin),
                                       ctypes.byref(byt), ctypes.byref(st)))
        return {"submitted": sub.value, "admitted": adm.value, "finished": fin.value, "bytes_in_use": byt.value,
                "engine": st.as_dict()}

    def close(self):
        if getattr(self, "_h", None):
            lib().ep2d_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
