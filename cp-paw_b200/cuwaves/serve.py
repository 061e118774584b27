"""Binding of the serving runtime (cuwaves_server_* in include/cuwaves.h).

`Server` queues complete wave-function sets (the inputs dictionary that
`systems.build_inputs` makes) as requests for a single point (nsteps = 0) or
a number of CP steps, admits them by an HBM budget and runs the admitted sets
concurrently on the GPU.  The reference has no counterpart: it runs one system
per program (PAW_DRIVER's time loop, src/paw_driver.f90:280-561).
"""
from __future__ import annotations

import ctypes as C
import time
from typing import Optional

import numpy as np

from .capi import CUW_PREC_FP64, Dims, WavesError, _D, _I, load_library


class Request(C.Structure):
    _fields_ = [
        ("dims", Dims),
        ("igvec", _I), ("minusg", _I), ("gbas", _D), ("gvec", _D), ("g2", _D), ("pro", _D), ("ylm", _D),
        ("mpsi", _D), ("gweight", C.c_double), ("v", _D), ("lmnxx", C.c_int), ("dh", _D), ("lnxx", C.c_int),
        ("dover", _D), ("r0", _D), ("occ", _D), ("psi", _D), ("delt", C.c_double), ("annee", C.c_double),
        ("nsteps", C.c_int), ("mass", _D), ("flags", C.c_int),
    ]


CUW_REQ_BORROW = 1


STATS = ("completed", "failed", "p50_ms", "p99_ms", "throughput_per_s", "peak_bytes", "bytes_in_use",
         "in_system", "mean_admitted", "max_ms")

_fns = None


def _bind():
    global _fns
    if _fns is None:
        lib = load_library()
        P, LL = C.c_void_p, C.c_longlong
        sig = {
            "create": [C.c_size_t, C.c_int, C.POINTER(P)],
            "set_max_active": [P, C.c_int],
            "submit": [P, C.POINTER(Request), C.POINTER(LL)],
            "poll": [P, LL, _I, _I, _D, _D, _D],
            "error": [P, LL, C.c_char_p, C.c_int],
            "release": [P, LL],
            "wait_all": [P],
            "stats": [P, _D, C.c_int],
            "destroy": [P],
        }
        fns = {}
        for name, args in sig.items():
            f = getattr(lib, "cuwaves_server_" + name)
            f.argtypes = args
            f.restype = C.c_int
            fns[name] = f
        _fns = fns
    return _fns


def _ptr(a, t):
    return a.ctypes.data_as(t)


class Server:
    """Continuous-batching request loop over wave-function sets on one GPU."""

    def __init__(self, hbm_budget: int, workers: int = 4, max_active: Optional[int] = None):
        self._f = _bind()
        h = C.c_void_p()
        rc = self._f["create"](C.c_size_t(int(hbm_budget)), int(workers), C.byref(h))
        if rc:
            raise WavesError(rc, "server_create", "invalid budget or worker count")
        self.h = h
        if max_active is not None:
            self._f["set_max_active"](h, int(max_active))
        self._keep = {}
        self._nat = {}

    def submit(self, inputs: dict, nsteps: int = 0, move_atoms: bool = False,
               precision: int = CUW_PREC_FP64, psi: Optional[np.ndarray] = None, borrow: bool = False) -> int:
        """Queues one set; with borrow the server reads the arrays in place and
        this object keeps them alive until the request is released."""
        i = inputs
        d = Dims()
        d.ngl, d.ndim, d.nb, d.nbh, d.tinv = i["ngl"], 1, i["nb"], i["nbh"], 1
        d.nr1, d.nr2, d.nr3 = i["grid"]
        d.nat, d.nsp, d.lmx, d.precision = i["nat"], i["nsp"], i["lmx"], precision
        for s in range(i["nsp"]):
            d.lnx[s] = i["lnx"][s]
            for ln, l in enumerate(i["lox"][s]):
                d.lox[s][ln] = l
        k = dict(
            isp=np.ascontiguousarray(i["isp"], dtype=np.int32),
            igvec=np.ascontiguousarray(i["igvec"], dtype=np.int32),
            minusg=np.ascontiguousarray(i["minusg"], dtype=np.int32),
            gbas=np.asfortranarray(i["gbas"], dtype=np.float64),
            gvec=np.ascontiguousarray(i["gvec"], dtype=np.float64),
            g2=np.ascontiguousarray(i["g2"], dtype=np.float64),
            pro=np.ascontiguousarray(i["pro"], dtype=np.float64),
            ylm=np.ascontiguousarray(i["ylm"], dtype=np.float64),
            mpsi=np.ascontiguousarray(i["mpsi"], dtype=np.float64),
            v=np.ascontiguousarray(i["v"], dtype=np.float64),
            dh=np.ascontiguousarray(i["dh"], dtype=np.complex128),
            dover=np.ascontiguousarray(i["dover"], dtype=np.float64),
            r0=np.ascontiguousarray(i["r0"], dtype=np.float64),
            occ=np.ascontiguousarray(i["occ"], dtype=np.float64),
            psi=np.ascontiguousarray(i["psi"] if psi is None else psi, dtype=np.complex128),
            mass=np.ascontiguousarray(i["masses"], dtype=np.float64),
        )
        d.isp = _ptr(k["isp"], _I)
        r = Request()
        r.dims = d
        for name in ("igvec", "minusg"):
            setattr(r, name, _ptr(k[name], _I))
        for name in ("gbas", "gvec", "g2", "pro", "ylm", "mpsi", "v", "dh", "dover", "r0", "occ", "psi"):
            setattr(r, name, _ptr(k[name], _D))
        r.gweight = float(i["omega"])
        r.lmnxx = int(k["dh"].shape[-1])
        r.lnxx = int(k["dover"].shape[-1])
        r.delt, r.annee = float(i["delt"]), float(i["annee"])
        r.nsteps = int(nsteps)
        r.mass = _ptr(k["mass"], _D) if move_atoms else None
        r.flags = CUW_REQ_BORROW if borrow else 0
        rid = C.c_longlong()
        rc = self._f["submit"](self.h, C.byref(r), C.byref(rid))
        if rc:
            raise WavesError(rc, "server_submit", "request rejected")
        self._nat[rid.value] = int(i["nat"])
        if borrow:
            self._keep[rid.value] = k
        return rid.value

    def poll(self, rid: int):
        """None while pending, else (status, out[8], force(NAT,3), latency_ms)."""
        done, st, lat = C.c_int(), C.c_int(), C.c_double()
        out = np.zeros(8)
        f = np.zeros((self._nat[rid], 3))
        rc = self._f["poll"](self.h, rid, C.byref(done), C.byref(st), _ptr(out, _D), _ptr(f, _D), C.byref(lat))
        if rc:
            raise WavesError(rc, "server_poll", f"unknown request {rid}")
        if not done.value:
            return None
        return st.value, out, f, lat.value

    def error(self, rid: int) -> str:
        buf = C.create_string_buffer(512)
        self._f["error"](self.h, rid, buf, 512)
        return buf.value.decode(errors="replace")

    def result(self, rid: int, timeout: float = 600.0):
        t0 = time.monotonic()
        while True:
            r = self.poll(rid)
            if r is not None:
                if r[0]:
                    raise WavesError(r[0], "server request", self.error(rid))
                return r
            if time.monotonic() - t0 > timeout:
                raise TimeoutError(f"request {rid} not finished after {timeout} s")
            time.sleep(0.0005)

    def release(self, rid: int):
        self._f["release"](self.h, rid)
        self._nat.pop(rid, None)
        self._keep.pop(rid, None)

    def wait_all(self) -> int:
        return self._f["wait_all"](self.h)

    def stats(self) -> dict:
        out = np.zeros(len(STATS))
        self._f["stats"](self.h, _ptr(out, _D), len(out))
        return dict(zip(STATS, out.tolist()))

    def close(self):
        if getattr(self, "h", None):
            self._f["destroy"](self.h)
            self.h = None
        self._keep = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
