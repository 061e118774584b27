"""ctypes binding of the C ABI in include/cuwaves.h.

`Waves` mirrors the reference's WAVES object for one (k-point, spin) set:
its methods carry the names of the reference routines they replace
(hpsi, projections, propagate, orthogonalize, switch, ekin, force, ...), take
the same arguments and raise `WavesError` where the reference calls
ERROR$STOP (src/paw_error.f90:221).  The same class drives any library that
exports the ABI under another symbol prefix.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

CUW_MAXSP = 16
CUW_MAXLN = 8
CUW_PSI0, CUW_PSIM, CUW_HPSI, CUW_OPSI = 0, 1, 2, 3
CUW_PREC_FP64, CUW_PREC_MIXED = 0, 1
CUW_OPT_LYAP_TOL = 1
CUW_OPT_GRAPHS = 2
CUW_OPT_LYAP_MAX_SWEEPS = 3
CUW_OPT_SELFCONSISTENT = 4
CUW_OPT_FFT_VARIANT = 5
CUW_OPT_STREAM_PRIORITY = 6
CUW_OPT_SAFEORTHO = 7
CUW_OPT_SWAPSTATES = 8
CUW_OPT_CONTRACTION_TILES = 9
CUW_OPT_SM_SHARE = 10

ERRORS = {1: "CUW_ERR_ARG", 2: "CUW_ERR_CUDA", 3: "CUW_ERR_STATE", 4: "CUW_ERR_NOT_CONVERGED",
          5: "CUW_ERR_DIVERGED", 6: "CUW_ERR_UNSUPPORTED", 7: "CUW_ERR_NAN", 8: "CUW_ERR_NOMEM"}


class WavesError(RuntimeError):
    def __init__(self, code: int, routine: str, message: str):
        self.code = code
        self.routine = routine
        super().__init__(f"{routine}: {ERRORS.get(code, code)}: {message}")


class Dims(C.Structure):
    _fields_ = [
        ("ngl", C.c_int), ("ndim", C.c_int), ("nb", C.c_int), ("nbh", C.c_int), ("tinv", C.c_int),
        ("nr1", C.c_int), ("nr2", C.c_int), ("nr3", C.c_int), ("nat", C.c_int), ("nsp", C.c_int),
        ("lmx", C.c_int), ("precision", C.c_int),
        ("lnx", C.c_int * CUW_MAXSP), ("lox", (C.c_int * CUW_MAXLN) * CUW_MAXSP),
        ("isp", C.POINTER(C.c_int)),
    ]


# (name, argtypes) of every entry point; handle pointers are c_void_p
_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)
SIGNATURES = {
    "create": [C.POINTER(Dims), C.POINTER(C.c_void_p)],
    "destroy": [_P],
    "last_error": [_P, C.c_char_p, C.c_int],
    "set_gset": [_P, _I, _I, _D, _D, _D, _D, _D, _D, _D, C.c_double],
    "set_potential": [_P, _D],
    "set_dh": [_P, C.c_int, _D],
    "set_do": [_P, C.c_int, _D],
    "set_atoms": [_P, _D, _D],
    "reset_atoms": [_P, _D],
    "get_atoms": [_P, _D, _D, _D],
    "set_occ": [_P, _D],
    "set_dynamics": [_P, C.c_double, C.c_double],
    "set_cell_friction": [_P, _D, C.c_double, C.c_double, _D],
    "upload_psi": [_P, C.c_int, _D],
    "download_psi": [_P, C.c_int, _D],
    "get_proj": [_P, _D],
    "set_proj": [_P, _D],
    "get_rlam0": [_P, _D],
    "set_rlam0": [_P, _D],
    "gramschmidt": [_P, C.c_int, _D],
    "projections": [_P],
    "hpsi": [_P],
    "ekin": [_P, _D],
    "expectation": [_P, _D],
    "wavekinetic": [_P, _D, _D],
    "force": [_P, _D],
    "density": [_P, _D],
    "write_restart": [_P, C.c_char_p, _D],
    "read_restart": [_P, C.c_char_p],
    "denmat": [_P, C.c_int, _D, _D],
    "propagate": [_P],
    "orthogonalize": [_P, C.c_int, C.c_double, _I],
    "switch": [_P],
    "stop": [_P],
    "cp_step": [_P, C.c_int, _D, C.c_int, C.c_double, _D, _D],
    "etot": [_P, _D, _D],
    "overlap_check": [_P, _D, _D],
    "set_rhoset": [_P, C.c_int, _I, _D, _D, C.c_int, _I, _D, _D, _D, _D, _D],
    "set_qlm": [_P, _D],
    "vofrho": [_P, _D, _D, _D, _D, _D, _D],
}
OPTIONAL = {
    "set_async": [_P, C.c_int],
    "synchronize": [_P],
    "set_timing": [_P, C.c_int],
    "get_timing": [_P, _D, C.c_int, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)],
    "get_stream": [_P, C.POINTER(C.c_void_p)],
    "get_ortho_stats": [_P, _D, C.c_int],
    "set_option": [_P, C.c_int, C.c_double],
    "get_graph_stats": [_P, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)],
    "autotune": [_P, _D, C.c_int],
    "tc_gemm_check": [C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _P],
    # batches of sets stepped by one graph launch (no handle argument)
    "batch_create": [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p)],
    "batch_step": [_P, C.c_int, C.POINTER(_D), C.c_int, C.c_double, _D],
    "batch_error": [_P, C.c_char_p, C.c_int],
    "batch_destroy": [_P],
    # device-pointer variant without allocation (no handle)
    "projections_noalloc": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _P, C.c_double, _P, _P],
    "get_atoms": [_P, _D, _D, _D],
    "set_threads": [_P, C.c_int],
}


def _dptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(_D)


def _iptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(_I)


def bind(lib: C.CDLL, prefix: str) -> dict:
    fns = {}
    for name, args in list(SIGNATURES.items()) + list(OPTIONAL.items()):
        sym = prefix + name
        if not hasattr(lib, sym):
            if name in OPTIONAL:
                continue
            raise OSError(f"{sym} not exported")
        f = getattr(lib, sym)
        f.argtypes = args
        f.restype = C.c_int
        fns[name] = f
    return fns


class Waves:
    """One wave-function set on an engine that implements the C ABI."""

    def __init__(self, fns: dict, inputs: dict, precision: int = CUW_PREC_FP64):
        self._f = fns
        self.inp = inputs
        d = Dims()
        d.ngl = inputs["ngl"]
        d.ndim = 1
        d.nb = inputs["nb"]
        d.nbh = inputs["nbh"]
        d.tinv = 1
        d.nr1, d.nr2, d.nr3 = inputs["grid"]
        d.nat = inputs["nat"]
        d.nsp = inputs["nsp"]
        d.lmx = inputs["lmx"]
        d.precision = precision
        for s in range(inputs["nsp"]):
            d.lnx[s] = inputs["lnx"][s]
            for ln, l in enumerate(inputs["lox"][s]):
                d.lox[s][ln] = l
        self._isp = np.ascontiguousarray(inputs["isp"], dtype=np.int32)
        d.isp = _iptr(self._isp)
        self.dims = d
        h = C.c_void_p()
        rc = fns["create"](C.byref(d), C.byref(h))
        if rc:
            buf = C.create_string_buffer(512)
            fns["last_error"](None, buf, 512)
            raise WavesError(rc, "create", buf.value.decode(errors="replace"))
        self.h = h
        self.ngl, self.nb, self.nbh, self.nat = d.ngl, d.nb, d.nbh, d.nat
        self.npro = sum(sum(2 * l + 1 for l in inputs["lox"][s - 1]) for s in self._isp.tolist())

    # -- error handling ------------------------------------------------------
    def _chk(self, rc: int, routine: str):
        if rc:
            buf = C.create_string_buffer(512)
            self._f["last_error"](self.h, buf, 512)
            raise WavesError(rc, routine, buf.value.decode(errors="replace"))

    def close(self):
        if getattr(self, "h", None):
            self._f["destroy"](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- set-up ----------------------------------------------------------------
    def setup(self, psi0: Optional[np.ndarray] = None, psim: Optional[np.ndarray] = None):
        """Loads G-set, potential, one-centre matrices, atoms, occupations and
        dynamics parameters from the inputs dictionary."""
        i = self.inp
        self._keep = dict(
            igvec=np.ascontiguousarray(i["igvec"], dtype=np.int32),
            minusg=np.ascontiguousarray(i["minusg"], dtype=np.int32),
            gbas=np.asfortranarray(i["gbas"], dtype=np.float64),
            gvec=np.ascontiguousarray(i["gvec"], dtype=np.float64),
            g2=np.ascontiguousarray(i["g2"], dtype=np.float64),
            pro=np.ascontiguousarray(i["pro"], dtype=np.float64),
            ylm=np.ascontiguousarray(i["ylm"], dtype=np.float64),
            mpsi=np.ascontiguousarray(i["mpsi"], dtype=np.float64),
        )
        k = self._keep
        self._chk(self._f["set_gset"](self.h, _iptr(k["igvec"]), _iptr(k["minusg"]), _dptr(k["gbas"]),
                                      _dptr(k["gvec"]), _dptr(k["g2"]), _dptr(k["pro"]), _dptr(k["ylm"]),
                                      _dptr(k["mpsi"]), None, float(i["omega"])), "set_gset")
        self.set_potential(i["v"])
        self.set_dh(i["dh"])
        self.set_do(i["dover"])
        self.reset_atoms(i["r0"])
        self.set_occ(i["occ"])
        self.set_dynamics(i["delt"], i["annee"])
        p0 = i["psi"] if psi0 is None else psi0
        self.upload_psi(CUW_PSI0, p0)
        self.upload_psi(CUW_PSIM, p0 if psim is None else psim)
        return self

    def set_potential(self, v):
        a = np.ascontiguousarray(v, dtype=np.float64)
        self._chk(self._f["set_potential"](self.h, _dptr(a)), "set_potential")

    def set_dh(self, dh):
        a = np.ascontiguousarray(dh, dtype=np.complex128)
        self._chk(self._f["set_dh"](self.h, int(a.shape[-1]), a.ctypes.data_as(_D)), "set_dh")

    def set_do(self, dover):
        a = np.ascontiguousarray(dover, dtype=np.float64)
        self._chk(self._f["set_do"](self.h, int(a.shape[-1]), _dptr(a)), "set_do")

    def set_atoms(self, r0=None, rp=None):
        a = None if r0 is None else np.ascontiguousarray(r0, dtype=np.float64)
        b = None if rp is None else np.ascontiguousarray(rp, dtype=np.float64)
        self._chk(self._f["set_atoms"](self.h, _dptr(a), _dptr(b)), "set_atoms")

    def get_atoms(self):
        """(R(-), R(0), R(+)) as (NAT, 3) arrays."""
        rs = [np.zeros((self.nat, 3)) for _ in range(3)]
        self._chk(self._f["get_atoms"](self.h, _dptr(rs[0]), _dptr(rs[1]), _dptr(rs[2])), "get_atoms")
        return tuple(rs)

    def reset_atoms(self, r0):
        a = np.ascontiguousarray(r0, dtype=np.float64)
        self._chk(self._f["reset_atoms"](self.h, _dptr(a)), "reset_atoms")

    def set_occ(self, occ):
        a = np.ascontiguousarray(occ, dtype=np.float64)
        self._chk(self._f["set_occ"](self.h, _dptr(a)), "set_occ")

    def set_dynamics(self, delt, annee=0.0):
        self._chk(self._f["set_dynamics"](self.h, float(delt), float(annee)), "set_dynamics")

    def set_cell_friction(self, fricmat=None, emass=0.0, emasscg2=0.0, dbucket=None):
        """G-dependent friction of a moving cell (WAVES_DMPSI with TSTRESS);
        fricmat (3, 3) = PSIANNEMAT, None switches it off."""
        f = None if fricmat is None else np.asfortranarray(fricmat, dtype=np.float64)
        d = None if dbucket is None else np.ascontiguousarray(dbucket, dtype=np.float64)
        self._chk(self._f["set_cell_friction"](self.h, _dptr(f), float(emass), float(emasscg2), _dptr(d)),
                  "set_cell_friction")

    # -- data movement -------------------------------------------------------
    def upload_psi(self, which: int, psi):
        a = np.ascontiguousarray(psi, dtype=np.complex128)
        assert a.size == self.ngl * self.nbh
        self._chk(self._f["upload_psi"](self.h, which, a.ctypes.data_as(_D)), "upload_psi")

    def download_psi(self, which: int) -> np.ndarray:
        a = np.empty((self.nbh, self.ngl), dtype=np.complex128)
        self._chk(self._f["download_psi"](self.h, which, a.ctypes.data_as(_D)), "download_psi")
        return a

    def get_proj(self) -> np.ndarray:
        """PROJ(1,NBH,NPRO) returned with shape (NPRO, NBH)."""
        a = np.empty((self.npro, self.nbh), dtype=np.complex128)
        self._chk(self._f["get_proj"](self.h, a.ctypes.data_as(_D)), "get_proj")
        return a

    def set_proj(self, proj):
        a = np.ascontiguousarray(proj, dtype=np.complex128)
        self._chk(self._f["set_proj"](self.h, a.ctypes.data_as(_D)), "set_proj")

    def get_rlam0(self) -> np.ndarray:
        """RLAM0(NB,NB) returned with shape (NB, NB) indexed [j, i]."""
        a = np.empty((self.nb, self.nb), dtype=np.complex128)
        self._chk(self._f["get_rlam0"](self.h, a.ctypes.data_as(_D)), "get_rlam0")
        return a

    def set_rlam0(self, r):
        a = np.ascontiguousarray(r, dtype=np.complex128)
        self._chk(self._f["set_rlam0"](self.h, a.ctypes.data_as(_D)), "set_rlam0")

    # -- the WAVES operations --------------------------------------------------
    def gramschmidt(self, which: int, r):
        a = np.ascontiguousarray(r, dtype=np.float64)
        self._chk(self._f["gramschmidt"](self.h, which, _dptr(a)), "WAVES_GRAMSCHMIDT")

    def projections(self):
        self._chk(self._f["projections"](self.h), "WAVES$PROJECTIONS")

    def hpsi(self):
        self._chk(self._f["hpsi"](self.h), "WAVES$HPSI")

    def ekin(self) -> float:
        x = C.c_double()
        self._chk(self._f["ekin"](self.h, C.byref(x)), "WAVES$EKIN")
        return x.value

    def expectation(self) -> np.ndarray:
        a = np.empty(self.nb)
        self._chk(self._f["expectation"](self.h, _dptr(a)), "WAVES$ETOT")
        return a

    def wavekinetic(self):
        x = C.c_double()
        a = np.empty(self.nb)
        self._chk(self._f["wavekinetic"](self.h, C.byref(x), _dptr(a)), "WAVES_WAVEKINETIC")
        return x.value, a

    def force(self) -> np.ndarray:
        a = np.empty((self.nat, 3))
        self._chk(self._f["force"](self.h, _dptr(a)), "WAVES$FORCE")
        return a

    def write_restart(self, path, rbas=None):
        """WAVES$WRITE: the WAVES section of a restart file for this set."""
        r = None if rbas is None else np.asfortranarray(rbas, dtype=np.float64)
        self._chk(self._f["write_restart"](self.h, str(path).encode(), _dptr(r)), "WAVES$WRITE")

    def read_restart(self, path):
        """WAVES$READ of a section written for the same bands."""
        self._chk(self._f["read_restart"](self.h, str(path).encode()), "WAVES$READ")

    def density(self) -> np.ndarray:
        """WAVES_DENSITY of this set: rho as an (NR3, NR2, NR1) array."""
        d = self.dims
        rho = np.empty(d.nr1 * d.nr2 * d.nr3)
        self._chk(self._f["density"](self.h, _dptr(rho)), "WAVES$RHO")
        return rho.reshape(d.nr3, d.nr2, d.nr1)

    def denmat(self, lmnxx=None):
        """WAVES$DENMAT of this set: (denmat, edenmat), each (NAT, LMNXX, LMNXX)
        complex with [a, lmn2, lmn1] = DENMAT(lmn1, lmn2, a)."""
        if lmnxx is None:
            lmnxx = max(sum(2 * l + 1 for l in self.inp["lox"][s - 1]) for s in self._isp.tolist())
        n = lmnxx * lmnxx * max(1, self.nat)
        dm = np.zeros(n, dtype=np.complex128)
        em = np.zeros(n, dtype=np.complex128)
        self._chk(self._f["denmat"](self.h, lmnxx, dm.ctypes.data_as(_D), em.ctypes.data_as(_D)), "WAVES$DENMAT")
        return dm.reshape(max(1, self.nat), lmnxx, lmnxx), em.reshape(max(1, self.nat), lmnxx, lmnxx)

    def propagate(self):
        self._chk(self._f["propagate"](self.h), "WAVES$PROPAGATE")

    def orthogonalize(self, max_iter: int = 200, eps: float = 1e-8) -> int:
        it = C.c_int()
        self._chk(self._f["orthogonalize"](self.h, max_iter, eps, C.byref(it)), "WAVES$ORTHOGONALIZE")
        return it.value

    def switch(self):
        self._chk(self._f["switch"](self.h), "WAVES$SWITCH")

    def stop(self):
        self._chk(self._f["stop"](self.h), "WAVES$STOP")

    def cp_step(self, move_atoms: bool = False, max_iter: int = 200, eps: float = 1e-8, want_force=True):
        out = np.zeros(8)
        f = np.zeros((self.nat, 3)) if want_force else None
        m = np.ascontiguousarray(self.inp["masses"], dtype=np.float64)
        self._chk(self._f["cp_step"](self.h, int(move_atoms), _dptr(m), max_iter, eps, _dptr(out), _dptr(f)),
                  "TIMESTEP")
        return out, f

    def etot(self, want_force=True):
        """Single-point energy (sum_n f_n <psi_n|H|psi_n>, kinetic energy) and forces
        at PSI0 and R(0), without propagation (WAVES$ETOT energy part)."""
        out = np.zeros(2)
        f = np.zeros((self.nat, 3)) if want_force else None
        self._chk(self._f["etot"](self.h, _dptr(out), _dptr(f)), "ETOT")
        return out, f

    def overlap_check(self):
        """(MAT, max|MAT - 1|): <psi_i|O|psi_j> of PSI0 with projections formed
        afresh at R(0), the orthonormality test of WAVES$ORTHOGONALIZE.  MAT is
        returned as an (NB, NB) array indexed [j, i]."""
        m = np.empty((self.nb, self.nb))
        x = C.c_double()
        self._chk(self._f["overlap_check"](self.h, _dptr(m), C.byref(x)), "overlap_check")
        return m, x.value

    def set_rhoset(self):
        """Loads the density G set and its tables (inputs key 'rhoset')."""
        r = self.inp["rhoset"]
        self._rk = dict(
            igvec=np.ascontiguousarray(r["igvec"], dtype=np.int32),
            gvec=np.ascontiguousarray(r["gvec"], dtype=np.float64),
            g2=np.ascontiguousarray(r["g2"], dtype=np.float64),
            lmrx=np.ascontiguousarray(r["lmrx"], dtype=np.int32),
            ylm=np.ascontiguousarray(r["ylm"], dtype=np.float64),
            g0=np.ascontiguousarray(r["g0"], dtype=np.float64),
            v0=np.ascontiguousarray(r["v0"], dtype=np.float64),
            pscore=np.ascontiguousarray(r["pscore"], dtype=np.float64),
            vbar=np.ascontiguousarray(r["vbar"], dtype=np.float64),
        )
        k = self._rk
        self._chk(self._f["set_rhoset"](self.h, int(len(k["g2"])), _iptr(k["igvec"]), _dptr(k["gvec"]),
                                        _dptr(k["g2"]), int(r["lmrxx"]), _iptr(k["lmrx"]), _dptr(k["ylm"]),
                                        _dptr(k["g0"]), _dptr(k["v0"]), _dptr(k["pscore"]), _dptr(k["vbar"])),
                  "POTENTIAL_UPDATE")
        self.set_qlm(r["qlm"])
        return self

    def set_qlm(self, qlm):
        a = np.ascontiguousarray(qlm, dtype=np.float64)
        self._chk(self._f["set_qlm"](self.h, _dptr(a)), "set_qlm")

    def vofrho(self, rho=None, qlm=None):
        """POTENTIAL$VOFRHO: (V as an (NR3, NR2, NR1) array, {EHARTREE, EXC, RHOB},
        forces (NAT, 3), VQLM (NAT, LMRXX)); the handle's potential becomes V."""
        d = self.dims
        nr = d.nr1 * d.nr2 * d.nr3
        r = None if rho is None else np.ascontiguousarray(rho, dtype=np.float64).reshape(-1)
        q = None if qlm is None else np.ascontiguousarray(qlm, dtype=np.float64)
        v = np.empty(nr)
        e = np.empty(3)
        f = np.empty((self.nat, 3))
        lmrxx = int(self.inp["rhoset"]["lmrxx"])
        vq = np.empty((self.nat, lmrxx))
        self._chk(self._f["vofrho"](self.h, _dptr(r), _dptr(q), _dptr(v), _dptr(e), _dptr(f), _dptr(vq)),
                  "POTENTIAL$VOFRHO")
        return v.reshape(d.nr3, d.nr2, d.nr1), dict(zip(("ehartree", "exc", "rhob"), e.tolist())), f, vq

    def set_async(self, flag: bool):
        if "set_async" in self._f:
            self._chk(self._f["set_async"](self.h, int(flag)), "set_async")

    def synchronize(self):
        if "synchronize" in self._f:
            self._chk(self._f["synchronize"](self.h), "synchronize")

    PHASES = ("reductions", "structure factors", "forces", "fft_vpsi", "addpro_propagate",
              "projections", "gram", "ortho_solve", "rotate", "bookkeeping", "potential")

    def set_option(self, option: int, value: float):
        self._chk(self._f["set_option"](self.h, int(option), float(value)), "set_option")

    def autotune(self) -> dict:
        """Times and fixes the FFT plan variant and band batch, the tile family of
        the contractions (mixed precision) and the split-K factors."""
        out = np.zeros(11)
        self._chk(self._f["autotune"](self.h, _dptr(out), len(out)), "autotune")
        keys = ("fft_batch", "split_proj", "split_gram", "fft_ms", "proj_ms", "gram_ms", "cached", "fft_variant",
                "dmma_tiles", "tc_tiles_ms", "dmma_tiles_ms")
        return dict(zip(keys, out.tolist()))

    def graph_stats(self) -> tuple:
        n, r = C.c_longlong(), C.c_longlong()
        self._chk(self._f["get_graph_stats"](self.h, C.byref(n), C.byref(r)), "get_graph_stats")
        return n.value, r.value

    def set_timing(self, on: bool):
        self._chk(self._f["set_timing"](self.h, int(on)), "set_timing")

    def get_timing(self):
        ms = np.zeros(len(self.PHASES))
        nl, ns = C.c_longlong(), C.c_longlong()
        self._chk(self._f["get_timing"](self.h, _dptr(ms), len(ms), C.byref(nl), C.byref(ns)), "get_timing")
        return dict(zip(self.PHASES, ms.tolist())), nl.value, ns.value

    ORTHO_STATS = ("eigendecompositions", "fixed_point_sweeps", "last_jacobi_sweeps", "last_ortho_iterations",
                   "fixed_point_fallbacks")

    def ortho_stats(self) -> dict:
        out = np.zeros(len(self.ORTHO_STATS))
        self._chk(self._f["get_ortho_stats"](self.h, _dptr(out), len(out)), "get_ortho_stats")
        return dict(zip(self.ORTHO_STATS, out.tolist()))

    def stream(self) -> int:
        s = C.c_void_p()
        self._chk(self._f["get_stream"](self.h, C.byref(s)), "get_stream")
        return s.value or 0

    def initialize(self, gram_schmidt: bool = True):
        """Start-up of WAVES$ETOT at TFIRST (src/paw_waves1.f90:1733-1748):
        Gram-Schmidt of PSI0 (at R(0)) and PSIM (at R(-)), then PROJ of PSI0."""
        if gram_schmidt:
            r = self.inp["r0"]
            self.gramschmidt(CUW_PSI0, r)
            self.gramschmidt(CUW_PSIM, r)
        self.projections()
        return self


class Batch:
    """Several wave-function sets advanced together by one CUDA graph launch
    (cuwaves_batch_*): step() advances every set by two CP steps."""

    def __init__(self, sets):
        self.sets = list(sets)
        self._f = self.sets[0]._f
        arr = (C.c_void_p * len(self.sets))(*[w.h for w in self.sets])
        b = C.c_void_p()
        rc = self._f["batch_create"](arr, len(self.sets), C.byref(b))
        if rc:
            raise WavesError(rc, "batch_create", "")
        self.b = b
        self._masses = [np.ascontiguousarray(w.inp["masses"], dtype=np.float64) for w in self.sets]
        self._mp = (_D * len(self.sets))(*[_dptr(m) for m in self._masses])

    def step(self, move_atoms: bool = False, max_iter: int = 200, eps: float = 1e-8) -> np.ndarray:
        """Two CP steps of every set; returns out[set, step, 8] as cuwaves_cp_step."""
        out = np.zeros((len(self.sets), 2, 8))
        rc = self._f["batch_step"](self.b, int(move_atoms), self._mp if move_atoms else None, max_iter, eps,
                                   _dptr(out))
        if rc:
            buf = C.create_string_buffer(512)
            self._f["batch_error"](self.b, buf, 512)
            raise WavesError(rc, "batch_step", buf.value.decode(errors="replace"))
        return out

    def close(self):
        if getattr(self, "b", None):
            self._f["batch_destroy"](self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(os.path.dirname(PKG_DIR), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libcuwaves.so")


def load_library(path: Optional[str] = None) -> C.CDLL:
    """Loads the B200 engine.  There is no fallback: a missing library or a
    machine without a CUDA device raises."""
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise OSError(f"libcuwaves.so not built: {p} (run __graft_entry__.build())")
    return C.CDLL(p, mode=C.RTLD_GLOBAL)


_engine_fns = None


def engine() -> dict:
    global _engine_fns
    if _engine_fns is None:
        _engine_fns = bind(load_library(), "cuwaves_")
    return _engine_fns


def open_waves(inputs: dict, precision: int = CUW_PREC_FP64) -> Waves:
    return Waves(engine(), inputs, precision)
