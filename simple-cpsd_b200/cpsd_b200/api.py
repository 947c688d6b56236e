"""Python mirror of the reference's entry points, backed by the CUDA library.

* ``cpsd(inp, state, inner)`` -- one call of the drop-in ``cpsd()`` of
  ccpsdv3/cpsd.c:33-71 with host numpy buffers (``state`` is updated in
  place exactly as the reference updates its arrays).
* ``GpuCell`` -- a persistent context: tables and orbitals stay resident in
  HBM between calls; ``run(inner)`` is the body of ``cpsd()``.
* ``cr_fft3b`` / ``rc_fft3f`` -- the fftpack3d 3-D FFT drop-ins.

Errors raise ``CpsdError``; the Lagrange non-convergence warning of the
reference (``ierr=10``, cpsd.c:477) is counted, not raised.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import lib as _l
from .lib import CpsdError

_P = ctypes.c_void_p


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.flags.c_contiguous, "arrays must be C-contiguous"
    return a.ctypes.data_as(_P)


class State:
    """The arrays cpsd() reads and writes (sizes as ccpsdv3/main.c:124-136)."""

    def __init__(self, inp):
        ne0, ne1 = int(inp.ne[0]), int(inp.ne[1])
        self.c2 = inp.c2.copy()
        self.c1 = inp.c2.copy()
        self.cpsi = np.zeros_like(inp.c2)
        self.dn = np.zeros(inp.ispin * inp.n2ft3d)
        self.hml = np.zeros(ne0 * ne0 + ne1 * ne1)
        self.lmd = np.zeros(ne0 * ne0 + ne1 * ne1)
        self.r2 = inp.r2.copy()
        self.r1 = inp.r2.copy()
        self.fion = np.zeros(3 * max(inp.nion, 1))
        self.E = np.zeros(10)
        self.deltae = 0.0
        self.deltac = 0.0
        self.deltar = 0.0
        self.lagrange_fail = 0


_DROPIN_INP = ("unitg", "katm", "amass", "zv", "rcell", "masker", "G", "tg", "vc", "vg", "lmmax", "vnlnrm",
               "vl", "vnl")
_DROPIN_ST = ("r1", "r2", "fion", "c1", "c2", "cpsi", "dn", "hml", "lmd", "E")


def _dropin_args(inp, st: State, inner: int, move: int):
    """The C arguments of one drop-in call, built once per (inputs, state)
    and reused while every array object and scalar they name is the same
    (marshalling 40 arguments costs about as much as a small cell's step)."""
    key = (id(inp), inner, move, int(inp.nion), int(inp.ispin), int(inp.nfft), int(inp.nfft3d), int(inp.n2ft3d),
           float(inp.omega), float(inp.dt), float(inp.fmass), int(inp.nsh), float(inp.cewald), float(inp.rcut),
           tuple(int(x) for x in inp.ne), tuple(id(getattr(inp, n)) for n in _DROPIN_INP),
           tuple(id(getattr(st, n)) for n in _DROPIN_ST))
    cached = getattr(st, "_dropin", None)
    if cached is not None and cached[0] == key:
        return cached[1], cached[2]
    ne = np.ascontiguousarray(inp.ne, dtype=np.int32)
    dd = [ctypes.c_double() for _ in range(3)]
    args = (ctypes.c_int(inner), ctypes.c_int(move), ctypes.c_int(inp.nion), ctypes.c_int(inp.ispin),
            _ptr(ne), ctypes.c_int(inp.nfft), ctypes.c_int(inp.nfft3d), ctypes.c_int(inp.n2ft3d),
            _ptr(inp.unitg), ctypes.c_double(inp.omega), ctypes.c_double(inp.dt),
            ctypes.c_double(inp.fmass), _ptr(inp.katm), _ptr(inp.amass), _ptr(inp.zv),
            ctypes.c_int(inp.nsh), _ptr(inp.rcell), ctypes.c_double(inp.cewald),
            ctypes.c_double(inp.rcut), _ptr(inp.masker), _ptr(inp.G), _ptr(inp.tg), _ptr(inp.vc),
            _ptr(inp.vg), _ptr(inp.lmmax), _ptr(inp.vnlnrm), _ptr(inp.vl), _ptr(inp.vnl),
            _ptr(st.r1), _ptr(st.r2), _ptr(st.fion), _ptr(st.c1), _ptr(st.c2), _ptr(st.cpsi),
            _ptr(st.dn), _ptr(st.hml), _ptr(st.lmd), _ptr(st.E), ctypes.byref(dd[0]),
            ctypes.byref(dd[1]), ctypes.byref(dd[2]))
    st._dropin = (key, args, dd, ne)  # ne stays alive with the pointer to it
    return args, dd


def cpsd(inp, st: State, inner: int, move: int = 0) -> State:
    """The drop-in: exactly the reference's cpsd() call with host buffers."""
    L = _l.load()
    args, dd = _dropin_args(inp, st, inner, move)
    rc = L.cpsd_gpu_cpsd(*args)
    if rc == _l.CPSD_WARN_LAGRANGE:
        st.lagrange_fail += 1
    elif rc != _l.CPSD_OK:
        raise CpsdError(rc, "cpsd")
    st.deltae, st.deltac, st.deltar = dd[0].value, dd[1].value, dd[2].value
    return st


class GpuCell:
    """A cell resident on one GPU (the persistent-context API)."""

    def __init__(self, inp, precision: int = _l.CPSD_PREC_FP64, device: int = 0):
        L = _l.load()
        self._L = L
        self.inp = inp
        p = _l.Params()
        p.nfft = inp.nfft
        p.ispin = inp.ispin
        p.ne[0] = int(inp.ne[0])
        p.ne[1] = int(inp.ne[1])
        p.nion = inp.nion
        p.nkatm = len(inp.zv)
        p.nsh = inp.nsh
        p.precision = precision
        p.device = device
        for i in range(9):
            p.unitg[i] = float(inp.unitg[i])
        p.omega, p.dt, p.fmass, p.cewald, p.rcut = inp.omega, inp.dt, inp.fmass, inp.cewald, inp.rcut
        h = ctypes.c_void_p()
        m1 = np.ascontiguousarray(inp.masker1, dtype=np.int32)
        rc = L.cpsd_gpu_create(ctypes.byref(p), _ptr(m1), ctypes.byref(h))
        if rc:
            raise CpsdError(rc, "cpsd_gpu_create")
        self.h = h
        self.device = device
        self._check(L.cpsd_gpu_set_tables(
            h, _ptr(inp.katm), _ptr(inp.amass), _ptr(inp.zv), _ptr(inp.rcell), _ptr(inp.G),
            _ptr(inp.tg), _ptr(inp.vc), _ptr(inp.vg), _ptr(inp.lmmax), _ptr(inp.vnlnrm),
            _ptr(inp.vl), _ptr(inp.vnl)), "cpsd_gpu_set_tables")
        self.E = np.zeros(10)
        self.deltae = self.deltac = self.deltar = 0.0
        self.lagrange_warnings = 0

    def _check(self, rc: int, what: str) -> int:
        if rc not in (_l.CPSD_OK, _l.CPSD_WARN_LAGRANGE):
            raise CpsdError(rc, what)
        return rc

    @property
    def npw(self) -> int:
        return self._L.cpsd_gpu_npw(self.h)

    def geometry(self) -> dict:
        out = (ctypes.c_int * 6)()
        self._check(self._L.cpsd_gpu_geometry(self.h, out), "cpsd_gpu_geometry")
        return dict(npw=out[0], npw_pad=out[1], ncol=out[2], KX=out[3], nproj=out[4], dens_chunks=out[5])

    @property
    def launches_per_step(self) -> int:
        return self._L.cpsd_gpu_launches_per_step(self.h)

    def counters(self):
        """(kernel launches, host-to-device bytes, device-to-host bytes) so far."""
        out = (ctypes.c_longlong * 3)()
        self._L.cpsd_gpu_counters(self.h, out)
        return int(out[0]), int(out[1]), int(out[2])

    def set_precision(self, precision: int) -> None:
        """CPSD_PREC_FP64 or CPSD_PREC_MIXED for the following steps."""
        self._check(self._L.cpsd_gpu_set_precision(self.h, int(precision)), "cpsd_gpu_set_precision")

    def use_graphs(self, on: bool) -> None:
        self._check(self._L.cpsd_gpu_use_graphs(self.h, 1 if on else 0), "cpsd_gpu_use_graphs")

    def phase_timing(self, on: bool) -> None:
        self._check(self._L.cpsd_gpu_phase_timing(self.h, 1 if on else 0), "cpsd_gpu_phase_timing")

    def phase_times(self):
        """{phase name: ms} of the last SD step (phase timing must be on)."""
        buf = (ctypes.c_float * 32)()
        n = self._L.cpsd_gpu_phase_times(self.h, buf, 32)
        return {self._L.cpsd_gpu_phase_name(i).decode(): float(buf[i]) for i in range(n)}

    @property
    def stream(self) -> int:
        return self._L.cpsd_gpu_stream(self.h) or 0

    def set_preconditioner(self, mlp) -> None:
        """Attach a trained Mlp (learned SD step scales) or None for plain SD."""
        self._check(self._L.cpsd_gpu_set_preconditioner(self.h, mlp.h if mlp is not None else None),
                    "cpsd_gpu_set_preconditioner")
        self._mlp = mlp  # keep it alive while attached

    def run_guarded(self, inner: int, cap: float, blocks: int = 1):
        """Blocks of learned steps with plain SD as the arbiter, in the library
        (cpsd_gpu_run_guarded): returns (energy, rejected blocks, new cap)."""
        c = np.array([cap], dtype=np.float64)
        de, dc = ctypes.c_double(), ctypes.c_double()
        rej = ctypes.c_int(0)
        rc = self._L.cpsd_gpu_run_guarded(self.h, int(blocks), int(inner), _ptr(c), _ptr(self.E), ctypes.byref(de),
                                          ctypes.byref(dc), ctypes.byref(rej))
        if rc == _l.CPSD_WARN_LAGRANGE:
            self.lagrange_warnings += 1
        elif rc != _l.CPSD_OK:
            raise CpsdError(rc, "cpsd_gpu_run_guarded")
        self.deltae, self.deltac = de.value, dc.value
        return float(self.E[0]), rej.value, float(c[0])

    # band-parallel SD (cpsd_b200.bands drives these)
    def set_band_range(self, lo: int, hi: int) -> None:
        self._check(self._L.cpsd_gpu_set_band_range(self.h, int(lo), int(hi)), "cpsd_gpu_set_band_range")

    def step_phase(self, phase: int) -> None:
        self._check(self._L.cpsd_gpu_step_phase(self.h, int(phase)), "cpsd_gpu_step_phase")

    def bp_buffers(self):
        """Device addresses (dn_part, dn, c2, cpsi) and the row length in doubles."""
        p = [ctypes.c_void_p() for _ in range(4)]
        ld = ctypes.c_long()
        self._check(self._L.cpsd_gpu_bp_buffers(self.h, *[ctypes.byref(x) for x in p], ctypes.byref(ld)),
                    "cpsd_gpu_bp_buffers")
        return tuple(x.value for x in p) + (ld.value,)

    def bp_finish(self, inner: int) -> np.ndarray:
        de, dc = ctypes.c_double(), ctypes.c_double()
        rc = self._L.cpsd_gpu_bp_finish(self.h, int(inner), _ptr(self.E), ctypes.byref(de), ctypes.byref(dc))
        if rc == _l.CPSD_WARN_LAGRANGE:
            self.lagrange_warnings += 1
        elif rc != _l.CPSD_OK:
            raise CpsdError(rc, "cpsd_gpu_bp_finish")
        self.deltae, self.deltac = de.value, dc.value
        return self.E

    def tuning(self) -> dict:
        """The kernel choices of this context (cpsd_gpu_get_tuning)."""
        t = _l.Tuning()
        self._check(self._L.cpsd_gpu_get_tuning(self.h, ctypes.byref(t)), "cpsd_gpu_get_tuning")
        return t.as_dict()

    def tuning_limits(self) -> dict:
        t = _l.Tuning()
        self._check(self._L.cpsd_gpu_tuning_limits(self.h, ctypes.byref(t)), "cpsd_gpu_tuning_limits")
        return t.as_dict()

    def set_tuning(self, **kw) -> None:
        """Change some kernel choices (cpsd_gpu_set_tuning); unnamed fields keep their values."""
        cur = self.tuning()
        cur.update(kw)
        t = _l.Tuning()
        for i, v in enumerate(cur["plane_occupancy"]):
            t.plane_occupancy[i] = int(v)
        t.tn_ctas_per_sm = int(cur["tn_ctas_per_sm"])
        t.density_chunks = int(cur["density_chunks"])
        t.lagrange_solver = int(cur["lagrange_solver"])
        self._check(self._L.cpsd_gpu_set_tuning(self.h, ctypes.byref(t)), "cpsd_gpu_set_tuning")

    def autotune(self, steps: int = 10, force: bool = False) -> dict:
        """Time the candidate kernel choices on this cell and keep the
        fastest (cpsd_gpu_autotune); returns the choices and ms per SD step
        before and after (-1 when the process cache had this shape)."""
        b, a = ctypes.c_float(), ctypes.c_float()
        self._check(self._L.cpsd_gpu_autotune(self.h, int(steps), int(force), ctypes.byref(b), ctypes.byref(a)),
                    "cpsd_gpu_autotune")
        return {"tuning": self.tuning(), "ms_per_step_before": b.value, "ms_per_step_after": a.value}

    def set_gemm(self, mode: int) -> None:
        """TN-product engine of the mixed path: CPSD_GEMM_FP64 or CPSD_GEMM_TF32X3."""
        self._check(self._L.cpsd_gpu_set_gemm(self.h, int(mode)), "cpsd_gpu_set_gemm")

    def set_preconditioner_range(self, min_log_k: float, max_log_k: float) -> None:
        """Range of the learned log step scale ([0, 0]: plain SD steps)."""
        self._check(self._L.cpsd_gpu_set_preconditioner_range(self.h, float(min_log_k), float(max_log_k)),
                    "cpsd_gpu_set_preconditioner_range")

    def save_orbitals(self) -> None:
        self._check(self._L.cpsd_gpu_save_orbitals(self.h), "cpsd_gpu_save_orbitals")

    def restore_orbitals(self) -> None:
        self._check(self._L.cpsd_gpu_restore_orbitals(self.h), "cpsd_gpu_restore_orbitals")

    def get_packed(self):
        """(c1, c2, cpsi) as complex (nbands, npw) arrays in sphere order."""
        nb, npw = self.inp.nbands, self.npw
        out = [np.zeros((nb, npw), dtype=np.complex128) for _ in range(3)]
        self._check(self._L.cpsd_gpu_get_packed(self.h, *[_ptr(o) for o in out]), "cpsd_gpu_get_packed")
        return out

    def get_c2(self) -> np.ndarray:
        """The current orbitals only, complex (nbands, npw) in sphere order."""
        out = np.zeros((self.inp.nbands, self.npw), dtype=np.complex128)
        self._check(self._L.cpsd_gpu_get_packed(self.h, None, _ptr(out), None), "cpsd_gpu_get_packed")
        return out

    def set_packed(self, c2: np.ndarray) -> None:
        c2 = np.ascontiguousarray(c2, dtype=np.complex128)
        self._check(self._L.cpsd_gpu_set_packed(self.h, _ptr(c2)), "cpsd_gpu_set_packed")

    def sphere(self):
        """(half-box index, Gamma weight, |G| shell) of every sphere point."""
        npw = self.npw
        idx = np.zeros(npw, dtype=np.int32)
        w = np.zeros(npw)
        sh = np.zeros(npw, dtype=np.int32)
        self._check(self._L.cpsd_gpu_get_sphere(self.h, _ptr(idx), _ptr(w), _ptr(sh)), "cpsd_gpu_get_sphere")
        return idx, w, sh

    def set_state(self, c2: np.ndarray, r2: np.ndarray) -> None:
        self._check(self._L.cpsd_gpu_set_state(self.h, _ptr(np.ascontiguousarray(c2)),
                                               _ptr(np.ascontiguousarray(r2))), "cpsd_gpu_set_state")

    def run(self, inner: int, move: int = 0) -> np.ndarray:
        dd = [ctypes.c_double() for _ in range(3)]
        rc = self._check(self._L.cpsd_gpu_run(self.h, inner, move, _ptr(self.E), ctypes.byref(dd[0]),
                                              ctypes.byref(dd[1]), ctypes.byref(dd[2])), "cpsd_gpu_run")
        if rc == _l.CPSD_WARN_LAGRANGE:
            self.lagrange_warnings += 1
        self.deltae, self.deltac, self.deltar = dd[0].value, dd[1].value, dd[2].value
        return self.E

    def get_state(self, st: State) -> State:
        self._check(self._L.cpsd_gpu_get_state(self.h, _ptr(st.c1), _ptr(st.c2), _ptr(st.cpsi),
                                                _ptr(st.dn), _ptr(st.hml), _ptr(st.lmd), _ptr(st.r1),
                                                _ptr(st.r2), _ptr(st.fion)), "cpsd_gpu_get_state")
        st.E[:] = self.E
        st.deltae, st.deltac, st.deltar = self.deltae, self.deltac, self.deltar
        return st

    def epilogue(self) -> dict:
        """The run's epilogue on the device (ccpsdv3/main.c:452-487): the
        orthonormality table <c1_i|c1_j>, the eigenvalues of hml per spin in
        descending order (eig[ms*ne0 + i]) with their eigenvectors (hml's
        layout), and c1 <- c2 V, which get_state then returns."""
        ne0, ne1 = int(self.inp.ne[0]), int(self.inp.ne[1])
        ortho = np.zeros(ne0 * ne0 + ne1 * ne1)
        vec = np.zeros_like(ortho)
        eig = np.zeros(ne0 + ne1)
        self._check(self._L.cpsd_gpu_epilogue(self.h, _ptr(ortho), _ptr(eig), _ptr(vec)), "cpsd_gpu_epilogue")
        return {"ortho": ortho, "eig": eig, "vec": vec}

    def close(self) -> None:
        if getattr(self, "h", None):
            self._L.cpsd_gpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuBatch:
    """Many resident cells stepped together: one CUDA graph launch per SD step."""

    def __init__(self, cells):
        self._L = _l.load()
        self.cells = list(cells)
        arr = (ctypes.c_void_p * len(self.cells))(*[c.h for c in self.cells])
        h = ctypes.c_void_p()
        rc = self._L.cpsd_gpu_batch_create(arr, len(self.cells), ctypes.byref(h))
        if rc:
            raise CpsdError(rc, "cpsd_gpu_batch_create")
        self.h = h
        self.E = np.zeros((len(self.cells), 10))
        self.deltae = np.zeros(len(self.cells))
        self.deltac = np.zeros(len(self.cells))
        self.lagrange_warnings = 0

    def run(self, inner: int) -> np.ndarray:
        rc = self._L.cpsd_gpu_batch_run(self.h, inner, _ptr(self.E), _ptr(self.deltae), _ptr(self.deltac))
        if rc == _l.CPSD_WARN_LAGRANGE:
            self.lagrange_warnings += 1
        elif rc != _l.CPSD_OK:
            raise CpsdError(rc, "cpsd_gpu_batch_run")
        for c, e, de, dc in zip(self.cells, self.E, self.deltae, self.deltac):
            c.E[:] = e
            c.deltae, c.deltac = float(de), float(dc)
        return self.E

    def launches(self) -> int:
        out = (ctypes.c_longlong * 1)()
        self._L.cpsd_gpu_batch_counters(self.h, out)
        return int(out[0])

    @property
    def stream(self) -> int:
        return self._L.cpsd_gpu_batch_stream(self.h) or 0

    def close(self) -> None:
        if getattr(self, "h", None):
            self._L.cpsd_gpu_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Mlp:
    """The preconditioner network on the GPU (forward, gradient, Adam training)."""

    def __init__(self, seed: int = 0):
        self._L = _l.load()
        h = ctypes.c_void_p()
        rc = self._L.cpsd_mlp_create(ctypes.c_ulonglong(seed), ctypes.byref(h))
        if rc:
            raise CpsdError(rc, "cpsd_mlp_create")
        self.h = h
        self.nparams = self._L.cpsd_mlp_nparams()

    def forward(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        y = np.zeros(X.shape[0], dtype=np.float32)
        rc = self._L.cpsd_mlp_forward(self.h, _ptr(X), X.shape[0], _ptr(y))
        if rc:
            raise CpsdError(rc, "cpsd_mlp_forward")
        return y

    def gradient(self, X: np.ndarray, T: np.ndarray):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        g = np.zeros(self.nparams, dtype=np.float32)
        loss = ctypes.c_float()
        rc = self._L.cpsd_mlp_gradient(self.h, _ptr(X), _ptr(T), X.shape[0], _ptr(g), ctypes.byref(loss))
        if rc:
            raise CpsdError(rc, "cpsd_mlp_gradient")
        return float(loss.value), g

    def train(self, X: np.ndarray, T: np.ndarray, steps: int, batch: int, lr: float) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        losses = np.zeros(steps, dtype=np.float32)
        rc = self._L.cpsd_mlp_train(self.h, _ptr(X), _ptr(T), X.shape[0], steps, batch, ctypes.c_float(lr),
                                    _ptr(losses))
        if rc:
            raise CpsdError(rc, "cpsd_mlp_train")
        return losses

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(self.nparams, dtype=np.float32)
        self._L.cpsd_mlp_get_params(self.h, _ptr(p))
        return p

    @params.setter
    def params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        rc = self._L.cpsd_mlp_set_params(self.h, _ptr(p))
        if rc:
            raise CpsdError(rc, "cpsd_mlp_set_params")

    def close(self) -> None:
        if getattr(self, "h", None):
            self._L.cpsd_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_elcout(path: str, inp, c1: np.ndarray) -> None:
    """ELCOUT as ccpsdv3/main.c:537-546 writes it (header, then c1)."""
    L = _l.load()
    ne = np.ascontiguousarray(inp.ne, dtype=np.int32)
    c1 = np.ascontiguousarray(c1, dtype=np.float64)
    if c1.size != int(ne.sum()) * inp.n2ft3d:
        raise ValueError("c1 must hold (ne0+ne1) * n2ft3d doubles")
    rc = L.cpsd_write_elcout(path.encode(), int(inp.spec.icube), int(inp.nfft), float(inp.spec.unit),
                             int(inp.ispin), _ptr(ne), _ptr(c1))
    if rc:
        raise CpsdError(rc, "cpsd_write_elcout")


def write_ionout(path: str, inp, fnames, r2: np.ndarray) -> None:
    """IONOUT as ccpsdv3/main.c:549-566 writes it; fnames are the psp file
    names of the kinds (as IONIN lists them)."""
    L = _l.load()
    species = inp.spec.species
    if len(fnames) != len(species):
        raise ValueError("one file name per kind")
    names = (ctypes.c_char_p * len(fnames))(*[f.encode() for f in fnames])
    lmax = np.array([sp.lmax for sp in species], dtype=np.int32)
    katm = np.ascontiguousarray(inp.katm, dtype=np.int32)
    r2 = np.ascontiguousarray(r2, dtype=np.float64)
    rc = L.cpsd_write_ionout(path.encode(), len(fnames), names, _ptr(lmax), int(inp.nion), _ptr(katm), _ptr(r2))
    if rc:
        raise CpsdError(rc, "cpsd_write_ionout")


def kbpp(table, G: np.ndarray, nfft3d: int):
    """Kleinman-Bylander tables on the half-box grid from a radial table
    (ckbppv3/dkbppv3.c kbpp(), on the GPU): returns (vl, vnl, vnlnrm, vp)
    with vp's nonlocal channels replaced by vp_l - vp_lmax, as kbpp() leaves
    them."""
    L = _l.load()
    lmax = int(table.lmax)
    vp = np.array(table.vp, dtype=np.float64)
    vl = np.zeros(nfft3d)
    vnl = np.zeros(max(lmax * lmax, 1) * nfft3d)
    vnlnrm = np.zeros(max(lmax * lmax, 1))
    rc = L.cpsd_gpu_kbpp(float(table.zv), lmax, int(table.nrho), float(table.drho),
                         _ptr(np.ascontiguousarray(table.rho, dtype=np.float64)), _ptr(vp),
                         _ptr(np.ascontiguousarray(table.wp, dtype=np.float64)), int(nfft3d),
                         _ptr(np.ascontiguousarray(G, dtype=np.float64)), _ptr(vl), _ptr(vnl), _ptr(vnlnrm))
    if rc:
        raise CpsdError(rc, "cpsd_gpu_kbpp")
    return vl, vnl[:lmax * lmax * nfft3d], vnlnrm[:lmax * lmax], vp


def makepsi(nfft: int, ispin: int, ne, waves) -> np.ndarray:
    """The initial plane-wave orbitals of cmakepsi/dmakepsi.c in the ELCIN
    layout; waves: the PSI0.DAT rows (i, j, k, l), at least ne[0] of them."""
    L = _l.load()
    ne = np.ascontiguousarray(ne, dtype=np.int32)
    w = np.ascontiguousarray(np.asarray(waves, dtype=np.int32)[:int(ne[0])].ravel())
    if w.size != 4 * int(ne[0]):
        raise ValueError("need ne[0] rows of (i, j, k, l)")
    psi = np.zeros((int(ne[0]) + (int(ne[1]) if ispin == 2 else 0)) * (nfft + 2) * nfft * nfft)
    rc = L.cpsd_makepsi(int(nfft), int(ispin), _ptr(ne), _ptr(w), _ptr(psi))
    if rc:
        raise CpsdError(rc, "cpsd_makepsi")
    return psi


def dropin_counters():
    """Counters of the context the drop-in cpsd() keeps between calls."""
    L = _l.load()
    h = L.cpsd_gpu_dropin_context()
    out = (ctypes.c_longlong * 3)()
    L.cpsd_gpu_counters(h, out)
    return int(out[0]), int(out[1]), int(out[2])


def _fft(fn, A: np.ndarray, nfft: int) -> None:
    assert A.dtype == np.float64 and A.flags.c_contiguous
    L = _l.load()
    i = lambda v: ctypes.byref(ctypes.c_int(v))  # noqa: E731
    nh = nfft // 2 + 1
    fn(_ptr(A), i(nh), i(nh * nfft), i(nfft + 2), i((nfft + 2) * nfft), i(nfft), i(nfft), i(nfft),
       None, i(0))
    rc = L.cpsd_gpu_fft_status()
    if rc:
        raise CpsdError(rc, "3-D FFT")


def cr_fft3b(A: np.ndarray, nfft: int) -> None:
    """In place: half box (complex) -> real (padded x lines), unnormalised."""
    _fft(_l.load().cr_fft3b_, A, nfft)


def rc_fft3f(A: np.ndarray, nfft: int) -> None:
    """In place: real (padded x lines) -> half box (complex), unnormalised."""
    _fft(_l.load().rc_fft3f_, A, nfft)


def overlap_tn(A, B, w=None, method: int = _l.CPSD_GEMM_FP64, out=None, stream=None):
    """C = A^T W B on device tensors (torch float64 CUDA tensors, rows of K
    reals with unit stride): C[i, j] = sum_k w[k // 2] A[i, k] B[j, k], the
    Gamma-point gcdotc of every row pair.  Returns C (M x N)."""
    import torch
    M, K = A.shape
    N = B.shape[0]
    for t in (A, B):
        if t.dtype != torch.float64 or not t.is_cuda or t.stride(1) != 1:
            raise ValueError("A and B must be float64 CUDA tensors with unit stride along K")
    if B.shape[1] != K:
        raise ValueError("A and B must have the same K")
    if out is None:
        out = torch.empty((M, N), dtype=torch.float64, device=A.device)
    s = stream if stream is not None else torch.cuda.current_stream(A.device).cuda_stream
    wp = None if w is None else w.data_ptr()
    rc = _l.load().cpsd_overlap_tn(int(method), M, N, K, A.data_ptr(), A.stride(0), B.data_ptr(), B.stride(0),
                                   wp, out.data_ptr(), out.stride(0), s)
    if rc != _l.CPSD_OK:
        raise CpsdError(rc, "cpsd_overlap_tn")
    return out
