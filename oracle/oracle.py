"""ORACLE / TEST INFRASTRUCTURE ONLY -- ctypes access to the CPU oracles.

* ``Restatement``  -- oracle/_build/liboracle.so, the project's plain-C
  restatement of ccpsdv3/cpsd.c (cpsd_oracle.c + fft3d.c).
* ``ReferenceBuild`` -- oracle/_ref/libcpsd_ref.so, the reference's own
  ccpsdv3/*.c compiled unmodified (oracle/Makefile target ``ref``).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  Both classes run the same state machine as the reference's
driver: ``run(inputs, inner, state)`` performs one ``cpsd()`` call and
updates ``state`` (c1, c2, cpsi, dn, hml, lmd, r1, r2, fion, E) in place.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "_build", "liboracle.so")
REFERENCE_SO = os.path.join(HERE, "_ref", "libcpsd_ref.so")

_P = ctypes.c_void_p


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_P)


def build_restatement() -> str:
    subprocess.run(["make", "-s", "-C", HERE, "restatement"], check=True)
    return RESTATEMENT_SO


class State:
    """Mutable arrays cpsd() reads and writes, sized like main.c:124-136."""

    def __init__(self, inp):
        nb = inp.nbands
        ne0 = int(inp.ne[0])
        ne1 = int(inp.ne[1])
        self.c2 = inp.c2.copy()
        self.c1 = inp.c2.copy()
        self.cpsi = np.zeros_like(inp.c2)
        self.dn = np.zeros(inp.ispin * inp.n2ft3d)
        self.hml = np.zeros(ne0 * ne0 + ne1 * ne1)
        self.lmd = np.zeros(ne0 * ne0 + ne1 * ne1)
        self.r2 = inp.r2.copy()
        self.r1 = inp.r2.copy()
        self.fion = np.zeros(3 * inp.nion)
        self.E = np.zeros(10)
        self.deltae = 0.0
        self.deltac = 0.0
        self.deltar = 0.0
        self.lagrange_fail = 0
        assert self.c2.size == nb * inp.n2ft3d


def _common_args(inp, inner: int, move: int):
    ne = np.ascontiguousarray(inp.ne, dtype=np.int32)
    return ne, [
        ctypes.c_int(inner), ctypes.c_int(move), ctypes.c_int(inp.nion), ctypes.c_int(inp.ispin),
        _ptr(ne), ctypes.c_int(inp.nfft), ctypes.c_int(inp.nfft3d), ctypes.c_int(inp.n2ft3d),
        _ptr(inp.unitg), ctypes.c_double(inp.omega), ctypes.c_double(inp.dt),
        ctypes.c_double(inp.fmass), _ptr(inp.katm), _ptr(inp.amass), _ptr(inp.zv),
        ctypes.c_int(inp.nsh), _ptr(inp.rcell), ctypes.c_double(inp.cewald),
        ctypes.c_double(inp.rcut), _ptr(inp.masker), _ptr(inp.G), _ptr(inp.tg), _ptr(inp.vc),
        _ptr(inp.vg), _ptr(inp.lmmax), _ptr(inp.vnlnrm), _ptr(inp.vl), _ptr(inp.vnl),
    ]


class _Bands(ctypes.Structure):
    """oracle_bands of oracle.h."""
    _fields_ = [("lo", ctypes.c_int), ("hi", ctypes.c_int), ("allreduce_sum", ctypes.c_void_p),
                ("allgather_rows", ctypes.c_void_p), ("user", ctypes.c_void_p)]

    def __init__(self, lo, hi, red, gat, user):
        super().__init__(lo, hi, ctypes.cast(red, ctypes.c_void_p), ctypes.cast(gat, ctypes.c_void_p), user)
        self._keep = (red, gat)


class Restatement:
    def __init__(self, path: str = RESTATEMENT_SO):
        if not os.path.exists(path):
            build_restatement()
        self.lib = ctypes.CDLL(path)
        self.lib.oracle_cpsd.restype = ctypes.c_int
        self.lib.oracle_gcdotc.restype = ctypes.c_double
        self.lib.oracle_gsdot.restype = ctypes.c_double
        self.lib.oracle_gssum.restype = ctypes.c_double

    def run(self, inp, inner: int, st: State, move: Optional[int] = None) -> State:
        move = inp.spec.move if move is None else move
        ne, args = _common_args(inp, inner, move)
        dd = [ctypes.c_double() for _ in range(3)]
        fail = ctypes.c_int()
        rc = self.lib.oracle_cpsd(*args, _ptr(st.r1), _ptr(st.r2), _ptr(st.fion), _ptr(st.c1),
                                  _ptr(st.c2), _ptr(st.cpsi), _ptr(st.dn), _ptr(st.hml),
                                  _ptr(st.lmd), _ptr(st.E), ctypes.byref(dd[0]),
                                  ctypes.byref(dd[1]), ctypes.byref(dd[2]), ctypes.byref(fail))
        if rc != 0:
            raise MemoryError("oracle_cpsd could not allocate scratch")
        st.deltae, st.deltac, st.deltar = dd[0].value, dd[1].value, dd[2].value
        st.lagrange_fail += fail.value
        return st

    def run_bands(self, inp, inner: int, st: State, lo: int, hi: int, allreduce_sum, allgather_rows) -> State:
        """The band-parallel form (oracle_cpsd_bands, move = 0): this rank
        steps bands [lo, hi); allreduce_sum(array) adds an array over the
        ranks in place and allgather_rows(array2d) fills every rank's rows
        of a (bands x row) array in place -- numpy views of the C buffers."""
        ne, args = _common_args(inp, inner, 0)
        del args[1]  # no move argument
        dd = [ctypes.c_double() for _ in range(3)]
        fail = ctypes.c_int()
        RED = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.c_long, ctypes.c_void_p)
        GAT = ctypes.CFUNCTYPE(None, ctypes.POINTER(ctypes.c_double), ctypes.c_long, ctypes.c_void_p)
        nb = inp.nbands
        red = RED(lambda p, n, u: allreduce_sum(np.ctypeslib.as_array(p, shape=(n,))))
        gat = GAT(lambda p, row, u: allgather_rows(np.ctypeslib.as_array(p, shape=(nb, row))))
        bp = _Bands(lo, hi, red, gat, None)
        rc = self.lib.oracle_cpsd_bands(*args, _ptr(st.r1), _ptr(st.r2), _ptr(st.fion), _ptr(st.c1),
                                        _ptr(st.c2), _ptr(st.cpsi), _ptr(st.dn), _ptr(st.hml),
                                        _ptr(st.lmd), _ptr(st.E), ctypes.byref(dd[0]),
                                        ctypes.byref(dd[1]), ctypes.byref(dd[2]), ctypes.byref(fail),
                                        ctypes.byref(bp))
        if rc != 0:
            raise ValueError("oracle_cpsd_bands: status %d" % rc)
        st.deltae, st.deltac, st.deltar = dd[0].value, dd[1].value, dd[2].value
        st.lagrange_fail += fail.value
        return st

    # FFT and helper entry points (same argument conventions as the reference)
    def cr_fft3b(self, A: np.ndarray, nfft: int) -> None:
        _fft(self.lib.cr_fft3b_, A, nfft)

    def rc_fft3f(self, A: np.ndarray, nfft: int) -> None:
        _fft(self.lib.rc_fft3f_, A, nfft)

    def gcdotc(self, nfft: int, a: np.ndarray, b: np.ndarray) -> float:
        return self.lib.oracle_gcdotc(ctypes.c_int(nfft), _ptr(a), _ptr(b))

    def xc(self, ispin: int, n2ft3d: int, dn: np.ndarray):
        xcp = np.zeros(ispin * n2ft3d)
        xce = np.zeros(n2ft3d)
        self.lib.oracle_xc(ctypes.c_int(ispin), ctypes.c_int(n2ft3d), _ptr(dn), _ptr(xcp), _ptr(xce))
        return xcp, xce


def _fft(fn, A: np.ndarray, nfft: int) -> None:
    assert A.dtype == np.float64 and A.flags.c_contiguous
    i = lambda v: ctypes.byref(ctypes.c_int(v))  # noqa: E731
    nh = nfft // 2 + 1
    fn(_ptr(A), i(nh), i(nh * nfft), i(nfft + 2), i((nfft + 2) * nfft), i(nfft), i(nfft), i(nfft),
       None, i(0))


KBPP_SO = os.path.join(HERE, "_ref", "libkbpp_ref.so")


def reference_kbpp(zv: float, lmax: int, rho: np.ndarray, vp: np.ndarray, wp: np.ndarray, drho: float,
                   G: np.ndarray, nfft3d: int, path: str = KBPP_SO):
    """The reference's own kbpp() (ckbppv3/dkbppv3.c, compiled unmodified into
    oracle/_ref/libkbpp_ref.so): returns (vl, vnl, vnlnrm, vp after the call)."""
    if not os.path.exists(path):
        raise FileNotFoundError(path + " (build with: make -C oracle ref)")
    lib = ctypes.CDLL(path)
    D = ctypes.c_double
    vp = np.array(vp, dtype=np.float64)
    lmmax = lmax * lmax
    vl = np.zeros(nfft3d)
    vnl = np.zeros(max(lmmax, 1) * nfft3d)
    vnlnrm = np.zeros(max(lmmax, 1))
    lib.kbpp(D(zv), ctypes.c_int(lmax), ctypes.c_int(len(rho)), D(drho),
             _ptr(np.ascontiguousarray(rho, dtype=np.float64)), _ptr(vp),
             _ptr(np.ascontiguousarray(wp, dtype=np.float64)), ctypes.c_int(nfft3d),
             _ptr(np.ascontiguousarray(G, dtype=np.float64)), _ptr(vl), _ptr(vnl), _ptr(vnlnrm))
    return vl, vnl[:lmmax * nfft3d], vnlnrm[:lmmax], vp


class ReferenceBuild:
    """The reference's own cpsd() (oracle/_ref/libcpsd_ref.so)."""

    def __init__(self, path: str = REFERENCE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path + " (build with: make -C oracle ref)")
        self.lib = ctypes.CDLL(path)
        self.lib.gcdotc.restype = ctypes.c_double
        self.lib.gssum.restype = ctypes.c_double

    @staticmethod
    def work_size(inp) -> int:
        """cpsdwork length, main.c:317-320 (+nion for dti when move, cpsd.c:119)."""
        ne0 = int(inp.ne[0])
        return ((6 + inp.ispin) * inp.n2ft3d + inp.nion * (5 * inp.nfft + 3) + 7 * ne0 * ne0)

    def run(self, inp, inner: int, st: State, move: Optional[int] = None) -> State:
        move = inp.spec.move if move is None else move
        ne, args = _common_args(inp, inner, move)
        work = np.zeros(self.work_size(inp))
        dd = [ctypes.c_double() for _ in range(3)]
        self.lib.cpsd(*args, _ptr(st.r1), _ptr(st.r2), _ptr(st.fion), _ptr(st.c1), _ptr(st.c2),
                      _ptr(st.cpsi), _ptr(st.dn), _ptr(st.hml), _ptr(st.lmd), _ptr(work),
                      _ptr(st.E), ctypes.byref(dd[0]), ctypes.byref(dd[1]), ctypes.byref(dd[2]))
        st.deltae, st.deltac, st.deltar = dd[0].value, dd[1].value, dd[2].value
        return st

    def cr_fft3b(self, A: np.ndarray, nfft: int) -> None:
        _fft(self.lib.cr_fft3b_, A, nfft)

    def rc_fft3f(self, A: np.ndarray, nfft: int) -> None:
        _fft(self.lib.rc_fft3f_, A, nfft)

    def get_g(self, nfft: int, unitg: np.ndarray) -> np.ndarray:
        nh = nfft // 2 + 1
        G = np.zeros(3 * nh * nfft * nfft)
        self.lib.get_g(ctypes.c_int(nfft), _ptr(unitg), _ptr(G))
        return G

    def get_masker(self, nfft: int, ggcut: float, unitg: np.ndarray) -> np.ndarray:
        nh = nfft // 2 + 1
        m = np.zeros(nh * nfft * nfft, dtype=np.int32)
        self.lib.get_masker(ctypes.c_int(nfft), ctypes.c_double(ggcut), _ptr(unitg), _ptr(m))
        return m

    def get_cube(self, icube: int, unit: float):
        vol = ctypes.c_double()
        unita = np.zeros(9)
        unitg = np.zeros(9)
        self.lib.get_cube(ctypes.c_int(icube), ctypes.c_double(unit), ctypes.byref(vol),
                          _ptr(unita), _ptr(unitg))
        return vol.value, unita, unitg

    def gssum(self, nfft: int, x: np.ndarray) -> float:
        return self.lib.gssum(ctypes.c_int(nfft), _ptr(x))

    def gcdotc(self, nfft: int, a: np.ndarray, b: np.ndarray) -> float:
        return self.lib.gcdotc(ctypes.c_int(nfft), _ptr(a), _ptr(b))

    def eigsrt(self, D: np.ndarray, V: np.ndarray, n: int) -> None:
        """The reference's eigsrt (ccpsdv3/eigsrt.c:9-36) in place; V column-major, ld n."""
        self.lib.eigsrt(_ptr(D), _ptr(V), ctypes.c_int(n))


def eigsrt(D: np.ndarray, V: np.ndarray) -> None:
    """ccpsdv3/eigsrt.c:9-36 restated: selection sort into descending order,
    ties to the later index; V[:, i] (eigenvector i) moves with D[i]."""
    n = len(D)
    for i in range(n - 1):
        k, p = i, D[i]
        for j in range(i + 1, n):
            if D[j] >= p:
                k, p = j, D[j]
        if k != i:
            D[k] = D[i]
            D[i] = p
            V[:, [i, k]] = V[:, [k, i]]


def epilogue(inp, st: State, gcdotc, sort=eigsrt, matmul=None) -> dict:
    """ccpsdv3/main.c:452-487 restated on a State after the last cpsd() call:

    * ``ortho``: <c1_i|c1_j> (gcdotc, main.c:455-467), per spin in hml's layout;
    * ``eig``, ``vec``: dsyev('V','U') of hml per spin (LAPACK, via scipy)
      then eigsrt (main.c:470-479): eig[ms*ne0 + i] descending, vec in hml's
      layout (column-major, ld ne[ms]);
    * ``c1``: c2 V per spin (main.c:481-487), the orbitals ELCOUT holds.

    ``gcdotc(nfft, a, b)`` is an oracle's Gamma-point dot; ``sort(D, V)``
    orders the eigenpairs (V as an array, column i = vector i); ``matmul(C2, V)``
    returns C2 @ V for C2 of shape (n2ft3d, m) (numpy by default)."""
    from scipy.linalg import lapack
    ne = [int(inp.ne[0]), int(inp.ne[1])]
    ne0 = ne[0]
    n2 = inp.n2ft3d
    ortho = np.zeros(ne[0] ** 2 + ne[1] ** 2)
    vec = np.zeros_like(ortho)
    eig = np.zeros(ne[0] + ne[1])
    c1 = np.zeros_like(st.c2)
    for ms in range(inp.ispin):
        m, b0 = ne[ms], ms * ne0
        o = ms * ne0 * ne0
        for i in range(m):
            for j in range(i, m):
                w = gcdotc(inp.nfft, st.c1[(b0 + i) * n2:(b0 + i + 1) * n2], st.c1[(b0 + j) * n2:(b0 + j + 1) * n2])
                ortho[o + i + j * m] = ortho[o + j + i * m] = w
        H = st.hml[o:o + m * m].reshape(m, m).T  # H[i, j] = hml[i + j*m]
        w, v, info = lapack.dsyev(np.array(H, order="F"), compute_v=1, lower=0)
        assert info == 0
        D = np.array(w)
        V = np.array(v)
        sort(D, V)
        eig[ms * ne0:ms * ne0 + m] = D
        vec[o:o + m * m] = V.T.ravel()  # column-major
        C2 = st.c2[b0 * n2:(b0 + m) * n2].reshape(m, n2).T
        C1 = matmul(C2, V) if matmul else C2 @ V
        c1[b0 * n2:(b0 + m) * n2] = C1.T.ravel()
    return {"ortho": ortho, "eig": eig, "vec": vec, "c1": c1}


def simp(f: np.ndarray, h: float) -> np.ndarray:
    """simp() of ckbppv3/dkbppv3.c along the last axis:
    h/3 (2 sum_even f + 4 sum_odd f - f_0 - f_{n-1})."""
    s = 2.0 * f[..., 0::2].sum(axis=-1) + 4.0 * f[..., 1::2].sum(axis=-1) - f[..., 0] - f[..., -1]
    return s * (h / 3.0)


def kbpp(zv: float, lmax: int, rho: np.ndarray, vp: np.ndarray, wp: np.ndarray, drho: float,
         G: np.ndarray, nfft3d: int, chunk: int = 2048):
    """kbpp() of ckbppv3/dkbppv3.c (kbppv3.c:335-444) restated with numpy:
    returns (vl, vnl, vnlnrm, vp with its nonlocal channels minus the local one)."""
    n = len(rho)
    vp = np.array(vp, dtype=np.float64).reshape(lmax + 1, n)
    wp = np.asarray(wp, dtype=np.float64).reshape(lmax + 1, n)
    for l in range(lmax):
        vp[l] -= vp[lmax]
    lmmax = lmax * lmax
    vnlnrm = np.zeros(lmmax)
    for l in range(lmax):
        vnlnrm[l * l:(l + 1) * (l + 1)] = simp(vp[l] * wp[l] * wp[l], drho)
    fourpi = 4.0 * np.pi
    p0, p1, p2 = np.sqrt(fourpi), np.sqrt(3.0 * fourpi), np.sqrt(15.0 * fourpi)
    vl = np.zeros(nfft3d)
    vnl = np.zeros((lmmax, nfft3d))
    G = np.asarray(G).reshape(3, nfft3d)
    for k0 in range(1, nfft3d, chunk):
        k = np.arange(k0, min(nfft3d, k0 + chunk))
        g = G[:, k]
        q = np.sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2])
        gx, gy, gz = g[0] / q, g[1] / q, g[2] / q
        x = q[:, None] * rho[None, :]
        sn, cs = np.sin(x), np.cos(x)
        if lmax > 2:
            a = 3.0 * (sn / x - cs) / x - sn
            f = a * wp[2] * vp[2]
            f[:, 0] = 0.0
            d = p2 * simp(f, drho) / q
            vnl[4, k] = d * (3.0 * gz * gz - 1.0) / (2.0 * np.sqrt(3.0))
            vnl[5, k] = d * gx * gy
            vnl[6, k] = d * gy * gz
            vnl[7, k] = d * gz * gx
            vnl[8, k] = d * (gx * gx - gy * gy) / 2.0
        if lmax > 1:
            f = (sn / x - cs) * wp[1] * vp[1]
            f[:, 0] = 0.0
            p = p1 * simp(f, drho) / q
            vnl[1, k], vnl[2, k], vnl[3, k] = p * gx, p * gy, p * gz
        if lmax > 0:
            vnl[0, k] = p0 * simp(sn * wp[0] * vp[0], drho) / q
        vl[k] = simp(rho * vp[lmax] * sn, drho) * fourpi / q - zv * fourpi * cs[:, -1] / (q * q)
    vl[0] = fourpi * simp(vp[lmax] * (rho * rho), drho) + 2.0 * np.pi * zv * rho[-1] * rho[-1]
    if lmax > 0:
        vnl[0, 0] = p0 * simp(rho * wp[0] * vp[0], drho)
    return vl, vnl.ravel(), vnlnrm, vp.ravel()


def makepsi(nfft: int, ispin: int, ne, waves) -> np.ndarray:
    """cmakepsi/dmakepsi.c:93-140 restated: one plane wave per band (PSI0.DAT
    rows i j k l), its Hermitian partner on the kx = 0 plane; spin 1 reuses
    the first ne[1] rows."""
    nh = nfft // 2 + 1
    nfft3 = (nfft + 2) * nfft * nfft
    s = 1.0 / np.sqrt(2.0)
    bands = []
    for ms in range(ispin):
        for n in range(int(ne[ms])):
            i, j, k, l = (int(v) for v in waves[n])
            c = (0.0, s) if l < 0 else ((1.0, 0.0) if l == 0 else (s, 0.0))
            b = np.zeros(nfft3)
            k2, k3 = (j + nfft) % nfft, (k + nfft) % nfft
            idx = 2 * (i + k2 * nh + k3 * nh * nfft)
            b[idx], b[idx + 1] = c
            if i == 0:
                idx = 2 * (((nfft - k2) % nfft) * nh + ((nfft - k3) % nfft) * nh * nfft)
                b[idx], b[idx + 1] = c[0], -c[1]
            bands.append(b)
    return np.concatenate(bands)
