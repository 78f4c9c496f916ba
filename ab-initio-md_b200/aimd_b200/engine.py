"""
Device engine: one native context per basis structure, re-targeted to each
new geometry. Owns nothing but the context handle; device memory for the
inputs and outputs of each call comes from torch (the caller's tensors).

Layout sent to the device:
  * contraction blocks (the reference's BasisSet.blk_*, aimd/qc/basis.py:
    185-228), with blocks whose contraction count exceeds the kernel cap
    (2 for s, 1 otherwise) split into consecutive smaller blocks; the
    coefficient matrix is [nprim][2] with zeros for unused columns;
  * segmented shells for the one-electron kernels.
Pairs are block index i(i+1)/2 + j for i >= j; without splitting they are
exactly the reference's pair indices.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .basis import BasisSet


def _ncon_cap(l: int) -> int:
    return 2 if l == 0 else 1


def device_blocks(basis: BasisSet) -> dict:
    """Block arrays for the device, splitting over-cap general contractions."""
    atom, lval, ncon, ao, p0, npr, exps, coefs, orig = [], [], [], [], [], [], [], [], []
    split = False
    for b in range(basis.nblock):
        l = int(basis.blk_l[b])
        nc = int(basis.blk_ncon[b])
        k0, k1 = int(basis.blk_prim[b]), int(basis.blk_prim[b + 1])
        cap = _ncon_cap(l)
        nct = (l + 1) * (l + 2) // 2
        for c0 in range(0, nc, cap):
            cols = list(range(c0, min(nc, c0 + cap)))
            if len(cols) < nc:
                split = True
            rows = [k for k in range(k0, k1) if any(basis.blk_coef[k, c] != 0.0 for c in cols)] if len(cols) < nc \
                else list(range(k0, k1))
            atom.append(int(basis.blk_atom[b]))
            orig.append(b)
            lval.append(l)
            ncon.append(len(cols))
            ao.append(int(basis.blk_ao[b]) + c0 * nct)
            p0.append(len(exps))
            npr.append(len(rows))
            for k in rows:
                exps.append(float(basis.blk_exp[k]))
                coefs.append([float(basis.blk_coef[k, c]) for c in cols] + [0.0] * (2 - len(cols)))
    i32 = lambda v: np.ascontiguousarray(np.array(v, dtype=np.int32))  # noqa: E731
    return {"atom": i32(atom), "l": i32(lval), "ncon": i32(ncon), "ao": i32(ao), "p0": i32(p0), "np": i32(npr),
            "exp": np.ascontiguousarray(np.array(exps, dtype=float)),
            "coef": np.ascontiguousarray(np.array(coefs, dtype=float).reshape(-1, 2)), "split": split,
            "orig": np.array(orig, dtype=np.int64)}


def _p32(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _p64(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class Engine:
    """Native context for one basis structure (any geometry)."""

    def __init__(self, basis: BasisSet, device: torch.device | None = None) -> None:
        if not torch.cuda.is_available():
            raise RuntimeError("aimd_b200 needs a CUDA device; none is visible")
        self.lib = _lib.load()
        self.device = torch.device(device or "cuda")
        self.natm, self.nao = basis.natm, basis.nao
        blk = device_blocks(basis)
        self.blocks = blk
        self.nblock = len(blk["l"])
        self.split = blk["split"]
        sh_np = np.diff(basis.shell_prim).astype(np.int32)
        self._keep = {
            "sh_atom": np.ascontiguousarray(basis.shell_atom.astype(np.int32)),
            "sh_l": np.ascontiguousarray(basis.shell_l.astype(np.int32)),
            "sh_ao": np.ascontiguousarray(basis.shell_ao[:-1].astype(np.int32)),
            "sh_p0": np.ascontiguousarray(basis.shell_prim[:-1].astype(np.int32)),
            "sh_np": np.ascontiguousarray(sh_np),
            "sh_exp": np.ascontiguousarray(basis.prim_exp.astype(float)),
            "sh_coef": np.ascontiguousarray(basis.prim_coef.astype(float)),
            "charges": np.ascontiguousarray(basis.nuclear_charges.astype(float)),
        }
        k = self._keep
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self.lib.aimd_create(
                ctypes.byref(h), self.natm, self.nao, self.nblock, _p32(blk["atom"]), _p32(blk["l"]),
                _p32(blk["ncon"]), _p32(blk["ao"]), _p32(blk["p0"]), _p32(blk["np"]), len(blk["exp"]),
                _p64(blk["exp"]), _p64(blk["coef"]), basis.nshell, _p32(k["sh_atom"]), _p32(k["sh_l"]),
                _p32(k["sh_ao"]), _p32(k["sh_p0"]), _p32(k["sh_np"]), len(k["sh_exp"]), _p64(k["sh_exp"]),
                _p64(k["sh_coef"]), _p64(k["charges"])), "aimd_create")
        self.handle = h
        self.npair = self.lib.aimd_pair_count(h)
        self._pos_key: bytes | None = None
        self.pos = torch.zeros((self.natm, 3), dtype=torch.float64, device=self.device)
        self._fp32_cutoff = 0.0

    def _precision(self, fp32_cutoff: float) -> None:
        """Quartets with Q1 Q2 < fp32_cutoff run in FP32 in the next calls (0: all FP64)."""
        c = float(fp32_cutoff)
        if c != self._fp32_cutoff:
            _lib.check(self.lib.aimd_set_fp32_cutoff(self.handle, c), "aimd_set_fp32_cutoff")
            self._fp32_cutoff = c

    def __del__(self) -> None:
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.aimd_destroy(h)
            except Exception:
                pass
            self.handle = None

    # ------------------------------------------------------------ geometry
    def set_geometry(self, positions) -> None:
        """Move to new positions (bohr); a no-op if they did not change."""
        if isinstance(positions, torch.Tensor):
            x = positions.detach().to(self.device, torch.float64).reshape(self.natm, 3)
            key = x.cpu().numpy().tobytes()
        else:
            arr = np.array(positions, dtype=float).reshape(self.natm, 3)
            key = arr.tobytes()
            x = torch.from_numpy(arr).to(self.device)
        if key == self._pos_key:
            return
        self.pos.copy_(x)
        _lib.check(self.lib.aimd_set_geometry(self.handle, ctypes.c_void_p(self.pos.data_ptr()), _stream()),
                   "aimd_set_geometry")
        self._pos_key = key

    # ------------------------------------------------------------ two-electron
    def schwarz(self) -> torch.Tensor:
        Q = torch.empty(self.npair, dtype=torch.float64, device=self.device)
        _lib.check(self.lib.aimd_schwarz(self.handle, ctypes.c_void_p(Q.data_ptr()), _stream()), "aimd_schwarz")
        return Q

    def jk_acc(self, D: torch.Tensor, thr: float, fp32_cutoff: float = 0.0) -> tuple[torch.Tensor, torch.Tensor]:
        """Un-symmetrised J/K accumulators for symmetric densities D[nset, n, n]."""
        self._precision(fp32_cutoff)
        D = D.contiguous()
        J = torch.empty_like(D)
        K = torch.empty_like(D)
        _lib.check(self.lib.aimd_jk(self.handle, D.shape[0], ctypes.c_void_p(D.data_ptr()),
                                    ctypes.c_void_p(J.data_ptr()), ctypes.c_void_p(K.data_ptr()), float(thr),
                                    _stream()), "aimd_jk")
        return J, K

    def jk_delta_acc(self, dD: torch.Tensor, thr: float, dthr: float,
                     fp32_cutoff: float = 0.0) -> tuple[torch.Tensor, torch.Tensor]:
        """Accumulators of J/K for difference densities with density-weighted screening."""
        self._precision(fp32_cutoff)
        dD = dD.contiguous()
        J = torch.empty_like(dD)
        K = torch.empty_like(dD)
        _lib.check(self.lib.aimd_jk_delta(self.handle, dD.shape[0], ctypes.c_void_p(dD.data_ptr()),
                                          ctypes.c_void_p(J.data_ptr()), ctypes.c_void_p(K.data_ptr()), float(thr),
                                          float(dthr), _stream()), "aimd_jk_delta")
        return J, K

    def eri_tensor(self, thr: float) -> torch.Tensor:
        self._precision(0.0)
        n = self.nao
        eri = torch.empty((n, n, n, n), dtype=torch.float64, device=self.device)
        _lib.check(self.lib.aimd_eri_tensor(self.handle, ctypes.c_void_p(eri.data_ptr()), float(thr), _stream()),
                   "aimd_eri_tensor")
        return eri

    def grad2e(self, Dc: torch.Tensor, Dx: torch.Tensor, kfac: float, thr: float, gamma_bound: float,
               fp32_cutoff: float = 0.0) -> torch.Tensor:
        self._precision(fp32_cutoff)
        Dc = Dc.contiguous()
        Dx = Dx.contiguous()
        g = torch.empty((self.natm, 3), dtype=torch.float64, device=self.device)
        _lib.check(self.lib.aimd_grad2e(self.handle, ctypes.c_void_p(Dc.data_ptr()), Dx.shape[0],
                                        ctypes.c_void_p(Dx.data_ptr()), float(kfac), float(thr), float(gamma_bound),
                                        ctypes.c_void_p(g.data_ptr()), _stream()), "aimd_grad2e")
        return g

    # ------------------------------------------------------------ one-electron
    def onee(self, origin=None):
        n = self.nao
        dev = self.device
        S = torch.empty((n, n), dtype=torch.float64, device=dev)
        T = torch.empty_like(S)
        V = torch.empty_like(S)
        M = torch.empty((3, n, n), dtype=torch.float64, device=dev)
        o = np.zeros(3) if origin is None else np.ascontiguousarray(np.asarray(origin, dtype=float).reshape(3))
        _lib.check(self.lib.aimd_onee(self.handle, _p64(o), ctypes.c_void_p(S.data_ptr()),
                                      ctypes.c_void_p(T.data_ptr()), ctypes.c_void_p(M.data_ptr()),
                                      ctypes.c_void_p(V.data_ptr()), _stream()), "aimd_onee")
        return S, T, M, V

    def onee_grad(self, W: torch.Tensor, D: torch.Tensor) -> torch.Tensor:
        """d/dR [sum W S + sum D (T + V)]."""
        W = W.contiguous()
        D = D.contiguous()
        g = torch.zeros((self.natm, 3), dtype=torch.float64, device=self.device)
        _lib.check(self.lib.aimd_onee_grad(self.handle, ctypes.c_void_p(W.data_ptr()), ctypes.c_void_p(D.data_ptr()),
                                           ctypes.c_void_p(g.data_ptr()), _stream()), "aimd_onee_grad")
        return g

    # ------------------------------------------------------------ launch shape
    DEFAULT_SHAPES = ((8, 32), (4, 32), (16, 32), (8, 16), (8, 64))

    @property
    def launch_shape(self) -> tuple[int, int]:
        """(work-plan chunks per resident CTA, primitive quartets per split column item)."""
        c, q = ctypes.c_int(), ctypes.c_int()
        _lib.check(self.lib.aimd_get_launch_shape(self.handle, ctypes.byref(c), ctypes.byref(q)),
                   "aimd_get_launch_shape")
        return int(c.value), int(q.value)

    def set_launch_shape(self, chunks_per_cta: int, item_pq: int) -> None:
        _lib.check(self.lib.aimd_set_launch_shape(self.handle, int(chunks_per_cta), int(item_pq)),
                   "aimd_set_launch_shape")

    def autotune(self, D: torch.Tensor, thr: float, grad: tuple | None = None, shapes=None,
                 jk_weight: float = 10.0, reps: int = 2, fp32_cutoff: float = 0.0) -> dict:
        """
        Pick the launch shape of this context by timing, at the current
        geometry: for every candidate (chunks per resident CTA, quartets per
        split item) one warm J/K build of the densities D[nset, n, n] and,
        if ``grad = (Dc, Dx, kfac, thr, gamma_bound)`` is given, one
        two-electron gradient, timed with CUDA events on the current stream
        (best of ``reps``); the score is jk_weight x J/K time + gradient
        time (an MD step runs about ten Fock builds per gradient). Sets and
        returns the fastest shape with every candidate's timings.
        """
        shapes = tuple(shapes or self.DEFAULT_SHAPES)
        if not shapes:
            raise ValueError("autotune: no candidate launch shapes")
        start = self.launch_shape

        def timed(fn) -> float:
            best = float("inf")
            for _ in range(reps):
                s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                s.record()
                fn()
                e.record()
                e.synchronize()
                best = min(best, s.elapsed_time(e))
            return best

        results = []
        try:
            for shape in shapes:
                self.set_launch_shape(*shape)
                self.jk_acc(D, thr, fp32_cutoff)                  # warm-up at this shape
                t_jk = timed(lambda: self.jk_acc(D, thr, fp32_cutoff))
                t_g = timed(lambda: self.grad2e(*grad, fp32_cutoff=fp32_cutoff)) if grad is not None else 0.0
                results.append({"shape": tuple(shape), "jk_ms": t_jk, "grad_ms": t_g,
                                "score": jk_weight * t_jk + t_g})
        except Exception:
            self.set_launch_shape(*start)
            raise
        best = min(results, key=lambda r: r["score"])
        self.set_launch_shape(*best["shape"])
        return {"shape": best["shape"], "candidates": results}

    # ------------------------------------------------------------ inspection
    def quartet_counts(self, which: int = 0) -> np.ndarray:
        out = np.zeros(36, dtype=np.int64)
        _lib.check(self.lib.aimd_quartet_counts(self.handle, which, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))),
                   "aimd_quartet_counts")
        return out.reshape(6, 6)

    def pair_data(self):
        npp = np.zeros(self.npair, dtype=np.int32)
        cls = np.zeros(self.npair, dtype=np.int32)
        srt = np.zeros(self.npair, dtype=np.int32)
        _lib.check(self.lib.aimd_pair_data(self.handle, _p32(npp), _p32(cls), _p32(srt)), "aimd_pair_data")
        return npp, cls, srt

    def launch_count(self) -> int:
        return int(self.lib.aimd_launch_count(self.handle))


def engine_for(basis: BasisSet) -> Engine:
    """The engine shared by every geometry of this basis (BasisSet.with_positions copies it)."""
    eng = basis._shared.get("engine")
    if eng is None:
        eng = Engine(basis)
        basis._shared["engine"] = eng
    eng.set_geometry(basis.positions)
    return eng
