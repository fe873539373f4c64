"""DF integral engine: device-resident bases, pair tables and class task lists.

``DFEngine`` owns everything the Rys kernels of ``libdfb.so`` read for one
(AO basis, aux basis) pair and exposes

* ``metric()``      -> V[P,Q] = (P|Q)                     (naux, naux)
* ``int3c(layout)`` -> X = (mu nu|P) as 'Qmn' (naux,nao,nao) or 'mnQ' (nao,nao,naux)
* ``deriv3c(bar)``  -> sum bar . d(mu nu|P)/dR  accumulated into grad (natm, 3)
* ``deriv2c(bar)``  -> sum bar . d(P|Q)/dR      accumulated into grad (natm, 3)

and the reference's DF-build seams as module functions with the same names and
argument meaning (``asuka/cueri/df.py:803,859,946,994``,
``asuka/integrals/cueri_df.py:33-133``): ``metric_2c2e_basis``,
``int3c2e_basis``, ``cholesky_metric``, ``whiten_3c2e``,
``build_df_B_from_cueri_packed_bases``.

Task enumeration follows the reference's unscreened DF build (every l-ordered
AO shell pair times every aux shell, ``asuka/cueri/gpu.py:1833-1834``; metric
over unordered aux pairs oriented l(P) >= l(Q), ``gpu.py:1590-1706``); the
tasks of one angular class go to the device as a (pairs x aux shells) grid.
"""

from __future__ import annotations

import ctypes
import functools
import os
import weakref

import numpy as np
import torch

from . import _lib
from . import linalg as _la
from .basis import BasisCartSoA, build_shell_pairs_l_order, from_reference_like, ncart

_DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
_TABLE_READY: set[int] = set()
PRIM_SCREEN = 1e-20  # primitive-pair magnitude bound below which a pair is skipped (0 = evaluate all)
NSTREAMS = int(os.environ.get("DFB_STREAMS", "8"))  # side streams for per-class launches (2/4/6/8 measured: 8 fastest)
NROOTS_SLOTS = 11  # DFB_NROOTS_MAX + 1
_SIDE_STREAMS: dict[int, list] = {}


class ScratchHolder:
    """Device scratch for the generic kernels, shared by engines that run one after another
    on the same streams (a batch of molecules): one buffer, grown to the largest need."""

    def __init__(self):
        self.t: torch.Tensor | None = None

    def get(self, need: int, device) -> torch.Tensor:
        if self.t is None or self.t.numel() < need:
            self.t = None
            self.t = torch.empty(need, dtype=torch.float64, device=device)
        return self.t[:need]


@functools.lru_cache(maxsize=1)
def _rys_table_host():
    with np.load(os.path.join(_DATA, "rys_table.npz")) as z:
        nmax, tmax, nint, deg = z["meta"]
        nmax, nint, deg = int(nmax), int(nint), int(deg)
        coefs, herms = [], []
        offs = np.zeros(NROOTS_SLOTS, dtype=np.int32)
        hoffs = np.zeros(NROOTS_SLOTS, dtype=np.int32)
        o = h = 0
        for n in range(1, nmax + 1):
            c = np.ascontiguousarray(z[f"coef{n}"], dtype=np.float64).ravel()
            w = np.ascontiguousarray(z[f"herm{n}"], dtype=np.float64).ravel()
            offs[n], hoffs[n] = o, h
            coefs.append(c)
            herms.append(w)
            o += c.size
            h += w.size
    return np.concatenate(coefs), offs, np.concatenate(herms), hoffs, nmax, nint, deg, float(tmax)


def ensure_rys_table(device: torch.device) -> None:
    """Upload the Rys node/weight table to ``device`` once per process."""
    idx = torch.device(device).index
    idx = torch.cuda.current_device() if idx is None else idx
    if idx in _TABLE_READY:
        return
    coef, offs, herm, hoffs, nmax, nint, deg, tmax = _rys_table_host()
    L = _lib.lib()
    with torch.cuda.device(idx):
        rc = L.dfb_rys_table_init(coef.ctypes.data, offs.ctypes.data, coef.size, herm.ctypes.data, hoffs.ctypes.data,
                                  herm.size, nmax, nint, deg, tmax)
    _lib.check(rc, "dfb_rys_table_init")
    _TABLE_READY.add(idx)


PREC_FP64, PREC_MIXED = 0, 1  # DFB_PREC_FP64 / DFB_PREC_MIXED of include/dfb.h
PREC_ALL_MIXED = -1  # 'mixed_all': every class in FP32 (measurement of the per-class errors)


def _prec_code(precision: str) -> int:
    """'fp64' -> DFB_PREC_FP64; 'mixed' -> DFB_PREC_MIXED for the classes the precision table
    admits (FP64 for the others); 'mixed_all' -> DFB_PREC_MIXED for every class."""
    if precision == "fp64":
        return PREC_FP64
    if precision == "mixed":
        return PREC_MIXED
    if precision == "mixed_all":
        return PREC_ALL_MIXED
    raise ValueError(f"precision must be 'fp64', 'mixed' or 'mixed_all', got {precision!r}")


@functools.lru_cache(maxsize=1)
def mixed_class_table() -> dict:
    """Angular classes whose FP32-component kernels the mixed mode uses, per kind ('int3c',
    'deriv3c', 'deriv2c'), as sets of (la, lb, lc).  Written by ``asuka_b200.tune_precision``
    from the measured first-order energy and gradient errors of every class (FP32 against FP64
    kernels); classes not listed run in FP64 in mixed mode too."""
    p = os.path.join(_DATA, "class_precision.json")
    if not os.path.exists(p):
        return {}
    import json

    with open(p) as f:
        t = json.load(f)
    return {k: {tuple(int(v) for v in c) for c in t.get(k, [])} for k in ("int3c", "deriv3c", "deriv2c")}


def _class_prec(code: int, kind: str, la: int, lb: int, lc: int) -> int:
    if code == PREC_FP64:
        return PREC_FP64
    if code == PREC_ALL_MIXED:
        return PREC_MIXED
    return PREC_MIXED if (la, lb, lc) in mixed_class_table().get(kind, ()) else PREC_FP64


def _stream() -> int:
    return int(torch.cuda.current_stream().cuda_stream)


def _as_soa(b) -> BasisCartSoA:
    return b if isinstance(b, BasisCartSoA) else from_reference_like(b)


class DFEngine:
    """Device-side state of the DF Rys integrals for one (AO, aux) basis pair."""

    def __init__(self, ao_basis, aux_basis, device=None, atom_coords_bohr: np.ndarray | None = None,
                 prim_screen: float = PRIM_SCREEN, scratch: ScratchHolder | None = None):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if self.device.type != "cuda":
            raise RuntimeError("DFEngine runs on CUDA devices only (no CPU fallback)")
        ensure_rys_table(self.device)
        ao = _as_soa(ao_basis)
        aux = _as_soa(aux_basis)
        if ao.shell_atom is None or aux.shell_atom is None:
            if atom_coords_bohr is None:
                raise ValueError("bases without shell->atom maps need atom_coords_bohr")
            from .basis import shell_to_atom_map

            ao = from_reference_like(ao, shell_to_atom_map(ao, atom_coords_bohr))
            aux = from_reference_like(aux, shell_to_atom_map(aux, atom_coords_bohr))
        self.ao, self.aux = ao, aux
        self.nao, self.naux = ao.nao, aux.nao
        self.natm = int(max(ao.shell_atom.max(initial=-1), aux.shell_atom.max(initial=-1))) + 1
        self.prim_screen = float(prim_screen)
        if ao.lmax > 8 or aux.lmax > 8:
            raise NotImplementedError("shells with l > 8 are not supported")
        dev = self.device
        i32 = self._i32
        f64 = self._f64

        # ---- AO side: basis arrays and l-ordered shell pairs
        self.sp = build_shell_pairs_l_order(ao)
        self.ao_cxyz = f64(ao.shell_cxyz)
        self.ao_pstart = i32(ao.shell_prim_start)
        self.ao_nprim = i32(ao.shell_nprim)
        self.ao_exp = f64(ao.prim_exp)
        self.ao_coef = f64(ao.prim_coef)
        self.ao_aostart = i32(ao.shell_ao_start)
        self.ao_atom = i32(ao.shell_atom)
        self.sp_A = i32(self.sp.sp_A)
        self.sp_B = i32(self.sp.sp_B)

        # ---- aux side: basis arrays and (P, dummy) self-pair tables for the metric
        self.ax_cxyz = f64(aux.shell_cxyz)
        self.ax_pstart = i32(aux.shell_prim_start)
        self.ax_nprim = i32(aux.shell_nprim)
        self.ax_exp = f64(aux.prim_exp)
        self.ax_coef = f64(aux.prim_coef)
        self.ax_rexp = f64(1.0 / np.asarray(aux.prim_exp, dtype=np.float64))
        self.ax_aostart = i32(aux.shell_ao_start)
        self.ax_atom = i32(aux.shell_atom)
        self.ax_self = i32(np.arange(aux.nshell, dtype=np.int32))
        self.ax_pp_sp = i32(np.repeat(np.arange(aux.nshell, dtype=np.int32), aux.shell_nprim))
        self.axpt = torch.empty((7, max(int(aux.shell_nprim.sum()), 1)), dtype=torch.float64, device=dev)
        self.ps_aux = _lib.PairSide(
            *[_lib.ptr(t) for t in (self.ax_self, self.ax_self, self.ax_pstart, self.ax_nprim, *self.axpt,
                                    self.ax_cxyz, self.ax_aostart, self.ax_atom)], 1)
        self.axs = _lib.AuxSide(*[_lib.ptr(t) for t in (self.ax_cxyz, self.ax_pstart, self.ax_nprim, self.ax_exp,
                                                        self.ax_coef, self.ax_rexp, self.ax_aostart, self.ax_atom)])
        aux_l = aux.shell_l
        self.aux_by_l = {}
        for l in np.unique(aux_l):
            idx = np.nonzero(aux_l == l)[0]
            idx = idx[np.argsort(-aux.shell_nprim[idx], kind="stable")]
            self.aux_by_l[int(l)] = i32(idx)
        # metric classes: unordered aux pairs oriented l(P) >= l(Q)
        self.classes2c = []
        nsh = aux.nshell
        Pi, Qi = np.tril_indices(nsh)
        lp, lq = aux_l[Pi], aux_l[Qi]
        swap = lp < lq
        P = np.where(swap, Qi, Pi)
        Q = np.where(swap, Pi, Qi)
        lP, lQ = aux_l[P], aux_l[Q]
        for a in np.unique(lP):
            for c in np.unique(lQ):
                sel = np.nonzero((lP == a) & (lQ == c))[0]
                if sel.size:
                    self.classes2c.append((int(a), int(c), i32(P[sel]), i32(Q[sel])))
        self._scratch = scratch if scratch is not None else ScratchHolder()
        self._build_ao_pairs(ao.shell_cxyz)
        self._build_pair_tables()

    # ------------------------------------------------------------ class launches over streams
    def _streams(self):
        """Side streams for class launches: classes write disjoint outputs (or add to the
        gradient atomically), so their kernels may overlap and fill each other's tails."""
        idx = self.device.index if self.device.index is not None else torch.cuda.current_device()
        if idx not in _SIDE_STREAMS:
            _SIDE_STREAMS[idx] = [torch.cuda.Stream(device=self.device) for _ in range(NSTREAMS)]
        return _SIDE_STREAMS[idx]

    def _fanout(self, launches):
        """Run launch(stream_ptr) callables round-robin over side streams, ordered after and
        before the current stream."""
        main = torch.cuda.current_stream(self.device)
        side = self._streams() if NSTREAMS > 1 else [main]
        if NSTREAMS > 1:
            start = torch.cuda.Event()
            start.record(main)
            for st in side:
                st.wait_event(start)
        for i, fn in enumerate(launches):
            fn(int(side[i % len(side)].cuda_stream))
        if NSTREAMS > 1:
            for st in side:
                ev = torch.cuda.Event()
                ev.record(st)
                main.wait_event(ev)

    @property
    def _i32(self):
        return lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device=self.device)

    @property
    def _f64(self):
        return lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=self.device)

    def _build_ao_pairs(self, shell_cxyz: np.ndarray) -> None:
        """Primitive-pair lists (screened) and the per-class AO pair lists for a geometry.

        A primitive pair is dropped when |c_a c_b| exp(-ab/(a+b) |AB|^2) (pi/(a+b))^(3/2),
        an upper bound of its overlap-like magnitude, is below ``prim_screen`` (1e-20 by
        default): its contribution to any integral is many orders below the FP64 rounding
        of the integral.  Shell pairs with no primitive pair left are dropped.  The
        reference evaluates every pair (``asuka/cueri/gpu.py:1833-1834``); ``prim_screen=0``
        reproduces that exactly.
        """
        ao, sp = self.ao, self.sp
        npr = sp.sp_npair.astype(np.int64)
        owner = np.repeat(np.arange(sp.nsp), npr)
        loc = (np.arange(owner.size) - np.repeat(sp.sp_pair_start[:-1].astype(np.int64), npr)).astype(np.int32)
        A = sp.sp_A[owner]
        B = sp.sp_B[owner]
        nb = ao.shell_nprim[B]
        pa = ao.shell_prim_start[A] + loc // nb
        pb = ao.shell_prim_start[B] + loc % nb
        if self.prim_screen > 0.0:
            a, b = ao.prim_exp[pa], ao.prim_exp[pb]
            R2 = ((shell_cxyz[A] - shell_cxyz[B]) ** 2).sum(1)
            p = a + b
            bound = np.abs(ao.prim_coef[pa] * ao.prim_coef[pb]) * np.exp(-a * b / p * R2) * (np.pi / p) ** 1.5
            keep = bound >= self.prim_screen
        else:
            keep = np.ones(owner.size, dtype=bool)
        kept_owner = owner[keep]
        cnt = np.bincount(kept_owner, minlength=sp.nsp).astype(np.int32)
        start = np.zeros(sp.nsp, dtype=np.int64)
        np.cumsum(cnt[:-1], out=start[1:])
        i32 = self._i32
        self.sp_pstart = i32(start)
        self.sp_npair = i32(cnt)
        self.pp_sp = i32(kept_owner)
        self.pp_local = i32(loc[keep])
        self.n_prim_pairs = int(keep.sum())
        self.n_prim_pairs_total = int(owner.size)
        self.pt = torch.empty((7, max(self.n_prim_pairs, 1)), dtype=torch.float64, device=self.device)
        self.ps_ao = _lib.PairSide(
            *[_lib.ptr(t) for t in (self.sp_A, self.sp_B, self.sp_pstart, self.sp_npair, *self.pt, self.ao_cxyz,
                                    self.ao_aostart, self.ao_atom)], 0)
        la = ao.shell_l[sp.sp_A]
        lb = ao.shell_l[sp.sp_B]
        live = cnt > 0
        # dropped shell pairs write nothing: outputs are zero-filled first when any exist
        self.n_dropped_pairs = int((~live).sum())
        self.classes3c = []  # (la, lb, lc, pairs tensor, aux tensor)
        for a in np.unique(la):
            for b in np.unique(lb):
                sel = np.nonzero((la == a) & (lb == b) & live)[0]
                if sel.size == 0:
                    continue
                # pairs by decreasing primitive-pair count: with the aux-major task
                # grid a warp walks pairs of similar cost against one aux shell
                sel = sel[np.argsort(-cnt[sel], kind="stable")]
                pairs = i32(sel)
                for c, auxs in self.aux_by_l.items():
                    self.classes3c.append((int(a), int(b), int(c), pairs, auxs))
        self._aux_blocks_n = None

    # ------------------------------------------------------------ helpers
    def _build_pair_tables(self) -> None:
        L = _lib.lib()
        p = _lib.ptr
        npp = self.n_prim_pairs
        rc = L.dfb_pair_tables(p(self.ao_cxyz), p(self.ao_pstart), p(self.ao_nprim), p(self.ao_exp), p(self.ao_coef),
                               p(self.sp_A), p(self.sp_B), p(self.sp_pstart), p(self.pp_sp), p(self.pp_local), npp, 0,
                               *[p(r) for r in self.pt], _stream())
        _lib.check(rc, "dfb_pair_tables(ao)")
        nax = int(self.ax_pp_sp.numel())
        rc = L.dfb_pair_tables(p(self.ax_cxyz), p(self.ax_pstart), p(self.ax_nprim), p(self.ax_exp), p(self.ax_coef),
                               p(self.ax_self), p(self.ax_self), p(self.ax_pstart), p(self.ax_pp_sp), 0, nax, 1,
                               *[p(r) for r in self.axpt], _stream())
        _lib.check(rc, "dfb_pair_tables(aux)")

    def set_coords(self, coords) -> None:
        """Move the shell centres to new atom positions ((natm, 3), bohr).

        Host coordinates (numpy or CPU tensor) also rebuild the screened primitive-pair
        lists for the new geometry; device coordinates update the centres and pair tables
        without a host round trip and keep the lists of the last host geometry (use them
        for small moves, such as finite differences or the timed steps of a fixed
        geometry).
        """
        if isinstance(coords, np.ndarray) or (isinstance(coords, torch.Tensor) and not coords.is_cuda):
            c_np = np.asarray(coords, dtype=np.float64).reshape(-1, 3)
            self._build_ao_pairs(c_np[self.ao.shell_atom])
        coords = torch.as_tensor(coords, dtype=torch.float64).to(device=self.device).reshape(-1, 3)
        self.ao_cxyz.copy_(coords.index_select(0, self.ao_atom.long()))
        self.ax_cxyz.copy_(coords.index_select(0, self.ax_atom.long()))
        self._build_pair_tables()

    def _scratch_for(self, deriv: bool, copies: int = 1) -> torch.Tensor:
        key = (deriv, os.environ.get("DFB_DISABLE_TMPL"), id(self.classes3c))
        cache = self.__dict__.setdefault("_need_cache", {})
        if key in cache:
            return self._scratch.get(cache[key] * copies, self.device)
        L = _lib.lib()
        need = 1
        for la, lb, lc, pairs, auxs in self.classes3c:
            n = L.dfb_rys_scratch_doubles(la, lb, lc, pairs.numel() * auxs.numel(), int(deriv))
            _lib.check(0 if n >= 0 else int(n), "dfb_rys_scratch_doubles")
            need = max(need, n)
        for lp, lq, P, Q in self.classes2c:
            n = L.dfb_rys_scratch_doubles(lp, 0, lq, P.numel(), int(deriv))
            _lib.check(0 if n >= 0 else int(n), "dfb_rys_scratch_doubles")
            need = max(need, n)
        cache[key] = need
        return self._scratch.get(need * copies, self.device)

    def aux_blocks(self, max_naux: int = 256):
        """Contiguous aux-shell blocks of at most ``max_naux`` functions, aligned to shells
        (``asuka/cueri/df.py:2059-2119`` plan_aux_blocks_cart); returns (p0, p1, AuxSide) tuples."""
        if getattr(self, "_aux_blocks_n", None) == max_naux:
            return self._aux_blocks
        aux = self.aux
        nc = np.array([ncart(int(l)) for l in aux.shell_l])
        blocks = []
        s0 = 0
        while s0 < aux.nshell:
            s1 = s0
            tot = 0
            while s1 < aux.nshell and (tot + nc[s1] <= max_naux or s1 == s0):
                tot += nc[s1]
                s1 += 1
            p0 = int(aux.shell_ao_start[s0])
            p1 = p0 + int(tot)
            shifted = torch.as_tensor(aux.shell_ao_start.astype(np.int32) - p0, device=self.device)
            axb = _lib.AuxSide(*[_lib.ptr(t) for t in (self.ax_cxyz, self.ax_pstart, self.ax_nprim, self.ax_exp,
                                                       self.ax_coef, self.ax_rexp, shifted, self.ax_atom)])
            byl = {}
            for l in np.unique(aux.shell_l[s0:s1]):
                idx = s0 + np.nonzero(aux.shell_l[s0:s1] == l)[0]
                byl[int(l)] = torch.as_tensor(idx.astype(np.int32), device=self.device)
            blocks.append((p0, p1, (axb, shifted, byl)))
            s0 = s1
        self._aux_blocks, self._aux_blocks_n = blocks, max_naux
        return blocks

    def int3c_block(self, blk, p0: int, p1: int, out: torch.Tensor | None = None,
                    dropped_zero: bool = False, precision: str = "fp64") -> torch.Tensor:
        """X rows for one aux block as (p1-p0, nao, nao) (streamed DF, ``gpu.py:2742``).

        Entries of screened-out shell pairs are not written; they are zeroed here
        unless ``dropped_zero`` says the buffer already holds zeros there (the set
        of dropped pairs is the same for every block, so a reused buffer needs
        zeroing once).
        """
        axb, _shifted, byl = blk
        nao = self.nao
        X = out if out is not None else torch.empty((p1 - p0, nao, nao), dtype=torch.float64, device=self.device)
        if self.n_dropped_pairs and not dropped_zero:
            X.zero_()
        self._slices_int = self._scratch_slices(False)
        launches = []
        seen = set()
        for la, lb, lc, pairs, _auxs in self.classes3c:
            if lc not in byl or (la, lb, lc) in seen:
                continue
            seen.add((la, lb, lc))
            auxs = byl[lc]
            launches.append(self._launch_int(la, lb, lc, self.ps_ao, axb, pairs, auxs, pairs.numel() * auxs.numel(),
                                             -pairs.numel(), 0, X, (nao * nao, nao, 1), _prec_code(precision)))
        self._fanout(launches)
        return X

    def deriv3c_block(self, blk, bar: torch.Tensor, grad: torch.Tensor, precision: str = "fp64") -> torch.Tensor:
        """grad += sum over one aux block of bar[P-p0, mu, nu] d(mu nu|P)/dR (block-local adjoint)."""
        axb, _shifted, byl = blk
        nao = self.nao
        bar = bar.contiguous()
        self._slices_der = self._scratch_slices(True)
        launches = []
        seen = set()
        for la, lb, lc, pairs, _auxs in self.classes3c:
            if lc not in byl or (la, lb, lc) in seen:
                continue
            seen.add((la, lb, lc))
            auxs = byl[lc]
            launches.append(self._launch_deriv(la, lb, lc, self.ps_ao, axb, pairs, auxs, pairs.numel() * auxs.numel(),
                                               -pairs.numel(), 0, bar, (nao * nao, nao, 1), grad,
                                               _prec_code(precision)))
        self._fanout(launches)
        return grad

    def _scratch_slices(self, deriv: bool):
        """Scratch for the generic kernels: one slice per side stream (launches overlap)."""
        n = max(NSTREAMS, 1)
        buf = self._scratch_for(deriv, copies=n)
        per = buf.numel() // n
        return [buf[i * per:(i + 1) * per] for i in range(n)]

    def _launch_int(self, la, lb, lc, ps, axs, pairs, auxs, ntask, ngrid, mode, out, strides, prec=PREC_FP64):
        L = _lib.lib()
        # the metric (mode 1) stays FP64: its Cholesky factor whitens everything downstream
        prec = PREC_FP64 if mode == 1 else _class_prec(prec, "int3c", la, lb, lc)
        key = (la, lb, lc, mode, prec)

        def fn(stream, _k=key):
            i = self._slot_of(stream)
            scr = self._slices_int[i]
            rc = L.dfb_rys_int_prec(la, lb, lc, ctypes.byref(ps), ctypes.byref(axs), _lib.ptr(pairs), _lib.ptr(auxs),
                                    ntask, ngrid, mode, prec, _lib.ptr(out), *strides, _lib.ptr(scr), scr.numel(),
                                    stream)
            _lib.check(rc, f"dfb_rys_int {_k}")
        return fn

    def _launch_deriv(self, la, lb, lc, ps, axs, pairs, auxs, ntask, ngrid, mode, bar, strides, grad, prec=PREC_FP64):
        L = _lib.lib()
        prec = _class_prec(prec, "deriv2c" if mode == 1 else "deriv3c", la, lb, lc)
        key = (la, lb, lc, mode, prec)

        def fn(stream, _k=key):
            i = self._slot_of(stream)
            scr = self._slices_der[i]
            rc = L.dfb_rys_deriv_prec(la, lb, lc, ctypes.byref(ps), ctypes.byref(axs), _lib.ptr(pairs),
                                      _lib.ptr(auxs), ntask, ngrid, mode, prec, _lib.ptr(bar), *strides,
                                      _lib.ptr(grad), self.natm, _lib.ptr(scr), scr.numel(), stream)
            _lib.check(rc, f"dfb_rys_deriv {_k}")
        return fn

    def _slot_of(self, stream_ptr: int) -> int:
        if NSTREAMS <= 1:
            return 0
        for i, st in enumerate(self._streams()):
            if int(st.cuda_stream) == stream_ptr:
                return i
        return 0

    # ------------------------------------------------------------ integrals
    def metric(self, out: torch.Tensor | None = None) -> torch.Tensor:
        """V[P, Q] = (P|Q), full symmetric (naux, naux)."""
        naux = self.naux
        V = out if out is not None else torch.empty((naux, naux), dtype=torch.float64, device=self.device)
        self._slices_int = self._scratch_slices(False)
        self._fanout([self._launch_int(lp, 0, lq, self.ps_aux, self.axs, P, Q, P.numel(), 0, 1, V, (naux, 1, 0))
                      for lp, lq, P, Q in self.classes2c])
        # diagonal shell blocks are written from one tile in both orders; make V
        # exactly symmetric as the reference does (cueri_df_cpu.py: V = (V+V^T)/2)
        V.copy_(0.5 * (V + V.T))
        return V

    def int3c(self, layout: str = "Qmn", out: torch.Tensor | None = None, precision: str = "fp64") -> torch.Tensor:
        """X = (mu nu|P): 'Qmn' -> (naux, nao, nao), 'mnQ' -> (nao, nao, naux).

        ``precision='mixed'`` runs the class kernels with FP32 recurrence tables and
        accumulators (``DFB_PREC_MIXED``); the output stays FP64."""
        nao, naux = self.nao, self.naux
        if layout == "Qmn":
            shape, s = (naux, nao, nao), (nao * nao, nao, 1)
        elif layout == "mnQ":
            shape, s = (nao, nao, naux), (1, nao * naux, naux)
        else:
            raise ValueError("layout must be 'Qmn' or 'mnQ'")
        X = out if out is not None else torch.empty(shape, dtype=torch.float64, device=self.device)
        if self.n_dropped_pairs:
            X.zero_()
        self._slices_int = self._scratch_slices(False)
        pc = _prec_code(precision)
        self._fanout([self._launch_int(la, lb, lc, self.ps_ao, self.axs, pairs, auxs, pairs.numel() * auxs.numel(),
                                       -pairs.numel(), 0, X, s, pc) for la, lb, lc, pairs, auxs in self.classes3c])
        return X

    def deriv3c(self, bar: torch.Tensor, grad: torch.Tensor, layout: str = "Qmn", precision: str = "fp64") -> torch.Tensor:
        """grad += sum_{mu nu P} bar[mu nu P] d(mu nu|P)/dR; bar symmetric in (mu, nu)."""
        nao, naux = self.nao, self.naux
        if layout == "Qmn":
            s = (nao * nao, nao, 1)
        elif layout == "mnQ":
            s = (1, nao * naux, naux)
        else:
            raise ValueError("layout must be 'Qmn' or 'mnQ'")
        bar = bar.contiguous()
        self._slices_der = self._scratch_slices(True)
        pc = _prec_code(precision)
        self._fanout([self._launch_deriv(la, lb, lc, self.ps_ao, self.axs, pairs, auxs, pairs.numel() * auxs.numel(),
                                         -pairs.numel(), 0, bar, s, grad, pc)
                      for la, lb, lc, pairs, auxs in self.classes3c])
        return grad

    def deriv2c(self, bar: torch.Tensor, grad: torch.Tensor, precision: str = "fp64") -> torch.Tensor:
        """grad += sum_{P,Q} bar[P,Q] d(P|Q)/dR; bar symmetric."""
        naux = self.naux
        bar = bar.contiguous()
        self._slices_der = self._scratch_slices(True)
        pc = _prec_code(precision)
        self._fanout([self._launch_deriv(lp, 0, lq, self.ps_aux, self.axs, P, Q, P.numel(), 0, 1, bar, (naux, 1, 0),
                                         grad, pc) for lp, lq, P, Q in self.classes2c])
        return grad


    # ------------------------------------------------------------ overlapped phases of one step
    def metric_cholesky_int3c(self, X: torch.Tensor | None = None, precision: str = "fp64"):
        """V = (P|Q), its Cholesky factor L and X = (mu nu|P) ('Qmn') with the phases overlapped.

        The metric classes go to the side streams first and the 3c classes after them; the
        main stream waits only for the metric launches, symmetrizes V and factorises it while
        the 3c classes still run, then joins.  Same results as metric(), cholesky_metric() and
        int3c() in sequence.
        """
        nao, naux = self.nao, self.naux
        if NSTREAMS <= 1:
            V = self.metric()
            return V, cholesky_metric(V), self.int3c("Qmn", out=X, precision=precision)
        V = torch.empty((naux, naux), dtype=torch.float64, device=self.device)
        X = X if X is not None else torch.empty((naux, nao, nao), dtype=torch.float64, device=self.device)
        if self.n_dropped_pairs:
            X.zero_()
        self._slices_int = self._scratch_slices(False)
        first = [self._launch_int(lp, 0, lq, self.ps_aux, self.axs, P, Q, P.numel(), 0, 1, V, (naux, 1, 0))
                 for lp, lq, P, Q in self.classes2c]
        pc = _prec_code(precision)
        second = [self._launch_int(la, lb, lc, self.ps_ao, self.axs, pairs, auxs, pairs.numel() * auxs.numel(),
                                   -pairs.numel(), 0, X, (nao * nao, nao, 1), pc)
                  for la, lb, lc, pairs, auxs in self.classes3c]
        main = torch.cuda.current_stream(self.device)
        side = self._streams()
        start = torch.cuda.Event()
        start.record(main)
        for st in side:
            st.wait_event(start)
        for i, fn in enumerate(first):
            fn(int(side[i % len(side)].cuda_stream))
        for st in side:
            ev = torch.cuda.Event()
            ev.record(st)
            main.wait_event(ev)
        for i, fn in enumerate(second):
            fn(int(side[(i + len(first)) % len(side)].cuda_stream))
        V.copy_(0.5 * (V + V.T))
        L, info = torch.linalg.cholesky_ex(V)
        for st in side:
            ev = torch.cuda.Event()
            ev.record(st)
            main.wait_event(ev)
        if int(info.item()) != 0:
            raise RuntimeError(f"metric Cholesky failed (leading minor {int(info.item())} not positive definite)")
        return V, L, X

    def deriv3c_2c(self, bar3: torch.Tensor, bar2: torch.Tensor, grad: torch.Tensor,
                   precision: str = "fp64") -> torch.Tensor:
        """deriv3c(bar3 'Qmn') and deriv2c(bar2) as one fan-out (both add into grad atomically)."""
        nao, naux = self.nao, self.naux
        bar3 = bar3.contiguous()
        bar2 = bar2.contiguous()
        self._slices_der = self._scratch_slices(True)
        pc = _prec_code(precision)
        launches = [self._launch_deriv(la, lb, lc, self.ps_ao, self.axs, pairs, auxs, pairs.numel() * auxs.numel(),
                                       -pairs.numel(), 0, bar3, (nao * nao, nao, 1), grad, pc)
                    for la, lb, lc, pairs, auxs in self.classes3c]
        launches += [self._launch_deriv(lp, 0, lq, self.ps_aux, self.axs, P, Q, P.numel(), 0, 1, bar2, (naux, 1, 0),
                                        grad, pc) for lp, lq, P, Q in self.classes2c]
        self._fanout(launches)
        return grad


# ---------------------------------------------------------------- reference seams

_ENGINES: "weakref.WeakValueDictionary" = weakref.WeakValueDictionary()
_ENGINE_KEEP: dict = {}


def get_engine(ao_basis, aux_basis, device=None) -> DFEngine:
    """Engine cached by (id(ao), id(aux), device) like the reference's plan caches (gpu.py:1602-1612)."""
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    key = (id(ao_basis), id(aux_basis), dev.index)
    eng = _ENGINE_KEEP.get(key)
    if eng is None or eng._bases_ref[0]() is not ao_basis or eng._bases_ref[1]() is not aux_basis:
        eng = DFEngine(ao_basis, aux_basis, device=dev)
        try:
            eng._bases_ref = (weakref.ref(ao_basis), weakref.ref(aux_basis))
        except TypeError:
            eng._bases_ref = (lambda: ao_basis, lambda: aux_basis)
        if len(_ENGINE_KEEP) > 8:
            _ENGINE_KEEP.clear()
        _ENGINE_KEEP[key] = eng
    return eng


def _dummy_ao_for(aux_basis):
    """Metric-only engines still need an AO side; an s shell at the first aux centre works."""
    aux = _as_soa(aux_basis)
    return BasisCartSoA(shell_cxyz=aux.shell_cxyz[:1].copy(), shell_prim_start=np.zeros(1, np.int32),
                        shell_nprim=np.ones(1, np.int32), shell_l=np.zeros(1, np.int32),
                        shell_ao_start=np.zeros(1, np.int32), prim_exp=np.ones(1), prim_coef=np.ones(1),
                        shell_atom=None if aux.shell_atom is None else aux.shell_atom[:1].copy())


def metric_2c2e_basis(aux_basis, *, stream=None, backend: str = "gpu_rys", mode: str = "warp", threads: int = 256,
                      mixed_precision: bool = False, atom_coords_bohr=None) -> torch.Tensor:
    """V[P,Q] = (P|Q) on the current CUDA device (``asuka/cueri/df.py:803``)."""
    if backend not in ("gpu_rys", "gpu_sp", "gpu_ss"):
        raise ValueError("backend must be one of gpu_rys/gpu_sp/gpu_ss")
    aux = _as_soa(aux_basis)
    if aux.shell_atom is None:
        aux = from_reference_like(aux, np.zeros(aux.nshell, np.int32))
    eng = DFEngine(_dummy_ao_for(aux), aux)
    return eng.metric()


def _check_ao_rep(ao_rep: str) -> str:
    if ao_rep not in ("cart", "sph"):
        raise ValueError("ao_rep must be 'cart' or 'sph'")
    return ao_rep


def int3c2e_basis(ao_basis, aux_basis, *, stream=None, backend: str = "gpu_rys", mode: str = "warp",
                  threads: int = 256, mixed_precision: bool = False, layout: str = "mnQ",
                  ao_rep: str = "cart") -> torch.Tensor:
    """X[mu,nu,P] = (mu nu|P) (``asuka/cueri/df.py:859``); layout 'mnQ' or 'Qmn'.

    ``ao_rep='sph'`` returns X over real spherical AOs (the aux index stays Cartesian).
    """
    _check_ao_rep(ao_rep)
    ao, aux = _as_soa(ao_basis), _as_soa(aux_basis)
    if ao.shell_atom is None:
        ao = from_reference_like(ao, np.zeros(ao.nshell, np.int32))
    if aux.shell_atom is None:
        aux = from_reference_like(aux, np.zeros(aux.nshell, np.int32))
    eng = DFEngine(ao, aux)
    if ao_rep == "cart":
        return eng.int3c(layout)
    from .sph import cart2sph_ao_matrix, int3c_cart_to_sph

    return int3c_cart_to_sph(eng.int3c("Qmn"), cart2sph_ao_matrix(ao.shell_l, eng.device),
                             "Qmn").permute(*((1, 2, 0) if layout == "mnQ" else (0, 1, 2))).contiguous()


def cholesky_metric(V: torch.Tensor, *, shift: float = 0.0) -> torch.Tensor:
    """Lower Cholesky factor of the metric.

    The reference's CPU DF build factorises V with no diagonal shift
    (``asuka/integrals/cueri_df_cpu.py:521``); that is the default here, so FP64
    results match the reference CPU path.  A non-zero ``shift`` is added to the
    diagonal first, as the reference's GPU builder does (``cueri_df.py:86-89``).
    """
    Vs = 0.5 * (V + V.T)
    if shift:
        Vs = Vs + float(shift) * torch.eye(V.shape[0], dtype=V.dtype, device=V.device)
    L, info = torch.linalg.cholesky_ex(Vs)
    if int(info.item()) != 0:
        raise RuntimeError(f"metric Cholesky failed (leading minor {int(info.item())} not positive definite)")
    return L


def whiten_3c2e(X: torch.Tensor, L: torch.Tensor, layout: str = "mnQ") -> torch.Tensor:
    """B = X L^-T over the aux index, in place (``asuka/cueri/df.py:994``)."""
    if layout == "mnQ":
        nao = X.shape[0]
        X2 = X.view(nao * nao, -1)
        _la.solve_lower_right_T(L, X2, out=X2)  # B = X L^-T over the last index
        return X
    if layout == "Qmn":
        naux = X.shape[0]
        X2 = X.view(naux, -1)
        _la.solve_lower(L, X2, out=X2)  # B_Q rows = L^-1 X
        return X
    raise ValueError("layout must be 'mnQ' or 'Qmn'")


def build_df_B_from_cueri_packed_bases(ao_basis, aux_basis, *, config=None, layout: str = "mnQ",
                                       ao_rep: str = "cart", profile: dict | None = None, return_L: bool = False):
    """Whitened DF factors B with (mu nu|ls) ~= sum_Q B[mu nu Q] B[ls Q] (``asuka/integrals/cueri_df.py:33``).

    FP64 device tensors; ``layout='mnQ'`` -> (nao, nao, naux), ``'Qmn'`` -> (naux, nao, nao).
    Errors raise RuntimeError/ValueError/NotImplementedError; there is no CPU fallback.
    """
    _check_ao_rep(ao_rep)
    ao, aux = _as_soa(ao_basis), _as_soa(aux_basis)
    if ao.shell_atom is None:
        ao = from_reference_like(ao, np.zeros(ao.nshell, np.int32))
    if aux.shell_atom is None:
        aux = from_reference_like(aux, np.zeros(aux.nshell, np.int32))
    eng = DFEngine(ao, aux)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)] if profile is not None else None
    if ev:
        ev[0].record()
    V = eng.metric()
    if ev:
        ev[1].record()
    if ao_rep == "cart":
        X = eng.int3c(layout)
    else:  # real spherical AOs on the AO side; the aux index stays Cartesian
        from .sph import cart2sph_ao_matrix, int3c_cart_to_sph

        X = int3c_cart_to_sph(eng.int3c("Qmn"), cart2sph_ao_matrix(ao.shell_l, eng.device), "Qmn")
        if layout == "mnQ":
            X = X.permute(1, 2, 0).contiguous()
    if ev:
        ev[2].record()
    L = cholesky_metric(V)
    if ev:
        ev[3].record()
    B = whiten_3c2e(X, L, layout)
    if ev:
        ev[4].record()
        torch.cuda.synchronize()
        profile.update(t_metric_s=ev[0].elapsed_time(ev[1]) / 1e3, t_int3c2e_s=ev[1].elapsed_time(ev[2]) / 1e3,
                       t_metric_cholesky_s=ev[2].elapsed_time(ev[3]) / 1e3,
                       t_whiten_s=ev[3].elapsed_time(ev[4]) / 1e3, nao=eng.nao, naux=eng.naux)
    return (B, L) if return_L else B
