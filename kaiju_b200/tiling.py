"""Domain decomposition of one problem into tiles along k, and the halo exchange between them.

This mirrors the reference's MPI tiling (src/gamera/mpi/gamapp_mpi.F90): every tile is a full problem of
its own (ghosts included) whose k faces inside the global domain carry the BC kind GAM_BC_HALO; after each
step the tiles' global dt is the minimum of their own (CalcDT_mpi, :501-518), the physical BCs run, the
4-layer halos of Gas, Bxyz and magFlux are exchanged (haloUpdate, :694-794) and Bxyz is recomputed from the
fluxes (updateMpiBCs, :579-663). The halo layers span the full i/j extent, ghosts included (the edge and
corner pieces of the reference's neighbour datatypes come from the same k neighbour when i and j are not
decomposed). Cells ks-n and their three faces come from the lower neighbour's cells ke-n+1; cells ke+n
and their I/J faces from the upper neighbour's cells ks+n-1; the K faces ke+1 .. ke+nG+1 from the upper
neighbour's K faces ks .. ks+nG, so the face the two tiles share belongs to the upper tile
(calcDatatypeFC, :1518-1664, nG+1 K-face layers for kData=1).

Indices here are zero-based positions in the Fortran arrays (0 = ksg), so they apply to the host arrays
of the C ABI and of any solver laid out like Grid_T/State_T.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple

GAM_BC_PERIODIC, GAM_BC_HALO = 0, 4
NG = 4


def split_k(Nkp: int, ntiles: int) -> List[Tuple[int, int]]:
    """(first active k counted from 0, active cells) of each tile; every tile needs at least NG cells."""
    if ntiles < 1 or Nkp < ntiles * NG:
        raise ValueError(f"cannot split {Nkp} cells into {ntiles} tiles of at least {NG}")
    base, extra = divmod(Nkp, ntiles)
    out, k0 = [], 0
    for q in range(ntiles):
        nk = base + (1 if q < extra else 0)
        out.append((k0, nk))
        k0 += nk
    return out


def tile_corners(xyz, k0: int, nk: int):
    """The corner coordinates of a tile, ghosts included: the global corner array (ghosts included) sliced
    at k0 .. k0 + nk + 2*NG."""
    return xyz[:, :, k0:k0 + nk + 2 * NG + 1, :]


def tile_bcs(global_bc: Sequence[int], q: int, ntiles: int) -> List[int]:
    """BC kinds of tile q: the global ones on the global faces, GAM_BC_HALO on faces between tiles (and on
    both global K faces when the global K boundary is periodic: the first and last tiles are neighbours)."""
    bc = list(global_bc)
    periodic = global_bc[4] == GAM_BC_PERIODIC and global_bc[5] == GAM_BC_PERIODIC
    if q > 0 or (periodic and ntiles > 1):
        bc[4] = GAM_BC_HALO
    if q < ntiles - 1 or (periodic and ntiles > 1):
        bc[5] = GAM_BC_HALO
    return bc


def neighbours(q: int, ntiles: int, periodic: bool):
    """(lower, upper) neighbour of tile q, None at a physical boundary."""
    lo = q - 1 if q > 0 else (ntiles - 1 if periodic and ntiles > 1 else None)
    up = q + 1 if q < ntiles - 1 else (0 if periodic and ntiles > 1 else None)
    return lo, up


def halo_from_below(nk_below: int):
    """Copies that fill a tile's lower halo from its lower neighbour (nk_below active cells):
    (array kind, component set, destination k slice, source k slice), kinds 'cell' (Gas, Bxyz) and
    'face' (magFlux, all components)."""
    src = slice(NG + nk_below - NG, NG + nk_below)
    return [("cell", None, slice(0, NG), src), ("face", (0, 1, 2), slice(0, NG), src)]


def halo_from_above(nk: int):
    """Copies that fill a tile's upper halo (the tile has nk active cells) from its upper neighbour."""
    return [("cell", None, slice(NG + nk, NG + nk + NG), slice(NG, 2 * NG)),
            ("face", (0, 1), slice(NG + nk, NG + nk + NG), slice(NG, 2 * NG)),
            ("face", (2,), slice(NG + nk, NG + nk + NG + 1), slice(NG, 2 * NG + 1))]


# ------------------------------------------------------------------ device tiles
def tile_models(model, ntiles: int):
    """(k0, nk, tile Model) for each k-tile of `model` (a gamera.Model): the tile's Nkp and BC kinds."""
    import dataclasses
    if model.ring is not None or model.do25D:
        raise ValueError("k tiling needs whole rings in k and more than one k layer")
    out = []
    for q, (k0, nk) in enumerate(split_k(model.Nkp, ntiles)):
        out.append((k0, nk, dataclasses.replace(model, Nkp=nk, bc=tuple(tile_bcs(model.bc, q, ntiles)))))
    return out


def make_tiles(model, xyz, ntiles: int, ic: str, fp32: bool = False, **kw):
    """Device tiles of one problem (each a gamera.GameraGPU on the current device) built from the global
    corner array with ghosts; returns (tiles, [(k0, nk), ...])."""
    from . import gamera as gm
    tiles, split = [], []
    for k0, nk, m in tile_models(model, ntiles):
        t = gm.GameraGPU.from_corners(m, tile_corners(xyz, k0, nk), ic, **kw)
        if fp32:
            t.set_precision(gm.GAM_FP32FLUX)
        tiles.append(t)
        split.append((k0, nk))
    return tiles, split


def periodic_k(model) -> bool:
    return model.bc[4] == GAM_BC_PERIODIC and model.bc[5] == GAM_BC_PERIODIC


def stitch(arrays: Sequence, split, face: bool = False):
    """The global array (Fortran layout, ghosts included) assembled from the tiles' arrays: every tile
    gives its active k layers (and, for face arrays, the last tile its upper face ke+1); the k ghosts
    come from the first and last tiles."""
    import numpy as np
    first, last = arrays[0], arrays[-1]
    nk_tot = sum(nk for _, nk in split)
    shape = list(first.shape)
    shape[2] = nk_tot + 2 * NG + (1 if face else 0)
    out = np.zeros(shape, dtype=first.dtype, order="F")
    out[:, :, :NG] = first[:, :, :NG]
    for a, (k0, nk) in zip(arrays, split):
        out[:, :, NG + k0:NG + k0 + nk] = a[:, :, NG:NG + nk]
    k0, nk = split[-1]
    out[:, :, NG + nk_tot:] = last[:, :, NG + nk:]
    return out


class DistTile:
    """One k-tile per process, its halos and dt minimum moved with torch.distributed: NCCL with CUDA
    tensors, or any backend through host copies (staging=True). The step is the reference's
    stepGamera_mpi (gamapp_mpi.F90:665-692) with haloUpdate (:694-794) as two send/recv pairs."""

    def __init__(self, tile, rank: int, world: int, periodic: bool, group=None, staging: bool = False):
        import ctypes as C
        import torch
        from . import gamera as gm
        self.gm, self.C, self.torch = gm, C, torch
        self.tile, self.rank, self.world, self.group, self.staging = tile, rank, world, group, staging
        self.lo, self.up = neighbours(rank, world, periodic)
        L = gm.load_library()
        s = C.c_void_p()
        self._check(L.gam_gpu_stream(tile.h, C.byref(s)), "gam_gpu_stream")
        self.stream = torch.cuda.ExternalStream(s.value)
        with torch.cuda.stream(self.stream):
            self.words = torch.zeros(2, dtype=torch.int64, device="cuda")

    def _check(self, rc, what):
        if rc:
            raise self.gm.GamError(rc, what)

    def _sizes(self, side, what):
        C = self.C
        sb, rb = C.c_longlong(), C.c_longlong()
        self._check(self.gm.load_library().gam_gpu_halo_bytes(self.tile.h, side, what, C.byref(sb), C.byref(rb)),
                    "gam_gpu_halo_bytes")
        return sb.value // 8, rb.value // 8

    def _allreduce_min(self):
        import torch.distributed as dist
        torch = self.torch
        with torch.cuda.stream(self.stream):
            if self.staging:
                w = self.words.cpu()
                dist.all_reduce(w, op=dist.ReduceOp.MIN, group=self.group)
                self.words.copy_(w)
            else:
                dist.all_reduce(self.words, op=dist.ReduceOp.MIN, group=self.group)

    def exchange(self, what):
        """Pack the two boundary slabs, swap them with the k neighbours, unpack the halos."""
        import torch.distributed as dist
        torch, L = self.torch, self.gm.load_library()
        h = self.tile.h
        sides = [s for s, nb in ((0, self.lo), (1, self.up)) if nb is not None]
        with torch.cuda.stream(self.stream):
            send, recv = {}, {}
            for s in sides:
                ns, nr = self._sizes(s, what)
                send[s] = torch.empty(ns, dtype=torch.float64, device="cuda")
                recv[s] = torch.empty(nr, dtype=torch.float64, device="cuda")
                self._check(L.gam_gpu_halo_pack(h, s, what, send[s].data_ptr()), "gam_gpu_halo_pack")
            peer = {0: self.lo, 1: self.up}
            if all(peer[s] == self.rank for s in sides):   # a single periodic tile is its own neighbour
                for s in sides:
                    recv[s].copy_(send[s ^ 1])
            else:
                # sends upward first, receives from below first: with two tiles on a periodic K boundary
                # both messages go to the same peer and must pair up in order
                order_send = [s for s in (1, 0) if s in sides]
                order_recv = [s for s in (0, 1) if s in sides]
                if self.staging:
                    sbuf = {s: send[s].cpu() for s in sides}
                    rbuf = {s: torch.empty(recv[s].shape, dtype=torch.float64) for s in sides}
                else:
                    sbuf, rbuf = send, recv
                ops = [dist.P2POp(dist.isend, sbuf[s], peer[s], self.group, tag=1 + s) for s in order_send]
                ops += [dist.P2POp(dist.irecv, rbuf[s], peer[s], self.group, tag=2 - s) for s in order_recv]
                for r in dist.batch_isend_irecv(ops):
                    r.wait()
                if self.staging:
                    for s in sides:
                        recv[s].copy_(rbuf[s])
            for s in sides:
                self._check(L.gam_gpu_halo_unpack(h, s, what, recv[s].data_ptr()), "gam_gpu_halo_unpack")

    def setup(self):
        """Hatch_mpi's set-up: halos of State and oState with Bxyz, then the tiles' minimum initial dt."""
        gm, L = self.gm, self.gm.load_library()
        self.exchange(gm.GAM_HALO_STATE | gm.GAM_HALO_OSTATE | gm.GAM_HALO_BXYZ)
        self._check(L.gam_gpu_calcdt_local(self.tile.h, self.words.data_ptr()), "gam_gpu_calcdt_local")
        self._allreduce_min()
        self._check(L.gam_gpu_calcdt_finish(self.tile.h, self.words.data_ptr()), "gam_gpu_calcdt_finish")

    def step(self) -> int:
        gm, L = self.gm, self.gm.load_library()
        h = self.tile.h
        self._check(L.gam_gpu_step_local(h, self.words.data_ptr()), "gam_gpu_step_local")
        self._allreduce_min()
        self._check(L.gam_gpu_step_bcs(h, self.words.data_ptr()), "gam_gpu_step_bcs")
        self.exchange(gm.GAM_HALO_STATE)
        return L.gam_gpu_step_ghosts(h)
