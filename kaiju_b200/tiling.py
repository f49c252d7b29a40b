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
