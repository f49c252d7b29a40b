"""Two ranks (gloo, CPU), each advancing one k-tile of a problem with the oracle, exchange their 4-layer
halos and take the global minimum dt every step (the reference's MPI tiling, gamapp_mpi.F90:501-794); the
tiles' active cells must match the undecomposed run exactly. This exercises the decomposition and the
exchange protocol of kaiju_b200/tiling.py that the multi-tile device path follows."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBLEMS = {
    # warped blast wave, zero-gradient in k: two tiles, a physical face at each end
    "bw": dict(n=(16, 16, 16), kw=dict(ic="BW", grid="warp", warp_amp=0.04, bounds=(-0.5, 0.5) * 3, CFL=0.3,
                                          bc=[1] * 6), corners=("warped", (-0.5, 0.5) * 3, 0.04)),
    # Orszag-Tang slab, periodic in k: the two tiles are each other's lower and upper neighbour
    "ot": dict(n=(16, 16, 8), kw=dict(ic="OT2D", grid="uniform", bounds=(0.0, 1.0, 0.0, 1.0, 0.0, 1.0 / 16), CFL=0.3,
                                         bc=[0] * 6), corners=("uniform", (0.0, 1.0, 0.0, 1.0, 0.0, 1.0 / 16), 0.0)),
}


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _exchange(o, q, nt, tiles, periodic, names):
    from kaiju_b200 import tiling as tl
    lo, up = tl.neighbours(q, nt, periodic)
    arrs = {nm: o.get(nm) for nm in names}
    nk = tiles[q][1]
    reqs, recvs = [], []

    def copies_for(kind_names, copies):
        return [(c, nm) for nm in kind_names for c in copies if (c[0] == "cell") == (nm != names[0])]

    cell_names, face_names = [names[1], names[2]], [names[0]]
    # messages up: what the upper neighbour's lower halo needs; messages down: the lower neighbour's upper halo
    if up is not None:
        for (kind, comps, _d, src), nm in copies_for(cell_names + face_names, tl.halo_from_below(nk)):
            a = arrs[nm]
            sl = a[:, :, src] if comps is None else a[:, :, src][..., list(comps)]
            reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(sl)), up, tag=1))
    if lo is not None:
        for (kind, comps, _d, src), nm in copies_for(cell_names + face_names, tl.halo_from_above(tiles[lo][1])):
            a = arrs[nm]
            sl = a[:, :, src] if comps is None else a[:, :, src][..., list(comps)]
            reqs.append(dist.isend(torch.from_numpy(np.ascontiguousarray(sl)), lo, tag=2))
    if lo is not None:
        for (kind, comps, dst, _s), nm in copies_for(cell_names + face_names, tl.halo_from_below(tiles[lo][1])):
            a = arrs[nm]
            shape = a[:, :, dst].shape if comps is None else a[:, :, dst][..., list(comps)].shape
            buf = torch.empty(shape, dtype=torch.float64)
            dist.recv(buf, lo, tag=1)
            recvs.append((nm, dst, comps, buf))
    if up is not None:
        for (kind, comps, dst, _s), nm in copies_for(cell_names + face_names, tl.halo_from_above(nk)):
            a = arrs[nm]
            shape = a[:, :, dst].shape if comps is None else a[:, :, dst][..., list(comps)].shape
            buf = torch.empty(shape, dtype=torch.float64)
            dist.recv(buf, up, tag=2)
            recvs.append((nm, dst, comps, buf))
    for r in reqs:
        r.wait()
    for nm, dst, comps, buf in recvs:
        if comps is None:
            arrs[nm][:, :, dst] = buf.numpy()
        else:
            for c, cc in enumerate(comps):
                arrs[nm][:, :, dst, cc] = buf.numpy()[..., c]
    for nm in names:
        o.set(nm, arrs[nm])


def _global_dt(o):
    sc = o.scalars()
    t = torch.tensor([sc["dt"]], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MIN)
    return float(t.item()), sc


def _rank(rank, world, port, name, nsteps):
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from kaiju_b200 import gamera as gm, tiling as tl
        from oracle.pyoracle import Oracle
        P = PROBLEMS[name]
        Nip, Njp, Nkp = P["n"]
        m = gm.Model(Nip, Njp, Nkp)
        kind, bds, amp = P["corners"]
        xyz = gm.corners_warped(m, bds, amp) if kind == "warped" else gm.corners_uniform(m, bds)
        tiles = tl.split_k(Nkp, world)
        k0, nk = tiles[rank]
        kw = dict(P["kw"])
        gbc = kw.pop("bc")
        periodic = gbc[4] == 0 and gbc[5] == 0
        o = Oracle(Nip, Njp, nk, bc=tl.tile_bcs(gbc, rank, world), xyz=tl.tile_corners(xyz, k0, nk), **kw)
        ref = Oracle(Nip, Njp, Nkp, bc=gbc, xyz=xyz, **kw)
        # set-up: halos of State and oState (Bxyz included, as the undecomposed set-up leaves it), global dt
        _exchange(o, rank, world, tiles, periodic, ("magflux", "gas", "bxyz"))
        _exchange(o, rank, world, tiles, periodic, ("omagflux", "ogas", "obxyz"))
        dt, sc = _global_dt(o)
        o.set_scalars(sc["t"], dt, sc["dt0"], sc["time"], sc["time"] - dt, sc["ts"])
        assert abs(dt - ref.scalars()["dt"]) <= 1e-15 * dt
        for _ in range(nsteps):
            o.step()
            ref.step()
            dt, sc = _global_dt(o)
            o.set_scalars(sc["t"], dt, sc["dt0"], sc["time"], sc["otime"], sc["ts"])
            _exchange(o, rank, world, tiles, periodic, ("magflux", "gas", "bxyz"))
            o.bflux2fld()
            if periodic:
                assert abs(dt - ref.scalars()["dt"]) <= 1e-14 * dt
            else:
                assert dt == ref.scalars()["dt"]
        G = 4
        for nm, face in (("gas", False), ("bxyz", False), ("magflux", True)):
            a, b = o.get(nm), ref.get(nm)
            act = (slice(G, G + Nip), slice(G, G + Njp))
            mine = a[act + (slice(G, G + nk),)]
            theirs = b[act + (slice(G + k0, G + k0 + nk),)]
            if periodic:
                # Across a periodic K boundary the last tile takes the wrap-around face ke+1 from the first
                # tile's face ks, as the reference's MPI exchange does; the undecomposed periodic BC keeps
                # its own face ke+1. Both are the same face from the same stencil values, equal to rounding.
                scale = max(np.abs(theirs).max(), 1.0)
                assert np.abs(mine - theirs).max() <= 1e-13 * scale, (rank, nm, np.abs(mine - theirs).max())
            else:
                assert np.array_equal(mine, theirs), (rank, nm, np.abs(mine - theirs).max())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["bw", "ot"])
def test_two_tiles_match_single_domain(oracle_lib, name):
    mp.spawn(_rank, args=(2, _free_port(), name, 4), nprocs=2, join=True)
