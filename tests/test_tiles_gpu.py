"""A problem split along k into tiles on the device (gam_tiles_* and the split-step pieces) must advance
exactly like the undecomposed problem: the tiles exchange 4-layer halos and take the minimum dt every step
(the reference's MPI tiling, gamapp_mpi.F90:501-794). The tiles run the same kernels on the same values as
the single domain, so zero-gradient problems match bit for bit; across a periodic K boundary the last tile
takes the wrap-around face from the first tile (as the reference's MPI exchange does) where the single
domain keeps its own copy, the same face from the same stencil values, so those match to rounding."""
import ctypes as C
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
G = 4
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _case(name):
    from kaiju_b200 import gamera as gm
    if name == "bw":   # warped blast wave, zero-gradient everywhere
        m = gm.Model(32, 16, 16, CFL=0.3, bc=(gm.GAM_BC_ZEROGRAD,) * 6, tFin=1e30)
        return m, gm.corners_warped(m, (-0.5, 0.5) * 3, 0.04), "BW"
    if name == "ot":   # Orszag-Tang slab, periodic everywhere
        m = gm.Model(32, 32, 8, CFL=0.3, bc=(gm.GAM_BC_PERIODIC,) * 6, tFin=1e30)
        return m, gm.corners_uniform(m, (0.0, 1.0, 0.0, 1.0, 0.0, 1.0 / 32)), "OT2D"
    raise ValueError(name)


def _single(name, fp32=False):
    from kaiju_b200 import gamera as gm
    m, xyz, ic = _case(name)
    g = gm.GameraGPU.from_corners(m, xyz, ic)
    if fp32:
        g.set_precision(gm.GAM_FP32FLUX)
    return g


def _compare(tiles, split, ref, periodic, what):
    from kaiju_b200 import tiling as tl
    m = ref.model
    act = (slice(G, G + m.Nip), slice(G, G + m.Njp), slice(G, G + m.Nkp))
    for nm in ("gas", "bxyz", "magflux"):
        mine = tl.stitch([t.fetch(nm) for t in tiles], split, face=(nm == "magflux"))[act]
        theirs = ref.fetch(nm)[act]
        if periodic:
            scale = max(np.abs(theirs).max(), 1.0)
            assert np.abs(mine - theirs).max() <= 1e-13 * scale, (what, nm, np.abs(mine - theirs).max())
        else:
            assert np.array_equal(mine, theirs), (what, nm, np.abs(mine - theirs).max())
    dts = [t.status()["dt"] for t in tiles]
    assert len(set(dts)) == 1, dts
    if periodic:
        assert abs(dts[0] - ref.status()["dt"]) <= 1e-13 * dts[0]
    else:
        assert dts[0] == ref.status()["dt"]
    assert all(t.status()["ts"] == ref.status()["ts"] for t in tiles)


@pytest.mark.parametrize("name,ntiles,fp32", [("bw", 2, False), ("bw", 3, False), ("ot", 2, False),
                                              ("bw", 2, True)])
def test_tile_group_matches_single_domain(name, ntiles, fp32):
    from kaiju_b200 import gamera as gm, tiling as tl
    m, xyz, ic = _case(name)
    ref = _single(name, fp32)
    tiles, split = tl.make_tiles(m, xyz, ntiles, ic, fp32=fp32)
    periodic = tl.periodic_k(m)
    with gm.TileGroup(tiles, periodic_k=periodic) as grp:
        _compare(tiles, split, ref, periodic, "set-up")
        grp.run_steps(6)
        ref.run_steps(6)
        _compare(tiles, split, ref, periodic, "6 steps")
        grp.run_steps(6)
        ref.run_steps(6)
        _compare(tiles, split, ref, periodic, "12 steps")


def _split_step(tiles, words, lo_up):
    """One step of every tile through the split-step pieces, halos moved between device buffers here."""
    import torch
    from kaiju_b200 import gamera as gm
    L = gm.load_library()
    for t, w in zip(tiles, words):
        assert L.gam_gpu_step_local(t.h, w.data_ptr()) == 0
    torch.cuda.synchronize()
    red = torch.stack(words).min(dim=0).values
    for w in words:
        w.copy_(red)
    torch.cuda.synchronize()
    for t, w in zip(tiles, words):
        assert L.gam_gpu_step_bcs(t.h, w.data_ptr()) == 0
    _exchange(tiles, gm.GAM_HALO_STATE, lo_up)
    for t in tiles:
        assert L.gam_gpu_step_ghosts(t.h) == 0


def _exchange(tiles, what, lo_up):
    import torch
    from kaiju_b200 import gamera as gm
    L = gm.load_library()
    torch.cuda.synchronize()
    msgs = {}
    for q, t in enumerate(tiles):
        for side, nb in enumerate(lo_up[q]):
            if nb is None:
                continue
            sb, rb = C.c_longlong(), C.c_longlong()
            assert L.gam_gpu_halo_bytes(t.h, side, what, C.byref(sb), C.byref(rb)) == 0
            buf = torch.empty(sb.value // 8, dtype=torch.float64, device="cuda")
            assert L.gam_gpu_halo_pack(t.h, side, what, buf.data_ptr()) == 0
            msgs[(q, side)] = buf
    torch.cuda.synchronize()
    for q, t in enumerate(tiles):
        for side, nb in enumerate(lo_up[q]):
            if nb is None:
                continue
            buf = msgs[(nb, side ^ 1)]   # the neighbour's message towards this tile
            sb, rb = C.c_longlong(), C.c_longlong()
            assert L.gam_gpu_halo_bytes(t.h, side, what, C.byref(sb), C.byref(rb)) == 0
            assert rb.value == buf.numel() * 8
            assert L.gam_gpu_halo_unpack(t.h, side, what, buf.data_ptr()) == 0
    torch.cuda.synchronize()


@pytest.mark.parametrize("name", ["bw", "ot"])
def test_split_step_pieces_match_single_domain(name):
    import torch
    from kaiju_b200 import gamera as gm, tiling as tl
    m, xyz, ic = _case(name)
    ref = _single(name)
    tiles, split = tl.make_tiles(m, xyz, 2, ic)
    periodic = tl.periodic_k(m)
    lo_up = [tl.neighbours(q, 2, periodic) for q in range(2)]
    L = gm.load_library()
    words = [torch.zeros(2, dtype=torch.int64, device="cuda") for _ in tiles]
    _exchange(tiles, gm.GAM_HALO_STATE | gm.GAM_HALO_OSTATE | gm.GAM_HALO_BXYZ, lo_up)
    for t, w in zip(tiles, words):
        assert L.gam_gpu_calcdt_local(t.h, w.data_ptr()) == 0
    torch.cuda.synchronize()
    red = torch.stack(words).min(dim=0).values
    for t, w in zip(tiles, words):
        w.copy_(red)
        torch.cuda.synchronize()
        assert L.gam_gpu_calcdt_finish(t.h, w.data_ptr()) == 0
    _compare(tiles, split, ref, periodic, "set-up")
    for _ in range(8):
        _split_step(tiles, words, lo_up)
    ref.run_steps(8)
    _compare(tiles, split, ref, periodic, "8 steps")
    # out-of-order calls are refused, not run
    assert L.gam_gpu_step_bcs(tiles[0].h, words[0].data_ptr()) == gm.GAM_ERR_ARG
    assert L.gam_gpu_step_ghosts(tiles[0].h) == gm.GAM_ERR_ARG


def test_tile_arguments_are_checked():
    from kaiju_b200 import gamera as gm, tiling as tl
    m, xyz, ic = _case("bw")
    tiles, _ = tl.make_tiles(m, xyz, 2, ic)
    L = gm.load_library()
    arr = (C.c_void_p * 2)(tiles[0].h.value, tiles[0].h.value)
    g = C.c_void_p()
    assert L.gam_tiles_create(C.byref(g), arr, 2, 0) == gm.GAM_ERR_ARG        # the same tile twice
    arr = (C.c_void_p * 2)(tiles[1].h.value, tiles[0].h.value)
    assert L.gam_tiles_create(C.byref(g), arr, 2, 0) == gm.GAM_ERR_ARG        # out of k order
    arr = (C.c_void_p * 2)(tiles[0].h.value, tiles[1].h.value)
    assert L.gam_tiles_create(C.byref(g), arr, 2, 1) == gm.GAM_ERR_ARG        # periodic, but ends not halos
    # a halo face on a ring-averaged or 2.5D problem is refused
    with pytest.raises(gm.GamError):
        bad = gm.Model(32, 16, 1, bc=(1, 1, 1, 1, gm.GAM_BC_HALO, gm.GAM_BC_HALO))
        gm.GameraGPU.from_corners(bad, gm.corners_uniform(bad, (0, 1, 0, 1, 0, 1)), "OT2D")


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _dist_rank(rank, world, port, name, nsteps):
    import sys
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from kaiju_b200 import gamera as gm, tiling as tl
        m, xyz, ic = _case(name)
        periodic = tl.periodic_k(m)
        k0, nk, tm = tl.tile_models(m, world)[rank]
        tile = gm.GameraGPU.from_corners(tm, tl.tile_corners(xyz, k0, nk), ic)
        dt = tl.DistTile(tile, rank, world, periodic, staging=True)
        dt.setup()
        for _ in range(nsteps):
            assert dt.step() == 0
        ref = _single(name)
        ref.run_steps(nsteps)
        for nm in ("gas", "bxyz", "magflux"):
            a, b = tile.fetch(nm), ref.fetch(nm)
            mine = a[G:G + m.Nip, G:G + m.Njp, G:G + nk]
            theirs = b[G:G + m.Nip, G:G + m.Njp, G + k0:G + k0 + nk]
            if periodic:
                assert np.abs(mine - theirs).max() <= 1e-13 * max(np.abs(theirs).max(), 1.0), (rank, nm)
            else:
                assert np.array_equal(mine, theirs), (rank, nm, np.abs(mine - theirs).max())
        tile.close()
        ref.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name", ["bw", "ot"])
def test_process_per_tile_over_torch_distributed(name):
    """Two processes, one tile each, on the one GPU: the host moves halos and the dt words with
    torch.distributed (gloo through host copies). No kernel of one rank waits on the other."""
    import torch.multiprocessing as mp
    mp.start_processes(_dist_rank, args=(2, _free_port(), name, 6), nprocs=2, join=True, start_method="spawn")
