"""The 2-D decomposition and its halo exchange (scale_b200/decomp.py), which
replaces COMM_vars8 of one periodic rank when the domain is split: with gloo
ranks on the CPU, every rank's halo after the exchange must equal the same
cells of the global domain filled periodically, for a 2x1 layout with a halo
of 2 and a 2x2 layout with a halo of 3; one rank is the periodic fill itself."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from scale_b200.decomp import Decomposition  # noqa: E402

KA = 7


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _global_field(imax_g, jmax_g, H, seed):
    """A periodic-filled global (KA, IA, JA) array in Fortran order."""
    rng = np.random.Generator(np.random.PCG64(seed))
    a = np.asfortranarray(rng.standard_normal((KA, imax_g + 2 * H, jmax_g + 2 * H)))
    IS, IE, JS, JE = H, H + imax_g, H, H + jmax_g
    a[:, :IS, :] = a[:, IE - H:IE, :]
    a[:, IE:, :] = a[:, IS:IS + H, :]
    a[:, :, :JS] = a[:, :, JE - H:JE]
    a[:, :, JE:] = a[:, :, JS:JS + H]
    return a


def _run_exchange(dec, nfields, seed):
    """Rank dec.rank's fields after the exchange, and the expected blocks."""
    got, want = [], []
    fields = []
    for q in range(nfields):
        g = _global_field(dec.imax_g, dec.jmax_g, dec.halo, seed + q)
        loc = np.asfortranarray(dec.local_of(g))
        want.append(loc.copy(order="F"))
        H = dec.halo
        garbled = loc.copy(order="F")
        garbled[:, :H, :] = np.nan
        garbled[:, -H:, :] = np.nan
        garbled[:, :, :H] = np.nan
        garbled[:, :, -H:] = np.nan
        fields.append(torch.from_numpy(np.ravel(garbled, order="F").copy()))
    dec.exchange(fields)
    for f, w in zip(fields, want):
        got.append(f.numpy().reshape(w.shape, order="F"))
    return got, want


def _worker(rank, world, port, nx, ny, imax_g, jmax_g, halo, out):
    import datetime

    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dec = Decomposition(imax_g, jmax_g, nx, ny, rank, halo)
        got, want = _run_exchange(dec, 3, 11)
        out[rank] = all(np.array_equal(g, w) for g, w in zip(got, want))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nx,ny,halo", [(2, 1, 2), (2, 2, 3)])
def test_exchange_matches_global_periodic_fill(nx, ny, halo):
    world = nx * ny
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, world, port, nx, ny, 12, 10, halo, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert all(out[r] for r in range(world)), dict(out)


@pytest.mark.parametrize("halo", [2, 3])
def test_single_rank_exchange_is_the_periodic_fill(halo):
    dec = Decomposition(9, 7, 1, 1, 0, halo)
    got, want = _run_exchange(dec, 2, 5)
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


def test_layout_and_neighbours():
    dec = Decomposition(16, 12, 4, 3, 5)  # rank 5 = (1, 1)
    assert (dec.px, dec.py, dec.imax, dec.jmax, dec.i0, dec.j0) == (1, 1, 4, 4, 4, 4)
    assert dec.neighbour(1, 0) == 6 and dec.neighbour(-1, 0) == 4
    assert dec.neighbour(0, 1) == 9 and dec.neighbour(0, -1) == 1
    assert Decomposition(16, 12, 4, 3, 0).neighbour(-1, -1) == 11  # periodic wrap to (3, 2)
    with pytest.raises(ValueError):
        Decomposition(15, 12, 4, 3, 0)
    with pytest.raises(ValueError):
        Decomposition(16, 12, 4, 3, 12)
