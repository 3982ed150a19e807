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


# ---- the dynamics on a decomposed domain: oracle RK4 stages per subdomain ----
STATE = ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")


def _local_inputs(dec, g_glob, a):
    """This rank's block of every input array (3-D and 2-D by its lateral
    block, 1-D lateral vectors by its slice, the rest as they are)."""
    H = dec.halo
    isl = slice(dec.i0, dec.i0 + dec.imax + 2 * H)
    jsl = slice(dec.j0, dec.j0 + dec.jmax + 2 * H)
    out = {}
    for k, v in a.items():
        if not isinstance(v, np.ndarray):
            out[k] = v
        elif v.ndim >= 3 and v.shape[:3] == g_glob.shape:
            out[k] = np.asfortranarray(v[:, isl, jsl])
        elif v.ndim >= 2 and v.shape[:2] == (g_glob.IA, g_glob.JA):
            out[k] = np.asfortranarray(v[isl, jsl])
        elif v.ndim == 1 and len(v) == g_glob.IA and k.endswith("X"):
            out[k] = v[isl].copy()
        elif v.ndim == 1 and len(v) == g_glob.JA and k.endswith("Y"):
            out[k] = v[jsl].copy()
        else:
            out[k] = v
    return out


def _rk4_decomposed(dec, g_loc, x, a, dt):
    """ATMOS_DYN_tinteg_short_rk4 (rk4.F90:376-650) with the oracle's stage on
    this rank's subdomain and dec.exchange in place of COMM_vars8."""
    import helpers
    import oracle

    x0 = {n: v.copy(order="F") for n, v in x.items()}
    rk, fl, cur = [], [], {n: x0[n] for n in STATE}
    for s, dtrk in enumerate((dt / 2.0, dt / 2.0, dt, dt)):
        o = helpers.stage_outputs(g_loc, 0.0)
        args = dict(a, dtrk=dtrk)
        args.update({n + "0": x0[n] for n in STATE})
        args.update(cur)
        if s == 3:
            o["mflx_hi"] = x0["mflx_hi"].copy(order="F")
            o["tflx_hi"] = x0["tflx_hi"].copy(order="F")
        oracle.tstep_short(g_loc, "CD4", o, args)
        st = {n: o[n + "_RK"] for n in STATE}
        if s < 3:
            t = [torch.from_numpy(np.ravel(st[n], order="F").copy()) for n in STATE]
            dec.exchange(t)
            st = {n: t[q].numpy().reshape(g_loc.shape, order="F").copy(order="F") for q, n in enumerate(STATE)}
        rk.append(st)
        fl.append((o["mflx_hi"], o["tflx_hi"]))
        cur = st
    g = g_loc
    sl = (slice(g.KS - 1, g.KE), slice(g.IS - 1, g.IE), slice(g.JS - 1, g.JE))
    for n in STATE:
        ks = slice(g.KS - 1, g.KE - 1) if n == "MOMZ" else sl[0]
        comb = (rk[0][n] * 2.0 + rk[1][n] * 4.0 + rk[2][n] * 2.0 + rk[3][n] - x0[n] * 3.0) / 6.0
        x[n][ks, sl[1], sl[2]] = comb[ks, sl[1], sl[2]]
    for f, name in enumerate(("mflx_hi", "tflx_hi")):
        comb = (fl[0][f] + fl[1][f] * 2.0 + fl[2][f] * 2.0 + fl[3][f]) / 6.0
        x[name][sl] = comb[sl]
    return x


def _dyn_worker(rank, world, port, nx, ny, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT / "tests"))
    import helpers
    import oracle

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        g = helpers.small_grid(IMAX=12, JMAX=10, KMAX=12)
        c = helpers.small_case(g, "CD4")
        helpers.perturb_state(c)
        a = helpers.short_inputs(c, full=True)
        for k in ("DENS0", "MOMZ0", "MOMX0", "MOMY0", "RHOT0", "DENS", "MOMZ", "MOMX", "MOMY", "RHOT", "dtrk"):
            a.pop(k)
        xg = {n: c.state[n].copy(order="F") for n in STATE}
        xg["mflx_hi"], xg["tflx_hi"] = g.zeros(3), g.zeros(3)
        dec = Decomposition(g.IMAX, g.JMAX, nx, ny, rank, g.halo)
        g_loc = helpers.small_grid(IMAX=dec.imax, JMAX=dec.jmax, KMAX=12)
        xl = {n: np.asfortranarray(v[:, dec.i0: dec.i0 + dec.imax + 4, dec.j0: dec.j0 + dec.jmax + 4])
              for n, v in xg.items()}
        al = _local_inputs(dec, g, a)
        oracle.tinteg_short_rk4(g, "CD4", xg, dict(a, dt=1.0))  # the global run
        _rk4_decomposed(dec, g_loc, xl, al, 1.0)
        ok = True
        for n in xl:
            glob = xg[n][:, dec.i0 + 2: dec.i0 + 2 + dec.imax, dec.j0 + 2: dec.j0 + 2 + dec.jmax]
            ok &= bool(np.array_equal(xl[n][:, 2:-2, 2:-2], glob))
        out[rank] = ok
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_decomposed_rk4_matches_global_run():
    """The RK4 short step on a 2x1 decomposition, each rank running the
    oracle's stage on its subdomain and exchanging the stage buffers, equals
    the global run on every rank's interior, bit for bit."""
    world, nx, ny = 2, 2, 1
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_dyn_worker, args=(r, world, port, nx, ny, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        assert all(out[r] for r in range(world)), dict(out)


# ---- exchanges inside the oracle's own call sequences: the FCT limiter's R+/R-
# (scale_atmos_dyn_common.F90:2526-2561) and the filter's work arrays at
# ND_ORDER > 1 (:1557-1563), through og_set_halo_exchange ----
def _block(dec, g, v):
    """This rank's block (halo included) of a global array: 3-D and more by its
    lateral block, (IA,JA) 2-D arrays likewise."""
    H = dec.halo
    isl = slice(dec.i0, dec.i0 + dec.imax + 2 * H)
    jsl = slice(dec.j0, dec.j0 + dec.jmax + 2 * H)
    if v.ndim >= 3 and v.shape[:3] == g.shape:
        return np.asfortranarray(v[:, isl, jsl])
    return np.asfortranarray(v[isl, jsl])


def _interior_equal(dec, g, glob, loc):
    H = dec.halo
    want = glob[:, dec.i0 + H: dec.i0 + H + dec.imax, dec.j0 + H: dec.j0 + H + dec.jmax]
    return bool(np.array_equal(loc[:, H:-H, H:-H], want))


def _inner_worker(rank, world, port, nx, ny, what, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT / "tests"))
    import helpers
    import oracle

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        g = helpers.small_grid(IMAX=12, JMAX=10, KMAX=12, stretched=True)
        c = helpers.small_case(g, "CD4")
        helpers.perturb_state(c)
        dec = Decomposition(g.IMAX, g.JMAX, nx, ny, rank, g.halo)
        g_loc = helpers.small_grid(IMAX=dec.imax, JMAX=dec.jmax, KMAX=12, stretched=True)
        exchange = lambda fields: dec.exchange([torch.from_numpy(f) for f in fields])  # noqa: E731
        ok = True
        if what == "fct":
            from test_gpu_parity import _tracer_inputs

            q0, q, d0, d, mflx, rhoq, GS, MAPF = _tracer_inputs(g, c)
            ndq = np.asfortranarray(1e-6 * np.random.default_rng(9).normal(size=g.shape + (3,)))
            for n in range(3):
                oracle.halo(g, np.asfortranarray(ndq[..., n]))
            for along in (True, False):
                qg = q.copy(order="F")
                oracle.tinteg_tracer_rk3(g, "UD3", qg, q0, rhoq, d0, d, mflx, ndq, GS, MAPF, 5.0, True, along)
                ql = _block(dec, g, q)
                oracle.set_halo_exchange(g_loc, exchange)
                try:
                    oracle.tinteg_tracer_rk3(g_loc, "UD3", ql, _block(dec, g, q0), _block(dec, g, rhoq),
                                             _block(dec, g, d0), _block(dec, g, d), _block(dec, g, mflx),
                                             _block(dec, g, ndq), _block(dec, g, GS), _block(dec, g, MAPF), 5.0,
                                             True, along)
                finally:
                    oracle.set_halo_exchange(g_loc, None)
                ok &= _interior_equal(dec, g, qg, ql)
        else:  # the filter at ND_ORDER = 2 and 3
            for order in (2, 3):
                ndg = g.zeros(5, 3)
                oracle.numfilter(g, ndg, c.state, c.ref, DT=0.5, ND_COEF=1e-3, ND_ORDER=order, ND_SFC_FACT=0.7)
                ndl = g_loc.zeros(5, 3)
                st = {n: _block(dec, g, v) for n, v in c.state.items()}
                ref = {n: _block(dec, g, v) for n, v in c.ref.items() if isinstance(v, np.ndarray) and v.ndim >= 3}
                oracle.set_halo_exchange(g_loc, exchange)
                try:
                    oracle.numfilter(g_loc, ndl, st, ref, DT=0.5, ND_COEF=1e-3, ND_ORDER=order, ND_SFC_FACT=0.7)
                finally:
                    oracle.set_halo_exchange(g_loc, None)
                for v in range(5):
                    for dd in range(3):
                        ok &= _interior_equal(dec, g, ndg[..., v, dd], ndl[..., v, dd])
        out[rank] = ok
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("what", ["fct", "nd_order"])
def test_decomposed_limiter_and_filter_match_global_run(what):
    """The tracer RK3 with the FCT limiter (its R+/R- exchanged between the
    limiter's passes) and the numerical filter at ND_ORDER 2 and 3 (its work
    arrays exchanged between the calc_diff4 applications), each rank running
    the oracle on its subdomain of a 2x1 layout with every halo fill replaced
    by the exchange, equal the global runs on every rank's interior, bit for
    bit."""
    world, nx, ny = 2, 2, 1
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_inner_worker, args=(r, world, port, nx, ny, what, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        assert all(out[r] for r in range(world)), dict(out)


def _budget_worker(rank, world, port, nx, ny, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT / "tests"))
    import helpers
    import oracle
    from scale_b200.decomp import budget_sums

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        g = helpers.small_grid(IMAX=12, JMAX=10, KMAX=12, stretched=True)
        c = helpers.small_case(g, "CD4")
        helpers.perturb_state(c)
        dec = Decomposition(g.IMAX, g.JMAX, nx, ny, rank, g.halo)
        g_loc = helpers.small_grid(IMAX=dec.imax, JMAX=dec.jmax, KMAX=12, stretched=True)
        st = {n: _block(dec, g, v) for n, v in c.state.items()}
        names = ("ENGT", "ENGP", "ENGK", "ENGI")
        e_loc, e_glob = oracle.energy_sum(g_loc, st, g_loc.CZ), oracle.energy_sum(g, c.state, g.CZ)
        tot = budget_sums([oracle.domain_sum(g_loc, st["DENS"])] + [e_loc[n] for n in names])
        want = [oracle.domain_sum(g, c.state["DENS"])] + [e_glob[n] for n in names]
        # every rank holds the same bits
        allt = [None] * world
        dist.all_gather_object(allt, tot)
        out[rank] = {"same_on_ranks": all(t == tot for t in allt),
                     "rel": max(abs(a - b) / abs(b) for a, b in zip(tot, want))}
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("nx,ny", [(2, 1), (2, 2)])
def test_budget_sums_over_ranks(nx, ny):
    """The FP64 mass and energy totals of a decomposed domain (each rank's
    subdomain sum, gathered and added in rank order) are the same bits on
    every rank and agree with the global domain's sums to rounding."""
    world = nx * ny
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_budget_worker, args=(r, world, port, nx, ny, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        for r in range(world):
            assert out[r]["same_on_ranks"], dict(out)
            assert out[r]["rel"] <= 1e-13, dict(out)
