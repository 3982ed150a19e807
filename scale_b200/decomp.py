"""2-D decomposition of a periodic domain over ranks, with the lateral halo
exchange that replaces COMM_vars8/COMM_wait (scale_comm_cartesC.F90:1600-2043,
2787-3023) when the domain is split.

The global domain of IMAX_G x JMAX_G interior columns is cut into
PRC_NUM_X x PRC_NUM_Y equal subdomains; rank r holds the subdomain at
(r % PRC_NUM_X, r // PRC_NUM_X), the rank layout of scale_prc_cartesC. Each
rank keeps its own (KA,IA,JA) arrays with the usual halo and runs the library
on them; the library calls the exchange below at every halo fill
(scale_hevi_set_halo_exchange).

The exchange runs in two phases, as a periodic fill of the global domain
would: first along x (the IHALO interior columns next to each lateral edge of
the interior rows go to the west and east neighbours), then along y (JHALO
whole rows, the x halo included, go to the south and north neighbours), which
also fills the corners. A neighbour that is the rank itself (one subdomain
along a direction) is a local copy. The transfers are torch.distributed
point-to-point operations on the fields' own device: NCCL between GPUs, gloo
on CPU tensors.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch


@dataclass(frozen=True)
class Decomposition:
    imax_g: int  # interior columns of the global domain along x
    jmax_g: int  # ... along y
    nx: int  # PRC_NUM_X
    ny: int  # PRC_NUM_Y
    rank: int
    halo: int = 2  # IHALO = JHALO

    def __post_init__(self):
        if self.nx < 1 or self.ny < 1 or not 0 <= self.rank < self.nx * self.ny:
            raise ValueError(f"rank {self.rank} is outside a {self.nx} x {self.ny} layout")
        if self.imax_g % self.nx or self.jmax_g % self.ny:
            raise ValueError(f"{self.imax_g} x {self.jmax_g} columns do not divide over {self.nx} x {self.ny} ranks")
        if self.imax_g // self.nx < self.halo or self.jmax_g // self.ny < self.halo:
            raise ValueError("a subdomain must be at least as wide as the halo")

    # ---- geometry ----
    @property
    def px(self) -> int:
        return self.rank % self.nx

    @property
    def py(self) -> int:
        return self.rank // self.nx

    @property
    def imax(self) -> int:
        return self.imax_g // self.nx

    @property
    def jmax(self) -> int:
        return self.jmax_g // self.ny

    @property
    def i0(self) -> int:
        """Global index (0-based, interior) of this subdomain's first column."""
        return self.px * self.imax

    @property
    def j0(self) -> int:
        return self.py * self.jmax

    def neighbour(self, dx: int, dy: int) -> int:
        """Rank of the periodic neighbour dx subdomains east and dy north."""
        return (self.px + dx) % self.nx + self.nx * ((self.py + dy) % self.ny)

    def local_of(self, glob):
        """This rank's (KA, IA, JA) block of a halo-filled global array
        (KA, IMAX_G + 2H, JMAX_G + 2H), halo included."""
        H = self.halo
        return glob[:, self.i0: self.i0 + self.imax + 2 * H, self.j0: self.j0 + self.jmax + 2 * H]

    # ---- the exchange ----
    def exchange(self, fields, group=None) -> None:
        """Fill the lateral halo of every field in place. A field is a tensor
        whose memory is a Fortran (KA,IA,JA) array of this subdomain: shape
        (JA, IA, KA) in torch's row-major order, or flat."""
        import torch.distributed as dist

        H, I, J = self.halo, self.imax, self.jmax
        IA, JA = I + 2 * H, J + 2 * H
        views = [f.view(JA, IA, -1) for f in fields]
        # phase 1, x: interior rows; phase 2, y: whole rows (corners included)
        phases = (
            ((1, 0), lambda v: v[H:H + J, I:I + H], lambda v: v[H:H + J, 0:H],         # east strip -> west halo of the east neighbour
             (-1, 0), lambda v: v[H:H + J, H:2 * H], lambda v: v[H:H + J, I + H:IA]),  # west strip -> east halo of the west neighbour
            ((0, 1), lambda v: v[J:J + H, :], lambda v: v[0:H, :],
             (0, -1), lambda v: v[H:2 * H, :], lambda v: v[J + H:JA, :]),
        )
        for fwd, send_f, recv_f, bwd, send_b, recv_b in phases:
            to_f, from_f = self.neighbour(*fwd), self.neighbour(-fwd[0], -fwd[1])
            to_b, from_b = self.neighbour(*bwd), self.neighbour(-bwd[0], -bwd[1])
            out_f = torch.stack([send_f(v) for v in views]).contiguous()
            out_b = torch.stack([send_b(v) for v in views]).contiguous()
            if to_f == self.rank:  # one subdomain along this direction: periodic in itself
                in_f, in_b = out_f, out_b
            else:
                in_f, in_b = torch.empty_like(out_f), torch.empty_like(out_b)
                ops = [dist.P2POp(dist.isend, out_f, to_f, group, 1), dist.P2POp(dist.irecv, in_f, from_f, group, 1),
                       dist.P2POp(dist.isend, out_b, to_b, group, 2), dist.P2POp(dist.irecv, in_b, from_b, group, 2)]
                for w in dist.batch_isend_irecv(ops):
                    w.wait()
            for q, v in enumerate(views):
                recv_f(v).copy_(in_f[q])
                recv_b(v).copy_(in_b[q])


class _DeviceField:
    """A raw device array exposed through __cuda_array_interface__."""

    def __init__(self, ptr: int, shape, elem_bytes: int):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8" if elem_bytes == 8 else "<f4",
                                         "data": (int(ptr), False), "version": 3, "strides": None}


def attach(lib, dec: Decomposition, KA: int, group=None) -> None:
    """Make dec's exchange the halo fill of the library `lib` (scale_b200.hevi),
    whose state was set up for this rank's subdomain of KA levels."""
    H = dec.halo
    shape = (dec.jmax + 2 * H, dec.imax + 2 * H, KA)

    def exchange(ptrs, nfields, elem_bytes):
        fields = [torch.as_tensor(_DeviceField(p, shape, elem_bytes), device="cuda") for p in ptrs]
        dec.exchange(fields, group)
        torch.cuda.synchronize()

    lib.set_halo_exchange(exchange)


def budget_sums(partials, group=None) -> list[float]:
    """The domain totals of a decomposed domain's budgets: every rank gives its
    subdomain's FP64 partial sums (scale_hevi_domain_sum_dev for the mass,
    scale_hevi_energy_sum_dev for ENGT/ENGP/ENGK/ENGI, the reference's
    MONITOR totals of scale_atmos_dyn.F90:530-688 and mod_atmos_vars.F90:768-777,
    which reduce over ranks with MPI_ALLREDUCE). The partials are gathered and
    added in rank order on every rank, so every rank holds the same bits
    whatever the transport does (a reduction inside the transport may
    associate the additions differently from one call to the next)."""
    import torch.distributed as dist

    v = torch.tensor([float(x) for x in partials], dtype=torch.float64)
    if dist.get_backend(group) == "nccl":
        v = v.cuda()
    world = dist.get_world_size(group)
    got = [torch.empty_like(v) for _ in range(world)]
    dist.all_gather(got, v, group)
    tot = [0.0] * len(partials)
    for r in range(world):  # rank order
        row = got[r].cpu().tolist()
        for q in range(len(tot)):
            tot[q] += row[q]
    return tot


def domain_budgets(lib, X, grid, group=None) -> dict[str, float]:
    """Mass and energy totals of the decomposed domain from this rank's state X
    (DENS, MOMZ, MOMX, MOMY, RHOT device arrays of its subdomain) and its grid
    vectors (CZ, CDZ, CDX, CDY)."""
    mass = lib.domain_sum_dev(X["DENS"], grid["CDZ"], grid["CDX"], grid["CDY"])
    eng = lib.energy_sum_dev(**X, CZ=grid["CZ"], CDZ=grid["CDZ"], CDX=grid["CDX"], CDY=grid["CDY"])
    names = ("ENGT", "ENGP", "ENGK", "ENGI")
    tot = budget_sums([mass] + [eng[n] for n in names], group)
    return {"mass": tot[0], **{n: tot[1 + q] for q, n in enumerate(names)}}
