"""Uneven ensembles on one GPU.

The members (domains of different sizes, each with its own initial state) live
in pooled device arrays, and one library state advances all of them: every
kernel of the short step (numerical filter, the four RK4 stages, halo and
boundary fills) covers all members in a single launch, and the short-step
sequence can be recorded once as a CUDA graph and replayed. With
persistent=True the whole short step is ONE cooperative launch
(scale_hevi_short_step_persistent_dev) whose CTAs take the blocks of each
phase in turn and meet at bounded grid barriers between the phases. This has no
counterpart in the reference, where each member is a separate run of
scale-rm; per member the arithmetic is that of the single-domain short step
(scale_atmos_dyn_tinteg_short_rk4.F90, scale_atmos_dyn_tstep_short_fvm_hevi.F90),
so a member advanced in the ensemble is bit-identical to the same member
advanced alone.

Pooled layout (the library's): a 3-D field holds member m's (KA,IA,JA) array
at point cell0[m]; component q of a multi-component array at
q*cell0[n] + cell0[m]; 2-D fields at col0[m]; 1-D z/x/y vectors at
z0[m]/x0[m]/y0[m] with KA/IA/JA slots per member.
"""
from __future__ import annotations

import numpy as np

from . import hevi, mkinit

STATE = ("DENS", "MOMZ", "MOMX", "MOMY", "RHOT")
TENDENCIES = ("DENS_t", "MOMZ_t", "MOMX_t", "MOMY_t", "RHOT_t")


class Ensemble:
    """Members given as mkinit.Case objects (same time step, filter coefficient
    and flux schemes), resident on cuda:0 from construction to close()."""

    def __init__(self, cases: list, mixed: bool = False, device: int = 0, persistent: bool = False):
        import torch

        c0 = cases[0]
        for c in cases:
            if (c.dt, c.nd_coef, c.scheme, c.scheme_tracer) != (c0.dt, c0.nd_coef, c0.scheme, c0.scheme_tracer):
                raise ValueError(f"{c.name}: members must share dt, ND_COEF and the flux schemes")
        self.cases, self.mixed, self.persistent = cases, mixed, persistent
        self.dt, self.nd_coef = c0.dt, c0.nd_coef
        self.shapes = [c.g.shape for c in cases]
        self.layout = L = hevi.ensemble_setup([c.g.index_dict() for c in cases], c0.scheme, c0.scheme_tracer, device)
        self.n3 = int(L["cell0"][-1])
        self.n2 = int(L["col0"][-1])
        cuda = torch.device("cuda", device)
        dev = lambda x: torch.from_numpy(x).to(cuda)  # noqa: E731
        cell0, col0 = L["cell0"], L["col0"]
        self.X = {n: dev(hevi.pool([c.state[n] for c in cases], cell0)) for n in STATE}
        prep = [mkinit.large_prep(c) for c in cases]
        self.RT2P = dev(hevi.pool([p[0] for p in prep], cell0))
        self.DPRES0 = dev(hevi.pool([p[1] for p in prep], cell0))
        self.REF_rhot = dev(hevi.pool([p[2] for p in prep], cell0))
        self.ref = {k: dev(hevi.pool([c.ref[k] for c in cases], cell0)) for k in ("REF_dens", "REF_pott", "PHI")}
        ft = torch.float32 if mixed else torch.float64
        z = lambda k=1: torch.zeros(k * self.n3, dtype=ft, device=cuda)  # noqa: E731
        self.mflx, self.tflx, self.num_diff = z(3), z(3), z(15)
        self.tend = {n: z() for n in TENDENCIES}
        self.GSQRT = torch.ones(7 * self.n3, dtype=torch.float64, device=cuda)
        self.J0 = torch.zeros(7 * self.n3, dtype=torch.float64, device=cuda)
        self.MAPF = torch.ones(8 * self.n2, dtype=torch.float64, device=cuda)
        self.CORIOLI = torch.zeros(self.n2, dtype=torch.float64, device=cuda)
        KA = [c.g.KA for c in cases]
        IA = [c.g.IA for c in cases]
        JA = [c.g.JA for c in cases]

        def vec(name, off, slots):
            return hevi.pool([getattr(c.g, name) for c in cases], L[off], slots=slots)

        self.grid = {n: vec(n, "z0", KA) for n in ("CDZ", "FDZ", "RCDZ", "RFDZ")}
        self.grid.update({n: vec(n, "x0", IA) for n in ("CDX", "FDX", "RCDX", "RFDX")})
        self.grid.update({n: vec(n, "y0", JA) for n in ("CDY", "FDY", "RCDY", "RFDY")})
        self.wdamp = np.zeros(int(L["z0"][-1]))
        self._graph = False

    # ---- one short step: numerical filter, RK4, boundary values and halos ----
    def step(self) -> None:
        gr = self.grid
        if self.persistent:
            # the whole step as one persistent launch over all members
            fn = hevi.short_step_persistent_mixed_dev if self.mixed else hevi.short_step_persistent_dev
            fn(mflx_hi=self.mflx, tflx_hi=self.tflx, num_diff=self.num_diff, DPRES0=self.DPRES0, RT2P=self.RT2P,
               CORIOLI=self.CORIOLI, wdamp_coef=self.wdamp, REF_dens=self.ref["REF_dens"],
               REF_pott=self.ref["REF_pott"], REF_rhot=self.REF_rhot, ND_COEF=self.nd_coef, ND_SFC_FACT=1.0,
               dt=self.dt, **self.X, **self.tend, **gr)
            return
        nf = hevi.ATMOS_DYN_numfilter_coef_mixed_dev if self.mixed else hevi.ATMOS_DYN_numfilter_coef_dev
        rk = hevi.ATMOS_DYN_Tinteg_short_rk4_mixed_dev if self.mixed else hevi.ATMOS_DYN_Tinteg_short_rk4_dev
        nf(num_diff=self.num_diff, CDZ=gr["CDZ"], CDX=gr["CDX"], CDY=gr["CDY"], FDZ=gr["FDZ"], FDX=gr["FDX"],
           FDY=gr["FDY"], DT=self.dt, REF_dens=self.ref["REF_dens"], REF_pott=self.ref["REF_pott"],
           ND_COEF=self.nd_coef, ND_ORDER=1, ND_SFC_FACT=1.0, ND_USE_RS=True, **self.X)
        rk(PROG=None, mflx_hi=self.mflx, tflx_hi=self.tflx, DPRES0=self.DPRES0, RT2P=self.RT2P,
           CORIOLI=self.CORIOLI, num_diff=self.num_diff, wdamp_coef=self.wdamp, divdmp_coef=0.0, DDIV=None,
           FLAG_FCT_MOMENTUM=False, FLAG_FCT_T=False, FLAG_FCT_ALONG_STREAM=True, PHI=self.ref["PHI"],
           GSQRT=self.GSQRT, J13G=self.J0, J23G=self.J0, J33G=1.0, MAPF=self.MAPF, REF_dens=self.ref["REF_dens"],
           REF_rhot=self.REF_rhot, BND_W=False, BND_E=False, BND_S=False, BND_N=False, dt=self.dt,
           **self.X, **self.tend, **{k: gr[k] for k in ("CDZ", "FDZ", "FDX", "FDY", "RCDZ", "RCDX", "RCDY", "RFDZ",
                                                        "RFDX", "RFDY")})
        hevi.boundary_dev(**self.X)

    def capture(self, steps: int = 1) -> None:
        """Record `steps` short steps as a CUDA graph (one eager step first
        completes the one-time table uploads; it advances the state)."""
        self.step()
        hevi.capture_begin()
        try:
            for _ in range(steps):
                self.step()
        finally:
            hevi.capture_end()
        self._graph = True

    def run(self, nsteps: int) -> None:
        """Advance nsteps short steps: graph replays when captured (nsteps a
        multiple of the captured steps is the caller's business), else eager."""
        if self._graph:
            hevi.replay(nsteps)
        else:
            for _ in range(nsteps):
                self.step()

    def members(self) -> list[dict[str, np.ndarray]]:
        """The members' state arrays on the host, each in its own (KA,IA,JA) shape."""
        hevi.check()
        per = {n: hevi.unpool(self.X[n].cpu().numpy(), self.layout["cell0"], self.shapes) for n in STATE}
        return [{n: per[n][m] for n in STATE} for m in range(len(self.cases))]

    def close(self) -> None:
        hevi.finalize()
