"""The moist large step composed from the oracle's operators - TEST
INFRASTRUCTURE ONLY.  The same phases, in the reference's large-step
schedule (src/cm1core/gm1_runtime.py:1969-2007), as the product's
composition, each phase calling the oracle restatement of the operator the
product calls there; left out identically: SGS stress and scalar diffusion,
Rayleigh damping, the dry-mass correction, surface fluxes.  A configuration
with a stretched column (cfg.column set) runs the flat (terrain_flag=.false.)
family on the column profiles its metrics carry."""

from __future__ import annotations

import numpy as np

from oracle import advection as oadv
from oracle import bridge as obr
from oracle import closure as ocl
from oracle import stress as ost
from oracle import kessler as oks
from oracle import moist_step as oms
from oracle import momentum as omom
from oracle import rk as ork
from oracle import terrain_open as otos
from oracle import tke as otke
from oracle import tke_evolution as otev
from oracle.periodic import REAL

NUMQ = 3
QMAG = 1.0e-2
EPS = 1.0e-18


def _f32(x):
    return float(np.float32(x))


def moisture_weps(r: int) -> float:
    return float(np.float32(np.float32(QMAG) * np.float32(EPS)))


def theta_weps() -> float:
    return float(np.float32(np.float32(10.0) * np.float32(EPS)))


# the column metrics the terrain texts of the SGS stress and turbs read
TERRAIN_METRICS = ("gz", "rgz", "gzu", "rgzu", "gzv", "rgzv", "gx", "gy", "gxu", "gyv")

class OracleMoistStep:
    def __init__(self, cfg, state: dict[str, np.ndarray], metrics: dict[str, np.ndarray]) -> None:
        self.cfg, self.s, self.m = cfg, state, metrics
        # CM1 apmasscon = 1 unless the configuration says otherwise; the
        # initial dry-air mass of the state unless it carries one
        self.apmasscon = bool(getattr(cfg, "apmasscon", True))
        if self.apmasscon:
            if "mass1" not in state:
                state["mass1"] = np.zeros(1, np.float64)
            if state["mass1"][0] == 0.0:
                state["mass1"][0] = oks.dry_mass(state["rho"], state["ruh"], state["rvh"], metrics["rmh"],
                                                 ni=cfg.ni, nj=cfg.nj, nk=cfg.nk)
        # the oracle's acoustic stage always writes its column diagnostics
        for n in ("tri_aa", "tri_bb", "tri_cc", "tri_dd", "tri_pivot", "tri_residual"):
            if state[n].shape != state["pp3d"].shape:
                state[n] = np.zeros(state["pp3d"].shape, REAL)
        self.k3 = dict(ni=cfg.ni, nj=cfg.nj, nk=cfg.nk)
        self.grid = dict(ni=cfg.ni, nj=cfg.nj, nk=cfg.nk, dx=cfg.dx, dy=cfg.dy, dz=cfg.dz)
        # a stretched column runs the flat (terrain_flag=.false.) family on
        # the column profiles of its metrics (the Cartesian stretched lane,
        # src/cm1core/cuda_cartesian_dynamics.py:1075-1104, :1148-1187,
        # :1220-1231, :1254-1269, :1293; cuda_cartesian_closure.py:1133-1141,
        # :1191-1197, :1658-1663)
        self.flat = getattr(cfg, "column", None) is not None
        # the SGS stress and scalar diffusion held tendencies (gettau +
        # turbu/turbv/turbw and turbs of the closure's held phase,
        # cuda_cartesian_closure.py:1268-1291): the flat texts on a
        # stretched column, the terrain texts (cpu_sgs_stress_tendency_inplace,
        # cpu_gm1_scalar_turbulence_inplace) on the uniform one
        self.sgs_diffusion = bool(getattr(cfg, "sgs_diffusion", False))
        # CM1's upper Rayleigh damping (irdamp = 1, solve1.F:412-454), its
        # coefficients and base-state winds from the metrics
        self.rayleigh = bool(getattr(cfg, "rayleigh", False))
        if self.sgs_diffusion or self.rayleigh:
            self.stress = ost.zeros(cfg.ni, cfg.nj, cfg.nk, ost.STRAIN_NAMES + ost.TAU_NAMES + ost.TENDENCY_NAMES)
        if self.flat:
            self.rdz = float(np.float32(np.float32(1.0) / np.float32(cfg.dz)))
            self.hx = dict(ni=cfg.ni, nj=cfg.nj, nk=cfg.nk, dx=cfg.dx, dy=cfg.dy)
            self.column = {"flat": True, "rho0p": metrics["rho0_padded"], "mh": metrics["mh_profile"],
                           "mf": metrics["mf_profile"], "rr0": metrics["rr0"], "rdz": self.rdz}

    def _pp3d_to_compact(self):
        c = self.cfg
        self.s["pp3d_c"][:] = self.s["pp3d"][1:c.nk + 1, 1:c.nj + 1, 1:c.ni + 1]

    def closure(self):
        s, m, c = self.s, self.m, self.cfg
        nk, nj, ni = c.nk, c.nj, c.ni
        s["uc"][:] = s["u3d"][1:nk + 1, 3:3 + nj, 3:4 + ni]
        s["vc"][:] = s["v3d"][1:nk + 1, 3:4 + nj, 3:3 + ni]
        s["wc"][:] = s["w3d"][1:nk + 2, 3:3 + nj, 3:3 + ni]
        self._pp3d_to_compact()
        ocl.moist_nm({"c1": m["c1"], "c2": m["c2"], "mf": m["mf"], "pi0": s["pi0"], "th0": s["th0"], "prs": s["prs"],
                      "pp3d": s["pp3d_c"], "th3d": s["th3d"], "q3d": s["q3d"], "nm": s["nm"],
                      "temperature": s["temperature"], "qt": s["qt"], "thv": s["thv_c"], "qvci": s["qvci"],
                      "saturation_mask": s["saturation_mask"]}, **self.k3, dz=c.dz)
        if self.flat:
            ocl.flat_calcdef({"u3d": s["uc"], "v3d": s["vc"], "w3d": s["wc"], "rho": s["rho"], "rf": s["rf"],
                              "mf": m["mf"], "c1": m["c1"], "c2": m["c2"], "mh_profile": m["mh_profile"],
                              "defv": s["defv"], "defh": s["defh"]}, **self.hx, rdz=self.rdz)
        else:
            ocl.calcdef({"u3d": s["uc"], "v3d": s["vc"], "w3d": s["wc"], "rho": s["rho"], "rf": s["rf"],
                         **{n: m[n] for n in ("c1", "c2", "gz", "rgz", "rgzu", "rgzv", "gx", "gy")},
                         "defv": s["defv"], "defh": s["defh"]}, **self.grid)
        otke.sgs_tke({"ruh": s["ruh"], "rvh": s["rvh"], "rmf": m["rmf"], **{n: s[n] for n in otke.NAMES
                                                                          if n not in ("ruh", "rvh", "rmf")}},
                     **self.grid)
        s["tke3d"][:] = s["tkea"]
        if self.flat:
            otev.tke_diffusion_flat(self._tke(), **self.hx, rdz=self.rdz, dt=c.dt)
        else:
            otev.tke_diffusion(self._tke(), **self.grid, dt=c.dt)
        if self.sgs_diffusion:
            self._held_stress()
        elif self.rayleigh:
            for n in ost.TENDENCY_NAMES:
                self.stress[n][:] = 0

    def _held_stress(self):
        """The held momentum tendencies: zero, then the SGS stress added
        (turbu/turbv/turbw into the zeroed tile tendencies; no Rayleigh
        damping, so uten1 = 0 and the held sum is the stress)."""
        s, m, c, st = self.s, self.m, self.cfg, self.stress
        for n in ost.TENDENCY_NAMES:
            st[n][:] = 0
        a = {"u3d": s["uc"], "v3d": s["vc"], "w3d": s["wc"], "rho": s["rho"], "rf": s["rf"], "mh": m["mh"],
             "mf": m["mf"], "kmh": s["kmh"], "kmv": s["kmv"], **st}
        if self.flat:
            ost.flat_sgs_stress({**a, "mh_profile": m["mh_profile"]}, **self.hx, rdz=self.rdz, dt=c.dt)
        else:
            ost.terrain_sgs_stress({**a, **{n: m[n] for n in TERRAIN_METRICS}}, **self.grid, dt=c.dt)

    def _tke(self):
        s, m = self.s, self.m
        return {"tkea": s["tkea"], "tke3d": s["tke3d"], "tketen": s["tketen"], "kmh": s["kmh"], "kmv": s["kmv"],
                "rho": s["rho"], "rf": s["rf"], "mh": m["mh"], "mf": m["mf"], "gz": m["gz"], "rgz": m["rgz"],
                "rgzu": m["rgzu"], "rgzv": m["rgzv"], "c1": m["c1"], "c2": m["c2"], "rrf0": m["rrf0"],
                "rru": s["rru"], "rrv": s["rrv"], "rrw": s["rrw"], "divx": s["divx"]}

    def held_tendencies(self):
        s, m, c = self.s, self.m, self.cfg
        s["thheld"][:] = 0
        s["qheld"][:] = 0
        if self.rayleigh:
            # added into the held momentum (uten1 + uten), assigned to thheld
            nk = c.nk
            a = {"tauh": m["tauh"], "taus": m["taus"], "tauf": m["tauf"], "u0": m["u0"], "v0": m["v0"],
                 "ua": s["uc"], "va": s["vc"], "wa": s["wc"][:nk], "tha": s["tha"], "uten1": self.stress["uten"],
                 "vten1": self.stress["vten"], "wten1": self.stress["wten"][:nk], "thten1": s["thheld"]}
            ost.rayleigh_held(a, ni=c.ni, nj=c.nj, nk=nk, rdalpha=getattr(c, "rayleigh_rdalpha", 3.3333333333e-3),
                              profiles=True, add_momentum=True)
        if getattr(c, "dissipative_heating", False):
            # idiss after the damping, before the subgrid turbulence
            ost.dissipative_heating({"dissten": s["dissten"], "pi0": s["pi0"], "ppi": s["pp3d_c"], "qa": s["qa"],
                                     "thten1": s["thheld"]}, **self.k3)
        if self.sgs_diffusion:
            # turbs for theta and the moisture rows into the held thten1/qten
            # the eqtset 2 composition then reads (solve1.F:1169-1233)
            a = {"th0": s["th0"], "tha": s["tha"], "qa": s["qa"], "rho": s["rho"], "rr": s["rr"], "rf": s["rf"],
                 "mh": m["mh"], "mf": m["mf"], "khh": s["khh"], "khv": s["khv"], "thten1": s["thheld"],
                 "qten": s["qheld"]}
            if self.flat:
                ost.flat_scalar_turbulence(a, **self.hx, numq=s["qheld"].shape[0], dz=c.dz, dt=c.dt)
            else:
                ost.terrain_scalar_turbulence({**a, **{n: m[n] for n in TERRAIN_METRICS}}, **self.grid,
                                              numq=s["qheld"].shape[0], dt=c.dt)
        oms.held_compose({"th0": s["th0_3d"], "pi0": s["pi0_3d"], "rho": s["rho"], "ppi": s["pp3d_c"],
                          "tha": s["tha"], "qa": s["qa"], "qpten": s["qpten"], "qtten": s["qtten"],
                          "qvten": s["qvten"], "qcten": s["qcten"], "thheld": s["thheld"], "qheld": s["qheld"],
                          "ppten": s["ppten"]}, **self.k3, dt=self.cfg.dt)

    def _mom(self):
        s, m = self.s, self.m
        return {n: (s[n] if n in s else m[n]) for n in omom.NAMES}

    def pre_acoustic(self, nrk):
        s, m, c = self.s, self.m, self.cfg
        obr.eqtset2_stage_terms(**self.k3, th0=s["th0"], qv0=s["qv0"], pi0=s["pi0"], th3d=s["th3d"], q3d=s["q3d"],
                                pp3d=s["pp3d"], thv=s["thv"], ppterm=s["ppterm"], buoyancy=s["dum8"],
                                thterm=s["thterm"], piadv=s["piadv"])
        oms.open_fill(s["thv"], "pressure", **self.k3)
        oms.open_fill(s["dum8"], "scalar", **self.k3)
        s["uten"][:] = 0
        s["vten"][:] = 0
        s["wten"][:] = 0
        if self.sgs_diffusion or self.rayleigh:
            # the held momentum seeds the stage tendencies' physical cells
            # (pack_cartesian_held_momentum, cuda_cartesian_dynamics.py:206)
            nk, nj, ni = c.nk, c.nj, c.ni
            s["uten"][1:nk + 1, 3:3 + nj, 3:4 + ni] = self.stress["uten"]
            s["vten"][1:nk + 1, 3:4 + nj, 3:3 + ni] = self.stress["vten"]
            s["wten"][1:nk + 2, 3:3 + nj, 3:3 + ni] = self.stress["wten"]
        if self.flat:
            omom.momentum_advection5_column(self._mom(), self.column, **self.hx, lateral_sides=c.lateral_sides)
            oms.moist_buoyancy_flat(s["dum8"], m["c1"], m["c2"], s["wten"], **self.k3)
            return
        if nrk >= 2:
            oms.bcwsfc(s["u3d"], s["v3d"], s["w3d"], m["gz"], m["dzdx"], m["dzdy"], **self.k3)
            oms.w_level1_fill(s["w3d"], **self.k3)
        a = self._mom()
        omom.momentum_advection5_phase(a, **self.grid, lateral_sides=c.lateral_sides, phase=1)
        oms.open_fill(s["rrw"], "w_keep_ends", **self.k3)
        omom.momentum_advection5_phase(a, **self.grid, lateral_sides=c.lateral_sides, phase=2)
        oms.moist_buoyancy(s["dum8"], m["c1"], m["c2"], m["gxu"], m["gyv"], s["uten"], s["vten"], s["wten"],
                           **self.k3)

    def acoustic(self, nrk):
        c = self.cfg
        if self.flat:
            otos.terrain_open_stage_flat(self.s, self.m, self.column, nrk=nrk, ni=c.ni, nj=c.nj, nk=c.nk, dt=c.dt,
                                         nsound=c.nsound, dx=c.dx, dy=c.dy, obc=c.obc, alph=_f32(c.alph),
                                         kdiv=_f32(c.kdiv), ablations=255 & ~128)
            return
        otos.terrain_open_stage(self.s, self.m, nrk=nrk, ni=c.ni, nj=c.nj, nk=c.nk, dt=c.dt, nsound=c.nsound,
                                dx=c.dx, dy=c.dy, dz=c.dz, alph=_f32(c.alph), kdiv=_f32(c.kdiv), ablations=255 & ~128)

    def post_acoustic(self, nrk):
        s, m = self.s, self.m
        a = {"rru": s["rru"], "rrv": s["rrv"], "rrw": s["rrw"], "rgzu": m["rgzu"], "rgzv": m["rgzv"],
             "dzdx": m["dzdx"], "dzdy": m["dzdy"], "gz": m["gz"], "rho0_3d": m["rho0_3d"], "rf0": m["rf0"],
             "thterm": s["thterm"], "divergence": s["divergence"], "theta_divergence_term": s["theta_div"],
             "divx": s["divx"]}
        if self.flat:
            oms.post_acoustic_flux_column(a, self.column, **self.hx)
        else:
            oms.post_acoustic_flux(a, **self.grid)

    def _advect(self, padded, tendency, nrk, weps):
        s, m, c = self.s, self.m, self.cfg
        a = {"scalar": padded, "rru": s["rru"], "rrv": s["rrv"], "rrw": s["rrw"], "c1": m["c1"], "c2": m["c2"],
             "rr0": m["rr0"], "gz": m["gz"], "divx": s["divx"], "tendency": tendency, "flux_x": s["fx"],
             "flux_y": s["fy"], "flux_z": s["fz"]}
        if self.flat:
            oadv.scalar_advection5_column(a, **self.hx, nrk=nrk, weps=weps, flat=True, profile=m["mh_profile"],
                                          rdz=self.rdz, lateral_obc=c.obc)
        else:
            oadv.scalar_advection5(a, **self.grid, nrk=nrk, weps=weps, lateral_obc=c.obc)

    def scalar_moist(self, nrk):
        s, m, c = self.s, self.m, self.cfg
        ork.theta_pack(s["th0"], s["th3d"], s["theta_padded"], **self.k3)
        oms.open_fill(s["theta_padded"], "scalar", **self.k3)
        s["theta_adv"][:] = 0
        self._advect(s["theta_padded"], s["theta_adv"], nrk, theta_weps())
        dttmp = ork.rk_stage_dt(c.dt, nrk)
        for r in range(NUMQ):
            oms.pack_scalar(s["q3d"][r], s["moisture_padded"], **self.k3)
            oms.open_fill(s["moisture_padded"], "scalar", **self.k3)
            s["moist_adv"][r] = 0
            if nrk < 3:
                self._advect(s["moisture_padded"], s["moist_adv"][r], nrk, moisture_weps(r))
            else:
                chain = {"scalar_a": s["qa"][r], "scalar_padded": s["moisture_padded"], "rho0_3d": m["rho0_3d"],
                         "gz": m["gz"], "rgz": m["rgz"], "rr0": m["rr0"], "c1": m["c1"], "c2": m["c2"],
                         "divx": s["divx"], "rru": s["rru"], "rrv": s["rrv"], "rrw": s["rrw"], "fx": s["fx"],
                         "fy": s["fy"], "fz": s["fz"], "advx": s["advx"], "advy": s["advy"], "advz": s["advz"],
                         "candidate": s["candidate"], "advection": s["moist_adv"][r]}
                if self.flat:
                    oms.pdef_moisture_chain_column(chain, **self.hx, dttmp=dttmp, weps=moisture_weps(r),
                                                   lateral_obc=c.obc, pdefweno=0 if r == 0 else 1, flat=True,
                                                   profile=m["mh_profile"], rdz=self.rdz)
                else:
                    oms.pdef_moisture_chain(chain, **self.grid, dttmp=dttmp, weps=moisture_weps(r),
                                            lateral_obc=c.obc, pdefweno=0 if r == 0 else 1)
        qa, q = s["qa"][:NUMQ], s["q3d"][:NUMQ]
        ork.compose(s["tha"], qa, s["thheld"], s["qheld"], s["theta_div"], s["theta_adv"], s["moist_adv"], s["th3d"],
                    q, nrk=nrk, dt=c.dt)

    def momentum_boundaries(self, nrk):
        s, m = self.s, self.m
        oms.open_fill(s["u3d"], "u", **self.k3)
        oms.open_fill(s["v3d"], "v", **self.k3)
        oms.open_fill(s["w3d"], "w", **self.k3)
        if not self.flat:
            oms.bcwsfc(s["u3d"], s["v3d"], s["w3d"], m["gz"], m["dzdx"], m["dzdy"], **self.k3)

    def scalar_boundaries(self, nrk):
        oms.open_fill(self.s["pp3d"], "pressure", **self.k3)

    def tke_rk(self, nrk):
        s = self.s
        if self.flat:
            otev.tke_rk_stage_flat(self._tke(), self.m["mf_profile"], s["tke3d"], s["tke_workspace"], **self.hx,
                                   nrk=nrk, rdz=self.rdz, dt=self.cfg.dt)
        else:
            otev.tke_rk_stage(self._tke(), s["tke3d"], s["tke_workspace"], **self.grid, nrk=nrk, dt=self.cfg.dt)
        s["tke3d"][:] = s["tke_workspace"]

    def microphysics(self):
        s, m, c = self.s, self.m, self.cfg
        self._pp3d_to_compact()
        a = {"ruh": s["ruh"], "rvh": s["rvh"], "rmh": m["rmh"], "mh": m["mh"], "pi0": s["pi0_3d"],
             "th0": s["th0_3d"], "rr": s["kessler_rr"], "rho": s["rho"], "pp3d": s["pp3d_c"], "th3d": s["th3d"],
             "prs": s["prs"], "qv": s["q3d"][0], "qc": s["q3d"][1], "qr": s["q3d"][2],
             "fall_velocity": s["fall_velocity"], "rain": s["rain"], "prate": s["prate"], "asq": s["asq"],
             "qbudget": s["qbudget"]}
        held = {"qpten": s["qpten"], "qtten": s["qtten"], "qvten": s["qvten"], "qcten": s["qcten"]}
        # with apmasscon the dry-air mass correction between the pre-physics
        # equation of state and the driver
        oks.kessler_large_step(a, held, **self.grid, dt=c.dt, eqtset=2,
                               mass1=s["mass1"] if self.apmasscon else None)
        s["pp3d"][1:c.nk + 1, 1:c.nj + 1, 1:c.ni + 1] = s["pp3d_c"]

    def solve3(self):
        s, m = self.s, self.m
        s["ppx"] += s["pp3d"]
        for cur, base in (("ua", "u3d"), ("va", "v3d"), ("wa", "w3d"), ("ppi", "pp3d"), ("tha", "th3d"),
                          ("qa", "q3d"), ("tkea", "tke3d")):
            s[cur][:] = s[base]
        oms.solve3_density(s["rho"], m["c1"], m["c2"], s["rr"], s["rf"], **self.k3)

    def step(self):
        self.closure()
        self.held_tendencies()
        for nrk in (1, 2, 3):
            self.pre_acoustic(nrk)
            self.acoustic(nrk)
            self.post_acoustic(nrk)
            self.scalar_moist(nrk)
            self.momentum_boundaries(nrk)
            if nrk < 3:
                self.scalar_boundaries(nrk)
            self.tke_rk(nrk)
        self.microphysics()
        self.solve3()
