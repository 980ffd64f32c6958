"""The differentiable form of the 2D step (pic_adj_* of include/pictor_b200.h).

Objective: J = sum over steps t of 1/2 sum over cells |B_t|^2 (the
time-integrated magnetic energy, CalcFldEnergy of savedata_routines.F90:310-326
times 1/2, summed over the run).  ``Adjoint.gradient`` returns dJ with respect
to every initial momentum (and position) and to the Weibel loader's drift and
per-species temperatures, from hand-written adjoint kernels run backwards
over the checkpointed forward run.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _capi
from ._capi import check, dptr, iptr
from .simulation import Particles, PicConfig


class Adjoint:
    def __init__(self, cfg: PicConfig):
        if cfg.dims != 2:
            raise ValueError("the differentiable form is 2D")
        self.cfg = cfg
        self.L = _capi.lib()
        h = C.c_void_p()
        check(self.L.pic_adj_create(C.byref(cfg.to_struct()), C.byref(h)), "pic_adj_create")
        self.h = h
        self.drift = 0.0
        self.temp = (0.0, 0.0)
        self.nsteps = 0

    def close(self):
        if getattr(self, "h", None):
            self.L.pic_adj_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_weibel(self, epc: float, density: float, drift: float, temp_ion: float, temp_elc: float,
                    seed: int) -> int:
        """Initial particles of pic_init_weibel with the same arguments (same
        seed, same particles); fields start at zero."""
        n = C.c_int64()
        check(self.L.pic_adj_init_weibel(self.h, epc, density, drift, temp_ion, temp_elc, seed, C.byref(n)),
              "pic_adj_init_weibel")
        self.drift, self.temp = drift, (temp_ion, temp_elc)
        return n.value

    def load_particles(self, p: Particles, drift_sign: np.ndarray | None = None) -> None:
        sgn = None if drift_sign is None else np.ascontiguousarray(drift_sign, dtype=np.float64)
        check(self.L.pic_adj_load_particles(self.h, len(p.x), dptr(p.q), dptr(p.x), dptr(p.y), dptr(p.z), dptr(p.u),
                                            dptr(p.v), dptr(p.w), iptr(p.flv), None if sgn is None else dptr(sgn)),
              "pic_adj_load_particles")

    def fetch_particles(self) -> tuple[Particles, np.ndarray]:
        """The initial particles (reference layout) and their drift signs."""
        n = C.c_int64()
        check(self.L.pic_adj_fetch_particles(self.h, C.byref(n), None, None, None, None, None, None, None, None, None),
              "pic_adj_fetch_particles")
        p = Particles.empty(n.value)
        sgn = np.zeros(n.value)
        check(self.L.pic_adj_fetch_particles(self.h, C.byref(n), dptr(p.q), dptr(p.x), dptr(p.y), dptr(p.z),
                                             dptr(p.u), dptr(p.v), dptr(p.w), iptr(p.flv), dptr(sgn)),
              "pic_adj_fetch_particles")
        return p, sgn

    def branches(self, mode: str) -> None:
        """'free' (default), 'record' the mover's discrete decisions in the
        next forward runs, or 'replay' them (pic_adj_branches)."""
        check(self.L.pic_adj_branches(self.h, {"free": 0, "record": 1, "replay": 2}[mode]), "pic_adj_branches")

    def forward(self, nsteps: int, checkpoint_every: int = 50) -> float:
        """J of nsteps steps from the initial state (state kept every
        checkpoint_every steps for the reverse sweep)."""
        obj = C.c_double()
        check(self.L.pic_adj_forward(self.h, int(nsteps), int(checkpoint_every), C.byref(obj)), "pic_adj_forward")
        self.nsteps = nsteps
        return obj.value

    def gradient(self, drift: float | None = None, temp: tuple | None = None) -> dict:
        """dJ/d(initial u, v, w, x, y) per particle and dJ/d(drift, temp_ion,
        temp_elc) of the last forward run."""
        n = C.c_int64()
        check(self.L.pic_adj_fetch_particles(self.h, C.byref(n), None, None, None, None, None, None, None, None, None),
              "pic_adj_fetch_particles")
        n = n.value
        out = {k: np.zeros(n) for k in ("u", "v", "w", "x", "y")}
        par = np.zeros(3)
        t = np.asarray(temp if temp is not None else self.temp, dtype=np.float64)
        check(self.L.pic_adj_gradient(self.h, float(self.drift if drift is None else drift), dptr(t), dptr(out["u"]),
                                      dptr(out["v"]), dptr(out["w"]), dptr(out["x"]), dptr(out["y"]), dptr(par)),
              "pic_adj_gradient")
        out["drift"], out["temp_ion"], out["temp_elc"] = float(par[0]), float(par[1]), float(par[2])
        return out
