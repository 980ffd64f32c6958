"""Host-side mirror of the reference's GPU entry points for the PIC step.

The reference's drop-in boundary is the set of argument-less subroutines that
``src/MAIN.F90`` calls under ``#ifdef gpu``; they act on module globals.
``Simulation`` owns one ``pic_handle`` (the device state those globals
describe) and exposes each of those subroutines under its reference name,
with a snake_case alias.  Arrays cross the boundary in the reference's layout:
fields are Fortran-ordered ``(mx, my, mz)`` float64 arrays with 2 low and 3
high ghost layers, particles are the SoA ``q,x,y,z,u,v,w`` (float64) and
``flv`` (int32) with absolute local cell coordinates.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _capi
from ._capi import check, dptr, iptr


def init_scale(c: float, c_ompe: float, epc: float, g0: float = 1.0, mi_me: float = 1.0) -> dict:
    """InitScale (src/init/initialise.F90:44-53) plus the default species
    table of AllocatePrtlVars (initialise.F90:84-87): flavour 1 = ions
    (q/m = 1/mi), flavour 2 = electrons (q/m = -1)."""
    me, mi = 1.0, mi_me
    ompe = c / c_ompe
    qi = (g0 * (ompe * ompe)) / ((float(epc) / 1.0) * (1.0 + me / mi))
    qe = -qi
    return {"ompe": ompe, "qi": qi, "qe": qe, "qmi": 1.0 / mi, "qme": -1.0,
            "masse": abs(qe) * me, "massi": qi * mi}


@dataclass
class PicConfig:
    """Runtime form of parameters.F90 (grid, Courant number, species, periods)."""

    nx: int
    ny: int
    nz: int = 1
    dims: int = 2
    c: float = 0.45
    qi: float = 1.0
    qm: tuple = (1.0, -1.0)
    fdtd: str = "yee"
    precision: str = "fp64"
    geom: str = "cartesian"
    bext: tuple = (0.0, 0.0, 0.0)
    reorder_period: int = 20
    curr_filter: int = 0
    capacity: int = 1 << 20
    rmin: float = 0.0
    inc_axis: int = 1
    brick: tuple = (0, 0, 0)   # FP32 form: brick shape in cells, (0, 0, 0) = from the fill
    cyl_modes: int = 0         # cylindrical: 0 = theta-gridded field solve, 2 = modes m = 0, 1
    slab_x: int = 0            # 1 = one slab of a domain split along x (pictor_b200.slab)
    exact_current: int = 0     # FP64: 1 = current summed in the reference's serial order (bit-exact J)
    fp64_tiles: int = 0        # FP64 mover after a reorder: 0 or 1 = by tiles, -1 = per particle
    exact_charge: int = 0      # FP32 3D: 1 = exactly charge-conserving deposit, 0 = the reference's weights

    def to_struct(self) -> _capi.Config:
        s = _capi.Config()
        s.nx, s.ny, s.nz = self.nx, self.ny, (self.nz if self.dims == 3 else 1)
        s.dims = self.dims
        s.geom = _capi.GEOM[self.geom]
        s.fdtd = _capi.FDTD[self.fdtd]
        s.precision = _capi.PRECISION[self.precision]
        s.nflvr = len(self.qm)
        s.c, s.qi = self.c, self.qi
        for d in range(3):
            s.bext[d] = self.bext[d]
        for i, v in enumerate(self.qm):
            s.qm[i + 1] = v
        s.reorder_period = self.reorder_period
        s.curr_filter = self.curr_filter
        s.capacity = int(self.capacity)
        s.rmin = self.rmin
        s.inc_axis = self.inc_axis
        for d in range(3):
            s.brick[d] = int(self.brick[d])
        s.cyl_modes = int(self.cyl_modes)
        s.slab_x = int(self.slab_x)
        s.exact_current = int(self.exact_current)
        s.fp64_tiles = int(self.fp64_tiles)
        s.exact_charge = int(self.exact_charge)
        return s

    @property
    def shape(self):
        return (self.nx + 5, self.ny + 5, (self.nz + 5) if self.dims == 3 else 1)


@dataclass
class Particles:
    """Reference-layout particle arrays (vars.F90:43-45)."""

    q: np.ndarray
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    flv: np.ndarray

    NAMES = ("q", "x", "y", "z", "u", "v", "w", "flv")

    @classmethod
    def empty(cls, n: int) -> "Particles":
        return cls(*(np.zeros(n) for _ in range(7)), np.zeros(n, dtype=np.int32))

    def __len__(self):
        return len(self.x)


@dataclass
class Fields:
    """Fortran-ordered (mx,my,mz) float64 field arrays."""

    Ex: np.ndarray
    Ey: np.ndarray
    Ez: np.ndarray
    Bx: np.ndarray
    By: np.ndarray
    Bz: np.ndarray
    Jx: np.ndarray = field(default=None)
    Jy: np.ndarray = field(default=None)
    Jz: np.ndarray = field(default=None)

    @classmethod
    def zeros(cls, shape) -> "Fields":
        return cls(*(np.zeros(shape, order="F") for _ in range(9)))


class Simulation:
    """One single-rank periodic PIC run on the GPU (one pic_handle)."""

    def __init__(self, cfg: PicConfig):
        self.cfg = cfg
        self.L = _capi.lib()
        h = C.c_void_p()
        check(self.L.pic_create(C.byref(cfg.to_struct()), C.byref(h)), "pic_create")
        self.h = h

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self.L.pic_destroy(self.h)
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

    # -- host <-> device (InitAll_gpu, CopyGPUDataToHostForOutput) ----------
    def load_fields(self, f: Fields) -> None:
        check(self.L.pic_load_fields(self.h, dptr(f.Ex), dptr(f.Ey), dptr(f.Ez), dptr(f.Bx), dptr(f.By), dptr(f.Bz)),
              "pic_load_fields")

    def load_current(self, Jx: np.ndarray, Jy: np.ndarray, Jz: np.ndarray) -> None:
        check(self.L.pic_load_current(self.h, dptr(Jx), dptr(Jy), dptr(Jz)), "pic_load_current")

    def fetch_fields(self, with_current: bool = True, out: Fields | None = None) -> Fields:
        """The fields in the reference layout; into the arrays of ``out`` when
        given (Fortran-ordered float64 of the grid's shape, e.g. views of
        pinned buffers, which the device writes at the full link rate)."""
        f = out if out is not None else Fields.zeros(self.cfg.shape)
        names = ("Ex", "Ey", "Ez", "Bx", "By", "Bz") + (("Jx", "Jy", "Jz") if with_current else ())
        for n in names:
            a = getattr(f, n)
            if a.shape != tuple(self.cfg.shape) or a.dtype != np.float64 or not a.flags["F_CONTIGUOUS"]:
                raise ValueError(f"fetch_fields: {n} must be a Fortran-ordered float64 array of shape {self.cfg.shape}")
        J = (dptr(f.Jx), dptr(f.Jy), dptr(f.Jz)) if with_current else (None, None, None)
        check(self.L.pic_fetch_fields(self.h, dptr(f.Ex), dptr(f.Ey), dptr(f.Ez), dptr(f.Bx), dptr(f.By), dptr(f.Bz), *J),
              "pic_fetch_fields")
        return f

    def load_particles(self, p: Particles) -> None:
        arrs = [np.ascontiguousarray(getattr(p, k), dtype=np.float64) for k in Particles.NAMES[:7]]
        flv = np.ascontiguousarray(p.flv, dtype=np.int32)
        check(self.L.pic_load_particles(self.h, len(flv), *[dptr(a) for a in arrs], iptr(flv)), "pic_load_particles")

    def particle_count(self) -> int:
        n = C.c_int64()
        check(self.L.pic_particle_count(self.h, C.byref(n)), "pic_particle_count")
        return n.value

    def fetch_particles(self) -> Particles:
        n = self.particle_count()
        p = Particles.empty(n)
        got = C.c_int64()
        check(self.L.pic_fetch_particles(self.h, C.byref(got), *[dptr(getattr(p, k)) for k in Particles.NAMES[:7]],
                                         iptr(p.flv)), "pic_fetch_particles")
        return p

    def init_weibel(self, epc: float, density: float, drift: float, temp_ion: float, temp_elc: float,
                    seed: int = 2930) -> int:
        """InitSetup of setup_weibel.F90 generated on the device (Philox-4x32-10)."""
        check(self.L.pic_init_weibel(self.h, epc, density, drift, temp_ion, temp_elc, seed), "pic_init_weibel")
        return self.particle_count()

    # -- phases of MAIN.F90 (reference names) -------------------------------
    def UpdateBfieldHalfGPU(self):
        """em_update_gpu.F90:44 + SendRecvFlds(B)."""
        check(self.L.pic_update_b_half(self.h), "pic_update_b_half")

    def MoveDepositPrtlGPU(self):
        """movdep_gpu.F90:14-49 (J cleared first, as ResetCurrent leaves it)."""
        check(self.L.pic_move_deposit(self.h), "pic_move_deposit")

    def ExchangePrtlGPU(self):
        """LoadPrtlOutliers + AppendParticles on one periodic rank."""
        check(self.L.pic_exchange_particles(self.h), "pic_exchange_particles")

    def UpdateEfieldGPU(self):
        """em_update_gpu.F90:12-42 + SendRecvFlds(E)."""
        check(self.L.pic_update_e(self.h), "pic_update_e")

    def UpdateCurrentsAllEdgesGPU(self):
        """UpdateCurrentAllFaces (comm_fld.F90:15-33): fold ghost J onto images."""
        check(self.L.pic_fold_current(self.h), "pic_fold_current")

    def smoothen_current_gpu(self):
        """smoothen_current (current.F90:19-30): curr_filter filter passes."""
        check(self.L.pic_filter_current(self.h), "pic_filter_current")

    def AddCurrentGPU(self):
        """em_update_gpu.F90:92-109 + EMfldExchangeGPU."""
        check(self.L.pic_add_current(self.h), "pic_add_current")

    def ResetCurrentGPU(self):
        check(self.L.pic_reset_current(self.h), "pic_reset_current")

    def ReorderPrtlGPU(self):
        """ReorderPrtlArr (mem_prtl.F90:166-301): stable cell-key sort (FP64
        form); the FP32 form groups the particles by brick instead."""
        check(self.L.pic_reorder(self.h), "pic_reorder")

    def RefBC_Prtl_x(self, side: int, pos: float):
        """RefBC_Prtl_Left (side 0) / RefBC_Prtl_Right (side 1), bc_reflect.F90:135-237:
        particles beyond the wall at pos mirrored, the current beyond it folded back."""
        check(self.L.pic_bc_reflect_x(self.h, int(side), float(pos)), "pic_bc_reflect_x")

    def CondBC_Fld_x(self, side: int, pos: float):
        """CondBC_Fld_Left (side 0) / CondBC_Fld_Right (side 1), bc_reflect.F90:43-72."""
        check(self.L.pic_bc_conducting_x(self.h, int(side), float(pos)), "pic_bc_conducting_x")

    def RefBC_Prtl_y(self, side: int, pos: float):
        """RefBC_Prtl_Bottom (side 0) / RefBC_Prtl_Top (side 1), bc_reflect.F90:79-128."""
        check(self.L.pic_bc_reflect_y(self.h, int(side), float(pos)), "pic_bc_reflect_y")

    def CondBC_Fld_y(self, side: int, pos: float):
        """CondBC_Fld_Bottom (side 0) / CondBC_Fld_Top (side 1), bc_reflect.F90:11-41."""
        check(self.L.pic_bc_conducting_y(self.h, int(side), float(pos)), "pic_bc_conducting_y")

    def RemovePrtl(self, face: int, pos: float):
        """RemovePrtl_Left / Right (bc_open.F90:8-62) at face 1..6 (x, y, z; low, high)."""
        check(self.L.pic_bc_remove(self.h, int(face), float(pos)), "pic_bc_remove")

    def Attenuate_EM_Vacuum(self, faces: dict):
        """Attenuate_EM_Vacuum (bc_attenuate.F90:151-290) for the faces of type
        'attn': ``faces`` maps bc_face index 1..6 to (pos_fld, attn_scale)."""
        mask = 0
        pos = (C.c_double * 6)()
        sc = (C.c_double * 6)(*([1.0] * 6))
        for n, (p, s) in faces.items():
            mask |= 1 << (int(n) - 1)
            pos[int(n) - 1] = float(p)
            sc[int(n) - 1] = float(s)
        check(self.L.pic_bc_attenuate(self.h, mask, pos, sc), "pic_bc_attenuate")

    def SetBC_PML(self, faces: dict):
        """The faces of type 'pml' (SetBC_Fld, bc.F90:45-50; bc_pml.F90):
        ``faces`` maps bc_face index 1..6 to (pos_fld, attn_thickness), the
        thickness 4 by default; an empty dict switches the PML off.  The
        auxiliary grids are zeroed on the first call and kept by later ones."""
        mask = 0
        pos = (C.c_double * 6)()
        th = (C.c_double * 6)(*([4.0] * 6))
        for n, v in faces.items():
            p, t = (v, 4.0) if isinstance(v, (int, float)) else v
            mask |= 1 << (int(n) - 1)
            pos[int(n) - 1] = float(p)
            th[int(n) - 1] = float(t)
        check(self.L.pic_bc_pml(self.h, mask, pos, th), "pic_bc_pml")

    def UpdateMagFld_PML(self):
        """UpdateMagFld_PML + SendRecvFlds(B), after the second B half step."""
        check(self.L.pic_bc_pml_b(self.h), "pic_bc_pml_b")

    def UpdateElcFld_PML(self):
        """UpdateElcFld_PML + SendRecvFlds(E), after the E update."""
        check(self.L.pic_bc_pml_e(self.h), "pic_bc_pml_e")

    def Attenuate_EM_Flow(self, face: int, pos: float, thickness: float = 1.0, scale: float = 4.0,
                          bflow=(0.0, 0.0, 0.0), drift=(0.0, 0.0, 0.0)):
        """Attenuate_EM_Flow (bc_attenuate.F90:16-131) of an 'iflw' face 1..4
        with a uniform flow (MagFld = bflow, DriftVelocity = drift); the
        defaults are SetBC_InflowFld's (bc.F90:163-205)."""
        b = (C.c_double * 3)(*map(float, bflow))
        v = (C.c_double * 3)(*map(float, drift))
        check(self.L.pic_bc_attenuate_flow(self.h, int(face), float(pos), float(thickness), float(scale), b, v),
              "pic_bc_attenuate_flow")

    def OpenBC_Fld_x(self, side: int, pos: float):
        """OpenBC_Fld_Left (side 0) / OpenBC_Fld_Right (side 1), bc.F90:411-469."""
        check(self.L.pic_bc_open_x(self.h, int(side), float(pos)), "pic_bc_open_x")

    def OpenBC_Prtl_x(self, side: int, pos: float):
        """OpenBC_Prtl_Left (side 0) / OpenBC_Prtl_Right (side 1), bc.F90:478-621,
        with dx = 1: particles beyond pos removed, the layer inside mirrored
        and appended with the column's mean x velocity taken out."""
        check(self.L.pic_bc_open_prtl_x(self.h, int(side), float(pos)), "pic_bc_open_prtl_x")

    update_b_half = UpdateBfieldHalfGPU
    move_deposit = MoveDepositPrtlGPU
    exchange_particles = ExchangePrtlGPU
    update_e = UpdateEfieldGPU
    fold_current = UpdateCurrentsAllEdgesGPU
    filter_current = smoothen_current_gpu
    add_current = AddCurrentGPU
    reset_current = ResetCurrentGPU
    reorder = ReorderPrtlGPU

    def set_sync(self, sync: bool = True) -> None:
        """False: the phase calls only enqueue their work on the handle's
        stream (``stream``); True (the default) waits and checks device errors."""
        check(self.L.pic_set_sync(self.h, 1 if sync else 0), "pic_set_sync")

    def step(self, nsteps: int = 1) -> None:
        """nsteps full steps of MAIN.F90:42-284 as one CUDA graph per step."""
        check(self.L.pic_step(self.h, int(nsteps)), "pic_step")

    def set_step(self, t: int) -> None:
        check(self.L.pic_set_step(self.h, int(t)), "pic_set_step")

    def diagnostics(self, masse: float = 1.0) -> dict:
        n = 4 + len(self.cfg.qm)
        out = np.zeros(n)
        check(self.L.pic_diagnostics(self.h, masse, dptr(out), n), "pic_diagnostics")
        return {"B2": out[0], "E2": out[1], "Benergy": 0.5 * out[0], "Eenergy": 0.5 * out[1],
                "gauss_linf": out[2], "rho_max": out[3], "kinetic": out[4:].copy()}

    def InflowBC_Prtl(self, face: int, pos: float, species, epc: float, density: float = 1.0,
                      drift=(0.0, 0.0, 0.0), speed: float = 0.0, vmax: float = 1.0, seed: int = 1, call: int = 0):
        """InjectNewPrtl (bc_inflow.F90:134-256) at the 'iflw' face 1..6 for a
        uniform density and drift; ``species`` lists (flv, temperature, charge)."""
        f = _capi.Inflow()
        f.face, f.pos, f.speed, f.vmax, f.epc, f.density = int(face), float(pos), float(speed), float(vmax), \
            float(epc), float(density)
        for d in range(3):
            f.drift[d] = float(drift[d])
        f.nspecies = len(species)
        for k, (fl, tp, q) in enumerate(species):
            f.flv[k], f.temp[k], f.charge[k] = int(fl), float(tp), float(q)
        f.seed, f.call = int(seed) & 0xFFFFFFFF, int(call) & 0xFFFFFFFF
        check(self.L.pic_bc_inflow(self.h, C.byref(f)), "pic_bc_inflow")

    def RefPrtlFluidFrameRight(self, pos: float, drift_x: float):
        """RefPrtlFluidFrameRight (bc_inflow.F90:62-121) at the right
        injector pos for the uniform flow drift_x, with its current."""
        check(self.L.pic_bc_inflow_reflect(self.h, float(pos), float(drift_x)), "pic_bc_inflow_reflect")

    def solve_gauss(self, tol: float = 1e-12, max_iter: int = 20000) -> dict:
        """The initial electrostatic field (pic_solve_gauss): E = -grad(phi)
        with the Gauss residual's node divergence equal to the particles' CIC
        density minus its mean; FP64 conjugate gradients on the device."""
        it = C.c_int32()
        rr, mean = C.c_double(), C.c_double()
        check(self.L.pic_solve_gauss(self.h, float(tol), int(max_iter), C.byref(it), C.byref(rr), C.byref(mean)),
              "pic_solve_gauss")
        return {"iters": it.value, "rel_residual": rr.value, "rho_mean": mean.value}

    def profile(self, enable: bool = True) -> None:
        check(self.L.pic_profile(self.h, 1 if enable else 0), "pic_profile")

    def phase_times(self) -> dict:
        """Summed device milliseconds and kernel launches per phase of the
        profiled pic_step calls (resets the accumulators)."""
        n = len(_capi.PHASES)
        ms = np.zeros(n)
        launches = np.zeros(n, dtype=np.int64)
        steps = C.c_int64()
        check(self.L.pic_phase_times(self.h, dptr(ms), launches.ctypes.data_as(_capi.PI64), n, C.byref(steps)),
              "pic_phase_times")
        return {"steps": steps.value, "ms": dict(zip(_capi.PHASES, ms)), "launches": dict(zip(_capi.PHASES, launches))}

    def launch_count(self) -> int:
        n = C.c_int64()
        check(self.L.pic_launch_count(self.h, C.byref(n)), "pic_launch_count")
        return n.value

    def device_errors(self) -> int:
        b = C.c_int32()
        check(self.L.pic_device_errors(self.h, C.byref(b)), "pic_device_errors")
        return b.value

    @property
    def stream(self) -> int:
        return self.L.pic_stream(self.h)


def step_many(sims, nsteps: int = 1, per_phase: bool = False, persistent: bool = False,
              spin_limit: int = 0, force_timeout: bool = False) -> None:
    """pic_step_many: nsteps steps of every simulation of an ensemble, their
    step graphs interleaved on their own streams so that small runs overlap
    on the GPU (all on the current device).  per_phase: pic_step_batched,
    one launch per phase for each group of runs (FP32, all reordered).
    persistent: pic_step_persistent, one persistent launch per span of steps
    between reorders (same requirements); spin_limit bounds every wait of
    its work items (0: about a second) and force_timeout makes the first
    wait run out (a test of that bound)."""
    sims = list(sims)
    if not sims:
        return
    L = sims[0].L
    arr = (C.c_void_p * len(sims))(*[s.h.value for s in sims])
    if persistent:
        check(L.pic_step_persistent(arr, len(sims), int(nsteps), int(spin_limit), int(bool(force_timeout))),
              "pic_step_persistent")
    elif per_phase:
        check(L.pic_step_batched(arr, len(sims), int(nsteps)), "pic_step_batched")
    else:
        check(L.pic_step_many(arr, len(sims), int(nsteps)), "pic_step_many")
