"""ctypes front end of the CPU restatement in ``pictor_oracle.c``.

TEST INFRASTRUCTURE ONLY.  This module is the checker: ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline arm of ``bench.py`` import it;
the product package ``pictor_b200`` never does.

Parity of this restatement against the reference itself is unpinned (the
reference is Fortran and ships no tests, fixtures or golden vectors); it is
pinned to the hand-derived known-answer vectors in ``tests/golden``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
MAX_FLVR = 8


def build(quiet: bool = True) -> None:
    """Compile the serial and OpenMP restatements with the Makefile beside this file."""
    out = subprocess.run(["make", "-C", _HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


_libs: dict = {}


def lib(openmp: bool = False) -> C.CDLL:
    name = "libpictor_oracle_omp.so" if openmp else "libpictor_oracle.so"
    if name not in _libs:
        path = os.path.join(_BUILD, name)
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        _declare(L)
        _libs[name] = L
    return _libs[name]


class Grid(C.Structure):
    _fields_ = [
        ("dims", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("mx", C.c_int), ("my", C.c_int), ("mz", C.c_int),
        ("fdtd", C.c_int), ("nflvr", C.c_int),
        ("c", C.c_double), ("qi", C.c_double), ("bext", C.c_double * 3),
        ("flvrqm", C.c_double * (MAX_FLVR + 1)),
    ]


class _Particles(C.Structure):
    _fields_ = [
        ("q", C.POINTER(C.c_double)), ("x", C.POINTER(C.c_double)), ("y", C.POINTER(C.c_double)),
        ("z", C.POINTER(C.c_double)), ("u", C.POINTER(C.c_double)), ("v", C.POINTER(C.c_double)),
        ("w", C.POINTER(C.c_double)), ("flv", C.POINTER(C.c_int32)),
        ("used", C.c_int64), ("capacity", C.c_int64),
    ]


class _Fields(C.Structure):
    _fields_ = [(n, C.POINTER(C.c_double)) for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Jx", "Jy", "Jz")]


class Inflow(C.Structure):
    _fields_ = [
        ("face", C.c_int32), ("pos", C.c_double), ("speed", C.c_double), ("vmax", C.c_double),
        ("epc", C.c_double), ("density", C.c_double), ("drift", C.c_double * 3), ("nspecies", C.c_int32),
        ("flv", C.c_int32 * 4), ("temp", C.c_double * 4), ("charge", C.c_double * 4), ("seed", C.c_uint32),
        ("call", C.c_uint32),
    ]


class _Pml(C.Structure):
    _fields_ = [
        ("faces", C.c_int32), ("pos", C.c_double * 6), ("thickness", C.c_double * 6),
        ("psiE", C.POINTER(C.c_double) * 6), ("psiB", C.POINTER(C.c_double) * 6),
    ]


class Pml:
    """The 'pml' faces {n: (pos, thickness)} (n = 1..6) and their twelve
    convolution arrays (pml_E_psi1/2, pml_B_psi1/2: x, y, z), zero at start."""

    def __init__(self, g: Grid, faces: dict):
        self.faces = {int(n): (float(p), float(t)) for n, (p, t) in faces.items()}
        shp = grid_shape(g)
        self.psiE = [np.zeros(shp, dtype=np.float64, order="F") for _ in range(6)]
        self.psiB = [np.zeros(shp, dtype=np.float64, order="F") for _ in range(6)]

    def struct(self) -> _Pml:
        s = _Pml()
        for n, (p, t) in self.faces.items():
            s.faces |= 1 << (n - 1)
            s.pos[n - 1] = p
            s.thickness[n - 1] = t
        for c in range(6):
            s.psiE[c] = _dp(self.psiE[c])
            s.psiB[c] = _dp(self.psiB[c])
        return s


class _Weibel(C.Structure):
    _fields_ = [
        ("dims", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("epc", C.c_double), ("density", C.c_double), ("drift", C.c_double),
        ("temp_ion", C.c_double), ("temp_elc", C.c_double), ("seed", C.c_uint32),
    ]


def _declare(L: C.CDLL) -> None:
    P = C.POINTER
    L.orc_grid_init.argtypes = [P(Grid)]
    for fn in ("orc_update_b_half", "orc_update_e", "orc_add_current", "orc_reset_current"):
        getattr(L, fn).argtypes = [P(Grid), P(_Fields)]
    L.orc_lehe_coefficients.argtypes = [P(Grid), P(C.c_double)]
    L.orc_send_recv_flds.argtypes = [P(Grid)] + [P(C.c_double)] * 3
    L.orc_update_current_all_faces.argtypes = [P(Grid)] + [P(C.c_double)] * 3
    L.orc_filter_current.argtypes = [P(Grid)] + [P(C.c_double)] * 3 + [C.c_int]
    L.orc_step_filtered.argtypes = [P(Grid), P(_Particles), P(_Fields), C.c_int, C.c_int, C.c_int]
    L.orc_step_filtered.restype = C.c_int
    L.orc_move_deposit.argtypes = [P(Grid), P(_Particles), P(_Fields)]
    L.orc_exchange_particles.argtypes = [P(Grid), P(_Particles)]
    L.orc_exchange_particles.restype = C.c_int
    L.orc_reorder.argtypes = [P(Grid), P(_Particles), P(C.c_int64)]
    for fn in ("orc_refl_prtl_left", "orc_refl_prtl_right"):
        getattr(L, fn).argtypes = [P(Grid), P(_Particles), P(_Fields), C.c_double]
    for fn in ("orc_cond_fld_left", "orc_cond_fld_right"):
        getattr(L, fn).argtypes = [P(Grid), P(_Fields), C.c_double]
    for fn in ("orc_refl_prtl_bottom", "orc_refl_prtl_top"):
        getattr(L, fn).argtypes = [P(Grid), P(_Particles), P(_Fields), C.c_double]
    for fn in ("orc_cond_fld_bottom", "orc_cond_fld_top"):
        getattr(L, fn).argtypes = [P(Grid), P(_Fields), C.c_double]
    L.orc_remove_prtl.argtypes = [P(Grid), P(_Particles), C.c_int, C.c_double]
    L.orc_attn_vacuum.argtypes = [P(Grid), P(_Fields), C.c_int, P(C.c_double), P(C.c_double)]
    L.orc_attn_flow.argtypes = [P(Grid), P(_Fields), C.c_int, C.c_double, C.c_double, C.c_double, P(C.c_double),
                                P(C.c_double)]
    for fn in ("orc_open_fld_right", "orc_open_fld_left"):
        getattr(L, fn).argtypes = [P(Grid), P(_Fields), C.c_double]
    L.orc_open_prtl.argtypes = [P(Grid), P(_Particles), C.c_int, C.c_double, C.c_double]
    L.orc_open_prtl.restype = C.c_int
    L.orc_inject.argtypes = [P(Grid), P(_Particles), P(Inflow)]
    L.orc_inject.restype = C.c_int64
    L.orc_refl_fluid_right.argtypes = [P(Grid), P(_Particles), P(_Fields), C.c_double, C.c_double]
    for fn in ("orc_pml_b", "orc_pml_e"):
        getattr(L, fn).argtypes = [P(Grid), P(_Fields), P(_Pml)]
    L.orc_step.argtypes = [P(Grid), P(_Particles), P(_Fields), C.c_int, C.c_int]
    L.orc_step.restype = C.c_int
    L.orc_field_energy.argtypes = [P(Grid), P(_Fields), P(C.c_double)]
    L.orc_set_exact_order.argtypes = [C.c_int]
    L.orc_particle_energy.argtypes = [P(Grid), P(_Particles), C.c_double, C.c_double, P(C.c_double)]
    L.orc_gauss_residual.argtypes = [P(Grid), P(_Fields), P(_Particles), P(C.c_double)]
    L.orc_gauss_residual.restype = C.c_double
    L.orc_philox4x32_10.argtypes = [P(C.c_uint32), P(C.c_uint32), P(C.c_uint32)]
    L.orc_u01.argtypes = [C.c_uint32, C.c_uint32]
    L.orc_u01.restype = C.c_double
    L.orc_load_weibel.argtypes = [P(_Weibel), P(_Particles)]
    L.orc_load_weibel.restype = C.c_int64
    L.orc_maxbolt_table.argtypes = [C.c_int, P(C.c_double), P(C.c_double)]
    for fn in ("orc_cyl_update_b_half", "orc_cyl_update_e", "orc_cyl_add_current"):
        getattr(L, fn).argtypes = [P(Grid), P(_Fields)]
    L.orc_cyl_params.argtypes = [P(Grid), P(C.c_double)]
    L.orc_cyl_send_recv_flds.argtypes = [P(Grid)] + [P(C.c_double)] * 3
    L.orc_cyl_fold.argtypes = [P(Grid)] + [P(C.c_double)] * 3
    L.orc_cyl_move_deposit.argtypes = [P(Grid), P(_Particles), P(_Fields)]
    L.orc_cyl_exchange.argtypes = [P(Grid), P(_Particles)]
    L.orc_cyl_exchange.restype = C.c_int
    L.orc_cyl_step.argtypes = [P(Grid), P(_Particles), P(_Fields), C.c_int, C.c_int]
    L.orc_cyl_step.restype = C.c_int
    L.orc_cyl_load_uniform.argtypes = [P(Grid), C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int,
                                       C.c_uint32, P(_Particles)]
    L.orc_cyl_load_uniform.restype = C.c_int64
    L.orc_cyl_field_energy.argtypes = [P(Grid), P(_Fields), P(C.c_double)]


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and (a.flags["C_CONTIGUOUS"] or a.flags["F_CONTIGUOUS"])
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_grid(dims: int, nx: int, ny: int, nz: int = 1, c: float = 0.45, qi: float = 1.0,
              fdtd: str = "yee", qm=(1.0, -1.0), bext=(0.0, 0.0, 0.0)) -> Grid:
    g = Grid()
    g.dims, g.nx, g.ny, g.nz = dims, nx, ny, (nz if dims == 3 else 1)
    g.fdtd = {"yee": 0, "lehe": 1}[fdtd]
    g.nflvr = len(qm)
    g.c, g.qi = c, qi
    for d in range(3):
        g.bext[d] = bext[d]
    for i, v in enumerate(qm):
        g.flvrqm[i + 1] = v
    lib().orc_grid_init(C.byref(g))
    return g


def grid_shape(g: Grid):
    """Fortran (mx,my,mz) array shape; arrays are stored column-major."""
    return (g.mx, g.my, g.mz)


class Fields:
    """E, B, J as Fortran-ordered (mx,my,mz) float64 arrays."""

    NAMES = ("Ex", "Ey", "Ez", "Bx", "By", "Bz", "Jx", "Jy", "Jz")

    def __init__(self, g: Grid):
        shp = grid_shape(g)
        for n in self.NAMES:
            setattr(self, n, np.zeros(shp, dtype=np.float64, order="F"))

    def struct(self) -> _Fields:
        s = _Fields()
        for n in self.NAMES:
            setattr(s, n, _dp(getattr(self, n)))
        return s

    def copy(self) -> "Fields":
        o = Fields.__new__(Fields)
        for n in self.NAMES:
            setattr(o, n, getattr(self, n).copy(order="F"))
        return o


class Particles:
    """Reference-layout particle SoA (q,x,y,z,u,v,w float64; flv int32)."""

    NAMES = ("q", "x", "y", "z", "u", "v", "w")

    def __init__(self, capacity: int):
        self.capacity = int(capacity)
        for n in self.NAMES:
            setattr(self, n, np.zeros(self.capacity, dtype=np.float64))
        self.flv = np.zeros(self.capacity, dtype=np.int32)
        self.used = 0
        self._s = None

    @classmethod
    def from_arrays(cls, capacity: int, **arrs) -> "Particles":
        p = cls(capacity)
        n = len(arrs["x"])
        for k in cls.NAMES + ("flv",):
            getattr(p, k)[:n] = arrs[k]
        p.used = n
        return p

    def struct(self) -> _Particles:
        s = _Particles()
        for n in self.NAMES:
            setattr(s, n, _dp(getattr(self, n)))
        s.flv = self.flv.ctypes.data_as(C.POINTER(C.c_int32))
        s.used = self.used
        s.capacity = self.capacity
        return s

    def copy(self) -> "Particles":
        o = Particles(self.capacity)
        for n in self.NAMES + ("flv",):
            getattr(o, n)[:] = getattr(self, n)
        o.used = self.used
        return o

    def view(self):
        return {k: getattr(self, k)[: self.used] for k in self.NAMES + ("flv",)}


class Oracle:
    """Stateful wrapper: one grid, its fields and particles."""

    def __init__(self, g: Grid, particles: Particles, fields: Fields | None = None, openmp: bool = False,
                 exact_order: bool = True):
        """openmp: the OpenMP build; exact_order (OpenMP build only): each
        cell's current summed in particle order, bit for bit the serial
        build's result; False: the reference's thread slices.  The setting is
        global to the OpenMP library and made again by every Oracle."""
        self.g = g
        self.p = particles
        self.f = fields if fields is not None else Fields(g)
        self.L = lib(openmp)
        if openmp:
            self.L.orc_set_exact_order(1 if exact_order else 0)

    def _call_p(self, fn, *extra):
        ps = self.p.struct()
        r = fn(C.byref(self.g), C.byref(ps), *extra)
        self.p.used = ps.used
        return r

    def update_b_half(self):
        fs = self.f.struct()
        self.L.orc_update_b_half(C.byref(self.g), C.byref(fs))

    def update_e(self):
        fs = self.f.struct()
        self.L.orc_update_e(C.byref(self.g), C.byref(fs))

    def add_current(self):
        fs = self.f.struct()
        self.L.orc_add_current(C.byref(self.g), C.byref(fs))

    def send_recv_flds(self, which: str):
        a = [getattr(self.f, which + c) for c in "xyz"]
        self.L.orc_send_recv_flds(C.byref(self.g), *[_dp(x) for x in a])

    def fold_current(self):
        self.L.orc_update_current_all_faces(C.byref(self.g), _dp(self.f.Jx), _dp(self.f.Jy), _dp(self.f.Jz))

    def filter_current(self, passes: int):
        self.L.orc_filter_current(C.byref(self.g), _dp(self.f.Jx), _dp(self.f.Jy), _dp(self.f.Jz), int(passes))

    def step_filtered(self, t: int, reorder_period: int, curr_filter: int) -> int:
        fs = self.f.struct()
        return self._call_p(self.L.orc_step_filtered, C.byref(fs), int(t), int(reorder_period), int(curr_filter))

    def move_deposit(self):
        fs = self.f.struct()
        self._call_p(self.L.orc_move_deposit, C.byref(fs))

    def exchange_particles(self) -> int:
        return self._call_p(self.L.orc_exchange_particles)

    def reflect_particles_x(self, side: int, pos: float):
        """RefBC_Prtl_Left (side 0) / RefBC_Prtl_Right (side 1) at wall pos."""
        fs = self.f.struct()
        fn = self.L.orc_refl_prtl_left if side == 0 else self.L.orc_refl_prtl_right
        self._call_p(fn, C.byref(fs), float(pos))

    def conducting_x(self, side: int, pos: float):
        """CondBC_Fld_Left (side 0) / CondBC_Fld_Right (side 1) at wall pos."""
        fs = self.f.struct()
        fn = self.L.orc_cond_fld_left if side == 0 else self.L.orc_cond_fld_right
        fn(C.byref(self.g), C.byref(fs), float(pos))

    def remove_particles(self, face: int, pos: float):
        """RemovePrtl_Left / Right for face 1..6 (x, y, z; low, high) at wall pos."""
        self._call_p(self.L.orc_remove_prtl, int(face), float(pos))

    def reflect_particles_y(self, side: int, pos: float):
        """RefBC_Prtl_Bottom (side 0) / RefBC_Prtl_Top (side 1) at wall pos."""
        fs = self.f.struct()
        fn = self.L.orc_refl_prtl_bottom if side == 0 else self.L.orc_refl_prtl_top
        self._call_p(fn, C.byref(fs), float(pos))

    def conducting_y(self, side: int, pos: float):
        """CondBC_Fld_Bottom (side 0) / CondBC_Fld_Top (side 1) at wall pos."""
        fs = self.f.struct()
        fn = self.L.orc_cond_fld_bottom if side == 0 else self.L.orc_cond_fld_top
        fn(C.byref(self.g), C.byref(fs), float(pos))

    def pml_b(self, pml: "Pml"):
        """UpdateMagFld_PML (after the second B half step; no halo refresh)."""
        fs, ps = self.f.struct(), pml.struct()
        self.L.orc_pml_b(C.byref(self.g), C.byref(fs), C.byref(ps))

    def pml_e(self, pml: "Pml"):
        """UpdateElcFld_PML (after the E update; no halo refresh)."""
        fs, ps = self.f.struct(), pml.struct()
        self.L.orc_pml_e(C.byref(self.g), C.byref(fs), C.byref(ps))

    def attenuate_vacuum(self, faces: dict):
        """Attenuate_EM_Vacuum for the 'attn' faces {n: (pos, scale)}, n = 1..6."""
        mask = 0
        pos = (C.c_double * 6)()
        sc = (C.c_double * 6)(*([1.0] * 6))
        for n, (p, s) in faces.items():
            mask |= 1 << (int(n) - 1)
            pos[int(n) - 1] = float(p)
            sc[int(n) - 1] = float(s)
        fs = self.f.struct()
        self.L.orc_attn_vacuum(C.byref(self.g), C.byref(fs), mask, pos, sc)

    def attenuate_flow(self, face: int, pos: float, thickness: float, scale: float, bflow, drift):
        """Attenuate_EM_Flow of face 1..4 with a uniform flow."""
        fs = self.f.struct()
        b = (C.c_double * 3)(*map(float, bflow))
        v = (C.c_double * 3)(*map(float, drift))
        self.L.orc_attn_flow(C.byref(self.g), C.byref(fs), int(face), float(pos), float(thickness), float(scale), b, v)

    def open_fld_x(self, side: int, pos: float):
        """OpenBC_Fld_Left (side 0) / OpenBC_Fld_Right (side 1) at pos."""
        fs = self.f.struct()
        fn = self.L.orc_open_fld_left if side == 0 else self.L.orc_open_fld_right
        fn(C.byref(self.g), C.byref(fs), float(pos))

    def inject(self, face: int, pos: float, species, epc: float, density: float = 1.0, drift=(0.0, 0.0, 0.0),
               speed: float = 0.0, vmax: float = 1.0, seed: int = 1, call: int = 0) -> int:
        """InjectNewPrtl at face 1..6; species = [(flv, temperature, charge)]."""
        f = Inflow()
        f.face, f.pos, f.speed, f.vmax, f.epc, f.density = int(face), float(pos), float(speed), float(vmax), \
            float(epc), float(density)
        for d in range(3):
            f.drift[d] = float(drift[d])
        f.nspecies = len(species)
        for k, (fl, tp, q) in enumerate(species):
            f.flv[k], f.temp[k], f.charge[k] = int(fl), float(tp), float(q)
        f.seed, f.call = int(seed) & 0xFFFFFFFF, int(call) & 0xFFFFFFFF
        return self._call_p(self.L.orc_inject, C.byref(f))

    def reflect_fluid_right(self, pos: float, vx: float):
        """RefPrtlFluidFrameRight at the right injector pos for the uniform drift vx."""
        fs = self.f.struct()
        self._call_p(self.L.orc_refl_fluid_right, C.byref(fs), float(pos), float(vx))

    def open_prtl_x(self, side: int, pos: float, dx: float = 1.0) -> int:
        """OpenBC_Prtl_Left (side 0) / OpenBC_Prtl_Right (side 1) at pos."""
        return self._call_p(self.L.orc_open_prtl, int(side), float(pos), float(dx))

    def reorder(self) -> np.ndarray:
        perm = np.zeros(max(self.p.used, 1), dtype=np.int64)
        self._call_p(self.L.orc_reorder, perm.ctypes.data_as(C.POINTER(C.c_int64)))
        return perm[: self.p.used]

    def step(self, t: int, reorder_period: int = 20) -> int:
        fs = self.f.struct()
        return self._call_p(self.L.orc_step, C.byref(fs), int(t), int(reorder_period))

    def field_energy(self):
        out = (C.c_double * 2)()
        fs = self.f.struct()
        self.L.orc_field_energy(C.byref(self.g), C.byref(fs), out)
        return out[0], out[1]

    def particle_energy(self, masse: float, massi: float = 0.0) -> np.ndarray:
        """CalcPrtlEnergy per species (orc_particle_energy)."""
        out = np.zeros(self.g.nflvr)
        ps = self.p.struct()
        self.L.orc_particle_energy(C.byref(self.g), C.byref(ps), float(masse), float(massi),
                                   out.ctypes.data_as(C.POINTER(C.c_double)))
        return out

    def gauss_residual(self):
        rm = C.c_double(0)
        fs = self.f.struct()
        ps = self.p.struct()
        r = self.L.orc_gauss_residual(C.byref(self.g), C.byref(fs), C.byref(ps), C.byref(rm))
        return r, rm.value


class CylOracle(Oracle):
    """The cylindrical (r, theta, z) restatement: same state, cylindrical phases."""

    def update_b_half(self):
        fs = self.f.struct()
        self.L.orc_cyl_update_b_half(C.byref(self.g), C.byref(fs))

    def update_e(self):
        fs = self.f.struct()
        self.L.orc_cyl_update_e(C.byref(self.g), C.byref(fs))

    def add_current(self):
        fs = self.f.struct()
        self.L.orc_cyl_add_current(C.byref(self.g), C.byref(fs))

    def send_recv_flds(self, which: str):
        a = [getattr(self.f, which + c) for c in "xyz"]
        self.L.orc_cyl_send_recv_flds(C.byref(self.g), *[_dp(x) for x in a])

    def fold_current(self):
        self.L.orc_cyl_fold(C.byref(self.g), _dp(self.f.Jx), _dp(self.f.Jy), _dp(self.f.Jz))

    def move_deposit(self):
        fs = self.f.struct()
        self._call_p(self.L.orc_cyl_move_deposit, C.byref(fs))

    def exchange_particles(self) -> int:
        return self._call_p(self.L.orc_cyl_exchange)

    def step(self, t: int, reorder_period: int = 20) -> int:
        fs = self.f.struct()
        return self._call_p(self.L.orc_cyl_step, C.byref(fs), int(t), int(reorder_period))

    def field_energy(self):
        out = (C.c_double * 2)()
        fs = self.f.struct()
        self.L.orc_cyl_field_energy(C.byref(self.g), C.byref(fs), out)
        return out[0], out[1]

    def params(self):
        out = (C.c_double * 4)()
        self.L.orc_cyl_params(C.byref(self.g), out)
        return {"dtheta": out[0], "ax_perm_area": out[1], "inv_dtheta": out[2], "rshift": out[3]}


def cyl_load_uniform(g: Grid, npx: int, npy: int, npz: int, density: float, temp: float, charge: float, flv: int,
                     seed: int, capacity: int) -> Particles:
    p = Particles(capacity)
    ps = p.struct()
    n = lib().orc_cyl_load_uniform(C.byref(g), npx, npy, npz, density, temp, charge, flv, seed, C.byref(ps))
    if n < 0:
        raise RuntimeError("capacity exceeded")
    p.used = ps.used
    return p


def lehe_coefficients(g: Grid) -> np.ndarray:
    out = (C.c_double * 12)()
    lib().orc_lehe_coefficients(C.byref(g), out)
    return np.array(out[:])


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return tuple(o[:])


def maxbolt_table(n: int = 10000):
    X = np.zeros(n)
    P = np.zeros(n)
    lib().orc_maxbolt_table(n, _dp(X), _dp(P))
    return X, P


def load_weibel(dims: int, nx: int, ny: int, nz: int = 1, epc: float = 16.0, density: float = 0.5,
                drift: float = 0.5, temp: float = 0.005, seed: int = 2930, capacity: int | None = None) -> Particles:
    """Weibel particle load (setup_weibel.F90 with Philox in place of random_number)."""
    vol = nx * ny * (nz if dims == 3 else 1)
    if capacity is None:
        capacity = int(2 * epc * vol * 1.3) + 4096
    p = Particles(capacity)
    w = _Weibel(dims, nx, ny, nz if dims == 3 else 1, float(epc), float(density), float(drift),
                float(temp), float(temp), int(seed))
    ps = p.struct()
    n = lib().orc_load_weibel(C.byref(w), C.byref(ps))
    if n < 0:
        raise RuntimeError("particle capacity exceeded in load_weibel")
    p.used = int(n)
    return p


def init_scale(c: float, c_ompe: float, epc: float, g0: float = 1.0, mi_me: float = 1.0):
    """InitScale, initialise.F90:44-53: returns (qi, qme, qmi, masse, massi)."""
    ompe = c / c_ompe
    qi = (g0 * (ompe * ompe)) / ((float(epc) / 1.0) * (1.0 + 1.0 / mi_me))
    return qi, -1.0, 1.0 / mi_me, abs(-qi) * 1.0, qi * mi_me
