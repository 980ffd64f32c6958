"""Host-side checks of the C ABI that need no GPU: the in-tree library loads,
exports every entry point include/pictor_b200.h declares, and the ctypes
mirror of pic_config has the C layout."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pictor_b200.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pic_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_entry_point():
    from pictor_b200 import _capi, build

    build.build()
    L = C.CDLL(_capi.library_path())
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding declares exactly these
    assert sorted(_capi.SIGNATURES) == names


def test_error_strings_without_gpu():
    from pictor_b200 import _capi

    L = _capi.lib()
    assert L.pic_error_string(0) == b"ok"
    assert b"capacity" in L.pic_error_string(-3)
    assert L.pic_version() >= 10000


@pytest.mark.parametrize("cname,pyname", [("pic_config", "Config"), ("pic_inflow", "Inflow")])
def test_struct_layout_matches_c(cname, pyname):
    from pictor_b200 import _capi

    st = getattr(_capi, pyname)
    fields = [f[0] for f in st._fields_]
    prog = "#include <stdio.h>\n#include <stddef.h>\n#include \"pictor_b200.h\"\nint main(){printf(\"%zu\\n\", sizeof(" + cname + "));"
    for f in fields:
        prog += f'printf("%zu\\n", offsetof({cname}, {f}));'
    prog += "return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = [int(x) for x in subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()]
    assert out[0] == C.sizeof(st)
    for f, off in zip(fields, out[1:]):
        assert getattr(st, f).offset == off, f


def test_create_without_gpu_fails_cleanly():
    """With no CUDA device the library reports PIC_ERR_NOGPU (never a CPU fallback)."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from pictor_b200 import PicConfig, PicError, Simulation

    with pytest.raises(PicError) as e:
        Simulation(PicConfig(nx=8, ny=8))
    assert e.value.code in (-8, -6)


def test_invalid_configs_rejected_before_device_use():
    from pictor_b200 import PicConfig, PicError, Simulation

    for bad in (PicConfig(nx=3, ny=8), PicConfig(nx=8, ny=8, c=1.5), PicConfig(nx=8, ny=8, dims=4),
                PicConfig(nx=8, ny=8, qm=()), PicConfig(nx=8, ny=8, capacity=0)):
        with pytest.raises(PicError) as e:
            Simulation(bad)
        assert e.value.code == -1


def test_cell_decode_division_is_exact():
    """The device decodes cell indices with n/d = (n * ceil(2^40/d)) >> 40,
    exact for n < 2^28 and d <= 4096 (checked at every quotient boundary)."""
    import numpy as np

    rng = np.random.default_rng(0)
    for d in (6, 21, 37, 261, 517, 1029, 4096):
        m = ((1 << 40) + d - 1) // d
        qmax = (1 << 28) // d
        q = np.unique(np.concatenate([rng.integers(0, qmax + 1, 20000), np.arange(max(0, qmax - 2000), qmax + 1)]))
        for r in (0, d - 1):
            for n in (int(x) * d + r for x in q):
                if n < (1 << 28):
                    assert ((n << 24) * m) >> 64 == n // d, (n, d)


def test_slab_and_wall_entry_points_validate_without_gpu():
    """The slab form is refused (before any device use) with a current
    filter, for the FP32 or modal cylindrical step, with the outer-radius
    form (slab_x = 2) outside a cylinder, and for a cylindrical slab whose
    radii would not all be positive; a cylinder without the axis must be a
    slab, one with it must have it at x = 3.5.  The slab, wall and sync
    entry points reject a null handle and bad arguments."""
    from pictor_b200 import PicConfig, PicError, Simulation, _capi

    cyl = dict(nx=12, ny=8, nz=8, dims=3, geom="cylindrical")
    for bad in (PicConfig(nx=12, ny=8, slab_x=2),
                PicConfig(nx=12, ny=8, slab_x=3),
                PicConfig(nx=12, ny=8, slab_x=1, curr_filter=1),
                PicConfig(**cyl, slab_x=1),                                    # rmin 0, no axis
                PicConfig(**cyl, slab_x=1, rmin=2.0),                          # ghost radii <= 0
                PicConfig(**cyl, slab_x=1, rmin=11.5, precision="fp32"),
                PicConfig(**cyl, slab_x=1, rmin=-0.5, inc_axis=1, cyl_modes=2),
                PicConfig(**cyl, rmin=11.5),                                   # no axis, one domain
                PicConfig(**cyl, rmin=0.0, inc_axis=1)):
        with pytest.raises(PicError) as e:
            Simulation(bad)
        assert e.value.code == -1
    L = _capi.lib()
    n = C.c_int64()
    a, b = C.c_int64(), C.c_int64()
    assert L.pic_slab_face_len(None, C.byref(n)) == -1
    assert L.pic_slab_pack_fields(None, 0, None, None) == -1
    assert L.pic_slab_unpack_fields(None, 0, None, None) == -1
    assert L.pic_slab_pack_particles(None, None, 0, C.byref(a), C.byref(b)) == -1
    assert L.pic_slab_unpack_particles(None, None, 0) == -1
    assert L.pic_slab_pack_particles_fixed(None, None, None, 0) == -1
    assert L.pic_slab_unpack_particles_fixed(None, None, None, 0) == -1
    assert L.pic_set_sync(None, 0) == -1
    for fn in (L.pic_bc_reflect_x, L.pic_bc_conducting_x, L.pic_bc_reflect_y, L.pic_bc_conducting_y):
        assert fn(None, 0, 1.5) == -1
    assert L.pic_bc_remove(None, 1, 1.5) == -1
    six = (C.c_double * 6)(*([1.0] * 6))
    three = (C.c_double * 3)()
    assert L.pic_bc_attenuate(None, 1, six, six) == -1
    assert L.pic_bc_attenuate_flow(None, 2, 30.0, 1.0, 4.0, three, three) == -1
    assert L.pic_bc_open_x(None, 1, 1.5) == -1
    assert L.pic_bc_open_prtl_x(None, 1, 1.5) == -1
    assert L.pic_solve_gauss(None, 1e-12, 100, None, None, None) == -1
    assert L.pic_bc_inflow(None, None) == -1
    assert L.pic_bc_inflow_reflect(None, 20.0, -0.3) == -1
    six = (C.c_double * 6)()
    assert L.pic_bc_pml(None, 1, six, six) == -1
    assert L.pic_bc_pml_b(None) == -1
    assert L.pic_bc_pml_e(None) == -1
