"""The allocation-free field-energy entry point against the existing one.

pic_field_energy_noalloc exists for callers that cannot allocate device
memory when they need the diagnostic (a host whose memory pool already owns
the GPU's memory, or one that must not let a library cudaMalloc/cudaFree
between its own steps).  It reads caller-owned device arrays and keeps its
reduction scratch in a fixed array inside the library.  Here the caller's
arrays are torch CUDA tensors in the reference layout; the result must match
pic_diagnostics of a handle holding the same fields, on two calls in a row
(the shared scratch keeps the previous call's partial sums)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


# (2, 40, 24, 1) and (3, 20, 12, 10) launch one block per 2048 interior cells;
# 160 x 128 x 128 = 2.6 M interior cells reaches the cap of 148 * 8 blocks, so
# the blocks stride over the grid and every slot of the fixed scratch is used.
@pytest.mark.parametrize("dims,nx,ny,nz", [(2, 40, 24, 1), (3, 20, 12, 10), (3, 160, 128, 128)])
def test_noalloc_energy_matches_diagnostics(dims, nx, ny, nz):
    import torch

    from pictor_b200 import Fields, PicConfig, Simulation, _capi

    cfg = PicConfig(nx=nx, ny=ny, nz=nz, dims=dims, capacity=1024)
    rng = np.random.default_rng(3)
    host = Fields.zeros(cfg.shape)
    for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz"):
        getattr(host, n)[...] = rng.normal(size=cfg.shape)
    with Simulation(cfg) as s:
        s.load_fields(host)
        ref = s.diagnostics()
    # device copies in the same column-major layout: torch shape (mz, my, mx)
    dev = {n: torch.from_numpy(np.ascontiguousarray(getattr(host, n).transpose(2, 1, 0))).cuda()
           for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz")}
    L = _capi.lib()
    for _ in range(2):
        out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        rc = L.pic_field_energy_noalloc(*[C.c_void_p(dev[n].data_ptr()) for n in ("Ex", "Ey", "Ez", "Bx", "By", "Bz")],
                                        nx, ny, nz, dims, C.c_void_p(out.data_ptr()), C.c_void_p(stream))
        assert rc == 0
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, [ref["B2"], ref["E2"]], rtol=1e-12)


def test_noalloc_rejects_bad_sizes():
    from pictor_b200 import _capi

    L = _capi.lib()
    p = C.c_void_p(8)
    assert L.pic_field_energy_noalloc(p, p, p, p, p, p, 0, 4, 4, 3, p, None) == -1
    assert L.pic_field_energy_noalloc(p, p, p, p, p, p, 4, 4, 4, 5, p, None) == -1
    assert L.pic_field_energy_noalloc(None, p, p, p, p, p, 4, 4, 4, 3, p, None) == -1
