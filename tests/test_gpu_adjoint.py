"""The differentiable form against its oracles: the FP64 forward of this
library (pic_step), central finite differences of the FP64 forward, and the
FP64 adjoint for the FP32 one.

The deposit is piecewise linear in the positions (floor and the relay
point's min/max), so a finite difference can straddle a cell crossing; the
steps here are short and the perturbations small, and the tolerances state
how far apart FD and adjoint may be."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

C_, CE = 0.45, 2.0


def _cfg(nx, ny, precision="fp64", capacity=1 << 16):
    from pictor_b200 import PicConfig, init_scale

    sc = init_scale(C_, CE, 4)
    return PicConfig(nx=nx, ny=ny, dims=2, c=C_, qi=sc["qi"], precision=precision, capacity=capacity,
                     reorder_period=0), sc


def test_forward_matches_the_fp64_step():
    """Same particles with no out-of-plane motion (w = 0, where the midpoint
    and the z-relay splits of the out-of-plane current agree): J of the
    differentiable forward equals sum_t 1/2 sum |B_t|^2 of the FP64 pic_step
    to round-off."""
    from pictor_b200 import Simulation
    from pictor_b200.adjoint import Adjoint

    cfg, sc = _cfg(32, 32)
    with Adjoint(cfg) as a:
        a.init_weibel(4, 0.5, 0.4, 0.005, 0.005, 77)
        p, sgn = a.fetch_particles()
        p.w[:] = 0.0
        a.load_particles(p, sgn)
        j = a.forward(10, 4)
    j_ref = 0.0
    with Simulation(cfg) as s:
        s.load_particles(p)
        for _ in range(10):
            s.step(1)
            j_ref += 0.5 * s.diagnostics(sc["masse"])["B2"]
    assert j_ref > 0
    assert abs(j - j_ref) <= 1e-10 * j_ref


def test_forward_tracks_the_fp32_step():
    """With out-of-plane motion the differentiable forward splits Jz as the
    FP32 form does: J agrees with pic_step in the FP32 form to 1e-4."""
    from pictor_b200 import Simulation
    from pictor_b200.adjoint import Adjoint

    cfg, sc = _cfg(32, 32)
    cfg32, _ = _cfg(32, 32, "fp32")
    with Adjoint(cfg) as a:
        a.init_weibel(4, 0.5, 0.4, 0.005, 0.005, 78)
        p, _ = a.fetch_particles()
        j = a.forward(10, 4)
    j_ref = 0.0
    with Simulation(cfg32) as s:
        s.load_particles(p)
        for _ in range(10):
            s.step(1)
            j_ref += 0.5 * s.diagnostics(sc["masse"])["B2"]
    assert abs(j - j_ref) <= 1e-4 * j_ref


def _fd(make, h):
    return (make(+h) - make(-h)) / (2 * h)


def test_gradient_matches_central_differences():
    """dJ/d(temperature), a random direction in the space of initial momenta
    and one in the initial positions, FP64, 8 steps with checkpoints every 3
    (the reverse sweep recomputes three segments): within 1e-6 of central FD
    with steps of 1e-4 of each parameter.  dJ/d(drift) over 3 steps, within
    1e-5: the drift moves every particle, and over longer runs its finite
    difference straddles jumps of the zigzag current (a move that crosses an
    x face while y changes shifts the x current's y weight by dy/4), which the
    adjoint, the derivative almost everywhere, does not see."""
    from pictor_b200.adjoint import Adjoint

    cfg, _ = _cfg(24, 24)
    D, T, seed, K = 0.4, 0.005, 5, 3
    res = []
    with Adjoint(cfg) as a:
        a.init_weibel(4, 0.5, D, T, T, seed)
        a.forward(3, K)
        g3 = a.gradient()

        def j_drift(dh):
            a.init_weibel(4, 0.5, D + dh, T, T, seed)
            return a.forward(3, K)

        res.append(("drift (3 steps)", g3["drift"], _fd(j_drift, 1e-4 * D), 1e-5))
        steps = 8
        a.init_weibel(4, 0.5, D, T, T, seed)
        a.forward(steps, K)
        g = a.gradient()
        p0, sgn = a.fetch_particles()

        def j_temp(dh):
            a.init_weibel(4, 0.5, D, T + dh, T, seed)
            return a.forward(steps, K)

        rng = np.random.default_rng(1)
        du, dv, dw = (rng.normal(size=len(p0.x)) for _ in range(3))
        nrm = np.sqrt((du * du + dv * dv + dw * dw).sum())
        du, dv, dw = du / nrm, dv / nrm, dw / nrm

        def j_dir(dh):
            p = type(p0)(*(getattr(p0, k).copy() for k in p0.NAMES))
            p.u += dh * du
            p.v += dh * dv
            p.w += dh * dw
            a.load_particles(p, sgn)
            return a.forward(steps, K)

        def j_pos(dh):
            p = type(p0)(*(getattr(p0, k).copy() for k in p0.NAMES))
            p.x += dh * du
            p.y += dh * dv
            a.load_particles(p, sgn)
            return a.forward(steps, K)

        res.append(("temp_ion", g["temp_ion"], _fd(j_temp, 1e-4 * T), 1e-6))
        res.append(("momenta", float((g["u"] * du + g["v"] * dv + g["w"] * dw).sum()), _fd(j_dir, 1e-4), 1e-6))
        res.append(("positions", float((g["x"] * du + g["y"] * dv).sum()), _fd(j_pos, 1e-4), 1e-6))
    for name, ad, fd, tol in res:
        assert abs(ad - fd) <= tol * abs(fd), res


def test_gradient_matches_frozen_branch_differences():
    """30 steps, where central differences of free runs straddle jumps of the
    zigzag current: with the mover's discrete decisions recorded in the base
    run and replayed in the perturbed runs, the run is smooth in its inputs
    and central differences (h = 1e-4 of each parameter, a unit direction)
    agree with the adjoint to 1e-6 for the drift, the temperature, a random
    direction of the momenta and one of the positions."""
    from pictor_b200.adjoint import Adjoint

    cfg, _ = _cfg(24, 24)
    D, T, seed, K, steps = 0.4, 0.005, 5, 7, 30
    res = []
    with Adjoint(cfg) as a:
        a.init_weibel(4, 0.5, D, T, T, seed)
        a.branches("record")
        a.forward(steps, K)
        g = a.gradient()
        p0, sgn = a.fetch_particles()
        a.branches("replay")

        def j_load(dd, dt):
            a.init_weibel(4, 0.5, D + dd, T + dt, T, seed)
            return a.forward(steps, K)

        rng = np.random.default_rng(3)
        du, dv, dw = (rng.normal(size=len(p0.x)) for _ in range(3))
        nrm = np.sqrt((du * du + dv * dv + dw * dw).sum())
        du, dv, dw = du / nrm, dv / nrm, dw / nrm

        def j_dir(dh, pos):
            p = type(p0)(*(getattr(p0, k).copy() for k in p0.NAMES))
            if pos:
                p.x += dh * du
                p.y += dh * dv
            else:
                p.u += dh * du
                p.v += dh * dv
                p.w += dh * dw
            a.load_particles(p, sgn)
            return a.forward(steps, K)

        res.append(("drift", g["drift"], _fd(lambda h: j_load(h, 0.0), 1e-4 * D)))
        res.append(("temp_ion", g["temp_ion"], _fd(lambda h: j_load(0.0, h), 1e-4 * T)))
        res.append(("momenta", float((g["u"] * du + g["v"] * dv + g["w"] * dw).sum()), _fd(lambda h: j_dir(h, False), 1e-4)))
        res.append(("positions", float((g["x"] * du + g["y"] * dv).sum()), _fd(lambda h: j_dir(h, True), 1e-4)))
        a.branches("free")
    for name, ad, fd in res:
        assert abs(ad - fd) <= 1e-6 * abs(fd), res


def test_fp32_adjoint_tracks_fp64():
    """The FP32 form's gradient against the FP64 reference adjoint on the same
    run: per-particle momentum gradients within 1e-2 (relative L2) and the
    drift gradient within 1e-2."""
    from pictor_b200.adjoint import Adjoint

    res = {}
    for prec in ("fp64", "fp32"):
        cfg, _ = _cfg(24, 24, prec)
        with Adjoint(cfg) as a:
            a.init_weibel(4, 0.5, 0.4, 0.005, 0.005, 9)
            a.forward(12, 5)
            res[prec] = a.gradient()
    g64, g32 = res["fp64"], res["fp32"]
    v64 = np.concatenate([g64[k] for k in ("u", "v", "w")])
    v32 = np.concatenate([g32[k] for k in ("u", "v", "w")])
    assert np.linalg.norm(v32 - v64) <= 1e-2 * np.linalg.norm(v64)
    assert abs(g32["drift"] - g64["drift"]) <= 1e-2 * abs(g64["drift"])
