"""Generates tests/golden/known_answers.json: hand-derived known answers that
pin the CPU restatement (the oracle).  Nothing here calls the oracle; every
expected value follows from closed-form arithmetic on the published
algorithms:

* Philox-4x32-10 known-answer vectors (Salmon et al., SC'11; the Random123
  kat_vectors file).
* Zigzag (Umeda 2003) deposit of one particle in zero field: with no cell
  crossing both segments go to the start cell and J_x(i,j) = q*qi*dx*(1-Wy),
  J_x(i,j+1) = q*qi*dx*Wy with Wy the particle's y offset; a crossing splits
  the path at the cell face (relay point xr = the face).
* Force-free motion: a particle with gamma*beta = 0.75 moves beta*c = 0.6*c
  per step.
* Boris rotation in a uniform B: |u| is invariant and the phase per step is
  2*atan(qm*B/(2*c*gamma)) (the effective field of movdep.F90:149-161).
* Yee vacuum dispersion of the step's E/B update (symplectic leapfrog):
  trace of the one-step amplification matrix = 2*cos(w) with
  sin(w/2) = c*sin(k/2).
* Periodic wrap (loadprtlout.F90 + comm_prtl.F90): a particle past x_max is
  re-appended at the end of the array at x - nx and its slot becomes a hole
  (x = y = 3.8, z = 1.5 in 2D).
"""
import json
import math
import os

HERE = os.path.dirname(os.path.abspath(__file__))

out = {}

out["philox"] = [
    {"ctr": [0, 0, 0, 0], "key": [0, 0], "out": [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]},
    {"ctr": [0xFFFFFFFF] * 4, "key": [0xFFFFFFFF, 0xFFFFFFFF], "out": [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]},
    {"ctr": [0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], "key": [0xA4093822, 0x299F31D0],
     "out": [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]},
]

# One particle, zero fields, c = 0.5, gamma*beta = 0.75 along x (beta = 0.6):
# displacement 0.3 per step.
c = 0.5
ub = 0.75
dx = 0.6 * c
cases = []
# (x0, y0, expected J entries [(component, i, j, value)], x1)
# no crossing: cell (7,6), Wy = 0.25
x0, y0 = 7.5, 6.25
cases.append({"name": "inside", "x0": x0, "y0": y0, "u": ub,
              "J": [["Jx", 7, 6, dx * (1 - 0.25)], ["Jx", 7, 7, dx * 0.25]], "x1": x0 + dx})
# x crossing at face 8: 0.1 in cell 7, 0.2 in cell 8
x0, y0 = 7.8, 6.5
cases.append({"name": "x_cross", "x0": x0, "y0": y0, "u": ub,
              "J": [["Jx", 7, 6, 0.2 * 0.5], ["Jx", 7, 7, 0.2 * 0.5], ["Jx", 8, 6, 0.1 * 0.5], ["Jx", 8, 7, 0.1 * 0.5]],
              "x1": x0 + dx})
out["deposit"] = {"c": c, "qi": 1.0, "q": 1.0, "cases": cases}

# Boris gyration: u along x, Bz uniform; qm = -1 for an electron
u0 = 0.3
gam = math.sqrt(1 + u0 * u0)
Bz = 0.2
qm = -1.0
phase = 2 * math.atan(abs(qm) * 0.5 * Bz / (c * gam))
out["boris"] = {"c": c, "u0": u0, "Bz": Bz, "qm": qm, "phase_per_step": phase, "umag": u0}

# Yee dispersion, waves along x on an nx-cell periodic grid, mode m
nx, m, cyee = 32, 3, 0.45
k = 2 * math.pi * m / nx
w = 2 * math.asin(cyee * math.sin(k / 2))
out["yee"] = {"nx": nx, "m": m, "c": cyee, "trace": 2 * math.cos(w)}

# periodic wrap, 2D grid 16x12: mx = 21, xmax = 19, xlen = 16
out["wrap"] = {"nx": 16, "ny": 12, "x": 19.1, "y": 7.3, "z": 1.4, "x_new": 19.1 - 16, "hole": [3.8, 3.8, 1.5]}

with open(os.path.join(HERE, "known_answers.json"), "w") as f:
    json.dump(out, f, indent=1, sort_keys=True)
print("wrote", os.path.join(HERE, "known_answers.json"))
