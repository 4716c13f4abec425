"""Batched ensembles of uneven members (the C5 configuration).

``c5_members(n, seed)`` draws n members from a seeded generator: horizontal sizes in
[64, 512], nz in {40, 64, 80}, and a mix of cases:

* warm bubble: +2 K cos^2 bubble on a 300 K hydrostatic base (dry);
* density current: a -15 K cold block (a box at the surface, not the reference's cos^2
  shape) on the same base, in pressure balance (rho*theta kept, the cold air denser; dry);
* mountain wave: Witch-of-Agnesi hill (400 m, 10 km half width) under a 10 m/s wind in a
  constant-N (0.01 1/s) atmosphere, Rayleigh layer over the top 30 % (dry, terrain);
* moist warm rain: the moist sounding with warm rain and 12 m/s fallout.

All members share dt and the substep count (one captured step advances all of them,
each on its own graph branch).  The step is 1 s: the reference discretisation is
unstable at 4 s with these level spacings (c dt / dz > 1.4).
"""
from __future__ import annotations

import importlib
from typing import List, Tuple

import numpy as np

CASES = ("warm_bubble", "cold_block", "mountain_wave", "moist")


def _gwm():
    return importlib.import_module("gpu-wm-next_b200")


def c5_members(n: int = 64, seed: int = 5, dt: float = 1.0, substeps: int = 4, size_range=(64, 512),
               nz_choices=(40, 64, 80)):
    """Grids, member specs, initial states, damping settings and case names of n members."""
    gwm = _gwm()
    rng = np.random.default_rng(seed)
    grids, specs, states, damping, kinds = [], [], [], [], []
    for m in range(n):
        kind = CASES[m % len(CASES)]
        nx, ny = (int(v) for v in rng.integers(size_range[0], size_range[1] + 1, 2))
        nz = int(rng.choice(nz_choices))
        step = gwm.StepConfig(dt=dt, fast_substeps=substeps)
        z_top = 250.0 * nz  # 10, 16 and 20 km tops for 40, 64 and 80 levels
        damp = None
        if kind == "moist":
            g = gwm.GridSpec(nx, ny, nz, dx=3000.0, dy=3000.0, z_top=z_top)
            p = gwm.CaseParams(theta_ref=300.0, noise_rms_k=0.5, seed=int(rng.integers(1, 1 << 30)))
            s = gwm.build_case("moist_sounding", g, p, moist=True)
            spec = gwm.MemberSpec(step=step, rain=gwm.WarmRainConfig(dt=dt, rain_terminal_velocity=12.0),
                                  moist=True)
        elif kind == "mountain_wave":
            terrain = gwm.build_terrain("agnesi", nx, ny, 1000.0, 1000.0, height=400.0, half_width_x=10000.0,
                                        half_width_y=10000.0)
            g = gwm.GridSpec(nx, ny, nz, dx=1000.0, dy=1000.0, z_top=z_top, terrain=terrain)
            p = gwm.CaseParams(theta_ref=288.0, p_surface=100000.0, u_background=10.0, brunt_vaisala=0.01)
            s = gwm.build_case("stratified_mountain_wave", g, p)
            s["u"][:, :, -1] = s["u"][:, :, 0]
            damp = (0.7 * z_top, 0.05, s["u"].astype(np.float64).mean(axis=(1, 2)))
            spec = gwm.MemberSpec(step=step)
        else:
            g = gwm.GridSpec(nx, ny, nz, dx=1000.0, dy=1000.0, z_top=z_top)
            p = gwm.CaseParams(rho_surface=1.16123, theta_ref=300.0, theta_perturbation=2.0,
                               center_z_fraction=0.2, radius_x_fraction=2000.0 / (nx * 1000.0),
                               radius_y_fraction=2000.0 / (ny * 1000.0), radius_z_fraction=2000.0 / z_top)
            s = gwm.build_case("hydrostatic_warm_bubble", g, p)
            if kind == "cold_block":
                # -15 K in a surface box, in pressure balance: the EOS depends on rho*theta
                # alone, so rho*theta (and p) keep their hydrostatic values and the cold air
                # is denser, rho = rho*theta / theta
                rt = (s["rho"].astype(np.float64) * 300.0)
                th = np.full(rt.shape, 300.0)
                zc = (np.arange(nz) + 0.5) * z_top / nz
                box = np.zeros(rt.shape, dtype=bool)
                box[zc < 2500.0, int(0.4 * ny):int(0.6 * ny), int(0.4 * nx):int(0.6 * nx)] = True
                th[box] -= 15.0
                s["rho_theta"] = rt.astype(np.float32)
                s["rho"] = (rt / th).astype(np.float32)
            spec = gwm.MemberSpec(step=step)
        grids.append(g)
        specs.append(spec)
        states.append(s)
        damping.append(damp)
        kinds.append(kind)
    return grids, specs, states, damping, kinds


def build_model(grids, specs, states, damping, concurrent: bool = True):
    """A model holding every member, states uploaded and damping layers set."""
    gwm = _gwm()
    m = gwm.Model(grids, specs)
    m.set_concurrent(concurrent)
    for i, (s, d) in enumerate(zip(states, damping)):
        m.upload(s, member=i)
        if d is not None:
            m.set_damping(d[0], d[1], u_ref=d[2], member=i)
    return m
