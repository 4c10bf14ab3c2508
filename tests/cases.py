"""Seeded test cases and the product-side runner shared by the tests.

A case is expressed in the reference's own terms (`oracle.refrun.ElasticCase` / `AcousticCase`)
so the same object drives the reference binaries, the C restatement and the CUDA product.
"""
from __future__ import annotations

import importlib.util
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import refrun  # noqa: E402


def load_twave():
    """Import the product package (tpu-wave_b200/) by path."""
    name = "twave"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "tpu-wave_b200", "__init__.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def random_model(Mx, My, seed, acoustic=False):
    """Padded (Mx+2)x(My+2) rho/vp/vs with per-node noise: rho U(1.8,2.7), vp U(1.5,4.5),
    vs = vp/sqrt(3) * U(0.9,1.1) (the elastic medium ranges of the 2048^2 benchmark)."""
    rng = np.random.default_rng(seed)
    P = (Mx + 2, My + 2)
    rho = rng.uniform(1.8, 2.7, P)
    vp = rng.uniform(1.5, 4.5, P)
    vs = np.zeros(P) if acoustic else vp / np.sqrt(3.0) * rng.uniform(0.9, 1.1, P)
    return rho, vp, vs


def layered_model(Mx, My, seed, n_layers=8, acoustic=False):
    """Horizontal layers along data x (depth): per-layer vp U(1.5,4.5), rho U(1.8,2.7);
    vs = vp/sqrt(3) * U(0.9,1.1) per node."""
    rng = np.random.default_rng(seed)
    edges = np.linspace(0, Mx + 2, n_layers + 1).astype(int)
    vp_l, rho_l = rng.uniform(1.5, 4.5, n_layers), rng.uniform(1.8, 2.7, n_layers)
    vp = np.zeros((Mx + 2, My + 2)); rho = np.zeros_like(vp)
    for k in range(n_layers):
        vp[edges[k]:edges[k + 1]] = vp_l[k]
        rho[edges[k]:edges[k + 1]] = rho_l[k]
    vs = np.zeros_like(vp) if acoustic else vp / np.sqrt(3.0) * rng.uniform(0.9, 1.1, vp.shape)
    return rho, vp, vs


def elastic_case(Mx, My, seed=0, cpst="00", Nt=40, src=None, rcvs=None, den_dx=None, cfl=0.4,
                 central_f=15.0, time_delay=None, model="random", acoustic=False):
    den_dx = den_dx or max(Mx, My)
    dx = 1.0 / den_dx
    rho, vp, vs = (random_model if model == "random" else layered_model)(Mx, My, seed, acoustic=acoustic)
    dt = cfl * dx / (np.sqrt(2.0) * 4.5)
    if time_delay is None:
        time_delay = 4 * dt
    if src is None:   # explosive source on an MM cell near the centre: (2i+1)/(2 den) -> cell i
        src = ("M", "M", 2 * (Mx // 2) + 1, 2 * den_dx, 2 * (My // 3) + 1, 2 * den_dx)
    if rcvs is None:
        rcvs = [("N", "M", 2, den_dx, 2 * 3 + 1, 2 * den_dx), ("M", "M", 2 * 5 + 1, 2 * den_dx, 2 * 7 + 1, 2 * den_dx),
                ("N", "N", Mx, den_dx, My, den_dx), ("M", "N", 2 * (Mx - 1) + 1, 2 * den_dx, 0, 1),
                ("N", "M", 0, 1, 2 * (My - 1) + 1, 2 * den_dx)]
    return refrun.ElasticCase(Mx=Mx, My=My, num_dx=1, den_dx=den_dx, dt=dt, rho=rho.reshape(-1),
                              vp=vp.reshape(-1), vs=vs.reshape(-1), src=src, rcvs=rcvs, Nt=Nt, cpst=cpst,
                              central_f=central_f, time_delay=time_delay)


def acoustic_periodic_case(Nx, Ny, seed=0, cpst="0", Nt=40, cfl=0.5, central_f=10.0):
    rng = np.random.default_rng(seed)
    dx = 1.0 / max(Nx, Ny)
    dt = cfl * dx / (np.sqrt(2.0) * 3.0)
    # the seam row of Vx and column of Vy carry their own medium, as the reference allows
    rho_vx, rho_vy = rng.uniform(1.0, 2.5, (Nx + 1, Ny)), rng.uniform(1.0, 2.5, (Nx, Ny + 1))
    kappa = rng.uniform(1.0, 9.0, (Nx, Ny))
    case = refrun.AcousticCase(Nx=Nx, Ny=Ny, dx=dx, dt=dt, coef_vx=1.0 / rho_vx, coef_vy=1.0 / rho_vy, coef_p=kappa,
                               src=(Nx // 2, Ny // 3), rcvs=[(2, 3, 3), (0, Nx, 2), (1, 1, Ny), (2, 0, 0), (0, 5, Ny - 1)],
                               Nt=Nt, cpst=cpst, central_f=central_f, time_delay=4 * dt)
    case.rho_vx, case.rho_vy = rho_vx, rho_vy
    return case


ELASTIC_KEYS = ("NN", "MN", "NM", "MM0", "MM1")


def product_elastic(case, precision, acoustic=False, fields0=None, resid0=None, energy=True, coef_fp16=False):
    """Run `case` through the C ABI; returns dict(fields, traces, E_k, E_p0, E_p1, resid)."""
    tw = load_twave()
    s = tw.Solver(case.Mx, case.My, case.num_dx, case.den_dx, case.dt,
                  physics=tw.ACOUSTIC if acoustic else tw.ELASTIC, precision=precision, cpst=case.cpst,
                  central_f=case.central_f, time_delay=case.time_delay, max_steps=max(case.Nt, 1), energy=energy,
                  coef_fp16=coef_fp16, bc_x=tw.SAT_INTERFACE if case.bc_x == "I" else tw.SAT_FREE,
                  sat_y=case.sat_y)
    try:
        Mx, My = case.Mx, case.My
        shp = (Mx + 2, My + 2)
        s.set_material_model(case.rho.reshape(shp), case.vp.reshape(shp), None if acoustic else case.vs.reshape(shp))
        if case.src is not None:
            s.set_source_location(*case.src)
        for r in case.rcvs:
            s.add_receiver_location(*r)
        slots = [(tw.MN, 0), (tw.NM, 0), (tw.MM, 0)] if acoustic else \
                [(tw.NN, 0), (tw.MN, 0), (tw.NM, 0), (tw.MM, 0), (tw.MM, 1)]
        if fields0 is not None:
            for (g, f), a in zip(slots, fields0):
                s.write_field(g, f, a)
        if resid0 is not None:
            for (g, f), a in zip(slots, resid0):
                s.write_resid(g, f, a)
        s.run(case.Nt)
        fields = [s.read_field(g, f) for g, f in slots]
        resid = [s.read_resid(g, f) for g, f in slots] if case.cpst != "00" else None
        out = {"fields": dict(zip(("MN", "NM", "MM0") if acoustic else ELASTIC_KEYS, fields)),
               "traces": s.read_receivers(), "resid": resid}
        if energy:
            out["E_k"], out["E_p0"], out["E_p1"] = s.read_energy()
        return out
    finally:
        s.close()


def product_acoustic_periodic(case, precision, fields0=None, resid0=None, energy=True):
    """energy=False runs the fused one-launch step (the energy records need the two-launch path)."""
    tw = load_twave()
    cp = {"0": "00", "3": "3R", "6": "6R"}[case.cpst]
    s = tw.Solver(case.Nx, case.Ny, 1, max(case.Nx, case.Ny), case.dt, physics=tw.ACOUSTIC, bc_x=tw.PERIODIC,
                  precision=precision, cpst=cp, central_f=case.central_f, time_delay=case.time_delay,
                  max_steps=max(case.Nt, 1), energy=energy)
    try:
        # Vx (N in x) is the NM grid, Vy (N in y) the MN grid
        s.set_material_grid(tw.NM, 0, case.rho_vx)
        s.set_material_grid(tw.MN, 0, case.rho_vy)
        s.set_material_grid(tw.MM, 0, np.asarray(case.coef_p).reshape(case.Nx, case.Ny))
        s.set_source(tw.MM, *case.src)
        mesh_grid = {0: tw.NM, 1: tw.MN, 2: tw.MM}
        for m, ix, iy in case.rcvs:
            s.add_receivers(mesh_grid[m], [ix], [iy])
        slots = [tw.NM, tw.MN, tw.MM]
        if fields0 is not None:
            for g, a in zip(slots, fields0):
                s.write_field(g, 0, a)
        if resid0 is not None:
            for g, a in zip(slots, resid0):
                s.write_resid(g, 0, a)
        s.run(case.Nt)
        out = {"fields": {"Vx": s.read_field(tw.NM), "Vy": s.read_field(tw.MN), "P": s.read_field(tw.MM)},
               "traces": s.read_receivers()[:, 0, :]}
        if energy:
            out["E_k"], out["E_p0"], out["E_p1"] = s.read_energy()
        if resid0 is not None:
            out["resid"] = [s.read_resid(g) for g in slots]
        return out
    finally:
        s.close()
