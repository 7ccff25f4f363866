"""The reverse mode of n steps of (LOD step, agents' update), composed from the
oracle's single-step adjoint (oracle/lod_oracle.c: orc_lod_step_adjoint) and
the agents' update reversed here in numpy. Test infrastructure only.

Agents' update at one voxel, in list order over its active agents
(BioFVM_basic_agent.cpp:291-296): x_k = (x_(k-1) + t1_k)/t2_k with
t1 = c*S*rho*, t2 = 1 + c*S + c*U, c = dt*volume/dx^3
(BioFVM_basic_agent.cpp:155-176). Backwards: dL/dt1_k += g/t2_k,
dL/dt2_k -= g*x_k/t2_k, g <- g/t2_k.
"""
from __future__ import annotations

import numpy as np


def oracle_adjoint(oracle, rho0, w, n_steps, dt, dx, D, lam, dirv, agents):
    """Returns dict(initial, D, lambda, final[, secretion, uptake, saturation]).

    dirv = (per-voxel Dirichlet values (nx, ny, nz, S), face mask (6, S));
    agents = dict(pos, vol, sec, upt, sat, active) or None."""
    dvals, fm = dirv
    shape = rho0.shape
    S = shape[-1]
    if agents is not None:
        bbox = (0, 0, 0, shape[0] * dx, shape[1] * dx, shape[2] * dx)
        vox = oracle.bin_agents(agents["pos"], bbox, dx, shape[:3])
        t1, t2 = oracle.agent_constants(dt, dx, agents["vol"], agents["sec"], agents["upt"], agents["sat"])
        act = np.ones(len(vox), bool) if agents.get("active") is None else agents["active"].astype(bool)
    us, vs = [], []
    u = np.array(rho0, dtype=np.float64)
    for _ in range(n_steps):
        us.append(u)
        v = oracle.lod_steps(u, dt, dx, D, lam, 1, dvals, fm)
        vs.append(v)
        u = oracle.cells_step(v, vox, t1, t2, act.astype(np.uint8)) if agents is not None else v
    final = u
    g = np.array(w, dtype=np.float64)
    gD, gL = np.zeros(S), np.zeros(S)
    if agents is not None:
        gt1, gt2 = np.zeros_like(t1), np.zeros_like(t2)
        by_vox = {}
        for a in range(len(vox)):
            if act[a]:
                by_vox.setdefault(int(vox[a]), []).append(a)
    for j in range(n_steps - 1, -1, -1):
        if agents is not None:
            g = g.copy()
            gf = g.reshape(-1, S)
            vf = vs[j].reshape(-1, S)
            for v_idx, lst in by_vox.items():
                xs = [vf[v_idx].copy()]
                for a in lst:
                    xs.append((xs[-1] + t1[a]) / t2[a])
                gg = gf[v_idx].copy()
                for q in range(len(lst) - 1, -1, -1):
                    a = lst[q]
                    gt1[a] += gg / t2[a]
                    gt2[a] -= gg * xs[q + 1] / t2[a]
                    gg = gg / t2[a]
                gf[v_idx] = gg
        g, dD, dL = oracle.lod_step_adjoint(us[j], g, dt, dx, D, lam, dvals, fm)
        gD += dD
        gL += dL
    out = {"initial": g, "D": gD, "lambda": gL, "final": final}
    if agents is not None:
        c = (dt * agents["vol"] / dx ** 3)[:, None]
        m = act[:, None]
        out["secretion"] = np.where(m, gt1 * (c * agents["sat"]) + gt2 * c, 0.0)
        out["uptake"] = np.where(m, gt2 * c, 0.0)
        out["saturation"] = np.where(m, gt1 * (c * agents["sec"]), 0.0)
    return out
