"""Reverse mode (bfb_adjoint_run) against the oracle and finite differences.

* FP64 adjoint == the oracle's adjoint (oracle/lod_oracle.c:
  orc_lod_step_adjoint, composed over steps, plus the agents' update reversed
  here in numpy) to 1e-11 relative, for one step, several steps with
  checkpoint segments of uneven length, Dirichlet faces and agents;
* FP64 adjoint == FP64 central finite differences of the GPU forward path to
  1e-6 relative, on initial-field entries, D, lambda and per-agent rates;
* FP32 adjoint against the FP64 one;
* the torch.autograd.Function wrapper;
* the inverse-problem workload: 128^3 x 2 substrates, 10k agents in a 300 um
  sphere, 200 steps, checkpoints every 20, L2 loss against a target made by
  hidden secretion rates, FP64 gradients checked by central differences on 32
  sampled parameters, FP32 gradients against FP64.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from adjoint_ref import oracle_adjoint
from conftest import log_uniform

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _dev_tensor(a, prec, bfb):
    dt = torch.float64 if prec == bfb.FP64 else torch.float32
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dt).contiguous()


def _setup(bfb, prec, shape, S, rng, dirichlet=True, n_agents=0, dt=0.01, dx=20.0):
    nx, ny, nz = shape
    D = log_uniform(rng, 1e2, 1e5, S)
    lam = log_uniform(rng, 1e-3, 1.0, S)
    rho0 = rng.random((nx, ny, nz, S))
    env = bfb.Env(shape, S, dx=dx, precision=prec)
    env.set_coefficients(D, lam)
    env.set_field(rho0)
    fm = np.zeros((6, S), np.uint8)
    act = np.zeros(S, np.uint8)
    vals = np.zeros(S)
    if dirichlet:
        act[0] = 1
        vals[0] = 2.5
        fm[:, 0] = [1, 1, 0, 1, 1, 0]  # x-lo, x-hi, y-hi, z-lo for substrate 0
        if S > 1:
            act[1] = 1
            vals[1] = 0.75
            fm[:, 1] = [0, 0, 1, 0, 0, 1]
        env.set_dirichlet_uniform(act, vals, face_mask=fm)
    agents = None
    if n_agents:
        L = np.array(shape) * dx
        pos = rng.random((n_agents, 3)) * L * 0.6 + 0.2 * L
        pos[: n_agents // 4] = pos[0]  # several agents share voxels
        vol = rng.uniform(500.0, 3000.0, n_agents)
        sec, upt, sat = log_uniform(rng, 1e-2, 10.0, (3, n_agents, S))
        active = (rng.random(n_agents) > 0.1).astype(np.uint8)
        env.set_agents(pos, vol, sec, upt, sat, dt, active=active)
        agents = dict(pos=pos, vol=vol, sec=sec, upt=upt, sat=sat, active=active)
    dvals = np.zeros((nx, ny, nz, S)) + vals
    return env, D, lam, rho0, (dvals, fm * act[None, :]), agents


def _gpu_adjoint(bfb, env, rho0, w, n_steps, dt, K, agents, prec=None, coef_grads=True):
    prec = env.precision if prec is None else prec
    env.set_field(rho0)
    wt = _dev_tensor(w, prec, bfb)
    gi = torch.empty_like(wt)
    fin = torch.empty_like(wt)
    flags = bfb.STEP_DIFFUSION | (bfb.STEP_CELLS if agents is not None else 0)
    torch.cuda.synchronize()
    r = env.adjoint_run(dt, n_steps, wt.data_ptr(), flags=flags, checkpoint_every=K, dL_dinitial_ptr=gi.data_ptr(),
                        final_ptr=fin.data_ptr(), agent_grads=agents is not None, coef_grads=coef_grads)
    r["initial"] = gi.double().cpu().numpy()
    r["final"] = fin.double().cpu().numpy()
    return r


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("n_steps,K,shape,S,agents", [
    (1, 1, (13, 11, 9), 2, 0),
    (7, 3, (12, 10, 17), 3, 0),
    (5, 2, (10, 12, 11), 2, 120),
    (4, 4, (33, 9, 40), 1, 60),
    (3, 2, (24, 20, 32), 8, 150),
    (4, 3, (9, 11, 13), 3, 80),  # rows of 39 doubles: the device field's rows are padded
])
def test_adjoint_fp64_matches_oracle(bfb, oracle, n_steps, K, shape, S, agents):
    rng = np.random.default_rng(500 + n_steps * 7 + S)
    dt = 0.01
    env, D, lam, rho0, dirv, ag = _setup(bfb, bfb.FP64, shape, S, rng, n_agents=agents, dt=dt)
    w = rng.standard_normal(rho0.shape)
    ref = oracle_adjoint(oracle, rho0, w, n_steps, dt, env.dx, D, lam, dirv, ag)
    got = _gpu_adjoint(bfb, env, rho0, w, n_steps, dt, K, ag)
    assert np.array_equal(got["final"], ref["final"])  # forward is bit-exact
    assert _rel(got["initial"], ref["initial"]) <= 1e-11
    assert _rel(got["D"], ref["D"]) <= 1e-11
    assert _rel(got["lambda"], ref["lambda"]) <= 1e-11
    if ag is not None:
        for k in ("secretion", "uptake", "saturation"):
            assert _rel(got[k], ref[k]) <= 1e-11, k
    env.close()


def test_adjoint_is_deterministic(bfb):
    rng = np.random.default_rng(9)
    env, D, lam, rho0, dirv, ag = _setup(bfb, bfb.FP64, (40, 36, 44), 3, rng, n_agents=300)
    w = rng.standard_normal(rho0.shape)
    a = _gpu_adjoint(bfb, env, rho0, w, 6, 0.01, 4, ag)
    b = _gpu_adjoint(bfb, env, rho0, w, 6, 0.01, 4, ag)
    for k in ("initial", "D", "lambda", "secretion", "uptake", "saturation"):
        assert np.array_equal(a[k], b[k]), k
    env.close()


def test_adjoint_without_coefficient_gradients(bfb):
    """With dL/dD and dL/dlambda not asked for (NULL), the reverse pass skips
    their per-line sums; every other gradient is bit for bit the same."""
    rng = np.random.default_rng(19)
    for prec in (bfb.FP64, bfb.FP32):
        env, D, lam, rho0, dirv, ag = _setup(bfb, prec, (40, 36, 44), 3, rng, n_agents=300)
        w = rng.standard_normal(rho0.shape)
        full = _gpu_adjoint(bfb, env, rho0, w, 6, 0.01, 4, ag)
        part = _gpu_adjoint(bfb, env, rho0, w, 6, 0.01, 4, ag, coef_grads=False)
        assert "D" not in part and "lambda" not in part
        for k in ("final", "initial", "secretion", "uptake", "saturation"):
            assert np.array_equal(full[k], part[k]), k
        env.close()


def _field_fd(bfb, env, rho0, n_steps, dt, flags):
    env.set_field(rho0)
    env.simulate(dt, n_steps, flags)
    return env.get_field()


def test_adjoint_fp64_matches_finite_differences(bfb):
    """Central differences of L = <w, u_n> through the GPU FP64 forward."""
    rng = np.random.default_rng(77)
    dt, n = 0.01, 6
    shape, S = (24, 20, 28), 2
    env, D, lam, rho0, dirv, ag = _setup(bfb, bfb.FP64, shape, S, rng, n_agents=200, dt=dt)
    w = rng.standard_normal(rho0.shape)
    flags = bfb.STEP_DIFFUSION | bfb.STEP_CELLS
    g = _gpu_adjoint(bfb, env, rho0, w, n, dt, 2, ag)

    def fd(apply, h):
        # L = <w, u> is linear in u: difference the fields, then weight, so
        # that the difference is not taken between two large sums
        apply(+h)
        up = _field_fd(bfb, env, rho0p[0], n, dt, flags)
        apply(-h)
        um = _field_fd(bfb, env, rho0p[0], n, dt, flags)
        apply(0.0)
        return float(np.sum(w * (up - um))) / (2 * h)

    rho0p = [rho0]
    checks = []
    for d in range(S):
        h = 1e-4 * D[d]

        def setD(e, d=d):
            Dp = D.copy()
            Dp[d] += e
            env.set_coefficients(Dp, lam)
        checks.append((fd(setD, h), g["D"][d], f"D[{d}]"))
        h = 1e-4 * lam[d]

        def setL(e, d=d):
            Lp = lam.copy()
            Lp[d] += e
            env.set_coefficients(D, Lp)
        checks.append((fd(setL, h), g["lambda"][d], f"lambda[{d}]"))
    act = np.flatnonzero(ag["active"])
    for a in act[:: max(1, len(act) // 4)][:4]:
        for key in ("sec", "upt", "sat"):
            d = int(rng.integers(S))
            base = ag[key][a, d]
            h = 1e-3 * base

            def setA(e, key=key, a=a, d=d, base=base):
                arr = ag[key].copy()
                arr[a, d] = base + e
                kw = dict(sec=ag["sec"], upt=ag["upt"], sat=ag["sat"])
                kw[key] = arr
                env.set_agents(ag["pos"], ag["vol"], kw["sec"], kw["upt"], kw["sat"], dt, active=ag["active"])
            name = {"sec": "secretion", "upt": "uptake", "sat": "saturation"}[key]
            checks.append((fd(setA, h), g[name][a, d], f"{name}[{a},{d}]"))
    for _ in range(4):
        i, j, k, d = (int(rng.integers(x)) for x in (*shape, S))
        h = 1e-4

        def setR(e, i=i, j=j, k=k, d=d):
            r = rho0.copy()
            r[i, j, k, d] += e
            rho0p[0] = r
        checks.append((fd(setR, h), g["initial"][i, j, k, d], f"rho0[{i},{j},{k},{d}]"))
    scale = max(abs(c[1]) for c in checks)
    for fdv, adj, name in checks:
        assert abs(fdv - adj) <= 1e-6 * max(abs(adj), 1e-3 * scale), (name, fdv, adj)
    env.close()


def test_adjoint_fp32_close_to_fp64(bfb):
    rng = np.random.default_rng(31)
    dt, n = 0.01, 20
    shape, S = (48, 40, 56), 2
    env64, D, lam, rho0, dirv, ag = _setup(bfb, bfb.FP64, shape, S, rng, n_agents=500, dt=dt)
    w = rng.standard_normal(rho0.shape)
    g64 = _gpu_adjoint(bfb, env64, rho0, w, n, dt, 5, ag)
    env32 = bfb.Env(shape, S, dx=20.0, precision=bfb.FP32)
    env32.set_coefficients(D, lam)
    fm = dirv[1]
    act = (fm.sum(axis=0) > 0).astype(np.uint8)
    env32.set_dirichlet_uniform(act, dirv[0][0, 0, 0], face_mask=fm)
    env32.set_agents(ag["pos"], ag["vol"], ag["sec"], ag["upt"], ag["sat"], dt, active=ag["active"])
    g32 = _gpu_adjoint(bfb, env32, rho0, w, n, dt, 5, ag)
    assert _rel(g32["initial"], g64["initial"]) <= 1e-4
    assert _rel(g32["D"], g64["D"]) <= 1e-4
    assert _rel(g32["lambda"], g64["lambda"]) <= 1e-4
    for k in ("secretion", "uptake", "saturation"):
        assert _rel(g32[k], g64[k]) <= 1e-4, k
    env64.close()
    env32.close()


def test_autograd_function(bfb):
    from biofvm_b_b200.autograd import simulate
    rng = np.random.default_rng(3)
    dt, n = 0.01, 5
    shape, S = (20, 18, 22), 2
    env, D, lam, rho0, dirv, ag = _setup(bfb, bfb.FP64, shape, S, rng, n_agents=80, dt=dt)
    w = rng.standard_normal(rho0.shape)
    ref = _gpu_adjoint(bfb, env, rho0, w, n, dt, 2, ag)
    r0 = torch.tensor(rho0, device="cuda", requires_grad=True)
    Dt = torch.tensor(D, requires_grad=True)
    Lt = torch.tensor(lam, requires_grad=True)
    sec = torch.tensor(ag["sec"], requires_grad=True)
    upt = torch.tensor(ag["upt"], requires_grad=True)
    sat = torch.tensor(ag["sat"], requires_grad=True)
    agents = dict(pos=ag["pos"], volume=ag["vol"], dt=dt, active=ag["active"])
    out = simulate(env, r0, Dt, Lt, dt, n, checkpoint_every=2, agents=agents, secretion=sec, uptake=upt,
                   saturation=sat)
    assert np.array_equal(out.detach().cpu().numpy(), ref["final"])
    loss = (out * torch.tensor(w, device="cuda")).sum()
    loss.backward()
    assert np.array_equal(r0.grad.cpu().numpy(), ref["initial"])
    assert np.array_equal(Dt.grad.numpy(), ref["D"])
    assert np.array_equal(Lt.grad.numpy(), ref["lambda"])
    assert np.array_equal(sec.grad.numpy(), ref["secretion"])
    assert np.array_equal(upt.grad.numpy(), ref["uptake"])
    assert np.array_equal(sat.grad.numpy(), ref["saturation"])
    env.close()


def test_adjoint_rejects_bad_arguments(bfb):
    env = bfb.Env((8, 8, 8), 1, precision=bfb.FP64)
    env.set_coefficients([1e3], [0.1])
    buf = torch.zeros(8 * 8 * 8, dtype=torch.float64, device="cuda")
    with pytest.raises(bfb.BFBError):
        env.adjoint_run(0.01, 2, buf.data_ptr(), flags=bfb.STEP_DIFFUSION | bfb.STEP_BULK)
    with pytest.raises(bfb.BFBError):
        env.adjoint_run(0.01, 0, buf.data_ptr())
    env.close()


# ---------------------------------------------------------------------------
# The inverse-problem workload at full size
# ---------------------------------------------------------------------------
def _inverse_problem(bfb, rng):
    n, S, dx, dt = 128, 2, 20.0, 0.01
    D = np.array([1e5, 2e3])
    lam = np.array([0.1, 0.01])
    rho0 = np.zeros((n, n, n, S))
    na = 10_000
    L = n * dx
    u = rng.normal(size=(na, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    pos = L / 2 + u * (300.0 * rng.random((na, 1)) ** (1.0 / 3.0))
    vol = np.full(na, 4.0 / 3.0 * math.pi * 1000.0)
    sec_true, upt, sat = log_uniform(rng, 1e-2, 10.0, (3, na, S))
    sec_guess = log_uniform(rng, 1e-2, 10.0, (na, S))
    return dict(n=n, S=S, dx=dx, dt=dt, D=D, lam=lam, rho0=rho0, pos=pos, vol=vol, sec_true=sec_true,
                sec=sec_guess, upt=upt, sat=sat)


def test_inverse_problem_128cube_10k_agents(bfb):
    """L = 0.5*||u_200 - target||^2; target from hidden secretion rates."""
    rng = np.random.default_rng(2024)
    P = _inverse_problem(bfb, rng)
    n, S, dt, steps, K = P["n"], P["S"], P["dt"], 200, 20
    flags = bfb.STEP_DIFFUSION | bfb.STEP_CELLS

    def make(prec, sec):
        env = bfb.Env((n, n, n), S, dx=P["dx"], precision=prec)
        env.set_coefficients(P["D"], P["lam"])
        env.set_field(P["rho0"])
        env.set_agents(P["pos"], P["vol"], sec, P["upt"], P["sat"], dt)
        return env

    env = make(bfb.FP64, P["sec_true"])
    env.simulate(dt, steps, flags)
    target = env.get_field()
    env.set_agents(P["pos"], P["vol"], P["sec"], P["upt"], P["sat"], dt)

    def loss():
        env.set_field(P["rho0"])
        env.simulate(dt, steps, flags)
        r = env.get_field() - target
        return 0.5 * float(np.sum(r * r)), r

    L0, resid = loss()
    assert L0 > 0
    g64 = _gpu_adjoint(bfb, env, P["rho0"], resid, steps, dt, K, P)

    # 32 sampled parameters: D, lambda and 28 per-agent rates
    samples = [("D", d) for d in range(S)] + [("lambda", d) for d in range(S)]
    agents = rng.choice(len(P["pos"]), 28, replace=False)
    kinds = ["secretion", "uptake", "saturation"]
    samples += [(kinds[q % 3], (int(a), int(rng.integers(S)))) for q, a in enumerate(agents)]
    key = {"secretion": "sec", "uptake": "upt", "saturation": "sat"}
    def perturbed_field(kind, idx, e):
        # every call sets all parameters, perturbing only (kind, idx)
        Dv, Lv = P["D"].copy(), P["lam"].copy()
        arrs = {k: P[k].copy() for k in ("sec", "upt", "sat")}
        if kind == "D":
            Dv[idx] += e
        elif kind == "lambda":
            Lv[idx] += e
        else:
            arrs[key[kind]][idx] += e
        env.set_coefficients(Dv, Lv)
        env.set_agents(P["pos"], P["vol"], arrs["sec"], arrs["upt"], arrs["sat"], dt)
        env.set_field(P["rho0"])
        env.simulate(dt, steps, flags)
        return env.get_field()

    def central(kind, idx, h):
        # L(+h) - L(-h) = sum (u+ - u-) ((u+ + u-)/2 - target): formed from the
        # field difference, not as the difference of two large sums
        up, um = perturbed_field(kind, idx, h), perturbed_field(kind, idx, -h)
        return float(np.sum((up - um) * (0.5 * (up + um) - target))) / (2 * h)

    worst = 0.0
    for kind, idx in samples:
        if kind in ("D", "lambda"):
            h = 1e-3 * (P["D"] if kind == "D" else P["lam"])[idx]
            adj = g64[kind][idx]
        else:
            h = 1e-3 * P[key[kind]][idx]
            adj = g64[kind][idx]
        # central differences at h and h/2, Richardson-extrapolated (error O(h^4))
        fdv = (4 * central(kind, idx, h / 2) - central(kind, idx, h)) / 3
        scale = max(abs(g64[kind]).max(), 1e-300)
        assert abs(fdv - adj) <= 1e-6 * max(abs(adj), 1e-3 * scale), (kind, idx, fdv, adj)
        worst = max(worst, abs(fdv - adj) / max(abs(adj), 1e-3 * scale))
    env.set_coefficients(P["D"], P["lam"])
    env.set_agents(P["pos"], P["vol"], P["sec"], P["upt"], P["sat"], dt)

    # FP32 gradients against FP64
    env32 = make(bfb.FP32, P["sec"])
    g32 = _gpu_adjoint(bfb, env32, P["rho0"], resid, steps, dt, K, P)
    errs = {k: _rel(g32[k], g64[k]) for k in ("D", "lambda", "secretion", "uptake", "saturation")}
    for k, e in errs.items():
        assert e <= 1e-3, k

    # the inverse problem itself: three steepest-descent steps on the secretion
    # rates (kept positive, step halved until the loss drops) lower the loss
    sec = P["sec"].copy()
    L_cur, g_cur = L0, g64["secretion"]
    eta = 0.5 * L0 / max(float(np.sum(g_cur * g_cur)), 1e-300)
    for _ in range(3):
        for _try in range(20):
            trial = np.maximum(sec - eta * g_cur, 1e-6)
            env.set_agents(P["pos"], P["vol"], trial, P["upt"], P["sat"], dt)
            L_try, r_try = loss()
            if L_try < L_cur:
                break
            eta *= 0.5
        assert L_try < L_cur
        sec, L_cur = trial, L_try
        g_cur = _gpu_adjoint(bfb, env, P["rho0"], r_try, steps, dt, K, P)["secretion"]
    print(f"\ninverse problem (128^3 x 2, 10k agents, 200 steps, checkpoints every {K}): "
          f"max FD mismatch on 32 parameters {worst:.2e} (relative); FP32 vs FP64 gradient rel Linf "
          + ", ".join(f"{k} {e:.1e}" for k, e in errs.items())
          + f"; loss {L0:.4e} -> {L_cur:.4e} after 3 descent steps")
    env32.close()
    env.close()
