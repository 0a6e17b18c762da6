"""Float64 PyTorch restatement of the substep with autograd: the reference gradient.

TEST INFRASTRUCTURE ONLY (see oracle/oracle.py): it stands in for the Taichi
autodiff gradient the reference would give (taichi is not installed), on small
instances.  It restates mpm_sim.py:153-340 like oracle/mpm_oracle.c, vectorised
over particles; branches become torch.where, so gradients follow the branch the
forward took (the same piecewise derivative a Taichi autodiff kernel takes).
The integer cell base (truncation) and the activation's floor carry no
gradient; clamps pass gradient only where inactive.
"""
from __future__ import annotations

import torch

E_base, nu_base = 0.1e4, 0.2
E_jelly, nu_jelly = 0.7e3, 0.3
E_payload, nu_payload = 2.0e5, 0.2
WATER_LAMBDA = 100000.0
GRAVITY = 10.0


def _lame(E, nu):
    return E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))


MU = {"base": _lame(E_base, nu_base)[0], "jelly": _lame(E_jelly, nu_jelly)[0],
      "payload": _lame(E_payload, nu_payload)[0]}
LA = {"base": _lame(E_base, nu_base)[1], "jelly": _lame(E_jelly, nu_jelly)[1],
      "payload": _lame(E_payload, nu_payload)[1]}


def activation(t, contraction, freq):
    """mpm_sim.py:173-180 with gradients w.r.t. contraction and freq."""
    period = 1.0 / (1.0 * freq)
    q = torch.floor(t / period).detach()
    phase = (t - period * q) / period
    arc = 0.5 * (1.0 - torch.cos(phase / contraction * 3.14159265))
    return torch.where(phase < contraction, arc, torch.zeros_like(arc))


def svd2(A):
    """taichi 1.7.4 _svd2d, vectorised: A (N,2,2) -> U, (s1, s2), V."""
    x = A[:, 0, 0] + A[:, 1, 1]
    y = A[:, 1, 0] - A[:, 0, 1]
    scale = 1.0 / torch.sqrt(x * x + y * y)
    c, s = x * scale, y * scale
    S00 = c * A[:, 0, 0] + s * A[:, 1, 0]
    S01 = c * A[:, 0, 1] + s * A[:, 1, 1]
    S11 = -s * A[:, 0, 1] + c * A[:, 1, 1]
    diag = S01.abs() < 1e-5
    tao = 0.5 * (S00 - S11)
    # the Jacobi branch is unused where |S01| < 1e-5; keep its sqrt away from 0
    # there so that its (discarded) derivative stays finite
    w = torch.sqrt(torch.where(diag, torch.ones_like(tao), tao * tao + S01 * S01))
    den = torch.where(tao > 0, tao + w, tao - w)
    den = torch.where(diag, torch.ones_like(den), den)
    t = torch.where(diag, torch.zeros_like(S01), S01 / den)
    cc = 1.0 / torch.sqrt(t * t + 1.0)
    ss = -t * cc
    s1 = torch.where(diag, S00, cc * cc * S00 - 2 * cc * ss * S01 + ss * ss * S11)
    s2 = torch.where(diag, S11, ss * ss * S00 + 2 * cc * ss * S01 + cc * cc * S11)
    cc = torch.where(diag, torch.ones_like(cc), cc)
    ss = torch.where(diag, torch.zeros_like(ss), ss)
    swap = s1 < s2
    s1n = torch.where(swap, s2, s1)
    s2n = torch.where(swap, s1, s2)
    V = torch.stack([torch.stack([torch.where(swap, -ss, cc), torch.where(swap, cc, ss)], -1),
                     torch.stack([torch.where(swap, -cc, -ss), torch.where(swap, -ss, cc)], -1)], -2)
    R = torch.stack([torch.stack([c, -s], -1), torch.stack([s, c], -1)], -2)
    U = R @ V
    return U, s1n, s2n, V


def substep(state, mat, fiber, p, t, nx, ny, domain_h, dt=2e-5):
    """One substep of one instance; state = dict(x, v, C, F) float64 tensors.

    p = dict(actuation, contraction, freq, payload_density) (0-d tensors).
    Returns the new state dict (functional, differentiable).
    """
    x, v, C, F = state["x"], state["v"], state["C"], state["F"]
    N = x.shape[0]
    dev = x.device
    inv_dx = float(nx)
    dx = 1.0 / nx
    p_vol = (dx * 0.5) ** 2
    p_mass = p_vol * 1
    live = mat >= 0
    base = torch.trunc(x.detach() * inv_dx - 0.5).long()
    inr = live & (base[:, 0] >= 0) & (base[:, 1] >= 0) & (base[:, 0] < nx - 2) & (base[:, 1] < ny - 2)
    fx = x * inv_dx - base.to(x.dtype)
    w = torch.stack([0.5 * (1.5 - fx) ** 2, 0.75 - (fx - 1) ** 2, 0.5 * (fx - 0.5) ** 2], 1)  # (N,3,2)
    eye = torch.eye(2, dtype=x.dtype, device=dev).expand(N, 2, 2)

    # P2G
    Fs = (eye + dt * C) @ F
    U, s1, s2, V = svd2(Fs)
    s1 = torch.clamp(s1, min=1e-6)
    s2 = torch.clamp(s2, min=1e-6)
    pay = mat == 2
    water = mat == 0
    jm = (mat == 1) | (mat == 3)
    n1 = torch.where(pay, torch.clamp(s1, 1 - 5e-3, 1 + 5e-3), s1)
    n2 = torch.where(pay, torch.clamp(s2, 1 - 5e-3, 1 + 5e-3), s2)
    J = n1 * n2
    sj = torch.sqrt(J)
    F_water = sj[:, None, None] * torch.eye(2, dtype=x.dtype, device=dev)
    Sig = torch.diag_embed(torch.stack([n1, n2], -1))
    F_pay = U @ Sig @ V.transpose(1, 2)
    Fn = torch.where(water[:, None, None], F_water, torch.where(pay[:, None, None], F_pay, Fs))
    def by_material(jelly, payload, water_v, other):
        full = lambda val: torch.full((N,), val, dtype=x.dtype, device=dev)  # noqa: E731
        return torch.where(jm, full(jelly), torch.where(pay, full(payload),
                                                        torch.where(water, full(water_v), full(other))))
    mu = by_material(MU["jelly"], MU["payload"], 0.0, MU["base"])
    la = by_material(LA["jelly"], LA["payload"], WATER_LAMBDA, LA["base"])
    R = U @ V.transpose(1, 2)
    stress = (2 * mu)[:, None, None] * (Fn - R) @ Fn.transpose(1, 2) + \
        (la * J * (J - 1))[:, None, None] * torch.eye(2, dtype=x.dtype, device=dev)
    a = activation(t, p["contraction"], p["freq"])
    pressure = p["actuation"] * a
    musc = (mat == 3)[:, None, None]
    fd = fiber
    stress = stress + torch.where(musc, fd[:, :, None] * fd[:, None, :] * (pressure * J)[:, None, None],
                                  torch.zeros_like(stress))
    mass = torch.where(pay, p_mass * p["payload_density"], torch.full_like(J, p_mass))
    stress = (-dt * p_vol * 4 * inv_dx * inv_dx) * stress
    affine = stress + mass[:, None, None] * C
    gp = torch.zeros((nx * ny, 2), dtype=x.dtype, device=dev)
    gm = torch.zeros((nx * ny,), dtype=x.dtype, device=dev)
    idx_live = torch.nonzero(inr).squeeze(1)
    for i in range(3):
        for j in range(3):
            off = torch.tensor([i, j], dtype=x.dtype, device=dev)
            dpos = (off - fx) * dx
            weight = w[:, i, 0] * w[:, j, 1]
            contrib = weight[:, None] * (mass[:, None] * v + (affine @ dpos[:, :, None])[:, :, 0])
            node = (base[:, 0] + i) * ny + (base[:, 1] + j)
            gp = gp.index_add(0, node[idx_live], contrib[idx_live])
            gm = gm.index_add(0, node[idx_live], (weight * mass)[idx_live])

    # grid update
    has = gm > 0
    gv = torch.where(has[:, None], gp / torch.where(has, gm, torch.ones_like(gm))[:, None], gp)
    ii = torch.arange(nx, device=dev, dtype=x.dtype)[:, None].expand(nx, ny).reshape(-1)
    jj = torch.arange(ny, device=dev, dtype=x.dtype)[None, :].expand(nx, ny).reshape(-1)
    dcx, dcy = nx // 20, ny // 20
    damp = torch.ones(nx * ny, dtype=x.dtype, device=dev)
    damp = torch.where(ii < dcx, damp * (0.95 + 0.05 * ii / dcx), damp)
    damp = torch.where(ii > nx - dcx, damp * (0.95 + 0.05 * (nx - ii) / dcx), damp)
    damp = torch.where(jj < dcy, damp * (0.95 + 0.05 * jj / dcy), damp)
    damp = torch.where(jj > ny - dcy, damp * (0.95 + 0.05 * (ny - jj) / dcy), damp)
    gv = torch.where(has[:, None], gv * damp[:, None], gv)
    g0, g1 = gv[:, 0], gv[:, 1]
    z = torch.zeros_like(g0)
    g0 = torch.where(has & (ii < 3) & (g0 < 0), z, g0)
    g0 = torch.where(has & (ii > nx - 3) & (g0 > 0), z, g0)
    g1 = torch.where(has & (jj < 3) & (g1 < 0), z, g1)
    g1 = torch.where(has & (jj > ny - 3) & (g1 > 0), z, g1)
    gv = torch.stack([g0, g1], -1)

    # G2P
    nv = torch.zeros_like(v)
    nC = torch.zeros_like(C)
    for i in range(3):
        for j in range(3):
            off = torch.tensor([i, j], dtype=x.dtype, device=dev)
            dpos = off - fx
            node = ((base[:, 0] + i) * ny + (base[:, 1] + j)).clamp(0, nx * ny - 1)
            g = gv[node]
            weight = w[:, i, 0] * w[:, j, 1]
            nv = nv + weight[:, None] * g
            nC = nC + (4 * inv_dx * weight)[:, None, None] * (g[:, :, None] * dpos[:, None, :])
    v_new = torch.where(inr[:, None], nv, v)
    C_new = torch.where(inr[:, None, None], nC, C)
    grav = torch.zeros_like(v_new)
    grav[:, 1] = dt * GRAVITY
    v_new = torch.where(live[:, None], v_new - grav, v)
    x_new = x + dt * v_new
    x_new = torch.stack([x_new[:, 0].clamp(0.001, 0.999), x_new[:, 1].clamp(0.001, domain_h - 0.001)], -1)
    x_new = torch.where(live[:, None], x_new, x)
    F_out = torch.where(inr[:, None, None], Fn, F)
    return {"x": x_new, "v": v_new, "C": C_new, "F": F_out}


def com_y(x, mat):
    """Payload CoM height, or jelly + muscle CoM without payload (mpm_sim.py:779-800)."""
    pay = mat == 2
    sel = pay if bool(pay.any()) else (mat == 1) | (mat == 3)
    return x[sel, 1].mean()


def displacement(x0, v0, mat, fiber, p, steps, nx, ny, domain_h, dt=2e-5, t0=0.0):
    """Payload displacement after `steps` substeps from rest-state (C = 0, F = I)."""
    N = x0.shape[0]
    st = {"x": x0, "v": v0, "C": torch.zeros((N, 2, 2), dtype=x0.dtype, device=x0.device),
          "F": torch.eye(2, dtype=x0.dtype, device=x0.device).repeat(N, 1, 1)}
    t = torch.tensor(t0, dtype=torch.float64, device=x0.device)
    for _ in range(steps):
        st = substep(st, mat, fiber, p, t, nx, ny, domain_h, dt)
        t = t + dt
    return com_y(st["x"], mat) - com_y(x0, mat), st
