"""Automatic-differentiation reference of the smoothing cost (TEST INFRASTRUCTURE).

The adjoint kernel's gradient is checked against central differences of the C
oracle and, here, against automatic differentiation of a pure-tensor
restatement of the same cost: float64 torch on the CPU, differentiated by
``torch.autograd``.  It stands in for ``jax.grad`` of a pure-JAX FK + SDF
reference, which cannot run here (jax is not installed): the "jax check" is
not run.  Only the test suite imports this module.

It restates ``orc_smooth_cost`` (oracle/prrtc_oracle.c:996-1030) term for term:
FK as the oracle's ``fk_sorted_f64`` (prrtc_oracle.c:124-196: parent transform
from the quaternion, SE(3) exponential of the twist times the joint value,
composition in table order, frames reordered by ``fk_topo_inv``), the primitive
distances of prrtc_oracle.c:228-264, softplus_beta(margin - d) over every
(robot sphere, world primitive) pair and every self pair, plus
w_len * sum |q_{w+1} - q_w|^2.
"""
from __future__ import annotations

import numpy as np
import torch

_F64 = torch.float64


def _t(x, dtype=_F64):
    return torch.as_tensor(np.asarray(x), dtype=dtype)


def _quat_to_mat(q7: torch.Tensor) -> torch.Tensor:
    """Rotation of the normalised quaternion (w, x, y, z) (prrtc_oracle.c:125-131)."""
    w, x, y, z = q7[0], q7[1], q7[2], q7[3]
    n = torch.sqrt(w * w + x * x + y * y + z * z)
    if float(n) > 0:
        w, x, y, z = w / n, x / n, y / n, z / n
    else:
        w, x, y, z = (torch.ones((), dtype=_F64), torch.zeros((), dtype=_F64), torch.zeros((), dtype=_F64),
                      torch.zeros((), dtype=_F64))
    return torch.stack([
        torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)]),
        torch.stack([2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)]),
        torch.stack([2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]),
    ])


def _se3_exp(tw: torch.Tensor, val: torch.Tensor):
    """R = I + A K + B K^2, t = (I + B K + C K^2) v for the twist (v, w) * val
    (prrtc_oracle.c:134-160); the series below theta = 1e-8 as the oracle,
    written so that autograd sees no square root of zero."""
    v = tw[:3] * val
    w = tw[3:] * val
    th2 = (w * w).sum()
    small = bool(th2 < 1e-16)
    if small:
        A, B, C = 1 - th2 / 6, 0.5 - th2 / 24, 1.0 / 6.0 - th2 / 120
    else:
        th = torch.sqrt(th2)
        s, c = torch.sin(th), torch.cos(th)
        A, B, C = s / th, (1 - c) / th2, (th - s) / (th2 * th)
    zero = torch.zeros((), dtype=_F64)
    K = torch.stack([torch.stack([zero, -w[2], w[1]]), torch.stack([w[2], zero, -w[0]]),
                     torch.stack([-w[1], w[0], zero])])
    K2 = torch.outer(w, w) - th2 * torch.eye(3, dtype=_F64)
    eye = torch.eye(3, dtype=_F64)
    R = eye + A * K + B * K2
    V = eye + B * K + C * K2
    return R, V @ v


def fk_frames(ctx: dict, q: torch.Tensor) -> list:
    """World frames (R, t) in output order: frame k is joint topo_inv[k] of the
    table order (prrtc_oracle.c:171-206)."""
    tw = _t(ctx["fk_twists"]).reshape(-1, 6)
    ptf = _t(ctx["fk_parent_tf"]).reshape(-1, 7)
    par = np.asarray(ctx["fk_parent_idx"]).reshape(-1)
    act = np.asarray(ctx["fk_act_idx"]).reshape(-1)
    J = tw.shape[0]
    mimic_idx = np.asarray(ctx.get("fk_mimic_act_idx", np.full(J, -1))).reshape(-1)
    mimic_mul = _t(ctx.get("fk_mimic_mul", np.zeros(J))).reshape(-1)
    mimic_off = _t(ctx.get("fk_mimic_off", np.zeros(J))).reshape(-1)
    topo = np.asarray(ctx.get("fk_topo_inv", np.arange(J))).reshape(-1)
    W = []
    for j in range(J):
        if mimic_idx.size == J and mimic_idx[j] >= 0:
            val = mimic_mul[j] * q[int(mimic_idx[j])] + mimic_off[j]
        elif act[j] >= 0:
            val = q[int(act[j])]
        else:
            val = torch.zeros((), dtype=_F64)
        P_R = _quat_to_mat(ptf[j, :4])
        P_t = ptf[j, 4:]
        E_R, E_t = _se3_exp(tw[j], val)
        L_R, L_t = P_R @ E_R, P_R @ E_t + P_t
        p = int(par[j])
        if 0 <= p < j:
            R0, t0 = W[p]
            W.append((R0 @ L_R, R0 @ L_t + t0))
        else:
            W.append((L_R, L_t))
    return [W[int(topo[k])] if topo.size == J else W[k] for k in range(J)]


def _softplus(x: torch.Tensor, beta: float) -> torch.Tensor:
    z = beta * x
    return (torch.clamp(z, min=0) + torch.log1p(torch.exp(-torch.abs(z)))) / beta


def _dist_spheres(c, r, ws):
    return torch.linalg.norm(c[:, None, :] - ws[None, :, :3], dim=-1) - r[:, None] - ws[None, :, 3]


def _dist_capsules(c, r, wc):
    p1, p2, rc = wc[:, :3], wc[:, 3:6], wc[:, 6]
    a = p2 - p1
    L2 = (a * a).sum(-1)
    w = c[:, None, :] - p1[None]
    t = torch.where(L2[None] > 0, (w * a[None]).sum(-1) / torch.where(L2 > 0, L2, torch.ones_like(L2))[None],
                    torch.zeros_like(w[..., 0]))
    t = torch.clamp(t, 0.0, 1.0)
    e = w - t[..., None] * a[None]
    return torch.linalg.norm(e, dim=-1) - r[:, None] - rc[None]


def _dist_boxes(c, r, wb):
    ctr, axes, half = wb[:, :3], wb[:, 3:12].reshape(-1, 3, 3), wb[:, 12:15]
    p = c[:, None, :] - ctr[None]
    l = torch.einsum("sbi,bki->sbk", p, axes)  # coordinate along each box axis
    q = torch.abs(l) - half[None]
    out = torch.linalg.norm(torch.clamp(q, min=0.0), dim=-1)
    inside = torch.clamp(q.max(dim=-1).values, max=0.0)
    return out + inside - r[:, None]


def _dist_halfspaces(c, r, wh):
    n, p = wh[:, :3], wh[:, 3:6]
    return ((c[:, None, :] - p[None]) * n[None]).sum(-1) - r[:, None]


def smooth_cost(ctx: dict, waypoints: torch.Tensor, margin: float = 0.02, beta: float = 50.0,
                w_len: float = 1.0) -> torch.Tensor:
    """Cost of one path [W, dim] (float64), differentiable by autograd.  The
    scalar parameters are rounded to float32 first, as the oracle and the
    kernel receive them."""
    margin, beta, w_len = (float(np.float32(v)) for v in (margin, beta, w_len))
    link = np.asarray(ctx["sphere_link_idx"]).reshape(-1)
    local = _t(ctx["sphere_local"]).reshape(-1, 3)
    rad = _t(ctx["sphere_radius"]).reshape(-1)
    tables = {k: _t(ctx[k]) for k in ("world_spheres", "world_capsules", "world_boxes", "world_halfspaces")
              if ctx.get(k) is not None and np.asarray(ctx[k]).size}
    pairs = np.asarray(ctx["self_pairs"]).reshape(-1, 2) if ctx.get("self_pairs") is not None else np.zeros((0, 2))
    total = torch.zeros((), dtype=_F64)
    for w in range(waypoints.shape[0]):
        F = fk_frames(ctx, waypoints[w])
        ok = [(s, int(link[s])) for s in range(link.size) if 0 <= link[s] < len(F)]
        idx = [s for s, _ in ok]
        c = torch.stack([F[f][0] @ local[s] + F[f][1] for s, f in ok])
        r = rad[idx]
        for key, fn in (("world_spheres", _dist_spheres), ("world_capsules", _dist_capsules),
                        ("world_boxes", _dist_boxes), ("world_halfspaces", _dist_halfspaces)):
            if key in tables:
                total = total + _softplus(margin - fn(c, r, tables[key]), beta).sum()
        pos = {s: k for k, s in enumerate(idx)}
        keep = [(pos[int(i)], pos[int(j)], int(i), int(j)) for i, j in pairs if int(i) in pos and int(j) in pos]
        if keep:
            a = torch.tensor([k[0] for k in keep])
            b = torch.tensor([k[1] for k in keep])
            d = torch.linalg.norm(c[a] - c[b], dim=-1) - r[a] - r[b]
            total = total + _softplus(margin - d, beta).sum()
    dq = waypoints[1:] - waypoints[:-1]
    return total + w_len * (dq * dq).sum()


def smooth_grad(ctx: dict, waypoints: np.ndarray, margin: float = 0.02, beta: float = 50.0,
                w_len: float = 1.0):
    """(cost, d cost / d waypoints) by torch.autograd in float64."""
    x = torch.tensor(np.asarray(waypoints, dtype=np.float64), requires_grad=True)
    cost = smooth_cost(ctx, x, margin, beta, w_len)
    (g,) = torch.autograd.grad(cost, x)
    return float(cost.detach()), g.numpy()
