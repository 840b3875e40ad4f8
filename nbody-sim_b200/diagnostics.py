"""Accuracy diagnostics: force error of the tree walk against an FP64 direct
sum, and the conserved quantities of a gravity-only disk.

The reference has no diagnostics of its own; these measure the quantities
its force criterion (src/physics/BHTree.cu:577) and KDK integrator
(src/main.cu:101-139) trade off.  Heavy sums run on the GPU
(``nbody_direct_f64``); the O(N) sums are FP64 numpy on the host.

Conventions (G = 1, star at the origin, disk in XZ, +Y pole):

* self-gravity  a_i = sum_{j != i} m_j d_ij / (|d_ij|^2 + eps^2)^{3/2}
* star term     -M x_i / (|x_i|^2 + eps^2)^{3/2}  (softened, BHTree.cu:547-553)
* energy        E = sum 1/2 m v^2 - sum M m / sqrt(r^2 + eps^2)
                    - sum_{i<j} m_i m_j / sqrt(r_ij^2 + eps^2)
* L_y           sum m (z v_x - x v_z)
"""
from __future__ import annotations

import importlib

import numpy as np


def _nb():
    return importlib.import_module("nbody-sim_b200")


def star_accel(x, y, z, eps, star_mass):
    r2 = x * x + y * y + z * z + eps * eps
    f = -star_mass / (r2 * np.sqrt(r2))
    return f * x, f * y, f * z


def _rel_err(a, ref):
    return np.linalg.norm(a - ref, axis=1) / np.linalg.norm(ref, axis=1)


def _summary(e):
    return {"median": float(np.median(e)), "p99": float(np.percentile(e, 99)),
            "max": float(np.max(e))}


def force_errors(st, theta: float, eps: float, star_mass: float, targets, leaf_max=None,
                 targets_per_lane=None, keep=False):
    """Walk accelerations (phase API: bbox, build, summarize, force) against the
    FP64 direct sum on the same float32 positions, at the target indices.

    ``st``: host arrays x, y, z (float32) and m.  Returns a dict with the
    relative error of the total acceleration and of the self-gravity part
    (walk with star_mass 0) as median / p99 / max, and the walk's
    interactions per body.  ``keep`` adds the per-target FP64 self-gravity
    yardstick ("direct_self", k x 3)."""
    import torch
    nb = _nb()
    n = len(st["x"])
    p = nb.allocate_particles_gpu(n)
    for k in ("x", "y", "z"):
        p.arrays[k].copy_(torch.from_numpy(np.ascontiguousarray(st[k], np.float32)))
    p.arrays["mass"].copy_(torch.from_numpy(np.ascontiguousarray(st["m"], np.float32)))
    tree = nb.Octree(n, leaf_max, targets_per_lane)
    tree.reset()
    tree.bbox(p)
    tree.build(p)
    tree.summarize()
    tree.sort()
    tg = np.asarray(targets, np.int64)
    out = {}
    acc = {}
    for name, sm in (("self", 0.0), ("total", star_mass)):
        tree.force(p, theta, eps, sm)
        a = np.stack([p.arrays[k].cpu().numpy()[tg] for k in ("ax", "ay", "az")], 1)
        acc[name] = a.astype(np.float64)
        if name == "self":
            out["interactions_per_body"] = tree.stats().interactions / n
    status = tree.stats().status
    tree.close()
    x64 = [torch.from_numpy(np.asarray(st[k], np.float32).astype(np.float64)).cuda()
           for k in ("x", "y", "z")]
    m32 = torch.from_numpy(np.ascontiguousarray(st["m"], np.float32)).cuda()
    t32 = torch.from_numpy(tg.astype(np.int32)).cuda()
    dx, dy, dz, _ = nb.direct_f64(*x64, m32, eps, targets=t32)
    d_self = np.stack([dx.cpu().numpy(), dy.cpu().numpy(), dz.cpu().numpy()], 1)
    xs = [np.asarray(st[k], np.float32)[tg].astype(np.float64) for k in ("x", "y", "z")]
    d_total = d_self + np.stack(star_accel(*xs, eps, star_mass), 1)
    out["self"] = _summary(_rel_err(acc["self"], d_self))
    out["total"] = _summary(_rel_err(acc["total"], d_total))
    out["status"] = status
    if keep:
        out["direct_self"] = d_self
    return out


def engine_force_errors(params, st, targets):
    """The engine's own walk (nbody_sim with ``params``: the groups, walk mode
    and leaf size a timed step uses) against the FP64 direct sum on the same
    float32 positions, at the target indices: relative error of the total
    acceleration and of the self-gravity part (a second engine with
    star_mass 0) as median / p99 / max."""
    import torch
    nb = _nb()
    n = len(st["x"])
    tg = np.asarray(targets, np.int64)
    acc = {}
    for name, sm in (("self", 0.0), ("total", params.star_mass)):
        p = type(params).from_buffer_copy(params)
        p.star_mass = sm
        p.state_precision = nb.STATE_F32
        sim = nb.Sim(p, n)
        sim.set_state(*[np.ascontiguousarray(st[k], np.float32)
                        for k in ("x", "y", "z", "vx", "vy", "vz")], st["m"])
        g = sim.get_state(accel=True)
        acc[name] = np.stack([g[k][tg] for k in ("ax", "ay", "az")], 1).astype(np.float64)
        status = sim.stats().status
        sim.close()
        if status:
            raise RuntimeError(f"engine status {status} in the force-error run")
    x64 = [torch.from_numpy(np.asarray(st[k], np.float32).astype(np.float64)).cuda()
           for k in ("x", "y", "z")]
    m32 = torch.from_numpy(np.ascontiguousarray(st["m"], np.float32)).cuda()
    t32 = torch.from_numpy(tg.astype(np.int32)).cuda()
    eps = params.softening
    dx, dy, dz, _ = nb.direct_f64(*x64, m32, eps, targets=t32)
    d_self = np.stack([dx.cpu().numpy(), dy.cpu().numpy(), dz.cpu().numpy()], 1)
    xs = [np.asarray(st[k], np.float32)[tg].astype(np.float64) for k in ("x", "y", "z")]
    d_total = d_self + np.stack(star_accel(*xs, eps, params.star_mass), 1)
    return {"self": _summary(_rel_err(acc["self"], d_self)),
            "total": _summary(_rel_err(acc["total"], d_total))}


def conserved(st, m, eps: float, star_mass: float):
    """Softened energy (kinetic, star, pair parts) and L_y of a state.

    ``st``: host arrays x..vz (any float type, taken as FP64); ``m`` float32.
    The pair term is the FP64 direct sum over every body (GPU)."""
    import torch
    nb = _nb()
    x, y, z, vx, vy, vz = [np.asarray(st[k], np.float64) for k in ("x", "y", "z", "vx", "vy",
                                                                    "vz")]
    md = np.asarray(m, np.float32).astype(np.float64)
    kin = 0.5 * np.sum(md * (vx * vx + vy * vy + vz * vz))
    u_star = -star_mass * np.sum(md / np.sqrt(x * x + y * y + z * z + eps * eps))
    xt = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (x, y, z)]
    mt = torch.from_numpy(np.ascontiguousarray(m, np.float32)).cuda()
    _, _, _, phi = nb.direct_f64(*xt, mt, eps, want_acc=False, want_phi=True)
    w = 0.5 * np.sum(md * phi.cpu().numpy())
    ly = np.sum(md * (z * vx - x * vz))
    return {"E": float(kin + u_star + w), "K": float(kin), "U_star": float(u_star),
            "W": float(w), "L_y": float(ly)}
