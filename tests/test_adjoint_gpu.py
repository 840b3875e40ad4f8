"""Adjoint of a disk trajectory (nbody_adjoint_*) against central finite
differences of the same frozen-tree forward.

The backward pass is the reverse mode of the recorded computation with the
tree frozen (sort order, warp groups, source lists).  The replay entry point
runs that function from perturbed inputs; its FP64-interaction variant is
the finite-difference reference (FP64 central differences, h = 1e-6
relative to the body's speed or radius): with FP32 interactions the
perturbed body's own rounding would scatter the difference quotient by
~1e-3.  The loss is the mass-weighted mean e^2 of the bodies that end inside
r < 2 AU; the two sides of a difference are subtracted body by body before
the sum, so the quotient does not cancel against the whole loss.  Bar: 1e-4
relative per checked component.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def setup(nb, cuda, n=3000, steps=40, theta=0.5, seed=3, drag=1e-3, pm=3.0, pr=10.0):
    prm = nb.sim_params(dt=0.005, theta=theta, softening=1e-3, star_mass=1.0, r_coll=0.0,
                        restitution=0.0, gas_drag_rate=drag, perturber_enabled=1,
                        perturber_mass_mjup=pm, perturber_radius_au=pr, perturber_phase0=0.0,
                        state_precision=nb.NBODY_STATE_F64)
    d = nb.make_disk(n, 0.5, 5.0, 0.01, 0.005, 1.0, seed)
    x0 = cuda.tensor(np.stack([d["x"], d["y"], d["z"]]), dtype=cuda.float64, device="cuda")
    v0 = cuda.tensor(np.stack([d["vx"], d["vy"], d["vz"]]), dtype=cuda.float64, device="cuda")
    mass = cuda.full((n,), 1e-8, dtype=cuda.float32, device="cuda")
    eng = nb.Adjoint(prm, n, steps)
    return eng, x0, v0, mass, pm, pr


def loss_diff(nb, cuda, plus, minus, mass):
    """L(plus) - L(minus), subtracted body by body (same r < 2 mask)."""
    (xp, vp), (xm, vm) = plus, minus
    rp = cuda.sqrt((xp * xp).sum(0))
    rm = cuda.sqrt((xm * xm).sum(0))
    assert cuda.equal(rp < 2.0, rm < 2.0)
    w = mass.to(cuda.float64) * (rp < 2.0).to(cuda.float64)
    d = nb.eccentricity2(xp, vp) - nb.eccentricity2(xm, vm)
    return float(((w * d).sum() / w.sum()).item())


def fd(nb, cuda, eng, mass, x0, v0, pm, pr, which, c=0, b=0, h=0.0, dpm=0.0, dpr=0.0):
    def run(sign):
        x, v = x0.clone(), v0.clone()
        if which == "x":
            x[c, b] += sign * h
        elif which == "v":
            v[c, b] += sign * h
        return eng.replay(x, v, pm + sign * dpm, pr + sign * dpr, fp64=True)
    step = h if which in ("x", "v") else (dpm or dpr)
    return loss_diff(nb, cuda, run(1.0), run(-1.0), mass) / (2.0 * step)


def test_replay_reproduces_the_recorded_forward(nb, cuda):
    eng, x0, v0, mass, pm, pr = setup(nb, cuda)
    x, v = eng.forward(x0, v0, mass, pm, pr)
    xr, vr = eng.replay(x0, v0, pm, pr)
    assert cuda.equal(x, xr) and cuda.equal(v, vr)
    st = eng.stats()
    assert st.ms_forward > 0 and st.tape_bytes > 0
    eng.close()


def gradients(nb, cuda, eng, x0, v0, mass, pm, pr):
    x0r = x0.clone().requires_grad_(True)
    v0r = v0.clone().requires_grad_(True)
    pmt = cuda.tensor(pm, dtype=cuda.float64, device="cuda", requires_grad=True)
    prt = cuda.tensor(pr, dtype=cuda.float64, device="cuda", requires_grad=True)
    x, v = nb.disk_trajectory(eng, x0r, v0r, pmt, prt, mass)
    loss = nb.eccentricity_loss(x, v, mass)
    loss.backward()
    return loss.item(), x0r.grad, v0r.grad, pmt.grad.item(), prt.grad.item()


def rel(a, b):
    return abs(a - b) / max(abs(a), abs(b), 1e-300)


@pytest.mark.parametrize("theta", [0.5, 0.0])
def test_velocity_gradient_matches_central_differences(nb, cuda, theta):
    eng, x0, v0, mass, pm, pr = setup(nb, cuda, theta=theta, n=3000 if theta else 1500)
    _, gx0, gv0, _, _ = gradients(nb, cuda, eng, x0, v0, mass, pm, pr)
    r0 = cuda.sqrt((x0 * x0).sum(0)).cpu().numpy()
    speed = cuda.sqrt((v0 * v0).sum(0)).cpu().numpy()
    rng = np.random.default_rng(0)
    inner = np.nonzero(r0 < 1.5)[0]
    bodies = rng.choice(inner, 12, replace=False)
    errs = []
    for k, b in enumerate(bodies):
        c = k % 3
        g = fd(nb, cuda, eng, mass, x0, v0, pm, pr, "v", c, int(b), 1e-6 * speed[b])
        errs.append(rel(float(gv0[c, b]), g))
    assert max(errs) <= 1e-4, errs
    # position components too
    for k, b in enumerate(bodies[:3]):
        g = fd(nb, cuda, eng, mass, x0, v0, pm, pr, "x", k, int(b), 1e-6 * r0[b])
        assert rel(float(gx0[k, b]), g) <= 1e-4, (k, b)
    eng.close()


def test_perturber_gradients_match_central_differences(nb, cuda):
    """A weak parameter: at h = 1e-6 the FP64 trajectories' own round-off
    (~1e-15 per step on positions that move ~1e-14 apart) scatters the
    quotient by ~1e-4, so the step is 1e-5 relative (the quotient is flat
    to ~1e-8 between 1e-4 and 1e-5)."""
    # a closer, heavier perturber so its parameters matter within the run
    eng, x0, v0, mass, pm, pr = setup(nb, cuda, pm=5.0, pr=6.0, steps=60)
    _, _, _, gm, gr = gradients(nb, cuda, eng, x0, v0, mass, pm, pr)
    fd_m = fd(nb, cuda, eng, mass, x0, v0, pm, pr, "m", dpm=1e-5 * pm)
    fd_r = fd(nb, cuda, eng, mass, x0, v0, pm, pr, "r", dpr=1e-5 * pr)
    assert rel(gm, fd_m) <= 1e-4, (gm, fd_m)
    assert rel(gr, fd_r) <= 1e-4, (gr, fd_r)
    eng.close()


def test_adjoint_rejects_collisions(nb, cuda):
    prm = nb.sim_params(dt=0.005, r_coll=1e-5, state_precision=nb.NBODY_STATE_F64)
    with pytest.raises(nb.NBodyError) as e:
        nb.Adjoint(prm, 100, 5)
    assert e.value.code == nb.NBODY_ERR_ARG


def test_checkpointed_engine_gives_the_tape_engine_gradient(nb, cuda):
    """NBODY_ADJOINT_CHECKPOINT keeps FP64 states every 25 levels only and
    rebuilds the others in the backward by running each step backwards in
    time (drag inverted in closed form), re-recording each level's tree and
    tape.  Its forward is the tape engine's, bit for bit; its gradient
    equals the tape engine's to the rounding of the reversed steps (their
    drift is reset at every checkpoint); it holds a fraction of the memory."""
    n, steps = 3000, 60
    eng_t, x0, v0, mass, pm, pr = setup(nb, cuda, n=n, steps=steps)
    eng_c = nb.Adjoint(eng_t.params, n, steps, mode="checkpoint", checkpoint_every=25)
    xt, vt = eng_t.forward(x0, v0, mass, pm, pr)
    xc, vc = eng_c.forward(x0, v0, mass, pm, pr)
    assert cuda.equal(xt, xc) and cuda.equal(vt, vc)
    _, gxt, gvt, gmt, grt = gradients(nb, cuda, eng_t, x0, v0, mass, pm, pr)
    _, gxc, gvc, gmc, grc = gradients(nb, cuda, eng_c, x0, v0, mass, pm, pr)
    scale_v = float(gvt.abs().max())
    scale_x = float(gxt.abs().max())
    dv = float((gvc - gvt).abs().max()) / scale_v
    dx = float((gxc - gxt).abs().max()) / scale_x
    print(f"checkpoint vs tape: velocity {dv:.3e} position {dx:.3e} of the largest; "
          f"mass {rel(gmc, gmt):.3e} radius {rel(grc, grt):.3e}")
    assert dv <= 1e-9 and dx <= 1e-9
    assert rel(gmc, gmt) <= 1e-9 and rel(grc, grt) <= 1e-9
    st_t, st_c = eng_t.stats(), eng_c.stats()
    assert st_c.tape_bytes + st_c.state_bytes < (st_t.tape_bytes + st_t.state_bytes) / 4
    eng_t.close()
    eng_c.close()


def test_direct_sum_gradient_matches_its_central_differences(nb, cuda):
    """NBODY_ADJOINT_DIRECT: the same loss with FP64 direct-sum self-gravity.
    Its dynamics are smooth (no tree), so its replay from perturbed inputs
    is the finite-difference reference for its own gradient."""
    n, steps = 1000, 30
    eng_t, x0, v0, mass, pm, pr = setup(nb, cuda, n=n, steps=steps)
    eng = nb.Adjoint(eng_t.params, n, steps, mode="direct")
    eng_t.close()
    _, gx0, gv0, gm, gr = gradients(nb, cuda, eng, x0, v0, mass, pm, pr)
    r0 = cuda.sqrt((x0 * x0).sum(0)).cpu().numpy()
    speed = cuda.sqrt((v0 * v0).sum(0)).cpu().numpy()
    bodies = np.random.default_rng(1).choice(np.nonzero(r0 < 1.5)[0], 9, replace=False)
    for k, b in enumerate(bodies):
        c = k % 3
        g = fd(nb, cuda, eng, mass, x0, v0, pm, pr, "v", c, int(b), 1e-6 * speed[b])
        assert rel(float(gv0[c, b]), g) <= 1e-4, (c, b, float(gv0[c, b]), g)
    fd_m = fd(nb, cuda, eng, mass, x0, v0, pm, pr, "m", dpm=1e-5 * pm)
    assert rel(gm, fd_m) <= 1e-4, (gm, fd_m)
    eng.close()


def test_tree_gradient_against_the_direct_sum_gradient(nb, cuda):
    """The frozen-tree adjoint (theta 0.5) against the FP64 direct-sum
    reference gradient of the same loss: they differ by the walk's force
    approximation, which is small against the star-dominated dynamics."""
    n, steps = 3000, 40
    eng_t, x0, v0, mass, pm, pr = setup(nb, cuda, n=n, steps=steps)
    eng_d = nb.Adjoint(eng_t.params, n, steps, mode="direct")
    _, gxt, gvt, gmt, grt = gradients(nb, cuda, eng_t, x0, v0, mass, pm, pr)
    _, gxd, gvd, gmd, grd = gradients(nb, cuda, eng_d, x0, v0, mass, pm, pr)
    dv = float((gvt - gvd).norm() / gvd.norm())
    dx = float((gxt - gxd).norm() / gxd.norm())
    print(f"tree vs direct-sum gradient: velocity {dv:.3e} position {dx:.3e} (relative "
          f"L2); mass {rel(gmt, gmd):.3e} radius {rel(grt, grd):.3e}")
    assert dv <= 1e-3 and dx <= 1e-3
    assert rel(gmt, gmd) <= 1e-2 and rel(grt, grd) <= 1e-2
    eng_t.close()
    eng_d.close()
