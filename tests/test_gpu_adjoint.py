"""The discrete adjoint (mbm_adjoint_run) against central finite differences of the
frozen-dt forward map: gradients of J = sum (qx^2 + qy^2) of the final state with
respect to the initial temperature field and to Kn, in seeded random directions;
the finite differences come from mbm_replay and, on a small case, from the C
oracle's own frozen-dt steps; and the torch.autograd.Function over it.

Where the map is smooth (limiters none and average; the HLL wave speeds are smooth
in subsonic flow) the check holds to 1e-6 at eps = 1e-6.  Minmod, superbee and
harmonic have kinks (sign changes of the one-sided differences, |d1| = |d2|); the
adjoint takes the forward branch there (a fixed subgradient), and a finite
difference of step eps crosses kinks in a fraction of cells that grows with eps,
so those limiters are checked at eps = 1e-8 with a bound that covers the crossings.
"""
import numpy as np
import pytest

import helpers as H
from multiblockmomentsfv_b200 import adjoint as adj
from multiblockmomentsfv_b200 import blockfile as bf
from multiblockmomentsfv_b200 import output
from multiblockmomentsfv_b200 import scenario as sc
from multiblockmomentsfv_b200 import solver as sv

pytestmark = pytest.mark.gpu


def _theta0(d, rng):
    return [1.0 + 0.2 * np.sin(np.linspace(0, 3, b.nx)[None, :] + np.linspace(0, 2, b.ny)[:, None])
            * rng.uniform(0.5, 1.0) for b in d.blocks]


def _fd_check(n, nsteps, every, ndirs, seed, limiter=bf.LIM_AVERAGE, eps=1e-6, Kn=0.01, mode="exact",
              functional="heat_flux", with_kn=False):
    d = H.quadrant_deck(n, Kn=Kn, limiter=limiter)
    base = adj.smooth_base(d, seed)
    rng = np.random.default_rng(seed)
    th0 = _theta0(d, rng)
    with adj.Sensitivity(d, base, mode=mode, functional=functional) as S:
        layers = adj.state_from_theta(d, base, th0)
        S.load(layers)
        J, g, gK, dts, ms = S.run(nsteps, every)
        gth = adj.theta_gradient(d, layers, g)
        worst = 0.0
        for _ in range(ndirs):
            v = [rng.standard_normal(t.shape) for t in th0]
            S.load(adj.state_from_theta(d, base, [t + eps * w for t, w in zip(th0, v)]))
            Jp = S.replay(dts)
            S.load(adj.state_from_theta(d, base, [t - eps * w for t, w in zip(th0, v)]))
            Jm = S.replay(dts)
            fd = (Jp - Jm) / (2 * eps)
            ad = sum(float(np.sum(a * w)) for a, w in zip(gth, v))
            worst = max(worst, abs(fd - ad) / max(abs(fd), 1e-300))
        S.load(layers, Kn=Kn * (1 + 1e-6))
        Jp = S.replay(dts)
        S.load(layers, Kn=Kn * (1 - 1e-6))
        Jm = S.replay(dts)
        fdK = (Jp - Jm) / (2 * Kn * 1e-6)
        S.load(layers, Kn=Kn)
        assert abs(S.replay(dts) - J) <= 1e-12 * abs(J)      # replay reproduces the forward run
    if with_kn:
        return worst, abs(fdK - gK) / abs(fdK), ms, J, fdK, gK
    return worst, abs(fdK - gK) / abs(fdK), ms, J


@pytest.mark.parametrize("functional", ["temperature", "deviatoric"])
def test_adjoint_other_functionals(functional):
    """The other functionals of mbm_set_functional (the sum of theta, and of the
    deviatoric temperature tensor's squares) against central differences of the same
    functional, smooth limiter."""
    worst, errK, ms, J, fdK, gK = _fd_check(n=24, nsteps=12, every=5, ndirs=6, seed=5,
                                            functional=functional, with_kn=True)
    assert J > 0
    assert worst < 1e-6, worst
    # dJ/dKn: relative agreement, or absolute where the functional barely depends on Kn
    assert abs(fdK - gK) <= max(1e-6 * abs(fdK), 1e-9 * abs(J)), (fdK, gK)


@pytest.mark.parametrize("limiter", [bf.LIM_NONE, bf.LIM_AVERAGE])
def test_adjoint_smooth_limiters(limiter):
    worst, errK, ms, J = _fd_check(n=24, nsteps=12, every=5, ndirs=6, seed=3, limiter=limiter)
    assert J > 0
    assert worst < 1e-6, worst
    assert errK < 1e-6, errK


def test_adjoint_with_the_fast_forward():
    """The same gradient checked against differences of the fast-arithmetic forward
    map (the adjoint differentiates the mathematics both modes compute)."""
    worst, errK, ms, J = _fd_check(n=24, nsteps=12, every=5, ndirs=6, seed=3, mode="fast")
    assert worst < 1e-6, worst
    assert errK < 1e-6, errK


@pytest.mark.parametrize("limiter", [bf.LIM_MINMOD, bf.LIM_SUPERBEE, bf.LIM_HARMONIC])
def test_adjoint_kinked_limiters(limiter):
    worst, errK, ms, J = _fd_check(n=24, nsteps=12, every=5, ndirs=6, seed=3, limiter=limiter, eps=1e-8)
    assert worst < 1e-3, worst
    assert errK < 1e-6, errK


def test_adjoint_benchmark_case():
    """4 blocks x 256^2, 200 steps, checkpoints every 20, 16 seeded directions,
    eps = 1e-6; the adjoint:forward device-time ratio is reported."""
    worst, errK, ms, J = _fd_check(n=256, nsteps=200, every=20, ndirs=16, seed=11)
    print(f"adjoint check: worst rel err {worst:.2e}, Kn rel err {errK:.2e}, "
          f"forward {ms[0]:.1f} ms, adjoint {ms[1]:.1f} ms, ratio {ms[1] / ms[0]:.2f}")
    assert worst < 1e-6, worst
    assert errK < 1e-6, errK


def test_adjoint_benchmark_case_harmonic():
    """The case the bench's adjoint leg times: 4 blocks x 256^2, 200 steps, checkpoints
    every 20, harmonic limiter, fast forward; 16 seeded directions at eps = 1e-6 and
    1e-8.  The harmonic limiter's weights |d| + 1e-10 have a kink where a one-sided
    difference d changes sign, and there the slope's derivative jumps by O(1); a
    central difference of step eps crosses such kinks (about 7e-4 of the one-sided
    differences per step change sign between the +eps and -eps runs of this case), so
    its error is that of the crossings, and it falls with eps -- a wrong adjoint
    would leave an error that does not.  Measured: median relative error 1.2e-3 at
    eps = 1e-6 (worst 1.4e-2), 6.1e-5 at 1e-8 (worst 4.6e-4)."""
    n, nsteps, every, seed = 256, 200, 20, 11
    d = H.quadrant_deck(n, Kn=0.01, limiter=bf.LIM_HARMONIC)
    base = adj.smooth_base(d, seed)
    rng = np.random.default_rng(seed)
    th0 = _theta0(d, rng)
    with adj.Sensitivity(d, base, mode="fast") as S:
        layers = adj.state_from_theta(d, base, th0)
        S.load(layers)
        J, g, gK, dts, ms = S.run(nsteps, every)
        gth = adj.theta_gradient(d, layers, g)
        dirs = [[rng.standard_normal(t.shape) for t in th0] for _ in range(16)]
        med, worst = {}, {}
        for eps in (1e-6, 1e-8):
            errs = []
            for v in dirs:
                S.load(adj.state_from_theta(d, base, [t + eps * w for t, w in zip(th0, v)]))
                Jp = S.replay(dts)
                S.load(adj.state_from_theta(d, base, [t - eps * w for t, w in zip(th0, v)]))
                Jm = S.replay(dts)
                fd = (Jp - Jm) / (2 * eps)
                ad = sum(float(np.sum(a * w)) for a, w in zip(gth, v))
                errs.append(abs(fd - ad) / abs(fd))
            med[eps], worst[eps] = float(np.median(errs)), float(np.max(errs))
        # kink crossings of the first direction: one-sided differences of the primitives
        # whose sign differs between the +eps and -eps runs, over every step
        eps, v = 1e-6, dirs[0]
        signs = []
        for sgn in (1.0, -1.0):
            S.load(adj.state_from_theta(d, base, [t + sgn * eps * w for t, w in zip(th0, v)]))
            run = []
            for k in range(len(dts) + 1):
                if k:
                    S.replay(dts[k - 1:k])
                for b in range(len(d.blocks)):
                    P = output.primitive(S.s.download(sv.L_DATA, b)[bf.NG - 1:-bf.NG + 1, bf.NG - 1:-bf.NG + 1])
                    run += [np.signbit(np.diff(P, axis=1)), np.signbit(np.diff(P, axis=0))]
            signs.append(run)
        flips = sum(int(np.count_nonzero(x != y)) for x, y in zip(*signs))
        total = sum(x.size for x in signs[0])
    print(f"harmonic adjoint check: eps 1e-6 median {med[1e-6]:.1e} worst {worst[1e-6]:.1e}; eps 1e-8 median "
          f"{med[1e-8]:.1e} worst {worst[1e-8]:.1e}; kink crossings {flips / total:.1e} of one-sided differences; "
          f"forward {ms[0]:.1f} ms, adjoint {ms[1]:.1f} ms")
    assert flips > 0
    assert med[1e-6] <= 5e-3 and worst[1e-6] <= 5e-2, (med, worst)
    assert med[1e-8] <= 3e-4 and worst[1e-8] <= 2e-3, (med, worst)
    assert med[1e-6] >= 5 * med[1e-8], med         # the error falls with eps


def _oracle_replay(O, d, layers, dts):
    """J after the frozen-dt steps of the C oracle (TimeUpdate, then NEW -> DATA)."""
    o = O.Oracle(d, sc.Scenario.named("riemann2d"))
    try:
        for b, U in enumerate(layers):
            o.set_layer(O.DATA, b, U)
        o.set_boundary(O.DATA, 0.0)
        t = 0.0
        for dt in dts:
            o.time_update(dt, t)
            for b in range(len(d.blocks)):
                o.set_layer(O.DATA, b, o.get_layer(O.NEW, b))
            t += dt
        final = o.layers(O.DATA)
    finally:
        o.close()
    J = 0.0
    for U in final:
        P = output.primitive(U[bf.NG:-bf.NG, bf.NG:-bf.NG])
        J += float(np.sum(P[..., 7] ** 2 + P[..., 8] ** 2))
    return J, final


def test_adjoint_against_oracle_differences(oracle_mod):
    """Directional derivatives from perturbed runs of the C oracle: its frozen-dt
    states equal the device replay bit for bit, and its central differences match
    the adjoint."""
    O = oracle_mod
    d = H.quadrant_deck(16, Kn=0.01, limiter=bf.LIM_AVERAGE)
    base = adj.smooth_base(d, 7)
    rng = np.random.default_rng(7)
    th0 = _theta0(d, rng)
    eps = 1e-6
    with adj.Sensitivity(d, base) as S:
        layers = adj.state_from_theta(d, base, th0)
        S.load(layers)
        J, g, gK, dts, ms = S.run(8, 3)
        gth = adj.theta_gradient(d, layers, g)
        S.load(layers)
        S.replay(dts)
        dev = [S.s.download(sv.L_DATA, b) for b in range(len(d.blocks))]
    Jo, final = _oracle_replay(O, d, layers, dts)
    for b in range(len(d.blocks)):
        H.assert_bitwise(dev[b][bf.NG:-bf.NG, bf.NG:-bf.NG], final[b][bf.NG:-bf.NG, bf.NG:-bf.NG], f"block {b + 1}")
    assert abs(Jo - J) <= 1e-13 * abs(J)
    for _ in range(4):
        v = [rng.standard_normal(t.shape) for t in th0]
        Jp, _ = _oracle_replay(O, d, adj.state_from_theta(d, base, [t + eps * w for t, w in zip(th0, v)]), dts)
        Jm, _ = _oracle_replay(O, d, adj.state_from_theta(d, base, [t - eps * w for t, w in zip(th0, v)]), dts)
        fd = (Jp - Jm) / (2 * eps)
        ad = sum(float(np.sum(a * w)) for a, w in zip(gth, v))
        assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)


def _reference_replay(O, d, layers, dts):
    """J after frozen-dt steps of the reference itself (its TimeUpdate from
    oracle/_ref/libmbmref.so, then NEW -> DATA as its Steps copies, src/Main.c:236-240)."""
    R = O.Reference(d)
    for b, U in enumerate(layers):
        R.set_layer(O.DATA, b, U)
    R.set_boundary(O.DATA, 0.0)
    t = 0.0
    for dt in dts:
        R.time_update(dt, t)
        for b in range(len(d.blocks)):
            R.set_layer(O.DATA, b, R.get_layer(O.NEW, b))
        t += dt
    J = 0.0
    final = [R.get_layer(O.DATA, b) for b in range(len(d.blocks))]
    for U in final:
        P = output.primitive(U[bf.NG:-bf.NG, bf.NG:-bf.NG])
        J += float(np.sum(P[..., 7] ** 2 + P[..., 8] ** 2))
    return J, final


def test_adjoint_against_reference_differences(oracle_mod):
    """Directional derivatives from perturbed runs of the reference's own TimeUpdate
    (the reference sources compiled into oracle/_ref), with the adjoint's frozen dt
    sequence: the reference's unperturbed states equal the device replay bit for bit,
    and its central differences (eps = 1e-6) match the adjoint to 1e-6."""
    O = oracle_mod
    if O.ref_lib() is None:
        pytest.skip("reference build absent (make -C oracle ref)")
    d = H.quadrant_deck(16, Kn=0.01, limiter=bf.LIM_AVERAGE)
    base = adj.smooth_base(d, 5)
    rng = np.random.default_rng(5)
    th0 = _theta0(d, rng)
    eps = 1e-6
    with adj.Sensitivity(d, base) as S:
        layers = adj.state_from_theta(d, base, th0)
        S.load(layers)
        J, g, gK, dts, ms = S.run(8, 3)
        gth = adj.theta_gradient(d, layers, g)
        S.load(layers)
        S.replay(dts)
        dev = [S.s.download(sv.L_DATA, b) for b in range(len(d.blocks))]
    Jr, final = _reference_replay(O, d, layers, dts)
    for b in range(len(d.blocks)):
        H.assert_bitwise(dev[b][bf.NG:-bf.NG, bf.NG:-bf.NG], final[b][bf.NG:-bf.NG, bf.NG:-bf.NG], f"block {b + 1}")
    assert abs(Jr - J) <= 1e-13 * abs(J)
    for _ in range(4):
        v = [rng.standard_normal(t.shape) for t in th0]
        Jp, _ = _reference_replay(O, d, adj.state_from_theta(d, base, [t + eps * w for t, w in zip(th0, v)]), dts)
        Jm, _ = _reference_replay(O, d, adj.state_from_theta(d, base, [t - eps * w for t, w in zip(th0, v)]), dts)
        fd = (Jp - Jm) / (2 * eps)
        ad = sum(float(np.sum(a * w)) for a, w in zip(gth, v))
        assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)


def test_autograd_function():
    torch = pytest.importorskip("torch")
    d = H.quadrant_deck(16, Kn=0.01)
    base = adj.smooth_base(d, 5)
    with adj.Sensitivity(d, base) as S:
        f = adj.make_autograd(S, nsteps=8, every=4)
        th = torch.ones((4, 16, 16), dtype=torch.float64, requires_grad=True)
        kn = torch.tensor(0.01, dtype=torch.float64, requires_grad=True)
        J = f(th, kn)
        J.backward()
        assert th.grad.shape == th.shape and torch.isfinite(th.grad).all()
        assert kn.grad is not None and torch.isfinite(kn.grad)
        # the gradient is the one mbm_adjoint_run returns for the same state
        layers = adj.state_from_theta(d, base, list(th.detach().numpy()))
        S.load(layers, 0.01)
        _, g, gK, _, _ = S.run(8, 4)
        ref = np.stack(adj.theta_gradient(d, layers, g))
        assert np.allclose(th.grad.numpy(), ref, rtol=1e-12, atol=0)
        assert abs(float(kn.grad) - gK) <= 1e-12 * abs(gK)


@pytest.mark.parametrize("limiter", [bf.LIM_NONE, bf.LIM_MINMOD, bf.LIM_SUPERBEE, bf.LIM_HARMONIC])
def test_row_march_equals_three_pass(limiter):
    """The row-marching adjoint pass (MBM_ADJ_MARCH=1) and the three-pass one (the
    default), two independent implementations of the stage adjoint, give the same
    gradient up to rounding (different association of the same sums)."""
    import os
    d = H.quadrant_deck(40, Kn=0.01, limiter=limiter)
    base = adj.smooth_base(d, 13)
    th0 = _theta0(d, np.random.default_rng(13))
    out = {}
    for march in ("1", "0"):
        os.environ["MBM_ADJ_MARCH"] = march
        try:
            with adj.Sensitivity(d, base) as S:
                layers = adj.state_from_theta(d, base, th0)
                S.load(layers)
                J, g, gK, dts, ms = S.run(16, 5)
                out[march] = (J, np.concatenate([x.ravel() for x in g]), gK)
        finally:
            del os.environ["MBM_ADJ_MARCH"]
    (J1, g1, k1), (J0, g0, k0) = out["1"], out["0"]
    assert J1 == J0
    scale = np.abs(g0).max()
    assert np.abs(g1 - g0).max() <= 1e-11 * scale, np.abs(g1 - g0).max() / scale
    assert abs(k1 - k0) <= 1e-11 * abs(k0)


@pytest.mark.parametrize("nsteps,every", [(16, 5), (12, 4), (3, 5)])
def test_tail_segment_kept_by_forward(nsteps, every):
    """The forward run keeps the last checkpoint segment's states for the reverse sweep
    (the default) or the sweep recomputes it (MBM_ADJ_TAIL=0): the same gradient, for a
    partial last segment, a full one, and a run shorter than one segment."""
    import os
    d = H.quadrant_deck(32, Kn=0.01, limiter=bf.LIM_HARMONIC)
    base = adj.smooth_base(d, 23)
    th0 = _theta0(d, np.random.default_rng(23))
    out = {}
    for tail in ("1", "0"):
        os.environ["MBM_ADJ_TAIL"] = tail
        try:
            with adj.Sensitivity(d, base, mode="fast") as S:
                S.load(adj.state_from_theta(d, base, th0))
                J, g, gK, dts, ms = S.run(nsteps, every)
                out[tail] = (J, np.concatenate([x.ravel() for x in g]), gK, dts)
        finally:
            del os.environ["MBM_ADJ_TAIL"]
    (J1, g1, k1, d1), (J0, g0, k0, d0) = out["1"], out["0"]
    assert J1 == J0
    H.assert_bitwise(d1, d0, "dt")
    scale = np.abs(g0).max()
    assert np.abs(g1 - g0).max() <= 1e-12 * scale, np.abs(g1 - g0).max() / scale
    assert abs(k1 - k0) <= 1e-12 * abs(k0)


@pytest.mark.parametrize("limiter", [bf.LIM_AVERAGE, bf.LIM_HARMONIC])
@pytest.mark.parametrize("mode", ["exact", "fast"])
def test_split_cell_pass_equals_whole(limiter, mode):
    """The cell pass in two halves with the Data0 term in the primitives pass (the
    default) and the whole cell pass (MBM_ADJ_SPLIT=0): the same gradient."""
    import os
    d = H.quadrant_deck(40, Kn=0.01, limiter=limiter)
    base = adj.smooth_base(d, 29)
    th0 = _theta0(d, np.random.default_rng(29))
    out = {}
    for split in ("1", "0"):
        os.environ["MBM_ADJ_SPLIT"] = split
        try:
            with adj.Sensitivity(d, base, mode=mode) as S:
                S.load(adj.state_from_theta(d, base, th0))
                J, g, gK, dts, ms = S.run(16, 5)
                out[split] = (J, np.concatenate([x.ravel() for x in g]), gK)
        finally:
            del os.environ["MBM_ADJ_SPLIT"]
    (J1, g1, k1), (J0, g0, k0) = out["1"], out["0"]
    assert J1 == J0
    scale = np.abs(g0).max()
    assert np.abs(g1 - g0).max() <= 1e-12 * scale, np.abs(g1 - g0).max() / scale
    assert abs(k1 - k0) <= 1e-12 * abs(k0)


def test_replay_before_the_first_adjoint_run():
    """A context whose first call is mbm_replay (which makes only the adjoint layer it
    needs) runs the adjoint afterwards with the same result as a context that runs it
    first: every work layer the adjoint needs is made on its first call.  (Gradients
    agree to rounding: the ghost-fill adjoint adds several ghosts into one source
    cell with atomic adds, in no fixed order.)"""
    d = H.quadrant_deck(32, Kn=0.01, limiter=bf.LIM_HARMONIC)
    base = adj.smooth_base(d, 21)
    th0 = _theta0(d, np.random.default_rng(21))
    layers = adj.state_from_theta(d, base, th0)
    with adj.Sensitivity(d, base) as S:
        S.load(layers)
        J, g, gK, dts, _ = S.run(12, 4)
    with adj.Sensitivity(d, base) as S:
        S.load(layers)
        assert abs(S.replay(dts) - J) <= 1e-12 * abs(J)
        S.load(layers)
        J2, g2, gK2, dts2, _ = S.run(12, 4)
    assert J2 == J and np.array_equal(dts2, dts)
    scale = max(np.abs(b).max() for b in g)
    assert scale > 0
    for a, b in zip(g2, g):
        assert np.abs(a - b).max() <= 1e-12 * scale
    assert abs(gK2 - gK) <= 1e-12 * abs(gK)
