"""Step-by-step parity of the GPU world with the reference step.

Oracles (all built from the reference's own sources, oracle/Makefile):
  - oracle():    contraction off — bit-exact target for scenes whose bodies
                 never reach libm's float transcendentals;
  - oracle_cr(): contraction off, libm sinf/cosf/atan2f evaluated in double
                 and rounded once like the GPU — bit-exact target for every
                 scene;
  - oracle_fast(): the reference's own release flags (FMA contraction) —
                 tolerance target (poses within 1e-5 m / 1e-5 rad per step).

Bit-exact comparisons, per step: every body's pose, velocities and sleep
state; the contact array (order, pairs, touch flags, manifold normals and
points); the step's begin and end contact events, in order; island
partitions; the greedy colouring of coloured islands; the profile counters.
"""
import gc
import os

import numpy as np
import pytest

from melon3d_b200 import api, harness

from . import _util as U

pytestmark = pytest.mark.gpu


def lockstep(ref, kind, steps, seed=1, a=0, b=0, c=0, substeps=4, check_colors=True, giant=None, compare=None,
             workers=0):
    """Step the oracle and the GPU world side by side; after every step that
    `compare(step)` selects (all by default) compare them bit for bit.
    `workers` sets the reference's thread count (its result does not depend
    on it: determinism across worker counts is one of its contracts)."""
    g = U.gpu()
    sr = harness.Scene(ref, kind, seed, a, b, c, workers=workers)
    sg = harness.Scene(g, kind, seed, a, b, c)
    if giant is not None:
        g.m3d_gpu_set_giant_island_contacts(sg.world, giant)
    coloured_steps = 0
    try:
        for step in range(steps):
            sr.run(1, substeps)
            sg.run(1, substeps)
            assert g.m3d_gpu_status(sg.world) == 0, g.m3d_gpu_last_error_string(sg.world)
            if compare is not None and not compare(step):
                continue
            cr, cg = U.contacts(ref, sr.world), U.contacts(g, sg.world)
            d = U.diff_contacts(cr, cg)
            assert d is None, "step %d: %s" % (step, d)
            d = U.diff_events(U.events(ref, sr.world), U.events(g, sg.world))
            assert d is None, "step %d: %s" % (step, d)
            br, bg = U.bodies(ref, sr.world), U.bodies(g, sg.world)
            d = U.diff_bodies(br, bg)
            assert d is None, "step %d: %s (pose error %s)" % (step, d, U.pose_error(br, bg))
            lr, lg = U.island_labels(ref, sr.world), U.island_labels(g, sg.world)
            live = br["inUse"] != 0
            assert np.array_equal(lr[live], lg[live]), "step %d: island partition differs" % step
            pr, pg = ref.m3d_world_profile(sr.world), g.m3d_world_profile(sg.world)
            for f in ("bodyCount", "awakeBodyCount", "contactCount", "touchingContactCount", "islandCount"):
                assert getattr(pr, f) == getattr(pg, f), "step %d: profile %s %d vs %d" % (
                    step, f, getattr(pr, f), getattr(pg, f))
            if check_colors and pr.touchingContactCount >= 300 and pr.islandCount > 0:
                kr, kg = U.contact_colors(ref, sr.world), U.contact_colors(g, sg.world)
                m = kr >= 0
                if m.any():
                    coloured_steps += 1
                    assert np.array_equal(kr[m], kg[m]), "step %d: colouring differs" % step
    finally:
        sr.close()
        sg.close()
    return coloured_steps


def test_pyramid_bit_exact_all_300_steps():
    # the pyramid workload as stated: 210 boxes (one island, > 300 contacts:
    # the coloured path), 300 steps at 60 Hz x 4 substeps, through sleep
    assert lockstep(U.oracle(), harness.PYRAMID, 300) > 0


def test_raft_coloured_path_bit_exact():
    assert lockstep(U.oracle(), harness.RAFT, 90) > 0


def test_pyramid_whole_gpu_coloured_path_bit_exact():
    # every coloured island through the cooperative whole-GPU kernel
    assert lockstep(U.oracle(), harness.PYRAMID, 80, giant=300) > 0


def test_raft_whole_gpu_coloured_path_bit_exact():
    assert lockstep(U.oracle(), harness.RAFT, 90, giant=300) > 0


def test_large_pile_whole_gpu_coloured_path_bit_exact():
    # 16,000 boxes: one island of ~38k touching contacts (above the default
    # giant threshold of 32768), 8 colours and a small overflow bucket
    assert lockstep(U.oracle_cr(), harness.PILE, 5, seed=3, a=20, b=40, c=20) > 0


def test_rain_20k_churn_200_first_60_steps_bit_exact():
    # the streaming rain workload at its stated size: 20,000 bodies, 200
    # destroyed and spawned per step, steps 0-59 compared after every step
    lockstep(U.oracle_cr(), harness.RAIN, 60, seed=2, a=20000, b=200, workers=os.cpu_count() or 1)


def test_rain_20k_churn_200_settled_phase_bit_exact():
    # the same workload pre-rolled to its settled phase (piles on the ground,
    # churn removing the lowest bodies): every 25th step of the first 300
    # compared, then steps 300-359 after every step
    lockstep(U.oracle_cr(), harness.RAIN, 360, seed=2, a=20000, b=200, workers=os.cpu_count() or 1,
             compare=lambda k: k >= 300 or k % 25 == 24)


def test_rain_with_churn_bit_exact():
    lockstep(U.oracle_cr(), harness.RAIN, 60, seed=2, a=1500, b=30)


def test_rain_churn_with_edits_between_steps_bit_exact():
    """After a step that followed destroys, the GPU world downloads what the
    next destroy needs on a second stream.  Edits that reach the device
    before that destroy (velocities, a material, flushed by the pose
    read-back of the churn) must drop it; the destroys then download afresh.
    Compared with the reference after every step: bodies, contacts, events."""
    ref, g = U.oracle_cr(), U.gpu()
    sr = harness.Scene(ref, harness.RAIN, 7, 3000, 60)
    sg = harness.Scene(g, harness.RAIN, 7, 3000, 60)
    try:
        for step in range(60):
            sr.run(1)
            sg.run(1)
            if step >= 20 and step % 5 == 0:
                ir, ig = sr.dynamic_ids(), sg.dynamic_ids()
                assert [(i.index, i.generation) for i in ir] == [(i.index, i.generation) for i in ig]
                for k in range(0, len(ir), 97):
                    v = api.Vec3(0.5, 3.0 + 0.01 * k, -0.25)
                    ref.m3d_body_set_linear_velocity(sr.world, ir[k], v)
                    g.m3d_body_set_linear_velocity(sg.world, ig[k], v)
                ref.m3d_body_set_friction(sr.world, ir[1], 0.9)
                g.m3d_body_set_friction(sg.world, ig[1], 0.9)
                sr.churn()  # destroys after the edits, without a step
                sg.churn()
                d = U.diff_events(U.events(ref, sr.world), U.events(g, sg.world))
                assert d is None, "step %d, churn: %s" % (step, d)
                sr.step_only()
                sg.step_only()
            d = U.diff_contacts(U.contacts(ref, sr.world), U.contacts(g, sg.world))
            assert d is None, "step %d: %s" % (step, d)
            d = U.diff_bodies(U.bodies(ref, sr.world), U.bodies(g, sg.world))
            assert d is None, "step %d: %s" % (step, d)
            d = U.diff_events(U.events(ref, sr.world), U.events(g, sg.world))
            assert d is None, "step %d: %s" % (step, d)
    finally:
        sr.close()
        sg.close()


def test_dense_rain_bit_exact():
    lockstep(U.oracle_cr(), harness.RAIN, 12, seed=5, a=20000, b=200)


def test_large_rain_bit_exact():
    # 150k bodies: per-body scans span 74 tiles and the grid sort ~120, so the
    # look-back walks several 32-tile windows; cell keys straddle the key
    # offset in every field, which the bias-subtracted sort digits cover
    lockstep(U.oracle_cr(), harness.RAIN, 4, seed=9, a=150000, b=500)


def _pile_contacts_equal(ref, g, wr, wg, step):
    cr = U.contacts(ref, wr)
    cg = U.contacts(g, wg)
    d = U.diff_contacts(cr, cg)
    n = len(cr)
    del cr, cg
    gc.collect()
    assert d is None, "step %d: %s" % (step, d)
    return n


def test_pile_250k_first_5_steps_bit_exact():
    """The settled-pile workload at its stated size: 250,000 boxes in a
    50x100x50 lattice (jitter), one giant island through the whole-GPU
    coloured solve; steps 0-4 compared bit for bit (bodies, every contact and
    manifold point, contact events, islands, colours, profile counters)."""
    ref, g = U.oracle_cr(), U.gpu()
    sr = harness.Scene(ref, harness.PILE, 3, 50, 100, 50, workers=os.cpu_count() or 1)
    sg = harness.Scene(g, harness.PILE, 3, 50, 100, 50)
    events_max = 0
    try:
        for step in range(5):
            sr.run(1)
            sg.run(1)
            assert g.m3d_gpu_status(sg.world) == 0, g.m3d_gpu_last_error_string(sg.world)
            br, bg = U.bodies(ref, sr.world), U.bodies(g, sg.world)
            d = U.diff_bodies(br, bg)
            assert d is None, "step %d: %s (pose error %s)" % (step, d, U.pose_error(br, bg))
            live = br["inUse"] != 0
            del bg
            lr, lg = U.island_labels(ref, sr.world), U.island_labels(g, sg.world)
            assert np.array_equal(lr[live], lg[live]), "step %d: island partition differs" % step
            n = _pile_contacts_equal(ref, g, sr.world, sg.world, step)
            er, eg = U.events(ref, sr.world), U.events(g, sg.world)
            d = U.diff_events(er, eg)
            assert d is None, "step %d: %s" % (step, d)
            events_max = max(events_max, len(er[0]), len(er[1]))
            pr, pg = ref.m3d_world_profile(sr.world), g.m3d_world_profile(sg.world)
            for f in ("bodyCount", "awakeBodyCount", "contactCount", "touchingContactCount", "islandCount"):
                assert getattr(pr, f) == getattr(pg, f), "step %d: profile %s" % (step, f)
            kr, kg = U.contact_colors(ref, sr.world), U.contact_colors(g, sg.world)
            m = kr >= 0
            assert np.array_equal(kr[m], kg[m]), "step %d: colouring differs" % step
            print("step %d: %d contacts, %d touching, %d coloured" % (step, n, pr.touchingContactCount, int(m.sum())))
        assert pr.touchingContactCount > 300000
        assert events_max > 1024  # longer than the event head copied with the step's counters
    finally:
        sr.close()
        sg.close()


def test_jointed_raft_every_joint_type_bit_exact():
    """Every joint type (rigid and soft distance, ball, weld, hinge with a
    limit, a motor, or both) inside one coloured island of > 300 contacts,
    plus a hinged chain, a motor-driven wheel and a soft pendulum: 120 steps
    compared bit for bit.  Hinge limits evaluate atan2, so the oracle is the
    one with correctly rounded float transcendentals."""
    assert lockstep(U.oracle_cr(), harness.JOINTED_RAFT, 120, seed=11) > 0


def test_small_pile_bit_exact():
    lockstep(U.oracle_cr(), harness.PILE, 40, seed=3, a=6, b=8, c=6)


def test_pyramid_pose_gate_60_steps():
    """Pose gate (1e-5 m / 1e-5 rad per step over 60 steps) against the
    contraction-off reference, which the GPU matches bit for bit (error 0).
    The reference's own release build (GCC free to contract a*b+c into FMAs)
    is a different float program: it drifts from its own contraction-off
    build by ~1e-3 m within ten pyramid steps.  The GPU's distance to that
    build is measured and must equal the contraction-off build's distance."""
    exact, stock, g = U.oracle(), U.oracle_fast(), U.gpu()
    se = harness.Scene(exact, harness.PYRAMID, 1)
    ss = harness.Scene(stock, harness.PYRAMID, 1)
    sg = harness.Scene(g, harness.PYRAMID, 1)
    worst_stock = (0.0, 0.0)
    try:
        for step in range(60):
            se.run(1)
            ss.run(1)
            sg.run(1)
            be, bs, bg = U.bodies(exact, se.world), U.bodies(stock, ss.world), U.bodies(g, sg.world)
            dx, dq = U.pose_error(be, bg)
            assert dx <= 1e-5 and dq <= 1e-5, "step %d: pose error %.3g m %.3g" % (step, dx, dq)
            assert U.pose_error(bs, bg) == U.pose_error(bs, be)
            e = U.pose_error(bs, bg)
            worst_stock = (max(worst_stock[0], e[0]), max(worst_stock[1], e[1]))
    finally:
        se.close()
        ss.close()
        sg.close()
    print("pyramid, GPU vs reference release build (FMA): max %.3g m, %.3g" % worst_stock)


def _gpu_twins(kind, steps, seed, a=0, b=0, c=0, giant=None):
    """Two GPU worlds built from the same seed and stepped alternately must
    agree bit for bit after every step (run-to-run determinism: no float
    atomics, fixed-order reductions, exact reorderings only)."""
    g = U.gpu()
    s1 = harness.Scene(g, kind, seed, a, b, c)
    s2 = harness.Scene(g, kind, seed, a, b, c)
    if giant is not None:
        g.m3d_gpu_set_giant_island_contacts(s1.world, giant)
        g.m3d_gpu_set_giant_island_contacts(s2.world, giant)
    try:
        for step in range(steps):
            s1.run(1)
            s2.run(1)
            d = U.diff_contacts(U.contacts(g, s1.world), U.contacts(g, s2.world))
            assert d is None, "step %d: %s" % (step, d)
            d = U.diff_bodies(U.bodies(g, s1.world), U.bodies(g, s2.world))
            assert d is None, "step %d: %s" % (step, d)
    finally:
        s1.close()
        s2.close()


def test_runs_are_bit_identical_rain():
    _gpu_twins(harness.RAIN, 40, 7, a=40000, b=400)


def test_runs_are_bit_identical_pile():
    _gpu_twins(harness.PILE, 6, 3, a=20, b=40, c=20)


def test_sleeping_world_fast_path_bit_exact():
    """2,400 boxes in 2-box stacks fall asleep after ~33 steps; once a step
    changes nothing, later steps take the host-only fast path.  Compared with
    the reference after every step (bodies, contacts, profile counters),
    before and after a body is woken by an impulse, which must end the fast
    path until the world is asleep again."""
    from melon3d_b200 import api
    ref, g = U.oracle(), U.gpu()
    sr = harness.Scene(ref, harness.SETTLED_STACKS, 1, 40, 30, 2)
    sg = harness.Scene(g, harness.SETTLED_STACKS, 1, 40, 30, 2)
    try:
        def compare(step):
            d = U.diff_contacts(U.contacts(ref, sr.world), U.contacts(g, sg.world))
            assert d is None, "step %d: %s" % (step, d)
            d = U.diff_bodies(U.bodies(ref, sr.world), U.bodies(g, sg.world))
            assert d is None, "step %d: %s" % (step, d)
            pr, pg = ref.m3d_world_profile(sr.world), g.m3d_world_profile(sg.world)
            for f in ("bodyCount", "awakeBodyCount", "contactCount", "touchingContactCount", "islandCount"):
                assert getattr(pr, f) == getattr(pg, f), "step %d: profile %s" % (step, f)
            assert len(U.contacts(g, sg.world)) == pg.contactCount
        for step in range(100):
            sr.run(1)
            sg.run(1)
            compare(step)
        fast = g.m3d_gpu_fast_path_steps(sg.world)
        assert fast >= 40, fast
        assert g.m3d_world_profile(sg.world).awakeBodyCount == 0
        # wake one box with an impulse on both worlds: normal steps resume
        ids_r, ids_g = sr.dynamic_ids(), sg.dynamic_ids()
        for lib, w, ids in ((ref, sr.world, ids_r), (g, sg.world, ids_g)):
            lib.m3d_body_apply_impulse(w, ids[7], api.Vec3(0.0, 4000.0, 0.0), lib.m3d_body_position(w, ids[7]))
        for step in range(100, 130):
            sr.run(1)
            sg.run(1)
            compare(step)
        assert g.m3d_gpu_fast_path_steps(sg.world) == fast  # the woken world stepped normally
    finally:
        sr.close()
        sg.close()
