"""Ensemble batching: members stepped together in one handle (one stage-kernel launch per RK stage for all
members) give each member the same result as running it alone; the autotuner measures both tile sizes
and keeps the faster.

Tolerance: FP64 members agree with their individual runs to 1e-12 of each variable's scale (the
per-element arithmetic and accumulation order do not depend on the tiling); wet flags identical."""
import numpy as np
import pytest

from dgswemv2_b200 import Problem, _lib, configs, ensemble

pytestmark = pytest.mark.gpu


def rel_err(a, b):
    out = 0.0
    for v in range(3):
        scale = max(np.max(np.abs(b[:, v, :])), 1e-300)
        out = max(out, np.max(np.abs(a[:, v, :] - b[:, v, :])) / scale)
    return out


def test_members_match_individual_runs_fp64():
    meshes, cfgs = configs.config5(n_members=5, seed=3, nmin=12, nmax=40, precision="fp64")
    E = ensemble(cfgs[0], meshes, [c.fn_params for c in cfgs], tile=0)
    assert E.ne == sum(m.n_elems for m in meshes)
    E.step_serial(40)
    q, w = E.get_state(), E.get_wet()
    for k, (m, c) in enumerate(zip(meshes, cfgs)):
        first, n = E.member_range(k)
        assert n == m.n_elems
        P = Problem(c, m)
        P.step_serial(40)
        assert rel_err(q[first:first + n], P.get_state()) <= 1e-12, k
        assert np.array_equal(w[first:first + n], P.get_wet()), k
    assert E.member_range(4)[0] + E.member_range(4)[1] == E.ne


def test_autotuner_times_every_candidate_and_keeps_the_fastest():
    """Tile size x register budget x tile order: eight candidates timed, the fastest kept."""
    meshes, cfgs = configs.config5(n_members=6, seed=1, nmin=32, nmax=64, precision="fp32")
    E = ensemble(cfgs[0], meshes, [c.fn_params for c in cfgs])  # tile = DGSW_TILE_AUTOTUNE
    rec = E.tuning()
    assert len(rec) == 8 and all(r[3] > 0 for r in rec)
    assert {(t, o, r) for t, o, r, _ in rec} == {(t, o, r) for t in (128, 256) for o in (0, 1) for r in (0, 1)}
    best = min(rec, key=lambda r: r[3])
    assert (E.info.tile, E.info.occupancy, E.info.tile_order) == best[:3]
    # the tuned handle starts from t = 0 like an untuned one
    assert E.time()[1] == 0
    F = ensemble(cfgs[0], meshes, [c.fn_params for c in cfgs], tile=E.info.tile, occupancy=E.info.occupancy,
                 tile_order=E.info.tile_order)
    E.step_serial(20)
    F.step_serial(20)
    assert np.array_equal(E.get_state(), F.get_state())
    # a second create of the same shape reuses the cached decision without timing
    G = ensemble(cfgs[0], meshes, [c.fn_params for c in cfgs])
    assert G.tuning() == [] and G.info.tile == E.info.tile


def test_fp32_ensemble_conserves_mass_and_stays_finite():
    meshes, cfgs = configs.config5(n_members=12, seed=7, nmin=40, nmax=90, precision="fp32")
    E = ensemble(cfgs[0], meshes, [c.fn_params for c in cfgs], tile=0)
    m0 = E.mass()
    E.step_serial(200)
    assert np.isfinite(E.get_state()).all()
    assert abs(E.mass() / m0 - 1) <= 1e-6
    assert E.get_wet().sum() > 0
