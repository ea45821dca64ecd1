"""Host side of the sensitivity surrogate (autoquantizer_b200.surrogate):
scene sampling, field groups, features, per-group targets and the scheme
derived from predicted sensitivities, on CPU."""
import numpy as np
import pytest

from autoquantizer_b200 import solvers
from autoquantizer_b200 import surrogate as S


@pytest.mark.parametrize("dim,fluid", [(2, False), (2, True), (3, False), (3, True)])
def test_groups_partition_the_record(dim, fluid):
    ns = 2 * dim + dim * dim + (1 if fluid else dim * dim)
    g = S.groups_of(dim, fluid)
    assert len(g) == S.N_OUT == 12
    flat = sum(g, [])
    assert sorted(flat) == list(range(ns))
    assert [len(x) for x in g[:3]] == [1] * dim + [0] * (3 - dim)  # x per component
    assert [len(x) for x in g[6:9]] == [dim] * dim + [0] * (3 - dim)  # C rows
    assert [len(x) for x in g[9:12]] == ([1, 0, 0] if fluid else [dim] * dim + [0] * (3 - dim))


def test_random_scenes_are_valid():
    rng = np.random.default_rng(3)
    for _ in range(20):
        cfg, vals = S.random_scene(rng, n_min=1000, n_max=5000, horizon=16)
        d = cfg.dim
        assert 1000 <= vals.shape[0] < 5000 and cfg.n_particles == vals.shape[0]
        assert vals.shape[1] == 2 * d + d * d + (1 if cfg.use_fluid else d * d)
        assert np.all((vals[:, :d] > 0.1) & (vals[:, :d] < 0.9))
        assert np.all(vals[:, d:2 * d] == vals[0, d:2 * d])  # one push for the whole body
        if cfg.use_fluid:
            assert np.all(vals[:, 2 * d + d * d] == 1.0)
        else:
            assert np.all(vals[:, 2 * d + d * d:] == np.eye(d).ravel())
        assert cfg.dt <= 2e-4 and cfg.n_timesteps == 17
        assert 1e3 <= cfg.E <= 1e5 and 0.2 <= cfg.nu <= 0.4


def test_features_from_known_statistics():
    cfg, vals = S.random_scene(np.random.default_rng(0), n_min=1000, n_max=1001)
    n, ns = vals.shape
    stats = np.zeros((ns, 5))
    for s in range(ns):  # sum |v|, sum v, sum v^2, max |v|, sum |v - v0|
        stats[s] = [n * (s + 1.0), -n * (s + 1.0), n * (s + 1.0) ** 2 * 2, 10.0 * (s + 1), n * 0.5]
    f = S.features(cfg, stats, n)
    assert f.shape == (S.N_IN,)
    # group 0 is x0 (slot 0): mean |.| 1, std sqrt(2 - 1) = 1, max 10, mean change 0.5
    assert f[0:4] == pytest.approx([0.0, 0.0, 1.0, np.log10(0.5)])
    absent = [gi for gi, sl in enumerate(S.groups_of(cfg.dim, cfg.use_fluid)) if not sl]
    for gi in absent:
        assert np.all(f[4 * gi:4 * gi + 4] == 0)
    assert f[48] == cfg.dim / 3.0 and f[49] == float(cfg.use_fluid) and f[63] == 1.0


def test_targets_and_scheme():
    cfg, vals = S.random_scene(np.random.default_rng(1), n_min=1000, n_max=1001)
    ns = vals.shape[1]
    sens = np.arange(1, ns + 1, dtype=np.float64)
    y, m = S.group_sensitivities(cfg, sens)
    groups = S.groups_of(cfg.dim, cfg.use_fluid)
    for gi, sl in enumerate(groups):
        if sl:
            assert m[gi] == 1 and y[gi] == pytest.approx(np.log10(sens[sl].sum()))
        else:
            assert m[gi] == 0
    stats = np.zeros((ns, 5))
    stats[:, 3] = np.linspace(0.5, 3.0, ns)
    r = S.group_ranges(cfg, stats)
    assert np.all(r[:3] == 1.0)
    for gi in range(3, 12):
        if groups[gi]:
            assert r[gi] == pytest.approx(2 * stats[groups[gi], 3].max())
    idx = np.where(m > 0)[0]
    want, _ = solvers.LagrangianEB(10.0 ** y[idx] * r[idx] ** 2, ref=123.0, tol_rel=1e-3)
    raw = S.scheme_bits(y, m, r, loss=123.0, tol_rel=1e-3, storable=False)
    assert raw[idx].tolist() == (want + 1).tolist() and np.all(raw[m == 0] == 0)
    bits = S.scheme_bits(y, m, r, loss=123.0, tol_rel=1e-3)
    assert bits[idx].tolist() == np.maximum(want + 1, S.MIN_WIDTH).tolist() and np.all(bits[m == 0] == 0)
    # a group whose error hardly matters gets a solver width below the
    # layout's minimum; the storable scheme clamps it, the solver's keeps it
    y2 = y.copy()
    y2[idx[0]] -= 12.0
    raw2 = S.scheme_bits(y2, m, r, loss=123.0, tol_rel=1e-3, storable=False)
    assert raw2[idx[0]] < S.MIN_WIDTH
    assert S.scheme_bits(y2, m, r, loss=123.0, tol_rel=1e-3)[idx[0]] == S.MIN_WIDTH


def test_adjoint_fallback_trades_agreement_for_speed():
    """evaluate_fallback: scenes whose ensemble is unsure take the adjoint's
    widths.  With no disagreement allowed every scene falls back (full
    agreement, speed-up t_adj / (t_sur + t_adj)); with any allowed, none
    does (the ensemble's own agreement); in between, only the uncertain
    scenes fall back, under both rules (members' spread, members' width
    span)."""
    rng = np.random.default_rng(0)
    n = 40
    Y = rng.uniform(-2, 2, (n, S.N_OUT))  # widths of about 10 bits: none clamped to the minimum
    M = np.ones((n, S.N_OUT))
    M[:, [2, 5, 8, 11]] = 0  # 2D scenes: third entries empty
    meta = [{"ranges": [1.0] * S.N_OUT, "loss": 1.0} for _ in range(n)]
    members = np.stack([Y.copy() for _ in range(4)])
    bad = np.arange(n) % 4 == 0  # a quarter of the scenes: wrong by 3 decades, and the members disagree
    members[:, bad] += 3.0
    members[0, bad, 4] -= 0.8
    members[1, bad, 4] += 0.8
    rows = S.evaluate_fallback(members, Y, M, meta, t_sur=1.0, t_adj=19.0, spreads=(-1.0, 0.2, 10.0),
                               spans=(-1, 1, 99))
    sp = [r for r in rows if r["rule"] == "spread"]
    sn = [r for r in rows if r["rule"] == "span"]
    assert [r["threshold"] for r in sp] == [-1.0, 0.2, 10.0] and [r["threshold"] for r in sn] == [-1, 1, 99]
    for r0, r1, r2 in (sp, sn):
        assert r0["fallback_share"] == 1.0 and r0["scenes_all_within_1_bit"] == 1.0
        assert r0["speedup_vs_adjoint"] == pytest.approx(19.0 / 20.0)
        assert r1["fallback_share"] == pytest.approx(0.25) and r1["scenes_all_within_1_bit"] == 1.0
        assert r1["speedup_vs_adjoint"] == pytest.approx(19.0 / (1.0 + 0.25 * 19.0))
        assert r2["fallback_share"] == 0.0 and r2["scenes_all_within_1_bit"] == pytest.approx(0.75)
