"""Mixed-resolution batches (hzlb_mixed_*): every schedule (serial, concurrent with capped
grids, the autotuner's choice) advances each resolution exactly as stepping it alone does —
bit for bit, since each work item's arithmetic does not depend on the grid size."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _configs(hzlb):
    return [hzlb.Config(n=32, members=5, precision=8, nu=1e-3, noise_sigma=0.05, seed=3),
            hzlb.Config(n=64, members=3, precision=4, nu=5e-4, noise_sigma=0.05, seed=4,
                        forcing_kmax=0),
            hzlb.Config(n=16, members=9, precision=4, nu=2e-3, seed=5)]


def _init(hzlb, ens, cfg, k):
    ens.set_state(np.array([hzlb.grf_spectrum(cfg.n, 11 + k, m) for m in range(cfg.members)]))
    if cfg.forcing_kmax >= 0:
        ens.set_forcing(hzlb.kolmogorov_forcing(cfg.n)[None])


def _alone(hzlb, cfgs, dts, steps):
    out = []
    for k, (c, dt) in enumerate(zip(cfgs, dts)):
        e = hzlb.Ensemble(c)
        _init(hzlb, e, c, k)
        e.step(dt, steps[k])
        out.append(e.get_state_compact())
        e.close()
    return out


@pytest.mark.parametrize("serial,caps", [(True, None), (False, None), (False, [3, 2, 1])])
def test_schedules_match_separate_stepping(hzlb, serial, caps):
    cfgs = _configs(hzlb)
    dts = [1e-3, 5e-4, 2e-3]
    m = hzlb.Mixed(cfgs)
    for k, (g, c) in enumerate(zip(m.groups, cfgs)):
        _init(hzlb, g, c, k)
    m.set_schedule(serial, caps, caps)
    m.step(dts, 11)
    got = [g.get_state_compact() for g in m.groups]
    for k, ref in enumerate(_alone(hzlb, cfgs, dts, [11] * 3)):
        np.testing.assert_array_equal(got[k], ref)
    m.close()


def test_autotuner_keeps_results_exact(hzlb):
    cfgs = _configs(hzlb)
    dts = [1e-3, 5e-4, 2e-3]
    m = hzlb.Mixed(cfgs)
    for k, (g, c) in enumerate(zip(m.groups, cfgs)):
        _init(hzlb, g, c, k)
    before = [g.get_state_compact() for g in m.groups]
    ms = m.tune(dts, repeats=1)
    assert ms > 0
    sched = m.schedule()
    assert len(sched["column_caps"]) == 3 and all(c > 0 for c in sched["column_caps"])
    # tuning leaves states and clocks as they were
    for g, b in zip(m.groups, before):
        np.testing.assert_array_equal(g.get_state_compact(), b)
        assert g.time()[1] == 0
    m.step(dts, 5)
    got = [g.get_state_compact() for g in m.groups]
    for k, ref in enumerate(_alone(hzlb, cfgs, dts, [5] * 3)):
        np.testing.assert_array_equal(got[k], ref)
    m.close()
