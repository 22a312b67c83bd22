"""Mixed-resolution batches (hzlb_mixed_*): every schedule (serial, concurrent with capped
grids, one fused persistent kernel per stage over the mixed work list, fused with a 512^2
branch, the autotuner's choice) advances each resolution exactly as stepping it alone does --
bit for bit, since each work item's arithmetic does not depend on the grid or on the other
resolutions in the launch."""
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


def _fused_configs(hzlb, with512=True):
    out = [hzlb.Config(n=64, members=37, precision=4, nu=1e-3, noise_sigma=0.05, seed=4,
                       forcing_kmax=0),
           hzlb.Config(n=128, members=11, precision=4, nu=5e-4, noise_sigma=0.05, seed=5,
                       forcing_kmax=0),
           hzlb.Config(n=256, members=3, precision=4, nu=2.5e-4, noise_sigma=0.05, seed=6,
                       forcing_kmax=0, member_base=48)]
    if with512:
        out.append(hzlb.Config(n=512, members=2, precision=4, nu=1.25e-4, noise_sigma=0.05,
                               seed=7, forcing_kmax=0))
    return out


@pytest.mark.parametrize("mode,with512", [("fused", True), ("fused", False),
                                          ("fused_branch", True)])
def test_fused_kernels_match_separate_stepping(hzlb, mode, with512):
    """One persistent row kernel and one column kernel per RK stage over the whole mixed work
    list (and with the 512^2 resolution on its own branch) equal each resolution stepped alone,
    bit for bit, including the step counters that key the noise across graph batches."""
    cfgs = _fused_configs(hzlb, with512)
    dts = [2e-3, 1e-3, 5e-4, 2.5e-4][:len(cfgs)]
    m = hzlb.Mixed(cfgs)
    for k, (g, c) in enumerate(zip(m.groups, cfgs)):
        _init(hzlb, g, c, k)
    m.set_mode(mode)
    assert m.schedule()["mode"] == mode
    m.step(dts, 11)
    assert all(g.status() == 0 for g in m.groups)
    got = [g.get_state_compact() for g in m.groups]
    for k, ref in enumerate(_alone(hzlb, cfgs, dts, [11] * len(cfgs))):
        np.testing.assert_array_equal(got[k], ref)
    m.close()


def test_fused_modes_are_refused_where_they_do_not_apply(hzlb):
    m = hzlb.Mixed(_configs(hzlb))   # FP64 and 16^2 / 32^2 groups
    with pytest.raises(hzlb.HzlbInvalidArgument):
        m.set_mode("fused")
    m.close()
    m = hzlb.Mixed(_fused_configs(hzlb, with512=False))
    with pytest.raises(hzlb.HzlbInvalidArgument):
        m.set_mode("fused_branch")
    m.close()


@pytest.mark.parametrize("serial,threads", [(False, [64, 64, 64]), (False, [128, 128, 128]),
                                            (True, [64, 128, 0])])
def test_row_block_shapes_match_separate_stepping(hzlb, serial, threads):
    """hzlb_mixed_set_row_threads: the row kernel in blocks of 64 or 128 threads (both compiled
    for every resolution) gives the same bits as each resolution stepped alone; the shapes in
    effect are reported, 0 resolving to the resolution's default."""
    cfgs = _configs(hzlb) + [hzlb.Config(n=256, members=3, precision=4, nu=2.5e-4, seed=6,
                                         forcing_kmax=0),
                             hzlb.Config(n=512, members=2, precision=4, nu=1.25e-4, seed=7,
                                         forcing_kmax=0)]
    dts = [1e-3, 5e-4, 2e-3, 2.5e-4, 1.25e-4]
    threads = threads + [threads[0], threads[1]]
    m = hzlb.Mixed(cfgs)
    for k, (g, c) in enumerate(zip(m.groups, cfgs)):
        _init(hzlb, g, c, k)
    m.set_schedule(serial)
    m.set_row_threads(threads)
    shapes = m.schedule()["row_threads"]
    assert all(s in (64, 128) for s in shapes)
    assert all(s == t for s, t in zip(shapes, threads) if t)
    m.step(dts, 9)
    got = [g.get_state_compact() for g in m.groups]
    for k, ref in enumerate(_alone(hzlb, cfgs, dts, [9] * 5)):
        np.testing.assert_array_equal(got[k], ref)
    with pytest.raises(hzlb.HzlbError):
        m.set_row_threads([96, 0, 0, 0, 0])
    m.close()
