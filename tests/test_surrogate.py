"""FNO surrogate trained on SOCS pairs, and surrogate-assisted ILT (High-NA EUV).

The trained network is compared with the same network untrained (the method
without training) on held-out clips and inside ILT; the exact SOCS judge must
take over once the surrogate's image error passes the bound.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    from highuvlith_b200 import surrogate as S
    from highuvlith_b200.fno import FnoSurrogate
    eng = S.high_na_engine()
    fno = FnoSurrogate(512, 16, 4, seed=3)
    untrained = FnoSurrogate(512, 16, 4, seed=3)
    losses = S.train(fno, S.PairSource(eng, seed=11), steps=120, batch=8, lr=2e-3, lr_final=1e-4)
    return eng, fno, untrained, losses


def test_training_reduces_image_error(trained):
    from highuvlith_b200 import surrogate as S
    eng, fno, untrained, losses = trained
    assert np.mean(losses[-10:]) < 0.1 * np.mean(losses[:3])
    held, _ = S.PairSource(eng, seed=99).batch(16)
    e_tr = S.relative_image_error(fno, eng, held)
    e_un = S.relative_image_error(untrained, eng, held)
    # max|I_fno - I_socs| / max I_socs over each held-out clip
    assert np.median(e_tr) < 0.5 * np.median(e_un), (e_tr, e_un)
    assert np.median(e_tr) < 0.5


def _targets(eng):
    from highuvlith_b200.targets import gen_contact_targets
    tg, _ = gen_contact_targets(4, eng.grid.size, eng.grid.pixel_nm, base_seed=5)
    return torch.from_numpy(tg).cuda()


def test_surrogate_ilt_gain_and_judge(trained):
    from highuvlith_b200 import ilt, surrogate as S
    eng, fno, untrained, _ = trained
    tg = _targets(eng)
    st = ilt.IltSettings(cost="resist", threshold=0.25, steepness=50.0, max_iterations=15)
    th0 = ilt.initial_theta_from_target(tg).contiguous()
    c0, _ = ilt.cost_and_gradient(eng, th0, tg, st, want_gradient=False)

    # Surrogate only (judge never takes over): the trained network lowers the
    # exact cost of every mask, the untrained one does not do as well.
    th_tr = th0.clone()
    r_tr = S.optimize_with_surrogate(eng, fno, th_tr, tg, st, judge_every=5, error_bound=1e9)
    th_un = th0.clone()
    r_un = S.optimize_with_surrogate(eng, untrained, th_un, tg, st, judge_every=5, error_bound=1e9)
    assert r_tr.takeover_iteration == -1 and r_tr.exact_iterations == 0
    assert np.all(r_tr.final_cost < 0.9 * c0), (r_tr.final_cost, c0)
    assert np.all(r_tr.final_cost < r_un.final_cost), (r_tr.final_cost, r_un.final_cost)
    # final_cost is the exact cost at the final masks
    ce, _ = ilt.cost_and_gradient(eng, th_tr, tg, st, want_gradient=False)
    np.testing.assert_allclose(r_tr.final_cost, ce, rtol=1e-6)

    # Judge every 5th iterate with a bound below the surrogate's error: SOCS
    # takes over at iteration 5 and exact iterations finish the run.
    th_j = th0.clone()
    r_j = S.optimize_with_surrogate(eng, fno, th_j, tg, st, judge_every=5, error_bound=0.05)
    assert r_j.takeover_iteration == 5
    assert r_j.judge_errors and r_j.judge_errors[0] > 0.05
    assert r_j.surrogate_iterations == 5 and r_j.exact_iterations >= 1
    # after the takeover the exact iterations finish the job: well below the
    # start, and no worse than letting the surrogate run on
    assert np.all(r_j.final_cost < 0.5 * c0), (r_j.final_cost, c0)
    assert np.all(r_j.final_cost < r_tr.final_cost * 1.05)


def test_surrogate_ilt_rejects_grid_mismatch(trained):
    from highuvlith_b200 import ilt, surrogate as S
    from highuvlith_b200._lib import HuvError
    from highuvlith_b200.fno import FnoSurrogate
    eng = trained[0]
    small = FnoSurrogate(256, 16, 4, seed=1)
    th = torch.zeros((1, 512, 512), device="cuda")
    with pytest.raises(HuvError):
        S.optimize_with_surrogate(eng, small, th, th.clone(), ilt.IltSettings(max_iterations=1))
