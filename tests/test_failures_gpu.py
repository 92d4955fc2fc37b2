"""Failure paths of the solvers and the device allocator, all raised on the
host side (nothing here faults, traps or hangs a GPU):

* a NaN or infinity in the initial Q or the unaries ends qp / lp with
  DCRF_E_NUMERIC, and the model stays usable;
* a device-memory budget smaller than a model needs ends its construction
  with DCRF_E_NOMEM before any device allocation, and lifting it lets the
  same construction succeed;
* the qp-gamma loop's cap (LP_inf_params::qp_max_iter, src/densecrf.cpp:
  650-675) runs out: with qp_max_iter = 1 and qp_tol = 0 every Frank-Wolfe
  iteration stops after exactly one qp-gamma iteration, as the reference's
  do-while does, and the solve still matches the CPU restatement.
"""
import numpy as np
import pytest

from densecrf_ho_b200 import (DCRFError, DenseCRF2D, device_memory_stats, set_device_memory_limit, synth)

pytestmark = pytest.mark.gpu

E_NOMEM, E_NUMERIC = 5, 6


def _model(img):
    m = DenseCRF2D(img["W"], img["H"], img["L"])
    m.setUnaryEnergy(img["unary"])
    m.addPairwiseGaussian(3.0, 3.0, 3.0)
    m.addPairwiseBilateral(50.0, 50.0, 15.0, 15.0, 15.0, img["rgb"], 5.0)
    return m


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_non_finite_initial_q_is_a_numeric_error(bad):
    img = synth.make_image(40, 30, 21, 3)
    m = _model(img)
    Q = m.unary_init()
    ref = m.qp_inference_super_pixels_non_convex(Q)
    Qb = Q.copy()
    Qb[17, 4] = bad
    with pytest.raises(DCRFError) as e:
        m.qp_inference_super_pixels_non_convex(Qb)
    assert e.value.code == E_NUMERIC and "NaN or an infinity" in str(e.value)
    with pytest.raises(DCRFError) as e:
        m.lp_inference_prox_super_pixels(Qb, prox_max_iter=2, fw_max_iter=2)
    assert e.value.code == E_NUMERIC
    # the model is still usable and gives the same answer as before
    assert np.array_equal(m.qp_inference_super_pixels_non_convex(Q), ref)


def test_non_finite_unary_is_a_numeric_error():
    img = synth.make_image(40, 30, 21, 4)
    m = _model(img)
    Q = m.unary_init()
    U = img["unary"].copy()
    U[5, 0] = np.nan
    m.setUnaryEnergy(U)
    for solve in (lambda: m.qp_inference_super_pixels_non_convex(Q),
                  lambda: m.lp_inference_prox_super_pixels(Q, prox_max_iter=1, fw_max_iter=2)):
        with pytest.raises(DCRFError) as e:
            solve()
        assert e.value.code == E_NUMERIC
    m.setUnaryEnergy(img["unary"])
    out = m.qp_inference_super_pixels_non_convex(Q)
    assert np.isfinite(out).all()


def test_device_memory_budget_refuses_on_the_host():
    img = synth.make_image(320, 240, 21, 5)
    in_use0, _, mallocs0 = device_memory_stats()
    set_device_memory_limit(in_use0 + (1 << 20))  # 1 MiB more than is held now
    try:
        with pytest.raises(DCRFError) as e:
            _model(img)
        assert e.value.code == E_NOMEM and "device memory limit" in str(e.value)
    finally:
        set_device_memory_limit(0)
    m = _model(img)  # the same construction without the budget
    assert np.isfinite(m.qp_inference_super_pixels_non_convex(m.unary_init())).all()
    in_use, _, mallocs = device_memory_stats()
    assert in_use > in_use0 and mallocs >= mallocs0


def test_qp_gamma_cap_runs_out(oracle_mod):
    W, H = 48, 36
    img = synth.make_image(W, H, 21, 6)
    orc = oracle_mod.build_model(oracle_mod.OracleModel, img)
    Q = orc.unary_init()
    m = _model(img)
    params = dict(prox_max_iter=3, fw_max_iter=4, qp_max_iter=1, qp_tol=0.0)
    out, st = m.lp_inference_prox_super_pixels(Q, stats=True, **params)
    assert st.inner_iters == 3 * 4
    assert st.gamma_iters == st.inner_iters  # the cap, not the tolerance, ended every qp-gamma loop
    ref, nit = orc.lp(Q, **params)
    assert st.iterations == nit
    assert (m.currentMap(out) == orc.current_map(ref)).mean() >= 0.999
    ea, eb = orc.energy_true(m.currentMap(out)), orc.energy_true(orc.current_map(ref))
    assert abs(ea - eb) <= 1e-4 * abs(eb)
