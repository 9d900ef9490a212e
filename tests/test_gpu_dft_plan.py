"""Bootstrapping DFT plans generated and encoded on the device (wg_dft_plan_create) against the
reference's own walsh15 plans, word for word: every stage's indices, baby steps, rescale flag
and all QP diagonal plaintexts (Montgomery form) of SlotToCoeff at the parameter scale and at
twice it, and CoeffToSlot (ckks_generate_bootstrap_dft_plan,
src/ckks/operations/bootstrap/ckks_bootstrap_dft.cpp:961-1079)."""
import numpy as np
import pytest

from test_dft_plan import _literals

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def walsh15_plans(ref_mod):
    return ref_mod.RefPlans(bootstrap_keys=True)


@pytest.mark.parametrize("which", ["s2c", "c2s", "s2c_x2"])
def test_device_plan_matches_reference(wg, walsh15_plans, which):
    R = walsh15_plans
    code, lit = _literals(wg, R)[which]
    if code is None:
        code = R.build_scaled_s2c(2)
    ctx = wg.Context(R.N, R.q, R.p, R.dnum)
    stages = ctx.dft_plan(lit)
    assert len(stages) == R.stages(code)
    for k, st in enumerate(stages):
        ref = R.stage(code, k)
        inf = st.info()
        assert (inf["nterms"], inf["baby"], inf["rescale"]) == (ref["nterms"], ref["baby"], ref["rescale"]), k
        assert inf["level"] + 1 + len(R.p) == ref["qp_limbs"], k
        idx, diags = st.download()
        assert (idx == ref["indices"]).all(), k
        bad = int((diags != ref["diagonals"]).sum())
        assert bad == 0, (which, k, bad)
    for st in stages:
        st.close()
