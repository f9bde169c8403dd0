"""The oracle against the reference's uniform-viscosity sweep
(tests/test_response_3d.f90:25-30, 63-81, 218-250): for every p of the sweep
and both degree-1 frames, the 3-D pseudo-spectral advance with a laterally
constant perturbation p equals the 1-D run with eta * 10^p, memory and
uplift to 1e-9 relative over 25 steps."""
import pytest

from oracle import orc
from sweep_util import PSWEEP, TOL, sweep_errors


@pytest.mark.parametrize("deg1_cm", [False, True])
@pytest.mark.parametrize("p_pert", PSWEEP)
def test_oracle_uniform_sweep(p_pert, deg1_cm):
    emem, eupl = sweep_errors(orc.Oracle, orc.default_params, p_pert, deg1_cm)
    assert emem <= TOL and eupl <= TOL, (emem, eupl)
