"""The reference's uniform-viscosity sweep (tests/test_response_3d.f90:25-30,
63-81, 218-250) on the device: for every p and both degree-1 frames, the 3-D
pseudo-spectral advance with a laterally constant perturbation p equals the
1-D run with eta * 10^p, memory and uplift to 1e-9 relative over 25 steps.
FP64 path; the tensor-core paths are held to the same tolerance in their own
test file."""
import pytest

from fastearth3d_b200 import lib as vlib
from sweep_util import PSWEEP, TOL, sweep_errors

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("deg1_cm", [False, True])
@pytest.mark.parametrize("p_pert", PSWEEP)
def test_gpu_uniform_sweep_fp64(p_pert, deg1_cm):
    emem, eupl = sweep_errors(vlib.Model, vlib.default_params, p_pert, deg1_cm)
    assert emem <= TOL and eupl <= TOL, (emem, eupl)
