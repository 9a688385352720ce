"""Full-grid plans (L = 1) on the device.

Forward = the centring prefold (CenteringPreFoldPlan, src/centering_prefold.jl:27-257):
the whole grid folds into parity channels of (N/2)^3, each channel is transformed and
the spectral-ASU points are merged from the channel spectra.  It needs only the
centring translations of the field, like the reference's prefold, and is checked
against fftn(u) on the ASU points for fields symmetrised over the centring only.
Backward = the full-grid inverse with symmetry fill (src/recursive_blocks_backward.jl:
531-545): spectral ASU -> whole grid, checked by round trip on symmetric fields.
The diffusion step on the full grid is checked against IFFT(K FFT(u))."""
import numpy as np
import pytest

from conftest import rel_err, to_oracle_ops, oracle_shifted_ops

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

LAT = np.eye(3)
DS = 0.05
TOL = {8: 1e-10, 4: 1e-5}


def to_dev(u, precision):
    dt = torch.float64 if precision == 8 else torch.float32
    return torch.tensor(np.asarray(u).ravel(order="F"), dtype=dt, device="cuda:0").view(*reversed(u.shape))


def from_dev(t, N):
    return t.detach().cpu().numpy().astype(np.float64).ravel().reshape(N, order="F")


def _plan(cf, sg, N, precision):
    ops_s = oracle_shifted_ops(cf, sg, N)
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    plan = cf.plan_krfft_prefold(ops_s, N, precision=precision, ds=DS, lattice=LAT)
    return plan, ops_s, spec


@pytest.mark.parametrize("sg,n,precision", [(229, 32, 8), (225, 32, 8), (63, 32, 8), (230, 48, 4), (229, 64, 4)])
def test_prefold_forward_needs_only_centring(cf, O, sg, n, precision):
    N = (n,) * 3
    plan, ops_s, spec = _plan(cf, sg, N, precision)
    assert plan.centered and tuple(plan.M) == N
    oops = to_oracle_ops(O, ops_s)
    # symmetric under the pure translations only (the centring), not the whole group
    cent = [op for op in oops if np.array_equal(op.Rm, np.eye(3, dtype=int))]
    u = O.make_symmetric(cent, N, seed=17)
    F = cf.execute_prefold_krfft(plan, to_dev(u, precision)).cpu().numpy()
    truth = O.spectrum_on_asu(u, O.calc_spectral_asu(oops, 3, N))
    assert rel_err(F, truth) < TOL[precision]
    plan.close()


@pytest.mark.parametrize("sg,n,precision", [(229, 32, 8), (227, 32, 8), (221, 16, 8), (230, 48, 4)])
def test_fullgrid_backward_symmetry_fill(cf, O, sg, n, precision):
    N = (n,) * 3
    plan, ops_s, spec = _plan(cf, sg, N, precision)
    u = O.make_symmetric(to_oracle_ops(O, ops_s), N, seed=3)
    F = plan.forward(to_dev(u, precision))
    back = from_dev(plan.backward(F), N)
    assert rel_err(back, u) < TOL[precision] * 10
    plan.close()


@pytest.mark.parametrize("sg", [229, 225, 221])
def test_fullgrid_scft_step(cf, O, sg):
    N = (32, 32, 32) if sg != 221 else (16, 16, 16)
    plan, ops_s, _ = _plan(cf, sg, N, 8)
    u = O.make_symmetric(to_oracle_ops(O, ops_s), N, seed=8)
    q = to_dev(u, 8)
    plan.scft_step(q)
    assert np.max(np.abs(from_dev(q, N) - O.fullgrid_reference(u, N, DS, LAT, [1, 1, 1]))) < 1e-12
    plan.close()
