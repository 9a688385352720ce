"""Fused 8-CTA cluster kernels (fold + x/y/z FFT in distributed shared memory; orbit
expansion + inverse z/y/x FFT + unfold) against the separate plane and z kernels of the
same plan (CFFT_CLUSTER=0) and against the FP64 oracle's full-grid truth.

Covers every centring that reaches the cluster kernels on cubic grids (plain, I, F, C),
channel edges H = 16, 24 and 32, both precisions, odd batches (the last workspace slot
holds one field) and the interaction-factor path of the diffusion step."""
import os

import numpy as np
import pytest

from conftest import rel_err, oracle_shifted_ops

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

LAT = np.eye(3)
DS = 0.05
SAME = {4: 2e-6, 8: 1e-13}   # cluster vs separate kernels: same arithmetic, different order
TRUTH = {4: 1e-5, 8: 1e-10}  # against the FP64 full-grid FFT

# (space group, grid edge, precision, expected centring type name)
CASES = [
    (229, 128, 4, "I"),   # Im-3m, H = 32, 4 channels
    (229, 64, 8, "I"),    # H = 16
    (230, 96, 4, "I"),    # Ia-3d, H = 24
    (225, 96, 4, "F"),    # Fm-3m, 2 channels
    (227, 64, 8, "F"),    # Fd-3m (origin choice 2)
    (63, 64, 4, "C"),     # Cmcm, 4 channels
    (65, 64, 8, "C"),     # Cmmm (the A-centred groups of the table reduce with L = (2, 2, 1) instead)
    (47, 64, 8, "P"),     # Pmmm, plain path, H = 32
    (221, 64, 4, "P"),    # Pm-3m
]


def _plans(cf, sg, n, precision, batch):
    N = (n,) * 3
    ops_s = oracle_shifted_ops(cf, sg, N)
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    outer = os.environ.get("CFFT_CLUSTER")
    try:
        os.environ["CFFT_CLUSTER"] = outer or "8"  # the cluster kernels are opt-in
        fused = cf.KRFFTPlan(spec, ops_s, precision=precision, max_batch=batch, ds=DS, lattice=LAT)
        os.environ["CFFT_CLUSTER"] = "0"
        sep = cf.KRFFTPlan(spec, ops_s, precision=precision, max_batch=batch, ds=DS, lattice=LAT)
    finally:
        if outer is None:
            del os.environ["CFFT_CLUSTER"]
        else:
            os.environ["CFFT_CLUSTER"] = outer
    return fused, sep, ops_s, spec


@pytest.mark.parametrize("sg,n,precision,cent", CASES)
def test_cluster_matches_separate_kernels(cf, sg, n, precision, cent):
    B = 3
    fused, sep, _, _ = _plans(cf, sg, n, precision, B)
    assert fused.info.exec_path & 4, "fused cluster kernels expected for this grid"
    assert not sep.info.exec_path & 4
    assert fused.centering == cent or (cent == "P" and not fused.centered)
    rdt = torch.float32 if precision == 4 else torch.float64
    g = torch.Generator(device="cuda:0").manual_seed(sg + n)
    shape = (B,) + tuple(reversed(fused.M))
    f0 = torch.randn(shape, generator=g, device="cuda:0", dtype=rdt)
    Fa, Fb = fused.forward(f0), sep.forward(f0)
    assert rel_err(Fa.cpu().numpy(), Fb.cpu().numpy()) < SAME[precision]
    ba, bb = fused.backward(Fa), sep.backward(Fa)
    assert rel_err(ba.cpu().numpy(), bb.cpu().numpy()) < SAME[precision]
    qa, qb = f0.clone(), f0.clone()
    fused.scft_step(qa)
    sep.scft_step(qb)
    assert rel_err(qa.cpu().numpy(), qb.cpu().numpy()) < SAME[precision]
    w = 0.3 * torch.randn(shape, generator=g, device="cuda:0", dtype=rdt)
    qa, qb = f0.clone(), f0.clone()
    fused.step_diffusion(qa, w, 0.02, n_steps=2)
    sep.step_diffusion(qb, w, 0.02, n_steps=2)
    assert rel_err(qa.cpu().numpy(), qb.cpu().numpy()) < SAME[precision]
    fused.close()
    sep.close()


@pytest.mark.parametrize("sg,n,precision", [(225, 96, 8), (63, 64, 8), (68, 64, 4), (229, 64, 4)])
def test_cluster_against_oracle(cf, O, sg, n, precision):
    from conftest import to_oracle_ops

    N = (n,) * 3
    fused, sep, ops_s, spec = _plans(cf, sg, n, precision, 1)
    sep.close()
    assert fused.info.exec_path & 4
    oops = to_oracle_ops(O, ops_s)
    u = O.make_symmetric(oops, N, seed=7)
    f0 = O.pack_stride(u, fused.L)
    rdt = torch.float32 if precision == 4 else torch.float64
    t = torch.tensor(np.asarray(f0).ravel(order="F"), dtype=rdt, device="cuda:0").view(*reversed(fused.M))
    F = fused.forward(t).cpu().numpy()
    truth = O.spectrum_on_asu(u, O.calc_spectral_asu(oops, 3, N))
    assert rel_err(F, truth) < TRUTH[precision]
    back = fused.backward(fused.forward(t)).cpu().numpy().astype(np.float64).ravel().reshape(fused.M, order="F")
    assert rel_err(back, f0) < TRUTH[precision] * 10
    fused.close()


@pytest.mark.parametrize("sg,n,precision", [(229, 128, 4), (47, 64, 8), (221, 64, 4)])
def test_cluster16_matches_separate_kernels(cf, sg, n, precision):
    """16-CTA clusters (two z-planes per CTA) where the device allows that size."""
    B = 3
    os.environ["CFFT_CLUSTER"] = "16"
    try:
        fused, sep, _, _ = _plans(cf, sg, n, precision, B)
    finally:
        os.environ.pop("CFFT_CLUSTER", None)
    assert fused.info.exec_path & 4
    rdt = torch.float32 if precision == 4 else torch.float64
    g = torch.Generator(device="cuda:0").manual_seed(sg)
    f0 = torch.randn((B,) + tuple(reversed(fused.M)), generator=g, device="cuda:0", dtype=rdt)
    Fa = fused.forward(f0)
    assert rel_err(Fa.cpu().numpy(), sep.forward(f0).cpu().numpy()) < SAME[precision]
    assert rel_err(fused.backward(Fa).cpu().numpy(), sep.backward(Fa).cpu().numpy()) < SAME[precision]
    fused.close()
    sep.close()
