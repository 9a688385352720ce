"""Legacy block path: plan_cfft + mul!/ldiv! (src/cfft_plan.jl, src/execution.jl) on the
device block transform, mirroring test/runtests.jl:80-115 and test/test_cfft.jl:74-110
(CFFT round trip, p2mm) and
checking every block against numpy's FFT."""
import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)


@pytest.mark.parametrize("N,sg,T", [((16, 16), 6, np.complex128), ((8, 8, 8), 47, np.complex128),
                                    ((16, 16, 16), 229, np.complex128), ((12, 12, 12), 221, np.complex64)])
def test_cfft_roundtrip_and_blocks(cf, N, sg, T):
    plan = cf.plan_cfft(N, sg, T)
    rng = np.random.default_rng(sg)
    inp = copy.deepcopy(plan.asu)
    for blocks in inp.dim_blocks.values():
        for b in blocks:
            b.data = (rng.standard_normal(b.data.shape) + 1j * rng.standard_normal(b.data.shape)).astype(T)
    spec = cf.mul(copy.deepcopy(plan.asu), plan, inp)
    tol = 1e-12 if T == np.complex128 else 2e-5
    for d, blocks in inp.dim_blocks.items():
        for b, s in zip(blocks, spec.dim_blocks[d]):
            want = np.fft.fftn(b.data.astype(np.complex128))
            assert np.max(np.abs(s.data - want)) <= tol * max(1.0, np.max(np.abs(want)))
    recon = cf.ldiv(copy.deepcopy(plan.asu), plan, spec)
    err = max(np.max(np.abs(r.data - b.data)) for d in inp.dim_blocks
              for r, b in zip(recon.dim_blocks[d], inp.dim_blocks[d]))
    assert err < (1e-12 if T == np.complex128 else 1e-5)
    plan.close()
