"""Parity of the headline configuration at its own batch size: Im-3m (No. 229) 128^3
FP32 centred KRFFT over 128 and 129 fields, which the library runs as several
workspace chunks on two or three concurrent lanes with programmatic dependent launch.

Every field's forward spectrum is compared with the FP64 truth on the spectral ASU,
and its backward with the input (the reference's bars, test/runtests.jl:199-216 and
test/test_centered_backward.jl:31-70; FP32 max relative error <= 1e-5 against FP64).
The fields are seeded combinations of k symmetric basis fields, so the truth of every
field is the same combination of the k bases' numpy FFTs.
"""
import os

import numpy as np
import pytest

from conftest import oracle_group

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

N = (128, 128, 128)
K_BASES = 4
TOL = 1e-5


@pytest.fixture(scope="module")
def headline(cf, O):
    ops, ops_s, oops = oracle_group(cf, O, 229, N)
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    ospec = O.calc_spectral_asu(oops, 3, N)
    bases, truths = [], []
    for k in range(K_BASES):
        u = O.make_symmetric(oops, N, seed=700 + k)
        bases.append(O.pack_stride(u, [2, 2, 2]))
        truths.append(O.spectrum_on_asu(u, ospec))
    return dict(ops_s=ops_s, spec=spec, ospec=ospec, bases=np.stack(bases), truths=np.stack(truths))


def _run(cf, h, B, lanes=None, chunk_bytes=None):
    env = {"CFFT_LANES": lanes, "CFFT_CHUNK_BYTES": chunk_bytes}
    old = {k: os.environ.get(k) for k in env}
    try:
        for k, v in env.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = str(v)
        plan = cf.KRFFTPlan(h["spec"], h["ops_s"], precision=4, max_batch=B, path=cf.PATH_CENTERED)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    info = (plan.info.chunk, plan.info.lanes)
    idx, _ = plan.spectral_asu()
    assert np.array_equal(idx, h["ospec"].idx)
    coef = np.random.default_rng(B * 7 + (lanes or 0)).standard_normal((B, K_BASES))
    f0 = np.einsum("bk,kxyz->bxyz", coef, h["bases"])                   # (B, M1, M2, M3)
    truth = coef @ h["truths"]                                          # (B, n_spec)
    dev = torch.tensor(np.ascontiguousarray(f0.transpose(0, 3, 2, 1)), dtype=torch.float32, device="cuda:0")
    F = plan.forward(dev)
    back = plan.backward(F)
    torch.cuda.synchronize()
    Fh = F.cpu().numpy().astype(np.complex128)
    bh = back.cpu().numpy().astype(np.float64).transpose(0, 3, 2, 1)
    plan.close()
    fwd_err = np.max(np.abs(Fh - truth), axis=1) / np.max(np.abs(truth), axis=1)
    bwd_err = np.max(np.abs(bh - f0).reshape(B, -1), axis=1) / np.max(np.abs(f0).reshape(B, -1), axis=1)
    return info, fwd_err, bwd_err


@pytest.mark.parametrize("B,lanes,chunk_bytes", [
    (128, None, None),            # the bench batch: 2 lanes x 64-field chunks
    (129, None, None),            # odd batch: a 1-field chunk at the end of the second pass
    (129, 3, None),               # three lanes, ragged last chunk
    (128, None, 10 * 2 ** 20),    # 20-field chunks: several chunks per lane
])
def test_headline_every_field_vs_fp64(cf, headline, B, lanes, chunk_bytes):
    (chunk, nl), fwd_err, bwd_err = _run(cf, headline, B, lanes, chunk_bytes)
    nchunks = -(-B // chunk)
    assert nl == (lanes or 2) and nchunks >= 2, (chunk, nl)
    worst_f, worst_b = int(np.argmax(fwd_err)), int(np.argmax(bwd_err))
    print(f"B={B} lanes={nl} chunk={chunk} chunks={nchunks}: forward max rel err {fwd_err.max():.3e} "
          f"(field {worst_f}), backward {bwd_err.max():.3e} (field {worst_b})")
    assert fwd_err.max() <= TOL, (worst_f, fwd_err.max())
    assert bwd_err.max() <= TOL, (worst_b, bwd_err.max())
