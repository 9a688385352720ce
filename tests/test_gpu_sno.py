"""The warm-start network on the device (cfft_sno_*) against its FP64 oracle
(oracle/sno_oracle.py, full-grid numpy FFTs; BF16 rounding emulated where the device
rounds: the weights and the inputs of the tensor-core channel products).

- forward: predicted fields [w_A | w_B] on the plan's subgrid, three groups (centred
  Im-3m and Ia-3d, primitive Pm-3m), relative error <= 2e-4;
- gradients of every parameter tensor, relative (to the tensor's largest entry)
  error <= 2e-3;
- a few Adam steps on fixed targets reduce the loss;
- weights survive a save / load round trip at BF16 precision.
"""
import numpy as np
import pytest

from conftest import oracle_group

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import sno_oracle as S  # noqa: E402

PARAMS = [(20.0, 0.4), (14.0, 0.33)]


def _case(cf, O, sg, N, nsamp=2):
    ops = O.get_ops(sg, 3, N)
    shift, oops = O.find_optimal_shift(ops, N)
    ops_s = [cf.SymOp(op.R, op.t) for op in oops]
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    plan = cf.KRFFTPlan(spec, ops_s, precision=4, max_batch=32 * nsamp)
    a = np.stack([S.features(sg, N, c, f, ops, shift) for c, f in PARAMS[:nsamp]])
    return plan, shift, oops, a


def _to_sub(x, L):
    """(S, C, N1, N2, N3) full grid [x, y, z] -> (S, C, M3, M2, M1) memory order."""
    sub = x[:, :, ::L[0], ::L[1], ::L[2]]
    return np.ascontiguousarray(sub.transpose(0, 1, 4, 3, 2))


def _targets(O, oops, N, nsamp):
    t = np.stack([np.stack([O.make_symmetric(oops, N, seed=10 * s + c) for c in range(2)]) for s in range(nsamp)])
    return 0.1 * t


@pytest.mark.parametrize("sg,n", [(229, 16), (230, 16), (221, 16), (230, 32), (229, 32)])
def test_sno_forward_matches_oracle(cf, O, sg, n):
    N = (n, n, n)
    plan, shift, oops, a = _case(cf, O, sg, N)
    model = cf.SpectralNeuralOperator()
    p = S.unflatten(model.get_params().astype(np.float64))
    ctx = model.bind(plan, sg, shift, 2)
    w = ctx.predict(PARAMS).cpu().numpy().astype(np.float64)
    out, _ = S.SNO(p, bf16_mode=True).forward(a)
    want = np.stack([np.stack(S.w_from_output(out[s], c, f)) for s, (c, f) in enumerate(PARAMS)])
    want = _to_sub(want, plan.L)
    dev = w - np.array([[c * (1 - f), c * f] for c, f in PARAMS])[:, :, None, None, None]
    ref = want - np.array([[c * (1 - f), c * f] for c, f in PARAMS])[:, :, None, None, None]
    err = np.max(np.abs(dev - ref)) / np.max(np.abs(ref))
    assert err <= 2e-4, err
    ctx.close()
    model.close()
    plan.close()


@pytest.mark.parametrize("sg", [229, 221])
def test_sno_gradients_match_oracle(cf, O, sg):
    N = (16, 16, 16)
    plan, shift, oops, a = _case(cf, O, sg, N)
    model = cf.SpectralNeuralOperator()
    p = S.unflatten(model.get_params().astype(np.float64))
    t = _targets(O, oops, N, 2)
    w_t = np.stack([np.stack(S.w_from_output(t[s], c, f)) for s, (c, f) in enumerate(PARAMS)])
    ctx = model.bind(plan, sg, shift, 2)
    wt_dev = torch.tensor(_to_sub(w_t, plan.L), dtype=torch.float32, device="cuda")
    loss = ctx.train_step(PARAMS, wt_dev, step=False)
    g_dev = S.unflatten(model.grads().astype(np.float64))
    net = S.SNO(p, bf16_mode=True)
    out, c = net.forward(a)
    assert abs(loss - net.loss(out, t)) <= 1e-4 * net.loss(out, t)
    g = net.backward(out, t, c)
    for k in S.PARAM_ORDER:
        scale = np.max(np.abs(g[k]))
        if scale == 0.0:
            assert np.max(np.abs(g_dev[k])) < 1e-12, k
            continue
        err = np.max(np.abs(g_dev[k] - g[k])) / scale
        assert err <= 2e-3, (k, err)
    ctx.close()
    model.close()
    plan.close()


def test_sno_training_reduces_loss_and_save_load(cf, O, tmp_path):
    N = (16, 16, 16)
    plan, shift, oops, a = _case(cf, O, 230, N)
    model = cf.SpectralNeuralOperator(lr=2e-3)
    ctx = model.bind(plan, 230, shift, 2)
    t = _targets(O, oops, N, 2)
    w_t = np.stack([np.stack(S.w_from_output(t[s], c, f)) for s, (c, f) in enumerate(PARAMS)])
    wt_dev = torch.tensor(_to_sub(w_t, plan.L), dtype=torch.float32, device="cuda")
    losses = [ctx.train_step(PARAMS, wt_dev) for _ in range(30)]
    assert losses[-1] < 0.5 * losses[0], losses
    path = tmp_path / "w.npy"
    model.save(str(path))
    before = ctx.predict(PARAMS).cpu().numpy()
    m2 = cf.SpectralNeuralOperator()
    m2.load(str(path))
    ctx2 = m2.bind(plan, 230, shift, 2)
    after = ctx2.predict(PARAMS).cpu().numpy()
    # the working copy is BF16 already, so only the FP32 biases move (by BF16 rounding)
    assert np.max(np.abs(after - before)) <= 2e-2 * np.max(np.abs(before))
    for o in (ctx, ctx2, model, m2, plan):
        o.close()



def _adam_first_step(w, g, lr, b1=0.9, b2=0.999, eps=1e-8):
    """Adam's first step from zero moments (cfft_sno_create's defaults, no weight decay)."""
    m = (1 - b1) * g / (1 - b1)
    v = (1 - b2) * g * g / (1 - b2)
    return w - lr * m / (np.sqrt(v) + eps)


def test_sno_split_step_and_data_parallel_step(cf, O):
    # cfft_sno_grads_device copies the gradients of the last train call; cfft_sno_apply_grads
    # takes one Adam step from a caller's gradient buffer; the data-parallel step on a
    # one-rank NCCL group (share 1, all-reduce of one rank) takes that step from the
    # all-reduced buffer.  Each is checked against Adam's first step on the host from the
    # exact gradients used (the gradient reductions use atomics, so two separate runs
    # may differ in the last bits).
    import datetime
    import socket

    import torch.distributed as dist

    N = (16, 16, 16)
    lr = 1e-3
    plan, shift, oops, a = _case(cf, O, 229, N)
    t = _targets(O, oops, N, 2)
    w_t = np.stack([np.stack(S.w_from_output(t[s], c, f)) for s, (c, f) in enumerate(PARAMS)])
    wt_dev = torch.tensor(_to_sub(w_t, plan.L), dtype=torch.float32, device="cuda")

    m1 = cf.SpectralNeuralOperator(lr=lr)
    c1 = m1.bind(plan, 229, shift, 2)
    w0 = m1.get_params().astype(np.float64)
    loss1 = c1.train_step(PARAMS, wt_dev, step=False)
    g = m1.grads_device()
    assert np.array_equal(g.cpu().numpy(), m1.grads())
    g_used = (0.5 * g).contiguous()  # any caller buffer, not the model's own gradients
    m1.apply_grads(g_used)
    want = _adam_first_step(w0, g_used.cpu().numpy().astype(np.float64), lr)
    assert np.max(np.abs(m1.get_params() - want)) <= 1e-6 * lr + 1e-7 * np.max(np.abs(w0))

    m2 = cf.SpectralNeuralOperator(lr=lr)
    c2 = m2.bind(plan, 229, shift, 2)
    assert np.array_equal(m2.get_params(), w0.astype(np.float32))  # seeded initial weights
    buf = torch.empty(cf.sno.N_PARAMS + 1, dtype=torch.float32, device="cuda")
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        loss2 = c2.train_step_data_parallel(PARAMS, wt_dev, len(PARAMS), dist, grad_buf=buf)
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
    assert abs(loss2 - loss1) <= 1e-5 * abs(loss1)
    assert abs(float(buf[-1]) - loss2) <= 1e-6 * abs(loss2)
    want2 = _adam_first_step(w0, buf[:-1].cpu().numpy().astype(np.float64), lr)
    assert np.max(np.abs(m2.get_params() - want2)) <= 1e-6 * lr + 1e-7 * np.max(np.abs(w0))
    for o in (c1, c2, m1, m2, plan):
        o.close()
