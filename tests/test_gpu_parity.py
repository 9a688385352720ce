"""GPU parity: the CUDA path (through the C ABI) against the FP64 oracle and full-grid
FFT truth, mirroring the reference's tests (test/runtests.jl, test/test_centered_*.jl,
test/test_m2_*.jl).  Tolerances: FP64 as the reference's own bars (1e-10 relative
for transforms, 1e-10 absolute for the diffusion step); FP32 max relative error
<= 1e-5 against FP64 (the target for the single-precision path)."""
import numpy as np
import pytest

from conftest import rel_err, oracle_shifted_ops

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

N16 = (16, 16, 16)
LAT = np.eye(3)
DS = 0.05
TOL = {8: 1e-10, 4: 1e-5}


def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def to_dev(f0, precision):
    """(M1,M2,M3) numpy field (x fastest) -> contiguous (M3,M2,M1) CUDA tensor."""
    M = f0.shape
    dt = torch.float64 if precision == 8 else torch.float32
    return torch.tensor(np.asarray(f0).ravel(order="F"), dtype=dt, device=dev()).view(*reversed(M))


def from_dev(t, M):
    return t.detach().cpu().numpy().astype(np.float64).ravel().reshape(M, order="F")


def make_plan(cf, p, N, precision, path=0, ds=DS, lattice=LAT, max_batch=1):
    return cf.KRFFTPlan(p["spec"], p["ops_s"], N=N, ds=ds, lattice=lattice, precision=precision,
                        max_batch=max_batch, path=path)


GROUPS = [221, 225, 227, 229, 230, 47, 63, 70, 72, 10, 2, 139, 136, 224, 166]


@pytest.mark.parametrize("precision", [8, 4])
@pytest.mark.parametrize("sg", GROUPS)
def test_forward_backward_scft(cf, O, prep, sg, precision):
    N = (12, 12, 12) if sg == 166 else N16
    lattice = np.array([[1.0, -0.5, 0], [0, np.sqrt(3) / 2, 0], [0, 0, 1.3]]) if sg == 166 else LAT
    p = prep(sg, N)
    plan = make_plan(cf, p, N, precision, lattice=lattice)
    ospec = O.calc_spectral_asu(p["oops"], 3, N)
    f0 = O.pack_stride(p["u"], plan.L)
    truth = O.spectrum_on_asu(p["u"], ospec)
    F = plan.forward(to_dev(f0, precision))
    torch.cuda.synchronize()
    assert rel_err(F.cpu().numpy(), truth) < TOL[precision]
    back = from_dev(plan.backward(F), plan.M)
    assert rel_err(back, f0) < TOL[precision] * 10
    q = to_dev(f0, precision)
    plan.scft_step(q)
    ref = O.fullgrid_reference(p["u"], N, DS, lattice, plan.L)
    if sg != 166:  # hexagonal K is not invariant at the Nyquist wrap on a tiny grid
        assert np.max(np.abs(from_dev(q, plan.M) - ref)) < (1e-10 if precision == 8 else 1e-5)
    plan.close()


@pytest.mark.parametrize("path", [0, 1])
def test_centered_and_m2_paths_agree(cf, O, prep, path):
    p = prep(229, N16)
    plan = make_plan(cf, p, N16, 8, path=path)
    assert plan.centered == (path == 0)
    f0 = O.pack_stride(p["u"], plan.L)
    F = plan.forward(to_dev(f0, 8)).cpu().numpy()
    truth = O.spectrum_on_asu(p["u"], O.calc_spectral_asu(p["oops"], 3, N16))
    assert rel_err(F, truth) < 1e-12
    plan.close()


def test_oracle_pipeline_bitwise_close(cf, O, prep):
    """CUDA FP64 against the oracle's own reference-style pipeline (not only truth)."""
    p = prep(230, N16)
    ospec = O.calc_spectral_asu(p["oops"], 3, N16)
    oplan = O.plan_centered_scft(ospec, p["oops"], N16, DS, LAT)
    f0 = O.pack_stride(p["u"], [2, 2, 2])
    F_o = O.fft_reconstruct_centered(oplan.fwd, f0)
    plan = make_plan(cf, p, N16, 8)
    F = plan.forward(to_dev(f0, 8)).cpu().numpy()
    assert np.max(np.abs(F - F_o)) < 1e-11
    out_o = O.execute_centered_scft(oplan, f0)
    q = to_dev(f0, 8)
    plan.scft_step(q)
    assert np.max(np.abs(from_dev(q, plan.M) - out_o)) < 1e-12
    plan.close()


@pytest.mark.parametrize("precision", [8, 4])
def test_batched_calls(cf, O, prep, precision):
    seeds = [1, 2, 3]
    ps = [prep(229, N16, seed=s) for s in seeds]
    plan = make_plan(cf, ps[0], N16, precision, max_batch=4)
    f0s = [O.pack_stride(p["u"], [2, 2, 2]) for p in ps]
    batch = torch.stack([to_dev(f, precision) for f in f0s])
    F = plan.forward(batch)
    assert F.shape == (3, plan.n_spec)
    for i, p in enumerate(ps):
        truth = O.spectrum_on_asu(p["u"], O.calc_spectral_asu(p["oops"], 3, N16))
        assert rel_err(F[i].cpu().numpy(), truth) < TOL[precision]
    back = plan.backward(F)
    for i in range(3):
        assert rel_err(from_dev(back[i], plan.M), f0s[i]) < TOL[precision] * 10
    with pytest.raises(cf.CFFTError):
        plan.forward(torch.zeros((5,) + tuple(reversed(plan.M)), dtype=batch.dtype, device=batch.device))
    plan.close()


def test_host_buffer_api(cf, O, prep):
    p = prep(225, N16)
    plan = make_plan(cf, p, N16, 8, max_batch=2)
    f0 = O.pack_stride(p["u"], [2, 2, 2])
    F = cf.fft_reconstruct_centered(plan, f0)  # numpy -> host entry point
    truth = O.spectrum_on_asu(p["u"], O.calc_spectral_asu(p["oops"], 3, N16))
    assert rel_err(F, truth) < 1e-10
    back = cf.ifft_unrecon_centered(plan, F)
    assert np.max(np.abs(back - f0)) < 1e-10
    out = cf.execute_centered_scft(plan, f0)
    assert np.max(np.abs(out - O.fullgrid_reference(p["u"], N16, DS, LAT, [2, 2, 2]))) < 1e-12
    plan.close()


@pytest.mark.parametrize("B", [5, 11])
def test_host_pipeline_pieces(cf, B):
    # Im-3m 128^3 FP32: 1 MiB per field, so the host entry points cut the batch into
    # several pieces (ragged for 5 and 11 fields) whose copies overlap.  The host
    # path must agree with the device-tensor path on the same fields.
    N = (128, 128, 128)
    ops_s = oracle_shifted_ops(cf, 229, N)
    spec = cf.calc_spectral_asu(ops_s, 3, N)
    plan = cf.KRFFTPlan(spec, ops_s, precision=4, max_batch=B, ds=DS, lattice=LAT)
    g = torch.Generator(device="cuda:0").manual_seed(B)
    f0 = torch.randn((B,) + tuple(reversed(plan.M)), generator=g, device="cuda:0", dtype=torch.float32)
    want_F = plan.forward(f0)
    host = np.stack([x.cpu().numpy().transpose(2, 1, 0) for x in f0])  # (B, M1, M2, M3) column-major fields
    F = plan.forward(host)
    assert rel_err(F, want_F.cpu().numpy()) < 1e-5
    back = plan.backward(F)
    want_back = plan.backward(want_F)
    assert rel_err(back, np.stack([x.cpu().numpy().transpose(2, 1, 0) for x in want_back])) < 1e-5
    stepped = plan.scft_step(host)
    want_step = plan.scft_step(f0.clone())
    assert rel_err(stepped, np.stack([x.cpu().numpy().transpose(2, 1, 0) for x in want_step])) < 1e-5
    plan.close()


def test_update_kernel(cf, O, prep):
    # test/runtests.jl:347-365: update equals a fresh plan
    p = prep(221, N16)
    plan = make_plan(cf, p, N16, 8, ds=0.05)
    f0 = O.pack_stride(p["u"], plan.L)
    plan.update_kernel(0.10)
    a = to_dev(f0, 8)
    plan.scft_step(a)
    fresh = make_plan(cf, p, N16, 8, ds=0.10)
    b = to_dev(f0, 8)
    fresh.scft_step(b)
    assert torch.max(torch.abs(a - b)).item() < 1e-14
    plan.close()
    fresh.close()


@pytest.mark.parametrize("sg", [229, 47, 230])
def test_step_diffusion(cf, O, prep, sg):
    """step_diffusion! (src/diffusion_solver.jl:254-267) applied 3 times vs the oracle."""
    p = prep(sg, N16)
    plan = make_plan(cf, p, N16, 8)
    L = plan.L
    f0 = O.pack_stride(p["u"], L)
    w = O.pack_stride(O.make_symmetric(p["oops"], N16, seed=99), L)
    q = to_dev(f0, 8)
    plan.step_diffusion(q, to_dev(w, 8), 0.02, n_steps=3)
    oplan = O.plan_m2_scft_ops(p["oops"], N16, DS, LAT)
    ref = f0
    for _ in range(3):
        ref = O.step_diffusion(lambda x: O.execute_m2_scft(oplan, x), ref, w, 0.02)
    assert np.max(np.abs(from_dev(q, plan.M) - ref)) < 1e-12
    plan.close()


def test_grid_conversion(cf, O, prep):
    p = prep(229, N16)
    plan = make_plan(cf, p, N16, 8)
    u = torch.tensor(p["u"].ravel(order="F"), dtype=torch.float64, device=dev()).view(*reversed(N16))
    f0 = plan.fullgrid_to_subgrid(u)
    assert np.array_equal(from_dev(f0, plan.M), O.pack_stride(p["u"], plan.L))
    full = plan.subgrid_to_fullgrid(f0)
    back = full.cpu().numpy().ravel().reshape(N16, order="F")
    assert np.max(np.abs(back - p["u"])) < 1e-12
    plan.close()


def test_pmmm_64_fp64_config(cf, O, prep):
    """Pmmm (No. 47) 64^3 Float64 forward+backward vs a full 3-D FFT."""
    N = (64, 64, 64)
    p = prep(47, N, seed=11)
    plan = make_plan(cf, p, N, 8)
    assert plan.L == [2, 2, 2] and plan.n_spec == 32 ** 3
    f0 = O.pack_stride(p["u"], plan.L)
    F = plan.forward(to_dev(f0, 8))
    truth = O.spectrum_on_asu(p["u"], O.calc_spectral_asu(p["oops"], 3, N))
    assert rel_err(F.cpu().numpy(), truth) < 1e-12
    back = from_dev(plan.backward(F), plan.M)
    assert np.max(np.abs(back - f0)) < 1e-12
    plan.close()


def test_im3m_128_fp32_config(cf, O, prep):
    """Im-3m (No. 229) 128^3 FP32 centred KRFFT: ASU spectrum vs FP64 full FFT (max
    relative error <= 1e-5), round trip, index tables bit-exact vs the oracle."""
    N = (128, 128, 128)
    p = prep(229, N, seed=5)
    plan = make_plan(cf, p, N, 4)
    assert plan.centered and plan.n_channels == 4 and plan.H == (32, 32, 32)
    ospec = O.calc_spectral_asu(p["oops"], 3, N)
    idx, mult = plan.spectral_asu()
    assert np.array_equal(idx, ospec.idx) and np.array_equal(mult, ospec.mult)
    f0 = O.pack_stride(p["u"], plan.L)
    F = plan.forward(to_dev(f0, 4))
    truth = O.spectrum_on_asu(p["u"], ospec)
    assert rel_err(F.cpu().numpy().astype(np.complex128), truth) <= 1e-5
    back = from_dev(plan.backward(F), plan.M)
    assert rel_err(back, f0) <= 1e-5
    plan.close()


def test_linearity_and_roundtrip_large(cf, O, prep):
    """Size-independent properties at 128^3: linearity of the forward transform and
    backward(forward(x)) == x for a batch."""
    N = (128, 128, 128)
    p1, p2 = prep(229, N, seed=5), prep(229, N, seed=6)
    plan = make_plan(cf, p1, N, 4, max_batch=2)
    a, b = O.pack_stride(p1["u"], plan.L), O.pack_stride(p2["u"], plan.L)
    Fa = plan.forward(to_dev(a, 4))
    Fb = plan.forward(to_dev(b, 4))
    Fab = plan.forward(to_dev(2.0 * a - 0.5 * b, 4))
    assert rel_err((2.0 * Fa - 0.5 * Fb).cpu().numpy(), Fab.cpu().numpy()) < 1e-5
    batch = torch.stack([to_dev(a, 4), to_dev(b, 4)])
    back = plan.backward(plan.forward(batch))
    assert torch.max(torch.abs(back - batch)).item() / torch.max(torch.abs(batch)).item() < 1e-5
    plan.close()


NEW_GROUPS = [76, 78, 88, 92, 98, 110, 122, 130, 142, 144, 152, 161, 167, 169, 176, 178, 186, 193]


@pytest.mark.parametrize("precision", [8, 4])
@pytest.mark.parametrize("sg", NEW_GROUPS)
def test_tetragonal_trigonal_hexagonal_groups(cf, O, prep, sg, precision):
    # forward vs full-grid FFT and backward round trip for groups of every crystal
    # system beyond the orthorhombic and cubic ones (screw axes 4_1, 3_1, 6_1; R lattices)
    N = (12, 12, 12) if sg >= 143 else N16
    p = prep(sg, N)
    plan = make_plan(cf, p, N, precision)
    f0 = O.pack_stride(p["u"], plan.L)
    truth = O.spectrum_on_asu(p["u"], O.calc_spectral_asu(p["oops"], 3, N))
    F = plan.forward(to_dev(f0, precision))
    assert rel_err(F.cpu().numpy(), truth) < TOL[precision]
    assert rel_err(from_dev(plan.backward(F), plan.M), f0) < TOL[precision] * 10
    plan.close()


def test_step_diffusion_graph_replay(cf, O, prep):
    # cfft_step_diffusion runs loops of >= 4 steps as a captured CUDA graph: replays
    # (same buffer), a new buffer and a kernel update must match direct launches exactly
    import os

    p = prep(229, (32, 32, 32))
    plan = make_plan(cf, p, (32, 32, 32), 4, max_batch=3)
    g = torch.Generator(device="cuda:0").manual_seed(5)
    shape = (3,) + tuple(reversed(plan.M))
    q0 = torch.randn(shape, generator=g, device="cuda:0")
    w = 0.2 * torch.randn(shape, generator=g, device="cuda:0")

    def direct(q, n):
        for _ in range(n):
            plan.step_diffusion(q, w, 0.02, n_steps=1)  # one step: never a graph
        return q

    want = direct(q0.clone(), 6)
    a = q0.clone()
    plan.step_diffusion(a, w, 0.02, n_steps=6)        # captured + replayed
    assert torch.equal(a, want)
    a.copy_(q0)
    plan.step_diffusion(a, w, 0.02, n_steps=6)        # cache hit
    assert torch.equal(a, want)
    b = q0.clone()
    plan.step_diffusion(b, w, 0.02, n_steps=6)        # another buffer: another graph
    assert torch.equal(b, want)
    plan.update_kernel(0.07, LAT)                     # the graph reads the new kernel
    a.copy_(q0)
    plan.step_diffusion(a, w, 0.02, n_steps=6)
    os.environ["CFFT_STEP_GRAPH"] = "0"
    try:
        c = q0.clone()
        plan.step_diffusion(c, w, 0.02, n_steps=6)
    finally:
        del os.environ["CFFT_STEP_GRAPH"]
    assert torch.equal(a, c) and not torch.equal(a, want)
    plan.close()
