"""The trace surrogate on the GPU: the BF16 tensor-core GEMM against a float32
product of the same bf16 inputs, forward and backward passes against the CPU
oracle, and training on traces the engine generates, against the method
without the network (the mean trace of the training set)."""

import numpy as np
import pytest

import oracle.surrogate as O

pytestmark = pytest.mark.gpu


def _bf16(t):
    import torch

    return t.to(torch.bfloat16)


@pytest.mark.parametrize("entry", ["ifdtd_nn_gemm_tc", "ifdtd_nn_gemm"])
@pytest.mark.parametrize("m,n,k", [(70, 45, 37), (1, 130, 8), (300, 4, 520), (64, 64, 64), (257, 300, 200), (128, 128, 128)])
@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
def test_gemm_matches_float32_product_of_the_bf16_inputs(m, n, k, ta, tb, entry):
    """Both GEMMs (tcgen05.mma with the accumulator in tensor memory, and the
    warp-level mma.sync) against a float64 product of the same bf16 inputs:
    ragged shapes, several 128 x 128 tiles, K over many 64-wide chunks (the
    two-stage ring reused), all transposes, alpha and beta."""

    import torch

    from ionosphere_fdtd_b200 import _native as N

    g = torch.Generator(device="cuda").manual_seed(m * 7 + n + k)
    a = _bf16(torch.randn((k, m) if ta else (m, k), device="cuda", generator=g))
    b = _bf16(torch.randn((n, k) if tb else (k, n), device="cuda", generator=g))
    c0 = torch.randn((m, n), device="cuda", generator=g)
    c = c0.clone()
    stream = torch.cuda.current_stream().cuda_stream
    N.check(getattr(N.load(), entry)(m, n, k, a.data_ptr(), a.shape[1], ta, b.data_ptr(), b.shape[1], tb, 0.5, 2.0,
                                     c.data_ptr(), n, stream), entry)
    A = (a.float().T if ta else a.float()).double()
    B = (b.float().T if tb else b.float()).double()
    expected = 0.5 * (A @ B) + 2.0 * c0.double()
    err = (c.double() - expected).norm() / expected.norm()
    assert float(err) < 1e-6
    if entry == "ifdtd_nn_gemm_tc":
        status = N.C.c_int32(-1)
        N.check(N.load().ifdtd_nn_gemm_tc_status(1, N.C.byref(status)), "ifdtd_nn_gemm_tc_status")
        assert status.value == 0


@pytest.mark.parametrize("m,n,k", [(1024, 2048, 520), (4096, 512, 8), (1000, 1500, 96), (8192, 512, 512),
                                   (4096, 4096, 192), (5000, 2600, 136)])
def test_tma_fed_gemm_matches_float32_product(m, n, k):
    """K-major operands with enough output tiles take the TMA-fed kernel
    (persistent CTAs over 128 x 256 tiles, 2-D TMA loads with the 128-byte
    swizzle into a 4-stage ring, two TMEM accumulators so a tile's epilogue
    overlaps the next tile's MMAs, zero fill outside the matrices): ragged M
    and N, K below one chunk and K with a partial last chunk, one tile per CTA
    and several (512 and 440 tiles on 148 SMs), against a float64 product,
    twice (the same bits)."""

    import torch

    from ionosphere_fdtd_b200 import _native as N

    g = torch.Generator(device="cuda").manual_seed(m + n + k)
    a = _bf16(torch.randn((m, k), device="cuda", generator=g))
    b = _bf16(torch.randn((n, k), device="cuda", generator=g))
    c0 = torch.randn((m, n), device="cuda", generator=g)
    stream = torch.cuda.current_stream().cuda_stream
    outs = []
    for _ in range(2):
        c = c0.clone()
        N.check(N.load().ifdtd_nn_gemm_tc(m, n, k, a.data_ptr(), k, 0, b.data_ptr(), k, 1, 0.75, 0.5, c.data_ptr(), n, stream),
                "ifdtd_nn_gemm_tc")
        outs.append(c)
    expected = 0.75 * (a.double() @ b.double().T) + 0.5 * c0.double()
    assert float((outs[0].double() - expected).norm() / expected.norm()) < 1e-6
    assert torch.equal(outs[0], outs[1])
    status = N.C.c_int32(-1)
    N.check(N.load().ifdtd_nn_gemm_tc_status(1, N.C.byref(status)), "ifdtd_nn_gemm_tc_status")
    assert status.value == 0


@pytest.mark.parametrize("m,n,k,ta,tb", [(4, 16, 65536, 1, 0), (64, 200, 3000, 1, 0), (32, 4, 20000, 0, 1), (130, 70, 1024, 0, 0)])
def test_split_k_gemm_matches_float32_product_and_repeats_bitwise(m, n, k, ta, tb):
    """The tcgen05 GEMM with a workspace splits a long K over CTAs (the decoder's
    weight gradients have K = rows) and adds the partial tiles in split order:
    the product of the float64 reference to 1e-6, and the same bits on every run."""

    import torch

    from ionosphere_fdtd_b200 import _native as N

    g = torch.Generator(device="cuda").manual_seed(m + n + k)
    a = _bf16(torch.randn((k, m) if ta else (m, k), device="cuda", generator=g))
    b = _bf16(torch.randn((n, k) if tb else (k, n), device="cuda", generator=g))
    ws = torch.empty(4 << 20, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    outs = []
    for _ in range(2):
        c = torch.full((m, n), 3.0, device="cuda")
        N.check(N.load().ifdtd_nn_gemm_tc_ws(m, n, k, a.data_ptr(), a.shape[1], ta, b.data_ptr(), b.shape[1], tb, 0.5, -1.0,
                                             c.data_ptr(), n, ws.data_ptr(), ws.numel() * 4, stream), "ifdtd_nn_gemm_tc_ws")
        outs.append(c)
    A = (a.float().T if ta else a.float()).double()
    B = (b.float().T if tb else b.float()).double()
    expected = 0.5 * (A @ B) - 3.0
    assert float((outs[0].double() - expected).norm() / expected.norm()) < 1e-6
    assert torch.equal(outs[0], outs[1])


@pytest.mark.parametrize("gemm", ["tcgen05", "mma"])
def test_forward_and_backward_match_the_cpu_oracle(gemm):
    import torch

    from ionosphere_fdtd_b200.surrogate import TraceSurrogate, architecture

    layers = architecture(inputs=8, width=48, depth=3, samples=64, t0=4, c0=8, channels=(4, 1), stride=4)
    net = TraceSurrogate(layers, seed=5, gemm=gemm)
    rng = np.random.default_rng(1)
    x = rng.standard_normal((6, 8))
    t = rng.standard_normal((6, 64)) * 0.1
    pred = net.forward(torch.tensor(x, dtype=torch.bfloat16, device="cuda"))
    _, grad = net.loss_and_grad(pred, torch.tensor(t, dtype=torch.float32, device="cuda"))
    net.backward(grad)
    spec = [(L.fan_in, L.fan_out, L.act, L.expand) for L in layers]
    w = [p.double().cpu().numpy() for p in net.w]
    b = [p.double().cpu().numpy() for p in net.b]
    opred, acts = O.forward(spec, w, b, x)
    _, ograd = O.mse(opred, t)
    gw, gb = O.backward(spec, w, acts, ograd)
    rel = lambda a, e: float(np.linalg.norm(a - e) / max(np.linalg.norm(e), 1e-30))  # noqa: E731
    assert rel(pred.double().cpu().numpy(), opred) < 5e-3
    for i in range(len(layers)):
        assert rel(net.gw[i].double().cpu().numpy(), gw[i]) < 2e-2, i
        assert rel(net.gb[i].double().cpu().numpy(), gb[i]) < 2e-2, i


def test_training_on_engine_traces_beats_the_mean_trace():
    import torch

    from ionosphere_fdtd_b200.surrogate import TraceSurrogate, architecture, encode_features, generate_traces, relative_l2

    params, traces = generate_traces(48, subdivision=3, radial_cells=16, steps=256, receivers=8, distance_deg=(2.0, 10.0),
                                     batch_members=24, seed=7)
    assert traces.shape == (384, 256) and np.all(np.isfinite(traces))
    scale = float(np.sqrt(np.mean(traces**2)))
    assert scale > 0.0
    x = torch.tensor(encode_features(params), dtype=torch.bfloat16, device="cuda")
    y = torch.tensor(traces / scale, dtype=torch.float32, device="cuda")
    train, test = slice(0, 288), slice(288, 384)  # whole runs held out
    net = TraceSurrogate(architecture(inputs=8, width=64, depth=3, samples=256, t0=16, c0=16, channels=(8, 1), stride=4), seed=1)
    losses = net.fit(x[train], y[train], iterations=1500, batch=64, lr=3e-3, lr_final=2e-4, seed=3)
    assert np.mean(losses[-50:]) < 0.5 * np.mean(losses[:10])
    pred = net.predict(x[test])
    mean_trace = y[train].mean(dim=0, keepdim=True).expand_as(y[test])
    keep = y[test].norm(dim=1) > 1e-3 * y[test].norm(dim=1).max()
    err_net = float(relative_l2(pred, y[test])[keep].median())
    err_mean = float(relative_l2(mean_trace, y[test])[keep].median())
    assert err_net < err_mean, (err_net, err_mean)


def test_weighted_squared_error_matches_a_float64_reference():
    import torch

    from ionosphere_fdtd_b200.surrogate import TraceSurrogate, architecture

    net = TraceSurrogate(architecture(inputs=8, width=16, depth=1, samples=16, t0=1, c0=4, channels=(4, 1), stride=4))
    g = torch.Generator(device="cuda").manual_seed(4)
    p = torch.randn((37, 53), device="cuda", generator=g)
    t = torch.randn((37, 53), device="cuda", generator=g)
    w = torch.rand(37, device="cuda", generator=g) + 0.5
    loss, grad = net.weighted_loss_and_grad(p, t, w)
    d = (p - t).double()
    expected = float((w.double()[:, None] * d * d).sum() / d.numel())
    assert float(loss) == pytest.approx(expected, rel=1e-5)
    torch.testing.assert_close(grad.double(), 2.0 * w.double()[:, None] * d / d.numel(), rtol=1e-6, atol=1e-9)


def test_training_data_does_not_depend_on_the_builder_threads():
    """generate_traces draws every member's parameters in order from one seeded
    generator and only then builds the members on host threads: one thread and
    four give the same parameters and the same traces, bit for bit."""

    from ionosphere_fdtd_b200.surrogate import generate_traces

    kw = dict(subdivision=3, radial_cells=12, steps=64, receivers=4, distance_deg=(2.0, 10.0), batch_members=6, seed=21)
    p1, t1 = generate_traces(9, workers=1, **kw)
    p4, t4 = generate_traces(9, workers=4, **kw)
    np.testing.assert_array_equal(p1, p4)
    np.testing.assert_array_equal(t1, t4)
    assert t1.shape == (36, 64) and np.abs(t1).max() > 0.0

