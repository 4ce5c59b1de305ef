"""The learned warm start's network on the device against the oracle (oracle/nn_oracle.py): every kernel on
BF16-rounded inputs, the whole forward and backward pass of the training wrapper, the C-ABI inference inside the CG
solve against the training forward pass, and what a trained network gains over the previous-step warm start."""
import ctypes as C

import numpy as np
import pytest

import nn_oracle as O
from edipic_b200 import (FIELD_PHI, FIELD_RHO_TOTAL, PRECOND_MG, PRECOND_NONE, WARM_LEARNED, WARM_PREVIOUS,
                         WARM_USER, Simulation, decks, library, warmstart)

torch = pytest.importorskip("torch")


def _bf(a):
    return torch.tensor(np.asarray(a, dtype=np.float32), device="cuda").to(torch.bfloat16)


def _f32(a):
    return torch.tensor(np.asarray(a, dtype=np.float32), device="cuda")


def _np(t):
    return t.detach().float().cpu().numpy().astype(np.float64)


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-30)


@pytest.mark.gpu
@pytest.mark.parametrize("c1,c2,cout", [(32, 0, 32), (64, 0, 128), (256, 128, 128), (64, 32, 32), (128, 0, 96),
                                        (128, 0, 256), (64, 128, 64)])
@pytest.mark.parametrize("n,h,w", [(2, 16, 24), (1, 13, 21)])
def test_conv_kernels_match_oracle(c1, c2, cout, n, h, w):
    """Forward (tcgen05 tensor cores, one CTA per 128 pixels and all output channels), data gradient through the
    same kernel on the flipped weights, weight and bias gradients; pixel counts that do and do not fill the last
    128-pixel tile."""
    lib = library()
    rng = np.random.default_rng(c1 + c2 + cout + h)
    x1 = O.bf16(rng.normal(0, 1, (n, h, w, c1)))
    x2 = O.bf16(rng.normal(0, 1, (n, h, w, c2))) if c2 else None
    cin = c1 + c2
    wt = O.bf16(rng.normal(0, 1.0 / np.sqrt(9 * cin), (cout, 9, cin)))
    b = rng.normal(0, 0.1, cout).astype(np.float32).astype(np.float64)
    xin = x1 if c2 == 0 else np.concatenate([x1, x2], axis=-1)
    tx1, tx2, tw, tb = _bf(x1), (_bf(x2) if c2 else None), _bf(wt), _f32(b)
    y = torch.empty((n, h, w, cout), device="cuda", dtype=torch.bfloat16)
    for relu in (0, 1):
        assert lib.edp_nn_conv3x3_fwd(n, h, w, _p(tx1), c1, _p(tx2), c2, _p(tw), _p(tb), cout, relu, _p(y),
                                      _stream()) == 0
        ref = O.conv_fwd(xin, wt, b, relu=bool(relu))
        assert _rel(_np(y), ref) < 8e-3   # BF16 output rounding
    # data gradient: the forward kernel on the flipped, transposed weights
    dz = O.bf16(rng.normal(0, 1, (n, h, w, cout)))
    tdz = _bf(dz)
    wtt = torch.empty((cin, 9, cout), device="cuda", dtype=torch.bfloat16)
    assert lib.edp_nn_flip_transpose(_p(tw), cout, cin, _p(wtt), _stream()) == 0
    dx = torch.empty((n, h, w, cin), device="cuda", dtype=torch.bfloat16)
    assert lib.edp_nn_conv3x3_fwd(n, h, w, _p(tdz), cout, None, 0, _p(wtt), None, cin, 0, _p(dx), _stream()) == 0
    assert _rel(_np(dx), O.conv_dgrad(dz, wt)) < 8e-3
    # weight and bias gradients (FP32, accumulated)
    dw = torch.zeros((cout, 9, cin), device="cuda", dtype=torch.float32)
    db = torch.zeros(cout, device="cuda", dtype=torch.float32)
    assert lib.edp_nn_conv3x3_wgrad(n, h, w, _p(tx1), c1, _p(tx2), c2, _p(tdz), cout, _p(dw), _p(db), _stream()) == 0
    rw, rb = O.conv_wgrad(xin, dz)
    assert _rel(_np(dw), rw) < 1e-5 and _rel(_np(db), rb) < 1e-5
    flag = C.c_int32(-1)
    assert lib.edp_nn_error(C.byref(flag)) == 0 and flag.value == 0


@pytest.mark.gpu
@pytest.mark.parametrize("c1,c2,cout", [(32, 0, 32), (64, 32, 32), (32, 0, 64), (64, 0, 64), (32, 0, 128),
                                        (128, 64, 64), (256, 0, 32)])
@pytest.mark.parametrize("n,h,w", [(1, 23, 13), (2, 40, 36), (3, 150, 97)])
def test_halo_conv_matches_oracle(c1, c2, cout, n, h, w):
    """The persistent halo kernel (edp_nn_conv_select(2): 8 x 16-pixel patches, one 10 x 18 halo per 32-channel
    chunk for all nine taps, weights resident or, above 112 KiB, streamed with each chunk, two tensor-memory
    accumulators) against the oracle, on images that do not fill their last patch, concatenated inputs, and more
    patches than CTAs (each CTA takes several); then the tile kernel gives the same output within the BF16 rounding
    of both."""
    lib = library()
    rng = np.random.default_rng(7 * c1 + c2 + cout + h)
    x1 = O.bf16(rng.normal(0, 1, (n, h, w, c1)))
    x2 = O.bf16(rng.normal(0, 1, (n, h, w, c2))) if c2 else None
    cin = c1 + c2
    wt = O.bf16(rng.normal(0, 1.0 / np.sqrt(9 * cin), (cout, 9, cin)))
    b = rng.normal(0, 0.1, cout).astype(np.float32).astype(np.float64)
    xin = x1 if c2 == 0 else np.concatenate([x1, x2], axis=-1)
    tx1, tx2, tw, tb = _bf(x1), (_bf(x2) if c2 else None), _bf(wt), _f32(b)
    y = torch.full((n, h, w, cout), 7.0, device="cuda", dtype=torch.bfloat16)
    try:
        assert lib.edp_nn_conv_select(2) == 0
        for relu in (0, 1):
            assert lib.edp_nn_conv3x3_fwd(n, h, w, _p(tx1), c1, _p(tx2), c2, _p(tw), _p(tb), cout, relu, _p(y),
                                          _stream()) == 0
            ref = O.conv_fwd(xin, wt, b, relu=bool(relu))
            assert _rel(_np(y), ref) < 8e-3   # BF16 output rounding
        flag = C.c_int32(-1)
        assert lib.edp_nn_error(C.byref(flag)) == 0 and flag.value == 0
        y1 = torch.empty_like(y)
        assert lib.edp_nn_conv_select(1) == 0
        assert lib.edp_nn_conv3x3_fwd(n, h, w, _p(tx1), c1, _p(tx2), c2, _p(tw), _p(tb), cout, 1, _p(y1),
                                      _stream()) == 0
        assert _rel(_np(y1), _np(y)) < 8e-3
    finally:
        lib.edp_nn_conv_select(0)
    # a layer whose weights do not fit is refused when the halo kernel is forced
    assert lib.edp_nn_conv_select(2) == 0
    try:
        big = torch.empty((256, 9, 256), device="cuda", dtype=torch.bfloat16)
        assert lib.edp_nn_conv3x3_fwd(n, h, w, _p(tx1), 256, None, 0, _p(big), None, 128, 0, _p(y), _stream()) != 0
    finally:
        lib.edp_nn_conv_select(0)


@pytest.mark.gpu
@pytest.mark.parametrize("c1,c2,cout", [(32, 0, 32), (64, 32, 32), (32, 0, 64), (128, 64, 128), (64, 0, 96),
                                        (32, 0, 256)])
@pytest.mark.parametrize("n,h,w", [(1, 9, 9), (3, 150, 97)])
def test_wgrad_kernels_match_oracle(c1, c2, cout, n, h, w):
    """The weight gradient on tcgen05 with the taps in M (edp_nn_wgrad_select(0): four shifted copies of the x patch
    per M = 128 MMA, tap 8 in an M = 64 one, K = the pixels of 8 x 16 patches), on tcgen05 with the taps in N
    (select 2: the nine taps' accumulators in tensor memory, M = output channels) and on mma.sync (select 1), against
    the oracle, accumulated onto a nonzero dw, with more patches than CTAs."""
    lib = library()
    rng = np.random.default_rng(5 * c1 + c2 + cout + h)
    x1 = O.bf16(rng.normal(0, 1, (n, h, w, c1)))
    x2 = O.bf16(rng.normal(0, 1, (n, h, w, c2))) if c2 else None
    cin = c1 + c2
    xin = x1 if c2 == 0 else np.concatenate([x1, x2], axis=-1)
    dz = O.bf16(rng.normal(0, 1, (n, h, w, cout)))
    tx1, tx2, tdz = _bf(x1), (_bf(x2) if c2 else None), _bf(dz)
    w0 = rng.normal(0, 1, (cout, 9, cin)).astype(np.float32)
    rw, rb = O.conv_wgrad(xin, dz)
    try:
        for mode in (0, 1, 2):
            assert lib.edp_nn_wgrad_select(mode) == 0
            dw = _f32(w0)
            db = torch.zeros(cout, device="cuda", dtype=torch.float32)
            assert lib.edp_nn_conv3x3_wgrad(n, h, w, _p(tx1), c1, _p(tx2), c2, _p(tdz), cout, _p(dw), _p(db),
                                            _stream()) == 0
            assert _rel(_np(dw) - w0, rw) < 1e-5, mode
            assert _rel(_np(db), rb) < 1e-5
    finally:
        lib.edp_nn_wgrad_select(0)
    flag = C.c_int32(-1)
    assert lib.edp_nn_error(C.byref(flag)) == 0 and flag.value == 0


@pytest.mark.gpu
def test_glue_kernels_match_oracle():
    lib = library()
    rng = np.random.default_rng(5)
    n, h, w, c = 2, 16, 24, 64
    x = O.bf16(rng.normal(0, 1, (n, h, w, c)))
    tx = _bf(x)
    for f in (2, 4):
        y = torch.empty((n, h // f, w // f, c), device="cuda", dtype=torch.bfloat16)
        assert lib.edp_nn_pool(n, h, w, c, f, _p(tx), _p(y), _stream()) == 0
        assert _rel(_np(y), O.pool(x, f)) < 5e-3
        dy = O.bf16(rng.normal(0, 1, (n, h // f, w // f, c)))
        dx = torch.empty((n, h, w, c), device="cuda", dtype=torch.bfloat16)
        assert lib.edp_nn_pool_bwd(n, h, w, c, f, _p(_bf(dy)), _p(dx), 0, _stream()) == 0
        assert _rel(_np(dx), O.pool_bwd(dy, f)) < 5e-3
        u = torch.empty((n, f * h, f * w, c), device="cuda", dtype=torch.bfloat16)
        assert lib.edp_nn_upsample(n, f * h, f * w, c, f, _p(tx), _p(u), _stream()) == 0
        assert np.array_equal(_np(u), O.up(x, f))
        du = O.bf16(rng.normal(0, 1, (n, f * h, f * w, c)))
        dxu = torch.empty((n, h, w, c), device="cuda", dtype=torch.bfloat16)
        assert lib.edp_nn_upsample_bwd(n, f * h, f * w, c, c, f, _p(_bf(du)), _p(dxu), _stream()) == 0
        assert _rel(_np(dxu), O.up_bwd(du, f)) < 5e-3
    yy = O.bf16(rng.normal(0, 1, (n, h, w, c)))
    dz = torch.empty((n, h, w, c), device="cuda", dtype=torch.bfloat16)
    assert lib.edp_nn_relu_bwd(n * h * w, c, _p(tx), c, 0, None, _p(_bf(yy)), _p(dz), _stream()) == 0
    assert np.array_equal(_np(dz), np.where(yy > 0, x, 0.0))
    # head (32 channels to one FP32 output)
    xh = O.bf16(rng.normal(0, 1, (n, h, w, 32)))
    wh = rng.normal(0, 0.1, 9 * 32).astype(np.float32).astype(np.float64)
    bh = np.array([0.25], dtype=np.float32)
    out = torch.empty((n, h, w), device="cuda", dtype=torch.float32)
    twh, tbh = _f32(wh), _f32(bh)
    assert lib.edp_nn_head_fwd(n, h, w, 32, _p(_bf(xh)), _p(twh), _p(tbh), _p(out), _stream()) == 0
    assert _rel(_np(out), O.head_fwd(xh, wh, 0.25)) < 1e-5
    dout = rng.normal(0, 1, (n, h, w)).astype(np.float32).astype(np.float64)
    dxh = torch.empty((n, h, w, 32), device="cuda", dtype=torch.bfloat16)
    dwh = torch.zeros(9 * 32, device="cuda", dtype=torch.float32)
    dbh = torch.zeros(1, device="cuda", dtype=torch.float32)
    assert lib.edp_nn_head_bwd(n, h, w, 32, _p(_bf(xh)), _p(twh), _p(_f32(dout)), _p(dxh), _p(dwh), _p(dbh),
                               _stream()) == 0
    rdx, rdw, rdb = O.head_bwd(xh, wh, dout)
    assert _rel(_np(dxh), rdx) < 5e-3 and _rel(_np(dwh), rdw) < 1e-5 and abs(float(dbh[0]) - rdb) < 1e-4 * abs(rdb) + 1e-4


@pytest.mark.gpu
def test_network_gradient_matches_oracle():
    """Forward and backward of the training wrapper (torch.autograd.Function over the device kernels) against the
    oracle on the same parameters and input. BF16 storage of activations and data gradients makes any two
    evaluations differ; the device's distance from the exact FP64 pass must stay within twice the distance of the
    oracle's own BF16-emulating pass from it, for the output, the whole gradient and every layer."""
    rng = np.random.default_rng(7)
    theta = warmstart.init_params(seed=3)
    heads0 = warmstart.param_layout()[1][0][0]
    theta[heads0:] *= 10.0   # livelier heads than at initialisation
    x = O.bf16(rng.normal(0, 1, (1, 64, 128, 32)))
    net = warmstart.WarmStartNet(theta)
    out = net.forward(_bf(x))
    dout = [rng.normal(0, 1, tuple(o.shape)) for o in out]
    sum((o * _f32(d)).sum() for o, d in zip(out, dout)).backward()
    g = _np(net.theta.grad)
    t64 = theta.astype(np.float64)
    rout_q, tape_q = O.net_forward(t64, x, quantize=True)
    rg_q = O.net_backward(t64, tape_q, dout)
    rout, tape = O.net_forward(t64, x, quantize=False)
    rg = O.net_backward(t64, tape, dout)
    for o, rq, r in zip(out, rout_q, rout):
        assert np.linalg.norm(_np(o) - r) <= 2.0 * np.linalg.norm(rq - r) + 1e-6 * np.linalg.norm(r)
    assert np.linalg.norm(g - rg) <= 2.0 * np.linalg.norm(rg_q - rg) + 1e-6 * np.linalg.norm(rg)
    cos = float(np.dot(g, rg) / (np.linalg.norm(g) * np.linalg.norm(rg)))
    assert cos > 0.99
    convs, heads, _ = warmstart.param_layout()
    for (wo, bo, ci, co) in convs + [(wh, bh, 32, 1) for (wh, bh) in heads]:
        err, noise = np.linalg.norm(g[wo:bo] - rg[wo:bo]), np.linalg.norm(rg_q[wo:bo] - rg[wo:bo])
        assert err <= 2.0 * noise + 1e-4 * np.linalg.norm(rg[wo:bo]) + 1e-9


def _input_from_fields(rho_t, phi, unk, K):
    """The network input and s of the library's inference, rebuilt on the host from rho_total and phi."""
    ny, nx = phi.shape
    H, W = warmstart.padded(ny), warmstart.padded(nx)
    p = np.pad(phi, 1)
    r0 = (rho_t - 4.0 * phi + p[1:-1, :-2] + p[1:-1, 2:] + p[:-2, 1:-1] + p[2:, 1:-1]) * unk
    s = np.sqrt((r0 ** 2).sum() / unk.sum())
    x = np.zeros((1, H, W, 32))
    x[0, :ny, :nx, 0] = r0 / s
    m = np.ones((H, W))
    m[:ny, :nx] = 1.0 - unk
    x[0, :, :, 1] = m
    return x, s


def _unknowns(p):
    ny, nx = p.ncy + 1, p.ncx + 1
    unk = np.zeros((ny, nx))
    unk[1:-1, 1:-1] = 1.0
    for o in range(p.n_inner):
        unk[p.inner_jbottom[o]:p.inner_jtop[o] + 1, p.inner_ileft[o]:p.inner_iright[o] + 1] = 0.0
    return unk


@pytest.mark.gpu
def test_library_inference_matches_training_forward(tmp_path):
    d = decks.write_deck(str(tmp_path), "cfg2", ncx=64, ncy=48, ppc=16, inner=(20, 12, 36, 20, -100.0))
    theta = warmstart.init_params(seed=11)
    theta[warmstart.param_layout()[1][0][0]:] *= 10.0
    with Simulation(d, sort_every=20) as sim:
        p = sim.params
        sim.distribute_particles(16)
        sim.solve_potential_with_cg(rtol=1e-10)
        for _ in range(2):
            sim.advance_electrons()
            sim.advance_ions()
            sim.end_ion_cycle()
        sim.load_warm_start(theta)
        guess, res = sim.predict_warm_start()
        phi = sim.field(FIELD_PHI)
        rho_t = sim.field(FIELD_RHO_TOTAL)
    unk = _unknowns(p)
    K = warmstart.k_factor(p.ncx, p.ncy)
    x, s = _input_from_fields(rho_t, phi, unk, K)
    net = warmstart.WarmStartNet(theta)
    with torch.no_grad():
        o0, o1 = (_np(o)[0] for o in net.forward(_bf(x)))
    ny, nx = phi.shape
    upd = s * (K * o0[:ny, :nx] + o1[:ny, :nx]) * unk
    assert np.abs(guess - phi - upd).max() <= 2e-2 * np.abs(upd).max()
    assert np.allclose(guess[unk == 0], phi[unk == 0])
    assert res[0] > 0 and np.isfinite(res[1])


@pytest.mark.gpu
def test_trained_warm_start_reduces_cg_work(tmp_path):
    """Trained on the potential updates of short plain runs of one geometry family, the network's start has a
    smaller residual than the previous potential on a held-out run, and CG needs fewer iterations from it."""
    dirs = []
    geo = [(20, 20, 36, 28, -100.0), (26, 30, 42, 38, -150.0), (16, 34, 32, 42, -60.0), (24, 22, 40, 30, -120.0)]
    for k, g in enumerate(geo):
        dirs.append(decks.write_deck(str(tmp_path / f"d{k}"), "cfg2", ncx=64, ncy=64, ppc=16, inner=g, seed=k))
    torch.manual_seed(0)
    dphi, unk = warmstart.generate_samples(dirs[:3], steps_per_deck=24, warmup=4)
    K = warmstart.k_factor(64, 64)
    net = warmstart.WarmStartNet(seed=0)
    hist = warmstart.train(net, dphi, unk, K, steps=400, batch=8, lr=1e-3)
    theta = net.blob()
    its = {}
    ratios = []
    for mode in (WARM_PREVIOUS, WARM_LEARNED):
        for pc in (PRECOND_NONE, PRECOND_MG):
            with Simulation(dirs[3], sort_every=20, seed=5) as sim:
                sim.set_cg_preconditioner(pc)
                sim.load_warm_start(theta)
                sim.distribute_particles(16)
                n = []
                for k in range(16):
                    if mode == WARM_LEARNED:
                        # the network's own start (used when its residual is smaller), whatever its wall time
                        guess, res = sim.predict_warm_start()
                        if pc == PRECOND_NONE and k >= 4:
                            ratios.append(res[1] / res[0])
                        if res[1] < res[0]:
                            sim.set_field(FIELD_PHI, guess)
                    it = sim.solve_potential_with_cg(rtol=1e-8, max_it=100000,
                                                     warm_start=WARM_USER if mode == WARM_LEARNED else mode)
                    if k >= 4:
                        n.append(it)
                    sim.advance_electrons()
                    sim.advance_ions()
                    sim.perform_electron_neutral_collisions()
                    sim.perform_resonant_charge_exchange()
                    sim.end_ion_cycle()
                its[(mode, pc)] = float(np.mean(n))
    print("train history", hist[-1:] if hist else None, "iterations", its, "residual ratio", np.mean(ratios))
    assert np.mean(ratios) < 0.5
    assert its[(WARM_LEARNED, PRECOND_NONE)] < its[(WARM_PREVIOUS, PRECOND_NONE)]
    assert its[(WARM_LEARNED, PRECOND_MG)] <= its[(WARM_PREVIOUS, PRECOND_MG)] + 0.5


@pytest.mark.gpu
def test_learned_start_is_judged_by_wall_time(tmp_path):
    """EDP_WARM_LEARNED with a network that predicts no update (its guess never has the smaller residual): the first
    two calls run the network, the third starts from the previous potential; the network's solves are then the
    slower ones, so over 70 calls it runs again only on the 64th (to re-measure), and every solve converges."""
    d = decks.write_deck(str(tmp_path), "cfg2", ncx=64, ncy=64, ppc=16, inner=(20, 20, 36, 28, -100.0))
    theta = warmstart.init_params(seed=3)
    theta[warmstart.param_layout()[1][0][0]:] = 0.0   # both heads zero: the update is 0
    with Simulation(d, sort_every=20, seed=2) as sim:
        sim.load_warm_start(theta)
        sim.distribute_particles(16)
        import ctypes as C
        for _ in range(70):
            assert sim.solve_potential_with_cg(rtol=1e-8, max_it=100000, warm_start=WARM_LEARNED) > 0
            sim.advance_electrons()
            sim.advance_ions()
            sim.end_ion_cycle()
        out = np.zeros(4)
        sim._check(sim.lib.edp_warmstart_timing(sim.ctx, out.ctypes.data_as(C.POINTER(C.c_double))), "timing")
    t_net, t_prev, calls, runs = out
    assert calls == 70 and 0 < t_prev < t_net
    assert runs == 3   # calls 0, 1 and 64
