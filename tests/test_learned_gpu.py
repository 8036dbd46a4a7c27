"""GPU checks of the BF16 tensor-core convolutions (pmhd_conv3x3,
pmhd_conv3x3_wgrad) and the training loss (pmhd_learned_loss_grad) against
the float64 network oracle, and of the trained correction.

Two kinds of case per kernel: small-integer data, for which every product
and partial sum is exact in the kernels' fp32 accumulators, so the results
must equal the oracle's exactly (any operand-layout mistake shows as a wrong
value, not a small error); and Gaussian data at sizes with partial tiles,
within the tolerances of bf16 outputs (8 significant bits) and fp32
accumulation.
"""
import ctypes
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import cnn_oracle as C  # noqa: E402

pytestmark = pytest.mark.gpu


def _dev_bf16(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16).cuda()


def _dev_f32(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def _host(t):
    import torch
    return t.float().cpu().numpy().astype(np.float64)


def _conv(pmhd, mode, x, W, b, c_out, zprev=None):
    import torch
    B, H, Wd, cin = x.shape
    xd, wd = _dev_bf16(x), _dev_bf16(W)
    bd = _dev_f32(b) if b is not None else None
    P = B * H * Wd
    if mode == pmhd.CONV_GELU:
        o0 = torch.empty((B, H, Wd, c_out), dtype=torch.bfloat16, device="cuda")
        o1 = torch.empty_like(o0)
    elif mode == pmhd.CONV_LINEAR:
        o0 = torch.empty((B, H, Wd, c_out), dtype=torch.float32, device="cuda")
        o1 = None
    else:
        o0 = torch.empty((B, H, Wd, c_out), dtype=torch.bfloat16, device="cuda")
        o1 = None
    zd = _dev_bf16(zprev) if zprev is not None else None
    rc = pmhd.load().pmhd_conv3x3(mode, xd.data_ptr(), B, H, Wd, cin, wd.data_ptr(),
                                  ctypes.cast(bd.data_ptr(), ctypes.POINTER(ctypes.c_float)) if bd is not None else None,
                                  c_out, zd.data_ptr() if zd is not None else None, o0.data_ptr(),
                                  o1.data_ptr() if o1 is not None else None, None)
    assert rc == pmhd.OK, pmhd.strerror(rc)
    return _host(o0), (_host(o1) if o1 is not None else None)


def _wgrad(pmhd, x, dz):
    import torch
    B, H, Wd, cin = x.shape
    co = dz.shape[3]
    dw = torch.zeros((co, 9, cin), dtype=torch.float32, device="cuda")
    db = torch.zeros((co,), dtype=torch.float32, device="cuda")
    fp = ctypes.POINTER(ctypes.c_float)
    xd, dzd = _dev_bf16(x), _dev_bf16(dz)  # kept alive across the call
    rc = pmhd.load().pmhd_conv3x3_wgrad(xd.data_ptr(), dzd.data_ptr(), B, H, Wd, cin, co,
                                        ctypes.cast(dw.data_ptr(), fp), ctypes.cast(db.data_ptr(), fp), None)
    assert rc == pmhd.OK, pmhd.strerror(rc)
    return _host(dw), _host(db)


def _ints(rng, shape, p_nonzero=1.0):
    v = rng.integers(-1, 2, size=shape).astype(np.float64)
    if p_nonzero < 1.0:
        v *= rng.random(shape) < p_nonzero
    return v


def _bf(a):
    return C.bf16_round(a).astype(np.float64)


# The last two shapes take the row kernel (width a multiple of 128, height
# of 8), the others the gather kernel.
SHAPES = [(1, 8, 16), (2, 9, 20), (1, 64, 64), (3, 17, 33), (1, 8, 128), (2, 16, 256)]


@pytest.mark.parametrize("shape", SHAPES)
def test_forward_gelu_exact_on_integers(pmhd_lib, shape):
    rng = np.random.default_rng(10)
    x = _ints(rng, shape + (32,))
    W = _ints(rng, (32, 9, 32), 0.2)
    b = rng.integers(-3, 4, 32).astype(np.float64)
    z, a = _conv(pmhd_lib, pmhd_lib.CONV_GELU, x, W, b, 32)
    zr = C.conv3x3(x, W, b)
    np.testing.assert_array_equal(z, zr)
    # gelu is evaluated in fp32 on the device: allow one bf16 ulp.
    np.testing.assert_allclose(a, _bf(C.gelu(zr)), rtol=2.0 ** -7, atol=1e-30)


@pytest.mark.parametrize("shape", SHAPES)
def test_forward_linear_exact_on_integers(pmhd_lib, shape):
    rng = np.random.default_rng(11)
    x = _ints(rng, shape + (32,))
    W = _ints(rng, (16, 9, 32))
    b = rng.integers(-3, 4, 16).astype(np.float64)
    out, _ = _conv(pmhd_lib, pmhd_lib.CONV_LINEAR, x, W, b, 16)
    np.testing.assert_array_equal(out, C.conv3x3(x, W, b))


@pytest.mark.parametrize("cin", [16, 32])
@pytest.mark.parametrize("shape", SHAPES[:3] + SHAPES[4:])
def test_backward_input_exact_on_integers(pmhd_lib, shape, cin):
    """x = the layer's output gradient (cin channels), W the layer weight
    [cin][9][32]; the kernel takes W transposed to [32][9][cin]."""
    rng = np.random.default_rng(12)
    dz = _ints(rng, shape + (cin,))
    W = _ints(rng, (cin, 9, 32), 0.3)
    zprev = _bf(rng.normal(0, 1.0, shape + (32,)))
    Wt = np.ascontiguousarray(W.transpose(2, 1, 0))
    out, _ = _conv(pmhd_lib, pmhd_lib.CONV_DGELU, dz, Wt, None, 32, zprev=zprev)
    da = C.conv3x3_backward_input(dz, W)  # exact integers
    ref = C.bf16_round((da * C.gelu_grad(zprev)).astype(np.float32)).astype(np.float64)
    # gelu' is evaluated in fp32 on the device: allow one bf16 ulp.
    np.testing.assert_allclose(out, ref, rtol=2.0 ** -7, atol=0)
    np.testing.assert_array_equal(out == 0, ref == 0)


@pytest.mark.parametrize("variant", ["gelu", "linear", "dgelu16", "dgelu32"])
def test_pipelined_row_kernel_matches_the_per_tile_row_kernel(pmhd_lib, monkeypatch, variant):
    """The persistent, pipelined row kernel (selected for large batches; here
    forced by its test hook with 2 CTAs, so each CTA runs 8 tiles through
    both staging and accumulator buffers) gives the per-tile row kernel's
    results bit for bit (same MMA sequence per row), and both equal the
    oracle on integer data."""
    rng = np.random.default_rng(15)
    shape = (4, 16, 256)
    if variant == "gelu":
        x, W, b, cout, zp, mode = _ints(rng, shape + (32,)), _ints(rng, (32, 9, 32), 0.2), \
            rng.integers(-3, 4, 32).astype(np.float64), 32, None, pmhd_lib.CONV_GELU
    elif variant == "linear":
        x, W, b, cout, zp, mode = _ints(rng, shape + (32,)), _ints(rng, (16, 9, 32)), \
            rng.integers(-3, 4, 16).astype(np.float64), 16, None, pmhd_lib.CONV_LINEAR
    else:
        cin = 16 if variant == "dgelu16" else 32
        x = _ints(rng, shape + (cin,))
        W = np.ascontiguousarray(_ints(rng, (cin, 9, 32), 0.3).transpose(2, 1, 0))
        b, cout, mode = None, 32, pmhd_lib.CONV_DGELU
        zp = _bf(rng.normal(0, 1.0, shape + (32,)))
    monkeypatch.delenv("PMHD_CONV_MAX_CTAS", raising=False)
    o0, o1 = _conv(pmhd_lib, mode, x, W, b, cout, zprev=zp)
    monkeypatch.setenv("PMHD_CONV_MAX_CTAS", "2")
    p0, p1 = _conv(pmhd_lib, mode, x, W, b, cout, zprev=zp)
    np.testing.assert_array_equal(p0, o0)
    if o1 is not None:
        np.testing.assert_array_equal(p1, o1)
    if variant in ("gelu", "linear"):
        np.testing.assert_array_equal(p0, C.conv3x3(x, W, b))


@pytest.mark.parametrize("cout", [32, 16])
@pytest.mark.parametrize("shape", SHAPES)
def test_weight_gradient_exact_on_integers(pmhd_lib, shape, cout):
    rng = np.random.default_rng(13)
    x = _ints(rng, shape + (32,))
    dz = _ints(rng, shape + (cout,))
    dw, db = _wgrad(pmhd_lib, x, dz)
    dwr, dbr = C.conv3x3_backward_weight(x, dz)
    np.testing.assert_array_equal(dw, dwr)
    np.testing.assert_array_equal(db, dbr)


def test_gaussian_layers_within_bf16_tolerance(pmhd_lib):
    rng = np.random.default_rng(14)
    shape = (2, 33, 47)
    x = _bf(rng.normal(0, 1, shape + (32,)))
    W1 = _bf(rng.normal(0, 0.08, (32, 9, 32)))
    b1 = rng.normal(0, 0.1, 32).astype(np.float32).astype(np.float64)
    z, a = _conv(pmhd_lib, pmhd_lib.CONV_GELU, x, W1, b1, 32)
    zr = C.conv3x3(x, W1, b1)
    scale = np.abs(zr).max()
    np.testing.assert_allclose(z, zr, rtol=2.0 ** -8, atol=1e-5 * scale)
    np.testing.assert_allclose(a, C.gelu(zr), rtol=2.0 ** -7, atol=1e-5 * scale)
    W3 = _bf(rng.normal(0, 0.08, (16, 9, 32)))
    b3 = rng.normal(0, 0.1, 16).astype(np.float32).astype(np.float64)
    out, _ = _conv(pmhd_lib, pmhd_lib.CONV_LINEAR, a, W3, b3, 16)
    outr = C.conv3x3(a, W3, b3)
    np.testing.assert_allclose(out, outr, rtol=1e-5, atol=1e-5 * np.abs(outr).max())
    dz = _bf(rng.normal(0, 1e-3, shape + (16,)))
    dw, db = _wgrad(pmhd_lib, a, dz)
    dwr, dbr = C.conv3x3_backward_weight(a, dz)
    np.testing.assert_allclose(dw, dwr, rtol=1e-4, atol=1e-4 * np.abs(dwr).max())
    np.testing.assert_allclose(db, dbr, rtol=1e-4, atol=1e-4 * np.abs(dbr).max())


def test_unsupported_channel_counts_are_rejected(pmhd_lib):
    import torch
    x = torch.zeros((1, 8, 8, 24), dtype=torch.bfloat16, device="cuda")
    w = torch.zeros((24, 9, 24), dtype=torch.bfloat16, device="cuda")
    b = torch.zeros((24,), dtype=torch.float32, device="cuda")
    o = torch.zeros((1, 8, 8, 24), dtype=torch.bfloat16, device="cuda")
    rc = pmhd_lib.load().pmhd_conv3x3(pmhd_lib.CONV_GELU, x.data_ptr(), 1, 8, 8, 24, w.data_ptr(),
                                      ctypes.cast(b.data_ptr(), ctypes.POINTER(ctypes.c_float)), 24, None,
                                      o.data_ptr(), o.data_ptr(), None)
    assert rc == pmhd_lib.ERR_UNSUPPORTED


def _loss_grad(pmhd, out, tgt, cx, cy):
    import torch
    B, H, Wd, _ = out.shape
    od, td = _dev_f32(out), _dev_f32(tgt)
    dz = torch.zeros((B, H, Wd, 16), dtype=torch.bfloat16, device="cuda")
    loss = ctypes.c_double()
    rc = pmhd.load().pmhd_learned_loss_grad(od.data_ptr(), td.data_ptr(), B, H, Wd, cx, cy, dz.data_ptr(),
                                            ctypes.byref(loss), None)
    assert rc == pmhd.OK, pmhd.strerror(rc)
    return loss.value, _host(dz)


def test_loss_kernel_matches_oracle(pmhd_lib):
    """The training loss and its gradient (direct channels and the field
    through the curl of the potential channel, periodic) against the float64
    oracle, on a batch with partial sizes; dz is bf16 (8 significant bits)."""
    rng = np.random.default_rng(31)
    out = rng.normal(0, 1, (3, 17, 23, 16)).astype(np.float32).astype(np.float64)
    tgt = rng.normal(0, 1, (3, 17, 23, 16)).astype(np.float32).astype(np.float64)
    cx, cy = 0.5, 0.625
    loss, dz = _loss_grad(pmhd_lib, out, tgt, cx, cy)
    rl, rg = C.curl_loss_and_grad(out, tgt, cx, cy)
    assert abs(loss - rl) < 1e-5 * rl
    np.testing.assert_allclose(dz, rg, rtol=2.0 ** -7, atol=1e-3 * np.abs(rg).max())
    assert np.all(dz[..., 8:] == 0)


def test_network_gradient_chain_matches_oracle(pmhd_lib):
    """The training iteration's chain (four layers: GELU, GELU, GELU, linear;
    the loss kernel's gradient; weight gradients; backward through the three
    GELUs) composed from the kernels matches the float64 oracle's analytic
    gradients."""
    rng = np.random.default_rng(21)
    shape = (2, 16, 24)
    x = _bf(np.concatenate([rng.normal(0, 1, shape + (18,)), np.zeros(shape + (14,))], axis=3))
    W1, W2, W3 = (_bf(rng.normal(0, 0.1, (32, 9, 32))) for _ in range(3))
    W4 = _bf(rng.normal(0, 0.1, (16, 9, 32)))
    b1, b2, b3, b4 = (rng.normal(0, 0.05, n).astype(np.float32).astype(np.float64) for n in (32, 32, 32, 16))
    tgt = rng.normal(0, 1, shape + (16,)).astype(np.float32).astype(np.float64)
    tgt[..., 10:] = 0
    tgt[..., 5] = 0
    cx, cy = 0.5, 0.5
    z1, a1 = _conv(pmhd_lib, pmhd_lib.CONV_GELU, x, W1, b1, 32)
    z2, a2 = _conv(pmhd_lib, pmhd_lib.CONV_GELU, a1, W2, b2, 32)
    z3, a3 = _conv(pmhd_lib, pmhd_lib.CONV_GELU, a2, W3, b3, 32)
    out, _ = _conv(pmhd_lib, pmhd_lib.CONV_LINEAR, a3, W4, b4, 16)
    _, dz4 = _loss_grad(pmhd_lib, out, tgt, cx, cy)
    gW4, gb4 = _wgrad(pmhd_lib, a3, dz4)
    dz3, _ = _conv(pmhd_lib, pmhd_lib.CONV_DGELU, dz4, np.ascontiguousarray(W4.transpose(2, 1, 0)), None, 32, zprev=z3)
    gW3, gb3 = _wgrad(pmhd_lib, a2, dz3)
    dz2, _ = _conv(pmhd_lib, pmhd_lib.CONV_DGELU, dz3, np.ascontiguousarray(W3.transpose(2, 1, 0)), None, 32, zprev=z2)
    gW2, gb2 = _wgrad(pmhd_lib, a1, dz2)
    dz1, _ = _conv(pmhd_lib, pmhd_lib.CONV_DGELU, dz2, np.ascontiguousarray(W2.transpose(2, 1, 0)), None, 32, zprev=z1)
    gW1, gb1 = _wgrad(pmhd_lib, x, dz1)
    _, grads = C.net_curl_loss_and_grads(x, [(W1, b1), (W2, b2), (W3, b3), (W4, b4)], tgt, cx, cy)
    for (gw, gb), (rw, rb) in zip([(gW1, gb1), (gW2, gb2), (gW3, gb3), (gW4, gb4)], grads):
        # bf16 activations and gradients: a few per cent of the largest entry.
        np.testing.assert_allclose(gw, rw, rtol=0, atol=0.03 * np.abs(rw).max())
        np.testing.assert_allclose(gb, rb, rtol=0, atol=0.03 * np.abs(rb).max())
        cos = np.sum(gw * rw) / np.sqrt(np.sum(gw * gw) * np.sum(rw * rw))
        assert cos > 0.999


def _rel(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


def _rel_rho_mean(a, ref):
    """Relative L2 of rho and the mean over the six non-trivial conserved
    variables (rho, mx, my, E, Bx, By), per-variable RMS(a - ref) / RMS(ref)."""
    r = [float(np.sqrt(np.mean((a[..., k] - ref[..., k]) ** 2)) / np.sqrt(np.mean(ref[..., k] ** 2)))
         for k in (0, 1, 2, 4, 5, 6)]
    return r[0], float(np.mean(r))


def test_learned_correction_trains_and_beats_the_plain_coarse_grid(pmhd_lib, tmp_path):
    """Orszag-Tang with the field scaled by B0: pairs from four training
    amplitudes (coarse 64^2, fine 256^2), evaluation on the held-out amplitude
    B0 = 1 at t = 0.25.  Judged against the restricted fine run, the corrected
    coarse run must beat the plain coarse run in rho AND in the mean over the
    variables; every correction passes the checks or is counted."""
    OT = pmhd_lib.PROBLEM_ORSZAG_TANG
    t_end = 0.25
    with pmhd_lib.Learned(nx=64, ny=64, refine=4, max_pairs=1500, seed=11) as L:
        assert L.cfg.relax == 0.25 and L.cfg.train_noise == 0.03  # the defaults
        for b0 in (0.7, 0.85, 1.15, 1.3):
            assert L.generate(OT, [b0], t_end=t_end, every=1) > 100
        losses = L.train(iters=1500, batch=8, lr=2e-3)
        assert np.all(np.isfinite(losses))
        assert losses[-100:].mean() < 0.2 * losses[:10].mean()
        fine, sf = L.fine_run(OT, [1.0], t_end=t_end, refine=4)
        plain, sp = L.run(OT, [1.0], t_end=t_end, use_net=False)
        corr, sc = L.run(OT, [1.0], t_end=t_end, use_net=True)
        assert sp.t == sc.t == t_end
        assert sc.accepted + sc.rejected_positivity + sc.rejected_divergence == sc.steps
        assert sc.accepted > 0.9 * sc.steps  # positivity-safe outputs, curl field: few rejections
        rho_p, mean_p = _rel_rho_mean(plain, fine)
        rho_c, mean_c = _rel_rho_mean(corr, fine)
        print(f"relL2 vs restricted fine: rho plain {rho_p:.4e} corrected {rho_c:.4e}; mean plain {mean_p:.4e} "
              f"corrected {mean_c:.4e}; accepted {sc.accepted}/{sc.steps}")
        assert rho_c < rho_p and mean_c < mean_p
        # The corrections of the conserved quantities are mean-free: the
        # corrected run keeps the periodic totals of rho, momentum and B_z that
        # the plain run keeps, to the rounding drift of the solver itself (the
        # plain run's x-momentum total moves by ~1e-8 over these 314 steps;
        # an uncorrected bias of the network would move them by orders of
        # magnitude more).  (E is left out: the GLM coupling makes its total
        # depend on the trajectory.)
        for k in (0, 1, 2, 3, 7):
            tc, tp = corr[..., k].sum(), plain[..., k].sum()
            assert abs(tc - tp) <= 1e-9 * np.abs(plain[..., k]).sum(), (k, tc, tp)
        # Weights and normalisation survive a save / load into a new handle.
        path = str(tmp_path / "net.bin")
        L.save(path)
        with pmhd_lib.Learned(nx=64, ny=64, refine=4, max_pairs=1, seed=99) as L2:
            L2.load_weights(path)
            corr2, sc2 = L2.run(OT, [1.0], t_end=t_end, use_net=True)
            assert sc2.steps == sc.steps
            np.testing.assert_allclose(corr2, corr, rtol=0, atol=1e-12 * np.abs(corr).max())


def test_corrected_trajectory_pairs_need_a_trained_network(pmhd_lib):
    """pmhd_learned_generate_corrected takes pairs along the run the current
    network corrects: refused before training, one pair per coarse step
    after it."""
    OT = pmhd_lib.PROBLEM_ORSZAG_TANG
    with pmhd_lib.Learned(nx=32, ny=32, refine=2, max_pairs=400, seed=5) as L:
        with pytest.raises(pmhd_lib.PmhdError) as e:
            L.generate(OT, [1.0], t_end=0.05, corrected=True)
        assert e.value.status == pmhd_lib.ERR_ARG
        n0 = L.generate(OT, [1.0], t_end=0.05)
        L.train(iters=100, batch=4, lr=1e-3)
        n1 = L.generate(OT, [1.0], t_end=0.05, corrected=True)
        assert n0 > 5 and abs(n1 - n0) <= 2 and L.num_pairs == n0 + n1


def test_rollout_pairs_follow_the_coarse_trajectory(pmhd_lib):
    """pmhd_learned_generate_rollout stores one pair per coarse step, as
    pmhd_learned_generate does (the coarse run keeps its own state instead of
    restarting from the restricted fine one, so its CFL steps and hence the
    pair count may differ slightly), and a network trains on them."""
    OT = pmhd_lib.PROBLEM_ORSZAG_TANG
    counts = []
    for rollout in (False, True):
        with pmhd_lib.Learned(nx=32, ny=32, refine=2, max_pairs=200, seed=5) as L:
            counts.append(L.generate(OT, [1.0], t_end=0.1, every=1, rollout=rollout))
            if rollout:
                losses = L.train(iters=200, batch=4, lr=2e-3)
                assert np.all(np.isfinite(losses)) and losses[-20:].mean() < losses[:5].mean()
    assert counts[0] > 10 and abs(counts[0] - counts[1]) <= 2
