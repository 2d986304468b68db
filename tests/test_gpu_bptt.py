"""GPU: the pyszsnn autograd function and its hand-written adjoint.

  * forward spikes / readout against the FP64 reference forward;
  * gradients against the FP64 BPTT reference run on the GPU's own forward
    trajectory (its spikes and pre-reset membrane): max |g_gpu - g_ref| <=
    1e-4 * max |g_ref| per weight tensor.  Against an FP64 forward of the same
    spike trains the gradients differ by up to ~1e-4 as well: the surrogate's
    slope (up to 2*beta) turns the fp32 forward's membrane rounding (~4e-7)
    into that much gradient change; the test bounds it at 5e-4;
  * finite differences of the GPU forward in the subthreshold regime with the
    surrogate off (beta = 0: the exact derivative);
  * checkpointing: results independent of the checkpoint interval.
"""
import numpy as np
import pytest
import torch

from oracle import bptt_ref as R
from szsnn_b200 import pyszsnn as P

pytestmark = pytest.mark.gpu


def _setup(N=300, M=60, K=6, B=4, T=130, density=0.1, w_in_scale=0.6, w_rec_scale=1.0, beta=10.0, ck=50, seed=0,
           shuffle_rows=False, store=False):
    dev = torch.device("cuda")
    rp, col, val = P.random_recurrent(N, density, seed, dev)
    if shuffle_rows:  # columns out of order inside each row
        rng = np.random.default_rng(seed + 99)
        rpn, cn, vn = rp.cpu().numpy(), col.cpu().numpy().copy(), val.cpu().numpy().copy()
        for j in range(N):
            perm = rng.permutation(rpn[j + 1] - rpn[j]) + rpn[j]
            cn[rpn[j]:rpn[j + 1]], vn[rpn[j]:rpn[j + 1]] = cn[perm], vn[perm]
        col, val = torch.from_numpy(cn).to(dev), torch.from_numpy(vn).to(dev)
    val = val * w_rec_scale
    g = torch.Generator(device="cpu").manual_seed(seed)
    w_in = (torch.randn((M, N), generator=g) * w_in_scale / np.sqrt(M)).to(dev)
    w_out = (torch.randn((N, K), generator=g) / np.sqrt(N)).to(dev)
    rates = torch.rand(M, generator=g) * 50.0
    x = P.poisson_bits(T, B, rates.to(dev), 1.0, seed)
    v0 = (torch.rand((B, N), generator=g) * 0.5).to(dev)
    net = P.LIFCurrExpRNN(N, M, K, rp, col, alpha=0.95, beta=beta, checkpoint_every=ck, store_trajectory=store)
    return net, w_in, val, w_out, x, v0


def _dense(net, val):
    N = net.n_neurons
    W = np.zeros((N, N), np.float64)
    rp = net.rec_row_ptr.cpu().numpy()
    col = net.rec_col.cpu().numpy()
    v = val.detach().cpu().numpy().astype(np.float64)
    for j in range(N):
        W[j, col[rp[j]:rp[j + 1]]] = v[rp[j]:rp[j + 1]]
    return W


def test_forward_matches_fp64_reference():
    net, w_in, val, w_out, x, v0 = _setup()
    out = P.simulate(net, w_in, val, w_out, x, v0)
    torch.cuda.synchronize()
    S_gpu = P.unpack_bits(out["spikes"], net.n_neurons).cpu().numpy()
    xs = P.unpack_bits(x, net.n_inputs).cpu().numpy()
    p = dict(net.params, alpha=net.alpha)
    fw = R.forward(p, w_in.cpu().numpy(), _dense(net, val), w_out.cpu().numpy(), xs, v0.cpu().numpy())
    assert S_gpu.sum() > 500
    agree = (S_gpu == fw["S"].astype(bool)).mean()
    assert np.array_equal(S_gpu[:20], fw["S"][:20].astype(bool))
    assert agree > 0.999
    # readout of the GPU's own spikes equals the FP64 readout of those spikes
    fw2 = R.forward(p, w_in.cpu().numpy(), _dense(net, val), w_out.cpu().numpy(), xs, v0.cpu().numpy(), spikes=S_gpu)
    assert np.allclose(out["ymax"].cpu().numpy(), fw2["ymax"], rtol=1e-5, atol=1e-5)
    assert np.allclose(out["vsum"].cpu().numpy(), fw2["vsum"], rtol=1e-4, atol=1e-3)


@pytest.mark.parametrize("ck,N,B,shuffle,store", [(50, 300, 4, False, False), (13, 300, 4, False, False),
                                                 (50, 1000, 37, False, False), (50, 3000, 64, False, False),
                                                 (50, 300, 4, True, False), (50, 300, 4, False, True),
                                                 (50, 1000, 37, False, True)])
def test_gradients_match_fp64_bptt(ck, N, B, shuffle, store):
    """B = 37: trials not a multiple of four (the SpMM's float4 trial groups
    are partly empty); N = 3000, B = 64: full trial groups, long rows;
    shuffle: columns out of order inside the rows; store: the backward reads
    the trajectory the forward kept instead of recomputing it."""
    net, w_in, val, w_out, x, v0 = _setup(ck=ck, N=N, B=B, T=130 if N <= 300 else 40, shuffle_rows=shuffle,
                                          store=store)
    w_in.requires_grad_(True)
    val.requires_grad_(True)
    w_out.requires_grad_(True)
    ymax, vsum = P.LIFCurrExpFunction.apply(w_in, val, w_out, x, v0, net)
    g = torch.Generator(device="cpu").manual_seed(1)
    gy = torch.randn(ymax.shape, generator=g).cuda()
    gv = (torch.randn(vsum.shape, generator=g) * 1e-3).cuda()
    (ymax * gy).sum().add_((vsum * gv).sum()).backward()
    torch.cuda.synchronize()
    out = P.simulate(net, w_in.detach(), val.detach(), w_out.detach(), x, v0, trace_u=True)
    S = P.unpack_bits(out["spikes"], net.n_neurons).cpu().numpy()
    xs = P.unpack_bits(x, net.n_inputs).cpu().numpy()
    p = dict(net.params, alpha=net.alpha)
    Wd = _dense(net, val)
    fw = R.forward(p, w_in.detach().cpu().numpy(), Wd, w_out.detach().cpu().numpy(), xs, v0.cpu().numpy(), spikes=S)
    assert np.array_equal(fw["tmax"], out["tmax"].cpu().numpy())
    fw_gpu = dict(fw, U=out["u_trace"].cpu().numpy().astype(np.float64))
    rp, col = net.rec_row_ptr.cpu().numpy(), net.rec_col.cpu().numpy()
    rows = np.repeat(np.arange(net.n_neurons), np.diff(rp))
    for traj, bound in ((fw_gpu, 1e-4), (fw, 5e-4)):
        dWin, dWrec, dWout = R.backward(p, w_in.detach().cpu().numpy(), Wd, w_out.detach().cpu().numpy(), xs, traj,
                                        gy.cpu().numpy(), gv.cpu().numpy(), beta=net.beta)
        for got, ref in ((w_in.grad, dWin), (val.grad, dWrec[rows, col]), (w_out.grad, dWout)):
            got = got.cpu().numpy().astype(np.float64)
            err = np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-30)
            assert err <= bound, (err, bound)
            assert np.max(np.abs(ref)) > 0


def test_full_size_gradients_match_fp64_bptt():
    """The benchmark's shape (N = 10,000, 10 % recurrent, M = 700 inputs,
    K = 20 readouts, B = 64 trials) over a short horizon: gradients within
    1e-4 of FP64 BPTT on the GPU's own trajectory."""
    net, w_in, val, w_out, x, v0 = _setup(N=10000, M=700, K=20, B=64, T=20, w_in_scale=1.0)
    for t in (w_in, val, w_out):
        t.requires_grad_(True)
    ymax, vsum = P.LIFCurrExpFunction.apply(w_in, val, w_out, x, v0, net)
    g = torch.Generator(device="cpu").manual_seed(2)
    gy = torch.randn(ymax.shape, generator=g).cuda()
    gv = (torch.randn(vsum.shape, generator=g) * 1e-3).cuda()
    (ymax * gy).sum().add_((vsum * gv).sum()).backward()
    torch.cuda.synchronize()
    out = P.simulate(net, w_in.detach(), val.detach(), w_out.detach(), x, v0, trace_u=True)
    S = P.unpack_bits(out["spikes"], net.n_neurons).cpu().numpy()
    assert S.sum() > 1000
    xs = P.unpack_bits(x, net.n_inputs).cpu().numpy()
    p = dict(net.params, alpha=net.alpha)
    Wd = _dense(net, val)
    fw = R.forward(p, w_in.detach().cpu().numpy(), Wd, w_out.detach().cpu().numpy(), xs, v0.cpu().numpy(), spikes=S)
    fw_gpu = dict(fw, U=out["u_trace"].cpu().numpy().astype(np.float64))
    dWin, dWrec, dWout = R.backward(p, w_in.detach().cpu().numpy(), Wd, w_out.detach().cpu().numpy(), xs, fw_gpu,
                                    gy.cpu().numpy(), gv.cpu().numpy(), beta=net.beta)
    rp, col = net.rec_row_ptr.cpu().numpy(), net.rec_col.cpu().numpy()
    rows = np.repeat(np.arange(net.n_neurons), np.diff(rp))
    for got, ref in ((w_in.grad, dWin), (val.grad, dWrec[rows, col]), (w_out.grad, dWout)):
        got = got.cpu().numpy().astype(np.float64)
        err = np.max(np.abs(got - ref)) / max(np.max(np.abs(ref)), 1e-30)
        assert err <= 1e-4, err
        assert np.max(np.abs(ref)) > 0


def test_finite_differences_subthreshold():
    """Below threshold the layer is linear in w_in on each sign pattern of the
    weights (the sign picks the exc / inh synaptic channel), so a central
    difference along a sign-preserving direction (w -> w (1 + eps n), |eps n|
    < 1) is exact up to rounding.  The fp32 forward limits that rounding, so
    the check uses one directional derivative over all input weights (large
    signal) and a loss summed in fp64."""
    net, w_in, val, w_out, x, v0 = _setup(w_in_scale=0.02, w_rec_scale=0.02, beta=0.0)
    c = torch.randn((x.shape[1], net.n_neurons), generator=torch.Generator().manual_seed(3)).cuda()

    def loss(wi):
        ymax, vsum = P.LIFCurrExpFunction.apply(wi, val, w_out, x, v0, net)
        return (vsum.double() * c.double()).sum()

    wi = w_in.clone().requires_grad_(True)
    loss(wi).backward()
    n = torch.randn(w_in.shape, generator=torch.Generator().manual_seed(5)).clamp(-3, 3).cuda()
    d = w_in * n
    eps = 0.2
    for wp in (w_in + eps * d, w_in - eps * d):
        out = P.simulate(net, wp, val, w_out, x, v0)
        assert int(P.unpack_bits(out["spikes"], net.n_neurons).sum()) == 0
    with torch.no_grad():
        fd = (float(loss(w_in + eps * d)) - float(loss(w_in - eps * d))) / (2 * eps)
    ad = float((wi.grad.double() * d.double()).sum())
    assert abs(fd - ad) <= 1e-3 * abs(fd), (fd, ad)


def test_backward_phase_times():
    net, w_in, val, w_out, x, v0 = _setup()
    net.phase_ms = np.zeros(4)
    val.requires_grad_(True)
    ymax, vsum = P.LIFCurrExpFunction.apply(w_in, val, w_out, x, v0, net)
    ymax.sum().backward()
    assert np.all(net.phase_ms > 0) and len(P.BACKWARD_PHASES) == 4


def test_checkpoint_interval_does_not_change_gradients():
    grads = []
    for ck in (50, 1000):
        net, w_in, val, w_out, x, v0 = _setup(ck=ck, seed=7)
        w_in.requires_grad_(True)
        ymax, vsum = P.LIFCurrExpFunction.apply(w_in, val, w_out, x, v0, net)
        ymax.sum().backward()
        grads.append(w_in.grad.clone())
    assert torch.equal(grads[0], grads[1])


def test_full_size_gradients_do_not_depend_on_the_checkpoint_interval():
    """The benchmark's BPTT shape (10,000 neurons, 10 % recurrent, 700 inputs,
    20 readouts, batch 64) over 100 steps: recomputing from checkpoints every
    25 or every 50 steps gives bit-identical input and recurrent weight
    gradients (a size-independent check of the recompute and of the recurrent
    term).  The readout-weight gradient is summed with fp32 atomics (its order
    varies from run to run), so it is compared within 1e-6 relative."""
    grads = []
    for ck in (25, 50):
        net, w_in, val, w_out, x, v0 = _setup(N=10000, M=700, K=20, B=64, T=100, ck=ck, seed=11)
        for t in (w_in, val, w_out):
            t.requires_grad_(True)
        ymax, vsum = P.LIFCurrExpFunction.apply(w_in, val, w_out, x, v0, net)
        (ymax.sum() + 1e-3 * vsum.sum()).backward()
        torch.cuda.synchronize()
        grads.append([t.grad.clone() for t in (w_in, val, w_out)])
    for g0, g1 in zip(*grads):
        assert torch.isfinite(g0).all() and float(g0.abs().max()) > 0
    assert torch.equal(grads[0][0], grads[1][0]) and torch.equal(grads[0][1], grads[1][1])
    g0, g1 = grads[0][2], grads[1][2]
    assert float((g0 - g1).abs().max()) <= 1e-6 * float(g0.abs().max())


def test_stored_trajectory_gives_the_recomputed_gradients():
    """The benchmark's shape over 100 steps: the backward reading the
    trajectory the forward kept and the backward recomputing it from
    checkpoints every 50 steps give bit-identical input and recurrent weight
    gradients (the readout's fp32 atomics: within 1e-6 relative); with the
    trajectory kept the recompute phase is empty."""
    grads, phases = [], []
    for store in (False, True):
        net, w_in, val, w_out, x, v0 = _setup(N=10000, M=700, K=20, B=64, T=100, ck=50, seed=11, store=store)
        net.phase_ms = np.zeros(4)
        for t in (w_in, val, w_out):
            t.requires_grad_(True)
        ymax, vsum = P.LIFCurrExpFunction.apply(w_in, val, w_out, x, v0, net)
        (ymax.sum() + 1e-3 * vsum.sum()).backward()
        torch.cuda.synchronize()
        grads.append([t.grad.clone() for t in (w_in, val, w_out)])
        phases.append(net.phase_ms.copy())
    assert torch.equal(grads[0][0], grads[1][0]) and torch.equal(grads[0][1], grads[1][1])
    g0, g1 = grads[0][2], grads[1][2]
    assert float((g0 - g1).abs().max()) <= 1e-6 * float(g0.abs().max())
    assert phases[0][0] > 0 and phases[1][0] == 0


def test_trajectory_kept_by_default_when_it_fits():
    net, *_ = _setup(N=300, B=4, T=130)
    net.store_trajectory = None
    assert net.stores_trajectory(130, 4, torch.device("cuda"))
    net.trajectory_budget = 1000
    assert not net.stores_trajectory(130, 4, torch.device("cuda"))
