"""The learned preconditioner on the device: forward and parameter gradient
against the numpy restatement (oracle/precnet_oracle.py), training with the
library's kernels, the FGMRES solve with the network, its gain over the
same solve without training, and the fallback to the plain solve."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


def test_forward_and_gradient_match_oracle(torch_cuda):
    from bamrex_b200.learned import PrecNet
    from oracle import precnet_oracle as P
    rng = np.random.default_rng(5)
    net = PrecNet(32, 24, batch=2, seed=11)
    net.set_tensor_cores(False)  # the FP32 forward, the one training differentiates
    w = net.get_weights().astype(np.float64)
    _, n = P.param_slices()
    assert net.num_params == n
    x = rng.standard_normal((2, 2, 24, 32)).astype(np.float32)
    out = net.forward(x)
    A = P.forward(w, x)
    ref = A[-1][:, 0]
    assert np.abs(out - ref).max() <= 1e-4 * np.abs(ref).max()
    dout = rng.standard_normal((2, 24, 32)).astype(np.float32)
    g = net.backward(dout)
    gref = P.backward(w, A, dout)
    assert np.linalg.norm(g - gref) <= 1e-4 * np.linalg.norm(gref)
    # per layer too: each conv's weight gradient
    sl, _ = P.param_slices()
    for s in sl:
        if s is None:
            continue
        a, b = g[s[0]:s[2]], gref[s[0]:s[2]]
        assert np.linalg.norm(a - b) <= 1e-3 * np.linalg.norm(b) + 1e-6
    net.close()


def test_tensor_core_forward_matches_fp32(torch_cuda):
    """The BF16 tensor-core convolutions agree with the FP32 ones to BF16
    rounding of the activations."""
    from bamrex_b200.learned import PrecNet
    rng = np.random.default_rng(6)
    net = PrecNet(128, 64, batch=2, seed=4)
    x = rng.standard_normal((2, 2, 64, 128)).astype(np.float32)
    net.set_tensor_cores(False)
    ref = net.forward(x)
    net.set_tensor_cores(True)
    got = net.forward(x)
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err <= 2e-2, err
    assert not np.array_equal(got, ref)  # the tensor-core path did run
    net.close()


def test_tcgen05_forward_matches_mma_and_fp32(torch_cuda):
    """The 16 -> 16 convolutions on tcgen05 agree with the FP32 CUDA cores to
    BF16 rounding.  The network is 1024 wide (every level a multiple of 128,
    so tcgen05 runs everywhere) and 48 high, so its coarsest level (6 rows)
    is one mma.sync cannot take: there mma.sync-only mode falls back to the
    FP32 kernel while tcgen05 runs, and the two modes differ."""
    from bamrex_b200.learned import PrecNet
    rng = np.random.default_rng(8)
    net = PrecNet(1024, 48, batch=2, seed=5)
    x = rng.standard_normal((2, 2, 48, 1024)).astype(np.float32)
    outs = {}
    for mode in (0, 1, 2):
        net.set_tensor_cores(mode)
        outs[mode] = net.forward(x)
        assert np.all(np.isfinite(outs[mode]))
    ref = np.linalg.norm(outs[0])
    assert np.linalg.norm(outs[1] - outs[0]) <= 2e-2 * ref
    assert np.linalg.norm(outs[2] - outs[0]) <= 2e-2 * ref
    assert not np.array_equal(outs[1], outs[2]) and not np.array_equal(outs[1], outs[0])
    # repeated forwards give the same result (no state left between calls)
    net.set_tensor_cores(1)
    np.testing.assert_array_equal(net.forward(x), outs[1])
    with pytest.raises(Exception):
        net.set_tensor_cores(3)
    net.close()


@pytest.fixture(scope="module")
def trained(torch_cuda):
    """A network trained on 160 pairs from the plain solver at 64^2."""
    from bamrex_b200.learned import PrecNet, make_training_pairs, train
    X, Y = make_training_pairs(160, n=64, seed=3, corr_cells=8)
    net = PrecNet(64, 64, batch=8, seed=2)
    w0 = net.get_weights()
    losses = train(net, X, Y, epochs=8, batch=8, lr=3e-3)
    return net, w0, losses


def test_training_lowers_the_loss(trained):
    net, w0, losses = trained
    first, last = np.mean(losses[:5]), np.mean(losses[-5:])
    assert last < 0.6 * first, (first, last)


def test_learned_solve_gain_and_fallback(trained):
    """On a held-out problem, FGMRES preconditioned by the trained network
    followed by one V-cycle needs fewer iterations than the same solve with
    the V-cycle alone (the method without the network) and than with the
    untrained network; a too-small iteration budget falls back to the plain
    solve, which reaches the tolerance."""
    from bamrex_b200 import problems
    from bamrex_b200._abi import PRECOND_NETWORK, PRECOND_NETWORK_VCYCLE, PRECOND_VCYCLE
    from bamrex_b200.helmholtz import Helmholtz
    from bamrex_b200.learned import PrecNet, solve_learned
    net, w0, _ = trained
    n, dx = 64, 1.0 / 2048
    mach = 0.01
    B = (0.8 * dx / mach) ** 2
    rng = np.random.default_rng(99)
    beta = np.exp(-problems.gaussian_random_field((n, n), 8, None, rng))[None]
    rhs = problems.gaussian_random_field((n, n), 4, None, rng)[None]
    h = Helmholtz(2, (n, n), [0.0, 0.0], [n * dx, n * dx])
    h.setScalars(1.0, B, 0.0)
    h.setACoeffs(mach * mach / 0.4)
    h.setBCoeffsFromCell(beta)
    net.resize(n, n, 1)
    fresh = PrecNet(n, n, batch=1, seed=2)
    fresh.set_weights(w0)
    its = {}
    for name, nn, mode in (("trained+V", net, PRECOND_NETWORK_VCYCLE), ("untrained+V", fresh, PRECOND_NETWORK_VCYCLE),
                           ("V", None, PRECOND_VCYCLE), ("trained", net, PRECOND_NETWORK),
                           ("untrained", fresh, PRECOND_NETWORK)):
        x, it, pit, rr, fb = solve_learned(h, nn, rhs, tol_rel=1e-8, max_iter=150, restart=30, mode=mode)
        assert rr <= 1e-8
        its[name] = it if not fb else 10 ** 6
    print("FGMRES iterations to 1e-8:", its)
    assert its["trained+V"] < its["V"] and its["trained+V"] <= its["untrained+V"]
    # one application of the network alone: the residual it leaves
    from bamrex_b200.learned import network_input
    inp, s = network_input(rhs[0], beta[0])
    left = {}
    for name, nn in (("trained", net), ("untrained", fresh)):
        e = nn.forward(inp[None])[0].astype(np.float64) * s * dx * dx / B
        r = rhs[0] - h.apply(e[None])[0]
        left[name] = np.linalg.norm(r) / np.linalg.norm(rhs)
    print("residual left by one network application:", left)
    assert left["trained"] < 0.7 and left["trained"] < 0.5 * left["untrained"]
    x3, it3, pit3, rr3, fb3 = solve_learned(h, net, rhs, tol_rel=1e-8, max_iter=2, restart=30, mode=PRECOND_NETWORK)
    assert fb3 and it3 == 2 and pit3 > 0 and rr3 <= 1e-8
    x, it, pit, rr, fb = solve_learned(h, net, rhs, tol_rel=1e-8, max_iter=150, restart=30)
    xp, itp, rrp = h.solve(rhs, tol_rel=1e-8)
    assert rr <= 1e-8 and rrp <= 1e-8
    assert np.abs(x - xp).max() <= 1e-4 * np.abs(xp).max()
    fresh.close()
    h.close()
