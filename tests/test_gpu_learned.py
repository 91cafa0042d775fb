"""The learned preconditioner's tensor-core convolution (tcgen05 + TMEM)
against a numpy restatement.

The numpy side rounds inputs and weights to BF16 exactly as the device does
(round to nearest even) and accumulates in FP64; the device accumulates in
FP32 and rounds its output to BF16, so the bound is 2^-8 of the output scale.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 2.0 ** -8


def _bf16(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16).to(torch.float32).numpy()


def conv_ref(x, w):
    """y[h, j, o] = sum_{dy, dx, i} x[h+dy-1, (j+dx-1) mod W, i] w[3 dy + dx, i, o],
    zero outside 0 <= h < H."""
    H, W, C = x.shape
    x, w = _bf16(x).astype(np.float64), _bf16(w).astype(np.float64)
    y = np.zeros((H, W, w.shape[2]))
    for dy in range(3):
        for dx in range(3):
            sh = np.roll(x, -(dx - 1), axis=1)               # sh[:, j] = x[:, j + dx - 1]
            pad = np.zeros_like(sh)
            lo, hi = max(0, 1 - dy), min(H, H + 1 - dy)      # rows h with 0 <= h + dy - 1 < H
            pad[lo:hi] = sh[lo + dy - 1:hi + dy - 1]
            y += pad @ w[3 * dy + dx]
    return y


def adjoint_weights(w):
    return np.stack([w[8 - t].T for t in range(9)])


@pytest.fixture(scope="module")
def G():
    from vvm_b200 import build, gpu
    build.build()
    return gpu


# W >= 144 runs the streamed TMA kernel (several rows a CTA once H * W / 128
# exceeds three CTAs a SM: 203 x 2048 gives 8 rows a CTA, a ring of 4 input
# slots refilled twice, and a last group of 3 rows); narrower rows the
# one-row-tile kernel
@pytest.mark.parametrize("H,W", [(3, 128), (5, 200), (4, 64), (2, 384), (203, 2048), (37, 1000)])
def test_conv_matches_reference(G, H, W):
    rng = np.random.default_rng(H * 1000 + W)
    x = rng.standard_normal((H, W, 32)).astype(np.float32)
    w = (rng.standard_normal((9, 32, 32)) / 16).astype(np.float32)
    y = G.conv3x3_c32(x, w)
    ref = conv_ref(x, w)
    assert np.abs(y - ref).max() <= TOL * np.abs(ref).max(), np.abs(y - ref).max()


@pytest.mark.parametrize("H,W", [(6, 256), (64, 1536)])
def test_adjoint_conv_matches_reference_and_transposes(G, H, W):
    rng = np.random.default_rng(7)
    x = rng.standard_normal((H, W, 32)).astype(np.float32)
    u = rng.standard_normal((H, W, 32)).astype(np.float32)
    w = (rng.standard_normal((9, 32, 32)) / 16).astype(np.float32)
    ya = G.conv3x3_c32(u, w, adjoint=True)
    ref = conv_ref(u, adjoint_weights(w))
    assert np.abs(ya - ref).max() <= TOL * np.abs(ref).max()
    # <A x, u> = <x, A^T u> up to the BF16 rounding of both results
    lhs = float(np.sum(G.conv3x3_c32(x, w).astype(np.float64) * _bf16(u)))
    rhs = float(np.sum(_bf16(x).astype(np.float64) * ya))
    assert abs(lhs - rhs) <= 1e-2 * abs(lhs)


# --------------------------------------------------------------- the network

def net_ref(params, x, NK):
    """The learned preconditioner in torch (CPU, FP64): the same layers, the
    same periodic-x / zero-y padding, the same parameter layout as
    vvm_gpu_learned_weights. x [H0][W0] -> z [H0][W0] (rows >= NK zero)."""
    import torch
    import torch.nn.functional as F
    C = 32

    def conv(a, w, cin, cout):          # a [cin, H, W], w [9][cin][cout] (tap = 3 dy + dx)
        ap = F.pad(a[None], (1, 1, 0, 0), mode="circular")
        ap = F.pad(ap, (0, 0, 1, 1))
        k = w.reshape(3, 3, cin, cout).permute(3, 2, 0, 1)
        return F.conv2d(ap, k)[0]

    def pool(a):
        return F.avg_pool2d(a[None], 2)[0]

    def up(a):
        return a.repeat_interleave(2, dim=1).repeat_interleave(2, dim=2)

    lift = params[:9 * C].reshape(9, 1, C)
    convs = [params[9 * C + i * 9 * C * C: 9 * C + (i + 1) * 9 * C * C].reshape(9, C, C) for i in range(6)]
    proj = params[9 * C + 6 * 9 * C * C:].reshape(9, C, 1)
    h0 = conv(x[None], lift, 1, C)
    h1 = conv(pool(h0), convs[0], C, C)
    h2 = conv(pool(h1), convs[1], C, C)
    h3 = conv(pool(h2), convs[2], C, C)
    g2 = conv(up(h3) + h2, convs[3], C, C)
    g1 = conv(up(g2) + h1, convs[4], C, C)
    g0 = conv(up(g1) + h0, convs[5], C, C)
    z = conv(g0, proj, C, 1)[0]
    mask = torch.zeros_like(z)
    mask[:NK] = 1.0
    return z * mask


def _net_case(G, NX=64, NZ=32):
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(NX, NZ)
    g = G.VVMGpu(st.grid, solver=G.VVM_SOLVER_LEARNED)
    g.upload(st)
    return g, st


def s_apply_ref(a, st, NK):
    """The operator the network works in on rows < NK of a [H0][W0] torch
    array, zero beyond: the cal_w operator in symmetric form (uniform levels:
    cx = 1/rhow_k, ru = 1/rhou_k, rd = 1/rhou_{k-1}) diagonally scaled,
    D^{-1/2} S D^{-1/2} with D = 2 cx + ru + rd: the energy norm of the loss."""
    import torch
    rhou, rhow = st.prof["rhou"], st.prof["rhow"]
    k = np.arange(NK) + 2
    cx0, ru0, rd0 = 1.0 / rhow[k], 1.0 / rhou[k], 1.0 / rhou[k - 1]
    s = 1.0 / np.sqrt(2 * cx0 + ru0 + rd0)
    s_up = np.append(s[1:], s[-1])
    s_dn = np.insert(s[:-1], 0, s[0])
    cx = torch.tensor(cx0 * s * s)[:, None]
    ru = torch.tensor(ru0 * s * s_up)[:, None]
    rd = torch.tensor(rd0 * s * s_dn)[:, None]
    b = a[:NK]
    y = b - cx * (torch.roll(b, 1, 1) + torch.roll(b, -1, 1))
    up = torch.zeros_like(b)
    up[:-1] = b[1:]
    dn = torch.zeros_like(b)
    dn[1:] = b[:-1]
    y = y - ru * up - rd * dn
    out = torch.zeros_like(a)
    out[:NK] = y
    return out


def test_network_forward_and_gradient_match_torch(G):
    """The loss L = 1 - (z, S t)^2 / ((z, S z)(t, S t)) (S the scaled operator
    of s_apply_ref) and dL/dweights against torch autograd in FP64 on the same weights (the device rounds
    weights and activations to BF16: relative bounds 2e-2 on z and L, 5e-2 on
    the gradient). The target is the network's own output plus noise of half
    its norm, so that (z, S t) is far from zero: with an unrelated target that
    sum cancels and the BF16 rounding of z moves it, and with it the gradient,
    by some 10 %."""
    import torch
    g, st = _net_case(G)
    H0, W0, n = g.learned_shape()
    NK = st.grid.NZ - 1
    rng = np.random.default_rng(3)
    x = np.zeros((H0, W0), np.float32)
    x[:NK] = rng.standard_normal((NK, W0))
    z_own = g.learned_eval(x)
    noise = np.zeros((H0, W0), np.float32)
    noise[:NK] = rng.standard_normal((NK, W0))
    t = (z_own + 0.5 * noise * np.linalg.norm(z_own) / np.linalg.norm(noise)).astype(np.float32)
    w = g.learned_weights()
    z, grad, loss = g.learned_eval(x, t)
    p = torch.tensor(_bf16(w).astype(np.float64), requires_grad=True)
    zr = net_ref(p, torch.tensor(_bf16(x).astype(np.float64)), NK)
    tt = torch.tensor(t.astype(np.float64))
    St = s_apply_ref(tt, st, NK)
    L = 1 - (zr * St).sum() ** 2 / ((zr * s_apply_ref(zr, st, NK)).sum() * (tt * St).sum())
    L.backward()
    zr = zr.detach().numpy()
    gr = p.grad.numpy()
    assert np.linalg.norm(z - zr) <= 2e-2 * np.linalg.norm(zr)
    assert abs(loss - float(L.detach())) <= 2e-2 * float(L.detach())
    assert np.linalg.norm(grad - gr) <= 5e-2 * np.linalg.norm(gr), np.linalg.norm(grad - gr) / np.linalg.norm(gr)
    g.close()


def test_training_reduces_the_loss_and_keeps_the_state(G):
    g, st = _net_case(G)
    g.step(2)
    before = g.download()
    first, last = g.learned_train(npairs=12, steps=80, batch=2, lr=2e-3, seed=1)
    after = g.download()
    assert all(np.array_equal(before.fields[f], after.fields[f]) for f in ("zeta", "th", "w", "u"))
    assert last < 0.5 * first, (first, last)
    g.close()


def test_learned_solve_meets_the_residual_and_beats_the_method_without_it(G):
    """Ablation: flexible CG preconditioned by the line solve plus the trained
    network against the line solve alone (the method without the network),
    same residual 1e-10; the solution matches the multigrid-PCG step to the
    solver tolerance."""
    from vvm_b200.initial_state import warm_bubble
    st = warm_bubble(128, 64)
    g = G.VVMGpu(st.grid, solver=G.VVM_SOLVER_LEARNED)
    g.upload(st)
    g.learned_train(npairs=24, steps=150, batch=2, lr=2e-3, seed=2)
    g.learned_config(mode=0, cap=400)
    g.step(3)
    it_net, fell = g.learned_last()
    _, rel = g.last_solve()
    assert not fell and rel <= 1e-10
    out = g.download()
    ref = G.VVMGpu(st.grid)
    ref.upload(st)
    ref.step(3)
    r = ref.download()
    for f in ("zeta", "th", "u", "w"):
        e = np.linalg.norm(out.fields[f] - r.fields[f]) / np.linalg.norm(r.fields[f])
        assert e <= 1e-8, (f, e)
    g2 = G.VVMGpu(st.grid, solver=G.VVM_SOLVER_LEARNED)
    g2.upload(st)
    g2.learned_config(mode=1, cap=4000)
    g2.step(3)
    it_plain, fell2 = g2.learned_last()
    assert not fell2
    assert it_net < it_plain, (it_net, it_plain)
    for h in (g, ref, g2):
        h.close()


def test_weights_from_small_workloads_serve_the_large_stretched_solve():
    """The network trained on the plain solver's pairs from the 128x64 warm
    bubble and the 1024x128 stretched squall line (few pairs here, to keep
    the test short) cuts the flexible-CG iterations of the 2048x256
    stretched-level solve against the same cycle without it, and the solve
    still meets the FP64 residual."""
    import torch
    from vvm_b200 import build
    from vvm_b200.gpu import VVM_SOLVER_LEARNED, VVMGpu
    from vvm_b200.initial_state import poisson_rhs, stretched_poisson_case
    from vvm_b200.learned_training import train_on_small_workloads
    build.build()
    w, rec = train_on_small_workloads(pairs_each=400, steps_each=150, batch=4)
    assert all(g["loss_last"] < g["loss_first"] for g in rec["grids"]), rec
    st = stretched_poisson_case(2048, 256, seed=7)
    b = poisson_rhs(st)
    d_b = torch.from_numpy(b).cuda()
    its = {}
    for mode in (0, 1):
        g = VVMGpu(st.grid, solver=VVM_SOLVER_LEARNED)
        g.upload(st)
        g.learned_weights(w)
        g.learned_config(mode=mode, cap=4000)
        d_W = torch.zeros_like(d_b)
        it, rel = g.poisson_solve_device(d_b.data_ptr(), d_W.data_ptr())
        fcg, fell = g.learned_last()
        assert not fell and rel <= 1e-10
        its[mode] = fcg
        g.close()
    assert its[0] * 3 < its[1], its
