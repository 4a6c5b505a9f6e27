"""Learned JCG initial guess (csrc/mpnn.cu) against a plain PyTorch FP32
reference of the same network.

The device stores inputs, weights and activations in BF16 and accumulates
in FP32 on the tensor cores; the reference rounds the same tensors to BF16
at the same points and computes in FP32, so the two agree to BF16 accuracy
(tolerances below), not bit for bit.  Gradients are checked against torch
autograd of the FP32 network (BF16-rounded weights and inputs).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

H, L = 64, 3


def _bf16(t):
    import torch
    return t.to(torch.bfloat16).to(torch.float32)


def _random_params(case, seed=3):
    from adcirc_b200 import learned
    a = case.arrays
    x = learned.features(a, case.params["prbckgrnd_mh2o"])
    p = learned.init_params(x.mean(axis=0), x.std(axis=0), 1e-4, seed)
    rng = np.random.default_rng(seed)
    v = learned.layer_views(p)
    v["w_out"][:] = rng.normal(0, 0.3, H)
    v["b_out"][:] = 0.05
    for l in range(L):
        v[f"b{l}"][:] = rng.normal(0, 0.05, H)
    return p


def _ring(case):
    a = case.arrays
    n = case.sizes["np"]
    nb = [[int(j) - 1 for j in a["neitab"][i, 1:a["nneigh"][i]] if 1 <= j <= n and j - 1 != i]
          for i in range(n)]
    return nb


def _torch_forward(case, p, rounding=True):
    """The network of csrc/mpnn.cu in torch FP32; with `rounding`, BF16
    rounding where the device stores BF16."""
    import torch
    from adcirc_b200 import learned
    r = _bf16 if rounding else (lambda t: t)
    a = case.arrays
    n = case.sizes["np"]
    v = {k: torch.tensor(np.array(t, np.float32)) for k, t in learned.layer_views(p).items()}
    f = torch.tensor(learned.features(a, case.params["prbckgrnd_mh2o"]), dtype=torch.float32)
    x = torch.zeros(n, 16)
    x[:, :9] = (f - v["mean"]) / v["std"]
    x[:, 9] = 1.0
    x = r(x)
    nb = _ring(case)
    idx = torch.tensor([j for lst in nb for j in lst])
    seg = torch.tensor([i for i, lst in enumerate(nb) for _ in lst])
    deg = torch.tensor([max(len(lst), 1) for lst in nb], dtype=torch.float32)
    W_in = r(v["W_in"]).requires_grad_(True)
    Ws = [r(v[f"Ws{l}"]).requires_grad_(True) for l in range(L)]
    Wn = [r(v[f"Wn{l}"]).requires_grad_(True) for l in range(L)]
    b = [v[f"b{l}"].clone().requires_grad_(True) for l in range(L)]
    w_out = v["w_out"].clone().requires_grad_(True)
    b_out = v["b_out"].clone().requires_grad_(True)
    h = r(torch.relu(x @ W_in.T))
    for l in range(L):
        m = torch.zeros(n, H).index_add_(0, seg, h[idx]) / deg[:, None]
        h = r(torch.relu(h @ Ws[l].T + r(m) @ Wn[l].T + b[l]))
    out = h @ w_out + b_out
    leaves = {"W_in": W_in, "Ws": Ws, "Wn": Wn, "b": b, "w_out": w_out, "b_out": b_out}
    return out, h, leaves


def _use_mask(case):
    from adcirc_b200 import learned
    return learned.use_mask(case.arrays)


HUBER = 3.0


def _huber(e):
    """The device's training loss of a normalised error (threshold 3)."""
    import torch
    ae = e.abs()
    return torch.where(ae <= HUBER, e * e, HUBER * (2.0 * ae - HUBER))


def _state(steps=40):
    from adcirc_b200 import model
    case = model.channel_case(vortex=True)
    g = model.GpuModel(case)
    g.run(1, steps)
    g.sync_to_host()
    return case, g


def test_predictor_forward_matches_torch(lib):
    case, g = _state()
    p = _random_params(case)
    g.set_predictor(p)
    guess, h3 = g.predictor_forward(hidden=True)
    g.close()
    out, h_ref, _ = _torch_forward(case, p)
    h_ref = h_ref.detach().numpy()
    scale = np.abs(h_ref).max()
    assert scale > 0.1
    err_h = np.abs(h3 - h_ref).max() / scale
    assert err_h <= 3e-2, err_h
    a = case.arrays
    use = _use_mask(case)
    s_out = float(p[-1])
    ref = a["etas"]
    corr_dev = (guess - ref) / s_out
    corr_ref = out.detach().numpy()
    assert np.array_equal(guess[~use], ref[~use])       # the reference guess off the wet interior
    err = np.abs(corr_dev[use] - corr_ref[use]).max() / max(np.abs(corr_ref[use]).max(), 1e-6)
    assert err <= 3e-2, err


def test_predictor_gradient_matches_torch(lib):
    import torch
    from adcirc_b200 import learned
    case, g = _state()
    p = _random_params(case, seed=5)
    g.set_predictor(p)
    rng = np.random.default_rng(9)
    a = case.arrays
    s_out = float(p[-1])
    target = a["etas"] + s_out * rng.normal(0.0, 1.5, a["etas"].size)
    grad = g.predictor_gradient_at(target)
    g.close()
    out, _, leaves = _torch_forward(case, p)
    use = torch.tensor(_use_mask(case))
    t = torch.tensor((target - a["etas"]) / s_out, dtype=torch.float32)
    loss = (_huber(out - t) * use).sum() / out.numel()
    loss.backward()
    gv = learned.layer_views(grad)

    def check(dev, ref, name):
        dev = np.asarray(dev, np.float64).ravel()
        ref = ref.detach().numpy().astype(np.float64).ravel()
        cos = dev @ ref / (np.linalg.norm(dev) * np.linalg.norm(ref) + 1e-30)
        rel = np.linalg.norm(dev - ref) / (np.linalg.norm(ref) + 1e-30)
        assert cos >= 0.995 and rel <= 6e-2, (name, cos, rel)

    check(gv["w_out"], leaves["w_out"].grad, "w_out")
    check(gv["b_out"], leaves["b_out"].grad, "b_out")
    for l in range(L):
        check(gv[f"Ws{l}"], leaves["Ws"][l].grad, f"Ws{l}")
        check(gv[f"Wn{l}"], leaves["Wn"][l].grad, f"Wn{l}")
        check(gv[f"b{l}"], leaves["b"][l].grad, f"b{l}")
    check(gv["W_in"][:, :10], leaves["W_in"].grad[:, :10], "W_in")


def test_training_keeps_the_plain_solve_and_learns(lib):
    """Training on the plain solver's pairs: the solve keeps the reference
    guess (the run is bit-identical to one without a predictor), and after
    training the network's loss on a new step is below that of predicting
    no correction at all (a zero head, where training starts)."""
    from adcirc_b200 import learned, model
    plain = model.channel_case(vortex=True)
    gp = model.GpuModel(plain)
    gp.run(1, 40)
    case, g = _state()
    a = case.arrays
    e0 = a["etas"].copy()
    g.run(41, 1)
    g.sync_to_host()
    use = _use_mask(case)
    s_out = float(np.sqrt(np.mean((a["etas"][use] - e0[use]) ** 2)))
    x = learned.features(a, case.params["prbckgrnd_mh2o"])
    p = learned.init_params(x.mean(axis=0), x.std(axis=0), s_out, seed=2)
    g.set_predictor(p)
    g.predictor_train(True, 2e-3)
    it = 42
    for k in range(5):
        g.run(it, 200)
        it += 200
    g.sync_to_host()
    ref = a["etas"].copy()
    use = _use_mask(case)
    g.run(it, 1)
    loss = g.predictor_stats()[0]
    g.sync_to_host()
    import torch
    base = float(_huber(torch.tensor((a["etas"] - ref) / s_out)[torch.tensor(use)]).sum()) / a["etas"].size
    gp.run(41, it - 40)
    gp.sync_to_host()
    assert g.predictor_stats()[1] == 1001
    assert np.array_equal(a["eta2"], plain.arrays["eta2"])
    assert np.isfinite(loss) and loss < 0.9 * base, (loss, base)
    g.close()
    gp.close()


def test_learned_start_converges_to_the_same_tolerance(lib):
    """With ADC_LEARNED_START the solve starts from the better of the two
    guesses and stops at the same tolerance: the run stays within the JCG
    tolerance's reach of the plain one, and every step is counted as used
    or fallen back."""
    from adcirc_b200 import _lib, model
    case, g = _state(20)
    p = _random_params(case)
    g.close()
    plain = model.channel_case(vortex=True)
    lc = model.channel_case(vortex=True)
    gp = model.GpuModel(plain)
    gl = model.GpuModel(lc, prec=_lib.ADC_LEARNED_START)
    gl.set_predictor(p)
    ip, _ = gp.run(1, 200)
    il, _ = gl.run(1, 200)
    used, fb = gl.warm_start_stats()
    gp.sync_to_host()
    gl.sync_to_host()
    gp.close()
    gl.close()
    assert used + fb == 200
    d = np.abs(lc.arrays["eta2"] - plain.arrays["eta2"]).max() / np.abs(plain.arrays["eta2"]).max()
    assert d <= 1e-6, d
    assert np.isfinite(lc.arrays["eta2"]).all()
