"""Numerics of the learned preconditioner stage against a PyTorch evaluation of the same network.

The stage is z_c = s * W3^T relu(W2^T relu(W1^T f_c / ...)) with f_c = [r_c, r of the six face neighbours, log k of
the cell and its neighbours] / s, s = |r| / sqrt(n) (the features k are not scaled).  On the GPU the inputs and
hidden activations are rounded to BF16 before each product and the products accumulate in FP32.  The tests export
the weights through the C ABI and compare:

* the forward pass with a PyTorch FP32 evaluation that rounds the same quantities to BF16 (tight), and with a plain
  FP32 evaluation (tolerance from BF16 rounding: 2^-8 relative per rounding, three roundings deep);
* the gradient of the training loss (z^T A z - 2 z^T r) / |r|^2 (mlp_bwd_kernel) with PyTorch autograd in FP64 and
  with central finite differences of the FP64 loss along random directions (tolerance: the BF16 roundings of the
  forward pass, which the GPU gradient inherits);
* that training collects the requested number of solver-generated residuals.
"""
import numpy as np
import pytest

from bosss_b200 import assembly as A
from bosss_b200.solvers import BlockMsrMatrix, FGMRESConfig, MultigridOperator, PmgConfig

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def stage():
    s = A.variable_coeff_3d(6, 2, seed=3)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    nbr = s.grid.face_neighbours()
    feats = A.log_coeff_features(s)
    op.SetCellGraph(nbr, feats)
    slv = FGMRESConfig(ConvergenceCriterion=1e-10, termination="relative", Learned="fgmres",
                       Preconditioners=[PmgConfig(DegreeHierarchy=(10, 4, 1), CoarseTolerance=1e-2)]
                       ).CreateInstance(op)
    yield s, op, slv, nbr, feats
    slv.Dispose()
    op.Dispose()


def _bf16(t):
    import torch
    return t.to(torch.bfloat16).to(t.dtype)


def _features(r, nbr, feats, Np, Fp, sc, dtype):
    import torch
    nc = nbr.shape[0]
    R = torch.from_numpy(r).reshape(nc, Np).to(dtype) / sc
    idx = torch.from_numpy(nbr.astype(np.int64))
    blocks = [R]
    for f in range(nbr.shape[1]):
        k = idx[:, f]
        blocks.append(torch.where((k >= 0)[:, None], R[k.clamp(min=0)], torch.zeros((), dtype=dtype)))
    X = torch.cat(blocks + [torch.from_numpy(feats).to(dtype)], dim=1)
    return torch.nn.functional.pad(X, (0, Fp - X.shape[1]))


def _forward(r, nbr, feats, W, info, dtype, bf16_rounding):
    import torch
    Np = info["Np"]
    sc = float(np.linalg.norm(r) / np.sqrt(len(r)))
    W1, W2, W3 = (torch.as_tensor(w).to(dtype) for w in W)
    X = _features(r, nbr, feats, Np, info["Fp"], sc, dtype)
    rnd = _bf16 if bf16_rounding else (lambda t: t)
    h1 = torch.relu(rnd(X) @ W1)
    h2 = torch.relu(rnd(h1) @ W2)
    y = rnd(h2) @ W3
    return y[:, :Np].reshape(-1) * sc


def test_learned_forward_matches_pytorch(cuda, stage):
    import torch
    s, op, slv, nbr, feats = stage
    info = slv.LearnedInfo()
    assert info["F"] == 7 * s.Np + 7 and info["H"] == 64
    W = slv.LearnedWeights()
    r = np.random.default_rng(5).standard_normal(s.N)
    z = slv.ApplyLearned(r)
    emul = _forward(r, nbr, feats, W, info, torch.float32, True).double().numpy()
    plain = _forward(r, nbr, feats, W, info, torch.float32, False).double().numpy()
    e_emul = np.linalg.norm(z - emul) / np.linalg.norm(emul)
    e_plain = np.linalg.norm(z - plain) / np.linalg.norm(plain)
    print(f"forward: vs BF16-emulating FP32 {e_emul:.2e}, vs plain FP32 {e_plain:.2e}")
    assert e_emul <= 2e-3, e_emul
    assert e_plain <= 3e-2, e_plain
    # positive homogeneity (no biases, ReLU): z(a r) = a z(r)
    z2 = slv.ApplyLearned(3.5 * r)
    assert np.linalg.norm(z2 - 3.5 * z) <= 1e-6 * np.linalg.norm(z2)


def test_learned_gradient_matches_autograd_and_finite_differences(cuda, stage):
    import torch
    s, op, slv, nbr, feats = stage
    info = slv.LearnedInfo()
    W = slv.LearnedWeights()
    # weights that are exact BF16 values, so that the FP32 masters the backward pass reads equal the BF16 copies
    rng = np.random.default_rng(9)
    Wb = [_bf16(torch.from_numpy(w + 0.05 * rng.standard_normal(w.shape).astype(np.float32) * np.abs(w).mean()))
          .numpy() for w in W]
    Wb[0][info["F"]:, :] = 0.0
    Wb[2][:, info["Np"]:] = 0.0
    slv.SetLearnedWeights(*Wb)
    assert all(np.array_equal(a, b) for a, b in zip(slv.LearnedWeights(), Wb))
    r = rng.standard_normal(s.N)
    loss_gpu, g = slv.LearnedGradient(r)

    # the operator the stage is trained on: the solver's (transformed) matrix
    Aop = op.OperatorMatrix
    from helpers import VarBsr
    v = VarBsr(Np=s.Np, row_ptr=s.row_ptr, col_idx=s.col_idx, values=Aop.read_values(),
               nspc=np.ones(s.nb, np.int32), rhs=np.zeros(s.N))
    Asp = v.to_scipy().tocsr()
    Ad = torch.from_numpy(Asp.toarray())
    rt = torch.from_numpy(r)

    def loss(Ws):
        z = _forward(r, nbr, feats, Ws, info, torch.float64, False)
        return (z @ (Ad @ z) - 2.0 * (z @ rt)) / (rt @ rt)

    Wt = [torch.from_numpy(w.astype(np.float64)).requires_grad_(True) for w in Wb]
    L = loss(Wt)
    L.backward()
    gt = np.concatenate([w.grad.numpy().ravel() for w in Wt])
    gg = np.concatenate([a.astype(np.float64).ravel() for a in g])
    e_grad = np.linalg.norm(gg - gt) / np.linalg.norm(gt)
    e_loss = abs(loss_gpu - L.item()) / abs(L.item())
    print(f"gradient vs FP64 autograd {e_grad:.2e}, loss {e_loss:.2e}")
    assert e_grad <= 3e-2, e_grad
    assert e_loss <= 3e-2, e_loss
    # central finite differences of the FP64 loss against the GPU gradient, along directions made of the descent
    # direction plus random components (so that the directional derivative is not a cancellation)
    with torch.no_grad():
        base = [torch.from_numpy(w.astype(np.float64)) for w in Wb]
        gnorm = float(np.linalg.norm(gt))
        for k in range(3):
            D = []
            for w in Wt:
                rd = torch.from_numpy(rng.standard_normal(tuple(w.shape)))
                D.append(w.grad / gnorm + 0.5 * rd / float(np.sqrt(gt.size)))
            D[0][info["F"]:, :] = 0.0
            D[2][:, info["Np"]:] = 0.0
            eps = 1e-5
            lp = loss([b + eps * d for b, d in zip(base, D)]).item()
            lm = loss([b - eps * d for b, d in zip(base, D)]).item()
            fd = (lp - lm) / (2 * eps)
            dd = sum(float((torch.from_numpy(a.astype(np.float64)) * d).sum()) for a, d in zip(g, D))
            print(f"direction {k}: finite difference {fd:.6e}, GPU gradient {dd:.6e}")
            assert abs(fd - dd) <= 3e-2 * abs(fd), (fd, dd)


def test_training_collects_requested_pairs(cuda):
    s = A.variable_coeff_3d(6, 2, seed=4)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    op.SetCellGraph(s.grid.face_neighbours(), A.log_coeff_features(s))
    slv = FGMRESConfig(ConvergenceCriterion=1e-10, termination="relative", Learned="fgmres", LearnedPairs=200,
                       Preconditioners=[PmgConfig(DegreeHierarchy=(10, 4, 1), CoarseTolerance=1e-2)]
                       ).CreateInstance(op)
    loss = slv.TrainLearned(n_rhs=40, steps=40, lr=1e-3, seed=2)
    assert np.isfinite(loss)
    assert slv.LearnedInfo()["pairs"] == 200
    x = np.zeros(s.N)
    slv.Solve(x, s.rhs)
    assert slv.Converged
    slv.Dispose()
    op.Dispose()


def test_learned_forward_twenty_modes(cuda):
    """Np = 20 (p = 3): the output layer has two 16-column halves in tensor memory; the forward pass against the
    BF16-emulating PyTorch evaluation."""
    import torch
    s = A.poisson_3d(5, 3, seed=2)
    op = MultigridOperator(BlockMsrMatrix.from_system(s))
    nbr = s.grid.face_neighbours()
    op.SetCellGraph(nbr)
    slv = FGMRESConfig(Learned="fgmres", Preconditioners=[PmgConfig(DegreeHierarchy=(20, 10, 4))]).CreateInstance(op)
    info = slv.LearnedInfo()
    assert info["Np"] == 20 and info["Op"] == 32 and info["F"] == 140
    W = slv.LearnedWeights()
    r = np.random.default_rng(8).standard_normal(s.N)
    z = slv.ApplyLearned(r)
    emul = _forward(r, nbr, np.zeros((s.nb, 0), np.float32), W, info, torch.float32, True).double().numpy()
    e = np.linalg.norm(z - emul) / np.linalg.norm(emul)
    assert e <= 2e-3, e
    slv.Dispose()
    op.Dispose()
