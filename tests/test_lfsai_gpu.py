"""Learned FSAI on the GPU against its FP64 CPU reference (oracle/lfsai_ref.py).

* features: FP32 on the GPU vs FP64, relative 1e-6;
* network outputs and the gradients of the probe loss and of the Kaporin
  loss: the GPU accumulates in FP32 and rounds layer inputs to BF16 from
  FP32 values, the reference from FP64 ones (and the tensor-core backward
  rounds the deltas to BF16 too), so a few inputs land on the other side of
  a BF16 rounding boundary; the bound is on the relative 2-norm of the
  difference (2e-2) and on the loss (1e-4 relative);
* the reference backpropagation itself is checked against central finite
  differences (BF16 rounding off) on the CPU in test_lfsai_reference_fd;
* the tensor-core forward and backward agree with the CUDA-core layers;
* training lowers the loss and the iteration count below the warm start,
  and the trained preconditioner needs fewer CG iterations than Jacobi on
  an unseen problem.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def small_problem(N=24, seed=3):
    from tnl_b200 import generators as g

    return g.diffusion_2d(N, 0.1, 1.5, seed)


@pytest.mark.parametrize("level", [0, 1])
def test_features_and_outputs_match_reference(level):
    from oracle import lfsai_ref as R
    import tnl_b200
    from tnl_b200.lfsai import LearnedFSAI

    A = small_problem()
    M = tnl_b200.SparseMatrix.from_csr(A)
    net = LearnedFSAI(seed=5, level=level)
    theta = net.params().astype(np.float64)
    assert np.array_equal(net.params(), R.init_params(5).astype(np.float32))
    f_gpu, o_gpu = net.evaluate(M)
    f_ref, s, pat = R.features(A, level=level)
    assert np.allclose(f_gpu, f_ref, rtol=1e-6, atol=1e-7)
    o_ref, _ = R.forward(theta, f_ref)
    rel = np.linalg.norm(o_gpu - o_ref) / np.linalg.norm(o_ref)
    assert rel < 2e-2, rel


@pytest.mark.parametrize("level", [0, 1])
@pytest.mark.parametrize("tensor_cores", [True, False])
def test_gradient_matches_reference(level, tensor_cores):
    """Probe-loss and Kaporin-loss gradients of the GPU (tensor-core or
    CUDA-core layers) against the FP64 reference."""
    from oracle import lfsai_ref as R
    import tnl_b200
    from tnl_b200.lfsai import LearnedFSAI

    A = small_problem(20, 4)
    M = tnl_b200.SparseMatrix.from_csr(A)
    net = LearnedFSAI(seed=9, level=level, tensor_cores=tensor_cores)
    theta = net.params().astype(np.float64)
    Z = LearnedFSAI.probes(M, 4, seed=1, residual_share=0.5)
    loss = net.gradient(M, Z)
    g_gpu = net.grad().astype(np.float64)
    L_ref, g_ref = R.loss_and_grad(theta, A, Z.cpu().numpy().T.copy(), level)
    assert loss == pytest.approx(L_ref, rel=1e-4)
    rel = np.linalg.norm(g_gpu - g_ref) / np.linalg.norm(g_ref)
    assert rel < 2e-2, rel
    loss = net.gradient(M, None, mode=2)
    g_gpu = net.grad().astype(np.float64)
    K_ref, g_ref = R.kaporin_and_grad(theta, A, level)
    assert loss == pytest.approx(K_ref, rel=1e-4, abs=1e-6)
    rel = np.linalg.norm(g_gpu - g_ref) / np.linalg.norm(g_ref)
    assert rel < 2e-2, rel


def test_level1_classical_fsai_matches_reference():
    """Classical FSAI on the level-1 pattern (tnlb_precond_create_fsai):
    pattern and values of G against the FP64 reference's local solves."""
    from oracle import lfsai_ref as R
    import tnl_b200

    A = small_problem(30, 6)
    M = tnl_b200.SparseMatrix.from_csr(A)
    P = tnl_b200.FSAI(level=1)
    P.update(M)
    rp, cols, vals = P.factor(0)
    pat = R.pattern(A, 1)
    assert np.array_equal(np.diff(rp), [len(J) for J in pat])
    assert np.array_equal(cols, np.concatenate([np.array(J) for J in pat]))
    ref = R.fsai_classical(A, 1)
    assert np.allclose(vals, ref, rtol=1e-10, atol=1e-12)


def test_warm_start_and_training_lower_the_loss():
    from tnl_b200.lfsai import LearnedFSAI, diffusion_problem

    train = [diffusion_problem(48, s) for s in range(4)]
    net = LearnedFSAI(seed=1)
    fit = net.fit_classical(train, steps=150, lr=3e-3)
    assert fit[-1] < 0.2 * fit[0]
    probes = [LearnedFSAI.probes(M, 8, 100 + i) for i, M in enumerate(train)]
    before = np.mean([net.gradient(M, Z) for M, Z in zip(train, probes)])
    net.train(train, steps=200, nprobes=8, lr=5e-4)
    after = np.mean([net.gradient(M, Z) for M, Z in zip(train, probes)])
    assert after < before


def test_learned_preconditioner_beats_jacobi_on_unseen_problem():
    import tnl_b200
    from tnl_b200 import generators as g
    from tnl_b200.lfsai import LearnedFSAI, diffusion_problem

    train = [diffusion_problem(64, s) for s in range(6)]
    net = LearnedFSAI(seed=2)
    net.fit_classical(train, steps=200, lr=3e-3)
    net.train(train, steps=150, nprobes=8, lr=5e-4)
    M = diffusion_problem(96, 1234)
    b = torch.tensor(g.uniform_vector(M.getRows(), 1), device="cuda")
    its = {}
    for name in ("jacobi", "learned"):
        S = tnl_b200.CG()
        S.setMatrix(M)
        S.setConvergenceResidue(1e-8)
        P = tnl_b200.Diagonal() if name == "jacobi" else None
        if P is not None:
            P.update(M)
        else:
            P = net.preconditioner(M)
        S.setPreconditioner(P)
        x = torch.zeros(M.getRows(), dtype=torch.float64, device="cuda")
        assert S.solve(b, x)
        its[name] = S.getIterations()
        assert tnl_b200.true_residual(M, b, x) < 1e-6
    assert its["learned"] < 0.8 * its["jacobi"], its


def test_mixed_precision_with_learned_preconditioner():
    import tnl_b200
    from tnl_b200 import generators as g
    from tnl_b200.lfsai import LearnedFSAI, diffusion_problem

    train = [diffusion_problem(48, s) for s in range(3)]
    net = LearnedFSAI(seed=4)
    net.fit_classical(train, steps=150, lr=3e-3)
    M = diffusion_problem(80, 77)
    A32 = tnl_b200.SparseMatrix(tnl_b200.CSR, torch.float32)
    A32.assign(M.segments.getOffsets(), M.getColumnIndexes().cpu().numpy(), M.getValues().cpu().numpy())
    P32 = net.preconditioner(A32)
    b = torch.tensor(g.uniform_vector(M.getRows(), 1), device="cuda")
    x = torch.zeros(M.getRows(), dtype=torch.float64, device="cuda")
    r = tnl_b200.solve_mixed(M, b, x, tol=1e-8, inner_tol=1e-4, inner=P32)
    assert r["converged"] and tnl_b200.true_residual(M, b, x) < 1e-8


def test_reliable_mixed_with_learned_preconditioner():
    """The learned FSAI (FP32) inside the reliable-update mixed PCG reaches
    the FP64 tolerance in fewer iterations than iterative refinement with
    it, and within 1.5x those of FP64 PCG with it (preconditioned residue
    1e-9)."""
    import tnl_b200
    from tnl_b200 import generators as g
    from tnl_b200.lfsai import LearnedFSAI, diffusion_problem

    train = [diffusion_problem(48, s) for s in range(3)]
    net = LearnedFSAI(seed=4)
    net.fit_classical(train, steps=150, lr=3e-3)
    M = diffusion_problem(80, 77)
    A32 = tnl_b200.SparseMatrix(tnl_b200.CSR, torch.float32)
    A32.assign(M.segments.getOffsets(), M.getColumnIndexes().cpu().numpy(), M.getValues().cpu().numpy())
    P32 = net.preconditioner(A32)
    P64 = net.preconditioner(M)
    b = torch.tensor(g.uniform_vector(M.getRows(), 1), device="cuda")
    S = tnl_b200.CG()
    S.setMatrix(M)
    S.setPreconditioner(P64)
    S.setup({"convergence-residue": 1e-9, "max-iterations": 20000})
    x64 = torch.zeros(M.getRows(), dtype=torch.float64, device="cuda")
    assert S.solve(b, x64)
    x = torch.zeros(M.getRows(), dtype=torch.float64, device="cuda")
    r = tnl_b200.solve_mixed_reliable(M, b, x, tol=1e-8, inner=P32)
    assert r["converged"] and tnl_b200.true_residual(M, b, x) < 1e-8
    assert r["iterations"] <= 1.5 * S.getIterations(), (r, S.getIterations())
    x2 = torch.zeros(M.getRows(), dtype=torch.float64, device="cuda")
    r2 = tnl_b200.solve_mixed_reliable(M, b, x2, tol=1e-8, inner=P32, vectors=torch.float64)
    assert r2["converged"] and tnl_b200.true_residual(M, b, x2) < 1e-8
    assert r2["iterations"] <= 1.5 * S.getIterations(), (r2, S.getIterations())
    xi = torch.zeros(M.getRows(), dtype=torch.float64, device="cuda")
    ir = tnl_b200.solve_mixed(M, b, xi, tol=1e-8, inner_tol=1e-4, inner=P32)
    assert ir["converged"] and r["iterations"] < ir["inner_iterations"], (r, ir)


def test_tensor_core_forward_matches_cuda_cores():
    """tcgen05 (BF16 in shared memory, FP32 accumulators in TMEM) against the
    CUDA-core layers: same BF16 operands, FP32 sums in another order."""
    from tnl_b200.lfsai import LearnedFSAI, diffusion_problem

    net = LearnedFSAI(seed=3, tensor_cores=False)
    for N in (16, 64, 181):  # 256, 4096 and 32761 rows (ragged last tile)
        M = diffusion_problem(N, 5 + N)
        _, o_cc = net.evaluate(M)
        net.set_tensor_cores(True)
        _, o_tc = net.evaluate(M)
        net.set_tensor_cores(False)
        rel = np.linalg.norm(o_tc - o_cc) / np.linalg.norm(o_cc)
        assert rel < 1e-3, (N, rel)
        assert np.max(np.abs(o_tc - o_cc)) < 1e-2


def test_tensor_core_backward_matches_cuda_cores():
    """The tcgen05 backward pass and weight gradients against the CUDA-core
    kernels on the same forward pass (the tensor-core path also rounds the
    deltas to BF16), for the probe loss and the Kaporin loss, on ragged row
    counts."""
    from tnl_b200.lfsai import LearnedFSAI, diffusion_problem

    net = LearnedFSAI(seed=11)
    net.fit_classical([diffusion_problem(32, 1)], steps=20, lr=3e-3)  # non-trivial deltas
    for N in (16, 64, 181):
        M = diffusion_problem(N, 7 + N)
        Z = LearnedFSAI.probes(M, 4, seed=N)
        for mode, probes in ((0, Z), (2, None)):
            net.set_tensor_cores(False)
            l_cc = net.gradient(M, probes, mode=mode)
            g_cc = net.grad().astype(np.float64)
            net.set_tensor_cores(True)
            l_tc = net.gradient(M, probes, mode=mode)
            g_tc = net.grad().astype(np.float64)
            assert l_tc == pytest.approx(l_cc, rel=1e-3, abs=1e-6), (N, mode)
            rel = np.linalg.norm(g_tc - g_cc) / np.linalg.norm(g_cc)
            assert rel < 1e-2, (N, mode, rel)


def _pcg_iterations(M, P, b):
    import tnl_b200

    S = tnl_b200.CG()
    S.setMatrix(M)
    S.setPreconditioner(P)
    S.setup({"convergence-residue": 1e-8, "max-iterations": 50000})
    x = torch.zeros(M.getRows(), dtype=torch.float64, device="cuda")
    assert S.solve(b, x)
    return S.getIterations()


def test_training_lowers_iterations_below_the_warm_start():
    """The warm start reproduces classical FSAI on A's own pattern; training
    on the Kaporin loss over the wider level-1 pattern must then cut the
    PCG iteration count on an unseen problem below the warm start's (and so
    below classical FSAI's on A's pattern)."""
    import tnl_b200
    from tnl_b200 import generators as g
    from tnl_b200.lfsai import LearnedFSAI, diffusion_problem

    train = [diffusion_problem(64, s) for s in range(8)]
    net = LearnedFSAI(seed=2)
    net.fit_classical(train, steps=400, lr=3e-3)
    M = diffusion_problem(128, 4321)
    b = torch.tensor(g.uniform_vector(M.getRows(), 1), device="cuda")
    warm = _pcg_iterations(M, net.preconditioner(M), b)
    P0 = tnl_b200.FSAI()
    P0.update(M)
    classical = _pcg_iterations(M, P0, b)
    assert warm <= 1.25 * classical, (warm, classical)
    hist = net.train_kaporin(train, steps=400, lr=1e-3)
    assert np.mean(hist[-8:]) < np.mean(hist[:8])
    trained = _pcg_iterations(M, net.preconditioner(M), b)
    assert trained < 0.95 * warm, (trained, warm, classical)


def _cd_problem(N, seed):
    import tnl_b200
    from tnl_b200 import generators as g

    return tnl_b200.SparseMatrix.from_csr(g.convection_diffusion_3d(N, seed=seed))


@pytest.mark.parametrize("tensor_cores", [True, False])
def test_two_factor_features_and_gradient_match_reference(tensor_cores):
    """The two-factor (nonsymmetric) form: features, and the probe-loss
    gradient through G_L and G_U (transposed products of G_L and A inside)
    against the FP64 reference."""
    from oracle import lfsai_ref as R
    from tnl_b200 import generators as g
    from tnl_b200.lfsai import LearnedFSAI
    import tnl_b200

    A = g.convection_diffusion_3d(6, seed=3)
    M = tnl_b200.SparseMatrix.from_csr(A)
    net = LearnedFSAI(seed=7, two_factor=True, tensor_cores=tensor_cores)
    f_gpu, _ = net.evaluate(M)
    f_ref, _, _ = R.features2(A)
    assert np.allclose(f_gpu, f_ref, rtol=1e-6, atol=1e-7)
    theta = net.params().astype(np.float64)
    Z = LearnedFSAI.probes(M, 4, seed=2, residual_share=0.0)
    loss = net.gradient(M, Z)
    g_gpu = net.grad().astype(np.float64)
    L_ref, g_ref = R.loss_and_grad2(theta, A, Z.cpu().numpy().T.copy())
    assert loss == pytest.approx(L_ref, rel=1e-4)
    rel = np.linalg.norm(g_gpu - g_ref) / np.linalg.norm(g_ref)
    assert rel < 2e-2, rel
    with pytest.raises(ValueError):
        net.gradient(M, None, mode=2)


def test_two_factor_learned_fsai_with_fgmres():
    """Warm start on the classical two-factor FSAI, then the probe loss on
    Rademacher vectors and BiCGStab residuals: the loss falls, and FGMRES(30)
    with the learned factors on an unseen convection-diffusion problem
    converges in fewer iterations than with Jacobi."""
    import tnl_b200
    from tnl_b200 import generators as g
    from tnl_b200.lfsai import LearnedFSAI

    train = [_cd_problem(16, s) for s in range(4)]
    net = LearnedFSAI(seed=3, two_factor=True)
    fit = net.fit_classical(train, steps=300, lr=3e-3)
    assert fit[-1] < 0.2 * fit[0]
    probes = [LearnedFSAI.probes(M, 8, 50 + i, symmetric=False) for i, M in enumerate(train)]
    before = np.mean([net.gradient(M, Z) for M, Z in zip(train, probes)])
    net.train(train, steps=120, nprobes=8, lr=2e-4)
    after = np.mean([net.gradient(M, Z) for M, Z in zip(train, probes)])
    assert after < before
    M = _cd_problem(24, 99)
    b = torch.tensor(g.uniform_vector(M.getRows(), 1), device="cuda")
    its = {}
    for name in ("jacobi", "learned"):
        S = tnl_b200.FGMRES()
        S.setMatrix(M)
        if name == "jacobi":
            P = tnl_b200.Diagonal()
            P.update(M)
        else:
            P = net.preconditioner(M)
        S.setPreconditioner(P)
        S.setup({"convergence-residue": 1e-8, "max-iterations": 20000, "gmres-restarting-min": 30,
                 "gmres-restarting-max": 30})
        x = torch.zeros(M.getRows(), dtype=torch.float64, device="cuda")
        assert S.solve(b, x), name
        its[name] = S.getIterations()
        assert tnl_b200.true_residual(M, b, x) < 1e-7
    assert its["learned"] < its["jacobi"], its
