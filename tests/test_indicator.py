"""Learned troubled-cell indicator: the CPU oracle (oracle/mlp_oracle.py) pinned by finite differences and
BF16 rounding cases, then the library's feature, forward (FP32 and tensor-core BF16), gradient and Adam
kernels against it, and the limiter gating inside the step.

Tolerances: features bit-exact (FP64 arithmetic with explicit roundings on both sides); FP32 forward
1e-5 on p; tensor-core forward within 5e-3 of the BF16-emulating oracle (mean difference below 2e-4:
only the FP32 accumulation order differs, which can flip a BF16 rounding of a hidden unit); gradient
max|g - g_oracle| <= 1e-4 max|g_oracle|; one Adam step 1e-6 relative."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

from dgswemv2_b200 import Problem, _lib, configs, mesh_topology

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import mlp_oracle as mo  # noqa: E402


# ---------------------------------------------------------------------------------------------- CPU


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    P = mo.init_params(1).astype(np.float64)
    P[mo.OFF_B1:mo.OFF_W2] = rng.normal(0, 0.1, mo.N_H)
    X = rng.normal(0, 1, (37, mo.N_IN))
    y = (rng.uniform(size=37) < 0.3).astype(np.float64)
    loss, g = mo.loss_and_grad(P, X, y, pos_weight=2.5)
    idx = np.concatenate([rng.choice(mo.N_PARAM, 60, replace=False), [mo.OFF_B3]])
    h = 1e-6
    for i in idx:
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += h
        Pm[i] -= h
        fd = (mo.loss_and_grad(Pp, X, y, 2.5)[0] - mo.loss_and_grad(Pm, X, y, 2.5)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, fd, g[i])


def test_bf16_rounding_cases():
    one = np.float32(1.0)
    half_ulp = np.float32(1.0 + 2.0 ** -8)  # halfway between 1 and the next BF16: ties to even -> 1
    above = np.float32(1.0 + 3 * 2.0 ** -9)  # above halfway -> 1 + 2^-7
    odd_half = np.float32(1.0 + 2.0 ** -7 + 2.0 ** -8)  # halfway from an odd mantissa -> rounds up
    out = mo.bf16_round(np.array([one, half_ulp, above, odd_half, -above], np.float32))
    assert list(out) == [1.0, 1.0, 1.0 + 2.0 ** -7, 1.0 + 2.0 ** -6, -(1.0 + 2.0 ** -7)]


def test_oracle_features_by_hand():
    """One element with two neighbours and a land face: the definition evaluated by hand."""
    q = np.zeros((3, 3, 3))         # [element][variable][mode]
    q[0, 0, :] = [1.0, 0.5, -0.2]   # ze of element 0: mean 1, slopes 0.5, -0.2
    q[0, 1, 0] = 0.25               # qx mean of element 0
    q[1, 0, 0], q[2, 0, 0] = 1.5, 0.0
    nbr = np.array([[1, 2, -1], [0, -1, -1], [0, -1, -1]])
    btype = np.array([[128, 128, 0], [128, 0, 0], [128, 0, 0]])
    wet = np.array([1, 1, 1])
    xyz = np.array([[0.0, 0.0, 2.0], [1.0, 0.0, 2.0], [0.0, 1.0, 2.0], [1.0, 1.0, 2.0]])
    en = np.array([[0, 1, 2], [1, 3, 2], [0, 2, 3]])
    g, M = 9.81, 0.5
    F, ok = mo.features(q, wet, nbr, btype, xyz, en, g, M)
    assert ok.all()
    ic = 1.0 / np.sqrt(g * 3.0)  # depth H = 1 + 2
    # common scale: ze slopes 0.5, -0.2, ze differences 0.5, -1, 0, qx differences -0.25 c^-1 -> s = 1;
    # r2 = (1/18 + 5/36 + 5/36) / 3 = 1/9 for the unit right triangle
    assert np.allclose(F[0, :3], [1.0 / (1.0 + M / 9.0), 0.25 / 3.0 * ic, 0.0])
    assert np.allclose(F[0, 3:8], [0.5, -0.2, 0.5, -1.0, 0.0])
    assert np.allclose(F[0, 8:13], [0.0, 0.0, -0.25 * ic, -0.25 * ic, 0.0])
    assert np.all(F[0, 13:] == 0)
    wet2 = np.array([1, 0, 1])
    assert list(mo.features(q, wet2, nbr, btype, xyz, en, g, M)[1]) == [False, False, True]
    # the raw set: element 0's modes of ze, qx, qy, then per face the neighbour means (own at the land face)
    R, okr = mo.features(q, wet, nbr, btype, xyz, en, g, M, fset=1)
    assert np.array_equal(okr, ok)
    assert np.allclose(R[0, :9], [1.0, 0.5, -0.2, 0.25, 0.0, 0.0, 0.0, 0.0, 0.0])
    assert np.allclose(R[0, 9:], [1.5, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 0.25, 0.0])


# ---------------------------------------------------------------------------------------------- GPU


def _dev(a, dtype=None):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a if dtype is None else a.astype(dtype))).cuda()


def _bowl(nq=24, precision="fp32", seed=3):
    mesh, cfg = configs.bowl_humps(nq=nq, seed=seed, precision=precision)
    return mesh, cfg


@pytest.mark.gpu
@pytest.mark.parametrize("precision,fset", [("fp32", 0), ("fp64", 0), ("fp64", 1)])
def test_features_match_oracle_bit_exact(precision, fset):
    """Both feature sets: 0 the characteristic set, 1 the raw modal coefficients and neighbour means."""
    import torch

    mesh, cfg = _bowl(precision=precision)
    P = Problem(cfg, mesh)
    P.step_serial(30)
    P.set_indicator_features(fset)
    feat = torch.empty((P.ne, 18), dtype=torch.float32, device="cuda")
    ok = torch.empty(P.ne, dtype=torch.uint8, device="cuda")
    P.indicator_features(feat.data_ptr(), ok.data_ptr())
    nbr, bt, _, _ = mesh_topology(mesh)
    F, okr = mo.features(P.get_state(), P.get_wet(), nbr, bt, mesh.node_xyz, mesh.elem_nodes, cfg.g, cfg.sl_M,
                         fset=fset)
    assert okr.sum() > P.ne // 4 and (~okr).sum() > 0  # wet and dry cells both present
    assert np.array_equal(ok.cpu().numpy() != 0, okr)
    assert np.array_equal(feat.cpu().numpy(), F)


@pytest.mark.gpu
def test_features_with_tide_flow_and_levee_faces():
    """Features on a mesh with tide and land boundaries and levee interfaces (the element across a levee
    is a neighbour; tide faces are boundary objects like land faces), bit-exact against the oracle."""
    import torch

    from dgswemv2_b200 import configs

    mesh, cfg = configs.levee_channel(p=1, dt=2.0, dry_right=True, limiter=True, precision="fp32")
    P = Problem(cfg, mesh)
    P.step_serial(500)
    feat = torch.empty((P.ne, 18), dtype=torch.float32, device="cuda")
    ok = torch.empty(P.ne, dtype=torch.uint8, device="cuda")
    P.indicator_features(feat.data_ptr(), ok.data_ptr())
    nbr, bt, _, _ = mesh_topology(mesh)
    F, okr = mo.features(P.get_state(), P.get_wet(), nbr, bt, mesh.node_xyz, mesh.elem_nodes, cfg.g, cfg.sl_M)
    tide_elems = np.any(bt == 1, axis=1)
    assert okr[tide_elems].any()  # cells on the tide boundary are eligible
    assert np.array_equal(ok.cpu().numpy() != 0, okr)
    assert np.array_equal(feat.cpu().numpy(), F)


def _random_batch(n, seed):
    rng = np.random.default_rng(seed)
    X = rng.uniform(-1, 1, (n, 18)).astype(np.float32)
    X[:, 0] = rng.uniform(0, 1, n)
    y = (rng.uniform(size=n) < 0.2).astype(np.uint8)
    P = mo.init_params(seed)
    P[mo.OFF_B1:mo.OFF_W2] = rng.normal(0, 0.05, 64)
    P[mo.OFF_B2:mo.OFF_W3] = rng.normal(0, 0.05, 64)
    P[mo.OFF_B3] = -0.3
    return X, y, P


@pytest.mark.gpu
@pytest.mark.parametrize("n", [1, 1000, 128 * 300 + 5])
def test_forward_fp32_and_tensor_cores(n):
    from dgswemv2_b200 import indicator

    X, _, P = _random_batch(n, 7)
    xd, pd = _dev(X), _dev(P)
    p32 = indicator.forward(xd, pd, tensor_cores=False).cpu().numpy()
    ptc = indicator.forward(xd, pd, tensor_cores=True).cpu().numpy()
    ref = mo.forward(P, X)[0]
    assert np.max(np.abs(p32 - ref)) <= 1e-5
    refb = mo.forward_bf16(P, X)
    assert np.max(np.abs(ptc - refb)) <= 5e-3
    assert np.mean(np.abs(ptc - refb)) <= 2e-4
    assert np.max(np.abs(ptc - ref)) <= 5e-2  # BF16 inputs/weights against exact FP64


@pytest.mark.gpu
def test_gradient_matches_oracle_and_is_deterministic():
    import torch

    from dgswemv2_b200 import indicator

    X, y, P = _random_batch(5000, 11)
    T = indicator.Trainer(P, max_batch=8192)
    g1 = T.grad(_dev(X), _dev(y), 3.0).cpu().numpy().copy()
    loss1 = float(T.loss.item())
    g2 = T.grad(_dev(X), _dev(y), 3.0).cpu().numpy().copy()
    loss_ref, g_ref = mo.loss_and_grad(P, X, y, 3.0)
    assert np.array_equal(g1, g2)
    assert abs(loss1 - loss_ref) <= 1e-5 * abs(loss_ref)
    assert np.max(np.abs(g1 - g_ref)) <= 1e-4 * np.max(np.abs(g_ref))
    # per block: every parameter group is exercised
    for a, b in [(mo.OFF_W1, mo.OFF_B1), (mo.OFF_W2, mo.OFF_B2), (mo.OFF_W3, mo.OFF_B3)]:
        assert np.max(np.abs(g_ref[a:b])) > 0
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_adam_step_matches_oracle():
    from dgswemv2_b200 import indicator

    X, y, P = _random_batch(2000, 5)
    T = indicator.Trainer(P, lr=1e-3, max_batch=4096)
    Pk, m, v = P.astype(np.float64), np.zeros(mo.N_PARAM), np.zeros(mo.N_PARAM)
    for t in range(1, 4):
        g = T.grad(_dev(X), _dev(y), 2.0).cpu().numpy().astype(np.float64)
        T.step(_dev(X), _dev(y), 2.0)
        Pk, m, v = mo.adam(Pk, m, v, g, t, 1e-3)
    got = T.params().astype(np.float64)
    assert np.max(np.abs(got - Pk)) <= 1e-6 * np.max(np.abs(Pk)) + 1e-7


@pytest.mark.gpu
def test_stage_record_is_the_plain_stage():
    """stage_record advances exactly like stage_serial and labels the cells the limiter looked at with
    its own decisions (255 elsewhere)."""
    import torch

    mesh, cfg = _bowl(nq=32)
    A, B = Problem(cfg, mesh), Problem(cfg, mesh)
    feat = torch.empty((A.ne, 18), dtype=torch.float32, device="cuda")
    lab = torch.empty(A.ne, dtype=torch.uint8, device="cuda")
    seen = 0
    for _ in range(40):
        A.stage_record(feat.data_ptr(), lab.data_ptr())
        B.stage_serial()
        lb = lab.cpu().numpy()
        lim = B.get_limited()
        assert set(np.unique(lb)) <= {0, 1, 255}
        look = lb != 255
        assert np.array_equal(lb[look], lim[look]) and not lim[~look].any()
        seen += int(lb[look].sum())
    assert np.array_equal(A.get_state(), B.get_state())
    assert seen > 0


def _gate_params(b3):
    P = np.zeros(mo.N_PARAM, np.float32)
    P[mo.OFF_B3] = b3
    return P


@pytest.mark.gpu
def test_gate_sending_everything_is_the_plain_limiter():
    mesh, cfg = _bowl(nq=32)
    A, B = Problem(cfg, mesh), Problem(cfg, mesh)
    A.set_indicator(_gate_params(50.0), confidence=0.9, mode=1)
    n_lim = 0
    for _ in range(60):
        A.stage_serial()
        B.stage_serial()
        assert np.array_equal(A.get_limited(), B.get_limited())
        n_lim += int(B.get_limited().sum())
    assert np.array_equal(A.get_state(), B.get_state())
    considered, sent, limited, missed = A.indicator_stats()
    assert considered > 0 and sent == considered and missed == 0 and limited == n_lim and n_lim > 0


@pytest.mark.gpu
def test_gate_sending_nothing_counts_every_limited_cell_as_missed():
    mesh, cfg = _bowl(nq=32)
    S, B = Problem(cfg, mesh), Problem(cfg, mesh)
    S.set_indicator(_gate_params(-50.0), confidence=0.9, mode=2)  # shadow: plain limiter decides, no write
    N = Problem(cfg, mesh)
    N.set_indicator(_gate_params(-50.0), confidence=0.9, mode=1)  # gate: the limiter visits nothing
    for _ in range(10):
        S.stage_serial()
        B.stage_serial()
        N.stage_serial()
        S_lim = S.get_limited()
        assert not S_lim.any()
    considered, sent, limited, missed = S.indicator_stats()
    assert sent == 0 and limited == 0 and missed > 0
    assert N.indicator_stats()[1] == 0 and not N.get_limited().any()
    # without limiting the two unlimited runs agree with each other
    assert np.array_equal(S.get_state(), N.get_state())


@pytest.mark.gpu
def test_trained_indicator_on_the_thacker_bowl():
    """The committed network (dgswemv2_b200/data/indicator_p1.f32) on the Thacker bowl at 256 x 256 quads,
    100 SSP-RK2 steps, FP32 bulk: the gate sends fewer cells to the limiter than the plain limiter visits,
    misses at most 2 % of the cells the plain limiter changes (shadow mode counts them), and the L2 error
    against the analytic solution stays within 0.1 % of the plain limiter's."""
    from dgswemv2_b200 import indicator

    W = indicator.load_weights()
    mesh, cfg = configs.config3(nq=256, dt=0.25, precision="fp32")
    runs = {}
    for mode in (0, 1, 2):
        P = Problem(cfg, mesh)
        if mode:
            P.set_indicator(W, confidence=0.9, mode=mode)
        P.step_serial(100)
        runs[mode] = (P.compute_residual_L2(), P.indicator_stats() if mode else None)
    considered, sent, limited, missed = runs[2][1]
    assert runs[1][1][1] == sent and sent < considered
    assert missed <= 0.02 * (limited + missed)
    assert abs(runs[1][0] / runs[0][0] - 1) <= 1e-3
