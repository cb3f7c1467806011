"""The engine's FP64 direct sums (csrc/direct.cu) pinned against the CPU oracle.

The large-configuration accuracy figures (bench.py, the large point-set tests, the tuner's error
gate) compare the engine with nnb_direct_type{1,2,3}_f64 on sampled outputs, because the CPU
oracle cannot sum 1e8 points in a test. This file pins those GPU sums to the oracle's FP64
direct NUDFT (oracle/nufft_oracle.cpp, restating the reference test oracle
tests/nuft_direct_kernels.cpp:73-293): 2e4 points, 1D/2D/3D, both signs, odd and even mode
counts, coordinates outside [-pi, pi), relative difference <= 1e-12 over every output.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

M = 20000
MODES = {1: [(101,), (100,)], 2: [(31, 24), (24, 31)], 3: [(9, 10, 11), (12, 7, 8)]}


def _mode_indices(modes):
    """Every mode of the CMCL box (k_d = -N_d/2 ...), x fastest, as an (S, dim) int64 array."""
    grids = np.meshgrid(*[np.arange(n) - n // 2 for n in modes], indexing="ij")
    return np.stack([g.transpose(tuple(reversed(range(len(modes))))).reshape(-1)
                     for g in grids], axis=1).astype(np.int64)


@pytest.mark.parametrize("sign", [-1, 1])
@pytest.mark.parametrize("dim,which", [(d, i) for d in (1, 2, 3) for i in (0, 1)])
def test_direct_type1_matches_oracle(dim, which, sign, cuda, engine, oracle):
    torch = cuda
    modes = MODES[dim][which]
    rng = np.random.default_rng(100 + 10 * dim + which)
    x = [rng.uniform(-3 * np.pi, 3 * np.pi, M) for _ in range(dim)]
    c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    ref = oracle.direct_type1(sign, x, c, list(modes)).reshape(-1)
    kidx = _mode_indices(modes)
    assert kidx.shape[0] == ref.size
    out = torch.empty(kidx.shape[0], dtype=torch.complex128, device="cuda")
    engine.direct_type1_f64(sign, [torch.from_numpy(a).cuda() for a in x],
                            torch.from_numpy(c).cuda(), torch.from_numpy(kidx).cuda(), out)
    got = out.cpu().numpy()
    assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("sign", [-1, 1])
@pytest.mark.parametrize("dim,which", [(d, i) for d in (1, 2, 3) for i in (0, 1)])
def test_direct_type2_matches_oracle(dim, which, sign, cuda, engine, oracle):
    torch = cuda
    modes = MODES[dim][which]
    rng = np.random.default_rng(200 + 10 * dim + which)
    x = [rng.uniform(-3 * np.pi, 3 * np.pi, M) for _ in range(dim)]
    nm = int(np.prod(modes))
    f = rng.standard_normal(nm) + 1j * rng.standard_normal(nm)
    ref = oracle.direct_type2(sign, list(modes), f, x)
    out = torch.empty(M, dtype=torch.complex128, device="cuda")
    pidx = torch.arange(M, dtype=torch.int64, device="cuda")
    engine.direct_type2_f64(sign, list(modes), torch.from_numpy(f).cuda(),
                            [torch.from_numpy(a).cuda() for a in x], pidx, out)
    got = out.cpu().numpy()
    assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)


@pytest.mark.parametrize("sign", [-1, 1])
@pytest.mark.parametrize("dim", [1, 2, 3])
def test_direct_type3_matches_oracle(dim, sign, cuda, engine, oracle):
    torch = cuda
    rng = np.random.default_rng(300 + dim)
    K = 2000
    x = [rng.uniform(-30.0, 30.0, M) for _ in range(dim)]
    s = [rng.uniform(-10.0, 10.0, K) for _ in range(dim)]
    c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    ref = oracle.direct_type3(sign, x, c, s)
    out = torch.empty(K, dtype=torch.complex128, device="cuda")
    tidx = torch.arange(K, dtype=torch.int64, device="cuda")
    engine.direct_type3_f64(sign, [torch.from_numpy(a).cuda() for a in x],
                            torch.from_numpy(c).cuda(), [torch.from_numpy(a).cuda() for a in s],
                            tidx, out)
    got = out.cpu().numpy()
    assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref)


def test_direct_type1_sampled_subset_matches_full_box(cuda, engine, oracle):
    """Sampling: the engine sums at arbitrary (repeated, unordered) mode indices, as the bench
    and the large tests use it."""
    torch = cuda
    modes = (16, 12, 10)
    rng = np.random.default_rng(7)
    x = [rng.uniform(-np.pi, np.pi, M) for _ in range(3)]
    c = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    full = oracle.direct_type1(-1, x, c, list(modes)).reshape(-1)
    kall = _mode_indices(modes)
    pick = rng.integers(0, full.size, 3000)
    out = torch.empty(pick.size, dtype=torch.complex128, device="cuda")
    engine.direct_type1_f64(-1, [torch.from_numpy(a).cuda() for a in x],
                            torch.from_numpy(c).cuda(),
                            torch.from_numpy(np.ascontiguousarray(kall[pick])).cuda(), out)
    ref = full[pick]
    assert np.linalg.norm(out.cpu().numpy() - ref) <= 1e-12 * np.linalg.norm(ref)
