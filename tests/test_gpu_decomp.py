"""Slab decomposition on one GPU: three contexts, each advancing its slab
(bbw_set_compute_range) with its halo refreshed after every stage through
bbw_gather_elements / bbw_scatter_elements; the owned elements must equal
the single-context run bit for bit."""
import numpy as np
import pytest

from bbwadg_b200 import WaveSolver, make_problem
from bbwadg_b200.decomp import LocalExchange, local_solver, local_state, run_decomposed, slab_partition

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("variant", ["nodal", "bb"])
@pytest.mark.parametrize("shots", [1, 2])
def test_three_slabs_equal_one_mesh(cuda, variant, shots):
    from bbwadg_b200 import RK4A, RK4B
    p = make_problem(4, 4, variant=variant, c2="sine", c2_jitter=0.5, seed=7)
    rng = np.random.default_rng(2)
    Q0 = np.stack([p.Q0 + 0.01 * s * rng.standard_normal(p.Q0.size) for s in range(shots)])
    Q0 = Q0.astype(np.float32).reshape(shots, p.K, -1)
    ref = WaveSolver(p)
    ref.set_shots(shots)
    ref.set_data(Q0)
    for _ in range(4):
        for i in range(5):
            ref.rk_stage(np.float32(RK4A[i]), np.float32(RK4B[i]), p.dt, 0.0)
    full = ref.get_data().reshape(shots, p.K, -1)
    ref.close()
    parts = slab_partition(p, 3)
    solvers = []
    for part in parts:
        s = local_solver(p, part)
        s.set_shots(shots)
        s.set_compute_range(part.Kc)
        s.set_data(np.stack([local_state(p, part, Q0[k]) for k in range(shots)]))
        solvers.append(s)
    run_decomposed(solvers, LocalExchange(parts, solvers), p.dt, 4)
    for part, s in zip(parts, solvers):
        q = s.get_data().reshape(shots, part.K, -1)[:, :part.Kc]
        assert np.array_equal(q, full[:, part.owned])
        s.close()


@pytest.mark.parametrize("shots", [1, 2])
def test_overlapped_exchange_equals_one_mesh(cuda, shots):
    """Interface elements first, halo exchange on side streams beside the
    interior elements (bbw_stage_part / bbw_move_elements / bbw_stage_commit):
    bit for bit the single-context run."""
    from bbwadg_b200 import RK4A, RK4B
    p = make_problem(4, 4, c2="sine", c2_jitter=0.5, seed=9)
    rng = np.random.default_rng(5)
    Q0 = np.stack([p.Q0 + 0.01 * s * rng.standard_normal(p.Q0.size) for s in range(shots)])
    Q0 = Q0.astype(np.float32).reshape(shots, p.K, -1)
    ref = WaveSolver(p)
    ref.set_shots(shots)
    ref.set_data(Q0)
    for _ in range(3):
        for i in range(5):
            ref.rk_stage(np.float32(RK4A[i]), np.float32(RK4B[i]), p.dt, 0.0)
    full = ref.get_data().reshape(shots, p.K, -1)
    ref.close()
    parts = slab_partition(p, 3, interface_first=True)
    assert all(0 < part.Ki < part.Kc for part in parts)
    solvers = []
    for part in parts:
        s = local_solver(p, part)
        s.set_shots(shots)
        s.set_compute_range(part.Kc)
        s.set_data(np.stack([local_state(p, part, Q0[k]) for k in range(shots)]))
        solvers.append(s)
    run_decomposed(solvers, LocalExchange(parts, solvers), p.dt, 3, overlap=True)
    for part, s in zip(parts, solvers):
        q = s.get_data().reshape(shots, part.K, -1)[:, :part.Kc]
        assert np.array_equal(q, full[:, part.owned])
        s.close()


def test_stage_part_arguments_are_validated(cuda):
    from bbwadg_b200._lib import BBWError
    p = make_problem(3, 2)
    s = WaveSolver(p)
    for k0, k1 in ((-1, 4), (4, 4), (0, p.K + 1)):
        with pytest.raises(BBWError):
            s.stage_part(0.0, 1.0, p.dt, k0, k1)
    s.close()


def test_compute_range_is_validated(cuda):
    from bbwadg_b200._lib import BBWError
    p = make_problem(3, 2)
    s = WaveSolver(p)
    for bad in (0, p.K + 1):
        with pytest.raises(BBWError):
            s.set_compute_range(bad)
    s.close()


@pytest.mark.parametrize("variant", ["nodal", "bb"])
@pytest.mark.parametrize("N", [3, 5])
def test_windows_equal_whole_stage(cuda, variant, N):
    """Element windows that start inside an element tile ([0,37), [37,200),
    [200,K)) advance the same elements as one whole-mesh stage, bit for bit,
    for every fused-stage variant (element tile, warps, operators in shared
    memory, double buffering) the device holds."""
    from bbwadg_b200 import RK4A, RK4B
    from bbwadg_b200._lib import BBWError
    p = make_problem(N, 4, variant=variant, c2="sine", c2_jitter=0.5, seed=11)
    ran = 0
    for tile in (32, 16):
      for warps in (8, 16):
        for ops in (True, False):
            for pipe in (True, False):
                a, b = WaveSolver(p), WaveSolver(p)
                try:
                    a.set_config(warps, ops, pipe, tile)
                    b.set_config(warps, ops, pipe, tile)
                except BBWError:  # this variant does not fit in shared memory
                    a.close(), b.close()
                    continue
                for i in range(5):
                    fa, fb = np.float32(RK4A[i]), np.float32(RK4B[i])
                    a.rk_stage(fa, fb, p.dt, 0.0)
                    for k0, k1 in ((0, 37), (37, 200), (200, p.K)):
                        b.stage_part(fa, fb, p.dt, k0, k1)
                    b.stage_commit()
                cfg = (warps, ops, pipe, tile)
                assert np.array_equal(a.get_data(), b.get_data()), cfg
                assert np.array_equal(a.get_residual(), b.get_residual()), cfg
                a.close(), b.close()
                ran += 1
    assert ran >= 4
