"""Lockstep batches (h3d_lockstep_*): designs of uneven resolution and hierarchy
depth stepping through their V-cycles together, one launch per V-cycle step over
all of them, give the C, V-cycle counts, residual estimates and statuses of the
same designs solved one at a time, to the last bit; and C of a lockstep design
agrees with the FP64 oracle (elasticMatrix, homogenization.cu:464-575, solved to
relthres 1e-10) as the single-design solve does."""
import numpy as np
import pytest

import homo3d_b200 as H
from tests.conftest import smooth_density
from tests.test_gpu_parity import rel_err
from tests.test_gpu_solve import oracle_C

pytestmark = pytest.mark.gpu

# resolutions with 3, 4 and 5 grid levels and coarsest grids of 4^3, 6^3 and 7^3
# (each a size the reference's rounding keeps: 40 would become 48)
DESIGNS = [(16, 0, 0.2), (32, 1, 0.4), (24, 2, 0.3), (28, 3, 0.15), (16, 4, 0.5), (64, 5, 0.3), (48, 6, 0.35),
           (56, 7, 0.25)]


def _rho(torch, n, seed, vol):
    return torch.tensor(smooth_density(n, seed=seed, vol=vol), dtype=torch.float32, device="cuda")


def _same_stats(a, b):
    assert a["status"] == b["status"] == H.H3D_OK
    assert a["vcycles"] == b["vcycles"]
    assert a["rel_res"] == b["rel_res"]


@pytest.mark.parametrize("tol", [1e-3, 1e-4])
def test_lockstep_matches_sequential_to_the_last_bit(torch_cuda, tol):
    torch = torch_cuda
    seq = [H.Homogenization(n, precision=H.PREC_FP32) for n, _, _ in DESIGNS]
    C1, C2, st1, st2 = [], [], [], []
    for hd, (n, seed, vol) in zip(seq, DESIGNS):
        hd.update(_rho(torch, n, seed, vol))
        C1.append(hd.elasticMatrix(tol))
        st1.append(hd.last_stats)
        C2.append(hd.elasticMatrix(tol))  # warm start from the stored solutions
        st2.append(hd.last_stats)
    for hd in seq:
        hd.close()
    homs = [H.Homogenization(n, precision=H.PREC_FP32) for n, _, _ in DESIGNS]
    H.batch_update(homs, [_rho(torch, n, seed, vol) for n, seed, vol in DESIGNS])
    with H.Lockstep(homs) as lk:
        L1 = lk.elasticMatrix(tol)
        for i, hd in enumerate(homs):
            _same_stats(hd.last_stats, st1[i])
            assert np.array_equal(L1[i], C1[i]), i
        L2 = lk.elasticMatrix(tol)  # the same graph again, from the stored solutions
        for i, hd in enumerate(homs):
            _same_stats(hd.last_stats, st2[i])
            assert np.array_equal(L2[i], C2[i]), i
    # the designs took different cycle counts, so some finished while others ran
    assert len({s["vcycles"] for s in st1}) > 1
    for hd in homs:
        hd.close()


def test_lockstep_design_matches_the_oracle(torch_cuda):
    torch = torch_cuda
    n, seed, vol = 32, 11, 0.3
    homs = [H.Homogenization(m, precision=H.PREC_FP32) for m in (n, 16)]
    H.batch_update(homs, [_rho(torch, n, seed, vol), _rho(torch, 16, 2, 0.4)])
    with H.Lockstep(homs) as lk:
        C = lk.elasticMatrix(1e-5)
    assert homs[0].last_stats["status"] == H.H3D_OK and max(homs[0].last_stats["rel_res"]) <= 1e-5
    Cref = oracle_C(n, smooth_density(n, seed=seed, vol=vol)).elastic_matrix()
    assert rel_err(C[0], Cref) < 1e-4
    for hd in homs:
        hd.close()


def test_lockstep_refuses_what_it_cannot_batch(torch_cuda):
    a = H.Homogenization(16, precision=H.PREC_FP32)
    cases = [
        [a, a],                                                              # a handle twice
        [a, H.Homogenization(16, precision=H.PREC_REFINE)],                  # not FP32
        [a, H.Homogenization(16, precision=H.PREC_FP32, E=2.0)],             # another material
        [a, H.Homogenization(16, precision=H.PREC_FP32, stencil=H.STENCIL_FP32)],  # other stencil storage
        [],                                                                  # empty
    ]
    for hs in cases:
        with pytest.raises(H.H3DError) as ei:
            H.Lockstep(hs)
        assert ei.value.code == H.H3D_ERR_ARG
    for hs in cases[1:4]:
        hs[1].close()
    # a closed handle or batch is refused before the library is called
    c = H.Homogenization(16, precision=H.PREC_FP32)
    lk = H.Lockstep([a, c])
    c.close()
    with pytest.raises(ValueError):
        lk.elasticMatrix(1e-3)
    lk.close()
    with pytest.raises(ValueError):
        lk.elasticMatrix(1e-3)
    a.close()


def test_lockstep_design_without_stencils_fails_alone(torch_cuda):
    torch = torch_cuda
    a, b = H.Homogenization(16, precision=H.PREC_FP32), H.Homogenization(24, precision=H.PREC_FP32)
    a.update(_rho(torch, 16, 0, 0.3))
    ref = H.Homogenization(16, precision=H.PREC_FP32)
    ref.update(_rho(torch, 16, 0, 0.3))
    Cr = ref.elasticMatrix(1e-3)
    with H.Lockstep([a, b]) as lk:
        with pytest.raises(H.H3DError) as ei:
            lk.elasticMatrix(1e-3)
        assert ei.value.code == H.H3D_ERR_STATE
        _same_stats(a.last_stats, ref.last_stats)
        # with its stencils the second design joins the next solve
        b.update(_rho(torch, 24, 1, 0.3))
        a.reset_solutions()
        C = lk.elasticMatrix(1e-3)
    assert np.array_equal(C[0], Cr)
    for hd in (a, b, ref):
        hd.close()


def test_short_density_is_refused(torch_cuda):
    """a density of the requested size where the reference rounds the grid up (40 ->
    48) is refused before the library reads past its end"""
    torch = torch_cuda
    hd = H.Homogenization(40, precision=H.PREC_FP32)
    assert hd.dims[0] == (48, 48, 48)
    with pytest.raises(ValueError):
        hd.update(_rho(torch, 40, 0, 0.3))
    with pytest.raises(ValueError):
        H.batch_update([hd], [_rho(torch, 40, 0, 0.3)])
    with pytest.raises(ValueError):
        hd.update(torch.ones(48 ** 3, dtype=torch.float64, device="cuda"))
    hd.update(_rho(torch, 48, 0, 0.3))
    hd.close()


@pytest.mark.parametrize("kw", [dict(coarse_mode=H.COARSE_PROJECT), dict(stencil=H.STENCIL_FP32),
                                dict(pin_mode=H.PIN_GALERKIN)])
def test_lockstep_other_modes(torch_cuda, kw):
    """the projected coarsest solve, FP32 coarse stencils and the Galerkin pin in
    lockstep, against the same designs one at a time"""
    torch = torch_cuda
    designs = [(16, 0, 0.3), (24, 1, 0.4), (32, 2, 0.2), (28, 5, 0.3)]
    ref = []
    for n, seed, vol in designs:
        hd = H.Homogenization(n, precision=H.PREC_FP32, **kw)
        hd.update(_rho(torch, n, seed, vol))
        ref.append((hd.elasticMatrix(1e-4), hd.last_stats))
        hd.close()
    homs = [H.Homogenization(n, precision=H.PREC_FP32, **kw) for n, _, _ in designs]
    H.batch_update(homs, [_rho(torch, n, seed, vol) for n, seed, vol in designs])
    with H.Lockstep(homs) as lk:
        C = lk.elasticMatrix(1e-4)
    for i, hd in enumerate(homs):
        _same_stats(hd.last_stats, ref[i][1])
        assert np.array_equal(C[i], ref[i][0]), i
        hd.close()


def test_lockstep_groups_give_the_same_result(torch_cuda):
    """the designs split into 1 to 4 parallel branches of the batch graph: the same
    C and statistics as one design at a time"""
    torch = torch_cuda
    ref = []
    for n, seed, vol in DESIGNS:
        hd = H.Homogenization(n, precision=H.PREC_FP32)
        hd.update(_rho(torch, n, seed, vol))
        ref.append((hd.elasticMatrix(1e-3), hd.last_stats))
        hd.close()
    homs = [H.Homogenization(n, precision=H.PREC_FP32) for n, _, _ in DESIGNS]
    H.batch_update(homs, [_rho(torch, n, seed, vol) for n, seed, vol in DESIGNS])
    for groups in (1, 2, 3, 4, len(DESIGNS)):
        for hd in homs:
            hd.reset_solutions()
        with H.Lockstep(homs, groups=groups) as lk:
            C = lk.elasticMatrix(1e-3)
        for i, hd in enumerate(homs):
            _same_stats(hd.last_stats, ref[i][1])
            assert np.array_equal(C[i], ref[i][0]), (groups, i)
    with pytest.raises(H.H3DError):
        H.Lockstep(homs, groups=len(DESIGNS) + 1)
    for hd in homs:
        hd.close()


def test_lockstep_launch_shapes_give_the_same_result(torch_cuda):
    """every combination of the sweeps' two launch shapes (level 0: six or three
    cases per thread; coarse levels: two or six) against one design at a time"""
    torch = torch_cuda
    ref = []
    for n, seed, vol in DESIGNS:
        hd = H.Homogenization(n, precision=H.PREC_FP32)
        hd.update(_rho(torch, n, seed, vol))
        ref.append((hd.elasticMatrix(1e-3), hd.last_stats))
        hd.close()
    homs = [H.Homogenization(n, precision=H.PREC_FP32) for n, _, _ in DESIGNS]
    H.batch_update(homs, [_rho(torch, n, seed, vol) for n, seed, vol in DESIGNS])
    with H.Lockstep(homs) as lk:
        for shapes in ((0, 0), (1, 0), (0, 1), (1, 1)):
            for hd in homs:
                hd.reset_solutions()
            lk.set_shapes(*shapes)
            C = lk.elasticMatrix(1e-3)
            for i, hd in enumerate(homs):
                _same_stats(hd.last_stats, ref[i][1])
                assert np.array_equal(C[i], ref[i][0]), (shapes, i)
        for hd in homs:
            hd.reset_solutions()
        lk.autotune()  # whatever it picks, the same results
        C = lk.elasticMatrix(1e-3)
        for i, hd in enumerate(homs):
            _same_stats(hd.last_stats, ref[i][1])
            assert np.array_equal(C[i], ref[i][0]), ("tuned", i)
        for bad in ((2, 0), (0, -1)):
            with pytest.raises(H.H3DError) as ei:
                lk.set_shapes(*bad)
            assert ei.value.code == H.H3D_ERR_ARG
    for hd in homs:
        hd.close()
