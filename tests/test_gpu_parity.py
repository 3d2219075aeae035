"""GPU (sm_100a) results through the C ABI against the C oracle: bit-exact."""
import numpy as np
import pytest

import oracle as O
from tests.helpers import ccs_case, ELL_D, D_SC, XS

Q = (1 << 64) - (1 << 32) + 1
pytestmark = pytest.mark.gpu


def _pp(kappa, m, seed):
    return np.random.default_rng(seed).integers(0, Q, size=(kappa, m, 54), dtype=np.uint64)


@pytest.mark.parametrize("m,n_vec", [(2, 1), (64, 1), (1024, 3), (1024, 5), (4096, 13), (1 << 16, 1), (1 << 16, 12)])
def test_commit_matches_oracle(ctx, m, n_vec):
    pp = _pp(16, m, m)
    rng = np.random.default_rng(m + n_vec)
    Z = rng.integers(-1, 2, size=(n_vec, 54, m)).astype(np.int8)
    ctx.pp_upload(pp)
    got = ctx.commit(Z)
    for v in range(n_vec):
        assert np.array_equal(got[v], O.commit_digits(pp, Z[v]))


def test_commit_edge_digits(ctx):
    m = 256
    pp = _pp(16, m, 1)
    ctx.pp_upload(pp)
    zeros = np.zeros((54, m), np.int8)
    assert np.all(ctx.commit(zeros) == 0)
    ones = np.ones((54, m), np.int8)
    big = np.full((54, m), -128, np.int8)
    top = np.full((54, m), 127, np.int8)
    for Z in (ones, big, top):
        assert np.array_equal(ctx.commit(Z), O.commit_digits(pp, Z))


def test_commit_int32_bound_extreme_pp(ctx):
    # all PP limbs 0xFF and all digits -128: the per-CTA int32 partials sit at the
    # overflow bound of the K split (512 K blocks of 128 bytes)
    m = 1 << 12
    pp = np.full((16, m, 54), (1 << 64) - (1 << 32), dtype=np.uint64)  # q - 1: every byte limb is 0xFF or 0x00
    pp[:, :, ::2] = np.uint64(0xFEFFFFFFFFFFFFFF)
    ctx.pp_upload(pp)
    Z = np.full((2, 54, m), -128, np.int8)
    got = ctx.commit(Z)
    assert np.array_equal(got[0], O.commit_digits(pp, Z[0]))


@pytest.mark.parametrize("n_vec", [1, 2, 4, 5])
def test_commit_small_digit_form_extremes(ctx, n_vec):
    """Digits with |z| <= 63 take the mod-Phi_81 tensor-core form, whose B
    entries are differences of two digits: alternating +-63 (|entry| = 126,
    the int8 limit of that form), constant +-63, random digits in [-63, 63]
    and one digit of 64 (the call falls back to the cyclic form) all equal the
    oracle, against PP limbs of 0xFF (the int32 bound of the partial sums)."""
    m = 2048
    pp = np.full((16, m, 54), (1 << 64) - (1 << 32), dtype=np.uint64)
    pp[:, :, ::2] = np.uint64(0xFEFFFFFFFFFFFFFF)
    pp[:, ::3] = _pp(16, m, 7)[:, ::3]
    ctx.pp_upload(pp)
    rng = np.random.default_rng(n_vec)
    alt = np.where(np.arange(54)[:, None] % 2 == 0, 63, -63).astype(np.int8) * np.ones((1, m), np.int8)
    cases = [np.stack([alt] * n_vec), np.full((n_vec, 54, m), -63, np.int8), np.full((n_vec, 54, m), 63, np.int8),
             rng.integers(-63, 64, size=(n_vec, 54, m)).astype(np.int8)]
    over = rng.integers(-63, 64, size=(n_vec, 54, m)).astype(np.int8)
    over[-1, 53, m - 1] = 64
    cases.append(over)
    for Z in cases:
        got = ctx.commit(Z)
        for v in range(n_vec):
            assert np.array_equal(got[v], O.commit_digits(pp, Z[v]))


def test_commit_device_ex_small_digits(ctx):
    """neo_gpu_commit_device_ex with NEO_COMMIT_SMALL_DIGITS (the form the fold
    step uses for its ternary planes) equals the host commitment and the
    any-int8 device form; digits that break the |z| <= 63 guarantee so that
    a window entry leaves int8 are reported as NEO_ERR_INVARIANT at the next
    synchronisation, and the context stays usable."""
    import torch
    from nightstream_b200.gpu import NeoGpuError
    m, n_vec = 4096, 12
    pp = _pp(16, m, 21)
    ctx.pp_upload(pp)
    Z = np.random.default_rng(8).integers(-1, 2, size=(n_vec, 54, m)).astype(np.int8)
    want = ctx.commit(Z)
    d = torch.from_numpy(Z).cuda()
    out = torch.zeros((n_vec, 16, 54), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    for small in (True, False, True):
        out.zero_()
        torch.cuda.synchronize()
        ctx.commit_device(d.data_ptr(), n_vec, m, out.data_ptr(), small_digits=small)
        ctx.synchronize()
        assert np.array_equal(out.cpu().numpy().view(np.uint64), want)
    bad = Z.copy()
    bad[3, 10, 100] = 100  # rows 10 and 37 (27 apart) meet in one window entry: 100 - (-100) leaves int8
    bad[3, 37, 100] = -100
    db = torch.from_numpy(bad).cuda()
    torch.cuda.synchronize()
    ctx.commit_device(db.data_ptr(), n_vec, m, out.data_ptr(), small_digits=True)
    with pytest.raises(NeoGpuError) as e:
        ctx.synchronize()
    assert e.value.code == 3
    ctx.commit_device(d.data_ptr(), n_vec, m, out.data_ptr(), small_digits=True)
    ctx.synchronize()
    assert np.array_equal(out.cpu().numpy().view(np.uint64), want)


def test_decomp_matches_oracle(ctx):
    rng = np.random.default_rng(3)
    z = np.concatenate([rng.integers(0, 1 << 32, size=5000, dtype=np.uint64),
                        (Q - rng.integers(1, 1 << 50, size=5000, dtype=np.uint64)).astype(np.uint64),
                        np.array([0, 1, Q - 1, 1 << 60], np.uint64)])
    assert np.array_equal(ctx.decomp_b2(z), O.decomp_b2(z))


def test_rlc_mix_and_split_match_oracle(ctx):
    rng = np.random.default_rng(4)
    count, m = 13, 4096
    rho = rng.integers(-2, 3, size=(count, 54)).astype(np.int8)
    Zs = rng.integers(-1, 2, size=(count, 54, m)).astype(np.int8)
    mix = ctx.rlc_mix(rho, Zs)
    assert np.array_equal(mix, O.rlc_mix(rho, Zs))
    planes, nz = ctx.split_b(mix, 12, 2)
    p2, nz2 = O.split_b(mix, 12, 2)
    assert np.array_equal(planes, p2) and np.array_equal(nz, nz2)
    assert np.array_equal(ctx.rlc_mix(rho[:1], Zs[:1]), Zs[0].astype(np.int32))


@pytest.mark.parametrize("count,m,wide", [(13, 100, False), (13, 1024, False), (2, 1024, True), (13, 8192, False), (13, 16384, False),
                                          (13, 65536, False), (3, 65536, True)])
def test_rlc_mix_every_grid_shape(ctx, count, m, wide):
    """The mix splits a column's 54 output rows over 1, 3, 9 or 54 threads
    depending on m (ragged m included); every shape equals the oracle, also
    for digits outside {-1, 0, 1}."""
    rng = np.random.default_rng(m + count)
    rho = rng.integers(-2, 3, size=(count, 54)).astype(np.int8)
    Zs = rng.integers(-7 if wide else -1, 8 if wide else 2, size=(count, 54, m)).astype(np.int8)
    assert np.array_equal(ctx.rlc_mix(rho, Zs), O.rlc_mix(rho, Zs))


def test_split_out_of_range_is_an_error(ctx):
    from nightstream_b200.gpu import NeoGpuError
    with pytest.raises(NeoGpuError) as e:
        ctx.split_b(np.array([[4096, 1]], np.int32), 12, 2)
    assert e.value.code == 3


def test_me_y_matches_oracle(ctx):
    ccs, z, Z, ch, chals = ccs_case(10, 3, True)
    r = chals[:10]
    y, ys = ctx.me_y(ccs, Z, r)
    for i in range(3):
        y2, ys2 = O.me_y_at_r(ccs, Z[i], 10, r)
        assert np.array_equal(y[i], y2) and np.array_equal(ys[i], ys2)


def _run_both(ctx, ell, k, inputs, seed=7):
    from nightstream_b200.gpu import GpuCcsOracle
    ccs, z, Z, ch, chals = ccs_case(ell, k, inputs, seed)
    args = (ccs, Z, 2, ch["alpha"], ch["beta_a"], ch["beta_r"], ch["gamma"], ch["r_inputs"], ELL_D, ell, D_SC)
    g = GpuCcsOracle(ctx, *args)
    o = O.CcsOracle(*args)
    assert g.num_rounds() == ell + ELL_D and g.degree_bound() == D_SC
    for r in range(ell + ELL_D):
        yg = g.evals_at(XS)
        yo = o.evals_at(XS)
        assert np.array_equal(yg, yo), f"round {r}"
        # a second evaluation in the same round (other points) must agree too
        xs2 = chals[r:r + 2]
        assert np.array_equal(g.evals_at(xs2), o.evals_at(xs2)), f"round {r} ext points"
        g.fold(chals[r])
        o.fold(chals[r])
    yg, ysg = g.me_outputs()
    yo, yso = o.me_outputs()
    assert np.array_equal(yg, yo) and np.array_equal(ysg, yso)
    g.close()


@pytest.mark.parametrize("ell,k,inputs", [(1, 1, False), (3, 2, True), (4, 2, True), (5, 3, False), (6, 1, False),
                                          (10, 13, True), (12, 3, True)])
def test_ccs_oracle_all_rounds_match(ctx, ell, k, inputs):
    _run_both(ctx, ell, k, inputs)


def test_ccs_oracle_wide_digits_match(ctx):
    """Digit rows outside {-1,0,1} (a corrupted or non-decomposed witness) take
    the general path of the digit-streaming rounds; the mix of general and
    ternary rows still matches the oracle in every round."""
    from nightstream_b200.gpu import GpuCcsOracle
    ell, k = 10, 3
    ccs, z, Z, ch, chals = ccs_case(ell, k, True, seed=23)
    rng = np.random.default_rng(5)
    Z = Z.copy()
    mask = rng.random(Z.shape) < 0.05
    Z[mask] = rng.integers(-7, 8, size=int(mask.sum())).astype(np.int8)
    args = (ccs, Z, 2, ch["alpha"], ch["beta_a"], ch["beta_r"], ch["gamma"], ch["r_inputs"], ELL_D, ell, D_SC)
    g = GpuCcsOracle(ctx, *args)
    o = O.CcsOracle(*args)
    for r in range(ell + ELL_D):
        assert np.array_equal(g.evals_at(XS), o.evals_at(XS)), f"round {r}"
        g.fold(chals[r])
        o.fold(chals[r])
    g.close()


def test_ccs_oracle_steady_state_full_size(ctx):
    # k = 13 (1 MCS + 12 carried children), n = m = 2^16
    _run_both(ctx, 16, 13, True, seed=11)


def test_row_rounds_device_matches_oracle(ctx):
    """The back-to-back device round sequence gives the same round polynomials
    as the transcript-driven rounds, and the Ajtai rounds continue from it."""
    import torch
    from nightstream_b200.gpu import GpuCcsOracle
    ell, k = 10, 3
    ccs, z, Z, ch, chals = ccs_case(ell, k, True)
    args = (ccs, Z, 2, ch["alpha"], ch["beta_a"], ch["beta_r"], ch["gamma"], ch["r_inputs"], ELL_D, ell, D_SC)
    g = GpuCcsOracle(ctx, *args)
    o = O.CcsOracle(*args)
    d = torch.zeros((ell, D_SC + 1, 2), dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    g.row_rounds_device(chals[:4], d.data_ptr())
    g.row_rounds_device(chals[4:ell], d[4:].data_ptr())
    ctx.synchronize()
    coeffs = d.cpu().numpy().view(np.uint64)
    for r in range(ell):
        yo = o.evals_at(XS)
        yg = np.stack([O.poly_eval_k(coeffs[r], x) for x in XS])
        assert np.array_equal(yg, yo), f"round {r}"
        o.fold(chals[r])
    for r in range(ell, ell + ELL_D):
        assert np.array_equal(g.evals_at(XS), o.evals_at(XS)), f"round {r}"
        g.fold(chals[r])
        o.fold(chals[r])
    yg, ysg = g.me_outputs()
    yo, yso = o.me_outputs()
    assert np.array_equal(yg, yo) and np.array_equal(ysg, yso)
    g.close()


def test_commit_mixers_match_definition(ctx):
    """CommitMixers on the device: sum_i rho_i c_i for general 54 x 54 F_q
    matrices and sum_i b^i c_i, against the definition in Python integers."""
    rng = np.random.default_rng(31)
    count, kappa = 13, 16
    rhos = rng.integers(0, Q, size=(count, 54, 54), dtype=np.uint64)
    rhos[0] = O.rot_matrix(rng.integers(-2, 3, size=54).astype(np.int8))  # a Pi_RLC rho = rot(a), a in {-2..2}^54
    cs = rng.integers(0, Q, size=(count, kappa, 54), dtype=np.uint64)
    got = ctx.mix_rhos_commits(rhos, cs)
    R = [[[int(x) for x in row] for row in m] for m in rhos]
    C = [[[int(x) for x in col] for col in c] for c in cs]
    want = [[sum(R[i][r][k] * C[i][c][k] for i in range(count) for k in range(54)) % Q for r in range(54)]
            for c in range(kappa)]
    assert np.array_equal(got, np.array(want, dtype=np.uint64))
    got = ctx.combine_b_pows(cs[:12], 2)
    want = [[sum(pow(2, i, Q) * C[i][c][r] for i in range(12)) % Q for r in range(54)] for c in range(kappa)]
    assert np.array_equal(got, np.array(want, dtype=np.uint64))


def test_autotuned_rounds_match_oracle(ctx):
    """The autotuner picks launch choices for (ell_n, k) on a real shape; an
    oracle created afterwards uses them and still equals the oracle in every
    round."""
    from nightstream_b200 import gpu
    ell, k = 11, 4
    ccs, z, Z, ch, chals = ccs_case(ell, k, True, seed=41)
    best = ctx.ccs_autotune(ccs, Z, reps=1)
    assert gpu.tune_get(ell, k) == best
    _run_both(ctx, ell, k, True, seed=41)
