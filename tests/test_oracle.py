"""The oracle is pinned before it is trusted (CPU only).

1. Against the golden fixtures recorded from the reference's public API
   (tests/golden/make_golden.py): value, map, entropy, value/map/entropy
   gradients, parameter sensitivities and the map VJP.
2. Against the reference's own CPU kernels compiled from source
   (oracle/_ref, when present): the float restatement must agree bit for bit.
"""

import numpy as np
import pytest

from oracle import oracle as O

CASES = ["sq", "rect", "ragged", "unit", "row"]
T0 = 0.7


def _case(golden, case):
    s = golden[f"{case}/scores"]
    ln = golden[f"{case}/lengths"] if f"{case}/lengths" in golden.files else None
    return s, ln, golden[f"{case}/cot"]


def _close(a, b, rtol=2e-5, atol=2e-6):
    np.testing.assert_allclose(np.asarray(a, np.float64), np.asarray(b, np.float64), rtol=rtol,
                               atol=atol)


@pytest.mark.parametrize("case", CASES)
def test_affine_oracle_vs_golden(golden, case):
    s, ln, cot = _case(golden, case)
    g = lambda k: golden[f"{case}/aff/{k}"]
    B = s.shape[0]
    o = O.affine(s, ln, -2.0, -0.5, T0)
    _close(o["value"], g("value"))
    _close(o["map"], g("map"))
    _close(-o["map"] / B, g("dvalue"))
    _close(o["grad_temp"], g("entropy"), atol=2e-5)
    sens = {p: O.affine_param_grad(s, ln, -2.0, -0.5, T0, p) for p in range(3)}
    _close(sens[0], g("sens_gap_open_score"), atol=1e-5)
    _close(sens[1], g("sens_gap_extend_score"), atol=1e-5)
    _close(sens[2], g("sens_temperature"), atol=1e-5)
    _close(sens[2], g("dentropy"), atol=1e-5)
    hv = O.affine_hvp(s, cot, ln, -2.0, -0.5, T0)
    _close(hv, g("dmap"), atol=1e-5)
    _close(hv, g("bw_pair_scores"), atol=1e-5)
    _close((cot * sens[0]).sum(), g("bw_gap_open_score"), atol=1e-4)
    _close((cot * sens[1]).sum(), g("bw_gap_extend_score"), atol=1e-4)
    _close((cot * sens[2]).sum(), g("bw_temperature"), atol=1e-4)


@pytest.mark.parametrize("case", CASES)
def test_linear_oracle_vs_golden(golden, case):
    s, ln, cot = _case(golden, case)
    g = lambda k: golden[f"{case}/lin/{k}"]
    B = s.shape[0]
    o = O.linear(s, ln, -1.0, T0)
    _close(o["value"], g("value"))
    _close(o["map"], g("map"))
    _close(-o["map"] / B, g("dvalue"))
    _close(o["grad_temp"], g("entropy"), atol=2e-5)
    sens = {p: O.linear_param_grad(s, ln, -1.0, T0, p) for p in range(2)}
    _close(sens[0], g("sens_gap_score"), atol=1e-5)
    _close(sens[1], g("sens_temperature"), atol=1e-5)
    _close(sens[1], g("dentropy"), atol=1e-5)
    hv = O.linear_hvp(s, cot, ln, -1.0, T0)
    _close(hv, g("dmap"), atol=1e-5)
    _close(hv, g("bw_pair_scores"), atol=1e-5)
    _close((cot * sens[0]).sum(), g("bw_gap_score"), atol=1e-4)
    _close((cot * sens[1]).sum(), g("bw_temperature"), atol=1e-4)


@pytest.mark.parametrize("case", CASES)
def test_nw_oracle_vs_golden(golden, case):
    """Global alignment (ohm.nw trio, ohm.ops.nw) against the recorded fixtures."""
    s, ln, cot = _case(golden, case)
    g = lambda k: golden[f"{case}/nw/{k}"]
    B = s.shape[0]
    o = O.nw(s, ln, -1.0, T0)
    _close(o["value"], g("value"))
    _close(o["map"], g("map"))
    _close(-o["map"] / B, g("dvalue"))
    _close(o["grad_temp"], g("entropy"), atol=2e-5)
    sens = {p: O.nw_param_grad(s, ln, -1.0, T0, p) for p in range(2)}
    _close(sens[0], g("sens_gap_score"), atol=1e-5)
    _close(sens[1], g("sens_temperature"), atol=1e-5)
    _close(sens[1], g("dentropy"), atol=1e-5)
    hv = O.nw_hvp(s, cot, ln, -1.0, T0)
    _close(hv, g("dmap"), atol=1e-5)
    _close(hv, g("bw_pair_scores"), atol=1e-5)
    _close((cot * sens[0]).sum(), g("bw_gap_score"), atol=1e-4)
    _close((cot * sens[1]).sum(), g("bw_temperature"), atol=1e-4)


@pytest.mark.parametrize("case", CASES)
def test_nw_affine_oracle_vs_golden(golden, case):
    """Global alignment with affine gaps (ohm.nw_affine trio, ohm.ops.nw_affine)
    against the recorded fixtures."""
    s, ln, cot = _case(golden, case)
    g = lambda k: golden[f"{case}/nwa/{k}"]
    B = s.shape[0]
    o = O.nw_affine(s, ln, -2.0, -0.5, T0)
    _close(o["value"], g("value"))
    _close(o["map"], g("map"))
    _close(-o["map"] / B, g("dvalue"))
    _close(o["grad_temp"], g("entropy"), atol=2e-5)
    sens = {p: O.nw_affine_param_grad(s, ln, -2.0, -0.5, T0, p) for p in range(3)}
    _close(sens[0], g("sens_gap_open_score"), atol=1e-5)
    _close(sens[1], g("sens_gap_extend_score"), atol=1e-5)
    _close(sens[2], g("sens_temperature"), atol=1e-5)
    _close(sens[2], g("dentropy"), atol=1e-5)
    hv = O.nw_affine_hvp(s, cot, ln, -2.0, -0.5, T0)
    _close(hv, g("dmap"), atol=1e-5)
    _close(hv, g("bw_pair_scores"), atol=1e-5)
    _close((cot * sens[0]).sum(), g("bw_gap_open_score"), atol=1e-4)
    _close((cot * sens[1]).sum(), g("bw_gap_extend_score"), atol=1e-4)
    _close((cot * sens[2]).sum(), g("bw_temperature"), atol=1e-4)


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("fam", ["svl", "sva"])
def test_sv_oracle_vs_golden(golden, case, fam):
    """Saigo-Vert, linear (ohm.sv trio, ohm.ops.sv) and affine (ohm.sv_affine
    trio, ohm.ops.sv_affine), against the recorded fixtures."""
    s, ln, cot = _case(golden, case)
    g = lambda k: golden[f"{case}/{fam}/{k}"]
    B = s.shape[0]
    lin = fam == "svl"
    go, ge = (-1.0, -1.0) if lin else (-2.0, -0.5)
    o = O.sv(s, ln, go, ge, T0, linear=lin)
    _close(o["value"], g("value"))
    _close(o["map"], g("map"))
    _close(-o["map"] / B, g("dvalue"))
    _close(o["grad_temp"], g("entropy"), atol=2e-5)
    names = ("gap_score", "temperature") if lin else ("gap_open_score", "gap_extend_score", "temperature")
    sens = {p: O.sv_param_grad(s, ln, go, ge, T0, p, linear=lin) for p in range(len(names))}
    for p, n in enumerate(names):
        _close(sens[p], g(f"sens_{n}"), atol=1e-5)
        _close((cot * sens[p]).sum(), g(f"bw_{n}"), atol=1e-4)
    _close(sens[len(names) - 1], g("dentropy"), atol=1e-5)
    hv = O.sv_hvp(s, cot, ln, go, ge, T0)
    _close(hv, g("dmap"), atol=1e-5)
    _close(hv, g("bw_pair_scores"), atol=1e-5)


def _mask_sentinel(scores, mask, T):
    """orihime/operator.py:334-386: masked cells -> amax - (sum(shape[1:])*80 + 200)*T."""
    x = np.where(mask, -np.inf, scores).astype(np.float32)
    amax = x.reshape(x.shape[0], -1).max(axis=1)
    amax = np.where(np.isfinite(amax), amax, 0.0)
    off = (float(sum(x.shape[1:])) * 80.0 + 200.0) * T
    sent = (amax - np.float32(off)).astype(np.float32)[:, None, None]
    return np.where(mask, sent, x).astype(np.float32)


def test_masked_batches_vs_golden(golden):
    s = golden["mask/scores"]
    mask = golden["mask/mask"].astype(bool)
    x = _mask_sentinel(s, mask, 0.8)
    o = O.affine(x, None, -2.0, -0.5, 0.8)
    _close(o["value"], golden["mask/aff/value"])
    _close(o["map"], golden["mask/aff/map"])
    _close(o["map"], golden["mask/aff/dx"])
    _close(o["grad_open"].sum(), golden["mask/aff/dgap_open"], atol=1e-4)
    _close(o["grad_ext"].sum(), golden["mask/aff/dgap_ext"], atol=1e-4)
    _close(o["grad_temp"].sum(), golden["mask/aff/dtemp"], atol=1e-4)
    o = O.linear(x, None, -1.0, 0.8)
    _close(o["value"], golden["mask/lin/value"])
    _close(o["map"], golden["mask/lin/map"])
    _close(o["grad_gap"].sum(), golden["mask/lin/dgap"], atol=1e-4)
    _close(o["grad_temp"].sum(), golden["mask/lin/dtemp"], atol=1e-4)
    assert np.all(o["map"][mask] == 0.0)
    o = O.nw(x, None, -1.0, 0.8)
    _close(o["value"], golden["mask/nw/value"])
    _close(o["map"], golden["mask/nw/map"])
    _close(o["map"], golden["mask/nw/dx"])
    _close(o["grad_gap"].sum(), golden["mask/nw/dgap"], atol=1e-4)
    _close(o["grad_temp"].sum(), golden["mask/nw/dtemp"], atol=1e-4)


def test_fp64_oracle_close_to_fp32(golden):
    s, ln, _ = _case(golden, "ragged")
    a = O.affine(s, ln, -2.0, -0.5, T0, dtype=np.float32)
    b = O.affine(s, ln, -2.0, -0.5, T0, dtype=np.float64)
    _close(a["value"], b["value"], rtol=1e-6)
    _close(a["map"], b["map"], atol=1e-6)


ref_only = pytest.mark.skipif(not O.ref_available(), reason="reference CPU kernels not built")


@ref_only
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_oracle_bit_exact_vs_reference_kernels(seed):
    rng = np.random.default_rng(seed)
    B, L1, L2 = 3, int(rng.integers(1, 17)), int(rng.integers(1, 17))
    s = (rng.standard_normal((B, L1, L2)) * 2).astype(np.float32)
    ln = np.stack([rng.integers(0, L1 + 1, B), rng.integers(0, L2 + 1, B)], 1).astype(np.int32)
    V = rng.standard_normal(s.shape).astype(np.float32)
    for lens in (None, ln):
        for T in (0.3, 1.0, 2.0):
            a, r = O.affine(s, lens, -2.0, -0.5, T), O.ref_affine(s, lens, -2.0, -0.5, T)
            for k in a:
                assert np.array_equal(a[k], r[k]), k
            assert np.array_equal(O.affine_hvp(s, V, lens, -2.0, -0.5, T),
                                  O.ref_affine_hvp(s, V, lens, -2.0, -0.5, T))
            for p in range(3):
                assert np.array_equal(O.affine_param_grad(s, lens, -2.0, -0.5, T, p),
                                      O.ref_affine_param_grad(s, lens, -2.0, -0.5, T, p))
            a, r = O.linear(s, lens, -1.0, T), O.ref_linear(s, lens, -1.0, T)
            for k in a:
                assert np.array_equal(a[k], r[k]), k
            assert np.array_equal(O.linear_hvp(s, V, lens, -1.0, T),
                                  O.ref_linear_hvp(s, V, lens, -1.0, T))
            for p in range(2):
                assert np.array_equal(O.linear_param_grad(s, lens, -1.0, T, p),
                                      O.ref_linear_param_grad(s, lens, -1.0, T, p))
            a, r = O.nw_affine(s, lens, -2.0, -0.5, T), O.ref_nw_affine(s, lens, -2.0, -0.5, T)
            for k in a:
                assert np.array_equal(a[k], r[k]), k
            assert np.array_equal(O.nw_affine_hvp(s, V, lens, -2.0, -0.5, T),
                                  O.ref_nw_affine_hvp(s, V, lens, -2.0, -0.5, T))
            for p in range(3):
                assert np.array_equal(O.nw_affine_param_grad(s, lens, -2.0, -0.5, T, p),
                                      O.ref_nw_affine_param_grad(s, lens, -2.0, -0.5, T, p))
            for lin, (go, ge) in ((False, (-2.0, -0.5)), (True, (-1.0, -1.0))):
                a, r = O.sv(s, lens, go, ge, T, linear=lin), O.ref_sv(s, lens, go, ge, T, linear=lin)
                for k in (("value", "map", "grad_open", "grad_temp") if lin else a):
                    assert np.array_equal(a[k], r[k]), (lin, k)
                assert np.array_equal(O.sv_hvp(s, V, lens, go, ge, T),
                                      O.ref_sv_hvp(s, V, lens, go, ge, T, linear=lin))
                for p in range(2 if lin else 3):
                    assert np.array_equal(O.sv_param_grad(s, lens, go, ge, T, p, linear=lin),
                                          O.ref_sv_param_grad(s, lens, go, ge, T, p, linear=lin))
            a, r = O.nw(s, lens, -1.0, T), O.ref_nw(s, lens, -1.0, T)
            for k in a:
                assert np.array_equal(a[k], r[k]), k
            assert np.array_equal(O.nw_hvp(s, V, lens, -1.0, T), O.ref_nw_hvp(s, V, lens, -1.0, T))
            for p in range(2):
                assert np.array_equal(O.nw_param_grad(s, lens, -1.0, T, p),
                                      O.ref_nw_param_grad(s, lens, -1.0, T, p))


def test_finite_difference_of_fp64_value():
    """dS/dscores (the map) and dS/dgap against central differences of the FP64 oracle."""
    rng = np.random.default_rng(5)
    s = rng.standard_normal((1, 6, 7))
    base = O.affine(s, None, -2.0, -0.5, 0.5, dtype=np.float64)
    eps = 1e-5
    for (i, j) in [(0, 0), (2, 3), (5, 6), (3, 1)]:
        sp, sm = s.copy(), s.copy()
        sp[0, i, j] += eps
        sm[0, i, j] -= eps
        fd = (O.affine(sp, None, -2.0, -0.5, 0.5, dtype=np.float64)["value"][0] -
              O.affine(sm, None, -2.0, -0.5, 0.5, dtype=np.float64)["value"][0]) / (2 * eps)
        assert abs(fd - base["map"][0, i, j]) < 1e-6
    fd = (O.affine(s, None, -2.0 + eps, -0.5, 0.5, dtype=np.float64)["value"][0] -
          O.affine(s, None, -2.0 - eps, -0.5, 0.5, dtype=np.float64)["value"][0]) / (2 * eps)
    assert abs(fd - base["grad_open"][0]) < 1e-6
    fd = (O.affine(s, None, -2.0, -0.5, 0.5 + eps, dtype=np.float64)["value"][0] -
          O.affine(s, None, -2.0, -0.5, 0.5 - eps, dtype=np.float64)["value"][0]) / (2 * eps)
    assert abs(fd - base["grad_temp"][0]) < 1e-5


def test_nw_finite_differences_of_fp64_value():
    """Global alignment: the map, dS/dgap (boundary cells included) and dS/dT
    against central differences of the FP64 oracle's value."""
    rng = np.random.default_rng(6)
    s = rng.standard_normal((1, 5, 8))
    ln = np.array([[5, 6]], np.int32)
    f = lambda x, g, t: O.nw(x, ln, g, t, dtype=np.float64)["value"][0]
    base = O.nw(s, ln, -0.7, 0.6, dtype=np.float64)
    eps = 1e-5
    for (i, j) in [(0, 0), (2, 3), (4, 5), (3, 1)]:
        sp, sm = s.copy(), s.copy()
        sp[0, i, j] += eps
        sm[0, i, j] -= eps
        assert abs((f(sp, -0.7, 0.6) - f(sm, -0.7, 0.6)) / (2 * eps) - base["map"][0, i, j]) < 1e-6
    assert abs((f(s, -0.7 + eps, 0.6) - f(s, -0.7 - eps, 0.6)) / (2 * eps) - base["grad_gap"][0]) < 1e-6
    assert abs((f(s, -0.7, 0.6 + eps) - f(s, -0.7, 0.6 - eps)) / (2 * eps) - base["grad_temp"][0]) < 1e-5
    assert np.all(base["map"][0, 5:, :] == 0) and np.all(base["map"][0, :, 6:] == 0)


@pytest.mark.parametrize("fam", ["sw", "sw_affine", "nw", "nw_affine", "sv_linear", "sv_affine"])
def test_second_order_homogeneity_identity(fam):
    """S is 1-homogeneous in (scores, gaps, T), so along any score direction v
    T * <v, dP/dT> = -<s, H v> - sum_k gap_k * <v, dP/dgap_k>: the identity
    from which the marginals_backward ops take their temperature tangent in
    the same pass as H v.  Checked on the fp64 oracle."""
    rng = np.random.default_rng(7)
    B, L1, L2, T = 2, 13, 17, 0.6
    s = (1.5 * rng.standard_normal((B, L1, L2))).astype(np.float32)
    v = rng.standard_normal((B, L1, L2)).astype(np.float32)
    ln = np.array([[13, 17], [9, 12]], np.int32)
    d = np.float64
    if fam == "sw":
        gaps = (-1.0,)
        hv = O.linear_hvp(s, v, ln, *gaps, T, dtype=d)
        jac = [O.linear_param_grad(s, ln, *gaps, T, p, dtype=d) for p in range(2)]
    elif fam == "nw":
        gaps = (-1.0,)
        hv = O.nw_hvp(s, v, ln, *gaps, T, dtype=d)
        jac = [O.nw_param_grad(s, ln, *gaps, T, p, dtype=d) for p in range(2)]
    elif fam == "sv_linear":
        gaps = (-1.0,)
        hv = O.sv_hvp(s, v, ln, -1.0, -1.0, T, dtype=d)
        jac = [O.sv_param_grad(s, ln, -1.0, -1.0, T, p, linear=True, dtype=d) for p in range(2)]
    else:
        gaps = (-2.0, -0.5)
        hvp, pg = {"sw_affine": (O.affine_hvp, O.affine_param_grad),
                   "nw_affine": (O.nw_affine_hvp, O.nw_affine_param_grad),
                   "sv_affine": (O.sv_hvp, O.sv_param_grad)}[fam]
        hv = hvp(s, v, ln, *gaps, T, dtype=d)
        jac = [pg(s, ln, *gaps, T, p, dtype=d) for p in range(3)]
    vd, sd = v.astype(d), s.astype(d)
    tan = [(vd * j).sum() for j in jac]
    lhs = T * tan[-1]
    rhs = -(sd * hv).sum() - sum(g * t for g, t in zip(gaps, tan[:-1]))
    assert abs(lhs - rhs) <= 1e-9 * (1 + abs(lhs) + np.abs(sd * hv).sum()), (fam, lhs, rhs)
