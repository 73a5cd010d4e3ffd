"""The public soft Smith-Waterman surface on CUDA tensors against the
reference's own public API.

The fixtures (tests/golden/sw_golden.npz, made by tests/golden/make_golden.py)
are the outputs of the reference package's ``orihime.sw*`` functions and
``orihime.ops.sw*.backward / .sensitivity`` (orihime/sw.py:32-200,
orihime/_public_ops.py:120-214), called on CPU tensors.  Here the same calls
go through this package's functions and named operations with the same
arguments on CUDA tensors: square, rectangular, ragged (``lengths=``),
1 x 1 and one-row batches, a boolean ``mask=`` batch, and learnable
(tensor, requires_grad) gap and temperature parameters.

First-order outputs are held to values rtol 1e-5, maps and score gradients
atol 1e-5, parameter gradients atol 1e-4, entropy atol 2e-5: tighter than the
reference's own CPU-vs-CUDA tests (tests/test_soft_sw_affine.py:425-575).
Second-order outputs (the named operations' sensitivities and backward
fields) are held as every second-order test here: to the fp64 oracle, no
further than max(1e-4 of the field's largest exact entry, the reference's own
recorded distance from fp64); and to the reference's recorded outputs at the
reference's own CPU-vs-CUDA tolerance for these fields (rtol 1e-2, atol 5e-3,
tests/test_soft_sw_affine.py:536-542).
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

CASES = ("sq", "rect", "ragged", "unit", "row")
FAMS = {
    "lin": ("sw", dict(gap_score=-1.0, temperature=0.7)),
    "aff": ("sw_affine", dict(gap_open_score=-2.0, gap_extend_score=-0.5, temperature=0.7)),
}


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    import orihime_b200  # noqa: F401


def _inputs(golden, case):
    s = torch.from_numpy(golden[f"{case}/scores"]).cuda()
    cot = torch.from_numpy(golden[f"{case}/cot"]).cuda()
    ln = (torch.from_numpy(golden[f"{case}/lengths"]).to(torch.int32).cuda()
          if f"{case}/lengths" in golden.files else None)
    return s, cot, ln


@pytest.mark.parametrize("fam", list(FAMS))
@pytest.mark.parametrize("case", CASES)
def test_public_functions_match_reference(golden, fam, case):
    import orihime_b200 as ob

    name, kw = FAMS[fam]
    fmap, fval, fent = getattr(ob, name), getattr(ob, f"{name}_value"), getattr(ob, f"{name}_entropy")
    s, cot, ln = _inputs(golden, case)
    g = lambda k: golden[f"{case}/{fam}/{k}"]  # noqa: E731

    x = s.clone().requires_grad_(True)
    v = fval(x, lengths=ln, **kw)
    (dv,) = torch.autograd.grad(-v.mean(), x)
    np.testing.assert_allclose(v.detach().cpu().numpy(), g("value"), rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(dv.cpu().numpy(), g("dvalue"), atol=1e-5)

    x = s.clone().requires_grad_(True)
    m = fmap(x, lengths=ln, **kw)
    (dm,) = torch.autograd.grad((m * cot).sum(), x)
    np.testing.assert_allclose(m.detach().cpu().numpy(), g("map"), atol=1e-5)
    np.testing.assert_allclose(dm.cpu().numpy(), g("dmap"), atol=1e-5)

    x = s.clone().requires_grad_(True)
    h = fent(x, lengths=ln, **kw)
    (dh,) = torch.autograd.grad(h.sum(), x)
    np.testing.assert_allclose(h.detach().cpu().numpy(), g("entropy"), atol=2e-5)
    np.testing.assert_allclose(dh.cpu().numpy(), g("dentropy"), atol=1e-4)


def _second_order_close(tag, got, ref_out, exact):
    """got within max(1e-4 of the largest exact entry, the reference's own
    distance from fp64) of fp64, and within the reference's CPU-vs-CUDA
    tolerance of its recorded output."""
    got, ref_out, exact = (np.asarray(x, np.float64) for x in (got, ref_out, exact))
    scale = float(np.abs(exact).max()) if exact.size else 0.0
    bound = max(1e-4 * scale, float(np.abs(ref_out - exact).max()) if exact.size else 0.0, 1e-7)
    err = float(np.abs(got - exact).max()) if exact.size else 0.0
    assert err <= bound, f"{tag}: ours-fp64 {err:.2e} > bound {bound:.2e}"
    np.testing.assert_allclose(got, ref_out, rtol=1e-2, atol=5e-3, err_msg=tag)


def _exact_second_order(fam, s, cot, ln, kw):
    """fp64 oracle: per parameter the map's sensitivity, and the map's VJP."""
    sn = s.cpu().numpy()
    lnn = None if ln is None else ln.cpu().numpy()
    cn = cot.cpu().numpy().astype(np.float64)
    if fam == "aff":
        p = (kw["gap_open_score"], kw["gap_extend_score"], kw["temperature"])
        sens = [O.affine_param_grad(sn, lnn, *p, k, dtype=np.float64) for k in range(3)]
        hv = O.affine_hvp(sn, cn, lnn, *p, dtype=np.float64)
    else:
        p = (kw["gap_score"], kw["temperature"])
        sens = [O.linear_param_grad(sn, lnn, *p, k, dtype=np.float64) for k in range(2)]
        hv = O.linear_hvp(sn, cn, lnn, *p, dtype=np.float64)
    return sens, hv, [float((cn * x).sum()) for x in sens]


@pytest.mark.parametrize("fam", list(FAMS))
@pytest.mark.parametrize("case", CASES)
def test_named_operations_match_reference(golden, fam, case):
    import orihime_b200 as ob

    name, kw = FAMS[fam]
    op = getattr(ob.ops, name)
    s, cot, ln = _inputs(golden, case)
    g = lambda k: golden[f"{case}/{fam}/{k}"]  # noqa: E731
    sens64, hv64, bw64 = _exact_second_order(fam, s, cot, ln, kw)

    sens = op.sensitivity(s, lengths=ln, **kw)
    assert tuple(sens) == op.sensitivity_fields
    for (k, t), e64 in zip(sens.items(), sens64):
        _second_order_close(f"sens_{k}", t.cpu().numpy(), g(f"sens_{k}"), e64)
    bw = op.backward(s, grad_map=cot, lengths=ln, **kw)
    assert tuple(bw) == op.backward_fields
    _second_order_close("bw_pair_scores", bw["pair_scores"].cpu().numpy(), g("bw_pair_scores"), hv64)
    for k, e64 in zip(op.parameter_fields, bw64):
        assert bw[k].shape == ()
        _second_order_close(f"bw_{k}", bw[k].item(), g(f"bw_{k}"), e64)
    # one field selected by name comes back bare; forward selects observables
    t = op.sensitivity(s, lengths=ln, output="temperature", **kw)
    assert torch.equal(t, sens["temperature"])
    fw = op.forward(s, lengths=ln, output=("value", "map"), **kw)
    np.testing.assert_allclose(fw["value"].cpu().numpy(), g("value"), rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(fw["map"].cpu().numpy(), g("map"), atol=1e-5)


def test_mask_and_learnable_parameters_match_reference(golden):
    import orihime_b200 as ob

    s = torch.from_numpy(golden["mask/scores"]).cuda()
    mask = torch.from_numpy(golden["mask/mask"]).bool().cuda()
    # linear gap: tensor gap and temperature with gradients
    x = s.clone().requires_grad_(True)
    gp = torch.tensor(-1.0, device="cuda", requires_grad=True)
    tp = torch.tensor(0.8, device="cuda", requires_grad=True)
    v = ob.sw_value(x, gap_score=gp, temperature=tp, mask=mask)
    dx, dg, dt = torch.autograd.grad(v.sum(), (x, gp, tp))
    np.testing.assert_allclose(v.detach().cpu().numpy(), golden["mask/lin/value"], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(dx.cpu().numpy(), golden["mask/lin/dx"], atol=1e-5)
    np.testing.assert_allclose(dg.item(), golden["mask/lin/dgap"], atol=1e-4)
    np.testing.assert_allclose(dt.item(), golden["mask/lin/dtemp"], atol=1e-4)
    m = ob.sw(s, gap_score=-1.0, temperature=0.8, mask=mask)
    np.testing.assert_allclose(m.cpu().numpy(), golden["mask/lin/map"], atol=1e-5)
    # affine gaps
    x = s.clone().requires_grad_(True)
    go = torch.tensor(-2.0, device="cuda", requires_grad=True)
    ge = torch.tensor(-0.5, device="cuda", requires_grad=True)
    tp = torch.tensor(0.8, device="cuda", requires_grad=True)
    v = ob.sw_affine_value(x, gap_open_score=go, gap_extend_score=ge, temperature=tp, mask=mask)
    grads = torch.autograd.grad(v.sum(), (x, go, ge, tp))
    np.testing.assert_allclose(v.detach().cpu().numpy(), golden["mask/aff/value"], rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(grads[0].cpu().numpy(), golden["mask/aff/dx"], atol=1e-5)
    for k, t in zip(("dgap_open", "dgap_ext", "dtemp"), grads[1:]):
        np.testing.assert_allclose(t.item(), golden[f"mask/aff/{k}"], atol=1e-4)
    m = ob.sw_affine(s, gap_open_score=-2.0, gap_extend_score=-0.5, temperature=0.8, mask=mask)
    np.testing.assert_allclose(m.cpu().numpy(), golden["mask/aff/map"], atol=1e-5)
