"""The fused input scan of the Python prelude (swb_scan_scores) against the
torch expressions it replaces (orihime/operator.py:249-386): the same errors
in the same order and the same mask sentinels, bit for bit."""

import pytest
import torch

pytestmark = pytest.mark.gpu

PARAMS = (-2.0, -0.5, 0.5)
NAMES = ("gap_open", "gap_ext", "temp")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("CUDA not available")
    import orihime_b200  # noqa: F401


def _both(x):
    from orihime_b200 import operator as op

    out = []
    for fused in (True, False):
        try:
            if fused:
                y = op._validate_and_normalize("pair_scores", x, PARAMS, NAMES)
            else:
                op._validate_domain("pair_scores", x, PARAMS, NAMES)
                y = op.normalize_mask(x, PARAMS[2])
            out.append(("ok", y))
        except (RuntimeError, ValueError) as e:
            out.append(("err", str(e)))
    return out


def _scores(*shape, seed=0):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(*shape, generator=g) * 3).cuda()


@pytest.mark.parametrize("shape", [(4, 37, 51), (3, 64, 64), (1, 1, 1), (2, 1, 1023)])
def test_fused_prelude_matches_torch_expressions(shape):
    from orihime_b200 import operator as op

    x = _scores(*shape)
    cases = {"clean": x.clone()}
    m = x.clone()
    m.view(-1)[:: max(1, m.numel() // 17)] = float("-inf")
    cases["masked"] = m
    am = x.clone()
    am[0] = float("-inf")                                 # an item masked everywhere
    cases["all_masked_item"] = am
    sv = x.clone()
    sv.view(-1)[0] = -op.MASK_SENTINEL_MAGNITUDE           # sentinel-valued cell is allowed
    cases["sentinel_cell"] = sv
    pi = x.clone()
    pi.view(-1)[-1] = float("inf")
    cases["posinf"] = pi
    na = x.clone()
    na.view(-1)[x.numel() // 2] = float("nan")
    cases["nan"] = na
    big = x.clone()
    big.view(-1)[0] = 81.0 * PARAMS[2]                      # |x| / T just over the 80 limit
    cases["out_of_domain"] = big
    both = x.clone()
    both.view(-1)[0] = float("inf")
    both.view(-1)[-1] = 1e6                                # +inf is reported before the domain
    cases["posinf_and_domain"] = both
    cases["non_contiguous"] = m.transpose(1, 2)
    for name, c in cases.items():
        (k1, v1), (k2, v2) = _both(c)
        assert k1 == k2, name
        if k1 == "ok":
            assert torch.equal(v1, v2), name
        else:
            assert v1 == v2, name


def test_scan_flags_and_amax():
    from orihime_b200 import _ops

    x = _scores(3, 40, 41)        # 1640 cells per item: the kernel's scalar path
    x[1, 2, 3] = float("-inf")
    x[2] = float("-inf")
    flags, amax = _ops.scan_scores(x, 1e9, 1e4)
    assert flags == _ops.SCAN_NEGINF
    assert torch.equal(amax, x.amax(dim=(1, 2)))
