"""Meta (fake) shapes and vmap argument checks of the namespaced ops, on the CPU
(reference registrations: orihime/_compile.py:25-140, orihime/_ops.py:178-406)."""

import pytest
import torch

import orihime_b200  # noqa: F401
from orihime_b200 import _ops

o = torch.ops.orihime
AFF = (-2.0, -0.5, 0.5)
LIN = (-1.0, 0.5)


@pytest.fixture(scope="module", autouse=True)
def _defined_here():
    if len(_ops.DEFINED_HERE) != len(_ops.SCHEMAS):
        pytest.skip("the reference extension defined the schemas; its package registers these")


def test_fake_shapes_of_all_ops():
    s = torch.empty(3, 5, 7, device="meta")
    ln = torch.empty(3, 2, dtype=torch.int32, device="meta")
    t = torch.empty((), device="meta")
    for name, args in (("sw_forward", (s, *LIN, None)), ("sw_affine_forward", (s, *AFF, None)),
                       ("sw_forward_t", (s, t, t, ln)), ("sw_affine_forward_t", (s, t, t, t, ln))):
        v, m = getattr(o, name)(*args)
        assert v.shape == (3,) and m.shape == (3, 5, 7), name
    assert [g.shape for g in o.sw_value_grad_params(s, *LIN, None)] == [(3,)] * 2
    assert [g.shape for g in o.sw_affine_value_grad_params(s, *AFF, None)] == [(3,)] * 3
    for name in ("sw_marginals_grad_gap", "sw_marginals_grad_temp"):
        assert getattr(o, name)(s, *LIN, None).shape == (3, 5, 7)
    for name in ("sw_affine_marginals_grad_gap_open", "sw_affine_marginals_grad_gap_ext",
                 "sw_affine_marginals_grad_temp"):
        assert getattr(o, name)(s, *AFF, None).shape == (3, 5, 7)
    assert o.sw_marginals_hvp(s, s, *LIN, None).shape == (3, 5, 7)
    assert o.sw_affine_marginals_hvp(s, s, *AFF, None).shape == (3, 5, 7)
    assert [g.shape for g in o.sw_marginals_backward(s, s, *LIN, None)] == [(3, 5, 7), (1,), (1,)]
    assert [g.shape for g in o.sw_affine_marginals_backward(s, s, *AFF, None)] == \
        [(3, 5, 7), (1,), (1,), (1,)]
    assert o.nw_marginals_hvp(s, s, *LIN, None).shape == (3, 5, 7)
    for name in ("nw_marginals_grad_gap", "nw_marginals_grad_temp"):
        assert getattr(o, name)(s, *LIN, None).shape == (3, 5, 7)
    assert [g.shape for g in o.nw_marginals_backward(s, s, *LIN, None)] == [(3, 5, 7), (1,), (1,)]
    v, m = o.nw_forward(s, *LIN, None)
    assert v.shape == (3,) and m.shape == (3, 5, 7)
    v, m = o.nw_forward_t(s, t, t, ln)
    assert v.shape == (3,) and m.shape == (3, 5, 7)
    assert [g.shape for g in o.nw_value_grad_params(s, *LIN, None)] == [(3,)] * 2


def test_vmap_rejects_a_mapped_scalar_parameter():
    s = torch.zeros(2, 3, 4, 5)
    ln = torch.full((3, 2), 4, dtype=torch.int32)
    temps = torch.ones(2)
    f = lambda sc, tt: o.sw_forward_t(sc, torch.tensor(-1.0), tt, ln)  # noqa: E731
    with pytest.raises(RuntimeError, match="does not support mapping scalar argument 'temp'"):
        torch.func.vmap(f)(s, temps)


def test_vmap_rejects_inconsistent_native_batches():
    s = torch.zeros(2, 3, 4, 5)
    v = torch.zeros(2, 4, 4, 5)
    with pytest.raises(RuntimeError, match="inconsistent native batch sizes 3 and 4"):
        torch.func.vmap(lambda a, b: o.sw_marginals_hvp(a, b, *LIN, None))(s, v)


def test_fake_shapes_of_value_only_ops():
    s = torch.empty(3, 5, 7, device="meta")
    assert torch.ops.orihime_b200.sw_value(s, *LIN, None).shape == (3,)
    assert torch.ops.orihime_b200.sw_affine_value(s, *AFF, None).shape == (3,)
    assert torch.ops.orihime_b200.nw_value(s, *LIN, None).shape == (3,)


def test_legacy_schemas_defined():
    """The 18 legacy soft_sw* / soft_nw* schemas (src/sw/registry.cpp:30-35,
    src/sw_affine/registry.cpp:27-32, src/nw/registry.cpp:34-39) exist beside
    the namespaced ones."""
    assert sorted(_ops.LEGACY_DEFINED_HERE) == sorted(_ops.LEGACY_SCHEMAS)
    for name in _ops.LEGACY_SCHEMAS:
        assert getattr(o, name).default._schema.name == f"orihime::{name}"


def test_legacy_schema_count():
    assert len(_ops.LEGACY_SCHEMAS) == 36
