"""Named operations ``orihime_b200.ops``: field names and ``output=``
selection (host logic, CPU; the computations are in test_gpu_public_api)."""

import pytest


def test_fields_follow_the_public_signatures():
    import orihime_b200 as ob

    assert ob.ops.sw_affine.backward_fields == ("pair_scores", "gap_open_score", "gap_extend_score",
                                                "temperature")
    assert ob.ops.sw_affine.sensitivity_fields == ("gap_open_score", "gap_extend_score", "temperature")
    assert ob.ops.sw.backward_fields == ("pair_scores", "gap_score", "temperature")
    for n in ("nw", "sv"):
        assert getattr(ob.ops, n).sensitivity_fields == ("gap_score", "temperature")
    for n in ("nw_affine", "sv_affine"):
        assert getattr(ob.ops, n).parameter_fields == ("gap_open_score", "gap_extend_score", "temperature")
    assert repr(ob.ops.sw_affine) == "<orihime_b200.ops.sw_affine>"


def test_output_selection_messages():
    from orihime_b200 import ops

    allowed = ops.FORWARD_FIELDS
    assert ops._select(None, allowed) == (allowed, False)
    assert ops._select("map", allowed) == (("map",), True)
    assert ops._select(["value", "map"], allowed) == (("value", "map"), False)
    with pytest.raises(ValueError, match="output must select at least one field"):
        ops._select([], allowed)
    with pytest.raises(ValueError, match="duplicate"):
        ops._select(["map", "map"], allowed)
    with pytest.raises(ValueError, match=r"unknown output field 'grad'; expected one of"):
        ops._select("grad", allowed)
    with pytest.raises(TypeError, match="output must be None, a field name, or a sequence of names"):
        ops._select(3, allowed)
    with pytest.raises(TypeError, match="output field names must be strings"):
        ops._select([1], allowed)


def test_primary_must_be_a_tensor():
    import orihime_b200 as ob

    with pytest.raises(TypeError, match="pair_scores must be a tensor"):
        ob.ops.sw_affine.sensitivity([[1.0]], gap_open_score=-1.0)
