"""Public Saigo-Vert (canonical local alignment, D <- I allowed, only M ends)
functions, linear and affine gaps, signature-compatible with
orihime/sv.py:33-215."""

from __future__ import annotations

from typing import Optional

import torch
from torch import Tensor

from .operator import SV_AFFINE, SV_LINEAR, Operator

_sv_linear_operator = Operator(SV_LINEAR)
_sv_affine_operator = Operator(SV_AFFINE)


def sv(pair_scores: Tensor, *, gap_score=0.0, temperature=1.0, lengths: Optional[Tensor] = None,
       mask: Optional[Tensor] = None, dtype: Optional[torch.dtype] = None) -> Tensor:
    """Saigo-Vert linear-gap alignment map (dS/dscores)."""
    return _sv_linear_operator(pair_scores, gap_score, temperature, lengths=lengths, mask=mask,
                               dtype=dtype)


def sv_value(pair_scores: Tensor, *, gap_score=0.0, temperature=1.0,
             lengths: Optional[Tensor] = None, mask: Optional[Tensor] = None,
             dtype: Optional[torch.dtype] = None) -> Tensor:
    """Saigo-Vert linear-gap value S = LSE(0, M cells) per pair [B]."""
    return _sv_linear_operator.value(pair_scores, gap_score, temperature, lengths=lengths, mask=mask,
                                     dtype=dtype)


def sv_entropy(pair_scores: Tensor, *, gap_score=0.0, temperature=1.0,
               lengths: Optional[Tensor] = None, mask: Optional[Tensor] = None,
               dtype: Optional[torch.dtype] = None) -> Tensor:
    """Saigo-Vert linear-gap entropy observable dS/dT [B]."""
    return _sv_linear_operator.entropy(pair_scores, gap_score, temperature, lengths=lengths,
                                       mask=mask, dtype=dtype)


def sv_affine(pair_scores: Tensor, *, gap_open_score=0.0, gap_extend_score=0.0, temperature=1.0,
              lengths: Optional[Tensor] = None, mask: Optional[Tensor] = None,
              dtype: Optional[torch.dtype] = None) -> Tensor:
    """Saigo-Vert affine-gap alignment map (dS/dscores)."""
    return _sv_affine_operator(pair_scores, gap_open_score, gap_extend_score, temperature,
                               lengths=lengths, mask=mask, dtype=dtype)


def sv_affine_value(pair_scores: Tensor, *, gap_open_score=0.0, gap_extend_score=0.0,
                    temperature=1.0, lengths: Optional[Tensor] = None,
                    mask: Optional[Tensor] = None, dtype: Optional[torch.dtype] = None) -> Tensor:
    """Saigo-Vert affine-gap value S per pair [B]."""
    return _sv_affine_operator.value(pair_scores, gap_open_score, gap_extend_score, temperature,
                                     lengths=lengths, mask=mask, dtype=dtype)


def sv_affine_entropy(pair_scores: Tensor, *, gap_open_score=0.0, gap_extend_score=0.0,
                      temperature=1.0, lengths: Optional[Tensor] = None,
                      mask: Optional[Tensor] = None, dtype: Optional[torch.dtype] = None) -> Tensor:
    """Saigo-Vert affine-gap entropy observable dS/dT [B]."""
    return _sv_affine_operator.entropy(pair_scores, gap_open_score, gap_extend_score, temperature,
                                       lengths=lengths, mask=mask, dtype=dtype)


__all__ = ["sv", "sv_value", "sv_entropy", "sv_affine", "sv_affine_value", "sv_affine_entropy"]


# The linear-gap family's kernel name, kept as aliases as in orihime/sv.py:117-122.
sv_linear = sv
sv_linear_value = sv_value
sv_linear_entropy = sv_entropy
