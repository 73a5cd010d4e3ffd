"""Public soft Smith-Waterman functions, signature-compatible with orihime/sw.py:32-200."""

from __future__ import annotations

from typing import Optional

import torch
from torch import Tensor

from .operator import SW, SW_AFFINE, Operator

_sw_operator = Operator(SW)
_sw_affine_operator = Operator(SW_AFFINE)


def sw(pair_scores: Tensor, *, gap_score=0.0, temperature=1.0, lengths: Optional[Tensor] = None,
       mask: Optional[Tensor] = None, dtype: Optional[torch.dtype] = None) -> Tensor:
    """Soft local-alignment map (dS/dscores) of the linear-gap soft Smith-Waterman."""
    return _sw_operator(pair_scores, gap_score, temperature, lengths=lengths, mask=mask, dtype=dtype)


def sw_value(pair_scores: Tensor, *, gap_score=0.0, temperature=1.0,
             lengths: Optional[Tensor] = None, mask: Optional[Tensor] = None,
             dtype: Optional[torch.dtype] = None) -> Tensor:
    """Soft Smith-Waterman value S [B] (linear gap)."""
    return _sw_operator.value(pair_scores, gap_score, temperature, lengths=lengths, mask=mask,
                              dtype=dtype)


def sw_entropy(pair_scores: Tensor, *, gap_score=0.0, temperature=1.0,
               lengths: Optional[Tensor] = None, mask: Optional[Tensor] = None,
               dtype: Optional[torch.dtype] = None) -> Tensor:
    """Entropy observable dS/dT [B] (linear gap); differentiable through pair_scores only."""
    return _sw_operator.entropy(pair_scores, gap_score, temperature, lengths=lengths, mask=mask,
                                dtype=dtype)


def sw_affine(pair_scores: Tensor, *, gap_open_score=0.0, gap_extend_score=0.0, temperature=1.0,
              lengths: Optional[Tensor] = None, mask: Optional[Tensor] = None,
              dtype: Optional[torch.dtype] = None) -> Tensor:
    """Soft local-alignment map (dS/dscores) of the affine-gap soft Smith-Waterman."""
    return _sw_affine_operator(pair_scores, gap_open_score, gap_extend_score, temperature,
                               lengths=lengths, mask=mask, dtype=dtype)


def sw_affine_value(pair_scores: Tensor, *, gap_open_score=0.0, gap_extend_score=0.0,
                    temperature=1.0, lengths: Optional[Tensor] = None,
                    mask: Optional[Tensor] = None, dtype: Optional[torch.dtype] = None) -> Tensor:
    """Soft Smith-Waterman value S [B] (affine gaps)."""
    return _sw_affine_operator.value(pair_scores, gap_open_score, gap_extend_score, temperature,
                                     lengths=lengths, mask=mask, dtype=dtype)


def sw_affine_entropy(pair_scores: Tensor, *, gap_open_score=0.0, gap_extend_score=0.0,
                      temperature=1.0, lengths: Optional[Tensor] = None,
                      mask: Optional[Tensor] = None, dtype: Optional[torch.dtype] = None) -> Tensor:
    """Entropy observable dS/dT [B] (affine gaps); differentiable through pair_scores only."""
    return _sw_affine_operator.entropy(pair_scores, gap_open_score, gap_extend_score, temperature,
                                       lengths=lengths, mask=mask, dtype=dtype)


__all__ = ["sw", "sw_value", "sw_entropy", "sw_affine", "sw_affine_value", "sw_affine_entropy"]
