"""Public soft Needleman-Wunsch (global alignment) functions, linear and
affine gaps, signature-compatible with orihime/nw.py:33-195."""

from __future__ import annotations

from typing import Optional

import torch
from torch import Tensor

from .operator import NW, NW_AFFINE, Operator

_nw_operator = Operator(NW)
_nw_affine_operator = Operator(NW_AFFINE)


def nw(pair_scores: Tensor, *, gap_score=0.0, temperature=1.0, lengths: Optional[Tensor] = None,
       mask: Optional[Tensor] = None, dtype: Optional[torch.dtype] = None) -> Tensor:
    """Soft global-alignment map (dS/dscores) of the linear-gap soft Needleman-Wunsch."""
    return _nw_operator(pair_scores, gap_score, temperature, lengths=lengths, mask=mask, dtype=dtype)


def nw_value(pair_scores: Tensor, *, gap_score=0.0, temperature=1.0,
             lengths: Optional[Tensor] = None, mask: Optional[Tensor] = None,
             dtype: Optional[torch.dtype] = None) -> Tensor:
    """Soft Needleman-Wunsch value S = A[L1, L2] per pair [B]."""
    return _nw_operator.value(pair_scores, gap_score, temperature, lengths=lengths, mask=mask,
                              dtype=dtype)


def nw_entropy(pair_scores: Tensor, *, gap_score=0.0, temperature=1.0,
               lengths: Optional[Tensor] = None, mask: Optional[Tensor] = None,
               dtype: Optional[torch.dtype] = None) -> Tensor:
    """Entropy observable dS/dT [B] of the global alignment; differentiable
    through pair_scores only."""
    return _nw_operator.entropy(pair_scores, gap_score, temperature, lengths=lengths, mask=mask,
                                dtype=dtype)


def nw_affine(pair_scores: Tensor, *, gap_open_score=0.0, gap_extend_score=0.0, temperature=1.0,
              lengths: Optional[Tensor] = None, mask: Optional[Tensor] = None,
              dtype: Optional[torch.dtype] = None) -> Tensor:
    """Soft global-alignment map (dS/dscores) of the affine-gap soft Needleman-Wunsch."""
    return _nw_affine_operator(pair_scores, gap_open_score, gap_extend_score, temperature,
                               lengths=lengths, mask=mask, dtype=dtype)


def nw_affine_value(pair_scores: Tensor, *, gap_open_score=0.0, gap_extend_score=0.0,
                    temperature=1.0, lengths: Optional[Tensor] = None,
                    mask: Optional[Tensor] = None, dtype: Optional[torch.dtype] = None) -> Tensor:
    """Soft Needleman-Wunsch value S = LSE(M, I, D at (L1, L2)) per pair [B] (affine gaps)."""
    return _nw_affine_operator.value(pair_scores, gap_open_score, gap_extend_score, temperature,
                                     lengths=lengths, mask=mask, dtype=dtype)


def nw_affine_entropy(pair_scores: Tensor, *, gap_open_score=0.0, gap_extend_score=0.0,
                      temperature=1.0, lengths: Optional[Tensor] = None,
                      mask: Optional[Tensor] = None, dtype: Optional[torch.dtype] = None) -> Tensor:
    """Entropy observable dS/dT [B] of the affine global alignment; differentiable
    through pair_scores only."""
    return _nw_affine_operator.entropy(pair_scores, gap_open_score, gap_extend_score, temperature,
                                       lengths=lengths, mask=mask, dtype=dtype)


__all__ = ["nw", "nw_value", "nw_entropy", "nw_affine", "nw_affine_value", "nw_affine_entropy"]
