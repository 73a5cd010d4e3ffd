"""Public soft Needleman-Wunsch (global alignment, linear gap) functions,
signature-compatible with orihime/nw.py:33-111."""

from __future__ import annotations

from typing import Optional

import torch
from torch import Tensor

from .operator import NW, Operator

_nw_operator = Operator(NW)


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


__all__ = ["nw", "nw_value", "nw_entropy"]
