"""Serialisation codes of voxel coordinates (reference o_voxel/serialize.py:7-36).

encode_seq / decode_seq with mode='z_order' run on CUDA tensors through the
library (ovx_z_order_encode / ovx_z_order_decode): 10 bits per coordinate, x
the most significant bit of each triple, int32 codes.  The reference also
offers CPU tensors and a Hilbert mode; neither is on the
mesh -> flexible dual grid path, and both raise here.
"""
from typing import List

import torch

from .convert.flexible_dual_grid import _ext

__all__ = ["encode_seq", "decode_seq"]


def _check_mode(mode: str, device: torch.device):
    if mode == "hilbert":
        raise NotImplementedError("mode='hilbert' is not provided by this implementation (z_order only)")
    if mode != "z_order":
        raise ValueError(f"Unknown encoding mode: {mode}")
    if device.type != "cuda":
        raise RuntimeError(f"this implementation runs on CUDA tensors only (got a {device} tensor)")


@torch.no_grad()
def encode_seq(coords: torch.Tensor, permute: List[int] = [0, 1, 2], mode: str = "z_order") -> torch.Tensor:
    """
    Encode [N, 3] voxel coordinates (each in [0, 1024)) into 30-bit int32 z-order codes.

    Args:
        coords: [N, 3] integer coordinates (CUDA).
        permute: which coordinate column is used as x, y and z.
        mode: 'z_order'.
    """
    assert coords.shape[-1] == 3 and coords.ndim == 2, "Input coordinates must be of shape [N, 3]"
    _check_mode(mode, coords.device)
    x = coords[:, permute[0]].int()
    y = coords[:, permute[1]].int()
    z = coords[:, permute[2]].int()
    return _ext().z_order_encode_cuda(x, y, z)


@torch.no_grad()
def decode_seq(code: torch.Tensor, permute: List[int] = [0, 1, 2], mode: str = "z_order") -> torch.Tensor:
    """
    Decode [N] z-order codes into [N, 3] int32 coordinates (inverse of encode_seq).
    """
    assert code.ndim == 1, "Input code must be of shape [N]"
    _check_mode(mode, code.device)
    x, y, z = _ext().z_order_decode_cuda(code)
    coords = torch.empty(code.shape[0], 3, dtype=torch.int32, device=code.device)
    coords[:, permute[0]] = x
    coords[:, permute[1]] = y
    coords[:, permute[2]] = z
    return coords
