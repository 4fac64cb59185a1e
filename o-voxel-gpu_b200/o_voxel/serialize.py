"""Serialisation codes of voxel coordinates (reference o_voxel/serialize.py:7-66).

encode_seq / decode_seq run on CUDA tensors through the library, with 10 bits
per coordinate and int32 codes:

* mode='z_order' (ovx_z_order_encode / ovx_z_order_decode): the bits of x, y
  and z interleaved, x the most significant of each triple;
* mode='hilbert' (ovx_hilbert_encode / ovx_hilbert_decode): J. Skilling's
  transposed Hilbert index, its three words interleaved the same way.

The reference also accepts CPU tensors (its CPU loops); here they raise.
"""
from typing import List

import torch

from .convert.flexible_dual_grid import _ext

__all__ = ["encode_seq", "decode_seq"]


def _check_mode(mode: str, device: torch.device):
    if mode not in ("z_order", "hilbert"):
        raise ValueError(f"Unknown encoding mode: {mode}")
    if device.type != "cuda":
        raise RuntimeError(f"this implementation runs on CUDA tensors only (got a {device} tensor)")


@torch.no_grad()
def encode_seq(coords: torch.Tensor, permute: List[int] = [0, 1, 2], mode: str = "z_order") -> torch.Tensor:
    """
    Encode [N, 3] voxel coordinates (each in [0, 1024)) into 30-bit int32 codes.

    Args:
        coords: [N, 3] integer coordinates (CUDA).
        permute: which coordinate column is used as x, y and z.
        mode: 'z_order' or 'hilbert'.
    """
    assert coords.shape[-1] == 3 and coords.ndim == 2, "Input coordinates must be of shape [N, 3]"
    _check_mode(mode, coords.device)
    x = coords[:, permute[0]].int()
    y = coords[:, permute[1]].int()
    z = coords[:, permute[2]].int()
    if mode == "hilbert":
        return _ext().hilbert_encode_cuda(x, y, z)
    return _ext().z_order_encode_cuda(x, y, z)


@torch.no_grad()
def decode_seq(code: torch.Tensor, permute: List[int] = [0, 1, 2], mode: str = "z_order") -> torch.Tensor:
    """
    Decode [N] codes into [N, 3] int32 coordinates (inverse of encode_seq with the same mode).
    """
    assert code.ndim == 1, "Input code must be of shape [N]"
    _check_mode(mode, code.device)
    x, y, z = (_ext().hilbert_decode_cuda if mode == "hilbert" else _ext().z_order_decode_cuda)(code)
    coords = torch.empty(code.shape[0], 3, dtype=torch.int32, device=code.device)
    coords[:, permute[0]] = x
    coords[:, permute[1]] = y
    coords[:, permute[2]] = z
    return coords
