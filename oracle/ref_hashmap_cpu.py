"""CPU restatement of the two reference hashmap operations that
o_voxel.convert.flexible_dual_grid_to_mesh calls (test infrastructure only).

The reference runs them as CUDA kernels (src/hash/hash.cu); the golden fixture
script (tests/golden/make_to_mesh_golden.py) runs the reference's own Python
function with these in their place, on CPU tensors.  A GPU test pins this
restatement against the reference kernels compiled from their source
(oracle/_ref/hash_ref, built by oracle/build.py).

* ``hashmap_insert_3d_idx_as_val_cuda(keys, vals, coords, W, H, D)``
  (hash.cu:366-420): coords are int32 [M,4] rows (b, x, y, z); row i is
  stored under the flat key b*W*H*D + x*H*D + y*D + z (size_t, then cast to
  the key type: uint32 or uint64) with value i.  No bounds check on insert.
  A repeated key overwrites the value (hash.cu:34-37; which of several
  threads writes last is unordered there, so repeats are not relied on).
* ``hashmap_lookup_3d_cuda(keys, vals, coords, W, H, D)`` (hash.cu:269-300):
  a row with x, y or z outside [0, W) x [0, H) x [0, D) gives the value
  type's maximum without a lookup; otherwise the value stored under the flat
  key, or the maximum when the key is absent (linear probing ends at an
  empty slot, hash.cu:70-88).

The table contents (and so the Murmur3 slot order, hash.cu:1-20) do not change
what a lookup returns while the table has a free slot, which the caller
guarantees with a capacity of 2N; the restatement keeps a dict beside the
caller's key tensor instead of probing it.
"""
import numpy as np
import torch

_TABLES = {}


def _key_mask(keys: torch.Tensor) -> int:
    return 0xFFFFFFFF if keys.dtype == torch.uint32 else 0xFFFFFFFFFFFFFFFF


def _flat(coords: np.ndarray, W: int, H: int, D: int) -> np.ndarray:
    c = coords.astype(np.int64)
    return (c[:, 0] * (W * H * D) + c[:, 1] * (H * D) + c[:, 2] * D + c[:, 3]).astype(np.uint64)


def hashmap_insert_3d_idx_as_val_cuda(keys: torch.Tensor, vals: torch.Tensor, coords: torch.Tensor, W: int, H: int, D: int):
    c = coords.cpu().numpy()
    flat = _flat(c, W, H, D) & np.uint64(_key_mask(keys))
    table = _TABLES.setdefault(id(keys), {})
    for i, k in enumerate(flat.tolist()):
        table[k] = i


def hashmap_lookup_3d_cuda(keys: torch.Tensor, vals: torch.Tensor, coords: torch.Tensor, W: int, H: int, D: int) -> torch.Tensor:
    c = coords.cpu().numpy().astype(np.int64)
    vmax = 0xFFFFFFFF if vals.dtype == torch.uint32 else 0xFFFFFFFFFFFFFFFF
    inside = (c[:, 1] >= 0) & (c[:, 1] < W) & (c[:, 2] >= 0) & (c[:, 2] < H) & (c[:, 3] >= 0) & (c[:, 3] < D)
    flat = _flat(c, W, H, D) & np.uint64(_key_mask(keys))
    table = _TABLES.get(id(keys), {})
    out = np.array([table.get(k, vmax) if ok else vmax for k, ok in zip(flat.tolist(), inside.tolist())], dtype=np.uint64)
    return torch.from_numpy(out.astype(np.uint32 if vals.dtype == torch.uint32 else np.uint64)).to(vals.device)


def clear():
    _TABLES.clear()
