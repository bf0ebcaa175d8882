"""Seeded synthetic inputs generated on the device (libzkp_gen.so), byte-identical to the
CPU oracle's generator: uniform Fr elements and bases P_i = k_i * G."""
from __future__ import annotations

import torch

from .native import check, load
from .scalar import require_cuda

LIB = "libzkp_gen.so"


def fr(seed: int, n: int, device="cuda", start: int = 0) -> torch.Tensor:
    """(n, 8) int32 device tensor of Montgomery-form Fr elements."""
    require_cuda()
    out = torch.empty((n, 8), dtype=torch.int32, device=device)
    check(load(LIB).zkp_gen_fr(seed, start, n, out.data_ptr(), torch.cuda.current_stream(out.device).cuda_stream),
          "zkp_gen_fr")
    return out


def points(seed: int, n: int, device="cuda", start: int = 0) -> torch.Tensor:
    """(n, 16) int32 device tensor of affine bases k_i * G (Montgomery Fq)."""
    require_cuda()
    out = torch.empty((n, 16), dtype=torch.int32, device=device)
    table = torch.empty((32 * 256, 16), dtype=torch.int32, device=device)
    check(load(LIB).zkp_gen_points(seed, start, n, table.data_ptr(), out.data_ptr(),
                                   torch.cuda.current_stream(out.device).cuda_stream), "zkp_gen_points")
    return out
