"""Turn-datagen helpers on the device: the pieces of the boundary-value
pipeline around the boundary-value network (cfvnet datagen, gpu-range-solver
batch.rs:765-790 and cfvnet/src/datagen/gpu_boundary_eval.rs:207-269)."""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .game import PostFlopGame


def boundary_reach(game: PostFlopGame):
    """Reach of each player at every depth boundary under the average strategy:
    a list over boundary ordinals of [reach of player 0 (H0), reach of player 1 (H1)]."""
    H0, H1 = game.num_private_hands(0), game.num_private_hands(1)
    nb = game.num_boundary_nodes()
    out = np.zeros(max(1, nb * (H0 + H1)), np.float32)
    N.check(N.lib().ps_boundary_reach(game._h, out.ctypes.data_as(C.POINTER(C.c_float))))
    return [[out[k * (H0 + H1):k * (H0 + H1) + H0].copy(), out[k * (H0 + H1) + H0:(k + 1) * (H0 + H1)].copy()]
            for k in range(nb)]


def boundary_river_reduce(boards, pots, stacks, net, reach, hands):
    """Reach-weighted average of boundary-network outputs over the 48 river
    cards, on the device (ps_boundary_river_reduce).

    boards [n, 4] card ids, pots / stacks [n] (host arrays); net [n, 2, 48, 1326],
    reach [n, 2, 1326] (OOP, IP) and hands [H] (int32 combo indices) are CUDA
    tensors.  Returns a CUDA tensor [n, 2, H]: player 0's values weighted by IP
    reach, player 1's by OOP reach, scaled by pot + stack."""
    import torch

    b = np.ascontiguousarray(boards, np.uint8).reshape(-1, 4)
    p = np.ascontiguousarray(pots, np.float32)
    s = np.ascontiguousarray(stacks, np.float32)
    n = b.shape[0]
    assert net.is_cuda and reach.is_cuda and hands.is_cuda
    net = net.contiguous().float()
    reach = reach.contiguous().float()
    hands = hands.contiguous().to(torch.int32)
    assert tuple(net.shape) == (n, 2, 48, 1326) and tuple(reach.shape) == (n, 2, 1326)
    out = torch.empty((n, 2, hands.numel()), dtype=torch.float32, device=net.device)
    stream = torch.cuda.current_stream(net.device).cuda_stream
    N.check(N.lib().ps_boundary_river_reduce(
        n, b.ctypes.data_as(C.POINTER(C.c_uint8)), p.ctypes.data_as(C.POINTER(C.c_float)),
        s.ctypes.data_as(C.POINTER(C.c_float)), C.c_void_p(net.data_ptr()), C.c_void_p(reach.data_ptr()),
        C.c_void_p(hands.data_ptr()), hands.numel(), C.c_void_p(out.data_ptr()), C.c_void_p(stream)))
    return out
