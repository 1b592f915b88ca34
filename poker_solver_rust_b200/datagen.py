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

    boards [n, 4] card ids, pots / stacks [n] (host arrays); net [n, 2, 48, 1326]
    (f32 or bf16), reach [n, 2, 1326] (OOP, IP) and hands [H] (int32 combo
    indices) are CUDA tensors.  Returns a CUDA tensor [n, 2, H]: player 0's
    values weighted by IP reach, player 1's by OOP reach, scaled by pot + stack."""
    import torch

    b = np.ascontiguousarray(boards, np.uint8).reshape(-1, 4)
    p = np.ascontiguousarray(pots, np.float32)
    s = np.ascontiguousarray(stacks, np.float32)
    n = b.shape[0]
    assert net.is_cuda and reach.is_cuda and hands.is_cuda
    bf16 = net.dtype == torch.bfloat16
    net = net.contiguous() if bf16 else net.contiguous().float()
    reach = reach.contiguous().float()
    hands = hands.contiguous().to(torch.int32)
    assert tuple(net.shape) == (n, 2, 48, 1326) and tuple(reach.shape) == (n, 2, 1326)
    out = torch.empty((n, 2, hands.numel()), dtype=torch.float32, device=net.device)
    stream = torch.cuda.current_stream(net.device).cuda_stream
    N.check(N.lib().ps_boundary_river_reduce(
        n, b.ctypes.data_as(C.POINTER(C.c_uint8)), p.ctypes.data_as(C.POINTER(C.c_float)),
        s.ctypes.data_as(C.POINTER(C.c_float)), C.c_void_p(net.data_ptr()), int(bf16), C.c_void_p(reach.data_ptr()),
        C.c_void_p(hands.data_ptr()), hands.numel(), C.c_void_p(out.data_ptr()), C.c_void_p(stream)))
    return out


_CARD_COMBOS = {}


def _card_combos(device):
    """[52, 51] combo indices holding each card (card_pair_to_index order)."""
    import torch

    key = str(device)
    if key not in _CARD_COMBOS:
        idx = [[a * (101 - a) // 2 + b - 1 if a < b else b * (101 - b) // 2 + a - 1 for b in range(52) if b != a]
               for a in range(52)]
        _CARD_COMBOS[key] = torch.tensor(idx, dtype=torch.int64, device=device)
    return _CARD_COMBOS[key]


def boundary_first_layer(boards, pots, stacks, reach, weight, bias=None, bf16: bool = False):
    """The first Linear layer (weight [h, 2720], bias [h]) of a boundary
    network over every input row of boundary_encode, without writing the rows
    (ps_boundary_first_layer): [n, 2, 48, h].  One GEMM over the n reach rows
    and one batched GEMM per card replace the layer's GEMM over 96 n rows."""
    import torch

    b = np.ascontiguousarray(boards, np.uint8).reshape(-1, 4)
    p = np.ascontiguousarray(pots, np.float32)
    s = np.ascontiguousarray(stacks, np.float32)
    n, h = b.shape[0], weight.shape[0]
    assert reach.is_cuda and tuple(reach.shape) == (n, 2, 1326) and tuple(weight.shape) == (h, 2720)
    W = weight.detach().float()
    R = reach.contiguous().float()
    Wr = W[:, :2652]
    base = (R.view(n, 2652) @ Wr.t()).contiguous()  # [n, h]
    idx = _card_combos(R.device)
    A = R[:, :, idx].permute(2, 0, 1, 3).reshape(52, n, 102)  # reach of the combos holding each card
    G = Wr.view(h, 2, 1326)[:, :, idx].permute(2, 1, 3, 0).reshape(52, 102, h)
    percard = torch.bmm(A, G).permute(1, 0, 2).contiguous()  # [n, 52, h]
    wcols = W[:, 2652:].t().contiguous()  # [68, h]
    bias_f = None if bias is None else bias.detach().float().contiguous()
    out = torch.empty((n, 2, 48, h), dtype=torch.bfloat16 if bf16 else torch.float32, device=R.device)
    if n == 0:
        return out
    stream = torch.cuda.current_stream(R.device).cuda_stream
    N.check(N.lib().ps_boundary_first_layer(
        n, b.ctypes.data_as(C.POINTER(C.c_uint8)), p.ctypes.data_as(C.POINTER(C.c_float)),
        s.ctypes.data_as(C.POINTER(C.c_float)), C.c_void_p(base.data_ptr()), C.c_void_p(percard.data_ptr()),
        C.c_void_p(wcols.data_ptr()), C.c_void_p(0 if bias_f is None else bias_f.data_ptr()), h,
        C.c_void_p(out.data_ptr()), int(bf16), C.c_void_p(stream)))
    return out


def boundary_encode(boards, pots, stacks, reach, bf16: bool = False):
    """Boundary-network input rows on the device (ps_boundary_encode):
    [n, 2, 48, 2720] for n items, their two players and the 48 river cards
    not on each 4-card board (cfvnet eval/boundary_evaluator.rs:27-60).

    boards [n, 4], pots / stacks [n] are host arrays; reach [n, 2, 1326]
    (OOP, IP) is a CUDA tensor.  Returns a CUDA tensor, f32 or bf16."""
    import torch

    b = np.ascontiguousarray(boards, np.uint8).reshape(-1, 4)
    p = np.ascontiguousarray(pots, np.float32)
    s = np.ascontiguousarray(stacks, np.float32)
    n = b.shape[0]
    assert reach.is_cuda and tuple(reach.shape) == (n, 2, 1326)
    reach = reach.contiguous().float()
    out = torch.empty((n, 2, 48, 2720), dtype=torch.bfloat16 if bf16 else torch.float32, device=reach.device)
    if n == 0:
        return out
    stream = torch.cuda.current_stream(reach.device).cuda_stream
    N.check(N.lib().ps_boundary_encode(
        n, b.ctypes.data_as(C.POINTER(C.c_uint8)), p.ctypes.data_as(C.POINTER(C.c_float)),
        s.ctypes.data_as(C.POINTER(C.c_float)), C.c_void_p(reach.data_ptr()), C.c_void_p(out.data_ptr()),
        int(bf16), C.c_void_p(stream)))
    return out


def _split_first_linear(net):
    """(first Linear(2720, h), the rest) of an nn.Sequential that starts with
    one, else None."""
    import torch

    if isinstance(net, torch.nn.Sequential) and len(net) > 1 and isinstance(net[0], torch.nn.Linear) \
            and net[0].in_features == 2720:
        return net[0], net[1:]
    return None


def evaluate_boundaries(items: dict, reach, net, pot_source: str = "boundary", denormalize: bool = False,
                        bf16: bool = False, chunk_items: int = 1024, factored: bool = True):
    """Boundary values of every item from a boundary-value network, all on
    the device: input rows (boundary_encode) -> net -> reach-weighted 48-river
    average (boundary_river_reduce); the host steps of the reference's
    datagen/gpu_boundary_eval.rs:107-269.

    items: BatchSolver.boundary_items(); reach: [items, 2, 1326] CUDA tensor
    (BatchSolver.boundary_reach(device=True)); net: a callable mapping
    [rows, 2720] to [rows, 1326].  pot_source: "boundary" encodes each
    boundary's own pot and stack (as cfvnet datagen/domain/
    neural_net_evaluator.rs:109-110 does), "root" the spot's starting pot and
    stack (as datagen/domain/pipeline.rs:818-819 does).  denormalize: scale
    the averages by pot + stack (chips), as gpu_boundary_eval.rs:238-256 does.
    factored: when net is an nn.Sequential that starts with Linear(2720, h),
    its first layer runs as boundary_first_layer (no input rows are written)
    and the rest of the net on its output.
    Returns [items, 2, 1326] (combo layout) for BatchSolver.set_boundary_cfvs."""
    import torch

    n = len(items["spot"])
    if pot_source == "root":
        pots, stacks = items["root_pots"], items["root_stacks"]
    else:
        pots, stacks = items["pots"], items["stacks"]
    out = torch.empty((n, 2, 1326), dtype=torch.float32, device=reach.device)
    combos = torch.arange(1326, dtype=torch.int32, device=reach.device)
    for a in range(0, n, chunk_items):
        z = slice(a, min(n, a + chunk_items))
        m = z.stop - z.start
        split = _split_first_linear(net) if factored else None
        p = next(net.parameters(), None) if hasattr(net, "parameters") else None
        with torch.no_grad():
            if split is not None:
                first, rest = split
                x = boundary_first_layer(items["boards"][z], pots[z], stacks[z], reach[z], first.weight, first.bias,
                                         bf16=p is not None and p.dtype == torch.bfloat16)
                x = x.view(m * 96, first.out_features)
                if p is not None and p.dtype != x.dtype:
                    x = x.to(p.dtype)
                y = rest(x).view(m, 2, 48, 1326)
            else:
                x = boundary_encode(items["boards"][z], pots[z], stacks[z], reach[z], bf16=bf16).view(m * 96, 2720)
                if p is not None and p.dtype != x.dtype:
                    x = x.to(p.dtype)
                y = net(x).view(m, 2, 48, 1326)
            if y.dtype not in (torch.float32, torch.bfloat16):
                y = y.float()
        if denormalize:
            dp, ds = pots[z], stacks[z]
        else:
            dp, ds = np.ones(m, np.float32), np.zeros(m, np.float32)
        out[z] = boundary_river_reduce(items["boards"][z], dp, ds, y, reach[z], combos)
    return out


def solve_with_boundary_net(batch, net, iterations: int, eval_interval: int, **eval_kwargs):
    """The turn-datagen loop of cfvnet datagen/domain/pipeline.rs:648-700 on a
    batch of depth-limited spots, with every step on the device: boundary
    values from the network under the uniform strategy, then every
    `eval_interval` iterations again from the reach under the current average
    strategy, until `iterations`.  One launch per interval runs its
    iterations plus the average-strategy epilogue that yields the next
    boundary reach; the last one also the exploitability and the root
    cfvalues (BatchSolver.results / root_cfvalues).  Returns the items."""
    items = batch.boundary_items()
    batch.reset()
    batch.run_iterations(0, 0, root=True)  # average strategy of zero sums: uniform
    t = 0
    while True:
        reach = batch.boundary_reach(device=True)
        batch.set_boundary_cfvs(evaluate_boundaries(items, reach, net, **eval_kwargs))
        end = min(iterations, t + eval_interval)
        batch.run_iterations(t, end, root=True, exploitability=end >= iterations)
        t = end
        if t >= iterations:
            return items
