"""G'-column sharding of one Sigma evaluation over several GPUs.

BerkeleyGW distributes the G' columns of the screened interaction over MPI
tasks (`ngpown = ncouls / (nodes_per_group * npes)`, GPP/gpp.cpp:144, 162;
"plane waves per MPI task", FF/ff.cpp:48-49).  Every sum of the GPP and FF
kernels is over independent (band, G', G) terms, so rank r evaluates the
contiguous column block [p0, p1) with its own GPU -- its slice of
inv_igp_index and of the [ngpown][...] arrays (wtilde_array, I_eps_array,
or I_epsR/I_epsA[:, p0:p1, :]) plus the replicated band arrays -- and the
only exchange is the gather of the partial outputs: 3 complex (GPP
achtemp; 6 with the screened exchange) or 1 + 2 nfreqeval complex (FF) per
rank.  The partials are all-gathered and
summed in rank order, so the result is bitwise reproducible for a given
world size.  One process per GPU; `torch.distributed` (NCCL on GPUs, gloo
on CPU) carries the gather.
"""
from __future__ import annotations

import dataclasses
from typing import Callable, Optional

import numpy as np

from .inputs import FFInputs, GppInputs


def _on_host(inp) -> bool:
    return isinstance(inp.wtilde_array if isinstance(inp, GppInputs) else inp.aqsmtemp, np.ndarray)


def column_range(ngpown: int, world: int, rank: int) -> tuple[int, int]:
    """Contiguous, balanced block of G' columns owned by `rank`."""
    base, extra = divmod(ngpown, world)
    p0 = rank * base + min(rank, extra)
    return p0, p0 + base + (1 if rank < extra else 0)


def _rows(a, p0: int, p1: int, axis: int = 0):
    """Contiguous copy of rows [p0, p1) along `axis` (numpy or torch)."""
    sl = (slice(None),) * axis + (slice(p0, p1),)
    if type(a).__module__.startswith("torch"):
        return a[sl].contiguous()
    return np.ascontiguousarray(a[sl])


def gpp_shard(inp: GppInputs, world: int, rank: int) -> GppInputs:
    p0, p1 = column_range(inp.ngpown, world, rank)
    return dataclasses.replace(
        inp, ngpown=p1 - p0,
        inv_igp_index=_rows(inp.inv_igp_index, p0, p1),
        wtilde_array=_rows(inp.wtilde_array, p0, p1),
        I_eps_array=_rows(inp.I_eps_array, p0, p1))


def ff_shard(inp: FFInputs, world: int, rank: int) -> FFInputs:
    p0, p1 = column_range(inp.ngpown, world, rank)
    return dataclasses.replace(
        inp, ngpown=p1 - p0,
        inv_igp_index=_rows(inp.inv_igp_index, p0, p1),
        I_epsR_array=_rows(inp.I_epsR_array, p0, p1, axis=1),
        I_epsA_array=_rows(inp.I_epsA_array, p0, p1, axis=1))


def gather_sum(partial, group=None, device=None) -> np.ndarray:
    """All-gathers a complex partial from every rank and sums it in rank
    order (fixed order: bitwise reproducible).  Collective: every rank of
    `group` must call it.  `partial`: numpy array or torch tensor.  Under
    NCCL the gather runs on `device` (default: the current CUDA device),
    since NCCL takes CUDA tensors only; under gloo it runs on the host."""
    import torch
    import torch.distributed as dist
    if type(partial).__module__.startswith("torch"):
        partial = partial.detach().cpu().numpy()
    x = np.ascontiguousarray(np.atleast_1d(partial).astype(np.complex128)).view(np.float64)
    t = torch.from_numpy(x.copy())
    if dist.get_backend(group) == "nccl":
        t = t.to(device if device is not None else torch.device("cuda", torch.cuda.current_device()))
    world = dist.get_world_size(group)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    total = np.zeros_like(x)
    for p in parts:                      # rank order
        total += p.cpu().numpy()
    return total.view(np.complex128)


def gpp_sharded(inp: GppInputs, world: int, rank: int, group=None,
                compute: Optional[Callable] = None, device=None) -> np.ndarray:
    """achtemp[3] of the whole problem; this rank computes its column block
    with `compute` (default: the GPU library)."""
    shard = gpp_shard(inp, world, rank)
    if compute is None:
        from . import noflagOCC_solver, to_device

        def compute(s):
            return noflagOCC_solver(to_device(s, device) if device is not None and _on_host(s) else s)
    local = compute(shard)
    if hasattr(local, "cpu"):
        local = local.cpu().numpy()
    return gather_sum(np.asarray(local, dtype=np.complex128), group, device)


def gpp_sigma_sharded(inp: GppInputs, world: int, rank: int, group=None,
                      compute: Optional[Callable] = None, device=None):
    """(achtemp[3], asxtemp[3]) of the whole problem (bgw_gpp_sigma: the
    Coulomb-hole sum and the occupied bands' screened exchange, both sums
    over G' columns); this rank computes its column block with `compute`
    (default: the GPU library), which returns the two outputs."""
    shard = gpp_shard(inp, world, rank)
    if compute is None:
        from . import gpp_sigma, to_device

        def compute(s):
            src = to_device(s, device) if device is not None and _on_host(s) else s
            return tuple(np.asarray(o.cpu().numpy() if hasattr(o, "cpu") else o) for o in gpp_sigma(src))
    ach, asx = compute(shard)
    tot = gather_sum(np.concatenate([np.atleast_1d(ach), np.atleast_1d(asx)]), group, device)
    return tot[:3], tot[3:6]


def ff_sharded(inp: FFInputs, world: int, rank: int, group=None,
               compute: Optional[Callable] = None, device=None):
    """(achsDtemp, asxDtemp[nfreqeval], achDtemp_cor[nfreqeval]) of the whole
    problem; this rank computes its column block with `compute` (default:
    the GPU library), which returns the three outputs."""
    shard = ff_shard(inp, world, rank)
    if compute is None:
        from . import ff_sigma, to_device

        def compute(s):
            src = to_device(s, device) if device is not None and _on_host(s) else s
            out = ff_sigma(src)
            return tuple(np.asarray(o.cpu().numpy() if hasattr(o, "cpu") else o) for o in out)
    achs, asx, cor = compute(shard)
    E = inp.nfreqeval
    flat = np.concatenate([np.atleast_1d(achs)[:1], np.atleast_1d(asx)[:E], np.atleast_1d(cor)[:E]])
    tot = gather_sum(flat, group, device)
    return tot[0], tot[1:1 + E], tot[1 + E:1 + 2 * E]
