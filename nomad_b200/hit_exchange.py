"""The per-object hit counters of a frame split over ranks.

A frame (or a camera path's views) can be rendered by several GPUs, one process per GPU, each with
a full scene replica: every rank renders its own views or pixel tiles with hit counting on. The
residency step must then see the whole frame's counts, or the ranks would keep different
resident sets. `allreduce_object_hits` sums the counts of all ranks (one all-reduce of
object_count 32-bit words, 8 KB at 2,048 objects) and writes the sum back into every rank's
counters, so the residency steps that follow take the same decisions on every rank. With the
radiance bands of a frame split by rows (nomad_b200.split_frame) it is the only exchange between
ranks on this path; geometry and rays never cross.

With the NCCL backend the counts stay on the device (device-to-device copies around the
all-reduce, over NVLink) and are summed as 32-bit integers, so an object's summed count must stay
below 2^31 in one frame (the rays of a frame are far fewer); with any other backend (gloo) they go
through host memory and are summed as 64-bit integers, with an error if a sum exceeds 32 bits.
"""
from __future__ import annotations

import numpy as np


def allreduce_object_hits(ctx, group=None) -> np.ndarray | None:
    """Sums the per-object closest-hit counts of every rank of `group` into each rank's context.

    `ctx` is a nomad_b200 Context (or any object with the same object_count, object_hits,
    write_object_hits and, for NCCL, object_hits_dev methods). Returns the summed counts as a
    host array for a host-memory backend, None for NCCL (where they never leave the device)."""
    import torch
    import torch.distributed as dist

    n = int(ctx.object_count)
    if dist.get_backend(group) == "nccl":
        t = torch.empty(n, dtype=torch.int32, device="cuda")
        ctx.sync()  # the counters are complete once the rank's render is
        ctx.object_hits_dev(t.data_ptr())
        ctx.sync()
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        torch.cuda.current_stream().synchronize()
        ctx.write_object_hits(dev_ptr=t.data_ptr())
        ctx.sync()
        return None
    local = np.asarray(ctx.object_hits(), np.uint32)
    # int64 on the wire: a sum of u32 counts over ranks does not fit int32
    t = torch.from_numpy(local.astype(np.int64))
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    total = t.numpy()
    if total.max(initial=0) > 0xFFFFFFFF:
        raise OverflowError("per-object hit counts exceed 32 bits after the sum over ranks")
    total = total.astype(np.uint32)
    ctx.write_object_hits(total)
    return total
