"""Sums of medium gradients over processes (no reference counterpart).

Shots are independent: each process (one per GPU) runs the misfit gradients
of its own shots, and one collective adds the gradient volumes of all ranks,
in FP64 whatever the simulation's precision: per grid, the 22 volumes (node
buoyancy and the 21 stiffness slots) are packed into one FP64 device buffer
on the library's stream, all-reduced there (NCCL over NVLink when the process
group's backend is nccl), and unpacked back into the gradient.
"""
import torch
import torch.distributed as dist


def reduce_gradients_on(sim, group, device):
    """Pack, all-reduce and unpack the gradient of every grid of sim with FP64
    buffers on `device`, on the current stream."""
    bufs = [torch.empty(sim.gradient_elems(g), dtype=torch.float64, device=device) for g in range(sim.ng)]
    for g, b in enumerate(bufs):
        sim.pack_gradient(g, b.data_ptr())
    for b in bufs:
        dist.all_reduce(b, op=dist.ReduceOp.SUM, group=group)
    for g, b in enumerate(bufs):
        sim.unpack_gradient(g, b.data_ptr())


def allreduce_gradients(sim, group=None):
    """Replace sim's medium gradient by its sum over the ranks of `group`.

    Every rank calls this once per gradient pass with a simulation of the same
    geometry (same grids), in the same order as its other collectives.  The
    collective is enqueued on the simulation's stream, so device timers on that
    stream (Simulation.timer_start/stop) cover it; the call returns after the
    unpack has completed."""
    device = torch.device("cuda", sim.device)
    stream = torch.cuda.ExternalStream(sim.stream(), device=device)
    with torch.cuda.device(device), torch.cuda.stream(stream):
        reduce_gradients_on(sim, group, device)
        stream.synchronize()
