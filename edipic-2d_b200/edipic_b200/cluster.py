"""Several GPUs sharing one cluster's particles, as the processes of one cluster do in the reference: every rank holds
the whole grid and pushes its own share of the particles; the densities each rank deposits are summed over the ranks
(the cluster reduce of c_rho, GATHER_ELECTRON_CHARGE_DENSITY pic2d_ElectronDynamics.f90:1641 and
GATHER_ION_CHARGE_DENSITY), and every rank then solves the same field, as the reference broadcasts E to the
cluster's processes. In mixed precision the densities are int64 fixed point, so the sum is exact and the field is
the same on every rank, bit for bit.

The sums run through torch.distributed (NCCL between GPUs, or gloo), in place on the library's device buffers and
ordered on the library's stream.
"""
import numpy as np

ID_SPACE = 1 << 32


class _Buffer:
    """A buffer of `count` int64 or FP64 values at `ptr`, seen through __cuda_array_interface__ (device memory) or
    __array_interface__ (host memory, for tests on the CPU)."""

    def __init__(self, ptr, count, is_int64, device):
        iface = {"shape": (int(count),), "typestr": "<i8" if is_int64 else "<f8", "data": (int(ptr), False),
                 "version": 3, "strides": None}
        if device:
            self.__cuda_array_interface__ = iface
        else:
            self.__array_interface__ = iface


def allreduce_buffers(entries, device=True, group=None, stream=None, blocking=False):
    """Sums every (ptr, count, is_int64) buffer over the ranks of `group`, in place. On a device, the operations are
    ordered on `stream` (a cudaStream_t as an integer); blocking waits for them on the host as well (for backends
    such as gloo whose device work is not ordered on the caller's stream)."""
    import torch
    import torch.distributed as dist

    if not entries:
        return 0
    if not device:
        for ptr, count, is_int64 in entries:
            dist.all_reduce(torch.from_numpy(np.asarray(_Buffer(ptr, count, is_int64, False))), group=group)
        return len(entries)
    ext = torch.cuda.ExternalStream(stream) if stream else torch.cuda.current_stream()
    if blocking:
        ext.synchronize()
    with torch.cuda.stream(ext):
        for ptr, count, is_int64 in entries:
            t = torch.as_tensor(_Buffer(ptr, count, is_int64, True), device="cuda")
            dist.all_reduce(t, group=group)
    if blocking:
        torch.cuda.synchronize()
    return len(entries)


class ClusterShare:
    """One rank's part of a cluster shared by `world` ranks: a disjoint range of particle ids, and the sum of the
    densities after each step."""

    def __init__(self, sim, rank, world, group=None, blocking=False, device=True):
        self.sim, self.rank, self.world, self.group, self.blocking = sim, rank, world, group, blocking
        self.device = device
        sim.set_id_base(rank * (ID_SPACE // world), (rank + 1) * (ID_SPACE // world))

    def reduce(self):
        """GATHER_*_CHARGE_DENSITY's cluster reduce: call after the distribution or upload and after every step."""
        if self.world == 1:
            self.sim.reduce_list()   # nothing to sum; clears the list
            return 0
        return allreduce_buffers(self.sim.reduce_list(), self.device, self.group,
                                 self.sim.stream() if self.device else None, self.blocking)

    def step(self, n=1):
        for _ in range(n):
            self.sim.step(1)
            self.reduce()
