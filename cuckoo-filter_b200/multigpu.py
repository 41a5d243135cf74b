"""Hash-partitioned filter over the GPUs of a process group (one process per GPU).

The reference's ``CuckooFilterMultiGPU<Config>(numGPUs, capacity)``
(``include/CuckooFilterMultiGPU.cuh``) drives N GPUs from one host thread.
Each GPU gets a slice of a host vector and groups it by destination GPU
(``hash64(key) % numGPUs``, its ``Partitioner`` at :44-50) with a gossip
multisplit (:226-234).  The groups are exchanged all-to-all over peer copies
(:247-254), each GPU runs the single-GPU batch operation on what it received
(:257-288), and lookups and deletes send their per-key results back the same
way (:292-312).  Each GPU owns an independent filter of
``SDIV(capacity, numGPUs) * 1.02`` slots (:337).

Here every GPU is its own process in a ``torch.distributed`` group (NCCL over
NVLink/NVSwitch), and every rank calls each operation with ITS OWN batch (the
slice the reference would have copied to that GPU):

1. ``cf_shard_partition`` groups the batch by destination rank on the device
   (two HBM passes, no host round trip);
2. one ``all_to_all_single`` of the per-rank key counts, then one of the keys;
3. the rank's own filter runs the batch operation on the keys it received;
4. for lookups and deletes, one ``all_to_all_single`` of the 1-byte results
   back, and ``cf_shard_unpartition`` puts them at their batch positions.

Results are aligned with the caller's keys; the reference leaves them in its
multisplit order.  Every rank makes the same calls in the same order, because
they are collectives.  Batches larger than ``max_keys_per_call`` on any rank
are processed in rounds that all ranks take together.
"""
from __future__ import annotations

import numpy as np

from . import CuckooConfig, CuckooFilter, _check, _stream_handle, library


# cf_shard_routing: the reference's hash64(key) % N, or splitmix64's output
# mixer applied to hash64(key) first (shard independent of the buckets)
ROUTING_REFERENCE, ROUTING_REMIXED = 0, 1
_ROUTINGS = {"reference": ROUTING_REFERENCE, "remixed": ROUTING_REMIXED}


def capacity_per_gpu(capacity: int, num_gpus: int) -> int:
    """``static_cast<size_t>(SDIV(capacity, numGPUs) * 1.02)``
    (CuckooFilterMultiGPU.cuh:337)."""
    return int(float(-(-int(capacity) // int(num_gpus))) * 1.02)


class KeyGrouping:
    """The grouping kernels (``cf_shard_partition`` / ``cf_shard_unpartition``)
    on one device, with their workspace.  ``unpartition`` reads the run starts
    that the last ``partition`` left in the workspace, so it takes the results
    of that batch."""

    def __init__(self, device, key_bytes: int):
        import torch

        self.torch, self.device, self.key_bytes = torch, torch.device(device), int(key_bytes)
        self._ws = None
        self._wsb = 0
        self._ns = 0
        self._L = library()

    def partition(self, keys, num_shards: int, routing: int = 0):
        """(keys grouped by shard, batch position of each grouped key (int32),
        keys per shard (int64)), all on the device.  `routing` is
        ROUTING_REFERENCE or ROUTING_REMIXED."""
        torch = self.torch
        n = keys.numel()
        wsb = int(self._L.cf_shard_workspace_bytes(n, num_shards))
        if wsb == 0:
            raise ValueError("num_shards must be 1..256")
        if self._ws is None or self._ws.numel() < wsb:
            self._ws = torch.empty(wsb, dtype=torch.uint8, device=self.device)
        grouped = torch.empty_like(keys)
        pos = torch.empty(n, dtype=torch.int32, device=self.device)
        counts = torch.empty(num_shards, dtype=torch.int64, device=self.device)
        _check(self._L.cf_shard_partition(keys.data_ptr() or None, n, self.key_bytes, num_shards, int(routing),
                                          grouped.data_ptr() or None, pos.data_ptr() or None, counts.data_ptr(),
                                          self._ws.data_ptr(), wsb, _stream_handle(None)))
        self._wsb, self._ns = wsb, num_shards
        return grouped, pos, counts

    def unpartition(self, grouped, pos):
        """Per-key bytes of the last partitioned batch, in group order, back
        at their batch positions."""
        n = grouped.numel()
        if self._ns == 0:
            raise RuntimeError("unpartition before any partition")
        out = self.torch.empty(n, dtype=self.torch.uint8, device=self.device)
        _check(self._L.cf_shard_unpartition(grouped.data_ptr() or None, pos.data_ptr() or None, n, self._ns,
                                            self._ws.data_ptr(), self._wsb, out.data_ptr() or None,
                                            _stream_handle(None)))
        return out


class DeviceShardOps:
    """The rank's device side: its filter shard and the grouping kernels, all
    through the C ABI of ``lib/libcuckoo_b200.so``."""

    def __init__(self, config: CuckooConfig, capacity: int):
        import torch

        self.torch = torch
        self.filter = CuckooFilter(config, capacity)
        self.device = torch.device("cuda", self.filter.device)
        self.key_bytes = config.key_bytes
        self.key_dtype = torch.int64 if self.key_bytes == 8 else torch.int32
        self.grouping = KeyGrouping(self.device, self.key_bytes)

    def to_device(self, keys):
        """This rank's keys as a contiguous device tensor of the key width."""
        torch = self.torch
        if isinstance(keys, np.ndarray):
            a = np.ascontiguousarray(keys, dtype=np.uint64 if self.key_bytes == 8 else np.uint32)
            t = torch.from_numpy(a.view(np.int64 if self.key_bytes == 8 else np.int32))
            return t.pin_memory().to(self.device, non_blocking=True)
        if keys.element_size() != self.key_bytes:
            raise ValueError(f"keys: element size {keys.element_size()} != {self.key_bytes}")
        return keys.contiguous().view(self.key_dtype).to(self.device)

    def partition(self, keys, num_shards: int, routing: int = 0):
        return self.grouping.partition(keys, num_shards, routing)

    def unpartition(self, grouped, pos):
        return self.grouping.unpartition(grouped, pos)

    def insert(self, keys) -> None:
        if keys.numel():
            self.filter.insertMany(keys)

    def contains(self, keys):
        out = self.torch.empty(keys.numel(), dtype=self.torch.uint8, device=self.device)
        if keys.numel():
            self.filter.containsMany(keys, out)
        return out

    def delete(self, keys):
        out = self.torch.empty(keys.numel(), dtype=self.torch.uint8, device=self.device)
        if keys.numel():
            self.filter.deleteMany(keys, out)
        return out

    def occupied(self) -> int:
        return self.filter.occupiedSlots()

    def capacity(self) -> int:
        return self.filter.capacity()

    def size_in_bytes(self) -> int:
        return self.filter.sizeInBytes()

    def clear(self) -> None:
        self.filter.clear()

    def synchronize(self) -> None:
        self.torch.cuda.synchronize(self.device)


class CuckooFilterMultiGPU:
    """Mirrors ``CuckooFilterMultiGPU<Config>``: ``insertMany`` (:452),
    ``containsMany`` (:469), ``deleteMany`` (:487, :504), ``loadFactor``
    (:520), ``synchronizeAllGPUs`` (:550), ``totalOccupiedSlots`` (:558),
    ``clear`` (:570), ``totalCapacity`` (:578) and ``sizeInBytes`` (:586),
    one process per GPU.

    ``group`` is the ``torch.distributed`` process group (default: the world);
    the number of GPUs is its size.  ``routing`` picks the shard of a key:
    ``"reference"`` is the reference's ``hash64(key) % numGPUs``; with the XOR
    policy and a power-of-two GPU count it leaves a shard's keys only
    1/numGPUs of its buckets as primary buckets, so inserts evict more and
    fail near full load.  ``"remixed"`` routes by splitmix64's output mixer
    of ``hash64(key)``, independent of the buckets.  ``ops`` replaces the
    rank's device side (its filter and grouping kernels); by default it is
    ``DeviceShardOps``.
    """

    def __init__(self, config: CuckooConfig, capacity: int, group=None, ops=None,
                 max_keys_per_call: int = 1 << 28, routing: str = "reference"):
        import torch
        import torch.distributed as dist

        if not dist.is_initialized():
            raise RuntimeError("CuckooFilterMultiGPU needs an initialized torch.distributed process group")
        self.torch, self.dist, self.group = torch, dist, group
        self.numGPUs = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        if self.numGPUs > 256:
            raise ValueError("at most 256 GPUs (shards)")
        self.config = config
        self.capacityPerGPU = capacity_per_gpu(capacity, self.numGPUs)
        self.ops = ops if ops is not None else DeviceShardOps(config, self.capacityPerGPU)
        self.max_keys_per_call = int(max_keys_per_call)
        if routing not in _ROUTINGS:
            raise ValueError(f"routing must be one of {sorted(_ROUTINGS)}")
        self.routing = _ROUTINGS[routing]

    # ------------------------------------------------------------ helpers
    def _sum(self, value: int) -> int:
        t = self.torch.tensor([int(value)], dtype=self.torch.int64, device=self.ops.device)
        self.dist.all_reduce(t, group=self.group)
        return int(t.item())

    def _rounds(self, n: int) -> int:
        t = self.torch.tensor([int(n)], dtype=self.torch.int64, device=self.ops.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX, group=self.group)
        m = int(t.item())
        return -(-m // self.max_keys_per_call) if m else 0

    def _exchange(self, keys, op: str):
        """One round: group, send keys, run `op` on the received keys and, for
        lookups and deletes, bring the results back in batch order."""
        torch, dist = self.torch, self.dist
        grouped, pos, counts = self.ops.partition(keys, self.numGPUs, self.routing)
        recv_counts = torch.empty_like(counts)
        dist.all_to_all_single(recv_counts, counts, group=self.group)
        send = [int(x) for x in counts.tolist()]
        recv = [int(x) for x in recv_counts.tolist()]
        mine = torch.empty(sum(recv), dtype=grouped.dtype, device=grouped.device)
        dist.all_to_all_single(mine, grouped, output_split_sizes=recv, input_split_sizes=send, group=self.group)
        if op == "insert":
            self.ops.insert(mine)
            return None
        res = self.ops.contains(mine) if op == "contains" else self.ops.delete(mine)
        back = torch.empty(keys.numel(), dtype=torch.uint8, device=res.device)
        dist.all_to_all_single(back, res, output_split_sizes=send, input_split_sizes=recv, group=self.group)
        return self.ops.unpartition(back, pos)

    def _run(self, keys, op: str, output=None):
        host = isinstance(keys, np.ndarray)
        d = self.ops.to_device(keys)
        n = d.numel()
        rounds = self._rounds(n)
        parts = []
        for r in range(rounds):
            lo = min(n, r * self.max_keys_per_call)
            hi = min(n, lo + self.max_keys_per_call)
            got = self._exchange(d[lo:hi], op)
            if got is not None:
                parts.append(got)
        if op == "insert":
            return None
        res = self.torch.cat(parts) if parts else self.torch.empty(0, dtype=self.torch.uint8, device=d.device)
        res = res.view(self.torch.bool)
        if output is not None:
            if isinstance(output, np.ndarray):
                output[:n] = res.cpu().numpy()
            else:
                output[:n].copy_(res)
            return output
        return res.cpu().numpy() if host else res

    # ------------------------------------------------------------ batch ops
    def insertMany(self, keys) -> int:
        """Insert this rank's keys; returns totalOccupiedSlots() afterwards."""
        self._run(keys, "insert")
        return self.totalOccupiedSlots()

    def containsMany(self, keys, output=None):
        """Membership of each of this rank's keys, aligned with `keys` (a host
        array for host keys, a device bool tensor for device keys, or `output`)."""
        return self._run(keys, "contains", output)

    def deleteMany(self, keys, output=None) -> int:
        """Remove one copy of each of this rank's keys; per-key outcomes go to
        `output` when given.  Returns totalOccupiedSlots() afterwards."""
        self._run(keys, "delete", output)
        return self.totalOccupiedSlots()

    # ------------------------------------------------------------ totals
    def totalOccupiedSlots(self) -> int:
        return self._sum(self.ops.occupied())

    def totalCapacity(self) -> int:
        return self._sum(self.ops.capacity())

    def sizeInBytes(self) -> int:
        return self._sum(self.ops.size_in_bytes())

    def loadFactor(self) -> float:
        return self.totalOccupiedSlots() / self.totalCapacity()

    def clear(self) -> None:
        self.ops.clear()

    def synchronizeAllGPUs(self) -> None:
        self.ops.synchronize()
        self.dist.barrier(group=self.group)


def remix64(h: np.ndarray) -> np.ndarray:
    """splitmix64's output mixer (Steele, Lea and Flood 2014; Vigna's constants)."""
    z = np.asarray(h, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def shard_of(keys: np.ndarray, num_shards: int, key_bytes: int = 8, routing: str = "reference") -> np.ndarray:
    """Destination shard of each key on the host: ``hash64(key) % num_shards``
    (the filter's own xxHash through ``cf_hash64``), remixed first for
    ``routing="remixed"``."""
    a = np.ascontiguousarray(keys, dtype=np.uint64 if key_bytes == 8 else np.uint32)
    h = np.empty(a.size, dtype=np.uint64)
    L = library()
    _check(L.cf_hash64(key_bytes, a.ctypes.data, a.size, h.ctypes.data))
    if _ROUTINGS[routing] == ROUTING_REMIXED:
        h = remix64(h)
    return (h % np.uint64(num_shards)).astype(np.int64)
