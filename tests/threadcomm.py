"""Ranks as threads of one process sharing one GPU and its default stream
(test harness for the partitioned solvers): a collective meets at a barrier,
copies between the ranks' tensors on the shared stream, and meets again once
every copy is enqueued, so no rank overwrites a buffer another still reads.
No kernel waits on another rank: all waiting is on the host."""
import threading


class ThreadComm:
    def __init__(self, size: int, timeout: float = 300.0):
        self.size = size
        self.bar = threading.Barrier(size, timeout=timeout)
        self.slot = [None] * size

    def rank_comm(self, rank: int):
        return _RankComm(self, rank)


class _RankComm:
    def __init__(self, shared: ThreadComm, rank: int):
        self.s, self.rank, self.size = shared, rank, shared.size

    def _publish(self, obj):
        self.s.slot[self.rank] = obj
        self.s.bar.wait()
        objs = list(self.s.slot)
        self.s.bar.wait()
        return objs

    def all_to_all_single(self, out, inp, out_splits, in_splits, async_op=False):
        import torch
        objs = self._publish((inp, [int(c) for c in in_splits]))
        parts = []
        for t, spl in objs:
            off = sum(spl[:self.rank])
            parts.append(t[off:off + spl[self.rank]])
        if out.numel():
            out.copy_(torch.cat(parts))
        self.s.bar.wait()
        return None

    def all_reduce(self, t):
        objs = self._publish(t)
        total = objs[0].clone()
        for o in objs[1:]:
            total += o
        self.s.bar.wait()
        t.copy_(total)
        return t

    def all_gather_v(self, t, counts):
        import torch
        objs = self._publish(t)
        out = torch.cat([o[:int(c)] for o, c in zip(objs, counts)])
        self.s.bar.wait()
        return out


def run_ranks(size: int, fn):
    """fn(rank) in `size` threads; returns their results, re-raising the
    first exception."""
    res, err = [None] * size, [None] * size

    def body(r):
        try:
            res[r] = fn(r)
        except BaseException as e:  # noqa: BLE001 - handed to the caller
            err[r] = e

    th = [threading.Thread(target=body, args=(r,)) for r in range(size)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for e in err:
        if e is not None:
            raise e
    return res
