"""A stand-in for the serving engine of mhd_gpu_solver_b200.serve (no GPU): each admitted
request finishes after `rounds` advances, or raises for request `fail_rid`; its result is a
small array holding its id. Used by the host tests of Server and of sharded serving."""

import time

import numpy as np


class FakeEngine:
    def __init__(self, stats, rounds=2, fail_rid=None):
        self.stats, self.rounds, self.fail_rid = stats, rounds, fail_rid
        self.active = {}
        self.closed = False
        self.start = time.perf_counter()

    def clock(self):
        return time.perf_counter() - self.start

    @property
    def busy(self):
        return bool(self.active)

    def order_queue(self, queue):
        return queue

    def admit(self, queue):
        while queue:
            r = queue.popleft()
            self.active[r.rid] = [r, self.rounds]
        self.stats.max_active = max(self.stats.max_active, len(self.active))

    def advance(self):
        from mhd_gpu_solver_b200.serve import Completion

        out = []
        for rid, item in list(self.active.items()):
            r, left = item
            if rid == self.fail_rid:
                raise RuntimeError("solve: reached max_steps before t_end")
            if left <= 1:
                del self.active[rid]
                c = Completion(rid, r.arrival, r.arrival, self.clock(), 7, r.t_end, r.n * r.n)
                self.stats.completions.append(c)
                self.stats.states[rid] = np.full(3, float(rid))
                out.append(c)
            else:
                item[1] = left - 1
        self.stats.chunks += 1
        return out

    def close(self):
        self.closed = True
