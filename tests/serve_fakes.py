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


class FakeBatch:
    """Stands in for BatchSolver under the real serving engine: solve `sid` finishes after
    `rounds` launches; results are zero arrays of the request's ghosted shape."""

    def __init__(self, rounds=2):
        self.rounds = rounds
        self.left = {}
        self.shape = {}
        self.launched = 0
        self.removed = []
        self.next_sid = 0

    def add_generated(self, nx, ny, init, params, bc):
        sid = self.next_sid
        self.next_sid += 1
        self.left[sid] = self.rounds
        self.shape[sid] = (9, ny + 4, nx + 4)
        return sid

    def launch(self, nsteps):
        self.launched += 1
        for sid in self.left:
            self.left[sid] -= 1

    def poll(self):
        return sum(1 for v in self.left.values() if v > 0)

    def status(self, sid):
        class R:
            steps, t = 5, 0.01
        return R(), self.left[sid] <= 0

    def download(self, sid, out=None):
        out = np.zeros(self.shape[sid]) if out is None else out
        out[...] = 0.0
        return out

    def remove(self, sid):
        self.removed.append(sid)
        del self.left[sid]

    def close(self):
        pass
