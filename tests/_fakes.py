"""Host-only stand-ins for device objects, for scheduling tests on the CPU."""
import numpy as np

from adaptflood_b200.batch import Arena


class FakeBatch:
    """Batch's interface on the host: each scenario advances by a fixed dt
    per batch step; a launch completes after a few polls."""

    def __init__(self, arena_bytes, dt=7.0, polls=3):
        self.arena_bytes = arena_bytes
        self.plan = Arena(arena_bytes)
        self.dt = dt
        self.polls = polls
        self.slots = {}
        self.in_flight = False
        self.launch_args = None
        self.attn = False
        self.attn_count = 0
        self.peak_used = 0
        self.next_slot = 0
        self.deferred = []

    def footprint(self, case, forcing=None, t_stop=None):
        return case.cells * 28

    def try_add(self, case, forcing=None, t_stop=None):
        off = self.plan.alloc(self.footprint(case))
        if off is None:
            return None
        s = self.next_slot
        self.next_slot += 1
        stop = case.sim_time if t_stop is None else t_stop
        self.slots[s] = dict(case=case, stop=stop, t=0.0, steps=0, off=off)
        self.peak_used = max(self.peak_used, self.plan.stats()[0])
        return s

    def _finished(self, s):
        d = self.slots[s]
        return not d["t"] < d["stop"]

    def launch(self, max_steps=1 << 40, stop_on_done=False):
        assert not self.in_flight, "launch while a launch is in flight"
        self.in_flight = True
        self.launch_args = (max_steps, stop_on_done)
        self.attn = False
        self.left = self.polls

    def attention(self):
        self.attn = True
        self.attn_count += 1

    def done(self):
        self.left -= 1
        return self.left <= 0

    def sync(self):
        assert self.in_flight
        max_steps, stop_on_done = self.launch_args
        for _ in range(max_steps):
            act = [s for s in self.slots if not self._finished(s)]
            if not act:
                break
            for s in act:
                self.slots[s]["t"] += self.dt
                self.slots[s]["steps"] += 1
            if self.attn or (stop_on_done and any(self._finished(s) for s in act)):
                break
        self.in_flight = False
        for s in self.deferred:
            self.plan.free(self.slots.pop(s)["off"])
        self.deferred.clear()

    def status(self, s):
        d = self.slots[s]
        return d["t"], self.dt, 0.0, d["steps"], 1 if self._finished(s) else 0

    def depth(self, s):
        assert self._finished(s) or not self.in_flight, "read-back of a running scenario"
        c = self.slots[s]["case"]
        return np.full((c.ny, c.nx), float(self.slots[s]["steps"]))

    def add(self, case, forcing=None, t_stop=None):
        s = self.try_add(case, forcing, t_stop if t_stop is not None else case.sim_time)
        assert s is not None, "no room"
        return s

    def run(self, max_steps=1 << 40):
        self.launch(max_steps)
        while not self.done():
            pass
        self.sync()

    def remove(self, s):
        if self.in_flight:
            self.deferred.append(s)
        else:
            self.plan.free(self.slots.pop(s)["off"])

    def close(self):
        pass
