"""A CPU model of the serving engine (simulated clock) for scheduler tests."""


class ModelEngine:
    """Simulated clock.  Host work (creating a box) advances the clock; a
    batch step is enqueued like a GPU launch: it costs (cells of the
    members) / rate seconds of device time, starting when the device is free,
    and the host sees its end only at ``sync``."""

    def __init__(self, rate=1e9, create_s=1e-3):
        self.t = 0.0
        self.busy = 0.0           # device time at which the enqueued work ends
        self.rate = rate
        self.create_s = create_s
        self.members = []
        self.log = []
        self.resident_max = 0

    def now(self):
        return self.t

    def wait_until(self, t):
        self.t = max(self.t, t)

    def create(self, req):
        self.t += self.create_s
        self.log.append(("create", req.rid, self.t))
        return {"req": req, "steps": 0}

    def add(self, box):
        self.members.append(box)

    def step(self, k):
        start = max(self.t, self.busy)
        self.busy = start + k * sum(b["req"].cells for b in self.members) / self.rate
        for b in self.members:
            b["steps"] += k
        self.log.append(("step", k, len(self.members)))

    def sync(self):
        self.t = max(self.t, self.busy)

    def detach(self, box):
        self.members.remove(box)

    def finish(self, box):
        self.log.append(("finish", box["req"].rid, self.t))
        return box["steps"]

    def release(self, box):
        pass
