"""A CPU model of the serving engine (simulated clock) for scheduler tests."""


class ModelEngine:
    """Simulated clock: a batch step costs (cells of the members) / rate
    seconds; creating a box costs ``create_s``."""

    def __init__(self, rate=1e9, create_s=1e-3):
        self.t = 0.0
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
        self.t += k * sum(b["req"].cells for b in self.members) / self.rate
        for b in self.members:
            b["steps"] += k

    def sync(self):
        pass

    def finish(self, box):
        self.members.remove(box)
        return box["steps"]

    def release(self, box):
        pass
